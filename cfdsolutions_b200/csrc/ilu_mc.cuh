// Block multicolour ILU(0) (ilu_mc.cu).
#pragma once

#include "ctx.cuh"

namespace cfd {

// Ordering, per-row slot lists and patch-local levels (once per mesh).
int mc_build(cfd_ctx *c);
// Factors A (block-CRS slots, storage TA) into M (storage TM), FP64 arithmetic.
template <typename TA, typename TM>
int mc_factor(cfd_ctx *c, const TA *A, TM *M);
// z = (LU)^-1 r with the factors in M; tmp holds the forward result.
template <typename TM>
int mc_apply(cfd_ctx *c, const TM *M, const double *r, double *tmp, double *z);

}  // namespace cfd
