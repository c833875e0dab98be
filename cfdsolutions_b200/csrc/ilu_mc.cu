// Block ILU(0) in block multicolour order.
//
// The level-scheduled ILU(0) in mesh order needs one launch per dependency
// level in the factorisation and in each triangular solve; on a banded
// (RCM-like) numbering of an n^3 mesh that is O(n) levels of a few thousand
// rows each, so the solves are bound by launch latency, not by HBM.  Here the
// rows are grouped in patches of kMcRows (32) consecutive rows and the
// patch graph (two patches adjacent when a matrix block couples them) is
// coloured by DSATUR.  The factorisation order is: colours in increasing
// order, rows of a colour in increasing index.  Two patches of one colour are
// never coupled, so every patch of a colour is factored (or solved) by its own
// CTA in one launch per colour; inside a patch the rows follow their local
// dependency levels, separated by __syncthreads().  This is ILU(0) of P A P^T
// for the permutation P of that order (the ordering idea is the algebraic block
// multicolour ordering of Iwashita, Nakashima and Takahashi, IPDPS 2012).
//
// Storage: `slot` lists each row's CRS slots as [lower, in factorisation
// order | diagonal | upper, in factorisation order]; the factors are stored
// in that order (entry u of row i at block IA[i] + u): L (unit diagonal) for
// the lower entries, inv(U_ii) for the diagonal, U for the upper entries.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <set>
#include <tuple>
#include <vector>

#include "ctx.cuh"
#include "kernels.cuh"
#include "ilu_mc.cuh"
#include "host_par.h"

namespace cfd {

namespace {

// Rows per patch of the ordering (five solve threads per row).
constexpr int kMcRows = 32;

template <typename T>
__device__ __forceinline__ double ld(const T *p);
template <>
__device__ __forceinline__ double ld<double>(const double *p) { return *p; }
template <>
__device__ __forceinline__ double ld<float>(const float *p) { return (double)*p; }
template <>
__device__ __forceinline__ double ld<uint16_t>(const uint16_t *p) { return load_low(p); }

template <typename T>
__device__ __forceinline__ void st(T *p, double v);
template <>
__device__ __forceinline__ void st<double>(double *p, double v) { *p = v; }
template <>
__device__ __forceinline__ void st<float>(float *p, double v) { *p = (float)v; }

// 5x5 inverse by Gauss-Jordan with partial pivoting across a warp: lane
// r*5+c (r, c < 5) holds entry (r,c) of the matrix (a) and of the inverse
// being formed (v); lanes 25-31 carry zeros.  The pivot of column k is the
// first row >= k of largest magnitude, as in the sequential elimination, and
// every entry sees the same operations in the same order.  Returns false
// (on every lane) when a pivot is zero.
__device__ __forceinline__ bool warp_inverse5(double &a, double &v, int lane) {
    const int r = lane / 5, c = lane - 5 * (lane / 5);
    const bool on = lane < 25;
    v = (on && r == c) ? 1.0 : 0.0;
    if (!on) a = 0.0;
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        // pivot: largest |a(r,k)| over r >= k, lowest r on ties
        double best = (on && c == k && r >= k) ? fabs(a) : -1.0;
        int brow = r;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int orow = __shfl_xor_sync(0xffffffffu, brow, o);
            if (ob > best || (ob == best && orow < brow)) { best = ob; brow = orow; }
        }
        if (!(best > 0.0)) ok = false;
        // swap rows k and brow
        const int sr = r == k ? brow : (r == brow ? k : r);
        const int from = on ? sr * 5 + c : lane;
        a = __shfl_sync(0xffffffffu, a, from);
        v = __shfl_sync(0xffffffffu, v, from);
        // scale row k by 1/a(k,k)
        const double d = 1.0 / __shfl_sync(0xffffffffu, a, k * 5 + k);
        if (on && r == k) { a *= d; v *= d; }
        // eliminate column k from the other rows
        const double f = __shfl_sync(0xffffffffu, a, (on ? r : 0) * 5 + k);
        const double ak = __shfl_sync(0xffffffffu, a, k * 5 + (on ? c : 0));
        const double vk = __shfl_sync(0xffffffffu, v, k * 5 + (on ? c : 0));
        if (on && r != k) { a -= f * ak; v -= f * vk; }
    }
    return ok;
}

// Shared-memory bytes of one warp of k_mc_factor (factor blocks staged in
// their storage type TM), rounded up to 16.
template <typename TM>
__host__ __device__ inline size_t mc_factor_warp_bytes(int maxrow, int maxstage) {
    const size_t b = (size_t)maxrow * sizeof(int4) + (size_t)maxrow * 25 * sizeof(double) +
                     (size_t)maxstage * 25 * sizeof(TM) + (size_t)(2 * maxstage + maxrow) * sizeof(int);
    return (b + 15) & ~(size_t)15;
}

// Factorisation of the patches of one colour, one warp per patch: the warp
// factors the patch's rows in increasing order (a row's lower blocks inside
// the patch belong to earlier rows of the same warp; the others to earlier
// colours), so no CTA-wide barrier is needed.  Row i's
// blocks are staged in shared memory in FP64 (CRS slot order) together with
// every factor block the row needs from earlier rows: inv(U_pp) for each lower
// block (i,p) and U_pj for each pair (p,j) with j in row i, listed per row at
// setup.  All those loads are issued together, then the elimination runs from
// shared memory: for each lower block, in factorisation order,
// L_ip = A_ip inv(U_pp) and A_ij -= L_ip U_pj over the row's pairs of p.
// The factors are stored in each row's factorisation order (row i's entry u of
// the slot list at M[(IA[i] + u) * 25]), so the solves read them as a stream.
// hdr[IA[i]+u] = (M position of inv(U_pp), pairs, CRS-local slot of (i,p));
// pairs are (M position of U_pj, CRS-local slot of (i,j)).
template <typename TA, typename TM>
__global__ void k_mc_factor(const int *__restrict__ patches, int npatch, int n, int maxrow, int maxstage,
                            const int *__restrict__ IA, const int *__restrict__ slot, const int4 *__restrict__ meta,
                            const int4 *__restrict__ hdr,
                            const int64_t *__restrict__ pair_ptr, const int2 *__restrict__ pairs,
                            const TA *__restrict__ A, TM *__restrict__ M, int *__restrict__ err) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int nwarp = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // per-warp region (a multiple of 16 bytes): headers first, so they stay
    // 16-byte aligned, then the FP64 blocks, then the integer lists
    unsigned char *reg = smraw + (size_t)wid * mc_factor_warp_bytes<TM>(maxrow, maxstage);
    int4 *hd = reinterpret_cast<int4 *>(reg);                                     // [maxrow]
    double *w = reinterpret_cast<double *>(reg + (size_t)maxrow * sizeof(int4));  // [maxrow][25] row blocks
    TM *stg = reinterpret_cast<TM *>(w + (size_t)maxrow * 25);       // [maxstage][25] staged factor blocks
    int *pm = reinterpret_cast<int *>(stg + (size_t)maxstage * 25);  // [maxstage] CRS-local slot of each pair
    int *src = pm + maxstage;                                         // [maxstage] M position of staged blocks
    int *sl = src + maxstage;                                         // [maxrow] CRS-local slot of list entry u
    const int pidx = blockIdx.x * nwarp + wid;
    if (pidx >= npatch) return;  // whole warp; no CTA barrier follows
    const int P = patches[pidx];
    const int p0 = P * kMcRows, nr = min(kMcRows, n - p0);
    const int a = lane / 5, b = lane - 5 * (lane / 5);
    {
        for (int q = 0; q < nr; q++) {
            const int i = p0 + q;
            const int4 mt = meta[i];
            const int base = IA[i], len = IA[i + 1] - base, nlo = mt.y;
            const int64_t pp = pair_ptr[i];
            const int npair = (int)(pair_ptr[i + 1] - pp);
            for (int e = lane; e < nlo; e += 32) {
                const int4 h = hdr[base + e];
                hd[e] = h;
                src[e] = h.x;
            }
            for (int e = lane; e < npair; e += 32) {
                const int2 pr = pairs[pp + e];
                pm[e] = pr.y;
                src[nlo + e] = pr.x;
            }
            for (int e = lane; e < len; e += 32) sl[e] = slot[base + e] - base;
            // one block per lane, its 25 loads in flight together
            for (int t = lane; t < len; t += 32) {
                const TA *ab = A + (int64_t)(base + t) * 25;
#pragma unroll
                for (int k = 0; k < 25; k++) w[t * 25 + k] = ld<TA>(ab + k);
            }
            __syncwarp();
            const int nst = nlo + npair;
            for (int t = lane; t < nst; t += 32) {
                const TM *mb = M + (int64_t)src[t] * 25;
#pragma unroll
                for (int k = 0; k < 25; k++) stg[t * 25 + k] = mb[k];
            }
            __syncwarp();
            int t0 = 0;
            for (int u = 0; u < nlo; u++) {
                const int4 h = hd[u];
                const int tk = h.z;
                // L_ip = A_ip inv(U_pp)
                double Lab = 0.0;
                if (lane < 25) {
#pragma unroll
                    for (int c = 0; c < 5; c++) Lab = fma(w[tk * 25 + a * 5 + c], (double)stg[u * 25 + c * 5 + b], Lab);
                }
                __syncwarp();
                if (lane < 25) w[tk * 25 + lane] = Lab;
                __syncwarp();
                // A_ij -= L_ip U_pj, the pairs' 25 entries spread over the lanes
                for (int e = lane; e < h.y * 25; e += 32) {
                    const int t = e / 25, ab = e - 25 * t, ea = ab / 5, eb = ab - 5 * ea;
                    const int mj = pm[t0 + t];
                    const TM *U = stg + (size_t)(nlo + t0 + t) * 25;
                    double s = w[mj * 25 + ab];
#pragma unroll
                    for (int c = 0; c < 5; c++) s = fma(-w[tk * 25 + ea * 5 + c], (double)U[c * 5 + eb], s);
                    w[mj * 25 + ab] = s;
                }
                __syncwarp();
                t0 += h.y;
            }
            const int td = sl[nlo];  // the diagonal follows the lower entries
            {
                double av = lane < 25 ? w[td * 25 + lane] : 0.0, iv;
                const bool ok = warp_inverse5(av, iv, lane);
                if (!ok && lane == 0) atomicOr(err, ERR_NAN);
                __syncwarp();
                if (lane < 25) w[td * 25 + lane] = iv;
            }
            __syncwarp();
            for (int e = lane; e < len * 25; e += 32) {
                const int u = e / 25;
                st<TM>(M + (int64_t)base * 25 + e, w[sl[u] * 25 + (e - 25 * u)]);
            }
            __syncwarp();
        }
    }
}

// Programmatic dependent launch (sm_90+): the solve of one colour lets the
// next colour's launch begin as soon as all of its own CTAs are resident
// (launch_dependents), and that launch stages its constant factor blocks
// before waiting (wait) for the vectors the earlier launches write.  Every
// CTA of the earlier grid is resident before a dependent CTA can start, so
// the earlier grid always completes.  Both are no-ops in a plain launch.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Resident CTAs per SM the triangular solves are compiled for: FP32 factors
// fit 8 in 48 registers; FP64 factors keep 6 (64 registers), which measured
// faster than 8 at 128^3 (2.69 against 2.88 ms per apply).
template <typename TM>
struct McMinBlocks {
    static constexpr int value = sizeof(TM) == 8 ? 6 : 8;
};

// Blocks of a row inside its own patch staged in shared memory before the
// level loop of a triangular solve (more go through the load path).
template <typename TM>
struct IntraCap {
    static constexpr int K = sizeof(TM) == 8 ? 3 : 6;
};

// Off-patch blocks of a row whose columns a triangular solve fetches before
// its dependency wait (the rest are read in its loop).
constexpr int kMcPrefetch = 4;

// Forward solve y = L^-1 r over the patches of one colour: five threads per
// row (thread m forms component m).  Lower blocks in other patches belong to
// earlier colours (complete in y) and are summed first; the row's blocks
// inside the patch are staged in shared memory before the level loop, which
// then only waits on shared memory.  CTA b takes the patch at position b of
// the colour and reads the factors in the packed layout k_mc_pack writes:
// slot t of every row of the patch side by side, so that for each (slot,
// component) the CTA's 160 threads read 160 consecutive values (thread q*5+m
// the entry (m, c) of row q's block) instead of five 32-byte sectors per row.
// rowf / rowl hold the rows' records ({i, off-patch lower slots, lower slots}
// and {level, last level of the patch, ..}; i = -1 past the mesh), L / cl the
// patch's factors and columns (off-patch slots: global columns, intra-patch
// slots: patch-local ones).  Everything constant is read before the wait;
// after it one round trip fetches the earlier colours' y.
template <typename TM>
__global__ void __launch_bounds__(5 * kMcRows, McMinBlocks<TM>::value)
    k_mc_fwd(const int4 *__restrict__ rowf, const int4 *__restrict__ rowl, const int64_t *__restrict__ lslot,
             const int *__restrict__ colL, const TM *__restrict__ PL, const double *__restrict__ r,
             double *__restrict__ y) {
    constexpr int K = IntraCap<TM>::K, PF = kMcPrefetch;
    constexpr int T = 5 * kMcRows;
    __shared__ double ys[T];
    __shared__ TM pa[K * 5][T];  // [t*5+c][thread]
    __shared__ unsigned char pj[K][T];
    const int tid = threadIdx.x;
    const int q = tid / 5, m = tid - 5 * q;
    const int4 rf = rowf[blockIdx.x * kMcRows + q];
    const int4 rl = rowl[blockIdx.x * kMcRows + q];
    const int64_t ls = lslot[blockIdx.x];
    const TM *L = PL + ls * (25 * kMcRows) + tid;  // slot t, column c of the block: L[(t * 5 + c) * T]
    const int *cl = colL + ls * kMcRows + q;       // column of slot t: cl[t * kMcRows]
    const bool act = rf.x >= 0;
    const int i = rf.x, nx = rf.y, nlo = rf.z, lev = rl.x;
    double s = 0.0;
    int col[PF];
    // the next colour's launch may start staging its constant factors now
    pdl_trigger();
    if (act) {
#pragma unroll
        for (int t = 0; t < K; t++)
            if (nx + t < nlo) {
                pj[t][tid] = (unsigned char)cl[(nx + t) * kMcRows];
#pragma unroll
                for (int c = 0; c < 5; c++) pa[t * 5 + c][tid] = L[((nx + t) * 5 + c) * T];
            }
#pragma unroll
        for (int t = 0; t < PF; t++) col[t] = t < nx ? cl[t * kMcRows] : 0;
        // r is complete before the first colour's launch starts, so before this one's
        s = r[(int64_t)i * 5 + m];
    }
    pdl_wait();  // the earlier colours' y are complete from here on
    if (act) {
#pragma unroll
        for (int t = 0; t < PF; t++)
            if (t < nx) {
                const double *yv = y + (int64_t)col[t] * 5;
#pragma unroll
                for (int c = 0; c < 5; c++) s = fma(-ld<TM>(L + (t * 5 + c) * T), yv[c], s);
            }
#pragma unroll 4
        for (int t = PF; t < nx; t++) {
            const double *yv = y + (int64_t)cl[t * kMcRows] * 5;
#pragma unroll
            for (int c = 0; c < 5; c++) s = fma(-ld<TM>(L + (t * 5 + c) * T), yv[c], s);
        }
    }
    const int last = rl.y;
    for (int l = 0; l <= last; l++) {
        if (act && lev == l) {
#pragma unroll
            for (int t = 0; t < K; t++)
                if (nx + t < nlo) {
                    const double *yv = ys + pj[t][tid] * 5;
#pragma unroll
                    for (int c = 0; c < 5; c++) s = fma(-(double)pa[t * 5 + c][tid], yv[c], s);
                }
            for (int t = nx + K; t < nlo; t++) {
                const double *yv = ys + cl[t * kMcRows] * 5;
#pragma unroll
                for (int c = 0; c < 5; c++) s = fma(-ld<TM>(L + (t * 5 + c) * T), yv[c], s);
            }
            ys[tid] = s;
        }
        __syncthreads();
    }
    if (act) y[(int64_t)i * 5 + m] = s;
}

// Backward solve z = U^-1 y over the patches of one colour (colours in
// decreasing order): upper blocks in other patches belong to later colours.
// rowb holds {i, intra-patch upper slots, upper slots, ..}; U / cu the
// packed upper blocks (intra-patch slots first, patch-local columns) and D the
// packed inverted diagonal blocks.  y is read after the wait: the last
// forward colour may still be writing it when the first backward one starts.
template <typename TM>
__global__ void __launch_bounds__(5 * kMcRows, McMinBlocks<TM>::value)
    k_mc_bwd(const int4 *__restrict__ rowb, const int4 *__restrict__ rowl, const int64_t *__restrict__ uslot,
             const int *__restrict__ colU, const TM *__restrict__ PU, const TM *__restrict__ PD,
             const double *__restrict__ y, double *__restrict__ z) {
    constexpr int K = IntraCap<TM>::K, PF = kMcPrefetch;
    constexpr int T = 5 * kMcRows;
    __shared__ double zs[T], ts[T];
    __shared__ TM pa[K * 5][T];
    __shared__ unsigned char pj[K][T];
    const int tid = threadIdx.x;
    const int q = tid / 5, m = tid - 5 * q;
    const int4 rb = rowb[blockIdx.x * kMcRows + q];
    const int4 rl = rowl[blockIdx.x * kMcRows + q];
    const int64_t us = uslot[blockIdx.x];
    const TM *U = PU + us * (25 * kMcRows) + tid;
    const int *cu = colU + us * kMcRows + q;
    const TM *D = PD + (int64_t)blockIdx.x * (25 * kMcRows) + tid;
    const bool act = rb.x >= 0;
    const int i = rb.x, nin = rb.y, nup = rb.z, lev = rl.z;
    double s = 0.0;
    TM dg[5];
    int col[PF];
    pdl_trigger();
    if (act) {
#pragma unroll
        for (int t = 0; t < K; t++)
            if (t < nin) {
                pj[t][tid] = (unsigned char)cu[t * kMcRows];
#pragma unroll
                for (int c = 0; c < 5; c++) pa[t * 5 + c][tid] = U[(t * 5 + c) * T];
            }
#pragma unroll
        for (int c = 0; c < 5; c++) dg[c] = D[c * T];
#pragma unroll
        for (int t = 0; t < PF; t++) col[t] = nin + t < nup ? cu[(nin + t) * kMcRows] : 0;
    }
    pdl_wait();  // y and the later colours' z are complete from here on
    if (act) {
        s = y[(int64_t)i * 5 + m];
#pragma unroll
        for (int t = 0; t < PF; t++)
            if (nin + t < nup) {
                const double *zv = z + (int64_t)col[t] * 5;
#pragma unroll
                for (int c = 0; c < 5; c++) s = fma(-ld<TM>(U + ((nin + t) * 5 + c) * T), zv[c], s);
            }
#pragma unroll 4
        for (int t = nin + PF; t < nup; t++) {
            const double *zv = z + (int64_t)cu[t * kMcRows] * 5;
#pragma unroll
            for (int c = 0; c < 5; c++) s = fma(-ld<TM>(U + (t * 5 + c) * T), zv[c], s);
        }
    }
    const int last = rl.w;
    for (int l = 0; l <= last; l++) {
        const bool mine = act && lev == l;
        if (mine) {
#pragma unroll
            for (int t = 0; t < K; t++)
                if (t < nin) {
                    const double *zv = zs + pj[t][tid] * 5;
#pragma unroll
                    for (int c = 0; c < 5; c++) s = fma(-(double)pa[t * 5 + c][tid], zv[c], s);
                }
            for (int t = K; t < nin; t++) {
                const double *zv = zs + cu[t * kMcRows] * 5;
#pragma unroll
                for (int c = 0; c < 5; c++) s = fma(-ld<TM>(U + (t * 5 + c) * T), zv[c], s);
            }
            ts[tid] = s;
        }
        __syncthreads();
        if (mine) {
            double o = 0.0;
#pragma unroll
            for (int c = 0; c < 5; c++) o = fma((double)dg[c], ts[q * 5 + c], o);
            zs[tid] = o;
        }
        __syncthreads();
    }
    if (act) z[(int64_t)i * 5 + m] = zs[tid];
}

// The factors of M (factorisation order) copied into the triangular solves'
// packed layout, one CTA per patch position: lower slot t, block entry (m, c)
// of row q at PL[lslot * 800 + (t * 5 + c) * 160 + q * 5 + m], the upper slots
// likewise in PU, the inverted diagonal block at PD[pos * 800 + c * 160 +
// q * 5 + m].  Slots past a row's own count are left unwritten and never read.
template <typename TM>
__global__ void __launch_bounds__(5 * kMcRows) k_mc_pack(const int4 *__restrict__ rowf, const int4 *__restrict__ rowb,
                                                        const int64_t *__restrict__ lslot,
                                                        const int64_t *__restrict__ uslot, const TM *__restrict__ M,
                                                        TM *__restrict__ PL, TM *__restrict__ PU,
                                                        TM *__restrict__ PD) {
    constexpr int T = 5 * kMcRows;
    const int pos = blockIdx.x, tid = threadIdx.x;
    const int q = tid / 5, m = tid - 5 * q;
    const int4 rf = rowf[pos * kMcRows + q], rb = rowb[pos * kMcRows + q];
    if (rf.x < 0) return;
    const int64_t l0 = lslot[pos], u0 = uslot[pos];
    TM *L = PL + l0 * (25 * kMcRows) + tid, *U = PU + u0 * (25 * kMcRows) + tid;
    for (int t = 0; t < rf.z; t++) {
        const TM *src = M + (int64_t)(rf.w + t) * 25 + m * 5;
#pragma unroll
        for (int c = 0; c < 5; c++) L[(t * 5 + c) * T] = src[c];
    }
    for (int t = 0; t < rb.z; t++) {
        const TM *src = M + (int64_t)(rb.w + 1 + t) * 25 + m * 5;
#pragma unroll
        for (int c = 0; c < 5; c++) U[(t * 5 + c) * T] = src[c];
    }
    const TM *dsrc = M + (int64_t)rb.w * 25 + m * 5;
#pragma unroll
    for (int c = 0; c < 5; c++) PD[(int64_t)pos * (25 * kMcRows) + c * T + tid] = dsrc[c];
}

}  // namespace

// Ordering, slot lists, patch-local levels and the factorisation's update
// lists (host, once per mesh).
int mc_build(cfd_ctx *c) {
    Abmc &mc = c->mc;
    if (mc.built) return CFD_OK;
    const int n = c->nnode;
    const std::vector<int> &IA = c->h_IA, &JA = c->h_JA, &IAU = c->h_IAU;
    const int np = (n + kMcRows - 1) / kMcRows;
    // DSATUR colouring of the patch graph (Brelaz 1979): repeatedly colour the
    // uncoloured patch with the most distinct colours among its neighbours
    // (ties: most neighbours, then lowest index) with the lowest colour free
    // there.  On the tet cubes and channels it needs 10-11 colours where the
    // greedy colouring in patch order needs 13-14, i.e. fewer launches per
    // factorisation and per triangular solve.
    std::vector<std::vector<int>> adj(np);
    parallel_ranges(np, [&](int, int64_t p0, int64_t p1) {
        for (int P = (int)p0; P < (int)p1; P++) {
            const int r0 = P * kMcRows, r1 = std::min(n, r0 + kMcRows);
            for (int i = r0; i < r1; i++)
                for (int k = IA[i]; k < IA[i + 1]; k++) {
                    const int Q = JA[k] / kMcRows;
                    if (Q != P) adj[P].push_back(Q);
                }
            std::sort(adj[P].begin(), adj[P].end());
            adj[P].erase(std::unique(adj[P].begin(), adj[P].end()), adj[P].end());
        }
    });
    std::vector<int> color(np, -1);
    std::vector<uint64_t> seen(np, 0);  // colours among a patch's neighbours
    std::set<std::tuple<int, int, int>> open;  // (-saturation, -degree, patch)
    for (int P = 0; P < np; P++) open.insert({0, -(int)adj[P].size(), P});
    int ncolor = 0;
    while (!open.empty()) {
        const int P = std::get<2>(*open.begin());
        open.erase(open.begin());
        const uint64_t m = seen[P];
        int col = 0;
        while (col < 64 && ((m >> col) & 1u)) col++;
        if (col >= 64) {
            set_error("ILU(0) multicolour: the patch graph needs more than 64 colours");
            return CFD_ERR_RANGE;
        }
        color[P] = col;
        ncolor = std::max(ncolor, col + 1);
        for (int Q : adj[P]) {
            if (color[Q] >= 0 || ((seen[Q] >> col) & 1u)) continue;
            const int sat = __builtin_popcountll(seen[Q]);
            open.erase({-sat, -(int)adj[Q].size(), Q});
            seen[Q] |= 1ull << col;
            open.insert({-(sat + 1), -(int)adj[Q].size(), Q});
        }
    }
    mc.ncolor = ncolor;
    mc.h_pcolor = color;
    mc.cptr.assign(ncolor + 1, 0);
    for (int P = 0; P < np; P++) mc.cptr[color[P] + 1]++;
    for (int k = 0; k < ncolor; k++) mc.cptr[k + 1] += mc.cptr[k];
    std::vector<int> patches(np), fill(mc.cptr.begin(), mc.cptr.end() - 1);
    for (int P = 0; P < np; P++) patches[fill[color[P]]++] = P;
    // position key of a row in the factorisation order
    auto key = [&](int j) { return (int64_t)color[j / kMcRows] * n + j; };
    std::vector<int> slot(c->nnzb), scol(c->nnzb);
    std::vector<int4> meta(n);
    std::vector<int> lf(n, 0), lb(n, 0);
    std::vector<int> maxrow_in(range_count(n), 0);
    parallel_ranges(n, [&](int rt, int64_t i0, int64_t i1) {
    std::vector<std::pair<int64_t, int>> lo, up;
    int &maxrow = maxrow_in[rt];
    for (int i = (int)i0; i < (int)i1; i++) {
        lo.clear();
        up.clear();
        const int64_t ki = key(i);
        const int Pi = i / kMcRows;
        int next = 0, nint = 0;
        for (int k = IA[i]; k < IA[i + 1]; k++) {
            if (k == IAU[i]) continue;
            const int64_t kj = key(JA[k]);
            if (kj < ki) lo.push_back({kj, k});
            else up.push_back({kj, k});
        }
        std::sort(lo.begin(), lo.end());
        std::sort(up.begin(), up.end());
        int w = IA[i];
        for (auto &e : lo) {
            slot[w++] = e.second;
            if (JA[e.second] / kMcRows != Pi) next++;
        }
        slot[w++] = IAU[i];
        for (auto &e : up) {
            slot[w++] = e.second;
            if (JA[e.second] / kMcRows == Pi) nint++;
        }
        // external lower blocks come first in key order (smaller colours),
        // intra-patch upper blocks first among the upper ones
        meta[i] = make_int4(next, (int)lo.size(), nint, 0);
        maxrow = std::max(maxrow, IA[i + 1] - IA[i]);
    }
    });
    const int maxrow = *std::max_element(maxrow_in.begin(), maxrow_in.end());
    parallel_ranges(c->nnzb, [&](int, int64_t u0, int64_t u1) {
        for (int64_t u = u0; u < u1; u++) scol[u] = JA[slot[u]];
    });
    // patch-local dependency levels (a patch's rows depend only on its own rows)
    std::vector<int2> plev(np, make_int2(0, 0));
    parallel_ranges(np, [&](int, int64_t q0, int64_t q1) {
    for (int P = (int)q0; P < (int)q1; P++) {
        const int r0 = P * kMcRows, r1 = std::min(n, r0 + kMcRows);
        for (int i = r0; i < r1; i++) {
            int l = 0;
            for (int u = IA[i] + meta[i].x; u < IA[i] + meta[i].y; u++) l = std::max(l, lf[scol[u]] + 1);
            lf[i] = l;
            plev[P].x = std::max(plev[P].x, l);
        }
        for (int i = r1 - 1; i >= r0; i--) {
            int l = 0;
            const int u0 = IA[i] + meta[i].y + 1;
            for (int u = u0; u < u0 + meta[i].z; u++) l = std::max(l, lb[scol[u]] + 1);
            lb[i] = l;
            plev[P].y = std::max(plev[P].y, l);
        }
    }
    });
    int maxlev = 0;
    for (int P = 0; P < np; P++) maxlev = std::max(maxlev, std::max(plev[P].x, plev[P].y));
    for (int i = 0; i < n; i++) meta[i].w = lf[i] | (lb[i] << 16);
    // update lists of the factorisation: for lower block (i,p), the upper
    // blocks (p,j) of row p whose column j row i also holds
    // Row i's pairs in order: for each lower block u, the upper entries v of
    // row p = JA[slot[base+u]] whose column row i holds (its CRS-local slot by
    // binary search, JA rows being sorted).  Counted, then written, per row.
    std::vector<int4> hdr(c->nnzb, make_int4(0, 0, 0, 0));
    std::vector<int64_t> pair_ptr(n + 1, 0);
    auto row_pairs = [&](int i, int2 *out) {  // returns the row's pair count; writes them when out != nullptr
        const int base = IA[i], end = IA[i + 1];
        const int nlo = meta[i].y;
        int total = 0;
        for (int u = 0; u < nlo; u++) {
            const int kk = slot[base + u], p = JA[kk];
            int cnt = 0;
            for (int v = IA[p] + meta[p].y + 1; v < IA[p + 1]; v++) {
                const int j = scol[v];
                const int *it = std::lower_bound(&JA[base], &JA[0] + end, j);
                if (it != &JA[0] + end && *it == j) {
                    if (out) out[total + cnt] = make_int2(v, (int)(it - &JA[base]));
                    cnt++;
                }
            }
            if (out) hdr[base + u] = make_int4(IA[p] + meta[p].y, cnt, kk - base, 0);
            total += cnt;
        }
        return total;
    };
    parallel_ranges(n, [&](int, int64_t i0, int64_t i1) {
        for (int i = (int)i0; i < (int)i1; i++) pair_ptr[i + 1] = row_pairs(i, nullptr);
    });
    int maxstage = 1;
    for (int i = 0; i < n; i++) {
        maxstage = std::max<int64_t>(maxstage, meta[i].y + pair_ptr[i + 1]);
        pair_ptr[i + 1] += pair_ptr[i];
    }
    std::vector<int2> pairs(std::max<int64_t>(pair_ptr[n], 1));
    parallel_ranges(n, [&](int, int64_t i0, int64_t i1) {
        for (int i = (int)i0; i < (int)i1; i++) row_pairs(i, pairs.data() + pair_ptr[i]);
    });
    // row records and packed-layout slots of the triangular solves, in launch
    // order (colour, then position of the patch in the colour, then row)
    std::vector<int4> rowf((size_t)np * kMcRows), rowb((size_t)np * kMcRows), rowl((size_t)np * kMcRows);
    std::vector<int64_t> lslot(np + 1, 0), uslot(np + 1, 0);
    for (int pos = 0; pos < np; pos++) {
        const int P = patches[pos];
        int lmax = 0, umax = 0;
        for (int q = 0; q < kMcRows; q++) {
            const int i = P * kMcRows + q;
            const size_t e = (size_t)pos * kMcRows + q;
            if (i < n) {
                const int base = IA[i], diag = base + meta[i].y;
                rowf[e] = make_int4(i, meta[i].x, meta[i].y, base);
                rowb[e] = make_int4(i, meta[i].z, IA[i + 1] - diag - 1, diag);
                rowl[e] = make_int4(lf[i], plev[P].x, lb[i], plev[P].y);
                lmax = std::max(lmax, meta[i].y);
                umax = std::max(umax, IA[i + 1] - diag - 1);
            } else {
                rowf[e] = rowb[e] = make_int4(-1, 0, 0, 0);
                rowl[e] = make_int4(-1, plev[P].x, -1, plev[P].y);
            }
        }
        lslot[pos + 1] = lslot[pos] + lmax;
        uslot[pos + 1] = uslot[pos] + umax;
    }
    std::vector<int> colL((size_t)lslot[np] * kMcRows, 0), colU((size_t)uslot[np] * kMcRows, 0);
    parallel_ranges(np, [&](int, int64_t q0, int64_t q1) {
    for (int pos = (int)q0; pos < (int)q1; pos++) {
        const int p0 = patches[pos] * kMcRows;
        for (int q = 0; q < kMcRows; q++) {
            const int4 rf = rowf[(size_t)pos * kMcRows + q], rb = rowb[(size_t)pos * kMcRows + q];
            if (rf.x < 0) continue;
            for (int t = 0; t < rf.z; t++) {
                const int j = scol[rf.w + t];
                colL[(size_t)(lslot[pos] + t) * kMcRows + q] = t < rf.y ? j : j - p0;
            }
            for (int t = 0; t < rb.z; t++) {
                const int j = scol[rb.w + 1 + t];
                colU[(size_t)(uslot[pos] + t) * kMcRows + q] = t < rb.y ? j - p0 : j;
            }
        }
    }
    });
    mc.nlslot = lslot[np];
    mc.nuslot = uslot[np];
    CFD_CUDA(mc.rowf.upload(rowf.data(), rowf.size(), c->stream));
    CFD_CUDA(mc.rowb.upload(rowb.data(), rowb.size(), c->stream));
    CFD_CUDA(mc.rowl.upload(rowl.data(), rowl.size(), c->stream));
    CFD_CUDA(mc.lslot.upload(lslot.data(), lslot.size(), c->stream));
    CFD_CUDA(mc.uslot.upload(uslot.data(), uslot.size(), c->stream));
    CFD_CUDA(mc.colL.upload(colL.data(), std::max<size_t>(1, colL.size()), c->stream));
    CFD_CUDA(mc.colU.upload(colU.data(), std::max<size_t>(1, colU.size()), c->stream));
    mc.maxrow = maxrow;
    mc.maxlev = maxlev;
    mc.maxstage = maxstage;
    CFD_CUDA(mc.patches.upload(patches.data(), patches.size(), c->stream));
    CFD_CUDA(mc.slot.upload(slot.data(), slot.size(), c->stream));
    CFD_CUDA(mc.scol.upload(scol.data(), scol.size(), c->stream));
    CFD_CUDA(mc.meta.upload(meta.data(), meta.size(), c->stream));
    CFD_CUDA(mc.plev.upload(plev.data(), plev.size(), c->stream));
    CFD_CUDA(mc.hdr.upload(hdr.data(), hdr.size(), c->stream));
    CFD_CUDA(mc.pair_ptr.upload(pair_ptr.data(), pair_ptr.size(), c->stream));
    CFD_CUDA(mc.pairs.upload(pairs.data(), (size_t)pair_ptr[n], c->stream));
    CFD_CUDA(stream_wait(c->stream));  // host vectors go out of scope
    mc.built = true;
    return CFD_OK;
}

template <typename TA, typename TM>
int mc_factor(cfd_ctx *c, const TA *A, TM *M) {
    Abmc &mc = c->mc;
    int st = mc_build(c);
    if (st) return st;
    // four warps (patches) per CTA, fewer when their staging does not fit in
    // 200 KB; several CTAs share an SM so every SM gets patches
    const size_t per_warp = mc_factor_warp_bytes<TM>(mc.maxrow, mc.maxstage);
    const int nwarp = (int)std::max<size_t>(1, std::min<size_t>(4, (200u << 10) / per_warp));
    if (per_warp > (200u << 10)) {
        set_error("ILU(0) multicolour: a row needs %d staged blocks, more than fit in shared memory",
                  mc.maxrow + mc.maxstage);
        return CFD_ERR_RANGE;
    }
    const size_t smem = per_warp * nwarp;
    int smax = 0;
    CFD_CUDA(allow_max_dynamic_smem(k_mc_factor<TA, TM>, c->device, &smax));
    if (smem > (size_t)smax) {
        set_error("ILU(0) multicolour: %zu bytes of shared memory needed, %d available", smem, smax);
        return CFD_ERR_RANGE;
    }
    for (int k = 0; k < mc.ncolor; k++) {
        const int cnt = mc.cptr[k + 1] - mc.cptr[k];
        k_mc_factor<TA, TM><<<grid_for(cnt, nwarp), 32 * nwarp, smem, c->stream>>>(
            mc.patches.p + mc.cptr[k], cnt, c->nnode, mc.maxrow, mc.maxstage, c->IA.p, mc.slot.p, mc.meta.p,
            mc.hdr.p, mc.pair_ptr.p, mc.pairs.p, A, M, c->err.p);
    }
    CFD_LAUNCH_CHECK();
    // the triangular solves read the factors in their packed layout
    McPack<TM> &pk = mc.pack<TM>();
    const int np = mc.cptr[mc.ncolor];
    const size_t nl = (size_t)mc.nlslot * 25 * kMcRows, nu = (size_t)mc.nuslot * 25 * kMcRows,
                 nd = (size_t)np * 25 * kMcRows;
    if (pk.L.n != std::max<size_t>(1, nl) || pk.U.n != std::max<size_t>(1, nu) || pk.D.n != nd) {
        mc.clear_graphs();  // captured applies hold the old addresses
        CFD_CUDA(pk.L.alloc(std::max<size_t>(1, nl)));
        CFD_CUDA(pk.U.alloc(std::max<size_t>(1, nu)));
        CFD_CUDA(pk.D.alloc(nd));
    }
    k_mc_pack<TM><<<np, 5 * kMcRows, 0, c->stream>>>(mc.rowf.p, mc.rowb.p, mc.lslot.p, mc.uslot.p, M, pk.L.p, pk.U.p,
                                                      pk.D.p);
    CFD_LAUNCH_CHECK();
    return CFD_OK;
}

template <typename TM>
static int mc_apply_launch(cfd_ctx *c, const TM *M, const double *r, double *tmp, double *z) {
    Abmc &mc = c->mc;
    (void)M;  // the solves read the packed copy mc_factor made of M
    struct {
        const TM *L, *U, *D;
    } pk{mc.pack<TM>().L.p, mc.pack<TM>().U.p, mc.pack<TM>().D.p};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t lc = {};
    lc.blockDim = dim3(5 * kMcRows);
    lc.dynamicSmemBytes = 0;
    lc.stream = c->stream;
    lc.attrs = at;
    lc.numAttrs = 1;
    for (int k = 0; k < mc.ncolor; k++) {
        lc.gridDim = dim3(mc.cptr[k + 1] - mc.cptr[k]);
        // the first colour starts after the stream's earlier work has completed
        // (no early start), so r is complete in every colour's launch
        lc.numAttrs = k == 0 ? 0 : 1;
        const size_t e = (size_t)mc.cptr[k] * kMcRows;
        CFD_CUDA(cudaLaunchKernelEx(&lc, k_mc_fwd<TM>, (const int4 *)(mc.rowf.p + e), (const int4 *)(mc.rowl.p + e),
                                    (const int64_t *)(mc.lslot.p + mc.cptr[k]), (const int *)mc.colL.p,
                                    (const TM *)pk.L, r, tmp));
    }
    lc.numAttrs = 1;
    for (int k = mc.ncolor - 1; k >= 0; k--) {
        lc.gridDim = dim3(mc.cptr[k + 1] - mc.cptr[k]);
        const size_t e = (size_t)mc.cptr[k] * kMcRows;
        CFD_CUDA(cudaLaunchKernelEx(&lc, k_mc_bwd<TM>, (const int4 *)(mc.rowb.p + e), (const int4 *)(mc.rowl.p + e),
                                    (const int64_t *)(mc.uslot.p + mc.cptr[k]), (const int *)mc.colU.p,
                                    (const TM *)pk.U, (const TM *)(pk.D + e * 25), (const double *)tmp, z));
    }
    CFD_LAUNCH_CHECK();
    return CFD_OK;
}

// The 2 x ncolor launches of an apply, replayed as one captured CUDA graph
// when the context has its own stream (the legacy stream cannot be
// captured): the host then issues one launch instead of 2 x ncolor, which is
// what bounds small systems.  Graphs are cached per pointer set.
template <typename TM>
int mc_apply(cfd_ctx *c, const TM *M, const double *r, double *tmp, double *z) {
    Abmc &mc = c->mc;
    if (!c->stream) return mc_apply_launch<TM>(c, M, r, tmp, z);
    for (const auto &g : mc.graphs)
        if (g.M == M && g.r == r && g.tmp == tmp && g.z == z) {
            CFD_CUDA(cudaGraphLaunch(g.exec, c->stream));
            return CFD_OK;
        }
    if (mc.graphs.size() >= 64) mc.clear_graphs();
    cudaGraph_t graph = nullptr;
    CFD_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int st = mc_apply_launch<TM>(c, M, r, tmp, z);
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (st) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    CFD_CUDA(e);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    CFD_CUDA(ei);
    mc.graphs.push_back({M, r, tmp, z, exec});
    CFD_CUDA(cudaGraphLaunch(exec, c->stream));
    return CFD_OK;
}

template int mc_factor<double, double>(cfd_ctx *, const double *, double *);
template int mc_factor<double, float>(cfd_ctx *, const double *, float *);
template int mc_factor<float, float>(cfd_ctx *, const float *, float *);
template int mc_factor<uint16_t, float>(cfd_ctx *, const uint16_t *, float *);
template int mc_apply<double>(cfd_ctx *, const double *, const double *, double *, double *);
template int mc_apply<float>(cfd_ctx *, const float *, const double *, double *, double *);

}  // namespace cfd

using namespace cfd;

extern "C" int cfd_ilu_mc_order(cfd_ctx *c, int *order, int *ncolor) {
    if (!c || !c->has_mesh) { cfd::set_error("cfd_ilu_mc_order: no mesh"); return CFD_ERR_STATE; }
    CFD_CUDA(cudaSetDevice(c->device));
    int st = mc_build(c);
    if (st) return st;
    const Abmc &mc = c->mc;
    if (ncolor) *ncolor = mc.ncolor;
    if (order) {
        const int n = c->nnode;
        int k = 0;
        for (int col = 0; col < mc.ncolor; col++)
            for (int P = 0; P * kMcRows < n; P++)
                if (mc.h_pcolor[P] == col)
                    for (int i = P * kMcRows; i < std::min(n, (P + 1) * kMcRows); i++) order[k++] = i;
    }
    return CFD_OK;
}
