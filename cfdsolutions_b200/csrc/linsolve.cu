// Block-CRS linear algebra of the implicit step: block SpMV (FP64 / FP32 /
// BF16 storage, FP64 accumulation), block-Jacobi and block-ILU(0)
// preconditioners (level-scheduled, FP32 or FP64 factors), restarted
// right-preconditioned GMRES(m) with FP64 Arnoldi and compensated dot
// products, FP64 iterative refinement around a reduced-precision inner solve,
// and the implicit steady driver.
//
// The reference has no block GMRES or ILU(0) on this path: its implicit
// drivers call block Gauss-Seidel / LU-SGS (Euler3D/src/Solver_Steady_Implicit.cpp:144,
// MATH/src/MC_Iterative_Jacobi.c:346,540) and its only GMRES is an unused
// MPI scalar-CRS, point-Jacobi GMRES (MATH/src/ParallelLinearAlgebra.cpp:27-278),
// whose restart/Givens structure this follows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.cuh"
#include "kernels.cuh"
#include "ilu_mc.cuh"

namespace cfd {

// ------------------------------------------------------------ reductions

__global__ void k_sum_partial(const double *__restrict__ x, int64_t n, double *__restrict__ part) {
    __shared__ double sh[256];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += x[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_sum_one(const double *__restrict__ part, int nblk, double *__restrict__ out) {
    __shared__ double sh[256];
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += part[b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

int reduce_sum_plain(cfd_ctx *c, const double *x, int64_t n, double *out_host) {
    const int nblk = 296;
    CFD_CUDA(c->red.alloc(std::max<size_t>(c->red.n, (size_t)nblk * 128)));
    CFD_CUDA(c->red_out.alloc(std::max<size_t>(c->red_out.n, 64)));
    k_sum_partial<<<nblk, 256, 0, c->stream>>>(x, n, c->red.p);
    CFD_LAUNCH_CHECK();
    k_sum_one<<<1, 256, 0, c->stream>>>(c->red.p, nblk, c->red_out.p);
    CFD_LAUNCH_CHECK();
    CFD_CUDA(cudaMemcpyAsync(out_host, c->red_out.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CFD_CUDA(stream_wait(c->stream));
    return CFD_OK;
}

// Error-free transformations (Knuth TwoSum, FMA TwoProd) for the compensated
// dot products of Ogita, Rump and Oishi, "Accurate sum and dot product"
// (SIAM J. Sci. Comput. 26, 2005), algorithm Dot2.
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
    s = a + b;
    const double z = s - a;
    e = (a - (s - z)) + (b - z);
}

// One product of a Dot2 sum: (s, c) += x * b with TwoProd and TwoSum.
__device__ __forceinline__ void dot2_acc(double x, double b, double &s, double &c) {
    const double p = x * b;
    const double pe = fma(x, b, -p);
    double t, e;
    two_sum(s, p, t, e);
    s = t;
    c += e + pe;
}

constexpr int MAXK = 64;
constexpr int MD_THREADS = 256;

// The block's CH (sum, compensation) pairs of vectors j0 .. j0+nj-1 combined
// and stored in part[block][j]: a warp butterfly (error-free TwoSum is
// symmetric in its arguments, so every lane holds the same pair), then the
// warps in order.
template <int CH>
__device__ __forceinline__ void dot2_block_store(double (&s)[CH], double (&c)[CH], int j0, int nj,
                                                 double (*shs)[MD_THREADS / 32], double (*shc)[MD_THREADS / 32],
                                                 double *__restrict__ part) {
    constexpr int NW = MD_THREADS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int jj = 0; jj < CH; jj++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double so = __shfl_xor_sync(0xffffffffu, s[jj], o);
            const double co = __shfl_xor_sync(0xffffffffu, c[jj], o);
            double t, e;
            two_sum(s[jj], so, t, e);
            s[jj] = t;
            c[jj] = (c[jj] + co) + e;
        }
        if (lane == 0) { shs[jj][wid] = s[jj]; shc[jj][wid] = c[jj]; }
    }
    __syncthreads();
    if (wid == 0 && lane < nj) {
        double ss = shs[lane][0], cc = shc[lane][0];
        for (int q = 1; q < NW; q++) {
            double t, e;
            two_sum(ss, shs[lane][q], t, e);
            ss = t;
            cc = (cc + shc[lane][q]) + e;
        }
        part[(blockIdx.x * MAXK + j0 + lane) * 2] = ss;
        part[(blockIdx.x * MAXK + j0 + lane) * 2 + 1] = cc;
    }
    __syncthreads();
}

// Dot2 of k vectors V[j] (stride ld) against w, one (sum, compensation)
// pair per vector per block.  Vectors are taken CH at a time (w is read
// once per chunk); each thread takes the elements i, i + G, i + 2G, ... of
// the grid G in that order, U of them per step with all their loads issued
// before the sums, so that U (CH + 1) loads are in flight per thread.  A
// vector's sum does not depend on CH or U: only on the grid, so results
// repeat run to run and between the instantiations.
template <int CH, int U>
__global__ void __launch_bounds__(MD_THREADS) k_mdot_partial(const double *__restrict__ V, int64_t ld, int k,
                                                             const double *__restrict__ w, int64_t n,
                                                             double *__restrict__ part) {
    __shared__ double shs[CH][MD_THREADS / 32], shc[CH][MD_THREADS / 32];
    const int64_t G = (int64_t)gridDim.x * blockDim.x;
    for (int j0 = 0; j0 < k; j0 += CH) {
        const int nj = min(CH, k - j0);
        double s[CH], c[CH];
#pragma unroll
        for (int jj = 0; jj < CH; jj++) { s[jj] = 0.0; c[jj] = 0.0; }
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        for (; i + (U - 1) * G < n; i += U * G) {
            double b[U], a[U][CH];
#pragma unroll
            for (int u = 0; u < U; u++) {
                b[u] = w[i + u * G];
#pragma unroll
                for (int jj = 0; jj < CH; jj++)
                    if (jj < nj) a[u][jj] = V[(int64_t)(j0 + jj) * ld + i + u * G];
            }
#pragma unroll
            for (int u = 0; u < U; u++)
#pragma unroll
                for (int jj = 0; jj < CH; jj++)
                    if (jj < nj) dot2_acc(a[u][jj], b[u], s[jj], c[jj]);
        }
        for (; i < n; i += G) {
            const double b = w[i];
#pragma unroll
            for (int jj = 0; jj < CH; jj++)
                if (jj < nj) dot2_acc(V[(int64_t)(j0 + jj) * ld + i], b, s[jj], c[jj]);
        }
        dot2_block_store<CH>(s, c, j0, nj, shs, shc, part);
    }
}

// A Gram-Schmidt update and the next reduction in one pass over w:
// w_i -= h_0 V_0i, then h_1 V_1i, ... (one fused multiply-add each, in j
// order), then the Dot2 partials of <V_j, w> for j < k or, SELF, of <w, w>,
// with k_mdot_partial's element order.  Each element's update is made and
// stored by the thread that reads it back in the later chunks, so the
// results are bit for bit those of the update followed by k_mdot_partial,
// with V read from DRAM once (k <= CH) instead of twice and w once instead
// of three times.
template <bool SELF, int CH, int U>
__global__ void __launch_bounds__(MD_THREADS) k_axpy_mdot_partial(const double *__restrict__ V, int64_t ld, int k,
                                                                  const double *__restrict__ h, double *__restrict__ w,
                                                                  int64_t n, double *__restrict__ part) {
    __shared__ double shs[CH][MD_THREADS / 32], shc[CH][MD_THREADS / 32];
    __shared__ double hs[MAXK];
    for (int j = threadIdx.x; j < k; j += blockDim.x) hs[j] = h[j];
    __syncthreads();
    const int64_t G = (int64_t)gridDim.x * blockDim.x;
    const int kd = SELF ? 1 : k;
    for (int j0 = 0; j0 < kd; j0 += CH) {
        const int nj = min(CH, kd - j0);
        double s[CH], c[CH];
#pragma unroll
        for (int jj = 0; jj < CH; jj++) { s[jj] = 0.0; c[jj] = 0.0; }
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        for (; i + (U - 1) * G < n; i += U * G) {
            double b[U];
#pragma unroll
            for (int u = 0; u < U; u++) b[u] = w[i + u * G];
            if (j0 == 0) {
#pragma unroll 2
                for (int j = 0; j < k; j++) {
                    double v[U];
#pragma unroll
                    for (int u = 0; u < U; u++) v[u] = V[(int64_t)j * ld + i + u * G];
#pragma unroll
                    for (int u = 0; u < U; u++) b[u] -= hs[j] * v[u];
                }
#pragma unroll
                for (int u = 0; u < U; u++) w[i + u * G] = b[u];
            }
#pragma unroll
            for (int u = 0; u < U; u++)
#pragma unroll
                for (int jj = 0; jj < CH; jj++)
                    if (jj < nj) {
                        // V_j again: the same thread has just read it (an L1 hit)
                        const double x = SELF ? b[u] : V[(int64_t)(j0 + jj) * ld + i + u * G];
                        dot2_acc(x, b[u], s[jj], c[jj]);
                    }
        }
        for (; i < n; i += G) {
            double b = w[i];
            if (j0 == 0) {
                for (int j = 0; j < k; j++) b -= hs[j] * V[(int64_t)j * ld + i];
                w[i] = b;
            }
#pragma unroll
            for (int jj = 0; jj < CH; jj++)
                if (jj < nj) dot2_acc(SELF ? b : V[(int64_t)(j0 + jj) * ld + i], b, s[jj], c[jj]);
        }
        dot2_block_store<CH>(s, c, j0, nj, shs, shc, part);
    }
}

__global__ void k_mdot_final(const double *__restrict__ part, int nblk, int k, double *__restrict__ out) {
    const int j = blockIdx.x;
    if (j >= k) return;
    __shared__ double shs[256], shc[256];
    double s = 0.0, c = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
        double t, e;
        two_sum(s, part[(b * MAXK + j) * 2], t, e);
        s = t;
        c += e + part[(b * MAXK + j) * 2 + 1];
    }
    shs[threadIdx.x] = s;
    shc[threadIdx.x] = c;
    __syncthreads();
    for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            double t, e;
            two_sum(shs[threadIdx.x], shs[threadIdx.x + o], t, e);
            shs[threadIdx.x] = t;
            shc[threadIdx.x] += shc[threadIdx.x + o] + e;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = shs[0] + shc[0];
}

static const int kRedBlocks = 1184;  // 8 x 148 SMs

// Device scalars of the GMRES driver, in c->dots (doubles):
//   [0, MAXK)        dot results read back by the host; [MAXK/2, MAXK) also
//                    holds the host-computed combination coefficients y
//   [MAXK, 2 MAXK)   first Gram-Schmidt coefficients h1
//   [2 MAXK, 3 MAXK) re-orthogonalisation coefficients h2
//   [3 MAXK, 4 MAXK) Hessenberg column h1 + h2 | ||w|| ; last entry 1/||w||
//   [4 MAXK]         ||w||^2
constexpr int DOT_H1 = MAXK, DOT_H2 = 2 * MAXK, DOT_COL = 3 * MAXK, DOT_NRM = 4 * MAXK, DOT_LEN = 5 * MAXK;

// out_dev[j] = <V_j, w>, j < k, compensated, deterministic; stays on the device.
// The chunk width follows k and the elements per step shrink as it grows, to
// keep the registers (and so the resident blocks) and the loads in flight up.
static int mdot_dev(cfd_ctx *c, const double *V, int64_t ld, int k, const double *w, int64_t n, double *out_dev) {
    if (k <= 1) k_mdot_partial<1, 8><<<kRedBlocks, MD_THREADS, 0, c->stream>>>(V, ld, k, w, n, c->red.p);
    else if (k <= 4) k_mdot_partial<4, 4><<<kRedBlocks, MD_THREADS, 0, c->stream>>>(V, ld, k, w, n, c->red.p);
    else k_mdot_partial<8, 2><<<kRedBlocks, MD_THREADS, 0, c->stream>>>(V, ld, k, w, n, c->red.p);
    CFD_LAUNCH_CHECK();
    k_mdot_final<<<k, 256, 0, c->stream>>>(c->red.p, kRedBlocks, k, out_dev);
    CFD_LAUNCH_CHECK();
    return CFD_OK;
}

// w -= V h (h = h_dev[0..k) on the device), then out_dev[j] = <V_j, w>
// (j < k) or, self, out_dev[0] = <w, w>: the update and mdot_dev in one pass.
static int axpy_mdot_dev(cfd_ctx *c, const double *V, int64_t ld, int k, const double *h_dev, double *w, int64_t n,
                         bool self, double *out_dev) {
    const int g = kRedBlocks, t = MD_THREADS;
    double *part = c->red.p;
    if (self) k_axpy_mdot_partial<true, 1, 4><<<g, t, 0, c->stream>>>(V, ld, k, h_dev, w, n, part);
    else if (k <= 4) k_axpy_mdot_partial<false, 4, 4><<<g, t, 0, c->stream>>>(V, ld, k, h_dev, w, n, part);
    else k_axpy_mdot_partial<false, 8, 2><<<g, t, 0, c->stream>>>(V, ld, k, h_dev, w, n, part);
    CFD_LAUNCH_CHECK();
    const int kd = self ? 1 : k;
    k_mdot_final<<<kd, 256, 0, c->stream>>>(c->red.p, kRedBlocks, kd, out_dev);
    CFD_LAUNCH_CHECK();
    return CFD_OK;
}

static int dot_buffers(cfd_ctx *c) {
    CFD_CUDA(c->red.alloc(std::max<size_t>(c->red.n, (size_t)kRedBlocks * 128)));
    CFD_CUDA(c->dots.alloc(std::max<size_t>(c->dots.n, (size_t)DOT_LEN)));
    return CFD_OK;
}

// out_host[j] = <V_j, w>, j < k, compensated, deterministic.
static int mdot(cfd_ctx *c, const double *V, int64_t ld, int k, const double *w, int64_t n, double *out_host) {
    int st = dot_buffers(c);
    if (st || (st = mdot_dev(c, V, ld, k, w, n, c->dots.p))) return st;
    CFD_CUDA(cudaMemcpyAsync(out_host, c->dots.p, sizeof(double) * k, cudaMemcpyDeviceToHost, c->stream));
    CFD_CUDA(stream_wait(c->stream));
    return CFD_OK;
}

// Hessenberg column j of the Arnoldi step: h1 + h2 (CGS2), ||w||, 1/||w||.
__global__ void k_arnoldi_column(int j, double *__restrict__ dots) {
    const int i = threadIdx.x;
    if (i <= j) dots[DOT_COL + i] = dots[DOT_H1 + i] + dots[DOT_H2 + i];
    if (i == 0) {
        const double hn = sqrt(fmax(dots[DOT_NRM], 0.0));
        dots[DOT_COL + j + 1] = hn;
        dots[DOT_COL + MAXK - 1] = hn > 0.0 ? 1.0 / hn : 0.0;
    }
}

// --------------------------------------------------------- vector kernels

__global__ void k_scale_copy(int64_t n, double a, const double *__restrict__ x, double *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = a * x[i];
}

// y = (*a) x with the factor read on the device.
__global__ void k_scale_copy_dev(int64_t n, const double *__restrict__ a, const double *__restrict__ x,
                                 double *__restrict__ y) {
    const double f = *a;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = f * x[i];
}

__global__ void k_comb(int64_t n, int k, const double *__restrict__ V, int64_t ld, const double *__restrict__ y,
                       double *__restrict__ out) {
    // out = sum_j y_j V_j
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < k; j++) s += y[j] * V[(int64_t)j * ld + i];
        out[i] = s;
    }
}

__global__ void k_add(int64_t n, const double *__restrict__ x, double *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += x[i];
}

__global__ void k_sub(int64_t n, const double *__restrict__ b, const double *__restrict__ ax, double *__restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = b[i] - ax[i];
}

// ----------------------------------------------------------- block SpMV
// y_i = sum_k A_k x_{JA[k]}, FP64 accumulation whatever the storage type.
// Five lanes per block row, lane m forming output m from row m of each 5x5
// block: the five lanes of a row read its 100-byte FP32 block together, and a
// warp covers 6.4 consecutive rows, whose blocks are consecutive in memory.
// Two blocks per step with their own partial sums (even and odd blocks of the
// row, added at the end) keep twice the loads in flight.  Measured at 128^3
// (2.15 M rows, 31.8 M blocks, FP32): 0.78 ms, 4.46 TB/s of algorithmic
// traffic; one warp per row (lane = block element, contiguous 100-byte block
// loads) reached only 1.7-2.3 TB/s, staging the row through shared memory
// 3.1 TB/s: fewer bytes in flight per warp.
template <typename TA>
__device__ __forceinline__ double ldA(const TA *p);
template <>
__device__ __forceinline__ double ldA<double>(const double *p) { return __ldg(p); }
template <>
__device__ __forceinline__ double ldA<float>(const float *p) { return (double)__ldg(p); }
template <>
__device__ __forceinline__ double ldA<uint16_t>(const uint16_t *p) { return load_low(p); }

// thread t of a block SpMV: row t/5, component t%5
template <typename TA>
__device__ __forceinline__ void bspmv_thread(int t, int nrow, const int *__restrict__ IA, const int *__restrict__ JA,
                                             const TA *__restrict__ A, const double *__restrict__ x,
                                             double *__restrict__ y) {
    const int r = t / 5, m = t - 5 * r;
    if (r >= nrow) return;
    double s0 = 0.0, s1 = 0.0;
    int k = IA[r];
    const int k1 = IA[r + 1];
    for (; k + 1 < k1; k += 2) {
        const TA *a = A + (int64_t)k * 25 + m * 5;
        const double *xv = x + (int64_t)JA[k] * 5, *xw = x + (int64_t)JA[k + 1] * 5;
        double av[10];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            av[q] = ldA<TA>(a + q);
            av[5 + q] = ldA<TA>(a + 25 + q);
        }
#pragma unroll
        for (int q = 0; q < 5; q++) {
            s0 = fma(av[q], __ldg(xv + q), s0);
            s1 = fma(av[5 + q], __ldg(xw + q), s1);
        }
    }
    if (k < k1) {
        const TA *a = A + (int64_t)k * 25 + m * 5;
        const double *xv = x + (int64_t)JA[k] * 5;
#pragma unroll
        for (int q = 0; q < 5; q++) s0 = fma(ldA<TA>(a + q), __ldg(xv + q), s0);
    }
    y[(int64_t)r * 5 + m] = s0 + s1;
}

template <typename TA>
__global__ void __launch_bounds__(160) k_bspmv(int nrow, const int *__restrict__ IA, const int *__restrict__ JA,
                                               const TA *__restrict__ A, const double *__restrict__ x,
                                               double *__restrict__ y) {
    bspmv_thread<TA>(blockIdx.x * blockDim.x + threadIdx.x, nrow, IA, JA, A, x, y);
}

// Several requests' SpMVs in one launch (the serving loop's fused SpMV): CTA
// b belongs to the job whose [block_begin, next block_begin) holds it, and
// computes that job's rows exactly as k_bspmv's CTA b - block_begin would.
template <typename TA>
__global__ void __launch_bounds__(160) k_bspmv_batch(const __grid_constant__ SpmvBatch B) {
    int j = 0;
    while (j + 1 < B.njobs && (int)blockIdx.x >= B.job[j + 1].block_begin) j++;
    const SpmvJob &J = B.job[j];
    bspmv_thread<TA>(((int)blockIdx.x - J.block_begin) * 160 + (int)threadIdx.x, J.nrow, J.IA, J.JA,
                     static_cast<const TA *>(J.A), J.x, J.y);
}

int launch_spmv_batch(int key, const SpmvBatch &b, cudaStream_t s) {
    int blocks = 0;
    for (int k = 0; k < b.njobs; k++) blocks += grid_for(5 * (int64_t)b.job[k].nrow, 160);
    if (blocks == 0) return CFD_OK;
    switch (key - kSpmvKey) {
        case CFD_PREC_FP64: k_bspmv_batch<double><<<blocks, 160, 0, s>>>(b); break;
        case CFD_PREC_FP32: k_bspmv_batch<float><<<blocks, 160, 0, s>>>(b); break;
        case CFD_PREC_BF16: k_bspmv_batch<uint16_t><<<blocks, 160, 0, s>>>(b); break;
        default: return CFD_ERR_UNSUPPORTED;
    }
    CFD_LAUNCH_CHECK();
    return CFD_OK;
}

// ------------------------------------------------------ preconditioners
// 5x5 inverse by Gauss-Jordan with partial pivoting (FP64).
__device__ __forceinline__ bool inv5(const double *a_in, double *inv) {
    double a[25];
#pragma unroll
    for (int k = 0; k < 25; k++) { a[k] = a_in[k]; inv[k] = (k % 6 == 0) ? 1.0 : 0.0; }
#pragma unroll
    for (int c = 0; c < 5; c++) {
        int p = c;
        double best = fabs(a[c * 5 + c]);
#pragma unroll
        for (int r = c + 1; r < 5; r++)
            if (fabs(a[r * 5 + c]) > best) { best = fabs(a[r * 5 + c]); p = r; }
        if (!(best > 0.0)) return false;
        if (p != c) {
#pragma unroll
            for (int j = 0; j < 5; j++) {
                double t = a[c * 5 + j]; a[c * 5 + j] = a[p * 5 + j]; a[p * 5 + j] = t;
                t = inv[c * 5 + j]; inv[c * 5 + j] = inv[p * 5 + j]; inv[p * 5 + j] = t;
            }
        }
        const double d = 1.0 / a[c * 5 + c];
#pragma unroll
        for (int j = 0; j < 5; j++) { a[c * 5 + j] *= d; inv[c * 5 + j] *= d; }
#pragma unroll
        for (int r = 0; r < 5; r++) {
            if (r == c) continue;
            const double f = a[r * 5 + c];
#pragma unroll
            for (int j = 0; j < 5; j++) { a[r * 5 + j] -= f * a[c * 5 + j]; inv[r * 5 + j] -= f * inv[c * 5 + j]; }
        }
    }
    return true;
}

template <typename TM>
__device__ __forceinline__ void stM(TM *p, double v);
template <>
__device__ __forceinline__ void stM<double>(double *p, double v) { *p = v; }
template <>
__device__ __forceinline__ void stM<float>(float *p, double v) { *p = (float)v; }

// Block-Jacobi: M_i = inv(A_ii).
template <typename TM>
__global__ void k_bjacobi_factor(int nrow, const int *__restrict__ IAU, const double *__restrict__ A,
                                 TM *__restrict__ M, int *__restrict__ err) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrow) return;
    double inv[25];
    if (!inv5(A + (int64_t)IAU[r] * 25, inv)) atomicOr(err, ERR_NAN);
#pragma unroll
    for (int k = 0; k < 25; k++) stM<TM>(M + (int64_t)r * 25 + k, inv[k]);
}

template <typename TM>
__global__ void __launch_bounds__(160) k_bjacobi_apply(int nrow, const TM *__restrict__ M, const double *__restrict__ r,
                                                       double *__restrict__ z) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / 5, m = t - 5 * i;
    if (i >= nrow) return;
    const TM *a = M + (int64_t)i * 25 + m * 5;
    const double *rv = r + (int64_t)i * 5;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 5; j++) s = fma(ldA<TM>(a + j), rv[j], s);
    z[(int64_t)i * 5 + m] = s;
}

// Block ILU(0), IKJ variant on the matrix pattern, one level of rows at a
// time (row i only reads rows p < i of earlier levels).  Factors are formed in
// FP64 in F (a copy of A) and stored as: strictly lower blocks L_ip
// (unit-diagonal L), strictly upper blocks U_ij, and the inverse of U_ii in the
// diagonal slot.
__global__ void __launch_bounds__(64) k_ilu0_level(int nrows, const int *__restrict__ rows, const int *__restrict__ IA,
                                                   const int *__restrict__ JA, const int *__restrict__ IAU,
                                                   double *__restrict__ F, int *__restrict__ err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    const int i = rows[t];
    const int rb = IA[i], re = IA[i + 1], di = IAU[i];
    for (int k = rb; k < di; k++) {
        const int p = JA[k];
        double *Lip = F + (int64_t)k * 25;
        const double *Dp = F + (int64_t)IAU[p] * 25;  // inverse of U_pp
        // blocks are staged in registers: F is read and written through the
        // same pointer, so direct use would serialise every load behind the
        // previous store
        double a_ip[25], d_p[25], L[25];
#pragma unroll
        for (int q = 0; q < 25; q++) { a_ip[q] = Lip[q]; d_p[q] = Dp[q]; }
#pragma unroll
        for (int a = 0; a < 5; a++)
#pragma unroll
            for (int b = 0; b < 5; b++) {
                double s = 0.0;
#pragma unroll
                for (int q = 0; q < 5; q++) s = fma(a_ip[a * 5 + q], d_p[q * 5 + b], s);
                L[a * 5 + b] = s;
            }
#pragma unroll
        for (int q = 0; q < 25; q++) Lip[q] = L[q];
        // row i, columns j > p  -=  L_ip U_pj  (merge of the two sorted rows)
        int m = k + 1;
        int pk = IAU[p] + 1;
        const int pe = IA[p + 1];
        while (m < re && pk < pe) {
            const int jm = JA[m], jp = JA[pk];
            if (jm < jp) { m++; continue; }
            if (jp < jm) { pk++; continue; }
            double *Aij = F + (int64_t)m * 25;
            const double *Upj = F + (int64_t)pk * 25;
            double u[25], t[25];
#pragma unroll
            for (int q = 0; q < 25; q++) { u[q] = Upj[q]; t[q] = Aij[q]; }
#pragma unroll
            for (int a = 0; a < 5; a++)
#pragma unroll
                for (int b = 0; b < 5; b++) {
                    double s = t[a * 5 + b];
#pragma unroll
                    for (int q = 0; q < 5; q++) s = fma(-L[a * 5 + q], u[q * 5 + b], s);
                    t[a * 5 + b] = s;
                }
#pragma unroll
            for (int q = 0; q < 25; q++) Aij[q] = t[q];
            m++;
            pk++;
        }
    }
    double inv[25];
    if (!inv5(F + (int64_t)di * 25, inv)) atomicOr(err, ERR_NAN);
#pragma unroll
    for (int q = 0; q < 25; q++) F[(int64_t)di * 25 + q] = inv[q];
}

template <typename TM>
__global__ void k_cast_factors(int64_t n, const double *__restrict__ F, TM *__restrict__ M) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        stM<TM>(M + i, F[i]);
}

// forward: y_i = r_i - sum_{p<i} L_ip y_p    (five lanes per row)
template <typename TM>
__global__ void __launch_bounds__(160) k_ilu_fwd(int nrows, const int *__restrict__ rows, const int *__restrict__ IA,
                                                 const int *__restrict__ JA, const int *__restrict__ IAU,
                                                 const TM *__restrict__ M, const double *__restrict__ r,
                                                 double *__restrict__ y) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = t / 5, m = t - 5 * q;
    if (q >= nrows) return;
    const int i = rows[q];
    double s = r[(int64_t)i * 5 + m];
    for (int k = IA[i]; k < IAU[i]; k++) {
        const TM *a = M + (int64_t)k * 25 + m * 5;
        const double *yv = y + (int64_t)JA[k] * 5;
#pragma unroll
        for (int j = 0; j < 5; j++) s = fma(-ldA<TM>(a + j), yv[j], s);
    }
    y[(int64_t)i * 5 + m] = s;
}

// backward: z_i = inv(U_ii) (y_i - sum_{j>i} U_ij z_j); the five lanes of a
// row exchange their partial sums through shared memory (a block of 160
// threads holds 32 whole rows, so a row never straddles blocks, but it can
// straddle warps).
template <typename TM>
__global__ void __launch_bounds__(160) k_ilu_bwd(int nrows, const int *__restrict__ rows, const int *__restrict__ IA,
                                                 const int *__restrict__ JA, const int *__restrict__ IAU,
                                                 const TM *__restrict__ M, const double *__restrict__ y,
                                                 double *__restrict__ z) {
    __shared__ double sh[160];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = t / 5, m = t - 5 * q;
    const bool act = q < nrows;
    int i = 0;
    double s = 0.0;
    if (act) {
        i = rows[q];
        s = y[(int64_t)i * 5 + m];
        for (int k = IAU[i] + 1; k < IA[i + 1]; k++) {
            const TM *a = M + (int64_t)k * 25 + m * 5;
            const double *zv = z + (int64_t)JA[k] * 5;
#pragma unroll
            for (int j = 0; j < 5; j++) s = fma(-ldA<TM>(a + j), zv[j], s);
        }
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    if (act) {
        const int base = threadIdx.x - m;
        const TM *d = M + (int64_t)IAU[i] * 25 + m * 5;
        double o = 0.0;
#pragma unroll
        for (int j = 0; j < 5; j++) o = fma(ldA<TM>(d + j), sh[base + j], o);
        z[(int64_t)i * 5 + m] = o;
    }
}

// ------------------------------------------------------------ GMRES driver

struct Precond {
    int kind = CFD_PC_NONE;
    int prec = CFD_PREC_FP64;
};

static int precond_setup(cfd_ctx *c, const Precond &pc) {
    const int n = c->nnode;
    if (pc.kind == CFD_PC_NONE) return CFD_OK;
    if (!c->a64_valid && pc.kind != CFD_PC_ILU0_MC) {
        set_error("gmres: with a low-precision-only system the preconditioner must be CFD_PC_ILU0_MC or none");
        return CFD_ERR_STATE;
    }
    if (pc.kind == CFD_PC_BLOCK_JACOBI) {
        if (pc.prec == CFD_PREC_FP64) {
            CFD_CUDA(c->M64.alloc((size_t)n * 25));
            k_bjacobi_factor<double><<<grid_for(n, 128), 128, 0, c->stream>>>(n, c->IAU.p, c->A64.p, c->M64.p, c->err.p);
        } else {
            CFD_CUDA(c->M32.alloc((size_t)n * 25));
            k_bjacobi_factor<float><<<grid_for(n, 128), 128, 0, c->stream>>>(n, c->IAU.p, c->A64.p, c->M32.p, c->err.p);
        }
        CFD_LAUNCH_CHECK();
        return check_device_error(c);
    }
    const size_t nz = (size_t)c->nnzb * 25;
    if (pc.kind == CFD_PC_ILU0_MC) {
        // block multicolour order: factors read straight from the stored
        // matrix (its own precision), FP64 arithmetic, stored in pc.prec
        if (pc.prec == CFD_PREC_FP64) {
            CFD_CUDA(c->M64.alloc(nz));
            int st = mc_factor<double, double>(c, c->A64.p, c->M64.p);
            if (st) return st;
        } else {
            CFD_CUDA(c->M32.alloc(nz));
            int st;
            if (c->a_precision == CFD_PREC_FP32 && c->A32.p) st = mc_factor<float, float>(c, c->A32.p, c->M32.p);
            else if (c->a_precision == CFD_PREC_BF16 && c->A16.p)
                st = mc_factor<uint16_t, float>(c, c->A16.p, c->M32.p);
            else st = mc_factor<double, float>(c, c->A64.p, c->M32.p);
            if (st) return st;
        }
        return check_device_error(c);
    }
    // ILU(0): factor in FP64 in M64, then cast when FP32 storage is wanted
    CFD_CUDA(c->M64.alloc(nz));
    CFD_CUDA(cudaMemcpyAsync(c->M64.p, c->A64.p, nz * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    Levels &L = c->lv_fwd;
    const int nl = (int)L.ptr.size() - 1;
    for (int l = 0; l < nl; l++) {
        const int lo = L.ptr[l], cnt = L.ptr[l + 1] - lo;
        k_ilu0_level<<<grid_for(cnt, 64), 64, 0, c->stream>>>(cnt, L.rows.p + lo, c->IA.p, c->JA.p, c->IAU.p,
                                                                c->M64.p, c->err.p);
    }
    CFD_LAUNCH_CHECK();
    if (pc.prec != CFD_PREC_FP64) {
        CFD_CUDA(c->M32.alloc(nz));
        k_cast_factors<float><<<1184, 256, 0, c->stream>>>((int64_t)nz, c->M64.p, c->M32.p);
        CFD_LAUNCH_CHECK();
    }
    return check_device_error(c);
}

template <typename TM>
static void ilu_apply(cfd_ctx *c, const TM *M, const double *r, double *tmp, double *z) {
    Levels &F = c->lv_fwd, &B = c->lv_bwd;
    for (int l = 0; l + 1 < (int)F.ptr.size(); l++) {
        const int lo = F.ptr[l], cnt = F.ptr[l + 1] - lo;
        k_ilu_fwd<TM><<<grid_for(5 * (int64_t)cnt, 160), 160, 0, c->stream>>>(cnt, F.rows.p + lo, c->IA.p, c->JA.p,
                                                                               c->IAU.p, M, r, tmp);
    }
    for (int l = 0; l + 1 < (int)B.ptr.size(); l++) {
        const int lo = B.ptr[l], cnt = B.ptr[l + 1] - lo;
        k_ilu_bwd<TM><<<grid_for(5 * (int64_t)cnt, 160), 160, 0, c->stream>>>(cnt, B.rows.p + lo, c->IA.p, c->JA.p,
                                                                               c->IAU.p, M, tmp, z);
    }
}

static int precond_apply(cfd_ctx *c, const Precond &pc, const double *r, double *tmp, double *z) {
    const int n = c->nnode;
    const int64_t len = (int64_t)n * 5;
    switch (pc.kind) {
        case CFD_PC_NONE:
            CFD_CUDA(cudaMemcpyAsync(z, r, len * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
            break;
        case CFD_PC_BLOCK_JACOBI:
            if (pc.prec == CFD_PREC_FP64)
                k_bjacobi_apply<double><<<grid_for(len, 160), 160, 0, c->stream>>>(n, c->M64.p, r, z);
            else
                k_bjacobi_apply<float><<<grid_for(len, 160), 160, 0, c->stream>>>(n, c->M32.p, r, z);
            break;
        case CFD_PC_ILU0_MC: {
            const int st = pc.prec == CFD_PREC_FP64 ? mc_apply<double>(c, c->M64.p, r, tmp, z)
                                                    : mc_apply<float>(c, c->M32.p, r, tmp, z);
            if (st) return st;
            break;
        }
        default:
            if (pc.prec == CFD_PREC_FP64) ilu_apply<double>(c, c->M64.p, r, tmp, z);
            else ilu_apply<float>(c, c->M32.p, r, tmp, z);
            break;
    }
    CFD_LAUNCH_CHECK();
    return CFD_OK;
}

static int spmv(cfd_ctx *c, int prec, const double *x, double *y) {
    const int n = c->nnode;
    const int g = grid_for(5 * (int64_t)n, 160), b = 160;
    if (prec == CFD_PREC_FP64 && !c->a64_valid) prec = c->a_precision;  // low-precision-only system
    const void *A = prec == CFD_PREC_FP32 && c->A32.p   ? (const void *)c->A32.p
                    : prec == CFD_PREC_BF16 && c->A16.p ? (const void *)c->A16.p
                                                        : (const void *)c->A64.p;
    if (A == c->A64.p) prec = CFD_PREC_FP64;
    if (c->batcher) {
        // the serving loop fuses this launch with other requests' (bit-identical per row)
        const SpmvJob job{n, c->IA.p, c->JA.p, A, x, y, 0};
        return c->batch_submit(c->batcher, c, kSpmvKey + prec, &job);
    }
    if (prec == CFD_PREC_FP32)
        k_bspmv<float><<<g, b, 0, c->stream>>>(n, c->IA.p, c->JA.p, static_cast<const float *>(A), x, y);
    else if (prec == CFD_PREC_BF16)
        k_bspmv<uint16_t><<<g, b, 0, c->stream>>>(n, c->IA.p, c->JA.p, static_cast<const uint16_t *>(A), x, y);
    else
        k_bspmv<double><<<g, b, 0, c->stream>>>(n, c->IA.p, c->JA.p, static_cast<const double *>(A), x, y);
    CFD_LAUNCH_CHECK();
    return CFD_OK;
}

static int vnorm(cfd_ctx *c, const double *x, int64_t n, double *out) {
    double s;
    int st = mdot(c, x, 0, 1, x, n, &s);
    if (st) return st;
    *out = sqrt(fmax(s, 0.0));
    return CFD_OK;
}

// Restarted right-preconditioned GMRES(m) for A_p d = r (A_p = A in storage
// precision `aprec`), d starting at zero.  Classical Gram-Schmidt with one
// re-orthogonalisation pass (CGS2), compensated FP64 dot products, Givens
// rotations on the host.  Returns inner iterations in *its.
static int gmres_inner(cfd_ctx *c, int aprec, const Precond &pc, int m, int max_iters, double tol_abs,
                       const double *r, double *d, int *its, int *restarts, double *res_est) {
    const int64_t n5 = (int64_t)c->nnode * 5;
    const int64_t ld = n5;
    double *V = c->V.p;
    double *w = c->work.p;           // [n5]
    double *tmp = c->work.p + n5;    // [n5]
    double *zz = c->work.p + 2 * n5; // [n5]
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), h(m + 1), y(m);
    int st0 = dot_buffers(c);
    if (st0) return st0;
    CFD_CUDA(cudaMemsetAsync(d, 0, n5 * sizeof(double), c->stream));
    CFD_CUDA(cudaMemcpyAsync(w, r, n5 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    int total = 0, nrst = 0;
    double beta;
    int st = vnorm(c, w, n5, &beta);
    if (st) return st;
    *res_est = beta;
    while (total < max_iters && beta > tol_abs) {
        if (!std::isfinite(beta)) { set_error("gmres: non-finite residual"); return CFD_ERR_NUMERIC; }
        k_scale_copy<<<1184, 256, 0, c->stream>>>(n5, 1.0 / beta, w, V);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        for (; j < m && total < max_iters; j++, total++) {
            // w = A M^-1 v_j
            if ((st = precond_apply(c, pc, V + j * ld, tmp, zz))) return st;
            if ((st = spmv(c, aprec, zz, w))) return st;
            // CGS2 with the coefficients kept on the device; one read-back
            // of the Hessenberg column per step
            double *dd = c->dots.p;
            if ((st = mdot_dev(c, V, ld, j + 1, w, n5, dd + DOT_H1))) return st;
            if ((st = axpy_mdot_dev(c, V, ld, j + 1, dd + DOT_H1, w, n5, false, dd + DOT_H2))) return st;
            if ((st = axpy_mdot_dev(c, V, ld, j + 1, dd + DOT_H2, w, n5, true, dd + DOT_NRM))) return st;
            k_arnoldi_column<<<1, MAXK, 0, c->stream>>>(j, dd);
            k_scale_copy_dev<<<1184, 256, 0, c->stream>>>(n5, dd + DOT_COL + MAXK - 1, w, V + (j + 1) * ld);
            CFD_LAUNCH_CHECK();
            CFD_CUDA(cudaMemcpyAsync(h.data(), dd + DOT_COL, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost,
                                     c->stream));
            CFD_CUDA(stream_wait(c->stream));
            const double hn = h[j + 1];
            if (!std::isfinite(hn)) { set_error("gmres: breakdown (non-finite)"); return CFD_ERR_NUMERIC; }
            // apply previous rotations, form a new one
            for (int i = 0; i < j; i++) {
                const double t = cs[i] * h[i] + sn[i] * h[i + 1];
                h[i + 1] = -sn[i] * h[i] + cs[i] * h[i + 1];
                h[i] = t;
            }
            const double den = std::hypot(h[j], h[j + 1]);
            if (den == 0.0) { set_error("gmres: zero Hessenberg column"); return CFD_ERR_NUMERIC; }
            cs[j] = h[j] / den;
            sn[j] = h[j + 1] / den;
            h[j] = den;
            h[j + 1] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            for (int i = 0; i <= j; i++) H[(size_t)i * m + j] = h[i];
            *res_est = std::fabs(g[j + 1]);
            if (*res_est <= tol_abs || hn == 0.0) { j++; total++; break; }
        }
        // y = H^-1 g (upper triangular j x j)
        for (int i = j - 1; i >= 0; i--) {
            double s = g[i];
            for (int k = i + 1; k < j; k++) s -= H[(size_t)i * m + k] * y[k];
            y[i] = s / H[(size_t)i * m + i];
        }
        // d += M^-1 (V y)
        CFD_CUDA(cudaMemcpyAsync(c->dots.p + MAXK / 2, y.data(), sizeof(double) * j, cudaMemcpyHostToDevice, c->stream));
        k_comb<<<1184, 256, 0, c->stream>>>(n5, j, V, ld, c->dots.p + MAXK / 2, tmp);
        if ((st = precond_apply(c, pc, tmp, w, zz))) return st;
        k_add<<<1184, 256, 0, c->stream>>>(n5, zz, d);
        CFD_LAUNCH_CHECK();
        // true residual for the restart: w = r - A d
        if ((st = spmv(c, aprec, d, tmp))) return st;
        k_sub<<<1184, 256, 0, c->stream>>>(n5, r, tmp, w);
        CFD_LAUNCH_CHECK();
        if ((st = vnorm(c, w, n5, &beta))) return st;
        *res_est = beta;
        nrst++;
    }
    *its = total;
    *restarts = nrst;
    return CFD_OK;
}

}  // namespace cfd

using namespace cfd;

// Physical-time terms of one inner iteration (Solver_Unsteady_Implicit.cpp:
// 181-216), one thread per node: s = V/dt ((1+theta)(Q - Q^n) - theta (Q^n -
// Q^n-1)) is subtracted from B and added to the convective residual (for
// the RMS), and (1+theta) V/dt joins the diagonal block of every stored
// precision.  qn / qn1 are [5][n] copies of the physical nodes.
template <typename TA>
__global__ void k_unsteady_terms(int n, int64_t ldq, const double *__restrict__ Q, const double *__restrict__ qn,
                                 const double *__restrict__ qn1, const double *__restrict__ vol, double dt,
                                 double theta, const int *__restrict__ IAU, double *__restrict__ B,
                                 double *__restrict__ res, double *__restrict__ A64, TA *__restrict__ Alow) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double eta = vol[i] / dt;
#pragma unroll
    for (int v = 0; v < 5; v++) {
        const double q = Q[v * ldq + i], a = qn[v * (int64_t)n + i], b = qn1[v * (int64_t)n + i];
        const double src = eta * ((1.0 + theta) * (q - a) - theta * (a - b));
        B[(int64_t)i * 5 + v] -= src;
        res[v * (int64_t)n + i] += src;
    }
    const double d = (1.0 + theta) * eta;
    const int64_t dg = (int64_t)IAU[i] * 25;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        if (A64) A64[dg + 6 * k] += d;
        if (Alow) store_low(Alow + dg + 6 * k, load_low(Alow + dg + 6 * k) + d);
    }
}

// Copies the physical part of Q ([5][ldq]) to a [5][n] history array.
__global__ void k_copy_state(int n, int64_t ldq, const double *__restrict__ Q, double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int v = 0; v < 5; v++) out[v * (int64_t)n + i] = Q[v * ldq + i];
}

extern "C" {

void cfd_gmres_default(cfd_gmres_opts *o) {
    if (!o) return;
    o->restart = 30;
    o->max_iters = 300;
    o->rtol = 1e-6;
    o->precond = CFD_PC_ILU0;
    o->precision = CFD_PREC_FP64;
    o->refine = 1;
    o->reuse_precond = 0;
}

int cfd_gmres(cfd_ctx *c, const cfd_gmres_opts *o, cfd_gmres_stats *stats) {
    if (!c || !c->has_mesh) { set_error("cfd_gmres: no mesh"); return CFD_ERR_STATE; }
    if (!c->has_system) { set_error("cfd_gmres: no system (call cfd_jacobian)"); return CFD_ERR_STATE; }
    cfd_gmres_opts opt;
    if (o) opt = *o; else cfd_gmres_default(&opt);
    if (opt.restart < 1 || opt.restart > MAXK / 2 - 1 || opt.max_iters < 1 || !(opt.rtol > 0.0)) {
        set_error("cfd_gmres: restart must be in [1,%d], max_iters >= 1, rtol > 0", MAXK / 2 - 1);
        return CFD_ERR_ARG;
    }
    if (opt.precond < CFD_PC_NONE || opt.precond > CFD_PC_ILU0_MC) return CFD_ERR_ARG;
    opt.precision &= ~CFD_PREC_LOW_ONLY;  // the matrix storage is decided by cfd_jacobian
    if (opt.precision < CFD_PREC_FP64 || opt.precision > CFD_PREC_BF16) return CFD_ERR_ARG;
    CFD_CUDA(cudaSetDevice(c->device));
    const int64_t n5 = (int64_t)c->nnode * 5;
    const int m = opt.restart;
    CFD_CUDA(c->V.alloc((size_t)(m + 1) * n5));
    CFD_CUDA(c->work.alloc(std::max<size_t>(c->work.n, (size_t)5 * n5)));
    // storage precision of the matrix used inside GMRES
    int aprec = opt.precision;
    if (aprec == CFD_PREC_FP32 && c->a_precision != CFD_PREC_FP32) aprec = CFD_PREC_FP64;
    if (aprec == CFD_PREC_BF16 && c->a_precision != CFD_PREC_BF16) aprec = CFD_PREC_FP64;
    if (!c->a64_valid) aprec = c->a_precision;  // only the low-precision matrix exists
    Precond pc;
    pc.kind = opt.precond;
    pc.prec = (opt.precision == CFD_PREC_FP64 && c->a64_valid) ? CFD_PREC_FP64 : CFD_PREC_FP32;
    int st = CFD_OK;
    if (!(opt.reuse_precond && c->pc_valid && c->pc_kind == pc.kind && c->pc_prec == pc.prec)) {
        c->pc_valid = false;
        if ((st = precond_setup(c, pc))) return st;
        c->pc_valid = true;
        c->pc_kind = pc.kind;
        c->pc_prec = pc.prec;
    }
    double *x = c->X.p;
    double *r = c->work.p + 3 * n5;
    double *d = c->work.p + 4 * n5;
    CFD_CUDA(cudaMemsetAsync(x, 0, n5 * sizeof(double), c->stream));
    double bnorm;
    if ((st = vnorm(c, c->B.p, n5, &bnorm))) return st;
    cfd_gmres_stats s{};
    if (bnorm == 0.0) {
        if (stats) *stats = s;
        return CFD_OK;
    }
    const int nref = std::max(1, opt.refine);
    double rel = 1.0;
    int left = opt.max_iters;
    for (int it = 0; it < nref && left > 0; it++) {
        // FP64 defect: r = B - A64 x
        if ((st = spmv(c, CFD_PREC_FP64, x, r))) return st;
        k_sub<<<1184, 256, 0, c->stream>>>(n5, c->B.p, r, r);
        CFD_LAUNCH_CHECK();
        double rn;
        if ((st = vnorm(c, r, n5, &rn))) return st;
        rel = rn / bnorm;
        if (rel <= opt.rtol) break;
        int its = 0, rs = 0;
        double est = 0.0;
        // inner tolerance relative to this defect; the final check is FP64
        const double tol_abs = std::max(opt.rtol * bnorm, (nref > 1 ? 1e-3 : 1.0) * opt.rtol * rn);
        st = gmres_inner(c, aprec, pc, m, left, nref > 1 ? std::max(opt.rtol * bnorm, 1e-4 * rn) : tol_abs, r, d,
                         &its, &rs, &est);
        if (st) return st;
        k_add<<<1184, 256, 0, c->stream>>>(n5, d, x);
        CFD_LAUNCH_CHECK();
        s.iterations += its;
        s.restarts += rs;
        s.refinements = it + 1;
        left -= its;
    }
    // final FP64 residual
    if ((st = spmv(c, CFD_PREC_FP64, x, r))) return st;
    k_sub<<<1184, 256, 0, c->stream>>>(n5, c->B.p, r, r);
    CFD_LAUNCH_CHECK();
    double rn;
    if ((st = vnorm(c, r, n5, &rn))) return st;
    s.rel_residual = rn / bnorm;
    if (stats) *stats = s;
    if (!std::isfinite(s.rel_residual)) {
        set_error("gmres: non-finite final residual (right-hand side norm %g)", bnorm);
        return CFD_ERR_NUMERIC;
    }
    return s.rel_residual <= opt.rtol * 1.0000001 ? CFD_OK : CFD_ERR_NOT_CONVERGED;
}

int cfd_spmv(cfd_ctx *c, int precision, const double *x, double *y) {
    if (!c || !c->has_mesh) { set_error("cfd_spmv: no mesh"); return CFD_ERR_STATE; }
    if (!c->has_system) { set_error("cfd_spmv: no system (call cfd_jacobian)"); return CFD_ERR_STATE; }
    if (!x || !y || precision < CFD_PREC_FP64 || precision > CFD_PREC_BF16) {
        set_error("cfd_spmv: device vectors x, y and a CFD_PREC_* precision");
        return CFD_ERR_ARG;
    }
    CFD_CUDA(cudaSetDevice(c->device));
    return spmv(c, precision, x, y);
}

int cfd_precond_apply(cfd_ctx *c, const double *r, double *z) {
    if (!c || !c->has_mesh) { set_error("cfd_precond_apply: no mesh"); return CFD_ERR_STATE; }
    if (!c->pc_valid) { set_error("cfd_precond_apply: no preconditioner (call cfd_gmres)"); return CFD_ERR_STATE; }
    if (!r || !z) { set_error("cfd_precond_apply: device vectors r, z"); return CFD_ERR_ARG; }
    CFD_CUDA(cudaSetDevice(c->device));
    const int64_t n5 = (int64_t)c->nnode * 5;
    CFD_CUDA(c->work.alloc(std::max<size_t>(c->work.n, (size_t)5 * n5)));
    Precond pc;
    pc.kind = c->pc_kind;
    pc.prec = c->pc_prec;
    return precond_apply(c, pc, r, c->work.p + 2 * n5, z);
}

int cfd_solve_unsteady(cfd_ctx *c, const cfd_unsteady_opts *o, cfd_unsteady_stats *stats) {
    if (!c || !c->has_mesh || !o) { set_error("cfd_solve_unsteady: no mesh / options"); return CFD_ERR_STATE; }
    if (!(o->dt > 0.0) || o->steps < 0 || o->inner_iterations < 1) {
        set_error("cfd_solve_unsteady: dt > 0, steps >= 0 and inner_iterations >= 1");
        return CFD_ERR_ARG;
    }
    if (c->params.variables != CFD_VARS_CONSERVATIVE) {
        // the physical-time terms difference conservative states (Solver_Unsteady_Implicit.cpp)
        set_error("cfd_solve_unsteady: conservative variables only");
        return CFD_ERR_UNSUPPORTED;
    }
    const int n = c->nnode;
    DevBuf<double> qn, qn1;
    CFD_CUDA(qn.alloc((size_t)5 * n));
    CFD_CUDA(qn1.alloc((size_t)5 * n));
    const int g = grid_for(n, 256);
    cfd_unsteady_stats s{};
    int st = CFD_OK;
    const int prec = o->linear_solver == 1 ? o->gmres.precision : CFD_PREC_FP64;
    for (int t = 0; t < o->steps && !st; t++) {
        const double theta = (o->bdf2 && t > 0) ? 0.5 : 0.0;
        if (o->bdf2) CFD_CUDA(cudaMemcpyAsync(qn1.p, qn.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToDevice, c->stream));
        k_copy_state<<<g, 256, 0, c->stream>>>(n, c->ldq, c->Q.p, qn.p);
        CFD_LAUNCH_CHECK();
        if (t == 0) CFD_CUDA(cudaMemcpyAsync(qn1.p, qn.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToDevice, c->stream));
        for (int it = 0; it < o->inner_iterations; it++) {
            if ((st = cfd_begin_iteration(c, it))) break;
            if (c->params.order == CFD_ORDER_SECOND) {
                if ((st = cfd_gradient(c))) break;
                if (c->params.limiter != CFD_LIMITER_NONE && (st = cfd_limiter(c))) break;
            }
            if ((st = cfd_apply_bc(c, it))) break;
            if ((st = cfd_residual(c, 0))) break;
            if ((st = cfd_jacobian(c, 0, o->include_diss, prec))) break;
            double *A64 = c->a64_valid ? c->A64.p : nullptr;
            if (c->a_precision == CFD_PREC_FP32)
                k_unsteady_terms<float><<<g, 256, 0, c->stream>>>(n, c->ldq, c->Q.p, qn.p, qn1.p, c->cvol.p, o->dt,
                                                                 theta, c->IAU.p, c->B.p, c->res.p, A64, c->A32.p);
            else if (c->a_precision == CFD_PREC_BF16)
                k_unsteady_terms<uint16_t><<<g, 256, 0, c->stream>>>(n, c->ldq, c->Q.p, qn.p, qn1.p, c->cvol.p,
                                                                    o->dt, theta, c->IAU.p, c->B.p, c->res.p, A64,
                                                                    c->A16.p);
            else
                k_unsteady_terms<float><<<g, 256, 0, c->stream>>>(n, c->ldq, c->Q.p, qn.p, qn1.p, c->cvol.p, o->dt,
                                                                 theta, c->IAU.p, c->B.p, c->res.p, A64,
                                                                 (float *)nullptr);
            CFD_LAUNCH_CHECK();
            double rms[6];
            if ((st = cfd_residual_rms(c, o->include_diss, rms))) break;
            if ((st = check_device_error(c))) break;
            s.rms_last = rms[5];
            s.inner_iterations++;
            if (!std::isfinite(rms[5])) { set_error("cfd_solve_unsteady: non-finite residual"); st = CFD_ERR_NUMERIC; break; }
            if (o->linear_solver == 1) {
                cfd_gmres_stats gs{};
                cfd_gmres_opts go = o->gmres;
                go.reuse_precond = 0;
                st = cfd_gmres(c, &go, &gs);
                s.linear_iterations += gs.iterations;
                if (st == CFD_ERR_NOT_CONVERGED) st = CFD_OK;
                if (st) break;
            } else {
                double lr;
                if ((st = cfd_block_gs(c, o->linear_iters, 0, &lr))) break;
                s.linear_iterations += o->linear_iters;
            }
            if ((st = cfd_update(c, o->relax))) break;
        }
        if (!st) s.steps = t + 1;
    }
    s.status = st;
    if (stats) *stats = s;
    return st;
}

int cfd_solve_steady(cfd_ctx *c, const cfd_solve_opts *o, cfd_solve_stats *stats) {
    if (!c || !c->has_mesh || !o) { set_error("cfd_solve_steady: no mesh / options"); return CFD_ERR_STATE; }
    cfd_solve_stats s{};
    int st = CFD_OK;
    for (int iter = 0; iter < o->max_iterations; iter++) {
        if ((st = cfd_begin_iteration(c, iter))) break;
        if ((st = cfd_apply_bc(c, iter))) break;
        if (c->params.order == CFD_ORDER_SECOND) {
            if ((st = cfd_gradient(c))) break;
            if (c->params.limiter != CFD_LIMITER_NONE && (st = cfd_limiter(c))) break;
        }
        if ((st = cfd_residual(c, 1))) break;
        if ((st = cfd_deltat(c, iter))) break;
        double rms[6];
        if ((st = cfd_residual_rms(c, o->include_diss, rms))) break;
        if ((st = check_device_error(c))) break;
        if (iter == 0) s.rms_first = rms[5];
        s.rms_last = rms[5];
        s.iterations = iter + 1;
        if (!std::isfinite(rms[5])) {
            set_error("cfd_solve_steady: non-finite residual at implicit iteration %d", iter);
            st = CFD_ERR_NUMERIC;
            break;
        }
        if (rms[5] <= o->drop * s.rms_first && iter > 0) break;
        if (rms[5] < 10.0 * DBL_EPSILON) break;  // Solver_Steady_Implicit.cpp:176
        const int prec = o->linear_solver == 1 ? o->gmres.precision : CFD_PREC_FP64;
        if ((st = cfd_jacobian(c, 1, o->include_diss, prec))) break;
        if (o->linear_solver == 1) {
            cfd_gmres_stats gs{};
            cfd_gmres_opts go = o->gmres;
            go.reuse_precond = (o->precond_update > 1 && iter % o->precond_update != 0) ? 1 : 0;
            st = cfd_gmres(c, &go, &gs);
            s.linear_iterations += gs.iterations;
            if (st == CFD_ERR_NOT_CONVERGED) st = CFD_OK;  // inexact Newton step
            if (st) break;
        } else {
            double lr;
            if ((st = cfd_block_gs(c, o->linear_iters, 0, &lr))) break;
            s.linear_iterations += o->linear_iters;
        }
        if ((st = cfd_update(c, o->relax))) break;
    }
    s.status = st;
    if (stats) *stats = s;
    return st;
}

}  // extern "C"
