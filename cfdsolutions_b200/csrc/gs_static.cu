// Block Gauss-Seidel for callers that cannot allocate device memory.
//
// cfd_block_gs allocates its work arrays (LU factors of the diagonal blocks,
// per-row residuals, reduction partials) with cudaMalloc on first use.  Some
// callers cannot let a library do that: a host framework that reserved all
// device memory up front and hands out only its own buffers, or a solver loop
// that must not reach the CUDA allocator once it is running.  For them,
// cfd_block_gs_static runs the same level-scheduled sweeps (same kernels,
// same arithmetic) on a system the caller already holds in device memory, and
// keeps every scratch value in one fixed-size static device array of this
// library instead.
//
// Cost and limits:
//   * the array holds scratch for CFD_GS_STATIC_MAX_ROWS block rows and is
//     reserved on every GPU that loads the library, until the process exits;
//   * systems with more rows are rejected with CFD_ERR_RANGE;
//   * all calls share the one array, so calls that overlap on the GPU (two
//     streams, or two host threads) race on it and give wrong results: order
//     them on one stream or synchronise between them;
//   * the array keeps the previous call's contents; everything that must start
//     at zero (the solution) is cleared by each call.
// The device address of the array is looked up once per device, with that
// device current, on the first call made on it; make that first call before
// any stream capture begins.  The address stays cached for the life of the
// process, so do not call cudaDeviceReset (or otherwise destroy the device's
// primary context) while this entry point is still in use.
//
// Host cost per call: the pattern (IA, IAU, then JA) is copied to the host
// with two synchronising copies and checked, both level schedules are rebuilt
// on the host (O(nnz)), and each sweep synchronises once to read its RMS.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cfloat>
#include <mutex>
#include <vector>

#include "ctx.cuh"
#include "kernels.cuh"

namespace cfd {

// LU blocks (25 doubles per row) | squared row residuals (1 per row) |
// level schedules, forward then backward (2 ints per row) | 296 partial sums
// | 1 total.  Sized in doubles.
constexpr int64_t kGsStaticDoubles = (int64_t)CFD_GS_STATIC_MAX_ROWS * 26 + CFD_GS_STATIC_MAX_ROWS + 296 + 8;
static __device__ __align__(256) double g_gs_scratch[kGsStaticDoubles];

namespace {
std::mutex g_gs_mutex;
double *g_gs_ptr[256] = {nullptr};  // device address of g_gs_scratch per device

int gs_scratch_address(int device, double **out) {
    std::lock_guard<std::mutex> lock(g_gs_mutex);
    if (device < 0 || device >= 256) return CFD_ERR_ARG;
    if (!g_gs_ptr[device]) {
        // the symbol's name is only a host-side handle; its device address is
        // looked up here with `device` current
        double *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_gs_scratch);
        if (e != cudaSuccess) {
            set_error("cfd_block_gs_static: cudaGetSymbolAddress failed on device %d: %s", device,
                      cudaGetErrorString(e));
            return CFD_ERR_CUDA;
        }
        g_gs_ptr[device] = p;
    }
    *out = g_gs_ptr[device];
    return CFD_OK;
}

// Level schedule of the forward (lower) or backward (upper) dependencies;
// rows of a level in ascending order.
void levels_host(const std::vector<int> &IA, const std::vector<int> &JA, int n, bool forward,
                 std::vector<int> &ptr, std::vector<int> &rows) {
    std::vector<int> lev(n, 0);
    int maxl = 0;
    for (int q = 0; q < n; q++) {
        const int i = forward ? q : n - 1 - q;
        int l = 0;
        for (int k = IA[i]; k < IA[i + 1]; k++) {
            const int j = JA[k];
            if (forward ? j < i : j > i) l = std::max(l, lev[j] + 1);
        }
        lev[i] = l;
        maxl = std::max(maxl, l);
    }
    ptr.assign(maxl + 2, 0);
    for (int i = 0; i < n; i++) ptr[lev[i] + 1]++;
    for (int l = 0; l <= maxl; l++) ptr[l + 1] += ptr[l];
    rows.assign(n, 0);
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < n; i++) rows[fill[lev[i]]++] = i;
}
}  // namespace

}  // namespace cfd

using namespace cfd;

extern "C" int cfd_block_gs_static(int nrow, const int *dIA, const int *dJA, const int *dIAU, const double *dA,
                                   const double *dB, double *dX, int iterations, int direction, void *stream,
                                   double *rms) {
    if (nrow <= 0 || !dIA || !dJA || !dIAU || !dA || !dB || !dX || direction < 0 || direction > 2) {
        set_error("cfd_block_gs_static: invalid arguments");
        return CFD_ERR_ARG;
    }
    if (nrow > CFD_GS_STATIC_MAX_ROWS) {
        set_error("cfd_block_gs_static: %d block rows exceed the static scratch capacity of %d rows "
                  "(use cfd_block_gs, which allocates)", nrow, CFD_GS_STATIC_MAX_ROWS);
        return CFD_ERR_RANGE;
    }
    int device = 0;
    CFD_CUDA(cudaGetDevice(&device));
    double *scr = nullptr;
    int st = gs_scratch_address(device, &scr);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    double *LU = scr;
    double *rowrms = scr + (int64_t)nrow * 25;
    int *lvl = reinterpret_cast<int *>(scr + (int64_t)CFD_GS_STATIC_MAX_ROWS * 26);  // 2*nrow ints
    double *part = scr + (int64_t)CFD_GS_STATIC_MAX_ROWS * 26 + CFD_GS_STATIC_MAX_ROWS;
    double *total = part + 296;

    // Pattern to the host for the level schedules (host memory only).  The
    // pattern comes from the caller, so it is checked in full before any
    // kernel reads A, JA or IAU through it: IA must be an increasing row
    // pointer starting at 0 (its last entry is the length of JA and A), every
    // column in range, and every IAU[r] the slot of row r's diagonal block.
    std::vector<int> IA(nrow + 1), IAU(nrow);
    CFD_CUDA(cudaMemcpyAsync(IA.data(), dIA, sizeof(int) * (nrow + 1), cudaMemcpyDeviceToHost, s));
    CFD_CUDA(cudaMemcpyAsync(IAU.data(), dIAU, sizeof(int) * nrow, cudaMemcpyDeviceToHost, s));
    CFD_CUDA(cudaStreamSynchronize(s));
    if (IA[0] != 0 || IA[nrow] < nrow) {
        set_error("cfd_block_gs_static: IA is not a block-CRS row pointer (IA[0] = %d, IA[nrow] = %d)", IA[0],
                  IA[nrow]);
        return CFD_ERR_ARG;
    }
    for (int i = 0; i < nrow; i++)
        if (IA[i + 1] <= IA[i]) {  // every row holds at least its diagonal block
            set_error("cfd_block_gs_static: IA is not increasing at row %d (IA[%d] = %d, IA[%d] = %d)", i, i,
                      IA[i], i + 1, IA[i + 1]);
            return CFD_ERR_ARG;
        }
    std::vector<int> JA(IA[nrow]);
    CFD_CUDA(cudaMemcpyAsync(JA.data(), dJA, sizeof(int) * IA[nrow], cudaMemcpyDeviceToHost, s));
    CFD_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < IA[nrow]; k++)
        if (JA[k] < 0 || JA[k] >= nrow) {
            set_error("cfd_block_gs_static: JA[%d] = %d out of range", k, JA[k]);
            return CFD_ERR_ARG;
        }
    for (int r = 0; r < nrow; r++)
        if (IAU[r] < IA[r] || IAU[r] >= IA[r + 1] || JA[IAU[r]] != r) {
            set_error("cfd_block_gs_static: IAU[%d] = %d is not the diagonal slot of row %d", r, IAU[r], r);
            return CFD_ERR_ARG;
        }
    std::vector<int> fptr, frows, bptr, brows;
    levels_host(IA, JA, nrow, true, fptr, frows);
    levels_host(IA, JA, nrow, false, bptr, brows);
    CFD_CUDA(cudaMemcpyAsync(lvl, frows.data(), sizeof(int) * nrow, cudaMemcpyHostToDevice, s));
    CFD_CUDA(cudaMemcpyAsync(lvl + nrow, brows.data(), sizeof(int) * nrow, cudaMemcpyHostToDevice, s));

    // X = 0 (MC_Iterative_Jacobi.c:375); the static array's old contents are
    // overwritten below before they are read
    CFD_CUDA(cudaMemsetAsync(dX, 0, sizeof(double) * 5 * (size_t)nrow, s));
    k_lu_nopivot<<<grid_for(nrow, 128), 128, 0, s>>>(nrow, dA, dIAU, LU);
    CFD_LAUNCH_CHECK();
    if (iterations <= 0) iterations = 10000;
    double r = 0.0;
    for (int it = 0; it < iterations; it++) {
        const bool fwd = direction == 0 || (direction == 2 && it % 2 == 0);
        const std::vector<int> &ptr = fwd ? fptr : bptr;
        const int *rows = fwd ? lvl : lvl + nrow;
        for (size_t l = 0; l + 1 < ptr.size(); l++) {
            const int lo = ptr[l], cnt = ptr[l + 1] - lo;
            k_gs_level<<<grid_for(cnt, 128), 128, 0, s>>>(cnt, rows + lo, dIA, dJA, dIAU, dA, dB, LU, dX, rowrms);
        }
        CFD_LAUNCH_CHECK();
        k_sum_partial<<<296, 256, 0, s>>>(rowrms, nrow, part);
        k_sum_one<<<1, 256, 0, s>>>(part, 296, total);
        CFD_LAUNCH_CHECK();
        double sum = 0.0;
        CFD_CUDA(cudaMemcpyAsync(&sum, total, sizeof(double), cudaMemcpyDeviceToHost, s));
        CFD_CUDA(cudaStreamSynchronize(s));
        r = sqrt(sum / (double)nrow);
        if (r < 100.0 * DBL_EPSILON) break;  // MC_Iterative_Jacobi.c:506
    }
    if (rms) *rms = r;
    return std::isnan(r) ? CFD_ERR_NUMERIC : CFD_OK;
}
