// Device context of the library: resident mesh, state, residual, block-CRS
// system and solver workspaces for one mesh on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <thread>
#include <utility>
#include <vector>

#include "cfd_internal.h"
#include "physics.cuh"

namespace cfd {

// Stream-ordered allocation for the serving workers (serve.cu): while set on
// the calling thread, DevBuf allocates and frees with cudaMallocAsync /
// cudaFreeAsync on that stream, so a worker never synchronises the device
// (cudaFree waits for all streams).  Off (plain cudaMalloc/cudaFree) otherwise.
inline thread_local bool g_alloc_async = false;
inline thread_local cudaStream_t g_alloc_stream = nullptr;

// Waits for the work queued on s.  On a serving worker it polls the stream and
// yields the core between polls instead of blocking in the driver's spin
// wait, so a dozen concurrent solves leave the host cores to the threads that
// issue the launches; elsewhere it is cudaStreamSynchronize.
inline cudaError_t stream_wait(cudaStream_t s) {
    if (!g_alloc_async) return cudaStreamSynchronize(s);
    for (;;) {
        const cudaError_t e = cudaStreamQuery(s);
        if (e != cudaErrorNotReady) return e;
        std::this_thread::yield();
    }
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            if (g_alloc_async) cudaFreeAsync(p, g_alloc_stream);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        if (count == n && p) return cudaSuccess;
        release();
        if (count == 0) return cudaSuccess;
        cudaError_t e = g_alloc_async ? cudaMallocAsync((void **)&p, count * sizeof(T), g_alloc_stream)
                                      : cudaMalloc((void **)&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
    void swap(DevBuf &o) {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
    cudaError_t upload(const T *h, size_t count, cudaStream_t s) {
        cudaError_t e = alloc(count);
        if (e != cudaSuccess || count == 0) return e;
        return cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s);
    }
};

// Level schedule of a sparse triangular dependency (rows grouped so that the
// rows of one level only depend on rows of earlier levels).
struct Levels {
    std::vector<int> ptr;  // host, nlevels+1
    DevBuf<int> rows;      // device, rows in level order
    int max_width = 0;
};

// Factors of one storage type in the triangular solves' packed layout
// (lower slots, upper slots, inverted diagonal blocks; see k_mc_pack).
template <typename TM>
struct McPack {
    DevBuf<TM> L, U, D;
};

// Block multicolour ordering of the ILU(0) preconditioner (ilu_mc.cu): rows
// are grouped in patches of consecutive rows, the patch graph is coloured
// (DSATUR), and the factorisation order is colour by colour, row index within
// a colour.
struct Abmc {
    bool built = false;
    int ncolor = 0, maxrow = 0, maxlev = 0, maxstage = 0;
    std::vector<int> cptr;            // host [ncolor+1] into patches
    std::vector<int> h_pcolor;        // host colour of each patch
    DevBuf<int> patches;              // patch ids in colour order
    DevBuf<int> slot;                 // [nnzb] per row: lower slots (factorisation order) | diag | upper slots
    DevBuf<int> scol;                 // [nnzb] column of each slot entry
    DevBuf<int4> meta;                // per row: external lower, lower, intra-patch upper, lev_f | lev_b << 16
    DevBuf<int2> plev;                // per patch: last forward level, last backward level
    DevBuf<int4> hdr;                 // [nnzb] per lower block: slot of inv(U_pp), pairs, local slot
    DevBuf<int64_t> pair_ptr;         // [n+1] update pairs of each row
    DevBuf<int2> pairs;               // (slot of U_pj, local slot of (i,j))
    // triangular solves: per row in launch order (colour, patch position, row)
    DevBuf<int4> rowf;                // {row, off-patch lower slots, lower slots, first lower slot in M}
    DevBuf<int4> rowb;                // {row, intra-patch upper slots, upper slots, diagonal slot in M}
    DevBuf<int4> rowl;                // {forward level, patch's last, backward level, patch's last}
    // packed layout: per patch position its first lower / upper slot row
    // (slots of 32 rows x 25 entries), and each slot's column per row
    int64_t nlslot = 0, nuslot = 0;
    DevBuf<int64_t> lslot, uslot;     // [npatch+1]
    DevBuf<int> colL, colU;           // [slots][32]
    McPack<float> pk32;
    McPack<double> pk64;
    template <typename TM>
    McPack<TM> &pack();
    // captured applies (one CUDA graph per factor / input / scratch / output
    // pointer set; the GMRES driver reuses a few such sets)
    struct Graph {
        const void *M, *r, *tmp, *z;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
    void clear_graphs() {
        for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }
    ~Abmc() { clear_graphs(); }
};
template <>
inline McPack<float> &Abmc::pack<float>() { return pk32; }
template <>
inline McPack<double> &Abmc::pack<double>() { return pk64; }

// Plan of the pipelined residual step (cfd_residual_step with host buffers):
// node chunks, their dependencies through the node graph's bandwidth, the
// boundary edges and boundary nodes of each chunk, and the copy streams.
struct StepPipe {
    bool built = false;
    int request = -1;              // cfd_set_step_pipeline: -1 automatic, 0/1 off, k: k chunks
    int K = 0;                     // chunks (0, 1: the step runs unpipelined)
    std::vector<int> lo;           // [K+1] node bounds, multiples of 128
    std::vector<int> dep;          // [K] last chunk holding a neighbour of chunk c
    std::vector<int> bc_lo;        // [K+1] bounds into bc_list
    std::vector<int> bn_lo;        // [K+1] bounds into bnode
    DevBuf<int> bc_list;           // boundary edges ordered by physical node
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaEvent_t ev_start = nullptr, ev_ghost = nullptr;
    std::vector<cudaEvent_t> ev_q, ev_r;  // [K] state chunk arrived, residual chunk done
    int *h_flags = nullptr;        // pinned: fix counters [2], device error word
    void release_events() {
        for (cudaEvent_t e : ev_q) cudaEventDestroy(e);
        for (cudaEvent_t e : ev_r) cudaEventDestroy(e);
        ev_q.clear();
        ev_r.clear();
    }
    ~StepPipe() {
        release_events();
        if (ev_start) cudaEventDestroy(ev_start);
        if (ev_ghost) cudaEventDestroy(ev_ghost);
        if (s_in) cudaStreamDestroy(s_in);
        if (s_out) cudaStreamDestroy(s_out);
        if (h_flags) cudaFreeHost(h_flags);
    }
};

}  // namespace cfd

namespace cfd {
// One request's interior gather residual as a job of a fused launch
// (k_residual_gather_batch): the arguments of k_residual_gather.
struct GatherJob {
    int nnode;
    int64_t ldq;
    const double *Q, *grad, *phi, *xyz;
    const int64_t *sell_ptr;
    const int *sell_nbr;
    const double4 *sell_geo;
    const int *deg;
    Flow f;
    int add_time, checks;
    int *roeflag, *fixcount;
    double *res, *resd, *dtsum;
    const double *lgrad;
    unsigned long long *ext;
    int block_begin;  // first CTA of this job in the fused grid
};
constexpr int kBatchMax = 16;
struct GatherBatch {
    GatherJob job[kBatchMax];
    int njobs;
};
static_assert(sizeof(GatherBatch) <= 32000, "the job table is passed as a kernel parameter");
// key of the kernel instantiation a job needs: (FLUX, second order, frac = 0,
// limited gradients); -1 when the fused launch does not carry that flux
inline int batch_key(int flux, bool second, bool k0, bool lg) {
    if (flux != CFD_FLUX_ROE && flux != CFD_FLUX_HLLC && flux != CFD_FLUX_AUSM) return -1;
    return (flux << 3) | (second ? 4 : 0) | (k0 ? 2 : 0) | (lg ? 1 : 0);
}
int launch_gather_batch(int key, const GatherBatch &b, cudaStream_t s);

// One request's block SpMV y = A x as a job of a fused launch
// (k_bspmv_batch): A in the storage type of the key.
struct SpmvJob {
    int nrow;
    const int *IA, *JA;
    const void *A;
    const double *x;
    double *y;
    int block_begin;  // first CTA of this job in the fused grid
};
struct SpmvBatch {
    SpmvJob job[kBatchMax];
    int njobs;
};
// keys of the fused SpMV launches: kSpmvKey + CFD_PREC_FP64 / FP32 / BF16
constexpr int kSpmvKey = 64;
int launch_spmv_batch(int key, const SpmvBatch &b, cudaStream_t s);
}  // namespace cfd

struct cfd_ctx {
    int device = 0;
    // serving: a fuser of the interior residual and block SpMV launches of
    // several contexts (nullptr: launches of its own); batch_submit takes a
    // GatherJob (key < kSpmvKey) or an SpmvJob and returns once the fused
    // launch is enqueued and this context's stream waits for it
    void *batcher = nullptr;
    int (*batch_submit)(void *batcher, cfd_ctx *c, int key, const void *job) = nullptr;
    int nsm = 148;  // SMs of the device (grids of the gated, usually empty passes)
    cudaStream_t stream = nullptr;
    cfd_params params{};
    cfd::Flow flow{};
    double cfl = 0.0;
    bool has_mesh = false;

    int nnode = 0, nghost = 0, nedge = 0, nbedge = 0;
    int64_t nnzb = 0;
    int64_t ldq = 0;  // leading dimension of Q (>= nnode + nghost)

    // mesh
    cfd::DevBuf<int2> edge_nodes;
    cfd::DevBuf<double4> edge_geo;    // unit normal (x,y,z) + |S|
    cfd::DevBuf<int2> bedge_nodes;
    cfd::DevBuf<double4> bedge_geo;
    cfd::DevBuf<int> bedge_type;
    cfd::DevBuf<double> cvol;
    cfd::DevBuf<double> xyz;          // SoA [3][nnode]
    cfd::DevBuf<double4> edge_sv;     // raw area vector (x,y,z) + 0, for Green-Gauss
    cfd::DevBuf<double4> bedge_sv;
    cfd::DevBuf<int> n2n_ia, n2n_ja;  // physical node graph (no diagonal)
    cfd::DevBuf<int> n2e_ptr, n2e;    // incident interior edges, ~e when the node is node_R
    cfd::DevBuf<int> n2b_ptr, n2b;    // incident boundary edges
    cfd::DevBuf<int> bnode;           // nodes with boundary edges, increasing
    int nbnode = 0;
    // block CRS (Create_CRS_SolverBlockMatrix layout)
    std::vector<int> h_IA, h_JA, h_IAU;
    cfd::DevBuf<int> IA, JA, IAU, tslot;  // tslot[k] = slot of (JA[k], row)
    cfd::DevBuf<int2> eslot;              // per edge: slot(L,R), slot(R,L)
    cfd::Levels lv_fwd, lv_bwd;
    // sliced-ELL incidence of the node-gather residual kernel
    cfd::DevBuf<int64_t> sell_ptr;    // [nslice+1] slot offset of each 32-node slice
    cfd::DevBuf<int> sell_nbr;        // [slots] neighbour id, ~id when the node is node_R
    // limited gradients phi * grad of the fused Green-Gauss + limiter pass
    // (frac = 0 only), read for the neighbours by the first residual pass;
    // valid while grad and phi are the ones they were formed from
    cfd::DevBuf<double> lgrad;        // [15][nnode]
    bool lgrad_pending = false;       // lgrad matches phi_next
    bool lgrad_valid = false;         // lgrad matches phi
    cfd::DevBuf<double4> sell_geo;    // [slots] edge unit normal (L->R) + |S|
    cfd::DevBuf<int> deg;             // [nnode] interior edges per node
    // patch layout of the residual kernel: patches are contiguous ranges of
    // CFD_PATCH_NODES nodes; each patch lists every interior edge touching it
    cfd::DevBuf<int> pe_ptr;          // [npatch+1]
    cfd::DevBuf<int> pe_loc;          // [sum] patch-local (L | R << 16)
    cfd::DevBuf<double4> pe_geo;      // [sum] unit normal + |S|
    cfd::DevBuf<int> ph_ptr, halo;    // per patch: halo node list (global ids, sorted)
    cfd::DevBuf<int> inc_ptr, inc;    // per node: (patch-local edge << 1) | (node is R), increasing
    int npatch = 0, patch_nlocmax = 0;
    bool use_patch = false;
    bool patch_built = false;  // the layout exists (built when residual_kernel = 1 is first asked for)
    // limiter fixes decided by the residual (see cfd_limiter): per node bit 0 =
    // Roe-average pressure fix, bit 1 = reconstructed-pressure correction;
    // fixcount = [nodes failing the Roe check, nodes failing the pressure check]
    cfd::DevBuf<int> roeflag;         // [nnode]
    cfd::DevBuf<int> fixcount;        // [2]
    bool roe_fix_pending = false;
    bool pc_fix_pending = false;
    // limiters formed by cfd_gradient's fused Green-Gauss + limiter pass for
    // the next cfd_limiter; cleared by anything that changes the state or the
    // parameters in between
    cfd::DevBuf<double> phi_next;     // [5][nnode]
    bool phi_next_valid = false;
    bool phi_next_defers_pc = false;

    // state and residual
    cfd::DevBuf<double> Q;      // [5][ldq]
    cfd::DevBuf<double> res;    // [5][nnode] convective
    cfd::DevBuf<double> resd;   // [5][nnode] dissipative
    cfd::DevBuf<double> dt;     // [nnode] sum(area*lambda) then DeltaT
    cfd::DevBuf<double> grad;   // [15][nnode]
    cfd::DevBuf<double> phi;    // [5][nnode]
    cfd::DevBuf<double> ggw;    // least-squares per-node coefficients [nnode][8]
    int lsq_weight = -1;        // weight the coefficients in ggw were built for
    cfd::DevBuf<unsigned long long> ext;  // 8 extrema as ordered bit patterns
    cfd::DevBuf<unsigned long long> ext_scratch;  // extrema of a residual pass a limiter fix may redo
    cfd::DevBuf<int> err;       // device error word
    cfd::DevBuf<double> red;    // reduction partials
    cfd::DevBuf<double> red_out;

    // linear system
    cfd::DevBuf<double> A64;    // [nnzb][25]
    cfd::DevBuf<float> A32;     // [nnzb][25] when FP32 storage requested
    cfd::DevBuf<uint16_t> A16;  // [nnzb][25] BF16 storage
    int a_precision = CFD_PREC_FP64;
    bool a64_valid = false;     // A64 holds the current system
    cfd::DevBuf<double> B, X;   // [nnode][5]
    cfd::DevBuf<double> LUd;    // [nnode][25] diagonal LU for block GS / LU-SGS
    cfd::DevBuf<int> lupiv;     // [nnode][5] row permutation of the LU-SGS pivoted factors
    cfd::DevBuf<double> rowrms; // [nnode]
    // GMRES / ILU workspaces (linsolve.cu)
    cfd::DevBuf<float> M32;     // ILU0 / block-Jacobi factors, FP32
    cfd::DevBuf<double> M64;    // ILU0 / block-Jacobi factors, FP64
    cfd::DevBuf<double> V;      // Krylov basis [(m+1)][5*nnode]
    cfd::DevBuf<double> Z;      // preconditioned vectors (flexible) [m][5*nnode]
    cfd::DevBuf<double> work;   // misc vectors
    cfd::DevBuf<double> dots;   // device dot results
    cfd::DevBuf<int> ilu_diag_inv_done;
    cfd::Abmc mc;               // block multicolour ILU(0) ordering
    cfd::StepPipe pipe;         // pipelined cfd_residual_step
    bool pc_valid = false;      // M64/M32 hold factors of kind pc_kind, precision pc_prec
    int pc_kind = -1, pc_prec = -1;
    int krylov_m = 0;
    bool has_system = false;
    bool has_grad = false;
};

namespace cfd {

#define CFD_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            cfd::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return CFD_ERR_CUDA;                                                         \
        }                                                                                \
    } while (0)

#define CFD_LAUNCH_CHECK()                                                               \
    do {                                                                                 \
        cudaError_t e_ = cudaGetLastError();                                             \
        if (e_ != cudaSuccess) {                                                         \
            cfd::set_error("%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            return CFD_ERR_CUDA;                                                         \
        }                                                                                \
    } while (0)

inline int grid_for(int64_t n, int block) { return (int)((n + block - 1) / block); }

// Raises a kernel's dynamic shared-memory limit to the device's opt-in
// maximum.  The limit is a process-wide attribute of the kernel: setting it to
// one fixed value (rather than each context's own need) keeps contexts that
// launch the kernel from different threads from undoing each other's setting.
template <typename K>
inline cudaError_t allow_max_dynamic_smem(K *kernel, int device, int *max_bytes) {
    int v = 0;
    cudaError_t e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, kernel)) != cudaSuccess) return e;
    v -= (int)fa.sharedSizeBytes;  // the kernel's static shared memory counts against the same limit
    if (max_bytes) *max_bytes = v;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
}

// Deterministic reductions (fixed grid -> fixed order): implemented in core.cu.
int reduce_sum_sq(cfd_ctx *c, const double *x, int64_t n, int64_t stride, int nvec, double *out_host);

// error word bits
enum : int {
    ERR_BC_NEG_PRESSURE = 1,
    ERR_BC_UNCLASSIFIED = 2,
    ERR_NAN = 4,
    ERR_NEG_STATE = 8,
};

int check_device_error(cfd_ctx *c);
// fused Green-Gauss + limiter pass over nodes [lo, hi) (gradient.cu), limiters
// to phi_out, the reconstructed-pressure check left to the residual
int gg_limiter_range(cfd_ctx *c, double *phi_out, int lo, int hi);

}  // namespace cfd
