// Drop-in replacement of the Euler3D hot-path functions by the CUDA library.
//
// Linked into the reference's own Euler3D executable in place of its
// implementations, this file defines the functions the implicit driver calls
// (Euler3D/src/Solver_Steady_Implicit.cpp:96-159) with their exact C++
// signatures, operating on the driver's process-global arrays:
//
//   void   Apply_Boundary_Condition(int)                (Euler3D/src/BC.cpp:1847)
//   void   Compute_Least_Square_Gradient(int)           (Euler3D/src/Gradient.cpp:232)
//   void   Compute_Limiter(void)                        (Euler3D/src/Limiters.cpp:20)
//   void   Compute_Residual(int)                        (Euler3D/src/Residual.cpp:18)
//   void   Compute_DeltaT(int)                          (Euler3D/src/Time_Step.cpp:23)
//   void   Compute_Jacobian(int, int)                   (Euler3D/src/Jacobian.cpp:18)
//   double MC_Iterative_Block_LU_Jacobi_CRS(int, int, MC_CRS)  (MATH/src/MC_Iterative_Jacobi.c:346)
//   double MC_Iterative_Block_LUSGS_CRS(int, MC_CRS)           (MATH/src/MC_Iterative_Jacobi.c:539)
//
// The mesh, state and block system live on the GPU; the host globals the
// driver reads (Q after the BC update, Res*/Res*_Diss for the RMS, DeltaT and
// the extrema for Residual.res, X after the linear solve) are copied back.
// The driver's own host update Q += relax*X is picked up by re-uploading Q at
// the first call of each iteration.  Environment:
//   CFD_B200_DEVICE=<n>       GPU to use (default 0)
//   CFD_B200_LINEAR=gmres     solve with GMRES(30)+ILU(0) instead of block
//                             Gauss-Seidel (the iteration argument is then the
//                             Krylov budget)
// The reference's globals are declared here with their own names and types;
// the struct layouts below are the reference's (Commons.h:97-102, MC.h:16-28).
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/cfd_b200.h"

// ---- reference types (layout-compatible declarations)
struct Vector3D_layout {
    double vec[3];
};
struct Edge3D {
    int type;
    int tag;
    int node[2];
    Vector3D_layout areav;
};
extern "C" {
typedef struct _MC_CRS {
    int Block_nRow, Block_nCol, DIM, nROW, nCOL;
    int *IA, *JA, *IAU;
    double ***A;
    double **B;
    double **X;
} MC_CRS;
}

// ---- reference globals (defined by the reference objects the driver links)
extern int nNode, nEdge, nBEdge, nBNode;
extern Edge3D *intEdge, *bndEdge;
extern double *cVolume, *coordXYZ;
extern int *crs_IA_Node2Node, *crs_JA_Node2Node;
extern double *Q1, *Q2, *Q3, *Q4, *Q5;
extern double *Res1, *Res2, *Res3, *Res4, *Res5;
extern double *Res1_Diss, *Res2_Diss, *Res3_Diss, *Res4_Diss, *Res5_Diss;
extern double *DeltaT, MinDeltaT, MaxDeltaT;
extern double MinEigenLamda1, MaxEigenLamda1, MinEigenLamda4, MaxEigenLamda4, MinEigenLamda5, MaxEigenLamda5;
extern double *Q1x, *Q1y, *Q1z, *Q2x, *Q2y, *Q2z, *Q3x, *Q3y, *Q3z, *Q4x, *Q4y, *Q4z, *Q5x, *Q5y, *Q5z;
extern double *Limiter_Phi1, *Limiter_Phi2, *Limiter_Phi3, *Limiter_Phi4, *Limiter_Phi5;
extern int FluxScheme, SolverOrder, LimiterMethod, LimiterOrder, LimiterSmooth, EntropyFix;
extern int TimeIntegrationType, CFL_Ramp, Mach_Ramp, ZPGIteration, JacobianUpdate, VariableType, PrecondMethod;
extern int JacobianMethod;
extern double CFL_MIN, CFL_MAX, Mach_MIN, Mach_MAX, Gamma, Ref_Alpha, Ref_Beta, Venkat_KThreshold;
extern double Inf_Rho, Inf_U, Inf_V, Inf_W, Inf_Et, Inf_Pressure, Inf_SpeedSound, Inf_Mach;
extern int SolverMethod;           // SOLVER_METHOD_STEADY (0) / SOLVER_METHOD_UNSTEADY (1)
extern MC_CRS SolverBlockMatrix;   // Solver.cpp:612-704

namespace {

struct Shim {
    cfd_ctx *ctx = nullptr;
    int nnode = 0, nghost = 0;
    std::vector<double> q, conv, diss, buf;
    bool gmres = false;
};
Shim g;

void die(const char *where, int code) {
    std::fprintf(stderr, "cfd_b200 shim: %s failed (%d): %s\n", where, code, cfd_last_error());
    std::exit(EXIT_FAILURE);  // the reference's error() convention (UTILS/src/Trim_Utils.c:31-52)
}
#define CHECK(call)                          \
    do {                                     \
        int rc_ = (call);                    \
        if (rc_ != CFD_OK) die(#call, rc_);  \
    } while (0)

void sync_params() {
    cfd_params p;
    cfd_params_default(&p);
    // PRECOND_METHOD_NONE (-1) or PRECOND_METHOD_ROE_LMFIX (0) with the Roe flux; FLUX_SCHEME_ROE,
    // _HLLC, _AUSM or _VANLEER (SolverParameters.h:109-117; the other families are empty stubs there)
    if (VariableType != 0 || !(PrecondMethod == -1 || (PrecondMethod == 0 && FluxScheme == CFD_FLUX_ROE)) ||
        FluxScheme < 0 || FluxScheme > 3) {
        std::fprintf(stderr, "cfd_b200 shim: only VARIABLE_CONSERVATIVE with the Roe (optionally with its low-Mach "
                             "fix), HLLC, AUSM or Van Leer flux is supported\n");
        std::exit(EXIT_FAILURE);
    }
    p.flux_scheme = PrecondMethod == 0 ? CFD_FLUX_ROE_LMFIX : (FluxScheme == 3 ? CFD_FLUX_VANLEER : FluxScheme);
    p.order = SolverOrder;
    p.limiter = LimiterMethod;
    p.limiter_order = LimiterOrder;
    p.limiter_smooth = LimiterSmooth;
    p.gradient = CFD_GRAD_LSQ;
    p.entropy_fix = EntropyFix;
    p.global_time = TimeIntegrationType == 1;
    p.cfl_ramp = CFL_Ramp;
    p.mach_ramp = Mach_Ramp;
    p.zpg_iteration = ZPGIteration;
    p.gamma = Gamma;
    p.mach = Mach_MAX;
    p.mach_min = Mach_MIN;
    p.alpha_deg = Ref_Alpha * 180.0 / M_PI;  // Material_Set_Properties stores radians
    p.beta_deg = Ref_Beta * 180.0 / M_PI;
    p.cfl_min = CFL_MIN;
    p.cfl_max = CFL_MAX;
    p.venkat_k = Venkat_KThreshold;
    CHECK(cfd_set_params(g.ctx, &p));
}

void ensure_init() {
    if (g.ctx) return;
    const char *dev = std::getenv("CFD_B200_DEVICE");
    const char *lin = std::getenv("CFD_B200_LINEAR");
    g.gmres = lin && std::strcmp(lin, "gmres") == 0;
    CHECK(cfd_create(dev ? std::atoi(dev) : 0, &g.ctx));
    sync_params();
    g.nnode = nNode;
    g.nghost = nBNode;
    std::vector<int> en(2 * (size_t)nEdge), bn(2 * (size_t)nBEdge), bt(nBEdge);
    std::vector<double> ea(3 * (size_t)nEdge), ba(3 * (size_t)nBEdge);
    for (int e = 0; e < nEdge; e++) {
        en[2 * e] = intEdge[e].node[0];
        en[2 * e + 1] = intEdge[e].node[1];
        for (int d = 0; d < 3; d++) ea[3 * (size_t)e + d] = intEdge[e].areav.vec[d];
    }
    for (int b = 0; b < nBEdge; b++) {
        bn[2 * b] = bndEdge[b].node[0];
        bn[2 * b + 1] = bndEdge[b].node[1];
        bt[b] = bndEdge[b].type;
        for (int d = 0; d < 3; d++) ba[3 * (size_t)b + d] = bndEdge[b].areav.vec[d];
    }
    CHECK(cfd_set_mesh(g.ctx, nNode, nBNode, nEdge, en.data(), ea.data(), nBEdge, bn.data(), ba.data(), bt.data(),
                       cVolume, coordXYZ, crs_IA_Node2Node, crs_JA_Node2Node));
    const size_t n = (size_t)nNode + nBNode;
    g.q.resize(5 * n);
    g.conv.resize(5 * (size_t)nNode);
    g.diss.resize(5 * (size_t)nNode);
}

// host Q1..Q5 -> device (SoA, nNode+nBNode each)
void upload_state() {
    const size_t n = (size_t)g.nnode + g.nghost;
    double *src[5] = {Q1, Q2, Q3, Q4, Q5};
    for (int k = 0; k < 5; k++) std::memcpy(&g.q[k * n], src[k], n * sizeof(double));
    CHECK(cfd_set_state(g.ctx, g.q.data()));
}

void download_state() {
    const size_t n = (size_t)g.nnode + g.nghost;
    CHECK(cfd_get_state(g.ctx, g.q.data()));
    double *dst[5] = {Q1, Q2, Q3, Q4, Q5};
    for (int k = 0; k < 5; k++) std::memcpy(dst[k], &g.q[k * n], n * sizeof(double));
}

// far field the driver computed for this iteration (ComputeFarFieldCondition)
void push_farfield() {
    const double inf[8] = {Inf_Rho, Inf_U, Inf_V, Inf_W, Inf_Et, Inf_Pressure, Inf_SpeedSound, Inf_Mach};
    CHECK(cfd_set_farfield(g.ctx, inf));
}

}  // namespace

void Compute_Least_Square_Gradient(int WeightType) {
    ensure_init();
    (void)WeightType;  // unweighted, as the driver requests (Solver_Steady_Implicit.cpp:97)
    upload_state();
    CHECK(cfd_gradient(g.ctx));
    if (Q1x) {
        g.buf.resize(15 * (size_t)g.nnode);
        CHECK(cfd_get_gradients(g.ctx, g.buf.data()));
        double *dst[15] = {Q1x, Q1y, Q1z, Q2x, Q2y, Q2z, Q3x, Q3y, Q3z, Q4x, Q4y, Q4z, Q5x, Q5y, Q5z};
        for (int k = 0; k < 15; k++) std::memcpy(dst[k], &g.buf[k * (size_t)g.nnode], g.nnode * sizeof(double));
    }
}

void Compute_Limiter(void) {
    ensure_init();
    CHECK(cfd_limiter(g.ctx));
}

void Apply_Boundary_Condition(int Iteration) {
    ensure_init();
    upload_state();
    push_farfield();
    CHECK(cfd_apply_bc(g.ctx, Iteration));
    download_state();  // the driver's later host code reads the ghost states
}

void Compute_Residual(int AddTime) {
    ensure_init();
    push_farfield();
    CHECK(cfd_begin_iteration(g.ctx, 0));  // resets device accumulators / extrema
    push_farfield();
    CHECK(cfd_residual(g.ctx, AddTime));
    CHECK(cfd_get_residual(g.ctx, g.conv.data(), g.diss.data()));
    const size_t n = g.nnode;
    double *c[5] = {Res1, Res2, Res3, Res4, Res5};
    double *d[5] = {Res1_Diss, Res2_Diss, Res3_Diss, Res4_Diss, Res5_Diss};
    for (int k = 0; k < 5; k++) {
        std::memcpy(c[k], &g.conv[k * n], n * sizeof(double));
        std::memcpy(d[k], &g.diss[k * n], n * sizeof(double));
    }
    if (AddTime) {
        CHECK(cfd_get_deltat(g.ctx, DeltaT));
        double ext[8];
        CHECK(cfd_get_extrema(g.ctx, ext));
        MinEigenLamda1 = ext[0]; MaxEigenLamda1 = ext[1];
        MinEigenLamda4 = ext[2]; MaxEigenLamda4 = ext[3];
        MinEigenLamda5 = ext[4]; MaxEigenLamda5 = ext[5];
    }
}

void Compute_DeltaT(int Iteration) {
    ensure_init();
    CHECK(cfd_deltat(g.ctx, Iteration));
    CHECK(cfd_get_deltat(g.ctx, DeltaT));
    double ext[8];
    CHECK(cfd_get_extrema(g.ctx, ext));
    MinDeltaT = ext[6];
    MaxDeltaT = ext[7];
}

namespace {

// The unsteady drivers add the physical-time terms to the host block system
// between Compute_Jacobian and the linear solve (Solver_Unsteady_Implicit.cpp:
// 100-121): with them the system is mirrored to SolverBlockMatrix after
// assembly and taken back from it before the solve.
bool mirror_system() { return SolverMethod == 1; }

void download_system() {
    const size_t nnzb = (size_t)SolverBlockMatrix.IA[g.nnode];
    g.buf.resize(25 * nnzb + 5 * (size_t)g.nnode);
    double *A = g.buf.data(), *B = A + 25 * nnzb;
    CHECK(cfd_get_system(g.ctx, A, B, nullptr));
    for (size_t k = 0; k < nnzb; k++)
        for (int r = 0; r < 5; r++)
            for (int c = 0; c < 5; c++) SolverBlockMatrix.A[k][r][c] = A[25 * k + 5 * r + c];
    for (int i = 0; i < g.nnode; i++)
        for (int v = 0; v < 5; v++) SolverBlockMatrix.B[i][v] = B[5 * (size_t)i + v];
}

void upload_system() {
    const size_t nnzb = (size_t)SolverBlockMatrix.IA[g.nnode];
    g.buf.resize(25 * nnzb + 5 * (size_t)g.nnode);
    double *A = g.buf.data(), *B = A + 25 * nnzb;
    for (size_t k = 0; k < nnzb; k++)
        for (int r = 0; r < 5; r++)
            for (int c = 0; c < 5; c++) A[25 * k + 5 * r + c] = SolverBlockMatrix.A[k][r][c];
    for (int i = 0; i < g.nnode; i++)
        for (int v = 0; v < 5; v++) B[5 * (size_t)i + v] = SolverBlockMatrix.B[i][v];
    CHECK(cfd_set_system(g.ctx, A, B));
}

}  // namespace

void Compute_Jacobian(int AddTime, int Iteration) {
    ensure_init();
    if (Iteration % JacobianUpdate != 0) return;  // Jacobian.cpp:26-28
    // Euler3D's right-hand side is B = -Res (its Res_Diss is never added, FluxTest.cpp:8143-8150)
    const bool mirror = mirror_system();
    if (JacobianMethod >= CFD_JAC_CENTRAL && JacobianMethod <= CFD_JAC_ALTERNATE)  // Roe_Jacobian.cpp:780-793
        CHECK(cfd_jacobian_fd(g.ctx, AddTime, 0, JacobianMethod, Iteration));
    else
        CHECK(cfd_jacobian(g.ctx, AddTime, 0, (g.gmres && !mirror) ? CFD_PREC_FP32 : CFD_PREC_FP64));
    if (mirror) download_system();
}

extern "C" double MC_Iterative_Block_LU_Jacobi_CRS(int Iteration, int Direction, MC_CRS Object) {
    ensure_init();
    if (mirror_system()) upload_system();
    double rms = 0.0;
    if (g.gmres) {
        cfd_gmres_opts o;
        cfd_gmres_default(&o);
        o.max_iters = Iteration > 0 ? Iteration : o.max_iters;
        o.precision = mirror_system() ? CFD_PREC_FP64 : CFD_PREC_FP32;
        o.refine = 4;
        cfd_gmres_stats st;
        const int rc = cfd_gmres(g.ctx, &o, &st);
        if (rc != CFD_OK && rc != CFD_ERR_NOT_CONVERGED) return NAN;
        rms = st.rel_residual;
    } else {
        const int rc = cfd_block_gs(g.ctx, Iteration, Direction, &rms);
        if (rc == CFD_ERR_NUMERIC) return NAN;
        if (rc != CFD_OK) die("cfd_block_gs", rc);
    }
    g.buf.resize(5 * (size_t)g.nnode);
    CHECK(cfd_get_system(g.ctx, nullptr, nullptr, g.buf.data()));
    for (int i = 0; i < Object.nROW; i++)
        for (int k = 0; k < 5; k++) Object.X[i][k] = g.buf[5 * (size_t)i + k];
    return rms;
}

extern "C" double MC_Iterative_Block_LUSGS_CRS(int Iteration, MC_CRS Object) {
    ensure_init();
    if (mirror_system()) upload_system();
    double rms = 0.0;
    const int rc = cfd_block_lusgs(g.ctx, Iteration, &rms);
    if (rc == CFD_ERR_NUMERIC) return NAN;
    if (rc != CFD_OK) die("cfd_block_lusgs", rc);
    g.buf.resize(5 * (size_t)g.nnode);
    CHECK(cfd_get_system(g.ctx, nullptr, nullptr, g.buf.data()));
    for (int i = 0; i < Object.nROW; i++)
        for (int k = 0; k < 5; k++) Object.X[i][k] = g.buf[5 * (size_t)i + k];
    return rms;
}
