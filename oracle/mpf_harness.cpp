/* Test harness around the reference MPFLOW3D objects (test infrastructure only).
 *
 * Linked with the reference's own MPFLOW3D, EOS, UTILS and MATH objects (plus
 * oracle/nist_stubs.c for the Fortran REFPROP symbols, which the ideal-gas
 * path never calls) into oracle/_ref/libmpflow3d_ref.so by oracle/Makefile.
 * Like ref_harness.cpp for Euler3D, it fills the reference's process-global
 * mesh arrays directly and calls the hot-path functions one at a time in the
 * order of MPFLOW3D/src/Solver_Steady_Implicit.cpp:60-175, so that each
 * function's output can be compared with the CUDA path.
 *
 * MPFLOW3D keeps its state in the solution variables of VARIABLE_TYPE
 * (VARIABLE_RUP here: rho, u, v, w, p; MPFLOW3D/src/Solver.cpp:356-364) and
 * caches thermodynamic properties per node in CogSolver
 * (MPFLOW3D/src/SolverDB.cpp:122-160), which the driver refreshes after every
 * state change (Solver_Steady_Implicit.cpp:59,118,126); the harness does the
 * same.  Residuals are conservative flux sums in either variable set; the
 * Jacobian and the update X are with respect to the solution variables.
 *
 * One mesh per process: the reference keeps static scratch, so callers run
 * each session in a fresh process.
 */
#include <cstring>
#include <cfloat>
#include "Trim_Utils.h"
#include "Commons.h"
#include "Solver.h"
#include "SolverParameters.h"
#include "Material.h"
#include "Gradient.h"
#include "Jacobian.h"
#include "MC.h"

static Edge3D *alloc_edges(int n) {
    Edge3D *e = (Edge3D *)malloc((size_t)(n > 0 ? n : 1) * sizeof(Edge3D));
    for (int i = 0; i < n; i++) {
        e[i].type = -1;
        e[i].tag = -1;
        e[i].node[0] = e[i].node[1] = -1;
        e[i].areav = 0.0;
    }
    return e;
}

static int g_save_order = 0, g_save_limiter = 0;

extern "C" {

/* Parameter file (MPFLOW3D/src/SolverParameters.cpp:191-1050); ends in
 * Material_Set_Properties (EOS set-up and non-dimensionalisation,
 * MPFLOW3D/src/Material.cpp:125-300). */
void mpf_read_params(const char *param_file) {
    Commons_Init();
    Solver_Parameters_Init();
    Solver_Parameters_Read(param_file);
}

/* Mesh into the reference globals, then Solver_Init,
 * Solver_Set_Initial_Conditions (boundary types, boundary flags, block-CRS
 * pattern; MPFLOW3D/src/Solver.cpp:98,330-492), and the set-up of
 * Solver() / Solver_Steady_Implicit (BC_Init, flux init, Jacobian_Init;
 * Solver.cpp:500-530, Solver_Steady_Implicit.cpp:48).  bedge_type[i] is the
 * BC_TYPE of boundary edge i, routed through bndType[tag-1] as
 * Initialize_Boundary_Condition does (MPFLOW3D/src/BC.cpp:91-95). */
void mpf_setup_mesh(int nnode, int nghost, int nedge, const int *edge_nodes, const double *edge_areav, int nbedge,
                    const int *bedge_nodes, const double *bedge_areav, const int *bedge_type, const double *cvol,
                    const double *coords, const int *n2n_ia, const int *n2n_ja) {
    nNode = nnode;
    nBNode = nghost;
    nEdge = nedge;
    nBEdge = nbedge;
    intEdge = alloc_edges(nedge);
    bndEdge = alloc_edges(nbedge);
    for (int i = 0; i < nedge; i++) {
        intEdge[i].node[0] = edge_nodes[2 * i];
        intEdge[i].node[1] = edge_nodes[2 * i + 1];
        for (int k = 0; k < 3; k++) intEdge[i].areav.vec[k] = edge_areav[3 * i + k];
    }
    nBC = 17;
    bndType = new int[nBC];
    for (int k = 0; k < nBC; k++) bndType[k] = k;
    for (int i = 0; i < nbedge; i++) {
        bndEdge[i].node[0] = bedge_nodes[2 * i];
        bndEdge[i].node[1] = bedge_nodes[2 * i + 1];
        bndEdge[i].tag = bedge_type[i] + 1;
        for (int k = 0; k < 3; k++) bndEdge[i].areav.vec[k] = bedge_areav[3 * i + k];
    }
    cVolume = (double *)malloc((size_t)nnode * sizeof(double));
    memcpy(cVolume, cvol, (size_t)nnode * sizeof(double));
    coordXYZ = (double *)malloc((size_t)3 * nnode * sizeof(double));
    memcpy(coordXYZ, coords, (size_t)3 * nnode * sizeof(double));
    crs_IA_Node2Node = (int *)malloc((size_t)(nnode + 1) * sizeof(int));
    memcpy(crs_IA_Node2Node, n2n_ia, (size_t)(nnode + 1) * sizeof(int));
    crs_JA_Node2Node = (int *)malloc((size_t)n2n_ia[nnode] * sizeof(int));
    memcpy(crs_JA_Node2Node, n2n_ja, (size_t)n2n_ia[nnode] * sizeof(int));

    Solver_Init();
    Solver_Set_Initial_Conditions();
    BC_Init();
    switch (FluxScheme) {
        case FLUX_SCHEME_ROE: Roe_Init(); break;
        case FLUX_SCHEME_HLLC: HLLC_Init(); break;
        default: break;
    }
    if (SolverScheme == SOLVER_SCHEME_IMPLICIT) Jacobian_Init();
    g_save_order = SolverOrder;
    g_save_limiter = LimiterMethod;
}

/* Q: SoA [5][nNode+nBNode] in the solution variables (RUP). */
void mpf_set_state(const double *Q) {
    int n = nNode + nBNode;
    double *dst[5] = {Q1, Q2, Q3, Q4, Q5};
    for (int k = 0; k < 5; k++) memcpy(dst[k], Q + (size_t)k * n, (size_t)n * sizeof(double));
    CogSolver.Compute_Bulk_Extended_Properties(0, nNode + nBNode);  // Solver_Steady_Implicit.cpp:59
}

void mpf_get_state(double *Q) {
    int n = nNode + nBNode;
    double *src[5] = {Q1, Q2, Q3, Q4, Q5};
    for (int k = 0; k < 5; k++) memcpy(Q + (size_t)k * n, src[k], (size_t)n * sizeof(double));
}

/* Per-iteration resets, far field with Mach ramp, first-order / limiter
 * switches and the physical nodes' properties
 * (Solver_Steady_Implicit.cpp:62-118). */
void mpf_begin_iteration(int iter) {
    for (int i = 0; i < nNode; i++) {
        Res1_Conv[i] = Res2_Conv[i] = Res3_Conv[i] = Res4_Conv[i] = Res5_Conv[i] = 0.0;
        Res1_Diss[i] = Res2_Diss[i] = Res3_Diss[i] = Res4_Diss[i] = Res5_Diss[i] = 0.0;
        DeltaT[i] = 0.0;
    }
    MinEigenLamda1 = DBL_MAX; MaxEigenLamda1 = DBL_MIN;
    MinEigenLamda4 = DBL_MAX; MaxEigenLamda4 = DBL_MIN;
    MinEigenLamda5 = DBL_MAX; MaxEigenLamda5 = DBL_MIN;
    MinDeltaT = DBL_MAX; MaxDeltaT = DBL_MIN;
    if (PrecondMethod != PRECOND_METHOD_NONE) {
        for (int i = 0; i < nNode; i++) PrecondSigma[i] = 0.0;
        MinPrecondSigma = DBL_MAX;
        MaxPrecondSigma = DBL_MIN;
    }
    Material_Set_InfinityCondition(iter);
    SolverOrder = g_save_order;
    if (FirstOrderNIteration > iter) SolverOrder = SOLVER_ORDER_FIRST;
    LimiterMethod = LIMITER_METHOD_NONE;
    if (LimiterStartSolverIteration < LimiterEndSolverIteration) {
        if ((LimiterStartSolverIteration <= iter + 1) && (LimiterEndSolverIteration > iter))
            LimiterMethod = g_save_limiter;
    }
    CogSolver.Compute_Bulk_Extended_Properties(0, nNode);
}

/* Second-order gradient (+ limiter), Solver_Steady_Implicit.cpp:121-126. */
void mpf_gradient(void) {
    if (SolverOrder == SOLVER_ORDER_SECOND) {
        Compute_Least_Square_Gradient(0);
        CogSolver.Smooth_Solution_Gradient();
        if (LimiterMethod != LIMITER_METHOD_NONE) Compute_Limiter();
    }
}

/* Characteristic BCs, then the ghosts' properties (:129-132). */
void mpf_apply_bc(int iter) {
    Apply_Boundary_Condition(iter);
    CogSolver.Compute_Bulk_Extended_Properties(nNode, nNode + nBNode);
}
void mpf_residual(int add_time) { Compute_Residual(add_time); }
void mpf_deltat(int iter) { Compute_DeltaT(iter); }
double mpf_rms(int iter) { return RMS_Writer(iter); }
void mpf_jacobian(int add_time, int iter) { Compute_Jacobian(add_time, iter); }
double mpf_lusgs(int niter) { return MC_Iterative_Block_LUSGS_CRS(niter, SolverBlockMatrix); }
double mpf_block_gs(int niter, int direction) {
    return MC_Iterative_Block_LU_Jacobi_CRS(niter, direction, SolverBlockMatrix);
}

/* Q += relax * X, Material_Limit_Solution and the preconditioning-variable
 * normalisation (Solver_Steady_Implicit.cpp:162-184). */
void mpf_update(double relax) {
    for (int i = 0; i < nNode; i++) {
        Q1[i] += relax * SolverBlockMatrix.X[i][0];
        Q2[i] += relax * SolverBlockMatrix.X[i][1];
        Q3[i] += relax * SolverBlockMatrix.X[i][2];
        Q4[i] += relax * SolverBlockMatrix.X[i][3];
        Q5[i] += relax * SolverBlockMatrix.X[i][4];
    }
    Material_Limit_Solution();
    if (PrecondMethod != PRECOND_METHOD_NONE) {
        for (int i = 0; i < nNode; i++) PrecondSigma[i] /= (crs_IA_Node2Node[i + 1] - crs_IA_Node2Node[i]);
    }
}

/* Residual arrays and extrema from the caller, then one RMS_Writer line
 * (MPFLOW3D/src/RMSIO.cpp:98-154 computes the RMS from Res*_Conv + Res*_Diss);
 * ext8 = {min/max lambda 1, 4, 5, min/max dt}, sigma2 = min/max sigma. */
double mpf_rms_write(int iteration, const double *conv, const double *diss, const double *ext8,
                     const double *sigma2) {
    double *c[5] = {Res1_Conv, Res2_Conv, Res3_Conv, Res4_Conv, Res5_Conv};
    double *d[5] = {Res1_Diss, Res2_Diss, Res3_Diss, Res4_Diss, Res5_Diss};
    for (int k = 0; k < 5; k++) {
        memcpy(c[k], conv + (size_t)k * nNode, (size_t)nNode * sizeof(double));
        memcpy(d[k], diss + (size_t)k * nNode, (size_t)nNode * sizeof(double));
    }
    MinEigenLamda1 = ext8[0]; MaxEigenLamda1 = ext8[1];
    MinEigenLamda4 = ext8[2]; MaxEigenLamda4 = ext8[3];
    MinEigenLamda5 = ext8[4]; MaxEigenLamda5 = ext8[5];
    MinDeltaT = ext8[6]; MaxDeltaT = ext8[7];
    MinPrecondSigma = sigma2[0]; MaxPrecondSigma = sigma2[1];
    return RMS_Writer(iteration);
}
void mpf_rms_close(void) { RMS_Writer_Finalize(); }

/* conv/diss: SoA [5][nNode] (Res*_Conv, Res*_Diss). */
void mpf_get_residual(double *conv, double *diss) {
    double *c[5] = {Res1_Conv, Res2_Conv, Res3_Conv, Res4_Conv, Res5_Conv};
    double *d[5] = {Res1_Diss, Res2_Diss, Res3_Diss, Res4_Diss, Res5_Diss};
    for (int k = 0; k < 5; k++) {
        memcpy(conv + (size_t)k * nNode, c[k], (size_t)nNode * sizeof(double));
        memcpy(diss + (size_t)k * nNode, d[k], (size_t)nNode * sizeof(double));
    }
}
void mpf_get_deltat(double *dt) { memcpy(dt, DeltaT, (size_t)nNode * sizeof(double)); }

/* {min1,max1,min4,max4,min5,max5,minDt,maxDt} */
void mpf_get_extrema(double *out) {
    out[0] = MinEigenLamda1; out[1] = MaxEigenLamda1;
    out[2] = MinEigenLamda4; out[3] = MaxEigenLamda4;
    out[4] = MinEigenLamda5; out[5] = MaxEigenLamda5;
    out[6] = MinDeltaT; out[7] = MaxDeltaT;
}

/* {rho,u,v,w,et,p,c,mach,T} of the far field (non-dimensional). */
void mpf_get_farfield(double *out) {
    out[0] = Inf_Rho; out[1] = Inf_U; out[2] = Inf_V; out[3] = Inf_W;
    out[4] = Inf_Et; out[5] = Inf_Pressure; out[6] = Inf_SpeedSound; out[7] = Inf_Mach;
    out[8] = Inf_Temperature;
}

int mpf_nnz_blocks(void) { return SolverBlockMatrix.DIM; }
void mpf_get_crs(int *IA, int *JA, int *IAU) {
    memcpy(IA, SolverBlockMatrix.IA, (size_t)(nNode + 1) * sizeof(int));
    memcpy(JA, SolverBlockMatrix.JA, (size_t)SolverBlockMatrix.DIM * sizeof(int));
    memcpy(IAU, SolverBlockMatrix.IAU, (size_t)nNode * sizeof(int));
}
/* A: [DIM][5][5] contiguous; B, X: [nNode][5]. */
void mpf_get_matrix(double *A, double *B, double *X) {
    for (int b = 0; b < SolverBlockMatrix.DIM; b++)
        for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++) A[(size_t)b * 25 + i * 5 + j] = SolverBlockMatrix.A[b][i][j];
    for (int r = 0; r < nNode; r++)
        for (int i = 0; i < 5; i++) {
            B[(size_t)r * 5 + i] = SolverBlockMatrix.B[r][i];
            X[(size_t)r * 5 + i] = SolverBlockMatrix.X[r][i];
        }
}
void mpf_set_matrix(const double *A, const double *B) {
    for (int b = 0; b < SolverBlockMatrix.DIM; b++)
        for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++) SolverBlockMatrix.A[b][i][j] = A[(size_t)b * 25 + i * 5 + j];
    for (int r = 0; r < nNode; r++)
        for (int i = 0; i < 5; i++) SolverBlockMatrix.B[r][i] = B[(size_t)r * 5 + i];
}

/* Transformation matrix d(to)/d(from) at one node, from the node's cached
 * properties (Material_Get_Transformation_Matrix, MPFLOW3D/src/Material.cpp);
 * m: [5][5] row-major.  Variable types as VARIABLE_* of SolverParameters.h. */
void mpf_transformation_matrix(int node, int from, int to, double *m) {
    double **M = new double *[5];
    for (int i = 0; i < 5; i++) M[i] = new double[5];
    Material_Get_Transformation_Matrix(node, from, to, M);
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) m[i * 5 + j] = M[i][j];
    for (int i = 0; i < 5; i++) delete[] M[i];
    delete[] M;
}

}  // extern "C"
