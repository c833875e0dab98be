/* Test harness around the reference Euler3D objects (test infrastructure only).
 *
 * Linked with the reference's own UTILS/MATH/Euler3D objects into
 * oracle/_ref/libeuler3d_ref.so by oracle/Makefile.  It fills the reference's
 * process-global mesh/state arrays directly (bypassing the reference's O(N^2)
 * setup for large meshes) and calls the reference's hot-path functions one at a
 * time, exactly as Euler3D/src/Solver_Steady_Implicit.cpp:45-159 does, so that
 * every function's output can be compared against the CUDA path.
 *
 * One mesh per process: the reference keeps static state (Roe scratch,
 * least-squares coefficients), so callers run each session in a fresh process.
 */
#include <cstring>
#include <cfloat>
#include "Trim_Utils.h"
#include "Commons.h"
#include "Solver.h"
#include "SolverParameters.h"
#include "MeshIO.h"
#include "Material.h"
#include "Gradient.h"
#include "MC.h"

void Roe_Init_New(void);
void HLLC_Init(void);
void VanLeer_Init(void);

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

extern "C" {

int ref_sizeof_edge3d(void) { return (int)sizeof(Edge3D); }

/* Read the reference parameter file (Euler3D/src/SolverParameters.cpp:184). */
void ref_read_params(const char *param_file) {
    Commons_Init();
    Solver_Parameters_Init();
    Solver_Parameters_Read(param_file);
}

/* Install a median-dual mesh into the reference globals and run the
 * reference's own Solver_Init / Solver_Set_Initial_Conditions
 * (Euler3D/src/Solver.cpp:98, :339) plus the flux-scheme init
 * (Euler3D/src/Solver.cpp:506-531).
 * bedge_type[i] is the BC_TYPE of boundary edge i (SolverParameters.h:40). */
void ref_setup_mesh(int nnode, int nghost, int nedge, const int *edge_nodes,
                    const double *edge_areav, int nbedge, const int *bedge_nodes,
                    const double *bedge_areav, const int *bedge_type,
                    const double *cvol, const double *coords,
                    const int *n2n_ia, const int *n2n_ja) {
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
    /* BC types are routed through the reference's tag->type table:
     * bndEdge.type = bndType[tag-1] (Euler3D/src/BC.cpp:23-27). */
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
    switch (FluxScheme) {
        case FLUX_SCHEME_ROE: Roe_Init_New(); break;
        case FLUX_SCHEME_HLLC: HLLC_Init(); break;
        case FLUX_SCHEME_VANLEER: VanLeer_Init(); break;
        default: break;
    }
}

/* Q is SoA [5][nNode+nBNode] (Euler3D/include/Solver.h:27-31). */
void ref_set_state(const double *Q) {
    int n = nNode + nBNode;
    double *dst[5] = {Q1, Q2, Q3, Q4, Q5};
    for (int k = 0; k < 5; k++) memcpy(dst[k], Q + (size_t)k * n, (size_t)n * sizeof(double));
}

void ref_get_state(double *Q) {
    int n = nNode + nBNode;
    double *src[5] = {Q1, Q2, Q3, Q4, Q5};
    for (int k = 0; k < 5; k++) memcpy(Q + (size_t)k * n, src[k], (size_t)n * sizeof(double));
}

/* Per-iteration resets of Euler3D/src/Solver_Steady_Implicit.cpp:45-75,81. */
void ref_begin_iteration(int iter) {
    for (int i = 0; i < nNode; i++) {
        Res1[i] = Res2[i] = Res3[i] = Res4[i] = Res5[i] = 0.0;
        Res1_Diss[i] = Res2_Diss[i] = Res3_Diss[i] = Res4_Diss[i] = Res5_Diss[i] = 0.0;
        DeltaT[i] = 0.0;
    }
    MinEigenLamda1 = DBL_MAX; MaxEigenLamda1 = DBL_MIN;
    MinEigenLamda4 = DBL_MAX; MaxEigenLamda4 = DBL_MIN;
    MinEigenLamda5 = DBL_MAX; MaxEigenLamda5 = DBL_MIN;
    MinDeltaT = DBL_MAX; MaxDeltaT = DBL_MIN;
    ComputeFarFieldCondition(iter);
}

void ref_gradient(int weight) { Compute_Least_Square_Gradient(weight); }
void ref_limiter(void) { Compute_Limiter(); }
void ref_apply_bc(int iter) { Apply_Boundary_Condition(iter); }
void ref_residual(int add_time) { Compute_Residual(add_time); }
void ref_deltat(int iter) { Compute_DeltaT(iter); }
void ref_jacobian(int add_time, int iter) { Compute_Jacobian(add_time, iter); }
double ref_block_gs(int niter, int direction) {
    return MC_Iterative_Block_LU_Jacobi_CRS(niter, direction, SolverBlockMatrix);
}
double ref_lusgs(int niter) { return MC_Iterative_Block_LUSGS_CRS(niter, SolverBlockMatrix); }

/* Q += relax * X  (Euler3D/src/Solver_Steady_Implicit.cpp:153-159). */
void ref_update(double relax) {
    for (int i = 0; i < nNode; i++) {
        Q1[i] += relax * SolverBlockMatrix.X[i][0];
        Q2[i] += relax * SolverBlockMatrix.X[i][1];
        Q3[i] += relax * SolverBlockMatrix.X[i][2];
        Q4[i] += relax * SolverBlockMatrix.X[i][3];
        Q5[i] += relax * SolverBlockMatrix.X[i][4];
    }
}

/* B = -(Res + Res_Diss), the right-hand side of MPFLOW3D's implicit driver
 * (MPFLOW3D/src/Roe_Jacobian.cpp:237-241), put into Euler3D's block system
 * after its Compute_Jacobian (which sets B = -Res, Euler3D/src/Roe_Jacobian.cpp),
 * so that the reference's own implicit loop converges to Res + Res_Diss = 0.
 * Returns the RMS over the five equations of Res + Res_Diss (the quantity
 * the loop drives to zero), sqrt(sum / (5 nNode)). */
double ref_rhs_include_diss(void) {
    double *c[5] = {Res1, Res2, Res3, Res4, Res5};
    double *d[5] = {Res1_Diss, Res2_Diss, Res3_Diss, Res4_Diss, Res5_Diss};
    double s = 0.0;
    for (int i = 0; i < nNode; i++)
        for (int k = 0; k < 5; k++) {
            const double r = c[k][i] + d[k][i];
            SolverBlockMatrix.B[i][k] = -r;
            s += r * r;
        }
    return sqrt(s / (5.0 * nNode));
}

/* One line of the reference's residual file (RMS_Writer, Euler3D/src/RMSIO.cpp:85-97)
 * with given values: rms6 = per-equation RMS and RMS_Res; ext8 = {min/max lambda 1,
 * 4, 5, min/max dt}; sigma2 = min/max preconditioner sigma.  The file is the
 * Residual.res that Solver_Init opened in the working directory. */
void ref_rms_write(int iteration, const double *rms6, const double *ext8, const double *sigma2) {
    double rms[5] = {rms6[0], rms6[1], rms6[2], rms6[3], rms6[4]};
    RMS_Res = rms6[5];
    MinEigenLamda1 = ext8[0]; MaxEigenLamda1 = ext8[1];
    MinEigenLamda4 = ext8[2]; MaxEigenLamda4 = ext8[3];
    MinEigenLamda5 = ext8[4]; MaxEigenLamda5 = ext8[5];
    MinDeltaT = ext8[6]; MaxDeltaT = ext8[7];
    MinPrecondSigma = sigma2[0]; MaxPrecondSigma = sigma2[1];
    RMS_Writer(iteration, rms);
}
void ref_rms_close(void) { RMS_Writer_Finalize(); }

/* conv/diss are SoA [5][nNode]. */
void ref_get_residual(double *conv, double *diss) {
    double *c[5] = {Res1, Res2, Res3, Res4, Res5};
    double *d[5] = {Res1_Diss, Res2_Diss, Res3_Diss, Res4_Diss, Res5_Diss};
    for (int k = 0; k < 5; k++) {
        memcpy(conv + (size_t)k * nNode, c[k], (size_t)nNode * sizeof(double));
        memcpy(diss + (size_t)k * nNode, d[k], (size_t)nNode * sizeof(double));
    }
}
void ref_set_residual(const double *conv, const double *diss) {
    double *c[5] = {Res1, Res2, Res3, Res4, Res5};
    double *d[5] = {Res1_Diss, Res2_Diss, Res3_Diss, Res4_Diss, Res5_Diss};
    for (int k = 0; k < 5; k++) {
        memcpy(c[k], conv + (size_t)k * nNode, (size_t)nNode * sizeof(double));
        memcpy(d[k], diss + (size_t)k * nNode, (size_t)nNode * sizeof(double));
    }
}
void ref_get_deltat(double *dt) { memcpy(dt, DeltaT, (size_t)nNode * sizeof(double)); }
void ref_set_deltat(const double *dt) { memcpy(DeltaT, dt, (size_t)nNode * sizeof(double)); }

/* out = {min1,max1,min4,max4,min5,max5,minDt,maxDt} */
void ref_get_extrema(double *out) {
    out[0] = MinEigenLamda1; out[1] = MaxEigenLamda1;
    out[2] = MinEigenLamda4; out[3] = MaxEigenLamda4;
    out[4] = MinEigenLamda5; out[5] = MaxEigenLamda5;
    out[6] = MinDeltaT; out[7] = MaxDeltaT;
}

/* Far-field globals after ComputeFarFieldCondition: rho,u,v,w,et,p,c,mach */
void ref_get_farfield(double *out) {
    out[0] = Inf_Rho; out[1] = Inf_U; out[2] = Inf_V; out[3] = Inf_W;
    out[4] = Inf_Et; out[5] = Inf_Pressure; out[6] = Inf_SpeedSound; out[7] = Inf_Mach;
}

int ref_nnz_blocks(void) { return SolverBlockMatrix.DIM; }
void ref_get_crs(int *IA, int *JA, int *IAU) {
    memcpy(IA, SolverBlockMatrix.IA, (size_t)(nNode + 1) * sizeof(int));
    memcpy(JA, SolverBlockMatrix.JA, (size_t)SolverBlockMatrix.DIM * sizeof(int));
    memcpy(IAU, SolverBlockMatrix.IAU, (size_t)nNode * sizeof(int));
}
/* A: [DIM][5][5] contiguous; B, X: [nNode][5]. */
void ref_get_matrix(double *A, double *B, double *X) {
    for (int b = 0; b < SolverBlockMatrix.DIM; b++)
        for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++) A[(size_t)b * 25 + i * 5 + j] = SolverBlockMatrix.A[b][i][j];
    for (int r = 0; r < nNode; r++)
        for (int i = 0; i < 5; i++) {
            B[(size_t)r * 5 + i] = SolverBlockMatrix.B[r][i];
            X[(size_t)r * 5 + i] = SolverBlockMatrix.X[r][i];
        }
}
void ref_set_matrix(const double *A, const double *B) {
    for (int b = 0; b < SolverBlockMatrix.DIM; b++)
        for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++) SolverBlockMatrix.A[b][i][j] = A[(size_t)b * 25 + i * 5 + j];
    for (int r = 0; r < nNode; r++)
        for (int i = 0; i < 5; i++) SolverBlockMatrix.B[r][i] = B[(size_t)r * 5 + i];
}

/* g: [15][nNode] in the order Q1x,Q1y,Q1z,...,Q5z; phi: [5][nNode]. */
void ref_get_gradients(double *g) {
    double *src[15] = {Q1x, Q1y, Q1z, Q2x, Q2y, Q2z, Q3x, Q3y, Q3z,
                       Q4x, Q4y, Q4z, Q5x, Q5y, Q5z};
    for (int k = 0; k < 15; k++) memcpy(g + (size_t)k * nNode, src[k], (size_t)nNode * sizeof(double));
}
void ref_set_gradients(const double *g) {
    double *dst[15] = {Q1x, Q1y, Q1z, Q2x, Q2y, Q2z, Q3x, Q3y, Q3z,
                       Q4x, Q4y, Q4z, Q5x, Q5y, Q5z};
    for (int k = 0; k < 15; k++) memcpy(dst[k], g + (size_t)k * nNode, (size_t)nNode * sizeof(double));
}
void ref_get_limiters(double *phi) {
    double *src[5] = {Limiter_Phi1, Limiter_Phi2, Limiter_Phi3, Limiter_Phi4, Limiter_Phi5};
    for (int k = 0; k < 5; k++) memcpy(phi + (size_t)k * nNode, src[k], (size_t)nNode * sizeof(double));
}

/* ---- Reference mesh pre-processing, for pinning the project's builder ----
 * UGrid_Reader (Euler3D/src/MeshIO.cpp:50) -> Create_Connectivity_Maps
 * (Connectivity_Maps.cpp:992) -> Calculate_Area_Volume (Area_Volume.cpp:903). */
void ref_mesh_from_ugrid(const char *path, int reorder) {
    Commons_Init();
    UGrid_Reader(path);
    Create_Connectivity_Maps(reorder);
    Calculate_Area_Volume();
}
void ref_mesh_sizes(int *out) {
    out[0] = nNode; out[1] = nBNode; out[2] = nEdge; out[3] = nBEdge;
    out[4] = crs_IA_Node2Node[nNode];
}
void ref_mesh_get(int *edge_nodes, double *edge_areav, int *bedge_nodes, double *bedge_areav,
                  int *bedge_tag, double *cvol, double *coords, int *n2n_ia, int *n2n_ja) {
    for (int i = 0; i < nEdge; i++) {
        edge_nodes[2 * i] = intEdge[i].node[0];
        edge_nodes[2 * i + 1] = intEdge[i].node[1];
        for (int k = 0; k < 3; k++) edge_areav[3 * i + k] = intEdge[i].areav.vec[k];
    }
    for (int i = 0; i < nBEdge; i++) {
        bedge_nodes[2 * i] = bndEdge[i].node[0];
        bedge_nodes[2 * i + 1] = bndEdge[i].node[1];
        bedge_tag[i] = bndEdge[i].tag;
        for (int k = 0; k < 3; k++) bedge_areav[3 * i + k] = bndEdge[i].areav.vec[k];
    }
    memcpy(cvol, cVolume, (size_t)nNode * sizeof(double));
    memcpy(coords, coordXYZ, (size_t)3 * nNode * sizeof(double));
    memcpy(n2n_ia, crs_IA_Node2Node, (size_t)(nNode + 1) * sizeof(int));
    memcpy(n2n_ja, crs_JA_Node2Node, (size_t)crs_IA_Node2Node[nNode] * sizeof(int));
}

}  // extern "C"
