/* cfd_b200.h -- C ABI of the B200-native implicit edge-based finite-volume
 * hot path (node-centred median-dual Euler solver: flux residual, 5x5
 * block-CRS Jacobian, block-CRS linear solves).
 *
 * Everything here is plain C: opaque handles, plain pointers and sizes, int
 * status codes.  No CUDA, C++ or torch types cross this boundary, so the
 * reference's C++ drivers (or ctypes, cgo, ...) can bind it directly.
 *
 * Data layout at the boundary is the reference's:
 *   - node state Q: SoA, 5 arrays of nNode+nGhost doubles, conservative
 *     variables (rho, rho*u, rho*v, rho*w, rho*et)
 *     (Euler3D/include/Solver.h:27-31);
 *   - interior edges: node[2] with node[0] < node[1] and the dual-face area
 *     vector pointing from node[0] to node[1]
 *     (Euler3D/include/Commons.h:97-105, Area_Volume.cpp:659-800);
 *   - boundary edges: node[0] physical, node[1] = its private ghost node
 *     (index >= nNode), outward area vector (Area_Volume.cpp:461-556,912);
 *   - block CRS: IA (nNode+1), JA (sorted, diagonal included), IAU (diagonal
 *     slot), A as [nnzb][5][5] row-major blocks, B and X as [nNode][5]
 *     (MATH/include/MC.h:16-28, Euler3D/src/Solver.cpp:612-704).
 *
 * Status codes: CFD_OK (0) or a negative CFD_ERR_*.  A numerical failure
 * detected on the device (NaN, negative density/pressure, Krylov breakdown)
 * is reported as CFD_ERR_NUMERIC and, for the linear solves, as a NaN RMS,
 * mirroring how the reference's drivers detect failure
 * (Euler3D/src/Solver_Steady_Implicit.cpp:131-150).  No entry point aborts
 * the process.
 */
#ifndef CFD_B200_H
#define CFD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFD_ABI_VERSION 6

/* ------------------------------------------------------------ status codes */
#define CFD_OK                 0
#define CFD_ERR_ARG           -1  /* bad argument / size                     */
#define CFD_ERR_MESH          -2  /* inconsistent mesh arrays                */
#define CFD_ERR_CUDA          -3  /* CUDA runtime error (see cfd_last_error) */
#define CFD_ERR_IO            -4  /* file I/O                                */
#define CFD_ERR_STATE         -5  /* call out of order (e.g. no mesh yet)    */
#define CFD_ERR_NUMERIC       -6  /* NaN / non-physical state on device      */
#define CFD_ERR_NOT_CONVERGED -7  /* Krylov budget exhausted                 */
#define CFD_ERR_UNSUPPORTED   -8  /* option not available on this path       */
#define CFD_ERR_RANGE         -9  /* size beyond a fixed capacity            */

/* ------------------------------------------- option values (reference enums)
 * Numeric values equal the reference's enums in
 * Euler3D/include/SolverParameters.h so parameter files map 1:1. */
#define CFD_FLUX_ROE   0   /* FLUX_SCHEME_ROE  (SolverParameters.h:111) */
#define CFD_FLUX_HLLC  1   /* FLUX_SCHEME_HLLC (SolverParameters.h:112) */
#define CFD_FLUX_AUSM  2   /* FLUX_SCHEME_AUSM (:113); AUSM+ (Liou 1996), the reference's is an empty stub */
#define CFD_FLUX_ROE_LMFIX 3 /* FLUX_SCHEME_ROE with PRECOND_METHOD_ROE_LMFIX (SolverParameters.h:136): the
                                low-Mach fix of Compute_Flux_Roe_LMFIX (Euler3D/src/FluxTest.cpp:2801) and the
                                preconditioned characteristic BC (BC.cpp:700) */
#define CFD_FLUX_ROE_PRECOND 4 /* FLUX_SCHEME_ROE with MPFLOW3D's Turkel-family preconditioning
                                (PRECOND_METHOD_BTW / _ERIKSSON / _TURKEL, MPFLOW3D/include/SolverParameters.h:141-144):
                                preconditioned Roe dissipation (Compute_Flux_Roe_Precondition_Turkel,
                                MPFLOW3D/src/Roe_Fluxes.cpp:2043), its eigenvalues in the time step,
                                the preconditioned pseudo-time term of the Jacobian (Roe_Jacobian.cpp:241)
                                and the preconditioned characteristic BC (MPFLOW3D/src/BC.cpp:113) */
#define CFD_FLUX_ROE_THORNBER 5 /* FLUX_SCHEME_ROE with MPFLOW3D's PRECOND_METHOD_THORNBER: the face velocities
                                blended toward each other by min(1, max Mach) before the Roe flux
                                (Compute_Flux_Roe_Thornber, MPFLOW3D/src/Roe_Fluxes.cpp:1081), plain
                                characteristic BCs */
#define CFD_FLUX_VANLEER 6    /* FLUX_SCHEME_VANLEER (SolverParameters.h:114): Van Leer flux-vector splitting
                                (Compute_VanLeerFlux, Euler3D/src/VanLeer_Fluxes.cpp:143), ideal gas only;
                                implicit steps use the approximate Roe Jacobian */
/* cfd_params.precond_method (MPFLOW3D PRECOND_METHOD values) */
#define CFD_PRECOND_BTW      2  /* Briley-Taylor-Whitfield: alpha 0, delta 1    */
#define CFD_PRECOND_ERIKSSON 3  /* Eriksson: alpha 0, delta beta                */
#define CFD_PRECOND_TURKEL   5  /* Turkel: alpha 0.4, delta beta                */
/* cfd_params.precond_type (MPFLOW3D PRECOND_TYPE values) */
#define CFD_PRECOND_LOCAL    0  /* beta from the local Mach and precond_mach    */
#define CFD_PRECOND_GLOBAL   1  /* beta = min(1, precond_mach)                  */
#define CFD_PRECOND_URLOCAL  2  /* beta = min(1, local Mach)                    */

#define CFD_ORDER_FIRST  0 /* SOLVER_ORDER_FIRST  (SolverParameters.h:316) */
#define CFD_ORDER_SECOND 1 /* SOLVER_ORDER_SECOND (SolverParameters.h:317) */

#define CFD_LIMITER_NONE  -1 /* LIMITER_METHOD_NONE           (:343) */
#define CFD_LIMITER_BJ     0 /* LIMITER_METHOD_BERTH_JESPERSEN(:344) */
#define CFD_LIMITER_VENKAT 1 /* LIMITER_METHOD_VENKATAKRISHNAN(:345) */

#define CFD_GRAD_LSQ 0   /* least squares (Euler3D/src/Gradient.cpp:232) */
#define CFD_GRAD_GG  1   /* Green-Gauss on the median dual (enum only in the reference, :329) */

#define CFD_BC_EULER_WALL 0  /* BC_TYPE_* (SolverParameters.h:40-58) */
#define CFD_BC_FAR_FIELD  1
#define CFD_BC_INFLOW     2
#define CFD_BC_OUTFLOW    3

#define CFD_PREC_FP64 0  /* Jacobian / preconditioner storage precision */
#define CFD_PREC_FP32 1
#define CFD_PREC_BF16 2
#define CFD_PREC_LOW_ONLY 0x10  /* or'ed with FP32/BF16 in cfd_jacobian / the GMRES precision: keep only the
                                   low-precision matrix (no FP64 copy); the outer FP64 correction is then the
                                   caller's nonlinear defect, and GMRES works with the stored matrix */

/* Solution variables (VARIABLE_TYPE, MPFLOW3D/include/SolverParameters.h:296-302): cfd_params.variables
 * (CONSERVATIVE or RUP) and the column names of cfd_rms_file_open (all four) */
#define CFD_VARS_CONSERVATIVE 0  /* VARIABLE_CONSERVATIVE / VARIABLE_CON: (rho, rho u, rho v, rho w, rho et) */
#define CFD_VARS_RUP          1  /* VARIABLE_RUP: (rho, u, v, w, p) */
#define CFD_VARS_PUT          2  /* (p, u, v, w, T)   */
#define CFD_VARS_RUT          3  /* (rho, u, v, w, T) */

#define CFD_PC_NONE      0  /* GMRES right preconditioner */
#define CFD_PC_BLOCK_JACOBI 1
#define CFD_PC_ILU0      2  /* ILU(0) in the mesh (row) order, level-scheduled */
#define CFD_PC_ILU0_MC   3  /* ILU(0) in block multicolour order: 32-row patches, patch graph coloured
                               by DSATUR, one launch per colour in factorisation and solves */

/* Solver options; mirrors the reference parameter file keys named beside
 * each field (Euler3D/src/SolverParameters.cpp:184-700). */
typedef struct cfd_params {
    int    flux_scheme;      /* FLUX_SCHEME                  */
    int    order;            /* SOLVER_ORDER                 */
    int    limiter;          /* LIMITER_METHOD               */
    int    limiter_order;    /* LIMITER_ORDER (0 first, 1 second) */
    int    limiter_smooth;   /* LIMITER_SMOOTH               */
    int    gradient;         /* CFD_GRAD_LSQ / CFD_GRAD_GG   */
    int    ls_weight;        /* 0 unweighted, 1 inverse distance (Gradient.cpp:151) */
    int    entropy_fix;      /* ENTROPY_FIX                  */
    int    global_time;      /* TIME_INTEGRATION_TYPE == GLOBAL */
    int    cfl_ramp;         /* CFL_RAMP                     */
    int    mach_ramp;        /* MACH_RAMP                    */
    int    zpg_iteration;    /* ZPG_ITERATION                */
    double gamma;            /* GAMMA                        */
    double mach;             /* REF_MACH (== MACH_MAX)       */
    double mach_min;         /* MACH_MIN                     */
    double alpha_deg;        /* REF_ALPHA (degrees)          */
    double beta_deg;         /* REF_BETA  (degrees)          */
    double cfl_min;          /* CFL_MIN                      */
    double cfl_max;          /* CFL_MAX                      */
    double venkat_k;         /* VENKAT_K_THRESHOLD           */
    int    residual_kernel;  /* 0: node-gather kernel (sliced-ELL), 1: shared-memory patch kernel
                                (its layout is built when 1 is first set on a context with a mesh) */
    /* Stiffened-gas constant p_inf / p_ref (0: the reference's ideal gas).
     * p = (gamma - 1) rho e - gamma pinf, c^2 = gamma (p + pinf) / rho; the
     * freestream keeps rho = 1, p = 1 and c = sqrt(gamma (1 + pinf)).  No
     * counterpart in the reference (Euler3D/MPFLOW3D are ideal-gas only,
     * EOS/src/EOS_IdealGas.c:73); at pinf = 0 every result is bit-identical
     * to the ideal-gas path. */
    double pinf;
    /* CFD_FLUX_ROE_PRECOND only (MPFLOW3D SolverParameters.cpp:75-78, Material.cpp:57):
     * PRECOND_METHOD, PRECOND_TYPE, PRECOND_GLOBAL_MACH and OUTFLOW_PRESSURE
     * (the subsonic-outflow pressure of the preconditioned BC; 0 = the
     * freestream pressure).  PRECOND_SMOOTH is NO (beta from the edge's own
     * states); the averages are Roe averages (AVERAGE_TYPE_ROE). */
    int    precond_method;
    int    precond_type;
    double precond_mach;
    double outflow_pressure;
    /* VARIABLE_TYPE: the variables the state Q holds, which the gradients and
     * limiters act on, the second-order faces are reconstructed in, the
     * boundary ghost states are written in, and the Jacobian's columns and the
     * update X refer to.
     *   CFD_VARS_CONSERVATIVE: Euler3D's formulation (and the layout at the top
     *     of this file);
     *   CFD_VARS_RUP: (rho, u, v, w, p), MPFLOW3D's implicit formulation
     *     (GUAGE_PRESSURE 0): faces take p directly (Material_Get_Properties,
     *     MPFLOW3D/src/Material.cpp:591-599), Thornber blends the velocities
     *     at fixed rho and p (Roe_Fluxes.cpp:1161-1168), and the Jacobian is
     *     d/d(rho,u,v,w,p): the convective blocks dF/dW at the nodes
     *     (CompressibleUtils.cpp:85-186), the dissipation Mop |A| at the Roe
     *     state (Roe_Fluxes.cpp:3185-3199) and the pseudo-time term
     *     (V/dt) Mop [Kinv] (Roe_Jacobian.cpp:241-264).  The residual is still
     *     the conservation-law residual.  Not on cfd_jacobian_fd or
     *     cfd_solve_unsteady (CFD_ERR_UNSUPPORTED).
     * The stiffened gas keeps its pressure exact in RUP (no gamma pinf
     * cancellation). */
    int    variables;
} cfd_params;

/* Fills p with the defaults used by the reference parameter files of this
 * path (ideal gas, generic non-dimensionalisation, first-order Roe). */
void cfd_params_default(cfd_params *p);

/* ------------------------------------------------------------- lifecycle */
typedef struct cfd_ctx cfd_ctx;

int  cfd_abi_version(void);
/* Text of the last error recorded on this thread (never NULL). */
const char *cfd_last_error(void);

int  cfd_create(int device, cfd_ctx **out);
int  cfd_destroy(cfd_ctx *ctx);
/* Run all work of ctx on this cudaStream_t (NULL = the legacy stream). */
int  cfd_set_stream(cfd_ctx *ctx, void *cuda_stream);
int  cfd_set_params(cfd_ctx *ctx, const cfd_params *p);
int  cfd_synchronize(cfd_ctx *ctx);

/* Install the median-dual mesh (host arrays, copied; the caller keeps
 * ownership).  Replaces the device mirror of the reference globals
 * nNode, nBNode, nEdge, intEdge, nBEdge, bndEdge, cVolume, coordXYZ,
 * crs_IA/JA_Node2Node (Euler3D/include/Commons.h:64-105) and builds the
 * block-CRS pattern of Create_CRS_SolverBlockMatrix (Solver.cpp:612-704).
 *   edge_nodes  [2*nedge]   edge_areav  [3*nedge]
 *   bedge_nodes [2*nbedge]  bedge_areav [3*nbedge]  bedge_type [nbedge]
 *   cvol [nnode]  coords [3*nnode] (xyz interleaved, as coordXYZ)
 *   n2n_ia [nnode+1]  n2n_ja [n2n_ia[nnode]]  (no diagonal) */
int  cfd_set_mesh(cfd_ctx *ctx, int nnode, int nghost,
                  int nedge, const int *edge_nodes, const double *edge_areav,
                  int nbedge, const int *bedge_nodes, const double *bedge_areav,
                  const int *bedge_type, const double *cvol, const double *coords,
                  const int *n2n_ia, const int *n2n_ja);

/* Block-CRS pattern built by cfd_set_mesh: sizes[0] = nnzb; IA/JA/IAU as
 * SolverBlockMatrix (any pointer may be NULL to query sizes only). */
int  cfd_get_block_pattern(cfd_ctx *ctx, int64_t *nnzb, int *IA, int *JA, int *IAU);

/* ----------------------------------------------------------- state I/O */
/* Q host SoA [5][nnode+nghost] <-> device. */
int  cfd_set_state(cfd_ctx *ctx, const double *Q);
int  cfd_get_state(cfd_ctx *ctx, double *Q);
/* Device pointer of the resident state (SoA, leading dimension *ld >=
 * nnode+nghost) for zero-copy callers.  A state written through it after
 * cfd_gradient needs cfd_gradient again before cfd_limiter. */
int  cfd_state_device_ptr(cfd_ctx *ctx, double **dQ, int64_t *ld);
/* Freestream state per node (Solver_Set_Initial_Conditions,
 * Euler3D/src/Solver.cpp:339-393) on the device, in the variables of the
 * context's cfd_params. */
int  cfd_set_freestream(cfd_ctx *ctx);

/* --------------------------------------------- hot path (device-resident)
 * Each call is stream-ordered on the context's stream. */

/* Per-iteration resets of Solver_Steady_Implicit.cpp:45-98: zero the residual
 * / spectral-radius accumulators, reset extrema, evaluate the far field with
 * Mach ramping (ComputeFarFieldCondition, Material.cpp:185-210). */
int  cfd_begin_iteration(cfd_ctx *ctx, int iteration);
/* Ghost-node states, characteristic BCs (Apply_Boundary_Condition,
 * Euler3D/src/BC.cpp:1440-1487, 381-677). */
int  cfd_apply_bc(cfd_ctx *ctx, int iteration);
/* Node gradients of Q1..Q5 (Compute_Least_Square_Gradient,
 * Euler3D/src/Gradient.cpp:232-296, or Green-Gauss).  With Green-Gauss,
 * second order and a limiter, the limiters of the same state are formed in
 * the same pass and taken by the next cfd_limiter. */
int  cfd_gradient(cfd_ctx *ctx);
/* Limiter (Compute_Limiter, Euler3D/src/Limiters.cpp:20-111) of the state
 * and gradients of the last cfd_gradient.  Its pressure fixes (:61-110,
 * :273-304) are completed by the next second-order cfd_residual, or by
 * cfd_get_limiters. */
int  cfd_limiter(cfd_ctx *ctx);
/* Flux residual (Compute_Residual, Euler3D/src/Residual.cpp:18 ->
 * FluxTest.cpp:7968 Roe / HLLC_Fluxes.cpp:519 HLLC / AUSM+).  Writes the
 * convective and dissipative residuals separately (Res*, Res*_Diss), and when
 * add_time != 0 accumulates sum(area*lambda_max) per node and the
 * eigenvalue extrema. */
int  cfd_residual(cfd_ctx *ctx, int add_time);
/* Local time step dt_i = V_i*CFL/sum (Compute_DeltaT, Time_Step.cpp:23-51). */
int  cfd_deltat(cfd_ctx *ctx, int iteration);
/* RMS of the residual as Solver_Steady_Implicit.cpp:107-126: out[0..4]
 * per equation, out[5] = RMS_Res.  include_diss adds Res_Diss first
 * (MPFLOW3D semantics). */
int  cfd_residual_rms(cfd_ctx *ctx, int include_diss, double out[6]);

/* Approximate first-order Roe Jacobian + right-hand side
 * (Compute_Jacobian, Euler3D/src/Jacobian.cpp:18 ->
 * Roe_Jacobian.cpp:29-228).  B = -(Res + include_diss*Res_Diss);
 * diagonal += V/dt when add_time.  precision: CFD_PREC_FP64/FP32/BF16 storage
 * of A; the FP64 copy is kept for the linear defect correction unless
 * CFD_PREC_LOW_ONLY is or'ed in, in which case the diagonal blocks are summed
 * (in FP64) from the stored low-precision off-diagonal blocks and only the
 * low-precision matrix exists (cfd_block_gs and the mesh-order ILU(0) /
 * block-Jacobi preconditioners then need a new FP64 Jacobian). */
int  cfd_jacobian(cfd_ctx *ctx, int add_time, int include_diss, int precision);

/* Block Gauss-Seidel with LU-factored diagonal blocks, X = 0 start
 * (MC_Iterative_Block_LU_Jacobi_CRS, MATH/src/MC_Iterative_Jacobi.c:346-535):
 * direction 0 forward, 1 backward, 2 alternating.  Level-scheduled on the
 * device, same row order and arithmetic as the reference.  *rms = RMS of the
 * last sweep's residual. */
int  cfd_block_gs(cfd_ctx *ctx, int iterations, int direction, double *rms);

/* Finite-difference Roe Jacobian (Compute_Jacobian_FiniteDifference_Roe,
 * Euler3D/src/Roe_Jacobian.cpp:236): difference quotients (eps = 1e-8) of the
 * reference's matrix-form Roe flux (Roe_Fluxes.cpp:552) of first-order states;
 * interior edges by `method`, boundary edges by central differences with the
 * ghost state rebuilt by the older characteristic BC (BC.cpp:33) for every
 * perturbed state.  FP64 system; B = -(Res + include_diss * Res_Diss).
 * method: JACOBIAN_METHOD_* (SolverParameters.h:274-279); ALTERNATE is forward
 * on even iterations, backward on odd ones. */
#define CFD_JAC_CENTRAL   0
#define CFD_JAC_FORWARD   1
#define CFD_JAC_BACKWARD  2
#define CFD_JAC_ALTERNATE 3
int  cfd_jacobian_fd(cfd_ctx *ctx, int add_time, int include_diss, int method, int iteration);

/* Block LU-SGS (MC_Iterative_Block_LUSGS_CRS, MATH/src/MC_Iterative_Jacobi.c:539):
 * X starts at each row's mean of B; each iteration is a forward then a
 * backward Gauss-Seidel sweep in which the diagonal block is solved by
 * Gaussian elimination with partial pivoting.  Bit-exact with the reference
 * (level-scheduled sweeps, explicitly rounded arithmetic).  *rms is the
 * reference's returned value (computed as it computes it). */
int  cfd_block_lusgs(cfd_ctx *ctx, int iterations, double *rms);

typedef struct cfd_gmres_opts {
    int    restart;        /* Krylov dimension m (30)                       */
    int    max_iters;      /* total inner iterations budget                 */
    double rtol;           /* relative residual target, e.g. 1e-6           */
    int    precond;        /* CFD_PC_*                                      */
    int    precision;      /* CFD_PREC_* of the preconditioner / A copy     */
    int    refine;         /* FP64 outer iterative-refinement sweeps (>=1)   */
    int    reuse_precond;  /* 1: keep the preconditioner factored by the previous
                              call (same kind and precision) instead of
                              factoring the current matrix again            */
} cfd_gmres_opts;

typedef struct cfd_gmres_stats {
    int    iterations;     /* inner iterations done                          */
    int    restarts;
    int    refinements;
    double rel_residual;   /* ||B - A X|| / ||B|| in FP64 at exit            */
} cfd_gmres_stats;

void cfd_gmres_default(cfd_gmres_opts *o);
/* Solves A X = B (A, B from cfd_jacobian) with right-preconditioned
 * restarted GMRES; FP64 Arnoldi with compensated dot products.  The
 * reference has no block GMRES on this path (its MPI scalar GMRES,
 * MATH/src/ParallelLinearAlgebra.cpp:27-278, is unused); this is the solver
 * the implicit drivers call in its place. */
int  cfd_gmres(cfd_ctx *ctx, const cfd_gmres_opts *o, cfd_gmres_stats *st);

/* The two operators of a Krylov iteration on their own, on DEVICE vectors of
 * the context's device ([nnode][5] FP64, stream-ordered on the context's
 * stream): cfd_spmv forms y = A x with the stored copy of the system of the
 * given CFD_PREC_* (the FP64 copy when that copy is not stored; the stored
 * low-precision copy when only that one exists); cfd_precond_apply forms
 * z = M^-1 r with the preconditioner factored by the last cfd_gmres
 * (CFD_ERR_STATE when there is none).  The reference's block products are
 * inside its Gauss-Seidel sweeps (MATH/src/MC_Iterative_Jacobi.c:346-535);
 * these give the GPU solver's products to a caller's own Krylov loop. */
int  cfd_spmv(cfd_ctx *ctx, int precision, const double *x, double *y);
int  cfd_precond_apply(cfd_ctx *ctx, const double *r, double *z);

/* Factorisation order of CFD_PC_ILU0_MC: order[k] = row at position k
 * (nnode entries; colours in increasing order, rows of a colour in increasing
 * index) and the number of colours.  Either pointer may be NULL. */
int  cfd_ilu_mc_order(cfd_ctx *ctx, int *order, int *ncolor);

/* Block Gauss-Seidel that allocates no device memory.  No counterpart in the
 * reference: it exists for callers that cannot let a library call cudaMalloc
 * (a host framework that reserved all device memory up front and passes in only
 * its own buffers, or a running solver loop that must not reach the CUDA
 * allocator).  Same sweeps and arithmetic as cfd_block_gs, on a system the
 * caller holds in device memory: IA/JA/IAU block-CRS pattern (as
 * SolverBlockMatrix), A [nnzb][5][5], B and X [nrow][5]; X is overwritten
 * (starts at zero), *rms as cfd_block_gs.  Its scratch is one static device
 * array of this library for up to CFD_GS_STATIC_MAX_ROWS rows (about 3.5 MB,
 * reserved on every GPU that loads the library until the process exits);
 * larger systems return CFD_ERR_RANGE.  The array is shared: calls that
 * overlap on the GPU race, so keep them on one stream.  The first call on a
 * device looks up the array's device address (make it before any stream
 * capture) and keeps it until exit: do not cudaDeviceReset the device while
 * the library is in use.  The caller's pattern is checked on the host before
 * any launch (IA increasing from 0, JA in range, JA[IAU[r]] == r with IAU[r] in
 * row r), CFD_ERR_ARG otherwise.  Each call copies the pattern to the host
 * (two synchronising copies), rebuilds its level schedules there (O(nnz)) and
 * synchronises once per sweep.  Work runs on `stream` (a cudaStream_t, NULL =
 * legacy stream). */
#define CFD_GS_STATIC_MAX_ROWS 16384
int  cfd_block_gs_static(int nrow, const int *IA, const int *JA, const int *IAU, const double *A,
                         const double *B, double *X, int iterations, int direction, void *stream,
                         double *rms);

/* Q += relax * X on physical nodes (Solver_Steady_Implicit.cpp:153-159). */
int  cfd_update(cfd_ctx *ctx, double relax);

/* -------------------------------------------------------------- readback */
int  cfd_get_residual(cfd_ctx *ctx, double *conv, double *diss);  /* [5][nnode] each */
int  cfd_get_deltat(cfd_ctx *ctx, double *dt);                    /* [nnode] */
/* {minL1,maxL1,minL4,maxL4,minL5,maxL5,minDt,maxDt}, DBL_MAX/DBL_MIN when unset */
int  cfd_get_extrema(cfd_ctx *ctx, double out[8]);
/* Far field {rho,u,v,w,et,p,c,mach} of the last cfd_begin_iteration. */
int  cfd_get_farfield(cfd_ctx *ctx, double out[8]);
/* Override the far field with values a driver computed itself (its globals
 * Inf_Rho, Inf_U, Inf_V, Inf_W, Inf_Et, Inf_Pressure, Inf_SpeedSound, Inf_Mach
 * after ComputeFarFieldCondition, Euler3D/src/Material.cpp:185-210); holds
 * until the next cfd_begin_iteration / cfd_deltat. */
int  cfd_set_farfield(cfd_ctx *ctx, const double in[8]);
int  cfd_get_gradients(cfd_ctx *ctx, double *g);                  /* [15][nnode] */
int  cfd_get_limiters(cfd_ctx *ctx, double *phi);                 /* [5][nnode]  */
/* A [nnzb][25] (FP64 copy), B [nnode][5], X [nnode][5]; NULL skips. */
int  cfd_get_system(cfd_ctx *ctx, double *A, double *B, double *X);
/* Replace A/B (host, FP64) -- lets a caller solve a system assembled elsewhere. */
int  cfd_set_system(cfd_ctx *ctx, const double *A, const double *B);

/* ------------------------------------------- fused steps and whole solves */
/* One residual evaluation of the hot path: begin_iteration + BC + (gradient
 * + limiter when second order) + residual + deltat.  With Q_host != NULL the
 * state is copied in first and, with conv_host/diss_host != NULL, the
 * residuals are copied back (the end-to-end form of the call).  In that
 * form, for second order with Green-Gauss gradients and a limiter on a
 * stream set by cfd_set_stream, the copies overlap the kernels: the state
 * goes up and the residuals come down in node chunks while other chunks are
 * computed (results identical to the unpipelined calls). */
int  cfd_residual_step(cfd_ctx *ctx, int iteration, const double *Q_host,
                       double *conv_host, double *diss_host);
/* Chunks of the pipelined cfd_residual_step: -1 automatic (the default: up to
 * 16 chunks of >= 131072 nodes, none below 262144 nodes), 0 or 1 off, k >= 2
 * k chunks (at most nnode / 256). */
int  cfd_set_step_pipeline(cfd_ctx *ctx, int chunks);

typedef struct cfd_solve_opts {
    int    max_iterations;   /* SOLVER_NITERATION                         */
    double drop;             /* stop when RMS <= drop * RMS(first), e.g. 1e-8 */
    int    include_diss;     /* 1: B = -(Res+Res_Diss) (MPFLOW3D), 0: Euler3D */
    int    linear_solver;    /* 0 block GS sweeps, 1 GMRES                 */
    int    linear_iters;     /* LINEAR_SOLVER_NITERATION / GMRES budget    */
    double relax;            /* SOLVER_RELAXATION                          */
    cfd_gmres_opts gmres;
    int    precond_update;   /* factor the GMRES preconditioner every k implicit
                                iterations (<= 1: every one); the Jacobian itself
                                is rebuilt every iteration                  */
} cfd_solve_opts;

typedef struct cfd_solve_stats {
    int    iterations;
    double rms_first;
    double rms_last;
    int    linear_iterations;  /* summed over the solve                   */
    int    status;
} cfd_solve_stats;

/* Implicit steady solve (Solver_Steady_Implicit, Euler3D/src/
 * Solver_Steady_Implicit.cpp:35-184) entirely on the device. */
int  cfd_solve_steady(cfd_ctx *ctx, const cfd_solve_opts *o, cfd_solve_stats *st);

/* Physical-time implicit solve (Solver_Unsteady_Implicit,
 * MPFLOW3D/src/Solver_Unsteady_Implicit.cpp:36-305): `steps` physical steps of
 * `dt`, each converged by `inner_iterations` Newton iterations of
 *   (J + (1+theta) V/dt I) dQ = -(Res + Res_Diss + V/dt ((1+theta)(Q - Q^n) - theta (Q^n - Q^n-1)))
 * with J the approximate Jacobian without a pseudo-time term (AddTime FALSE);
 * theta = 0 (TIME_INTEGRATION_METHOD_IMPLICIT_EULER_EULER) or, with bdf2,
 * 0.5 from the second step on (TIME_INTEGRATION_METHOD_IMPLICIT_EULER_BDF). */
typedef struct cfd_unsteady_opts {
    double dt;               /* PHYSICAL_DELTA_TIME (non-dimensional)       */
    int    steps;            /* physical time steps                          */
    int    inner_iterations; /* INNER_NITERATION                             */
    int    bdf2;             /* 1: second-order backward difference          */
    int    include_diss;     /* as cfd_solve_opts                            */
    int    linear_solver;    /* 0 block GS sweeps (the reference's), 1 GMRES */
    int    linear_iters;     /* LINEAR_SOLVER_NITERATION                     */
    double relax;            /* SOLVER_RELAXATION                            */
    cfd_gmres_opts gmres;
} cfd_unsteady_opts;

typedef struct cfd_unsteady_stats {
    int    steps;              /* physical steps completed                   */
    int    inner_iterations;   /* summed                                    */
    double rms_last;           /* RMS of the last inner iteration           */
    int    linear_iterations;  /* summed                                    */
    int    status;
} cfd_unsteady_stats;

int  cfd_solve_unsteady(cfd_ctx *ctx, const cfd_unsteady_opts *o, cfd_unsteady_stats *st);

/* ----------------------------------------------------- host mesh builder */
typedef struct cfd_mesh cfd_mesh;

/* Node numberings of the builder.  PATCH_RCM: recursive-coordinate-bisection
 * patches of CFD_PATCH_NODES nodes, patches ordered by reverse Cuthill-McKee of
 * the patch graph; the residual kernel computes each edge flux once per patch
 * (patches are contiguous node ranges of this size), so this numbering makes
 * the patches spatially compact. */
#define CFD_NUMBERING_NATURAL   0
#define CFD_NUMBERING_RCM       1
#define CFD_NUMBERING_PATCH_RCM 2
#define CFD_PATCH_NODES 128

/* Tet-split box of nx*ny*nz hexes (6 tets each) over [0,lx]x[0,ly]x[0,lz],
 * interior nodes jittered by U(+-jitter*h) from seed, node numbering
 * CFD_NUMBERING_*, face BC types {xmin,xmax,ymin,ymax,zmin,zmax}.
 * Median-dual metrics as Calculate_Area_Volume (Area_Volume.cpp:903). */
int  cfd_mesh_box(int nx, int ny, int nz, double lx, double ly, double lz,
                  double jitter, uint64_t seed, int numbering, const int face_bc[6],
                  cfd_mesh **out);
/* Same from explicit cells: tets [4*ntet] positively oriented, boundary
 * triangles [3*ntri] with outward right-hand normals, tri_bc [ntri]. */
int  cfd_mesh_from_cells(int nnode, const double *coords, int64_t ntet, const int *tets,
                         int64_t ntri, const int *tris, const int *tri_bc, cfd_mesh **out);
/* sizes: {nnode, nghost, nedge, nbedge, ntet, ntri, n2n_nnz} */
int  cfd_mesh_sizes(const cfd_mesh *m, int64_t sizes[7]);
/* Copies out the arrays cfd_set_mesh takes (any pointer may be NULL). */
int  cfd_mesh_export(const cfd_mesh *m, int *edge_nodes, double *edge_areav,
                     int *bedge_nodes, double *bedge_areav, int *bedge_type,
                     double *cvol, double *coords, int *n2n_ia, int *n2n_ja);
int  cfd_mesh_export_cells(const cfd_mesh *m, int *tets, int *tris, int *tri_bc);
/* UGRID ASCII in the layout of UGrid_Reader (Euler3D/src/MeshIO.cpp:50). */
int  cfd_mesh_write_ugrid(const cfd_mesh *m, const char *path);
/* Reads a UGRID ASCII mesh of tetrahedra, pyramids, prisms and hexahedra
 * with boundary triangles and quadrilaterals (UGrid_Reader,
 * Euler3D/src/MeshIO.cpp:50-216, its winding translation :22-45) and builds
 * its median dual as Calculate_Area_Volume (Area_Volume.cpp:461-902): per
 * element edge the two triangles mid-edge -> face centroid -> cell centroid,
 * control volumes from the small tetrahedra, one boundary edge and ghost per
 * boundary-face vertex (triangles first, then quadrilaterals).  Boundary tag t
 * gets BC type tag_bc[t-1] (the BC file's list, ntag entries; NULL: far field
 * everywhere).  numbering: CFD_NUMBERING_* applied before the dual is built. */
int  cfd_mesh_read_ugrid(const char *path, int ntag, const int *tag_bc, int numbering, cfd_mesh **out);
/* Convenience: cfd_set_mesh from a builder mesh. */
int  cfd_set_mesh_from(cfd_ctx *ctx, const cfd_mesh *m);
void cfd_mesh_free(cfd_mesh *m);

/* Initial state of a request: the generic freestream (rho = 1, p = 1,
 * c = sqrt(gamma), velocity from mach, alpha, beta) with density, each
 * velocity component and pressure of every physical node multiplied by
 * (1 + noise * U(-1,1)), U from a counter-based hash of (seed, variable,
 * node); ghosts at freestream.  Q is SoA [5][nnode+nghost] (host). */
int  cfd_perturbed_freestream(const cfd_mesh *m, double gamma, double mach, double alpha_deg, double beta_deg,
                              double noise, uint64_t seed, double *Q);
/* The same for any gas of p (gamma, pinf, mach, alpha, beta): the freestream
 * of p with density, velocity and pressure noise of their own amplitudes
 * noise[0..2] (same hash streams as above); with pinf = 0 and three equal
 * amplitudes it equals cfd_perturbed_freestream.  Q is in p->variables. */
int  cfd_initial_state(const cfd_mesh *m, const cfd_params *p, const double noise[3], uint64_t seed, double *Q);

/* ------------------------------------------------------------ serving loop
 * No counterpart in the reference (its drivers run one solve per process).
 * A server runs steady-solve requests concurrently on one GPU: requests queue
 * in arrival order; a worker (one host thread and one CUDA stream each) takes
 * the head request when its device-memory estimate fits in what is left of
 * the budget, builds its tet-split box mesh on the host, sets the seeded
 * initial state and runs cfd_solve_steady.  Workers allocate device memory
 * stream-ordered, so solves of different sizes overlap on the GPU without
 * device-wide synchronisation.  Results do not depend on the other requests
 * (all kernels are deterministic). */
#define CFD_PENDING 1  /* cfd_server_wait: not finished within the timeout */

typedef struct cfd_server cfd_server;

typedef struct cfd_serve_request {
    int      nx, ny, nz;        /* tet-split box of nx*ny*nz hexes ...        */
    double   lx, ly, lz;        /* ... over [0,lx]x[0,ly]x[0,lz]               */
    double   jitter;            /* interior node jitter (fraction of h)       */
    uint64_t mesh_seed;
    int      numbering;         /* CFD_NUMBERING_*                           */
    int      face_bc[6];        /* CFD_BC_* of xmin,xmax,ymin,ymax,zmin,zmax  */
    double   noise;             /* initial state, see cfd_perturbed_freestream */
    uint64_t state_seed;
    cfd_params params;
    cfd_solve_opts opts;
    int      keep_state;        /* 1: keep the final state (cfd_server_state) */
} cfd_serve_request;

typedef struct cfd_serve_result {
    int    status;              /* CFD_OK, CFD_PENDING, or the failing call's code */
    cfd_solve_stats stats;
    int    nnode, nghost;
    double t_submit, t_admit, t_start_solve, t_done;  /* seconds on the server's clock */
    double bytes_estimate;      /* device memory reserved against the budget  */
    char   message[160];        /* error text when status < 0                  */
} cfd_serve_result;

/* workers: concurrent solves; budget_bytes: device memory the admitted
 * requests may reserve together (each request's estimate is
 * 1.2 * (N*(1644 + 40*(m+6)) + 15.5*N*(A + M + 60)) + 16 MiB bytes for N
 * nodes, GMRES restart m, A bytes per stored Jacobian block and M = 3 x
 * the bytes per factor block, for the factors and their packed copy). */
int  cfd_server_create(int device, int workers, double budget_bytes, cfd_server **out);
/* Queues a request; CFD_ERR_RANGE when its estimate exceeds the budget. */
int  cfd_server_submit(cfd_server *srv, const cfd_serve_request *req, int64_t *id);
/* Waits up to timeout_s (< 0: forever); CFD_PENDING on timeout. */
int  cfd_server_wait(cfd_server *srv, int64_t id, double timeout_s, cfd_serve_result *out);
/* Final state [5][nnode+nghost] of a finished request that kept it. */
int  cfd_server_state(cfd_server *srv, int64_t id, double *Q);
/* Forgets a finished request (its result and state). */
int  cfd_server_release(cfd_server *srv, int64_t id);
/* {active, queued, reserved bytes, peak reserved bytes, server clock s} */
int  cfd_server_stats(cfd_server *srv, double out[5]);
/* Fused launches across requests (on by default, window 50 us): the
 * interior residual launch and the GMRES block SpMV launches of each request
 * in its solve are handed to a batcher, which launches the jobs of one kernel
 * that are waiting when as many jobs as requests in their solves have
 * arrived, or window_us after the first, as one kernel over a request table
 * (k_residual_gather_batch, k_bspmv_batch; conservative-variable requests);
 * each request's results agree either way to round-off, with the same
 * iteration counts.  Set before the first submit.  batch_stats:
 * {fused residual launches, residual jobs in them, fused SpMV launches, SpMV
 * jobs in them}. */
int  cfd_server_set_batching(cfd_server *srv, int enable, double window_us);
int  cfd_server_batch_stats(cfd_server *srv, double out[4]);
/* Running requests finish; queued ones are dropped. */
int  cfd_server_destroy(cfd_server *srv);

/* ------------------------------------------------------ VTK solution file
 * VTK_Writer (Euler3D/src/MeshIO.cpp:219-372), conservative variables: the
 * legacy ASCII file the reference writes at the end of a run (points,
 * surface triangles then tetrahedra with 0-based node indices, cell types,
 * boundary ids = tri_tag or 1 when NULL, density, velocity components,
 * pressure, temperature, Mach number, velocity vector of the nnode physical
 * nodes of Q, SoA [5][ld]).  Byte-identical to the reference's file for the
 * same mesh and state with pinf = 0 (derived fields in its operation order);
 * with pinf > 0 pressure, temperature and Mach follow the stiffened gas.  Q is
 * in p->variables (a RUP state is written through its conservative form). */
int  cfd_vtk_write(const char *path, int nnode, const double *coords, int64_t ntri, const int *tris,
                   const int *tri_tag, int64_t ntet, const int *tets, const cfd_params *p, const double *Q,
                   int64_t ld);

/* ------------------------------------------------- restart file (binary)
 * Byte-compatible with Restart_Writer / Restart_Reader
 * (Euler3D/src/RestartIO.cpp:45-179): int32 {iteration, nNode, nBNode, 5}
 * then (nNode+nBNode) rows of 5 doubles. */
int  cfd_restart_write(const char *path, int iteration, int nnode, int nghost, const double *Q);
int  cfd_restart_read(const char *path, int *iteration, int nnode, int nghost, double *Q);

/* ------------------------------------------ residual history (Residual.res)
 * The text file the reference's RMS writers keep, one line per iteration.
 *   CFD_RMSFILE_EULER3D  (Euler3D/src/RMSIO.cpp:21-97): iteration, RMS per
 *     equation, RMS_Res, min/max time step, min/max lambda 1, 4, 5 (and the
 *     preconditioner's min/max sigma when precond != 0);
 *   CFD_RMSFILE_MPFLOW3D (MPFLOW3D/src/RMSIO.cpp:21-154): the same with every
 *     RMS first given normalised by the scale MPFLOW3D accumulates over its
 *     first five writes.
 * Header, column names, widths and number formats as the reference's, so the
 * file is byte-identical for the same values.  variables: the solution
 * variables the column names refer to (CFD_VARS_*).  cfd_rms_file_write
 * takes rms[6] as cfd_residual_rms gives it (per equation, then RMS_Res),
 * extrema[8] in cfd_get_extrema's order and sigma[2] (min, max) when the file
 * has a preconditioner; cfd_rms_file_write_ctx reads both from a context
 * (non-preconditioned files).  close writes the closing rule line. */
#define CFD_RMSFILE_EULER3D  0
#define CFD_RMSFILE_MPFLOW3D 1
typedef struct cfd_rms_file cfd_rms_file;
int  cfd_rms_file_open(const char *path, int layout, int variables, int precond, cfd_rms_file **out);
int  cfd_rms_file_write(cfd_rms_file *f, int iteration, const double rms[6], const double extrema[8],
                        const double sigma[2]);
int  cfd_rms_file_write_ctx(cfd_rms_file *f, cfd_ctx *ctx, int iteration, int include_diss);
int  cfd_rms_file_close(cfd_rms_file *f);

#ifdef __cplusplus
}
#endif
#endif /* CFD_B200_H */
