/* CPU restatement of the reference's implicit edge-based FV hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; it is never linked into or called by the product library.  Plain
 * C, FP64, sequential loops in the reference's order.  Parity of this
 * restatement with the reference itself is pinned by tests/test_oracle_pin.py
 * against the reference objects compiled in oracle/_ref.  Functions for
 * methods the reference does not implement (Green-Gauss, AUSM+, block ILU(0),
 * GMRES) are restated from the published methods; those are "parity unpinned"
 * by the reference and are pinned by property tests (linear exactness,
 * conservation, agreement with a dense direct solve).
 */
#ifndef CFD_ORACLE_H
#define CFD_ORACLE_H

typedef struct {
    double gamma, mach, alpha_deg, beta_deg, cfl, venkat_k;
    int flux, order, limiter, limiter_order, limiter_smooth, entropy_fix;
    int global_time, ls_weight, gradient, iteration, zpg_iteration;
    double pinf; /* stiffened-gas constant (0: ideal gas) */
    /* flux 4, preconditioned Roe (MPFLOW3D enum values): method 2 BTW, 3 Eriksson,
     * 5 Turkel; type 0 local, 1 global, 2 unrestricted local; reference Mach;
     * subsonic outflow pressure (0: freestream) */
    int pc_method, pc_type;
    double pc_mach, outflow_p;
    /* face average of the preconditioned Roe: 0 Roe (MPFLOW3D AVERAGE_TYPE_ROE), 1 simple
     * arithmetic mean of rho, u, v, w, h (Euler3D's Compute_Flux_Roe_Precondition_BTW,
     * FluxTest.cpp:3917-3940) */
    int pc_avg;
    /* Roe dissipation form (test pins only): 0 the closed form of Euler3D's
     * Compute_Flux_Roe_Optimized (FluxTest.cpp:3143-3200, the library's form);
     * 1 MPFLOW3D's matrix form Mop P dW (MPFLOW3D/src/Roe_Fluxes.cpp:1605-1683)
     * exactly as written, whose w-momentum diagonal reads E1 (1 - ny^2); 2 the
     * same matrix form with E1 (1 - nz^2) */
    int mpf_form;
    /* state variables: 0 conservative, 1 (rho, u, v, w, p) (MPFLOW3D VARIABLE_RUP) */
    int variables;
} orc_params;

typedef struct {
    int nnode, nghost, nedge, nbedge;
    const int *en;    /* [2*nedge]  L < R            */
    const double *ea; /* [3*nedge]  area L -> R      */
    const int *bn;    /* [2*nbedge] node, ghost      */
    const double *ba; /* [3*nbedge] outward area     */
    const int *bt;    /* [nbedge]   BC type          */
    const double *vol;/* [nnode]                     */
    const double *xyz;/* [3*nnode]  interleaved      */
    const int *ia, *ja; /* node graph, no diagonal   */
} orc_mesh;

/* far field {rho,u,v,w,et,p,c,mach} */
void orc_farfield(const orc_params *p, double out[8]);
void orc_apply_bc(const orc_mesh *m, const orc_params *p, double *Q);
void orc_gradient_lsq(const orc_mesh *m, const orc_params *p, const double *Q, double *grad);
void orc_gradient_gg(const orc_mesh *m, const double *Q, double *grad);
void orc_limiter(const orc_mesh *m, const orc_params *p, const double *Q, const double *grad, double *phi);
/* conv/diss [5][nnode], dtsum [nnode], ext {min1,max1,min4,max4,min5,max5} */
void orc_residual(const orc_mesh *m, const orc_params *p, const double *Q, const double *grad, const double *phi,
                  double *conv, double *diss, double *dtsum, double ext[6]);
/* dt: in = sum(area*lambda), out = time step; ext2 {min, max} */
void orc_deltat(const orc_mesh *m, const orc_params *p, double *dt, double ext2[2]);
/* block CRS pattern; returns nnzb (arrays may be NULL to query) */
long orc_block_pattern(const orc_mesh *m, int *IA, int *JA, int *IAU);
void orc_jacobian(const orc_mesh *m, const orc_params *p, const double *Q, const double *dt, const double *conv,
                  const double *diss, int add_time, int include_diss, const int *IA, const int *JA, const int *IAU,
                  double *A, double *B);
double orc_block_gs(int n, const int *IA, const int *JA, const int *IAU, const double *A, const double *B, double *X,
                    int iters, int direction);
int orc_ilu0(int n, const int *IA, const int *JA, const int *IAU, const double *A, double *F);
void orc_ilu0_apply(int n, const int *IA, const int *JA, const int *IAU, const double *F, const double *r,
                    double *z);
int orc_gmres(int n, const int *IA, const int *JA, const int *IAU, const double *A, const double *B, double *X,
              int m, int maxit, double rtol, int precond, int *iters, double *relres);
double orc_block_lusgs(int n, const int *IA, const int *JA, const int *IAU, const double *A, const double *B,
                       double *X, int iters);
void orc_bspmv(int n, const int *IA, const int *JA, const double *A, const double *x, double *y);

#endif
