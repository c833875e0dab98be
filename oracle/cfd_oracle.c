/* CPU restatement of the reference's implicit edge-based FV hot path.
 * TEST INFRASTRUCTURE ONLY -- the checker of the CUDA path, never part of the
 * product.  See cfd_oracle.h.  Every routine cites the reference lines it
 * restates (paths relative to the reference's Trunk/).
 */
#include "cfd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(v, i, ld) ((size_t)(v) * (size_t)(ld) + (size_t)(i))

static double dmin(double a, double b) { return a < b ? a : b; }
static double dmax(double a, double b) { return a > b ? a : b; }

/* Vector3D::normalize / magnitude (MATH/src/Vector3D.cpp:216-229) */
static void unit(const double *a, double *n, double *mag) {
    double m = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    n[0] = a[0]; n[1] = a[1]; n[2] = a[2];
    if (m > 1.0e-20) { n[0] = a[0] / m; n[1] = a[1] / m; n[2] = a[2] / m; }
    *mag = m;
}

/* ComputeFarFieldCondition, generic non-dimensionalisation
 * (Euler3D/src/Material.cpp:112-210). */
void orc_farfield(const orc_params *p, double out[8]) {
    double R = 1.0 / p->gamma, rho = 1.0, T = p->gamma, pr = R * rho * T;
    double a = p->alpha_deg * M_PI / 180.0, b = p->beta_deg * M_PI / 180.0;
    /* stiffened gas: c^2 = gamma (p + pinf) / rho, rho e = (p + gamma pinf) / (gamma - 1) */
    double c = p->pinf != 0.0 ? sqrt(p->gamma * (pr + p->pinf) / rho) : sqrt(p->gamma * R * T);
    double u = p->mach * c * cos(a) * cos(b), v = p->mach * c * sin(a), w = p->mach * c * sin(b) * cos(a);
    double q2 = u * u + v * v + w * w;
    out[0] = rho; out[1] = u; out[2] = v; out[3] = w;
    out[4] = (pr + p->gamma * p->pinf) / ((p->gamma - 1.0) * rho) + 0.5 * q2;
    out[5] = pr; out[6] = c; out[7] = p->mach;
}

typedef struct { double rho, u, v, w, et, p, ht, ubar, c; } face_t;

/* Compute_EOS_Variables_Face, conservative branch (Material.cpp:216-248),
 * extended to the stiffened gas p = (g - 1) rho e - g pinf, c^2 = g (p + pinf) / rho
 * (pinf = 0: the reference's ideal gas).  With p->variables == 1 the state is
 * (rho, u, v, w, p), taken as stored (MPFLOW3D Material_Get_Properties,
 * VARIABLE_RUP, MPFLOW3D/src/Material.cpp:591-599). */
static void eos_face(const double *q, double nx, double ny, double nz, const orc_params *p, face_t *s) {
    double g = p->gamma, pinf = p->pinf;
    s->rho = q[0];
    if (p->variables == 1) {
        s->u = q[1]; s->v = q[2]; s->w = q[3]; s->p = q[4];
        double q2 = s->u * s->u + s->v * s->v + s->w * s->w;
        s->et = (s->p + g * pinf) / ((g - 1.0) * s->rho) + 0.5 * q2;
        s->ht = s->et + s->p / s->rho;
        s->c = sqrt((g * (s->p + pinf)) / s->rho);
        s->ubar = s->u * nx + s->v * ny + s->w * nz;
        return;
    }
    s->u = q[1] / s->rho;
    s->v = q[2] / s->rho;
    s->w = q[3] / s->rho;
    s->et = q[4] / s->rho;
    double q2 = s->u * s->u + s->v * s->v + s->w * s->w;
    s->p = (g - 1.0) * (s->rho * s->et - 0.5 * s->rho * q2) - g * pinf;
    s->ht = (s->rho * s->et + s->p) / s->rho;
    s->c = sqrt((g * (s->p + pinf)) / s->rho);
    s->ubar = s->u * nx + s->v * ny + s->w * nz;
}

/* A ghost state from (rho, u, v, w, p) in the state's variables (Get_TotalEnergy,
 * Material.cpp:1012-1040, for conservative states). */
static void put_state(double rb, double ub, double vb, double wb, double pb, const orc_params *p, double *qB) {
    if (p->variables == 1) { qB[0] = rb; qB[1] = ub; qB[2] = vb; qB[3] = wb; qB[4] = pb; return; }
    double et = ub * ub + vb * vb + wb * wb;
    et = (pb + p->gamma * p->pinf) / ((p->gamma - 1.0) * rb) + 0.5 * et;
    qB[0] = rb; qB[1] = rb * ub; qB[2] = rb * vb; qB[3] = rb * wb; qB[4] = rb * et;
}

/* ---- Low-Mach preconditioned Roe of the Turkel family (MPFLOW3D) ----------
 * Compute_Flux_Roe_Precondition_Turkel (MPFLOW3D/src/Roe_Fluxes.cpp:2043-2526):
 * preconditioner K in (rho, u, v, w, p) with parameters alpha, delta and
 * beta = Mr^2 (BTW: alpha 0, delta 1; Eriksson: alpha 0, delta beta; Turkel:
 * alpha 0.4, delta beta), dissipation Mop Kinv R |Lambda| L Mpr dQ with the
 * eigenvalues |u.n|, |u'.n +- c'| of K A, the Roe average, the solution in
 * conservative variables and the pressure smoothing off (PRECOND_SMOOTH NO). */
typedef struct {
    double L[5][5], R[5][5], lam[5], kc[5]; /* left/right eigenvectors, |eigenvalues|, Kinv column 4 */
    double ubar, ubp, cp;
} pc_sys_t;

/* beta (squared) of PRECOND_TYPE LOCAL (0) / GLOBAL (1) / URLOCAL (2) (Roe_Fluxes.cpp:2225-2248). */
static double pc_beta(const orc_params *p, double mach, double mach_max) {
    double b = 1.0;
    if (p->pc_type == 0) {
        double M = dmax(mach, mach_max), G = p->pc_mach;
        b = M < G ? 0.5 * (M * M) / (G * G) - M / G + 1.0 : 0.5;
        b = dmin(1.0, b * (sqrt(M * G) + M));
    } else if (p->pc_type == 2) {
        b = dmin(1.0, mach);
    } else {
        b = dmin(1.0, p->pc_mach);
    }
    return b * b;
}

static void pc_params(const orc_params *p, double beta, double *alpha, double *delta) {
    *alpha = p->pc_method == 5 ? 0.4 : 0.0;
    *delta = p->pc_method == 2 ? 1.0 : beta;
}

/* Eigen-system of K A in (rho, u, v, w, p) at (rho, u, v, w, c), normal n
 * (Roe_Fluxes.cpp:2266-2400; BC.cpp:260-305). */
static void pc_system(double rho, double u, double v, double w, double c, const double *n, double beta, double alpha,
                      double delta, pc_sys_t *S) {
    double nx = n[0], ny = n[1], nz = n[2];
    double ubar = u * nx + v * ny + w * nz, c2 = c * c, bc2 = beta * c2;
    double zp = 0.5 * (1.0 + beta - alpha), zm = 0.5 * (1.0 - beta + alpha);
    double ubp = zp * ubar, cp = sqrt(beta * (c2 - ubar * ubar) + zp * zp * ubar * ubar);
    double pv1 = rho * (beta - delta), pv2 = pv1 * ubar, pv3 = bc2 - alpha * ubar * ubar;
    double pv4 = (bc2 * (cp + ubar * zm)) / (2.0 * cp * pv3), pv5 = (bc2 * (cp - ubar * zm)) / (2.0 * cp * pv3);
    S->ubar = ubar; S->ubp = ubp; S->cp = cp;
    S->lam[0] = S->lam[1] = S->lam[2] = fabs(ubar);
    S->lam[3] = fabs(ubp + cp);
    S->lam[4] = fabs(ubp - cp);
    /* left eigenvectors (rows) */
    double (*L)[5] = S->L;
    L[0][0] = nx;
    L[0][1] = nx * ubar * (alpha * (v * nz - w * ny) + pv1 * nx) / pv3;
    L[0][2] = (bc2 * nz - alpha * ubar * (w * ny * ny + u * nx * nz + w * nz * nz) + pv2 * nx * ny) / pv3;
    L[0][3] = (-bc2 * ny + alpha * ubar * (v * ny * ny + u * nx * ny + v * nz * nz) + pv2 * nx * nz) / pv3;
    L[0][4] = (-rho * delta * c2 * nx + alpha * c2 * (v * nz - w * ny) + alpha * rho * ubar * ubar * nx) / (rho * c2 * pv3);
    L[1][0] = ny;
    L[1][1] = (-bc2 * nz + alpha * ubar * (w * nx * nx + v * ny * nz + w * nz * nz) + pv2 * nx * ny) / pv3;
    L[1][2] = ny * ubar * (alpha * (w * nx - u * nz) + pv1 * ny) / pv3;
    L[1][3] = (bc2 * nx - alpha * ubar * (u * nx * nx + v * nx * ny + u * nz * nz) + pv2 * ny * nz) / pv3;
    L[1][4] = (-rho * delta * c2 * ny + alpha * c2 * (w * nx - u * nz) + alpha * rho * ubar * ubar * ny) / (rho * c2 * pv3);
    L[2][0] = nz;
    L[2][1] = (bc2 * ny - alpha * ubar * (v * nx * nx + w * ny * nz + v * ny * ny) + pv2 * nx * nz) / pv3;
    L[2][2] = (-bc2 * nx + alpha * ubar * (u * nx * nx + w * nx * nz + u * ny * ny) + pv2 * ny * nz) / pv3;
    L[2][3] = nz * ubar * (alpha * (u * ny - v * nx) + pv1 * nz) / pv3;
    L[2][4] = (-rho * delta * c2 * nz + alpha * c2 * (u * ny - v * nx) + alpha * rho * ubar * ubar * nz) / (rho * c2 * pv3);
    L[3][0] = 0.0; L[3][1] = pv4 * nx; L[3][2] = pv4 * ny; L[3][3] = pv4 * nz;
    L[3][4] = (bc2 + alpha * ubar * (cp - ubar * zp)) / (2.0 * rho * cp * pv3);
    L[4][0] = 0.0; L[4][1] = -pv5 * nx; L[4][2] = -pv5 * ny; L[4][3] = -pv5 * nz;
    L[4][4] = (bc2 - alpha * ubar * (cp + ubar * zp)) / (2.0 * rho * cp * pv3);
    /* right eigenvectors (columns) */
    double (*R)[5] = S->R;
    R[0][0] = nx; R[0][1] = ny; R[0][2] = nz;
    R[0][3] = rho * ((zp * delta - beta) * ubar + cp * delta) / bc2;
    R[0][4] = -rho * ((zp * delta - beta) * ubar - cp * delta) / bc2;
    R[1][0] = 0.0; R[1][1] = -nz; R[1][2] = ny;
    R[1][3] = nx - alpha * u * (cp + zp * ubar) / bc2;
    R[1][4] = -nx - alpha * u * (cp - zp * ubar) / bc2;
    R[2][0] = nz; R[2][1] = 0.0; R[2][2] = -nx;
    R[2][3] = ny - alpha * v * (cp + zp * ubar) / bc2;
    R[2][4] = -ny - alpha * v * (cp - zp * ubar) / bc2;
    R[3][0] = -ny; R[3][1] = nx; R[3][2] = 0.0;
    R[3][3] = nz - alpha * w * (cp + zp * ubar) / bc2;
    R[3][4] = -nz - alpha * w * (cp - zp * ubar) / bc2;
    R[4][0] = 0.0; R[4][1] = 0.0; R[4][2] = 0.0;
    R[4][3] = rho * (cp - zm * ubar);
    R[4][4] = rho * (cp + zm * ubar);
    /* Kinv = I except column 4 */
    S->kc[0] = (1.0 - delta) / bc2;
    S->kc[1] = (alpha * u) / (beta * rho * c2);
    S->kc[2] = (alpha * v) / (beta * rho * c2);
    S->kc[3] = (alpha * w) / (beta * rho * c2);
    S->kc[4] = 1.0 / beta;
}

/* Mpr = d(rho, u, v, w, p) / dQ_cons and Mop = dQ_cons / d(rho, u, v, w, p) at
 * (rho, u, v, w) (Material_Get_Transformation_Matrix; the stiffened gas has
 * the same derivatives as the ideal gas). */
static void pc_transforms(double rho, double u, double v, double w, double g, double Mpr[5][5], double Mop[5][5]) {
    double q2 = u * u + v * v + w * w, g1 = g - 1.0;
    double a[5][5] = {{1, 0, 0, 0, 0}, {-u / rho, 1.0 / rho, 0, 0, 0}, {-v / rho, 0, 1.0 / rho, 0, 0},
                      {-w / rho, 0, 0, 1.0 / rho, 0}, {0.5 * g1 * q2, -g1 * u, -g1 * v, -g1 * w, g1}};
    double b[5][5] = {{1, 0, 0, 0, 0}, {u, rho, 0, 0, 0}, {v, 0, rho, 0, 0}, {w, 0, 0, rho, 0},
                      {0.5 * q2, rho * u, rho * v, rho * w, 1.0 / g1}};
    memcpy(Mpr, a, sizeof a);
    memcpy(Mop, b, sizeof b);
}

static void mm5g(double A[5][5], double B[5][5], double C[5][5]) {
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            C[i][j] = 0.0;
            for (int k = 0; k < 5; k++) C[i][j] += A[i][k] * B[k][j];
        }
}

/* The edge's averaged state and eigen-system (first-order states or
 * reconstructed face states); returns the spectral radius. */
static double pc_edge(const double *qL, const double *qR, const double *n, const orc_params *p, face_t *Lf, face_t *Rf,
                      double avg[4], pc_sys_t *S) {
    double g = p->gamma;
    eos_face(qL, n[0], n[1], n[2], p, Lf);
    eos_face(qR, n[0], n[1], n[2], p, Rf);
    double rho, u, v, w, ht, c;
    if (p->pc_avg == 1) { /* simple mean, |c^2| (Euler3D FluxTest.cpp:3927-3940) */
        rho = 0.5 * (Rf->rho + Lf->rho);
        u = 0.5 * (Rf->u + Lf->u); v = 0.5 * (Rf->v + Lf->v); w = 0.5 * (Rf->w + Lf->w);
        ht = 0.5 * (Rf->ht + Lf->ht);
        c = sqrt(fabs((g - 1.0) * (ht - 0.5 * (u * u + v * v + w * w))));
    } else {
        double sigma;
        rho = sqrt(Rf->rho * Lf->rho), sigma = rho / (Lf->rho + rho);
        u = Lf->u + sigma * (Rf->u - Lf->u), v = Lf->v + sigma * (Rf->v - Lf->v), w = Lf->w + sigma * (Rf->w - Lf->w);
        ht = Lf->ht + sigma * (Rf->ht - Lf->ht);
        c = sqrt((g - 1.0) * (ht - 0.5 * (u * u + v * v + w * w))); /* Material_Get_DH_SpeedSound: c^2 = (g - 1) h */
    }
    double q2 = u * u + v * v + w * w;
    double mach = sqrt(q2) / c;
    double mL = sqrt(Lf->u * Lf->u + Lf->v * Lf->v + Lf->w * Lf->w) / Lf->c;
    double mR = sqrt(Rf->u * Rf->u + Rf->v * Rf->v + Rf->w * Rf->w) / Rf->c;
    double beta = pc_beta(p, mach, dmax(mL, mR)), alpha, delta;
    pc_params(p, beta, &alpha, &delta);
    pc_system(rho, u, v, w, c, n, beta, alpha, delta, S);
    avg[0] = rho; avg[1] = u; avg[2] = v; avg[3] = w;
    return dmax(S->lam[0], dmax(S->lam[3], S->lam[4]));
}

/* |A|_p = Mop Kinv R |Lambda| L Mpr (Compute_Dissipation_Matrix_Roe_Precondition_Turkel,
 * Roe_Fluxes.cpp:3440-3810). */
static void pc_absA(const pc_sys_t *S, const double avg[4], const orc_params *p, double A[5][5]) {
    double Mpr[5][5], Mop[5][5], T[5][5], U[5][5], V[5][5];
    pc_transforms(avg[0], avg[1], avg[2], avg[3], p->gamma, Mpr, Mop);
    if (p->variables == 1) /* the state's own (rho, u, v, w, p): Mpr = I */
        for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++) Mpr[i][j] = i == j ? 1.0 : 0.0;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) U[i][j] = S->lam[i] * S->L[i][j];       /* |Lambda| L */
    mm5g((double (*)[5])S->R, U, T);                                       /* R |Lambda| L */
    for (int j = 0; j < 5; j++) {                                          /* Kinv (R |Lambda| L) */
        double t4 = T[4][j];
        for (int i = 0; i < 5; i++) V[i][j] = (i == 4 ? 0.0 : T[i][j]) + S->kc[i] * t4;
    }
    mm5g(Mop, V, T);
    mm5g(T, Mpr, A);
}

static double roe_pc(const double *qL, const double *qR, const double *n, double area, const orc_params *p,
                     double *conv, double *diss, double lam[3]) {
    face_t L, R;
    pc_sys_t S;
    double avg[4], A[5][5];
    double lmax = pc_edge(qL, qR, n, p, &L, &R, avg, &S);
    double mL = L.rho * L.ubar, mR = R.rho * R.ubar;
    double FL[5] = {mL, L.u * mL + L.p * n[0], L.v * mL + L.p * n[1], L.w * mL + L.p * n[2], L.ht * mL};
    double FR[5] = {mR, R.u * mR + R.p * n[0], R.v * mR + R.p * n[1], R.w * mR + R.p * n[2], R.ht * mR};
    pc_absA(&S, avg, p, A);
    for (int i = 0; i < 5; i++) {
        double fa = 0.0;
        for (int j = 0; j < 5; j++) fa += A[i][j] * (qR[j] - qL[j]);
        conv[i] = 0.5 * (FL[i] + FR[i]) * area;
        diss[i] = -0.5 * fa * area;
    }
    lam[0] = S.lam[0]; lam[1] = S.lam[3]; lam[2] = S.lam[4];
    return lmax;
}

/* Cinv = Mop Kinv Mpr at a node (Compute_Transformed_Preconditioner_Matrix_Roe_Turkel
 * with reqInv, Roe_Fluxes.cpp:261-441): the pseudo-time term of the Jacobian. */
static void pc_node_cinv(const double *q, const orc_params *p, double C[5][5]) {
    face_t F;
    double n0[3] = {1.0, 0.0, 0.0};
    eos_face(q, n0[0], n0[1], n0[2], p, &F);
    double mach = sqrt(F.u * F.u + F.v * F.v + F.w * F.w) / F.c;
    double beta = pc_beta(p, mach, 0.0), alpha, delta;
    pc_params(p, beta, &alpha, &delta);
    double c2 = F.c * F.c, kc[5] = {(1.0 - delta) / (beta * c2), (alpha * F.u) / (beta * F.rho * c2),
                                    (alpha * F.v) / (beta * F.rho * c2), (alpha * F.w) / (beta * F.rho * c2), 1.0 / beta};
    double Mpr[5][5], Mop[5][5], K[5][5] = {{0}}, T[5][5];
    pc_transforms(F.rho, F.u, F.v, F.w, p->gamma, Mpr, Mop);
    if (p->variables == 1)
        for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++) Mpr[i][j] = i == j ? 1.0 : 0.0;
    for (int i = 0; i < 5; i++) { K[i][i] = i == 4 ? 0.0 : 1.0; K[i][4] += kc[i]; }
    mm5g(Mop, K, T);
    mm5g(T, Mpr, C);
}

/* Gaussian elimination with partial pivoting on a 5x5 system (the
 * GaussainLUDecompose + pivoted substitutions the preconditioned BC uses). */
static void solve5(double A[5][5], const double *b, double *x) {
    double M[5][6];
    for (int i = 0; i < 5; i++) { for (int j = 0; j < 5; j++) M[i][j] = A[i][j]; M[i][5] = b[i]; }
    for (int c = 0; c < 5; c++) {
        int pi = c;
        for (int i = c + 1; i < 5; i++) if (fabs(M[i][c]) > fabs(M[pi][c])) pi = i;
        if (pi != c) for (int j = 0; j < 6; j++) { double t = M[c][j]; M[c][j] = M[pi][j]; M[pi][j] = t; }
        for (int i = c + 1; i < 5; i++) {
            double f = M[i][c] / M[c][c];
            for (int j = c; j < 6; j++) M[i][j] -= f * M[c][j];
        }
    }
    for (int i = 4; i >= 0; i--) {
        double t = M[i][5];
        for (int j = i + 1; j < 5; j++) t -= M[i][j] * x[j];
        x[i] = t / M[i][i];
    }
}

static void lmul5(double L[5][5], const double *q, double *out) {
    for (int i = 0; i < 5; i++) {
        out[i] = 0.0;
        for (int j = 0; j < 5; j++) out[i] += L[i][j] * q[j];
    }
}

/* Ghost state of Compute_Precondition_Characteristic_BoundaryCondition_Turkel
 * (MPFLOW3D/src/BC.cpp:113-700), BC_METHOD_CHARCTERISTIC, in (rho, u, v, w, p)
 * through the preconditioned characteristic variables L q.  The subsonic
 * outflow imposes p->outflow_p (the freestream pressure when 0). */
static int bc_state_pc(const double *qI, const double *qG, const double *areav, int type, const orc_params *p,
                       const double *inf, double *qB) {
    double n[3], mag;
    unit(areav, n, &mag);
    face_t I, G, O;
    double q0[5];
    eos_face(qI, n[0], n[1], n[2], p, &I);
    eos_face(qG, n[0], n[1], n[2], p, &G);
    for (int k = 0; k < 5; k++) q0[k] = 0.5 * (qI[k] + qG[k]);
    eos_face(q0, n[0], n[1], n[2], p, &O);
    double mach = sqrt(O.u * O.u + O.v * O.v + O.w * O.w) / O.c;
    double mI = sqrt(I.u * I.u + I.v * I.v + I.w * I.w) / I.c, mG = sqrt(G.u * G.u + G.v * G.v + G.w * G.w) / G.c;
    double beta = pc_beta(p, mach, dmax(mI, mG)), alpha, delta;
    pc_params(p, beta, &alpha, &delta);
    pc_sys_t S;
    pc_system(O.rho, O.u, O.v, O.w, O.c, n, beta, alpha, delta, &S);
    double l1 = S.ubar, l4 = S.ubp + S.cp, l5 = S.ubp - S.cp;
    int inst = -1, st = 0;
    switch (type) {
        case 0: inst = 0; break;
        case 1:
            if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 10;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 11;
            else if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 9;
            else if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 8;
            else { inst = 1; st = 2; }
            break;
        case 2:
            if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 4;
            else if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 6;
            else inst = fabs(l1) < O.c ? 4 : 6;
            break;
        case 3:
            if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 5;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 7;
            else inst = fabs(l1) < O.c ? 5 : 7;
            break;
        default: inst = type; break;
    }
    double qi[5] = {I.rho, I.u, I.v, I.w, I.p}, qinf[5] = {inf[0], inf[1], inf[2], inf[3], inf[5]};
    double B[5], X[5], xb[5] = {inf[0], inf[1], inf[2], inf[3], inf[5]};
    double outp = p->outflow_p != 0.0 ? p->outflow_p : inf[5];
    switch (inst) {
        case 0: /* wall: four characteristics from inside, zero normal velocity */
            lmul5(S.L, qi, B);
            B[4] = 0.0;
            S.L[4][0] = 0.0; S.L[4][1] = n[0]; S.L[4][2] = n[1]; S.L[4][3] = n[2]; S.L[4][4] = 0.0;
            solve5(S.L, B, xb);
            if (p->iteration < p->zpg_iteration && xb[4] + p->pinf < 0.0) {
                xb[0] = I.rho; xb[4] = I.p;
                xb[1] = I.u - n[0] * I.ubar; xb[2] = I.v - n[1] * I.ubar; xb[3] = I.w - n[2] * I.ubar;
            }
            if (xb[4] + p->pinf < 0.0) st = st ? st : 1;
            break;
        case 4: case 8: { /* subsonic inflow: the u.n + c characteristic from inside */
            double qe[5] = {qinf[0], qinf[1], qinf[2], qinf[3], inst == 4 ? I.p : qinf[4]};
            lmul5(S.L, qe, B);
            lmul5(S.L, qi, X);
            B[3] = X[3];
            solve5(S.L, B, xb);
        } break;
        case 5: /* subsonic outflow: pressure imposed */
            lmul5(S.L, qi, B);
            for (int j = 0; j < 4; j++) S.L[4][j] = 0.0;
            S.L[4][4] = 1.0;
            B[4] = outp;
            solve5(S.L, B, xb);
            break;
        case 9: /* far-field subsonic outflow: the u.n - c characteristic from outside */
            lmul5(S.L, qi, B);
            lmul5(S.L, qinf, X);
            B[4] = X[4];
            solve5(S.L, B, xb);
            break;
        case 7: case 11:
            for (int k = 0; k < 5; k++) xb[k] = qi[k];
            break;
        default: break; /* 1, 6, 10: freestream */
    }
    put_state(xb[0], xb[1], xb[2], xb[3], xb[4], p, qB);
    return st;
}

/* Characteristic BC ghost state (Compute_Characteristic_BoundaryCondition_New,
 * Euler3D/src/BC.cpp:381-677), conservative variables.  Returns nonzero where
 * the reference would abort. */
static int bc_state(const double *qI, const double *qG, const double *areav, int type, const orc_params *p,
                    const double *inf, double *qB) {
    double n[3], mag;
    unit(areav, n, &mag);
    face_t I, G, O;
    double q0[5];
    eos_face(qI, n[0], n[1], n[2], p, &I);
    eos_face(qG, n[0], n[1], n[2], p, &G);
    for (int k = 0; k < 5; k++) q0[k] = 0.5 * (qI[k] + qG[k]);
    eos_face(q0, n[0], n[1], n[2], p, &O);
    double l1 = O.ubar, l4 = l1 + O.c, l5 = l1 - O.c;
    double pb = inf[5], rb = inf[0], ub = inf[1], vb = inf[2], wb = inf[3];
    double outflow_p = 0.935 * inf[5];
    int inst = -1, st = 0;
    switch (type) {
        case 0: inst = 0; break;
        case 1:
            if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 10;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 11;
            else if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 9;
            else if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 8;
            else st = 2;
            break;
        case 2:
            if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 4;
            else if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 6;
            else inst = fabs(l1) < O.c ? 4 : 6;
            break;
        case 3:
            if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 5;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 7;
            else inst = fabs(l1) < O.c ? 5 : 7;
            break;
        default: inst = type; break;
    }
    /* the preconditioned characteristic BC used with the low-Mach fix keeps the
     * freestream at subsonic and supersonic outflow (BC.cpp:1229-1236) */
    if (p->flux == 3 && (inst == 5 || inst == 7)) inst = 4;
    switch (inst) {
        case 0:
            pb = I.p + O.rho * O.c * I.ubar;
            if (p->iteration < p->zpg_iteration && pb + p->pinf < 0.0) pb = I.p;
            rb = I.rho + (pb - I.p) / (O.c * O.c);
            ub = I.u - n[0] * (pb - I.p) / (O.rho * O.c);
            vb = I.v - n[1] * (pb - I.p) / (O.rho * O.c);
            wb = I.w - n[2] * (pb - I.p) / (O.rho * O.c);
            break;
        case 5: case 9:
            pb = inst == 5 ? outflow_p : inf[5];
            rb = I.rho + (pb - I.p) / (O.c * O.c);
            ub = I.u - n[0] * (pb - I.p) / (O.rho * O.c);
            vb = I.v - n[1] * (pb - I.p) / (O.rho * O.c);
            wb = I.w - n[2] * (pb - I.p) / (O.rho * O.c);
            break;
        case 7: case 11:
            pb = I.p; rb = I.rho; ub = I.u; vb = I.v; wb = I.w;
            break;
        case 8: {
            double t = n[0] * (inf[1] - I.u) + n[1] * (inf[2] - I.v) + n[2] * (inf[3] - I.w);
            pb = 0.5 * (inf[5] + I.p - O.rho * O.c * t);
            rb = inf[0] + (pb - inf[5]) / (O.c * O.c);
            ub = inf[1] + n[0] * (pb - inf[5]) / (O.rho * O.c);
            vb = inf[2] + n[1] * (pb - inf[5]) / (O.rho * O.c);
            wb = inf[3] + n[2] * (pb - inf[5]) / (O.rho * O.c);
        } break;
        default: break;
    }
    if (pb + p->pinf < 0.0) st = st ? st : 1;
    put_state(rb, ub, vb, wb, pb, p, qB);
    return st;
}

/* Apply_Characteristic_Boundary_Condition (BC.cpp:1440-1487). */
void orc_apply_bc(const orc_mesh *m, const orc_params *p, double *Q) {
    const int ld = m->nnode + m->nghost;
    double inf[8];
    orc_farfield(p, inf);
    for (int b = 0; b < m->nbedge; b++) {
        int L = m->bn[2 * b], R = m->bn[2 * b + 1];
        double qI[5], qG[5], qB[5];
        for (int k = 0; k < 5; k++) { qI[k] = Q[IDX(k, L, ld)]; qG[k] = Q[IDX(k, R, ld)]; }
        if (p->flux == 4) bc_state_pc(qI, qG, m->ba + 3 * (size_t)b, m->bt[b], p, inf, qB);
        else bc_state(qI, qG, m->ba + 3 * (size_t)b, m->bt[b], p, inf, qB);
        for (int k = 0; k < 5; k++) Q[IDX(k, R, ld)] = qB[k];
    }
}

/* Roe_EntropyFix (Euler3D/src/Roe_EntropyFix.cpp:19-59). */
static void entropy_fix(double ubL, double cL, double ubR, double cR, double ub, double c, double E[3]) {
    E[0] = fabs(ub);
    double lL = ubL + cL, lR = ubR + cR, l = ub + c;
    double eps = 4.0 * dmax(0.0, dmax(l - lL, lR - l));
    E[1] = fabs(l) < eps ? (l * l + eps * eps) / (2.0 * eps) : fabs(l);
    lL = ubL - cL; lR = ubR - cR; l = ub - c;
    eps = 4.0 * dmax(0.0, dmax(l - lL, lR - l));
    E[2] = fabs(l) < eps ? (l * l + eps * eps) / (2.0 * eps) : fabs(l);
}

/* Thornber modification (Compute_Flux_Roe_Thornber, MPFLOW3D/src/Roe_Fluxes.cpp:1141-1165,
 * conservative variables): z = min(1, max(M_L, M_R)); u_L' = ((1+z) u_L + (1-z) u_R)/2,
 * u_R' symmetric; density and total energy unchanged. */
static void thornber(const double *qL, const double *qR, const orc_params *p, double *mL, double *mR) {
    face_t L, R;
    eos_face(qL, 1.0, 0.0, 0.0, p, &L);
    eos_face(qR, 1.0, 0.0, 0.0, p, &R);
    double z = dmin(1.0, dmax(sqrt(L.u * L.u + L.v * L.v + L.w * L.w) / L.c,
                              sqrt(R.u * R.u + R.v * R.v + R.w * R.w) / R.c));
    mL[0] = qL[0]; mR[0] = qR[0]; mL[4] = qL[4]; mR[4] = qR[4];
    if (p->variables == 1) { /* velocities blended at fixed rho and p (MPFLOW3D Roe_Fluxes.cpp:1161-1168) */
        for (int i = 1; i < 4; i++) {
            double t1 = 0.5 * ((1.0 + z) * qL[i] + (1.0 - z) * qR[i]);
            double t2 = 0.5 * ((1.0 + z) * qR[i] + (1.0 - z) * qL[i]);
            mL[i] = t1;
            mR[i] = t2;
        }
        return;
    }
    for (int i = 1; i < 4; i++) {
        double t1 = 0.5 * ((1.0 + z) * qL[i] / qL[0] + (1.0 - z) * qR[i] / qR[0]);
        double t2 = 0.5 * ((1.0 + z) * qR[i] / qR[0] + (1.0 - z) * qL[i] / qL[0]);
        mL[i] = qL[0] * t1;
        mR[i] = qR[0] * t2;
    }
}

/* Compute_Flux_Roe_Optimized (Euler3D/src/FluxTest.cpp:3026-3200). */
static double roe(const double *qL, const double *qR, const double *n, double area, const orc_params *p,
                  double *conv, double *diss, double lam[3]) {
    face_t L, R;
    double g = p->gamma;
    eos_face(qL, n[0], n[1], n[2], p, &L);
    eos_face(qR, n[0], n[1], n[2], p, &R);
    double FL[5], FR[5];
    FL[0] = L.rho * L.ubar; FL[1] = L.u * FL[0] + L.p * n[0]; FL[2] = L.v * FL[0] + L.p * n[1];
    FL[3] = L.w * FL[0] + L.p * n[2]; FL[4] = L.ht * FL[0];
    FR[0] = R.rho * R.ubar; FR[1] = R.u * FR[0] + R.p * n[0]; FR[2] = R.v * FR[0] + R.p * n[1];
    FR[3] = R.w * FR[0] + R.p * n[2]; FR[4] = R.ht * FR[0];
    double rho = sqrt(R.rho * L.rho), sigma = rho / (L.rho + rho);
    double u = L.u + sigma * (R.u - L.u), v = L.v + sigma * (R.v - L.v), w = L.w + sigma * (R.w - L.w);
    double ht = L.ht + sigma * (R.ht - L.ht);
    double phi = 0.5 * (g - 1.0) * (u * u + v * v + w * w);
    double c = sqrt((g - 1.0) * ht - phi);   /* Get_SpeedSound, Material.cpp:939-960 */
    double ub = u * n[0] + v * n[1] + w * n[2];
    double E[3];
    if (p->entropy_fix) entropy_fix(L.ubar, L.c, R.ubar, R.c, ub, c, E);
    else { E[0] = fabs(ub); E[1] = fabs(ub + c); E[2] = fabs(ub - c); }
    lam[0] = E[0]; lam[1] = E[1]; lam[2] = E[2];
    /* M = dQ/dq_RUP (Compute_Transformation_Conservative_To_RUP, Material.cpp:1172-1236) */
    double M[5][5] = {{1, 0, 0, 0, 0}, {u, rho, 0, 0, 0}, {v, 0, rho, 0, 0}, {w, 0, 0, rho, 0},
                      {phi / (g - 1.0), rho * u, rho * v, rho * w, 1.0 / (g - 1.0)}};
    double dQ[5] = {R.rho - L.rho, R.u - L.u, R.v - L.v, R.w - L.w, R.p - L.p};
    double E0 = E[0], E1 = E[1], E2 = E[2];
    double dU = dQ[1] * n[0] + dQ[2] * n[1] + dQ[3] * n[2];
    if (p->flux == 3) {
        /* low-Mach fix (Compute_Flux_Roe_LMFIX, FluxTest.cpp:2943-3005): the normal velocity
         * jump times min(1, (|u.n| + |u.t1| + |u.t2|) / c); t1 in the face plane from the
         * largest normal component, t2 = t1 x n, both normalised */
        double nmax = fabs(n[0]), t1[3] = {1.0, 1.0, 1.0}, t2[3];
        int mc = 0;
        if (nmax < fabs(n[1])) { nmax = fabs(n[1]); mc = 1; }
        if (nmax < fabs(n[2])) { nmax = fabs(n[2]); mc = 2; }
        t1[mc] = -(n[(mc + 1) % 3] + n[(mc + 2) % 3]) / n[mc];
        double m1 = sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
        if (m1 > 1.0e-20) for (int k = 0; k < 3; k++) t1[k] /= m1;
        t2[0] = t1[1] * n[2] - t1[2] * n[1];
        t2[1] = -t1[0] * n[2] + t1[2] * n[0];
        t2[2] = t1[0] * n[1] - t1[1] * n[0];
        double m2 = sqrt(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
        if (m2 > 1.0e-20) for (int k = 0; k < 3; k++) t2[k] /= m2;
        double mach = (fabs(ub) + fabs(u * t1[0] + v * t1[1] + w * t1[2]) + fabs(u * t2[0] + v * t2[1] + w * t2[2])) / c;
        dU = dmin(mach, 1.0) * dU;
    }
    if (p->mpf_form) {
        /* MPFLOW3D's matrix form (Roe_Fluxes.cpp:1598-1683, VARIABLE_RUP): |A| dQ =
         * (Mop P) dW with P = |A| in (rho, u, v, w, p), Mop at the Roe state and dW the
         * jump of (rho, u, v, w, p); E4 = |u.n + c|, E5 = |u.n - c| */
        double Em = E1 - E2, Ep = E1 + E2, c2 = c * c, P[5][5], T[5][5];
        double dd = p->mpf_form == 1 ? n[1] * n[1] : n[2] * n[2];
        P[0][0] = E0; P[0][1] = 0.5 * Em * rho * n[0] / c; P[0][2] = 0.5 * Em * rho * n[1] / c;
        P[0][3] = 0.5 * Em * rho * n[2] / c; P[0][4] = -E0 / c2 + 0.5 * Ep / c2;
        P[1][0] = 0.0; P[1][1] = E0 * (1.0 - n[0] * n[0]) + 0.5 * Ep * n[0] * n[0];
        P[1][2] = -E0 * n[0] * n[1] + 0.5 * Ep * n[0] * n[1]; P[1][3] = -E0 * n[0] * n[2] + 0.5 * Ep * n[0] * n[2];
        P[1][4] = 0.5 * Em * n[0] / (rho * c);
        P[2][0] = 0.0; P[2][1] = -E0 * n[0] * n[1] + 0.5 * Ep * n[1] * n[0];
        P[2][2] = E0 * (1.0 - n[1] * n[1]) + 0.5 * Ep * n[1] * n[1];
        P[2][3] = -E0 * n[1] * n[2] + 0.5 * Ep * n[1] * n[2]; P[2][4] = 0.5 * Em * n[1] / (rho * c);
        P[3][0] = 0.0; P[3][1] = -E0 * n[0] * n[2] + 0.5 * Ep * n[2] * n[0];
        P[3][2] = -E0 * n[1] * n[2] + 0.5 * Ep * n[2] * n[1];
        P[3][3] = E0 * (1.0 - dd) + 0.5 * Ep * n[2] * n[2]; P[3][4] = 0.5 * Em * n[2] / (rho * c);
        P[4][0] = 0.0; P[4][1] = 0.5 * Em * c * rho * n[0]; P[4][2] = 0.5 * Em * c * rho * n[1];
        P[4][3] = 0.5 * Em * c * rho * n[2]; P[4][4] = 0.0 + 0.5 * Ep;
        mm5g(M, P, T);
        for (int i = 0; i < 5; i++) {
            double fa = 0.0;
            for (int j = 0; j < 5; j++) fa += T[i][j] * dQ[j];
            conv[i] = 0.5 * (FL[i] + FR[i]) * area;
            diss[i] = -0.5 * fa * area;
        }
        return dmax(E0, dmax(E1, E2));
    }
    double dw[5];
    dw[0] = E0 * dQ[0] + (E1 + E2 - 2.0 * E0) * dQ[4] / (2.0 * c * c) + rho * (E1 - E2) * dU / (2.0 * c);
    for (int k = 1; k < 4; k++)
        dw[k] = E0 * dQ[k] + 0.5 * n[k - 1] * dU * ((E1 + E2) - 2.0 * E0) + n[k - 1] * (E1 - E2) * dQ[4] / (2.0 * rho * c);
    dw[4] = 0.5 * dQ[4] * (E1 + E2) + 0.5 * rho * c * dU * (E1 - E2);
    for (int i = 0; i < 5; i++) {
        double fa = 0.0;   /* MC_Matrix_Mul_Vector (MATH/src/MC_Iterative_Jacobi.c:174-187) */
        for (int j = 0; j < 5; j++) fa += M[i][j] * dw[j];
        conv[i] = 0.5 * (FL[i] + FR[i]) * area;
        diss[i] = -0.5 * fa * area;
    }
    return dmax(E0, dmax(E1, E2));
}

/* Compute_HLLCFlux (Euler3D/src/HLLC_Fluxes.cpp:143-326). */
static double hllc(const double *qL, const double *qR, const double *n, double area, const orc_params *p,
                   double *conv, double *diss) {
    face_t L, R;
    double g = p->gamma;
    eos_face(qL, n[0], n[1], n[2], p, &L);
    eos_face(qR, n[0], n[1], n[2], p, &R);
    double rho = sqrt(R.rho * L.rho), sigma = rho / (L.rho + rho);
    double u = L.u + sigma * (R.u - L.u), v = L.v + sigma * (R.v - L.v), w = L.w + sigma * (R.w - L.w);
    double ht = L.ht + sigma * (R.ht - L.ht);
    double phi = 0.5 * (g - 1.0) * (u * u + v * v + w * w);
    double c = sqrt((g - 1.0) * ht - phi);
    double ub = u * n[0] + v * n[1] + w * n[2];
    double lmax = dmax(fabs(ub), dmax(fabs(ub + c), fabs(ub - c)));
    double SL = dmin(L.ubar - L.c, ub - c), SR = dmax(R.ubar + R.c, ub + c);
    double SM = (R.rho * R.ubar * (SR - R.ubar) - L.rho * L.ubar * (SL - L.ubar) + L.p - R.p) /
                (R.rho * (SR - R.ubar) - L.rho * (SL - L.ubar));
    double F[5];
    const face_t *S = 0;
    double Sk = 0.0;
    if (SL > 0.0 || SR < 0.0) {
        S = SL > 0.0 ? &L : &R;
        F[0] = S->rho * S->ubar; F[1] = S->u * F[0] + S->p * n[0]; F[2] = S->v * F[0] + S->p * n[1];
        F[3] = S->w * F[0] + S->p * n[2]; F[4] = S->ht * F[0];
    } else {
        if (SM > 0.0) { S = &L; Sk = SL; } else { S = &R; Sk = SR; }
        double pstar = S->p + S->rho * (S->ubar - Sk) * (S->ubar - SM);
        double om = 1.0 / (Sk - SM), c1 = Sk - S->ubar, c2 = pstar - S->p;
        double rs = om * (c1 * S->rho), rus = om * (c1 * S->rho * S->u + c2 * n[0]);
        double rvs = om * (c1 * S->rho * S->v + c2 * n[1]), rws = om * (c1 * S->rho * S->w + c2 * n[2]);
        double res = om * (c1 * S->rho * S->et - S->p * S->ubar + pstar * SM);
        F[0] = rs * SM; F[1] = rus * SM + pstar * n[0]; F[2] = rvs * SM + pstar * n[1];
        F[3] = rws * SM + pstar * n[2]; F[4] = (res + pstar) * SM;
    }
    for (int k = 0; k < 5; k++) { conv[k] = F[k] * area; diss[k] = 0.0; }
    return lmax;
}

/* Compute_VanLeerFlux (Euler3D/src/VanLeer_Fluxes.cpp:143-305): Van Leer flux-vector
 * splitting, F+ of the left and F- of the right face state by the normal Mach number;
 * the time step takes the eigenvalues of the arithmetic mean state. */
static double vanleer(const double *qL, const double *qR, const double *n, double area, const orc_params *p,
                      double *conv, double *diss) {
    face_t L, R;
    double g = p->gamma, nx = n[0], ny = n[1], nz = n[2];
    eos_face(qL, nx, ny, nz, p, &L);
    eos_face(qR, nx, ny, nz, p, &R);
    double rho_a = 0.5 * (L.rho + R.rho), ub_a = 0.5 * ((L.u + R.u) * nx + (L.v + R.v) * ny + (L.w + R.w) * nz);
    double p_a = 0.5 * (L.p + R.p), c_a = sqrt(g * p_a / rho_a);
    double lmax = dmax(fabs(ub_a), dmax(fabs(ub_a + c_a), fabs(ub_a - c_a)));
    double fp[5] = {0, 0, 0, 0, 0}, fm[5] = {0, 0, 0, 0, 0};
    double M = L.ubar / L.c, q2 = L.u * L.u + L.v * L.v + L.w * L.w;
    if (fabs(M) < 1.0) {
        double b = -L.ubar + 2.0 * L.c;
        fp[0] = 0.25 * L.rho * L.c * (M + 1.0) * (M + 1.0);
        fp[1] = fp[0] * (nx * b / g + L.u);
        fp[2] = fp[0] * (ny * b / g + L.v);
        fp[3] = fp[0] * (nz * b / g + L.w);
        fp[4] = fp[0] * ((-(g - 1.0) * L.ubar * L.ubar + 2.0 * (g - 1.0) * L.ubar * L.c + 2.0 * L.c * L.c) / (g * g - 1.0) + 0.5 * q2);
    } else if (M >= 1.0) {
        fp[0] = L.rho * L.ubar;
        fp[1] = L.rho * L.u * L.ubar + nx * L.p;
        fp[2] = L.rho * L.v * L.ubar + ny * L.p;
        fp[3] = L.rho * L.w * L.ubar + nz * L.p;
        fp[4] = (L.rho * L.et + L.p) * L.ubar;
    }
    M = R.ubar / R.c;
    q2 = R.u * R.u + R.v * R.v + R.w * R.w;
    if (fabs(M) < 1.0) {
        double b = -R.ubar - 2.0 * R.c;
        fm[0] = -0.25 * R.rho * R.c * (M - 1.0) * (M - 1.0);
        fm[1] = fm[0] * (nx * b / g + R.u);
        fm[2] = fm[0] * (ny * b / g + R.v);
        fm[3] = fm[0] * (nz * b / g + R.w);
        fm[4] = fm[0] * ((-(g - 1.0) * R.ubar * R.ubar - 2.0 * (g - 1.0) * R.ubar * R.c + 2.0 * R.c * R.c) / (g * g - 1.0) + 0.5 * q2);
    } else if (M <= -1.0) {
        fm[0] = R.rho * R.ubar;
        fm[1] = R.rho * R.u * R.ubar + nx * R.p;
        fm[2] = R.rho * R.v * R.ubar + ny * R.p;
        fm[3] = R.rho * R.w * R.ubar + nz * R.p;
        fm[4] = (R.rho * R.et + R.p) * R.ubar;
    }
    for (int k = 0; k < 5; k++) { conv[k] = (fp[k] + fm[k]) * area; diss[k] = 0.0; }
    return lmax;
}

/* AUSM+ restated from Liou, J. Comput. Phys. 129 (1996) 364-382: c_1/2 =
 * min(c^_L, c^_R), c^ = c*^2/max(c*, |u|), c*^2 = 2(g-1)/(g+1) H; M+-(M)
 * degree-4 polynomials with beta = 1/8, P+-(M) degree-5 with alpha = 3/16.
 * (The reference's AUSM is an empty stub, Euler3D/src/AUSM_Fluxes.cpp:45-54.) */
static double ausmp(const double *qL, const double *qR, const double *n, double area, const orc_params *p,
                    double *conv, double *diss) {
    face_t L, R;
    double g = p->gamma;
    eos_face(qL, n[0], n[1], n[2], p, &L);
    eos_face(qR, n[0], n[1], n[2], p, &R);
    double k = 2.0 * (g - 1.0) / (g + 1.0);
    double csL = sqrt(k * L.ht), csR = sqrt(k * R.ht);
    double c12 = dmin(csL * csL / dmax(csL, L.ubar), csR * csR / dmax(csR, -R.ubar));
    double ML = L.ubar / c12, MR = R.ubar / c12;
    double Mp, Pp, Mm, Pm;
    if (fabs(ML) >= 1.0) { Mp = 0.5 * (ML + fabs(ML)); Pp = ML > 0.0 ? 1.0 : 0.0; }
    else {
        Mp = 0.25 * (ML + 1.0) * (ML + 1.0) + 0.125 * (ML * ML - 1.0) * (ML * ML - 1.0);
        Pp = 0.25 * (ML + 1.0) * (ML + 1.0) * (2.0 - ML) + (3.0 / 16.0) * ML * (ML * ML - 1.0) * (ML * ML - 1.0);
    }
    if (fabs(MR) >= 1.0) { Mm = 0.5 * (MR - fabs(MR)); Pm = MR < 0.0 ? 1.0 : 0.0; }
    else {
        Mm = -0.25 * (MR - 1.0) * (MR - 1.0) - 0.125 * (MR * MR - 1.0) * (MR * MR - 1.0);
        Pm = 0.25 * (MR - 1.0) * (MR - 1.0) * (2.0 + MR) - (3.0 / 16.0) * MR * (MR * MR - 1.0) * (MR * MR - 1.0);
    }
    double m12 = Mp + Mm, mp = 0.5 * (m12 + fabs(m12)), mm = 0.5 * (m12 - fabs(m12));
    double p12 = Pp * L.p + Pm * R.p;
    double aL = c12 * mp * L.rho, aR = c12 * mm * R.rho;
    conv[0] = area * (aL + aR);
    conv[1] = area * (aL * L.u + aR * R.u + p12 * n[0]);
    conv[2] = area * (aL * L.v + aR * R.v + p12 * n[1]);
    conv[3] = area * (aL * L.w + aR * R.w + p12 * n[2]);
    conv[4] = area * (aL * L.ht + aR * R.ht);
    for (int j = 0; j < 5; j++) diss[j] = 0.0;
    double rho = sqrt(R.rho * L.rho), sigma = rho / (L.rho + rho);
    double u = L.u + sigma * (R.u - L.u), v = L.v + sigma * (R.v - L.v), w = L.w + sigma * (R.w - L.w);
    double ht = L.ht + sigma * (R.ht - L.ht);
    double c = sqrt((g - 1.0) * ht - 0.5 * (g - 1.0) * (u * u + v * v + w * w));
    return fabs(u * n[0] + v * n[1] + w * n[2]) + c;
}

/* Compute_SecondOrderReconstructQ (Euler3D/src/HigherOrderReconstructQ.cpp:21-72). */
static void reconstruct(const orc_mesh *m, const orc_params *p, const double *Q, const double *grad,
                        const double *phi, int a, int b, double *qa) {
    const int ld = m->nnode + m->nghost, nn = m->nnode;
    double frac = p->limiter_order == 1 ? 0.5 : 0.0;
    double r[3];
    for (int d = 0; d < 3; d++) r[d] = 0.5 * (m->xyz[3 * (size_t)b + d] - m->xyz[3 * (size_t)a + d]);
    for (int k = 0; k < 5; k++) {
        double ph = (p->limiter != -1 && phi) ? phi[IDX(k, a, nn)] : 1.0;
        double gr = grad[IDX(3 * k, a, nn)] * r[0] + grad[IDX(3 * k + 1, a, nn)] * r[1] + grad[IDX(3 * k + 2, a, nn)] * r[2];
        qa[k] = Q[IDX(k, a, ld)] + ph * (frac * (Q[IDX(k, b, ld)] - Q[IDX(k, a, ld)]) + (1.0 - frac) * gr);
    }
}

/* Compute_Residual_Roe_New (FluxTest.cpp:7968-8151) / Compute_Residual_HLLC
 * (HLLC_Fluxes.cpp:519-573): interior edges then boundary edges, scatter. */
void orc_residual(const orc_mesh *m, const orc_params *p, const double *Q, const double *grad, const double *phi,
                  double *conv, double *diss, double *dtsum, double ext[6]) {
    const int ld = m->nnode + m->nghost, nn = m->nnode;
    memset(conv, 0, sizeof(double) * 5 * nn);
    memset(diss, 0, sizeof(double) * 5 * nn);
    memset(dtsum, 0, sizeof(double) * nn);
    ext[0] = ext[2] = ext[4] = DBL_MAX;
    ext[1] = ext[3] = ext[5] = DBL_MIN;
    for (int pass = 0; pass < 2; pass++) {
        int ne = pass == 0 ? m->nedge : m->nbedge;
        const int *en = pass == 0 ? m->en : m->bn;
        const double *ea = pass == 0 ? m->ea : m->ba;
        for (int e = 0; e < ne; e++) {
            int L = en[2 * e], R = en[2 * e + 1];
            double n[3], area, qL[5], qR[5], fc[5], fd[5], lam[3] = {0, 0, 0}, lmax;
            unit(ea + 3 * (size_t)e, n, &area);
            if (pass == 0 && p->order == 1) {
                reconstruct(m, p, Q, grad, phi, L, R, qL);
                reconstruct(m, p, Q, grad, phi, R, L, qR);
            } else {
                for (int k = 0; k < 5; k++) { qL[k] = Q[IDX(k, L, ld)]; qR[k] = Q[IDX(k, R, ld)]; }
            }
            if (p->flux == 1) lmax = hllc(qL, qR, n, area, p, fc, fd);
            else if (p->flux == 2) lmax = ausmp(qL, qR, n, area, p, fc, fd);
            else if (p->flux == 6) lmax = vanleer(qL, qR, n, area, p, fc, fd);
            else {
                if (p->flux == 5) {
                    double mL[5], mR[5];
                    thornber(qL, qR, p, mL, mR);
                    lmax = roe(mL, mR, n, area, p, fc, fd, lam);
                } else {
                    lmax = p->flux == 4 ? roe_pc(qL, qR, n, area, p, fc, fd, lam) : roe(qL, qR, n, area, p, fc, fd, lam);
                }
                ext[0] = dmin(ext[0], lam[0]); ext[1] = dmax(ext[1], lam[0]);
                ext[2] = dmin(ext[2], lam[1]); ext[3] = dmax(ext[3], lam[1]);
                ext[4] = dmin(ext[4], lam[2]); ext[5] = dmax(ext[5], lam[2]);
            }
            dtsum[L] += area * lmax;
            if (R < nn) dtsum[R] += area * lmax;
            for (int k = 0; k < 5; k++) {
                conv[IDX(k, L, nn)] += fc[k];
                diss[IDX(k, L, nn)] += fd[k];
                if (pass == 0) {
                    conv[IDX(k, R, nn)] -= fc[k];
                    diss[IDX(k, R, nn)] -= fd[k];
                }
            }
        }
    }
}

/* Compute_DeltaT (Euler3D/src/Time_Step.cpp:23-51); p->cfl is the ramped CFL. */
void orc_deltat(const orc_mesh *m, const orc_params *p, double *dt, double ext2[2]) {
    ext2[0] = DBL_MAX;
    ext2[1] = DBL_MIN;
    for (int i = 0; i < m->nnode; i++) {
        dt[i] = m->vol[i] * p->cfl / dt[i];
        ext2[0] = dmin(ext2[0], dt[i]);
        ext2[1] = dmax(ext2[1], dt[i]);
    }
    if (p->global_time)
        for (int i = 0; i < m->nnode; i++) dt[i] = ext2[0];
}

/* Least-squares coefficients and gradient (Euler3D/src/Gradient.cpp:137-296). */
void orc_gradient_lsq(const orc_mesh *m, const orc_params *p, const double *Q, double *grad) {
    const int ld = m->nnode + m->nghost, nn = m->nnode;
    for (int i = 0; i < nn; i++) {
        double r11 = 0, r12 = 0, r13 = 0, r22 = 0, r23 = 0, r33 = 0, ro22 = 0, ro33 = 0;
        const double *xi = m->xyz + 3 * (size_t)i;
        for (int pass = 0; pass < 4; pass++) {
            for (int k = m->ia[i]; k < m->ia[i + 1]; k++) {
                int j = m->ja[k];
                const double *xj = m->xyz + 3 * (size_t)j;
                double dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
                double a = p->ls_weight ? 1.0 / sqrt(dx * dx + dy * dy + dz * dz) : 1.0;
                dx *= a; dy *= a; dz *= a;
                if (pass == 0) { r11 += dx * dx; r12 += dx * dy; r13 += dx * dz; }
                else if (pass == 1) {
                    double t = dy - (r12 / r11) * dx;
                    r22 += t * t; r23 += t * dz; ro22 += t * dy;
                } else if (pass == 2) {
                    double t = dz - (r13 / r11) * dx - (r23 / r22) * (dy - (r12 / r11) * dx);
                    r33 += t * t; ro33 += t * dz;
                } else {
                    double Wz = (dz - (r13 / r11) * dx - (r23 / r22) * (dy - (r12 / r11) * dx)) / ro33;
                    double Wy = (dy - (r12 / r11) * dx - r23 * Wz) / ro22;
                    double Wx = (dx - r12 * Wy - r13 * Wz) / r11;
                    for (int v = 0; v < 5; v++) {
                        double d = Q[IDX(v, j, ld)] - Q[IDX(v, i, ld)];
                        if (k == m->ia[i]) {
                            grad[IDX(3 * v, i, nn)] = grad[IDX(3 * v + 1, i, nn)] = grad[IDX(3 * v + 2, i, nn)] = 0.0;
                        }
                        grad[IDX(3 * v, i, nn)] += Wx * a * d;
                        grad[IDX(3 * v + 1, i, nn)] += Wy * a * d;
                        grad[IDX(3 * v + 2, i, nn)] += Wz * a * d;
                    }
                }
            }
        }
        (void)r33;
    }
}

/* Green-Gauss on the median dual (restated: the reference only declares the
 * option, SolverParameters.h:329): grad_i = (1/V_i) sum_j (Q_j - Q_i)/2 S_ij
 * over interior dual faces; boundary dual faces carry Q_i and drop out. */
void orc_gradient_gg(const orc_mesh *m, const double *Q, double *grad) {
    const int ld = m->nnode + m->nghost, nn = m->nnode;
    memset(grad, 0, sizeof(double) * 15 * nn);
    for (int e = 0; e < m->nedge; e++) {
        int L = m->en[2 * e], R = m->en[2 * e + 1];
        const double *S = m->ea + 3 * (size_t)e;
        for (int v = 0; v < 5; v++) {
            double h = 0.5 * (Q[IDX(v, R, ld)] - Q[IDX(v, L, ld)]);
            for (int d = 0; d < 3; d++) {
                grad[IDX(3 * v + d, L, nn)] += h * S[d];
                grad[IDX(3 * v + d, R, nn)] += h * S[d];
            }
        }
    }
    for (int i = 0; i < nn; i++)
        for (int k = 0; k < 15; k++) grad[IDX(k, i, nn)] /= m->vol[i];
}

/* Compute_Limiter (Euler3D/src/Limiters.cpp:20-111) with Venkatakrishnan
 * (:185-267) or Barth-Jespersen (:117-178), the pressure correction
 * (:273-304) and, for the Roe flux, the sequential Roe-average pressure
 * correction (:61-110, :311-356). */
void orc_limiter(const orc_mesh *m, const orc_params *p, const double *Q, const double *grad, double *phi) {
    const int ld = m->nnode + m->nghost, nn = m->nnode;
    const double frac = p->limiter_order == 1 ? 0.5 : 0.0;
    for (int i = 0; i < nn; i++)
        for (int v = 0; v < 5; v++) phi[IDX(v, i, nn)] = 1.0;
    for (int i = 0; i < nn; i++) {
        double ph[5] = {1, 1, 1, 1, 1}, qmin[5], qmax[5], qc[5];
        for (int v = 0; v < 5; v++) qc[v] = qmin[v] = qmax[v] = Q[IDX(v, i, ld)];
        double eps2 = pow(p->venkat_k, 3.0);
        eps2 = 6.0 * eps2 * m->vol[i] / M_PI;
        for (int k = m->ia[i]; k < m->ia[i + 1]; k++)
            for (int v = 0; v < 5; v++) {
                qmin[v] = dmin(qmin[v], Q[IDX(v, m->ja[k], ld)]);
                qmax[v] = dmax(qmax[v], Q[IDX(v, m->ja[k], ld)]);
            }
        for (int k = m->ia[i]; k < m->ia[i + 1]; k++) {
            int j = m->ja[k];
            double r[3];
            for (int d = 0; d < 3; d++) r[d] = 0.5 * (m->xyz[3 * (size_t)j + d] - m->xyz[3 * (size_t)i + d]);
            for (int v = 0; v < 5; v++) {
                double gr = grad[IDX(3 * v, i, nn)] * r[0] + grad[IDX(3 * v + 1, i, nn)] * r[1] + grad[IDX(3 * v + 2, i, nn)] * r[2];
                double q = qc[v] + frac * (Q[IDX(v, j, ld)] - qc[v]) + (1.0 - frac) * gr;
                double dm = q - qc[v];
                if (p->limiter == 1) {
                    if (dm != 0.0) {
                        double dp = (dm > 0.0 ? qmax[v] : qmin[v]) - qc[v];
                        double t = (dp * dp + eps2) + 2.0 * (dm * dp);
                        t = t / (dp * dp + 2.0 * dm * dm + dm * dp + eps2);
                        ph[v] = dmin(ph[v], t);
                    } else ph[v] = dmin(ph[v], 1.0);
                } else {
                    if (dm > 0.0) ph[v] = dmin(ph[v], dmin(1.0, (qmax[v] - qc[v]) / dm));
                    else if (dm < 0.0) ph[v] = dmin(ph[v], dmin(1.0, (qmin[v] - qc[v]) / dm));
                    else ph[v] = dmin(ph[v], 1.0);
                }
                ph[v] = dmax(0.0, ph[v]);
            }
        }
        if (p->limiter_smooth) {
            for (int v = 1; v < 5; v++) ph[0] = dmin(ph[0], ph[v]);
            for (int v = 1; v < 5; v++) ph[v] = ph[0];
        }
        for (int k = m->ia[i]; k < m->ia[i + 1]; k++) {
            int j = m->ja[k];
            double r[3], q[5];
            for (int d = 0; d < 3; d++) r[d] = 0.5 * (m->xyz[3 * (size_t)j + d] - m->xyz[3 * (size_t)i + d]);
            for (int v = 0; v < 5; v++) {
                double gr = grad[IDX(3 * v, i, nn)] * r[0] + grad[IDX(3 * v + 1, i, nn)] * r[1] + grad[IDX(3 * v + 2, i, nn)] * r[2];
                q[v] = qc[v] + ph[v] * (frac * (Q[IDX(v, j, ld)] - qc[v]) + (1.0 - frac) * gr);
            }
            /* p < 0 (Limiters.cpp:296-301); for the stiffened gas p + pinf < 0 */
            double pc = p->variables == 1 ? q[4] + p->pinf
                                          : (p->gamma - 1.0) * ((q[4] - p->pinf) - (0.5 / q[0]) * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]));
            if (pc < 0.0)
                for (int v = 0; v < 5; v++) ph[v] = 0.0;
        }
        for (int v = 0; v < 5; v++) phi[IDX(v, i, nn)] = ph[v];
    }
    if (p->flux != 0 && p->flux != 3 && p->flux != 4 && p->flux != 5) return;
    for (int i = 0; i < nn; i++) {
        for (int k = m->ia[i]; k < m->ia[i + 1]; k++) {
            int j = m->ja[k];
            double r[3], qa[5], qb[5];
            for (int d = 0; d < 3; d++) r[d] = 0.5 * (m->xyz[3 * (size_t)j + d] - m->xyz[3 * (size_t)i + d]);
            for (int v = 0; v < 5; v++) {
                double gi = grad[IDX(3 * v, i, nn)] * r[0] + grad[IDX(3 * v + 1, i, nn)] * r[1] + grad[IDX(3 * v + 2, i, nn)] * r[2];
                double gj = -(grad[IDX(3 * v, j, nn)] * r[0] + grad[IDX(3 * v + 1, j, nn)] * r[1] + grad[IDX(3 * v + 2, j, nn)] * r[2]);
                double ci = Q[IDX(v, i, ld)], cj = Q[IDX(v, j, ld)];
                qa[v] = ci + phi[IDX(v, i, nn)] * (frac * (cj - ci) + (1.0 - frac) * gi);
                qb[v] = cj + phi[IDX(v, j, nn)] * (frac * (ci - cj) + (1.0 - frac) * gj);
            }
            /* Compute_RoeVariables (Roe_Fluxes.cpp:3609-3633) */
            face_t A, B;
            eos_face(qa, 0, 0, 0, p, &A);
            eos_face(qb, 0, 0, 0, p, &B);
            double rho = sqrt(B.rho * A.rho), sg = rho / (A.rho + rho);
            double u = A.u + sg * (B.u - A.u), v = A.v + sg * (B.v - A.v), w = A.w + sg * (B.w - A.w);
            double ht = A.ht + sg * (B.ht - A.ht);
            double qr[5] = {rho, rho * u, rho * v, rho * w,
                            (rho / p->gamma) * (ht + 0.5 * (p->gamma - 1.0) * (u * u + v * v + w * w))};
            /* for the stiffened gas this is p + pinf of the Roe state (c^2 = (g - 1) h) */
            double pr = (p->gamma - 1.0) * (qr[4] - (0.5 / qr[0]) * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]));
            if (pr < 0.0)
                for (int v2 = 0; v2 < 5; v2++) { phi[IDX(v2, i, nn)] = 0.0; phi[IDX(v2, j, nn)] = 0.0; }
        }
    }
}

/* Create_CRS_SolverBlockMatrix pattern (Euler3D/src/Solver.cpp:612-672). */
long orc_block_pattern(const orc_mesh *m, int *IA, int *JA, int *IAU) {
    long nnz = 0;
    for (int i = 0; i < m->nnode; i++) nnz += m->ia[i + 1] - m->ia[i] + 1;
    if (!IA) return nnz;
    IA[0] = 0;
    for (int i = 0; i < m->nnode; i++) {
        int k = IA[i], n0 = k;
        JA[k++] = i;
        for (int q = m->ia[i]; q < m->ia[i + 1]; q++) JA[k++] = m->ja[q];
        /* selection sort as the reference does */
        for (int a = n0; a < k; a++) {
            int mi = a;
            for (int b = a + 1; b < k; b++) if (JA[b] < JA[mi]) mi = b;
            int t = JA[a]; JA[a] = JA[mi]; JA[mi] = t;
            if (JA[a] == i) IAU[i] = a;
        }
        IA[i + 1] = k;
    }
    return nnz;
}

/* ConservativeEulerFluxJacobian (Euler3D/src/CompressibleUtils.cpp:558-609). */
static void flux_jac(const double *q, const double *n, double g, double pinf, double J[5][5]) {
    double rho = q[0], u = q[1] / rho, v = q[2] / rho, w = q[3] / rho, rhoet = q[4];
    double ek = 0.5 * (u * u + v * v + w * w), p = (g - 1.0) * (rhoet - rho * ek) - g * pinf, ht = (rhoet + p) / rho;
    double ub = u * n[0] + v * n[1] + w * n[2];
    double nx = n[0], ny = n[1], nz = n[2];
    J[0][0] = 0.0; J[1][0] = (g - 1.0) * ek * nx - u * ub; J[2][0] = (g - 1.0) * ek * ny - v * ub;
    J[3][0] = (g - 1.0) * ek * nz - w * ub; J[4][0] = ((g - 1.0) * ek - ht) * ub;
    J[0][1] = nx; J[1][1] = ub - (g - 2.0) * u * nx; J[2][1] = v * nx - (g - 1.0) * u * ny;
    J[3][1] = w * nx - (g - 1.0) * u * nz; J[4][1] = ht * nx - (g - 1.0) * u * ub;
    J[0][2] = ny; J[1][2] = u * ny - (g - 1.0) * v * nx; J[2][2] = ub - (g - 2.0) * v * ny;
    J[3][2] = w * ny - (g - 1.0) * v * nz; J[4][2] = ht * ny - (g - 1.0) * v * ub;
    J[0][3] = nz; J[1][3] = u * nz - (g - 1.0) * w * nx; J[2][3] = v * nz - (g - 1.0) * w * ny;
    J[3][3] = ub - (g - 2.0) * w * nz; J[4][3] = ht * nz - (g - 1.0) * w * ub;
    J[0][4] = 0.0; J[1][4] = (g - 1.0) * nx; J[2][4] = (g - 1.0) * ny; J[3][4] = (g - 1.0) * nz; J[4][4] = g * ub;
}

/* dF.n/d(rho, u, v, w, p) (Compute_Flux_Jacobian_Euler_Convective, VARIABLE_RUP,
 * MPFLOW3D/src/CompressibleUtils.cpp:85-186), rho ht = g (p + pinf) / (g - 1) + rho q^2 / 2. */
static void flux_jac_rup(const double *q, const double *n, double g, double pinf, double J[5][5]) {
    double rho = q[0], u = q[1], v = q[2], w = q[3], pr = q[4];
    double ub = u * n[0] + v * n[1] + w * n[2], q2 = u * u + v * v + w * w;
    double ht = g * (pr + pinf) / ((g - 1.0) * rho) + 0.5 * q2;
    double vel[3] = {u, v, w};
    J[0][0] = ub;
    for (int d = 0; d < 3; d++) J[0][1 + d] = rho * n[d];
    J[0][4] = 0.0;
    for (int k = 0; k < 3; k++) {
        J[1 + k][0] = vel[k] * ub;
        for (int d = 0; d < 3; d++) J[1 + k][1 + d] = rho * vel[k] * n[d] + (k == d ? rho * ub : 0.0);
        J[1 + k][4] = n[k];
    }
    J[4][0] = 0.5 * q2 * ub;
    for (int d = 0; d < 3; d++) J[4][1 + d] = rho * (vel[d] * ub + ht * n[d]);
    J[4][4] = g / (g - 1.0) * ub;
}

static void mm5(double A[5][5], double B[5][5], double C[5][5]) {
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            C[i][j] = 0.0;
            for (int k = 0; k < 5; k++) C[i][j] += A[i][k] * B[k][j];
        }
}

/* Compute_RoeAJacobian: |A| = M P |Lambda| P^-1 M^-1 (Euler3D/src/Roe_Fluxes.cpp:149-273). */
static void roe_absA(const double *qL, const double *qR, const double *n, const orc_params *p, double A[5][5]) {
    face_t L, R;
    double g = p->gamma;
    eos_face(qL, n[0], n[1], n[2], p, &L);
    eos_face(qR, n[0], n[1], n[2], p, &R);
    double rho = sqrt(R.rho * L.rho), sigma = rho / (L.rho + rho);
    double u = L.u + sigma * (R.u - L.u), v = L.v + sigma * (R.v - L.v), w = L.w + sigma * (R.w - L.w);
    double ht = L.ht + sigma * (R.ht - L.ht);
    double phi = 0.5 * (g - 1.0) * (u * u + v * v + w * w);
    double c = sqrt((g - 1.0) * ht - phi);
    double ub = u * n[0] + v * n[1] + w * n[2];
    double nx = n[0], ny = n[1], nz = n[2];
    double M[5][5] = {{1, 0, 0, 0, 0}, {u, rho, 0, 0, 0}, {v, 0, rho, 0, 0}, {w, 0, 0, rho, 0},
                      {phi / (g - 1.0), rho * u, rho * v, rho * w, 1.0 / (g - 1.0)}};
    double Mi[5][5] = {{1, 0, 0, 0, 0}, {-u / rho, 1.0 / rho, 0, 0, 0}, {-v / rho, 0, 1.0 / rho, 0, 0},
                       {-w / rho, 0, 0, 1.0 / rho, 0}, {phi, -u * (g - 1.0), -v * (g - 1.0), -w * (g - 1.0), g - 1.0}};
    double P[5][5] = {{nx, ny, nz, rho / c, rho / c}, {0.0, -nz, ny, nx, -nx}, {nz, 0.0, -nx, ny, -ny},
                      {-ny, nx, 0.0, nz, -nz}, {0.0, 0.0, 0.0, rho * c, rho * c}};
    double Pi[5][5] = {{nx, 0.0, nz, -ny, -nx / (c * c)}, {ny, -nz, 0.0, nx, -ny / (c * c)},
                       {nz, ny, -nx, 0.0, -nz / (c * c)}, {0.0, 0.5 * nx, 0.5 * ny, 0.5 * nz, 1.0 / (2.0 * rho * c)},
                       {0.0, -0.5 * nx, -0.5 * ny, -0.5 * nz, 1.0 / (2.0 * rho * c)}};
    double E[3];
    if (p->entropy_fix) entropy_fix(L.ubar, L.c, R.ubar, R.c, ub, c, E);
    else { E[0] = fabs(ub); E[1] = fabs(ub + c); E[2] = fabs(ub - c); }
    double Lm[5][5] = {{0}};
    Lm[0][0] = Lm[1][1] = Lm[2][2] = E[0]; Lm[3][3] = E[1]; Lm[4][4] = E[2];
    double T[5][5], Ti[5][5], LT[5][5];
    mm5(M, P, T);
    if (p->variables == 1) {
        /* columns in (rho, u, v, w, p): Mop |A| (MPFLOW3D Compute_Dissipation_Matrix_Roe_Optimized,
         * Roe_Fluxes.cpp:3185-3199, Mpr = I); mpf_form 1 carries its E1 (1 - ny^2) w-momentum
         * diagonal (:3146), i.e. |A|[3][3] + E0 (nz^2 - ny^2) in (rho, u, v, w, p) */
        mm5(Lm, Pi, LT);
        mm5(T, LT, A);
        if (p->mpf_form == 1)
            for (int a = 0; a < 5; a++) A[a][3] += M[a][3] * E[0] * (nz * nz - ny * ny);
        return;
    }
    mm5(Pi, Mi, Ti);
    mm5(Lm, Ti, LT);
    mm5(T, LT, A);
}

/* Compute_Jacobian_Approximate_Roe (Euler3D/src/Roe_Jacobian.cpp:29-228);
 * A is [nnzb][5][5] contiguous, B [nnode][5]. */
void orc_jacobian(const orc_mesh *m, const orc_params *p, const double *Q, const double *dt, const double *conv,
                  const double *diss, int add_time, int include_diss, const int *IA, const int *JA, const int *IAU,
                  double *A, double *B) {
    const int ld = m->nnode + m->nghost, nn = m->nnode;
    memset(A, 0, sizeof(double) * 25 * (size_t)IA[nn]);
    for (int i = 0; i < nn; i++) {
        for (int k = 0; k < 5; k++)
            B[5 * (size_t)i + k] = -(conv[IDX(k, i, nn)] + (include_diss ? diss[IDX(k, i, nn)] : 0.0));
        if (add_time && p->flux == 4) {
            /* pseudo-time term (V / dt) Cinv of the preconditioned system (Roe_Jacobian.cpp:241-264) */
            double q[5], C[5][5];
            for (int k = 0; k < 5; k++) q[k] = Q[IDX(k, i, ld)];
            pc_node_cinv(q, p, C);
            for (int a = 0; a < 5; a++)
                for (int b = 0; b < 5; b++) A[25 * (size_t)IAU[i] + 5 * a + b] = m->vol[i] / dt[i] * C[a][b];
        } else if (add_time && p->variables == 1) {
            /* (V / dt) dQ/d(rho, u, v, w, p) (MPFLOW3D Roe_Jacobian.cpp:241-264, PRECOND_METHOD_NONE) */
            double q[5], Mpr[5][5], Mop[5][5];
            for (int k = 0; k < 5; k++) q[k] = Q[IDX(k, i, ld)];
            pc_transforms(q[0], q[1], q[2], q[3], p->gamma, Mpr, Mop);
            for (int a = 0; a < 5; a++)
                for (int b = 0; b < 5; b++) A[25 * (size_t)IAU[i] + 5 * a + b] = m->vol[i] / dt[i] * Mop[a][b];
        } else if (add_time)
            for (int k = 0; k < 5; k++) A[25 * (size_t)IAU[i] + 6 * k] = m->vol[i] / dt[i];
    }
    for (int pass = 0; pass < 2; pass++) {
        int ne = pass == 0 ? m->nedge : m->nbedge;
        const int *en = pass == 0 ? m->en : m->bn;
        const double *ea = pass == 0 ? m->ea : m->ba;
        for (int e = 0; e < ne; e++) {
            int L = en[2 * e], R = en[2 * e + 1];
            double n[3], area, qL[5], qR[5], JL[5][5], JR[5][5], Ab[5][5];
            unit(ea + 3 * (size_t)e, n, &area);
            for (int k = 0; k < 5; k++) { qL[k] = Q[IDX(k, L, ld)]; qR[k] = Q[IDX(k, R, ld)]; }
            if (p->variables == 1) {
                flux_jac_rup(qL, n, p->gamma, p->pinf, JL);
                flux_jac_rup(qR, n, p->gamma, p->pinf, JR);
            } else {
                flux_jac(qL, n, p->gamma, p->pinf, JL);
                flux_jac(qR, n, p->gamma, p->pinf, JR);
            }
            if (p->flux == 4) {
                face_t Lf, Rf;
                pc_sys_t S;
                double avg[4];
                pc_edge(qL, qR, n, p, &Lf, &Rf, avg, &S);
                pc_absA(&S, avg, p, Ab);
            } else if (p->flux == 5) {
                double mL[5], mR[5];
                thornber(qL, qR, p, mL, mR);
                roe_absA(mL, mR, n, p, Ab);
            } else {
                roe_absA(qL, qR, n, p, Ab);
            }
            double *dL = A + 25 * (size_t)IAU[L];
            if (pass == 1) {
                for (int a = 0; a < 5; a++)
                    for (int b = 0; b < 5; b++) dL[5 * a + b] += 0.5 * (JL[a][b] + Ab[a][b]) * area;
                continue;
            }
            int oL = -1, oR = -1;
            for (int k = IA[L]; k < IA[L + 1]; k++) if (JA[k] == R) { oL = k; break; }
            for (int k = IA[R]; k < IA[R + 1]; k++) if (JA[k] == L) { oR = k; break; }
            double *dR = A + 25 * (size_t)IAU[R], *aL = A + 25 * (size_t)oL, *aR = A + 25 * (size_t)oR;
            for (int a = 0; a < 5; a++)
                for (int b = 0; b < 5; b++) {
                    double fl = 0.5 * (JL[a][b] + Ab[a][b]) * area, fr = 0.5 * (JR[a][b] - Ab[a][b]) * area;
                    dL[5 * a + b] += fl;
                    dR[5 * a + b] -= fr;
                    aL[5 * a + b] += fr;
                    aR[5 * a + b] -= fl;
                }
        }
    }
}

/* MC_Iterative_Block_LU_Jacobi_CRS (MATH/src/MC_Iterative_Jacobi.c:346-535). */
double orc_block_gs(int n, const int *IA, const int *JA, const int *IAU, const double *A, const double *B, double *X,
                    int iters, int direction) {
    double *LU = (double *)malloc(sizeof(double) * 25 * (size_t)n);
    double rms = 0.0;
    memset(X, 0, sizeof(double) * 5 * (size_t)n);
    for (int r = 0; r < n; r++) {
        double *a = LU + 25 * (size_t)r;
        memcpy(a, A + 25 * (size_t)IAU[r], sizeof(double) * 25);
        for (int k = 0; k < 4; k++) {
            for (int j = k + 1; j < 5; j++) a[5 * j + k] = a[5 * j + k] / a[5 * k + k];
            for (int j = k + 1; j < 5; j++)
                for (int i = k + 1; i < 5; i++) a[5 * i + j] -= a[5 * i + k] * a[5 * k + j];
        }
    }
    if (iters <= 0) iters = 10000;
    for (int it = 0; it < iters; it++) {
        rms = 0.0;
        int fwd = direction == 0 || (direction == 2 && it % 2 == 0);
        for (int q = 0; q < n; q++) {
            int r = fwd ? q : n - 1 - q;
            double rhs[5], t[5];
            for (int k = 0; k < 5; k++) rhs[k] = B[5 * (size_t)r + k];
            for (int k = IA[r]; k < IA[r + 1]; k++) {
                const double *a = A + 25 * (size_t)k, *x = X + 5 * (size_t)JA[k];
                for (int ii = 0; ii < 5; ii++) {
                    t[ii] = 0.0;
                    for (int jj = 0; jj < 5; jj++) t[ii] += a[5 * ii + jj] * x[jj];
                }
                for (int ii = 0; ii < 5; ii++) rhs[ii] -= t[ii];
            }
            for (int k = 0; k < 5; k++) rms += rhs[k] * rhs[k];
            const double *ad = A + 25 * (size_t)IAU[r], *xr = X + 5 * (size_t)r;
            for (int ii = 0; ii < 5; ii++) {
                t[ii] = 0.0;
                for (int jj = 0; jj < 5; jj++) t[ii] += ad[5 * ii + jj] * xr[jj];
            }
            for (int ii = 0; ii < 5; ii++) rhs[ii] += t[ii];
            const double *lu = LU + 25 * (size_t)r;
            for (int ii = 0; ii < 5; ii++) {
                t[ii] = rhs[ii];
                for (int jj = 0; jj < ii; jj++) t[ii] -= lu[5 * ii + jj] * t[jj];
            }
            double *xo = X + 5 * (size_t)r;
            for (int ii = 4; ii >= 0; ii--) {
                xo[ii] = t[ii];
                for (int jj = 4; jj > ii; jj--) xo[ii] -= lu[5 * ii + jj] * xo[jj];
                xo[ii] = xo[ii] / lu[5 * ii + ii];
            }
        }
        rms = sqrt(rms / (double)n);
        if (rms < 100.0 * DBL_EPSILON) break;
    }
    free(LU);
    return rms;
}

/* MC_Iterative_Block_LUSGS_CRS (MATH/src/MC_Iterative_Jacobi.c:539-717) with
 * the pivoted elimination of GaussainLUDecompose and the pivoted
 * substitutions (MATH/src/LinearAlgebra.c:20-43, 117-150); the returned RMS is
 * computed as the reference computes it (block 6 of the storage against X at
 * its column for every row, the running sum divided by 5 after each row). */
static void lu_pivot5(double a[25], int P[5]) {
    for (int i = 0; i < 5; i++) P[i] = i;
    for (int c = 0; c < 5; c++) {
        double pmax = a[P[c] * 5 + c];
        int pi = c;
        for (int i = c + 1; i < 5; i++)
            if (fabs(a[P[i] * 5 + c]) > fabs(pmax)) { pmax = a[P[i] * 5 + c]; pi = i; }
        if (pi != c) { int t = P[c]; P[c] = P[pi]; P[pi] = t; }
        for (int i = c + 1; i < 5; i++) a[P[i] * 5 + c] /= a[P[c] * 5 + c];
        for (int i = c + 1; i < 5; i++)
            for (int j = c + 1; j < 5; j++) a[P[i] * 5 + j] -= a[P[i] * 5 + c] * a[P[c] * 5 + j];
    }
}

double orc_block_lusgs(int n, const int *IA, const int *JA, const int *IAU, const double *A, const double *B,
                       double *X, int iters) {
    for (int r = 0; r < n; r++) {
        double m = 0.0;
        for (int j = 0; j < 5; j++) m += B[5 * (size_t)r + j];
        m /= 5;
        for (int j = 0; j < 5; j++) X[5 * (size_t)r + j] = m;
    }
    if (iters <= 0) iters = 100;
    for (int it = 0; it < iters; it++)
        for (int dir = 0; dir < 2; dir++)
            for (int q = 0; q < n; q++) {
                const int r = dir == 0 ? q : n - 1 - q;
                double rhs[5], t[5], lu[25], y[5], x[5];
                int P[5];
                for (int k = 0; k < 5; k++) rhs[k] = B[5 * (size_t)r + k];
                for (int k = IA[r]; k < IA[r + 1]; k++) {
                    if (k == IAU[r]) continue;
                    const double *a = A + 25 * (size_t)k, *xv = X + 5 * (size_t)JA[k];
                    for (int ii = 0; ii < 5; ii++) {
                        t[ii] = 0.0;
                        for (int jj = 0; jj < 5; jj++) t[ii] += a[5 * ii + jj] * xv[jj];
                    }
                    for (int ii = 0; ii < 5; ii++) rhs[ii] -= t[ii];
                }
                memcpy(lu, A + 25 * (size_t)IAU[r], sizeof lu);
                lu_pivot5(lu, P);
                y[0] = rhs[P[0]];
                for (int i = 1; i < 5; i++) {
                    y[i] = rhs[P[i]];
                    for (int j = 0; j < i; j++) y[i] -= y[j] * lu[P[i] * 5 + j];
                }
                x[4] = y[4] / lu[P[4] * 5 + 4];
                for (int i = 3; i >= 0; i--) {
                    x[i] = y[i];
                    for (int j = 4; j > i; j--) x[i] -= x[j] * lu[P[i] * 5 + j];
                    x[i] /= lu[P[i] * 5 + i];
                }
                for (int k = 0; k < 5; k++) X[5 * (size_t)r + k] = x[k];
            }
    double t[5], rms = 0.0;
    const double *a = A + 25 * 5, *xv = X + 5 * (size_t)JA[5];
    for (int ii = 0; ii < 5; ii++) {
        t[ii] = 0.0;
        for (int jj = 0; jj < 5; jj++) t[ii] += a[5 * ii + jj] * xv[jj];
    }
    for (int r = 0; r < n; r++) {
        for (int j = 0; j < 5; j++) rms += (B[5 * (size_t)r + j] - t[j]) * (B[5 * (size_t)r + j] - t[j]);
        rms /= 5;
    }
    return sqrt(rms / (double)n);
}

void orc_bspmv(int n, const int *IA, const int *JA, const double *A, const double *x, double *y) {
    for (int r = 0; r < n; r++)
        for (int a = 0; a < 5; a++) {
            double s = 0.0;
            for (int k = IA[r]; k < IA[r + 1]; k++)
                for (int b = 0; b < 5; b++) s += A[25 * (size_t)k + 5 * a + b] * x[5 * (size_t)JA[k] + b];
            y[5 * (size_t)r + a] = s;
        }
}

/* 5x5 inverse, Gauss-Jordan with partial pivoting. */
static int inv5(const double *in, double *out) {
    double a[25];
    memcpy(a, in, sizeof a);
    for (int k = 0; k < 25; k++) out[k] = (k % 6 == 0) ? 1.0 : 0.0;
    for (int c = 0; c < 5; c++) {
        int p = c;
        for (int r = c + 1; r < 5; r++) if (fabs(a[5 * r + c]) > fabs(a[5 * p + c])) p = r;
        if (a[5 * p + c] == 0.0) return 1;
        for (int j = 0; j < 5; j++) {
            double t = a[5 * c + j]; a[5 * c + j] = a[5 * p + j]; a[5 * p + j] = t;
            t = out[5 * c + j]; out[5 * c + j] = out[5 * p + j]; out[5 * p + j] = t;
        }
        double d = 1.0 / a[5 * c + c];
        for (int j = 0; j < 5; j++) { a[5 * c + j] *= d; out[5 * c + j] *= d; }
        for (int r = 0; r < 5; r++) {
            if (r == c) continue;
            double f = a[5 * r + c];
            for (int j = 0; j < 5; j++) { a[5 * r + j] -= f * a[5 * c + j]; out[5 * r + j] -= f * out[5 * c + j]; }
        }
    }
    return 0;
}

/* Block ILU(0), IKJ variant in natural row order (Saad, "Iterative Methods
 * for Sparse Linear Systems", 2nd ed., Alg. 10.4, with 5x5 blocks): F holds
 * the strictly lower L blocks, the strictly upper U blocks and inv(U_ii) on
 * the diagonal. */
int orc_ilu0(int n, const int *IA, const int *JA, const int *IAU, const double *A, double *F) {
    memcpy(F, A, sizeof(double) * 25 * (size_t)IA[n]);
    for (int i = 0; i < n; i++) {
        for (int k = IA[i]; k < IAU[i]; k++) {
            int p = JA[k];
            double L[25], *Lip = F + 25 * (size_t)k;
            const double *Dp = F + 25 * (size_t)IAU[p];
            for (int a = 0; a < 5; a++)
                for (int b = 0; b < 5; b++) {
                    double s = 0.0;
                    for (int q = 0; q < 5; q++) s += Lip[5 * a + q] * Dp[5 * q + b];
                    L[5 * a + b] = s;
                }
            memcpy(Lip, L, sizeof L);
            for (int mi = k + 1; mi < IA[i + 1]; mi++) {
                int j = JA[mi];
                for (int pk = IAU[p] + 1; pk < IA[p + 1]; pk++) {
                    if (JA[pk] != j) continue;
                    double *Aij = F + 25 * (size_t)mi;
                    const double *U = F + 25 * (size_t)pk;
                    for (int a = 0; a < 5; a++)
                        for (int b = 0; b < 5; b++)
                            for (int q = 0; q < 5; q++) Aij[5 * a + b] -= L[5 * a + q] * U[5 * q + b];
                }
            }
        }
        double inv[25];
        if (inv5(F + 25 * (size_t)IAU[i], inv)) return 1;
        memcpy(F + 25 * (size_t)IAU[i], inv, sizeof inv);
    }
    return 0;
}

static void ilu_apply(int n, const int *IA, const int *JA, const int *IAU, const double *F, const double *r,
                      double *z) {
    double *y = (double *)malloc(sizeof(double) * 5 * (size_t)n);
    for (int i = 0; i < n; i++)
        for (int a = 0; a < 5; a++) {
            double s = r[5 * (size_t)i + a];
            for (int k = IA[i]; k < IAU[i]; k++)
                for (int b = 0; b < 5; b++) s -= F[25 * (size_t)k + 5 * a + b] * y[5 * (size_t)JA[k] + b];
            y[5 * (size_t)i + a] = s;
        }
    for (int i = n - 1; i >= 0; i--) {
        double t[5];
        for (int a = 0; a < 5; a++) {
            double s = y[5 * (size_t)i + a];
            for (int k = IAU[i] + 1; k < IA[i + 1]; k++)
                for (int b = 0; b < 5; b++) s -= F[25 * (size_t)k + 5 * a + b] * z[5 * (size_t)JA[k] + b];
            t[a] = s;
        }
        const double *D = F + 25 * (size_t)IAU[i];
        for (int a = 0; a < 5; a++) {
            double s = 0.0;
            for (int b = 0; b < 5; b++) s += D[5 * a + b] * t[b];
            z[5 * (size_t)i + a] = s;
        }
    }
    free(y);
}

/* z = (LU)^-1 r with the factors of orc_ilu0 (the apply of orc_gmres' ILU(0)). */
void orc_ilu0_apply(int n, const int *IA, const int *JA, const int *IAU, const double *F, const double *r,
                    double *z) {
    ilu_apply(n, IA, JA, IAU, F, r, z);
}

static double dot(const double *a, const double *b, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* Restarted right-preconditioned GMRES(m), modified Gram-Schmidt, Givens
 * rotations (Saad, Alg. 9.5; the restart/Givens structure of the reference's
 * unused ParallelSparseGMRES, MATH/src/ParallelLinearAlgebra.cpp:27-278).
 * precond: 0 none, 1 block Jacobi, 2 block ILU(0).  X starts at zero. */
int orc_gmres(int n, const int *IA, const int *JA, const int *IAU, const double *A, const double *B, double *X, int m,
              int maxit, double rtol, int precond, int *iters, double *relres) {
    const size_t N = 5 * (size_t)n;
    double *F = NULL;
    if (precond == 2) {
        F = (double *)malloc(sizeof(double) * 25 * (size_t)IA[n]);
        if (orc_ilu0(n, IA, JA, IAU, A, F)) { free(F); return 2; }
    } else if (precond == 1) {
        F = (double *)malloc(sizeof(double) * 25 * (size_t)n);
        for (int i = 0; i < n; i++)
            if (inv5(A + 25 * (size_t)IAU[i], F + 25 * (size_t)i)) { free(F); return 2; }
    }
    double *V = (double *)malloc(sizeof(double) * N * (m + 1));
    double *w = (double *)malloc(sizeof(double) * N), *z = (double *)malloc(sizeof(double) * N);
    double *H = (double *)calloc((size_t)(m + 1) * m, sizeof(double));
    double *cs = (double *)malloc(sizeof(double) * m), *sn = (double *)malloc(sizeof(double) * m);
    double *g = (double *)malloc(sizeof(double) * (m + 1)), *y = (double *)malloc(sizeof(double) * m);
    memset(X, 0, sizeof(double) * N);
    double bn = sqrt(dot(B, B, N));
    int tot = 0, rc = 1;
    if (bn == 0.0) { *iters = 0; *relres = 0.0; rc = 0; goto done; }
#define PREC(in, out)                                                                         \
    do {                                                                                      \
        if (precond == 2) ilu_apply(n, IA, JA, IAU, F, in, out);                              \
        else if (precond == 1)                                                                \
            for (int i_ = 0; i_ < n; i_++)                                                    \
                for (int a_ = 0; a_ < 5; a_++) {                                              \
                    double s_ = 0.0;                                                          \
                    for (int b_ = 0; b_ < 5; b_++) s_ += F[25 * (size_t)i_ + 5 * a_ + b_] * in[5 * (size_t)i_ + b_]; \
                    out[5 * (size_t)i_ + a_] = s_;                                            \
                }                                                                             \
        else memcpy(out, in, sizeof(double) * N);                                             \
    } while (0)
    while (tot < maxit) {
        orc_bspmv(n, IA, JA, A, X, w);
        for (size_t i = 0; i < N; i++) w[i] = B[i] - w[i];
        double beta = sqrt(dot(w, w, N));
        *relres = beta / bn;
        if (*relres <= rtol) { rc = 0; break; }
        for (size_t i = 0; i < N; i++) V[i] = w[i] / beta;
        for (int i = 0; i <= m; i++) g[i] = 0.0;
        g[0] = beta;
        int j = 0;
        for (; j < m && tot < maxit; j++, tot++) {
            PREC((V + N * j), z);
            orc_bspmv(n, IA, JA, A, z, w);
            for (int i = 0; i <= j; i++) {
                double h = dot(w, V + N * i, N);
                H[(size_t)i * m + j] = h;
                for (size_t q = 0; q < N; q++) w[q] -= h * V[N * i + q];
            }
            double hn = sqrt(dot(w, w, N));
            H[(size_t)(j + 1) * m + j] = hn;
            if (hn > 0.0)
                for (size_t q = 0; q < N; q++) V[N * (j + 1) + q] = w[q] / hn;
            for (int i = 0; i < j; i++) {
                double t = cs[i] * H[(size_t)i * m + j] + sn[i] * H[(size_t)(i + 1) * m + j];
                H[(size_t)(i + 1) * m + j] = -sn[i] * H[(size_t)i * m + j] + cs[i] * H[(size_t)(i + 1) * m + j];
                H[(size_t)i * m + j] = t;
            }
            double den = hypot(H[(size_t)j * m + j], H[(size_t)(j + 1) * m + j]);
            cs[j] = H[(size_t)j * m + j] / den;
            sn[j] = H[(size_t)(j + 1) * m + j] / den;
            H[(size_t)j * m + j] = den;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            if (fabs(g[j + 1]) / bn <= rtol || hn == 0.0) { j++; tot++; break; }
        }
        for (int i = j - 1; i >= 0; i--) {
            double s = g[i];
            for (int k = i + 1; k < j; k++) s -= H[(size_t)i * m + k] * y[k];
            y[i] = s / H[(size_t)i * m + i];
        }
        for (size_t q = 0; q < N; q++) {
            double s = 0.0;
            for (int i = 0; i < j; i++) s += y[i] * V[N * i + q];
            w[q] = s;
        }
        PREC(w, z);
        for (size_t q = 0; q < N; q++) X[q] += z[q];
    }
    orc_bspmv(n, IA, JA, A, X, w);
    for (size_t i = 0; i < N; i++) w[i] = B[i] - w[i];
    *relres = sqrt(dot(w, w, N)) / bn;
    if (*relres <= rtol) rc = 0;
    *iters = tot;
#undef PREC
done:
    free(V); free(w); free(z); free(H); free(cs); free(sn); free(g); free(y);
    if (F) free(F);
    return rc;
}
