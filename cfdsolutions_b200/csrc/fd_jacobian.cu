// Finite-difference Roe Jacobian (Compute_Jacobian_FiniteDifference_Roe,
// Euler3D/src/Roe_Jacobian.cpp:236-775).
//
// Every block is a difference quotient of the reference's matrix-form Roe flux
// (Compute_RoeFlux, Euler3D/src/Roe_Fluxes.cpp:552-870, first-order states):
// central (coefficient 1/2, fluxes at +-eps), forward or backward (one side
// against the unperturbed flux), or alternating forward / backward by
// iteration parity, with eps = 1e-8.  Interior edges give the four blocks of
// their two nodes; boundary edges give the diagonal block of their node, always
// by central differences, the ghost state being rebuilt for every perturbed
// interior state by the older characteristic boundary condition
// (Compute_Characteristic_BoundaryCondition, Euler3D/src/BC.cpp:33-380).
//
// A difference quotient amplifies any change in the last bits of the flux by
// |F| / (eps |dF|), so this file is compiled without floating-point
// contraction (-fmad=false): each expression rounds exactly as the
// reference's scalar code, and the flux evaluations, hence the quotients, are
// the reference's bit for bit.  Off-diagonal blocks are written once per edge;
// the diagonal blocks are summed per row in a fixed order (no atomics).
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>

#include "ctx.cuh"
#include "kernels.cuh"

namespace cfd {

namespace {

constexpr double kFdEps = 1.0e-8;  // Roe_Jacobian.cpp:249

struct RefFace {
    double rho, u, v, w, et, q2, p, ht, c, ubar;
};

// Compute_EOS_Variables_Face, generic non-dimensionalisation, conservative
// variables (Euler3D/src/Material.cpp:216-240), in the reference's order, with
// the stiffened-gas terms (exact zeros at pinf = 0).
__device__ void ref_face(const double q[5], double nx, double ny, double nz, const Flow &f, RefFace &s) {
    const double gamma = f.gamma;
    s.rho = q[0];
    s.u = q[1] / s.rho;
    s.v = q[2] / s.rho;
    s.w = q[3] / s.rho;
    s.et = q[4] / s.rho;
    s.q2 = s.u * s.u + s.v * s.v + s.w * s.w;
    s.p = (gamma - 1.0) * (s.rho * s.et - 0.5 * s.rho * s.q2) - f.gpinf;
    s.ht = (s.rho * s.et + s.p) / s.rho;
    s.c = sqrt((gamma * (s.p + f.pinf)) / s.rho);
    s.ubar = s.u * nx + s.v * ny + s.w * nz;
}

// Out = A B for 5x5 row-major matrices, accumulated from 0 in k order
// (MC_Matrix_Mul_Matrix, MATH/src/MC_Iterative_Jacobi.c:192-207).
__device__ void mat5_mul(const double *A, const double *B, double *Out) {
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            double s = 0.0;
            for (int k = 0; k < 5; k++) s += A[i * 5 + k] * B[k * 5 + j];
            Out[i * 5 + j] = s;
        }
}

// Matrix-form Roe flux of two first-order states (Compute_RoeFlux, with its
// low-Mach-fix branch for CFD_FLUX_ROE_LMFIX): conv = 1/2 (F_L + F_R) area,
// diss = -1/2 (M P |Lambda| Pinv Minv) (Q_R - Q_L) area.
__device__ void ref_roe_flux(const double qL[5], const double qR[5], double nx, double ny, double nz, double area,
                             const Flow &f, double conv[5], double diss[5]) {
    const double g = f.gamma;
    RefFace L, R;
    ref_face(qL, nx, ny, nz, f, L);
    ref_face(qR, nx, ny, nz, f, R);
    double fl[5], fr[5];
    fl[0] = L.rho * L.ubar;
    fl[1] = L.u * fl[0] + L.p * nx;
    fl[2] = L.v * fl[0] + L.p * ny;
    fl[3] = L.w * fl[0] + L.p * nz;
    fl[4] = L.ht * fl[0];
    fr[0] = R.rho * R.ubar;
    fr[1] = R.u * fr[0] + R.p * nx;
    fr[2] = R.v * fr[0] + R.p * ny;
    fr[3] = R.w * fr[0] + R.p * nz;
    fr[4] = R.ht * fr[0];
    const double rho = sqrt(R.rho * L.rho);
    const double sigma = rho / (L.rho + rho);
    const double u = L.u + sigma * (R.u - L.u);
    const double v = L.v + sigma * (R.v - L.v);
    const double w = L.w + sigma * (R.w - L.w);
    const double ht = L.ht + sigma * (R.ht - L.ht);
    // Get_SpeedSound(u, v, w, ht) (Material.cpp:939-960)
    const double phi = 0.5 * (g - 1.0) * (u * u + v * v + w * w);
    const double c = sqrt((g - 1.0) * ht - phi);
    const double ubar = u * nx + v * ny + w * nz;
    // Compute_Transformation_Conservative_To_RUP / RUP_To_Conservative (Material.cpp:1172-1300)
    double M[25] = {1.0, 0.0, 0.0, 0.0, 0.0,  u, rho, 0.0, 0.0, 0.0,  v, 0.0, rho, 0.0, 0.0,
                    w, 0.0, 0.0, rho, 0.0,  phi / (g - 1.0), rho * u, rho * v, rho * w, 1.0 / (g - 1.0)};
    double Minv[25] = {1.0, 0.0, 0.0, 0.0, 0.0,  -u / rho, 1.0 / rho, 0.0, 0.0, 0.0,
                       -v / rho, 0.0, 1.0 / rho, 0.0, 0.0,  -w / rho, 0.0, 0.0, 1.0 / rho, 0.0,
                       phi, -u * (g - 1.0), -v * (g - 1.0), -w * (g - 1.0), (g - 1.0)};
    // eigenvectors in the (rho, u, v, w, p) variables (Roe_Fluxes.cpp:664-719)
    double P[25] = {nx, ny, nz, rho / c, rho / c,  0.0, -nz, ny, nx, -nx,  nz, 0.0, -nx, ny, -ny,
                    -ny, nx, 0.0, nz, -nz,  0.0, 0.0, 0.0, rho * c, rho * c};
    double Pinv[25] = {nx, 0.0, nz, -ny, -nx / (c * c),  ny, -nz, 0.0, nx, -ny / (c * c),
                       nz, ny, -nx, 0.0, -nz / (c * c),  0.0, 0.5 * nx, 0.5 * ny, 0.5 * nz, 1.0 / (2.0 * rho * c),
                       0.0, -0.5 * nx, -0.5 * ny, -0.5 * nz, 1.0 / (2.0 * rho * c)};
    double T[25], Tinv[25], A[25], E[25];
    mat5_mul(M, P, T);
    for (int k = 0; k < 25; k++) E[k] = 0.0;
    // Roe_EntropyFix (Euler3D/src/Roe_EntropyFix.cpp:19-59)
    E[0] = fabs(ubar);
    E[6] = E[0];
    E[12] = E[0];
    if (f.entropy_fix == 1) {
        double lL = L.ubar + L.c, lR = R.ubar + R.c, l = ubar + c;
        double a = l - lL, b = lR - l;
        double m = a > b ? a : b;
        double eps = 4.0 * (0.0 > m ? 0.0 : m);
        E[18] = fabs(l) < eps ? (l * l + eps * eps) / (2.0 * eps) : fabs(l);
        lL = L.ubar - L.c;
        lR = R.ubar - R.c;
        l = ubar - c;
        a = l - lL;
        b = lR - l;
        m = a > b ? a : b;
        eps = 4.0 * (0.0 > m ? 0.0 : m);
        E[24] = fabs(l) < eps ? (l * l + eps * eps) / (2.0 * eps) : fabs(l);
    } else {
        E[18] = fabs(ubar + c);
        E[24] = fabs(ubar - c);
    }
    if (f.lmfix) {
        // PRECOND_METHOD_ROE_LMFIX branch of Compute_RoeFlux (Roe_Fluxes.cpp:641-685, :820-848):
        // fix = min(1, (|u.n| + |u.t1| + |u.t2|) / c) at the Roe average; |A| acts on the
        // density and pressure jumps, and the velocity jump enters through fix * (du.n)
        double nmax = fabs(nx);
        int mc = 1;
        if (nmax < fabs(ny)) { nmax = fabs(ny); mc = 2; }
        if (nmax < fabs(nz)) { nmax = fabs(nz); mc = 3; }
        double t1[3] = {1.0, 1.0, 1.0};
        if (mc == 1) t1[0] = -(ny + nz) / nx;
        else if (mc == 2) t1[1] = -(nx + nz) / ny;
        else t1[2] = -(nx + ny) / nz;
        double mg = sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
        if (mg > 1.0e-20) { t1[0] = t1[0] / mg; t1[1] = t1[1] / mg; t1[2] = t1[2] / mg; }
        const double ub1 = u * t1[0] + v * t1[1] + w * t1[2];
        double t2[3] = {+t1[1] * nz - t1[2] * ny, -t1[0] * nz + t1[2] * nx, +t1[0] * ny - t1[1] * nx};
        mg = sqrt(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
        if (mg > 1.0e-20) { t2[0] = t2[0] / mg; t2[1] = t2[1] / mg; t2[2] = t2[2] / mg; }
        const double ub2 = u * t2[0] + v * t2[1] + w * t2[2];
        double mach = fabs(ubar) + fabs(ub1) + fabs(ub2);
        mach = mach / c;
        const double fix = mach < 1.0 ? mach : 1.0;
        mat5_mul(E, Pinv, Tinv);
        mat5_mul(T, Tinv, A);  // M P |Lambda| Pinv
        const double d1[5] = {R.rho - L.rho, 0.0, 0.0, 0.0, R.p - L.p};
        double fa[5], dw[5], md[5];
        for (int i = 0; i < 5; i++) {
            fa[i] = 0.0;
            for (int k = 0; k < 5; k++) fa[i] += A[i * 5 + k] * d1[k];
        }
        const double fixUn = fix * ((R.u - L.u) * nx + (R.v - L.v) * ny + (R.w - L.w) * nz);
        const double ap = fabs(ubar + c), am = fabs(ubar - c);
        dw[0] = (0.5 * rho * fixUn * (ap - am)) / c;
        dw[1] = fabs(ubar) * ((R.u - L.u) - fixUn * nx) + 0.5 * nx * fixUn * (ap + am);
        dw[2] = fabs(ubar) * ((R.v - L.v) - fixUn * ny) + 0.5 * ny * fixUn * (ap + am);
        dw[3] = fabs(ubar) * ((R.w - L.w) - fixUn * nz) + 0.5 * nz * fixUn * (ap + am);
        dw[4] = 0.5 * rho * c * fixUn * (ap - am);
        for (int i = 0; i < 5; i++) {
            md[i] = 0.0;
            for (int k = 0; k < 5; k++) md[i] += M[i * 5 + k] * dw[k];
        }
        for (int i = 0; i < 5; i++) {
            conv[i] = 0.5 * (fl[i] + fr[i]) * area;
            diss[i] = -0.5 * (fa[i] + md[i]) * area;
        }
        return;
    }
    mat5_mul(Pinv, Minv, Tinv);
    mat5_mul(E, Tinv, A);
    mat5_mul(T, A, Tinv);  // |A| = T (|Lambda| Pinv Minv)
    double dq[5];
    for (int k = 0; k < 5; k++) dq[k] = qR[k] - qL[k];
    for (int i = 0; i < 5; i++) {
        double s = 0.0;
        for (int k = 0; k < 5; k++) s += Tinv[i * 5 + k] * dq[k];
        conv[i] = 0.5 * (fl[i] + fr[i]) * area;
        diss[i] = -0.5 * s * area;
    }
}

// Ghost state of the older characteristic boundary condition
// (Compute_Characteristic_BoundaryCondition, Euler3D/src/BC.cpp:33-380) for
// interior state qi and current ghost qg.  Sets err bits where the reference
// aborts (unclassifiable far field, negative pressure).
__device__ void old_characteristic_bc(const double qi[5], const double qg[5], double nx, double ny, double nz,
                                      int type, int iteration, const Flow &f, double qb[5], int *err) {
    const double g = f.gamma;
    RefFace I, Z;
    ref_face(qi, nx, ny, nz, f, I);
    double q0[5];
    for (int k = 0; k < 5; k++) q0[k] = 0.5 * (qi[k] + qg[k]);
    ref_face(q0, nx, ny, nz, f, Z);
    const double l1 = Z.ubar, l4 = l1 + Z.c, l5 = l1 - Z.c;
    int inst = type;
    switch (type) {
        case 0: inst = 0; break;
        case 1:
            if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 10;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 11;
            else if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 9;
            else if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 8;
            else { atomicOr(err, ERR_BC_UNCLASSIFIED); inst = 1; }
            break;
        case 2:
            if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 4;
            else if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 6;
            else inst = fabs(l1) < Z.c ? 4 : 6;
            break;
        case 3:
            if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 5;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 7;
            else inst = fabs(l1) < Z.c ? 5 : 7;
            break;
        default: inst = type; break;  // 4-7 keep their type (the reference only warns)
    }
    double pb = f.inf_p, rb = f.inf_rho, ub = f.inf_u, vb = f.inf_v, wb = f.inf_w;
    const double rc = Z.rho * Z.c, cc = Z.c * Z.c;
    switch (inst) {
        case 0:
            pb = I.p + Z.rho * Z.c * I.ubar;
            if (iteration < f.zpg_iteration && pb + f.pinf < 0.0) pb = I.p;
            rb = I.rho + (pb - I.p) / cc;
            ub = I.u - nx * (pb - I.p) / rc;
            vb = I.v - ny * (pb - I.p) / rc;
            wb = I.w - nz * (pb - I.p) / rc;
            break;
        case 5: case 9:
            pb = inst == 5 ? f.outflow_p : f.inf_p;
            rb = I.rho + (pb - I.p) / cc;
            ub = I.u - nx * (pb - I.p) / rc;
            vb = I.v - ny * (pb - I.p) / rc;
            wb = I.w - nz * (pb - I.p) / rc;
            break;
        case 7: case 11:
            pb = I.p; rb = I.rho; ub = I.u; vb = I.v; wb = I.w;
            break;
        case 8: {
            const double temp = nx * (f.inf_u - I.u) + ny * (f.inf_v - I.v) + nz * (f.inf_w - I.w);
            pb = 0.5 * (f.inf_p + I.p - Z.rho * Z.c * temp);
            rb = f.inf_rho + (pb - f.inf_p) / cc;
            ub = f.inf_u + nx * (pb - f.inf_p) / rc;
            vb = f.inf_v + ny * (pb - f.inf_p) / rc;
            wb = f.inf_w + nz * (pb - f.inf_p) / rc;
            break;
        }
        default: break;  // 1, 4, 6, 10: freestream values
    }
    if (pb + f.pinf < 0.0) atomicOr(err, ERR_BC_NEG_PRESSURE);
    // Get_TotalEnergy (Material.cpp:1012-1021)
    double et = ub * ub + vb * vb + wb * wb;
    et = (pb + f.gpinf) / ((g - 1.0) * rb) + 0.5 * et;
    qb[0] = rb;
    qb[1] = rb * ub;
    qb[2] = rb * vb;
    qb[3] = rb * wb;
    qb[4] = rb * et;
}

// Difference quotient of one column: coef ((FP_c + FP_d) - (FM_c + FM_d)) / eps.
__device__ __forceinline__ void fd_column(const double pc[5], const double pd[5], const double mc[5],
                                          const double md[5], double coef, double *col /* stride 5 */) {
    for (int i = 0; i < 5; i++) col[i * 5] = coef * ((pc[i] + pd[i]) - (mc[i] + md[i])) / kFdEps;
}

// Interior edges: dFdL, dFdR by perturbing each of the ten states; writes
// A[L,R] = 0 + dFdR and A[R,L] = 0 - dFdL (Roe_Jacobian.cpp:291-557).
__global__ void k_fd_edges(int nedge, int64_t ldq, const double *__restrict__ Q, const int2 *__restrict__ en,
                           const double4 *__restrict__ eg, const int2 *__restrict__ eslot, Flow f, int method,
                           double *__restrict__ A) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nedge) return;
    const int2 nd = en[e];
    const double4 gm = eg[e];
    double q[2][5];
    for (int v = 0; v < 5; v++) {
        q[0][v] = Q[v * ldq + nd.x];
        q[1][v] = Q[v * ldq + nd.y];
    }
    const bool plus = method == CFD_JAC_CENTRAL || method == CFD_JAC_FORWARD;
    const bool minus = method == CFD_JAC_CENTRAL || method == CFD_JAC_BACKWARD;
    const double coef = method == CFD_JAC_CENTRAL ? 0.5 : 1.0;
    double bc[5], bd[5];
    if (!plus || !minus) ref_roe_flux(q[0], q[1], gm.x, gm.y, gm.z, gm.w, f, bc, bd);
    double d[2][25];
    for (int side = 0; side < 2; side++)
        for (int k = 0; k < 5; k++) {
            double pc[5], pd[5], mc[5], md[5];
            const double base = q[side][k];
            if (plus) {
                q[side][k] = base + kFdEps;
                ref_roe_flux(q[0], q[1], gm.x, gm.y, gm.z, gm.w, f, pc, pd);
            } else {
                for (int i = 0; i < 5; i++) { pc[i] = bc[i]; pd[i] = bd[i]; }
            }
            if (minus) {
                q[side][k] = base - kFdEps;
                ref_roe_flux(q[0], q[1], gm.x, gm.y, gm.z, gm.w, f, mc, md);
            } else {
                for (int i = 0; i < 5; i++) { mc[i] = bc[i]; md[i] = bd[i]; }
            }
            q[side][k] = base;
            fd_column(pc, pd, mc, md, coef, &d[side][k]);
        }
    const int2 sl = eslot[e];
    for (int k = 0; k < 25; k++) {
        A[(int64_t)sl.x * 25 + k] = 0.0 + d[1][k];
        A[(int64_t)sl.y * 25 + k] = 0.0 - d[0][k];
    }
}

// Boundary edges: dFdL by central differences with the ghost rebuilt for each
// perturbed interior state (Roe_Jacobian.cpp:559-774); one block per edge.
__global__ void k_fd_bedges(int nbedge, int64_t ldq, const double *__restrict__ Q, const int2 *__restrict__ bn,
                            const double4 *__restrict__ bg, const int *__restrict__ btype, Flow f, int iteration,
                            double *__restrict__ out, int *__restrict__ err) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbedge) return;
    const int2 nd = bn[b];
    const double4 gm = bg[b];
    const int type = btype[b];
    double qi[5], qg[5];
    for (int v = 0; v < 5; v++) {
        qi[v] = Q[v * ldq + nd.x];
        qg[v] = Q[v * ldq + nd.y];
    }
    double d[25];
    for (int k = 0; k < 5; k++) {
        double pc[5], pd[5], mc[5], md[5], qb[5];
        const double base = qi[k];
        qi[k] = base + kFdEps;
        old_characteristic_bc(qi, qg, gm.x, gm.y, gm.z, type, iteration, f, qb, err);
        ref_roe_flux(qi, qb, gm.x, gm.y, gm.z, gm.w, f, pc, pd);
        qi[k] = base - kFdEps;
        old_characteristic_bc(qi, qg, gm.x, gm.y, gm.z, type, iteration, f, qb, err);
        ref_roe_flux(qi, qb, gm.x, gm.y, gm.z, gm.w, f, mc, md);
        qi[k] = base;
        fd_column(pc, pd, mc, md, 0.5, &d[k]);
    }
    for (int k = 0; k < 25; k++) out[(int64_t)b * 25 + k] = d[k];
}

// Diagonal blocks and right-hand side: V/dt I + sum_j dFdL or -dFdR of the
// node's edges (= -A[j,i]) + its boundary blocks; B = -(Res [+ Res_Diss]).
__global__ void k_fd_rows(int nnode, const int *__restrict__ IA, const int *__restrict__ IAU,
                          const int *__restrict__ tslot, const int *__restrict__ n2b_ptr, const int *__restrict__ n2b,
                          const double *__restrict__ fdb, const double *__restrict__ vol, const double *__restrict__ dt,
                          const double *__restrict__ res, const double *__restrict__ resd, int add_time,
                          int include_diss, double *__restrict__ A, double *__restrict__ B) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnode) return;
    double D[25];
    for (int k = 0; k < 25; k++) D[k] = 0.0;
    if (add_time)
        for (int k = 0; k < 5; k++) D[k * 6] = vol[i] / dt[i];
    const int dg = IAU[i];
    for (int k = IA[i]; k < IA[i + 1]; k++) {
        if (k == dg) continue;
        const double *blk = A + (int64_t)tslot[k] * 25;
        for (int m = 0; m < 25; m++) D[m] -= blk[m];
    }
    for (int k = n2b_ptr[i]; k < n2b_ptr[i + 1]; k++) {
        const double *blk = fdb + (int64_t)n2b[k] * 25;
        for (int m = 0; m < 25; m++) D[m] += blk[m];
    }
    for (int m = 0; m < 25; m++) A[(int64_t)dg * 25 + m] = D[m];
    for (int v = 0; v < 5; v++) {
        double r = res[v * (int64_t)nnode + i];
        if (include_diss) r += resd[v * (int64_t)nnode + i];
        B[(int64_t)i * 5 + v] = -r;
    }
}

}  // namespace

}  // namespace cfd

using namespace cfd;

extern "C" int cfd_jacobian_fd(cfd_ctx *c, int add_time, int include_diss, int method, int iteration) {
    if (!c || !c->has_mesh) { set_error("cfd_jacobian_fd: no mesh"); return CFD_ERR_STATE; }
    if (method < CFD_JAC_CENTRAL || method > CFD_JAC_ALTERNATE) {
        set_error("cfd_jacobian_fd: method must be CFD_JAC_CENTRAL, _FORWARD, _BACKWARD or _ALTERNATE");
        return CFD_ERR_ARG;
    }
    if (c->params.variables != CFD_VARS_CONSERVATIVE) {
        // Euler3D's difference quotients perturb conservative states (Roe_Jacobian.cpp:236-775)
        set_error("cfd_jacobian_fd: conservative variables only");
        return CFD_ERR_UNSUPPORTED;
    }
    if (c->params.flux_scheme != CFD_FLUX_ROE && c->params.flux_scheme != CFD_FLUX_ROE_LMFIX) {
        // Compute_Jacobian_FiniteDifference_Roe differences the Roe flux (Roe_Jacobian.cpp:236)
        set_error("cfd_jacobian_fd: the finite-difference Jacobian is defined for the Roe flux (with or "
                  "without the low-Mach fix)");
        return CFD_ERR_UNSUPPORTED;
    }
    CFD_CUDA(cudaSetDevice(c->device));
    if (method == CFD_JAC_ALTERNATE)  // Roe_Jacobian.cpp:282-287
        method = iteration % 2 == 0 ? CFD_JAC_FORWARD : CFD_JAC_BACKWARD;
    CFD_CUDA(c->A64.alloc((size_t)c->nnzb * 25));
    CFD_CUDA(c->B.alloc((size_t)c->nnode * 5));
    CFD_CUDA(c->X.alloc((size_t)c->nnode * 5));
    CFD_CUDA(c->work.alloc(std::max<size_t>(c->work.n, (size_t)25 * std::max(c->nbedge, 1))));
    if (c->nedge)
        k_fd_edges<<<grid_for(c->nedge, 64), 64, 0, c->stream>>>(c->nedge, c->ldq, c->Q.p, c->edge_nodes.p,
                                                                   c->edge_geo.p, c->eslot.p, c->flow, method,
                                                                   c->A64.p);
    CFD_LAUNCH_CHECK();
    if (c->nbedge)
        k_fd_bedges<<<grid_for(c->nbedge, 64), 64, 0, c->stream>>>(c->nbedge, c->ldq, c->Q.p, c->bedge_nodes.p,
                                                                     c->bedge_geo.p, c->bedge_type.p, c->flow,
                                                                     iteration, c->work.p, c->err.p);
    CFD_LAUNCH_CHECK();
    k_fd_rows<<<grid_for(c->nnode, 128), 128, 0, c->stream>>>(c->nnode, c->IA.p, c->IAU.p, c->tslot.p, c->n2b_ptr.p,
                                                                c->n2b.p, c->work.p, c->cvol.p, c->dt.p, c->res.p,
                                                                c->resd.p, add_time, include_diss, c->A64.p, c->B.p);
    CFD_LAUNCH_CHECK();
    c->a_precision = CFD_PREC_FP64;
    c->a64_valid = true;
    c->has_system = true;
    c->pc_valid = false;
    return check_device_error(c);
}
