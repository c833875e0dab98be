// Device physics of the node-centred edge-based Euler path: ideal-gas EOS in
// the generic non-dimensionalisation (or the stiffened gas
// p = (gamma - 1) rho e - gamma pinf, which is the ideal gas at pinf = 0), Roe / HLLC / AUSM+ edge fluxes,
// characteristic ghost states and the approximate Roe flux Jacobian.
// The state holds either the conservative variables (rho, rho u, rho v, rho w,
// rho et), as Euler3D with VARIABLE_TYPE=VARIABLE_CONSERVATIVE, or (rho, u, v,
// w, p), as MPFLOW3D with VARIABLE_RUP (Flow::rup): the face properties, ghost
// states and Jacobian columns follow the state's variables, the fluxes are
// the conservation-law fluxes either way.
#pragma once

#include <cuda_runtime.h>

#include "../../include/cfd_b200.h"

namespace cfd {

// Flow constants of one iteration (ComputeFarFieldCondition,
// Euler3D/src/Material.cpp:185-210) and the options the kernels branch on.
struct Flow {
    double gamma, gm1, inv_gm1;
    double inf_rho, inf_u, inf_v, inf_w, inf_p, inf_et, inf_c, inf_mach;
    double outflow_p;
    double pinf, gpinf;   // stiffened-gas constant and gamma * pinf (both 0 for the ideal gas)
    double frac;          // 0.5 for LIMITER_ORDER_SECOND else 0 (HigherOrderReconstructQ.cpp:27-29)
    double venkat_eps_k3; // K^3 (Limiters.cpp:205)
    int flux;             // CFD_FLUX_*
    int order;            // CFD_ORDER_*
    int limiter;          // CFD_LIMITER_*
    int limiter_smooth;
    int entropy_fix;
    int zpg_iteration, iteration;
    int lmfix;            // Roe low-Mach fix and the preconditioned characteristic BC (CFD_FLUX_ROE_LMFIX)
    // preconditioned Roe (CFD_FLUX_ROE_PRECOND): CFD_PRECOND_* method and type,
    // reference Mach and the pressure its subsonic outflow imposes
    int pc_method, pc_type;
    double pc_mach, pc_outflow_p;
    int rup;              // state in (rho, u, v, w, p) (CFD_VARS_RUP), else conservative
};

struct Face {
    double rho, u, v, w, p, ht, ubar, c;
};

// Whether the state holds (rho, u, v, w, p): V = 0 (conservative) or 1 (RUP)
// as a compile-time constant of the caller, or V = -1, read from f.rup.
template <int V>
__device__ __forceinline__ bool vars_rup(const Flow &f) {
    if constexpr (V < 0) return f.rup != 0;
    else return V == 1;
}

// Compute_EOS_Variables_Face, conservative branch (Euler3D/src/Material.cpp:216-248),
// with the stiffened-gas terms: p = (gamma - 1)(rho et - rho q^2 / 2) - gamma pinf and
// c^2 = gamma (p + pinf) / rho.  At pinf = 0 both added terms are exact zeros, so
// the ideal-gas results are bit-identical.  c is only formed when `want_c`.
// RUP states (MPFLOW3D Material_Get_Properties, VARIABLE_RUP branch,
// MPFLOW3D/src/Material.cpp:591-599) take rho, u, v, w, p as stored and
// ht = gamma (p + pinf) / ((gamma - 1) rho) + q^2 / 2.
template <int V = -1>
__device__ __forceinline__ void eos_face(const double q[5], double nx, double ny, double nz, const Flow &f,
                                         bool want_c, Face &s) {
    s.rho = q[0];
    const double ri = 1.0 / s.rho;
    if (vars_rup<V>(f)) {
        s.u = q[1];
        s.v = q[2];
        s.w = q[3];
        s.p = q[4];
        s.ht = f.gamma * f.inv_gm1 * (s.p + f.pinf) * ri + 0.5 * (s.u * s.u + s.v * s.v + s.w * s.w);
    } else {
        s.u = q[1] * ri;
        s.v = q[2] * ri;
        s.w = q[3] * ri;
        const double q2 = s.u * s.u + s.v * s.v + s.w * s.w;
        s.p = f.gm1 * (q[4] - 0.5 * s.rho * q2) - f.gpinf;
        s.ht = (q[4] + s.p) * ri;
    }
    s.ubar = s.u * nx + s.v * ny + s.w * nz;
    s.c = want_c ? sqrt(f.gamma * (s.p + f.pinf) * ri) : 0.0;
}

// A state from (rho, u, v, w, p) in the state's variables; the conservative
// total energy by Get_TotalEnergy (Material.cpp:1012-1040),
// rho e = (p + gamma pinf) / (gamma - 1).
__device__ __forceinline__ void store_state(double rho, double u, double v, double w, double p, const Flow &f,
                                            double q[5]) {
    if (f.rup) {
        q[0] = rho; q[1] = u; q[2] = v; q[3] = w; q[4] = p;
        return;
    }
    const double et = (p + f.gpinf) / (f.gm1 * rho) + 0.5 * (u * u + v * v + w * w);
    q[0] = rho;
    q[1] = rho * u;
    q[2] = rho * v;
    q[3] = rho * w;
    q[4] = rho * et;
}

// dQ_cons/d(rho,u,v,w,p) at (rho, u, v, w) (Compute_Transformation_Conservative_To_RUP,
// MPFLOW3D/src/Material.cpp:1172-1236), row-major; the same for either gas.
__device__ __forceinline__ void dcons_drup(double rho, double u, double v, double w, const Flow &f, double M[25]) {
    M[0] = 1.0;  M[1] = 0.0;     M[2] = 0.0;     M[3] = 0.0;     M[4] = 0.0;
    M[5] = u;    M[6] = rho;     M[7] = 0.0;     M[8] = 0.0;     M[9] = 0.0;
    M[10] = v;   M[11] = 0.0;    M[12] = rho;    M[13] = 0.0;    M[14] = 0.0;
    M[15] = w;   M[16] = 0.0;    M[17] = 0.0;    M[18] = rho;    M[19] = 0.0;
    M[20] = 0.5 * (u * u + v * v + w * w);
    M[21] = rho * u; M[22] = rho * v; M[23] = rho * w; M[24] = f.inv_gm1;
}

// Kermani entropy fix on the acoustic eigenvalues (Euler3D/src/Roe_EntropyFix.cpp:19-59).
__device__ __forceinline__ void roe_entropy_fix(double ubar_L, double c_L, double ubar_R, double c_R,
                                                double ubar, double c, double &E0, double &E1, double &E2) {
    E0 = fabs(ubar);
    // lambda_4 = ubar + c
    {
        double lL = ubar_L + c_L, lR = ubar_R + c_R, l = ubar + c;
        double eps = 4.0 * fmax(0.0, fmax(l - lL, lR - l));
        E1 = (fabs(l) < eps) ? (l * l + eps * eps) / (2.0 * eps) : fabs(l);
    }
    // lambda_5 = ubar - c
    {
        double lL = ubar_L - c_L, lR = ubar_R - c_R, l = ubar - c;
        double eps = 4.0 * fmax(0.0, fmax(l - lL, lR - l));
        E2 = (fabs(l) < eps) ? (l * l + eps * eps) / (2.0 * eps) : fabs(l);
    }
}

// Roe flux of Compute_Flux_Roe_Optimized (Euler3D/src/FluxTest.cpp:3026-3200):
// central part 0.5 (F_L + F_R) area and dissipation -0.5 |A| dQ area with
// |A| dQ = M_{cons<-RUP} * dw, dw in closed form (FluxTest.cpp:3180-3190).
// Returns the largest |eigenvalue| (for the time step) and the three
// eigenvalue magnitudes |ubar|, |ubar+c|, |ubar-c| in lam[3].
// c2_out, when not null, receives the Roe-averaged c^2 (see edge_flux).
template <bool LMFIX, int V = -1>
__device__ __forceinline__ double roe_flux(const double qL[5], const double qR[5], double nx, double ny,
                                           double nz, double area, const Flow &f, double conv[5],
                                           double diss[5], double lam[3], double *c2_out = nullptr) {
    Face L, R;
    const bool want_c = f.entropy_fix != 0;
    eos_face<V>(qL, nx, ny, nz, f, want_c, L);
    eos_face<V>(qR, nx, ny, nz, f, want_c, R);

    const double mL = L.rho * L.ubar, mR = R.rho * R.ubar;
    const double ha = 0.5 * area;
    conv[0] = ha * (mL + mR);
    conv[1] = ha * ((L.u * mL + L.p * nx) + (R.u * mR + R.p * nx));
    conv[2] = ha * ((L.v * mL + L.p * ny) + (R.v * mR + R.p * ny));
    conv[3] = ha * ((L.w * mL + L.p * nz) + (R.w * mR + R.p * nz));
    conv[4] = ha * (L.ht * mL + R.ht * mR);

    // Roe averages (FluxTest.cpp:3107-3115); rho and 1/rho, c and 1/c from one
    // reciprocal square root each
    const double rr = R.rho * L.rho;
    const double rho_i = rsqrt(rr);
    const double rho = rr * rho_i;
    const double sigma = rho / (L.rho + rho);
    const double u = L.u + sigma * (R.u - L.u);
    const double v = L.v + sigma * (R.v - L.v);
    const double w = L.w + sigma * (R.w - L.w);
    const double ht = L.ht + sigma * (R.ht - L.ht);
    const double q2 = u * u + v * v + w * w;
    // Get_SpeedSound(u,v,w,ht), generic non-dimensionalisation (Material.cpp:939-960)
    const double c2 = f.gm1 * ht - 0.5 * f.gm1 * q2;
    if (c2_out) *c2_out = c2;
    const double ci = rsqrt(c2);
    const double c = c2 * ci;
    const double ubar = u * nx + v * ny + w * nz;

    double E0, E1, E2;
    if (f.entropy_fix) {
        roe_entropy_fix(L.ubar, L.c, R.ubar, R.c, ubar, c, E0, E1, E2);
    } else {
        E0 = fabs(ubar);
        E1 = fabs(ubar + c);
        E2 = fabs(ubar - c);
    }
    lam[0] = E0;
    lam[1] = E1;
    lam[2] = E2;

    const double drho = R.rho - L.rho, du = R.u - L.u, dv = R.v - L.v, dw_ = R.w - L.w, dp = R.p - L.p;
    double dU = du * nx + dv * ny + dw_ * nz;
    if (LMFIX) {
        // Low-Mach fix (Compute_Flux_Roe_LMFIX, Euler3D/src/FluxTest.cpp:2929-2966): the normal
        // velocity jump scaled by min(1, (|u.n| + |u.t1| + |u.t2|) / c), t1 from the largest normal
        // component, t2 = t1 x n, both normalised
        double nmax = fabs(nx);
        int mc = 1;
        if (nmax < fabs(ny)) { nmax = fabs(ny); mc = 2; }
        if (nmax < fabs(nz)) { nmax = fabs(nz); mc = 3; }
        double a0 = 1.0, a1 = 1.0, a2 = 1.0;
        if (mc == 1) a0 = -(ny + nz) / nx;
        else if (mc == 2) a1 = -(nx + nz) / ny;
        else a2 = -(nx + ny) / nz;
        double m1 = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
        if (m1 > 1.0e-20) { a0 = a0 / m1; a1 = a1 / m1; a2 = a2 / m1; }
        const double ub1 = u * a0 + v * a1 + w * a2;
        double b0 = a1 * nz - a2 * ny, b1 = -a0 * nz + a2 * nx, b2 = a0 * ny - a1 * nx;
        const double m2 = sqrt(b0 * b0 + b1 * b1 + b2 * b2);
        if (m2 > 1.0e-20) { b0 = b0 / m2; b1 = b1 / m2; b2 = b2 / m2; }
        const double ub2 = u * b0 + v * b1 + w * b2;
        const double mach = (fabs(ubar) + fabs(ub1) + fabs(ub2)) / c;
        dU = (mach < 1.0 ? mach : 1.0) * dU;
    }
    const double Es = E1 + E2 - 2.0 * E0;
    const double Ed = E1 - E2;
    const double t1 = 0.5 * dU * Es;
    const double t2 = Ed * dp * (0.5 * ci) * rho_i;
    const double w0 = E0 * drho + Es * dp * (0.5 * ci * ci) + rho * Ed * dU * (0.5 * ci);
    const double w1 = E0 * du + nx * t1 + nx * t2;
    const double w2 = E0 * dv + ny * t1 + ny * t2;
    const double w3 = E0 * dw_ + nz * t1 + nz * t2;
    const double w4 = 0.5 * dp * (E1 + E2) + 0.5 * rho * c * dU * Ed;
    // M = dQ_cons/dq_RUP (Compute_Transformation_Conservative_To_RUP, Material.cpp:1172-1236)
    const double hd = -0.5 * area;
    diss[0] = hd * w0;
    diss[1] = hd * (u * w0 + rho * w1);
    diss[2] = hd * (v * w0 + rho * w2);
    diss[3] = hd * (w * w0 + rho * w3);
    diss[4] = hd * (0.5 * q2 * w0 + rho * (u * w1 + v * w2 + w * w3) + w4 * f.inv_gm1);
    return fmax(E0, fmax(E1, E2));
}

// Ghost state of the characteristic boundary condition
// (Compute_Characteristic_BoundaryCondition_New, Euler3D/src/BC.cpp:381-677),
// conservative variables.  Returns 0 on success, 1 on negative pressure,
// 2 when the far-field case cannot be classified (the reference aborts).
__device__ __forceinline__ int characteristic_bc(const double qI[5], const double qG[5], double nx, double ny,
                                                 double nz, int bc_type, const Flow &f, double qB[5]) {
    Face I, G, O;
    eos_face(qI, nx, ny, nz, f, true, I);
    eos_face(qG, nx, ny, nz, f, true, G);
    double q0[5];
    for (int k = 0; k < 5; k++) q0[k] = 0.5 * (qI[k] + qG[k]);
    eos_face(q0, nx, ny, nz, f, true, O);
    const double l1 = O.ubar, l4 = O.ubar + O.c, l5 = O.ubar - O.c;
    double p_b = f.inf_p, rho_b = f.inf_rho, u_b = f.inf_u, v_b = f.inf_v, w_b = f.inf_w;
    int inst;
    int status = 0;
    // case selection (BC.cpp:428-560); values of the BC_TYPE enum
    switch (bc_type) {
        case 0: inst = 0; break;  // Euler wall
        case 1:                   // far field
            if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 10;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 11;
            else if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 9;
            else if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 8;
            else { inst = 1; status = 2; }
            break;
        case 2:  // inflow
            if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 4;
            else if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 6;
            else inst = (fabs(l1) < O.c) ? 4 : 6;
            break;
        case 3:  // outflow
            if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 5;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 7;
            else inst = (fabs(l1) < O.c) ? 5 : 7;
            break;
        case 4: case 5: case 6: case 7: inst = bc_type; break;
        default: inst = -1; status = 2; break;
    }
    const double rc = O.rho * O.c, c2 = O.c * O.c;
    switch (inst) {
        case 0: {  // Euler wall (BC.cpp:582-594)
            p_b = I.p + rc * I.ubar;
            if (f.iteration < f.zpg_iteration && p_b + f.pinf < 0.0) p_b = I.p;
            const double dp = p_b - I.p;
            rho_b = I.rho + dp / c2;
            u_b = I.u - nx * dp / rc;
            v_b = I.v - ny * dp / rc;
            w_b = I.w - nz * dp / rc;
        } break;
        case 4: case 6: case 10: case 1: break;  // freestream values
        case 5: case 7:
            // the preconditioned characteristic BC (used with the low-Mach fix,
            // BC.cpp:1229-1236) keeps the freestream values for these two
            if (f.lmfix) break;
            if (inst == 7) { p_b = I.p; rho_b = I.rho; u_b = I.u; v_b = I.v; w_b = I.w; break; }
            [[fallthrough]];
        case 9: {                                 // subsonic outflow / far-field subsonic outflow
            p_b = (inst == 5) ? f.outflow_p : f.inf_p;
            const double dp = p_b - I.p;
            rho_b = I.rho + dp / c2;
            u_b = I.u - nx * dp / rc;
            v_b = I.v - ny * dp / rc;
            w_b = I.w - nz * dp / rc;
        } break;
        case 11:  // far-field supersonic outflow: extrapolate
            p_b = I.p; rho_b = I.rho; u_b = I.u; v_b = I.v; w_b = I.w;
            break;
        case 8: {  // far-field subsonic inflow (BC.cpp:621-628)
            const double t = nx * (f.inf_u - I.u) + ny * (f.inf_v - I.v) + nz * (f.inf_w - I.w);
            p_b = 0.5 * (f.inf_p + I.p - rc * t);
            const double dp = p_b - f.inf_p;
            rho_b = f.inf_rho + dp / c2;
            u_b = f.inf_u + nx * dp / rc;
            v_b = f.inf_v + ny * dp / rc;
            w_b = f.inf_w + nz * dp / rc;
        } break;
        default: break;
    }
    if (p_b + f.pinf < 0.0) status = status ? status : 1;
    store_state(rho_b, u_b, v_b, w_b, p_b, f, qB);
    return status;
}

// Conservative Euler flux Jacobian dF.n/dQ (ConservativeEulerFluxJacobian,
// Euler3D/src/CompressibleUtils.cpp:558-609).  J row-major [5][5].  The
// stiffened gas only shifts p (dp/dQ is unchanged), so only ht carries gpinf.
__device__ __forceinline__ void euler_flux_jacobian(const double q[5], double nx, double ny, double nz,
                                                    double g, double gpinf, double J[25]) {
    const double rho = q[0], ri = 1.0 / rho;
    const double u = q[1] * ri, v = q[2] * ri, w = q[3] * ri, rhoet = q[4];
    const double ek = 0.5 * (u * u + v * v + w * w);
    const double p = (g - 1.0) * (rhoet - rho * ek) - gpinf;
    const double ht = (rhoet + p) * ri;
    const double ub = u * nx + v * ny + w * nz;
    const double g1 = g - 1.0, g2 = g - 2.0;
    J[0] = 0.0;                    J[1] = nx;                    J[2] = ny;                    J[3] = nz;                    J[4] = 0.0;
    J[5] = g1 * ek * nx - u * ub;  J[6] = ub - g2 * u * nx;      J[7] = u * ny - g1 * v * nx;  J[8] = u * nz - g1 * w * nx;  J[9] = g1 * nx;
    J[10] = g1 * ek * ny - v * ub; J[11] = v * nx - g1 * u * ny; J[12] = ub - g2 * v * ny;     J[13] = v * nz - g1 * w * ny; J[14] = g1 * ny;
    J[15] = g1 * ek * nz - w * ub; J[16] = w * nx - g1 * u * nz; J[17] = w * ny - g1 * v * nz; J[18] = ub - g2 * w * nz;     J[19] = g1 * nz;
    J[20] = (g1 * ek - ht) * ub;   J[21] = ht * nx - g1 * u * ub; J[22] = ht * ny - g1 * v * ub; J[23] = ht * nz - g1 * w * ub; J[24] = g * ub;
}

// dF.n/dW for W = (rho, u, v, w, p) (Compute_Flux_Jacobian_Euler_Convective,
// VARIABLE_RUP, MPFLOW3D/src/CompressibleUtils.cpp:85-186), with
// rho ht = gamma (p + pinf) / (gamma - 1) + rho q^2 / 2.
__device__ __forceinline__ void rup_flux_jacobian(const double q[5], double nx, double ny, double nz, const Flow &f,
                                                  double J[25]) {
    const double rho = q[0], u = q[1], v = q[2], w = q[3];
    const double ub = u * nx + v * ny + w * nz, q2 = u * u + v * v + w * w;
    const double ht = f.gamma * f.inv_gm1 * (q[4] + f.pinf) / rho + 0.5 * q2;
    J[0] = ub;             J[1] = rho * nx;               J[2] = rho * ny;               J[3] = rho * nz;               J[4] = 0.0;
    J[5] = u * ub;         J[6] = rho * (ub + u * nx);    J[7] = rho * u * ny;           J[8] = rho * u * nz;           J[9] = nx;
    J[10] = v * ub;        J[11] = rho * v * nx;          J[12] = rho * (ub + v * ny);   J[13] = rho * v * nz;          J[14] = ny;
    J[15] = w * ub;        J[16] = rho * w * nx;          J[17] = rho * w * ny;          J[18] = rho * (ub + w * nz);   J[19] = nz;
    J[20] = 0.5 * q2 * ub; J[21] = rho * (u * ub + ht * nx); J[22] = rho * (v * ub + ht * ny); J[23] = rho * (w * ub + ht * nz);
    J[24] = f.gamma * f.inv_gm1 * ub;
}

// Convective flux Jacobian with respect to the state's variables.
__device__ __forceinline__ void flux_jacobian(const double q[5], double nx, double ny, double nz, const Flow &f,
                                              double J[25]) {
    if (f.rup) rup_flux_jacobian(q, nx, ny, nz, f, J);
    else euler_flux_jacobian(q, nx, ny, nz, f.gamma, f.gpinf, J);
}

// Pseudo-time matrix dQ_cons/dW of a node (V/dt times it is added to the
// diagonal block; the identity for conservative states).
__device__ __forceinline__ void state_time_matrix(const double q[5], const Flow &f, double M[25]) {
    if (f.rup) {
        dcons_drup(q[0], q[1], q[2], q[3], f, M);
    } else {
#pragma unroll
        for (int k = 0; k < 25; k++) M[k] = (k % 6 == 0) ? 1.0 : 0.0;
    }
}

// Roe dissipation matrix |A| = M P |Lambda| P^-1 M^-1 (Compute_RoeAJacobian,
// Euler3D/src/Roe_Fluxes.cpp:149-273), assembled as M * D * M^-1 where
// D = P |Lambda| P^-1 is written out in closed form in the (rho,u,v,w,p)
// variables -- the same matrix whose action on dq is the flux's dw.
__device__ __forceinline__ void roe_abs_jacobian(const double qL[5], const double qR[5], double nx, double ny,
                                                 double nz, const Flow &f, double Aout[25]) {
    Face L, R;
    const bool want_c = f.entropy_fix != 0;
    eos_face(qL, nx, ny, nz, f, want_c, L);
    eos_face(qR, nx, ny, nz, f, want_c, R);
    const double rho = sqrt(R.rho * L.rho);
    const double sigma = rho / (L.rho + rho);
    const double u = L.u + sigma * (R.u - L.u);
    const double v = L.v + sigma * (R.v - L.v);
    const double w = L.w + sigma * (R.w - L.w);
    const double ht = L.ht + sigma * (R.ht - L.ht);
    const double q2 = u * u + v * v + w * w;
    const double c = sqrt(f.gm1 * ht - 0.5 * f.gm1 * q2);
    const double ubar = u * nx + v * ny + w * nz;
    double E0, E1, E2;
    if (f.entropy_fix) roe_entropy_fix(L.ubar, L.c, R.ubar, R.c, ubar, c, E0, E1, E2);
    else { E0 = fabs(ubar); E1 = fabs(ubar + c); E2 = fabs(ubar - c); }
    const double n[3] = {nx, ny, nz};
    const double Es = E1 + E2 - 2.0 * E0, Ed = E1 - E2;
    // D in RUP variables
    double D[25];
    D[0] = E0;
    for (int j = 0; j < 3; j++) D[1 + j] = 0.5 * rho * Ed / c * n[j];
    D[4] = Es / (2.0 * c * c);
    for (int k = 0; k < 3; k++) {
        D[5 * (k + 1) + 0] = 0.0;
        for (int j = 0; j < 3; j++) D[5 * (k + 1) + 1 + j] = (k == j ? E0 : 0.0) + 0.5 * n[k] * n[j] * Es;
        D[5 * (k + 1) + 4] = n[k] * Ed / (2.0 * rho * c);
    }
    D[20] = 0.0;
    for (int j = 0; j < 3; j++) D[21 + j] = 0.5 * rho * c * Ed * n[j];
    D[24] = 0.5 * (E1 + E2);
    // M^-1 = dq_RUP/dQ_cons (Compute_Transformation_RUP_To_Conservative, Material.cpp:1240-1300);
    // with RUP states the columns stay in (rho,u,v,w,p): Mop |A| with Mpr = I
    // (Compute_Dissipation_Matrix_Roe_Optimized, MPFLOW3D/src/Roe_Fluxes.cpp:3185-3199)
    const double ri = 1.0 / rho, phi = 0.5 * f.gm1 * q2;
    double DM[25];
    if (f.rup) {
        for (int k = 0; k < 25; k++) DM[k] = D[k];
    } else {
        double Mi[25] = {1.0, 0.0, 0.0, 0.0, 0.0,
                         -u * ri, ri, 0.0, 0.0, 0.0,
                         -v * ri, 0.0, ri, 0.0, 0.0,
                         -w * ri, 0.0, 0.0, ri, 0.0,
                         phi, -u * f.gm1, -v * f.gm1, -w * f.gm1, f.gm1};
        for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++) {
                double s = 0.0;
                for (int k = 0; k < 5; k++) s += D[5 * i + k] * Mi[5 * k + j];
                DM[5 * i + j] = s;
            }
    }
    // M = dQ_cons/dq_RUP
    for (int j = 0; j < 5; j++) {
        const double d0 = DM[j], d1 = DM[5 + j], d2 = DM[10 + j], d3 = DM[15 + j], d4 = DM[20 + j];
        Aout[j] = d0;
        Aout[5 + j] = u * d0 + rho * d1;
        Aout[10 + j] = v * d0 + rho * d2;
        Aout[15 + j] = w * d0 + rho * d3;
        Aout[20 + j] = (phi / f.gm1) * d0 + rho * (u * d1 + v * d2 + w * d3) + d4 / f.gm1;
    }
}

// Thornber's low-Mach modification (Compute_Flux_Roe_Thornber,
// MPFLOW3D/src/Roe_Fluxes.cpp:1141-1165): with z = min(1, max(M_L, M_R)) the
// face velocities become u_L' = ((1+z) u_L + (1-z) u_R)/2 and symmetrically
// u_R'; density and total energy stay, so the pressure follows the changed
// kinetic energy.  With RUP states the velocities are blended at fixed
// density and pressure (Roe_Fluxes.cpp:1161-1168).  The Roe flux is then
// formed from the modified states.
template <int V = -1>
__device__ __forceinline__ void thornber_states(const double qL[5], const double qR[5], const Flow &f,
                                                double mL[5], double mR[5]) {
    Face L, R;
    eos_face<V>(qL, 1.0, 0.0, 0.0, f, true, L);
    eos_face<V>(qR, 1.0, 0.0, 0.0, f, true, R);
    const double ml = sqrt(L.u * L.u + L.v * L.v + L.w * L.w) / L.c;
    const double mr = sqrt(R.u * R.u + R.v * R.v + R.w * R.w) / R.c;
    const double z = fmin(1.0, fmax(ml, mr));
    mL[0] = qL[0];
    mR[0] = qR[0];
    mL[4] = qL[4];
    mR[4] = qR[4];
    if (vars_rup<V>(f)) {
#pragma unroll
        for (int i = 1; i < 4; i++) {
            mL[i] = 0.5 * ((1.0 + z) * qL[i] + (1.0 - z) * qR[i]);
            mR[i] = 0.5 * ((1.0 + z) * qR[i] + (1.0 - z) * qL[i]);
        }
        return;
    }
#pragma unroll
    for (int i = 1; i < 4; i++) {
        const double ul = qL[i] / qL[0], ur = qR[i] / qR[0];
        mL[i] = qL[0] * (0.5 * ((1.0 + z) * ul + (1.0 - z) * ur));
        mR[i] = qR[0] * (0.5 * ((1.0 + z) * ur + (1.0 - z) * ul));
    }
}

// ---------------------------------------------------------------------------
// Low-Mach preconditioned Roe of the Turkel family (MPFLOW3D:
// Compute_Flux_Roe_Precondition_Turkel, MPFLOW3D/src/Roe_Fluxes.cpp:2043-2526;
// Compute_Dissipation_Matrix_Roe_Precondition_Turkel, :3440-3810;
// Compute_Transformed_Preconditioner_Matrix_Roe_Turkel, :261-441).  The
// preconditioner K acts on (rho, u, v, w, p):
//   K = I except K[0][4] = (delta - 1)/c^2, K[1..3][4] = -alpha (u,v,w)/(rho c^2), K[4][4] = beta
// with beta = Mr^2 and (alpha, delta) = (0, 1) BTW, (0, beta) Eriksson,
// (0.4, beta) Turkel.  The edge dissipation is Mop Kinv R |Lambda| L Mpr dQ
// with L, R the left/right eigenvectors of K A at the Roe average and the
// eigenvalues |u.n|, |zp u.n +- c'|, zp = (1 + beta - alpha)/2,
// c'^2 = beta (c^2 - (u.n)^2) + zp^2 (u.n)^2.  Conservative solution
// variables, pressure smoothing off (PRECOND_SMOOTH NO).

// beta = Mr^2 for CFD_PRECOND_LOCAL / GLOBAL / URLOCAL (Roe_Fluxes.cpp:2225-2248)
__device__ __forceinline__ double pc_beta(const Flow &f, double mach, double mach_max) {
    double b;
    if (f.pc_type == CFD_PRECOND_LOCAL) {
        const double M = fmax(mach, mach_max), G = f.pc_mach;
        b = M < G ? 0.5 * (M * M) / (G * G) - M / G + 1.0 : 0.5;
        b = fmin(1.0, b * (sqrt(M * G) + M));
    } else if (f.pc_type == CFD_PRECOND_URLOCAL) {
        b = fmin(1.0, mach);
    } else {
        b = fmin(1.0, f.pc_mach);
    }
    return b * b;
}

struct PcSys {
    double rho, u, v, w, c, beta, alpha, delta, zp, zm, ubar, ubp, cp;
    double lam0, lam3, lam4;      // |u.n|, |ubp + cp|, |ubp - cp|
};

__device__ __forceinline__ void pc_system(double rho, double u, double v, double w, double c, double nx, double ny,
                                          double nz, double beta, const Flow &f, PcSys &S) {
    const double alpha = f.pc_method == CFD_PRECOND_TURKEL ? 0.4 : 0.0;
    const double delta = f.pc_method == CFD_PRECOND_BTW ? 1.0 : beta;
    const double ubar = u * nx + v * ny + w * nz;
    const double zp = 0.5 * (1.0 + beta - alpha), zm = 0.5 * (1.0 - beta + alpha);
    const double ubp = zp * ubar, cp = sqrt(beta * (c * c - ubar * ubar) + zp * zp * ubar * ubar);
    S.rho = rho; S.u = u; S.v = v; S.w = w; S.c = c;
    S.beta = beta; S.alpha = alpha; S.delta = delta; S.zp = zp; S.zm = zm;
    S.ubar = ubar; S.ubp = ubp; S.cp = cp;
    S.lam0 = fabs(ubar);
    S.lam3 = fabs(ubp + cp);
    S.lam4 = fabs(ubp - cp);
}

// Row k of the left eigenvectors of K A (rows of the reference's right-
// eigenvector array, Roe_Fluxes.cpp:2353-2387; BC.cpp:279-305).  Called with
// a constant k so each row is formed where it is consumed.
__device__ __forceinline__ void pc_left_row(int k, const PcSys &S, double nx, double ny, double nz, double L[5]) {
    const double rho = S.rho, u = S.u, v = S.v, w = S.w, ubar = S.ubar, c2 = S.c * S.c;
    const double beta = S.beta, alpha = S.alpha, delta = S.delta, zp = S.zp, zm = S.zm, cp = S.cp;
    const double bc2 = beta * c2, pv1 = rho * (beta - delta), pv2 = pv1 * ubar, pv3 = bc2 - alpha * ubar * ubar;
    const double ipv3 = 1.0 / pv3, aub = alpha * ubar;
    if (k < 3) {
        const double irc = 1.0 / (rho * c2 * pv3), aub2r = alpha * rho * ubar * ubar, rdc = rho * delta * c2;
        if (k == 0) {
            L[0] = nx;
            L[1] = nx * ubar * (alpha * (v * nz - w * ny) + pv1 * nx) * ipv3;
            L[2] = (bc2 * nz - aub * (w * ny * ny + u * nx * nz + w * nz * nz) + pv2 * nx * ny) * ipv3;
            L[3] = (-bc2 * ny + aub * (v * ny * ny + u * nx * ny + v * nz * nz) + pv2 * nx * nz) * ipv3;
            L[4] = (-rdc * nx + alpha * c2 * (v * nz - w * ny) + aub2r * nx) * irc;
        } else if (k == 1) {
            L[0] = ny;
            L[1] = (-bc2 * nz + aub * (w * nx * nx + v * ny * nz + w * nz * nz) + pv2 * nx * ny) * ipv3;
            L[2] = ny * ubar * (alpha * (w * nx - u * nz) + pv1 * ny) * ipv3;
            L[3] = (bc2 * nx - aub * (u * nx * nx + v * nx * ny + u * nz * nz) + pv2 * ny * nz) * ipv3;
            L[4] = (-rdc * ny + alpha * c2 * (w * nx - u * nz) + aub2r * ny) * irc;
        } else {
            L[0] = nz;
            L[1] = (bc2 * ny - aub * (v * nx * nx + w * ny * nz + v * ny * ny) + pv2 * nx * nz) * ipv3;
            L[2] = (-bc2 * nx + aub * (u * nx * nx + w * nx * nz + u * ny * ny) + pv2 * ny * nz) * ipv3;
            L[3] = nz * ubar * (alpha * (u * ny - v * nx) + pv1 * nz) * ipv3;
            L[4] = (-rdc * nz + alpha * c2 * (u * ny - v * nx) + aub2r * nz) * irc;
        }
    } else if (k == 3) {
        const double pv4 = (bc2 * (cp + ubar * zm)) / (2.0 * cp * pv3);
        L[0] = 0.0; L[1] = pv4 * nx; L[2] = pv4 * ny; L[3] = pv4 * nz;
        L[4] = (bc2 + aub * (cp - ubar * zp)) / (2.0 * rho * cp * pv3);
    } else {
        const double pv5 = (bc2 * (cp - ubar * zm)) / (2.0 * cp * pv3);
        L[0] = 0.0; L[1] = -pv5 * nx; L[2] = -pv5 * ny; L[3] = -pv5 * nz;
        L[4] = (bc2 - aub * (cp + ubar * zp)) / (2.0 * rho * cp * pv3);
    }
}

// out = Mop Kinv R |Lambda| L Mpr dQ at the system's averaged state, with
// Mpr = d(rho,u,v,w,p)/dQ and Mop its inverse (the same for either gas);
// Mpr = I when dQ is already a (rho,u,v,w,p) difference (RUP states).
template <int V = -1>
__device__ __forceinline__ void pc_dissipation(const PcSys &S, double nx, double ny, double nz, const Flow &f,
                                               const double dQ[5], double out[5]) {
    const double rho = S.rho, u = S.u, v = S.v, w = S.w, ri = 1.0 / rho;
    const double q2 = u * u + v * v + w * w;
    double dq[5];
    if (vars_rup<V>(f)) {
#pragma unroll
        for (int k = 0; k < 5; k++) dq[k] = dQ[k];
    } else {
        dq[0] = dQ[0];
        dq[1] = (dQ[1] - u * dQ[0]) * ri;
        dq[2] = (dQ[2] - v * dQ[0]) * ri;
        dq[3] = (dQ[3] - w * dQ[0]) * ri;
        dq[4] = f.gm1 * (0.5 * q2 * dQ[0] - u * dQ[1] - v * dQ[2] - w * dQ[3] + dQ[4]);
    }
    double a[5];
#pragma unroll
    for (int k = 0; k < 5; k++) {
        double l[5];
        pc_left_row(k, S, nx, ny, nz, l);
        a[k] = l[0] * dq[0] + l[1] * dq[1] + l[2] * dq[2] + l[3] * dq[3] + l[4] * dq[4];
    }
    a[0] *= S.lam0; a[1] *= S.lam0; a[2] *= S.lam0; a[3] *= S.lam3; a[4] *= S.lam4;
    // right eigenvectors
    const double bc2 = S.beta * S.c * S.c, ibc2 = 1.0 / bc2, zp = S.zp, zm = S.zm, ub = S.ubar, cp = S.cp;
    const double r03 = rho * ((zp * S.delta - S.beta) * ub + cp * S.delta) * ibc2;
    const double r04 = -rho * ((zp * S.delta - S.beta) * ub - cp * S.delta) * ibc2;
    const double sp = S.alpha * (cp + zp * ub) * ibc2, sm = S.alpha * (cp - zp * ub) * ibc2;
    double z[5];
    z[0] = nx * a[0] + ny * a[1] + nz * a[2] + r03 * a[3] + r04 * a[4];
    z[1] = -nz * a[1] + ny * a[2] + (nx - u * sp) * a[3] + (-nx - u * sm) * a[4];
    z[2] = nz * a[0] - nx * a[2] + (ny - v * sp) * a[3] + (-ny - v * sm) * a[4];
    z[3] = -ny * a[0] + nx * a[1] + (nz - w * sp) * a[3] + (-nz - w * sm) * a[4];
    z[4] = rho * (cp - zm * ub) * a[3] + rho * (cp + zm * ub) * a[4];
    // Kinv: identity except column 4
    const double k4 = z[4] / S.beta, kr = S.alpha * z[4] / (S.beta * rho * S.c * S.c);
    z[0] += (1.0 - S.delta) * ibc2 * z[4];
    z[1] += u * kr;
    z[2] += v * kr;
    z[3] += w * kr;
    z[4] = k4;
    out[0] = z[0];
    out[1] = u * z[0] + rho * z[1];
    out[2] = v * z[0] + rho * z[2];
    out[3] = w * z[0] + rho * z[3];
    out[4] = 0.5 * q2 * z[0] + rho * (u * z[1] + v * z[2] + w * z[3]) + z[4] * f.inv_gm1;
}

// Roe-averaged eigen-system of an edge; beta from the average's Mach and the
// larger of the two states' (PRECOND_TYPE LOCAL without smoothing).
__device__ __forceinline__ void pc_edge_system(const Face &L, const Face &R, double nx, double ny, double nz,
                                               const Flow &f, PcSys &S) {
    const double rr = R.rho * L.rho;
    const double rho = sqrt(rr);
    const double sigma = rho / (L.rho + rho);
    const double u = L.u + sigma * (R.u - L.u);
    const double v = L.v + sigma * (R.v - L.v);
    const double w = L.w + sigma * (R.w - L.w);
    const double ht = L.ht + sigma * (R.ht - L.ht);
    const double q2 = u * u + v * v + w * w;
    const double c = sqrt(f.gm1 * (ht - 0.5 * q2));  // c^2 = (gamma - 1) h for either gas
    const double mach = sqrt(q2) / c;
    const double mL = sqrt(L.u * L.u + L.v * L.v + L.w * L.w) / L.c;
    const double mR = sqrt(R.u * R.u + R.v * R.v + R.w * R.w) / R.c;
    pc_system(rho, u, v, w, c, nx, ny, nz, pc_beta(f, mach, fmax(mL, mR)), f, S);
}

// Preconditioned Roe flux: central part as Roe, dissipation -1/2 |A|_p dQ area;
// returns the spectral radius of K A (time step), lam = |u.n|, |ubp+cp|, |ubp-cp|.
template <int V = -1>
__device__ __forceinline__ double roe_precond_flux(const double qL[5], const double qR[5], double nx, double ny,
                                                   double nz, double area, const Flow &f, double conv[5],
                                                   double diss[5], double lam[3]) {
    Face L, R;
    eos_face<V>(qL, nx, ny, nz, f, true, L);
    eos_face<V>(qR, nx, ny, nz, f, true, R);
    const double mL = L.rho * L.ubar, mR = R.rho * R.ubar;
    const double ha = 0.5 * area;
    conv[0] = ha * (mL + mR);
    conv[1] = ha * ((L.u * mL + L.p * nx) + (R.u * mR + R.p * nx));
    conv[2] = ha * ((L.v * mL + L.p * ny) + (R.v * mR + R.p * ny));
    conv[3] = ha * ((L.w * mL + L.p * nz) + (R.w * mR + R.p * nz));
    conv[4] = ha * (L.ht * mL + R.ht * mR);
    PcSys S;
    pc_edge_system(L, R, nx, ny, nz, f, S);
    double dQ[5], d[5];
#pragma unroll
    for (int k = 0; k < 5; k++) dQ[k] = qR[k] - qL[k];
    pc_dissipation<V>(S, nx, ny, nz, f, dQ, d);
#pragma unroll
    for (int k = 0; k < 5; k++) diss[k] = -ha * d[k];
    lam[0] = S.lam0;
    lam[1] = S.lam3;
    lam[2] = S.lam4;
    return fmax(S.lam0, fmax(S.lam3, S.lam4));
}

// |A|_p as a matrix (row-major), column j = the dissipation of dQ = e_j.
__device__ __forceinline__ void pc_abs_jacobian(const double qL[5], const double qR[5], double nx, double ny,
                                                double nz, const Flow &f, double A[25]) {
    Face L, R;
    eos_face(qL, nx, ny, nz, f, true, L);
    eos_face(qR, nx, ny, nz, f, true, R);
    PcSys S;
    pc_edge_system(L, R, nx, ny, nz, f, S);
    // fully unrolled so that every index is a constant (no local-memory arrays)
#pragma unroll
    for (int j = 0; j < 5; j++) {
        double e[5], col[5];
#pragma unroll
        for (int k = 0; k < 5; k++) e[k] = k == j ? 1.0 : 0.0;
        pc_dissipation(S, nx, ny, nz, f, e, col);
#pragma unroll
        for (int i = 0; i < 5; i++) A[5 * i + j] = col[i];
    }
}

// Pseudo-time matrix Cinv = Mop Kinv Mpr at a node state (beta from the
// node's Mach; Roe_Jacobian.cpp:241-264 adds (V/dt) Cinv to the diagonal);
// Mpr = I for RUP states.
__device__ __forceinline__ void pc_node_cinv(const double q[5], const Flow &f, double C[25]) {
    Face F;
    eos_face(q, 1.0, 0.0, 0.0, f, true, F);
    const double mach = sqrt(F.u * F.u + F.v * F.v + F.w * F.w) / F.c;
    const double beta = pc_beta(f, mach, 0.0);
    const double alpha = f.pc_method == CFD_PRECOND_TURKEL ? 0.4 : 0.0;
    const double delta = f.pc_method == CFD_PRECOND_BTW ? 1.0 : beta;
    const double rho = F.rho, u = F.u, v = F.v, w = F.w, c2 = F.c * F.c, q2 = u * u + v * v + w * w;
    const double kc0 = (1.0 - delta) / (beta * c2), kr = alpha / (beta * rho * c2), k4 = 1.0 / beta;
    // Mpr rows: (1,0,0,0,0), (-u,1,0,0,0)/rho, (-v,0,1,0,0)/rho, (-w,0,0,1,0)/rho, gm1 (q2/2,-u,-v,-w,1)
#pragma unroll
    for (int j = 0; j < 5; j++) {
        double m[5];
        if (f.rup) {
#pragma unroll
            for (int k = 0; k < 5; k++) m[k] = k == j ? 1.0 : 0.0;
        } else {
            m[0] = j == 0 ? 1.0 : 0.0;
            m[1] = (j == 0 ? -u : (j == 1 ? 1.0 : 0.0)) / rho;
            m[2] = (j == 0 ? -v : (j == 2 ? 1.0 : 0.0)) / rho;
            m[3] = (j == 0 ? -w : (j == 3 ? 1.0 : 0.0)) / rho;
            m[4] = f.gm1 * (j == 0 ? 0.5 * q2 : (j == 4 ? 1.0 : (j == 1 ? -u : (j == 2 ? -v : -w))));
        }
        double z0 = m[0] + kc0 * m[4], z1 = m[1] + u * kr * m[4], z2 = m[2] + v * kr * m[4], z3 = m[3] + w * kr * m[4];
        double z4 = k4 * m[4];
        C[j] = z0;
        C[5 + j] = u * z0 + rho * z1;
        C[10 + j] = v * z0 + rho * z2;
        C[15 + j] = w * z0 + rho * z3;
        C[20 + j] = 0.5 * q2 * z0 + rho * (u * z1 + v * z2 + w * z3) + z4 * f.inv_gm1;
    }
}

// x = A^-1 b for a 5x5 system by Gaussian elimination with partial pivoting
// (the pivoted LU the preconditioned BC solves with); A is overwritten.
// Returns false (x then undefined) when a pivot is zero.
__device__ __forceinline__ bool solve5_pivot(double A[25], double b[5], double x[5]) {
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 5; c++) {
        int p = c;
#pragma unroll
        for (int i = c + 1; i < 5; i++)
            if (fabs(A[5 * i + c]) > fabs(A[5 * p + c])) p = i;
        if (p != c) {
#pragma unroll
            for (int j = 0; j < 5; j++) {
                const double t = A[5 * c + j];
                A[5 * c + j] = A[5 * p + j];
                A[5 * p + j] = t;
            }
            const double t = b[c];
            b[c] = b[p];
            b[p] = t;
        }
        if (A[5 * c + c] == 0.0) ok = false;
#pragma unroll
        for (int i = c + 1; i < 5; i++) {
            const double m = A[5 * i + c] / A[5 * c + c];
#pragma unroll
            for (int j = c; j < 5; j++) A[5 * i + j] -= m * A[5 * c + j];
            b[i] -= m * b[c];
        }
    }
#pragma unroll
    for (int i = 4; i >= 0; i--) {
        double t = b[i];
#pragma unroll
        for (int j = i + 1; j < 5; j++) t -= A[5 * i + j] * x[j];
        x[i] = t / A[5 * i + i];
    }
    return ok;
}

// Ghost state of the preconditioned characteristic BC
// (Compute_Precondition_Characteristic_BoundaryCondition_Turkel,
// MPFLOW3D/src/BC.cpp:113-700, BC_METHOD_CHARCTERISTIC) through the
// characteristic variables L (rho,u,v,w,p) at the interior/ghost average:
// wall = four outgoing characteristics and zero normal velocity; subsonic
// inflow = freestream (rho, u, v, w) with the interior's p and the u.n + c'
// characteristic from inside; subsonic outflow = four characteristics from
// inside and the outflow pressure.  Returns as characteristic_bc (2 also for
// a singular characteristic system).
__device__ __forceinline__ int precond_characteristic_bc(const double qI[5], const double qG[5], double nx,
                                                         double ny, double nz, int bc_type, const Flow &f,
                                                         double qB[5]) {
    Face I, G, O;
    eos_face(qI, nx, ny, nz, f, true, I);
    eos_face(qG, nx, ny, nz, f, true, G);
    double q0[5];
#pragma unroll
    for (int k = 0; k < 5; k++) q0[k] = 0.5 * (qI[k] + qG[k]);
    eos_face(q0, nx, ny, nz, f, true, O);
    const double mach = sqrt(O.u * O.u + O.v * O.v + O.w * O.w) / O.c;
    const double mI = sqrt(I.u * I.u + I.v * I.v + I.w * I.w) / I.c;
    const double mG = sqrt(G.u * G.u + G.v * G.v + G.w * G.w) / G.c;
    PcSys S;
    pc_system(O.rho, O.u, O.v, O.w, O.c, nx, ny, nz, pc_beta(f, mach, fmax(mI, mG)), f, S);
    double Lm[25];
#pragma unroll
    for (int k = 0; k < 5; k++) pc_left_row(k, S, nx, ny, nz, Lm + 5 * k);
    const double l1 = S.ubar, l4 = S.ubp + S.cp, l5 = S.ubp - S.cp;
    int inst, status = 0;
    switch (bc_type) {
        case 0: inst = 0; break;
        case 1:
            if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 10;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 11;
            else if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 9;
            else if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 8;
            else { inst = 1; status = 2; }
            break;
        case 2:
            if (l1 <= 0.0 && l4 >= 0.0 && l5 <= 0.0) inst = 4;
            else if (l1 <= 0.0 && l4 <= 0.0 && l5 <= 0.0) inst = 6;
            else inst = (fabs(l1) < O.c) ? 4 : 6;
            break;
        case 3:
            if (l1 >= 0.0 && l5 <= 0.0 && l4 >= 0.0) inst = 5;
            else if (l1 >= 0.0 && l4 >= 0.0 && l5 >= 0.0) inst = 7;
            else inst = (fabs(l1) < O.c) ? 5 : 7;
            break;
        case 4: case 5: case 6: case 7: inst = bc_type; break;
        default: inst = -1; status = 2; break;
    }
    const double qi[5] = {I.rho, I.u, I.v, I.w, I.p};
    const double qf[5] = {f.inf_rho, f.inf_u, f.inf_v, f.inf_w, f.inf_p};
    double xb[5] = {f.inf_rho, f.inf_u, f.inf_v, f.inf_w, f.inf_p};
    auto lrow = [&](int k, const double q[5]) {
        return Lm[5 * k] * q[0] + Lm[5 * k + 1] * q[1] + Lm[5 * k + 2] * q[2] + Lm[5 * k + 3] * q[3] +
               Lm[5 * k + 4] * q[4];
    };
    double B[5];
    switch (inst) {
        case 0:
#pragma unroll
            for (int k = 0; k < 4; k++) B[k] = lrow(k, qi);
            B[4] = 0.0;
            Lm[20] = 0.0; Lm[21] = nx; Lm[22] = ny; Lm[23] = nz; Lm[24] = 0.0;
            if (!solve5_pivot(Lm, B, xb)) status = status ? status : 2;
            if (f.iteration < f.zpg_iteration && xb[4] + f.pinf < 0.0) {
                xb[0] = I.rho; xb[4] = I.p;
                xb[1] = I.u - nx * I.ubar; xb[2] = I.v - ny * I.ubar; xb[3] = I.w - nz * I.ubar;
            }
            if (xb[4] + f.pinf < 0.0) status = status ? status : 1;
            break;
        case 4: case 8: {
            const double qe[5] = {qf[0], qf[1], qf[2], qf[3], inst == 4 ? I.p : qf[4]};
#pragma unroll
            for (int k = 0; k < 5; k++) B[k] = k == 3 ? lrow(3, qi) : lrow(k, qe);
            if (!solve5_pivot(Lm, B, xb)) status = status ? status : 2;
        } break;
        case 5:
#pragma unroll
            for (int k = 0; k < 4; k++) B[k] = lrow(k, qi);
            B[4] = f.pc_outflow_p;
            Lm[20] = 0.0; Lm[21] = 0.0; Lm[22] = 0.0; Lm[23] = 0.0; Lm[24] = 1.0;
            if (!solve5_pivot(Lm, B, xb)) status = status ? status : 2;
            break;
        case 9:
#pragma unroll
            for (int k = 0; k < 5; k++) B[k] = k == 4 ? lrow(4, qf) : lrow(k, qi);
            if (!solve5_pivot(Lm, B, xb)) status = status ? status : 2;
            break;
        case 7: case 11:
#pragma unroll
            for (int k = 0; k < 5; k++) xb[k] = qi[k];
            break;
        default: break;  // 1, 6, 10: freestream
    }
    store_state(xb[0], xb[1], xb[2], xb[3], xb[4], f, qB);
    return status;
}

}  // namespace cfd
