// Device physics of the node-centred edge-based Euler path: ideal-gas EOS in
// the generic non-dimensionalisation (or the stiffened gas
// p = (gamma - 1) rho e - gamma pinf, which is the ideal gas at pinf = 0), Roe / HLLC / AUSM+ edge fluxes,
// characteristic ghost states and the approximate Roe flux Jacobian.
// Conservative variables (rho, rho u, rho v, rho w, rho et) throughout, as
// Euler3D with VARIABLE_TYPE=VARIABLE_CONSERVATIVE.
#pragma once

#include <cuda_runtime.h>

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
};

struct Face {
    double rho, u, v, w, p, ht, ubar, c;
};

// Compute_EOS_Variables_Face, conservative branch (Euler3D/src/Material.cpp:216-248),
// with the stiffened-gas terms: p = (gamma - 1)(rho et - rho q^2 / 2) - gamma pinf and
// c^2 = gamma (p + pinf) / rho.  At pinf = 0 both added terms are exact zeros, so
// the ideal-gas results are bit-identical.  c is only formed when `want_c`.
__device__ __forceinline__ void eos_face(const double q[5], double nx, double ny, double nz, const Flow &f,
                                         bool want_c, Face &s) {
    s.rho = q[0];
    const double ri = 1.0 / s.rho;
    s.u = q[1] * ri;
    s.v = q[2] * ri;
    s.w = q[3] * ri;
    const double q2 = s.u * s.u + s.v * s.v + s.w * s.w;
    s.p = f.gm1 * (q[4] - 0.5 * s.rho * q2) - f.gpinf;
    s.ht = (q[4] + s.p) * ri;
    s.ubar = s.u * nx + s.v * ny + s.w * nz;
    s.c = want_c ? sqrt(f.gamma * (s.p + f.pinf) * ri) : 0.0;
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
template <bool LMFIX>
__device__ __forceinline__ double roe_flux(const double qL[5], const double qR[5], double nx, double ny,
                                           double nz, double area, const Flow &f, double conv[5],
                                           double diss[5], double lam[3]) {
    Face L, R;
    const bool want_c = f.entropy_fix != 0;
    eos_face(qL, nx, ny, nz, f, want_c, L);
    eos_face(qR, nx, ny, nz, f, want_c, R);

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
    // Get_TotalEnergy (Material.cpp:1012-1040), rho e = (p + gamma pinf) / (gamma - 1)
    const double et = (p_b + f.gpinf) / (f.gm1 * rho_b) + 0.5 * (u_b * u_b + v_b * v_b + w_b * w_b);
    qB[0] = rho_b;
    qB[1] = rho_b * u_b;
    qB[2] = rho_b * v_b;
    qB[3] = rho_b * w_b;
    qB[4] = rho_b * et;
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
    // M^-1 = dq_RUP/dQ_cons (Compute_Transformation_RUP_To_Conservative, Material.cpp:1240-1300)
    const double ri = 1.0 / rho, phi = 0.5 * f.gm1 * q2;
    double Mi[25] = {1.0, 0.0, 0.0, 0.0, 0.0,
                     -u * ri, ri, 0.0, 0.0, 0.0,
                     -v * ri, 0.0, ri, 0.0, 0.0,
                     -w * ri, 0.0, 0.0, ri, 0.0,
                     phi, -u * f.gm1, -v * f.gm1, -w * f.gm1, f.gm1};
    double DM[25];
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            double s = 0.0;
            for (int k = 0; k < 5; k++) s += D[5 * i + k] * Mi[5 * k + j];
            DM[5 * i + j] = s;
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

}  // namespace cfd
