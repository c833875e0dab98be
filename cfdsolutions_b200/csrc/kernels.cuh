// Edge-flux dispatch (Roe / HLLC / AUSM+) and small device helpers shared by
// the residual, Jacobian and linear-solver translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "ctx.cuh"
#include "physics.cuh"

namespace cfd {

// HLLC flux (Compute_HLLCFlux, Euler3D/src/HLLC_Fluxes.cpp:143-326): Roe-averaged
// wave speeds SL = min(ubar_L - c_L, ubar - c), SR = max(ubar_R + c_R, ubar + c),
// contact speed SM, star states.  The whole flux goes to the convective
// residual (Compute_Residual_HLLC, :519-573); the dissipative part is zero.
template <int V = -1>
__device__ __forceinline__ double hllc_flux(const double qL[5], const double qR[5], double nx, double ny, double nz,
                                            double area, const Flow &f, double conv[5], double diss[5],
                                            double lam[3]) {
    Face L, R;
    eos_face<V>(qL, nx, ny, nz, f, true, L);
    eos_face<V>(qR, nx, ny, nz, f, true, R);
    const double rho = sqrt(R.rho * L.rho);
    const double sigma = rho / (L.rho + rho);
    const double u = L.u + sigma * (R.u - L.u);
    const double v = L.v + sigma * (R.v - L.v);
    const double w = L.w + sigma * (R.w - L.w);
    const double ht = L.ht + sigma * (R.ht - L.ht);
    const double phi = 0.5 * f.gm1 * (u * u + v * v + w * w);
    const double c = sqrt(f.gm1 * ht - phi);
    const double ubar = u * nx + v * ny + w * nz;
    const double SL = fmin(L.ubar - L.c, ubar - c);
    const double SR = fmax(R.ubar + R.c, ubar + c);
    const double SM = (R.rho * R.ubar * (SR - R.ubar) - L.rho * L.ubar * (SL - L.ubar) + L.p - R.p) /
                      (R.rho * (SR - R.ubar) - L.rho * (SL - L.ubar));
    double F[5];
    if (SL > 0.0 || SR < 0.0) {
        const Face &S = SL > 0.0 ? L : R;
        const double m = S.rho * S.ubar;
        F[0] = m;
        F[1] = S.u * m + S.p * nx;
        F[2] = S.v * m + S.p * ny;
        F[3] = S.w * m + S.p * nz;
        F[4] = S.ht * m;
    } else {
        const bool left = SM > 0.0;
        const Face &S = left ? L : R;
        const double Sk = left ? SL : SR;
        const double pstar = S.p + S.rho * (S.ubar - Sk) * (S.ubar - SM);
        const double om = 1.0 / (Sk - SM);
        const double c1 = Sk - S.ubar, c2 = pstar - S.p;
        const double et = S.ht - S.p / S.rho;
        const double rs = om * (c1 * S.rho);
        const double rus = om * (c1 * S.rho * S.u + c2 * nx);
        const double rvs = om * (c1 * S.rho * S.v + c2 * ny);
        const double rws = om * (c1 * S.rho * S.w + c2 * nz);
        const double res_ = om * (c1 * S.rho * et - S.p * S.ubar + pstar * SM);
        F[0] = rs * SM;
        F[1] = rus * SM + pstar * nx;
        F[2] = rvs * SM + pstar * ny;
        F[3] = rws * SM + pstar * nz;
        F[4] = (res_ + pstar) * SM;
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
        conv[k] = F[k] * area;
        diss[k] = 0.0;
    }
    // HLLC leaves the eigenvalue extrema untouched in the reference; NaN is
    // ignored by fmin/fmax.
    lam[0] = lam[1] = lam[2] = __longlong_as_double(0x7ff8000000000000LL);
    return fmax(fabs(ubar), fmax(fabs(ubar + c), fabs(ubar - c)));
}

// AUSM+ (M.-S. Liou, "A sequel to AUSM: AUSM+", J. Comput. Phys. 129, 1996):
// interface sound speed c_1/2 = min(c^_L, c^_R), c^ = c*^2/max(c*, |u_n|) with
// c*^2 = 2 (gamma-1)/(gamma+1) H; split Mach numbers of degree 4 (beta = 1/8)
// and split pressures of degree 5 (alpha = 3/16); upwinded convective flux
// c_1/2 (m+ Phi_L + m- Phi_R) plus p_1/2 n.  The reference's AUSM entry points
// are empty stubs (Euler3D/src/AUSM_Fluxes.cpp:45-54), so this follows the
// published method.  The dissipative residual is zero; the time-step spectral
// radius is the Roe-averaged |ubar| + c, as for HLLC.
template <int V = -1>
__device__ __forceinline__ double ausmp_flux(const double qL[5], const double qR[5], double nx, double ny,
                                             double nz, double area, const Flow &f, double conv[5], double diss[5],
                                             double lam[3]) {
    Face L, R;
    eos_face<V>(qL, nx, ny, nz, f, false, L);
    eos_face<V>(qR, nx, ny, nz, f, false, R);
    const double k = 2.0 * f.gm1 / (f.gamma + 1.0);
    const double csL = sqrt(k * L.ht), csR = sqrt(k * R.ht);
    const double chL = csL * csL / fmax(csL, L.ubar);
    const double chR = csR * csR / fmax(csR, -R.ubar);
    const double c12 = fmin(chL, chR);
    const double ML = L.ubar / c12, MR = R.ubar / c12;
    const double beta = 0.125, alpha = 3.0 / 16.0;
    double Mp, Pp, Mm, Pm;
    if (fabs(ML) >= 1.0) {
        Mp = 0.5 * (ML + fabs(ML));
        Pp = ML > 0.0 ? 1.0 : 0.0;
    } else {
        const double a = ML + 1.0, b = ML * ML - 1.0;
        Mp = 0.25 * a * a + beta * b * b;
        Pp = 0.25 * a * a * (2.0 - ML) + alpha * ML * b * b;
    }
    if (fabs(MR) >= 1.0) {
        Mm = 0.5 * (MR - fabs(MR));
        Pm = MR < 0.0 ? 1.0 : 0.0;
    } else {
        const double a = MR - 1.0, b = MR * MR - 1.0;
        Mm = -0.25 * a * a - beta * b * b;
        Pm = 0.25 * a * a * (2.0 + MR) - alpha * MR * b * b;
    }
    const double m12 = Mp + Mm;
    const double mpos = 0.5 * (m12 + fabs(m12)), mneg = 0.5 * (m12 - fabs(m12));
    const double p12 = Pp * L.p + Pm * R.p;
    const double aL = c12 * mpos * L.rho, aR = c12 * mneg * R.rho;
    conv[0] = area * (aL + aR);
    conv[1] = area * (aL * L.u + aR * R.u + p12 * nx);
    conv[2] = area * (aL * L.v + aR * R.v + p12 * ny);
    conv[3] = area * (aL * L.w + aR * R.w + p12 * nz);
    conv[4] = area * (aL * L.ht + aR * R.ht);
#pragma unroll
    for (int j = 0; j < 5; j++) diss[j] = 0.0;
    lam[0] = lam[1] = lam[2] = __longlong_as_double(0x7ff8000000000000LL);
    const double rho = sqrt(R.rho * L.rho);
    const double sigma = rho / (L.rho + rho);
    const double u = L.u + sigma * (R.u - L.u);
    const double v = L.v + sigma * (R.v - L.v);
    const double w = L.w + sigma * (R.w - L.w);
    const double ht = L.ht + sigma * (R.ht - L.ht);
    const double c = sqrt(f.gm1 * ht - 0.5 * f.gm1 * (u * u + v * v + w * w));
    return fabs(u * nx + v * ny + w * nz) + c;
}

// Van Leer flux-vector splitting (Compute_VanLeerFlux, Euler3D/src/VanLeer_Fluxes.cpp:143-305):
// F+ of the left state and F- of the right state by the face-normal Mach
// number, the full flux beyond |M| = 1; no dissipative part; the time-step
// eigenvalue from the arithmetic means (c of the mean rho and p).  Ideal gas.
template <int V = -1>
__device__ __forceinline__ double vanleer_flux(const double qL[5], const double qR[5], double nx, double ny,
                                               double nz, double area, const Flow &f, double conv[5],
                                               double diss[5], double lam[3]) {
    Face L, R;
    eos_face<V>(qL, nx, ny, nz, f, true, L);
    eos_face<V>(qR, nx, ny, nz, f, true, R);
    const double g = f.gamma, gg = g * g - 1.0;
    const double rho_a = 0.5 * (L.rho + R.rho);
    const double ub_a = 0.5 * ((L.u + R.u) * nx + (L.v + R.v) * ny + (L.w + R.w) * nz);
    const double p_a = 0.5 * (L.p + R.p);
    const double c_a = sqrt(g * p_a / rho_a);
    double fp[5], fm[5];
    {
        const double M = L.ubar / L.c, q2 = L.u * L.u + L.v * L.v + L.w * L.w;
        if (fabs(M) < 1.0) {
            const double b = -L.ubar + 2.0 * L.c;
            fp[0] = 0.25 * L.rho * L.c * (M + 1.0) * (M + 1.0);
            fp[1] = fp[0] * (nx * b / g + L.u);
            fp[2] = fp[0] * (ny * b / g + L.v);
            fp[3] = fp[0] * (nz * b / g + L.w);
            fp[4] = fp[0] * ((-(g - 1.0) * L.ubar * L.ubar + 2.0 * (g - 1.0) * L.ubar * L.c + 2.0 * L.c * L.c) / gg +
                             0.5 * q2);
        } else if (M >= 1.0) {
            fp[0] = L.rho * L.ubar;
            fp[1] = L.rho * L.u * L.ubar + nx * L.p;
            fp[2] = L.rho * L.v * L.ubar + ny * L.p;
            fp[3] = L.rho * L.w * L.ubar + nz * L.p;
            fp[4] = (qL[4] + L.p) * L.ubar;
        } else {
            fp[0] = fp[1] = fp[2] = fp[3] = fp[4] = 0.0;
        }
    }
    {
        const double M = R.ubar / R.c, q2 = R.u * R.u + R.v * R.v + R.w * R.w;
        if (fabs(M) < 1.0) {
            const double b = -R.ubar - 2.0 * R.c;
            fm[0] = -0.25 * R.rho * R.c * (M - 1.0) * (M - 1.0);
            fm[1] = fm[0] * (nx * b / g + R.u);
            fm[2] = fm[0] * (ny * b / g + R.v);
            fm[3] = fm[0] * (nz * b / g + R.w);
            fm[4] = fm[0] * ((-(g - 1.0) * R.ubar * R.ubar - 2.0 * (g - 1.0) * R.ubar * R.c + 2.0 * R.c * R.c) / gg +
                             0.5 * q2);
        } else if (M <= -1.0) {
            fm[0] = R.rho * R.ubar;
            fm[1] = R.rho * R.u * R.ubar + nx * R.p;
            fm[2] = R.rho * R.v * R.ubar + ny * R.p;
            fm[3] = R.rho * R.w * R.ubar + nz * R.p;
            fm[4] = (qR[4] + R.p) * R.ubar;
        } else {
            fm[0] = fm[1] = fm[2] = fm[3] = fm[4] = 0.0;
        }
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
        conv[k] = (fp[k] + fm[k]) * area;
        diss[k] = 0.0;
    }
    // the reference leaves the eigenvalue extrema untouched for this flux
    lam[0] = lam[1] = lam[2] = __longlong_as_double(0x7ff8000000000000LL);
    return fmax(fabs(ub_a), fmax(fabs(ub_a + c_a), fabs(ub_a - c_a)));
}

// roe_c2, when not null and FLUX is the plain or low-Mach-fix Roe flux (the
// fluxes that average qL and qR themselves, roe_c2_of), receives the c^2 of
// their Roe average: (gamma - 1)(h - q^2/2), of the sign of the Roe state's
// pressure (Compute_Limiter_RoePressureCorrection, Limiters.cpp:311-356, forms
// p = (rho/gamma)(gamma - 1)(h - q^2/2) from the same averages, or p + pinf for
// the stiffened gas), so the limiter's Roe-average pressure check costs no
// second average.  The two agree in sign except within rounding of zero.
template <int FLUX>
__host__ __device__ constexpr bool roe_c2_of() { return FLUX == CFD_FLUX_ROE || FLUX == CFD_FLUX_ROE_LMFIX; }

template <int FLUX, int V = -1>
__device__ __forceinline__ double edge_flux(const double qL[5], const double qR[5], double nx, double ny, double nz,
                                            double area, const Flow &f, double conv[5], double diss[5],
                                            double lam[3], double *roe_c2 = nullptr) {
    if (FLUX == CFD_FLUX_HLLC) return hllc_flux<V>(qL, qR, nx, ny, nz, area, f, conv, diss, lam);
    if (FLUX == CFD_FLUX_AUSM) return ausmp_flux<V>(qL, qR, nx, ny, nz, area, f, conv, diss, lam);
    if (FLUX == CFD_FLUX_VANLEER) return vanleer_flux<V>(qL, qR, nx, ny, nz, area, f, conv, diss, lam);
    if (FLUX == CFD_FLUX_ROE_PRECOND) return roe_precond_flux<V>(qL, qR, nx, ny, nz, area, f, conv, diss, lam);
    if (FLUX == CFD_FLUX_ROE_THORNBER) {
        double mL[5], mR[5];
        thornber_states<V>(qL, qR, f, mL, mR);
        return roe_flux<false, V>(mL, mR, nx, ny, nz, area, f, conv, diss, lam);
    }
    return roe_flux<FLUX == CFD_FLUX_ROE_LMFIX, V>(qL, qR, nx, ny, nz, area, f, conv, diss, lam, roe_c2);
}

// The Roe family (plain, low-Mach fix, preconditioned): the limiter pressure fix applies.
__host__ __device__ constexpr bool is_roe_flux(int flux) {
    return flux == CFD_FLUX_ROE || flux == CFD_FLUX_ROE_LMFIX || flux == CFD_FLUX_ROE_PRECOND ||
           flux == CFD_FLUX_ROE_THORNBER;
}

// Pressure of the Roe-averaged state of two reconstructed face states
// (Compute_RoeVariables, Roe_Fluxes.cpp:3609-3633, tested in
// Compute_Limiter_RoePressureCorrection, Limiters.cpp:311-356).
// For the stiffened gas the value returned is p + pinf of the Roe state (its
// c^2 = (g - 1) h holds for either gas), the quantity whose sign matters.
// Roe-averaged p + pinf of two reconstructed (rho, u, v, w, p) face states:
// Compute_RoeAverage_Q and Material_Get_Pressure with VARIABLE_RUP
// (MPFLOW3D/src/Limiters.cpp:350-352), p + pinf = (gamma - 1) rho (ht - q^2/2) / gamma.
__device__ __forceinline__ double roe_avg_pressure_rup(const double qa[5], const double qb[5], const Flow &f) {
    const double ra = qa[0], rb = qb[0];
    const double k = f.gamma * f.inv_gm1;
    const double ha = k * (qa[4] + f.pinf) / ra + 0.5 * (qa[1] * qa[1] + qa[2] * qa[2] + qa[3] * qa[3]);
    const double hb = k * (qb[4] + f.pinf) / rb + 0.5 * (qb[1] * qb[1] + qb[2] * qb[2] + qb[3] * qb[3]);
    const double rho = sqrt(ra * rb), sg = rho / (ra + rho);
    const double u = qa[1] + sg * (qb[1] - qa[1]), v = qa[2] + sg * (qb[2] - qa[2]), w = qa[3] + sg * (qb[3] - qa[3]);
    const double ht = ha + sg * (hb - ha);
    return f.gm1 * rho * (ht - 0.5 * (u * u + v * v + w * w)) / f.gamma;
}

template <int V = -1>
__device__ __forceinline__ double roe_avg_pressure(const double qa[5], const double qb[5], const Flow &f) {
    if (vars_rup<V>(f)) return roe_avg_pressure_rup(qa, qb, f);
    const double g = f.gamma, gpinf = f.gpinf;
    const double ra = qa[0], rb = qb[0];
    const double ia = 1.0 / ra, ib = 1.0 / rb;
    const double ua = qa[1] * ia, va = qa[2] * ia, wa = qa[3] * ia;
    const double ub = qb[1] * ib, vb = qb[2] * ib, wb = qb[3] * ib;
    const double pa = (g - 1.0) * (qa[4] - 0.5 * ra * (ua * ua + va * va + wa * wa)) - gpinf;
    const double pb = (g - 1.0) * (qb[4] - 0.5 * rb * (ub * ub + vb * vb + wb * wb)) - gpinf;
    const double ha = (qa[4] + pa) * ia, hb = (qb[4] + pb) * ib;
    const double rho = sqrt(ra * rb), sg = rho / (ra + rho);
    const double u = ua + sg * (ub - ua), v = va + sg * (vb - va), w = wa + sg * (wb - wa);
    const double ht = ha + sg * (hb - ha);
    const double q2 = u * u + v * v + w * w;
    const double e = (rho / g) * (ht + 0.5 * (g - 1.0) * q2);
    return (g - 1.0) * (e - 0.5 * rho * q2);
}

// Reconstructed-pressure test of Compute_Limiter_PressureCorrection
// (Euler3D/src/Limiters.cpp:296-301): p < 0, without the division when rho > 0
// (p + pinf < 0 for the stiffened gas).
template <int V = -1>
__device__ __forceinline__ bool recon_pressure_negative(const double q[5], const Flow &f) {
    if (vars_rup<V>(f)) return q[4] + f.pinf < 0.0;  // Material_Get_Pressure of a RUP state (Limiters.cpp:296-297)
    const double m2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    return q[0] > 0.0 ? (2.0 * q[0] * (q[4] - f.pinf) < m2) : (f.gm1 * ((q[4] - f.pinf) - (0.5 / q[0]) * m2) < 0.0);
}

__device__ __forceinline__ void store_low(float *p, double v) { *p = (float)v; }
__device__ __forceinline__ void store_low(uint16_t *p, double v) {
    __nv_bfloat16 b = __double2bfloat16(v);
    *p = *reinterpret_cast<uint16_t *>(&b);
}
__device__ __forceinline__ double load_low(const float *p) { return (double)*p; }
__device__ __forceinline__ double load_low(const uint16_t *p) {
    __nv_bfloat16 b = *reinterpret_cast<const __nv_bfloat16 *>(p);
    return (double)__bfloat162float(b);
}

// Kernels shared across translation units (defined in core.cu / linsolve.cu).
__global__ void k_lu_nopivot(int nnode, const double *__restrict__ A, const int *__restrict__ IAU,
                             double *__restrict__ LU);
__global__ void k_gs_level(int nrows, const int *__restrict__ rows, const int *__restrict__ IA,
                           const int *__restrict__ JA, const int *__restrict__ IAU, const double *__restrict__ A,
                           const double *__restrict__ B, const double *__restrict__ LU, double *__restrict__ X,
                           double *__restrict__ rowrms);
__global__ void k_sum_partial(const double *__restrict__ x, int64_t n, double *__restrict__ part);
__global__ void k_sum_one(const double *__restrict__ part, int nblk, double *__restrict__ out);

// Deterministic sum of a plain vector (host result).
int reduce_sum_plain(cfd_ctx *c, const double *x, int64_t n, double *out_host);

// Patch residual kernel: threads per CTA (= edges per chunk), node variables
// staged per patch node for second order (Q 5, gradients 15, limiters 5,
// coordinates 3), and the dynamic shared memory it needs.  128-node patches of
// a tet mesh have ~350 patch + halo nodes (~78 KB + 22 KB chunk buffer, two
// CTAs per SM); larger halos still run, one CTA per SM, up to kPatchSmemMax.
constexpr int PATCH_CHUNK = 256;
constexpr int PATCH_NV2 = 28;
constexpr size_t kPatchSmemMax = 220 * 1024;
inline size_t patch_smem_bytes(int nlocmax, bool second) {
    return ((size_t)(second ? PATCH_NV2 : 5) * nlocmax + 11 * PATCH_CHUNK) * sizeof(double);
}

// The limiter fixes left to the residual (reconstructed-pressure correction,
// Roe-average pressure fix) as their own passes over the node graph
// (gradient.cu); used when the limiters are needed before a gather residual.
int limiter_fix_standalone(cfd_ctx *c);
// k_roe_pressure_fix from c->work into c->phi; gate as in the kernel
int launch_roe_pressure_fix(cfd_ctx *c, const int *gate);

// The patch residual kernel is selected (it carries no reconstructed-pressure check).
inline bool patch_kernel(const cfd_ctx *c) { return c->use_patch && c->params.residual_kernel == 1; }

}  // namespace cfd
