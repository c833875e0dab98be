// Node gradients (least squares as the reference, or Green-Gauss on the median
// dual) and the Venkatakrishnan limiter with the reference's pressure
// corrections.  One thread per node, neighbour loops in the node graph's fixed
// (sorted) order, so every result is deterministic.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>

#include "ctx.cuh"
#include "kernels.cuh"

namespace cfd {

// Least-squares Gram-Schmidt coefficients r11..r33, ro22, ro33
// (Compute_Least_Square_Gradient_Coefficients, Euler3D/src/Gradient.cpp:137-228).
__global__ void k_lsq_coeff(int nnode, const int64_t *__restrict__ sell_ptr, const int *__restrict__ sell_nbr,
                            const int *__restrict__ deg,
                            const double *__restrict__ xyz, int weighted, double *__restrict__ cf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnode) return;
    const int64_t sb = sell_ptr[i >> 5] + (i & 31);
    const int dgi = deg[i];
    const double xi = xyz[i], yi = xyz[nnode + i], zi = xyz[2 * nnode + i];
    double r11 = 0, r12 = 0, r13 = 0, r22 = 0, r23 = 0, r33 = 0, ro22 = 0, ro33 = 0;
    for (int k = 0; k < dgi; k++) {
        int j = sell_nbr[sb + 32 * k];
        j = j >= 0 ? j : ~j;
        double dx = xyz[j] - xi, dy = xyz[nnode + j] - yi, dz = xyz[2 * nnode + j] - zi;
        const double a = weighted ? 1.0 / sqrt(dx * dx + dy * dy + dz * dz) : 1.0;
        dx *= a; dy *= a; dz *= a;
        r11 += dx * dx; r12 += dx * dy; r13 += dx * dz;
    }
    for (int k = 0; k < dgi; k++) {
        int j = sell_nbr[sb + 32 * k];
        j = j >= 0 ? j : ~j;
        double dx = xyz[j] - xi, dy = xyz[nnode + j] - yi, dz = xyz[2 * nnode + j] - zi;
        const double a = weighted ? 1.0 / sqrt(dx * dx + dy * dy + dz * dz) : 1.0;
        dx *= a; dy *= a; dz *= a;
        const double t = dy - (r12 / r11) * dx;
        r22 += t * t; r23 += t * dz; ro22 += t * dy;
    }
    for (int k = 0; k < dgi; k++) {
        int j = sell_nbr[sb + 32 * k];
        j = j >= 0 ? j : ~j;
        double dx = xyz[j] - xi, dy = xyz[nnode + j] - yi, dz = xyz[2 * nnode + j] - zi;
        const double a = weighted ? 1.0 / sqrt(dx * dx + dy * dy + dz * dz) : 1.0;
        dx *= a; dy *= a; dz *= a;
        const double t = dz - (r13 / r11) * dx - (r23 / r22) * (dy - (r12 / r11) * dx);
        r33 += t * t; ro33 += t * dz;
    }
    double *o = cf + (int64_t)i * 8;
    o[0] = r11; o[1] = r12; o[2] = r13; o[3] = r22; o[4] = r23; o[5] = r33; o[6] = ro22; o[7] = ro33;
}

// Least-squares gradient of Q1..Q5 (Compute_Least_Square_Gradient, Gradient.cpp:232-296).
__global__ void __launch_bounds__(128) k_lsq_grad(int nnode, int64_t ldq, const double *__restrict__ Q,
                                                  const int64_t *__restrict__ sell_ptr, const int *__restrict__ sell_nbr,
                            const int *__restrict__ deg,
                                                  const double *__restrict__ xyz, int weighted,
                                                  const double *__restrict__ cf, double *__restrict__ g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnode) return;
    const int64_t sb = sell_ptr[i >> 5] + (i & 31);
    const int dgi = deg[i];
    const double *c = cf + (int64_t)i * 8;
    const double r11 = c[0], r12 = c[1], r13 = c[2], r22 = c[3], r23 = c[4], ro22 = c[6], ro33 = c[7];
    const double xi = xyz[i], yi = xyz[nnode + i], zi = xyz[2 * nnode + i];
    double qi[5], gx[5] = {0, 0, 0, 0, 0}, gy[5] = {0, 0, 0, 0, 0}, gz[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int v = 0; v < 5; v++) qi[v] = Q[v * ldq + i];
    for (int k = 0; k < dgi; k++) {
        int j = sell_nbr[sb + 32 * k];
        j = j >= 0 ? j : ~j;
        double dx = xyz[j] - xi, dy = xyz[nnode + j] - yi, dz = xyz[2 * nnode + j] - zi;
        const double a = weighted ? 1.0 / sqrt(dx * dx + dy * dy + dz * dz) : 1.0;
        dx *= a; dy *= a; dz *= a;
        const double Wz = (dz - (r13 / r11) * dx - (r23 / r22) * (dy - (r12 / r11) * dx)) / ro33;
        const double Wy = (dy - (r12 / r11) * dx - r23 * Wz) / ro22;
        const double Wx = (dx - r12 * Wy - r13 * Wz) / r11;
#pragma unroll
        for (int v = 0; v < 5; v++) {
            const double d = Q[v * ldq + j] - qi[v];
            gx[v] += Wx * a * d;
            gy[v] += Wy * a * d;
            gz[v] += Wz * a * d;
        }
    }
#pragma unroll
    for (int v = 0; v < 5; v++) {
        g[(3 * v) * (int64_t)nnode + i] = gx[v];
        g[(3 * v + 1) * (int64_t)nnode + i] = gy[v];
        g[(3 * v + 2) * (int64_t)nnode + i] = gz[v];
    }
}

// Green-Gauss on the median dual: grad Q_i = (1/V_i) sum_faces Q_f S_f with
// Q_f = (Q_i + Q_j)/2 on interior dual faces and Q_f = Q_i on boundary dual
// faces; written with the closed-surface identity sum_f S_f = 0 as
// (1/V_i) sum_j (Q_j - Q_i)/2 S_ij so that uniform fields give exactly zero.
// (The reference declares GRADINET_METHOD_GREEN_GAUSS, SolverParameters.h:329,
// without implementing it.)
__global__ void __launch_bounds__(128) k_gg_grad(int nnode, int64_t ldq, const double *__restrict__ Q,
                                                 const int64_t *__restrict__ sell_ptr, const int *__restrict__ sell_nbr,
                                                 const int *__restrict__ deg, const double4 *__restrict__ sell_geo,
                                                 const double *__restrict__ vol, double *__restrict__ g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnode) return;
    const int64_t sb = sell_ptr[i >> 5] + (i & 31);
    const int dgi = deg[i];
    double qi[5], gx[5] = {0, 0, 0, 0, 0}, gy[5] = {0, 0, 0, 0, 0}, gz[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int v = 0; v < 5; v++) qi[v] = Q[v * ldq + i];
    for (int k = 0; k < dgi; k++) {
        const int sn = sell_nbr[sb + 32 * k];
        const int j = sn >= 0 ? sn : ~sn;
        const double4 S = sell_geo[sb + 32 * k];  // unit normal L->R and |S|
        const double sg = sn >= 0 ? 0.5 * S.w : -0.5 * S.w;  // outward from i
        const double sx = sg * S.x, sy = sg * S.y, sz = sg * S.z;
#pragma unroll
        for (int v = 0; v < 5; v++) {
            const double d = Q[v * ldq + j] - qi[v];
            gx[v] += d * sx;
            gy[v] += d * sy;
            gz[v] += d * sz;
        }
    }
    const double vi = 1.0 / vol[i];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        g[(3 * v) * (int64_t)nnode + i] = gx[v] * vi;
        g[(3 * v + 1) * (int64_t)nnode + i] = gy[v] * vi;
        g[(3 * v + 2) * (int64_t)nnode + i] = gz[v] * vi;
    }
}

// Reconstructed increment of node i towards neighbour j (Compute_SecondOrderReconstructQ,
// MPFLOW3D/src/HigherOrderReconstructQ.cpp:56-60, without phi):
// frac (Q_j - Q_i) + (1 - frac) grad_i . r.  KAPPA0 is the frac = 0 case (the
// default LIMITER_ORDER): frac (Q_j - Q_i) is then a signed zero and
// (1 - frac) g.r is g.r exactly, so the neighbour's state is not loaded and
// every sum below rounds as in the general form (up to the sign of an exact zero).
template <bool KAPPA0>
__device__ __forceinline__ double recon_incr(double qj, double qi, double gr, double frac) {
    return KAPPA0 ? gr : frac * (qj - qi) + (1.0 - frac) * gr;
}

// Limiter of node i from its state qc, gradient (gx, gy, gz) and the extremes
// of its neighbours' states, as differences dmax = max_j Q_j - qc >= 0 and
// dmin = min_j Q_j - qc <= 0: Venkatakrishnan (Compute_Limiter_Venkatakrishnan,
// Euler3D/src/Limiters.cpp:185-267) or Barth-Jespersen (:117-178), the
// optional variable smoothing (:50-58) and, when PC, the reconstructed-
// pressure correction (Compute_Limiter_PressureCorrection, :273-304).
template <bool KAPPA0, bool PC>
__device__ __forceinline__ void limit_node(int i, int nnode, int64_t ldq, const double *__restrict__ Q, int64_t sb,
                                           int dgi, const int *__restrict__ sell_nbr, const double *__restrict__ xyz,
                                           const Flow &f, const double qc[5], const double dmin[5],
                                           const double dmax[5], const double gx[5], const double gy[5],
                                           const double gz[5], double eps2, double ph[5]) {
    const double frac = f.frac;
    const double xi = xyz[i], yi = xyz[nnode + i], zi = xyz[2 * nnode + i];
#pragma unroll
    for (int v = 0; v < 5; v++) ph[v] = 1.0;
    if (f.limiter == CFD_LIMITER_VENKAT) {
        // phi = min(1, min_edges num/den) with num, den >= 0 (dm and dp share
        // their sign).  The running minimum is kept as a fraction and compared
        // by cross-multiplication, so one division per variable replaces one
        // per edge; the result is the same rounded quotient the reference's
        // per-edge divisions select, except for ties closer than an ulp.
        double bn[5] = {1, 1, 1, 1, 1}, bd[5] = {1, 1, 1, 1, 1};
        // neighbour ids two slots ahead, coordinates one slot ahead
        int sn1 = 0, sn2 = 0;
        double xn = 0.0, yn = 0.0, zn = 0.0;
        if (dgi > 0) {
            sn1 = sell_nbr[sb];
            const int j0 = sn1 >= 0 ? sn1 : ~sn1;
            xn = xyz[j0]; yn = xyz[nnode + j0]; zn = xyz[2 * nnode + j0];
        }
        if (dgi > 1) sn2 = sell_nbr[sb + 32];
        for (int k = 0; k < dgi; k++) {
            const double rx = 0.5 * (xn - xi), ry = 0.5 * (yn - yi), rz = 0.5 * (zn - zi);
            int j = sn1;
            if (k + 1 < dgi) {
                sn1 = sn2;
                const int j1 = sn1 >= 0 ? sn1 : ~sn1;
                xn = xyz[j1]; yn = xyz[nnode + j1]; zn = xyz[2 * nnode + j1];
                if (k + 2 < dgi) sn2 = sell_nbr[sb + 32 * (k + 2)];
            }
            j = j >= 0 ? j : ~j;
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const double qj = KAPPA0 ? 0.0 : Q[v * ldq + j];
                const double q = qc[v] + recon_incr<KAPPA0>(qj, qc[v], gx[v] * rx + gy[v] * ry + gz[v] * rz, frac);
                const double dm = q - qc[v];
                if (dm != 0.0) {
                    const double dp = dm > 0.0 ? dmax[v] : dmin[v];
                    const double num = (dp * dp + eps2) + 2.0 * (dm * dp);
                    const double den = dp * dp + 2.0 * dm * dm + dm * dp + eps2;
                    if (num * bd[v] < bn[v] * den) { bn[v] = num; bd[v] = den; }
                }
            }
        }
#pragma unroll
        for (int v = 0; v < 5; v++) ph[v] = fmax(0.0, bn[v] == bd[v] ? 1.0 : bn[v] / bd[v]);
    } else {  // Barth-Jespersen
        for (int k = 0; k < dgi; k++) {
            int j = sell_nbr[sb + 32 * k];
            j = j >= 0 ? j : ~j;
            const double rx = 0.5 * (xyz[j] - xi), ry = 0.5 * (xyz[nnode + j] - yi), rz = 0.5 * (xyz[2 * nnode + j] - zi);
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const double qj = KAPPA0 ? 0.0 : Q[v * ldq + j];
                const double q = qc[v] + recon_incr<KAPPA0>(qj, qc[v], gx[v] * rx + gy[v] * ry + gz[v] * rz, frac);
                const double dm = q - qc[v];
                double t = 1.0;
                if (dm > 0.0) t = fmin(1.0, dmax[v] / dm);
                else if (dm < 0.0) t = fmin(1.0, dmin[v] / dm);
                ph[v] = fmax(0.0, fmin(ph[v], t));
            }
        }
    }
    if (f.limiter_smooth) {
        double m = ph[0];
#pragma unroll
        for (int v = 1; v < 5; v++) m = fmin(m, ph[v]);
#pragma unroll
        for (int v = 0; v < 5; v++) ph[v] = m;
    }
    // pressure correction: any negative reconstructed pressure -> first order
    if (PC) {
        bool neg = false;
        for (int k = 0; k < dgi; k++) {
            int j = sell_nbr[sb + 32 * k];
            j = j >= 0 ? j : ~j;
            const double rx = 0.5 * (xyz[j] - xi), ry = 0.5 * (xyz[nnode + j] - yi), rz = 0.5 * (xyz[2 * nnode + j] - zi);
            double q[5];
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const double qj = KAPPA0 ? 0.0 : Q[v * ldq + j];
                q[v] = qc[v] + ph[v] * recon_incr<KAPPA0>(qj, qc[v], gx[v] * rx + gy[v] * ry + gz[v] * rz, frac);
            }
            if (recon_pressure_negative(q, f)) neg = true;
        }
        if (neg) {
#pragma unroll
            for (int v = 0; v < 5; v++) ph[v] = 0.0;
        }
    }
}

// Limiter pass over stored gradients (any gradient method).  Without PC the
// pressure correction is left to the residual, whose gather kernel forms the
// same reconstructed states (k_residual_gather, check bit 1), or to k_venkat_pc.
template <bool KAPPA0, bool PC>
__global__ void __launch_bounds__(128) k_venkat(int nnode, int64_t ldq, const double *__restrict__ Q,
                                                const int64_t *__restrict__ sell_ptr, const int *__restrict__ sell_nbr,
                                                const int *__restrict__ deg, const double *__restrict__ xyz,
                                                const double *__restrict__ g, const double *__restrict__ vol, Flow f,
                                                double *__restrict__ phi, int *__restrict__ roeflag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnode) return;
    const int64_t sb = sell_ptr[i >> 5] + (i & 31);
    const int dgi = deg[i];
    roeflag[i] = 0;
    double qc[5], qmin[5], qmax[5], ph[5], gx[5], gy[5], gz[5];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        qc[v] = Q[v * ldq + i];
        qmin[v] = qmax[v] = qc[v];
        gx[v] = g[(3 * v) * (int64_t)nnode + i];
        gy[v] = g[(3 * v + 1) * (int64_t)nnode + i];
        gz[v] = g[(3 * v + 2) * (int64_t)nnode + i];
    }
    const double eps2 = 6.0 * f.venkat_eps_k3 * vol[i] / M_PI;
    for (int k = 0; k < dgi; k++) {
        int j = sell_nbr[sb + 32 * k];
        j = j >= 0 ? j : ~j;
#pragma unroll
        for (int v = 0; v < 5; v++) {
            const double q = Q[v * ldq + j];
            qmin[v] = fmin(qmin[v], q);
            qmax[v] = fmax(qmax[v], q);
        }
    }
#pragma unroll
    for (int v = 0; v < 5; v++) {
        qmin[v] -= qc[v];
        qmax[v] -= qc[v];
    }
    limit_node<KAPPA0, PC>(i, nnode, ldq, Q, sb, dgi, sell_nbr, xyz, f, qc, qmin, qmax, gx, gy, gz, eps2, ph);
#pragma unroll
    for (int v = 0; v < 5; v++) phi[v * (int64_t)nnode + i] = ph[v];
}

// Green-Gauss gradient and limiter in one pass over the node graph: the
// gradient loop of k_gg_grad (same sums, same order, so the same gradients
// bit for bit) also takes the neighbours' extremes, and the limiter then
// reads the gradient from registers.  Saves the limiter's own neighbour pass
// and its re-read of the 15 gradient components.
template <bool KAPPA0, bool PC>
__global__ void __launch_bounds__(128, 4) k_gg_limiter(int nnode, int64_t ldq, const double *__restrict__ Q,
                                                    const int64_t *__restrict__ sell_ptr,
                                                    const int *__restrict__ sell_nbr, const int *__restrict__ deg,
                                                    const double4 *__restrict__ sell_geo,
                                                    const double *__restrict__ xyz, const double *__restrict__ vol,
                                                    Flow f, double *__restrict__ g, double *__restrict__ phi,
                                                    int *__restrict__ roeflag, double *__restrict__ lg, int lo,
                                                    int hi) {
    // nodes [lo, hi); the whole mesh is 0, nnode
    const int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi) return;
    const int64_t sb = sell_ptr[i >> 5] + (i & 31);
    const int dgi = deg[i];
    roeflag[i] = 0;
    double qi[5], qmin[5], qmax[5], gx[5] = {0, 0, 0, 0, 0}, gy[5] = {0, 0, 0, 0, 0}, gz[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int v = 0; v < 5; v++) qmin[v] = qmax[v] = qi[v] = Q[v * ldq + i];
    // slot k+1's neighbour id and face are loaded while slot k is summed
    int sn_next = dgi > 0 ? sell_nbr[sb] : 0, sn_far = dgi > 1 ? sell_nbr[sb + 32] : 0;
    double4 S_next = dgi > 0 ? sell_geo[sb] : make_double4(0, 0, 0, 0);
    double qn[5] = {0, 0, 0, 0, 0};
    if (dgi > 0) {
        const int j0 = sn_next >= 0 ? sn_next : ~sn_next;
#pragma unroll
        for (int v = 0; v < 5; v++) qn[v] = Q[v * ldq + j0];
    }
    for (int k = 0; k < dgi; k++) {
        const int sn = sn_next;
        const double4 S = S_next;
        double qcur[5];
#pragma unroll
        for (int v = 0; v < 5; v++) qcur[v] = qn[v];
        if (k + 1 < dgi) {
            sn_next = sn_far;
            S_next = sell_geo[sb + 32 * (k + 1)];
            const int j1 = sn_next >= 0 ? sn_next : ~sn_next;
#pragma unroll
            for (int v = 0; v < 5; v++) qn[v] = Q[v * ldq + j1];
            if (k + 2 < dgi) sn_far = sell_nbr[sb + 32 * (k + 2)];
        }
        const double sg = sn >= 0 ? 0.5 * S.w : -0.5 * S.w;
        const double sx = sg * S.x, sy = sg * S.y, sz = sg * S.z;
#pragma unroll
        for (int v = 0; v < 5; v++) {
            const double qj = qcur[v];
            const double d = qj - qi[v];
            gx[v] += d * sx;
            gy[v] += d * sy;
            gz[v] += d * sz;
            qmin[v] = fmin(qmin[v], qj);
            qmax[v] = fmax(qmax[v], qj);
        }
    }
    const double vinv = 1.0 / vol[i];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        gx[v] *= vinv;
        gy[v] *= vinv;
        gz[v] *= vinv;
        g[(3 * v) * (int64_t)nnode + i] = gx[v];
        g[(3 * v + 1) * (int64_t)nnode + i] = gy[v];
        g[(3 * v + 2) * (int64_t)nnode + i] = gz[v];
        qmin[v] -= qi[v];
        qmax[v] -= qi[v];
    }
    const double eps2 = 6.0 * f.venkat_eps_k3 * vol[i] / M_PI;
    double ph[5];
    limit_node<KAPPA0, PC>(i, nnode, ldq, Q, sb, dgi, sell_nbr, xyz, f, qi, qmin, qmax, gx, gy, gz, eps2, ph);
#pragma unroll
    for (int v = 0; v < 5; v++) phi[v * (int64_t)nnode + i] = ph[v];
    if (KAPPA0 && lg) {
        // limited gradients for the residual's neighbour gathers: with frac = 0
        // the face state is Q + phi grad.r, and a neighbour's (phi grad) is 15
        // loads where grad and phi are 20
#pragma unroll
        for (int v = 0; v < 5; v++) {
            lg[(3 * v) * (int64_t)nnode + i] = ph[v] * gx[v];
            lg[(3 * v + 1) * (int64_t)nnode + i] = ph[v] * gy[v];
            lg[(3 * v + 2) * (int64_t)nnode + i] = ph[v] * gz[v];
        }
    }
}

// The reconstructed-pressure correction alone (Compute_Limiter_PressureCorrection,
// Euler3D/src/Limiters.cpp:273-304), in place: node i reads only its own
// limiters.  Resolves a correction that k_venkat<.., false> left to the residual
// when the limiters are needed before (or without) a gather residual.
template <bool KAPPA0>
__global__ void __launch_bounds__(128) k_venkat_pc(int nnode, int64_t ldq, const double *__restrict__ Q,
                                                   const int64_t *__restrict__ sell_ptr,
                                                   const int *__restrict__ sell_nbr, const int *__restrict__ deg,
                                                   const double *__restrict__ xyz, const double *__restrict__ g,
                                                   Flow f, double *__restrict__ phi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnode) return;
    const int64_t sb = sell_ptr[i >> 5] + (i & 31);
    const int dgi = deg[i];
    const double frac = f.frac;
    double qc[5], ph[5], gx[5], gy[5], gz[5];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        qc[v] = Q[v * ldq + i];
        ph[v] = phi[v * (int64_t)nnode + i];
        gx[v] = g[(3 * v) * (int64_t)nnode + i];
        gy[v] = g[(3 * v + 1) * (int64_t)nnode + i];
        gz[v] = g[(3 * v + 2) * (int64_t)nnode + i];
    }
    const double xi = xyz[i], yi = xyz[nnode + i], zi = xyz[2 * nnode + i];
    bool neg = false;
    for (int k = 0; k < dgi && !neg; k++) {
        int j = sell_nbr[sb + 32 * k];
        j = j >= 0 ? j : ~j;
        const double rx = 0.5 * (xyz[j] - xi), ry = 0.5 * (xyz[nnode + j] - yi), rz = 0.5 * (xyz[2 * nnode + j] - zi);
        double q[5];
#pragma unroll
        for (int v = 0; v < 5; v++) {
            const double qj = KAPPA0 ? 0.0 : Q[v * ldq + j];
            q[v] = qc[v] + ph[v] * recon_incr<KAPPA0>(qj, qc[v], gx[v] * rx + gy[v] * ry + gz[v] * rz, frac);
        }
        neg = recon_pressure_negative(q, f);
    }
    if (neg) {
#pragma unroll
        for (int v = 0; v < 5; v++) phi[v * (int64_t)nnode + i] = 0.0;
    }
}

// Roe-average pressure correction (Compute_Limiter_RoePressureCorrection,
// Limiters.cpp:311-356, applied for the Roe flux at :61-110): a node's limiters
// drop to zero when the Roe-averaged state of any of its reconstructed edges
// has negative pressure.  Evaluated against the limiters of the previous
// pass (Jacobi order); the reference sweeps nodes in sequence, which gives
// the same result whenever this fix does not cascade.
__global__ void __launch_bounds__(128) k_roe_pressure_fix(int nnode, int64_t ldq, const double *__restrict__ Q,
                                                          const int64_t *__restrict__ sell_ptr, const int *__restrict__ sell_nbr,
                            const int *__restrict__ deg,
                                                          const double *__restrict__ xyz,
                                                          const double *__restrict__ g, Flow f,
                                                          const int *__restrict__ gate,
                                                          const double *__restrict__ phi_in, double *__restrict__ phi) {
    // gate: the residual's fix counters; this full pass is needed only when the
    // reconstructed-pressure correction changed some limiter (gate[1] > 0)
    if (gate && gate[1] == 0) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnode; i += gridDim.x * blockDim.x) {
        const int64_t sb = sell_ptr[i >> 5] + (i & 31);
        const int dgi = deg[i];
        const double frac = f.frac;
        bool neg = false;
        const double xi = xyz[i], yi = xyz[nnode + i], zi = xyz[2 * nnode + i];
        for (int k = 0; k < dgi && !neg; k++) {
            int j = sell_nbr[sb + 32 * k];
            j = j >= 0 ? j : ~j;
            const double rx = 0.5 * (xyz[j] - xi), ry = 0.5 * (xyz[nnode + j] - yi), rz = 0.5 * (xyz[2 * nnode + j] - zi);
            double qa[5], qb[5];
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const double ci = Q[v * ldq + i], cj = Q[v * ldq + j];
                const double pi_ = phi_in[v * (int64_t)nnode + i], pj = phi_in[v * (int64_t)nnode + j];
                qa[v] = ci + pi_ * (frac * (cj - ci) + (1.0 - frac) * (g[(3 * v) * (int64_t)nnode + i] * rx +
                                                                      g[(3 * v + 1) * (int64_t)nnode + i] * ry +
                                                                      g[(3 * v + 2) * (int64_t)nnode + i] * rz));
                qb[v] = cj + pj * (frac * (ci - cj) - (1.0 - frac) * (g[(3 * v) * (int64_t)nnode + j] * rx +
                                                                     g[(3 * v + 1) * (int64_t)nnode + j] * ry +
                                                                     g[(3 * v + 2) * (int64_t)nnode + j] * rz));
            }
            if (f.rup) {
                if (roe_avg_pressure_rup(qa, qb, f) < 0.0) neg = true;
                continue;
            }
            // Compute_RoeVariables (Roe_Fluxes.cpp:3609-3633)
            const double ra = qa[0], rb = qb[0];
            const double ua = qa[1] / ra, va = qa[2] / ra, wa = qa[3] / ra;
            const double ub = qb[1] / rb, vb = qb[2] / rb, wb = qb[3] / rb;
            const double pa = f.gm1 * (qa[4] - 0.5 * ra * (ua * ua + va * va + wa * wa)) - f.gpinf;
            const double pb = f.gm1 * (qb[4] - 0.5 * rb * (ub * ub + vb * vb + wb * wb)) - f.gpinf;
            const double ha = (qa[4] + pa) / ra, hb = (qb[4] + pb) / rb;
            const double rho = sqrt(ra * rb), sg = rho / (ra + rho);
            const double u = ua + sg * (ub - ua), v = va + sg * (vb - va), w = wa + sg * (wb - wa);
            const double ht = ha + sg * (hb - ha);
            double qr[5];
            qr[0] = rho; qr[1] = rho * u; qr[2] = rho * v; qr[3] = rho * w;
            qr[4] = (rho / f.gamma) * (ht + 0.5 * f.gm1 * (u * u + v * v + w * w));
            const double p = f.gm1 * (qr[4] - (0.5 / qr[0]) * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]));
            if (p < 0.0) neg = true;
        }
#pragma unroll
        for (int v = 0; v < 5; v++) phi[v * (int64_t)nnode + i] = neg ? 0.0 : phi_in[v * (int64_t)nnode + i];
    }
}

template <bool KAPPA0, bool PC>
static void launch_venkat(cfd_ctx *c) {
    k_venkat<KAPPA0, PC><<<grid_for(c->nnode, 128), 128, 0, c->stream>>>(
        c->nnode, c->ldq, c->Q.p, c->sell_ptr.p, c->sell_nbr.p, c->deg.p, c->xyz.p, c->grad.p, c->cvol.p, c->flow,
        c->phi.p, c->roeflag.p);
}

template <bool KAPPA0, bool PC>
static void launch_gg_limiter(cfd_ctx *c, double *lg, double *phi_out, int lo, int hi) {
    k_gg_limiter<KAPPA0, PC><<<grid_for(hi - lo, 128), 128, 0, c->stream>>>(
        c->nnode, c->ldq, c->Q.p, c->sell_ptr.p, c->sell_nbr.p, c->deg.p, c->sell_geo.p, c->xyz.p, c->cvol.p, c->flow,
        c->grad.p, phi_out, c->roeflag.p, lg, lo, hi);
}

template <bool KAPPA0, bool PC>
static void launch_gg_limiter(cfd_ctx *c, double *lg) {
    launch_gg_limiter<KAPPA0, PC>(c, lg, c->phi_next.p, 0, c->nnode);
}

// Whether the next limiter leaves its reconstructed-pressure correction to
// the residual: only the gather residual kernel carries that check.
static bool limiter_defers_pc(const cfd_ctx *c) { return !patch_kernel(c); }

}  // namespace cfd

using namespace cfd;

extern "C" {

int cfd_gradient(cfd_ctx *c) {
    if (!c || !c->has_mesh) { set_error("cfd_gradient: no mesh"); return CFD_ERR_STATE; }
    CFD_CUDA(cudaSetDevice(c->device));
    const int n = c->nnode;
    CFD_CUDA(c->grad.alloc((size_t)15 * n));
    c->phi_next_valid = false;
    c->lgrad_valid = c->lgrad_pending = false;  // grad changes
    const bool with_limiter = c->params.order == CFD_ORDER_SECOND && c->params.limiter != CFD_LIMITER_NONE;
    if (c->params.gradient == CFD_GRAD_GG && with_limiter) {
        // second order with a limiter: the limiter of this state is formed in
        // the same pass and taken by the next cfd_limiter unless the state or
        // the parameters change before it (phi_next_valid)
        CFD_CUDA(c->phi_next.alloc((size_t)5 * n));
        const bool kappa0 = c->flow.frac == 0.0, defer = limiter_defers_pc(c);
        // the gather residual reads the limited gradients (frac = 0)
        double *lg = nullptr;
        if (kappa0 && !patch_kernel(c)) {
            CFD_CUDA(c->lgrad.alloc((size_t)15 * n));
            lg = c->lgrad.p;
        }
        if (kappa0) {
            if (defer) launch_gg_limiter<true, false>(c, lg);
            else launch_gg_limiter<true, true>(c, lg);
        } else {
            if (defer) launch_gg_limiter<false, false>(c, lg);
            else launch_gg_limiter<false, true>(c, lg);
        }
        CFD_LAUNCH_CHECK();
        c->phi_next_valid = true;
        c->phi_next_defers_pc = defer;
        c->lgrad_pending = lg != nullptr;
    } else if (c->params.gradient == CFD_GRAD_GG) {
        k_gg_grad<<<grid_for(n, 128), 128, 0, c->stream>>>(n, c->ldq, c->Q.p, c->sell_ptr.p, c->sell_nbr.p, c->deg.p,
                                                             c->sell_geo.p, c->cvol.p, c->grad.p);
    } else {
        // coefficients depend on the mesh and the weight only (FlagLSCoeff, Gradient.cpp:245-252)
        if (c->lsq_weight != c->params.ls_weight || c->ggw.n != (size_t)8 * n) {
            CFD_CUDA(c->ggw.alloc((size_t)8 * n));
            k_lsq_coeff<<<grid_for(n, 128), 128, 0, c->stream>>>(n, c->sell_ptr.p, c->sell_nbr.p, c->deg.p, c->xyz.p,
                                                                   c->params.ls_weight, c->ggw.p);
            CFD_LAUNCH_CHECK();
            c->lsq_weight = c->params.ls_weight;
        }
        k_lsq_grad<<<grid_for(n, 128), 128, 0, c->stream>>>(n, c->ldq, c->Q.p, c->sell_ptr.p, c->sell_nbr.p, c->deg.p, c->xyz.p,
                                                              c->params.ls_weight, c->ggw.p, c->grad.p);
    }
    CFD_LAUNCH_CHECK();
    c->has_grad = true;
    return CFD_OK;
}

int cfd_limiter(cfd_ctx *c) {
    if (!c || !c->has_mesh) { set_error("cfd_limiter: no mesh"); return CFD_ERR_STATE; }
    if (!c->has_grad) { set_error("cfd_limiter: call cfd_gradient first"); return CFD_ERR_STATE; }
    CFD_CUDA(cudaSetDevice(c->device));
    const int n = c->nnode;
    CFD_CUDA(c->phi.alloc((size_t)5 * n));
    if (c->params.limiter == CFD_LIMITER_NONE) {
        // Compute_Limiter initialises phi = 1 (Limiters.cpp:24-31)
        CFD_CUDA(c->work.alloc(std::max<size_t>(c->work.n, (size_t)5 * n)));
        return CFD_OK;
    }
    // The reconstructed-pressure correction (Limiters.cpp:273-304) and, for
    // the Roe fluxes, the Roe-average pressure fix (:61-110) test the face
    // states the second-order residual forms anyway: both are left to the
    // next cfd_residual (k_residual_gather flags the nodes that fail and a
    // gated pass applies the fixes), or to limiter_fix_standalone when the
    // limiters are read back or consumed by another kernel first.
    bool defer_pc;
    c->lgrad_valid = false;
    if (c->phi_next_valid) {
        // formed by cfd_gradient together with the gradient of this state
        c->phi.swap(c->phi_next);
        c->phi_next_valid = false;
        defer_pc = c->phi_next_defers_pc;
        c->lgrad_valid = c->lgrad_pending;
    } else {
        const bool kappa0 = c->flow.frac == 0.0;
        defer_pc = limiter_defers_pc(c);
        if (kappa0) {
            if (defer_pc) launch_venkat<true, false>(c);
            else launch_venkat<true, true>(c);
        } else {
            if (defer_pc) launch_venkat<false, false>(c);
            else launch_venkat<false, true>(c);
        }
        CFD_LAUNCH_CHECK();
    }
    c->pc_fix_pending = defer_pc;
    c->roe_fix_pending = is_roe_flux(c->params.flux_scheme);
    if (c->pc_fix_pending || c->roe_fix_pending)
        CFD_CUDA(cudaMemsetAsync(c->fixcount.p, 0, 2 * sizeof(int), c->stream));
    return CFD_OK;
}

}  // extern "C"

namespace cfd {
int gg_limiter_range(cfd_ctx *c, double *phi_out, int lo, int hi) {
    if (hi <= lo) return CFD_OK;
    if (c->flow.frac == 0.0) launch_gg_limiter<true, false>(c, c->lgrad.p, phi_out, lo, hi);
    else launch_gg_limiter<false, false>(c, nullptr, phi_out, lo, hi);
    CFD_LAUNCH_CHECK();
    return CFD_OK;
}

int launch_roe_pressure_fix(cfd_ctx *c, const int *gate) {
    const int n = c->nnode;
    // gated: usually a no-op, so a short grid that strides when it runs
    const int grid = gate ? std::min(grid_for(n, 128), 4 * c->nsm) : grid_for(n, 128);
    k_roe_pressure_fix<<<grid, 128, 0, c->stream>>>(n, c->ldq, c->Q.p, c->sell_ptr.p, c->sell_nbr.p,
                                                                  c->deg.p, c->xyz.p, c->grad.p, c->flow, gate,
                                                                  c->work.p, c->phi.p);
    CFD_LAUNCH_CHECK();
    return CFD_OK;
}

int limiter_fix_standalone(cfd_ctx *c) {
    const int n = c->nnode;
    c->lgrad_valid = false;  // the fixes may change phi
    if (c->pc_fix_pending) {
        if (c->flow.frac == 0.0)
            k_venkat_pc<true><<<grid_for(n, 128), 128, 0, c->stream>>>(n, c->ldq, c->Q.p, c->sell_ptr.p, c->sell_nbr.p,
                                                                         c->deg.p, c->xyz.p, c->grad.p, c->flow, c->phi.p);
        else
            k_venkat_pc<false><<<grid_for(n, 128), 128, 0, c->stream>>>(n, c->ldq, c->Q.p, c->sell_ptr.p, c->sell_nbr.p,
                                                                          c->deg.p, c->xyz.p, c->grad.p, c->flow, c->phi.p);
        CFD_LAUNCH_CHECK();
        c->pc_fix_pending = false;
    }
    if (!c->roe_fix_pending) return CFD_OK;
    CFD_CUDA(c->work.alloc(std::max<size_t>(c->work.n, (size_t)5 * n)));
    CFD_CUDA(cudaMemcpyAsync(c->work.p, c->phi.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToDevice, c->stream));
    int st = launch_roe_pressure_fix(c, nullptr);
    if (st) return st;
    c->roe_fix_pending = false;
    return CFD_OK;
}
}  // namespace cfd

extern "C" {

int cfd_get_gradients(cfd_ctx *c, double *g) {
    if (!c || !g || !c->has_grad) return CFD_ERR_STATE;
    CFD_CUDA(cudaMemcpyAsync(g, c->grad.p, sizeof(double) * 15 * c->nnode, cudaMemcpyDeviceToHost, c->stream));
    CFD_CUDA(stream_wait(c->stream));
    return CFD_OK;
}

int cfd_get_limiters(cfd_ctx *c, double *phi) {
    if (!c || !phi || !c->phi.p) return CFD_ERR_STATE;
    int st = limiter_fix_standalone(c);
    if (st) return st;
    CFD_CUDA(cudaMemcpyAsync(phi, c->phi.p, sizeof(double) * 5 * c->nnode, cudaMemcpyDeviceToHost, c->stream));
    CFD_CUDA(stream_wait(c->stream));
    return CFD_OK;
}

}  // extern "C"
