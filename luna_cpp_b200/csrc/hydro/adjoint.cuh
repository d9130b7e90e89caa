// The adjoint of one static step (luna-cpp's step_adjoint, src/hydro/finite_volume.hpp:2201-2231): Qbar^n = J^T Qbar^n+1
// at fixed dt, for the FP64 policy, order 1, the per-face loop. Four passes, no atomics (the same bits every run):
//   k_sweep_fit      the forward sweep again, keeping the fit the gradient's adjoint needs (SweepFitHook<false>,
//                    finite_volume.hpp:1763-1926): M's Cholesky factor, M's row 0, the unlimited gradient g0, per
//                    variable the last clip (offset, bound, flags) and the face its bound came through;
//   k_faces_adjoint  once per face: the Riemann adjoint -> the bars of both face states (AdjointFaces, :2078-2102);
//   k_cell_adjoint   per cell, one walk: face-state adjoints -> W and g bars, the limited gradient's adjoint from the
//                    stored fit -> the fit's b bars, bound bars, the cell's own W bar (AdjointCell, :2107-2169);
//   k_gather_adjoint per cell: the neighbours' b and bound bars, then the primitive adjoint into Qbar (:2171-2195).
#pragma once

#include "kernels.cuh"

namespace luna {

template <int D>
struct FitLayout {
    static constexpr int U = D + 1, V = D + 2;
    static constexpr int factor = 0, row0 = U * U, g0 = row0 + U, offset = g0 + V * D, bound = offset + V * D, width = bound + V;
};

// primitive_adjoint (euler.hpp:143-162).
template <int D>
__device__ __forceinline__ void primitive_adjoint(const double* U, const double* Wbar, const GasDev& gas, double* Ubar) {
    constexpr int P = D + 1;
    const double rho = fmax(U[0], gas.smallr), inv_rho = 1.0 / rho;
    double v[D], vb[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        v[k] = U[1 + k] * inv_rho;
        vb[k] = U[1 + k] * (1.0 / rho);
    }
    const double smalle = gas.smallc * gas.smallc / gas.gamma / (gas.gamma - 1.0);
    const int floors = (U[0] >= gas.smallr ? 0 : 1) | (U[P] - 0.5 * rho * dot<D>(vb, vb) >= smalle * rho ? 0 : 2);
    const double ebar = (gas.gamma - 1.0) * Wbar[P];
    double rhobar = Wbar[0], energybar = 0;
    double vbar[D];
#pragma unroll
    for (int k = 0; k < D; ++k) vbar[k] = Wbar[1 + k];
    if (floors & 2) {
        rhobar += smalle * ebar;
    } else {
        energybar = ebar;
        rhobar -= 0.5 * dot<D>(v, v) * ebar;
        const double s = rho * ebar;
#pragma unroll
        for (int k = 0; k < D; ++k) vbar[k] = vbar[k] - v[k] * s;
    }
    rhobar -= dot<D>(v, vbar) * inv_rho;
    Ubar[0] = floors & 1 ? 0.0 : rhobar;
#pragma unroll
    for (int k = 0; k < D; ++k) Ubar[1 + k] = vbar[k] * inv_rho;
    Ubar[P] = energybar;
}

// half_step_adjoint (euler.hpp:241-272): adds J^T halfbar to Wbar and gbar.
template <int D>
__device__ __forceinline__ void half_step_adjoint(const double* W, const double* g, double dt, double gamma, const double* halfbar, double* Wbar,
                                                  double* gbar) {
    constexpr int P = D + 1;
    const double rho = W[0], inv_rho = 1.0 / W[0], rho_c2 = gamma * W[P];
    double Abar[D + 2];
#pragma unroll
    for (int v = 0; v < D + 2; ++v) {
        Wbar[v] += halfbar[v];
        Abar[v] = -0.5 * dt * halfbar[v];
    }
    double inv_rhobar = 0, rho_c2bar = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double vn = W[1 + d];
        Wbar[1 + d] += Abar[0] * g[0 * D + d];
        gbar[0 * D + d] += Abar[0] * vn;
        Wbar[0] += Abar[0] * g[(1 + d) * D + d];
        gbar[(1 + d) * D + d] += Abar[0] * rho;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            Wbar[1 + d] += Abar[1 + k] * g[(1 + k) * D + d];
            gbar[(1 + k) * D + d] += Abar[1 + k] * vn;
            if (k == d) {
                inv_rhobar += Abar[1 + k] * g[P * D + d];
                gbar[P * D + d] += Abar[1 + k] * inv_rho;
            }
        }
        rho_c2bar += Abar[P] * g[(1 + d) * D + d];
        gbar[(1 + d) * D + d] += Abar[P] * rho_c2;
        Wbar[1 + d] += Abar[P] * g[P * D + d];
        gbar[P * D + d] += Abar[P] * vn;
    }
    Wbar[0] -= inv_rho * inv_rho * inv_rhobar;
    Wbar[P] += gamma * rho_c2bar;
}

// detail::side_with_adjoint (euler.hpp:375-398); vbar_in may be null (zero). Returns vn's bar.
template <int D>
__device__ __forceinline__ double side_with_adjoint(const double* W, const double* n, double inverse_gm1, const Side<D, double>& s,
                                                    const double* Fbar, const double* Ubar, double Ebar, const double* vbar_in, double* Wbar) {
    constexpr int P = D + 1;
    const double m = W[0] * s.vn;
    double vbar[D];
#pragma unroll
    for (int k = 0; k < D; ++k) vbar[k] = vbar_in ? vbar_in[k] : 0.0;
    Ebar += Fbar[P] * s.vn + Ubar[P];
    double Pbar = Fbar[P] * s.vn, vnbar = Fbar[P] * (s.E + W[P]), mbar = Fbar[0], rhobar = Ubar[0];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        Pbar += Fbar[1 + k] * n[k];
        mbar += Fbar[1 + k] * s.v[k];
        vbar[k] += Fbar[1 + k] * m + Ubar[1 + k] * W[0];
        rhobar += Ubar[1 + k] * s.v[k];
    }
    rhobar += mbar * s.vn;
    vnbar += mbar * W[0];
    Pbar += Ebar * inverse_gm1;
    rhobar += Ebar * (0.5 * dot<D>(s.v, s.v));
    const double e = Ebar * W[0];
#pragma unroll
    for (int k = 0; k < D; ++k) vbar[k] = vbar[k] + s.v[k] * e;
    Wbar[0] += rhobar;
#pragma unroll
    for (int k = 0; k < D; ++k) Wbar[1 + k] += vbar[k];
    Wbar[P] += Pbar;
    return vnbar;
}

// HLLC::flux_adjoint (euler.hpp:738-832) for a static face (w = 0): only the case the forward took is differentiated; a
// guarded divisor has derivative 0.
template <int D>
__device__ void hllc_flux_adjoint(const double* L, const double* R, const double* n, const GasDev& gas, const double* Fbar, double* Lbar,
                                  double* Rbar) {
    constexpr int P = D + 1;
    constexpr double eps = 1e-20;
    const double vnL = dot<D>(L + 1, n), vnR = dot<D>(R + 1, n);
    const double inv_rhoL = 1.0 / L[0], inv_rhoR = 1.0 / R[0];
    const double c2L = gas.gamma * L[P] * inv_rhoL, c2R = gas.gamma * R[P] * inv_rhoR;
    const bool ok = c2L >= 0 && c2R >= 0;
    const double cL = c2L > 0 ? sqrt(c2L) : 0.0, cR = c2R > 0 ? sqrt(c2R) : 0.0;
    const double sl = vnL - cL, sr = vnR - cR, tl = vnL + cL, tr = vnR + cR;
    const double SL = fmin(sl, sr), SR = fmax(tl, tr);
    const double denomL = L[0] * (SL - vnL), denomR = R[0] * (SR - vnR);
    const double den_raw = denomL - denomR;
    const double SM = (R[P] - L[P] + denomL * vnL - denomR * vnR) / nonzero(den_raw);
    const bool left = ok && (SL >= 0 || SM >= 0);
    const bool star = ok && SL < 0 && (SM >= 0 || SR > 0);
    const bool sl_from_left = !(sr < sl), sr_from_left = !(tr > tl);
    double W[D + 2];
#pragma unroll
    for (int v = 0; v < D + 2; ++v) W[v] = left ? L[v] : R[v];
    const double zero[D] = {};
    Side<D, double> s;
    side_with<D, double>(W, n, zero, gas.inverse_gm1, left ? vnL : vnR, s);
    double Wbar[D + 2];
#pragma unroll
    for (int v = 0; v < D + 2; ++v) Wbar[v] = 0;
    double vnLbar = 0, vnRbar = 0;
    if (!star) {
        const double zeroU[D + 2] = {};
        const double r = side_with_adjoint<D>(W, n, gas.inverse_gm1, s, Fbar, zeroU, 0.0, nullptr, Wbar);
        if (left)
            vnLbar += r;
        else
            vnRbar += r;
    } else {
        const double S = left ? SL : SR, denom = left ? denomL : denomR, inv_side = left ? inv_rhoL : inv_rhoR;
        const bool guard_q = fabs(S - SM) < eps, guard_denom = fabs(denom) < eps, guard_den = fabs(den_raw) < eps;
        const double q = nonzero(S - SM), rho_star = denom / q, inv_denom = 1.0 / nonzero(denom);
        const double a2 = SM - s.vn, a3 = SM + W[P] * inv_denom, E_star = s.E * inv_side + a2 * a3;
        double v_star[D];
#pragma unroll
        for (int k = 0; k < D; ++k) v_star[k] = s.v[k] + n[k] * a2;
        double Sbar = 0, rho_starbar = 0, E_starbar = 0;
        double sUbar[D + 2], v_starbar[D];
#pragma unroll
        for (int v = 0; v < D + 2; ++v) {
            const double U_star = v == 0 ? rho_star : v == P ? rho_star * E_star : rho_star * v_star[v - 1];
            Sbar += Fbar[v] * (U_star - s.U[v]);
            sUbar[v] = -S * Fbar[v];
            const double U_starbar = S * Fbar[v];
            if (v == 0) {
                rho_starbar += U_starbar;
            } else if (v == P) {
                rho_starbar += U_starbar * E_star;
                E_starbar = U_starbar * rho_star;
            } else {
                rho_starbar += U_starbar * v_star[v - 1];
                v_starbar[v - 1] = U_starbar * rho_star;
            }
        }
        const double a2bar = dot<D>(v_starbar, n) + E_starbar * a3, a3bar = E_starbar * a2;
        double SMbar = a3bar + a2bar, vnbar = -a2bar;
        const double inv_denombar = a3bar * W[P];
        const double denombar = (guard_denom ? 0.0 : -inv_denom * inv_denom * inv_denombar) + rho_starbar / q;
        const double qbar = guard_q ? 0.0 : -rho_starbar * rho_star / q;
        Sbar += qbar;
        SMbar -= qbar;
        const double sEbar = E_starbar * inv_side, inv_sidebar = E_starbar * s.E;
        vnbar += side_with_adjoint<D>(W, n, gas.inverse_gm1, s, Fbar, sUbar, sEbar, v_starbar, Wbar);
        Wbar[P] += a3bar * inv_denom;
        const double den = nonzero(den_raw), numbar = SMbar / den, denbar = guard_den ? 0.0 : -SMbar * SM / den;
        double denomLbar = denbar + numbar * vnL, denomRbar = -denbar - numbar * vnR;
        if (left)
            denomLbar += denombar;
        else
            denomRbar += denombar;
        vnLbar += numbar * denomL;
        vnRbar -= numbar * denomR;
        Rbar[P] += numbar;
        Lbar[P] -= numbar;
        if (left)
            vnLbar += vnbar;
        else
            vnRbar += vnbar;
        double invLbar = left ? inv_sidebar : 0.0, invRbar = left ? 0.0 : inv_sidebar;
        double SLbar = denomLbar * L[0], SRbar = denomRbar * R[0];
        if (left)
            SLbar += Sbar;
        else
            SRbar += Sbar;
        Lbar[0] += denomLbar * (SL - vnL);
        vnLbar -= denomLbar * L[0];
        Rbar[0] += denomRbar * (SR - vnR);
        vnRbar -= denomRbar * R[0];
        double cLbar = 0, cRbar = 0;
        if (sl_from_left) {
            vnLbar += SLbar;
            cLbar -= SLbar;
        } else {
            vnRbar += SLbar;
            cRbar -= SLbar;
        }
        if (sr_from_left) {
            vnLbar += SRbar;
            cLbar += SRbar;
        } else {
            vnRbar += SRbar;
            cRbar += SRbar;
        }
        if (c2L > 0) {
            const double c2bar = cLbar / (2 * cL);
            Lbar[P] += c2bar * gas.gamma * inv_rhoL;
            invLbar += c2bar * gas.gamma * L[P];
        }
        if (c2R > 0) {
            const double c2bar = cRbar / (2 * cR);
            Rbar[P] += c2bar * gas.gamma * inv_rhoR;
            invRbar += c2bar * gas.gamma * R[P];
        }
        Lbar[0] -= inv_rhoL * inv_rhoL * invLbar;
        Rbar[0] -= inv_rhoR * inv_rhoR * invRbar;
    }
#pragma unroll
    for (int v = 0; v < D + 2; ++v) {
        Lbar[v] += left ? Wbar[v] : 0.0;
        Rbar[v] += left ? 0.0 : Wbar[v];
    }
#pragma unroll
    for (int k = 0; k < D; ++k) {
        Lbar[1 + k] += vnLbar * n[k];
        Rbar[1 + k] += vnRbar * n[k];
    }
}

// HLL::flux_adjoint (euler.hpp:509-540) for a static face, with detail::side_adjoint (:402-413).
template <int D>
__device__ void hll_flux_adjoint(const double* L, const double* R, const double* n, const GasDev& gas, const double* Fbar, double* Lbar,
                                 double* Rbar) {
    constexpr int P = D + 1;
    const double zero[D] = {};
    Side<D, double> l, r;
    side_with<D, double>(L, n, zero, gas.inverse_gm1, dot<D>(L + 1, n), l);
    side_with<D, double>(R, n, zero, gas.inverse_gm1, dot<D>(R + 1, n), r);
    const double c2l = gas.gamma * L[P] / L[0], c2r = gas.gamma * R[P] / R[0];
    l.c = c2l > 0 ? sqrt(c2l) : 0.0;
    r.c = c2r > 0 ? sqrt(c2r) : 0.0;
    const double a = l.vn - l.c, b = r.vn - r.c, A = l.vn + l.c, B = r.vn + r.c;
    const double SLm = fmin(a, b), SRm = fmax(A, B);
    const int wave = SLm >= 0 ? 1 : SRm <= 0 ? 2 : 0;
    const bool sl_from_left = !(b < a), sr_from_left = !(B > A);
    const double SL = sl_from_left ? l.vn - l.c : r.vn - r.c, SR = sr_from_left ? l.vn + l.c : r.vn + r.c;
    double lF[D + 2], rF[D + 2], lU[D + 2], rU[D + 2];
#pragma unroll
    for (int v = 0; v < D + 2; ++v) lF[v] = rF[v] = lU[v] = rU[v] = 0;
    double SLbar = 0, SRbar = 0;
    if (wave == 1) {
#pragma unroll
        for (int v = 0; v < D + 2; ++v) lF[v] = Fbar[v];
    } else if (wave == 2) {
#pragma unroll
        for (int v = 0; v < D + 2; ++v) rF[v] = Fbar[v];
    } else {
        const double inv_dS = 1.0 / (SR - SL);
#pragma unroll
        for (int v = 0; v < D + 2; ++v) {
            const double dU = r.U[v] - l.U[v], F = (SR * l.F[v] - SL * r.F[v] + SL * SR * dU) * inv_dS;
            const double N = Fbar[v] * inv_dS;
            SRbar += -Fbar[v] * F * inv_dS + N * (l.F[v] + SL * dU);
            SLbar += Fbar[v] * F * inv_dS + N * (-r.F[v] + SR * dU);
            lF[v] = SR * N;
            rF[v] = -SL * N;
            rU[v] = SL * SR * N;
            lU[v] = -SL * SR * N;
        }
    }
    double lvn = 0, lc = 0, rvn = 0, rc = 0;
    if (sl_from_left) {
        lvn += SLbar;
        lc -= SLbar;
    } else {
        rvn += SLbar;
        rc -= SLbar;
    }
    if (sr_from_left) {
        lvn += SRbar;
        lc += SRbar;
    } else {
        rvn += SRbar;
        rc += SRbar;
    }
    // detail::side_adjoint for both sides
    lvn += side_with_adjoint<D>(L, n, gas.inverse_gm1, l, lF, lU, 0.0, nullptr, Lbar);
    rvn += side_with_adjoint<D>(R, n, gas.inverse_gm1, r, rF, rU, 0.0, nullptr, Rbar);
#pragma unroll
    for (int k = 0; k < D; ++k) {
        Lbar[1 + k] += lvn * n[k];
        Rbar[1 + k] += rvn * n[k];
    }
    if (c2l > 0) {
        const double c2bar = lc / (2 * l.c);
        Lbar[P] += c2bar * gas.gamma / L[0];
        Lbar[0] -= c2bar * c2l / L[0];
    }
    if (c2r > 0) {
        const double c2bar = rc / (2 * r.c);
        Rbar[P] += c2bar * gas.gamma / R[0];
        Rbar[0] -= c2bar * c2r / R[0];
    }
}

// FaceFlux::side_value (finite_volume.hpp:1342-1347): the double face state and whether it fell back to W.
template <int D>
__device__ __forceinline__ bool side_value(const double* W, const double* g, const double* r, double dt, double gamma, double* Wf) {
    constexpr int V = D + 2;
    double A[V];
    half_step_rate<D, double>(W, g, gamma, A);
#pragma unroll
    for (int v = 0; v < V; ++v) Wf[v] = W[v] - 0.5 * dt * A[v];
#pragma unroll
    for (int v = 0; v < V; ++v) Wf[v] += dot<D>(g + D * v, r);
    const bool fallback = !(Wf[0] > 0 && Wf[D + 1] > 0);
    if (fallback)
#pragma unroll
        for (int v = 0; v < V; ++v) Wf[v] = W[v];
    return fallback;
}

// Resident blocks an SM the adjoint's register-heavy kernels are cut for, and the list entries the gather requests
// together. Measured at 128^3 (step_adjoint, FP64): no cap (128-164 registers) 9.66 ms, 4 blocks (128 registers, a few
// spills) 8.32 ms; a gather batch of 4 changed nothing (9.68 / 8.34 ms); 3 blocks 8.65 ms, and the fit's entry loop
// unrolled by 2 8.54 ms (8.28 for the default).
#ifndef LUNA_ADJ_MIN_BLOCKS
#define LUNA_ADJ_MIN_BLOCKS 4
#endif
#ifndef LUNA_ADJ_GATHER_BATCH
#define LUNA_ADJ_GATHER_BATCH 1
#endif

// The sweep again with the fit kept (Sweep<false, true, SweepFitHook<false>>): the same gradients as k_sweep's FP64
// policy, plus fit rows [N][FitLayout::width] and flags [N][2V] (clipped | upper << 1 | zero << 2; the bound's face).
template <int D, bool Limit>
__global__ void __launch_bounds__(128, LUNA_ADJ_MIN_BLOCKS) k_sweep_fit(MeshDev<D> m, const double* __restrict__ prims, double* __restrict__ grad_out,
                                                   double* __restrict__ fit, int32_t* __restrict__ flags) {
    constexpr int V = D + 2, U = D + 1, GS = grad_stride<D>();
    using FL = FitLayout<D>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    const double* pi = prims + PS * i;
    double Wi[V];
#pragma unroll
    for (int v = 0; v < V; ++v) Wi[v] = pi[v];
    double surface = 0, smallest = __longlong_as_double(0x7ff0000000000000ll);
    double lo[V], hi[V];
    int lo_f[V], hi_f[V];
    double M[U][U], b[V][U];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        lo[v] = finite_max<double>();
        hi[v] = -finite_max<double>();
        lo_f[v] = hi_f[v] = -1;
#pragma unroll
        for (int p = 0; p < U; ++p) b[v][p] = 0;
    }
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s < U; ++s) M[p][s] = 0;
    double centroid[D];
#pragma unroll
    for (int a = 0; a < D; ++a) centroid[a] = m.cen[D * i + a];
    const int first = m.start[i], end = m.start[i + 1];
    for (int k = first; k < end; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e);
        const int j = e >= 0 ? m.neighbour[f] : m.owner[f];
        const double* pj = prims + PS * j;
        double d[D];
        m.separation(i, j, d);
        const double magnitude = m.mag[f];
        surface += magnitude;
        smallest = fmin(smallest, magnitude);
        double X[U];
        X[0] = 1;
#pragma unroll
        for (int p = 1; p < U; ++p) X[p] = d[p - 1] + m.cen[D * j + p - 1] - centroid[p - 1];
#pragma unroll
        for (int p = 0; p < U; ++p)
#pragma unroll
            for (int s = p; s < U; ++s) M[p][s] += magnitude * X[p] * X[s];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const double Wj = pj[v];
            const double dW = Wj - Wi[v];
#pragma unroll
            for (int p = 0; p < U; ++p) b[v][p] += magnitude * X[p] * dW;
            if (Wj < lo[v]) lo[v] = Wj, lo_f[v] = f;
            if (Wj > hi[v]) hi[v] = Wj, hi_f[v] = f;
        }
    }
    const double tiny = 1e-6 * surface;
    const bool any_tiny = smallest < tiny;
    if (any_tiny) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            lo[v] = finite_max<double>();
            hi[v] = -finite_max<double>();
        }
        for (int k = first; k < end; ++k) {
            const int32_t e = m.list[k];
            const int f = list_face(e);
            if (m.mag[f] < tiny) continue;
            const int j = e >= 0 ? m.neighbour[f] : m.owner[f];
            const double* pj = prims + PS * j;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                if (pj[v] < lo[v]) lo[v] = pj[v], lo_f[v] = f;
                if (pj[v] > hi[v]) hi[v] = pj[v], hi_f[v] = f;
            }
        }
    }
    double* fr = fit + static_cast<int64_t>(FL::width) * i;
    {  // cholesky (finite_volume.hpp:677-687), kept in the fit row
        double Lc[U][U];
#pragma unroll
        for (int p = 0; p < U; ++p)
#pragma unroll
            for (int s = 0; s < U; ++s) Lc[p][s] = 0;
#pragma unroll
        for (int p = 0; p < U; ++p)
#pragma unroll
            for (int s = 0; s <= p; ++s) {
                double sum = M[s][p];
#pragma unroll
                for (int k = 0; k < s; ++k) sum -= Lc[p][k] * Lc[s][k];
                Lc[p][s] = p == s ? sqrt(sum) : sum / Lc[s][s];
            }
#pragma unroll
        for (int p = 0; p < U; ++p) {
#pragma unroll
            for (int s = 0; s < U; ++s) fr[FL::factor + p * U + s] = Lc[p][s];
            fr[FL::row0 + p] = M[0][p];
        }
    }
    double g[V * D];
    cholesky_solve<D, double>(M, b, g);
#pragma unroll
    for (int c = 0; c < V * D; ++c) fr[FL::g0 + c] = g[c];
    bool clipped[V], upper[V], zero[V];
    int clip_f[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        clipped[v] = upper[v] = zero[v] = false;
        clip_f[v] = -1;
    }
    if constexpr (Limit) {
        for (int k = first; k < end; ++k) {
            const int f = list_face(m.list[k]);
            if (any_tiny && m.mag[f] < tiny) continue;
            double offset[D];
            m.face_offset(f, i, offset);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                double* gv = g + D * v;
                const double dp = dot<D>(gv, offset);
                if (dp > 0 && Wi[v] + dp > hi[v]) {
                    const double s = hi[v] > Wi[v] ? (hi[v] - Wi[v]) / dp : 0.0;
#pragma unroll
                    for (int a = 0; a < D; ++a) gv[a] = gv[a] * s;
                    clipped[v] = true, upper[v] = true, zero[v] = !(hi[v] > Wi[v]), clip_f[v] = f;
                } else if (dp < 0 && Wi[v] + dp < lo[v]) {
                    const double s = lo[v] < Wi[v] ? (lo[v] - Wi[v]) / dp : 0.0;
#pragma unroll
                    for (int a = 0; a < D; ++a) gv[a] = gv[a] * s;
                    clipped[v] = true, upper[v] = false, zero[v] = !(lo[v] < Wi[v]), clip_f[v] = f;
                }
            }
        }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
        double offset[D];
#pragma unroll
        for (int a = 0; a < D; ++a) offset[a] = 0;
        if (clipped[v]) m.face_offset(clip_f[v], i, offset);
#pragma unroll
        for (int a = 0; a < D; ++a) fr[FL::offset + D * v + a] = offset[a];
        fr[FL::bound + v] = upper[v] ? hi[v] : lo[v];
        flags[2 * V * i + v] = (clipped[v] ? 1 : 0) | (upper[v] ? 2 : 0) | (zero[v] ? 4 : 0);
        flags[2 * V * i + V + v] = upper[v] ? hi_f[v] : lo_f[v];
    }
    double* out = grad_out + static_cast<int64_t>(GS) * i;
#pragma unroll
    for (int c = 0; c < V * D; ++c) out[c] = g[c];
}

// AdjointFaces (finite_volume.hpp:2078-2102): per face, the bars of its two face states from Qbar's jump across it.
template <int D, int Riemann>
__global__ void __launch_bounds__(128, LUNA_ADJ_MIN_BLOCKS) k_faces_adjoint(MeshDev<D> m, const double* __restrict__ prims, const double* __restrict__ grad,
                                                       const double* __restrict__ qbar, double dt, GasDev gas, double* __restrict__ face_bar) {
    constexpr int V = D + 2, GS = grad_stride<D>();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.f) return;
    double a[D];
#pragma unroll
    for (int k = 0; k < D; ++k) a[k] = m.area[D * f + k];
    const double magnitude = sqrt(dot<D>(a, a));
    double Lbar[V], Rbar[V];
#pragma unroll
    for (int v = 0; v < V; ++v) Lbar[v] = Rbar[v] = 0;
    if (magnitude != 0) {
        const int o = m.owner[f], j = m.neighbour[f];
        double ro[D], rj[D], L[V], R[V], Wo[V], Wj[V], go[V * D], gj[V * D], n[D], Fbar[V];
        m.face_offset(f, o, ro);
        m.face_offset(f, j, rj);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            Wo[v] = prims[PS * o + v];
            Wj[v] = prims[PS * j + v];
        }
#pragma unroll
        for (int c = 0; c < V * D; ++c) {
            go[c] = grad[static_cast<int64_t>(GS) * o + c];
            gj[c] = grad[static_cast<int64_t>(GS) * j + c];
        }
        side_value<D>(Wo, go, ro, dt, gas.gamma, L);
        side_value<D>(Wj, gj, rj, dt, gas.gamma, R);
#pragma unroll
        for (int v = 0; v < V; ++v) Fbar[v] = magnitude * dt * (qbar[V * j + v] - qbar[V * o + v]);
        const double inv = 1.0 / magnitude;
#pragma unroll
        for (int k = 0; k < D; ++k) n[k] = a[k] * inv;
        if constexpr (Riemann == 1)
            hll_flux_adjoint<D>(L, R, n, gas, Fbar, Lbar, Rbar);
        else
            hllc_flux_adjoint<D>(L, R, n, gas, Fbar, Lbar, Rbar);
    }
    double* row = face_bar + 2 * V * static_cast<int64_t>(f);
#pragma unroll
    for (int v = 0; v < V; ++v) {
        row[v] = Lbar[v];
        row[V + v] = Rbar[v];
    }
}

// AdjointCell (finite_volume.hpp:2107-2169).
template <int D>
__global__ void __launch_bounds__(128, LUNA_ADJ_MIN_BLOCKS) k_cell_adjoint(MeshDev<D> m, const double* __restrict__ prims, const double* __restrict__ grad,
                                                      const double* __restrict__ face_bar, const double* __restrict__ fit,
                                                      const int32_t* __restrict__ flags, double dt, GasDev gas, double* __restrict__ wbar,
                                                      double* __restrict__ bbar, double* __restrict__ boundbar, int32_t* __restrict__ bound_face) {
    constexpr int V = D + 2, U = D + 1, GS = grad_stride<D>();
    using FL = FitLayout<D>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double Wi[V], gi[V * D], Wi_bar[V], gi_bar[V * D];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        Wi[v] = prims[PS * i + v];
        Wi_bar[v] = 0;
    }
#pragma unroll
    for (int c = 0; c < V * D; ++c) {
        gi[c] = grad[static_cast<int64_t>(GS) * i + c];
        gi_bar[c] = 0;
    }
    for (int k = m.start[i]; k < m.start[i + 1]; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e);
        double a[D];
#pragma unroll
        for (int q = 0; q < D; ++q) a[q] = m.area[D * f + q];
        if (dot<D>(a, a) == 0) continue;
        const double* mine = face_bar + 2 * V * static_cast<int64_t>(f) + (e >= 0 ? 0 : V);
        double r[D], Wf[V], mb[V];
        m.face_offset(f, i, r);
#pragma unroll
        for (int v = 0; v < V; ++v) mb[v] = mine[v];
        if (side_value<D>(Wi, gi, r, dt, gas.gamma, Wf)) {
#pragma unroll
            for (int v = 0; v < V; ++v) Wi_bar[v] += mb[v];
        } else {
#pragma unroll
            for (int v = 0; v < V; ++v)
#pragma unroll
                for (int q = 0; q < D; ++q) gi_bar[D * v + q] = gi_bar[D * v + q] + r[q] * mb[v];
            half_step_adjoint<D>(Wi, gi, dt, gas.gamma, mb, Wi_bar, gi_bar);
        }
    }
    const double* fr = fit + static_cast<int64_t>(FL::width) * i;
    double Lc[U][U];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s < U; ++s) Lc[p][s] = fr[FL::factor + p * U + s];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int flag = flags[2 * V * i + v];
        double g0[D], g0bar[D], xbar[U], z[U], bs[U];
#pragma unroll
        for (int a = 0; a < D; ++a) {
            g0[a] = fr[FL::g0 + D * v + a];
            g0bar[a] = gi_bar[D * v + a];
        }
        double self = 0, bound = 0;
        int face = -1;
        if ((flag & 1) && (flag & 4)) {
#pragma unroll
            for (int a = 0; a < D; ++a) g0bar[a] = 0;
        } else if (flag & 1) {
            double o[D];
#pragma unroll
            for (int a = 0; a < D; ++a) o[a] = fr[FL::offset + D * v + a];
            const double den = dot<D>(g0, o);
            const double s = (fr[FL::bound + v] - Wi[v]) / den, t = dot<D>(gi_bar + D * v, g0) / den;
#pragma unroll
            for (int a = 0; a < D; ++a) g0bar[a] = gi_bar[D * v + a] * s - o[a] * (s * t);
            bound = t;
            face = flags[2 * V * i + V + v];
            self -= t;
        }
        xbar[0] = 0;
#pragma unroll
        for (int a = 0; a < D; ++a) xbar[1 + a] = g0bar[a];
        // solve_factored (finite_volume.hpp:688-702): b bar = M^-1 x bar
#pragma unroll
        for (int p = 0; p < U; ++p) {
            double sum = xbar[p];
#pragma unroll
            for (int q = 0; q < p; ++q) sum -= Lc[p][q] * z[q];
            z[p] = sum / Lc[p][p];
        }
#pragma unroll
        for (int p = U - 1; p >= 0; --p) {
            double sum = z[p];
#pragma unroll
            for (int q = p + 1; q < U; ++q) sum -= Lc[q][p] * bs[q];
            bs[p] = sum / Lc[p][p];
        }
#pragma unroll
        for (int p = 0; p < U; ++p) self -= fr[FL::row0 + p] * bs[p];
        wbar[V * i + v] = Wi_bar[v] + self;
#pragma unroll
        for (int p = 0; p < U; ++p) bbar[static_cast<int64_t>(U * V) * i + U * v + p] = bs[p];
        boundbar[V * i + v] = bound;
        bound_face[V * i + v] = face;
    }
}

// AdjointGather (finite_volume.hpp:2171-2195): Qbar_j += primitive_adjoint(W_j bar) / V_j.
template <int D>
__global__ void __launch_bounds__(128) k_gather_adjoint(MeshDev<D> m, const double* __restrict__ q, const double* __restrict__ wbar,
                                                        const double* __restrict__ bbar, const double* __restrict__ boundbar,
                                                        const int32_t* __restrict__ bound_face, GasDev gas, double* __restrict__ qbar) {
    constexpr int V = D + 2, U = D + 1;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m.n) return;
    double W_bar[V];
#pragma unroll
    for (int v = 0; v < V; ++v) W_bar[v] = wbar[V * j + v];
    double cj[D];
#pragma unroll
    for (int a = 0; a < D; ++a) cj[a] = m.cen[D * j + a];
    constexpr int B = LUNA_ADJ_GATHER_BATCH;
    const int first = m.start[j], end = m.start[j + 1];
    for (int k0 = first; k0 < end; k0 += B) {
        int f[B], i[B];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int32_t e = k0 + b < end ? m.list[k0 + b] : 0;
            f[b] = list_face(e);
            i[b] = k0 + b < end ? (e >= 0 ? m.neighbour[f[b]] : m.owner[f[b]]) : j;
        }
#pragma unroll
        for (int b = 0; b < B; ++b) {
            if (k0 + b >= end) break;
            double sep[D], between[D];
            m.separation(i[b], j, sep);
#pragma unroll
            for (int a = 0; a < D; ++a) between[a] = sep[a] + cj[a] - m.cen[D * i[b] + a];
            const double w = m.mag[f[b]];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const double* bb = bbar + static_cast<int64_t>(U * V) * i[b] + U * v;
                double sum = bb[0];
#pragma unroll
                for (int p = 1; p < U; ++p) sum += between[p - 1] * bb[p];
                W_bar[v] += w * sum + (bound_face[V * i[b] + v] == f[b] ? boundbar[V * i[b] + v] : 0.0);
            }
        }
    }
    const double inv = 1.0 / m.vol[j];
    double Uj[V], U_bar[V];
#pragma unroll
    for (int v = 0; v < V; ++v) Uj[v] = q[V * j + v] * inv;
    primitive_adjoint<D>(Uj, W_bar, gas, U_bar);
#pragma unroll
    for (int v = 0; v < V; ++v) qbar[V * j + v] += U_bar[v] * inv;
}

}  // namespace luna
