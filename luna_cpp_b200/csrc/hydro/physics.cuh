// Device physics of the hydro step: the ideal-gas conversions, the MUSCL-Hancock half step, the face-frame boost and the
// HLLC/HLL Riemann solvers of luna-cpp's src/hydro/euler.hpp, written for registers (fixed-size arrays, D a template
// parameter, T = double or float). Operation order follows the reference's, so that the results differ from the CPU
// oracle only by the compiler's multiply-add contraction.
#pragma once

#include <cuda_runtime.h>

namespace luna {

struct GasDev {
    double gamma, smallr, smallc, inverse_gm1;
    float inverse_gm1_float;
};

template <int D, class T>
__device__ __forceinline__ T dot(const T* a, const T* b) {
    T s = a[0] * b[0];
#pragma unroll
    for (int k = 1; k < D; ++k) s = s + a[k] * b[k];
    return s;
}

// primitive(): U -> W with LUNA's RAMSES floors (euler.hpp:104-113).
template <int D>
__device__ __forceinline__ void primitive(const double* U, const GasDev& gas, double* W) {
    const double rho = fmax(U[0], gas.smallr);
    const double inv_rho = 1.0 / rho;
    double v[D];
#pragma unroll
    for (int k = 0; k < D; ++k) v[k] = U[1 + k] * inv_rho;
    const double smalle = gas.smallc * gas.smallc / gas.gamma / (gas.gamma - 1.0);
    const double kinetic = 0.5 * rho * dot<D>(v, v);
    const double e = fmax(U[D + 1] - kinetic, smalle * rho);
    W[0] = rho;
#pragma unroll
    for (int k = 0; k < D; ++k) W[1 + k] = v[k];
    W[D + 1] = (gas.gamma - 1.0) * e;
}

// The radius of a sphere (3D) or circle (2D) of volume v (FiniteVolume::radius, finite_volume.hpp:241-246).
template <int D>
__device__ __forceinline__ double radius(double v) {
    if constexpr (D == 3)
        return cbrt(v * (3.0 / (4.0 * 3.14159265358979323846)));
    else
        return sqrt(v * (1.0 / 3.14159265358979323846));
}
// AREPO's face angle size (FiniteVolume::face_angle, finite_volume.hpp:248-253).
template <int D>
__device__ __forceinline__ double face_angle(double area) {
    if constexpr (D == 3)
        return sqrt(area / 3.14159265358979323846);
    else
        return 0.5 * area;
}

// half_step_rate(): sum_d A_d(W) dW/dx_d (euler.hpp:186-204); g[v * D + d] = dW_v/dx_d.
template <int D, class T>
__device__ __forceinline__ void half_step_rate(const T* W, const T* g, T gamma, T* A) {
    constexpr int P = D + 1;
    const T rho = W[0], inv_rho = T(1) / W[0], rho_c2 = gamma * W[P];
#pragma unroll
    for (int v = 0; v < D + 2; ++v) A[v] = T(0);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const T vn = W[1 + d];
        A[0] += vn * g[0 * D + d] + rho * g[(1 + d) * D + d];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            T row = vn * g[(1 + k) * D + d];
            if (k == d) row = row + inv_rho * g[P * D + d];
            A[1 + k] += row;
        }
        A[P] += rho_c2 * g[(1 + d) * D + d] + vn * g[P * D + d];
    }
}

// One side of a face in the face frame (detail::Side / side_with, euler.hpp:313-336).
template <int D, class T>
struct Side {
    T v[D], vn, c, E, F[D + 2], U[D + 2];
};

template <int D, class T>
__device__ __forceinline__ void side_with(const T* W, const T* n, const T* w, T inverse_gm1, T vn, Side<D, T>& s) {
    constexpr int P = D + 1;
#pragma unroll
    for (int k = 0; k < D; ++k) s.v[k] = W[1 + k] - w[k];
    s.vn = vn;
    s.c = T(0);
    s.E = W[P] * inverse_gm1 + W[0] * (T(0.5) * dot<D>(s.v, s.v));
    const T m = W[0] * s.vn;
    s.F[0] = m;
#pragma unroll
    for (int k = 0; k < D; ++k) s.F[1 + k] = m * s.v[k] + W[P] * n[k];
    s.F[P] = (s.E + W[P]) * s.vn;
    s.U[0] = W[0];
#pragma unroll
    for (int k = 0; k < D; ++k) s.U[1 + k] = W[0] * s.v[k];
    s.U[P] = s.E;
}

// to_lab(): the face-frame flux back to the lab frame (euler.hpp:350-356).
template <int D, class T>
__device__ __forceinline__ void to_lab(T* F, const T* w) {
    constexpr int P = D + 1;
    T e = w[0] * F[1];
#pragma unroll
    for (int k = 1; k < D; ++k) e = e + w[k] * F[1 + k];
    F[P] += e + T(0.5) * dot<D>(w, w) * F[0];
#pragma unroll
    for (int k = 0; k < D; ++k) F[1 + k] += w[k] * F[0];
}

template <class T>
__device__ __forceinline__ T nonzero(T d) {
    const T eps = T(1e-20);
    return fabs(d) < eps ? (d < T(0) ? -eps : eps) : d;
}

// HLLC with LUNA's guards (euler.hpp:609-642): c^2 < 0 on a side takes F_R, divisors kept off zero by 1e-20, LUNA's
// branch order F_L, F*_L, F*_R, F_R; the flux is built for the upwind side only. Frame: velocities relative to w.
template <int D, class T>
__device__ __forceinline__ void hllc_flux(const T* L, const T* R, const T* n, const T* w, T gamma, T inverse_gm1, T* F,
                                          bool moving_frame) {
    constexpr int P = D + 1;
    T rl[D], rr[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        rl[k] = L[1 + k] - w[k];
        rr[k] = R[1 + k] - w[k];
    }
    const T vnL = dot<D>(rl, n), vnR = dot<D>(rr, n);
    const T inv_rhoL = T(1) / L[0], inv_rhoR = T(1) / R[0];
    const T c2L = gamma * L[P] * inv_rhoL, c2R = gamma * R[P] * inv_rhoR;
    const bool ok = c2L >= T(0) && c2R >= T(0);
    const T cL = c2L > T(0) ? sqrt(c2L) : T(0), cR = c2R > T(0) ? sqrt(c2R) : T(0);
    const T SL = fmin(vnL - cL, vnR - cR);
    const T SR = fmax(vnL + cL, vnR + cR);
    const T denomL = L[0] * (SL - vnL), denomR = R[0] * (SR - vnR);
    const T SM = (R[P] - L[P] + denomL * vnL - denomR * vnR) / nonzero(denomL - denomR);
    const bool left = ok && (SL >= T(0) || SM >= T(0));
    const bool star = ok && SL < T(0) && (SM >= T(0) || SR > T(0));
    T W[D + 2];
#pragma unroll
    for (int v = 0; v < D + 2; ++v) W[v] = left ? L[v] : R[v];
    Side<D, T> s;
    side_with<D, T>(W, n, w, inverse_gm1, left ? vnL : vnR, s);
    if (!star) {
#pragma unroll
        for (int v = 0; v < D + 2; ++v) F[v] = s.F[v];
    } else {
        const T S = left ? SL : SR, denom = left ? denomL : denomR;
        const T rho_star = denom / nonzero(S - SM);
        const T E_star = s.E * (left ? inv_rhoL : inv_rhoR) + (SM - s.vn) * (SM + W[P] * (T(1) / nonzero(denom)));
        T U_star[D + 2];
        U_star[0] = rho_star;
#pragma unroll
        for (int k = 0; k < D; ++k) U_star[1 + k] = rho_star * (s.v[k] + n[k] * (SM - s.vn));
        U_star[P] = rho_star * E_star;
#pragma unroll
        for (int v = 0; v < D + 2; ++v) F[v] = s.F[v] + S * (U_star[v] - s.U[v]);
    }
    if (moving_frame) to_lab<D, T>(F, w);
}

// HLL with Davis wave speeds (euler.hpp:444-461).
template <int D>
__device__ __forceinline__ void hll_flux(const double* L, const double* R, const double* n, const double* w, const GasDev& gas,
                                         double* F, bool moving_frame) {
    constexpr int P = D + 1;
    Side<D, double> l, r;
    double rel[D];
#pragma unroll
    for (int k = 0; k < D; ++k) rel[k] = L[1 + k] - w[k];
    side_with<D, double>(L, n, w, gas.inverse_gm1, dot<D>(rel, n), l);
    {
        const double c2 = gas.gamma * L[P] / L[0];
        l.c = c2 > 0 ? sqrt(c2) : 0.0;
    }
#pragma unroll
    for (int k = 0; k < D; ++k) rel[k] = R[1 + k] - w[k];
    side_with<D, double>(R, n, w, gas.inverse_gm1, dot<D>(rel, n), r);
    {
        const double c2 = gas.gamma * R[P] / R[0];
        r.c = c2 > 0 ? sqrt(c2) : 0.0;
    }
    const double SL = fmin(l.vn - l.c, r.vn - r.c);
    const double SR = fmax(l.vn + l.c, r.vn + r.c);
    if (SL >= 0) {
#pragma unroll
        for (int v = 0; v < D + 2; ++v) F[v] = l.F[v];
    } else if (SR <= 0) {
#pragma unroll
        for (int v = 0; v < D + 2; ++v) F[v] = r.F[v];
    } else {
        const double inv_dS = 1.0 / (SR - SL);
#pragma unroll
        for (int v = 0; v < D + 2; ++v) F[v] = (SR * l.F[v] - SL * r.F[v] + SL * SR * (r.U[v] - l.U[v])) * inv_dS;
    }
    if (moving_frame) to_lab<D, double>(F, w);
}

}  // namespace luna
