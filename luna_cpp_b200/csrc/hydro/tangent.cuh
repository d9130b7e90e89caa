// The tangent of one static step (luna-cpp's step_tangent, src/hydro/finite_volume.hpp:2023-2062): dQ^n+1 = J dQ^n at
// fixed dt, for the FP64 policy, order 1, the per-face loop; the step itself runs after it with the production kernels,
// so Q^n+1 is step()'s. The linearisation point is the adjoint's (k_sweep_fit: the reference's fit, its clip pattern and
// gradients), so the tangent and the adjoint are transposes of one map (the dot test). Passes:
//   k_tangent_prims   dW = J dU of primitive() per cell (primitive_tangent, euler.hpp:131-142);
//   k_tangent_sweep   dg per cell: the fit's tangent right-hand side over the list, solved with the stored Cholesky
//                     factor, then the limited gradient's tangent at its clip pattern (limited_gradient_tangent,
//                     finite_volume.hpp:811-833: a clipped variable is g0 (bound - W_i) / (g0 . o_last));
//   k_tangent_fluxes  per face: both face states' tangents (side_tangent: the half step and g . r, a fallen-back side
//                     carries dW) and the Riemann solve's, by forward-mode dual numbers through the same HLLC/HLL code
//                     as the step (each branch the forward took), times |A| (TangentFluxes, :1971-2004);
//   k_tangent_update  dQ_i -= dt sum_k sign_k dF_k in list order (TangentUpdate, :2006-2022).
#pragma once

#include "adjoint.cuh"

namespace luna {
namespace fwd {

// A forward-mode dual number: a value and its derivative along one direction. The free functions below are found by
// argument-dependent lookup from the templated device physics (T = Dual), so the tangent differentiates the very
// expressions the step evaluates; comparisons look at values only (the forward's branch).
struct Dual {
    double v, d;
    __device__ __forceinline__ Dual() : v(0), d(0) {}
    __device__ __forceinline__ Dual(double x) : v(x), d(0) {}  // NOLINT: constants enter the physics as T(c)
    __device__ __forceinline__ Dual(double x, double dx) : v(x), d(dx) {}
    __device__ __forceinline__ Dual& operator+=(const Dual& o) {
        v += o.v;
        d += o.d;
        return *this;
    }
    __device__ __forceinline__ Dual& operator-=(const Dual& o) {
        v -= o.v;
        d -= o.d;
        return *this;
    }
    __device__ __forceinline__ Dual& operator*=(const Dual& o) {
        d = d * o.v + v * o.d;
        v *= o.v;
        return *this;
    }
};
__device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(const Dual& a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
__device__ __forceinline__ Dual sqrt(const Dual& a) {
    const double r = ::sqrt(a.v);
    return {r, r > 0 ? a.d / (2 * r) : 0.0};
}
__device__ __forceinline__ Dual fabs(const Dual& a) { return a.v < 0 ? -a : a; }
__device__ __forceinline__ Dual fmin(const Dual& a, const Dual& b) { return b.v < a.v ? b : a; }
__device__ __forceinline__ Dual fmax(const Dual& a, const Dual& b) { return b.v > a.v ? b : a; }

// HLL (euler.hpp:444-461) for any arithmetic type T (the step's hll_flux is double only).
template <int D, class T>
__device__ __forceinline__ void hll_flux_t(const T* L, const T* R, const T* n, const T* w, T gamma, T inverse_gm1, T* F,
                                           bool moving_frame = false) {
    constexpr int P = D + 1;
    Side<D, T> l, r;
    T rel[D];
#pragma unroll
    for (int k = 0; k < D; ++k) rel[k] = L[1 + k] - w[k];
    side_with<D, T>(L, n, w, inverse_gm1, dot<D>(rel, n), l);
    {
        const T c2 = gamma * L[P] / L[0];
        l.c = c2 > T(0) ? sqrt(c2) : T(0);
    }
#pragma unroll
    for (int k = 0; k < D; ++k) rel[k] = R[1 + k] - w[k];
    side_with<D, T>(R, n, w, inverse_gm1, dot<D>(rel, n), r);
    {
        const T c2 = gamma * R[P] / R[0];
        r.c = c2 > T(0) ? sqrt(c2) : T(0);
    }
    const T SL = fmin(l.vn - l.c, r.vn - r.c);
    const T SR = fmax(l.vn + l.c, r.vn + r.c);
    if (SL >= T(0)) {
#pragma unroll
        for (int v = 0; v < D + 2; ++v) F[v] = l.F[v];
    } else if (SR <= T(0)) {
#pragma unroll
        for (int v = 0; v < D + 2; ++v) F[v] = r.F[v];
    } else {
        const T inv_dS = T(1) / (SR - SL);
#pragma unroll
        for (int v = 0; v < D + 2; ++v) F[v] = (SR * l.F[v] - SL * r.F[v] + SL * SR * (r.U[v] - l.U[v])) * inv_dS;
    }
    if (moving_frame) to_lab<D, T>(F, w);
}

}  // namespace fwd

// primitive_tangent (euler.hpp:131-142): dW = J dU; a floored density or energy has derivative 0 in what it replaced.
template <int D>
__device__ __forceinline__ void primitive_tangent(const double* U, const double* dU, const GasDev& gas, double* dW) {
    constexpr int P = D + 1;
    const double rho = fmax(U[0], gas.smallr), inv_rho = 1.0 / rho;
    double v[D];
#pragma unroll
    for (int k = 0; k < D; ++k) v[k] = U[1 + k] * inv_rho;
    const double smalle = gas.smallc * gas.smallc / gas.gamma / (gas.gamma - 1.0);
    const int floors = (U[0] >= gas.smallr ? 0 : 1) | (U[P] - 0.5 * rho * dot<D>(v, v) >= smalle * rho ? 0 : 2);
    const double drho = floors & 1 ? 0.0 : dU[0];
    double dv[D];
#pragma unroll
    for (int k = 0; k < D; ++k) dv[k] = (dU[1 + k] - v[k] * drho) * inv_rho;
    const double dkinetic = 0.5 * drho * dot<D>(v, v) + rho * dot<D>(v, dv);
    const double de = floors & 2 ? smalle * drho : dU[P] - dkinetic;
    dW[0] = drho;
#pragma unroll
    for (int k = 0; k < D; ++k) dW[1 + k] = dv[k];
    dW[P] = (gas.gamma - 1.0) * de;
}

template <int D>
__global__ void __launch_bounds__(256) k_tangent_prims(int n, const double* __restrict__ q, const double* __restrict__ dq,
                                                       const double* __restrict__ vol, GasDev gas, double* __restrict__ dprims) {
    constexpr int V = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double inv = 1.0 / vol[i];
    double U[V], dU[V], dW[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        U[v] = q[V * static_cast<int64_t>(i) + v] * inv;
        dU[v] = dq[V * static_cast<int64_t>(i) + v] * inv;
    }
    primitive_tangent<D>(U, dU, gas, dW);
#pragma unroll
    for (int v = 0; v < V; ++v) dprims[V * static_cast<int64_t>(i) + v] = dW[v];
}

// The limited gradient's tangent per cell at the stored fit and clip pattern (k_sweep_fit's rows and flags).
template <int D>
__global__ void __launch_bounds__(128) k_tangent_sweep(MeshDev<D> m, const double* __restrict__ prims, const double* __restrict__ dprims,
                                                       const double* __restrict__ fit, const int32_t* __restrict__ flags,
                                                       double* __restrict__ dgrad) {
    constexpr int V = D + 2, U = D + 1;
    using FL = FitLayout<D>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double dWi[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dWi[v] = dprims[V * static_cast<int64_t>(i) + v];
    double centroid[D];
#pragma unroll
    for (int a = 0; a < D; ++a) centroid[a] = m.cen[D * i + a];
    double db[V][U];
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
        for (int p = 0; p < U; ++p) db[v][p] = 0;
    for (int k = m.start[i]; k < m.start[i + 1]; ++k) {  // the fit's tangent right-hand side (limited_core, :733-737)
        const int32_t e = m.list[k];
        const int f = list_face(e);
        const int j = e >= 0 ? m.neighbour[f] : m.owner[f];
        double d[D], X[U];
        m.separation(i, j, d);
        X[0] = 1;
#pragma unroll
        for (int p = 1; p < U; ++p) X[p] = d[p - 1] + m.cen[D * j + p - 1] - centroid[p - 1];
        const double w = m.mag[f];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const double ddW = w * (dprims[V * static_cast<int64_t>(j) + v] - dWi[v]);
#pragma unroll
            for (int p = 0; p < U; ++p) db[v][p] += X[p] * ddW;
        }
    }
    const double* fr = fit + static_cast<int64_t>(FL::width) * i;
    double Lc[U][U];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s < U; ++s) Lc[p][s] = fr[FL::factor + p * U + s];
    double* out = dgrad + static_cast<int64_t>(V * D) * i;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        double z[U], x[U];  // solve_factored (:688-699)
#pragma unroll
        for (int p = 0; p < U; ++p) {
            double sum = db[v][p];
#pragma unroll
            for (int q = 0; q < p; ++q) sum -= Lc[p][q] * z[q];
            z[p] = sum / Lc[p][p];
        }
#pragma unroll
        for (int p = U - 1; p >= 0; --p) {
            double sum = z[p];
#pragma unroll
            for (int q = p + 1; q < U; ++q) sum -= Lc[q][p] * x[q];
            x[p] = sum / Lc[p][p];
        }
        double dg0[D], g0[D], o[D];
#pragma unroll
        for (int a = 0; a < D; ++a) {
            dg0[a] = x[1 + a];
            g0[a] = fr[FL::g0 + D * v + a];
            o[a] = fr[FL::offset + D * v + a];
        }
        const int flag = flags[2 * V * static_cast<int64_t>(i) + v];
        if (!(flag & 1)) {
#pragma unroll
            for (int a = 0; a < D; ++a) out[D * v + a] = dg0[a];
        } else if (flag & 4) {
#pragma unroll
            for (int a = 0; a < D; ++a) out[D * v + a] = 0.0;
        } else {
            // the bound came through face bf from its other cell
            const int bf = flags[2 * V * static_cast<int64_t>(i) + V + v];
            const int holder = m.owner[bf] == i ? m.neighbour[bf] : m.owner[bf];
            const double dbound = dprims[V * static_cast<int64_t>(holder) + v];
            const double den = dot<D>(g0, o);
            const double s = (fr[FL::bound + v] - prims[PS * static_cast<int64_t>(i) + v]) / den;
            const double ds = (dbound - dWi[v] - s * dot<D>(dg0, o)) / den;
#pragma unroll
            for (int a = 0; a < D; ++a) out[D * v + a] = dg0[a] * s + g0[a] * ds;
        }
    }
}

// side_tangent (finite_volume.hpp:1346-1366): the face state's tangent, by duals through the half step; a side that
// fell back (rho or P of the face state not positive) carries dW.
template <int D>
__device__ __forceinline__ void side_tangent(const double* W, const double* dW, const double* g, const double* dg, const double* r, double dt,
                                             double gamma, bool fallback, double* dWf) {
    constexpr int V = D + 2;
    if (fallback) {
#pragma unroll
        for (int v = 0; v < V; ++v) dWf[v] = dW[v];
        return;
    }
    fwd::Dual Wd[V], gd[V * D], A[V];
#pragma unroll
    for (int v = 0; v < V; ++v) Wd[v] = fwd::Dual(W[v], dW[v]);
#pragma unroll
    for (int c = 0; c < V * D; ++c) gd[c] = fwd::Dual(g[c], dg[c]);
    half_step_rate<D, fwd::Dual>(Wd, gd, fwd::Dual(gamma), A);
#pragma unroll
    for (int v = 0; v < V; ++v) {
        fwd::Dual f = Wd[v] - fwd::Dual(0.5 * dt) * A[v];
#pragma unroll
        for (int a = 0; a < D; ++a) f += gd[D * v + a] * fwd::Dual(r[a]);
        dWf[v] = f.d;
    }
}

template <int D, int Riemann>
__global__ void __launch_bounds__(128) k_tangent_fluxes(MeshDev<D> m, const double* __restrict__ prims, const double* __restrict__ grad,
                                                        const double* __restrict__ dprims, const double* __restrict__ dgrad, double dt, GasDev gas,
                                                        double* __restrict__ dflux) {
    constexpr int V = D + 2, GS = grad_stride<D>();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.f) return;
    const double magnitude = m.mag[f];
    double dF[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dF[v] = 0;
    if (magnitude != 0) {
        const int o = m.owner[f], j = m.neighbour[f];
        double ro[D], rj[D];
        m.face_offset(f, o, ro);
        m.face_offset(f, j, rj);
        double L[V], R[V], dL[V], dR[V];
        const double *Wo = prims + PS * static_cast<int64_t>(o), *Wj = prims + PS * static_cast<int64_t>(j);
        const double *go = grad + static_cast<int64_t>(GS) * o, *gj = grad + static_cast<int64_t>(GS) * j;
        const bool fo = side_value<D>(Wo, go, ro, dt, gas.gamma, L), fj = side_value<D>(Wj, gj, rj, dt, gas.gamma, R);
        side_tangent<D>(Wo, dprims + V * static_cast<int64_t>(o), go, dgrad + static_cast<int64_t>(V * D) * o, ro, dt, gas.gamma, fo, dL);
        side_tangent<D>(Wj, dprims + V * static_cast<int64_t>(j), gj, dgrad + static_cast<int64_t>(V * D) * j, rj, dt, gas.gamma, fj, dR);
        fwd::Dual Ld[V], Rd[V], n[D], w[D], F[V];
        const double inv = 1.0 / magnitude;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            Ld[v] = fwd::Dual(L[v], dL[v]);
            Rd[v] = fwd::Dual(R[v], dR[v]);
        }
#pragma unroll
        for (int a = 0; a < D; ++a) {
            n[a] = fwd::Dual(m.area[D * static_cast<int64_t>(f) + a] * inv);
            w[a] = fwd::Dual(0.0);
        }
        if constexpr (Riemann == 1)
            fwd::hll_flux_t<D, fwd::Dual>(Ld, Rd, n, w, fwd::Dual(gas.gamma), fwd::Dual(gas.inverse_gm1), F);
        else
            hllc_flux<D, fwd::Dual>(Ld, Rd, n, w, fwd::Dual(gas.gamma), fwd::Dual(gas.inverse_gm1), F, false);
#pragma unroll
        for (int v = 0; v < V; ++v) dF[v] = F[v].d * magnitude;
    }
#pragma unroll
    for (int v = 0; v < V; ++v) dflux[V * static_cast<int64_t>(f) + v] = dF[v];
}

template <int D>
__global__ void __launch_bounds__(256) k_tangent_update(MeshDev<D> m, double* __restrict__ dq, const double* __restrict__ dflux, double dt) {
    constexpr int V = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double dsum[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dsum[v] = 0;
    for (int k = m.start[i]; k < m.start[i + 1]; ++k) {
        const int32_t e = m.list[k];
        const double sign = e >= 0 ? 1.0 : -1.0;
        const double* r = dflux + V * static_cast<int64_t>(list_face(e));
#pragma unroll
        for (int v = 0; v < V; ++v) dsum[v] += sign * r[v];
    }
#pragma unroll
    for (int v = 0; v < V; ++v) dq[V * static_cast<int64_t>(i) + v] = dq[V * static_cast<int64_t>(i) + v] - dt * dsum[v];
}

}  // namespace luna
