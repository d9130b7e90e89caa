// The derivatives of the order-0 moving step at fixed topology (luna-cpp's step_moving_tangent / step_moving_adjoint,
// src/hydro/finite_volume.hpp:2431-2604): the state is (Q, x); the fluxes read W = primitive(Q / V), the face areas A and
// face centroids x_f, the separations d = x_j - x_o and the face velocities from the point velocities w; w reads W, the
// sound speed, the cell centroid c and, through AREPO's roundness term, the cell's largest face angle; Q advances by
// dt times the fluxes and x by dt w. The geometry's own derivative in x (V, c, A, x_f) is the caller's (the mesh
// library's GeometryDerivative, mesh_derivative.hpp:10-29): the tangent takes its dV, dc, dA, dx_f, the adjoint hands back
// the bars of V, c, A, x_f for it. FP64, the per-face loop, HLLC or HLL. No atomics: every bar is gathered.
//
// Every local derivative is taken by forward-mode dual numbers (fwd::Dual) through the step's own expressions, each
// branch the forward took: the tangent in one pass along the caller's direction, the adjoint from the local Jacobian's
// columns (one pass per input) times the output's bar, so the two are transposes of one linearisation.
//   tangent: k_mv_prims (W, c_s and their tangents) -> k_mv_velocity (w, dw) -> k_mv_faces_tangent (dG per face)
//            -> k_mv_update_tangent (dQ -= dt sum sign dG, dx += dt dw);
//   adjoint: k_mv_prims, k_mv_velocity (values) -> k_mv_faces_adjoint (per face: the flux's and the face velocity's
//            bars) -> k_mv_cells_adjoint (per cell: W's and w's bars gathered, the point velocity's and the primitives'
//            adjoints into Q's bar, V's and c's bars) -> k_mv_area_adjoint (A's bar) -> k_mv_separation_adjoint (x's bar).
#pragma once

#include "tangent.cuh"

namespace luna {
namespace mvd {

using fwd::Dual;

// primitive() (euler.hpp:104-113) on any arithmetic type, floors included.
template <int D, class T>
__device__ __forceinline__ void primitive_t(const T* U, const GasDev& gas, T* W) {
    const T rho = fmax(U[0], T(gas.smallr));
    const T inv_rho = T(1.0) / rho;
    T v[D];
#pragma unroll
    for (int k = 0; k < D; ++k) v[k] = U[1 + k] * inv_rho;
    const double smalle = gas.smallc * gas.smallc / gas.gamma / (gas.gamma - 1.0);
    const T kinetic = T(0.5) * rho * dot<D>(v, v);
    const T e = fmax(U[D + 1] - kinetic, T(smalle) * rho);
    W[0] = rho;
#pragma unroll
    for (int k = 0; k < D; ++k) W[1 + k] = v[k];
    W[D + 1] = T(gas.gamma - 1.0) * e;
}

// sound_speed(): sqrt(gamma P / rho).
template <class T>
__device__ __forceinline__ T sound_t(const T* W, int P, double gamma) {
    const T c2 = T(gamma) * W[P] / W[0];
    return c2 > T(0) ? sqrt(c2) : T(0);
}

// The largest face angle of cell i (Regularised, finite_volume.hpp:2246-2262): the face, the cell across it, the angle.
template <int D>
struct AngleFace {
    int f = -1, other = -1;
    double amax = 0;
};
template <int D>
__device__ __forceinline__ AngleFace<D> angle_face(const MeshDev<D>& m, int i) {
    AngleFace<D> r;
    for (int k = m.start[i]; k < m.start[i + 1]; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e), j = e >= 0 ? m.neighbour[f] : m.owner[f];
        double d[D], a[D];
        m.separation(i, j, d);
#pragma unroll
        for (int q = 0; q < D; ++q) a[q] = m.area[D * f + q];
        const double angle = face_angle<D>(sqrt(dot<D>(a, a))) / (0.5 * sqrt(dot<D>(d, d)));
        if (angle > r.amax) {
            r.amax = angle;
            r.f = f;
            r.other = j;
        }
    }
    return r;
}

// face_angle() on any arithmetic type.
template <int D, class T>
__device__ __forceinline__ T face_angle_t(T area) {
    if constexpr (D == 3)
        return sqrt(area / T(3.14159265358979323846));
    else
        return T(0.5) * area;
}

// Sweep<true>'s point velocity (finite_volume.hpp:526-537): w = v + c (fraction c_s / |c|), fraction from the largest
// face angle (0 below 0.75 of 2.25, 0.5 above 2.25, linear between), on any arithmetic type: W's velocity, c_s, c, and
// the angle face's area vector A and separation d (the angle itself recomputed from them, so that it carries their
// derivative).
template <int D, class T>
__device__ __forceinline__ void point_velocity_t(const AngleFace<D>& af, const T* W, T cs, const T* c, const T* A, const T* d, T* w) {
    constexpr double factor = 2.25, speed = 0.5;
#pragma unroll
    for (int a = 0; a < D; ++a) w[a] = W[1 + a];
    if (!(af.amax > 0.75 * factor)) return;
    T fraction;
    if (af.amax > factor) {
        fraction = T(speed);
    } else {
        const T angle = face_angle_t<D, T>(sqrt(dot<D>(A, A))) / (T(0.5) * sqrt(dot<D>(d, d)));
        fraction = T(speed) * (angle - T(0.75 * factor)) / T(0.25 * factor);
    }
    const T cd = sqrt(dot<D>(c, c));
    if (!(cd > T(0))) return;
    const T s = fraction * cs / cd;
#pragma unroll
    for (int a = 0; a < D; ++a) w[a] = w[a] + c[a] * s;
}

// FaceFlux::face_velocity (finite_volume.hpp:1380-1397) on any arithmetic type: d owner -> neighbour, x_f relative to the
// owner, the two point velocities.
template <int D, class T>
__device__ __forceinline__ void face_velocity_t(const T* d, const T* xf, const T* wL, const T* wR, T* out) {
    const T dist = sqrt(dot<D>(d, d));
    const T inv_dist = T(1.0) / dist;
    T c[D], dw[D];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        c[a] = xf[a] - d[a] * T(0.5);
        dw[a] = wL[a] - wR[a];
    }
    T facv = dot<D>(c, dw) * inv_dist;
    const T limit = T(0.9) * dist, c2 = dot<D>(c, c);
    if (c2 > limit * limit) facv = facv * (limit / sqrt(c2));
    const T s = facv * inv_dist;
#pragma unroll
    for (int a = 0; a < D; ++a) out[a] = (wL[a] + wR[a]) * T(0.5) + d[a] * s;
}

// The moving face's flux times |A| (FaceFlux<0, true>::operator(), :1415-1434) on any arithmetic type.
template <int D, int Riemann, class T>
__device__ __forceinline__ void face_flux_t(const T* L, const T* R, const T* A, const T* wf, const GasDev& gas, T* G) {
    constexpr int V = D + 2;
    const T mag = sqrt(dot<D>(A, A));
    T n[D];
    const T inv = T(1.0) / mag;
#pragma unroll
    for (int a = 0; a < D; ++a) n[a] = A[a] * inv;
    if constexpr (Riemann == 1)
        fwd::hll_flux_t<D, T>(L, R, n, wf, T(gas.gamma), T(gas.inverse_gm1), G, true);
    else
        hllc_flux<D, T>(L, R, n, wf, T(gas.gamma), T(gas.inverse_gm1), G, true);
#pragma unroll
    for (int v = 0; v < V; ++v) G[v] = G[v] * mag;
}

template <int D>
__device__ __forceinline__ void load_vec(const double* p, int64_t i, double* out) {
#pragma unroll
    for (int a = 0; a < D; ++a) out[a] = p[D * i + a];
}

// W and c_s of every cell, rows of V + 1 (moving_primitives, :2412-2428); with dq and dV, their tangents: dU = (dq - U dV) / V.
template <int D>
__global__ void k_mv_prims(MeshDev<D> m, const double* __restrict__ q, const double* __restrict__ dq, const double* __restrict__ dV,
                           GasDev gas, double* __restrict__ W, double* __restrict__ dW) {
    constexpr int V = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    const double inv = 1.0 / m.vol[i];
    Dual U[V], Wd[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const double u = q[V * i + v] * inv;
        U[v] = Dual(u, dq ? (dq[V * i + v] - u * dV[i]) * inv : 0.0);
    }
    primitive_t<D, Dual>(U, gas, Wd);
    const Dual cs = sound_t<Dual>(Wd, D + 1, gas.gamma);
#pragma unroll
    for (int v = 0; v < V; ++v) W[(V + 1) * i + v] = Wd[v].v;
    W[(V + 1) * i + V] = cs.v;
    if (dW) {
#pragma unroll
        for (int v = 0; v < V; ++v) dW[(V + 1) * i + v] = Wd[v].d;
        dW[(V + 1) * i + V] = cs.d;
    }
}

// The point velocities w and (with the tangents) dw; the angle face of every cell.
template <int D>
__global__ void k_mv_velocity(MeshDev<D> m, const double* __restrict__ W, const double* __restrict__ dW, const double* __restrict__ dx,
                              const double* __restrict__ dc, const double* __restrict__ dA, double* __restrict__ w, double* __restrict__ dw,
                              int32_t* __restrict__ angle_f) {
    constexpr int V = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    const AngleFace<D> af = angle_face<D>(m, i);
    angle_f[i] = af.f;
    Dual Wd[V], cs, c[D], A[D], d[D], out[D];
#pragma unroll
    for (int v = 0; v < V; ++v) Wd[v] = Dual(W[(V + 1) * i + v], dW ? dW[(V + 1) * i + v] : 0.0);
    cs = Dual(W[(V + 1) * i + V], dW ? dW[(V + 1) * i + V] : 0.0);
    double sep[D];
    if (af.f >= 0) m.separation(i, af.other, sep);
#pragma unroll
    for (int a = 0; a < D; ++a) {
        c[a] = Dual(m.cen[D * i + a], dW ? dc[D * i + a] : 0.0);
        A[a] = af.f >= 0 ? Dual(m.area[D * af.f + a], dW ? dA[D * af.f + a] : 0.0) : Dual(0.0);
        d[a] = af.f >= 0 ? Dual(sep[a], dW ? dx[D * af.other + a] - dx[D * i + a] : 0.0) : Dual(1.0);
    }
    point_velocity_t<D, Dual>(af, Wd, cs, c, A, d, out);
#pragma unroll
    for (int a = 0; a < D; ++a) {
        w[D * i + a] = out[a].v;
        if (dw) dw[D * i + a] = out[a].d;
    }
}

// The tangent of each face's flux times |A| (moving_faces_tangent, :2457-2472).
template <int D, int Riemann>
__global__ void k_mv_faces_tangent(MeshDev<D> m, const double* __restrict__ W, const double* __restrict__ dW, const double* __restrict__ w,
                                   const double* __restrict__ dw, const double* __restrict__ dx, const double* __restrict__ dA,
                                   const double* __restrict__ dxf, GasDev gas, double* __restrict__ dG) {
    constexpr int V = D + 2;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.f) return;
    const int o = m.owner[f], j = m.neighbour[f];
    double a[D];
    load_vec<D>(m.area, f, a);
    if (dot<D>(a, a) == 0) {
#pragma unroll
        for (int v = 0; v < V; ++v) dG[V * static_cast<int64_t>(f) + v] = 0;
        return;
    }
    double sep[D];
    m.separation(o, j, sep);
    Dual d[D], xf[D], wL[D], wR[D], A[D], wf[D], L[V], R[V], G[V];
#pragma unroll
    for (int q = 0; q < D; ++q) {
        d[q] = Dual(sep[q], dx[D * j + q] - dx[D * o + q]);
        xf[q] = Dual(m.fcen[D * f + q], dxf[D * f + q]);
        wL[q] = Dual(w[D * o + q], dw[D * o + q]);
        wR[q] = Dual(w[D * j + q], dw[D * j + q]);
        A[q] = Dual(a[q], dA[D * f + q]);
    }
    face_velocity_t<D, Dual>(d, xf, wL, wR, wf);
#pragma unroll
    for (int v = 0; v < V; ++v) {
        L[v] = Dual(W[(V + 1) * o + v], dW[(V + 1) * o + v]);
        R[v] = Dual(W[(V + 1) * j + v], dW[(V + 1) * j + v]);
    }
    face_flux_t<D, Riemann, Dual>(L, R, A, wf, gas, G);
#pragma unroll
    for (int v = 0; v < V; ++v) dG[V * static_cast<int64_t>(f) + v] = G[v].d;
}

// dQ_i -= dt sum_k sign_k dG_k in list order, dx_i += dt dw_i (moving_update_tangent, :2473-2484).
template <int D>
__global__ void k_mv_update_tangent(MeshDev<D> m, const double* __restrict__ dG, const double* __restrict__ dw, double dt,
                                    double* __restrict__ dq, double* __restrict__ dx) {
    constexpr int V = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double sum[V];
#pragma unroll
    for (int v = 0; v < V; ++v) sum[v] = 0;
    for (int k = m.start[i]; k < m.start[i + 1]; ++k) {
        const int32_t e = m.list[k];
        const double sign = e >= 0 ? 1.0 : -1.0;
        const int64_t f = list_face(e);
#pragma unroll
        for (int v = 0; v < V; ++v) sum[v] += sign * dG[V * f + v];
    }
#pragma unroll
    for (int v = 0; v < V; ++v) dq[V * i + v] -= dt * sum[v];
#pragma unroll
    for (int a = 0; a < D; ++a) dx[D * i + a] += dt * dw[D * i + a];
}

// The face rows of the adjoint: W_L, W_R bars, w_L, w_R bars, d's bar, A's bar (bar_width entries).
template <int D>
__host__ __device__ constexpr int bar_width() {
    return 2 * (D + 2) + 4 * D;
}

// Per face: G's bar from both cells' Q bars, then through the flux and the face velocity to the bars of W_L, W_R, A,
// d, x_f, w_L, w_R (moving_faces_adjoint, :2510-2540), from the local Jacobians' columns.
template <int D, int Riemann>
__global__ void k_mv_faces_adjoint(MeshDev<D> m, const double* __restrict__ W, const double* __restrict__ w, const double* __restrict__ qbar,
                                   double dt, GasDev gas, double* __restrict__ face_bar, double* __restrict__ xfbar) {
    constexpr int V = D + 2, B = bar_width<D>();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.f) return;
    double* row = face_bar + static_cast<int64_t>(B) * f;
#pragma unroll
    for (int s = 0; s < B; ++s) row[s] = 0;
#pragma unroll
    for (int q = 0; q < D; ++q) xfbar[D * f + q] = 0;
    const int o = m.owner[f], j = m.neighbour[f];
    double a[D];
    load_vec<D>(m.area, f, a);
    if (dot<D>(a, a) == 0) return;
    double sep[D], xfv[D], wLv[D], wRv[D], Lv[V], Rv[V], Gbar[V];
    m.separation(o, j, sep);
    load_vec<D>(m.fcen, f, xfv);
    load_vec<D>(w, o, wLv);
    load_vec<D>(w, j, wRv);
#pragma unroll
    for (int v = 0; v < V; ++v) {
        Lv[v] = W[(V + 1) * o + v];
        Rv[v] = W[(V + 1) * j + v];
        Gbar[v] = -dt * (qbar[V * o + v] - qbar[V * j + v]);
    }
    double wf[D];
    {
        double tmp[D];
        face_velocity_t<D, double>(sep, xfv, wLv, wRv, tmp);
#pragma unroll
        for (int q = 0; q < D; ++q) wf[q] = tmp[q];
    }
    // the flux's inputs: W_L (V), W_R (V), A (D), w_f (D)
    double wfbar[D];
#pragma unroll
    for (int q = 0; q < D; ++q) wfbar[q] = 0;
    for (int s = 0; s < 2 * V + 2 * D; ++s) {
        Dual L[V], R[V], A[D], wd[D], G[V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            L[v] = Dual(Lv[v], s == v ? 1.0 : 0.0);
            R[v] = Dual(Rv[v], s == V + v ? 1.0 : 0.0);
        }
#pragma unroll
        for (int q = 0; q < D; ++q) {
            A[q] = Dual(a[q], s == 2 * V + q ? 1.0 : 0.0);
            wd[q] = Dual(wf[q], s == 2 * V + D + q ? 1.0 : 0.0);
        }
        face_flux_t<D, Riemann, Dual>(L, R, A, wd, gas, G);
        double bar = 0;
#pragma unroll
        for (int v = 0; v < V; ++v) bar += Gbar[v] * G[v].d;
        if (s < 2 * V)
            row[s] = bar;  // W_L then W_R
        else if (s < 2 * V + D)
            row[2 * V + 3 * D + (s - 2 * V)] = bar;  // A
        else
            wfbar[s - 2 * V - D] = bar;
    }
    // the face velocity's inputs: d (D), x_f (D), w_L (D), w_R (D)
    for (int s = 0; s < 4 * D; ++s) {
        Dual d[D], xf[D], wL[D], wR[D], out[D];
#pragma unroll
        for (int q = 0; q < D; ++q) {
            d[q] = Dual(sep[q], s == q ? 1.0 : 0.0);
            xf[q] = Dual(xfv[q], s == D + q ? 1.0 : 0.0);
            wL[q] = Dual(wLv[q], s == 2 * D + q ? 1.0 : 0.0);
            wR[q] = Dual(wRv[q], s == 3 * D + q ? 1.0 : 0.0);
        }
        face_velocity_t<D, Dual>(d, xf, wL, wR, out);
        double bar = 0;
#pragma unroll
        for (int q = 0; q < D; ++q) bar += wfbar[q] * out[q].d;
        if (s < D)
            row[2 * V + 2 * D + s] = bar;  // d
        else if (s < 2 * D)
            xfbar[D * f + (s - D)] = bar;
        else
            row[2 * V + (s - 2 * D)] = bar;  // w_L then w_R
    }
}

// Per cell (moving_cells_adjoint, :2544-2585): w's bar (dt x bar and the faces'), W's bar from the faces; through the
// point velocity to W, c_s, c and the angle face's A and d; c_s's bar into W's; through W = primitive(Q / V) into Q's bar
// (added) and V's bar (written).
template <int D>
__global__ void k_mv_cells_adjoint(MeshDev<D> m, const double* __restrict__ q, const double* __restrict__ W, const double* __restrict__ face_bar,
                                   const double* __restrict__ xbar, const int32_t* __restrict__ angle_f, double dt, GasDev gas,
                                   double* __restrict__ qbar, double* __restrict__ Vbar, double* __restrict__ cbar,
                                   double* __restrict__ angle_Abar, double* __restrict__ angle_dbar) {
    constexpr int V = D + 2, B = bar_width<D>();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double wbar[D], Wbar[V];
#pragma unroll
    for (int a = 0; a < D; ++a) wbar[a] = xbar[D * i + a] * dt;
#pragma unroll
    for (int v = 0; v < V; ++v) Wbar[v] = 0;
    for (int k = m.start[i]; k < m.start[i + 1]; ++k) {
        const int32_t e = m.list[k];
        const bool owned = e >= 0;
        const double* row = face_bar + static_cast<int64_t>(B) * list_face(e);
#pragma unroll
        for (int v = 0; v < V; ++v) Wbar[v] += row[(owned ? 0 : V) + v];
#pragma unroll
        for (int a = 0; a < D; ++a) wbar[a] += row[2 * V + (owned ? 0 : D) + a];
    }
    AngleFace<D> af;
    af.f = angle_f[i];
    double Wv[V], csv, cv[D], Av[D], dv[D];
#pragma unroll
    for (int v = 0; v < V; ++v) Wv[v] = W[(V + 1) * i + v];
    csv = W[(V + 1) * i + V];
    load_vec<D>(m.cen, i, cv);
    if (af.f >= 0) {
        const int32_t o = m.owner[af.f];
        af.other = o == i ? m.neighbour[af.f] : o;
        load_vec<D>(m.area, af.f, Av);
        m.separation(i, af.other, dv);
        af.amax = face_angle<D>(sqrt(dot<D>(Av, Av))) / (0.5 * sqrt(dot<D>(dv, dv)));
    } else {
#pragma unroll
        for (int a = 0; a < D; ++a) Av[a] = 0, dv[a] = 1;
    }
    // the point velocity's inputs: W (V), c_s, c (D), A (D), d (D)
    double csbar = 0;
    for (int s = 0; s < V + 1 + 3 * D; ++s) {
        Dual Wd[V], cs, c[D], A[D], d[D], out[D];
#pragma unroll
        for (int v = 0; v < V; ++v) Wd[v] = Dual(Wv[v], s == v ? 1.0 : 0.0);
        cs = Dual(csv, s == V ? 1.0 : 0.0);
#pragma unroll
        for (int a = 0; a < D; ++a) {
            c[a] = Dual(cv[a], s == V + 1 + a ? 1.0 : 0.0);
            A[a] = Dual(Av[a], s == V + 1 + D + a ? 1.0 : 0.0);
            d[a] = Dual(dv[a], s == V + 1 + 2 * D + a ? 1.0 : 0.0);
        }
        point_velocity_t<D, Dual>(af, Wd, cs, c, A, d, out);
        double bar = 0;
#pragma unroll
        for (int a = 0; a < D; ++a) bar += wbar[a] * out[a].d;
        if (s < V)
            Wbar[s] += bar;
        else if (s == V)
            csbar = bar;
        else if (s < V + 1 + D)
            cbar[D * i + (s - V - 1)] = bar;
        else if (s < V + 1 + 2 * D)
            angle_Abar[D * i + (s - V - 1 - D)] = bar;
        else
            angle_dbar[D * i + (s - V - 1 - 2 * D)] = bar;
    }
    // c_s = sqrt(gamma P / rho): its bar into W's
    for (int s = 0; s < V; ++s) {
        Dual Wd[V];
#pragma unroll
        for (int v = 0; v < V; ++v) Wd[v] = Dual(Wv[v], s == v ? 1.0 : 0.0);
        Wbar[s] += csbar * sound_t<Dual>(Wd, D + 1, gas.gamma).d;
    }
    // W = primitive(U), U = Q / V
    const double inv = 1.0 / m.vol[i];
    double Uv[V], Ubar[V];
#pragma unroll
    for (int v = 0; v < V; ++v) Uv[v] = q[V * i + v] * inv;
    for (int s = 0; s < V; ++s) {
        Dual U[V], Wd[V];
#pragma unroll
        for (int v = 0; v < V; ++v) U[v] = Dual(Uv[v], s == v ? 1.0 : 0.0);
        primitive_t<D, Dual>(U, gas, Wd);
        double bar = 0;
#pragma unroll
        for (int v = 0; v < V; ++v) bar += Wbar[v] * Wd[v].d;
        Ubar[s] = bar;
    }
    double vb = 0;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        qbar[V * i + v] += Ubar[v] * inv;
        vb -= Ubar[v] * Uv[v] * inv;
    }
    Vbar[i] = vb;
}

// A's bar: the faces' and the angle faces' of its two cells (moving_area_bar, :2587-2592).
template <int D>
__global__ void k_mv_area_adjoint(MeshDev<D> m, const double* __restrict__ face_bar, const int32_t* __restrict__ angle_f,
                                  const double* __restrict__ angle_Abar, double* __restrict__ Abar) {
    constexpr int V = D + 2, B = bar_width<D>();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.f) return;
    const int o = m.owner[f], j = m.neighbour[f];
#pragma unroll
    for (int a = 0; a < D; ++a)
        Abar[D * f + a] = face_bar[static_cast<int64_t>(B) * f + 2 * V + 3 * D + a] + (angle_f[o] == f ? angle_Abar[D * o + a] : 0.0) +
                          (angle_f[j] == f ? angle_Abar[D * j + a] : 0.0);
}

// x's bar from the separations (moving_separation_bar, :2593-2603): the faces' d = x_j - x_o and the angle faces'
// d = x_other - x_i, added to x bar (the geometry's part is the caller's).
template <int D>
__global__ void k_mv_separation_adjoint(MeshDev<D> m, const double* __restrict__ face_bar, const int32_t* __restrict__ angle_f,
                                        const double* __restrict__ angle_dbar, double* __restrict__ xbar) {
    constexpr int V = D + 2, B = bar_width<D>();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double sum[D];
#pragma unroll
    for (int a = 0; a < D; ++a) sum[a] = -angle_dbar[D * i + a];
    for (int k = m.start[i]; k < m.start[i + 1]; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e);
        const bool owned = e >= 0;
        const int j = owned ? m.neighbour[f] : m.owner[f];
        const double* db = face_bar + static_cast<int64_t>(B) * f + 2 * V + 2 * D;
#pragma unroll
        for (int a = 0; a < D; ++a) sum[a] += owned ? -db[a] : db[a];
        if (angle_f[j] == f)
#pragma unroll
            for (int a = 0; a < D; ++a) sum[a] += angle_dbar[D * j + a];
    }
#pragma unroll
    for (int a = 0; a < D; ++a) xbar[D * i + a] += sum[a];
}

}  // namespace mvd
}  // namespace luna
