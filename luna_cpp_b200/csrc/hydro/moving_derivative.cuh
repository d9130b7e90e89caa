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

#include "adjoint.cuh"
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
// The transpose of face_flux_t in reverse mode (MovingFace::adjoint, euler.hpp:883-916): G = |A| to_lab(F, w), F the
// static solve of the face-frame states L - w, R - w along n = A / |A|. The solve's adjoint in its states
// (hllc_flux_adjoint / hll_flux_adjoint), to_lab's in F and w, and n's bar from the solve's invariance under rotations:
// for dn orthogonal to n, <Fbar, dF/dn dn> = dn . (turn(Fbar, F) - turn(Lbar, L') - turn(Rbar, R')) on the velocity parts,
// turn(a, b) = a (n . b) - b (n . a). Adds into Lbar, Rbar, Abar, wbar.
template <int D, int Riemann>
__device__ void moving_face_adjoint(const double* L, const double* R, const double* A, const double* w, const GasDev& gas,
                                    const double* Gbar, double* Lbar, double* Rbar, double* Abar, double* wbar) {
    constexpr int V = D + 2, P = D + 1;
    const double mag = sqrt(dot<D>(A, A)), inv = 1.0 / mag;
    double n[D];
#pragma unroll
    for (int a = 0; a < D; ++a) n[a] = A[a] * inv;
    double Lr[V], Rr[V], F[V];
#pragma unroll
    for (int v = 0; v < V; ++v) Lr[v] = L[v], Rr[v] = R[v];
#pragma unroll
    for (int k = 0; k < D; ++k) Lr[1 + k] -= w[k], Rr[1 + k] -= w[k];
    const double zero[D] = {};
    if constexpr (Riemann == 1)
        hll_flux<D>(Lr, Rr, n, zero, gas, F, false);
    else
        hllc_flux<D, double>(Lr, Rr, n, zero, gas.gamma, gas.inverse_gm1, F, false);
    double lab[V];
#pragma unroll
    for (int v = 0; v < V; ++v) lab[v] = F[v];
    to_lab<D, double>(lab, w);
    // G = |A| lab
    double magbar = 0, labbar[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        magbar += Gbar[v] * lab[v];
        labbar[v] = mag * Gbar[v];
    }
    // lab = to_lab(F, w): momentum += w F_0, energy += w . F_mom + |w|^2 / 2 F_0
    double Fbar[V];
    Fbar[0] = labbar[0] + 0.5 * dot<D>(w, w) * labbar[P];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        Fbar[0] += w[k] * labbar[1 + k];
        Fbar[1 + k] = labbar[1 + k] + w[k] * labbar[P];
        wbar[k] += labbar[1 + k] * F[0] + labbar[P] * (F[1 + k] + w[k] * F[0]);
    }
    Fbar[P] = labbar[P];
    double Lrb[V], Rrb[V];
#pragma unroll
    for (int v = 0; v < V; ++v) Lrb[v] = Rrb[v] = 0;
    if constexpr (Riemann == 1)
        hll_flux_adjoint<D>(Lr, Rr, n, gas, Fbar, Lrb, Rrb);
    else
        hllc_flux_adjoint<D>(Lr, Rr, n, gas, Fbar, Lrb, Rrb);
    const auto turn = [&](const double* a, const double* b, double* out, double sign) {
        const double nb = dot<D>(n, b), na = dot<D>(n, a);
#pragma unroll
        for (int k = 0; k < D; ++k) out[k] += sign * (a[k] * nb - b[k] * na);
    };
    double nbar[D] = {};
    turn(Fbar + 1, F + 1, nbar, 1.0);
    turn(Lrb + 1, Lr + 1, nbar, -1.0);
    turn(Rrb + 1, Rr + 1, nbar, -1.0);
    const double nn = dot<D>(n, nbar);
#pragma unroll
    for (int a = 0; a < D; ++a) Abar[a] += magbar * n[a] + (nbar[a] - n[a] * nn) * inv;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        Lbar[v] += Lrb[v];
        Rbar[v] += Rrb[v];
    }
#pragma unroll
    for (int k = 0; k < D; ++k) wbar[k] -= Lrb[1 + k] + Rrb[1 + k];
}

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
    // the flux's inputs, W_L (V), W_R (V), A (D), w_f (D), by the face's reverse mode
    double wfbar[D], Lbar[V], Rbar[V], Ab[D];
#pragma unroll
    for (int q = 0; q < D; ++q) wfbar[q] = Ab[q] = 0;
#pragma unroll
    for (int v = 0; v < V; ++v) Lbar[v] = Rbar[v] = 0;
    moving_face_adjoint<D, Riemann>(Lv, Rv, a, wf, gas, Gbar, Lbar, Rbar, Ab, wfbar);
#pragma unroll
    for (int v = 0; v < V; ++v) {
        row[v] = Lbar[v];  // W_L then W_R
        row[V + v] = Rbar[v];
    }
#pragma unroll
    for (int q = 0; q < D; ++q) row[2 * V + 3 * D + q] = Ab[q];  // A
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

// ---- Order 1 (step_moving_tangent_1 / step_moving_adjoint_1, finite_volume.hpp:2626-3155): the MUSCL-Hancock moving
// step's two passes (W + g r on the mesh of t^n; W a whole step on, to the face of t^n+1) with the limited gradients, the
// grid-step point velocities w-hat (their quantisation taken as the identity: tangent dw) and the meshes of t^n and t^n+1.
// The gradients are the reference's direct fit (an area-weighted least squares with intercept, its Cholesky solve and the
// face-centroid clip in list order, limited_core :1008-1034), here on dual numbers so that it carries the derivative in
// every input: W of the cell and its neighbours, the separations, the centroids, the areas and the face centroids.

// The direction of the fit's inputs for one dual pass: the caller's tangents, one unit seed, or none.
template <int D>
struct FitDirection {
    static constexpr int V = D + 2, R = V + 1;
    const double *dW = nullptr, *dx = nullptr, *dc = nullptr, *dA = nullptr, *dxf = nullptr;  // tangents (null: zero)
    int kind = -1, entry = -1, comp = -1;  // a unit seed: 0 W_i, 1 c_i, 2 W_j, 3 d (x_j - x_i), 4 c_j, 5 A, 6 x_f of an entry
    __device__ double Wi(int i, int v) const { return kind >= 0 ? (kind == 0 && comp == v ? 1.0 : 0.0) : dW ? dW[R * i + v] : 0.0; }
    __device__ double ci(int i, int a) const { return kind >= 0 ? (kind == 1 && comp == a ? 1.0 : 0.0) : dc ? dc[D * i + a] : 0.0; }
    __device__ double Wj(int k, int j, int v) const {
        return kind >= 0 ? (kind == 2 && entry == k && comp == v ? 1.0 : 0.0) : dW ? dW[R * j + v] : 0.0;
    }
    __device__ double d(int k, int i, int j, int a) const {
        return kind >= 0 ? (kind == 3 && entry == k && comp == a ? 1.0 : 0.0) : dx ? dx[D * j + a] - dx[D * i + a] : 0.0;
    }
    __device__ double cj(int k, int j, int a) const { return kind >= 0 ? (kind == 4 && entry == k && comp == a ? 1.0 : 0.0) : dc ? dc[D * j + a] : 0.0; }
    __device__ double A(int k, int f, int a) const { return kind >= 0 ? (kind == 5 && entry == k && comp == a ? 1.0 : 0.0) : dA ? dA[D * f + a] : 0.0; }
    __device__ double xf(int k, int f, int a) const {
        return kind >= 0 ? (kind == 6 && entry == k && comp == a ? 1.0 : 0.0) : dxf ? dxf[D * f + a] : 0.0;
    }
};

// Cell i's limited gradient on dual numbers (the adjoint's k_sweep_fit arithmetic: Sweep with the fit, finite_volume.hpp:
// 486-515, 591-615, the tiny-face rule and the face-centroid clip, :1008-1034). W: rows of V + 1 (W, c_s).
template <int D>
__device__ void fit_gradient_t(const MeshDev<D>& m, int i, const double* __restrict__ W, bool limit, const FitDirection<D>& dir,
                               Dual (&g)[(D + 2) * D]) {
    constexpr int V = D + 2, U = D + 1, R = V + 1;
    Dual Wi[V], ci[D];
#pragma unroll
    for (int v = 0; v < V; ++v) Wi[v] = Dual(W[R * i + v], dir.Wi(i, v));
#pragma unroll
    for (int a = 0; a < D; ++a) ci[a] = Dual(m.cen[D * i + a], dir.ci(i, a));
    const int first = m.start[i], end = m.start[i + 1];
    double surface = 0, smallest = __longlong_as_double(0x7ff0000000000000ll);
    Dual M[U][U], b[V][U], lo[V], hi[V];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s < U; ++s) M[p][s] = Dual(0.0);
#pragma unroll
    for (int v = 0; v < V; ++v) {
        lo[v] = Dual(finite_max<double>());
        hi[v] = Dual(-finite_max<double>());
#pragma unroll
        for (int p = 0; p < U; ++p) b[v][p] = Dual(0.0);
    }
    for (int k = first; k < end; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e), j = e >= 0 ? m.neighbour[f] : m.owner[f], kk = k - first;
        Dual A[D], d[D], X[U];
        double sep[D];
        m.separation(i, j, sep);
#pragma unroll
        for (int a = 0; a < D; ++a) {
            A[a] = Dual(m.area[D * f + a], dir.A(kk, f, a));
            d[a] = Dual(sep[a], dir.d(kk, i, j, a));
        }
        const Dual w = sqrt(dot<D>(A, A));
        surface += w.v;
        smallest = fmin(smallest, w.v);
        X[0] = Dual(1.0);
#pragma unroll
        for (int p = 1; p < U; ++p) X[p] = d[p - 1] + Dual(m.cen[D * j + p - 1], dir.cj(kk, j, p - 1)) - ci[p - 1];
#pragma unroll
        for (int p = 0; p < U; ++p)
#pragma unroll
            for (int s = p; s < U; ++s) M[p][s] += w * X[p] * X[s];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const Dual Wj = Dual(W[R * j + v], dir.Wj(kk, j, v));
            const Dual dW = Wj - Wi[v];
#pragma unroll
            for (int p = 0; p < U; ++p) b[v][p] += w * X[p] * dW;
            if (Wj.v < lo[v].v) lo[v] = Wj;
            if (Wj.v > hi[v].v) hi[v] = Wj;
        }
    }
    const double tiny = 1e-6 * surface;
    const bool any_tiny = smallest < tiny;
    if (any_tiny) {  // the range without the tiny faces' neighbours
#pragma unroll
        for (int v = 0; v < V; ++v) {
            lo[v] = Dual(finite_max<double>());
            hi[v] = Dual(-finite_max<double>());
        }
        for (int k = first; k < end; ++k) {
            const int32_t e = m.list[k];
            const int f = list_face(e), j = e >= 0 ? m.neighbour[f] : m.owner[f], kk = k - first;
            if (m.mag[f] < tiny) continue;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const Dual Wj = Dual(W[R * j + v], dir.Wj(kk, j, v));
                if (Wj.v < lo[v].v) lo[v] = Wj;
                if (Wj.v > hi[v].v) hi[v] = Wj;
            }
        }
    }
    // M is symmetric: the solve reads its upper triangle
    cholesky_solve<D, Dual>(M, b, g);
    if (!limit) return;
    for (int k = first; k < end; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e), kk = k - first;
        if (any_tiny && m.mag[f] < tiny) continue;
        Dual o[D];
        if (e >= 0) {
#pragma unroll
            for (int a = 0; a < D; ++a) o[a] = Dual(m.fcen[D * f + a], dir.xf(kk, f, a)) - ci[a];
        } else {  // face_offset: the owner j's face centroid moved to i's generator, x_f + (x_j - x_i)
            const int j = m.owner[f];
            double sep[D];
            m.separation(i, j, sep);
#pragma unroll
            for (int a = 0; a < D; ++a) o[a] = Dual(m.fcen[D * f + a], dir.xf(kk, f, a)) + Dual(sep[a], dir.d(kk, i, j, a)) - ci[a];
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            Dual* gv = g + D * v;
            const Dual dp = dot<D>(gv, o);
            if (dp.v > 0 && Wi[v].v + dp.v > hi[v].v) {
                const Dual sc = hi[v].v > Wi[v].v ? (hi[v] - Wi[v]) / dp : Dual(0.0);
#pragma unroll
                for (int a = 0; a < D; ++a) gv[a] = gv[a] * sc;
            } else if (dp.v < 0 && Wi[v].v + dp.v < lo[v].v) {
                const Dual sc = lo[v].v < Wi[v].v ? (lo[v] - Wi[v]) / dp : Dual(0.0);
#pragma unroll
                for (int a = 0; a < D; ++a) gv[a] = gv[a] * sc;
            }
        }
    }
}

// Per cell: the limited gradient g [N][V D] and (with the tangents) dg; c^n (the centroids the second pass starts from);
// w-hat, the whole grid steps of x + dt w per dt (k_keep_centroids' rounding), and its tangent dw (0 with the steps held).
template <int D>
__global__ void k_mv1_cells(MeshDev<D> m, const double* __restrict__ W, const double* __restrict__ dW, const double* __restrict__ dx,
                            const double* __restrict__ dc, const double* __restrict__ dA, const double* __restrict__ dxf,
                            const double* __restrict__ x, const double* __restrict__ w, bool limit, double dt, double step, double per_step,
                            long long p0, long long p1, long long p2, double* __restrict__ g, double* __restrict__ dg, double* __restrict__ wh,
                            double* __restrict__ c0, double* __restrict__ dc0) {
    constexpr int V = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    FitDirection<D> dir;
    dir.dW = dW, dir.dx = dx, dir.dc = dc, dir.dA = dA, dir.dxf = dxf;
    Dual gd[V * D];
    fit_gradient_t<D>(m, i, W, limit, dir, gd);
#pragma unroll
    for (int c = 0; c < V * D; ++c) {
        g[V * D * static_cast<int64_t>(i) + c] = gd[c].v;
        if (dg) dg[V * D * static_cast<int64_t>(i) + c] = gd[c].d;
    }
    const long long period[3] = {p0, p1, p2};
    const double unit = step / dt;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const long long p = period[a];
        long long k0 = llround(x[D * i + a] * per_step);
        k0 = ((k0 % p) + p) % p;
        long long k1 = llround((x[D * i + a] + dt * w[D * i + a]) * per_step);
        k1 = ((k1 % p) + p) % p;
        long long s = k1 - k0;
        if (s > p / 2) s -= p;
        if (s < -(p / 2)) s += p;
        wh[D * i + a] = static_cast<double>(s) * unit;
        c0[D * i + a] = m.cen[D * i + a];
        if (dc0) dc0[D * i + a] = dc ? dc[D * i + a] : 0.0;
    }
}

// One side of a pass: W + g r (pass 1), or W a whole step on (the half-step rate at 2 dt) plus g r (pass 2); the cell's W
// where rho or P would not stay positive (FaceFlux::side_value, :1342-1347).
template <int D, bool Second, class T>
__device__ __forceinline__ void pass_side_t(const T* W, const T* g, const T* r, double dt, double gamma, T* Wf, bool& fallback) {
    constexpr int V = D + 2;
    if constexpr (Second) {
        T A[V];
        half_step_rate<D, T>(W, g, T(gamma), A);
#pragma unroll
        for (int v = 0; v < V; ++v) Wf[v] = W[v] - T(0.5 * (2 * dt)) * A[v];
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) Wf[v] = W[v];
    }
#pragma unroll
    for (int v = 0; v < V; ++v) Wf[v] += dot<D>(g + D * v, r);
    fallback = !(Wf[0] > T(0) && Wf[D + 1] > T(0));
    if (fallback)
#pragma unroll
        for (int v = 0; v < V; ++v) Wf[v] = W[v];
}

// The offset r of cell i's side of face f in a pass (pass_offset, :2876-2880): face_offset(f, i) on this mesh; pass 2 from the
// old centroid to the new face plus dt w-hat. Values only.
template <int D, bool Second>
__device__ __forceinline__ void pass_offset(const MeshDev<D>& m, int f, int i, const double* wh, const double* c0, double dt, double* r) {
    m.face_offset(f, i, r);
    if constexpr (Second)
#pragma unroll
        for (int a = 0; a < D; ++a) r[a] = r[a] + m.cen[D * i + a] - c0[D * i + a] + wh[D * i + a] * (0.5 * (2 * dt));
}

// One pass's tangent per face (moving_pass_tangent, :2833-2865): both sides' tangents (W, g, the offset through x, c, x_f and
// pass 2's c^n and w-hat), the face velocity's (w-hat, d, x_f) and the area's, through the flux.
template <int D, int Riemann, bool Second>
__global__ void k_mv1_pass_tangent(MeshDev<D> m, const double* __restrict__ W, const double* __restrict__ dW, const double* __restrict__ g,
                                   const double* __restrict__ dg, const double* __restrict__ wh, const double* __restrict__ dw,
                                   const double* __restrict__ c0, const double* __restrict__ dc0, const double* __restrict__ dx,
                                   const double* __restrict__ dc, const double* __restrict__ dA, const double* __restrict__ dxf, double dt,
                                   GasDev gas, double* __restrict__ dG) {
    constexpr int V = D + 2, R = V + 1;
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
    Dual side[2][V];
    for (int s = 0; s < 2; ++s) {
        const int i = s == 0 ? o : j;
        Dual Wi[V], gi[V * D], r[D];
#pragma unroll
        for (int v = 0; v < V; ++v) Wi[v] = Dual(W[R * i + v], dW[R * i + v]);
#pragma unroll
        for (int c = 0; c < V * D; ++c) gi[c] = Dual(g[V * D * static_cast<int64_t>(i) + c], dg[V * D * static_cast<int64_t>(i) + c]);
        double rv[D];
        pass_offset<D, Second>(m, f, i, wh, c0, dt, rv);
#pragma unroll
        for (int q = 0; q < D; ++q) {  // offset_tangent (:2618-2621): dx_f - dc_i (+ dx_o - dx_i off the owner)
            double dr = dxf[D * f + q] - dc[D * i + q] + (i != o ? dx[D * o + q] - dx[D * i + q] : 0.0);
            if constexpr (Second) dr += dc[D * i + q] - dc0[D * i + q] + dw[D * i + q] * dt;
            r[q] = Dual(rv[q], dr);
        }
        bool fallback;
        pass_side_t<D, Second, Dual>(Wi, gi, r, dt, gas.gamma, side[s], fallback);
    }
    double sep[D];
    m.separation(o, j, sep);
    Dual d[D], xf[D], wL[D], wR[D], A[D], wf[D], G[V];
#pragma unroll
    for (int q = 0; q < D; ++q) {
        d[q] = Dual(sep[q], dx[D * j + q] - dx[D * o + q]);
        xf[q] = Dual(m.fcen[D * f + q], dxf[D * f + q]);
        wL[q] = Dual(wh[D * o + q], dw[D * o + q]);
        wR[q] = Dual(wh[D * j + q], dw[D * j + q]);
        A[q] = Dual(a[q], dA[D * f + q]);
    }
    face_velocity_t<D, Dual>(d, xf, wL, wR, wf);
    face_flux_t<D, Riemann, Dual>(side[0], side[1], A, wf, gas, G);
#pragma unroll
    for (int v = 0; v < V; ++v) dG[V * static_cast<int64_t>(f) + v] = G[v].d;
}

// dQ_i -= dt / 2 sum_k sign_k dG_k in list order (moving_pass_update_tangent, :2866-2875).
template <int D>
__global__ void k_mv1_pass_update_tangent(MeshDev<D> m, const double* __restrict__ dG, double dt, double* __restrict__ dq) {
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
    for (int v = 0; v < V; ++v) dq[V * i + v] -= 0.5 * dt * sum[v];
}

// x^n+1's tangent: dx += dt dw.
template <int D>
__global__ void k_mv1_drift_tangent(int n, const double* __restrict__ dw, double dt, double* __restrict__ dx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int a = 0; a < D; ++a) dx[D * i + a] += dt * dw[D * i + a];
}

// A pass's face rows in the adjoint: the two sides' bars, w-hat's two bars, d's bar, the neighbour side's offset bar.
template <int D>
__host__ __device__ constexpr int pass_width() {
    return 2 * (D + 2) + 4 * D;
}

// One pass's adjoint per face (moving_pass_adjoint, :2882-2929): the flux's local Jacobian columns times G's bar -> the sides',
// the area's and the face velocity's bars; the face velocity's -> d, x_f, w-hat; the sides' offsets' bars g^T S-bar (where
// the side did not fall back) into x_f's bar and, for the neighbour's side (whose offset carries x_owner), the row.
template <int D, int Riemann, bool Second>
__global__ void k_mv1_pass_faces_adjoint(MeshDev<D> m, const double* __restrict__ W, const double* __restrict__ g, const double* __restrict__ wh,
                                         const double* __restrict__ c0, const double* __restrict__ qbar, double dt, GasDev gas,
                                         double* __restrict__ rows, double* __restrict__ Abar, double* __restrict__ xfbar) {
    constexpr int V = D + 2, R = V + 1, B = pass_width<D>();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.f) return;
    double* row = rows + static_cast<int64_t>(B) * f;
#pragma unroll
    for (int s = 0; s < B; ++s) row[s] = 0;
#pragma unroll
    for (int q = 0; q < D; ++q) Abar[D * f + q] = xfbar[D * f + q] = 0;
    const int o = m.owner[f], j = m.neighbour[f];
    double a[D];
    load_vec<D>(m.area, f, a);
    if (dot<D>(a, a) == 0) return;
    double side[2][V], Gbar[V];
    bool fallback[2];
    for (int s = 0; s < 2; ++s) {
        const int i = s == 0 ? o : j;
        double r[D];
        pass_offset<D, Second>(m, f, i, wh, c0, dt, r);
        pass_side_t<D, Second, double>(W + R * i, g + V * D * static_cast<int64_t>(i), r, dt, gas.gamma, side[s], fallback[s]);
    }
#pragma unroll
    for (int v = 0; v < V; ++v) Gbar[v] = -0.5 * dt * (qbar[V * o + v] - qbar[V * j + v]);
    double sep[D], xfv[D], wLv[D], wRv[D], wf[D];
    m.separation(o, j, sep);
    load_vec<D>(m.fcen, f, xfv);
    load_vec<D>(wh, o, wLv);
    load_vec<D>(wh, j, wRv);
    face_velocity_t<D, double>(sep, xfv, wLv, wRv, wf);
    double Sbar[2][V], wfbar[D], Ab[D];
#pragma unroll
    for (int q = 0; q < D; ++q) wfbar[q] = Ab[q] = 0;
#pragma unroll
    for (int v = 0; v < V; ++v) Sbar[0][v] = Sbar[1][v] = 0;
    moving_face_adjoint<D, Riemann>(side[0], side[1], a, wf, gas, Gbar, Sbar[0], Sbar[1], Ab, wfbar);
#pragma unroll
    for (int q = 0; q < D; ++q) Abar[D * f + q] = Ab[q];
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
            xfbar[D * f + (s - D)] += bar;
        else
            row[2 * V + (s - 2 * D)] = bar;  // w-hat of the owner, then of the neighbour
    }
    for (int s = 0; s < 2; ++s) {
        const int i = s == 0 ? o : j;
        double rbar[D];
#pragma unroll
        for (int q = 0; q < D; ++q) {
            rbar[q] = 0;
            if (!fallback[s])
#pragma unroll
                for (int v = 0; v < V; ++v) rbar[q] += g[V * D * static_cast<int64_t>(i) + D * v + q] * Sbar[s][v];
            xfbar[D * f + q] += rbar[q];
            if (s == 1) row[2 * V + 3 * D + q] = rbar[q];
        }
#pragma unroll
        for (int v = 0; v < V; ++v) row[(s == 0 ? 0 : V) + v] = Sbar[s][v];
    }
}

// Each cell's sides of one pass (moving_pass_gather, :2931-2985): the side's adjoint into W's and g's bars (the local
// Jacobian's columns), its offset's bar into c^n's (and w-hat's on pass 2) and x's, its share of the face velocity's
// adjoint into w-hat's and x's bars. Added to the running bars.
template <int D, bool Second>
__global__ void k_mv1_pass_gather(MeshDev<D> m, const double* __restrict__ W, const double* __restrict__ g, const double* __restrict__ wh,
                                  const double* __restrict__ c0, const double* __restrict__ rows, double dt, GasDev gas, double* __restrict__ Wb,
                                  double* __restrict__ gb, double* __restrict__ whb, double* __restrict__ cb, double* __restrict__ xb) {
    constexpr int V = D + 2, R = V + 1, B = pass_width<D>();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double Wv[V], gv[V * D];
#pragma unroll
    for (int v = 0; v < V; ++v) Wv[v] = W[R * i + v];
#pragma unroll
    for (int c = 0; c < V * D; ++c) gv[c] = g[V * D * static_cast<int64_t>(i) + c];
    double Wbar[V], gbar[V * D], whbar[D], cbar[D], xbar[D];
#pragma unroll
    for (int v = 0; v < V; ++v) Wbar[v] = 0;
#pragma unroll
    for (int c = 0; c < V * D; ++c) gbar[c] = 0;
#pragma unroll
    for (int q = 0; q < D; ++q) whbar[q] = cbar[q] = xbar[q] = 0;
    for (int k = m.start[i]; k < m.start[i + 1]; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e);
        double a[D];
        load_vec<D>(m.area, f, a);
        if (dot<D>(a, a) == 0) continue;
        const bool owned = e >= 0;
        const double* row = rows + static_cast<int64_t>(B) * f;
        double Sbar[V], r[D];
#pragma unroll
        for (int v = 0; v < V; ++v) Sbar[v] = row[(owned ? 0 : V) + v];
        pass_offset<D, Second>(m, f, i, wh, c0, dt, r);
        bool fallback = false;
        for (int s = 0; s < V + V * D; ++s) {  // the side's columns in W and g
            Dual Wd[V], gd[V * D], rd[D], out[V];
#pragma unroll
            for (int v = 0; v < V; ++v) Wd[v] = Dual(Wv[v], s == v ? 1.0 : 0.0);
#pragma unroll
            for (int c = 0; c < V * D; ++c) gd[c] = Dual(gv[c], s == V + c ? 1.0 : 0.0);
#pragma unroll
            for (int q = 0; q < D; ++q) rd[q] = Dual(r[q]);
            pass_side_t<D, Second, Dual>(Wd, gd, rd, dt, gas.gamma, out, fallback);
            double bar = 0;
#pragma unroll
            for (int v = 0; v < V; ++v) bar += Sbar[v] * out[v].d;
            if (s < V)
                Wbar[s] += bar;
            else
                gbar[s - V] += bar;
        }
        double rbar[D];
#pragma unroll
        for (int q = 0; q < D; ++q) {
            rbar[q] = 0;
            if (!fallback)
#pragma unroll
                for (int v = 0; v < V; ++v) rbar[q] += gv[D * v + q] * Sbar[v];
            cbar[q] -= rbar[q];
            if constexpr (Second) whbar[q] += rbar[q] * dt;
            if (!owned) xbar[q] -= rbar[q];                     // own offset: + x_o - x_i
            if (owned) xbar[q] += row[2 * V + 3 * D + q];      // the neighbour's offset carries x_i
            whbar[q] += row[2 * V + (owned ? 0 : D) + q];      // the face velocity's share
            xbar[q] += owned ? -row[2 * V + 2 * D + q] : row[2 * V + 2 * D + q];  // d = x_j - x_o
        }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) Wb[V * i + v] += Wbar[v];
#pragma unroll
    for (int c = 0; c < V * D; ++c) gb[V * D * static_cast<int64_t>(i) + c] += gbar[c];
#pragma unroll
    for (int q = 0; q < D; ++q) {
        whb[D * i + q] += whbar[q];
        cb[D * i + q] += cbar[q];
        xb[D * i + q] += xbar[q];
    }
}

// x^n+1 = x^n + dt w-hat: w-hat's bar takes dt x^n+1's; x^n's bar is x^n+1's (moving_drift_adjoint, :3034-3038).
template <int D>
__global__ void k_mv1_drift_adjoint(int n, const double* __restrict__ xb, double dt, double* __restrict__ whb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int a = 0; a < D; ++a) whb[D * i + a] += dt * xb[D * i + a];
}

// The fit's entry rows: per list entry, the bars of the neighbour's W, the separation, the neighbour's centroid, the area
// and the face centroid (V + 4 D).
template <int D>
__host__ __device__ constexpr int entry_width() {
    return (D + 2) + 4 * D;
}

// Per cell at t^n (moving_cells_adjoint_1, :3068-3105): w-hat's bar through the point velocity (W, c_s, c, the angle face's
// A and d); c_s's bar into W's; g's bar through the fit: the cell's own W and c bars, and each entry's bars into the entry
// rows. Wb and cb hold the passes' sums on entry and the cell's own totals on return.
// The transpose of fit_gradient_t's Jacobian in reverse mode, for the bars gbar of cell i's limited gradient: the
// forward fit again (M, b, the range and its entries, the clips in list order), then the last clip's scale
// s = (bound - W_i) / (g0 . o) backwards onto g0, the bound's entry and the offset; M x = b once more for b's bars
// (bbar = M^-1 xbar, M symmetric) and M's (-bbar x^T); and each entry's share through w = |A| and X = (1, d + c_j - c_i)
// (the reference's moving_gradient_adjoint, finite_volume.hpp:2690-2760). Adds into Wibar, cibar; writes each entry's
// row of entry_width: W_j, d, c_j, A, x_f.
template <int D>
__device__ void fit_gradient_adjoint(const MeshDev<D>& m, int i, const double* __restrict__ W, bool limit, const double* gbar,
                                     double (&Wibar)[D + 2], double (&cibar)[D], double* __restrict__ rows) {
    constexpr int V = D + 2, U = D + 1, R = V + 1, E = entry_width<D>();
    double Wi[V], ci[D];
#pragma unroll
    for (int v = 0; v < V; ++v) Wi[v] = W[R * i + v];
#pragma unroll
    for (int a = 0; a < D; ++a) ci[a] = m.cen[D * i + a];
    const int first = m.start[i], end = m.start[i + 1];
    double surface = 0, smallest = __longlong_as_double(0x7ff0000000000000ll);
    double M[U][U], b[V][U], lo[V], hi[V];
    int lo_k[V], hi_k[V];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int q = 0; q < U; ++q) M[p][q] = 0.0;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        lo[v] = finite_max<double>();
        hi[v] = -finite_max<double>();
        lo_k[v] = hi_k[v] = -1;
#pragma unroll
        for (int p = 0; p < U; ++p) b[v][p] = 0.0;
    }
    // the entry k's face, neighbour, area vector, |A|, X and W_j
    const auto entry = [&](int k, int& f, int& j, bool& owned, double (&A)[D], double& w, double (&X)[U]) {
        const int32_t e = m.list[k];
        f = list_face(e);
        owned = e >= 0;
        j = owned ? m.neighbour[f] : m.owner[f];
        double sep[D];
        m.separation(i, j, sep);
#pragma unroll
        for (int a = 0; a < D; ++a) A[a] = m.area[D * f + a];
        w = sqrt(dot<D>(A, A));
        X[0] = 1.0;
#pragma unroll
        for (int p = 1; p < U; ++p) X[p] = sep[p - 1] + m.cen[D * j + p - 1] - ci[p - 1];
    };
    for (int k = first; k < end; ++k) {
        int f, j;
        bool owned;
        double A[D], w, X[U];
        entry(k, f, j, owned, A, w, X);
        surface += w;
        smallest = fmin(smallest, w);
#pragma unroll
        for (int p = 0; p < U; ++p)
#pragma unroll
            for (int q = p; q < U; ++q) M[p][q] += w * X[p] * X[q];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const double Wj = W[R * j + v], dW = Wj - Wi[v];
#pragma unroll
            for (int p = 0; p < U; ++p) b[v][p] += w * X[p] * dW;
            if (Wj < lo[v]) lo[v] = Wj, lo_k[v] = k - first;
            if (Wj > hi[v]) hi[v] = Wj, hi_k[v] = k - first;
        }
    }
    const double tiny = 1e-6 * surface;
    const bool any_tiny = smallest < tiny;
    if (any_tiny) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            lo[v] = finite_max<double>();
            hi[v] = -finite_max<double>();
            lo_k[v] = hi_k[v] = -1;
        }
        for (int k = first; k < end; ++k) {
            const int32_t e = m.list[k];
            const int f = list_face(e), j = e >= 0 ? m.neighbour[f] : m.owner[f];
            if (m.mag[f] < tiny) continue;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const double Wj = W[R * j + v];
                if (Wj < lo[v]) lo[v] = Wj, lo_k[v] = k - first;
                if (Wj > hi[v]) hi[v] = Wj, hi_k[v] = k - first;
            }
        }
    }
    // Cholesky of M (its upper triangle) and the fit of every variable, as cholesky_solve
    double L[U][U];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int q = 0; q < U; ++q) L[p][q] = 0.0;
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int q = 0; q <= p; ++q) {
            double sum = M[q][p];
#pragma unroll
            for (int k = 0; k < q; ++k) sum -= L[p][k] * L[q][k];
            L[p][q] = p == q ? sqrt(sum) : sum / L[q][q];
        }
    const auto solve = [&](const double (&r)[U], double (&x)[U]) {
        double z[U];
#pragma unroll
        for (int p = 0; p < U; ++p) {
            double sum = r[p];
#pragma unroll
            for (int k = 0; k < p; ++k) sum -= L[p][k] * z[k];
            z[p] = sum / L[p][p];
        }
#pragma unroll
        for (int p = U - 1; p >= 0; --p) {
            double sum = z[p];
#pragma unroll
            for (int k = p + 1; k < U; ++k) sum -= L[k][p] * x[k];
            x[p] = sum / L[p][p];
        }
    };
    double xs[V][U], g[V][D];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        solve(b[v], xs[v]);
#pragma unroll
        for (int a = 0; a < D; ++a) g[v][a] = xs[v][1 + a];
    }
    // the clips in list order: each variable's last one (entry, which bound, to zero or not, its face offset)
    int last[V];
    bool upper[V], zero[V], last_owned[V];
    double offset[V][D];
#pragma unroll
    for (int v = 0; v < V; ++v) last[v] = -1, upper[v] = zero[v] = false, last_owned[v] = true;
    if (limit)
        for (int k = first; k < end; ++k) {
            const int32_t e = m.list[k];
            const int f = list_face(e);
            if (any_tiny && m.mag[f] < tiny) continue;
            double o[D];
            if (e >= 0) {
#pragma unroll
                for (int a = 0; a < D; ++a) o[a] = m.fcen[D * f + a] - ci[a];
            } else {
                double sep[D];
                m.separation(i, m.owner[f], sep);
#pragma unroll
                for (int a = 0; a < D; ++a) o[a] = m.fcen[D * f + a] + sep[a] - ci[a];
            }
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const double dp = dot<D>(g[v], o);
                bool clip = false, up = false;
                double sc = 0.0;
                if (dp > 0 && Wi[v] + dp > hi[v]) {
                    clip = up = true;
                    sc = hi[v] > Wi[v] ? (hi[v] - Wi[v]) / dp : 0.0;
                } else if (dp < 0 && Wi[v] + dp < lo[v]) {
                    clip = true;
                    sc = lo[v] < Wi[v] ? (lo[v] - Wi[v]) / dp : 0.0;
                }
                if (!clip) continue;
#pragma unroll
                for (int a = 0; a < D; ++a) g[v][a] = g[v][a] * sc;
                last[v] = k - first;
                upper[v] = up;
                zero[v] = up ? !(hi[v] > Wi[v]) : !(lo[v] < Wi[v]);
                last_owned[v] = e >= 0;
#pragma unroll
                for (int a = 0; a < D; ++a) offset[v][a] = o[a];
            }
        }
    // backwards through the clip: g = g0 s, s = (bound - W_i) / (g0 . o)
    double xbar[V][U], bound_bar[V], obar[V][D];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const double* gb = gbar + D * v;
        xbar[v][0] = 0.0;
        bound_bar[v] = 0.0;
#pragma unroll
        for (int a = 0; a < D; ++a) obar[v][a] = 0.0;
        if (last[v] < 0) {
#pragma unroll
            for (int a = 0; a < D; ++a) xbar[v][1 + a] = gb[a];
        } else if (zero[v]) {
#pragma unroll
            for (int a = 0; a < D; ++a) xbar[v][1 + a] = 0.0;
        } else {
            double g0[D];
#pragma unroll
            for (int a = 0; a < D; ++a) g0[a] = xs[v][1 + a];
            const double den = dot<D>(g0, offset[v]);
            const double sc = ((upper[v] ? hi[v] : lo[v]) - Wi[v]) / den;
            const double sbar = dot<D>(gb, g0);
            bound_bar[v] = sbar / den;
            Wibar[v] -= sbar / den;
            const double denbar = -sbar * sc / den;
#pragma unroll
            for (int a = 0; a < D; ++a) {
                xbar[v][1 + a] = sc * gb[a] + denbar * offset[v][a];
                obar[v][a] = denbar * g0[a];
            }
        }
    }
    // x = M^-1 b: b's bars M^-1 xbar; M's -sum_v bbar x^T
    double bbar[V][U], G[U][U];
#pragma unroll
    for (int v = 0; v < V; ++v) solve(xbar[v], bbar[v]);
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int q = 0; q < U; ++q) {
            double sum = 0.0;
#pragma unroll
            for (int v = 0; v < V; ++v) sum -= bbar[v][p] * xs[v][q];
            G[p][q] = sum;
        }
    // each entry's bars: M = sum w X X^T, b_v = sum w X (W_j - W_i), X = (1, d + c_j - c_i), w = |A|
    for (int k = first; k < end; ++k) {
        const int kk = k - first;
        int f, j;
        bool owned;
        double A[D], w, X[U];
        entry(k, f, j, owned, A, w, X);
        double Xbar[U], wbar = 0.0;
#pragma unroll
        for (int p = 0; p < U; ++p) {
            double sum = 0.0;
#pragma unroll
            for (int q = 0; q < U; ++q) {
                wbar += G[p][q] * X[p] * X[q];
                sum += (G[p][q] + G[q][p]) * X[q];
            }
            Xbar[p] = w * sum;
        }
        double* row = rows + static_cast<int64_t>(E) * kk;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const double dW = W[R * j + v] - Wi[v], xb = dot<U>(X, bbar[v]);
            wbar += xb * dW;
#pragma unroll
            for (int p = 0; p < U; ++p) Xbar[p] += w * bbar[v][p] * dW;
            Wibar[v] -= w * xb;
            double Wjbar = w * xb;
            if (last[v] >= 0 && !zero[v] && (upper[v] ? hi_k[v] : lo_k[v]) == kk) Wjbar += bound_bar[v];
            row[v] = Wjbar;
        }
        double dbar[D], xfbar[D];
#pragma unroll
        for (int a = 0; a < D; ++a) {
            dbar[a] = Xbar[1 + a];
            xfbar[a] = 0.0;
            cibar[a] -= Xbar[1 + a];
            row[V + D + a] = Xbar[1 + a];                                   // c_j
            row[V + 2 * D + a] = w > 0 ? wbar * A[a] / w : 0.0;              // A
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            if (last[v] != kk || zero[v]) continue;
#pragma unroll
            for (int a = 0; a < D; ++a) {
                xfbar[a] += obar[v][a];
                cibar[a] -= obar[v][a];
                if (!last_owned[v]) dbar[a] += obar[v][a];
            }
        }
#pragma unroll
        for (int a = 0; a < D; ++a) {
            row[V + a] = dbar[a];               // d
            row[V + 3 * D + a] = xfbar[a];      // x_f
        }
    }
}

template <int D>
__global__ void k_mv1_cells_adjoint(MeshDev<D> m, const double* __restrict__ W, const double* __restrict__ gb, const double* __restrict__ whb,
                                    const int32_t* __restrict__ angle_f, bool limit, bool steps_fixed, GasDev gas, double* __restrict__ Wb,
                                    double* __restrict__ cb, double* __restrict__ entry_bar, double* __restrict__ angle_Abar,
                                    double* __restrict__ angle_dbar) {
    constexpr int V = D + 2, R = V + 1, E = entry_width<D>();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double Wbar[V], cbar[D], wbar[D];
#pragma unroll
    for (int v = 0; v < V; ++v) Wbar[v] = Wb[V * i + v];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        cbar[a] = cb[D * i + a];
        wbar[a] = steps_fixed ? 0.0 : whb[D * i + a];
        angle_Abar[D * i + a] = angle_dbar[D * i + a] = 0;
    }
    // the point velocity (as the order-0 adjoint's cells)
    AngleFace<D> af;
    af.f = angle_f[i];
    double Wv[V], csv = W[R * i + V], cv[D], Av[D], dv[D];
#pragma unroll
    for (int v = 0; v < V; ++v) Wv[v] = W[R * i + v];
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
            cbar[s - V - 1] += bar;
        else if (s < V + 1 + 2 * D)
            angle_Abar[D * i + (s - V - 1 - D)] = bar;
        else
            angle_dbar[D * i + (s - V - 1 - 2 * D)] = bar;
    }
    for (int s = 0; s < V; ++s) {
        Dual Wd[V];
#pragma unroll
        for (int v = 0; v < V; ++v) Wd[v] = Dual(Wv[v], s == v ? 1.0 : 0.0);
        Wbar[s] += csbar * sound_t<Dual>(Wd, D + 1, gas.gamma).d;
    }
    // the fit's transpose: the cell's W and c, and every entry's row (W_j, d, c_j, A, x_f)
    double gbv[V * D];
#pragma unroll
    for (int c = 0; c < V * D; ++c) gbv[c] = gb[V * D * static_cast<int64_t>(i) + c];
    fit_gradient_adjoint<D>(m, i, W, limit, gbv, Wbar, cbar, entry_bar + static_cast<int64_t>(E) * m.start[i]);
#pragma unroll
    for (int v = 0; v < V; ++v) Wb[V * i + v] = Wbar[v];
#pragma unroll
    for (int a = 0; a < D; ++a) cb[D * i + a] = cbar[a];
}

// The list position of face f in cell i's list (entry_of, :2622-2626).
template <int D>
__device__ __forceinline__ int entry_of(const MeshDev<D>& m, int i, int f) {
    for (int k = m.start[i]; k < m.start[i + 1]; ++k)
        if (list_face(m.list[k]) == f) return k;
    return -1;
}

// Per cell at t^n (moving_gather_adjoint_1, :3106-3140): the W bars the neighbours' fits hold for it, then the primitives'
// adjoint into Q's bar (added) and V's bar (written); c's bar (written) and x's (added) from its own and its neighbours'
// entries (the separations, the neighbours' centroids, the offsets off the owner) and the angle faces.
template <int D>
__global__ void k_mv1_gather_adjoint(MeshDev<D> m, const double* __restrict__ q, const double* __restrict__ Wb, const double* __restrict__ cb,
                                     const double* __restrict__ entry_bar, const int32_t* __restrict__ angle_f,
                                     const double* __restrict__ angle_dbar, GasDev gas, double* __restrict__ qbar, double* __restrict__ Vbar,
                                     double* __restrict__ cbar_out, double* __restrict__ xb) {
    constexpr int V = D + 2, E = entry_width<D>();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double Wbar[V], cbar[D], xsum[D];
#pragma unroll
    for (int v = 0; v < V; ++v) Wbar[v] = Wb[V * i + v];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        cbar[a] = cb[D * i + a];
        xsum[a] = -angle_dbar[D * i + a];
    }
    for (int k = m.start[i]; k < m.start[i + 1]; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e), j = e >= 0 ? m.neighbour[f] : m.owner[f];
        const int kj = entry_of<D>(m, j, f);
        const double* own = entry_bar + static_cast<int64_t>(E) * k;
        const double* mirror = entry_bar + static_cast<int64_t>(E) * kj;
#pragma unroll
        for (int v = 0; v < V; ++v) Wbar[v] += mirror[v];  // j's fit reads W_i
#pragma unroll
        for (int a = 0; a < D; ++a) {
            xsum[a] += -own[V + a] + mirror[V + a];  // d = x_j - x_i here, x_i - x_j in j's fit
            cbar[a] += mirror[V + D + a];           // j's fit reads c_i as its neighbour's centroid
        }
        if (angle_f[j] == f)
#pragma unroll
            for (int a = 0; a < D; ++a) xsum[a] += angle_dbar[D * j + a];
    }
    const double inv = 1.0 / m.vol[i];
    double Uv[V];
#pragma unroll
    for (int v = 0; v < V; ++v) Uv[v] = q[V * i + v] * inv;
    double vb = 0;
    for (int s = 0; s < V; ++s) {
        Dual U[V], Wd[V];
#pragma unroll
        for (int v = 0; v < V; ++v) U[v] = Dual(Uv[v], s == v ? 1.0 : 0.0);
        primitive_t<D, Dual>(U, gas, Wd);
        double bar = 0;
#pragma unroll
        for (int v = 0; v < V; ++v) bar += Wbar[v] * Wd[v].d;
        qbar[V * i + s] += bar * inv;
        vb -= bar * Uv[s] * inv;
    }
    Vbar[i] = vb;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        cbar_out[D * i + a] = cbar[a];
        xb[D * i + a] += xsum[a];
    }
}

// Per face at t^n (moving_faces_bar_1, :3141-3153): A's bar from both cells' fit entries and angle faces, x_f's from the fit
// entries, added to the passes'.
template <int D>
__global__ void k_mv1_faces_bar(MeshDev<D> m, const double* __restrict__ entry_bar, const int32_t* __restrict__ angle_f,
                                const double* __restrict__ angle_Abar, double* __restrict__ Abar, double* __restrict__ xfbar) {
    constexpr int V = D + 2, E = entry_width<D>();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.f) return;
    const int o = m.owner[f], j = m.neighbour[f];
    const int ko = entry_of<D>(m, o, f), kj = entry_of<D>(m, j, f);
    const double* ro = entry_bar + static_cast<int64_t>(E) * ko;
    const double* rj = entry_bar + static_cast<int64_t>(E) * kj;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        Abar[D * f + a] += ro[V + 2 * D + a] + rj[V + 2 * D + a] + (angle_f[o] == f ? angle_Abar[D * o + a] : 0.0) +
                           (angle_f[j] == f ? angle_Abar[D * j + a] : 0.0);
        xfbar[D * f + a] += ro[V + 3 * D + a] + rj[V + 3 * D + a];
    }
}

}  // namespace mvd
}  // namespace luna
