// The 1D solver's stencil (src/hydro/finite_volume_1d.hpp, Stencil :70-329 and Kernel::face_state :492-506), shared by
// the static line (line.cu) and the moving line (moving_line.cu): the line's slots with their gaps, volumes and centroid
// offsets, the five-cell load with ghosts behind walls, the limited slopes, the face states and the flux.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "kernels.cuh"
#include "luna_b200.h"

namespace {

constexpr int V1 = 3;  // rho, rho v, E

struct LineDev {
    int n, lines, periodic, order, limiter, riemann;
    int wall[2];
    double inflow[2][3];
    double step;
    const double* __restrict__ gap;       // [n + 1]: gap[s + 1] from slot s to s + 1 in grid steps; gap[0], gap[n] over the ends
    const double* __restrict__ volume;    // [n]
    const double* __restrict__ centroid;  // [n]: the centroid's offset from the generator
    luna::GasDev gas;
};

struct Cell1 {
    double W[3], c;
    bool real;
};

__device__ __forceinline__ int slot_at(const LineDev& L, int s, int k) {
    const int t = s + k;
    if (L.periodic) return t < 0 ? t + L.n : t >= L.n ? t - L.n : t;
    return t >= 0 && t < L.n ? t : -1;
}

__device__ __forceinline__ void primitive_of(const LineDev& L, const double* q, int s, double* W) {
    const double inv = 1.0 / L.volume[s];
    double U[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) U[v] = q[3 * s + v] * inv;
    luna::primitive<1>(U, L.gas, W);
}

// Stencil::ghost (finite_volume_1d.hpp:117-122): behind a wall, next to an end cell of state W.
__device__ __forceinline__ void ghost(const LineDev& L, const double* W, bool left, double* out) {
    const int wall = L.wall[left ? 0 : 1];
    if (wall == LUNA_WALL_REFLECTIVE) {
        out[0] = W[0];
        out[1] = -W[1];
        out[2] = W[2];
    } else if (wall == LUNA_WALL_INFLOW) {
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = L.inflow[left ? 0 : 1][v];
    } else {
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = W[v];
    }
}
// Stencil::ghost_face (:124-128).
__device__ __forceinline__ void ghost_face(const LineDev& L, const double* Wf, const double* W, bool left, double* out) {
    if (L.wall[left ? 0 : 1] == LUNA_WALL_REFLECTIVE) {
        out[0] = Wf[0];
        out[1] = -Wf[1];
        out[2] = Wf[2];
    } else {
        ghost(L, W, left, out);
    }
}

// Stencil::load<2> (:132-156): cells s - 2 .. s + 2 (a ghost next to an end cell behind a wall), the distances between
// their generators.
__device__ __forceinline__ void load(const LineDev& L, const double* q, int s, Cell1 (&cell)[5], double (&gap)[4]) {
    int slot[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        slot[k] = slot_at(L, s, k - 2);
        cell[k].real = slot[k] >= 0;
        cell[k].c = 0;
#pragma unroll
        for (int v = 0; v < 3; ++v) cell[k].W[v] = 0;
        if (slot[k] >= 0) {
            primitive_of(L, q, slot[k], cell[k].W);
            cell[k].c = L.centroid[slot[k]];
        }
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        if (slot[k] >= 0) continue;
        const int end = k < 2 ? k + 1 : k - 1;
        if (slot[end] < 0) continue;
        ghost(L, cell[end].W, k < 2, cell[k].W);
        cell[k].c = -cell[end].c;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int a = slot[k], b = slot[k + 1];
        gap[k] = a >= 0 ? L.gap[a + 1] * L.step : b >= 0 ? L.gap[0] * L.step : 0.0;
    }
}

// Stencil::gradient (:183-207): the limited slope of variable v of *cell between its neighbours.
__device__ __forceinline__ double gradient(const LineDev& L, const Cell1* cell, double gapL, double gapR, int v) {
    const Cell1& me = *cell;
    const double dL = -gapL + cell[-1].c - me.c, dR = gapR + cell[1].c - me.c;
    const double Wi = me.W[v], left = cell[-1].W[v], right = cell[1].W[v];
    if (L.limiter == LUNA_LIMITER_MINMOD || L.limiter == LUNA_LIMITER_VAN_LEER) {
        const double sL = (left - Wi) / dL, sR = (right - Wi) / dR;
        if (!(sL * sR > 0)) return 0.0;
        if (L.limiter == LUNA_LIMITER_VAN_LEER) return 2 * sL * sR / (sL + sR);
        return fabs(sL) < fabs(sR) ? sL : sR;
    }
    double g = ((right - Wi) - (left - Wi)) / (dR - dL);
    if (L.limiter == LUNA_LIMITER_NONE) return g;
    const double r[2] = {-0.5 * gapL - me.c, 0.5 * gapR - me.c};
    const double lo = fmin(left, right), hi = fmax(left, right);
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        const double dp = g * r[f];
        if (dp > 0 && Wi + dp > hi)
            g = g * (hi > Wi ? (hi - Wi) / dp : 0.0);
        else if (dp < 0 && Wi + dp < lo)
            g = g * (lo < Wi ? (lo - Wi) / dp : 0.0);
    }
    return g;
}

// Kernel::face_state (:492-506): half a step on, to the face at offset r; the cell's W if rho or P would not stay positive.
template <int Order>
__device__ __forceinline__ void face_state(const LineDev& L, const double* W, const double* g, double r, double dt, double* out) {
    if constexpr (Order == 0) {
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = W[v];
    } else {
        double A[3];
        luna::half_step_rate<1, double>(W, g, L.gas.gamma, A);
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = W[v] - 0.5 * dt * A[v];
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] += g[v] * r;
        if (out[0] > 0 && out[2] > 0) return;
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = W[v];
    }
}

__device__ __forceinline__ void line_flux(const LineDev& L, const double* Wl, const double* Wr, double* F) {
    const double n[1] = {1.0}, w[1] = {0.0};
    if (L.riemann == LUNA_HLL)
        luna::hll_flux<1>(Wl, Wr, n, w, L.gas, F, false);
    else
        luna::hllc_flux<1, double>(Wl, Wr, n, w, L.gas.gamma, L.gas.inverse_gm1, F, false);
}

}  // namespace
