// The 1D solver on a moving line: hydro::FiniteVolume<1> with Motion::moving (src/hydro/finite_volume_1d.hpp) on the GPU.
//
// Layout: the line's slots (its generators sorted along it) hold everything: Q [slots][3], the positions x, the grid
// keys and each slot's cell id (the caller's cell order, cells from the walls appended); the slots' gaps, volumes and
// centroid offsets follow from the keys (the step writes the next ones beside its update; after a re-sort or new cells,
// k_mline_geometry). A step is one launch and one pinned read of its counters (the next dt, the slots out of order, the
// error word, the end slots' wishes), as the reference reads its dt and order check. One thread per slot does what the
// reference's Kernel::body does for a moving line (:552-660): the five-cell stencil, the slopes and point velocities of
// s - 1, s, s + 1, their new keys (each point moves by whole grid steps), the two faces' fluxes on the meshes of t^n and
// t^n+1 in the frame of the face's move (each computed once, shared through the block), the update and the slot's next
// position and key; the fused variant also reduces the next dt of LUNA's rule and counts the slots out of order. When
// points cross, the slots re-sort by (key, cell) (CUB's
// radix sort, then one gather of every slot array). Cells from the walls (supply_cells) are decided on the host from the
// two end slots, as the reference does, and inserted by one kernel that shifts the slot arrays.
//
// This object is compiled without multiply-add contraction (the reference's operation order; explicit fma where it calls
// Kokkos::fma): a point's grid step depends on the last bit of its velocity.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "line_stencil.cuh"
#include "luna_b200.h"

namespace luna {
luna_status report_error(luna_status s, const std::string& what);
}  // namespace luna

namespace {

luna_status mfail(luna_status s, const std::string& what) { return luna::report_error(s, what); }

#define MLINE_CUDA(call)                                                                                     \
    do {                                                                                                     \
        const cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return mfail(LUNA_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr double kShapingSpeed = 0.5;  // FiniteVolume<1>::cell_shaping_speed (finite_volume_1d.hpp:26)

// What the moving kernels read beyond the stencil's LineDev.
struct MovingDev {
    const int64_t* __restrict__ keys;  // [slots]
    const int* __restrict__ cell;      // [slots]: the slot's cell id
    const double* __restrict__ x;      // [slots]
    double* __restrict__ x_next;       // [slots]
    int64_t* __restrict__ keys_next;   // [slots]
    double* __restrict__ gap_next;     // [slots + 1]: the next step's geometry, from the new keys
    double* __restrict__ volume_next;  // [slots]
    double* __restrict__ centroid_next;  // [slots]
    double length, spacing;
    int64_t period;
    int regularise, supply[2];
};

// sorted_mesh::snap: the grid point nearest y (ties to even); periodic: modulo the period, else within [0, period].
__device__ __forceinline__ int64_t snap(const LineDev& L, const MovingDev& M, double y) {
    int64_t k = static_cast<int64_t>(nearbyint(y / L.step));
    if (L.periodic) {
        k %= M.period;
        if (k < 0) k += M.period;
    } else {
        k = k < 0 ? 0 : k > M.period ? M.period : k;
    }
    return k;
}
// sorted_mesh::before: the slots' order, by key, then by cell.
__device__ __forceinline__ bool before(int64_t ka, int ia, int64_t kb, int ib) { return ka < kb || (ka == kb && ia < ib); }

__device__ __forceinline__ double sound1(const LineDev& L, const double* W) { return sqrt(L.gas.gamma * W[2] / W[0]); }

// Stencil::drift (:301-316): AREPO-ng's regularisation, the point velocity's difference from the fluid's.
__device__ __forceinline__ double drift(const LineDev& L, const MovingDev& M, const double* W, double g, double c, double volume) {
    const double r = 0.5 * volume;
    if (!M.regularise || fabs(c) <= 0.5 * r) return 0.0;
    double offset = c;
    const double dgrad = fabs(g);
    if (dgrad > 0) {
        const double tmp = 3 * r + W[0] / dgrad;
        const double x = (tmp - sqrt(tmp * tmp - 8 * r * r)) / 4;
        if (x < 0.25 * r) offset += x / dgrad * g;
    }
    const double d = fabs(offset);
    if (d <= 0.75 * r) return 0.0;
    const double fraction = d > r ? kShapingSpeed : kShapingSpeed * (d - 0.75 * r) / (0.25 * r);
    return offset * (fraction * sound1(L, W) / d);
}
// Stencil::point_velocity (:320-329): drift(), plus, for a generator beyond 0.75 r of its centroid, up to the fluid's
// velocity at the generator, linear between the centroids of this cell and its neighbour there (luna-cpp #25).
__device__ __forceinline__ double point_velocity(const LineDev& L, const MovingDev& M, const Cell1* cell, double gapL, double gapR,
                                                 double g_rho, double volume) {
    const Cell1& me = *cell;
    const double r = 0.5 * volume, d = fabs(me.c), weight = fmin(1.0, (d - 0.75 * r) / (0.25 * r));
    const double drifting = drift(L, M, me.W, g_rho, me.c, volume);
    if (!(weight > 0)) return drifting;
    const int side = me.c < 0 ? 1 : -1;
    const double between = side > 0 ? gapR + cell[1].c - me.c : gapL + me.c - cell[-1].c;
    return drifting + weight * (cell[side].W[1] - me.W[1]) * (d / between);
}
// Stencil::wants_cell (:88-98): 0..2 cells an end slot asks its wall for.
__device__ __forceinline__ int wants_cell(const LineDev& L, const MovingDev& M, int s) {
    int wants = 0;
    if (s == 0 && M.supply[0])
        wants += L.volume[0] > 2 * M.spacing && static_cast<double>(M.keys[0]) * L.step >= 1.5 * M.spacing;
    if (s == L.n - 1 && M.supply[1])
        wants += L.volume[s] > 2 * M.spacing && static_cast<double>(M.period - M.keys[s]) * L.step >= 1.5 * M.spacing;
    return wants;
}
// Kernel::extrapolated (:507-523): W + g r, a whole step on (MUSCL-Hancock) when second; W if rho or P would not stay
// positive.
template <int Order>
__device__ __forceinline__ void extrapolated(const LineDev& L, const double* W, const double* g, double r, int second, double dt, double* out) {
    if constexpr (Order == 0) {
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = W[v];
    } else {
        if (second) {
            double A[3];
            luna::half_step_rate<1, double>(W, g, L.gas.gamma, A);
            const double whole = 2 * dt;
#pragma unroll
            for (int v = 0; v < 3; ++v) out[v] = W[v] - 0.5 * whole * A[v];
        } else {
#pragma unroll
            for (int v = 0; v < 3; ++v) out[v] = W[v];
        }
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] += g[v] * r;
        if (out[0] > 0 && out[2] > 0) return;
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = W[v];
    }
}
// Kernel::moved (:546-550): where a point at x0 ends up after dt.
__device__ __forceinline__ double moved(const LineDev& L, const MovingDev& M, double x0, double velocity, double dt) {
    const double side = M.length;
    const double y = fma(dt, velocity, x0);
    return L.periodic ? y - side * floor(y / side) : fmin(fmax(y, 0.0), side);
}
// Riemann::flux(L, R, n = 1, w) through a face moving at w, back in the lab frame.
__device__ __forceinline__ void moving_flux(const LineDev& L, const double* Wl, const double* Wr, double w, double* F) {
    const double n[1] = {1.0}, wv[1] = {w};
    if (L.riemann == LUNA_HLL)
        luna::hll_flux<1>(Wl, Wr, n, wv, L.gas, F, true);
    else
        luna::hllc_flux<1, double>(Wl, Wr, n, wv, L.gas.gamma, L.gas.inverse_gm1, F, true);
}

// What one launch hands back, in one read: the next dt's bits (the Min reducer), the error word, the slots out of order
// and the end slots' wishes for a cell. Two of them alternate: each launch zeroes the other for the next one.
struct Counters {
    unsigned long long dt_bits, error;
    int descents, wants;
};
__device__ __forceinline__ void reset_spare(Counters* spare) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        spare->dt_bits = 0x7fefffffffffffffull;  // DBL_MAX, the Min reducer's identity
        spare->error = 0;
        spare->descents = 0;
        spare->wants = 0;
    }
}

constexpr int kLineBlock = 128;

// Kernel::body, moving (:552-660), one thread per slot, a block sharing what the reference computes per slot three times
// (the slope, point velocity and new key of s - 1, s, s + 1) and twice (each face's flux): each thread computes them for
// its own slot (the block's first and last slots also for their outer neighbours) and the flux of its right face (the
// first slot also its left one), and reads the rest from shared memory; the same operations on the same operands, so
// the same bits as the per-slot body. Writes the slot's next Q, position, key and geometry; counts the slots out of
// order against their right neighbour; Fused: the next dt of LUNA's rule with the volume of the new keys and |w - v| of
// t^n (:632-658) into dt_bits, and with `watching` the end slots' wishes for a cell (the line before the step).
template <int Order, bool Fused>
__global__ void __launch_bounds__(kLineBlock) k_mline_step(LineDev L, MovingDev M, const double* __restrict__ q, double* __restrict__ next, double dt,
                                                           double courant, int watching, Counters* __restrict__ use, Counters* __restrict__ spare) {
    __shared__ double s_grad[kLineBlock][3], s_point[kLineBlock], s_moves[kLineBlock], s_F[kLineBlock][3];
    __shared__ long long s_key[kLineBlock];
    const int t = threadIdx.x, s = blockIdx.x * blockDim.x + t;
    reset_spare(spare);
    const bool active = s < L.n;
    const bool last = active && (t == blockDim.x - 1 || s == L.n - 1);
    double smallest = 1.0e300;
    Cell1 cell[5];
    double gap[4], grad[5][3], point[5] = {0, 0, 0, 0, 0}, moves[5] = {0, 0, 0, 0, 0};
    int64_t key[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int v = 0; v < 3; ++v) grad[k][v] = 0;
    if (active) {
        load(L, q, s, cell, gap);
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
            if (!(k == 2 || (k == 1 && t == 0) || (k == 3 && last)) || !cell[k].real) continue;
            if constexpr (Order == 1)
#pragma unroll
                for (int v = 0; v < 3; ++v) grad[k][v] = gradient(L, cell + k, gap[k - 1], gap[k], v);
            point[k] = cell[k].W[1] + point_velocity(L, M, cell + k, gap[k - 1], gap[k], grad[k][0], 0.5 * (gap[k - 1] + gap[k]));
            const int u = slot_at(L, s, k - 2);
            key[k] = snap(L, M, moved(L, M, M.x[u], point[k], dt));
            int64_t d = key[k] - M.keys[u];
            if (L.periodic) d = d > M.period / 2 ? d - M.period : d < -M.period / 2 ? d + M.period : d;
            moves[k] = static_cast<double>(d);
        }
#pragma unroll
        for (int v = 0; v < 3; ++v) s_grad[t][v] = grad[2][v];
        s_point[t] = point[2];
        s_moves[t] = moves[2];
        s_key[t] = key[2];
    }
    __syncthreads();
    // the flux through the face between stencil cells a and b = a + 1, positive along +x
    const auto face = [&](int a, double (&F)[3]) {
        const int b = a + 1;
        // a wall's face is static; between cells the face moves by the mean of its generators' moves
        const bool inside = cell[a].real && cell[b].real;
        const double travel = inside ? 0.5 * (moves[a] + moves[b]) * L.step : 0.0;
        const double w = travel / dt;
        const double ra = 0.5 * gap[a] - cell[a].c, rb = -0.5 * gap[a] - cell[b].c;
        double pass[2][3];
#pragma unroll
        for (int second = 0; second < (Order == 1 ? 2 : 1); ++second) {
            double Wl[3] = {0, 0, 0}, Wr[3] = {0, 0, 0};
            if (cell[a].real) extrapolated<Order>(L, cell[a].W, grad[a], ra + second * travel, second, dt, Wl);
            if (cell[b].real) extrapolated<Order>(L, cell[b].W, grad[b], rb + second * travel, second, dt, Wr);
            if (!cell[a].real) ghost_face(L, Wr, cell[b].W, true, Wl);
            if (!cell[b].real) ghost_face(L, Wl, cell[a].W, false, Wr);
            moving_flux(L, Wl, Wr, w, pass[second]);
        }
#pragma unroll
        for (int v = 0; v < 3; ++v) F[v] = Order == 1 ? 0.5 * (pass[0][v] + pass[1][v]) : pass[0][v];
    };
    double F[2][3];
    if (active) {
        if (!last) {  // the right neighbour's from its thread
#pragma unroll
            for (int v = 0; v < 3; ++v) grad[3][v] = cell[3].real ? s_grad[t + 1][v] : 0.0;
            point[3] = cell[3].real ? s_point[t + 1] : 0.0;
            moves[3] = cell[3].real ? s_moves[t + 1] : 0.0;
            key[3] = cell[3].real ? s_key[t + 1] : 0;
        }
        face(2, F[1]);
#pragma unroll
        for (int v = 0; v < 3; ++v) s_F[t][v] = F[1][v];
        if (t == 0) face(1, F[0]);
    }
    __syncthreads();
    if (active) {
        if (t > 0) {
#pragma unroll
            for (int v = 0; v < 3; ++v) F[0][v] = s_F[t - 1][v];
            key[1] = cell[1].real ? s_key[t - 1] : 0;
        }
        double U[3];
        bool finite = true;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            U[v] = q[3 * s + v] - dt * (F[1][v] - F[0][v]);
            next[3 * s + v] = U[v];
            finite = finite && isfinite(U[v]);
        }
        if (!finite) atomicOr(&use->error, 2ull);
        M.x_next[s] = moved(L, M, M.x[s], point[2], dt);
        M.keys_next[s] = key[2];
        const int i = M.cell[s];
        double left, right;
        if (cell[1].real) {
            const int64_t d = key[2] - key[1];
            left = static_cast<double>(d < 0 && L.periodic ? d + M.period : d);
        } else {
            left = static_cast<double>(2 * key[2]);
        }
        if (cell[3].real) {
            const int u = slot_at(L, s, 1);
            const int64_t d = key[3] - key[2];
            right = static_cast<double>(d < 0 && L.periodic ? d + M.period : d);
            if (!before(key[2], i, key[3], M.cell[u])) atomicAdd(&use->descents, 1);
        } else {
            right = static_cast<double>(2 * (M.period - key[2]));
        }
        // the next step's geometry from the new keys (k_mline_geometry's, as long as the slots stay in order)
        M.gap_next[s + 1] = right;
        if (s == 0) M.gap_next[0] = left;
        M.volume_next[s] = (left + right) * (0.5 * L.step);
        M.centroid_next[s] = (right - left) * (0.25 * L.step);
        if constexpr (Fused) {
            const double volume = (left + right) * (0.5 * L.step), inv = 1.0 / volume;
            double Un[3], Wn[3];
#pragma unroll
            for (int v = 0; v < 3; ++v) Un[v] = U[v] * inv;
            luna::primitive<1>(Un, L.gas, Wn);
            const double relative = fabs(point[2] - cell[2].W[1]);
            smallest = courant * volume / (relative + sound1(L, Wn));
            if (!(smallest == smallest)) atomicOr(&use->error, 1ull);
            if (watching && (s == 0 || s == L.n - 1)) {
                const int wants = wants_cell(L, M, s);
                if (wants) atomicAdd(&use->wants, wants);
            }
        }
    }
    if constexpr (Fused) luna::block_min_to(smallest, &use->dt_bits);
}

// time_step (:332-384), moving: per slot the point velocity's |w - v| (order 1: with the limited density slope) in place
// of |v|; LUNA's rule (Rule 1) courant V / (|w - v| + c), AREPO's (Rule 0) the smallest of r / (c + |w - v|) and, per
// side, (distance + r) / vsig. With `watching`, the end slots' wishes for a cell.
template <int Order, int Rule>
__global__ void __launch_bounds__(128) k_mline_time_step(LineDev L, MovingDev M, const double* __restrict__ q, double courant, int watching,
                                                         Counters* __restrict__ use, Counters* __restrict__ spare) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    reset_spare(spare);
    double smallest = 1.0e300;
    if (s < L.n) {
        Cell1 cell[5];
        double gap[4];
        load(L, q, s, cell, gap);  // load<1>'s cells and gaps are cell[1..3], gap[1..2]
        const double* Wi = cell[2].W;
        const double ci = sound1(L, Wi);
        const double volume = L.volume[s];
        const double g = Order == 1 ? gradient(L, cell + 2, gap[1], gap[2], 0) : 0.0;
        const double vi = fabs(point_velocity(L, M, cell + 2, gap[1], gap[2], g, volume));
        if (watching && (s == 0 || s == L.n - 1)) {
            const int wants = wants_cell(L, M, s);
            if (wants) atomicAdd(&use->wants, wants);
        }
        if constexpr (Rule == 1) {
            smallest = courant * volume / (vi + ci);
        } else {
            const double r = 0.5 * volume;
            double step = r / (ci + vi);
#pragma unroll
            for (int side = -1; side <= 1; side += 2) {
                const int t = slot_at(L, s, side);
                double Wj[3];
                if (t >= 0)
                    primitive_of(L, q, t, Wj);
                else
                    ghost(L, Wi, side < 0, Wj);
                const double dist = (side < 0 ? L.gap[s] : L.gap[s + 1]) * L.step;
                const double vsig = ci + sound1(L, Wj) - (Wj[1] - Wi[1]) * side;
                if (vsig > 0) step = fmin(step, (dist + r) / vsig);
            }
            smallest = courant * step;
        }
        if (!(smallest == smallest)) atomicOr(&use->error, 1ull);
    }
    luna::block_min_to(smallest, &use->dt_bits);
}

// Line::gap, volume, centroid from the keys (load_inner :163-176): between neighbours the key difference (a periodic
// line's seam wraps), at a wall twice the end generator's distance to it.
__global__ void k_mline_geometry(int n, int periodic, int64_t period, double step, const int64_t* __restrict__ keys, double* __restrict__ gap,
                                 double* __restrict__ volume, double* __restrict__ centroid) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const auto after = [&](int t) {  // the gap after slot t, t = -1 .. n - 1, in grid steps
        if (t >= 0 && t + 1 < n) {
            int64_t d = keys[t + 1] - keys[t];
            if (d < 0 && periodic) d += period;
            return static_cast<double>(d);
        }
        if (periodic) {
            int64_t d = keys[0] - keys[n - 1];
            if (d < 0) d += period;
            return static_cast<double>(d);
        }
        return t < 0 ? static_cast<double>(2 * keys[0]) : static_cast<double>(2 * (period - keys[n - 1]));
    };
    const double gl = after(s - 1), gr = after(s);
    gap[s + 1] = gr;
    if (s == 0) gap[0] = gl;
    volume[s] = (gl + gr) * (0.5 * step);
    centroid[s] = (gr - gl) * (0.25 * step);
}

// The sort's two stable passes (by cell, then by key): the cells of the slots as keys; then the keys of the slots in
// the first pass's order.
__global__ void k_mline_sort_cells(int n, const int* __restrict__ cell, unsigned int* __restrict__ by_cell, int* __restrict__ slot) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    by_cell[s] = static_cast<unsigned int>(cell[s]);
    slot[s] = s;
}
__global__ void k_mline_sort_keys(int n, const int64_t* __restrict__ keys, const int* __restrict__ slot, unsigned long long* __restrict__ by_key) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    by_key[t] = static_cast<unsigned long long>(keys[slot[t]]);
}
// Every slot array gathered by the sorted permutation.
__global__ void k_mline_gather(int n, const int* __restrict__ from, const double* __restrict__ q, const double* __restrict__ x,
                               const int64_t* __restrict__ keys, const int* __restrict__ cell, double* __restrict__ q_out, double* __restrict__ x_out,
                               int64_t* __restrict__ keys_out, int* __restrict__ cell_out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int t = from[s];
#pragma unroll
    for (int v = 0; v < 3; ++v) q_out[3 * s + v] = q[3 * t + v];
    x_out[s] = x[t];
    keys_out[s] = keys[t];
    cell_out[s] = cell[t];
}

// The two end slots as supply_cells reads them (:424-431): keys of the two slots at each end, the end cells' volumes and
// velocities.
struct Ends {
    long long k0, k1, kb, kl;
    double v0, vl, volume0, volumel;
};
__global__ void k_mline_ends(LineDev L, const int64_t* __restrict__ keys, const double* __restrict__ q, Ends* __restrict__ out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int n = L.n, last = n - 1;
    double W[3];
    Ends e;
    e.k0 = keys[0];
    e.k1 = n > 1 ? keys[1] : 0;
    e.kb = n > 1 ? keys[last - 1] : 0;
    e.kl = keys[last];
    primitive_of(L, q, 0, W);
    e.v0 = W[1];
    primitive_of(L, q, last, W);
    e.vl = W[1];
    e.volume0 = L.volume[0];
    e.volumel = L.volume[last];
    *out = e;
}

// mesh_->insert + the split (:441-468): the slot arrays shifted by one when a cell enters at the left; each new cell takes
// `fraction` of its old neighbour's Q. Slot t of the new line from the old arrays.
struct Insert {
    int left, right, cell_left, cell_right;
    double fraction_left, fraction_right, x_left, x_right;
    long long key_left, key_right;
};
__global__ void k_mline_insert(int n_old, Insert in, const double* __restrict__ q, const double* __restrict__ x, const int64_t* __restrict__ keys,
                               const int* __restrict__ cell, double* __restrict__ q_out, double* __restrict__ x_out, int64_t* __restrict__ keys_out,
                               int* __restrict__ cell_out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_new = n_old + in.left + in.right;
    if (t >= n_new) return;
    if (in.left && t == 0) {
#pragma unroll
        for (int v = 0; v < 3; ++v) q_out[v] = in.fraction_left * q[v];
        x_out[0] = in.x_left;
        keys_out[0] = in.key_left;
        cell_out[0] = in.cell_left;
        return;
    }
    if (in.right && t == n_new - 1) {
        const int last = n_old - 1;
#pragma unroll
        for (int v = 0; v < 3; ++v) q_out[3 * t + v] = in.fraction_right * q[3 * last + v];
        x_out[t] = in.x_right;
        keys_out[t] = in.key_right;
        cell_out[t] = in.cell_right;
        return;
    }
    const int s = t - in.left;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        double value = q[3 * s + v];
        if (in.left && s == 0) value -= in.fraction_left * q[v];
        if (in.right && s == n_old - 1) value -= in.fraction_right * q[3 * s + v];
        q_out[3 * t + v] = value;
    }
    x_out[t] = x[s];
    keys_out[t] = keys[s];
    cell_out[t] = cell[s];
}

// Caller cell order <-> slot order: to[s] = from[cell[s]] (gather) or to[cell[s]] = from[s], `width` doubles a row.
template <bool Gather>
__global__ void k_mline_permute(int n, int width, const int* __restrict__ cell, const double* __restrict__ from, double* __restrict__ to) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int i = cell[s];
    for (int v = 0; v < width; ++v) {
        if (Gather)
            to[width * s + v] = from[width * i + v];
        else
            to[width * i + v] = from[width * s + v];
    }
}

template <class T>
struct DevBuffer {
    T* ptr = nullptr;
    size_t count = 0;
    DevBuffer() = default;
    DevBuffer(const DevBuffer&) = delete;
    DevBuffer& operator=(const DevBuffer&) = delete;
    ~DevBuffer() {
        if (ptr) cudaFree(ptr);
    }
    void swap(DevBuffer& other) {
        std::swap(ptr, other.ptr);
        std::swap(count, other.count);
    }
    luna_status alloc(size_t n, const char* what) {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
        const cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();
            return mfail(e == cudaErrorMemoryAllocation ? LUNA_ENOMEM : LUNA_ECUDA, std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
        }
        count = n;
        return LUNA_OK;
    }
};

unsigned int blocks_of(int64_t n) { return static_cast<unsigned int>((std::max<int64_t>(n, 1) + 127) / 128); }

}  // namespace

struct luna_mline {
    ~luna_mline() {
        if (host_counters) cudaFreeHost(host_counters);
    }
    LineDev dev{};
    MovingDev mdev{};
    int n = 0, cap = 0, order = 1;
    double length = 0, step = 0;
    int64_t period = int64_t(1) << 52;  // the 1D mesh's grid: 2^52 steps (research_notes/stage1_1d_2026-11-04.md:35)
    cudaStream_t stream = nullptr;
    // slot arrays and their spares (the step's outputs, the sort's and the insertion's targets)
    DevBuffer<double> q, q2, x, x2, gap, volume, centroid, gap2, volume2, centroid2, staging;
    DevBuffer<int64_t> keys, keys2;
    DevBuffer<int> cell, cell2, slot, slot2;
    DevBuffer<unsigned long long> composite, composite2;
    DevBuffer<unsigned int> by_cell, by_cell2;
    DevBuffer<Counters> counters;  // two, alternating
    Counters* host_counters = nullptr;  // pinned
    int epoch = 0;
    DevBuffer<unsigned char> sort_temp;
    DevBuffer<Ends> ends;
    // supply_cells' bookkeeping (:924-1000)
    bool supply[2] = {false, false}, watching = false, looked = false;
    double spacing = 0;
    int wants = 0, until_look = 0;
    int64_t added = 0, sorts = 0, updates = 0;

    void bind() {
        dev.n = n;
        dev.gap = gap.ptr;
        dev.volume = volume.ptr;
        dev.centroid = centroid.ptr;
        mdev.keys = keys.ptr;
        mdev.cell = cell.ptr;
        mdev.x = x.ptr;
        mdev.x_next = x2.ptr;
        mdev.keys_next = keys2.ptr;
        mdev.gap_next = gap2.ptr;
        mdev.volume_next = volume2.ptr;
        mdev.centroid_next = centroid2.ptr;
        mdev.spacing = spacing;
        mdev.supply[0] = supply[0];
        mdev.supply[1] = supply[1];
    }
    luna_status geometry() {
        k_mline_geometry<<<blocks_of(n), 128, 0, stream>>>(n, dev.periodic, period, step, keys.ptr, gap.ptr, volume.ptr, centroid.ptr);
        MLINE_CUDA(cudaGetLastError());
        return LUNA_OK;
    }
    // Room for `count` slots, by a quarter more when full (reserve_cells :967-983); the slot arrays keep their rows.
    luna_status reserve(int count) {
        if (count <= cap) return LUNA_OK;
        // the sort's first pass takes 31 bits of a cell id
        if (count >= (1 << 30)) return mfail(LUNA_EINVAL, "the moving line holds fewer than 2^30 cells");
        const int grown = std::max(count, cap + cap / 4);
        MLINE_CUDA(cudaStreamSynchronize(stream));  // the rows to keep are final before they are copied
        luna_status st = LUNA_OK;
        const auto grow = [&](auto& buffer, size_t width, const char* what) {
            using T = std::remove_pointer_t<decltype(buffer.ptr)>;
            if (st != LUNA_OK) return;
            DevBuffer<T> fresh;
            st = fresh.alloc(static_cast<size_t>(grown) * width, what);
            if (st != LUNA_OK) return;
            if (buffer.ptr && n > 0) {
                const cudaError_t e = cudaMemcpy(fresh.ptr, buffer.ptr, sizeof(T) * width * n, cudaMemcpyDeviceToDevice);
                if (e != cudaSuccess) st = mfail(LUNA_ECUDA, std::string("reserve: ") + cudaGetErrorString(e));
            }
            buffer.swap(fresh);
        };
        grow(q, 3, "moving line state");
        grow(q2, 3, "moving line next state");
        grow(x, 1, "moving line positions");
        grow(x2, 1, "moving line next positions");
        grow(keys, 1, "moving line keys");
        grow(keys2, 1, "moving line next keys");
        grow(cell, 1, "moving line cells");
        grow(cell2, 1, "moving line spare cells");
        grow(volume, 1, "moving line volumes");
        grow(centroid, 1, "moving line centroids");
        grow(volume2, 1, "moving line next volumes");
        grow(centroid2, 1, "moving line next centroids");
        grow(staging, 3, "moving line staging");
        grow(slot, 1, "moving line sort slots");
        grow(slot2, 1, "moving line sorted slots");
        grow(composite, 1, "moving line sort keys");
        grow(composite2, 1, "moving line sorted keys");
        grow(by_cell, 1, "moving line sort cells");
        grow(by_cell2, 1, "moving line sorted cells");
        if (st != LUNA_OK) return st;
        DevBuffer<double> g, g2;
        st = g.alloc(static_cast<size_t>(grown) + 1, "moving line gaps");
        if (st == LUNA_OK) st = g2.alloc(static_cast<size_t>(grown) + 1, "moving line next gaps");
        if (st != LUNA_OK) return st;
        gap.swap(g);
        gap2.swap(g2);
        cap = grown;
        size_t temp_keys = 0, temp_cells = 0;
        MLINE_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_keys, composite.ptr, composite2.ptr, slot.ptr, slot2.ptr, cap, 0, 53, stream));
        MLINE_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_cells, by_cell.ptr, by_cell2.ptr, slot.ptr, slot2.ptr, cap, 0, 31, stream));
        st = sort_temp.alloc(std::max(temp_keys, temp_cells), "moving line sort scratch");
        if (st != LUNA_OK) return st;
        bind();
        return LUNA_OK;
    }
    // mesh_->order(): the slots sorted by (key, cell) (two stable radix passes: by cell, then by key), every slot array
    // gathered.
    luna_status sort() {
        k_mline_sort_cells<<<blocks_of(n), 128, 0, stream>>>(n, cell.ptr, by_cell.ptr, slot.ptr);
        MLINE_CUDA(cudaGetLastError());
        size_t temp = sort_temp.count;
        MLINE_CUDA(cub::DeviceRadixSort::SortPairs(sort_temp.ptr, temp, by_cell.ptr, by_cell2.ptr, slot.ptr, slot2.ptr, n, 0, 31, stream));
        k_mline_sort_keys<<<blocks_of(n), 128, 0, stream>>>(n, keys.ptr, slot2.ptr, composite.ptr);
        MLINE_CUDA(cudaGetLastError());
        temp = sort_temp.count;
        MLINE_CUDA(cub::DeviceRadixSort::SortPairs(sort_temp.ptr, temp, composite.ptr, composite2.ptr, slot2.ptr, slot.ptr, n, 0, 53, stream));
        k_mline_gather<<<blocks_of(n), 128, 0, stream>>>(n, slot.ptr, q.ptr, x.ptr, keys.ptr, cell.ptr, q2.ptr, x2.ptr, keys2.ptr, cell2.ptr);
        MLINE_CUDA(cudaGetLastError());
        q.swap(q2);
        x.swap(x2);
        keys.swap(keys2);
        cell.swap(cell2);
        bind();
        return LUNA_OK;
    }
    // The launch's counters (one pinned read); the next launch uses the other pair.
    luna_status read_counters(Counters* out, double* dt_out) {
        MLINE_CUDA(cudaMemcpyAsync(host_counters, counters.ptr + epoch, sizeof(Counters), cudaMemcpyDeviceToHost, stream));
        MLINE_CUDA(cudaStreamSynchronize(stream));
        *out = *host_counters;
        epoch ^= 1;
        if (out->error)
            return mfail(LUNA_ENONFINITE, out->error & 1ull ? "the moving line's time step is not finite" : "the moving line's state is not finite after the update");
        if (dt_out) std::memcpy(dt_out, &out->dt_bits, sizeof(double));
        return LUNA_OK;
    }
    Counters* use() { return counters.ptr + epoch; }
    Counters* spare() { return counters.ptr + (epoch ^ 1); }
    // due() (:957-964).
    bool due() {
        if (!supply[0] && !supply[1]) return false;
        if (watching) return !looked || wants > 0;
        if (--until_look > 0) return false;
        until_look = 64;
        return true;
    }
    luna_status time_step(double courant, int rule, double* dt) {
        bind();
        const int w = watching ? 1 : 0;
        if (order == 1)
            (rule == 1 ? k_mline_time_step<1, 1> : k_mline_time_step<1, 0>)<<<blocks_of(n), 128, 0, stream>>>(dev, mdev, q.ptr, courant, w, use(), spare());
        else
            (rule == 1 ? k_mline_time_step<0, 1> : k_mline_time_step<0, 0>)<<<blocks_of(n), 128, 0, stream>>>(dev, mdev, q.ptr, courant, w, use(), spare());
        MLINE_CUDA(cudaGetLastError());
        Counters c;
        const luna_status st = read_counters(&c, dt);
        if (st != LUNA_OK) return st;
        if (watching) {
            wants = c.wants;
            looked = true;
        }
        return LUNA_OK;
    }
    // supply_cells (:421-470).
    luna_status supply_cells(int* added_now) {
        if (added_now) *added_now = 0;
        bind();
        k_mline_ends<<<1, 1, 0, stream>>>(dev, keys.ptr, q.ptr, ends.ptr);
        MLINE_CUDA(cudaGetLastError());
        Ends e;
        MLINE_CUDA(cudaMemcpyAsync(&e, ends.ptr, sizeof(Ends), cudaMemcpyDeviceToHost, stream));
        MLINE_CUDA(cudaStreamSynchronize(stream));
        const auto room = [&](double vol, int64_t d) { return vol > 2 * spacing && static_cast<double>(d) * step >= 1.5 * spacing; };
        const int want_left = supply[0] && room(e.volume0, e.k0);
        const int want_right = supply[1] && room(e.volumel, period - e.kl);
        watching = watching || (supply[0] && e.v0 > 0) || (supply[1] && e.vl < 0);
        if (!want_left && !want_right) return LUNA_OK;
        const auto snap_host = [&](double y) {
            int64_t k = static_cast<int64_t>(std::nearbyint(y / step));
            return k < 0 ? int64_t(0) : k > period ? period : k;
        };
        Insert in{};
        int done = 0;
        if (want_left) {
            const double p = static_cast<double>(e.k0) * step - spacing;
            const int64_t kp = snap_host(p), k0 = e.k0, k1 = n > 1 ? e.k1 : period;
            if (kp > 0 && kp < k0) {
                in.left = 1;
                in.cell_left = n + done++;
                in.fraction_left = (static_cast<double>(kp + k0) * (0.5 * step)) / (static_cast<double>(k0 + k1) * (0.5 * step));
                in.x_left = p;
                in.key_left = kp;
            }
        }
        if (want_right) {
            const double p = length - (static_cast<double>(period - e.kl) * step - spacing);
            const int64_t kp = snap_host(p), kl = e.kl, kb = n > 1 ? e.kb : 0;
            if (kp > kl && kp < period) {
                in.right = 1;
                in.cell_right = n + done++;
                in.fraction_right = (static_cast<double>(2 * period - kl - kp) * (0.5 * step)) / (static_cast<double>(2 * period - kb - kl) * (0.5 * step));
                in.x_right = p;
                in.key_right = kp;
            }
        }
        if (done == 0) return LUNA_OK;
        luna_status st = reserve(n + done);
        if (st != LUNA_OK) return st;
        k_mline_insert<<<blocks_of(n + done), 128, 0, stream>>>(n, in, q.ptr, x.ptr, keys.ptr, cell.ptr, q2.ptr, x2.ptr, keys2.ptr, cell2.ptr);
        MLINE_CUDA(cudaGetLastError());
        q.swap(q2);
        x.swap(x2);
        keys.swap(keys2);
        cell.swap(cell2);
        n += done;
        added += done;
        bind();
        st = geometry();
        if (st != LUNA_OK) return st;
        if (added_now) *added_now = done;
        return LUNA_OK;
    }
    // One step's kernel, then Q, x and the keys move, the slots re-sort when out of order. Returns whether they did.
    luna_status advance(double dt, double courant, bool fused, double* smallest, bool* again) {
        if (!(dt > 0) || !std::isfinite(dt)) return mfail(LUNA_EINVAL, "dt must be finite and > 0");
        bind();
        const int w = fused && watching ? 1 : 0;
        const dim3 grid(blocks_of(n));
        if (order == 1)
            (fused ? k_mline_step<1, true> : k_mline_step<1, false>)<<<grid, kLineBlock, 0, stream>>>(dev, mdev, q.ptr, q2.ptr, dt, courant, w, use(), spare());
        else
            (fused ? k_mline_step<0, true> : k_mline_step<0, false>)<<<grid, kLineBlock, 0, stream>>>(dev, mdev, q.ptr, q2.ptr, dt, courant, w, use(), spare());
        MLINE_CUDA(cudaGetLastError());
        Counters c;
        luna_status st = read_counters(&c, smallest);
        if (st != LUNA_OK) return st;
        q.swap(q2);
        x.swap(x2);
        keys.swap(keys2);
        gap.swap(gap2);
        volume.swap(volume2);
        centroid.swap(centroid2);
        updates += 1;
        *again = false;
        bind();
        if (c.descents != (dev.periodic ? 1 : 0)) {
            st = sort();
            if (st == LUNA_OK) st = geometry();
            if (st != LUNA_OK) return st;
            sorts += 1;
            *again = true;
        }
        if (fused) {
            wants = c.wants;
            looked = watching;
        }
        return LUNA_OK;
    }
};

extern "C" {

LUNA_API luna_status luna_mline_create(int64_t n_cells, const double* positions, double length, int periodic, const int* walls,
                                       const double* inflow, const luna_gas* gas, int order, int limiter, int riemann, int regularise,
                                       luna_mline** out) {
    if (!out || !positions || !gas) return mfail(LUNA_EINVAL, "luna_mline_create: null argument");
    *out = nullptr;
    if (n_cells < 3 || n_cells >= (int64_t(1) << 30)) return mfail(LUNA_EINVAL, "luna_mline_create: 3 <= cells < 2^30");
    if (!(length > 0) || !std::isfinite(length)) return mfail(LUNA_EINVAL, "luna_mline_create: length must be positive");
    if (order != 0 && order != 1) return mfail(LUNA_EINVAL, "luna_mline_create: order 0 or 1");
    if (limiter < LUNA_LIMITER_FACE_CENTROID || limiter > LUNA_LIMITER_VAN_LEER) return mfail(LUNA_EINVAL, "luna_mline_create: unknown limiter");
    if (riemann != LUNA_HLLC && riemann != LUNA_HLL) return mfail(LUNA_EINVAL, "luna_mline_create: riemann HLLC or HLL");
    if (!(gas->gamma > 1.0)) return mfail(LUNA_EINVAL, "luna_mline_create: gamma must be > 1");
    const int w0 = walls ? walls[0] : LUNA_WALL_OUTFLOW, w1 = walls ? walls[1] : LUNA_WALL_OUTFLOW;
    if (!periodic && (w0 < LUNA_WALL_REFLECTIVE || w0 > LUNA_WALL_INFLOW || w1 < LUNA_WALL_REFLECTIVE || w1 > LUNA_WALL_INFLOW))
        return mfail(LUNA_EINVAL, "luna_mline_create: unknown wall");
    if (!periodic && (w0 == LUNA_WALL_INFLOW || w1 == LUNA_WALL_INFLOW) && !inflow)
        return mfail(LUNA_EINVAL, "luna_mline_create: an inflow wall needs its state");
    auto* ml = new luna_mline();
    ml->n = static_cast<int>(n_cells);
    ml->order = order;
    ml->length = length;
    ml->step = std::ldexp(length, -52);
    const int64_t period = ml->period;
    // the slots: the points snapped to the grid, sorted by (key, cell)
    std::vector<int64_t> key(n_cells);
    for (int64_t i = 0; i < n_cells; ++i) {
        const double p = positions[i];
        if (!(p >= 0 && p <= length)) {
            delete ml;
            return mfail(LUNA_EINVAL, "luna_mline_create: positions must lie in [0, length]");
        }
        int64_t k = static_cast<int64_t>(std::nearbyint(p / ml->step));
        if (periodic) {
            k %= period;
            if (k < 0) k += period;
        } else {
            k = std::min(std::max<int64_t>(k, 0), period);
        }
        key[i] = k;
    }
    std::vector<int> cells(n_cells);
    for (int64_t i = 0; i < n_cells; ++i) cells[i] = static_cast<int>(i);
    std::sort(cells.begin(), cells.end(), [&](int a, int b) { return key[a] < key[b] || (key[a] == key[b] && a < b); });
    std::vector<int64_t> skeys(n_cells);
    std::vector<double> sx(n_cells);
    for (int64_t s = 0; s < n_cells; ++s) {
        skeys[s] = key[cells[s]];
        sx[s] = positions[cells[s]];
    }
    luna_status st = LUNA_OK;
    ml->n = 0;  // nothing to keep in reserve()
    if (st == LUNA_OK) st = ml->counters.alloc(2, "moving line counters");
    if (st == LUNA_OK && cudaMallocHost(&ml->host_counters, sizeof(Counters)) != cudaSuccess) {
        cudaGetLastError();
        ml->host_counters = nullptr;
        st = mfail(LUNA_ENOMEM, "luna_mline_create: pinned counters");
    }
    if (st == LUNA_OK) st = ml->ends.alloc(1, "moving line ends");
    if (st == LUNA_OK) st = ml->reserve(static_cast<int>(n_cells));
    if (st != LUNA_OK) {
        delete ml;
        return st;
    }
    ml->n = static_cast<int>(n_cells);
    cudaError_t e = cudaMemcpy(ml->keys.ptr, skeys.data(), sizeof(int64_t) * n_cells, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ml->cell.ptr, cells.data(), sizeof(int) * n_cells, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ml->x.ptr, sx.data(), sizeof(double) * n_cells, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(ml->q.ptr, 0, sizeof(double) * 3 * n_cells);
    if (e == cudaSuccess) {
        Counters fresh[2];
        for (Counters& f : fresh) f = Counters{0x7fefffffffffffffull, 0, 0, 0};
        e = cudaMemcpy(ml->counters.ptr, fresh, sizeof(fresh), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        delete ml;
        return mfail(LUNA_ECUDA, std::string("luna_mline_create: ") + cudaGetErrorString(e));
    }
    LineDev& d = ml->dev;
    d.lines = 1;
    d.periodic = periodic != 0;
    d.order = order;
    d.limiter = limiter;
    d.riemann = riemann;
    d.wall[0] = w0;
    d.wall[1] = w1;
    for (int a = 0; a < 2; ++a)
        for (int v = 0; v < 3; ++v) d.inflow[a][v] = inflow ? inflow[3 * a + v] : 0.0;
    d.step = ml->step;
    d.gas.gamma = gas->gamma;
    d.gas.smallr = gas->smallr;
    d.gas.smallc = gas->smallc;
    d.gas.inverse_gm1 = 1.0 / (gas->gamma - 1.0);
    d.gas.inverse_gm1_float = static_cast<float>(1.0 / (gas->gamma - 1.0));
    MovingDev& m = ml->mdev;
    m.length = length;
    m.period = period;
    m.regularise = regularise != 0;
    // set_inflow_spacing(box / n) (:46, :61-66)
    ml->spacing = length / static_cast<double>(n_cells);
    for (int a = 0; a < 2; ++a) ml->supply[a] = !periodic && d.wall[a] != LUNA_WALL_REFLECTIVE && ml->spacing > 0;
    ml->bind();
    st = ml->geometry();
    if (st == LUNA_OK && cudaDeviceSynchronize() != cudaSuccess) st = mfail(LUNA_ECUDA, "luna_mline_create: the geometry kernel failed");
    if (st != LUNA_OK) {
        delete ml;
        return st;
    }
    *out = ml;
    return LUNA_OK;
}

LUNA_API luna_status luna_mline_destroy(luna_mline* ml) {
    delete ml;
    return LUNA_OK;
}

LUNA_API luna_status luna_mline_set_stream(luna_mline* ml, void* stream) {
    if (!ml) return mfail(LUNA_EINVAL, "luna_mline_set_stream: null line");
    ml->stream = static_cast<cudaStream_t>(stream);
    return LUNA_OK;
}

LUNA_API luna_status luna_mline_cells(luna_mline* ml, int64_t* cells) {
    if (!ml || !cells) return mfail(LUNA_EINVAL, "luna_mline_cells: null argument");
    *cells = ml->n;
    return LUNA_OK;
}

static luna_status mline_in(luna_mline* ml, const double* from, int width, double* slots, int on_device) {
    const double* src = from;
    if (!on_device) {
        MLINE_CUDA(cudaMemcpyAsync(ml->staging.ptr, from, sizeof(double) * width * ml->n, cudaMemcpyHostToDevice, ml->stream));
        src = ml->staging.ptr;
    }
    k_mline_permute<true><<<blocks_of(ml->n), 128, 0, ml->stream>>>(ml->n, width, ml->cell.ptr, src, slots);
    MLINE_CUDA(cudaGetLastError());
    if (!on_device) MLINE_CUDA(cudaStreamSynchronize(ml->stream));
    return LUNA_OK;
}
static luna_status mline_out(luna_mline* ml, const double* slots, int width, double* to, int on_device) {
    double* dst = on_device ? to : ml->staging.ptr;
    k_mline_permute<false><<<blocks_of(ml->n), 128, 0, ml->stream>>>(ml->n, width, ml->cell.ptr, slots, dst);
    MLINE_CUDA(cudaGetLastError());
    if (!on_device) {
        MLINE_CUDA(cudaMemcpyAsync(to, ml->staging.ptr, sizeof(double) * width * ml->n, cudaMemcpyDeviceToHost, ml->stream));
        MLINE_CUDA(cudaStreamSynchronize(ml->stream));
    }
    return LUNA_OK;
}

LUNA_API luna_status luna_mline_set_state(luna_mline* ml, const double* q, int on_device) {
    if (!ml || !q) return mfail(LUNA_EINVAL, "luna_mline_set_state: null argument");
    return mline_in(ml, q, 3, ml->q.ptr, on_device);
}

LUNA_API luna_status luna_mline_get_state(luna_mline* ml, double* q, int on_device) {
    if (!ml || !q) return mfail(LUNA_EINVAL, "luna_mline_get_state: null argument");
    return mline_out(ml, ml->q.ptr, 3, q, on_device);
}

LUNA_API luna_status luna_mline_positions(luna_mline* ml, double* x, int on_device) {
    if (!ml || !x) return mfail(LUNA_EINVAL, "luna_mline_positions: null argument");
    return mline_out(ml, ml->x.ptr, 1, x, on_device);
}

LUNA_API luna_status luna_mline_geometry(luna_mline* ml, double* generator, double* volume, double* centroid) {
    if (!ml || !generator || !volume || !centroid) return mfail(LUNA_EINVAL, "luna_mline_geometry: null argument");
    const int n = ml->n;
    std::vector<int64_t> k(n);
    std::vector<int> c(n);
    std::vector<double> v(n), m(n);
    MLINE_CUDA(cudaMemcpyAsync(k.data(), ml->keys.ptr, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ml->stream));
    MLINE_CUDA(cudaMemcpyAsync(c.data(), ml->cell.ptr, sizeof(int) * n, cudaMemcpyDeviceToHost, ml->stream));
    MLINE_CUDA(cudaMemcpyAsync(v.data(), ml->volume.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, ml->stream));
    MLINE_CUDA(cudaMemcpyAsync(m.data(), ml->centroid.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, ml->stream));
    MLINE_CUDA(cudaStreamSynchronize(ml->stream));
    for (int s = 0; s < n; ++s) {
        generator[c[s]] = static_cast<double>(k[s]) * ml->step;
        volume[c[s]] = v[s];
        centroid[c[s]] = m[s];
    }
    return LUNA_OK;
}

LUNA_API luna_status luna_mline_set_inflow_spacing(luna_mline* ml, double spacing) {
    if (!ml || !(spacing >= 0) || !std::isfinite(spacing)) return mfail(LUNA_EINVAL, "luna_mline_set_inflow_spacing: spacing >= 0");
    ml->spacing = spacing;
    for (int a = 0; a < 2; ++a) ml->supply[a] = !ml->dev.periodic && ml->dev.wall[a] != LUNA_WALL_REFLECTIVE && spacing > 0;
    ml->bind();
    return LUNA_OK;
}

LUNA_API luna_status luna_mline_supply_cells(luna_mline* ml, int* added) {
    if (!ml) return mfail(LUNA_EINVAL, "luna_mline_supply_cells: null line");
    return ml->supply_cells(added);
}

LUNA_API luna_status luna_mline_time_step(luna_mline* ml, double courant, int rule, double* dt) {
    if (!ml || !dt) return mfail(LUNA_EINVAL, "luna_mline_time_step: null argument");
    if (rule != 0 && rule != 1) return mfail(LUNA_EINVAL, "luna_mline_time_step: rule 0 (AREPO's) or 1 (LUNA's)");
    if (!(courant > 0)) return mfail(LUNA_EINVAL, "luna_mline_time_step: courant must be positive");
    return ml->time_step(courant, rule, dt);
}

LUNA_API luna_status luna_mline_step(luna_mline* ml, double dt) {
    if (!ml) return mfail(LUNA_EINVAL, "luna_mline_step: null line");
    bool again = false;
    luna_status st = ml->advance(dt, 0.0, false, nullptr, &again);
    if (st != LUNA_OK) return st;
    if (ml->due()) st = ml->supply_cells(nullptr);
    ml->looked = false;
    return st;
}

LUNA_API luna_status luna_mline_step_and_time_step(luna_mline* ml, double dt, double courant, double* dt_next) {
    if (!ml || !dt_next) return mfail(LUNA_EINVAL, "luna_mline_step_and_time_step: null argument");
    if (!(courant > 0)) return mfail(LUNA_EINVAL, "luna_mline_step_and_time_step: courant must be positive");
    bool again = false;
    double smallest = 0;
    luna_status st = ml->advance(dt, courant, true, &smallest, &again);
    if (st != LUNA_OK) return st;
    if (ml->due()) {
        int added = 0;
        st = ml->supply_cells(&added);
        if (st != LUNA_OK) return st;
        again = added > 0 || again;
    }
    ml->looked = false;
    if (again) return ml->time_step(courant, 1, dt_next);
    *dt_next = smallest;
    return LUNA_OK;
}

LUNA_API luna_status luna_mline_stats(luna_mline* ml, int64_t* cells_added, int64_t* sorts, int64_t* updates) {
    if (!ml) return mfail(LUNA_EINVAL, "luna_mline_stats: null line");
    if (cells_added) *cells_added = ml->added;
    if (sorts) *sorts = ml->sorts;
    if (updates) *updates = ml->updates;
    return LUNA_OK;
}

}  // extern "C"
