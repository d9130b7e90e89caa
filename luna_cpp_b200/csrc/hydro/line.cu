// The 1D solver of luna-cpp, FiniteVolume<1> on a static line (src/hydro/finite_volume_1d.hpp), on the GPU: a batch of
// independent lines that share one geometry (the reference runs one line; a batch of them is the data factory of the
// learned limiter's 1D Riemann problems, one launch for all of them).
//
// Layout: the line's generators sorted along it (slot order), per slot the cell's volume and centroid offset and the
// grid-step gaps to its neighbours (walls: twice the end generator's distance; periodic: the seam), shared by the batch;
// Q [lines][slots][3], slot order (the caller's cell order at the boundary). One thread per (line, slot) does what the
// reference's fused kernel does per slot (Kernel::body, :555-660): the five-cell stencil from HBM (neighbouring threads
// share it through L1), the limited slopes of s - 1, s, s + 1, the MUSCL-Hancock face states and the HLLC/HLL fluxes of
// its two faces, the update; the fused variant also reduces the next dt of LUNA's rule per line. Each face's flux is
// computed by both its cells, as in the reference: the step is latency-bound on the stencil loads, not flop-bound.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "line_stencil.cuh"
#include "luna_b200.h"
#include "tangent.cuh"

namespace luna {
luna_status report_error(luna_status s, const std::string& what);
}  // namespace luna

namespace {

// Kernel::body, static (:555-660), one thread per (line, slot): blockIdx.y is the line. Fused: the next dt of LUNA's rule,
// courant V / (|v| + c) of the updated cell (Kernel::body :632-658), reduced per line into dt_bits.
template <int Order, bool Fused>
__global__ void __launch_bounds__(128) k_line_step(LineDev L, const double* __restrict__ q_all, double* __restrict__ next_all,
                                                   const double* __restrict__ dt_of, double courant, unsigned long long* __restrict__ dt_bits,
                                                   unsigned long long* __restrict__ error) {
    const int line = blockIdx.y, s = blockIdx.x * blockDim.x + threadIdx.x;
    const double* q = q_all + static_cast<int64_t>(line) * L.n * V1;
    double* next = next_all + static_cast<int64_t>(line) * L.n * V1;
    const double dt = dt_of[line];
    double smallest = 1.0e300;
    if (s < L.n) {
        Cell1 cell[5];
        double gap[4], grad[5][3];
        load(L, q, s, cell, gap);
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
#pragma unroll
            for (int v = 0; v < 3; ++v) grad[k][v] = 0;
            if constexpr (Order == 1)
                if (cell[k].real)
#pragma unroll
                    for (int v = 0; v < 3; ++v) grad[k][v] = gradient(L, cell + k, gap[k - 1], gap[k], v);
        }
        double F[2][3];
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            const int a = 1 + f, b = 2 + f;
            double Wl[3] = {0, 0, 0}, Wr[3] = {0, 0, 0};
            if (cell[a].real) face_state<Order>(L, cell[a].W, grad[a], 0.5 * gap[a] - cell[a].c, dt, Wl);
            if (cell[b].real) face_state<Order>(L, cell[b].W, grad[b], -0.5 * gap[a] - cell[b].c, dt, Wr);
            if (!cell[a].real) ghost_face(L, Wr, cell[b].W, true, Wl);
            if (!cell[b].real) ghost_face(L, Wl, cell[a].W, false, Wr);
            line_flux(L, Wl, Wr, F[f]);
        }
        double U[3];
        bool finite = true;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            U[v] = q[3 * s + v] - dt * (F[1][v] - F[0][v]);
            next[3 * s + v] = U[v];
            finite = finite && isfinite(U[v]);
        }
        if (!finite) atomicOr(error, 2ull);
        if constexpr (Fused) {
            const double volume = L.volume[s], inv = 1.0 / volume;
            double Un[3], Wn[3];
#pragma unroll
            for (int v = 0; v < 3; ++v) Un[v] = U[v] * inv;
            luna::primitive<1>(Un, L.gas, Wn);
            smallest = courant * volume / (fabs(Wn[1]) + sqrt(L.gas.gamma * Wn[2] / Wn[0]));
            if (!(smallest == smallest)) atomicOr(error, 1ull);
        }
    }
    if constexpr (Fused) luna::block_min_to(smallest, dt_bits + line);
}

// time_step (:332-384), static: LUNA's rule (Rule 1) courant V / (|v| + c); AREPO's (Rule 0) courant times the smallest of
// r / (c + |v|) and, per side, (distance + r) / vsig, vsig = c_i + c_j - (v_j - v_i) side > 0, r = V / 2.
template <int Rule>
__global__ void __launch_bounds__(128) k_line_time_step(LineDev L, const double* __restrict__ q_all, double courant,
                                                        unsigned long long* __restrict__ dt_bits, unsigned long long* __restrict__ error) {
    const int line = blockIdx.y, s = blockIdx.x * blockDim.x + threadIdx.x;
    const double* q = q_all + static_cast<int64_t>(line) * L.n * V1;
    double smallest = 1.0e300;
    if (s < L.n) {
        double Wi[3];
        primitive_of(L, q, s, Wi);
        const double ci = sqrt(L.gas.gamma * Wi[2] / Wi[0]);
        const double volume = L.volume[s], vi = fabs(Wi[1]);
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
                const double vsig = ci + sqrt(L.gas.gamma * Wj[2] / Wj[0]) - (Wj[1] - Wi[1]) * side;
                if (vsig > 0) step = fmin(step, (dist + r) / vsig);
            }
            smallest = courant * step;
        }
        if (!(smallest == smallest)) atomicOr(error, 1ull);
    }
    luna::block_min_to(smallest, dt_bits + line);
}

__global__ void k_line_reset(int lines, unsigned long long* dt_bits) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < lines) dt_bits[k] = 0x7fefffffffffffffull;  // DBL_MAX, the Min reducer's identity
}

// Caller cell order <-> slot order: to[line][s] = from[line][order[s]] (gather) or to[line][order[s]] = from[line][s].
template <bool Gather>
__global__ void k_line_permute(int64_t n, int lines, const int64_t* __restrict__ order, const double* __restrict__ from, double* __restrict__ to) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n * lines) return;
    const int64_t line = k / n, s = k - line * n, i = order[s];
    const int64_t a = (line * n + s) * V1, b = (line * n + i) * V1;
#pragma unroll
    for (int v = 0; v < V1; ++v) {
        if (Gather)
            to[a + v] = from[b + v];
        else
            to[b + v] = from[a + v];
    }
}

// ---- The step's derivatives at fixed dt (the reference's FiniteVolume<1>::step_tangent / step_adjoint,
// finite_volume_1d.hpp:711-823, checked against LUNA's jax.jvp / jax.vjp). Cell s's update reads the cells s - 2 .. s + 2
// (its two faces, each from the two cells' slopes). Both derivatives run the step's expressions on forward-mode dual
// numbers (fwd::Dual; each branch the forward took): the tangent in one pass a slot seeded by dq; the adjoint forms each
// row's 3 x 15 block of the band Jacobian (one pass per input) and gathers J^T w from it (no atomics: the same bits every
// run).

// primitive() (euler.hpp:104-113) on any arithmetic type: the step's operations, floors included.
template <class T>
__device__ __forceinline__ void primitive1(const T* U, const luna::GasDev& gas, T* W) {
    const T rho = fmax(U[0], T(gas.smallr));
    const T inv_rho = T(1.0) / rho;
    const T v = U[1] * inv_rho;
    const double smalle = gas.smallc * gas.smallc / gas.gamma / (gas.gamma - 1.0);
    const T kinetic = T(0.5) * rho * (v * v);
    const T e = fmax(U[2] - kinetic, T(smalle) * rho);
    W[0] = rho;
    W[1] = v;
    W[2] = T(gas.gamma - 1.0) * e;
}
template <class T>
__device__ __forceinline__ void ghost_t(const LineDev& L, const T* W, bool left, T* out) {
    const int wall = L.wall[left ? 0 : 1];
    if (wall == LUNA_WALL_REFLECTIVE) {
        out[0] = W[0];
        out[1] = -W[1];
        out[2] = W[2];
    } else if (wall == LUNA_WALL_INFLOW) {
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = T(L.inflow[left ? 0 : 1][v]);
    } else {
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = W[v];
    }
}
template <class T>
__device__ __forceinline__ void ghost_face_t(const LineDev& L, const T* Wf, const T* W, bool left, T* out) {
    if (L.wall[left ? 0 : 1] == LUNA_WALL_REFLECTIVE) {
        out[0] = Wf[0];
        out[1] = -Wf[1];
        out[2] = Wf[2];
    } else {
        ghost_t(L, W, left, out);
    }
}
struct CellT {
    luna::fwd::Dual W[3];
    double c;
    bool real;
};
// gradient() on dual numbers (Stencil::gradient, finite_volume_1d.hpp:183-207).
__device__ __forceinline__ luna::fwd::Dual gradient_t(const LineDev& L, const CellT* cell, double gapL, double gapR, int v) {
    using T = luna::fwd::Dual;
    const CellT& me = *cell;
    const double dL = -gapL + cell[-1].c - me.c, dR = gapR + cell[1].c - me.c;
    const T Wi = me.W[v], left = cell[-1].W[v], right = cell[1].W[v];
    if (L.limiter == LUNA_LIMITER_MINMOD || L.limiter == LUNA_LIMITER_VAN_LEER) {
        const T sL = (left - Wi) / T(dL), sR = (right - Wi) / T(dR);
        if (!(sL * sR > T(0))) return T(0);
        if (L.limiter == LUNA_LIMITER_VAN_LEER) return T(2) * sL * sR / (sL + sR);
        return fabs(sL) < fabs(sR) ? sL : sR;
    }
    T g = ((right - Wi) - (left - Wi)) / T(dR - dL);
    if (L.limiter == LUNA_LIMITER_NONE) return g;
    const double r[2] = {-0.5 * gapL - me.c, 0.5 * gapR - me.c};
    const T lo = fmin(left, right), hi = fmax(left, right);
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        const T dp = g * T(r[f]);
        if (dp > T(0) && Wi + dp > hi)
            g = g * (hi > Wi ? (hi - Wi) / dp : T(0));
        else if (dp < T(0) && Wi + dp < lo)
            g = g * (lo < Wi ? (lo - Wi) / dp : T(0));
    }
    return g;
}

// The tangent of slot s's update for the tangents dU of the stencil's U = Q / V (d[k][u], positions k = 0 .. 4; a ghost
// position's ignored): d Q'_s = -dt (dF_right - dF_left), on dual numbers (the step's operations and branches).
template <int Order>
__device__ __forceinline__ void update_tangent(const LineDev& L, const double* q, const int (&slot)[5], const double (&gap)[4], double dt,
                                               const double (&d)[5][3], double (&out)[3]) {
    using T = luna::fwd::Dual;
    CellT cell[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        cell[k].real = slot[k] >= 0;
        cell[k].c = 0;
#pragma unroll
        for (int v = 0; v < 3; ++v) cell[k].W[v] = T(0);
        if (slot[k] >= 0) {
            const double inv = 1.0 / L.volume[slot[k]];
            T U[3];
#pragma unroll
            for (int v = 0; v < 3; ++v) U[v] = T(q[3 * slot[k] + v] * inv, d[k][v]);
            primitive1(U, L.gas, cell[k].W);
            cell[k].c = L.centroid[slot[k]];
        }
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        if (slot[k] >= 0) continue;
        const int end = k < 2 ? k + 1 : k - 1;
        if (slot[end] < 0) continue;
        ghost_t(L, cell[end].W, k < 2, cell[k].W);
        cell[k].c = -cell[end].c;
    }
    T grad[5][3];
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
#pragma unroll
        for (int v = 0; v < 3; ++v) grad[k][v] = T(0);
        if constexpr (Order == 1)
            if (cell[k].real)
#pragma unroll
                for (int v = 0; v < 3; ++v) grad[k][v] = gradient_t(L, cell + k, gap[k - 1], gap[k], v);
    }
    T F[2][3];
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        const int a = 1 + f, b = 2 + f;
        T Wl[3] = {T(0), T(0), T(0)}, Wr[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int c = side == 0 ? a : b;
            if (!cell[c].real) continue;
            T* o = side == 0 ? Wl : Wr;
            const double r = side == 0 ? 0.5 * gap[a] - cell[a].c : -0.5 * gap[a] - cell[b].c;
            if constexpr (Order == 0) {
#pragma unroll
                for (int v = 0; v < 3; ++v) o[v] = cell[c].W[v];
            } else {  // Kernel::face_state (:492-506)
                T A[3];
                luna::half_step_rate<1, T>(cell[c].W, grad[c], T(L.gas.gamma), A);
#pragma unroll
                for (int v = 0; v < 3; ++v) o[v] = cell[c].W[v] - T(0.5 * dt) * A[v];
#pragma unroll
                for (int v = 0; v < 3; ++v) o[v] += grad[c][v] * T(r);
                if (!(o[0] > T(0) && o[2] > T(0)))
#pragma unroll
                    for (int v = 0; v < 3; ++v) o[v] = cell[c].W[v];
            }
        }
        if (!cell[a].real) ghost_face_t(L, Wr, cell[b].W, true, Wl);
        if (!cell[b].real) ghost_face_t(L, Wl, cell[a].W, false, Wr);
        const T n[1] = {T(1.0)}, w[1] = {T(0.0)};
        if (L.riemann == LUNA_HLL)
            luna::fwd::hll_flux_t<1, T>(Wl, Wr, n, w, T(L.gas.gamma), T(L.gas.inverse_gm1), F[f]);
        else
            luna::hllc_flux<1, T>(Wl, Wr, n, w, T(L.gas.gamma), T(L.gas.inverse_gm1), F[f], false);
    }
#pragma unroll
    for (int v = 0; v < 3; ++v) out[v] = -dt * (F[1][v].d - F[0][v].d);
}

__device__ __forceinline__ void stencil_of(const LineDev& L, int s, int (&slot)[5], double (&gap)[4]) {
#pragma unroll
    for (int k = 0; k < 5; ++k) slot[k] = slot_at(L, s, k - 2);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int a = slot[k], b = slot[k + 1];
        gap[k] = a >= 0 ? L.gap[a + 1] * L.step : b >= 0 ? L.gap[0] * L.step : 0.0;
    }
}

// step_tangent's derivative (:852-883): dout = dq + d Q' for the tangent dq, one dual pass a slot (slot order).
template <int Order>
__global__ void __launch_bounds__(128) k_line_tangent(LineDev L, const double* __restrict__ q_all, const double* __restrict__ dt_of,
                                                      const double* __restrict__ dq_all, double* __restrict__ dout_all) {
    const int line = blockIdx.y, s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= L.n) return;
    const int64_t base = static_cast<int64_t>(line) * L.n * V1;
    const double *q = q_all + base, *dq = dq_all + base;
    int slot[5];
    double gap[4], d[5][3], out[3];
    stencil_of(L, s, slot, gap);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const double inv = slot[k] >= 0 ? 1.0 / L.volume[slot[k]] : 0.0;
#pragma unroll
        for (int v = 0; v < 3; ++v) d[k][v] = slot[k] >= 0 ? dq[3 * slot[k] + v] * inv : 0.0;
    }
    update_tangent<Order>(L, q, slot, gap, dt_of[line], d, out);
#pragma unroll
    for (int v = 0; v < 3; ++v) dout_all[base + 3 * s + v] = dq[3 * s + v] + out[v];
}

// Row s's block of the step's Jacobian for step_adjoint: jac[line][s][v][3 k + u] = d Q'_s,v / d Q_{s + k - 2},u, one
// dual pass per input (a ghost position's column 0: a ghost's dependence on its wall's end cell runs through that cell's
// column).
template <int Order>
__global__ void __launch_bounds__(128) k_line_jacobian(LineDev L, const double* __restrict__ q_all, const double* __restrict__ dt_of,
                                                       double* __restrict__ jac_all) {
    const int line = blockIdx.y, s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= L.n) return;
    const double* q = q_all + static_cast<int64_t>(line) * L.n * V1;
    double* jac = jac_all + (static_cast<int64_t>(line) * L.n + s) * 45;
    const double dt = dt_of[line];
    int slot[5];
    double gap[4];
    stencil_of(L, s, slot, gap);
    for (int seed = 0; seed < 15; ++seed) {
        const int sk = seed / 3, sv = seed % 3;
        double out[3] = {0, 0, 0};
        if (slot[sk] >= 0) {
            double d[5][3];
#pragma unroll
            for (int k = 0; k < 5; ++k)
#pragma unroll
                for (int v = 0; v < 3; ++v) d[k][v] = k == sk && v == sv ? 1.0 / L.volume[slot[sk]] : 0.0;
            update_tangent<Order>(L, q, slot, gap, dt, d, out);
        }
#pragma unroll
        for (int v = 0; v < 3; ++v) jac[15 * v + seed] = (sk == 2 && sv == v ? 1.0 : 0.0) + out[v];
    }
}

// out = J^T w with the blocks of k_line_jacobian, slot order: column t gathers the rows s whose stencil position k is t
// (s = t + 2 - k), no atomics (the same bits every run).
__global__ void __launch_bounds__(128) k_line_band_adjoint(LineDev L, const double* __restrict__ jac_all, const double* __restrict__ w_all,
                                                           double* __restrict__ out_all) {
    const int line = blockIdx.y, t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.n) return;
    const int64_t base = static_cast<int64_t>(line) * L.n;
    const double* w = w_all + base * V1;
    double out[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int s = slot_at(L, t, 2 - k);
        if (s < 0) continue;
        const double* J = jac_all + (base + s) * 45;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double ws = w[3 * s + v];
#pragma unroll
            for (int u = 0; u < 3; ++u) out[u] += J[15 * v + 3 * k + u] * ws;
        }
    }
    double* o = out_all + (base + t) * V1;
#pragma unroll
    for (int v = 0; v < 3; ++v) o[v] = out[v];
}

luna_status fail(luna_status s, const std::string& what) { return luna::report_error(s, what); }

#define LINE_CUDA(call)                                                                                     \
    do {                                                                                                    \
        const cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return fail(LUNA_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
struct Buffer {
    T* ptr = nullptr;
    size_t count = 0;
    Buffer() = default;
    Buffer(const Buffer&) = delete;
    Buffer& operator=(const Buffer&) = delete;
    void swap(Buffer& other) {
        std::swap(ptr, other.ptr);
        std::swap(count, other.count);
    }
    ~Buffer() {
        if (ptr) cudaFree(ptr);
    }
    luna_status alloc(size_t n, const char* what) {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
        const cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();
            return fail(e == cudaErrorMemoryAllocation ? LUNA_ENOMEM : LUNA_ECUDA, std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
        }
        count = n;
        return LUNA_OK;
    }
};

}  // namespace

struct luna_line {
    LineDev dev{};
    int64_t n = 0, period = 0;
    int lines = 0;
    cudaStream_t stream = nullptr;
    std::vector<int64_t> keys, order;  // sorted keys; slot -> caller cell
    std::vector<double> host_volume, host_centroid;
    Buffer<double> q, next, gap, volume, centroid, dt, staging;
    Buffer<double> jac, dvec, dout;  // the derivatives (allocated by their first call): Jacobian blocks, vectors in slot order
    Buffer<int64_t> order_dev;
    Buffer<unsigned long long> bits, error;
    std::vector<unsigned long long> host_bits;

    dim3 grid() const { return dim3(static_cast<unsigned int>((n + 127) / 128), static_cast<unsigned int>(lines)); }

    luna_status read_dt(double* out) {
        LINE_CUDA(cudaMemcpyAsync(host_bits.data(), bits.ptr, sizeof(unsigned long long) * lines, cudaMemcpyDeviceToHost, stream));
        unsigned long long err = 0;
        LINE_CUDA(cudaMemcpyAsync(&err, error.ptr, sizeof(err), cudaMemcpyDeviceToHost, stream));
        LINE_CUDA(cudaStreamSynchronize(stream));
        if (err) {
            LINE_CUDA(cudaMemsetAsync(error.ptr, 0, sizeof(unsigned long long), stream));
            return fail(LUNA_ENONFINITE, err & 1ull ? "a line's time step is not finite" : "a line's state is not finite after the update");
        }
        for (int k = 0; k < lines; ++k) {
            double d;
            std::memcpy(&d, &host_bits[k], sizeof(d));
            out[k] = d;
        }
        return LUNA_OK;
    }
    luna_status upload_dt(const double* dt_host) {
        for (int k = 0; k < lines; ++k)
            if (!(dt_host[k] >= 0) || !std::isfinite(dt_host[k])) return fail(LUNA_EINVAL, "dt must be finite and >= 0");
        LINE_CUDA(cudaMemcpyAsync(dt.ptr, dt_host, sizeof(double) * lines, cudaMemcpyHostToDevice, stream));
        return LUNA_OK;
    }
};

extern "C" {

LUNA_API luna_status luna_line_create(int64_t n_cells, int lines, const double* positions, double length, int periodic, const int* walls,
                                      const double* inflow, const luna_gas* gas, int order, int limiter, int riemann, luna_line** out) {
    if (!out || !positions || !gas) return fail(LUNA_EINVAL, "luna_line_create: null argument");
    *out = nullptr;
    if (n_cells < 3 || n_cells >= (int64_t(1) << 30)) return fail(LUNA_EINVAL, "luna_line_create: 3 <= cells < 2^30");
    if (lines < 1 || lines > 65535) return fail(LUNA_EINVAL, "luna_line_create: 1 <= lines <= 65535");
    if (!(length > 0) || !std::isfinite(length)) return fail(LUNA_EINVAL, "luna_line_create: length must be positive");
    if (order != 0 && order != 1) return fail(LUNA_EINVAL, "luna_line_create: order 0 or 1");
    if (limiter < LUNA_LIMITER_FACE_CENTROID || limiter > LUNA_LIMITER_VAN_LEER) return fail(LUNA_EINVAL, "luna_line_create: unknown limiter");
    if (riemann != LUNA_HLLC && riemann != LUNA_HLL) return fail(LUNA_EINVAL, "luna_line_create: riemann HLLC or HLL");
    if (!(gas->gamma > 1.0)) return fail(LUNA_EINVAL, "luna_line_create: gamma must be > 1");
    const int w0 = walls ? walls[0] : LUNA_WALL_OUTFLOW, w1 = walls ? walls[1] : LUNA_WALL_OUTFLOW;
    if (!periodic && (w0 < LUNA_WALL_REFLECTIVE || w0 > LUNA_WALL_INFLOW || w1 < LUNA_WALL_REFLECTIVE || w1 > LUNA_WALL_INFLOW))
        return fail(LUNA_EINVAL, "luna_line_create: unknown wall");
    if (!periodic && (w0 == LUNA_WALL_INFLOW || w1 == LUNA_WALL_INFLOW) && !inflow)
        return fail(LUNA_EINVAL, "luna_line_create: an inflow wall needs its state");

    auto* ln = new luna_line();
    ln->n = n_cells;
    ln->lines = lines;
    // the 1D mesh's grid: 2^52 steps across the line (research_notes/stage1_1d_2026-11-04.md:35, :64-78)
    const double step = std::ldexp(length, -52);
    ln->period = int64_t(1) << 52;
    std::vector<int64_t> key(n_cells);
    for (int64_t i = 0; i < n_cells; ++i) {
        const double x = positions[i];
        if (!(x >= 0 && x <= length)) {
            delete ln;
            return fail(LUNA_EINVAL, "luna_line_create: positions must lie in [0, length]");
        }
        key[i] = std::llrint(x / step);
    }
    ln->order.resize(n_cells);
    for (int64_t i = 0; i < n_cells; ++i) ln->order[i] = i;
    std::stable_sort(ln->order.begin(), ln->order.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
    ln->keys.resize(n_cells);
    for (int64_t s = 0; s < n_cells; ++s) ln->keys[s] = key[ln->order[s]];
    for (int64_t s = 0; s + 1 < n_cells; ++s)
        if (ln->keys[s + 1] == ln->keys[s]) {
            delete ln;
            return fail(LUNA_EINVAL, "luna_line_create: two generators on one grid point");
        }
    // Line::gap, volume, centroid (finite_volume_1d.hpp load_inner :163-176)
    std::vector<double> gap(n_cells + 1);
    for (int64_t s = 0; s + 1 < n_cells; ++s) gap[s + 1] = static_cast<double>(ln->keys[s + 1] - ln->keys[s]);
    if (periodic) {
        gap[0] = gap[n_cells] = static_cast<double>(ln->keys[0] + ln->period - ln->keys[n_cells - 1]);
    } else {
        gap[0] = static_cast<double>(2 * ln->keys[0]);
        gap[n_cells] = static_cast<double>(2 * (ln->period - ln->keys[n_cells - 1]));
    }
    ln->host_volume.resize(n_cells);
    ln->host_centroid.resize(n_cells);
    for (int64_t s = 0; s < n_cells; ++s) {
        ln->host_volume[s] = (gap[s] + gap[s + 1]) * (0.5 * step);
        ln->host_centroid[s] = (gap[s + 1] - gap[s]) * (0.25 * step);
    }
    luna_status st = LUNA_OK;
    const size_t cells = static_cast<size_t>(n_cells) * lines;
    if (st == LUNA_OK) st = ln->q.alloc(cells * V1, "line state");
    if (st == LUNA_OK) st = ln->next.alloc(cells * V1, "line next state");
    if (st == LUNA_OK) st = ln->staging.alloc(cells * V1, "line staging");
    if (st == LUNA_OK) st = ln->gap.alloc(n_cells + 1, "line gaps");
    if (st == LUNA_OK) st = ln->volume.alloc(n_cells, "line volumes");
    if (st == LUNA_OK) st = ln->centroid.alloc(n_cells, "line centroids");
    if (st == LUNA_OK) st = ln->order_dev.alloc(n_cells, "line order");
    if (st == LUNA_OK) st = ln->dt.alloc(lines, "line dt");
    if (st == LUNA_OK) st = ln->bits.alloc(lines, "line dt bits");
    if (st == LUNA_OK) st = ln->error.alloc(1, "line error word");
    if (st != LUNA_OK) {
        delete ln;
        return st;
    }
    cudaError_t e = cudaMemcpy(ln->gap.ptr, gap.data(), sizeof(double) * gap.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ln->volume.ptr, ln->host_volume.data(), sizeof(double) * n_cells, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ln->centroid.ptr, ln->host_centroid.data(), sizeof(double) * n_cells, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ln->order_dev.ptr, ln->order.data(), sizeof(int64_t) * n_cells, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(ln->q.ptr, 0, sizeof(double) * cells * V1);
    if (e == cudaSuccess) e = cudaMemset(ln->error.ptr, 0, sizeof(unsigned long long));
    if (e != cudaSuccess) {
        delete ln;
        return fail(LUNA_ECUDA, std::string("luna_line_create: ") + cudaGetErrorString(e));
    }
    ln->host_bits.resize(lines);
    LineDev& d = ln->dev;
    d.n = static_cast<int>(n_cells);
    d.lines = lines;
    d.periodic = periodic != 0;
    d.order = order;
    d.limiter = limiter;
    d.riemann = riemann;
    d.wall[0] = w0;
    d.wall[1] = w1;
    for (int a = 0; a < 2; ++a)
        for (int v = 0; v < 3; ++v) d.inflow[a][v] = inflow ? inflow[3 * a + v] : 0.0;
    d.step = step;
    d.gap = ln->gap.ptr;
    d.volume = ln->volume.ptr;
    d.centroid = ln->centroid.ptr;
    d.gas.gamma = gas->gamma;
    d.gas.smallr = gas->smallr;
    d.gas.smallc = gas->smallc;
    d.gas.inverse_gm1 = 1.0 / (gas->gamma - 1.0);
    d.gas.inverse_gm1_float = static_cast<float>(1.0 / (gas->gamma - 1.0));
    *out = ln;
    return LUNA_OK;
}

LUNA_API luna_status luna_line_destroy(luna_line* ln) {
    delete ln;
    return LUNA_OK;
}

LUNA_API luna_status luna_line_set_stream(luna_line* ln, void* stream) {
    if (!ln) return fail(LUNA_EINVAL, "line is null");
    ln->stream = static_cast<cudaStream_t>(stream);
    return LUNA_OK;
}

// The cells' geometry in the caller's order: volume and centroid offset from the generator.
LUNA_API luna_status luna_line_geometry(luna_line* ln, double* volume, double* centroid) {
    if (!ln) return fail(LUNA_EINVAL, "line is null");
    for (int64_t s = 0; s < ln->n; ++s) {
        if (volume) volume[ln->order[s]] = ln->host_volume[s];
        if (centroid) centroid[ln->order[s]] = ln->host_centroid[s];
    }
    return LUNA_OK;
}

LUNA_API luna_status luna_line_set_state(luna_line* ln, const double* q, int on_device) {
    if (!ln || !q) return fail(LUNA_EINVAL, "null argument");
    const size_t bytes = sizeof(double) * static_cast<size_t>(ln->n) * ln->lines * V1;
    LINE_CUDA(cudaMemcpyAsync(ln->staging.ptr, q, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ln->stream));
    const int64_t total = ln->n * ln->lines;
    k_line_permute<true><<<static_cast<unsigned int>((total + 255) / 256), 256, 0, ln->stream>>>(ln->n, ln->lines, ln->order_dev.ptr, ln->staging.ptr,
                                                                                                 ln->q.ptr);
    LINE_CUDA(cudaGetLastError());
    if (!on_device) LINE_CUDA(cudaStreamSynchronize(ln->stream));  // the caller may reuse its host buffer
    return LUNA_OK;
}

LUNA_API luna_status luna_line_get_state(luna_line* ln, double* q, int on_device) {
    if (!ln || !q) return fail(LUNA_EINVAL, "null argument");
    const int64_t total = ln->n * ln->lines;
    k_line_permute<false><<<static_cast<unsigned int>((total + 255) / 256), 256, 0, ln->stream>>>(ln->n, ln->lines, ln->order_dev.ptr, ln->q.ptr,
                                                                                                  ln->staging.ptr);
    LINE_CUDA(cudaGetLastError());
    const size_t bytes = sizeof(double) * static_cast<size_t>(total) * V1;
    LINE_CUDA(cudaMemcpyAsync(q, ln->staging.ptr, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ln->stream));
    if (!on_device) LINE_CUDA(cudaStreamSynchronize(ln->stream));
    return LUNA_OK;
}

// time_step(courant, rule) (finite_volume_1d.hpp:332-384): per line; rule 0 AREPO's, 1 LUNA's. Synchronises.
LUNA_API luna_status luna_line_time_step(luna_line* ln, double courant, int rule, double* dt_out) {
    if (!ln || !dt_out) return fail(LUNA_EINVAL, "null argument");
    if (!(courant > 0)) return fail(LUNA_EINVAL, "courant must be positive");
    k_line_reset<<<(ln->lines + 255) / 256, 256, 0, ln->stream>>>(ln->lines, ln->bits.ptr);
    if (rule == 1)
        k_line_time_step<1><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, courant, ln->bits.ptr, ln->error.ptr);
    else
        k_line_time_step<0><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, courant, ln->bits.ptr, ln->error.ptr);
    LINE_CUDA(cudaGetLastError());
    return ln->read_dt(dt_out);
}

// step(dt) (:389-410), static: every line by its own dt (host array [lines]). Asynchronous.
LUNA_API luna_status luna_line_step(luna_line* ln, const double* dt) {
    if (!ln || !dt) return fail(LUNA_EINVAL, "null argument");
    const luna_status st = ln->upload_dt(dt);
    if (st != LUNA_OK) return st;
    if (ln->dev.order == 1)
        k_line_step<1, false><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, ln->next.ptr, ln->dt.ptr, 0.0, nullptr, ln->error.ptr);
    else
        k_line_step<0, false><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, ln->next.ptr, ln->dt.ptr, 0.0, nullptr, ln->error.ptr);
    LINE_CUDA(cudaGetLastError());
    ln->q.swap(ln->next);
    return LUNA_OK;
}

// step_and_time_step(dt, courant) (:412-418): the step and the next dt of LUNA's rule in one launch. Synchronises.
LUNA_API luna_status luna_line_step_and_time_step(luna_line* ln, const double* dt, double courant, double* dt_next) {
    if (!ln || !dt || !dt_next) return fail(LUNA_EINVAL, "null argument");
    if (!(courant > 0)) return fail(LUNA_EINVAL, "courant must be positive");
    const luna_status st = ln->upload_dt(dt);
    if (st != LUNA_OK) return st;
    k_line_reset<<<(ln->lines + 255) / 256, 256, 0, ln->stream>>>(ln->lines, ln->bits.ptr);
    if (ln->dev.order == 1)
        k_line_step<1, true><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, ln->next.ptr, ln->dt.ptr, courant, ln->bits.ptr, ln->error.ptr);
    else
        k_line_step<0, true><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, ln->next.ptr, ln->dt.ptr, courant, ln->bits.ptr, ln->error.ptr);
    LINE_CUDA(cudaGetLastError());
    ln->q.swap(ln->next);
    return ln->read_dt(dt_next);
}

// The step's derivatives at fixed dt (finite_volume_1d.hpp:711-823): x in the caller's cell order [lines][n][3] (device
// or host memory). tangent: x <- J x in one dual pass, then the step itself (Q advances as luna_line_step); adjoint: the
// Jacobian blocks at the current state and x <- J^T x, Q unchanged (the state must be the step's start).
static luna_status line_derivative(luna_line* ln, const double* dt, double* x, int on_device, bool tangent) {
    if (!ln || !dt || !x) return fail(LUNA_EINVAL, "null argument");
    if (ln->dev.periodic && ln->n < 5) return fail(LUNA_EINVAL, "the derivatives of a periodic line need 5 cells or more");
    const size_t cells = static_cast<size_t>(ln->n) * ln->lines;
    if (!ln->dvec.ptr) {
        luna_status st = ln->dvec.alloc(cells * V1, "line derivative vector");
        if (st == LUNA_OK) st = ln->dout.alloc(cells * V1, "line derivative vector");
        if (st != LUNA_OK) return st;
    }
    if (!tangent && !ln->jac.ptr) {
        const luna_status st = ln->jac.alloc(cells * 45, "line Jacobian blocks");
        if (st != LUNA_OK) return st;
    }
    luna_status st = ln->upload_dt(dt);
    if (st != LUNA_OK) return st;
    const size_t bytes = sizeof(double) * cells * V1;
    const int64_t total = ln->n * ln->lines;
    const unsigned int pblocks = static_cast<unsigned int>((total + 255) / 256);
    LINE_CUDA(cudaMemcpyAsync(ln->staging.ptr, x, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ln->stream));
    k_line_permute<true><<<pblocks, 256, 0, ln->stream>>>(ln->n, ln->lines, ln->order_dev.ptr, ln->staging.ptr, ln->dvec.ptr);
    if (tangent) {
        if (ln->dev.order == 1)
            k_line_tangent<1><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, ln->dt.ptr, ln->dvec.ptr, ln->dout.ptr);
        else
            k_line_tangent<0><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, ln->dt.ptr, ln->dvec.ptr, ln->dout.ptr);
    } else {
        if (ln->dev.order == 1)
            k_line_jacobian<1><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, ln->dt.ptr, ln->jac.ptr);
        else
            k_line_jacobian<0><<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->q.ptr, ln->dt.ptr, ln->jac.ptr);
        k_line_band_adjoint<<<ln->grid(), 128, 0, ln->stream>>>(ln->dev, ln->jac.ptr, ln->dvec.ptr, ln->dout.ptr);
    }
    k_line_permute<false><<<pblocks, 256, 0, ln->stream>>>(ln->n, ln->lines, ln->order_dev.ptr, ln->dout.ptr, ln->staging.ptr);
    LINE_CUDA(cudaGetLastError());
    LINE_CUDA(cudaMemcpyAsync(x, ln->staging.ptr, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ln->stream));
    if (!on_device) LINE_CUDA(cudaStreamSynchronize(ln->stream));
    if (tangent) return luna_line_step(ln, dt);
    return LUNA_OK;
}

LUNA_API luna_status luna_line_step_tangent(luna_line* ln, const double* dt, double* dq, int on_device) {
    return line_derivative(ln, dt, dq, on_device, true);
}

LUNA_API luna_status luna_line_step_adjoint(luna_line* ln, const double* dt, double* qbar, int on_device) {
    return line_derivative(ln, dt, qbar, on_device, false);
}

}  // extern "C"
