// Kernels of the hydro step on a periodic Voronoi mesh (luna-cpp's FiniteVolume<D>, src/hydro/finite_volume.hpp).
//
// Data layout in HBM (the library's own copies, made once per mesh):
//   cells  q[N][V] (extensive Q), prims[N][8] (W, c, r, pad: two 32-B sectors a row), gradient rows [N][GS] of G
//          (GS = 16 in 3D: 15 used, 128 B in double / 64 B in float), vol[N], cen[N][D] (relative to the generator),
//          pos[N][D] (generators)
//   faces  owner[F], neighbour[F], area[F][D], mag[F] (|A|, computed once per mesh), fcen[F][D] (relative to the
//          owner's generator), flux rows [F][V] (per-face update)
//   lists  start[N + 1], list[2F] (voronoi-cpp's lists with the owner bit: ~f marks a face the cell does not own)
#pragma once

#include <cstdint>

#include <cuda_fp16.h>

#include "physics.cuh"

namespace luna {

constexpr int PS = 8;  // doubles per primitive row: W (V), c, r, pad
template <int D>
constexpr int grad_stride() {
    return D == 3 ? 16 : 8;
}

template <int D>
struct MeshDev {
    const int32_t* __restrict__ owner;
    const int32_t* __restrict__ neighbour;
    const int32_t* __restrict__ start;
    const int32_t* __restrict__ list;
    const double* __restrict__ area;
    const double* __restrict__ mag;
    const double* __restrict__ fcen;
    const double* __restrict__ cen;
    const double* __restrict__ vol;
    const double* __restrict__ pos;
    double side[3], inv[3];
    int32_t n, f;

    // tet_mesh::wrap (voronoi-cpp): the nearest periodic image of a separation.
    __device__ __forceinline__ double wrap(double d, int a) const { return d - side[a] * rint(d * inv[a]); }
    // Geometry::separation (finite_volume.hpp:282-285).
    __device__ __forceinline__ void separation(int i, int j, double* d) const {
#pragma unroll
        for (int a = 0; a < D; ++a) d[a] = wrap(pos[D * j + a] - pos[D * i + a], a);
    }
    // Geometry::face_offset (finite_volume.hpp:322-326): face centroid of f relative to the centroid of cell i.
    __device__ __forceinline__ void face_offset(int f, int i, double* out) const {
        const int o = owner[f];
        double rel[D];
        if (o == i) {
#pragma unroll
            for (int a = 0; a < D; ++a) rel[a] = fcen[D * f + a];
        } else {
            double s[D];
            separation(i, o, s);
#pragma unroll
            for (int a = 0; a < D; ++a) rel[a] = fcen[D * f + a] + s[a];
        }
#pragma unroll
        for (int a = 0; a < D; ++a) out[a] = rel[a] - cen[D * i + a];
    }
};

__device__ __forceinline__ int list_face(int32_t e) { return e >= 0 ? e : ~e; }

// One 256-bit read-only load (sm_100: a whole 32-B sector per lane, one request instead of four scalar ones).
// p must be 32-B aligned and unwritten during the kernel.
__device__ __forceinline__ void ldg256(const double* p, double* out) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(out[0]), "=d"(out[1]), "=d"(out[2]), "=d"(out[3]) : "l"(p));
}
__device__ __forceinline__ void ldg256(const float* p, float* out) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(out[0]), "=f"(out[1]), "=f"(out[2]), "=f"(out[3]), "=f"(out[4]), "=f"(out[5]), "=f"(out[6]), "=f"(out[7])
        : "l"(p));
}

// L2 eviction priority for rows streamed once per step (the rows gathered by every neighbour keep the default).
__device__ __forceinline__ unsigned long long l2_evict_first() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// Read-only loads with an L2 policy.
__device__ __forceinline__ unsigned int ldg_hint(const unsigned int* p, unsigned long long pol) {
    unsigned int v;
    asm("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ldg_hint(const double* p, unsigned long long pol) {
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ldg_hint(const float* p, unsigned long long pol) {
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double2 ldg_hint(const double2* p, unsigned long long pol) {
    double2 v;
    asm("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float2 ldg_hint(const float2* p, unsigned long long pol) {
    float2 v;
    asm("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ void ldg256_hint(const double* p, double* out, unsigned long long pol) {
    asm("ld.global.nc.L2::cache_hint.v4.f64 {%0, %1, %2, %3}, [%4], %5;"
        : "=d"(out[0]), "=d"(out[1]), "=d"(out[2]), "=d"(out[3])
        : "l"(p), "l"(pol));
}
__device__ __forceinline__ void ldg256_hint(const float* p, float* out, unsigned long long pol) {
    asm("ld.global.nc.L2::cache_hint.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8], %9;"
        : "=f"(out[0]), "=f"(out[1]), "=f"(out[2]), "=f"(out[3]), "=f"(out[4]), "=f"(out[5]), "=f"(out[6]), "=f"(out[7])
        : "l"(p), "l"(pol));
}
__device__ __forceinline__ void prefetch_l2_hint(const void* p, unsigned int bytes, unsigned long long pol) {
    asm volatile("cp.async.bulk.prefetch.L2.global.L2::cache_hint [%0], %1, %2;" ::"l"(p), "r"(bytes), "l"(pol) : "memory");
}

// A TMA bulk prefetch of [p, p + bytes) into L2 (p 16-B aligned, bytes a multiple of 16): one instruction per range,
// no registers or shared memory held while the data is in flight.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned int bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// A shared-memory load the compiler keeps where it is written (not hoisted, not merged with another).
__device__ __forceinline__ double lds_volatile(const double* p) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(static_cast<unsigned int>(__cvta_generic_to_shared(p))));
    return v;
}

// Asynchronous copies global -> shared (no registers held while in flight); cp_async_wait_all waits for this
// thread's copies, a barrier after it makes them visible to the block. 16 B: both addresses 16-B aligned; 8 B: 8-B.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned int s = static_cast<unsigned int>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned int s = static_cast<unsigned int>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// A merged row of the FP64 static per-face step: the cell's W (V doubles) then its gradient (V D), padded to whole
// 32-B sectors: 20 doubles (160 B, 5 sectors) in 3D against the 2 + 4 sectors of a primitive row and a gradient row.
template <int D>
constexpr int wg_stride() {
    return ((D + 2) * (D + 1) + 3) / 4 * 4;
}

// A cell's primitive row (W, c, r, pad: 64 B, 64-B aligned) in two vector loads (3D), one (2D: W only).
template <int D>
__device__ __forceinline__ void load_prim_row(const double* prims, int i, double* row) {
    const double* p = prims + 8 * static_cast<int64_t>(i);
    ldg256(p, row);
    ldg256(p + 4, row + 4);
}

// Counters a step's kernels write; read back with dt (one copy).
struct Counters {
    unsigned long long dt_bits;       // min over the time-step terms, as the bits of a positive double
    unsigned long long fallbacks[2];  // face sides that took the cell's state (pass 0, moving pass 1)
    unsigned long long error;         // bit 0 non-finite dt term, bit 1 non-finite state, bit 2 index out of range
};

__device__ __forceinline__ void block_min_to(double value, unsigned long long* target) {
    __shared__ double warp_min[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) value = fmin(value, __shfl_xor_sync(0xffffffffu, value, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_min[warp] = value;
    __syncthreads();
    if (warp == 0) {
        const int warps = (blockDim.x + 31) >> 5;
        value = lane < warps ? warp_min[lane] : 1.0e300;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) value = fmin(value, __shfl_xor_sync(0xffffffffu, value, o));
        // Positive doubles order as their bit patterns; NaN (skipped by fmin) and +inf never win.
        if (lane == 0 && value > 0.0 && value < 1.0e300) atomicMin(target, static_cast<unsigned long long>(__double_as_longlong(value)));
    }
}

// The warp's minimum (positive, finite values) into *target, without a block barrier.
__device__ __forceinline__ void warp_min_to(double value, unsigned long long* target) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) value = fmin(value, __shfl_xor_sync(0xffffffffu, value, o));
    if ((threadIdx.x & 31) == 0 && value > 0.0 && value < 1.0e300) atomicMin(target, static_cast<unsigned long long>(__double_as_longlong(value)));
}

__device__ __forceinline__ void block_sum_to(unsigned long long value, unsigned long long* target) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) value += __shfl_xor_sync(0xffffffffu, value, o);
    if ((threadIdx.x & 31) == 0 && value) atomicAdd(target, value);
}

// primitives() (finite_volume.hpp:403-415): W = primitive(Q / V), c = sqrt(gamma P / rho), r = radius(V).
template <int D>
__global__ void __launch_bounds__(256) k_primitives(MeshDev<D> m, const double* __restrict__ q, double* __restrict__ prims, GasDev gas) {
    constexpr int V = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    const double inv = 1.0 / m.vol[i];
    double U[V], W[V];
#pragma unroll
    for (int v = 0; v < V; ++v) U[v] = q[V * i + v] * inv;
    primitive<D>(U, gas, W);
    double* p = prims + PS * i;
#pragma unroll
    for (int v = 0; v < V; ++v) p[v] = W[v];
    p[V] = sqrt(gas.gamma * W[D + 1] / W[0]);
    p[V + 1] = radius<D>(m.vol[i]);
}

// |A| per face, once per mesh (the magnitudes the reference caches, finite_volume.hpp:1598-1601).
template <int D>
__global__ void k_magnitudes(const double* __restrict__ area, double* __restrict__ mag, int f_count) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= f_count) return;
    double a[D];
#pragma unroll
    for (int k = 0; k < D; ++k) a[k] = area[D * f + k];
    mag[f] = sqrt(dot<D>(a, a));
}

// Sweep::solve (finite_volume.hpp:591-615): M = L L^T by Cholesky, then every variable's fit; the gradient is x[1..D].
template <int D, class G>
__device__ __forceinline__ void cholesky_solve(G (&M)[D + 1][D + 1], G (&b)[D + 2][D + 1], G* grad) {
    constexpr int U = D + 1, V = D + 2;
    G L[U][U];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s < U; ++s) L[p][s] = G(0);
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s <= p; ++s) {
            G sum = M[s][p];
#pragma unroll
            for (int k = 0; k < s; ++k) sum -= L[p][k] * L[s][k];
            L[p][s] = p == s ? sqrt(sum) : sum / L[s][s];
        }
#pragma unroll
    for (int v = 0; v < V; ++v) {
        G z[U], x[U];
#pragma unroll
        for (int p = 0; p < U; ++p) {
            G sum = b[v][p];
#pragma unroll
            for (int k = 0; k < p; ++k) sum -= L[p][k] * z[k];
            z[p] = sum / L[p][p];
        }
#pragma unroll
        for (int p = U - 1; p >= 0; --p) {
            G sum = z[p];
#pragma unroll
            for (int k = p + 1; k < U; ++k) sum -= L[k][p] * x[k];
            x[p] = sum / L[p][p];
        }
#pragma unroll
        for (int a = 0; a < D; ++a) grad[D * v + a] = x[1 + a];
    }
}

template <class G>
__device__ __forceinline__ G finite_max();
template <>
__device__ __forceinline__ double finite_max<double>() {
    return 1.7976931348623157e308;
}
template <>
__device__ __forceinline__ float finite_max<float>() {
    return 3.40282347e38f;
}

// What a flux pass needs beyond the mesh: the state rows and the moving step's extra rows.
template <int D, class G>
struct FluxArgs {
    const double* __restrict__ q;
    const double* __restrict__ prims;
    const G* __restrict__ grad;
    const int32_t* __restrict__ steps;      // moving: grid steps per point over the step
    const double* __restrict__ old_cen;     // moving: centroids of t^n
    double dt;                              // the flux's dt (FaceFlux::dt)
    double unit;                            // moving: grid step / dt
    GasDev gas;
    const double* __restrict__ wg = nullptr;           // FP64 static per-face step: merged rows [N][wg_stride] (W, g)
    const double* __restrict__ w = nullptr;            // order-0 moving step: the point velocities [N][D]
    const uint16_t* __restrict__ grad16 = nullptr;    // Grad16: binary16 rows [N][16] instead of grad (G = float)
    const uint32_t* __restrict__ exponents = nullptr;  // Grad16: the three int8 group exponents of each row
    const double* __restrict__ dt_at = nullptr;        // set: dt read from device memory (the sweep's reduction)
};

// The group (0 rho, 1 the velocity, 2 P) of gradient component c = D v + a: each has its own exponent in a Grad16 row.
template <int D>
__host__ __device__ constexpr int half_group(int c) {
    return c < D ? 0 : c < D + D * D ? 1 : 2;
}
// 2^k as a float, k in [-126, 127] (exact).
__device__ __forceinline__ float two_to(int k) { return __uint_as_float(static_cast<uint32_t>(k + 127) << 23); }

// FaceFlux::side at order 1 (finite_volume.hpp:1306-1329): W + g . r - dt/2 A(W) g, or W if rho or P fall to <= 0.
// A cell's gradient row (GS values of G, 32-B aligned) in vector loads.
template <int D, class G>
__device__ __forceinline__ void load_grad_row(const G* grad, int i, G* row) {
    constexpr int GS = grad_stride<D>(), per = 32 / sizeof(G);
    const G* p = grad + static_cast<int64_t>(GS) * i;
#pragma unroll
    for (int c = 0; c < GS; c += per) ldg256(p + c, row + c);
}

// FaceFlux::gradient (finite_volume.hpp:1289-1302): a cell's gradient row; H (Grad16): one 32-B load of 16 binary16
// values, each decoded to float times 2^-k of its group.
template <int D, class G, bool H = false>
__device__ __forceinline__ void load_side_grad(const FluxArgs<D, G>& x, int i, G* g) {
    if constexpr (H && sizeof(G) == sizeof(float)) {
        constexpr int GS = grad_stride<D>();
        float raw[8];
        ldg256(reinterpret_cast<const float*>(x.grad16 + 16 * static_cast<int64_t>(i)), raw);
        const uint32_t k = __ldg(x.exponents + i);
        float scale[3];
#pragma unroll
        for (int s = 0; s < 3; ++s) scale[s] = two_to(-static_cast<int>(static_cast<int8_t>((k >> (8 * s)) & 0xffu)));
#pragma unroll
        for (int c = 0; c < GS; ++c) {
            const uint32_t pair = __float_as_uint(raw[c >> 1]);
            const unsigned short h = static_cast<unsigned short>(c & 1 ? pair >> 16 : pair & 0xffffu);
            g[c] = __half2float(__ushort_as_half(h)) * scale[half_group<D>(c)];
        }
    } else {
        load_grad_row<D, G>(x.grad, i, g);
    }
}

template <int D, class G, bool H = false, bool WG = false>
__device__ __forceinline__ void face_side(const FluxArgs<D, G>& x, int i, const double* r, double dt, double* Wf, int& fallbacks) {
    constexpr int V = D + 2, GS = grad_stride<D>();
    double W[V];
    G g[GS];
    if constexpr (WG && sizeof(G) == sizeof(double)) {  // one merged row: W then g
        constexpr int S = wg_stride<D>();
        double row[S];
        const double* p = x.wg + static_cast<int64_t>(S) * i;
#pragma unroll
        for (int c = 0; c < S; c += 4) ldg256(p + c, row + c);
#pragma unroll
        for (int v = 0; v < V; ++v) W[v] = row[v];
#pragma unroll
        for (int c = 0; c < V * D; ++c) g[c] = row[V + c];
    } else {
        double prow[8];
        load_prim_row<D>(x.prims, i, prow);
#pragma unroll
        for (int v = 0; v < V; ++v) W[v] = prow[v];
        load_side_grad<D, G, H>(x, i, g);
    }
    if constexpr (sizeof(G) == sizeof(double)) {
        double A[V];
        half_step_rate<D, double>(W, g, x.gas.gamma, A);
#pragma unroll
        for (int v = 0; v < V; ++v) Wf[v] = W[v] - 0.5 * dt * A[v];
#pragma unroll
        for (int v = 0; v < V; ++v) Wf[v] += dot<D>(g + D * v, r);
    } else {
        float Wg[V], rate[V], rg[D];
#pragma unroll
        for (int v = 0; v < V; ++v) Wg[v] = static_cast<float>(W[v]);
        half_step_rate<D, float>(Wg, g, static_cast<float>(x.gas.gamma), rate);
#pragma unroll
        for (int a = 0; a < D; ++a) rg[a] = static_cast<float>(r[a]);
        const float h = 0.5f * static_cast<float>(dt);
#pragma unroll
        for (int v = 0; v < V; ++v) Wf[v] = W[v] + static_cast<double>(dot<D>(g + D * v, rg) - h * rate[v]);
    }
    if (Wf[0] > 0 && Wf[D + 1] > 0) return;
    ++fallbacks;
#pragma unroll
    for (int v = 0; v < V; ++v) Wf[v] = W[v];
}

// MovingFlux<false>::pass_side (finite_volume.hpp:1457-1467): W + g . r on the mesh of t^n, no half step.
template <int D, class G, bool H = false>
__device__ __forceinline__ void pass1_side(const FluxArgs<D, G>& x, int i, const double* r, double* Wf, int& fallbacks) {
    constexpr int V = D + 2, GS = grad_stride<D>();
    double prow[8];
    load_prim_row<D>(x.prims, i, prow);
    double W[V];
#pragma unroll
    for (int v = 0; v < V; ++v) W[v] = prow[v];
    G g[GS];
    load_side_grad<D, G, H>(x, i, g);
    if constexpr (sizeof(G) == sizeof(double)) {
#pragma unroll
        for (int v = 0; v < V; ++v) Wf[v] = W[v] + dot<D>(g + D * v, r);
    } else {
        float rg[D];
#pragma unroll
        for (int a = 0; a < D; ++a) rg[a] = static_cast<float>(r[a]);
#pragma unroll
        for (int v = 0; v < V; ++v) Wf[v] = W[v] + static_cast<double>(dot<D>(g + D * v, rg));
    }
    if (Wf[0] > 0 && Wf[D + 1] > 0) return;
    ++fallbacks;
#pragma unroll
    for (int v = 0; v < V; ++v) Wf[v] = W[v];
}

// FaceFlux::solve (finite_volume.hpp:1400-1413): along the unit normal n; RF: in float in the face's frame.
template <int D, bool RF, int Riemann>
__device__ __forceinline__ void riemann_solve(const double* L, const double* R, const double* n, const double* wf, const GasDev& gas,
                                              double* F, bool moving) {
    constexpr int V = D + 2;
    if constexpr (!RF) {
        if constexpr (Riemann == 1)
            hll_flux<D>(L, R, n, wf, gas, F, moving);
        else
            hllc_flux<D, double>(L, R, n, wf, gas.gamma, gas.inverse_gm1, F, moving);
    } else {
        float Lf[V], Rf[V], nf[D], Ff[V], zero[D];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            Lf[v] = static_cast<float>(v >= 1 && v <= D ? L[v] - wf[v - 1] : L[v]);
            Rf[v] = static_cast<float>(v >= 1 && v <= D ? R[v] - wf[v - 1] : R[v]);
        }
#pragma unroll
        for (int a = 0; a < D; ++a) {
            nf[a] = static_cast<float>(n[a]);
            zero[a] = 0.0f;
        }
        hllc_flux<D, float>(Lf, Rf, nf, zero, static_cast<float>(gas.gamma), gas.inverse_gm1_float, Ff, false);
#pragma unroll
        for (int v = 0; v < V; ++v) F[v] = static_cast<double>(Ff[v]);
        if (moving) to_lab<D, double>(F, wf);
    }
}

// FaceFlux::face_velocity (finite_volume.hpp:1380-1397): the mean point velocity plus a correction along d, |c| <= 0.9|d|.
template <int D>
__device__ __forceinline__ void face_velocity(const MeshDev<D>& m, int f, int o, int j, const double* wL, const double* wR, double* out) {
    double d[D], c[D], dw[D];
    m.separation(o, j, d);
    const double dist = sqrt(dot<D>(d, d));
    const double inv_dist = 1.0 / dist;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        c[a] = m.fcen[D * f + a] - d[a] * 0.5;
        dw[a] = wL[a] - wR[a];
    }
    double facv = dot<D>(c, dw) * inv_dist;
    const double limit = 0.9 * dist, c2 = dot<D>(c, c);
    if (c2 > limit * limit) facv *= limit / sqrt(c2);
    const double s = facv * inv_dist;
#pragma unroll
    for (int a = 0; a < D; ++a) out[a] = (wL[a] + wR[a]) * 0.5 + d[a] * s;
}

// The flux through face f times |A| (FaceFlux::operator(), finite_volume.hpp:1415-1434; MovingFlux::operator(),
// :1469-1490). Pass: -1 static, 0 moving on the mesh of t^n, 1 moving on the mesh of t^n+1, 2 the order-0 moving step
// (FaceFlux<0, true>: each side the cell's W, the face velocity from the point velocities).
template <int D, int Order, int Pass, class G, bool RF, int Riemann, bool H = false>
__device__ __forceinline__ void face_flux(const MeshDev<D>& m, const FluxArgs<D, G>& x, int f, double* F, int& fb_o, int& fb_j) {
    constexpr int V = D + 2;
    const int o = m.owner[f], j = m.neighbour[f];
    double a[D];
#pragma unroll
    for (int k = 0; k < D; ++k) a[k] = m.area[D * f + k];
    const double magnitude = sqrt(dot<D>(a, a));
    if (magnitude == 0) {
#pragma unroll
        for (int v = 0; v < V; ++v) F[v] = 0;
        return;
    }
    double L[V], R[V], n[D], wf[D];
    const double inv = 1.0 / magnitude;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        n[k] = a[k] * inv;
        wf[k] = 0;
    }
    if constexpr (Pass == 2) {
        static_assert(Order == 0, "the order-0 moving step");
        face_velocity<D>(m, f, o, j, x.w + D * o, x.w + D * j, wf);
        double U[V];
        const double io = 1.0 / m.vol[o], ij = 1.0 / m.vol[j];
#pragma unroll
        for (int v = 0; v < V; ++v) U[v] = x.q[V * o + v] * io;
        primitive<D>(U, x.gas, L);
#pragma unroll
        for (int v = 0; v < V; ++v) U[v] = x.q[V * j + v] * ij;
        primitive<D>(U, x.gas, R);
    } else if constexpr (Pass < 0) {
        if constexpr (Order == 0) {
            double U[V];
            const double io = 1.0 / m.vol[o], ij = 1.0 / m.vol[j];
#pragma unroll
            for (int v = 0; v < V; ++v) U[v] = x.q[V * o + v] * io;
            primitive<D>(U, x.gas, L);
#pragma unroll
            for (int v = 0; v < V; ++v) U[v] = x.q[V * j + v] * ij;
            primitive<D>(U, x.gas, R);
        } else {
            double ro[D], rj[D];
            m.face_offset(f, o, ro);
            m.face_offset(f, j, rj);
            face_side<D, G, H>(x, o, ro, x.dt, L, fb_o);
            face_side<D, G, H>(x, j, rj, x.dt, R, fb_j);
        }
    } else {
        double wo[D], wj[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            wo[k] = static_cast<double>(x.steps[D * o + k]) * x.unit;
            wj[k] = static_cast<double>(x.steps[D * j + k]) * x.unit;
        }
        face_velocity<D>(m, f, o, j, wo, wj, wf);
        double ro[D], rj[D];
        m.face_offset(f, o, ro);
        m.face_offset(f, j, rj);
        if constexpr (Pass == 0) {
            pass1_side<D, G, H>(x, o, ro, L, fb_o);
            pass1_side<D, G, H>(x, j, rj, R, fb_j);
        } else {
            double r2[D];
#pragma unroll
            for (int k = 0; k < D; ++k) r2[k] = ro[k] + m.cen[D * o + k] - x.old_cen[D * o + k] + wo[k] * (0.5 * x.dt);
            face_side<D, G, H>(x, o, r2, x.dt, L, fb_o);
#pragma unroll
            for (int k = 0; k < D; ++k) r2[k] = rj[k] + m.cen[D * j + k] - x.old_cen[D * j + k] + wj[k] * (0.5 * x.dt);
            face_side<D, G, H>(x, j, r2, x.dt, R, fb_j);
        }
    }
    riemann_solve<D, RF, Riemann>(L, R, n, wf, x.gas, F, Pass >= 0);
#pragma unroll
    for (int v = 0; v < V; ++v) F[v] *= magnitude;
}

// Flux rows in the precision policy's flux storage (Precision::flux, precision.hpp:26-39; FaceFluxes, finite_volume.hpp:65):
// double rows of V values, or float rows rounded once as the reference's static_cast<FluxStore> does, padded to 8 floats
// (3D, one 32-B sector) or 4 (2D, 16 B) so that a row is one aligned vector store and one aligned vector load.
template <int D, class FS>
__host__ __device__ constexpr int flux_stride() {
    return sizeof(FS) == sizeof(double) ? D + 2 : (D == 3 ? 8 : 4);
}
template <int D, class FS>
__device__ __forceinline__ void store_flux_row(FS* flux, int64_t f, const double* F) {
    constexpr int V = D + 2;
    if constexpr (sizeof(FS) == sizeof(double)) {
#pragma unroll
        for (int v = 0; v < V; ++v) flux[V * f + v] = F[v];
    } else {
        constexpr int S = flux_stride<D, FS>();
        float r[S];
#pragma unroll
        for (int c = 0; c < S; ++c) r[c] = c < V ? static_cast<float>(F[c]) : 0.0f;
        float4* p = reinterpret_cast<float4*>(flux + S * f);
#pragma unroll
        for (int c = 0; c < S; c += 4) p[c / 4] = make_float4(r[c], r[c + 1], r[c + 2], r[c + 3]);
    }
}

// apply()'s flux pass (finite_volume.hpp:1591-1602): one flux row per face.
#ifndef LUNA_KFLUX_MIN_BLOCKS_F
#define LUNA_KFLUX_MIN_BLOCKS_F 8  // the float policies' flux passes over the mesh arrays (the moving step's); measured at
#endif                             // 128^3 (moving hydro ms): unbounded (72-80 registers) 4.70, 7 blocks 4.20, 8 4.16
template <int D, int Order, int Pass, class G, bool RF, int Riemann, bool H = false, class FS = double>
__global__ void __launch_bounds__(128, sizeof(G) == sizeof(float) ? LUNA_KFLUX_MIN_BLOCKS_F : 1) k_flux(MeshDev<D> m, FluxArgs<D, G> x, FS* __restrict__ flux,
                                              unsigned long long* __restrict__ fallbacks) {
    constexpr int V = D + 2;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    int count = 0;
    if (f < m.f) {
        double F[V];
        face_flux<D, Order, Pass, G, RF, Riemann, H>(m, x, f, F, count, count);
        store_flux_row<D, FS>(flux, f, F);
    }
    block_sum_to(static_cast<unsigned long long>(count), fallbacks);
}

// A flux row of V doubles at p (8-B aligned) through the 32-B aligned 64-B window that holds it (V <= 5: a row starts at
// most 24 B into its window): two 256-bit loads instead of V scalar ones, the row picked out of the window by its offset
// (V = 4: rows are 32 B, aligned, one load). The buffer must be 32-B aligned and extend at least 24 B past its last row.
template <int V>
__device__ __forceinline__ void load_row_windowed(const double* p, double* row) {
    static_assert(V == 4 || V == 5, "2D or 3D flux rows");
    if constexpr (V == 4) {  // 32-B rows of a 32-B aligned buffer: one load
        double w[4];
        ldg256(p, w);
#pragma unroll
        for (int v = 0; v < 4; ++v) row[v] = w[v];
    } else {
        const uintptr_t a = reinterpret_cast<uintptr_t>(p);
        const double* w = reinterpret_cast<const double*>(a & ~static_cast<uintptr_t>(31));
        const int off = static_cast<int>((a >> 3) & 3);
        double win[8];
        ldg256(w, win);
        ldg256(w + 4, win + 4);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double lo = (off & 1) ? win[v + 1] : win[v];
            const double hi = (off & 1) ? win[v + 3] : win[v + 2];
            row[v] = (off & 2) ? hi : lo;
        }
    }
}

// The end of a cell's update (finite_volume.hpp:1603-1615): Q_i -= dt sum, the error word's bit 1 if not finite; NextPrims:
// the next primitive rows (Windowed: the library's rows, 16-B vector stores).
template <int D, bool NextPrims, bool Windowed>
__device__ __forceinline__ void update_cell(const MeshDev<D>& m, double* __restrict__ q, int i, const double (&sum)[D + 2], double dt,
                                            double* __restrict__ prims, const GasDev& gas, Counters* __restrict__ ctr) {
    constexpr int V = D + 2;
    double next[V];
    bool finite = true;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        next[v] = q[V * i + v] - dt * sum[v];
        q[V * i + v] = next[v];
        finite = finite && isfinite(next[v]);
    }
    if (!finite) atomicOr(&ctr->error, 2ull);
    if constexpr (NextPrims) {
        const double inv = 1.0 / m.vol[i];
        double U[V], W[V];
#pragma unroll
        for (int v = 0; v < V; ++v) U[v] = next[v] * inv;
        primitive<D>(U, gas, W);
        double row[PS];
#pragma unroll
        for (int v = 0; v < V; ++v) row[v] = W[v];
        row[V] = sqrt(gas.gamma * W[D + 1] / W[0]);
        row[V + 1] = radius<D>(m.vol[i]);
#pragma unroll
        for (int c = V + 2; c < PS; ++c) row[c] = 0.0;
        if constexpr (Windowed) {
            double2* p = reinterpret_cast<double2*>(prims + PS * static_cast<int64_t>(i));
#pragma unroll
            for (int c = 0; c < PS; c += 2) p[c / 2] = make_double2(row[c], row[c + 1]);
        } else {
            double* p = prims + PS * i;
#pragma unroll
            for (int c = 0; c < V + 2; ++c) p[c] = row[c];
        }
    }
}

// apply()'s update (finite_volume.hpp:1603-1615): Q_i -= dt sum_k sign_k F_k in list order; NextPrims: the next
// primitive rows (a moving step's second pass; here every per-face step, which makes the next primitives() pass free).
// Windowed: flux rows through load_row_windowed (the library's own flux buffer, padded for it).
// The library's update (windowed rows): resident blocks of 256 its registers are cut for, and the entries whose rows are
// requested together; measured at 128^3 (update ms, every policy alike): 1 / 4 0.395, 4 / 2 0.391, 4 / 3 0.410,
// 4 / 4 0.444 (spills), 3 / 6 0.477. The no-allocation path's instantiation keeps 1 / 4.
#ifndef LUNA_UPDATE_MIN_BLOCKS
#define LUNA_UPDATE_MIN_BLOCKS 4
#endif
#ifndef LUNA_UPDATE_BATCH
#define LUNA_UPDATE_BATCH 2
#endif
#ifndef LUNA_UPDATE_MIN_BLOCKS_F
#define LUNA_UPDATE_MIN_BLOCKS_F LUNA_UPDATE_MIN_BLOCKS  // single's float flux rows
#endif
#ifndef LUNA_UPDATE_BATCH_F
#define LUNA_UPDATE_BATCH_F LUNA_UPDATE_BATCH  // single's float flux rows (32-B rows, half the registers a row)
#endif
// FS = float: the rows of store_flux_row, one aligned vector load each, widened to double before the sum (the
// reference's static_cast<double>(F(f, v)), finite_volume.hpp:1607).
template <int D, bool NextPrims, bool Windowed = false, class FS = double>
__global__ void __launch_bounds__(256, Windowed ? (sizeof(FS) == sizeof(float) ? LUNA_UPDATE_MIN_BLOCKS_F : LUNA_UPDATE_MIN_BLOCKS) : 1) k_update(MeshDev<D> m, double* __restrict__ q, const FS* __restrict__ flux, double dt,
                                                double* __restrict__ prims, GasDev gas, Counters* __restrict__ ctr) {
    constexpr int V = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double sum[V];
#pragma unroll
    for (int v = 0; v < V; ++v) sum[v] = 0;
    const int first = m.start[i], end = m.start[i + 1];
    // kBatch entries at a time: their list words, then their flux rows, are all requested before any is used (the
    // gathers of a list are independent); the sums stay in list order.
    constexpr int kBatch = Windowed ? (sizeof(FS) == sizeof(float) ? LUNA_UPDATE_BATCH_F : LUNA_UPDATE_BATCH) : 4;
    for (int k0 = first; k0 < end; k0 += kBatch) {
        int32_t e[kBatch];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) e[b] = k0 + b < end ? m.list[k0 + b] : 0;
        double row[kBatch][V];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            if (k0 + b < end) {
                if constexpr (sizeof(FS) == sizeof(float)) {
                    constexpr int S = flux_stride<D, FS>();
                    const float* r = reinterpret_cast<const float*>(flux) + S * static_cast<int64_t>(list_face(e[b]));
                    float w[8];
                    if constexpr (S == 8) {
                        ldg256(r, w);
                    } else {
                        const float4 t = __ldg(reinterpret_cast<const float4*>(r));
                        w[0] = t.x, w[1] = t.y, w[2] = t.z, w[3] = t.w;
                    }
#pragma unroll
                    for (int v = 0; v < V; ++v) row[b][v] = static_cast<double>(w[v]);
                } else {
                    const double* r = reinterpret_cast<const double*>(flux) + V * static_cast<int64_t>(list_face(e[b]));
                    if constexpr (Windowed) {
                        load_row_windowed<V>(r, row[b]);
                    } else {
#pragma unroll
                        for (int v = 0; v < V; ++v) row[b][v] = __ldg(r + v);
                    }
                }
            }
        }
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            if (k0 + b >= end) break;
            const double sign = e[b] >= 0 ? 1.0 : -1.0;
#pragma unroll
            for (int v = 0; v < V; ++v) sum[v] += sign * row[b][v];
        }
    }
    update_cell<D, NextPrims, Windowed>(m, q, i, sum, dt, prims, gas, ctr);
}

// apply()'s per-cell loop (finite_volume.hpp:1543-1562): each cell computes the fluxes of its faces itself, in list order.
template <int D, int Order, class G, bool RF, int Riemann, bool H = false>
__global__ void __launch_bounds__(128) k_fluxes_and_update(MeshDev<D> m, FluxArgs<D, G> x, double* __restrict__ next, double dt,
                                                           Counters* __restrict__ ctr) {
    constexpr int V = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int count = 0;
    if (i < m.n) {
        double sum[V];
#pragma unroll
        for (int v = 0; v < V; ++v) sum[v] = 0;
        for (int k = m.start[i]; k < m.start[i + 1]; ++k) {
            const int32_t e = m.list[k];
            const int f = list_face(e);
            int fo = 0, fj = 0;
            double F[V];
            face_flux<D, Order, -1, G, RF, Riemann, H>(m, x, f, F, fo, fj);
            const bool owned = e >= 0;
            count += owned ? fo : fj;
            const double sign = owned ? 1.0 : -1.0;
#pragma unroll
            for (int v = 0; v < V; ++v) sum[v] += sign * F[v];
        }
        bool finite = true;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            next[V * i + v] = x.q[V * i + v] - dt * sum[v];
            finite = finite && isfinite(next[V * i + v]);
        }
        if (!finite) atomicOr(&ctr->error, 2ull);
    }
    block_sum_to(static_cast<unsigned long long>(count), &ctr->fallbacks[0]);
}

// The moving step's start (finite_volume.hpp:1506-1514): keep the centroids of t^n, snap the points to the mesh grid,
// their move over dt as whole grid steps.
template <int D>
__global__ void k_keep_centroids(int n, const double* __restrict__ cen, double* __restrict__ old_cen, double* __restrict__ x,
                                 const double* __restrict__ w, int32_t* __restrict__ steps, double dt, double step, double per_step,
                                 long long p0, long long p1, long long p2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long period[3] = {p0, p1, p2};
#pragma unroll
    for (int a = 0; a < D; ++a) {
        old_cen[D * i + a] = cen[D * i + a];
        const long long p = period[a];
        long long k0 = llround(x[D * i + a] * per_step);
        k0 = ((k0 % p) + p) % p;
        long long k1 = llround((x[D * i + a] + dt * w[D * i + a]) * per_step);
        k1 = ((k1 % p) + p) % p;
        x[D * i + a] = static_cast<double>(k0) * step;
        long long d = k1 - k0;
        if (d > p / 2) d -= p;
        if (d < -(p / 2)) d += p;
        steps[D * i + a] = static_cast<int32_t>(d);
    }
}

// move() of the order-0 moving step (finite_volume.hpp:1212-1228, off the grid): x + dt w, wrapped into the box.
template <int D>
__global__ void k_drift_free(int n, double* __restrict__ x, const double* __restrict__ w, double dt, double s0, double s1, double s2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double side[3] = {s0, s1, s2};
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const double moved = x[D * i + a] + dt * w[D * i + a];
        x[D * i + a] = moved - side[a] * floor(moved / side[a]);
    }
}

// move()'s drift on the grid (finite_volume.hpp:1219-1231).
template <int D>
__global__ void k_drift(int n, double* __restrict__ x, const int32_t* __restrict__ steps, double step, double per_step, long long p0,
                        long long p1, long long p2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long period[3] = {p0, p1, p2};
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const long long k = llround(x[D * i + a] * per_step) + steps[D * i + a];
        const long long p = period[a];
        x[D * i + a] = static_cast<double>(((k % p) + p) % p) * step;
    }
}

}  // namespace luna
