// The mesh reordered for the step's kernels, once per mesh (a static mesh: once; a moving mesh: after each remesh).
//
// luna-cpp's sweep and flux kernels walk voronoi-cpp's lists and recompute the same geometry every step: each list entry
// costs three dependent loads (list -> face -> neighbour -> rows) plus the separation, the fit row X = [1, d + c_j - c_i]
// and the face offset. Everything there except the neighbours' primitive rows depends on the mesh only, so this pass
// computes it once, in the reference's arithmetic, into rows that the step streams in list order:
//   entries          per list entry: the entry's row of the cell's gradient operator c_k (see k_geometry) instead of
//                    the fit's sums, the face offset x_f - c_i, the neighbour as a row of the tile's staged cells
//                    (tiles.h), whether the cell owns the face and whether the face is below 1e-6 of the cell's
//                    surface; sliced by 32 cells (a warp): entry k of the slice's lane l sits at
//                    (slice_base + k) * 32 + l, each field in an array of its own, so a warp's load of entry k of its
//                    32 cells is one contiguous run;
//   face rows [F]    the unit normal A / |A|, |A|, both cells' face offsets and the two cells (FaceFlux, :1415-1434);
//   cell angle [N]   the largest AREPO face angle of the cell (the moving mesh's regularisation, :509, :526-537).
// The sweep runs one block per tile: it stages the primitive rows and generators of the tile's cells and of their
// neighbours into shared memory, then each thread walks its cell's streamed entries and reads the neighbours' rows
// there, so no list entry waits on a gather from HBM.
#pragma once

#include <cuda_bf16.h>

#include <type_traits>

#include "kernels.cuh"
#include "tiles.h"

namespace luna {

template <class G>
using Pair = typename std::conditional<sizeof(G) == sizeof(double), double2, float2>::type;

constexpr unsigned int kOwnedBit = 0x80000000u, kTinyBit = 0x40000000u, kIndexMask = 0x3fffffffu;

// A face's row for the flux pass: n = A / |A| (double in every policy: grad32 solves in double; riemann32 rounds it to
// float itself, as FaceFlux::solve does), |A|, the cells, and the face offsets from each cell's centroid in G.
struct alignas(32) FaceRow64 {
    double n[3];
    double mag;
    double offo[3];
    int o, j;
    double offj[3];
    double pad;
};
struct alignas(32) FaceRow32 {
    double n[3];
    double mag;
    float offo[3];
    float offj[3];
    int o, j;
};
template <class G>
using FaceRow = typename std::conditional<sizeof(G) == sizeof(double), FaceRow64, FaceRow32>::type;

// A staged row in shared memory (12 doubles, 96 B): the cell's primitive row (W, c, r, pad: as in HBM), then its
// generator (D doubles).
constexpr int kStagedDoubles = 12;
constexpr int kStagedPos = 8;

template <int D, class G>
struct GeometryDev {
    const int32_t* __restrict__ order;        // [tiles * kTileCells]: thread t sweeps cell order[t] (-1: idle)
    const int32_t* __restrict__ slice_base;   // [tiles * kTileCells / 32 + 1], in slots of 32 entries
    const int32_t* __restrict__ stage_start;  // [tiles + 1]
    const int32_t* __restrict__ stage_cells;  // each tile's staged cells: its own in thread order, then the halo
    unsigned int* __restrict__ nbr;           // staged row of the neighbour | tiny << 30 | owned << 31
    Pair<G>* __restrict__ c01;                // gradient operator row c_k, x and y
    G* __restrict__ c2;                       // z (3D)
    Pair<G>* __restrict__ off01;              // face offset x, y
    G* __restrict__ off2;                     // z (3D)
    FaceRow<G>* __restrict__ faces;           // [F]
    double* __restrict__ max_angle;           // [N]
    double* __restrict__ reach2;              // [N]: the largest |x_f - c_i|^2 over the cell's faces
    int64_t threads;                          // tiles * kTileCells
};

// One thread a cell (in sweep order): the cell's geometry in list order. The least-squares fit of Sweep (an area-
// weighted fit with intercept over the face neighbours, finite_volume.hpp:486-515, 591-615) is linear in the
// neighbours' differences: x_v = M^-1 sum_k w_k X_k (W_kv - W_iv) with M = sum_k w_k X_k X_k^T, so the gradient is
// g_v = sum_k c_k (W_kv - W_iv) with c_k = rows 1..D of M^-1 w_k X_k. M, its Cholesky factor and each c_k are formed
// here in double, in the reference's order; the sweep then only sums c_k times the differences. Also the face rows of
// the faces the cell owns and the largest face angle. g.nbr holds each entry's staged row on entry (from the host's
// tiles); the kernel adds the owned and tiny bits.
// Both walks take the list in batches of LUNA_GEOMETRY_BATCH entries whose loads are all issued before any is used:
// the entries' list words, then their faces' cells and |A| (and the face's centroid), then the neighbours' generators
// and centroids. The cell's own generator is read once and each face offset is formed from the loaded rows. The
// arithmetic is the per-entry one, in list order. Measured on the 128^3 moving blast's hydro part (the rows rebuilt
// every step): batches of 1, 2, 4 entries 5.16, 5.44, 6.08 ms a step (the larger batches' registers cost occupancy),
// against 5.8 ms before the own generator and the offsets were taken from registers; 16 lanes a cell (the fit's sums
// by a shuffle tree) 6.55 ms.
#ifndef LUNA_GEOMETRY_BATCH
#define LUNA_GEOMETRY_BATCH 1
#endif
// FaceRows: also the static flux pass's face rows (a moving mesh's flux passes read the mesh arrays, not the rows).
// One block a tile, tiles [tile0, tile0 + gridDim.x). Staged: the generators and centroids of the tile's staged cells
// (its own and the halo, tiles.h) copied into shared memory first (2 D doubles a row), each entry's neighbour read there
// through its staged row (the tiler's entry words) instead of through the face's owner / neighbour; the same values, so
// the same rows.
#ifndef LUNA_GEOMETRY_MIN_BLOCKS
#define LUNA_GEOMETRY_MIN_BLOCKS 5  // measured at 128^3 (moving hydro ms): unbounded (114 registers) 4.70, 5 4.62, 6 4.69
#endif
template <int D, class G, bool FaceRows = true, bool Staged = false>
__global__ void __launch_bounds__(128, LUNA_GEOMETRY_MIN_BLOCKS) k_geometry(MeshDev<D> m, GeometryDev<D, G> g, int tile0) {
    constexpr int U = D + 1, B = LUNA_GEOMETRY_BATCH;
    extern __shared__ double geo_rows[];  // Staged: [staged rows][2 D]: generator, centroid
    const int tile = tile0 + static_cast<int>(blockIdx.x);
    const int64_t t = static_cast<int64_t>(tile) * kTileCells + threadIdx.x;
    int s0 = 0;
    if constexpr (Staged) {
        s0 = g.stage_start[tile];
        const int staged = g.stage_start[tile + 1] - s0;
        for (int r = threadIdx.x; r < staged; r += kTileCells) {
            const int c = g.stage_cells[s0 + r];
#pragma unroll
            for (int a = 0; a < D; ++a) {
                geo_rows[2 * D * r + a] = m.pos[D * static_cast<int64_t>(c) + a];
                geo_rows[2 * D * r + D + a] = m.cen[D * static_cast<int64_t>(c) + a];
            }
        }
        __syncthreads();
    }
    if (t >= g.threads) return;
    const int i = g.order[t];
    if (i < 0) return;
    double centroid[D], pi[D];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        centroid[a] = m.cen[D * i + a];
        pi[a] = m.pos[D * i + a];
    }
    const int first = m.start[i], end = m.start[i + 1];
    const int64_t slot0 = static_cast<int64_t>(g.slice_base[t >> 5]) * 32 + (t & 31);
    double surface = 0, smallest = __longlong_as_double(0x7ff0000000000000ll), max_angle = 0;
    double M[U][U];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s < U; ++s) M[p][s] = 0;
    for (int k0 = first; k0 < end; k0 += B) {
        int32_t e[B];
        int j[B];
        double mag[B], pj[B][D], cj[B][D];
#pragma unroll
        for (int b = 0; b < B; ++b) e[b] = k0 + b < end ? m.list[k0 + b] : 0;
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int f = list_face(e[b]);
            if constexpr (Staged)
                j[b] = k0 + b < end ? static_cast<int>(g.nbr[slot0 + 32 * static_cast<int64_t>(k0 + b - first)] & kIndexMask) : 0;
            else
                j[b] = k0 + b < end ? (e[b] >= 0 ? m.neighbour[f] : m.owner[f]) : i;
            mag[b] = k0 + b < end ? m.mag[f] : 0.0;
        }
#pragma unroll
        for (int b = 0; b < B; ++b)
#pragma unroll
            for (int a = 0; a < D; ++a) {
                if constexpr (Staged) {  // j: the staged row
                    pj[b][a] = geo_rows[2 * D * j[b] + a];
                    cj[b][a] = geo_rows[2 * D * j[b] + D + a];
                } else {
                    pj[b][a] = m.pos[D * j[b] + a];
                    cj[b][a] = m.cen[D * j[b] + a];
                }
            }
#pragma unroll
        for (int b = 0; b < B; ++b) {
            if (k0 + b >= end) break;
            double d[D];
#pragma unroll
            for (int a = 0; a < D; ++a) d[a] = m.wrap(pj[b][a] - pi[a], a);  // Geometry::separation(i, j)
            const double magnitude = mag[b];
            surface += magnitude;
            smallest = fmin(smallest, magnitude);
            const double d2 = dot<D>(d, d);
            max_angle = fmax(max_angle, face_angle<D>(magnitude) / (0.5 * sqrt(d2)));
            double X[U];
            X[0] = 1;
#pragma unroll
            for (int p = 1; p < U; ++p) X[p] = d[p - 1] + cj[b][p - 1] - centroid[p - 1];
#pragma unroll
            for (int p = 0; p < U; ++p)
#pragma unroll
                for (int s = p; s < U; ++s) M[p][s] += magnitude * X[p] * X[s];
        }
    }
    double L[U][U];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s < U; ++s) L[p][s] = 0;
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s <= p; ++s) {
            double sum = M[s][p];
#pragma unroll
            for (int q = 0; q < s; ++q) sum -= L[p][q] * L[s][q];
            L[p][s] = p == s ? sqrt(sum) : sum / L[s][s];
        }
    const double tiny = 1e-6 * surface;
    const bool any_tiny = smallest < tiny;
    double reach2 = 0;
    for (int k0 = first; k0 < end; k0 += B) {
        int32_t e[B];
        int j[B];
        double mag[B], fc[B][D], pj[B][D], cj[B][D];
#pragma unroll
        for (int b = 0; b < B; ++b) e[b] = k0 + b < end ? m.list[k0 + b] : 0;
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int f = list_face(e[b]);
            const bool in = k0 + b < end;
            if constexpr (Staged)
                j[b] = in ? static_cast<int>(g.nbr[slot0 + 32 * static_cast<int64_t>(k0 + b - first)] & kIndexMask) : 0;
            else
                j[b] = in ? (e[b] >= 0 ? m.neighbour[f] : m.owner[f]) : i;
            mag[b] = in ? m.mag[f] : 0.0;
#pragma unroll
            for (int a = 0; a < D; ++a) fc[b][a] = in ? m.fcen[D * f + a] : 0.0;
        }
#pragma unroll
        for (int b = 0; b < B; ++b)
#pragma unroll
            for (int a = 0; a < D; ++a) {
                if constexpr (Staged) {
                    pj[b][a] = geo_rows[2 * D * j[b] + a];
                    cj[b][a] = geo_rows[2 * D * j[b] + D + a];
                } else {
                    pj[b][a] = m.pos[D * j[b] + a];
                    cj[b][a] = m.cen[D * j[b] + a];
                }
            }
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int k = k0 + b;
            if (k >= end) break;
            const int f = list_face(e[b]);
            const bool owned = e[b] >= 0;
            const int64_t slot = slot0 + 32 * static_cast<int64_t>(k - first);
            // c_k: M^-1 (w X_k) by the factor, rows 1..D
            double d[D], z[U], x[U], wX[U];
#pragma unroll
            for (int a = 0; a < D; ++a) d[a] = m.wrap(pj[b][a] - pi[a], a);
            const double magnitude = mag[b];
            wX[0] = magnitude;
#pragma unroll
            for (int p = 1; p < U; ++p) wX[p] = magnitude * (d[p - 1] + cj[b][p - 1] - centroid[p - 1]);
#pragma unroll
            for (int p = 0; p < U; ++p) {
                double sum = wX[p];
#pragma unroll
                for (int q = 0; q < p; ++q) sum -= L[p][q] * z[q];
                z[p] = sum / L[p][p];
            }
#pragma unroll
            for (int p = U - 1; p >= 0; --p) {
                double sum = z[p];
#pragma unroll
                for (int q = p + 1; q < U; ++q) sum -= L[q][p] * x[q];
                x[p] = sum / L[p][p];
            }
            g.c01[slot] = Pair<G>{static_cast<G>(x[1]), static_cast<G>(x[2])};
            if constexpr (D == 3) g.c2[slot] = static_cast<G>(x[3]);
            // Geometry::face_offset(f, i): the face centroid (relative to the owner) moved to i's generator when the
            // owner is the other cell, minus i's centroid
            double off[D];
#pragma unroll
            for (int a = 0; a < D; ++a) off[a] = (owned ? fc[b][a] : fc[b][a] + d[a]) - centroid[a];
            g.off01[slot] = Pair<G>{static_cast<G>(off[0]), static_cast<G>(off[1])};
            if constexpr (D == 3) g.off2[slot] = static_cast<G>(off[2]);
            {
                double r2 = 0;
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    const double o = static_cast<double>(static_cast<G>(off[a]));
                    r2 += o * o;
                }
                reach2 = fmax(reach2, r2);
            }
            const bool tiny_face = any_tiny && magnitude < tiny;
            g.nbr[slot] = (g.nbr[slot] & kIndexMask) | (owned ? kOwnedBit : 0u) | (tiny_face ? kTinyBit : 0u);
            if (FaceRows && owned) {  // the face row, written once by the owner
                double a[D];
#pragma unroll
                for (int q = 0; q < D; ++q) a[q] = m.area[D * f + q];
                const double amag = sqrt(dot<D>(a, a));
                // face_offset(f, j): the owner i seen from j, minus j's centroid
                double offj[D];
#pragma unroll
                for (int q = 0; q < D; ++q) offj[q] = (fc[b][q] + m.wrap(pi[q] - pj[b][q], q)) - cj[b][q];
                FaceRow<G> r;
                const double inv = amag == 0 ? 0.0 : 1.0 / amag;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    r.n[q] = q < D ? a[q] * inv : 0.0;
                    if constexpr (sizeof(G) == sizeof(double)) {
                        r.offo[q] = q < D ? off[q] : 0.0;
                        r.offj[q] = q < D ? offj[q] : 0.0;
                    } else {
                        r.offo[q] = q < D ? static_cast<float>(off[q]) : 0.0f;
                        r.offj[q] = q < D ? static_cast<float>(offj[q]) : 0.0f;
                    }
                }
                r.mag = amag;
                r.o = i;
                if constexpr (Staged)
                    r.j = g.stage_cells[s0 + j[b]];
                else
                    r.j = j[b];
                if constexpr (sizeof(G) == sizeof(double)) r.pad = 0;
                g.faces[f] = r;
            }
        }
    }
    g.max_angle[i] = max_angle;
    g.reach2[i] = reach2;
}

// The sweep over the reordered rows (Sweep<Moving, Grad>::operator(), finite_volume.hpp:463-569), one block per tile:
// the block stages the primitive rows and generators of the tile's cells and their neighbours into shared memory (the
// rows are independent: all copies are in flight at once); then walk 1 sums the gradient g_v = sum_k c_k (W_jv - W_iv)
// in list order, the neighbours' range (tiny faces left out) and the owned faces' CFL terms (FaceStep, :1074-1090,
// the separation formed from the staged generators); walk 2 clips at each face offset in list order. Per entry: the
// streamed coalesced entry rows and one shared-memory row.
// The learned limiter's 32 features of a cell (FP64 policy: lo/hi are the neighbours' values): per variable v,
//   alpha_v / 2                        the admissible factor (how far the slope may steepen or must flatten),
//   (W_v - lo_v) / (hi_v - lo_v) - 1/2 where the cell sits in its neighbours' range,
//   tanh(|g_v| r / (hi_v - lo_v))      the unlimited slope across the cell relative to the range (smoothness),
//   tanh((hi_v - lo_v) / scale_v)      the size of the range relative to the values (a jump or a smooth region);
// then tanh(log(hi_P / lo_P)) (a pressure jump), tanh(|v| / c), min_v min(alpha_v, 1) (the plain limiter's strongest
// clip), 1, and zeros.
template <int D, class G>
__device__ __forceinline__ void write_learned_inputs(const struct LearnedInputs& out, int i, const double* Wi, double c, double r, const G* g,
                                                     const G* lo, const G* hi, const double* alpha);

// The learned limiter's inputs, written by the sweep in its learned mode (see write_learned_inputs). Dense (cells null):
// row i is cell i. Compact: only cells whose slopes are not round-off get a row (their factor is the network's; the
// others keep the factor 1, the plain limiter's there), taken in arrival order; cells[row] names the row's cell and
// *count ends as the number of rows.
struct LearnedInputs {
    __nv_bfloat16* features;  // [rows][32]
    double* alpha;            // [rows][5]: the admissible slope factor per variable
    int* cells;               // [N] or null (dense)
    unsigned int* count;      // the compact rows taken (reset to 0 before the sweep)
};
constexpr double kAlphaCap = 2.0;  // the largest steepening the learned limiter may choose

// The Grad16 policy's gradient storage (Sweep::store with P::half, finite_volume.hpp:616-641): rows of 16 binary16
// values (32 B) and a word of three int8 group exponents per cell; null rows: the gradients are stored as G.
struct HalfRows {
    uint16_t* rows;
    uint32_t* exponents;
};

// Each group (rho, the velocity, P) scaled by 2^k that puts its largest magnitude in [2^14, 2^15) (k = 0 for an all-zero
// group, within [-114, 126]; precision.hpp half::group_exponent), rounded to binary16 (nearest, ties to even).
template <int D>
__device__ __forceinline__ void store_half_row(const HalfRows& out, int i, const float* g) {
    constexpr int V = D + 2;
    float largest[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int c = 0; c < V * D; ++c) largest[half_group<D>(c)] = fmaxf(largest[half_group<D>(c)], fabsf(g[c]));
    int k[3];
    float scale[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const int e = static_cast<int>((__float_as_uint(largest[s]) >> 23) & 0xffu) - 127;
        k[s] = largest[s] > 0.0f ? min(max(14 - e, -114), 126) : 0;
        scale[s] = two_to(k[s]);
    }
    uint32_t packed[8];
#pragma unroll
    for (int w = 0; w < 8; ++w) packed[w] = 0;
#pragma unroll
    for (int c = 0; c < V * D; ++c)
        packed[c >> 1] |= static_cast<uint32_t>(__half_as_ushort(__float2half_rn(g[c] * scale[half_group<D>(c)]))) << (16 * (c & 1));
    uint4* dst = reinterpret_cast<uint4*>(out.rows + 16 * static_cast<int64_t>(i));
    dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
    dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
    out.exponents[i] = static_cast<uint32_t>(static_cast<uint8_t>(static_cast<int8_t>(k[0]))) |
                       static_cast<uint32_t>(static_cast<uint8_t>(static_cast<int8_t>(k[1]))) << 8 |
                       static_cast<uint32_t>(static_cast<uint8_t>(static_cast<int8_t>(k[2]))) << 16;
}

// Resident blocks per SM the register budget is cut for, and the entries whose streamed rows are requested together;
// measured at 128^3 FP64 (sweep ms): 3 blocks / 4 entries 1.74, 4 / 2 1.31 (a few spilled registers), 5 / 1 1.65.
#ifndef LUNA_SWEEP_MIN_BLOCKS
#define LUNA_SWEEP_MIN_BLOCKS 4
#endif
#ifndef LUNA_SWEEP_MIN_BLOCKS_F
#define LUNA_SWEEP_MIN_BLOCKS_F LUNA_SWEEP_MIN_BLOCKS  // the float policies' sweep
#endif
#ifndef LUNA_SWEEP_BATCH
#define LUNA_SWEEP_BATCH 0  // 0: 2 entries in FP64, 3 in the float policies (128^3 sweep ms: FP64 2: 0.748, 1: 0.760,
                            // 3: 0.794; riemann32 3: 0.536, 2: 0.545)
#endif
#ifndef LUNA_SWEEP_L2_PREFETCH
#define LUNA_SWEEP_L2_PREFETCH 2  // TMA bulk prefetches into L2: 1 the walk-1 entry rows at block start, 2 also walk 2's
#endif                            // (measured at 128^3 FP64, sweep ms: none 0.800, 1: 0.775, 2: 0.772)
#ifndef LUNA_CLIP_BATCH
#define LUNA_CLIP_BATCH 4  // entries of the clip walk whose offset rows are requested together
#endif
// Limit: 0 none, 1 the plain face-centroid limiter, 2 the learned limiter's inputs (the gradient left unlimited).
// KB: entries whose streamed rows are requested together. Launched with blocks of kTileCells threads over tiles [tile0, tile0 + gridDim.x) and the shared memory of the most
// rows one of them stages (kStagedDoubles doubles a row).
template <int D, bool Moving, bool Grad, class G, int Limit, int KB = LUNA_SWEEP_BATCH,
          int MINB = sizeof(G) == sizeof(double) ? LUNA_SWEEP_MIN_BLOCKS : LUNA_SWEEP_MIN_BLOCKS_F>
__global__ void __launch_bounds__(kTileCells, MINB) k_sweep_tiles(MeshDev<D> m, GeometryDev<D, G> geo, int tile0, const double* __restrict__ prims,
                                                               G* __restrict__ grad_out, double* __restrict__ w_out, double courant,
                                                               double round_off2, Counters* __restrict__ ctr, LearnedInputs learned,
                                                               HalfRows half, double* __restrict__ wg_out) {
    extern __shared__ double2 staged_rows[];
    double* rows = reinterpret_cast<double*>(staged_rows);
    constexpr int V = D + 2, GS = grad_stride<D>(), R = kStagedDoubles;
    constexpr bool exact = sizeof(G) == sizeof(double);
    const int tile = tile0 + static_cast<int>(blockIdx.x);
    const int64_t t = static_cast<int64_t>(tile) * kTileCells + threadIdx.x;
    const int i = geo.order[t];
    const int count = i >= 0 ? m.start[i + 1] - m.start[i] : 0;
    const int64_t row0 = static_cast<int64_t>(geo.slice_base[t >> 5]) * 32;  // the warp's first slot
    const int64_t slot0 = row0 + (t & 31);
    const unsigned long long once = l2_evict_first();  // entry rows are read once per step
#if LUNA_SWEEP_L2_PREFETCH
    if ((threadIdx.x & 31) == 0) {  // the warp's walk-1 entry rows, on their way to L2 while the block stages
        const int64_t rows = geo.slice_base[(t >> 5) + 1] - geo.slice_base[t >> 5];
        if (rows > 0) {
            prefetch_l2(geo.nbr + row0, static_cast<unsigned int>(rows * 32 * sizeof(unsigned int)));
            if constexpr (Grad) {
                prefetch_l2(geo.c01 + row0, static_cast<unsigned int>(rows * 32 * sizeof(Pair<G>)));
                if constexpr (D == 3) prefetch_l2(geo.c2 + row0, static_cast<unsigned int>(rows * 32 * sizeof(G)));
            }
        }
    }
#endif
    {
        const int s0 = geo.stage_start[tile], staged = geo.stage_start[tile + 1] - s0;
        constexpr int kRowsInFlight = 4;
        for (int r0 = 0; r0 < staged; r0 += kRowsInFlight * kTileCells) {
            int cell[kRowsInFlight];
#pragma unroll
            for (int b = 0; b < kRowsInFlight; ++b) {
                const int r = r0 + b * kTileCells + static_cast<int>(threadIdx.x);
                cell[b] = r < staged ? geo.stage_cells[s0 + r] : -1;
            }
#pragma unroll
            for (int b = 0; b < kRowsInFlight; ++b) {
                if (cell[b] < 0) continue;
                double* dst = rows + R * (r0 + b * kTileCells + static_cast<int>(threadIdx.x));
                const double* src = prims + PS * static_cast<int64_t>(cell[b]);
#pragma unroll
                for (int q = 0; q < PS; q += 2) cp_async16(dst + q, src + q);
#pragma unroll
                for (int a = 0; a < D; ++a) cp_async8(dst + kStagedPos + a, m.pos + D * static_cast<int64_t>(cell[b]) + a);
            }
        }
        cp_async_wait_all();
        __syncthreads();
    }
    double smallest_dt = 1.0e300;
    if (i >= 0) {
        // the cell's own row: tile cells are staged first, in thread order
        const double* own = rows + R * threadIdx.x;
        double Wi[V];
#pragma unroll
        for (int v = 0; v < V; ++v) Wi[v] = own[v];
        // The own row's sound speed, radius and generator are read from shared memory where they are used. FP64:
        // volatile loads, not held in registers through walk 1, whose double sums need them all (measured at 128^3:
        // the sweep 0.772 -> 0.747 ms); the float policies have registers to spare and keep them (0.546 against 0.601).
        double held[3 + D];  // the float policies: c, r, the generator, read once
        if constexpr (!exact) {
            held[0] = own[V];
            held[1] = own[V + 1];
#pragma unroll
            for (int a = 0; a < D; ++a) held[2 + a] = own[kStagedPos + a];
        }
        const auto own_at = [own, &held](int k) -> double {
            if constexpr (exact) return lds_volatile(own + k);
            else return k == V ? held[0] : k == V + 1 ? held[1] : held[2 + k - kStagedPos];
        };
        G lo[V], hi[V], g[V * D];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            lo[v] = finite_max<G>();
            hi[v] = -finite_max<G>();
#pragma unroll
            for (int a = 0; a < D; ++a) g[D * v + a] = G(0);
        }
        // kBatch entries at a time: their streamed rows are all requested before any is used; the staged rows they
        // name are shared-memory reads.
        constexpr int kBatch = KB > 0 ? KB : (exact ? 2 : 3);
        // The smallest face term courant (dist + r) / vsig, vsig = c_i + c_j - dv.d / dist (FaceStep), held as the
        // fraction num / den = (dist + r) dist / ((c_i + c_j) dist - dv.d) and compared by cross products: one division
        // a cell instead of two a face (the same minimum, rounded once).
        double best_num = 1.0e300, best_den = 1.0;
        bool any_tiny = false;  // a face below 1e-6 of the surface (rare): walk 2 then reads the entry words again
        for (int k0 = 0; k0 < count; k0 += kBatch) {
            unsigned int word[kBatch];
            G c[kBatch][D];
#pragma unroll
            for (int b = 0; b < kBatch; ++b) {
                const int64_t slot = slot0 + 32 * static_cast<int64_t>(k0 + b);
                if (k0 + b < count) {
                    word[b] = ldg_hint(geo.nbr + slot, once);
                    if constexpr (Grad) {
                        const Pair<G> c01 = ldg_hint(geo.c01 + slot, once);
                        c[b][0] = c01.x;
                        c[b][1] = c01.y;
                        if constexpr (D == 3) c[b][2] = ldg_hint(geo.c2 + slot, once);
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < kBatch; ++b) {
                if (k0 + b >= count) break;
                const bool owned = (word[b] & kOwnedBit) != 0, tiny_face = (word[b] & kTinyBit) != 0;
                any_tiny = any_tiny || tiny_face;
                const double* rj = rows + R * static_cast<int>(word[b] & kIndexMask);
                double pj[8];
#pragma unroll
                for (int q = 0; q < 6; q += 2) {
                    const double2 w2 = *reinterpret_cast<const double2*>(rj + q);
                    pj[q] = w2.x;
                    pj[q + 1] = w2.y;
                }
                if (owned) {  // FaceStep (finite_volume.hpp:1074-1090)
                    const double2 w2 = *reinterpret_cast<const double2*>(rj + 6);
                    pj[6] = w2.x;
                    pj[7] = w2.y;
                    double dv[D], d[D];
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        dv[a] = pj[1 + a] - Wi[1 + a];
                        d[a] = m.wrap(rj[kStagedPos + a] - own_at(kStagedPos + a), a);  // Geometry::separation of owner and neighbour
                    }
                    const double dist = sqrt(dot<D>(d, d));
                    // Both cells' terms: the smaller radius gives the smaller one. den > 0 is vsig > 0.
                    const double num = (dist + fmin(own_at(V + 1), pj[V + 1])) * dist, den = (own_at(V) + pj[V]) * dist - dot<D>(dv, d);
                    if (den > 0 && num * best_den < best_num * den) {
                        best_num = num;
                        best_den = den;
                    }
                }
                if constexpr (Grad) {
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        const double dW = pj[v] - Wi[v];
                        const G dWg = static_cast<G>(dW);
#pragma unroll
                        for (int a = 0; a < D; ++a) g[D * v + a] += c[b][a] * dWg;
                        if (!tiny_face) {
                            const G value = exact ? static_cast<G>(pj[v]) : dWg;
                            lo[v] = fmin(lo[v], value);
                            hi[v] = fmax(hi[v], value);
                        }
                    }
                }
            }
        }
        if (best_num < 1.0e300) smallest_dt = courant * (best_num / best_den);
        const double ci = own_at(V), ri = own_at(V + 1);
        double wi[D];
#pragma unroll
        for (int a = 0; a < D; ++a) wi[a] = Wi[1 + a];
        if constexpr (Moving) {
            const double max_angle = geo.max_angle[i];
            const double factor = 2.25, speed = 0.5;
            double fraction = 0;
            if (max_angle > 0.75 * factor) fraction = max_angle > factor ? speed : speed * (max_angle - 0.75 * factor) / (0.25 * factor);
            double centroid[D];
#pragma unroll
            for (int a = 0; a < D; ++a) centroid[a] = m.cen[D * i + a];
            const double cd = sqrt(dot<D>(centroid, centroid));
            if (cd > 0 && fraction > 0) {
                const double s = fraction * ci / cd;
#pragma unroll
                for (int a = 0; a < D; ++a) wi[a] = wi[a] + centroid[a] * s;
            }
#pragma unroll
            for (int a = 0; a < D; ++a) w_out[D * i + a] = wi[a];
        }
        {
            double rel[D];
#pragma unroll
            for (int a = 0; a < D; ++a) rel[a] = Wi[1 + a] - (Moving ? wi[a] : 0.0);
            smallest_dt = fmin(smallest_dt, courant * (ri / (ci + sqrt(dot<D>(rel, rel)))));
        }
        if constexpr (Grad) {
            // A slope that moves every face value of its variable by at most the policy's round-off of the variable's
            // scale (|g_v| max_k |r_k| <= e s_v; s = |rho|, |v| + c for the velocity components, |P|; e = 2^-50 when
            // the face states are solved in double, 2^-24 when the Riemann solve rounds them to float) is round-off of
            // a uniform region, where a clip could change face states only at that level; when every variable's slope
            // is such, walk 2 is left out (the learned limiter's inputs then take the admissible factor 1, the plain
            // limiter's choice there). The step then differs from the reference's arithmetic only at that level in
            // those cells' face states. round_off2 = e^2.
            bool round_off_only = false;
            if constexpr (Limit != 0) {
                const double reach2 = geo.reach2[i];
                const double kNoise2 = round_off2;
                double speed2 = 0;
#pragma unroll
                for (int a = 0; a < D; ++a) speed2 += Wi[1 + a] * Wi[1 + a];
                const double signal = sqrt(speed2) + ci;
                round_off_only = true;
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    double gg = 0;
#pragma unroll
                    for (int a = 0; a < D; ++a) gg += static_cast<double>(g[D * v + a]) * static_cast<double>(g[D * v + a]);
                    const double scale = (v >= 1 && v <= D) ? signal : fabs(Wi[v]);
                    round_off_only = round_off_only && gg * reach2 <= kNoise2 * (scale * scale);
                }
            }
#if LUNA_SWEEP_L2_PREFETCH >= 2
            if constexpr (Limit != 0) {  // the warp's walk-2 offset rows, when a lane of it clips
                const unsigned int here = __activemask();
                const unsigned int need = __ballot_sync(here, !round_off_only);
                if (need && static_cast<int>(threadIdx.x & 31) == __ffs(here) - 1) {
                    const int64_t rows = geo.slice_base[(t >> 5) + 1] - geo.slice_base[t >> 5];
                    prefetch_l2(geo.off01 + row0, static_cast<unsigned int>(rows * 32 * sizeof(Pair<G>)));
                    if constexpr (D == 3) prefetch_l2(geo.off2 + row0, static_cast<unsigned int>(rows * 32 * sizeof(G)));
                }
            }
#endif
            if constexpr (Limit == 2) if (!(learned.cells && round_off_only)) {
                // The admissible factor per variable: the smallest over the faces (tiny ones left out) of the factor that
                // puts the face value on its bound, max(room, 0) / |dp|, the min-factor form of the limiter
                // (finite_volume.hpp:1008-1034), here capped at kAlphaCap instead of 1; held as a fraction and compared
                // by cross products (one division a variable).
                double alpha[V], num[V], den[V];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    num[v] = round_off_only ? 1.0 : kAlphaCap;
                    den[v] = 1.0;
                }
                for (int k = 0; k < (round_off_only ? 0 : count); ++k) {
                    const int64_t slot = slot0 + 32 * static_cast<int64_t>(k);
                    if (any_tiny && (ldg_hint(geo.nbr + slot, once) & kTinyBit)) continue;
                    const Pair<G> o01 = ldg_hint(geo.off01 + slot, once);
                    G rg[D];
                    rg[0] = o01.x;
                    rg[1] = o01.y;
                    if constexpr (D == 3) rg[2] = ldg_hint(geo.off2 + slot, once);
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        const double dp = static_cast<double>(dot<D>(g + D * v, rg));
                        if (dp == 0) continue;
                        const double room = dp > 0 ? static_cast<double>(hi[v]) - Wi[v] : Wi[v] - static_cast<double>(lo[v]);
                        const double n = room > 0 ? room : 0.0, d = fabs(dp);
                        if (n * den[v] < num[v] * d) {
                            num[v] = n;
                            den[v] = d;
                        }
                    }
                }
#pragma unroll
                for (int v = 0; v < V; ++v) alpha[v] = num[v] / den[v];
                int row = i;
                if (learned.cells) {  // one atomic a warp: the lanes here take consecutive rows
                    const unsigned int here = __activemask();
                    const int lane = static_cast<int>(threadIdx.x & 31), leader = __ffs(here) - 1;
                    unsigned int base = 0;
                    if (lane == leader) base = atomicAdd(learned.count, static_cast<unsigned int>(__popc(here)));
                    base = __shfl_sync(here, base, leader);
                    row = static_cast<int>(base) + __popc(here & ((1u << lane) - 1u));
                    learned.cells[row] = i;
                }
                write_learned_inputs<D>(learned, row, Wi, ci, ri, g, lo, hi, alpha);
            }
            if constexpr (Limit == 1 && exact) if (!round_off_only) {
                // The clip (Sweep walk 2, finite_volume.hpp:538-565): each face in list order (tiny ones left out)
                // scales a variable's gradient so that its face value stays in [lo, hi].
                constexpr int kClipBatch = LUNA_CLIP_BATCH;
                for (int k0 = 0; k0 < count; k0 += kClipBatch) {
                    unsigned int word[kClipBatch];
                    G rg[kClipBatch][D];
#pragma unroll
                    for (int b = 0; b < kClipBatch; ++b) {
                        const int64_t slot = slot0 + 32 * static_cast<int64_t>(k0 + b);
                        if (k0 + b < count) {
                            word[b] = any_tiny ? ldg_hint(geo.nbr + slot, once) : 0u;
                            const Pair<G> o01 = ldg_hint(geo.off01 + slot, once);
                            rg[b][0] = o01.x;
                            rg[b][1] = o01.y;
                            if constexpr (D == 3) rg[b][2] = ldg_hint(geo.off2 + slot, once);
                        }
                    }
#pragma unroll
                    for (int b = 0; b < kClipBatch; ++b) {
                        if (k0 + b >= count) break;
                        if (word[b] & kTinyBit) continue;
#pragma unroll
                        for (int v = 0; v < V; ++v) {
                            G* gv = g + D * v;
                            const G dp = dot<D>(gv, rg[b]);
                            if (dp > 0 && Wi[v] + dp > hi[v]) {
                                const G s = hi[v] > Wi[v] ? (hi[v] - Wi[v]) / dp : G(0);
#pragma unroll
                                for (int a = 0; a < D; ++a) gv[a] = gv[a] * s;
                            } else if (dp < 0 && Wi[v] + dp < lo[v]) {
                                const G s = lo[v] < Wi[v] ? (lo[v] - Wi[v]) / dp : G(0);
#pragma unroll
                                for (int a = 0; a < D; ++a) gv[a] = gv[a] * s;
                            }
                        }
                    }
                }
            }
            if constexpr (Limit == 1 && !exact) if (!round_off_only) {
                // The float policies' clip (the range is of differences, lo <= 0 <= hi) in its min-factor form
                // (finite_volume.hpp:1008-1034): scaling g by each face's factor in list order ends at g times the
                // smallest factor, since after a clip the face sits on its bound and a later face clips again only
                // with a smaller one. Per variable the smallest room / |dp| over the faces is held as a fraction and
                // compared by cross products: no division in the walk, one per clipped variable (measured: the
                // grad32 sweep 0.91 -> 0.80 ms at 128^3; the FP64 sweep keeps the list-order form, which is faster
                // there).
                G best_num[V], best_den[V];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    best_num[v] = G(1);
                    best_den[v] = G(1);
                }
                constexpr int kClipBatch = LUNA_CLIP_BATCH;
                for (int k0 = 0; k0 < count; k0 += kClipBatch) {
                    unsigned int word[kClipBatch];
                    G rg[kClipBatch][D];
#pragma unroll
                    for (int b = 0; b < kClipBatch; ++b) {
                        const int64_t slot = slot0 + 32 * static_cast<int64_t>(k0 + b);
                        if (k0 + b < count) {
                            word[b] = any_tiny ? ldg_hint(geo.nbr + slot, once) : 0u;
                            const Pair<G> o01 = ldg_hint(geo.off01 + slot, once);
                            rg[b][0] = o01.x;
                            rg[b][1] = o01.y;
                            if constexpr (D == 3) rg[b][2] = ldg_hint(geo.off2 + slot, once);
                        }
                    }
#pragma unroll
                    for (int b = 0; b < kClipBatch; ++b) {
                        if (k0 + b >= count) break;
                        if (word[b] & kTinyBit) continue;
#pragma unroll
                        for (int v = 0; v < V; ++v) {
                            const G dp = dot<D>(g + D * v, rg[b]);
                            const G room = dp > G(0) ? hi[v] : -lo[v], size = fabs(dp);
                            if (dp != G(0) && size > room) {  // the face value would leave the range
                                const G num = room > G(0) ? room : G(0);
                                if (num * best_den[v] < best_num[v] * size) {
                                    best_num[v] = num;
                                    best_den[v] = size;
                                }
                            }
                        }
                    }
                }
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    if (best_num[v] < best_den[v]) {
                        const G s = best_num[v] / best_den[v];
#pragma unroll
                        for (int a = 0; a < D; ++a) g[D * v + a] = g[D * v + a] * s;
                    }
                }
            }
            bool stored = false;
            if constexpr (!exact)
                if (half.rows) {
                    store_half_row<D>(half, i, g);
                    stored = true;
                }
            if constexpr (exact)
                if (wg_out) {  // the merged row of the static per-face step: W (as staged) then g
                    constexpr int S = wg_stride<D>();
                    double row[S];
#pragma unroll
                    for (int v = 0; v < V; ++v) row[v] = Wi[v];
#pragma unroll
                    for (int c = 0; c < V * D; ++c) row[V + c] = g[c];
#pragma unroll
                    for (int c = V + V * D; c < S; ++c) row[c] = 0.0;
                    double2* dst = reinterpret_cast<double2*>(wg_out + static_cast<int64_t>(S) * i);
#pragma unroll
                    for (int c = 0; c < S; c += 2) dst[c / 2] = make_double2(row[c], row[c + 1]);
                    stored = true;
                }
            if (!stored) {  // the row in 16-B vector stores (pad zeroed)
                G row[GS];
#pragma unroll
                for (int c = 0; c < GS; ++c) row[c] = c < V * D ? g[c] : G(0);
                using Vec16 = typename std::conditional<sizeof(G) == sizeof(double), double2, float4>::type;
                constexpr int per = 16 / static_cast<int>(sizeof(G));
                Vec16* out = reinterpret_cast<Vec16*>(grad_out + static_cast<int64_t>(GS) * i);
#pragma unroll
                for (int c = 0; c < GS; c += per) {
                    if constexpr (sizeof(G) == sizeof(double))
                        out[c / per] = make_double2(row[c], row[c + 1]);
                    else
                        out[c / per] = make_float4(row[c], row[c + 1], row[c + 2], row[c + 3]);
                }
            }
        }
    }
    warp_min_to(smallest_dt, &ctr->dt_bits);  // no block barrier: a warp done with its lists leaves
    if (i >= 0 && !(smallest_dt == smallest_dt)) atomicOr(&ctr->error, 1ull);
}

// The network's slot of variable v, by role in every dimension: density 0, velocity components 1 .. D, pressure 4 (in 2D
// slot 3, the z velocity's, stays empty), so that one network serves 2D and 3D meshes.
template <int D>
__host__ __device__ constexpr int learned_slot(int v) {
    return v == D + 1 ? 4 : v;
}

template <int D, class G>
__device__ __forceinline__ void write_learned_inputs(const LearnedInputs& out, int i, const double* Wi, double c, double r, const G* g,
                                                     const G* lo, const G* hi, const double* alpha) {
    constexpr int V = D + 2;
    float f[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) f[k] = 0.0f;
    double plain = 1.0;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        if (v >= V) break;
        const double range = static_cast<double>(hi[v]) - static_cast<double>(lo[v]);
        const double scale = fabs(Wi[v]) + fabs(static_cast<double>(hi[v])) + fabs(static_cast<double>(lo[v])) + 1e-300;
        const double safe = range > 1e-12 * scale ? range : 1e-12 * scale;
        double gn = 0;
#pragma unroll
        for (int a = 0; a < D; ++a) gn += static_cast<double>(g[D * v + a]) * static_cast<double>(g[D * v + a]);
        gn = sqrt(gn);
        const double pos = fmin(fmax((Wi[v] - static_cast<double>(lo[v])) / safe, -1.0), 2.0);
        const int slot = learned_slot<D>(v);
        f[4 * slot + 0] = static_cast<float>(alpha[v] / kAlphaCap);
        f[4 * slot + 1] = static_cast<float>(pos - 0.5);
        f[4 * slot + 2] = tanhf(static_cast<float>(gn * r / safe));  // the features are BF16: float is ample
        f[4 * slot + 3] = tanhf(static_cast<float>(range / scale * 3.0));
        plain = fmin(plain, fmin(alpha[v], 1.0));
        out.alpha[5 * static_cast<int64_t>(i) + v] = alpha[v];
    }
    const double plo = fmax(static_cast<double>(lo[D + 1]), 1e-300), phi = fmax(static_cast<double>(hi[D + 1]), plo);
    double speed = 0;
#pragma unroll
    for (int a = 0; a < D; ++a) speed += Wi[1 + a] * Wi[1 + a];
    f[20] = tanhf(logf(static_cast<float>(phi / plo)));
    f[21] = tanhf(static_cast<float>(sqrt(speed) / fmax(c, 1e-300)));
    f[22] = static_cast<float>(plain);
    f[23] = 1.0f;
    __nv_bfloat16* row = out.features + 32 * static_cast<int64_t>(i);
#pragma unroll
    for (int k = 0; k < 32; k += 2) *reinterpret_cast<__nv_bfloat162*>(row + k) = __floats2bfloat162_rn(f[k], f[k + 1]);
}

// The learned slope factors applied to the rows of LearnedInputs (dense: row s is cell s; compact: cells[s], the first
// *count rows): g_v *= alpha_v sigmoid(logit_v) (use_net), or min(alpha_v, 1), the plain limiter's factor in min-factor
// form (a check of alpha against the plain sweep).
template <int D>
__global__ void k_apply_factors(int rows, const int* __restrict__ cells, const unsigned int* __restrict__ count, double* __restrict__ grad,
                                const double* __restrict__ alpha, const float* __restrict__ logits, bool use_net) {
    constexpr int V = D + 2, GS = grad_stride<D>();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= rows || (count && s >= static_cast<int>(*count))) return;
    const int64_t i = cells ? cells[s] : s;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const double a = alpha[5 * static_cast<int64_t>(s) + v];
        double phi;
        if (use_net) {
            const double o = logits[16 * static_cast<int64_t>(s) + learned_slot<D>(v)];
            phi = a / (1.0 + exp(-o));
        } else {
            phi = fmin(a, 1.0);
        }
#pragma unroll
        for (int d = 0; d < D; ++d) grad[GS * i + D * v + d] *= phi;
    }
}

// The static flux pass over the face rows (FaceFlux::operator(), finite_volume.hpp:1415-1434): one streamed row per
// face, then the two cells' primitive and gradient rows.
// Resident blocks per SM the flux pass's registers are cut for; measured at 128^3 FP64 (fluxes ms): unbounded (96
// registers, 5 blocks) 0.80-0.84, 6 blocks 0.77 (0.699 with the later rows), 7 blocks 0.767, 8 blocks 1.03 (spills).
#ifndef LUNA_FLUX_MIN_BLOCKS
#define LUNA_FLUX_MIN_BLOCKS 6
#endif
#ifndef LUNA_FLUX_MIN_BLOCKS_F
#define LUNA_FLUX_MIN_BLOCKS_F 8  // the float policies' flux pass (128^3 single, fluxes ms: 6 blocks 0.534, 7 0.492, 8 0.458)
#endif
// One face row, 32-B aligned, in vector loads (streamed once per step: evict-first in L2).
template <class G>
__device__ __forceinline__ void load_face_row(const FaceRow<G>* p, FaceRow<G>& r) {
    double* words = reinterpret_cast<double*>(&r);
    const unsigned long long once = l2_evict_first();
#pragma unroll
    for (int c = 0; c < static_cast<int>(sizeof(FaceRow<G>) / 8); c += 4) ldg256_hint(reinterpret_cast<const double*>(p) + c, words + c, once);
}

// The flux of one face row (FaceFlux::operator() :1415-1434): both sides' face states from the cells' rows, the Riemann
// solve in the face's frame, times the area. count: the sides that fell back to the cell's state.
template <int D, int Order, class G, bool RF, int Riemann, bool H, bool WG>
__device__ __forceinline__ void row_flux(const MeshDev<D>& m, const FluxArgs<D, G>& x, const FaceRow<G>& r, double (&F)[D + 2], int& count) {
    constexpr int V = D + 2;
    if (r.mag == 0) {
#pragma unroll
        for (int v = 0; v < V; ++v) F[v] = 0;
        return;
    }
    double L[V], R[V], n[D], wf[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        n[k] = r.n[k];
        wf[k] = 0;
    }
    if constexpr (Order == 0) {
        double U[V];
        const double io = 1.0 / m.vol[r.o], ij = 1.0 / m.vol[r.j];
#pragma unroll
        for (int v = 0; v < V; ++v) U[v] = x.q[V * r.o + v] * io;
        primitive<D>(U, x.gas, L);
#pragma unroll
        for (int v = 0; v < V; ++v) U[v] = x.q[V * r.j + v] * ij;
        primitive<D>(U, x.gas, R);
    } else {
        double ro[D], rj[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            ro[k] = static_cast<double>(r.offo[k]);
            rj[k] = static_cast<double>(r.offj[k]);
        }
        face_side<D, G, H, WG>(x, r.o, ro, x.dt, L, count);
        face_side<D, G, H, WG>(x, r.j, rj, x.dt, R, count);
    }
    riemann_solve<D, RF, Riemann>(L, R, n, wf, x.gas, F, false);
#pragma unroll
    for (int v = 0; v < V; ++v) F[v] *= r.mag;
}

template <int D, int Order, class G, bool RF, int Riemann, bool H = false, bool WG = false, class FS = double>
__global__ void __launch_bounds__(128, sizeof(G) == sizeof(double) ? LUNA_FLUX_MIN_BLOCKS : LUNA_FLUX_MIN_BLOCKS_F) k_flux_rows(MeshDev<D> m, GeometryDev<D, G> geo, FluxArgs<D, G> x, FS* __restrict__ flux,
                                                   unsigned long long* __restrict__ fallbacks) {
    constexpr int V = D + 2;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    int count = 0;
    if (x.dt_at) x.dt = *x.dt_at;  // launched behind the sweep before the host has read the dt
    if (f < m.f) {
        FaceRow<G> r;
        load_face_row<G>(geo.faces + f, r);
        double F[V];
        row_flux<D, Order, G, RF, Riemann, H, WG>(m, x, r, F, count);
        store_flux_row<D, FS>(flux, f, F);
    }
    block_sum_to(static_cast<unsigned long long>(count), fallbacks);
}

// The fused flux-and-update pass of a static FP64 mesh (apply(), :1538-1631), one block a sweep tile (tiles.h
// TileFaces): the tile's interior face rows (contiguous, tile order) prefetched into L2 by one bulk copy and solved into
// shared memory, then each cell of the tile sums its faces' fluxes in list order, from shared memory or, for a face
// between tiles, from the crossing pass's flux row in HBM, and updates Q and its next primitive row. The same fluxes and
// the same sums in the same order as k_flux_rows then k_update: the same bits.
#ifndef LUNA_FUSED_MIN_BLOCKS
#define LUNA_FUSED_MIN_BLOCKS 6
#endif
template <int D, int Riemann>
__global__ void __launch_bounds__(kTileCells, LUNA_FUSED_MIN_BLOCKS) k_tile_flux_update(MeshDev<D> m, FluxArgs<D, double> x, const int32_t* __restrict__ order,
                                                                                       const int32_t* __restrict__ tstart, const FaceRow64* __restrict__ trows,
                                                                                       const int32_t* __restrict__ eslot, const double* __restrict__ xflux,
                                                                                       double* q, double dt, double* __restrict__ prims,
                                                                                       Counters* __restrict__ ctr) {
    constexpr int V = D + 2;
    extern __shared__ double tile_flux[];  // [interior faces][V]
    const int tile = blockIdx.x;
    const int s0 = tstart[tile], slots = tstart[tile + 1] - s0;
    if (threadIdx.x == 0 && slots > 0) prefetch_l2(trows + s0, static_cast<unsigned int>(slots * sizeof(FaceRow64)));
    int count = 0;
    for (int j = threadIdx.x; j < slots; j += kTileCells) {
        FaceRow64 r;
        load_face_row<double>(trows + s0 + j, r);
        double F[V];
        row_flux<D, 1, double, false, Riemann, false, true>(m, x, r, F, count);
#pragma unroll
        for (int v = 0; v < V; ++v) tile_flux[V * j + v] = F[v];
    }
    __syncthreads();
    const int i = order[static_cast<int64_t>(tile) * kTileCells + threadIdx.x];
    if (i >= 0) {
        double sum[V];
#pragma unroll
        for (int v = 0; v < V; ++v) sum[v] = 0;
        const int first = m.start[i], end = m.start[i + 1];
        constexpr int kBatch = 4;  // the entries' words, then their rows, requested before any is summed
        for (int k0 = first; k0 < end; k0 += kBatch) {
            int32_t e[kBatch];
#pragma unroll
            for (int b = 0; b < kBatch; ++b) e[b] = k0 + b < end ? eslot[k0 + b] : 0;
            double row[kBatch][V];
#pragma unroll
            for (int b = 0; b < kBatch; ++b) {
                const int32_t w = e[b] >= 0 ? e[b] : ~e[b];
                if (k0 + b < end && (w & kCrossing)) load_row_windowed<V>(xflux + V * static_cast<int64_t>(w & ~kCrossing), row[b]);
            }
#pragma unroll
            for (int b = 0; b < kBatch; ++b) {
                if (k0 + b >= end) break;
                const int32_t w = e[b] >= 0 ? e[b] : ~e[b];
                if (!(w & kCrossing))
#pragma unroll
                    for (int v = 0; v < V; ++v) row[b][v] = tile_flux[V * w + v];
                const double sign = e[b] >= 0 ? 1.0 : -1.0;
#pragma unroll
                for (int v = 0; v < V; ++v) sum[v] += sign * row[b][v];
            }
        }
        update_cell<D, true, true>(m, q, i, sum, dt, prims, x.gas, ctr);
    }
    block_sum_to(static_cast<unsigned long long>(count), &ctr->fallbacks[0]);
}

// rows[k] = faces[index[k]] (Gather: the face rows of the fused pass, interior in tile order, crossing in face order),
// or faces[index[k]] = rows[k] (the face-ordered rows back, for a step that leaves the fused pass).
template <class G, bool Gather>
__global__ void k_move_face_rows(FaceRow<G>* __restrict__ faces, const int32_t* __restrict__ index, int64_t count, FaceRow<G>* __restrict__ rows) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= count) return;
    if (Gather)
        rows[k] = faces[index[k]];
    else
        faces[index[k]] = rows[k];
}

}  // namespace luna
