// libluna_b200: the C ABI of include/luna_b200.h over the sm_100a kernels of kernels.cuh.
//
// A luna_fv mirrors luna-cpp's FiniteVolume<D> (src/hydro/finite_volume.hpp:47-239): it owns Q and its rows, copies the
// caller's mesh arrays once per mesh, and runs time_step() (primitives, the sweep with the CFL reduction riding in it) and
// step() (face fluxes, then the per-cell update in list order, which also writes the next step's primitive rows).

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <algorithm>
#include <utility>
#include <vector>

#include "adjoint.cuh"
#include "tangent.cuh"
#include "geometry.cuh"
#include "kernels.cuh"
#include "mlp.cuh"
#include "moving_derivative.cuh"
#include "luna_b200.h"

namespace {

thread_local std::string g_last_error;

luna_status set_error(luna_status s, const std::string& what) {
    g_last_error = what;
    return s;
}

#define LUNA_CUDA(call)                                                                                           \
    do {                                                                                                          \
        cudaError_t err_ = (call);                                                                                \
        if (err_ != cudaSuccess) return set_error(LUNA_ECUDA, std::string(#call) + ": " + cudaGetErrorString(err_)); \
    } while (0)

#define LUNA_TRY(call)                      \
    do {                                    \
        luna_status st_ = (call);           \
        if (st_ != LUNA_OK) return st_;     \
    } while (0)

// A device allocation that frees itself. It only grows: a smaller request (the next mesh of a moving run, whose face
// count changes every step) reuses the allocation instead of freeing it (cudaFree synchronises the device).
template <class T>
struct DevArray {
    T* ptr = nullptr;
    size_t count = 0, capacity = 0;
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    ~DevArray() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = capacity = 0;
    }
    luna_status alloc(size_t n, const char* what) {
        if (ptr && n <= capacity) {
            count = n;
            return LUNA_OK;
        }
        release();
        if (n == 0) return LUNA_OK;
        cudaError_t e = cudaMalloc(&ptr, n * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();
            return set_error(e == cudaErrorMemoryAllocation ? LUNA_ENOMEM : LUNA_ECUDA,
                             std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
        }
        count = capacity = n;
        return LUNA_OK;
    }
    size_t bytes() const { return capacity * sizeof(T); }
};

constexpr int kBlockCells = 128;
constexpr int kBlockFaces = 128;

int blocks(int64_t n, int per) { return static_cast<int>((n + per - 1) / per); }

}  // namespace

namespace luna {
// Other translation units of the library report through the same last-error slot as the entry points here.
luna_status report_error(luna_status s, const std::string& what) { return set_error(s, what); }
}  // namespace luna

struct luna_fv {
    int dim = 3, order = 1, update = LUNA_UPDATE_PER_FACE, limiter = LUNA_LIMITER_FACE_CENTROID, motion = LUNA_STATIC_MESH,
        riemann = LUNA_HLLC, precision = LUNA_FP64;
    int64_t n = 0, f = 0;
    luna::GasDev gas{};
    double box[3] = {1, 1, 1};
    cudaStream_t stream = nullptr;

    // mesh
    DevArray<int32_t> owner, neighbour, start, list;
    DevArray<double> area, mag, fcen, cen, vol, pos;
    // state and rows
    DevArray<double> q, next, prims, grad64, flux, w, x, old_cen;
    DevArray<float> grad32;
    DevArray<double> wg64;          // FP64 static per-face step: merged rows (W, g) [N][wg_stride] the flux reads
    bool grads_in_wg = false;       // the last sweep wrote wg64 (not grad64)
    DevArray<uint16_t> grad16;     // Grad16: binary16 gradient rows [N][16]
    DevArray<uint32_t> grad16_exp;  // Grad16: the rows' group exponents [N]
    DevArray<int32_t> steps;
    DevArray<luna::Counters> counters;
    // the mesh reordered for the step (geometry.cuh), rebuilt by every load_mesh
    DevArray<unsigned char> geo_c01, geo_c2, geo_off01, geo_off2, geo_faces;
    DevArray<unsigned int> geo_nbr;
    DevArray<int32_t> geo_slice_base, geo_order, geo_stage_start, geo_stage_cells;
    DevArray<double> geo_angle, geo_reach2;
    int64_t tiles = 0, normal_tiles = 0;  // the sweep's tiles (tiles.h)
    int normal_rows = 0, big_rows = 0;
    // the learned limiter: inputs written by the sweep, the network's logits; mlp_params is the caller's device vector
    DevArray<unsigned char> lim_features;
    DevArray<double> lim_alpha;
    DevArray<float> lim_logits;
    DevArray<int32_t> lim_cells;       // the compact rows' cells (a step that applies the limiter)
    DevArray<unsigned int> lim_count;  // the compact rows taken
    const float* mlp_params = nullptr;
    bool learned_inputs = false, apply_learned = false;
    // adjoint (allocated by the first luna_fv_step_adjoint)
    DevArray<double> adj_fit, adj_face_bar, adj_wbar, adj_bbar, adj_boundbar, adj_qbar;
    // tangent (allocated by the first luna_fv_step_tangent): dW, dg per cell, dF per face, a device copy of dq
    DevArray<double> tan_dprims, tan_dgrad, tan_dflux, tan_dq;
    DevArray<int32_t> adj_flags, adj_bound_face;
    // the order-0 moving step's derivatives (allocated by their first call): W and c_s rows and their tangents, w, dw, the
    // faces' dG or bar rows, the angle faces' bars, and device copies of the caller's host arrays
    DevArray<double> mv_W, mv_dW, mv_w, mv_dw, mv_face, mv_angle_Abar, mv_angle_dbar, mv_in[6];
    DevArray<int32_t> mv_angle_f;
    // order 1: the gradients and their tangents, w-hat, c^n and its tangent, the running bars, the fit's entry rows;
    // stage: 1 a tangent's first pass done (its second pass due after the step), 2 an adjoint begun, 3 its second pass done
    DevArray<double> mv_g, mv_dg, mv_wh, mv_c0, mv_dc0, mv_Wb, mv_gb, mv_whb, mv_cb, mv_xb, mv_entry;
    int mv_stage = 0;
    bool mv_steps_fixed = false;  // the reference's steps_fixed: the grid steps held, no derivative through w-hat
    luna::Counters* host_counters = nullptr;  // pinned

    // Per-phase timing: event pairs recorded around each launch, reduced on request.
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> event_pool;
    std::vector<std::pair<int, size_t>> pending;  // (phase, pool index) recorded since the last reduction
    double phase_ms[5] = {0, 0, 0, 0, 0};
    int64_t phase_launches[5] = {0, 0, 0, 0, 0};

    bool prims_ready = false, swept = false, moving_pending = false;
    // The static per-face step's flux pass, launched by time_step behind the sweep with the dt of the sweep's reduction
    // read on the device (no idle gap while the host reads dt); step(dt) with that dt, bit for bit, then only updates.
    bool flux_ready = false;
    unsigned long long flux_dt_bits = 0;
    cudaEvent_t counters_read = nullptr;
    double pending_dt = 0;
    double grid_step = 0, per_step = 0;
    long long period[3] = {1, 1, 1};

    // The fused flux-and-update pass of the static FP64 step (tiles.h TileFaces), planned by the first step on a mesh
    // when LUNA_FUSED_STEP=1: fused 0 not planned, 1 ready, -1 not used (not asked for, or the mesh does not fit it).
    int fused = 0;
    int fused_smem = 0;
    int64_t fused_crossing = 0;
    DevArray<int32_t> fz_tstart, fz_eslot, fz_tface, fz_xface;
    DevArray<unsigned char> fz_trows, fz_xrows;
    DevArray<double> fz_xflux;

    luna::DeviceTiler* tiler = nullptr;  // the sweep's tiles cut on the device, for meshes given in device memory
    DevArray<unsigned int> list_check;   // bad entries found in a device mesh's lists

    ~luna_fv() {
        if (tiler) luna::device_tiler_destroy(tiler);
        if (host_counters) cudaFreeHost(host_counters);
        if (counters_read) cudaEventDestroy(counters_read);
        for (auto& e : event_pool) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
    }

    // Opens a timed launch of `phase`; returns the pool slot (or -1 with timing off). close_timed records its end.
    long open_timed(int phase) {
        if (!timing) return -1;
        const size_t slot = pending.size();
        if (slot >= event_pool.size()) {
            cudaEvent_t a, b;
            if (cudaEventCreate(&a) != cudaSuccess) return -1;
            if (cudaEventCreate(&b) != cudaSuccess) {
                cudaEventDestroy(a);
                return -1;
            }
            event_pool.push_back({a, b});
        }
        cudaEventRecord(event_pool[slot].first, stream);
        pending.push_back({phase, slot});
        return static_cast<long>(slot);
    }
    void close_timed(long slot) {
        if (slot >= 0) cudaEventRecord(event_pool[static_cast<size_t>(slot)].second, stream);
    }

    template <int D, class G>
    luna::GeometryDev<D, G> geometry_dev() const {
        luna::GeometryDev<D, G> g;
        g.order = geo_order.ptr;
        g.slice_base = geo_slice_base.ptr;
        g.stage_start = geo_stage_start.ptr;
        g.stage_cells = geo_stage_cells.ptr;
        g.nbr = geo_nbr.ptr;
        g.c01 = reinterpret_cast<luna::Pair<G>*>(geo_c01.ptr);
        g.c2 = reinterpret_cast<G*>(geo_c2.ptr);
        g.off01 = reinterpret_cast<luna::Pair<G>*>(geo_off01.ptr);
        g.off2 = reinterpret_cast<G*>(geo_off2.ptr);
        g.faces = reinterpret_cast<luna::FaceRow<G>*>(geo_faces.ptr);
        g.max_angle = geo_angle.ptr;
        g.reach2 = geo_reach2.ptr;
        g.threads = tiles * luna::kTileCells;
        return g;
    }

    template <int D>
    luna::MeshDev<D> mesh_dev() const {
        luna::MeshDev<D> m;
        m.owner = owner.ptr;
        m.neighbour = neighbour.ptr;
        m.start = start.ptr;
        m.list = list.ptr;
        m.area = area.ptr;
        m.mag = mag.ptr;
        m.fcen = fcen.ptr;
        m.cen = cen.ptr;
        m.vol = vol.ptr;
        m.pos = pos.ptr;
        for (int a = 0; a < 3; ++a) {
            m.side[a] = box[a];
            m.inv[a] = box[a] > 0 ? 1.0 / box[a] : 0.0;
        }
        m.n = static_cast<int32_t>(n);
        m.f = static_cast<int32_t>(f);
        return m;
    }
};

// The Riemann solve in float in the face's frame (riemann32 and single), and float flux rows (single).
inline bool float_riemann(const luna_fv* fv) { return fv->precision == LUNA_FP32 || fv->precision == LUNA_SINGLE; }
inline bool float_flux(const luna_fv* fv) { return fv->precision == LUNA_SINGLE; }


namespace {

template <class T>
luna_status upload(DevArray<T>& dst, const T* src, size_t count, bool on_device, cudaStream_t s, const char* what) {
    LUNA_TRY(dst.alloc(count, what));
    if (count == 0) return LUNA_OK;
    if (!src) return set_error(LUNA_EINVAL, std::string("mesh array ") + what + " is null");
    LUNA_CUDA(cudaMemcpyAsync(dst.ptr, src, count * sizeof(T), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    return LUNA_OK;
}

luna_status validate_mesh(const luna_mesh_desc* m, int dim, int64_t n) {
    if (!m) return set_error(LUNA_EINVAL, "mesh is null");
    if (m->dim != 2 && m->dim != 3) return set_error(LUNA_EINVAL, "mesh dim must be 2 or 3");
    if (dim && m->dim != dim) return set_error(LUNA_EINVAL, "mesh dim differs from the solver's");
    if (m->n_cells <= 0 || m->n_cells >= (int64_t(1) << 31)) return set_error(LUNA_EINVAL, "n_cells out of range");
    if (n && m->n_cells != n) return set_error(LUNA_EINVAL, "a new mesh must have the same cells");
    if (m->n_faces < 0 || 2 * m->n_faces >= (int64_t(1) << 31)) return set_error(LUNA_EINVAL, "n_faces out of range");
    for (int a = 0; a < m->dim; ++a)
        if (!(m->box[a] > 0)) return set_error(LUNA_EINVAL, "box sides must be positive");
    if (!m->on_device) {  // host lists: checked here, once per mesh (device lists are the caller's responsibility)
        const int64_t N = m->n_cells, F = m->n_faces;
        if (!m->cell_face_start || !m->cell_face || !m->owner || !m->neighbour) return set_error(LUNA_EINVAL, "mesh lists are null");
        if (m->cell_face_start[0] != 0 || m->cell_face_start[N] != 2 * F) return set_error(LUNA_EINVAL, "cell_face_start must run 0 .. 2F");
        for (int64_t i = 0; i < N; ++i)
            if (m->cell_face_start[i + 1] < m->cell_face_start[i]) return set_error(LUNA_EINVAL, "cell_face_start not monotone");
        for (int64_t k = 0; k < 2 * F; ++k) {
            const int32_t e = m->cell_face[k];
            const int32_t face = e >= 0 ? e : ~e;
            if (face >= F) return set_error(LUNA_EINVAL, "cell_face entry out of range");
        }
        for (int64_t k = 0; k < F; ++k)
            if (m->owner[k] < 0 || m->owner[k] >= N || m->neighbour[k] < 0 || m->neighbour[k] >= N)
                return set_error(LUNA_EINVAL, "owner/neighbour out of range");
    }
    return LUNA_OK;
}

// The reordered rows of the current mesh (geometry.cuh::k_geometry), in the policy's gradient type, once the tiles are
// in place (geo_order, geo_slice_base, geo_stage_start, geo_stage_cells, geo_nbr holding each entry's staged row).
template <int D, class G>
luna_status finish_geometry(luna_fv* fv, size_t slots) {
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f);
    LUNA_TRY(fv->geo_c01.alloc(sizeof(luna::Pair<G>) * slots, "entry gradient rows"));
    LUNA_TRY(fv->geo_c2.alloc(sizeof(G) * slots, "entry gradient rows"));
    LUNA_TRY(fv->geo_off01.alloc(sizeof(luna::Pair<G>) * slots, "entry offsets"));
    LUNA_TRY(fv->geo_off2.alloc(sizeof(G) * slots, "entry offsets"));
    // a moving mesh's flux passes read the mesh arrays: no face rows
    const bool face_rows = fv->motion != LUNA_MOVING;
    if (face_rows)
        LUNA_TRY(fv->geo_faces.alloc(sizeof(luna::FaceRow<G>) * (F > 0 ? F : 1), "face rows"));
    else
        fv->geo_faces.release();
    LUNA_TRY(fv->geo_angle.alloc(N, "face angles"));
    LUNA_TRY(fv->geo_reach2.alloc(N, "cell reach"));
    const int64_t threads = fv->tiles * luna::kTileCells;
    if (threads > 0) {
        // timed with the sweep: the fit's operator rows, which the reference's sweep forms every step (a moving mesh
        // forms them every step here too)
        const long timed_ = fv->open_timed(1);
        // the tiles within the staged-row budget read their neighbours from shared memory; the single-cell tiles past it
        // through the face's cells
        const auto m = fv->mesh_dev<D>();
        const auto g = fv->geometry_dev<D, G>();
        const unsigned int normal = static_cast<unsigned int>(fv->normal_tiles), big = static_cast<unsigned int>(fv->tiles - fv->normal_tiles);
        const size_t smem = sizeof(double) * 2 * D * static_cast<size_t>(fv->normal_rows > 0 ? fv->normal_rows : 1);
        if (face_rows) {
            if (normal > 0) luna::k_geometry<D, G, true, true><<<normal, luna::kTileCells, smem, fv->stream>>>(m, g, 0);
            if (big > 0) luna::k_geometry<D, G, true, false><<<big, luna::kTileCells, 0, fv->stream>>>(m, g, static_cast<int>(normal));
        } else {
            if (normal > 0) luna::k_geometry<D, G, false, true><<<normal, luna::kTileCells, smem, fv->stream>>>(m, g, 0);
            if (big > 0) luna::k_geometry<D, G, false, false><<<big, luna::kTileCells, 0, fv->stream>>>(m, g, static_cast<int>(normal));
        }
        fv->close_timed(timed_);
        LUNA_CUDA(cudaGetLastError());
    }
    // The host vectors' contents (host tiles) must outlive the asynchronous uploads.
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

luna_status finish_geometry_any(luna_fv* fv, size_t slots) {
    const int D = fv->dim;
    return fv->precision == LUNA_FP64 ? (D == 3 ? finish_geometry<3, double>(fv, slots) : finish_geometry<2, double>(fv, slots))
                                      : (D == 3 ? finish_geometry<3, float>(fv, slots) : finish_geometry<2, float>(fv, slots));
}

// Geometry from tiles cut on the host.
luna_status build_geometry(luna_fv* fv, const luna::SweepTiles& tiles) {
    const size_t slots = tiles.local.size();
    fv->tiles = tiles.tiles;
    fv->normal_tiles = tiles.normal_tiles;
    fv->normal_rows = tiles.normal_rows;
    fv->big_rows = tiles.big_rows;
    LUNA_TRY(upload(fv->geo_order, tiles.order.data(), tiles.order.size(), false, fv->stream, "sweep order"));
    LUNA_TRY(upload(fv->geo_slice_base, tiles.slice_base.data(), tiles.slice_base.size(), false, fv->stream, "slice bases"));
    LUNA_TRY(upload(fv->geo_stage_start, tiles.stage_start.data(), tiles.stage_start.size(), false, fv->stream, "tile row starts"));
    LUNA_TRY(upload(fv->geo_stage_cells, tiles.stage_cells.data(), tiles.stage_cells.size() > 0 ? tiles.stage_cells.size() : 0, false, fv->stream,
                    "tile rows"));
    // the entries' staged rows; k_geometry adds the owned and tiny bits in place
    LUNA_TRY(upload(fv->geo_nbr, tiles.local.data(), slots, false, fv->stream, "entry neighbours"));
    return finish_geometry_any(fv, slots);
}

// Geometry from tiles cut on the device (tiles_device.cu), for a mesh the caller holds in device memory; false in
// *done when a tile does not fit the device cut (the caller cuts on the host instead).
luna_status build_geometry_device(luna_fv* fv, bool* done) {
    *done = false;
    if (!fv->tiler) fv->tiler = luna::device_tiler_create();
    luna::DeviceTilePlan plan;
    LUNA_TRY(luna::device_tiles_plan(fv->tiler, fv->dim, fv->n, fv->pos.ptr, fv->box, fv->start.ptr, fv->list.ptr, fv->owner.ptr,
                                     fv->neighbour.ptr, fv->stream, &plan));
    if (!plan.fits) return LUNA_OK;
    const size_t slots = static_cast<size_t>(plan.slots > 0 ? plan.slots : 1);
    fv->tiles = plan.tiles;
    fv->normal_tiles = plan.normal_tiles;
    fv->normal_rows = plan.normal_rows;
    fv->big_rows = plan.big_rows;
    LUNA_TRY(fv->geo_order.alloc(static_cast<size_t>(plan.tiles) * luna::kTileCells, "sweep order"));
    LUNA_TRY(fv->geo_slice_base.alloc(static_cast<size_t>(plan.tiles) * (luna::kTileCells / 32) + 1, "slice bases"));
    LUNA_TRY(fv->geo_stage_start.alloc(static_cast<size_t>(plan.tiles) + 1, "tile row starts"));
    LUNA_TRY(fv->geo_stage_cells.alloc(static_cast<size_t>(plan.staged > 0 ? plan.staged : 1), "tile rows"));
    LUNA_TRY(fv->geo_nbr.alloc(slots, "entry neighbours"));
    LUNA_TRY(luna::device_tiles_fill(fv->tiler, fv->geo_order.ptr, fv->geo_slice_base.ptr, fv->geo_stage_start.ptr, fv->geo_stage_cells.ptr,
                                     fv->geo_nbr.ptr, fv->stream));
    LUNA_TRY(finish_geometry_any(fv, slots));
    *done = true;
    return LUNA_OK;
}

// A device mesh's lists checked in place before any kernel follows them (the host's are checked by validate_mesh): the
// list starts run from 0 to 2F and do not fall, list entries name faces below F, owners and neighbours name cells below
// N. Counts the bad entries.
__global__ void k_check_lists(int64_t N, int64_t F, const int32_t* __restrict__ start, const int32_t* __restrict__ list,
                              const int32_t* __restrict__ owner, const int32_t* __restrict__ neighbour, unsigned int* __restrict__ bad) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    unsigned int wrong = 0;
    if (i < N) {
        const int64_t s0 = start[i], s1 = start[i + 1];
        wrong += s0 < 0 || s1 < s0 || s1 > 2 * F || (i == 0 && s0 != 0) || (i == N - 1 && s1 != 2 * F);
    }
    if (i < 2 * F) {
        const int32_t e = list[i];
        wrong += (e >= 0 ? e : ~e) >= F;
    }
    if (i < F) wrong += owner[i] < 0 || owner[i] >= N || neighbour[i] < 0 || neighbour[i] >= N;
    if (wrong) atomicAdd(bad, wrong);
}

luna_status check_device_lists(luna_fv* fv, int64_t N, int64_t F) {
    LUNA_TRY(fv->list_check.alloc(1, "list check"));
    LUNA_CUDA(cudaMemsetAsync(fv->list_check.ptr, 0, sizeof(unsigned int), fv->stream));
    const int64_t threads = N > 2 * F ? N : 2 * F;
    k_check_lists<<<blocks(threads, 256), 256, 0, fv->stream>>>(N, F, fv->start.ptr, fv->list.ptr, fv->owner.ptr, fv->neighbour.ptr,
                                                                 fv->list_check.ptr);
    LUNA_CUDA(cudaGetLastError());
    unsigned int bad = 0;
    LUNA_CUDA(cudaMemcpyAsync(&bad, fv->list_check.ptr, sizeof(bad), cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    if (bad) return set_error(LUNA_EINVAL, "mesh: " + std::to_string(bad) + " bad entries in the device lists");
    return LUNA_OK;
}

luna_status load_mesh(luna_fv* fv, const luna_mesh_desc* m) {
    const int D = m->dim;
    fv->fused = 0;
    const size_t N = static_cast<size_t>(m->n_cells), F = static_cast<size_t>(m->n_faces);
    const bool dev = m->on_device != 0;
    cudaStream_t s = fv->stream;
    LUNA_TRY(upload(fv->owner, m->owner, F, dev, s, "owner"));
    LUNA_TRY(upload(fv->neighbour, m->neighbour, F, dev, s, "neighbour"));
    LUNA_TRY(upload(fv->start, m->cell_face_start, N + 1, dev, s, "cell_face_start"));
    LUNA_TRY(upload(fv->list, m->cell_face, 2 * F, dev, s, "cell_face"));
    LUNA_TRY(upload(fv->area, m->area, F * D, dev, s, "area"));
    LUNA_TRY(upload(fv->fcen, m->face_centroid, F * D, dev, s, "face_centroid"));
    LUNA_TRY(upload(fv->cen, m->centroid, N * D, dev, s, "centroid"));
    LUNA_TRY(upload(fv->vol, m->volume, N, dev, s, "volume"));
    LUNA_TRY(upload(fv->pos, m->positions, N * D, dev, s, "positions"));
    LUNA_TRY(fv->mag.alloc(F, "magnitudes"));
    fv->f = static_cast<int64_t>(F);
    for (int a = 0; a < 3; ++a) fv->box[a] = a < D ? m->box[a] : 0.0;
    if (F > 0) {
        if (D == 3)
            luna::k_magnitudes<3><<<blocks(F, 256), 256, 0, s>>>(fv->area.ptr, fv->mag.ptr, static_cast<int>(F));
        else
            luna::k_magnitudes<2><<<blocks(F, 256), 256, 0, s>>>(fv->area.ptr, fv->mag.ptr, static_cast<int>(F));
        LUNA_CUDA(cudaGetLastError());
    }
    // 4 doubles past the last row: the update reads each row through its 32-B aligned 64-B window (load_row_windowed)
    if (fv->update == LUNA_UPDATE_PER_FACE) LUNA_TRY(fv->flux.alloc(F * (D + 2) + 4, "flux rows"));
    // The sweep's tiles: cut on the device when the caller's arrays are there (a mesh rebuilt every step stays on the
    // device), else on the host from the lists and the generators (also the fallback for a tile the device cut cannot
    // hold). Lists in device memory are checked for indices out of range first.
    if (dev) {
        LUNA_TRY(check_device_lists(fv, static_cast<int64_t>(N), static_cast<int64_t>(F)));
        bool done = false;
        LUNA_TRY(build_geometry_device(fv, &done));
        if (done) return LUNA_OK;
    }
    std::vector<int32_t> h_start, h_list, h_owner, h_neighbour;
    std::vector<double> h_pos;
    const int32_t *start = m->cell_face_start, *list = m->cell_face, *own = m->owner, *nbr = m->neighbour;
    const double* pos = m->positions;
    if (dev) {
        h_start.resize(N + 1);
        h_list.resize(2 * F);
        h_owner.resize(F);
        h_neighbour.resize(F);
        h_pos.resize(N * D);
        LUNA_CUDA(cudaMemcpy(h_start.data(), start, (N + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (F > 0) {
            LUNA_CUDA(cudaMemcpy(h_list.data(), list, 2 * F * sizeof(int32_t), cudaMemcpyDeviceToHost));
            LUNA_CUDA(cudaMemcpy(h_owner.data(), own, F * sizeof(int32_t), cudaMemcpyDeviceToHost));
            LUNA_CUDA(cudaMemcpy(h_neighbour.data(), nbr, F * sizeof(int32_t), cudaMemcpyDeviceToHost));
        }
        LUNA_CUDA(cudaMemcpy(h_pos.data(), pos, N * D * sizeof(double), cudaMemcpyDeviceToHost));
        start = h_start.data();
        list = h_list.data();
        own = h_owner.data();
        nbr = h_neighbour.data();
        pos = h_pos.data();
    }
    luna::SweepTiles tiles;
    const std::string why = luna::build_sweep_tiles(D, static_cast<int64_t>(N), pos, m->box, start, list, own, nbr, tiles);
    if (!why.empty()) return set_error(LUNA_EINVAL, "mesh: " + why);
    return build_geometry(fv, tiles);
}

template <int D>
luna_status run_primitives(luna_fv* fv) {
    {
        const long timed_ = fv->open_timed(0);
        luna::k_primitives<D><<<blocks(fv->n, 256), 256, 0, fv->stream>>>(fv->mesh_dev<D>(), fv->q.ptr, fv->prims.ptr, fv->gas);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    return LUNA_OK;
}

// The sweep's launches: the tiles within the row budget, then (rare) the single-cell tiles that stage more rows.
template <int D, bool Moving, bool Grad, class G, int Limit>
luna_status launch_sweep_tiles(luna_fv* fv, G* grad, double courant) {
    const auto m = fv->mesh_dev<D>();
    const auto geo = fv->geometry_dev<D, G>();
    // compact rows when the factors are applied (a step); every cell's row when the inputs are read (training data)
    const bool compact = fv->apply_learned;
    const luna::LearnedInputs learned{reinterpret_cast<__nv_bfloat16*>(fv->lim_features.ptr), fv->lim_alpha.ptr,
                                      compact ? fv->lim_cells.ptr : nullptr, compact ? fv->lim_count.ptr : nullptr};
    if (Limit == 2 && compact) LUNA_CUDA(cudaMemsetAsync(fv->lim_count.ptr, 0, sizeof(unsigned int), fv->stream));
    auto kernel = luna::k_sweep_tiles<D, Moving, Grad, G, Limit>;
    const luna::HalfRows half{fv->precision == LUNA_GRAD16 ? fv->grad16.ptr : nullptr, fv->grad16_exp.ptr};
    // merged rows for the static per-face FP64 step (the learned limiter's mode scales plain gradient rows)
    double* const wg_out = (Grad && Limit != 2 && sizeof(G) == sizeof(double)) ? fv->wg64.ptr : nullptr;
    fv->grads_in_wg = wg_out != nullptr;
    const int64_t groups[2][2] = {{0, fv->normal_tiles}, {fv->normal_tiles, fv->tiles}};
    const int most_rows[2] = {fv->normal_rows, fv->big_rows};
    // the round-off of the face states, squared: double face states (FP64, grad32), float ones (riemann32)
    const double round_off2 = float_riemann(fv) ? 0x1p-48 : 0x1p-100;
    for (int k = 0; k < 2; ++k) {
        const int64_t first = groups[k][0], count = groups[k][1] - groups[k][0];
        if (count <= 0) continue;
        const size_t smem = sizeof(double) * luna::kStagedDoubles * static_cast<size_t>(most_rows[k]);
        if (smem > 48 * 1024) LUNA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        kernel<<<static_cast<unsigned int>(count), luna::kTileCells, smem, fv->stream>>>(m, geo, static_cast<int>(first), fv->prims.ptr, grad, fv->w.ptr,
                                                                                        courant, round_off2, fv->counters.ptr, learned, half, wg_out);
        LUNA_CUDA(cudaGetLastError());
    }
    return LUNA_OK;
}

template <int D, bool Moving, bool Grad, class G>
luna_status launch_sweep(luna_fv* fv, G* grad, double courant) {
    const bool learned_mode = Grad && fv->learned_inputs && fv->limiter == LUNA_LIMITER_FACE_CENTROID;
    {
        const long timed_ = fv->open_timed(1);
        luna_status st = LUNA_OK;
        if (fv->limiter == LUNA_LIMITER_NONE)
            st = launch_sweep_tiles<D, Moving, Grad, G, 0>(fv, grad, courant);
        else if (learned_mode) {
            if constexpr (sizeof(G) == sizeof(double)) st = launch_sweep_tiles<D, Moving, Grad, G, 2>(fv, grad, courant);
        } else
            st = launch_sweep_tiles<D, Moving, Grad, G, 1>(fv, grad, courant);
        fv->close_timed(timed_);
        if (st != LUNA_OK) return st;
    }
    LUNA_CUDA(cudaGetLastError());
    if constexpr (sizeof(G) == sizeof(double)) {
        if (learned_mode && fv->apply_learned) {  // the network's factors, then the gradients scaled
            const long timed_ = fv->open_timed(1);
            if (fv->mlp_params) {
                const luna_status st = luna::mlp::forward_tc(fv->mlp_params, reinterpret_cast<const __nv_bfloat16*>(fv->lim_features.ptr),
                                                             static_cast<int>(fv->n), fv->lim_count.ptr, fv->lim_logits.ptr,
                                                             &fv->counters.ptr->error, fv->stream);
                if (st != LUNA_OK) {
                    fv->close_timed(timed_);
                    return st;
                }
            }
            luna::k_apply_factors<D><<<blocks(fv->n, 256), 256, 0, fv->stream>>>(static_cast<int>(fv->n), fv->lim_cells.ptr, fv->lim_count.ptr, grad,
                                                                                 fv->lim_alpha.ptr, fv->lim_logits.ptr, fv->mlp_params != nullptr);
            fv->close_timed(timed_);
            LUNA_CUDA(cudaGetLastError());
        }
    }
    return LUNA_OK;
}

// sweep() (finite_volume.hpp:1107-1149): the dt word is reset, then one kernel writes gradients, point velocities and dt.
template <int D>
luna_status run_sweep(luna_fv* fv, double courant) {
    const unsigned long long init = 0x7fefffffffffffffull;  // DBL_MAX: the Min reducer's identity
    LUNA_CUDA(cudaMemcpyAsync(&fv->counters.ptr->dt_bits, &init, sizeof(init), cudaMemcpyHostToDevice, fv->stream));
    const bool moving = fv->motion == LUNA_MOVING, grad = fv->order == 1;
    if (fv->precision != LUNA_FP64) {
        if (moving) return grad ? launch_sweep<D, true, true, float>(fv, fv->grad32.ptr, courant) : launch_sweep<D, true, false, float>(fv, fv->grad32.ptr, courant);
        return grad ? launch_sweep<D, false, true, float>(fv, fv->grad32.ptr, courant) : launch_sweep<D, false, false, float>(fv, fv->grad32.ptr, courant);
    }
    if (moving) return grad ? launch_sweep<D, true, true, double>(fv, fv->grad64.ptr, courant) : launch_sweep<D, true, false, double>(fv, fv->grad64.ptr, courant);
    return grad ? launch_sweep<D, false, true, double>(fv, fv->grad64.ptr, courant) : launch_sweep<D, false, false, double>(fv, fv->grad64.ptr, courant);
}

luna_status read_counters(luna_fv* fv) {
    LUNA_CUDA(cudaMemcpyAsync(fv->host_counters, fv->counters.ptr, sizeof(luna::Counters), cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

template <int D>
luna_status prepare_sweep(luna_fv* fv, double courant) {
    if (!fv->prims_ready) LUNA_TRY(run_primitives<D>(fv));
    fv->prims_ready = false;
    return run_sweep<D>(fv, courant);
}

template <int D>
luna_status ensure_step_rows(luna_fv* fv);

template <int D, int Order, int Pass, class G, bool RF, int Riemann, bool H = false>
luna_status launch_flux(luna_fv* fv, const luna::FluxArgs<D, G>& x) {
    if (fv->f == 0) return LUNA_OK;
    LUNA_TRY(ensure_step_rows<D>(fv));
    {
        const long timed_ = fv->open_timed(2);
        bool single = false;
        if constexpr (sizeof(G) == sizeof(float) && RF) {
            single = float_flux(fv);
            if (single)
                luna::k_flux<D, Order, Pass, G, RF, Riemann, H, float><<<blocks(fv->f, kBlockFaces), kBlockFaces, 0, fv->stream>>>(
                    fv->mesh_dev<D>(), x, reinterpret_cast<float*>(fv->flux.ptr), &fv->counters.ptr->fallbacks[Pass == 1 ? 1 : 0]);
        }
        if (!single)
            luna::k_flux<D, Order, Pass, G, RF, Riemann, H><<<blocks(fv->f, kBlockFaces), kBlockFaces, 0, fv->stream>>>(
                fv->mesh_dev<D>(), x, fv->flux.ptr, &fv->counters.ptr->fallbacks[Pass == 1 ? 1 : 0]);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    return LUNA_OK;
}

template <int D, int Order, class G, bool RF, int Riemann, bool H = false, bool WG = false, class FS = double>
luna_status launch_flux_rows(luna_fv* fv, const luna::FluxArgs<D, G>& x) {
    if (fv->f == 0) return LUNA_OK;
    LUNA_TRY(ensure_step_rows<D>(fv));
    {
        const long timed_ = fv->open_timed(2);
        luna::k_flux_rows<D, Order, G, RF, Riemann, H, WG, FS><<<blocks(fv->f, kBlockFaces), kBlockFaces, 0, fv->stream>>>(
                fv->mesh_dev<D>(), fv->geometry_dev<D, G>(), x, reinterpret_cast<FS*>(fv->flux.ptr), &fv->counters.ptr->fallbacks[0]);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    return LUNA_OK;
}

template <int D, int Order, class G>
luna_status dispatch_flux_rows(luna_fv* fv, const luna::FluxArgs<D, G>& x) {
    if constexpr (sizeof(G) == sizeof(double) && Order == 1)
        if (fv->grads_in_wg) {
            auto y = x;
            y.wg = fv->wg64.ptr;
            return fv->riemann == LUNA_HLL ? launch_flux_rows<D, Order, G, false, 1, false, true>(fv, y)
                                           : launch_flux_rows<D, Order, G, false, 0, false, true>(fv, y);
        }
    if (fv->precision == LUNA_GRAD16) return launch_flux_rows<D, Order, G, false, 0, true>(fv, x);
    if (float_flux(fv)) return launch_flux_rows<D, Order, G, true, 0, false, false, float>(fv, x);
    if (float_riemann(fv)) return launch_flux_rows<D, Order, G, true, 0>(fv, x);
    if (fv->riemann == LUNA_HLL) return launch_flux_rows<D, Order, G, false, 1>(fv, x);
    return launch_flux_rows<D, Order, G, false, 0>(fv, x);
}

template <int D, int Order, int Pass, class G>
luna_status dispatch_flux(luna_fv* fv, const luna::FluxArgs<D, G>& x) {
    if (fv->precision == LUNA_GRAD16) return launch_flux<D, Order, Pass, G, false, 0, true>(fv, x);
    if (float_riemann(fv)) return launch_flux<D, Order, Pass, G, true, 0>(fv, x);
    if (fv->riemann == LUNA_HLL) return launch_flux<D, Order, Pass, G, false, 1>(fv, x);
    return launch_flux<D, Order, Pass, G, false, 0>(fv, x);
}

template <int D, int Order, class G, bool RF, int Riemann, bool H = false>
luna_status launch_per_cell(luna_fv* fv, const luna::FluxArgs<D, G>& x, double dt) {
    double* out = Order == 0 ? fv->next.ptr : fv->q.ptr;
    {
        const long timed_ = fv->open_timed(2);
        luna::k_fluxes_and_update<D, Order, G, RF, Riemann, H><<<blocks(fv->n, kBlockCells), kBlockCells, 0, fv->stream>>>(fv->mesh_dev<D>(), x, out, dt,
                                                                                                                     fv->counters.ptr);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    if (Order == 0) std::swap(fv->q.ptr, fv->next.ptr);
    return LUNA_OK;
}

template <int D, class G>
luna::FluxArgs<D, G> flux_args(luna_fv* fv, const G* grad, double dt) {
    luna::FluxArgs<D, G> x;
    x.q = fv->q.ptr;
    x.prims = fv->prims.ptr;
    x.grad = grad;
    x.steps = fv->steps.ptr;
    x.old_cen = fv->old_cen.ptr;
    x.dt = dt;
    x.unit = 0;
    x.gas = fv->gas;
    if (fv->precision == LUNA_GRAD16) {
        x.grad16 = fv->grad16.ptr;
        x.exponents = fv->grad16_exp.ptr;
    }
    return x;
}

// apply()'s update of the library's flux rows (windowed double rows, or single's float rows).
template <int D, bool NextPrims>
void launch_update(luna_fv* fv, double dt) {
    if (float_flux(fv))
        luna::k_update<D, NextPrims, true, float><<<blocks(fv->n, 256), 256, 0, fv->stream>>>(
            fv->mesh_dev<D>(), fv->q.ptr, reinterpret_cast<const float*>(fv->flux.ptr), dt, fv->prims.ptr, fv->gas, fv->counters.ptr);
    else
        luna::k_update<D, NextPrims, true><<<blocks(fv->n, 256), 256, 0, fv->stream>>>(fv->mesh_dev<D>(), fv->q.ptr, fv->flux.ptr, dt, fv->prims.ptr,
                                                                                      fv->gas, fv->counters.ptr);
}

// The fused pass's plan for the current mesh (tiles.h build_tile_faces on the host, from the device arrays), its face
// rows gathered from the step's rows (k_geometry's) in tile order and in crossing order. Leaves fv->fused at 1, or -1
// where the plan does not apply (the step then runs k_flux_rows and k_update).
template <int D>
luna_status plan_fused(luna_fv* fv) {
    fv->fused = -1;
    const char* env = std::getenv("LUNA_FUSED_STEP");
    if (!(env && env[0] == '1') || fv->f == 0 || fv->tiles == 0) return LUNA_OK;
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f), T = static_cast<size_t>(fv->tiles);
    std::vector<int32_t> order(T * luna::kTileCells), start(N + 1), list(2 * F), owner(F), neighbour(F);
    LUNA_CUDA(cudaMemcpyAsync(order.data(), fv->geo_order.ptr, order.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaMemcpyAsync(start.data(), fv->start.ptr, start.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaMemcpyAsync(list.data(), fv->list.ptr, list.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaMemcpyAsync(owner.data(), fv->owner.ptr, F * sizeof(int32_t), cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaMemcpyAsync(neighbour.data(), fv->neighbour.ptr, F * sizeof(int32_t), cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    luna::TileFaces plan;
    const std::string why = luna::build_tile_faces(fv->n, fv->f, fv->tiles, order.data(), start.data(), list.data(), owner.data(),
                                                   neighbour.data(), plan);
    if (!why.empty()) return LUNA_OK;
    const size_t smem = sizeof(double) * (D + 2) * static_cast<size_t>(plan.max_slots);
    if (smem > 200 * 1024) return LUNA_OK;
    using Row = luna::FaceRow<double>;
    const size_t inner = plan.tface.size(), crossing = plan.xface.size();
    LUNA_TRY(upload(fv->fz_tstart, plan.tstart.data(), plan.tstart.size(), false, fv->stream, "fused tile starts"));
    LUNA_TRY(upload(fv->fz_eslot, plan.eslot.data(), plan.eslot.size(), false, fv->stream, "fused entry slots"));
    LUNA_TRY(upload(fv->fz_tface, plan.tface.data(), inner, false, fv->stream, "fused interior faces"));
    LUNA_TRY(upload(fv->fz_xface, plan.xface.data(), crossing, false, fv->stream, "fused crossing faces"));
    LUNA_TRY(fv->fz_trows.alloc(sizeof(Row) * (inner > 0 ? inner : 1), "fused interior face rows"));
    LUNA_TRY(fv->fz_xrows.alloc(sizeof(Row) * (crossing > 0 ? crossing : 1), "fused crossing face rows"));
    // 4 doubles past the last row: the update reads each row through its 32-B aligned 64-B window
    LUNA_TRY(fv->fz_xflux.alloc((D + 2) * crossing + 4, "fused crossing flux rows"));
    auto* faces = reinterpret_cast<Row*>(fv->geo_faces.ptr);
    if (inner > 0)
        luna::k_move_face_rows<double, true><<<blocks(inner, 256), 256, 0, fv->stream>>>(faces, fv->fz_tface.ptr, static_cast<int64_t>(inner),
                                                                                          reinterpret_cast<Row*>(fv->fz_trows.ptr));
    if (crossing > 0)
        luna::k_move_face_rows<double, true><<<blocks(crossing, 256), 256, 0, fv->stream>>>(faces, fv->fz_xface.ptr, static_cast<int64_t>(crossing),
                                                                                             reinterpret_cast<Row*>(fv->fz_xrows.ptr));
    LUNA_CUDA(cudaGetLastError());
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));  // the host plan must outlive the copies
    // The fused pass keeps the face rows in its own two orders and needs no flux row of an interior face: the face-ordered
    // rows and the flux rows are released (a step that leaves the fused pass takes them back, ensure_step_rows).
    fv->geo_faces.release();
    fv->flux.release();
    fv->fused_smem = static_cast<int>(smem);
    fv->fused_crossing = static_cast<int64_t>(crossing);
    fv->fused = 1;
    return LUNA_OK;
}

// The face-ordered rows and the flux rows of the two-kernel passes, after the fused pass released them.
template <int D>
luna_status ensure_step_rows(luna_fv* fv) {
    if (fv->update == LUNA_UPDATE_PER_FACE) LUNA_TRY(fv->flux.alloc(static_cast<size_t>(fv->f) * (D + 2) + 4, "flux rows"));
    if (fv->fused == 1 && !fv->geo_faces.ptr && fv->f > 0 && fv->precision == LUNA_FP64) {
        using Row = luna::FaceRow<double>;
        LUNA_TRY(fv->geo_faces.alloc(sizeof(Row) * static_cast<size_t>(fv->f), "face rows"));
        auto* faces = reinterpret_cast<Row*>(fv->geo_faces.ptr);
        const int64_t inner = static_cast<int64_t>(fv->fz_tface.count), crossing = fv->fused_crossing;
        if (inner > 0)
            luna::k_move_face_rows<double, false><<<blocks(inner, 256), 256, 0, fv->stream>>>(faces, fv->fz_tface.ptr, inner,
                                                                                               reinterpret_cast<Row*>(fv->fz_trows.ptr));
        if (crossing > 0)
            luna::k_move_face_rows<double, false><<<blocks(crossing, 256), 256, 0, fv->stream>>>(faces, fv->fz_xface.ptr, crossing,
                                                                                                  reinterpret_cast<Row*>(fv->fz_xrows.ptr));
        LUNA_CUDA(cudaGetLastError());
    }
    return LUNA_OK;
}

// The fused static FP64 pass: the crossing faces' rows (k_flux_rows over the crossing rows), then one block a tile.
template <int D, int Riemann>
luna_status launch_fused(luna_fv* fv, const luna::FluxArgs<D, double>& x, double dt) {
    auto m = fv->mesh_dev<D>();
    auto geo = fv->geometry_dev<D, double>();
    if (fv->fused_crossing > 0) {
        auto mx = m;
        mx.f = static_cast<int32_t>(fv->fused_crossing);
        geo.faces = reinterpret_cast<luna::FaceRow<double>*>(fv->fz_xrows.ptr);
        const long timed_ = fv->open_timed(2);
        luna::k_flux_rows<D, 1, double, false, Riemann, false, true><<<blocks(fv->fused_crossing, kBlockFaces), kBlockFaces, 0, fv->stream>>>(
            mx, geo, x, fv->fz_xflux.ptr, &fv->counters.ptr->fallbacks[0]);
        fv->close_timed(timed_);
    }
    auto kernel = luna::k_tile_flux_update<D, Riemann>;
    if (fv->fused_smem > 48 * 1024) LUNA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, fv->fused_smem));
    {
        const long timed_ = fv->open_timed(3);
        kernel<<<static_cast<unsigned int>(fv->tiles), luna::kTileCells, fv->fused_smem, fv->stream>>>(
            m, x, fv->geo_order.ptr, fv->fz_tstart.ptr, reinterpret_cast<const luna::FaceRow64*>(fv->fz_trows.ptr), fv->fz_eslot.ptr,
            fv->fz_xflux.ptr, fv->q.ptr, dt, fv->prims.ptr, fv->counters.ptr);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    return LUNA_OK;
}

// apply() for a static mesh (finite_volume.hpp:1538-1631).
template <int D, class G>
luna_status run_apply(luna_fv* fv, const G* grad, double dt) {
    const auto x = flux_args<D, G>(fv, grad, dt);
    if (fv->update == LUNA_UPDATE_PER_CELL) {
        if (fv->order == 0) {
            if (float_riemann(fv)) return launch_per_cell<D, 0, G, true, 0>(fv, x, dt);
            if (fv->precision == LUNA_GRAD16) return launch_per_cell<D, 0, G, false, 0, true>(fv, x, dt);
            return fv->riemann == LUNA_HLL ? launch_per_cell<D, 0, G, false, 1>(fv, x, dt) : launch_per_cell<D, 0, G, false, 0>(fv, x, dt);
        }
        if (float_riemann(fv)) return launch_per_cell<D, 1, G, true, 0>(fv, x, dt);
        if (fv->precision == LUNA_GRAD16) return launch_per_cell<D, 1, G, false, 0, true>(fv, x, dt);
        return fv->riemann == LUNA_HLL ? launch_per_cell<D, 1, G, false, 1>(fv, x, dt) : launch_per_cell<D, 1, G, false, 0>(fv, x, dt);
    }
    if constexpr (sizeof(G) == sizeof(double)) {
        if (fv->order == 1 && fv->grads_in_wg) {
            if (fv->fused == 0) LUNA_TRY(plan_fused<D>(fv));
            if (fv->fused == 1) {
                auto y = x;
                y.wg = fv->wg64.ptr;
                LUNA_TRY(fv->riemann == LUNA_HLL ? (launch_fused<D, 1>(fv, y, dt)) : (launch_fused<D, 0>(fv, y, dt)));
                fv->prims_ready = true;  // the update wrote the next primitive rows
                return LUNA_OK;
            }
        }
    }
    if (fv->order == 0)
        LUNA_TRY((dispatch_flux_rows<D, 0, G>(fv, x)));
    else
        LUNA_TRY((dispatch_flux_rows<D, 1, G>(fv, x)));
    {
        const long timed_ = fv->open_timed(3);
        launch_update<D, true>(fv, dt);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    fv->prims_ready = true;  // the update wrote the next primitive rows
    return LUNA_OK;
}

// Whether time_step may launch the step's flux pass itself: a static mesh stepped per face by the two-kernel pass.
template <int D>
luna_status flux_ahead(luna_fv* fv, bool* ahead) {
    *ahead = false;
    if (fv->motion == LUNA_MOVING || fv->update != LUNA_UPDATE_PER_FACE) return LUNA_OK;
    if (fv->precision == LUNA_FP64 && fv->order == 1 && fv->grads_in_wg) {
        if (fv->fused == 0) LUNA_TRY(plan_fused<D>(fv));
        if (fv->fused == 1) return LUNA_OK;
    }
    *ahead = true;
    return LUNA_OK;
}

// The flux pass of the static step with the dt of the sweep's reduction (read on the device).
template <int D, class G>
luna_status launch_flux_ahead(luna_fv* fv, const G* grad) {
    auto x = flux_args<D, G>(fv, grad, 0.0);
    x.dt_at = reinterpret_cast<const double*>(&fv->counters.ptr->dt_bits);
    if (fv->order == 0) return dispatch_flux_rows<D, 0, G>(fv, x);
    return dispatch_flux_rows<D, 1, G>(fv, x);
}

template <int D>
luna_status step_static(luna_fv* fv, double dt) {
    unsigned long long bits;
    std::memcpy(&bits, &dt, sizeof(bits));
    const bool ahead = fv->swept && fv->flux_ready && bits == fv->flux_dt_bits;
    fv->flux_ready = false;
    if (!fv->swept) LUNA_TRY(prepare_sweep<D>(fv, 1.0));
    fv->swept = false;
    if (ahead) {  // time_step launched this dt's flux pass: the update alone
        {
            const long timed_ = fv->open_timed(3);
            launch_update<D, true>(fv, dt);
            fv->close_timed(timed_);
        }
        LUNA_CUDA(cudaGetLastError());
        fv->prims_ready = true;  // the update wrote the next primitive rows
        return LUNA_OK;
    }
    LUNA_CUDA(cudaMemsetAsync(&fv->counters.ptr->fallbacks[0], 0, 2 * sizeof(unsigned long long), fv->stream));
    if (fv->precision != LUNA_FP64) return run_apply<D, float>(fv, fv->grad32.ptr, dt);
    return run_apply<D, double>(fv, fv->grad64.ptr, dt);
}

template <int D>
luna_status moving_begin(luna_fv* fv, double dt) {
    if (!fv->swept) LUNA_TRY(prepare_sweep<D>(fv, 1.0));
    fv->swept = false;
    LUNA_CUDA(cudaMemsetAsync(&fv->counters.ptr->fallbacks[0], 0, 2 * sizeof(unsigned long long), fv->stream));
    if (fv->order == 0) {  // step(): advance<0, true>() on this mesh, then move() (finite_volume.hpp:205-226, :1212-1228)
        fv->pending_dt = dt;
        if (fv->precision != LUNA_FP64) {
            auto x = flux_args<D, float>(fv, fv->grad32.ptr, dt);
            x.w = fv->w.ptr;
            LUNA_TRY(float_riemann(fv) ? (launch_flux<D, 0, 2, float, true, 0>(fv, x)) : (launch_flux<D, 0, 2, float, false, 0>(fv, x)));
        } else {
            auto x = flux_args<D, double>(fv, fv->grad64.ptr, dt);
            x.w = fv->w.ptr;
            LUNA_TRY(fv->riemann == LUNA_HLL ? (launch_flux<D, 0, 2, double, false, 1>(fv, x)) : (launch_flux<D, 0, 2, double, false, 0>(fv, x)));
        }
        {
            const long timed_ = fv->open_timed(3);
            launch_update<D, false>(fv, dt);
            fv->close_timed(timed_);
        }
        LUNA_CUDA(cudaGetLastError());
        {
            const long timed_ = fv->open_timed(4);
            luna::k_drift_free<D><<<blocks(fv->n, 256), 256, 0, fv->stream>>>(static_cast<int>(fv->n), fv->x.ptr, fv->w.ptr, dt, fv->box[0],
                                                                              fv->box[1], fv->box[2]);
            fv->close_timed(timed_);
        }
        LUNA_CUDA(cudaGetLastError());
        fv->moving_pending = true;
        return LUNA_OK;
    }
    {
        const long timed_ = fv->open_timed(4);
        luna::k_keep_centroids<D><<<blocks(fv->n, 256), 256, 0, fv->stream>>>(static_cast<int>(fv->n), fv->cen.ptr, fv->old_cen.ptr, fv->x.ptr, fv->w.ptr,
                                                                               fv->steps.ptr, dt, fv->grid_step, fv->per_step, fv->period[0],
                                                                               fv->period[1], fv->period[2]);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    fv->pending_dt = dt;
    if (fv->precision != LUNA_FP64) {
        auto x = flux_args<D, float>(fv, fv->grad32.ptr, 0.0);
        x.unit = fv->grid_step / dt;
        if (float_riemann(fv))
            LUNA_TRY((launch_flux<D, 1, 0, float, true, 0>(fv, x)));
        else if (fv->precision == LUNA_GRAD16)
            LUNA_TRY((launch_flux<D, 1, 0, float, false, 0, true>(fv, x)));
        else
            LUNA_TRY((launch_flux<D, 1, 0, float, false, 0>(fv, x)));
    } else {
        auto x = flux_args<D, double>(fv, fv->grad64.ptr, 0.0);
        x.unit = fv->grid_step / dt;
        if (fv->riemann == LUNA_HLL)
            LUNA_TRY((launch_flux<D, 1, 0, double, false, 1>(fv, x)));
        else
            LUNA_TRY((launch_flux<D, 1, 0, double, false, 0>(fv, x)));
    }
    {
        const long timed_ = fv->open_timed(3);
        launch_update<D, false>(fv, 0.5 * dt);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    {
        const long timed_ = fv->open_timed(4);
        luna::k_drift<D><<<blocks(fv->n, 256), 256, 0, fv->stream>>>(static_cast<int>(fv->n), fv->x.ptr, fv->steps.ptr, fv->grid_step, fv->per_step,
                                                                     fv->period[0], fv->period[1], fv->period[2]);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    fv->moving_pending = true;
    return LUNA_OK;
}

template <int D>
luna_status moving_end(luna_fv* fv) {
    const double dt = fv->pending_dt;
    if (fv->order == 0) {  // the new mesh is taken; its volumes change W, so the next step recomputes the primitive rows
        LUNA_CUDA(cudaMemcpyAsync(fv->x.ptr, fv->pos.ptr, static_cast<size_t>(fv->n) * fv->dim * sizeof(double), cudaMemcpyDeviceToDevice,
                                  fv->stream));
        fv->prims_ready = false;
        fv->moving_pending = false;
        return LUNA_OK;
    }
    if (fv->precision != LUNA_FP64) {
        auto x = flux_args<D, float>(fv, fv->grad32.ptr, 2 * dt);
        x.unit = fv->grid_step / dt;
        if (float_riemann(fv))
            LUNA_TRY((launch_flux<D, 1, 1, float, true, 0>(fv, x)));
        else if (fv->precision == LUNA_GRAD16)
            LUNA_TRY((launch_flux<D, 1, 1, float, false, 0, true>(fv, x)));
        else
            LUNA_TRY((launch_flux<D, 1, 1, float, false, 0>(fv, x)));
    } else {
        auto x = flux_args<D, double>(fv, fv->grad64.ptr, 2 * dt);
        x.unit = fv->grid_step / dt;
        if (fv->riemann == LUNA_HLL)
            LUNA_TRY((launch_flux<D, 1, 1, double, false, 1>(fv, x)));
        else
            LUNA_TRY((launch_flux<D, 1, 1, double, false, 0>(fv, x)));
    }
    {
        const long timed_ = fv->open_timed(3);
        launch_update<D, true>(fv, 0.5 * dt);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    fv->prims_ready = true;
    fv->moving_pending = false;
    return LUNA_OK;
}

// step_adjoint (finite_volume.hpp:2201-2231): the forward recompute (primitives, the sweep keeping its fit), then the
// faces' Riemann adjoints, the cells' adjoints and the gather into Qbar.
template <int D>
luna_status run_adjoint(luna_fv* fv, double dt, double* qbar) {
    fv->grads_in_wg = false;  // k_sweep_fit writes grad64
    constexpr int V = D + 2, U = D + 1;
    using FL = luna::FitLayout<D>;
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f);
    LUNA_TRY(fv->adj_fit.alloc(N * FL::width, "adjoint fit rows"));
    LUNA_TRY(fv->adj_flags.alloc(N * 2 * V, "adjoint flags"));
    LUNA_TRY(fv->adj_face_bar.alloc(F > 0 ? F * 2 * V : 1, "adjoint face bars"));
    LUNA_TRY(fv->adj_wbar.alloc(N * V, "adjoint W bars"));
    LUNA_TRY(fv->adj_bbar.alloc(N * V * U, "adjoint b bars"));
    LUNA_TRY(fv->adj_boundbar.alloc(N * V, "adjoint bound bars"));
    LUNA_TRY(fv->adj_bound_face.alloc(N * V, "adjoint bound faces"));
    const auto m = fv->mesh_dev<D>();
    LUNA_TRY(run_primitives<D>(fv));
    {
        const long timed_ = fv->open_timed(1);
        if (fv->limiter == LUNA_LIMITER_NONE)
            luna::k_sweep_fit<D, false><<<blocks(N, kBlockCells), kBlockCells, 0, fv->stream>>>(m, fv->prims.ptr, fv->grad64.ptr, fv->adj_fit.ptr,
                                                                                              fv->adj_flags.ptr);
        else
            luna::k_sweep_fit<D, true><<<blocks(N, kBlockCells), kBlockCells, 0, fv->stream>>>(m, fv->prims.ptr, fv->grad64.ptr, fv->adj_fit.ptr,
                                                                                             fv->adj_flags.ptr);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    if (F > 0) {
        const long timed_ = fv->open_timed(2);
        if (fv->riemann == LUNA_HLL)
            luna::k_faces_adjoint<D, 1><<<blocks(F, kBlockFaces), kBlockFaces, 0, fv->stream>>>(m, fv->prims.ptr, fv->grad64.ptr, qbar, dt, fv->gas,
                                                                                              fv->adj_face_bar.ptr);
        else
            luna::k_faces_adjoint<D, 0><<<blocks(F, kBlockFaces), kBlockFaces, 0, fv->stream>>>(m, fv->prims.ptr, fv->grad64.ptr, qbar, dt, fv->gas,
                                                                                              fv->adj_face_bar.ptr);
        fv->close_timed(timed_);
        LUNA_CUDA(cudaGetLastError());
    }
    {
        const long timed_ = fv->open_timed(3);
        luna::k_cell_adjoint<D><<<blocks(N, kBlockCells), kBlockCells, 0, fv->stream>>>(m, fv->prims.ptr, fv->grad64.ptr, fv->adj_face_bar.ptr,
                                                                                        fv->adj_fit.ptr, fv->adj_flags.ptr, dt, fv->gas, fv->adj_wbar.ptr,
                                                                                        fv->adj_bbar.ptr, fv->adj_boundbar.ptr, fv->adj_bound_face.ptr);
        luna::k_gather_adjoint<D><<<blocks(N, kBlockCells), kBlockCells, 0, fv->stream>>>(m, fv->q.ptr, fv->adj_wbar.ptr, fv->adj_bbar.ptr,
                                                                                          fv->adj_boundbar.ptr, fv->adj_bound_face.ptr, fv->gas, qbar);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    fv->prims_ready = true;  // Q is unchanged
    fv->swept = false;
    return LUNA_OK;
}

// step_tangent (finite_volume.hpp:2023-2062) before the step: dq <- J dq at fixed dt, linearised where step_adjoint is
// (the reference's fit and clip pattern, k_sweep_fit), then the production step advances Q.
template <int D>
luna_status run_tangent(luna_fv* fv, double dt, double* dq) {
    fv->grads_in_wg = false;  // k_sweep_fit writes grad64
    constexpr int V = D + 2;
    using FL = luna::FitLayout<D>;
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f);
    LUNA_TRY(fv->adj_fit.alloc(N * FL::width, "adjoint fit rows"));
    LUNA_TRY(fv->adj_flags.alloc(N * 2 * V, "adjoint flags"));
    LUNA_TRY(fv->tan_dprims.alloc(N * V, "tangent dW"));
    LUNA_TRY(fv->tan_dgrad.alloc(N * V * D, "tangent dg"));
    LUNA_TRY(fv->tan_dflux.alloc(F > 0 ? F * V : 1, "tangent dF"));
    const auto m = fv->mesh_dev<D>();
    LUNA_TRY(run_primitives<D>(fv));
    {
        const long timed_ = fv->open_timed(1);
        if (fv->limiter == LUNA_LIMITER_NONE)
            luna::k_sweep_fit<D, false><<<blocks(N, kBlockCells), kBlockCells, 0, fv->stream>>>(m, fv->prims.ptr, fv->grad64.ptr, fv->adj_fit.ptr,
                                                                                              fv->adj_flags.ptr);
        else
            luna::k_sweep_fit<D, true><<<blocks(N, kBlockCells), kBlockCells, 0, fv->stream>>>(m, fv->prims.ptr, fv->grad64.ptr, fv->adj_fit.ptr,
                                                                                             fv->adj_flags.ptr);
        luna::k_tangent_prims<D><<<blocks(N, 256), 256, 0, fv->stream>>>(static_cast<int>(N), fv->q.ptr, dq, fv->vol.ptr, fv->gas, fv->tan_dprims.ptr);
        luna::k_tangent_sweep<D><<<blocks(N, kBlockCells), kBlockCells, 0, fv->stream>>>(m, fv->prims.ptr, fv->tan_dprims.ptr, fv->adj_fit.ptr,
                                                                                        fv->adj_flags.ptr, fv->tan_dgrad.ptr);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    if (F > 0) {
        const long timed_ = fv->open_timed(2);
        if (fv->riemann == LUNA_HLL)
            luna::k_tangent_fluxes<D, 1><<<blocks(F, kBlockFaces), kBlockFaces, 0, fv->stream>>>(m, fv->prims.ptr, fv->grad64.ptr, fv->tan_dprims.ptr,
                                                                                               fv->tan_dgrad.ptr, dt, fv->gas, fv->tan_dflux.ptr);
        else
            luna::k_tangent_fluxes<D, 0><<<blocks(F, kBlockFaces), kBlockFaces, 0, fv->stream>>>(m, fv->prims.ptr, fv->grad64.ptr, fv->tan_dprims.ptr,
                                                                                               fv->tan_dgrad.ptr, dt, fv->gas, fv->tan_dflux.ptr);
        fv->close_timed(timed_);
        LUNA_CUDA(cudaGetLastError());
    }
    {
        const long timed_ = fv->open_timed(3);
        luna::k_tangent_update<D><<<blocks(N, 256), 256, 0, fv->stream>>>(m, dq, fv->tan_dflux.ptr, dt);
        fv->close_timed(timed_);
    }
    LUNA_CUDA(cudaGetLastError());
    fv->prims_ready = true;  // Q is unchanged
    fv->swept = false;       // grad64 holds the fit's gradients: the step sweeps again
    return LUNA_OK;
}

// IEEE binary16 -> float on the host (exact), for the Grad16 rows copied out.
float half_to_float(uint16_t h) {
    const int field = (h >> 10) & 0x1f, mant = h & 0x3ff;
    const float sign = (h & 0x8000) ? -1.0f : 1.0f;
    if (field == 0x1f) return mant ? std::nanf("") : sign * INFINITY;
    if (field == 0) return sign * std::ldexp(static_cast<float>(mant), -24);
    return sign * std::ldexp(static_cast<float>(mant | 0x400), field - 25);
}

luna_status copy_out(const double* src, double* dst, size_t count, int on_device, cudaStream_t s) {
    if (!dst) return set_error(LUNA_EINVAL, "output is null");
    LUNA_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    LUNA_CUDA(cudaStreamSynchronize(s));
    return LUNA_OK;
}

// The order-0 moving step's derivatives (finite_volume.hpp:2431-2604; kernels in moving_derivative.cuh).

luna_status check_moving_derivative(luna_fv* fv, double dt, const char* what) {
    if (fv->motion != LUNA_MOVING || fv->update != LUNA_UPDATE_PER_FACE || fv->precision != LUNA_FP64)
        return set_error(LUNA_EINVAL, std::string("hydro::FiniteVolume::") + what + ": a moving mesh, the per-face loop, the FP64 policy");
    if (fv->moving_pending) return set_error(LUNA_ESTATE, "inside a moving step");
    if (!(dt >= 0)) return set_error(LUNA_EINVAL, "dt must be >= 0");
    return LUNA_OK;
}

// The caller's arrays on the device: the array itself (on_device) or a copy into the library's slot k.
luna_status device_view(luna_fv* fv, int k, const double* src, size_t count, int on_device, const double** out) {
    if (!src) return set_error(LUNA_EINVAL, "null argument");
    if (on_device) {
        *out = src;
        return LUNA_OK;
    }
    LUNA_TRY(fv->mv_in[k].alloc(count > 0 ? count : 1, "moving derivative input"));
    if (count) LUNA_CUDA(cudaMemcpyAsync(fv->mv_in[k].ptr, src, count * sizeof(double), cudaMemcpyHostToDevice, fv->stream));
    *out = fv->mv_in[k].ptr;
    return LUNA_OK;
}

template <int D>
luna_status moving_work(luna_fv* fv) {
    constexpr int V = D + 2;
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f);
    LUNA_TRY(fv->mv_W.alloc(N * (V + 1), "moving W rows"));
    LUNA_TRY(fv->mv_dW.alloc(N * (V + 1), "moving W tangents"));
    LUNA_TRY(fv->mv_w.alloc(N * D, "moving point velocities"));
    LUNA_TRY(fv->mv_dw.alloc(N * D, "moving point velocity tangents"));
    LUNA_TRY(fv->mv_face.alloc((F > 0 ? F : 1) * luna::mvd::bar_width<D>(), "moving face rows"));
    LUNA_TRY(fv->mv_angle_Abar.alloc(N * D, "angle faces' area bars"));
    LUNA_TRY(fv->mv_angle_dbar.alloc(N * D, "angle faces' separation bars"));
    LUNA_TRY(fv->mv_angle_f.alloc(N, "angle faces"));
    return LUNA_OK;
}

template <int D>
luna_status run_moving_tangent(luna_fv* fv, double dt, double* dq, double* dx, const double* dV, const double* dc, const double* dA,
                               const double* dxf) {
    LUNA_TRY(moving_work<D>(fv));
    const auto m = fv->mesh_dev<D>();
    const unsigned int cb = blocks(fv->n, 128), fb = blocks(fv->f > 0 ? fv->f : 1, 128);
    luna::mvd::k_mv_prims<D><<<cb, 128, 0, fv->stream>>>(m, fv->q.ptr, dq, dV, fv->gas, fv->mv_W.ptr, fv->mv_dW.ptr);
    luna::mvd::k_mv_velocity<D><<<cb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_dW.ptr, dx, dc, dA, fv->mv_w.ptr, fv->mv_dw.ptr,
                                                            fv->mv_angle_f.ptr);
    if (fv->f > 0) {
        if (fv->riemann == LUNA_HLL)
            luna::mvd::k_mv_faces_tangent<D, 1><<<fb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_dW.ptr, fv->mv_w.ptr, fv->mv_dw.ptr, dx, dA, dxf,
                                                                            fv->gas, fv->mv_face.ptr);
        else
            luna::mvd::k_mv_faces_tangent<D, 0><<<fb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_dW.ptr, fv->mv_w.ptr, fv->mv_dw.ptr, dx, dA, dxf,
                                                                            fv->gas, fv->mv_face.ptr);
    }
    luna::mvd::k_mv_update_tangent<D><<<cb, 128, 0, fv->stream>>>(m, fv->mv_face.ptr, fv->mv_dw.ptr, dt, dq, dx);
    LUNA_CUDA(cudaGetLastError());
    return LUNA_OK;
}

template <int D>
luna_status moving_work1(luna_fv* fv) {
    constexpr int V = D + 2;
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f > 0 ? fv->f : 1);
    LUNA_TRY(fv->mv_g.alloc(N * V * D, "moving gradients"));
    LUNA_TRY(fv->mv_dg.alloc(N * V * D, "moving gradient tangents"));
    LUNA_TRY(fv->mv_wh.alloc(N * D, "grid-step velocities"));
    LUNA_TRY(fv->mv_c0.alloc(N * D, "centroids of t^n"));
    LUNA_TRY(fv->mv_dc0.alloc(N * D, "centroid tangents of t^n"));
    LUNA_TRY(fv->mv_Wb.alloc(N * V, "W bars"));
    LUNA_TRY(fv->mv_gb.alloc(N * V * D, "gradient bars"));
    LUNA_TRY(fv->mv_whb.alloc(N * D, "grid-step velocity bars"));
    LUNA_TRY(fv->mv_cb.alloc(N * D, "centroid bars"));
    LUNA_TRY(fv->mv_xb.alloc(N * D, "position bars"));
    LUNA_TRY(fv->mv_entry.alloc(2 * F * luna::mvd::entry_width<D>(), "fit entry bars"));
    return LUNA_OK;
}

template <int D>
void launch_mv1_cells(luna_fv* fv, double dt, const double* dW, const double* dx, const double* dc, const double* dA, const double* dxf) {
    const unsigned int cb = blocks(fv->n, 128);
    luna::mvd::k_mv1_cells<D><<<cb, 128, 0, fv->stream>>>(fv->mesh_dev<D>(), fv->mv_W.ptr, dW, dx, dc, dA, dxf, fv->x.ptr, fv->mv_w.ptr,
                                                          fv->limiter == LUNA_LIMITER_FACE_CENTROID, dt, fv->grid_step, fv->per_step, fv->period[0],
                                                          fv->period[1], fv->period[2], fv->mv_g.ptr, dW ? fv->mv_dg.ptr : nullptr, fv->mv_wh.ptr,
                                                          fv->mv_c0.ptr, dW ? fv->mv_dc0.ptr : nullptr);
}

template <int D, bool Second>
void launch_mv1_pass_tangent(luna_fv* fv, double dt, double* dq, const double* dx, const double* dc, const double* dA, const double* dxf) {
    const auto m = fv->mesh_dev<D>();
    const unsigned int cb = blocks(fv->n, 128), fb = blocks(fv->f > 0 ? fv->f : 1, 128);
    if (fv->f > 0) {
        if (fv->riemann == LUNA_HLL)
            luna::mvd::k_mv1_pass_tangent<D, 1, Second><<<fb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_dW.ptr, fv->mv_g.ptr, fv->mv_dg.ptr,
                                                                                    fv->mv_wh.ptr, fv->mv_dw.ptr, fv->mv_c0.ptr, fv->mv_dc0.ptr, dx, dc,
                                                                                    dA, dxf, dt, fv->gas, fv->mv_face.ptr);
        else
            luna::mvd::k_mv1_pass_tangent<D, 0, Second><<<fb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_dW.ptr, fv->mv_g.ptr, fv->mv_dg.ptr,
                                                                                    fv->mv_wh.ptr, fv->mv_dw.ptr, fv->mv_c0.ptr, fv->mv_dc0.ptr, dx, dc,
                                                                                    dA, dxf, dt, fv->gas, fv->mv_face.ptr);
    }
    luna::mvd::k_mv1_pass_update_tangent<D><<<cb, 128, 0, fv->stream>>>(m, fv->mv_face.ptr, dt, dq);
}

// Order 1, the first part (step_moving_tangent_1, :2767-2815): the gradients, the point velocities and their tangents, the
// first pass's tangent, then x^n+1's (dx += dt dw). The second pass's tangent follows the step (run_moving_tangent1_end).
template <int D>
luna_status run_moving_tangent1(luna_fv* fv, double dt, double* dq, double* dx, const double* dV, const double* dc, const double* dA,
                                const double* dxf) {
    LUNA_TRY(moving_work<D>(fv));
    LUNA_TRY(moving_work1<D>(fv));
    const auto m = fv->mesh_dev<D>();
    const unsigned int cb = blocks(fv->n, 128);
    luna::mvd::k_mv_prims<D><<<cb, 128, 0, fv->stream>>>(m, fv->q.ptr, dq, dV, fv->gas, fv->mv_W.ptr, fv->mv_dW.ptr);
    luna::mvd::k_mv_velocity<D><<<cb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_dW.ptr, dx, dc, dA, fv->mv_w.ptr, fv->mv_dw.ptr,
                                                            fv->mv_angle_f.ptr);
    launch_mv1_cells<D>(fv, dt, fv->mv_dW.ptr, dx, dc, dA, dxf);
    if (fv->mv_steps_fixed) LUNA_CUDA(cudaMemsetAsync(fv->mv_dw.ptr, 0, static_cast<size_t>(fv->n) * D * sizeof(double), fv->stream));
    launch_mv1_pass_tangent<D, false>(fv, dt, dq, dx, dc, dA, dxf);
    luna::mvd::k_mv1_drift_tangent<D><<<cb, 128, 0, fv->stream>>>(static_cast<int>(fv->n), fv->mv_dw.ptr, dt, dx);
    LUNA_CUDA(cudaGetLastError());
    fv->mv_stage = 1;
    return LUNA_OK;
}

template <int D>
luna_status run_moving_tangent1_end(luna_fv* fv, double dt, double* dq, const double* dx, const double* dc, const double* dA, const double* dxf) {
    launch_mv1_pass_tangent<D, true>(fv, dt, dq, dx, dc, dA, dxf);
    LUNA_CUDA(cudaGetLastError());
    fv->mv_stage = 0;
    return LUNA_OK;
}

// Order 1 adjoint (step_moving_adjoint_1, :2987-3155), in three parts around the caller's step and restore: begin at t^n
// (W, g, w-hat, c^n kept; the bars zeroed), the second pass on the mesh of t^n+1, then the rest on the mesh of t^n.
template <int D>
luna_status run_moving_adjoint1_begin(luna_fv* fv, double dt) {
    constexpr int V = D + 2;
    LUNA_TRY(moving_work<D>(fv));
    LUNA_TRY(moving_work1<D>(fv));
    const auto m = fv->mesh_dev<D>();
    const unsigned int cb = blocks(fv->n, 128);
    const size_t N = static_cast<size_t>(fv->n);
    luna::mvd::k_mv_prims<D><<<cb, 128, 0, fv->stream>>>(m, fv->q.ptr, nullptr, nullptr, fv->gas, fv->mv_W.ptr, nullptr);
    luna::mvd::k_mv_velocity<D><<<cb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, nullptr, nullptr, nullptr, nullptr, fv->mv_w.ptr, nullptr,
                                                            fv->mv_angle_f.ptr);
    launch_mv1_cells<D>(fv, dt, nullptr, nullptr, nullptr, nullptr, nullptr);
    LUNA_CUDA(cudaMemsetAsync(fv->mv_Wb.ptr, 0, N * V * sizeof(double), fv->stream));
    LUNA_CUDA(cudaMemsetAsync(fv->mv_gb.ptr, 0, N * V * D * sizeof(double), fv->stream));
    LUNA_CUDA(cudaMemsetAsync(fv->mv_whb.ptr, 0, N * D * sizeof(double), fv->stream));
    LUNA_CUDA(cudaMemsetAsync(fv->mv_cb.ptr, 0, N * D * sizeof(double), fv->stream));
    LUNA_CUDA(cudaGetLastError());
    fv->mv_stage = 2;
    return LUNA_OK;
}

template <int D, bool Second>
void launch_mv1_pass_adjoint(luna_fv* fv, double dt, const double* qbar, double* Abar, double* xfbar) {
    const auto m = fv->mesh_dev<D>();
    const unsigned int cb = blocks(fv->n, 128), fb = blocks(fv->f > 0 ? fv->f : 1, 128);
    if (fv->f > 0) {
        if (fv->riemann == LUNA_HLL)
            luna::mvd::k_mv1_pass_faces_adjoint<D, 1, Second><<<fb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_g.ptr, fv->mv_wh.ptr, fv->mv_c0.ptr,
                                                                                          qbar, dt, fv->gas, fv->mv_face.ptr, Abar, xfbar);
        else
            luna::mvd::k_mv1_pass_faces_adjoint<D, 0, Second><<<fb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_g.ptr, fv->mv_wh.ptr, fv->mv_c0.ptr,
                                                                                          qbar, dt, fv->gas, fv->mv_face.ptr, Abar, xfbar);
    }
    luna::mvd::k_mv1_pass_gather<D, Second><<<cb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_g.ptr, fv->mv_wh.ptr, fv->mv_c0.ptr, fv->mv_face.ptr,
                                                                        dt, fv->gas, fv->mv_Wb.ptr, fv->mv_gb.ptr, fv->mv_whb.ptr, fv->mv_cb.ptr,
                                                                        fv->mv_xb.ptr);
}

template <int D>
luna_status run_moving_adjoint1_new_mesh(luna_fv* fv, double dt, const double* qbar, const double* xbar, double* Abar, double* xfbar) {
    LUNA_CUDA(cudaMemcpyAsync(fv->mv_xb.ptr, xbar, static_cast<size_t>(fv->n) * D * sizeof(double), cudaMemcpyDeviceToDevice, fv->stream));
    launch_mv1_pass_adjoint<D, true>(fv, dt, qbar, Abar, xfbar);
    LUNA_CUDA(cudaGetLastError());
    fv->mv_stage = 3;
    return LUNA_OK;
}

template <int D>
luna_status run_moving_adjoint1_end(luna_fv* fv, double dt, double* qbar, const double* xbar, double* Vbar, double* cbar, double* Abar,
                                    double* xfbar) {
    const auto m = fv->mesh_dev<D>();
    const unsigned int cb = blocks(fv->n, 128), fb = blocks(fv->f > 0 ? fv->f : 1, 128);
    LUNA_CUDA(cudaMemcpyAsync(fv->mv_xb.ptr, xbar, static_cast<size_t>(fv->n) * D * sizeof(double), cudaMemcpyDeviceToDevice, fv->stream));
    luna::mvd::k_mv1_drift_adjoint<D><<<cb, 128, 0, fv->stream>>>(static_cast<int>(fv->n), fv->mv_xb.ptr, dt, fv->mv_whb.ptr);
    launch_mv1_pass_adjoint<D, false>(fv, dt, qbar, Abar, xfbar);
    luna::mvd::k_mv1_cells_adjoint<D><<<cb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_gb.ptr, fv->mv_whb.ptr, fv->mv_angle_f.ptr,
                                                                  fv->limiter == LUNA_LIMITER_FACE_CENTROID, fv->mv_steps_fixed, fv->gas, fv->mv_Wb.ptr,
                                                                  fv->mv_cb.ptr,
                                                                  fv->mv_entry.ptr, fv->mv_angle_Abar.ptr, fv->mv_angle_dbar.ptr);
    luna::mvd::k_mv1_gather_adjoint<D><<<cb, 128, 0, fv->stream>>>(m, fv->q.ptr, fv->mv_Wb.ptr, fv->mv_cb.ptr, fv->mv_entry.ptr, fv->mv_angle_f.ptr,
                                                                   fv->mv_angle_dbar.ptr, fv->gas, qbar, Vbar, cbar, fv->mv_xb.ptr);
    if (fv->f > 0)
        luna::mvd::k_mv1_faces_bar<D><<<fb, 128, 0, fv->stream>>>(m, fv->mv_entry.ptr, fv->mv_angle_f.ptr, fv->mv_angle_Abar.ptr, Abar, xfbar);
    LUNA_CUDA(cudaGetLastError());
    fv->mv_stage = 0;
    return LUNA_OK;
}

template <int D>
luna_status run_moving_adjoint(luna_fv* fv, double dt, double* qbar, double* xbar, double* Vbar, double* cbar, double* Abar, double* xfbar) {
    LUNA_TRY(moving_work<D>(fv));
    const auto m = fv->mesh_dev<D>();
    const unsigned int cb = blocks(fv->n, 128), fb = blocks(fv->f > 0 ? fv->f : 1, 128);
    luna::mvd::k_mv_prims<D><<<cb, 128, 0, fv->stream>>>(m, fv->q.ptr, nullptr, nullptr, fv->gas, fv->mv_W.ptr, nullptr);
    luna::mvd::k_mv_velocity<D><<<cb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, nullptr, nullptr, nullptr, nullptr, fv->mv_w.ptr, nullptr,
                                                            fv->mv_angle_f.ptr);
    if (fv->f > 0) {
        if (fv->riemann == LUNA_HLL)
            luna::mvd::k_mv_faces_adjoint<D, 1><<<fb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_w.ptr, qbar, dt, fv->gas, fv->mv_face.ptr, xfbar);
        else
            luna::mvd::k_mv_faces_adjoint<D, 0><<<fb, 128, 0, fv->stream>>>(m, fv->mv_W.ptr, fv->mv_w.ptr, qbar, dt, fv->gas, fv->mv_face.ptr, xfbar);
    }
    luna::mvd::k_mv_cells_adjoint<D><<<cb, 128, 0, fv->stream>>>(m, fv->q.ptr, fv->mv_W.ptr, fv->mv_face.ptr, xbar, fv->mv_angle_f.ptr, dt, fv->gas,
                                                                 qbar, Vbar, cbar, fv->mv_angle_Abar.ptr, fv->mv_angle_dbar.ptr);
    if (fv->f > 0)
        luna::mvd::k_mv_area_adjoint<D><<<fb, 128, 0, fv->stream>>>(m, fv->mv_face.ptr, fv->mv_angle_f.ptr, fv->mv_angle_Abar.ptr, Abar);
    luna::mvd::k_mv_separation_adjoint<D><<<cb, 128, 0, fv->stream>>>(m, fv->mv_face.ptr, fv->mv_angle_f.ptr, fv->mv_angle_dbar.ptr, xbar);
    LUNA_CUDA(cudaGetLastError());
    return LUNA_OK;
}

}  // namespace

extern "C" {

LUNA_API const char* luna_status_string(luna_status s) {
    switch (s) {
        case LUNA_OK: return "ok";
        case LUNA_EINVAL: return "invalid argument";
        case LUNA_ENOMEM: return "out of memory";
        case LUNA_ECUDA: return "CUDA error";
        case LUNA_ENONFINITE: return "non-finite value";
        case LUNA_ETIMEOUT: return "device wait timed out";
        case LUNA_ESTATE: return "call out of order";
    }
    return "unknown status";
}

LUNA_API const char* luna_last_error(void) { return g_last_error.c_str(); }

LUNA_API luna_status luna_fv_create(const luna_mesh_desc* mesh, const luna_gas* gas, int order, int update, int limiter, int motion, int riemann,
                                    int precision, luna_fv** out) {
    if (!out) return set_error(LUNA_EINVAL, "out is null");
    *out = nullptr;
    if (!gas || !(gas->gamma > 1.0)) return set_error(LUNA_EINVAL, "gas: gamma must be > 1");
    if (order != 0 && order != 1) return set_error(LUNA_EINVAL, "hydro::FiniteVolume: order 0 or 1");
    if (update != LUNA_UPDATE_PER_CELL && update != LUNA_UPDATE_PER_FACE) return set_error(LUNA_EINVAL, "update: per_cell or per_face");
    if (limiter != LUNA_LIMITER_FACE_CENTROID && limiter != LUNA_LIMITER_NONE) return set_error(LUNA_EINVAL, "limiter: face_centroid or none");
    if (motion != LUNA_STATIC_MESH && motion != LUNA_MOVING) return set_error(LUNA_EINVAL, "motion: static_mesh or moving");
    if (riemann != LUNA_HLLC && riemann != LUNA_HLL) return set_error(LUNA_EINVAL, "riemann: HLLC or HLL");
    if (precision != LUNA_FP64 && precision != LUNA_FP32 && precision != LUNA_GRAD32 && precision != LUNA_GRAD16 && precision != LUNA_SINGLE)
        return set_error(LUNA_EINVAL, "precision: FP64, FP32, GRAD32, GRAD16 or SINGLE");
    if (precision != LUNA_FP64 && riemann == LUNA_HLL)
        return set_error(LUNA_EINVAL, "the FP32 policy takes HLLC (the reference's reduced presets are HLLC only)");
    if (motion == LUNA_MOVING && update != LUNA_UPDATE_PER_FACE) return set_error(LUNA_EINVAL, "a moving mesh runs the per-face update");
    LUNA_TRY(validate_mesh(mesh, 0, 0));
    luna_fv* fv = new (std::nothrow) luna_fv();
    if (!fv) return set_error(LUNA_ENOMEM, "luna_fv");
    fv->dim = mesh->dim;
    fv->order = order;
    fv->update = update;
    fv->limiter = limiter;
    fv->motion = motion;
    fv->riemann = riemann;
    fv->precision = precision;
    fv->n = mesh->n_cells;
    fv->gas.gamma = gas->gamma;
    fv->gas.smallr = gas->smallr;
    fv->gas.smallc = gas->smallc;
    fv->gas.inverse_gm1 = 1.0 / (gas->gamma - 1.0);
    fv->gas.inverse_gm1_float = 1.0f / (static_cast<float>(gas->gamma) - 1.0f);
    auto fail = [&](luna_status s) {
        delete fv;
        return s;
    };
    const int D = fv->dim, V = D + 2;
    const size_t N = static_cast<size_t>(fv->n);
    if (cudaMallocHost(&fv->host_counters, sizeof(luna::Counters)) != cudaSuccess) {
        cudaGetLastError();
        fv->host_counters = nullptr;
        return fail(set_error(LUNA_ENOMEM, "pinned counters"));
    }
    luna_status s;
    if ((s = fv->counters.alloc(1, "counters")) != LUNA_OK) return fail(s);
    if (cudaMemsetAsync(fv->counters.ptr, 0, sizeof(luna::Counters), fv->stream) != cudaSuccess) return fail(set_error(LUNA_ECUDA, "memset counters"));
    if ((s = fv->q.alloc(N * V, "Q")) != LUNA_OK) return fail(s);
    if (cudaMemsetAsync(fv->q.ptr, 0, N * V * sizeof(double), fv->stream) != cudaSuccess) return fail(set_error(LUNA_ECUDA, "memset Q"));
    if (order == 0 && update == LUNA_UPDATE_PER_CELL && (s = fv->next.alloc(N * V, "Q next")) != LUNA_OK) return fail(s);
    if ((s = fv->prims.alloc(N * luna::PS, "primitive rows")) != LUNA_OK) return fail(s);
    const size_t GS = D == 3 ? luna::grad_stride<3>() : luna::grad_stride<2>();
    if (order == 1) {
        if (precision == LUNA_GRAD16) {
            if ((s = fv->grad16.alloc(N * 16, "binary16 gradient rows")) != LUNA_OK) return fail(s);
            if ((s = fv->grad16_exp.alloc(N, "gradient exponents")) != LUNA_OK) return fail(s);
            if ((s = fv->grad32.alloc(1, "gradient rows (unused)")) != LUNA_OK) return fail(s);
        } else if (precision != LUNA_FP64) {
            if ((s = fv->grad32.alloc(N * GS, "gradient rows")) != LUNA_OK) return fail(s);
        } else if ((s = fv->grad64.alloc(N * GS, "gradient rows")) != LUNA_OK) {
            return fail(s);
        }
        if (precision == LUNA_FP64 && motion == LUNA_STATIC_MESH && update == LUNA_UPDATE_PER_FACE) {
            const size_t S = D == 3 ? luna::wg_stride<3>() : luna::wg_stride<2>();
            if ((s = fv->wg64.alloc(N * S, "merged W and gradient rows")) != LUNA_OK) return fail(s);
        }
    }
    if ((s = fv->w.alloc(N * D, "point velocities")) != LUNA_OK) return fail(s);
    if (cudaMemsetAsync(fv->w.ptr, 0, N * D * sizeof(double), fv->stream) != cudaSuccess) return fail(set_error(LUNA_ECUDA, "memset w"));
    if ((s = load_mesh(fv, mesh)) != LUNA_OK) return fail(s);
    if (motion == LUNA_MOVING) {
        if ((s = fv->x.alloc(N * D, "positions")) != LUNA_OK) return fail(s);
        if ((s = fv->old_cen.alloc(N * D, "old centroids")) != LUNA_OK) return fail(s);
        if ((s = fv->steps.alloc(N * D, "grid steps")) != LUNA_OK) return fail(s);
        if (cudaMemcpyAsync(fv->x.ptr, fv->pos.ptr, N * D * sizeof(double), cudaMemcpyDeviceToDevice, fv->stream) != cudaSuccess)
            return fail(set_error(LUNA_ECUDA, "copy positions"));
        double longest = mesh->box[0];
        for (int a = 1; a < D; ++a) longest = longest > mesh->box[a] ? longest : mesh->box[a];
        fv->grid_step = std::ldexp(longest, -30);
        fv->per_step = 1.0 / fv->grid_step;
        for (int a = 0; a < D; ++a) fv->period[a] = std::llround(mesh->box[a] / fv->grid_step);
    }
    if (cudaStreamSynchronize(fv->stream) != cudaSuccess) return fail(set_error(LUNA_ECUDA, cudaGetErrorString(cudaGetLastError())));
    *out = fv;
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_destroy(luna_fv* fv) {
    if (!fv) return LUNA_OK;
    cudaStreamSynchronize(fv->stream);
    delete fv;
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_set_stream(luna_fv* fv, void* stream) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    fv->stream = static_cast<cudaStream_t>(stream);
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_state(luna_fv* fv, double** dev_q) {
    if (!fv || !dev_q) return set_error(LUNA_EINVAL, "null argument");
    fv->prims_ready = false;
    fv->swept = false;
    *dev_q = fv->q.ptr;
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_set_state(luna_fv* fv, const double* q, int on_device) {
    if (!fv || !q) return set_error(LUNA_EINVAL, "null argument");
    const size_t bytes = static_cast<size_t>(fv->n) * (fv->dim + 2) * sizeof(double);
    LUNA_CUDA(cudaMemcpyAsync(fv->q.ptr, q, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, fv->stream));
    if (!on_device) LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    fv->prims_ready = false;
    fv->swept = false;
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_get_state(luna_fv* fv, double* q, int on_device) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    return copy_out(fv->q.ptr, q, static_cast<size_t>(fv->n) * (fv->dim + 2), on_device, fv->stream);
}

LUNA_API luna_status luna_fv_time_step(luna_fv* fv, double courant, double* dt_out) {
    if (!fv || !dt_out) return set_error(LUNA_EINVAL, "null argument");
    if (fv->moving_pending) return set_error(LUNA_ESTATE, "time_step inside a moving step (call luna_fv_step_moving_end first)");
    LUNA_TRY(fv->dim == 3 ? prepare_sweep<3>(fv, courant) : prepare_sweep<2>(fv, courant));
    fv->flux_ready = false;
    bool ahead = false;
    LUNA_TRY(fv->dim == 3 ? flux_ahead<3>(fv, &ahead) : flux_ahead<2>(fv, &ahead));
    if (ahead) {
        // the counters (dt, error word) read behind the sweep; the step's flux pass queued behind that read with the
        // reduced dt read on the device, so it runs while the host takes dt
        if (!fv->counters_read) LUNA_CUDA(cudaEventCreateWithFlags(&fv->counters_read, cudaEventDisableTiming));
        LUNA_CUDA(cudaMemsetAsync(&fv->counters.ptr->fallbacks[0], 0, 2 * sizeof(unsigned long long), fv->stream));
        LUNA_CUDA(cudaMemcpyAsync(fv->host_counters, fv->counters.ptr, sizeof(luna::Counters), cudaMemcpyDeviceToHost, fv->stream));
        LUNA_CUDA(cudaEventRecord(fv->counters_read, fv->stream));
        luna_status st;
        if (fv->precision != LUNA_FP64)
            st = fv->dim == 3 ? launch_flux_ahead<3, float>(fv, fv->grad32.ptr) : launch_flux_ahead<2, float>(fv, fv->grad32.ptr);
        else
            st = fv->dim == 3 ? launch_flux_ahead<3, double>(fv, fv->grad64.ptr) : launch_flux_ahead<2, double>(fv, fv->grad64.ptr);
        LUNA_TRY(st);
        LUNA_CUDA(cudaEventSynchronize(fv->counters_read));
        std::memcpy(&fv->flux_dt_bits, &fv->host_counters->dt_bits, sizeof(fv->flux_dt_bits));
        fv->flux_ready = (fv->host_counters->error & 17ull) == 0;
    } else {
        LUNA_TRY(read_counters(fv));
    }
    fv->swept = true;
    double dt;
    std::memcpy(&dt, &fv->host_counters->dt_bits, sizeof(dt));
    *dt_out = dt;
    if (fv->host_counters->error & 1ull) return set_error(LUNA_ENONFINITE, "a time-step term is not finite");
    if (fv->host_counters->error & 16ull) return set_error(LUNA_ETIMEOUT, "the learned limiter's tensor-core completion wait gave up");
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step(luna_fv* fv, double dt) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    if (fv->motion == LUNA_MOVING) return set_error(LUNA_ESTATE, "a moving mesh steps with luna_fv_step_moving_begin/end");
    if (!(dt >= 0)) return set_error(LUNA_EINVAL, "dt must be >= 0");
    return fv->dim == 3 ? step_static<3>(fv, dt) : step_static<2>(fv, dt);
}

LUNA_API luna_status luna_fv_fallbacks(luna_fv* fv, int64_t* out) {
    if (!fv || !out) return set_error(LUNA_EINVAL, "null argument");
    LUNA_TRY(read_counters(fv));
    *out = static_cast<int64_t>(fv->host_counters->fallbacks[0] + fv->host_counters->fallbacks[1]);
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_error_word(luna_fv* fv, uint32_t* out) {
    if (!fv || !out) return set_error(LUNA_EINVAL, "null argument");
    LUNA_TRY(read_counters(fv));
    *out = static_cast<uint32_t>(fv->host_counters->error);
    LUNA_CUDA(cudaMemsetAsync(&fv->counters.ptr->error, 0, sizeof(unsigned long long), fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step_moving_begin(luna_fv* fv, double dt, double* positions_out, int on_device) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    if (fv->motion != LUNA_MOVING) return set_error(LUNA_ESTATE, "not a moving mesh");
    if (fv->moving_pending) return set_error(LUNA_ESTATE, "a moving step is already open");
    if (!(dt > 0)) return set_error(LUNA_EINVAL, "dt must be > 0");
    LUNA_TRY(fv->dim == 3 ? moving_begin<3>(fv, dt) : moving_begin<2>(fv, dt));
    if (positions_out) LUNA_TRY(copy_out(fv->x.ptr, positions_out, static_cast<size_t>(fv->n) * fv->dim, on_device, fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step_moving_end(luna_fv* fv, const luna_mesh_desc* new_mesh) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    if (!fv->moving_pending) return set_error(LUNA_ESTATE, "luna_fv_step_moving_end without begin");
    LUNA_TRY(validate_mesh(new_mesh, fv->dim, fv->n));
    LUNA_TRY(load_mesh(fv, new_mesh));
    return fv->dim == 3 ? moving_end<3>(fv) : moving_end<2>(fv);
}

LUNA_API luna_status luna_fv_set_mesh(luna_fv* fv, const luna_mesh_desc* mesh) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    if (fv->moving_pending) return set_error(LUNA_ESTATE, "inside a moving step (use luna_fv_step_moving_end)");
    LUNA_TRY(validate_mesh(mesh, fv->dim, fv->n));
    LUNA_TRY(load_mesh(fv, mesh));
    if (fv->motion == LUNA_MOVING)
        LUNA_CUDA(cudaMemcpyAsync(fv->x.ptr, fv->pos.ptr, static_cast<size_t>(fv->n) * fv->dim * sizeof(double), cudaMemcpyDeviceToDevice, fv->stream));
    fv->prims_ready = false;
    fv->swept = false;
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_positions(luna_fv* fv, double* out, int on_device) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    const double* src = fv->motion == LUNA_MOVING ? fv->x.ptr : fv->pos.ptr;
    return copy_out(src, out, static_cast<size_t>(fv->n) * fv->dim, on_device, fv->stream);
}

LUNA_API luna_status luna_fv_point_velocities(luna_fv* fv, double* out, int on_device) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    return copy_out(fv->w.ptr, out, static_cast<size_t>(fv->n) * fv->dim, on_device, fv->stream);
}

LUNA_API luna_status luna_fv_prims(luna_fv* fv, double* out, int on_device) {
    if (!fv || !out) return set_error(LUNA_EINVAL, "null argument");
    const int width = fv->dim + 4;
    LUNA_CUDA(cudaMemcpy2DAsync(out, width * sizeof(double), fv->prims.ptr, luna::PS * sizeof(double), width * sizeof(double),
                                static_cast<size_t>(fv->n), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_gradients(luna_fv* fv, double* out, int on_device) {
    if (!fv || !out) return set_error(LUNA_EINVAL, "null argument");
    if (fv->order != 1) return set_error(LUNA_ESTATE, "order 0 has no gradients");
    const int D = fv->dim, width = (D + 2) * D;
    const size_t GS = D == 3 ? luna::grad_stride<3>() : luna::grad_stride<2>();
    const size_t N = static_cast<size_t>(fv->n);
    if (fv->precision == LUNA_FP64) {
        const double* src = fv->grad64.ptr;
        size_t pitch = GS;
        if (fv->grads_in_wg) {  // the merged rows: g after the row's V values of W
            src = fv->wg64.ptr + (D + 2);
            pitch = D == 3 ? luna::wg_stride<3>() : luna::wg_stride<2>();
        }
        LUNA_CUDA(cudaMemcpy2DAsync(out, width * sizeof(double), src, pitch * sizeof(double), width * sizeof(double), N,
                                    on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, fv->stream));
        LUNA_CUDA(cudaStreamSynchronize(fv->stream));
        return LUNA_OK;
    }
    if (on_device) return set_error(LUNA_EINVAL, "FP32 gradients are copied to host memory only");
    if (fv->precision == LUNA_GRAD16) {  // decoded as the flux reads them: binary16 times 2^-k of the group
        std::vector<uint16_t> rows(N * 16);
        std::vector<uint32_t> k(N);
        LUNA_CUDA(cudaMemcpyAsync(rows.data(), fv->grad16.ptr, N * 16 * sizeof(uint16_t), cudaMemcpyDeviceToHost, fv->stream));
        LUNA_CUDA(cudaMemcpyAsync(k.data(), fv->grad16_exp.ptr, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, fv->stream));
        LUNA_CUDA(cudaStreamSynchronize(fv->stream));
        for (size_t i = 0; i < N; ++i)
            for (int c = 0; c < width; ++c) {
                const int group = c < D ? 0 : c < D + D * D ? 1 : 2;
                const int e = static_cast<int8_t>((k[i] >> (8 * group)) & 0xffu);
                out[i * width + c] = std::ldexp(static_cast<double>(half_to_float(rows[i * 16 + c])), -e);
            }
        return LUNA_OK;
    }
    float* tmp = nullptr;
    LUNA_CUDA(cudaMallocHost(&tmp, N * GS * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(tmp, fv->grad32.ptr, N * GS * sizeof(float), cudaMemcpyDeviceToHost, fv->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(fv->stream);
    if (e == cudaSuccess)
        for (size_t i = 0; i < N; ++i)
            for (int c = 0; c < width; ++c) out[i * width + c] = static_cast<double>(tmp[i * GS + c]);
    cudaFreeHost(tmp);
    if (e != cudaSuccess) return set_error(LUNA_ECUDA, cudaGetErrorString(e));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step_adjoint(luna_fv* fv, double dt, double* qbar, int on_device) {
    if (!fv || !qbar) return set_error(LUNA_EINVAL, "null argument");
    if (fv->motion != LUNA_STATIC_MESH || fv->order != 1 || fv->update != LUNA_UPDATE_PER_FACE || fv->precision != LUNA_FP64)
        return set_error(LUNA_EINVAL, "hydro::FiniteVolume::step_adjoint: a static mesh, order 1, the per-face loop, the FP64 policy");
    if (fv->moving_pending) return set_error(LUNA_ESTATE, "inside a moving step");
    const size_t count = static_cast<size_t>(fv->n) * (fv->dim + 2);
    double* dev = qbar;
    if (!on_device) {
        LUNA_TRY(fv->adj_qbar.alloc(count, "adjoint Q bar"));
        LUNA_CUDA(cudaMemcpyAsync(fv->adj_qbar.ptr, qbar, count * sizeof(double), cudaMemcpyHostToDevice, fv->stream));
        dev = fv->adj_qbar.ptr;
    }
    LUNA_TRY(fv->dim == 3 ? run_adjoint<3>(fv, dt, dev) : run_adjoint<2>(fv, dt, dev));
    if (!on_device) LUNA_TRY(copy_out(dev, qbar, count, 0, fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step_tangent(luna_fv* fv, double dt, double* dq, int on_device) {
    if (!fv || !dq) return set_error(LUNA_EINVAL, "null argument");
    if (fv->motion != LUNA_STATIC_MESH || fv->order != 1 || fv->update != LUNA_UPDATE_PER_FACE || fv->precision != LUNA_FP64)
        return set_error(LUNA_EINVAL, "hydro::FiniteVolume::step_tangent: a static mesh, order 1, the per-face loop, the FP64 policy");
    if (fv->moving_pending) return set_error(LUNA_ESTATE, "inside a moving step");
    if (!(dt >= 0)) return set_error(LUNA_EINVAL, "dt must be >= 0");
    const size_t count = static_cast<size_t>(fv->n) * (fv->dim + 2);
    double* dev = dq;
    if (!on_device) {
        LUNA_TRY(fv->tan_dq.alloc(count, "tangent dq"));
        LUNA_CUDA(cudaMemcpyAsync(fv->tan_dq.ptr, dq, count * sizeof(double), cudaMemcpyHostToDevice, fv->stream));
        dev = fv->tan_dq.ptr;
    }
    LUNA_TRY(fv->dim == 3 ? run_tangent<3>(fv, dt, dev) : run_tangent<2>(fv, dt, dev));
    LUNA_TRY(fv->dim == 3 ? step_static<3>(fv, dt) : step_static<2>(fv, dt));
    if (!on_device) LUNA_TRY(copy_out(dev, dq, count, 0, fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step_moving_tangent(luna_fv* fv, double dt, double* dq, double* dx, const double* dV, const double* dc,
                                                 const double* dA, const double* dxf, int on_device) {
    if (!fv || !dq || !dx) return set_error(LUNA_EINVAL, "null argument");
    LUNA_TRY(check_moving_derivative(fv, dt, "step_moving_tangent"));
    if (fv->mv_stage != 0) return set_error(LUNA_ESTATE, "step_moving_tangent: another moving derivative is open");
    const int D = fv->dim;
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f), nq = N * (D + 2), nx = N * D;
    const double *gV, *gc, *gA, *gxf, *gq, *gx;
    LUNA_TRY(device_view(fv, 0, dq, nq, on_device, &gq));
    LUNA_TRY(device_view(fv, 1, dx, nx, on_device, &gx));
    LUNA_TRY(device_view(fv, 2, dV, N, on_device, &gV));
    LUNA_TRY(device_view(fv, 3, dc, nx, on_device, &gc));
    LUNA_TRY(device_view(fv, 4, dA, F * D, on_device, &gA));
    LUNA_TRY(device_view(fv, 5, dxf, F * D, on_device, &gxf));
    double* q_dev = const_cast<double*>(gq);
    double* x_dev = const_cast<double*>(gx);
    if (fv->order == 1)
        LUNA_TRY(D == 3 ? run_moving_tangent1<3>(fv, dt, q_dev, x_dev, gV, gc, gA, gxf) : run_moving_tangent1<2>(fv, dt, q_dev, x_dev, gV, gc, gA, gxf));
    else
        LUNA_TRY(D == 3 ? run_moving_tangent<3>(fv, dt, q_dev, x_dev, gV, gc, gA, gxf) : run_moving_tangent<2>(fv, dt, q_dev, x_dev, gV, gc, gA, gxf));
    if (!on_device) {
        LUNA_CUDA(cudaMemcpyAsync(dq, q_dev, nq * sizeof(double), cudaMemcpyDeviceToHost, fv->stream));
        LUNA_CUDA(cudaMemcpyAsync(dx, x_dev, nx * sizeof(double), cudaMemcpyDeviceToHost, fv->stream));
    }
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step_moving_tangent_end(luna_fv* fv, double dt, double* dq, const double* dx, const double* dV, const double* dc,
                                                     const double* dA, const double* dxf, int on_device) {
    if (!fv || !dq || !dx) return set_error(LUNA_EINVAL, "null argument");
    LUNA_TRY(check_moving_derivative(fv, dt, "step_moving_tangent"));
    if (fv->order != 1 || fv->mv_stage != 1) return set_error(LUNA_ESTATE, "step_moving_tangent_end: after an order-1 step_moving_tangent and the step");
    const int D = fv->dim;
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f), nq = N * (D + 2), nx = N * D;
    const double *gV, *gc, *gA, *gxf, *gq, *gx;
    LUNA_TRY(device_view(fv, 0, dq, nq, on_device, &gq));
    LUNA_TRY(device_view(fv, 1, dx, nx, on_device, &gx));
    LUNA_TRY(device_view(fv, 2, dV, N, on_device, &gV));
    LUNA_TRY(device_view(fv, 3, dc, nx, on_device, &gc));
    LUNA_TRY(device_view(fv, 4, dA, F * D, on_device, &gA));
    LUNA_TRY(device_view(fv, 5, dxf, F * D, on_device, &gxf));
    double* q_dev = const_cast<double*>(gq);
    LUNA_TRY(D == 3 ? run_moving_tangent1_end<3>(fv, dt, q_dev, gx, gc, gA, gxf) : run_moving_tangent1_end<2>(fv, dt, q_dev, gx, gc, gA, gxf));
    if (!on_device) LUNA_CUDA(cudaMemcpyAsync(dq, q_dev, nq * sizeof(double), cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_set_steps_fixed(luna_fv* fv, int held) {
    if (!fv) return set_error(LUNA_EINVAL, "null argument");
    fv->mv_steps_fixed = held != 0;
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step_moving_adjoint_begin(luna_fv* fv, double dt) {
    if (!fv) return set_error(LUNA_EINVAL, "null argument");
    LUNA_TRY(check_moving_derivative(fv, dt, "step_moving_adjoint"));
    if (fv->order != 1) return set_error(LUNA_EINVAL, "step_moving_adjoint_begin: order 1 (order 0 takes luna_fv_step_moving_adjoint alone)");
    if (fv->mv_stage != 0) return set_error(LUNA_ESTATE, "step_moving_adjoint_begin: another moving derivative is open");
    LUNA_TRY(fv->dim == 3 ? run_moving_adjoint1_begin<3>(fv, dt) : run_moving_adjoint1_begin<2>(fv, dt));
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step_moving_adjoint_new_mesh(luna_fv* fv, double dt, const double* qbar, double* xbar, double* Abar, double* xfbar,
                                                          int on_device) {
    if (!fv || !qbar || !xbar || !Abar || !xfbar) return set_error(LUNA_EINVAL, "null argument");
    LUNA_TRY(check_moving_derivative(fv, dt, "step_moving_adjoint"));
    if (fv->order != 1 || fv->mv_stage != 2) return set_error(LUNA_ESTATE, "step_moving_adjoint_new_mesh: after step_moving_adjoint_begin and the step");
    const int D = fv->dim;
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f), nq = N * (D + 2), nx = N * D;
    const double *gq, *gx;
    LUNA_TRY(device_view(fv, 0, qbar, nq, on_device, &gq));
    LUNA_TRY(device_view(fv, 1, xbar, nx, on_device, &gx));
    double* outs[2] = {Abar, xfbar};
    double* dev_out[2];
    for (int k = 0; k < 2; ++k) {
        if (on_device) {
            dev_out[k] = outs[k];
        } else {
            LUNA_TRY(fv->mv_in[2 + k].alloc(F * D > 0 ? F * D : 1, "moving derivative output"));
            dev_out[k] = fv->mv_in[2 + k].ptr;
        }
    }
    LUNA_TRY(D == 3 ? run_moving_adjoint1_new_mesh<3>(fv, dt, gq, gx, dev_out[0], dev_out[1]) : run_moving_adjoint1_new_mesh<2>(fv, dt, gq, gx, dev_out[0], dev_out[1]));
    LUNA_CUDA(cudaMemcpyAsync(xbar, fv->mv_xb.ptr, nx * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, fv->stream));
    if (!on_device)
        for (int k = 0; k < 2; ++k)
            if (F) LUNA_CUDA(cudaMemcpyAsync(outs[k], dev_out[k], F * D * sizeof(double), cudaMemcpyDeviceToHost, fv->stream));
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_step_moving_adjoint(luna_fv* fv, double dt, double* qbar, double* xbar, double* Vbar, double* cbar, double* Abar,
                                                 double* xfbar, int on_device) {
    if (!fv || !qbar || !xbar || !Vbar || !cbar || !Abar || !xfbar) return set_error(LUNA_EINVAL, "null argument");
    LUNA_TRY(check_moving_derivative(fv, dt, "step_moving_adjoint"));
    if (fv->order == 1 && fv->mv_stage != 3) return set_error(LUNA_ESTATE, "step_moving_adjoint (order 1): after begin, the step, new_mesh and the restore");
    if (fv->order == 0 && fv->mv_stage != 0) return set_error(LUNA_ESTATE, "step_moving_adjoint: another moving derivative is open");
    const int D = fv->dim;
    const size_t N = static_cast<size_t>(fv->n), F = static_cast<size_t>(fv->f), nq = N * (D + 2), nx = N * D;
    const double *gq, *gx;
    LUNA_TRY(device_view(fv, 0, qbar, nq, on_device, &gq));
    LUNA_TRY(device_view(fv, 1, xbar, nx, on_device, &gx));
    double* outs[4] = {Vbar, cbar, Abar, xfbar};
    const size_t counts[4] = {N, nx, F * D, F * D};
    double* dev_out[4];
    for (int k = 0; k < 4; ++k) {
        if (on_device) {
            dev_out[k] = outs[k];
        } else {
            LUNA_TRY(fv->mv_in[2 + k].alloc(counts[k] > 0 ? counts[k] : 1, "moving derivative output"));
            dev_out[k] = fv->mv_in[2 + k].ptr;
        }
    }
    double* q_dev = const_cast<double*>(gq);
    double* x_dev = const_cast<double*>(gx);
    if (fv->order == 1) {
        LUNA_TRY(D == 3 ? run_moving_adjoint1_end<3>(fv, dt, q_dev, x_dev, dev_out[0], dev_out[1], dev_out[2], dev_out[3])
                        : run_moving_adjoint1_end<2>(fv, dt, q_dev, x_dev, dev_out[0], dev_out[1], dev_out[2], dev_out[3]));
        LUNA_CUDA(cudaMemcpyAsync(x_dev, fv->mv_xb.ptr, nx * sizeof(double), cudaMemcpyDeviceToDevice, fv->stream));
    } else {
        LUNA_TRY(D == 3 ? run_moving_adjoint<3>(fv, dt, q_dev, x_dev, dev_out[0], dev_out[1], dev_out[2], dev_out[3])
                        : run_moving_adjoint<2>(fv, dt, q_dev, x_dev, dev_out[0], dev_out[1], dev_out[2], dev_out[3]));
    }
    if (!on_device) {
        LUNA_CUDA(cudaMemcpyAsync(qbar, q_dev, nq * sizeof(double), cudaMemcpyDeviceToHost, fv->stream));
        LUNA_CUDA(cudaMemcpyAsync(xbar, x_dev, nx * sizeof(double), cudaMemcpyDeviceToHost, fv->stream));
        for (int k = 0; k < 4; ++k)
            if (counts[k]) LUNA_CUDA(cudaMemcpyAsync(outs[k], dev_out[k], counts[k] * sizeof(double), cudaMemcpyDeviceToHost, fv->stream));
    }
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

// The learned limiter's buffers (64 B of features, 40 B of admissible factors, 64 B of logits and a compact row's cell a
// cell, and the row count).
static luna_status alloc_learned(luna_fv* fv) {
    const size_t N = static_cast<size_t>(fv->n);
    LUNA_TRY(fv->lim_features.alloc(N * 32 * sizeof(__nv_bfloat16), "limiter features"));
    LUNA_TRY(fv->lim_alpha.alloc(N * 5, "limiter admissible factors"));
    LUNA_TRY(fv->lim_logits.alloc(N * 16, "limiter logits"));
    LUNA_TRY(fv->lim_cells.alloc(N, "limiter rows' cells"));
    LUNA_TRY(fv->lim_count.alloc(1, "limiter row count"));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_set_limiter_mlp(luna_fv* fv, const float* params, int mode) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    if (mode == 0) {
        fv->learned_inputs = fv->apply_learned = false;
        fv->mlp_params = nullptr;
        return LUNA_OK;
    }
    if (fv->order != 1 || fv->precision != LUNA_FP64 || fv->limiter != LUNA_LIMITER_FACE_CENTROID)
        return set_error(LUNA_EINVAL, "the learned limiter needs order 1, the FP64 policy and the face-centroid limiter");
    if (mode == 1 && !params) return set_error(LUNA_EINVAL, "mode 1 needs the network's parameters");
    LUNA_TRY(alloc_learned(fv));
    fv->learned_inputs = fv->apply_learned = true;
    fv->mlp_params = mode == 1 ? params : nullptr;  // mode 2: the plain factor min(alpha, 1) through the same path
    fv->swept = false;
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_limiter_inputs(luna_fv* fv, void* features, double* alpha, double* gradients) {
    if (!fv || !features || !alpha || !gradients) return set_error(LUNA_EINVAL, "null argument");
    if (fv->order != 1 || fv->precision != LUNA_FP64 || fv->limiter != LUNA_LIMITER_FACE_CENTROID)
        return set_error(LUNA_EINVAL, "the learned limiter needs order 1, the FP64 policy and the face-centroid limiter");
    if (fv->moving_pending) return set_error(LUNA_ESTATE, "inside a moving step");
    LUNA_TRY(alloc_learned(fv));
    const bool inputs = fv->learned_inputs, apply = fv->apply_learned;
    fv->learned_inputs = true;
    fv->apply_learned = false;
    fv->prims_ready = false;
    luna_status s = fv->dim == 3 ? prepare_sweep<3>(fv, 1.0) : prepare_sweep<2>(fv, 1.0);
    fv->learned_inputs = inputs;
    fv->apply_learned = apply;
    fv->swept = false;
    if (s != LUNA_OK) return s;
    const size_t N = static_cast<size_t>(fv->n);
    const int D = fv->dim, width = (D + 2) * D;
    const size_t GS = D == 3 ? luna::grad_stride<3>() : luna::grad_stride<2>();
    LUNA_CUDA(cudaMemcpyAsync(features, fv->lim_features.ptr, N * 32 * sizeof(__nv_bfloat16), cudaMemcpyDeviceToDevice, fv->stream));
    LUNA_CUDA(cudaMemcpyAsync(alpha, fv->lim_alpha.ptr, N * 5 * sizeof(double), cudaMemcpyDeviceToDevice, fv->stream));
    LUNA_CUDA(cudaMemcpy2DAsync(gradients, width * sizeof(double), fv->grad64.ptr, GS * sizeof(double), width * sizeof(double), N,
                                cudaMemcpyDeviceToDevice, fv->stream));
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_set_timing(luna_fv* fv, int on) {
    if (!fv) return set_error(LUNA_EINVAL, "fv is null");
    fv->timing = on != 0;
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_timings(luna_fv* fv, luna_timings* out, int reset) {
    if (!fv || !out) return set_error(LUNA_EINVAL, "null argument");
    LUNA_CUDA(cudaStreamSynchronize(fv->stream));
    for (const auto& p : fv->pending) {
        float ms = 0;
        LUNA_CUDA(cudaEventElapsedTime(&ms, fv->event_pool[p.second].first, fv->event_pool[p.second].second));
        fv->phase_ms[p.first] += ms;
        fv->phase_launches[p.first] += 1;
    }
    fv->pending.clear();
    for (int k = 0; k < 5; ++k) {
        out->ms[k] = fv->phase_ms[k];
        out->launches[k] = fv->phase_launches[k];
        if (reset) {
            fv->phase_ms[k] = 0;
            fv->phase_launches[k] = 0;
        }
    }
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_fused_pass(luna_fv* fv, int* fused, int64_t* crossing_faces) {
    if (!fv || !fused) return set_error(LUNA_EINVAL, "null argument");
    *fused = fv->fused == 1 ? 1 : 0;
    if (crossing_faces) *crossing_faces = fv->fused == 1 ? fv->fused_crossing : 0;
    return LUNA_OK;
}

LUNA_API luna_status luna_fv_device_bytes(luna_fv* fv, int64_t* out) {
    if (!fv || !out) return set_error(LUNA_EINVAL, "null argument");
    size_t b = 0;
    b += fv->owner.bytes() + fv->neighbour.bytes() + fv->start.bytes() + fv->list.bytes();
    b += fv->area.bytes() + fv->mag.bytes() + fv->fcen.bytes() + fv->cen.bytes() + fv->vol.bytes() + fv->pos.bytes();
    b += fv->q.bytes() + fv->next.bytes() + fv->prims.bytes() + fv->grad64.bytes() + fv->grad32.bytes() + fv->flux.bytes();
    b += fv->grad16.bytes() + fv->grad16_exp.bytes() + fv->wg64.bytes();
    b += fv->w.bytes() + fv->x.bytes() + fv->old_cen.bytes() + fv->steps.bytes() + fv->counters.bytes();
    b += fv->adj_fit.bytes() + fv->adj_face_bar.bytes() + fv->adj_wbar.bytes() + fv->adj_bbar.bytes() + fv->adj_boundbar.bytes();
    b += fv->adj_qbar.bytes() + fv->adj_flags.bytes() + fv->adj_bound_face.bytes();
    b += fv->tan_dprims.bytes() + fv->tan_dgrad.bytes() + fv->tan_dflux.bytes() + fv->tan_dq.bytes();
    b += fv->geo_c01.bytes() + fv->geo_c2.bytes() + fv->geo_off01.bytes() + fv->geo_off2.bytes() + fv->geo_nbr.bytes();
    b += fv->geo_slice_base.bytes() + fv->geo_order.bytes() + fv->geo_stage_start.bytes() + fv->geo_stage_cells.bytes() + fv->geo_faces.bytes();
    b += fv->geo_angle.bytes() + fv->geo_reach2.bytes() + fv->lim_features.bytes() + fv->lim_alpha.bytes() + fv->lim_logits.bytes();
    b += fv->lim_cells.bytes() + fv->lim_count.bytes();
    b += fv->fz_tstart.bytes() + fv->fz_eslot.bytes() + fv->fz_tface.bytes() + fv->fz_xface.bytes() + fv->fz_trows.bytes() + fv->fz_xrows.bytes();
    b += fv->fz_xflux.bytes();
    b += fv->mv_W.bytes() + fv->mv_dW.bytes() + fv->mv_w.bytes() + fv->mv_dw.bytes() + fv->mv_face.bytes() + fv->mv_angle_Abar.bytes();
    b += fv->mv_angle_dbar.bytes() + fv->mv_angle_f.bytes();
    b += fv->mv_g.bytes() + fv->mv_dg.bytes() + fv->mv_wh.bytes() + fv->mv_c0.bytes() + fv->mv_dc0.bytes() + fv->mv_Wb.bytes() + fv->mv_gb.bytes();
    b += fv->mv_whb.bytes() + fv->mv_cb.bytes() + fv->mv_xb.bytes() + fv->mv_entry.bytes();
    for (const auto& a : fv->mv_in) b += a.bytes();
    *out = static_cast<int64_t>(b);
    return LUNA_OK;
}

}  // extern "C"
