// The flux-and-update pass of a static step without any device allocation, for callers that cannot allocate device
// memory themselves. Its only scratch (the per-face flux rows and the pass's counters) lives in one fixed-size
// file-scope device array; the caller passes every input and output.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "kernels.cuh"
#include "luna_b200.h"

namespace {

// 32 MiB: 256 bytes of counters, then flux rows of D + 2 doubles per face.
constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr size_t kCounterBytes = 256;
constexpr size_t kFluxDoubles = (kScratchBytes - kCounterBytes) / sizeof(double);

static_assert(sizeof(luna::Counters) <= kCounterBytes, "counters fit their slot");

// Held by every GPU that loads the library, until the process exits. Calls that overlap on the GPU share it and race.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The device address of g_noalloc_scratch per device, looked up once per device with that device current: in host
// code the array's name is only a host-side stand-in, not an address a kernel may use.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
unsigned char* g_scratch_address[kMaxDevices] = {};

}  // namespace

namespace luna {
// The library's error report (luna_last_error), defined with the other entry points.
luna_status report_error(luna_status s, const std::string& what);
}  // namespace luna

namespace {

luna_status fail(luna_status s, const std::string& what) { return luna::report_error(s, what); }

luna_status scratch_of_current_device(unsigned char** out) {
    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(LUNA_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices) return fail(LUNA_EINVAL, "device ordinal beyond the no-allocation table");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_address[device]) {
        void* address = nullptr;
        e = cudaGetSymbolAddress(&address, g_noalloc_scratch);
        if (e != cudaSuccess || !address)
            return fail(LUNA_ECUDA, std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(e));
        g_scratch_address[device] = static_cast<unsigned char*>(address);
    }
    *out = g_scratch_address[device];
    return LUNA_OK;
}

template <int D>
luna::MeshDev<D> mesh_of(const luna_mesh_desc* d) {
    luna::MeshDev<D> m;
    m.owner = d->owner;
    m.neighbour = d->neighbour;
    m.start = d->cell_face_start;
    m.list = d->cell_face;
    m.area = d->area;
    m.mag = nullptr;  // the flux and update passes take |A| from the area vectors
    m.fcen = d->face_centroid;
    m.cen = d->centroid;
    m.vol = d->volume;
    m.pos = d->positions;
    for (int a = 0; a < 3; ++a) {
        m.side[a] = a < D ? d->box[a] : 0.0;
        m.inv[a] = a < D ? 1.0 / d->box[a] : 0.0;
    }
    m.n = static_cast<int32_t>(d->n_cells);
    m.f = static_cast<int32_t>(d->n_faces);
    return m;
}

template <int D, int Order, int Riemann>
luna_status launch(const luna_mesh_desc* mesh, const luna::GasDev& gas, const double* prims, const double* gradients, double* q, double dt,
                   cudaStream_t stream, unsigned char* scratch) {
    auto* counters = reinterpret_cast<luna::Counters*>(scratch);
    double* flux = reinterpret_cast<double*>(scratch + kCounterBytes);
    const auto m = mesh_of<D>(mesh);
    luna::FluxArgs<D, double> x;
    x.q = q;
    x.prims = prims;
    x.grad = gradients;
    x.steps = nullptr;
    x.old_cen = nullptr;
    x.dt = dt;
    x.unit = 0;
    x.gas = gas;
    // The array keeps the last call's contents: the counters must start at zero; every flux row is written before it
    // is read.
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(luna::Counters), stream);
    if (e != cudaSuccess) return fail(LUNA_ECUDA, std::string("cudaMemsetAsync(counters): ") + cudaGetErrorString(e));
    const int64_t F = mesh->n_faces, N = mesh->n_cells;
    if (F > 0)
        luna::k_flux<D, Order, -1, double, false, Riemann>
            <<<static_cast<int>((F + 127) / 128), 128, 0, stream>>>(m, x, flux, &counters->fallbacks[0]);
    luna::k_update<D, false><<<static_cast<int>((N + 255) / 256), 256, 0, stream>>>(m, q, flux, dt, nullptr, gas, counters);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LUNA_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
    return LUNA_OK;
}

}  // namespace

extern "C" {

LUNA_API luna_status luna_apply_static_noalloc(const luna_mesh_desc* mesh, const luna_gas* gas, int order, int riemann, const double* prims,
                                               const double* gradients, double* q, double dt, void* stream, int64_t* fallbacks_out) {
    if (!mesh || !gas || !q) return fail(LUNA_EINVAL, "luna_apply_static_noalloc: null argument");
    if (!mesh->on_device) return fail(LUNA_EINVAL, "luna_apply_static_noalloc: the mesh arrays must be device pointers (on_device = 1)");
    if (mesh->dim != 2 && mesh->dim != 3) return fail(LUNA_EINVAL, "luna_apply_static_noalloc: dim must be 2 or 3");
    if (order != 0 && order != 1) return fail(LUNA_EINVAL, "luna_apply_static_noalloc: order 0 or 1");
    if (riemann != LUNA_HLLC && riemann != LUNA_HLL) return fail(LUNA_EINVAL, "luna_apply_static_noalloc: riemann HLLC or HLL");
    if (order == 1 && (!prims || !gradients)) return fail(LUNA_EINVAL, "luna_apply_static_noalloc: order 1 needs the primitive and gradient rows");
    if (!(gas->gamma > 1.0)) return fail(LUNA_EINVAL, "luna_apply_static_noalloc: gamma must be > 1");
    if (!(dt >= 0)) return fail(LUNA_EINVAL, "luna_apply_static_noalloc: dt must be >= 0");
    if (mesh->n_cells <= 0 || mesh->n_cells >= (int64_t(1) << 31) || mesh->n_faces < 0)
        return fail(LUNA_EINVAL, "luna_apply_static_noalloc: cell or face count out of range");
    for (int a = 0; a < mesh->dim; ++a)
        if (!(mesh->box[a] > 0)) return fail(LUNA_EINVAL, "luna_apply_static_noalloc: box sides must be positive");
    const int V = mesh->dim + 2;
    const int64_t max_faces = static_cast<int64_t>(kFluxDoubles / V);
    if (mesh->n_faces > max_faces)
        return fail(LUNA_EINVAL, "luna_apply_static_noalloc: the mesh has " + std::to_string(mesh->n_faces) + " faces; its fixed scratch holds at most " +
                                     std::to_string(max_faces) + " (" + std::to_string(mesh->dim) + "D flux rows in 32 MiB)");
    unsigned char* scratch = nullptr;
    luna_status s = scratch_of_current_device(&scratch);
    if (s != LUNA_OK) return s;
    luna::GasDev g;
    g.gamma = gas->gamma;
    g.smallr = gas->smallr;
    g.smallc = gas->smallc;
    g.inverse_gm1 = 1.0 / (gas->gamma - 1.0);
    g.inverse_gm1_float = 1.0f / (static_cast<float>(gas->gamma) - 1.0f);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (mesh->dim == 3) {
        if (order == 0)
            s = riemann == LUNA_HLL ? launch<3, 0, 1>(mesh, g, prims, gradients, q, dt, st, scratch) : launch<3, 0, 0>(mesh, g, prims, gradients, q, dt, st, scratch);
        else
            s = riemann == LUNA_HLL ? launch<3, 1, 1>(mesh, g, prims, gradients, q, dt, st, scratch) : launch<3, 1, 0>(mesh, g, prims, gradients, q, dt, st, scratch);
    } else {
        if (order == 0)
            s = riemann == LUNA_HLL ? launch<2, 0, 1>(mesh, g, prims, gradients, q, dt, st, scratch) : launch<2, 0, 0>(mesh, g, prims, gradients, q, dt, st, scratch);
        else
            s = riemann == LUNA_HLL ? launch<2, 1, 1>(mesh, g, prims, gradients, q, dt, st, scratch) : launch<2, 1, 0>(mesh, g, prims, gradients, q, dt, st, scratch);
    }
    if (s != LUNA_OK) return s;
    if (fallbacks_out) {
        // The pass's counters in one copy: the fallback count and the error word the update writes (bit 1: a state
        // that is not finite, bit 2: an index out of range), reported as every other entry point reports them.
        luna::Counters host{};
        const auto* counters = reinterpret_cast<const luna::Counters*>(scratch);
        cudaError_t e = cudaMemcpyAsync(&host, counters, sizeof(host), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(LUNA_ECUDA, std::string("reading the pass's counters: ") + cudaGetErrorString(e));
        *fallbacks_out = static_cast<int64_t>(host.fallbacks[0]);
        if (host.error & 7ull)
            return fail(LUNA_ENONFINITE, "luna_apply_static_noalloc: the update produced a state that is not finite (error word " +
                                             std::to_string(host.error) + ")");
    }
    return LUNA_OK;
}

}  // extern "C"
