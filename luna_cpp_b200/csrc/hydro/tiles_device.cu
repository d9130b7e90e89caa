// The sweep's tiles cut on the device (tiles.h: DeviceTilePlan), for meshes rebuilt on the device every step.
//
// One block of kTileCells threads per tile of 128 consecutive cells in Morton order. The block orders its cells by list
// length (longest first, then Morton position), puts their lists' neighbours into a shared-memory hash table and keeps
// each neighbour that is not a cell of the tile once: the halo, by cell index (sorted in the fill), as the host cut
// stages it. A planning pass counts each tile's rows and its warps' longest lists; scans turn them into the row and slot
// offsets; a filling pass repeats the table and writes the tiles.
#include <cuda_runtime.h>

#include <climits>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <string>

#include "luna_b200.h"
#include "tiles.h"

namespace luna {
luna_status report_error(luna_status s, const std::string& what);
}  // namespace luna

namespace {

constexpr int kCandidates = 8192;  // list entries of one tile's cells a block takes
static_assert(luna::kTileCells == 128, "4 warps a tile");

luna_status fail(luna_status s, const std::string& what) { return luna::report_error(s, what); }

#define TL_CUDA(call)                                                                                        \
    do {                                                                                                     \
        cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess) return fail(LUNA_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define TL_TRY(call)                  \
    do {                              \
        luna_status s_ = (call);      \
        if (s_ != LUNA_OK) return s_; \
    } while (0)

template <class T>
struct Buf {
    T* ptr = nullptr;
    size_t count = 0;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() {
        if (ptr) cudaFree(ptr);
    }
    luna_status reserve(size_t n, const char* what) {
        if (n == 0) n = 1;
        if (ptr && n <= count) return LUNA_OK;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
        const cudaError_t e = cudaMalloc(&ptr, n * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();
            return fail(e == cudaErrorMemoryAllocation ? LUNA_ENOMEM : LUNA_ECUDA, std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
        }
        count = n;
        return LUNA_OK;
    }
};

struct TileCounters {
    int normal_rows;
    int big_rows;
    int overflow;  // a tile with more list entries than kCandidates, or more rows than kBigTileRows
    int pad;
};

struct Box3 {
    double s[3];
};

int nblocks(int64_t n, int per) { return static_cast<int>((n + per - 1) / per); }

template <int D>
__global__ void k_morton(int64_t n, const double* __restrict__ pos, Box3 box, uint64_t* __restrict__ keys, int32_t* __restrict__ cells) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    keys[i] = luna::morton_key(D, pos + D * i, box.s);
    cells[i] = static_cast<int32_t>(i);
}

struct MeshLists {
    const int32_t* start;
    const int32_t* list;
    const int32_t* owner;
    const int32_t* neighbour;
    __device__ __forceinline__ int32_t other(int32_t e) const {  // the entry's other cell (~f: not owned)
        return e >= 0 ? neighbour[e] : owner[~e];
    }
};

struct PlanOut {
    int32_t* rows;       // [T]
    int32_t* slice_len;  // [T * 4]: each warp's longest list
    TileCounters* ctr;
};

struct FillOut {
    const int32_t* tile_pos;     // [T]: the tile's place u (normal tiles first)
    const int32_t* stage_start;  // [T + 1], by u
    const int32_t* slice_base;   // [T * 4 + 1], by u
    int32_t* order;
    int32_t* stage_cells;
    uint32_t* local;
};

// A tile's distinct list neighbours are kept in a shared-memory hash table (open addressing, linear probing): kHash
// slots, at most kHashFill distinct neighbours (more send the mesh to the host cut, as a tile with too many entries does).
constexpr int kHash = 4096;
constexpr int kHashFill = 3072;
__device__ __forceinline__ int hash_slot(int32_t x) { return static_cast<int>((static_cast<uint32_t>(x) * 2654435761u) >> 20); }

// One tile: plan (Fill false) or fill (Fill true). Each cell's thread inserts its list's neighbours into the block's
// table; a neighbour seen for the first time that is not a cell of the tile joins the halo. The plan counts the rows
// (the tile's cells and the halo); the fill sorts the halo by cell index, stages the rows and gives each list entry its
// neighbour's row (a binary search among the tile's cells, else a table lookup).
template <bool Fill>
__global__ void __launch_bounds__(luna::kTileCells) k_tiles(int64_t n, const int32_t* __restrict__ sorted_cells, MeshLists m, PlanOut plan,
                                                            FillOut fill) {
    constexpr int C = luna::kTileCells;
    __shared__ int32_t key[kHash];
    __shared__ int16_t row_of[kHash];
    __shared__ int32_t halo[kHash];
    __shared__ int32_t own_cell[C], own_len[C], ordered[C], own_sorted[C], own_row[C];
    __shared__ int n_halo, n_entries, table_full;
    const int64_t t = blockIdx.x;
    const int k = threadIdx.x;
    const int64_t idx = t * C + k;
    const int32_t c = idx < n ? sorted_cells[idx] : -1;
    const int len = c >= 0 ? m.start[c + 1] - m.start[c] : -1;
    own_cell[k] = c;
    own_len[k] = len;
    for (int q = k; q < kHash; q += C) key[q] = -1;
    if (k == 0) n_halo = n_entries = table_full = 0;
    __syncthreads();
    // place in the tile: longest list first, then Morton position (idle threads last); rank among the cells by index
    int rank = 0, by_index = 0, n_own = 0;
    for (int q = 0; q < C; ++q) {
        const int lq = own_len[q];
        rank += (lq > len) || (lq == len && q < k);
        by_index += own_cell[q] >= 0 && own_cell[q] < c;
        n_own += own_cell[q] >= 0;
    }
    ordered[rank] = c;
    if (c >= 0) {
        own_sorted[by_index] = c;
        own_row[by_index] = rank;
    }
    __syncthreads();
    auto own_index = [&](int32_t x) {  // x's place among the tile's cells by index, or -1
        int lo = 0, hi = n_own;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (own_sorted[mid] < x)
                lo = mid + 1;
            else
                hi = mid;
        }
        return lo < n_own && own_sorted[lo] == x ? lo : -1;
    };
    if (c >= 0) {
        atomicAdd(&n_entries, len);
        const int first = m.start[c];
        for (int e = 0; e < len; ++e) {
            const int32_t x = m.other(m.list[first + e]);
            int h = hash_slot(x);
            int probe = 0;
            for (; probe < kHash; ++probe) {
                const int32_t prev = atomicCAS(&key[h], -1, x);
                if (prev == -1) {
                    if (own_index(x) < 0) {
                        const int q = atomicAdd(&n_halo, 1);
                        if (q < kHashFill) halo[q] = x;
                    }
                    break;
                }
                if (prev == x) break;
                h = (h + 1) & (kHash - 1);
            }
            if (probe == kHash) table_full = 1;
        }
    }
    __syncthreads();
    const int halo_n = n_halo;
    if (n_entries > kCandidates || halo_n > kHashFill || table_full) {
        if (!Fill && k == 0) atomicOr(&plan.ctr->overflow, 1);
        return;
    }
    const int rows = n_own + halo_n;
    if constexpr (!Fill) {
        if (k < C / 32) {
            const int32_t lead = ordered[32 * k];  // a warp's first cell has its longest list
            plan.slice_len[4 * t + k] = lead >= 0 ? m.start[lead + 1] - m.start[lead] : 0;
        }
        if (k == 0) {
            plan.rows[t] = rows;
            if (rows > luna::kBigTileRows)
                atomicOr(&plan.ctr->overflow, 1);
            else
                atomicMax(rows > luna::kTileRows ? &plan.ctr->big_rows : &plan.ctr->normal_rows, rows);
        }
    } else {
        // the halo by cell index (bitonic, ascending)
        int P = 1;
        while (P < halo_n) P <<= 1;
        for (int q = halo_n + k; q < P; q += C) halo[q] = INT_MAX;
        __syncthreads();
        for (int size = 2; size <= P; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int q = k; q < P; q += C) {
                    const int r = q ^ stride;
                    if (r > q) {
                        const int32_t a = halo[q], b = halo[r];
                        if ((a > b) == ((q & size) == 0)) {
                            halo[q] = b;
                            halo[r] = a;
                        }
                    }
                }
                __syncthreads();
            }
        for (int q = k; q < halo_n; q += C) {  // each halo cell's row, in the table (x was inserted: found within kHash)
            const int32_t x = halo[q];
            int h = hash_slot(x);
            for (int probe = 0; probe < kHash && key[h] != x; ++probe) h = (h + 1) & (kHash - 1);
            if (key[h] == x) row_of[h] = static_cast<int16_t>(n_own + q);
        }
        __syncthreads();
        const int64_t u = fill.tile_pos[t];
        const int64_t s0 = fill.stage_start[u];
        const int32_t mine_cell = ordered[k];
        fill.order[u * C + k] = mine_cell;
        if (k < n_own) fill.stage_cells[s0 + k] = mine_cell;
        for (int q = k; q < halo_n; q += C) fill.stage_cells[s0 + n_own + q] = halo[q];
        if (mine_cell >= 0) {  // each entry's neighbour as a staged row
            const int64_t tg = u * C + k;
            const int64_t slot0 = static_cast<int64_t>(fill.slice_base[tg >> 5]) * 32 + (tg & 31);
            const int first = m.start[mine_cell], count = m.start[mine_cell + 1] - first;
            for (int e = 0; e < count; ++e) {
                const int32_t x = m.other(m.list[first + e]);
                const int o = own_index(x);
                int row;
                if (o >= 0) {
                    row = own_row[o];
                } else {  // a row the tile check rejects if x were missing (it was inserted: found within kHash)
                    int h = hash_slot(x);
                    for (int probe = 0; probe < kHash && key[h] != x; ++probe) h = (h + 1) & (kHash - 1);
                    row = key[h] == x ? row_of[h] : rows;
                }
                fill.local[slot0 + 32 * static_cast<int64_t>(e)] = static_cast<uint32_t>(row);
            }
        }
    }
}

__global__ void k_tile_flags(int64_t T, const int32_t* __restrict__ rows, int32_t* __restrict__ normal, int32_t* __restrict__ big) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t > T) return;
    const bool is_big = t < T && rows[t] > luna::kTileRows;
    normal[t] = t < T && !is_big;
    big[t] = is_big;
}

// Each tile's place u (normal tiles in order, then the big ones), and its rows and warp lengths moved to u.
__global__ void k_tile_place(int64_t T, const int32_t* __restrict__ rows, const int32_t* __restrict__ slice_len,
                             const int32_t* __restrict__ normal_before, const int32_t* __restrict__ big_before, int32_t* __restrict__ pos,
                             int32_t* __restrict__ rows_u, int32_t* __restrict__ len_u) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t > T) return;
    if (t == T) {
        rows_u[T] = 0;
        len_u[4 * T] = 0;
        return;
    }
    const int32_t normals = normal_before[T];
    const bool is_big = rows[t] > luna::kTileRows;
    const int32_t u = is_big ? normals + big_before[t] : normal_before[t];
    pos[t] = u;
    rows_u[u] = rows[t];
    for (int s = 0; s < 4; ++s) len_u[4 * u + s] = slice_len[4 * t + s];
}

// Every tile checked against the lists before the sweep stages by it: a thread's cell is its tile's staged row of that
// thread, each entry's row lies within its tile's rows and stages the entry's neighbour, each slot within the slots,
// and no tile stages more rows than its launch holds. Counts the bad cells.
__global__ void k_check_tiles(int64_t T, int64_t normal_tiles, int normal_rows, int big_rows, int64_t staged, int64_t slots, MeshLists m,
                              const int32_t* __restrict__ order, const int32_t* __restrict__ slice_base, const int32_t* __restrict__ stage_start,
                              const int32_t* __restrict__ stage_cells, const uint32_t* __restrict__ local, unsigned int* __restrict__ bad) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= T * luna::kTileCells) return;
    const int32_t c = order[t];
    if (c < 0) return;
    const int64_t u = t / luna::kTileCells;
    const int64_t s0 = stage_start[u], s1 = stage_start[u + 1];
    const int64_t most = u < normal_tiles ? normal_rows : big_rows;
    const int64_t lane = t % luna::kTileCells;
    if (s0 < 0 || s1 > staged || s1 - s0 > most || lane >= s1 - s0 || stage_cells[s0 + lane] != c) {
        atomicAdd(bad, 1u);
        return;
    }
    const int64_t slot0 = static_cast<int64_t>(slice_base[t >> 5]) * 32 + (t & 31);
    const int first = m.start[c], count = m.start[c + 1] - first;
    for (int e = 0; e < count; ++e) {
        const int64_t slot = slot0 + 32 * static_cast<int64_t>(e);
        if (slot >= slots) {
            atomicAdd(bad, 1u);
            return;
        }
        const uint32_t row = local[slot];
        if (row >= static_cast<uint32_t>(s1 - s0) || stage_cells[s0 + row] != m.other(m.list[first + e])) {
            atomicAdd(bad, 1u);
            return;
        }
    }
}

}  // namespace

namespace luna {

class DeviceTiler {
public:
    Buf<uint64_t> keys, keys_sorted;
    Buf<int32_t> cells, cells_sorted, rows, slice_len, normal, big, normal_before, big_before, pos, rows_u, len_u, stage_start, slice_base;
    Buf<TileCounters> ctr;
    Buf<unsigned int> bad;
    Buf<unsigned char> temp;
    MeshLists lists{};
    int64_t n = 0, T = 0;
    DeviceTilePlan plan;

    template <class F>
    luna_status with_temp(F call) {  // cub's two-call protocol with a kept scratch buffer
        size_t bytes = 0;
        TL_CUDA(call(static_cast<void*>(nullptr), bytes));
        TL_TRY(temp.reserve(bytes, "tile scratch"));
        TL_CUDA(call(static_cast<void*>(temp.ptr), bytes));
        return LUNA_OK;
    }
};

DeviceTiler* device_tiler_create() { return new DeviceTiler(); }
void device_tiler_destroy(DeviceTiler* t) { delete t; }

luna_status device_tiles_plan(DeviceTiler* d, int dim, int64_t n, const double* pos, const double* box, const int32_t* start,
                              const int32_t* list, const int32_t* owner, const int32_t* neighbour, cudaStream_t s, DeviceTilePlan* out) {
    const int64_t T = (n + kTileCells - 1) / kTileCells;
    d->n = n;
    d->T = T;
    d->lists = MeshLists{start, list, owner, neighbour};
    TL_TRY(d->keys.reserve(n, "Morton keys"));
    TL_TRY(d->keys_sorted.reserve(n, "Morton keys"));
    TL_TRY(d->cells.reserve(n, "Morton order"));
    TL_TRY(d->cells_sorted.reserve(n, "Morton order"));
    TL_TRY(d->rows.reserve(T, "tile rows"));
    TL_TRY(d->slice_len.reserve(4 * T, "tile slices"));
    TL_TRY(d->normal.reserve(T + 1, "tile flags"));
    TL_TRY(d->big.reserve(T + 1, "tile flags"));
    TL_TRY(d->normal_before.reserve(T + 1, "tile places"));
    TL_TRY(d->big_before.reserve(T + 1, "tile places"));
    TL_TRY(d->pos.reserve(T, "tile places"));
    TL_TRY(d->rows_u.reserve(T + 1, "tile rows"));
    TL_TRY(d->len_u.reserve(4 * T + 1, "tile slices"));
    TL_TRY(d->stage_start.reserve(T + 1, "tile row starts"));
    TL_TRY(d->slice_base.reserve(4 * T + 1, "slice bases"));
    TL_TRY(d->ctr.reserve(1, "tile counters"));
    const Box3 b{{box[0], box[1], dim == 3 ? box[2] : 1.0}};
    if (dim == 3)
        k_morton<3><<<nblocks(n, 256), 256, 0, s>>>(n, pos, b, d->keys.ptr, d->cells.ptr);
    else
        k_morton<2><<<nblocks(n, 256), 256, 0, s>>>(n, pos, b, d->keys.ptr, d->cells.ptr);
    TL_CUDA(cudaGetLastError());
    const int key_bits = dim == 3 ? 63 : 64;
    TL_TRY(d->with_temp([&](void* tmp, size_t& bytes) {
        return cub::DeviceRadixSort::SortPairs(tmp, bytes, d->keys.ptr, d->keys_sorted.ptr, d->cells.ptr, d->cells_sorted.ptr, n, 0, key_bits, s);
    }));
    TL_CUDA(cudaMemsetAsync(d->ctr.ptr, 0, sizeof(TileCounters), s));
    k_tiles<false><<<static_cast<unsigned int>(T), kTileCells, 0, s>>>(n, d->cells_sorted.ptr, d->lists, PlanOut{d->rows.ptr, d->slice_len.ptr, d->ctr.ptr},
                                                                       FillOut{});
    TL_CUDA(cudaGetLastError());
    k_tile_flags<<<nblocks(T + 1, 256), 256, 0, s>>>(T, d->rows.ptr, d->normal.ptr, d->big.ptr);
    TL_TRY(d->with_temp([&](void* tmp, size_t& bytes) { return cub::DeviceScan::ExclusiveSum(tmp, bytes, d->normal.ptr, d->normal_before.ptr, T + 1, s); }));
    TL_TRY(d->with_temp([&](void* tmp, size_t& bytes) { return cub::DeviceScan::ExclusiveSum(tmp, bytes, d->big.ptr, d->big_before.ptr, T + 1, s); }));
    k_tile_place<<<nblocks(T + 1, 256), 256, 0, s>>>(T, d->rows.ptr, d->slice_len.ptr, d->normal_before.ptr, d->big_before.ptr, d->pos.ptr,
                                                     d->rows_u.ptr, d->len_u.ptr);
    TL_CUDA(cudaGetLastError());
    TL_TRY(d->with_temp([&](void* tmp, size_t& bytes) { return cub::DeviceScan::ExclusiveSum(tmp, bytes, d->rows_u.ptr, d->stage_start.ptr, T + 1, s); }));
    TL_TRY(d->with_temp([&](void* tmp, size_t& bytes) { return cub::DeviceScan::ExclusiveSum(tmp, bytes, d->len_u.ptr, d->slice_base.ptr, 4 * T + 1, s); }));
    TileCounters h{};
    int32_t normals = 0, staged = 0, slices = 0;
    TL_CUDA(cudaMemcpyAsync(&h, d->ctr.ptr, sizeof(h), cudaMemcpyDeviceToHost, s));
    TL_CUDA(cudaMemcpyAsync(&normals, d->normal_before.ptr + T, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    TL_CUDA(cudaMemcpyAsync(&staged, d->stage_start.ptr + T, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    TL_CUDA(cudaMemcpyAsync(&slices, d->slice_base.ptr + 4 * T, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    TL_CUDA(cudaStreamSynchronize(s));
    DeviceTilePlan p;
    p.fits = h.overflow == 0;
    p.tiles = T;
    p.normal_tiles = normals;
    p.staged = staged;
    p.slots = static_cast<int64_t>(slices) * 32;
    p.normal_rows = h.normal_rows;
    p.big_rows = h.big_rows;
    d->plan = p;
    *out = p;
    return LUNA_OK;
}

luna_status device_tiles_fill(DeviceTiler* d, int32_t* order, int32_t* slice_base, int32_t* stage_start, int32_t* stage_cells, uint32_t* local,
                              cudaStream_t s) {
    if (!d->plan.fits) return fail(LUNA_EINVAL, "device tiles: the plan does not fit");
    const int64_t T = d->T;
    TL_CUDA(cudaMemcpyAsync(stage_start, d->stage_start.ptr, (T + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    TL_CUDA(cudaMemcpyAsync(slice_base, d->slice_base.ptr, (4 * T + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    TL_CUDA(cudaMemsetAsync(local, 0, (d->plan.slots > 0 ? d->plan.slots : 1) * sizeof(uint32_t), s));
    const FillOut f{d->pos.ptr, d->stage_start.ptr, d->slice_base.ptr, order, stage_cells, local};
    k_tiles<true><<<static_cast<unsigned int>(T), kTileCells, 0, s>>>(d->n, d->cells_sorted.ptr, d->lists, PlanOut{}, f);
    TL_CUDA(cudaGetLastError());
    TL_TRY(d->bad.reserve(1, "tile check"));
    TL_CUDA(cudaMemsetAsync(d->bad.ptr, 0, sizeof(unsigned int), s));
    const DeviceTilePlan& p = d->plan;
    k_check_tiles<<<nblocks(T * kTileCells, 256), 256, 0, s>>>(T, p.normal_tiles, p.normal_rows, p.big_rows, p.staged, p.slots, d->lists, order,
                                                               slice_base, stage_start, stage_cells, local, d->bad.ptr);
    TL_CUDA(cudaGetLastError());
    unsigned int bad = 0;
    TL_CUDA(cudaMemcpyAsync(&bad, d->bad.ptr, sizeof(bad), cudaMemcpyDeviceToHost, s));
    TL_CUDA(cudaStreamSynchronize(s));
    if (bad) return fail(LUNA_EINVAL, "device tiles: " + std::to_string(bad) + " cells failed the tile check");
    return LUNA_OK;
}

}  // namespace luna
