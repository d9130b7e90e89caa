// The moving mesh's remesh on the device (include/luna_remesh.h).
//
// One thread clips one cell with the host builder's code (voronoi_cell.h; this file is compiled with -fmad=false, so
// the cells have the host builder's bits). The rest is assembly in the host builder's order, done with scans and
// per-segment sorts instead of its serial passes:
//   buckets   counts (atomics), an exclusive scan, a fill (atomics), then each bucket's items sorted by index;
//   cells     each cell's faces, by neighbour, appended to one face buffer at an atomic cursor (a cell's faces stay
//             together; where they land does not matter, every later pass addresses them through the cell);
//   faces     per owner (the lower-numbered cell): its faces towards higher cells plus the faces higher cells saw and it
//             missed (flipped into its frame); a scan gives the face numbers, a segment with flipped faces is re-sorted
//             by neighbour;
//   lists     per cell, every face it is a side of (f, or ~f where it is not the owner), sorted by neighbour.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>
#include <string>
#include <type_traits>

#include "luna_b200.h"
#include "luna_remesh.h"
#include "voronoi_cell.h"
#include "voronoi_grid.h"

#ifndef LUNA_REMESH_DUAL
#define LUNA_REMESH_DUAL 1  // 3D cells kept as triangles of plane triples (DualT), as the host builder's default; 0: face
                            // loops (Poly3T), as the host builder with LUNA_MESH_DUAL=0
#endif

namespace luna {
luna_status report_error(luna_status s, const std::string& what);
}  // namespace luna

namespace {

using namespace luna_voronoi;

luna_status fail(luna_status s, const std::string& what) { return luna::report_error(s, what); }

#define RM_CUDA(call)                                                                                                 \
    do {                                                                                                              \
        cudaError_t e_ = (call);                                                                                      \
        if (e_ != cudaSuccess) return fail(LUNA_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
    } while (0)
#define RM_TRY(call)                     \
    do {                                 \
        luna_status s_ = (call);         \
        if (s_ != LUNA_OK) return s_;    \
    } while (0)

// A device buffer that only grows.
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
            return fail(e == cudaErrorMemoryAllocation ? LUNA_ENOMEM : LUNA_ECUDA,
                        std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
        }
        count = n;
        return LUNA_OK;
    }
    size_t bytes() const { return count * sizeof(T); }
};

struct Counters {
    unsigned long long faces;         // face records the cells appended
    unsigned long long inconsistent;  // faces seen from one side only
    int error;                        // the first cell error (voronoi_cell.h), 0: none
    int error_cell;
    int nonfinite;                    // a generator coordinate was not finite
    unsigned int retry;               // cells the fast path handed to the far search
};

struct Box {
    double s[3];
};

int grid_blocks(int64_t n, int per) { return static_cast<int>((n + per - 1) / per); }

template <int D>
__global__ void k_wrap(int64_t n, const double* __restrict__ in, double* __restrict__ pos, Box box, Counters* c) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n * D) return;
    double x = in[k];
    if (!isfinite(x)) {
        atomicOr(&c->nonfinite, 1);
        x = 0;
    }
    pos[k] = wrap_coordinate(x, box.s[k % D]);
}

template <int D>
__global__ void k_bucket_count(int64_t n, const double* __restrict__ pos, Grid g, int64_t* __restrict__ bucket,
                               unsigned long long* __restrict__ count) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int64_t b = 0;
    for (int a = 0; a < D; ++a) b = b * g.nb[a] + bucket_of(g, pos + D * i, a);
    bucket[i] = b;
    atomicAdd(count + b, 1ull);
}

__global__ void k_bucket_fill(int64_t n, const int64_t* __restrict__ bucket, const int64_t* __restrict__ start,
                              unsigned int* __restrict__ cursor, int32_t* __restrict__ items) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int64_t b = bucket[i];
    items[start[b] + atomicAdd(cursor + b, 1u)] = static_cast<int32_t>(i);
}

// Each bucket's items by index, as the host fills them.
__global__ void k_bucket_sort(int64_t buckets, const int64_t* __restrict__ start, int32_t* __restrict__ items) {
    const int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (b >= buckets) return;
    const int64_t s0 = start[b], s1 = start[b + 1];
    for (int64_t k = s0 + 1; k < s1; ++k) {
        const int32_t x = items[k];
        int64_t j = k - 1;
        while (j >= s0 && items[j] > x) {
            items[j + 1] = items[j];
            --j;
        }
        items[j + 1] = x;
    }
}

struct CellOut {
    double* volume;       // [n]
    double* centroid;     // [n][D]
    int64_t* first;       // [n]: the cell's first record in the face buffer
    int32_t* count;       // [n]
    int32_t* fj;          // [capacity]: neighbour
    double* fa;           // [capacity][D]: area vector out of the cell
    double* fc;           // [capacity][D]: centroid relative to the cell's generator
    unsigned long long capacity;
};

// The cells (all of them, or those of the list), each built by one thread. Without Far, a cell whose search would
// pass the grid's sorted offsets or fill the candidate store is put on the retry list for the Far pass (the same cell
// either way, voronoi_cell.h), which keeps the common cell's code small. 1,024 threads an SM (64 registers, a few
// spilled): 57.5 ms for the 128^3 jittered remesh against 62 ms at 80 registers, 58.6 ms at 896 threads and 58 ms at
// 1,280; in 64-thread blocks (16 an SM) about 1 % faster than in 128-thread blocks, and no faster with the L1 carveout
// preferred.
template <int D, bool Far>
__global__ void __launch_bounds__(64, 16) k_cells(int64_t n, const int32_t* __restrict__ list, const double* __restrict__ pos, Box box, Grid g,
                                               CellOut out, Counters* c, int32_t* __restrict__ retry) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const int64_t i = list ? list[k] : k;
#if LUNA_REMESH_DUAL
    using Poly = std::conditional_t<D == 3, Dual, Poly2>;
#else
    using Poly = std::conditional_t<D == 3, Poly3, Poly2>;
#endif
    Poly poly;
    CellFaces faces;
    Candidates cand;
    double volume = 0, centroid[3] = {0, 0, 0};
#if LUNA_REMESH_DUAL
    int code;
    if constexpr (D == 3)
        code = build_cell_dual<Far>(i, pos, box.s, g, poly, faces, cand, volume, centroid);
    else
        code = build_cell<D, Far>(i, pos, box.s, g, poly, faces, cand, volume, centroid);
#else
    const int code = build_cell<D, Far>(i, pos, box.s, g, poly, faces, cand, volume, centroid);
#endif
    if (code != kCellOk) {
        out.first[i] = 0;
        out.count[i] = 0;
        if (!Far && (code == kOutOfOffsets || code == kCandidates))
            retry[atomicAdd(&c->retry, 1u)] = static_cast<int32_t>(i);
        else if (atomicCAS(&c->error, 0, code) == 0)
            c->error_cell = static_cast<int>(i);
        return;
    }
    out.volume[i] = volume;
    for (int a = 0; a < D; ++a) out.centroid[D * i + a] = centroid[a];
    const unsigned long long base = atomicAdd(&c->faces, static_cast<unsigned long long>(faces.n));
    out.first[i] = static_cast<int64_t>(base);
    out.count[i] = faces.n;
    if (base + faces.n > out.capacity) return;  // the host grows the buffer and runs the cells again
    for (int e = 0; e < faces.n; ++e) {
        const int f = faces.order[e];
        const int64_t r = static_cast<int64_t>(base) + e;
        out.fj[r] = faces.j[f];
        for (int a = 0; a < D; ++a) {
            out.fa[D * r + a] = faces.a[f][a];
            out.fc[D * r + a] = faces.c[f][a];
        }
    }
}

// Whether cell c has a face towards j (its records are sorted by neighbour).
__device__ __forceinline__ bool has_face(const int64_t* first, const int32_t* count, const int32_t* fj, int32_t c, int32_t j) {
    int64_t lo = first[c], hi = lo + count[c];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (fj[mid] < j)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < first[c] + count[c] && fj[lo] == j;
}

// Per owner: its faces towards higher cells (fwd), and (flips) the faces higher cells saw that it missed.
__global__ void k_count_owned(int64_t n, const int64_t* __restrict__ first, const int32_t* __restrict__ count,
                              const int32_t* __restrict__ fj, int32_t* __restrict__ fwd, int32_t* __restrict__ flips,
                              Counters* c) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int own = 0;
    unsigned long long inconsistent = 0;
    const int64_t f0 = first[i];
    for (int k = 0; k < count[i]; ++k) {
        const int32_t j = fj[f0 + k];
        const bool seen = has_face(first, count, fj, j, static_cast<int32_t>(i));
        if (j > i) {
            ++own;
            if (!seen) ++inconsistent;
        } else if (!seen) {
            ++inconsistent;
            atomicAdd(flips + j, 1);
        }
    }
    fwd[i] = own;
    if (inconsistent) atomicAdd(&c->inconsistent, inconsistent);
}

__global__ void k_segment_lengths(int64_t n, const int32_t* __restrict__ fwd, const int32_t* __restrict__ flips,
                                  int64_t* __restrict__ length) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i > n) return;
    length[i] = i < n ? static_cast<int64_t>(fwd[i]) + flips[i] : 0;
}

struct FaceOut {
    int32_t* owner;
    int32_t* neighbour;
    double* area;
    double* fcen;
};

template <int D>
__global__ void k_emit(int64_t n, const int64_t* __restrict__ first, const int32_t* __restrict__ count,
                       const int32_t* __restrict__ fj, const double* __restrict__ fa, const double* __restrict__ fc,
                       const double* __restrict__ pos, Box box, const int64_t* __restrict__ face_start,
                       const int32_t* __restrict__ fwd, unsigned int* __restrict__ flip_cursor, FaceOut out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int64_t f0 = first[i];
    int64_t next = face_start[i];
    for (int k = 0; k < count[i]; ++k) {
        const int64_t r = f0 + k;
        const int32_t j = fj[r];
        if (j > i) {
            const int64_t f = next++;
            out.owner[f] = static_cast<int32_t>(i);
            out.neighbour[f] = j;
            for (int a = 0; a < D; ++a) {
                out.area[D * f + a] = fa[D * r + a];
                out.fcen[D * f + a] = fc[D * r + a];
            }
        } else if (!has_face(first, count, fj, j, static_cast<int32_t>(i))) {
            // owner j missed it: the area flips; the centroid, relative to j's generator, is this cell's centroid plus
            // the nearest image of x_i - x_j
            const int64_t f = face_start[j] + fwd[j] + atomicAdd(flip_cursor + j, 1u);
            out.owner[f] = j;
            out.neighbour[f] = static_cast<int32_t>(i);
            for (int a = 0; a < D; ++a) {
                double d = pos[D * i + a] - pos[D * j + a];
                d -= box.s[a] * nearbyint(d / box.s[a]);
                out.area[D * f + a] = -fa[D * r + a];
                out.fcen[D * f + a] = fc[D * r + a] + d;
            }
        }
    }
}

// An owner's segment holding flipped faces, sorted by neighbour.
template <int D>
__global__ void k_sort_segments(int64_t n, const int64_t* __restrict__ face_start, const int32_t* __restrict__ flips,
                                FaceOut out) {
    const int64_t o = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (o >= n || flips[o] == 0) return;
    const int64_t s0 = face_start[o], s1 = face_start[o + 1];
    for (int64_t k = s0 + 1; k < s1; ++k) {
        const int32_t key = out.neighbour[k];
        double a[D], c[D];
        for (int x = 0; x < D; ++x) {
            a[x] = out.area[D * k + x];
            c[x] = out.fcen[D * k + x];
        }
        int64_t j = k - 1;
        while (j >= s0 && out.neighbour[j] > key) {
            out.neighbour[j + 1] = out.neighbour[j];
            for (int x = 0; x < D; ++x) {
                out.area[D * (j + 1) + x] = out.area[D * j + x];
                out.fcen[D * (j + 1) + x] = out.fcen[D * j + x];
            }
            --j;
        }
        out.neighbour[j + 1] = key;
        for (int x = 0; x < D; ++x) {
            out.area[D * (j + 1) + x] = a[x];
            out.fcen[D * (j + 1) + x] = c[x];
        }
    }
}

__global__ void k_degree(int64_t F, const int32_t* __restrict__ owner, const int32_t* __restrict__ neighbour,
                         int32_t* __restrict__ degree) {
    const int64_t f = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (f >= F) return;
    atomicAdd(degree + owner[f], 1);
    atomicAdd(degree + neighbour[f], 1);
}

__global__ void k_list_fill(int64_t F, const int32_t* __restrict__ owner, const int32_t* __restrict__ neighbour,
                            const int32_t* __restrict__ start, unsigned int* __restrict__ cursor, int32_t* __restrict__ list,
                            int32_t* __restrict__ key) {
    const int64_t f = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (f >= F) return;
    const int32_t o = owner[f], j = neighbour[f];
    int32_t s = start[o] + static_cast<int32_t>(atomicAdd(cursor + o, 1u));
    list[s] = static_cast<int32_t>(f);
    key[s] = j;
    s = start[j] + static_cast<int32_t>(atomicAdd(cursor + j, 1u));
    list[s] = ~static_cast<int32_t>(f);
    key[s] = o;
}

// Each cell's list by neighbour.
__global__ void k_list_sort(int64_t n, const int32_t* __restrict__ start, int32_t* __restrict__ list, int32_t* __restrict__ key) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int32_t s0 = start[i], s1 = start[i + 1];
    for (int32_t k = s0 + 1; k < s1; ++k) {
        const int32_t x = key[k], e = list[k];
        int32_t j = k - 1;
        while (j >= s0 && key[j] > x) {
            key[j + 1] = key[j];
            list[j + 1] = list[j];
            --j;
        }
        key[j + 1] = x;
        list[j + 1] = e;
    }
}

const char* cell_error(int code) {
    switch (code) {
        case kOutOfOffsets: return "a cell reaches farther than a box side from its generator (too few points for the box)";
        case kReachesBox: return "a cell reaches the box (box too small for the points)";
        case kTouchesSelf: return "a cell touches its own periodic image (box too small for the points)";
        case kDuplicatePair: return "two faces between the same pair of cells (box too small for unique nearest images)";
        case kCapacity: return "a cell has more vertices or faces than the remesher holds";
        case kCandidates: return "more generators at one distance from a cell than the remesher holds";
        default: return "unknown cell error";
    }
}

}  // namespace

struct luna_remesh {
    int dim = 3;
    Box box{};
    cudaStream_t stream = nullptr;
    int64_t shape_n = -1;
    GridShape shape;
    Buf<int32_t> offsets;
    Buf<double> bound2;
    Buf<double> input, pos;
    Buf<int64_t> bucket, bucket_start;
    Buf<unsigned long long> bucket_count;
    Buf<unsigned int> cursor;
    Buf<int32_t> items;
    Buf<double> volume, centroid;
    Buf<int64_t> first;
    Buf<int32_t> retry;  // cells the fast path handed to the far search
    Buf<int32_t> count, fj;
    Buf<double> fa, fc;
    Buf<int32_t> fwd, flips;
    Buf<int64_t> seg_length, face_start;
    Buf<int32_t> owner, neighbour, degree, start, list, key;
    Buf<double> area, fcen;
    Buf<Counters> counters;
    Buf<unsigned char> scan_temp;
    unsigned long long capacity = 0;

    template <class T>
    luna_status exclusive_scan(const T* in, T* out, int64_t items) {
        size_t bytes = 0;
        RM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, items, stream));
        RM_TRY(scan_temp.reserve(bytes, "scan scratch"));
        RM_CUDA(cub::DeviceScan::ExclusiveSum(scan_temp.ptr, bytes, in, out, items, stream));
        return LUNA_OK;
    }

    template <int D>
    luna_status build(int64_t n, const double* points, bool on_device, luna_mesh_desc* mesh, int64_t* inconsistent);
};

template <int D>
luna_status luna_remesh::build(int64_t n, const double* points, bool on_device, luna_mesh_desc* mesh, int64_t* inconsistent) {
    const int T = 256;
    if (shape_n != n) {  // the grid's shape depends on n and the box only
        shape.build(D, n, box.s);
        RM_TRY(offsets.reserve(shape.offsets.size(), "bucket offsets"));
        RM_TRY(bound2.reserve(shape.bound2.size(), "bucket bounds"));
        RM_CUDA(cudaMemcpy(offsets.ptr, shape.offsets.data(), shape.offsets.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        RM_CUDA(cudaMemcpy(bound2.ptr, shape.bound2.data(), shape.bound2.size() * sizeof(double), cudaMemcpyHostToDevice));
        shape_n = n;
    }
    const int64_t B = shape.buckets;
    RM_TRY(counters.reserve(1, "remesh counters"));
    RM_TRY(pos.reserve(n * D, "generators"));
    RM_TRY(bucket.reserve(n, "buckets"));
    RM_TRY(bucket_count.reserve(B + 1, "bucket counts"));
    RM_TRY(bucket_start.reserve(B + 1, "bucket starts"));
    RM_TRY(cursor.reserve(B > n + 1 ? B : n + 1, "cursors"));
    RM_TRY(items.reserve(n, "bucket items"));
    RM_TRY(volume.reserve(n, "volumes"));
    RM_TRY(centroid.reserve(n * D, "centroids"));
    RM_TRY(first.reserve(n, "cell records"));
    RM_TRY(retry.reserve(n, "far cells"));
    RM_TRY(count.reserve(n, "cell records"));
    RM_TRY(fwd.reserve(n, "owned faces"));
    RM_TRY(flips.reserve(n, "flipped faces"));
    RM_TRY(seg_length.reserve(n + 1, "segments"));
    RM_TRY(face_start.reserve(n + 1, "segments"));
    RM_TRY(degree.reserve(n + 1, "degrees"));
    RM_TRY(start.reserve(n + 1, "cell_face_start"));

    const double* src = points;
    if (!on_device) {
        RM_TRY(input.reserve(n * D, "generators"));
        RM_CUDA(cudaMemcpyAsync(input.ptr, points, n * D * sizeof(double), cudaMemcpyHostToDevice, stream));
        src = input.ptr;
    }
    RM_CUDA(cudaMemsetAsync(counters.ptr, 0, sizeof(Counters), stream));
    k_wrap<D><<<grid_blocks(n * D, T), T, 0, stream>>>(n, src, pos.ptr, box, counters.ptr);
    RM_CUDA(cudaGetLastError());

    // buckets
    const Grid g = shape.view(bucket_start.ptr, items.ptr, offsets.ptr, bound2.ptr);
    RM_CUDA(cudaMemsetAsync(bucket_count.ptr, 0, (B + 1) * sizeof(unsigned long long), stream));
    k_bucket_count<D><<<grid_blocks(n, T), T, 0, stream>>>(n, pos.ptr, g, bucket.ptr, bucket_count.ptr);
    RM_CUDA(cudaGetLastError());
    RM_TRY(exclusive_scan(reinterpret_cast<const int64_t*>(bucket_count.ptr), bucket_start.ptr, B + 1));
    RM_CUDA(cudaMemsetAsync(cursor.ptr, 0, B * sizeof(unsigned int), stream));
    k_bucket_fill<<<grid_blocks(n, T), T, 0, stream>>>(n, bucket.ptr, bucket_start.ptr, cursor.ptr, items.ptr);
    k_bucket_sort<<<grid_blocks(B, T), T, 0, stream>>>(B, bucket_start.ptr, items.ptr);
    RM_CUDA(cudaGetLastError());

    // cells: a first guess of the face records (16 a cell in 3D, 6 in 2D on a jittered lattice), grown once if short
    if (capacity == 0) capacity = static_cast<unsigned long long>(n) * (D == 3 ? 18 : 7);
    Counters h{};
    for (int attempt = 0; attempt < 2; ++attempt) {
        RM_TRY(fj.reserve(capacity, "face records"));
        RM_TRY(fa.reserve(capacity * D, "face records"));
        RM_TRY(fc.reserve(capacity * D, "face records"));
        if (attempt > 0) RM_CUDA(cudaMemsetAsync(counters.ptr, 0, sizeof(Counters), stream));
        const CellOut out{volume.ptr, centroid.ptr, first.ptr, count.ptr, fj.ptr, fa.ptr, fc.ptr, capacity};
        k_cells<D, false><<<grid_blocks(n, 64), 64, 0, stream>>>(n, nullptr, pos.ptr, box, g, out, counters.ptr, retry.ptr);
        RM_CUDA(cudaGetLastError());
        RM_CUDA(cudaMemcpyAsync(&h, counters.ptr, sizeof(Counters), cudaMemcpyDeviceToHost, stream));
        RM_CUDA(cudaStreamSynchronize(stream));
        if (h.retry > 0 && !h.error && !h.nonfinite) {  // the far search for the cells the fast path handed on
            k_cells<D, true><<<grid_blocks(h.retry, 64), 64, 0, stream>>>(h.retry, retry.ptr, pos.ptr, box, g, out, counters.ptr, nullptr);
            RM_CUDA(cudaGetLastError());
            RM_CUDA(cudaMemcpyAsync(&h, counters.ptr, sizeof(Counters), cudaMemcpyDeviceToHost, stream));
            RM_CUDA(cudaStreamSynchronize(stream));
        }
        if (h.nonfinite) return fail(LUNA_EINVAL, "luna_remesh_build: non-finite point");
        if (h.error) return fail(LUNA_EINVAL, std::string("luna_remesh_build: cell ") + std::to_string(h.error_cell) + ": " + cell_error(h.error));
        if (h.faces <= capacity) break;
        capacity = h.faces + h.faces / 16;
    }

    // faces, by owner then neighbour
    RM_CUDA(cudaMemsetAsync(flips.ptr, 0, n * sizeof(int32_t), stream));
    k_count_owned<<<grid_blocks(n, T), T, 0, stream>>>(n, first.ptr, count.ptr, fj.ptr, fwd.ptr, flips.ptr, counters.ptr);
    k_segment_lengths<<<grid_blocks(n + 1, T), T, 0, stream>>>(n, fwd.ptr, flips.ptr, seg_length.ptr);
    RM_CUDA(cudaGetLastError());
    RM_TRY(exclusive_scan(static_cast<const int64_t*>(seg_length.ptr), face_start.ptr, n + 1));
    int64_t F = 0;
    RM_CUDA(cudaMemcpyAsync(&F, face_start.ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
    RM_CUDA(cudaMemcpyAsync(&h, counters.ptr, sizeof(Counters), cudaMemcpyDeviceToHost, stream));
    RM_CUDA(cudaStreamSynchronize(stream));
    if (2 * F >= (int64_t(1) << 31) - 1) return fail(LUNA_EINVAL, "luna_remesh_build: too many faces for int32 lists");
    RM_TRY(owner.reserve(F, "owner"));
    RM_TRY(neighbour.reserve(F, "neighbour"));
    RM_TRY(area.reserve(F * D, "area"));
    RM_TRY(fcen.reserve(F * D, "face_centroid"));
    RM_TRY(list.reserve(2 * F, "cell_face"));
    RM_TRY(key.reserve(2 * F, "list keys"));
    const FaceOut faces{owner.ptr, neighbour.ptr, area.ptr, fcen.ptr};
    RM_CUDA(cudaMemsetAsync(cursor.ptr, 0, n * sizeof(unsigned int), stream));
    k_emit<D><<<grid_blocks(n, T), T, 0, stream>>>(n, first.ptr, count.ptr, fj.ptr, fa.ptr, fc.ptr, pos.ptr, box, face_start.ptr,
                                                    fwd.ptr, cursor.ptr, faces);
    k_sort_segments<D><<<grid_blocks(n, T), T, 0, stream>>>(n, face_start.ptr, flips.ptr, faces);
    RM_CUDA(cudaGetLastError());

    // lists, by neighbour
    RM_CUDA(cudaMemsetAsync(degree.ptr, 0, (n + 1) * sizeof(int32_t), stream));
    if (F > 0) k_degree<<<grid_blocks(F, T), T, 0, stream>>>(F, owner.ptr, neighbour.ptr, degree.ptr);
    RM_CUDA(cudaGetLastError());
    RM_TRY(exclusive_scan(static_cast<const int32_t*>(degree.ptr), start.ptr, n + 1));
    RM_CUDA(cudaMemsetAsync(cursor.ptr, 0, n * sizeof(unsigned int), stream));
    if (F > 0) k_list_fill<<<grid_blocks(F, T), T, 0, stream>>>(F, owner.ptr, neighbour.ptr, start.ptr, cursor.ptr, list.ptr, key.ptr);
    k_list_sort<<<grid_blocks(n, T), T, 0, stream>>>(n, start.ptr, list.ptr, key.ptr);
    RM_CUDA(cudaGetLastError());
    RM_CUDA(cudaStreamSynchronize(stream));

    *mesh = luna_mesh_desc{};
    mesh->dim = D;
    mesh->n_cells = n;
    mesh->n_faces = F;
    mesh->owner = owner.ptr;
    mesh->neighbour = neighbour.ptr;
    mesh->cell_face_start = start.ptr;
    mesh->cell_face = list.ptr;
    mesh->area = area.ptr;
    mesh->face_centroid = fcen.ptr;
    mesh->centroid = centroid.ptr;
    mesh->volume = volume.ptr;
    mesh->positions = pos.ptr;
    for (int a = 0; a < 3; ++a) mesh->box[a] = a < D ? box.s[a] : 0.0;
    mesh->on_device = 1;
    if (inconsistent) *inconsistent = static_cast<int64_t>(h.inconsistent);
    return LUNA_OK;
}

extern "C" {

LUNA_API luna_status luna_remesh_create(int dim, const double* box, luna_remesh** out) {
    if (!out || !box) return fail(LUNA_EINVAL, "luna_remesh_create: null argument");
    *out = nullptr;
    if (dim != 2 && dim != 3) return fail(LUNA_EINVAL, "luna_remesh_create: dim must be 2 or 3");
    for (int a = 0; a < dim; ++a)
        if (!(box[a] > 0) || !std::isfinite(box[a])) return fail(LUNA_EINVAL, "luna_remesh_create: box sides must be positive");
    auto* r = new luna_remesh();
    r->dim = dim;
    for (int a = 0; a < 3; ++a) r->box.s[a] = a < dim ? box[a] : 1.0;
    *out = r;
    return LUNA_OK;
}

LUNA_API luna_status luna_remesh_destroy(luna_remesh* r) {
    delete r;
    return LUNA_OK;
}

LUNA_API luna_status luna_remesh_set_stream(luna_remesh* r, void* stream) {
    if (!r) return fail(LUNA_EINVAL, "luna_remesh_set_stream: null remesher");
    r->stream = static_cast<cudaStream_t>(stream);
    return LUNA_OK;
}

LUNA_API luna_status luna_remesh_build(luna_remesh* r, int64_t n, const double* points, int on_device, luna_mesh_desc* mesh,
                                       int64_t* inconsistent) {
    if (!r || !points || !mesh) return fail(LUNA_EINVAL, "luna_remesh_build: null argument");
    if (n < 2 || n >= (int64_t(1) << 30)) return fail(LUNA_EINVAL, "luna_remesh_build: n out of range");
    return r->dim == 3 ? r->build<3>(n, points, on_device != 0, mesh, inconsistent) : r->build<2>(n, points, on_device != 0, mesh, inconsistent);
}

LUNA_API luna_status luna_remesh_points(luna_remesh* r, int64_t n, double** points) {
    if (!r || !points) return fail(LUNA_EINVAL, "luna_remesh_points: null argument");
    if (n < 2 || n >= (int64_t(1) << 30)) return fail(LUNA_EINVAL, "luna_remesh_points: n out of range");
    RM_TRY(r->input.reserve(static_cast<size_t>(n) * r->dim, "generators"));
    *points = r->input.ptr;
    return LUNA_OK;
}

LUNA_API luna_status luna_remesh_device_bytes(const luna_remesh* r, int64_t* out) {
    if (!r || !out) return fail(LUNA_EINVAL, "luna_remesh_device_bytes: null argument");
    const size_t b = r->offsets.bytes() + r->bound2.bytes() + r->input.bytes() + r->pos.bytes() + r->bucket.bytes() +
                     r->bucket_start.bytes() + r->bucket_count.bytes() + r->cursor.bytes() + r->items.bytes() + r->volume.bytes() +
                     r->centroid.bytes() + r->first.bytes() + r->retry.bytes() + r->count.bytes() + r->fj.bytes() + r->fa.bytes() + r->fc.bytes() +
                     r->fwd.bytes() + r->flips.bytes() + r->seg_length.bytes() + r->face_start.bytes() + r->owner.bytes() +
                     r->neighbour.bytes() + r->degree.bytes() + r->start.bytes() + r->list.bytes() + r->key.bytes() + r->area.bytes() +
                     r->fcen.bytes() + r->counters.bytes() + r->scan_temp.bytes();
    *out = static_cast<int64_t>(b);
    return LUNA_OK;
}

}  // extern "C"
