// Periodic Voronoi mesh builder: cells by half-space clipping (voronoi_cell.h), faces in voronoi-cpp's layout (see luna_mesh.h).
//
// Each cell starts as the periodic box centred on its generator (its own images bound it there) and is clipped by the
// bisector plane (2D: line) of every generator image that can still cut it. Candidates come from a bucket grid visited in
// order of a lower bound on their distance; the walk stops once that bound exceeds twice the largest vertex radius of the
// cell (no farther generator can cut it). Each face is then emitted once, by its owner, the lower-numbered of its two
// cells; faces are numbered by owner, then by neighbour, and every cell's list is ordered by neighbour.

#include "luna_mesh.h"
#include "voronoi_cell.h"
#include "voronoi_grid.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_error;

int fail(const std::string& what) {
    g_error = what;
    return 1;
}

// One emitted face of a cell: the neighbour, area vector out of the cell, face centroid relative to the cell's generator.
struct CellFace {
    int32_t j;
    double a[3];
    double c[3];
};

// The grid's buckets filled on the host: items in index order within each bucket.
struct HostGrid {
    luna_voronoi::GridShape shape;
    std::vector<int64_t> start;
    std::vector<int32_t> items;

    void build(int d, int64_t n, const double* pts, const double* side) {
        shape.build(d, n, side);
        const luna_voronoi::Grid g = view();
        std::vector<int64_t> count(shape.buckets + 1, 0);
        std::vector<int64_t> of(n);
        for (int64_t i = 0; i < n; ++i) {
            int64_t b = 0;
            for (int a = 0; a < d; ++a) b = b * shape.nb[a] + luna_voronoi::bucket_of(g, pts + d * i, a);
            of[i] = b;
            ++count[b + 1];
        }
        for (int64_t b = 0; b < shape.buckets; ++b) count[b + 1] += count[b];
        start = count;
        items.resize(n);
        std::vector<int64_t> fill(count.begin(), count.end() - 1);
        for (int64_t i = 0; i < n; ++i) items[fill[of[i]]++] = static_cast<int32_t>(i);
    }
    luna_voronoi::Grid view() const {
        return shape.view(start.data(), items.data(), shape.offsets.data(), shape.bound2.data());
    }
};

const char* cell_error(int code) {
    switch (code) {
        case luna_voronoi::kOutOfOffsets: return "voronoi: a cell reaches farther than a box side from its generator (too few points for the box)";
        case luna_voronoi::kReachesBox: return "voronoi: a cell reaches the box (box too small for the points)";
        case luna_voronoi::kTouchesSelf: return "voronoi: a cell touches its own periodic image (box too small for the points)";
        case luna_voronoi::kDuplicatePair: return "voronoi: two faces between the same pair of cells (box too small for unique nearest images)";
        case luna_voronoi::kCapacity: return "voronoi: a cell has more vertices or faces than the builder holds";
        case luna_voronoi::kCandidates: return "voronoi: more generators at one distance from a cell than the builder holds";
        default: return "voronoi: unknown cell error";
    }
}

}  // namespace

struct luna_mesh_build {
    int dim = 3;
    int64_t n = 0, f = 0, inconsistent = 0;
    double box[3] = {1, 1, 1};
    std::vector<int32_t> owner, neighbour, start, list;
    std::vector<double> area, face_centroid, centroid, volume, positions;
};

namespace {

// 3D cells are built as DualT (voronoi_cell.h: triangles of plane triples), as the device remesher builds them, unless
// LUNA_MESH_DUAL=0 in the environment (read once per process) selects the face-loop cell (Poly3T).
bool dual_cells() {
    static const bool on = [] {
        const char* v = std::getenv("LUNA_MESH_DUAL");
        return !(v && v[0] == '0');
    }();
    return on;
}

// Cell i: clipped (voronoi_cell.h), then its faces by neighbour, volume and centroid. Returns 0 or a cell error.
struct CellWork {
    luna_voronoi::HostPoly3 p3;
    luna_voronoi::HostPoly2 p2;
    luna_voronoi::HostCellFaces faces;
    luna_voronoi::HostCandidates cand;
    luna_voronoi::HostDual dual;
};

int cell(int dim, int64_t i, const double* pos, const double* side, const luna_voronoi::Grid& grid, CellWork& work,
         std::vector<CellFace>& faces, double& volume, double* centroid) {
    const int code = dim == 3 ? (dual_cells() ? luna_voronoi::build_cell_dual<true>(i, pos, side, grid, work.dual, work.faces, work.cand, volume, centroid)
                                              : luna_voronoi::build_cell<3>(i, pos, side, grid, work.p3, work.faces, work.cand, volume, centroid))
                              : luna_voronoi::build_cell<2>(i, pos, side, grid, work.p2, work.faces, work.cand, volume, centroid);
    if (code != luna_voronoi::kCellOk) return code;
    faces.resize(work.faces.n);
    for (int k = 0; k < work.faces.n; ++k) {
        const int e = work.faces.order[k];
        faces[k].j = work.faces.j[e];
        for (int a = 0; a < 3; ++a) {
            faces[k].a[a] = work.faces.a[e][a];
            faces[k].c[a] = work.faces.c[e][a];
        }
    }
    return 0;
}

}  // namespace

extern "C" {

const char* luna_mesh_error(void) { return g_error.c_str(); }

int luna_mesh_create(int dim, int64_t n, const double* points, const double* box, int threads, luna_mesh_build** out) {
    if (!out || !points || !box) return fail("luna_mesh_create: null argument");
    *out = nullptr;
    if (dim != 2 && dim != 3) return fail("luna_mesh_create: dim must be 2 or 3");
    if (n < 2 || n >= (int64_t(1) << 30)) return fail("luna_mesh_create: n out of range");
    for (int a = 0; a < dim; ++a)
        if (!(box[a] > 0)) return fail("luna_mesh_create: box sides must be positive");
    auto m = new luna_mesh_build();
    m->dim = dim;
    m->n = n;
    for (int a = 0; a < 3; ++a) m->box[a] = a < dim ? box[a] : 0.0;
    // Generators wrapped into [0, side).
    m->positions.resize(static_cast<size_t>(n) * dim);
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < dim; ++a) {
            double x = points[dim * i + a];
            if (!std::isfinite(x)) {
                delete m;
                return fail("luna_mesh_create: non-finite point");
            }
            m->positions[dim * i + a] = luna_voronoi::wrap_coordinate(x, box[a]);
        }
    HostGrid grid;
    grid.build(dim, n, m->positions.data(), box);
    const luna_voronoi::Grid view = grid.view();
    m->volume.resize(n);
    m->centroid.resize(static_cast<size_t>(n) * dim);
    // Per cell faces, kept per thread chunk and gathered after.
    std::vector<std::vector<CellFace>> per_cell(n);
    std::string first_error;
    bool ok = true;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel
    {
        std::unique_ptr<CellWork> work(new CellWork());
        std::vector<CellFace> faces;
#pragma omp for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            if (!ok) continue;
            double vol = 0;
            const int code = cell(dim, i, m->positions.data(), box, view, *work, faces, vol, &m->centroid[dim * i]);
            if (code != 0) {
#pragma omp critical
                {
                    if (ok) first_error = cell_error(code);
                    ok = false;
                }
                continue;
            }
            m->volume[i] = vol;
            per_cell[i] = faces;
        }
    }
    if (!ok) {
        delete m;
        return fail(first_error);
    }
    // Faces by owner (the lower-numbered cell), then neighbour. A face seen only by the higher-numbered cell is kept in
    // that cell's geometry, flipped to the owner's frame.
    auto has = [&](int64_t c, int32_t j) {
        const auto& v = per_cell[c];
        auto it = std::lower_bound(v.begin(), v.end(), j, [](const CellFace& f, int32_t x) { return f.j < x; });
        return it != v.end() && it->j == j;
    };
    std::vector<int64_t> owned(n + 1, 0);
    int64_t inconsistent = 0;
#pragma omp parallel for reduction(+ : inconsistent) schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; ++i) {
        int64_t c = 0;
        for (const auto& f : per_cell[i]) {
            if (f.j > i) {
                ++c;
                if (!has(f.j, static_cast<int32_t>(i))) ++inconsistent;
            } else if (!has(f.j, static_cast<int32_t>(i))) {
                ++c;  // only this (higher) side saw it: emitted here for the owner f.j, see below
                ++inconsistent;
            }
        }
        owned[i + 1] = c;
    }
    m->inconsistent = inconsistent;
    // The emitting cell e holds faces owned by e (j > e) and faces owned by j < e that j missed; counts by emitter first.
    for (int64_t i = 0; i < n; ++i) owned[i + 1] += owned[i];
    const int64_t F = owned[n];
    if (F >= (int64_t(1) << 31) - 1) {
        delete m;
        return fail("luna_mesh_create: too many faces for int32 indices");
    }
    struct Raw {
        int32_t o, j;
        double a[3], c[3];
    };
    std::vector<Raw> raw(F);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; ++i) {
        int64_t k = owned[i];
        for (const auto& f : per_cell[i]) {
            if (f.j > i) {
                Raw r;
                r.o = static_cast<int32_t>(i);
                r.j = f.j;
                for (int a = 0; a < 3; ++a) {
                    r.a[a] = f.a[a];
                    r.c[a] = f.c[a];
                }
                raw[k++] = r;
            } else if (!has(f.j, static_cast<int32_t>(i))) {
                // Owner f.j: area flips; centroid relative to the owner's generator = own centroid + (x_i - x_o) nearest image.
                Raw r;
                r.o = f.j;
                r.j = static_cast<int32_t>(i);
                for (int a = 0; a < dim; ++a) {
                    double d = m->positions[dim * i + a] - m->positions[dim * f.j + a];
                    d -= box[a] * std::nearbyint(d / box[a]);
                    r.a[a] = -f.a[a];
                    r.c[a] = f.c[a] + d;
                }
                for (int a = dim; a < 3; ++a) r.a[a] = r.c[a] = 0;
                raw[k++] = r;
            }
        }
    }
    std::stable_sort(raw.begin(), raw.end(), [](const Raw& p, const Raw& q) { return p.o != q.o ? p.o < q.o : p.j < q.j; });
    m->f = F;
    m->owner.resize(F);
    m->neighbour.resize(F);
    m->area.resize(static_cast<size_t>(F) * dim);
    m->face_centroid.resize(static_cast<size_t>(F) * dim);
    std::vector<int64_t> deg(n + 1, 0);
    for (int64_t f = 0; f < F; ++f) {
        m->owner[f] = raw[f].o;
        m->neighbour[f] = raw[f].j;
        for (int a = 0; a < dim; ++a) {
            m->area[dim * f + a] = raw[f].a[a];
            m->face_centroid[dim * f + a] = raw[f].c[a];
        }
        ++deg[raw[f].o + 1];
        ++deg[raw[f].j + 1];
    }
    for (int64_t i = 0; i < n; ++i) deg[i + 1] += deg[i];
    m->start.resize(n + 1);
    for (int64_t i = 0; i <= n; ++i) m->start[i] = static_cast<int32_t>(deg[i]);
    // Lists ordered by neighbour: collect (neighbour, entry) per cell and sort.
    std::vector<std::pair<int32_t, int32_t>> entries(2 * F);
    {
        std::vector<int64_t> fill(deg.begin(), deg.end() - 1);
        for (int64_t f = 0; f < F; ++f) {
            entries[fill[raw[f].o]++] = {raw[f].j, static_cast<int32_t>(f)};
            entries[fill[raw[f].j]++] = {raw[f].o, ~static_cast<int32_t>(f)};
        }
    }
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < n; ++i) std::sort(entries.begin() + deg[i], entries.begin() + deg[i + 1]);
    m->list.resize(2 * F);
    for (int64_t k = 0; k < 2 * F; ++k) m->list[k] = entries[k].second;
    *out = m;
    return 0;
}

int luna_mesh_arrays_of(const luna_mesh_build* m, luna_mesh_arrays* out) {
    if (!m || !out) return fail("luna_mesh_arrays_of: null argument");
    out->dim = m->dim;
    out->n_cells = m->n;
    out->n_faces = m->f;
    out->owner = m->owner.data();
    out->neighbour = m->neighbour.data();
    out->cell_face_start = m->start.data();
    out->cell_face = m->list.data();
    out->area = m->area.data();
    out->face_centroid = m->face_centroid.data();
    out->centroid = m->centroid.data();
    out->volume = m->volume.data();
    out->positions = m->positions.data();
    for (int a = 0; a < 3; ++a) out->box[a] = m->box[a];
    out->inconsistent = m->inconsistent;
    return 0;
}

void luna_mesh_free(luna_mesh_build* m) { delete m; }

int luna_jittered_points(int dim, const int* cells, const double* side, double jitter, uint64_t seed, double* out) {
    if (!cells || !side || !out || (dim != 2 && dim != 3)) return fail("luna_jittered_points: bad argument");
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> shift(-jitter, jitter);
    int64_t p = 0;
    const int nz = dim == 3 ? cells[2] : 1;
    for (int i = 0; i < cells[0]; ++i)
        for (int j = 0; j < cells[1]; ++j)
            for (int k = 0; k < nz; ++k) {
                const int index[3] = {i, j, k};
                for (int a = 0; a < dim; ++a) {
                    const double h = side[a] / cells[a];
                    out[dim * p + a] = std::fmod((index[a] + 0.5 + shift(rng)) * h + side[a], side[a]);
                }
                ++p;
            }
    return 0;
}

}  // extern "C"
