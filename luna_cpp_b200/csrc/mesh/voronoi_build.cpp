// Periodic Voronoi mesh builder: cells by half-space clipping, faces in voronoi-cpp's layout (see luna_mesh.h).
//
// Each cell starts as the periodic box centred on its generator (its own images bound it there) and is clipped by the
// bisector plane (2D: line) of every generator image that can still cut it. Candidates come from a bucket grid visited in
// order of a lower bound on their distance; the walk stops once that bound exceeds twice the largest vertex radius of the
// cell (no farther generator can cut it). Each face is then emitted once, by its owner, the lower-numbered of its two
// cells; faces are numbered by owner, then by neighbour, and every cell's list is ordered by neighbour.

#include "luna_mesh.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <type_traits>
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

using V3 = std::array<double, 3>;

inline double dot3(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3 cross3(const V3& a, const V3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline V3 sub3(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }

// One emitted face of a cell: the neighbour, area vector out of the cell, face centroid relative to the cell's generator.
struct CellFace {
    int32_t j;
    double a[3];
    double c[3];
};

// A convex polyhedron around the origin: vertices, and faces as CCW (seen from outside) vertex loops with a tag each.
struct Poly3 {
    std::vector<V3> v, nv;
    std::vector<int> idx, nidx;           // face loops, concatenated
    std::vector<int> fo, nfo;             // face offsets into idx (size faces + 1)
    std::vector<int64_t> tag, ntag;       // neighbour per face (-1: box)
    std::vector<double> s;                // signed distances of the vertices to the cutting plane
    std::vector<int> remap;               // old vertex -> new vertex (-1: removed)
    std::vector<std::pair<uint64_t, int>> edge_memo;  // intersection vertex per cut edge
    std::vector<int> cut;                 // vertices of the new face
    double eps = 0;

    void box(const double* half) {
        v.clear();
        for (int k = 0; k < 8; ++k)
            v.push_back({(k & 1) ? half[0] : -half[0], (k & 2) ? half[1] : -half[1], (k & 4) ? half[2] : -half[2]});
        // Faces CCW seen from outside (-x, +x, -y, +y, -z, +z).
        const int loops[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
        idx.clear();
        fo.assign(1, 0);
        tag.clear();
        for (auto& l : loops) {
            for (int k = 0; k < 4; ++k) idx.push_back(l[k]);
            fo.push_back(static_cast<int>(idx.size()));
            tag.push_back(-1);
        }
    }
    double max_radius2() const {
        double r = 0;
        for (const V3& p : v) r = std::max(r, dot3(p, p));
        return r;
    }
    int memo(int a, int b) {
        const uint64_t key = a < b ? (uint64_t(a) << 32 | uint32_t(b)) : (uint64_t(b) << 32 | uint32_t(a));
        for (const auto& e : edge_memo)
            if (e.first == key) return e.second;
        const double t = s[a] / (s[a] - s[b]);
        const V3& p = v[a];
        const V3& q = v[b];
        nv.push_back({p[0] + t * (q[0] - p[0]), p[1] + t * (q[1] - p[1]), p[2] + t * (q[2] - p[2])});
        const int id = static_cast<int>(nv.size()) - 1;
        edge_memo.push_back({key, id});
        cut.push_back(id);
        return id;
    }
    // Keeps {y : n.y <= c}; the new face gets tag t. Returns whether anything was cut.
    bool clip(const V3& n, double c, int64_t t) {
        const int nvert = static_cast<int>(v.size());
        s.resize(nvert);
        double smax = -1e300;
        for (int k = 0; k < nvert; ++k) {
            s[k] = dot3(n, v[k]) - c;
            smax = std::max(smax, s[k]);
        }
        if (smax <= eps) return false;
        remap.assign(nvert, -1);
        nv.clear();
        cut.clear();
        edge_memo.clear();
        for (int k = 0; k < nvert; ++k)
            if (s[k] <= eps) {
                remap[k] = static_cast<int>(nv.size());
                nv.push_back(v[k]);
                if (s[k] >= -eps) cut.push_back(remap[k]);
            }
        nidx.clear();
        nfo.assign(1, 0);
        ntag.clear();
        const int nf = static_cast<int>(tag.size());
        for (int f = 0; f < nf; ++f) {
            const int a0 = fo[f], m = fo[f + 1] - fo[f];
            const size_t begin = nidx.size();
            for (int k = 0; k < m; ++k) {
                const int a = idx[a0 + k], b = idx[a0 + (k + 1) % m];
                if (s[a] <= eps) nidx.push_back(remap[a]);
                if ((s[a] < -eps && s[b] > eps) || (s[a] > eps && s[b] < -eps)) nidx.push_back(memo(a, b));
            }
            if (nidx.size() - begin >= 3) {
                nfo.push_back(static_cast<int>(nidx.size()));
                ntag.push_back(tag[f]);
            } else {
                nidx.resize(begin);
            }
        }
        // The new face: the cut vertices sorted by angle around their mean, CCW about n (outward).
        std::sort(cut.begin(), cut.end());
        cut.erase(std::unique(cut.begin(), cut.end()), cut.end());
        if (cut.size() >= 3) {
            V3 mean{0, 0, 0};
            for (int id : cut)
                for (int a = 0; a < 3; ++a) mean[a] += nv[id][a];
            for (int a = 0; a < 3; ++a) mean[a] /= static_cast<double>(cut.size());
            V3 u = std::fabs(n[0]) < 0.6 ? V3{1, 0, 0} : V3{0, 1, 0};
            const double un = dot3(u, n);
            u = {u[0] - un * n[0], u[1] - un * n[1], u[2] - un * n[2]};
            const double ul = std::sqrt(dot3(u, u));
            u = {u[0] / ul, u[1] / ul, u[2] / ul};
            const V3 w = cross3(n, u);
            std::vector<std::pair<double, int>> order;
            order.reserve(cut.size());
            for (int id : cut) {
                const V3 d = sub3(nv[id], mean);
                order.push_back({std::atan2(dot3(d, w), dot3(d, u)), id});
            }
            std::sort(order.begin(), order.end());
            for (const auto& o : order) nidx.push_back(o.second);
            nfo.push_back(static_cast<int>(nidx.size()));
            ntag.push_back(t);
        }
        v.swap(nv);
        idx.swap(nidx);
        fo.swap(nfo);
        tag.swap(ntag);
        return true;
    }
};

// A convex polygon around the origin, CCW, with the tag of the edge leaving each vertex.
struct Poly2 {
    std::vector<std::array<double, 2>> v, nv;
    std::vector<int64_t> tag, ntag;
    double eps = 0;
    void box(const double* half) {
        v = {{-half[0], -half[1]}, {half[0], -half[1]}, {half[0], half[1]}, {-half[0], half[1]}};
        tag = {-1, -1, -1, -1};
    }
    double max_radius2() const {
        double r = 0;
        for (const auto& p : v) r = std::max(r, p[0] * p[0] + p[1] * p[1]);
        return r;
    }
    bool clip(const double* n, double c, int64_t t) {
        const int m = static_cast<int>(v.size());
        std::vector<double> s(m);
        double smax = -1e300;
        for (int k = 0; k < m; ++k) {
            s[k] = n[0] * v[k][0] + n[1] * v[k][1] - c;
            smax = std::max(smax, s[k]);
        }
        if (smax <= eps) return false;
        nv.clear();
        ntag.clear();
        for (int k = 0; k < m; ++k) {
            const int b = (k + 1) % m;
            const bool ain = s[k] <= eps, bin = s[b] <= eps;
            if (ain) {
                nv.push_back(v[k]);
                // The edge k -> b stays (tag[k]) if b is inside; if b is outside, the edge is cut and continues to the
                // exit point with tag[k].
                ntag.push_back(tag[k]);
                if (!bin && s[k] < -eps) {
                    const double u = s[k] / (s[k] - s[b]);
                    nv.push_back({v[k][0] + u * (v[b][0] - v[k][0]), v[k][1] + u * (v[b][1] - v[k][1])});
                    ntag.push_back(t);  // from the exit point along the cut
                } else if (!bin) {
                    ntag.back() = t;  // k sits on the line: the cut starts here
                }
            } else if (bin && s[b] < -eps) {
                const double u = s[k] / (s[k] - s[b]);
                nv.push_back({v[k][0] + u * (v[b][0] - v[k][0]), v[k][1] + u * (v[b][1] - v[k][1])});
                ntag.push_back(tag[k]);  // entry point, then along edge k to b
            }
        }
        v.swap(nv);
        tag.swap(ntag);
        return true;
    }
};

struct Grid {
    int dim;
    int nb[3];
    double w[3];
    std::vector<int64_t> start;   // bucket -> first item
    std::vector<int32_t> items;   // point ids by bucket
    std::vector<std::array<int, 3>> offsets;  // sorted by the lower bound of their distance
    std::vector<double> bound2;

    int bucket_of(const double* x, int a) const {
        int b = static_cast<int>(std::floor(x[a] / w[a]));
        return std::min(std::max(b, 0), nb[a] - 1);
    }
    void build(int d, int64_t n, const double* pts, const double* side) {
        dim = d;
        double vol = 1;
        for (int a = 0; a < d; ++a) vol *= side[a];
        const double spacing = std::pow(vol / static_cast<double>(n), 1.0 / d);
        int64_t total = 1;
        for (int a = 0; a < 3; ++a) {
            nb[a] = a < d ? std::max(1, static_cast<int>(std::floor(side[a] / spacing))) : 1;
            w[a] = a < d ? side[a] / nb[a] : 1.0;
            total *= nb[a];
        }
        std::vector<int64_t> count(total + 1, 0);
        std::vector<int64_t> of(n);
        for (int64_t i = 0; i < n; ++i) {
            int64_t b = 0;
            for (int a = 0; a < d; ++a) b = b * nb[a] + bucket_of(pts + d * i, a);
            of[i] = b;
            ++count[b + 1];
        }
        for (int64_t b = 0; b < total; ++b) count[b + 1] += count[b];
        start = count;
        items.resize(n);
        std::vector<int64_t> fill(count.begin(), count.end() - 1);
        for (int64_t i = 0; i < n; ++i) items[fill[of[i]]++] = static_cast<int32_t>(i);
        const int K = 8;
        offsets.clear();
        for (int x = -K; x <= K; ++x)
            for (int y = (d >= 2 ? -K : 0); y <= (d >= 2 ? K : 0); ++y)
                for (int z = (d >= 3 ? -K : 0); z <= (d >= 3 ? K : 0); ++z) offsets.push_back({x, y, z});
        auto lower = [&](const std::array<int, 3>& o) {
            double s = 0;
            for (int a = 0; a < d; ++a) {
                const double g = std::max(0, std::abs(o[a]) - 1) * w[a];
                s += g * g;
            }
            return s;
        };
        std::stable_sort(offsets.begin(), offsets.end(), [&](const auto& p, const auto& q) { return lower(p) < lower(q); });
        bound2.resize(offsets.size());
        for (size_t k = 0; k < offsets.size(); ++k) bound2[k] = lower(offsets[k]);
    }
};

}  // namespace

struct luna_mesh_build {
    int dim = 3;
    int64_t n = 0, f = 0, inconsistent = 0;
    double box[3] = {1, 1, 1};
    std::vector<int32_t> owner, neighbour, start, list;
    std::vector<double> area, face_centroid, centroid, volume, positions;
};

namespace {

// Cell i: clipped, then its faces (sorted by neighbour), volume and centroid. Returns false with a message on error.
template <class Poly>
bool cell(int dim, int64_t i, const double* pos, const double* side, const Grid& grid, Poly& poly, std::vector<CellFace>& faces,
          double& volume, double* centroid, std::string& err) {
    const double* xi = pos + dim * i;
    double half[3];
    double scale = 0;
    for (int a = 0; a < dim; ++a) {
        half[a] = 0.5 * side[a];
        scale = std::max(scale, side[a]);
    }
    poly.box(half);
    poly.eps = 1e-13 * scale;
    int bi[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) bi[a] = grid.bucket_of(xi, a);
    double rmax2 = poly.max_radius2();
    bool done = false;
    for (size_t k = 0; k < grid.offsets.size(); ++k) {
        if (grid.bound2[k] > 4.0 * rmax2) {
            done = true;
            break;
        }
        const auto& o = grid.offsets[k];
        int64_t b = 0;
        double shift[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) {
            const int t = bi[a] + o[a];
            const int tw = ((t % grid.nb[a]) + grid.nb[a]) % grid.nb[a];
            shift[a] = static_cast<double>((t - tw) / grid.nb[a]) * side[a];
            b = b * grid.nb[a] + tw;
        }
        for (int64_t q = grid.start[b]; q < grid.start[b + 1]; ++q) {
            const int32_t j = grid.items[q];
            double d[3] = {0, 0, 0};
            double d2 = 0;
            for (int a = 0; a < dim; ++a) {
                d[a] = pos[dim * j + a] + shift[a] - xi[a];
                d2 += d[a] * d[a];
            }
            if (d2 == 0) continue;  // the generator itself
            if (d2 > 4.0 * rmax2) continue;
            const double inv = 1.0 / std::sqrt(d2);
            if constexpr (std::is_same_v<Poly, Poly3>) {
                const V3 n{d[0] * inv, d[1] * inv, d[2] * inv};
                if (poly.clip(n, 0.5 * d2 * inv, j)) rmax2 = poly.max_radius2();
            } else {
                const double n[2] = {d[0] * inv, d[1] * inv};
                if (poly.clip(n, 0.5 * d2 * inv, j)) rmax2 = poly.max_radius2();
            }
        }
    }
    if (!done) {
        err = "voronoi: the bucket search ran out of offsets (points too sparse for the grid)";
        return false;
    }
    faces.clear();
    volume = 0;
    double cm[3] = {0, 0, 0};
    if constexpr (std::is_same_v<Poly, Poly3>) {
        const int nf = static_cast<int>(poly.tag.size());
        for (int f = 0; f < nf; ++f) {
            const int a0 = poly.fo[f], m = poly.fo[f + 1] - a0;
            const V3& p0 = poly.v[poly.idx[a0]];
            V3 A{0, 0, 0};
            V3 C{0, 0, 0};
            double wsum = 0;
            std::vector<std::pair<V3, V3>> tris;
            for (int k = 1; k + 1 < m; ++k) {
                const V3& p1 = poly.v[poly.idx[a0 + k]];
                const V3& p2 = poly.v[poly.idx[a0 + k + 1]];
                const V3 t = cross3(sub3(p1, p0), sub3(p2, p0));
                for (int a = 0; a < 3; ++a) A[a] += 0.5 * t[a];
                // Tetrahedron (origin, p0, p1, p2): 6 V = p0 . (p1 x p2).
                const double v6 = dot3(p0, cross3(p1, p2));
                volume += v6 / 6.0;
                for (int a = 0; a < 3; ++a) cm[a] += v6 / 6.0 * (p0[a] + p1[a] + p2[a]) / 4.0;
                tris.push_back({t, {(p0[0] + p1[0] + p2[0]) / 3.0, (p0[1] + p1[1] + p2[1]) / 3.0, (p0[2] + p1[2] + p2[2]) / 3.0}});
            }
            const double amag = std::sqrt(dot3(A, A));
            if (poly.tag[f] < 0) {
                err = "voronoi: a cell reaches the box (box too small for the points)";
                return false;
            }
            if (poly.tag[f] == i) {
                err = "voronoi: a cell touches its own periodic image (box too small for the points)";
                return false;
            }
            for (const auto& tr : tris) {
                const double wgt = amag > 0 ? dot3(tr.first, A) / amag : 0.0;
                for (int a = 0; a < 3; ++a) C[a] += wgt * tr.second[a];
                wsum += wgt;
            }
            if (wsum > 0)
                for (int a = 0; a < 3; ++a) C[a] /= wsum;
            else
                C = p0;
            CellFace cf;
            cf.j = static_cast<int32_t>(poly.tag[f]);
            for (int a = 0; a < 3; ++a) {
                cf.a[a] = A[a];
                cf.c[a] = C[a];
            }
            faces.push_back(cf);
        }
    } else {
        const int m = static_cast<int>(poly.v.size());
        for (int k = 0; k < m; ++k) {
            const auto& p = poly.v[k];
            const auto& q = poly.v[(k + 1) % m];
            const double cr = p[0] * q[1] - p[1] * q[0];
            volume += 0.5 * cr;
            cm[0] += cr * (p[0] + q[0]) / 6.0;
            cm[1] += cr * (p[1] + q[1]) / 6.0;
            if (poly.tag[k] < 0) {
                err = "voronoi: a cell reaches the box (box too small for the points)";
                return false;
            }
            if (poly.tag[k] == i) {
                err = "voronoi: a cell touches its own periodic image (box too small for the points)";
                return false;
            }
            CellFace cf{};
            cf.j = static_cast<int32_t>(poly.tag[k]);
            cf.a[0] = q[1] - p[1];
            cf.a[1] = -(q[0] - p[0]);
            cf.c[0] = 0.5 * (p[0] + q[0]);
            cf.c[1] = 0.5 * (p[1] + q[1]);
            faces.push_back(cf);
        }
    }
    for (int a = 0; a < dim; ++a) centroid[a] = cm[a] / volume;
    std::sort(faces.begin(), faces.end(), [](const CellFace& p, const CellFace& q) { return p.j < q.j; });
    for (size_t k = 1; k < faces.size(); ++k)
        if (faces[k].j == faces[k - 1].j) {
            err = "voronoi: two faces between the same pair of cells (box too small for unique nearest images)";
            return false;
        }
    return true;
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
            x -= box[a] * std::floor(x / box[a]);
            if (x >= box[a]) x -= box[a];
            m->positions[dim * i + a] = x;
        }
    Grid grid;
    grid.build(dim, n, m->positions.data(), box);
    m->volume.resize(n);
    m->centroid.resize(static_cast<size_t>(n) * dim);
    std::vector<int64_t> count(n + 1, 0);
    // Per cell faces, kept per thread chunk and gathered after.
    std::vector<std::vector<CellFace>> per_cell(n);
    std::string first_error;
    bool ok = true;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel
    {
        Poly3 p3;
        Poly2 p2;
        std::vector<CellFace> faces;
        std::string err;
#pragma omp for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            if (!ok) continue;
            double vol = 0;
            bool good = dim == 3 ? cell(dim, i, m->positions.data(), box, grid, p3, faces, vol, &m->centroid[dim * i], err)
                                 : cell(dim, i, m->positions.data(), box, grid, p2, faces, vol, &m->centroid[dim * i], err);
            if (!good) {
#pragma omp critical
                {
                    if (ok) first_error = err;
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
