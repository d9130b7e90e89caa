// One periodic Voronoi cell by half-space clipping, in fixed-capacity storage, for the host builder
// (voronoi_build.cpp) and the device remesher (remesh.cu) alike. Both compile this one source without floating-point
// contraction (-ffp-contract=off on the host, -fmad=false on the device) and use only correctly rounded operations
// (+ - * /, sqrt, floor, nearbyint), so a mesh built on the device has the host builder's bits.
//
// A cell starts as the periodic box centred on its generator (its own images bound it there) and is clipped by the
// bisector plane (2D: line) of every generator image that can still cut it. Candidates come from a bucket grid visited
// in order of a lower bound on their distance; the walk stops once that bound exceeds twice the largest vertex radius of
// the cell (no farther generator can cut it).
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define LUNA_VC_HD __host__ __device__ __forceinline__
#else
#define LUNA_VC_HD inline
#endif

namespace luna_voronoi {

// The storage of a cell is fixed at compile time (the template arguments below): the device remesher's is sized for the
// cells of gas meshes (a thread's local memory), the host builder's for cells of up to a thousand faces; a cell that
// outgrows its storage is an error, never a different result.

// Why a cell could not be built (0: it was).
enum : int {
    kCellOk = 0,
    kOutOfOffsets = 1,   // the search reached its limit (the grid's offsets; with Far, a box side)
    kReachesBox = 2,     // a face of the starting box survived: the box is too small for the points
    kTouchesSelf = 3,    // a face towards the cell's own image
    kDuplicatePair = 4,  // two faces towards the same cell (no unique nearest images)
    kCapacity = 5,       // more vertices, faces or loop entries than the storage holds
    kCandidates = 6,     // more generator images at one distance than the candidate storage holds
};

// The bucket grid: nb buckets of width w per axis, items by bucket (CSR), and the bucket offsets to visit, sorted by a
// lower bound bound2 on the squared distance of any point in the offset bucket.
struct Grid {
    int dim;
    int nb[3];
    double w[3];
    const int64_t* start;
    const int32_t* items;
    const int32_t* offsets;  // [n_offsets][3]
    const double* bound2;    // [n_offsets]
    int n_offsets;
    int reach;               // the offsets cover -reach .. reach buckets per axis
};

LUNA_VC_HD int bucket_of(const Grid& g, const double* x, int a) {
    const int b = static_cast<int>(floor(x[a] / g.w[a]));
    return b < 0 ? 0 : (b > g.nb[a] - 1 ? g.nb[a] - 1 : b);
}

LUNA_VC_HD double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
LUNA_VC_HD void cross3(const double* a, const double* b, double* out) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

// A monotone stand-in for the polar angle of (x, y) in [0, 4): the position along the unit diamond |x| + |y| = 1,
// counter-clockwise from +x. One division, so the host and the device order a face's vertices alike.
LUNA_VC_HD double diamond_angle(double x, double y) {
    if (x == 0 && y == 0) return 0;
    if (y >= 0) return x >= 0 ? y / (x + y) : 1 - x / (y - x);
    return x < 0 ? 2 + y / (x + y) : 3 + x / (x - y);
}

// A convex polyhedron around the origin: vertices, and faces as counter-clockwise (seen from outside) vertex loops, each
// with the neighbour across it (-1: the starting box). Two copies, the current one and the one a clip builds. Room for
// kMaxVerts vertices, kMaxFaces faces, kMaxLoop loop entries and kMaxCut vertices of one new face.
template <int kMaxVerts, int kMaxFaces, int kMaxLoop, int kMaxCut>
struct Poly3T {
    double v[2][kMaxVerts][3];
    int idx[2][kMaxLoop];
    int fo[2][kMaxFaces + 1];  // face offsets into idx
    int32_t tag[2][kMaxFaces];
    int nv[2], nf[2];
    int cur;
    double s[kMaxVerts];  // signed distances of the vertices to the cutting plane
    int remap[kMaxVerts];  // old vertex -> new vertex (-1: removed)
    uint64_t memo_key[kMaxCut];  // the intersection vertex of each cut edge
    int memo_id[kMaxCut];
    int nmemo;
    int cut[kMaxCut];  // vertices of the new face
    double angle[kMaxCut];
    int ncut;
    double eps;
    bool full;  // a capacity ran out

    LUNA_VC_HD void box(const double* half) {
        cur = 0;
        full = false;
        nv[0] = 8;
        for (int k = 0; k < 8; ++k) {
            v[0][k][0] = (k & 1) ? half[0] : -half[0];
            v[0][k][1] = (k & 2) ? half[1] : -half[1];
            v[0][k][2] = (k & 4) ? half[2] : -half[2];
        }
        // faces counter-clockwise seen from outside: -x, +x, -y, +y, -z, +z
        const int loops[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
        nf[0] = 6;
        fo[0][0] = 0;
        for (int f = 0; f < 6; ++f) {
            for (int k = 0; k < 4; ++k) idx[0][4 * f + k] = loops[f][k];
            fo[0][f + 1] = 4 * f + 4;
            tag[0][f] = -1;
        }
    }
    LUNA_VC_HD double max_radius2() const {
        double r = 0;
        for (int k = 0; k < nv[cur]; ++k) {
            const double d = dot3(v[cur][k], v[cur][k]);
            r = d > r ? d : r;
        }
        return r;
    }
    // The new vertex on the edge a-b (each cut edge once).
    LUNA_VC_HD int memo(int a, int b) {
        const uint64_t key = a < b ? (uint64_t(a) << 32 | uint32_t(b)) : (uint64_t(b) << 32 | uint32_t(a));
        for (int k = 0; k < nmemo; ++k)
            if (memo_key[k] == key) return memo_id[k];
        const int o = cur, n = cur ^ 1;
        if (nv[n] >= kMaxVerts || nmemo >= kMaxCut || ncut >= kMaxCut) {
            full = true;
            return 0;
        }
        const double t = s[a] / (s[a] - s[b]);
        const double* p = v[o][a];
        const double* q = v[o][b];
        const int id = nv[n]++;
        v[n][id][0] = p[0] + t * (q[0] - p[0]);
        v[n][id][1] = p[1] + t * (q[1] - p[1]);
        v[n][id][2] = p[2] + t * (q[2] - p[2]);
        memo_key[nmemo] = key;
        memo_id[nmemo++] = id;
        cut[ncut++] = id;
        return id;
    }
    // Keeps {y : n.y <= c}; the new face gets tag t. Returns whether anything was cut.
    LUNA_VC_HD bool clip(const double* nrm, double c, int32_t t) {
        const int o = cur, n = cur ^ 1;
        const int nvert = nv[o];
        double smax = -1e300;
        for (int k = 0; k < nvert; ++k) {
            s[k] = dot3(nrm, v[o][k]) - c;
            smax = s[k] > smax ? s[k] : smax;
        }
        if (smax <= eps) return false;
        nv[n] = 0;
        nmemo = 0;
        ncut = 0;
        for (int k = 0; k < nvert; ++k) {
            remap[k] = -1;
            if (s[k] <= eps) {
                remap[k] = nv[n];
                v[n][nv[n]][0] = v[o][k][0];
                v[n][nv[n]][1] = v[o][k][1];
                v[n][nv[n]][2] = v[o][k][2];
                if (s[k] >= -eps) {
                    if (ncut >= kMaxCut) {
                        full = true;
                        return false;
                    }
                    cut[ncut++] = nv[n];
                }
                ++nv[n];
            }
        }
        int li = 0, fi = 0;
        fo[n][0] = 0;
        for (int f = 0; f < nf[o]; ++f) {
            const int a0 = fo[o][f], m = fo[o][f + 1] - fo[o][f];
            const int begin = li;
            for (int k = 0; k < m; ++k) {
                const int a = idx[o][a0 + k], b = idx[o][a0 + (k + 1) % m];
                if (li + 2 > kMaxLoop) {
                    full = true;
                    return false;
                }
                if (s[a] <= eps) idx[n][li++] = remap[a];
                if ((s[a] < -eps && s[b] > eps) || (s[a] > eps && s[b] < -eps)) {
                    const int id = memo(a, b);
                    if (full) return false;
                    idx[n][li++] = id;
                }
            }
            if (li - begin >= 3) {
                if (fi >= kMaxFaces) {
                    full = true;
                    return false;
                }
                tag[n][fi] = tag[o][f];
                fo[n][++fi] = li;
            } else {
                li = begin;
            }
        }
        // The new face: the cut vertices (sorted, once each) ordered counter-clockwise about nrm (outward) around their
        // mean, by diamond angle, then by vertex.
        for (int k = 1; k < ncut; ++k) {
            const int x = cut[k];
            int j = k - 1;
            while (j >= 0 && cut[j] > x) {
                cut[j + 1] = cut[j];
                --j;
            }
            cut[j + 1] = x;
        }
        int unique = 0;
        for (int k = 0; k < ncut; ++k)
            if (unique == 0 || cut[unique - 1] != cut[k]) cut[unique++] = cut[k];
        ncut = unique;
        if (ncut >= 3) {
            double mean[3] = {0, 0, 0};
            for (int k = 0; k < ncut; ++k)
                for (int a = 0; a < 3; ++a) mean[a] += v[n][cut[k]][a];
            for (int a = 0; a < 3; ++a) mean[a] /= static_cast<double>(ncut);
            double u[3] = {0, 0, 0};
            u[fabs(nrm[0]) < 0.6 ? 0 : 1] = 1;
            const double un = dot3(u, nrm);
            for (int a = 0; a < 3; ++a) u[a] = u[a] - un * nrm[a];
            const double ul = sqrt(dot3(u, u));
            for (int a = 0; a < 3; ++a) u[a] = u[a] / ul;
            double w[3];
            cross3(nrm, u, w);
            for (int k = 0; k < ncut; ++k) {
                const double* p = v[n][cut[k]];
                const double d[3] = {p[0] - mean[0], p[1] - mean[1], p[2] - mean[2]};
                angle[k] = diamond_angle(dot3(d, u), dot3(d, w));
            }
            for (int k = 1; k < ncut; ++k) {  // by angle, then by vertex (cut is sorted by vertex: a stable sort)
                const int x = cut[k];
                const double ax = angle[k];
                int j = k - 1;
                while (j >= 0 && angle[j] > ax) {
                    cut[j + 1] = cut[j];
                    angle[j + 1] = angle[j];
                    --j;
                }
                cut[j + 1] = x;
                angle[j + 1] = ax;
            }
            if (fi >= kMaxFaces || li + ncut > kMaxLoop) {
                full = true;
                return false;
            }
            for (int k = 0; k < ncut; ++k) idx[n][li++] = cut[k];
            tag[n][fi] = t;
            fo[n][++fi] = li;
        }
        nf[n] = fi;
        cur = n;
        return true;
    }
};

// A convex polygon around the origin, counter-clockwise, with the neighbour across the edge leaving each vertex; room
// for kMaxFaces vertices.
template <int kMaxFaces>
struct Poly2T {
    double v[2][kMaxFaces][2];
    int32_t tag[2][kMaxFaces];
    int nv[2];
    int cur;
    double s[kMaxFaces];
    double eps;
    bool full;

    LUNA_VC_HD void box(const double* half) {
        cur = 0;
        full = false;
        nv[0] = 4;
        const double x[4] = {-half[0], half[0], half[0], -half[0]}, y[4] = {-half[1], -half[1], half[1], half[1]};
        for (int k = 0; k < 4; ++k) {
            v[0][k][0] = x[k];
            v[0][k][1] = y[k];
            tag[0][k] = -1;
        }
    }
    LUNA_VC_HD double max_radius2() const {
        double r = 0;
        for (int k = 0; k < nv[cur]; ++k) {
            const double d = v[cur][k][0] * v[cur][k][0] + v[cur][k][1] * v[cur][k][1];
            r = d > r ? d : r;
        }
        return r;
    }
    LUNA_VC_HD bool clip(const double* nrm, double c, int32_t t) {
        const int o = cur, n = cur ^ 1;
        const int m = nv[o];
        double smax = -1e300;
        for (int k = 0; k < m; ++k) {
            s[k] = nrm[0] * v[o][k][0] + nrm[1] * v[o][k][1] - c;
            smax = s[k] > smax ? s[k] : smax;
        }
        if (smax <= eps) return false;
        int q = 0;
        for (int k = 0; k < m; ++k) {
            const int b = (k + 1) % m;
            const bool ain = s[k] <= eps, bin = s[b] <= eps;
            if (q + 2 > kMaxFaces) {
                full = true;
                return false;
            }
            if (ain) {
                v[n][q][0] = v[o][k][0];
                v[n][q][1] = v[o][k][1];
                // The edge k -> b stays (tag k) if b is inside; if b is outside the edge is cut, and continues to the
                // exit point with tag k.
                tag[n][q++] = tag[o][k];
                if (!bin && s[k] < -eps) {
                    const double u = s[k] / (s[k] - s[b]);
                    v[n][q][0] = v[o][k][0] + u * (v[o][b][0] - v[o][k][0]);
                    v[n][q][1] = v[o][k][1] + u * (v[o][b][1] - v[o][k][1]);
                    tag[n][q++] = t;  // from the exit point along the cut
                } else if (!bin) {
                    tag[n][q - 1] = t;  // k sits on the line: the cut starts here
                }
            } else if (bin && s[b] < -eps) {
                const double u = s[k] / (s[k] - s[b]);
                v[n][q][0] = v[o][k][0] + u * (v[o][b][0] - v[o][k][0]);
                v[n][q][1] = v[o][k][1] + u * (v[o][b][1] - v[o][k][1]);
                tag[n][q++] = tag[o][k];  // entry point, then along edge k to b
            }
        }
        nv[n] = q;
        cur = n;
        return true;
    }
};

// The faces of one built cell, by neighbour: area vector out of the cell, centroid relative to the cell's generator.
template <int kMaxFaces>
struct CellFacesT {
    int32_t j[kMaxFaces];
    double a[kMaxFaces][3];
    double c[kMaxFaces][3];
    int order[kMaxFaces];  // faces by neighbour
    int n;
};

// The generator images a cell is clipped by, one batch at a time: the image's periodic wraps, squared distance,
// index; in clipping order. The clip recomputes an image's offset from its generator, its wraps and the cell's generator
// in the gather's own operations, so the offset is the gathered one bit for bit, and the store keeps 4 bytes an image
// instead of 24.
template <int kMax>
struct CandidatesT {
    uint32_t w[kMax];  // the image's wraps per axis, each + 128 in a byte
    double d2[kMax];
    int32_t j[kMax];
    int order[kMax];
    double key[kMax];  // d2 in clipping order
    int n;
};

// Whether the bucket at offset o from the cell's bucket bi can hold an image with lo2 < d2 <= hi2 from the cell's
// generator xi: the distance from xi to the bucket's box, per axis, against hi2, and to its far corner against lo2. A
// point in bucket b lies within [b w, (b + 1) w) up to the rounding of floor(x / w) and of b w, which the margin of a
// millionth of a bucket covers, so a bucket it skips holds no image of the shell and the batch is the same without it.
template <int D>
LUNA_VC_HD bool bucket_reaches(const double* xi, const int* bi, const int32_t* o, const Grid& grid, double lo2, double hi2) {
    double near2 = 0, far2 = 0;
    for (int a = 0; a < D; ++a) {
        const double w = grid.w[a], m = 1e-6 * w;
        const double lo = static_cast<double>(bi[a] + o[a]) * w - xi[a];  // the bucket's low face from xi
        const double hi = lo + w;
        double near = 0;
        if (lo > 0)
            near = lo - m;
        else if (hi < 0)
            near = -hi - m;
        near = near > 0 ? near : 0;
        const double far = (-lo > hi ? -lo : hi) + m;
        near2 += near * near;
        far2 += far * far;
    }
    return near2 <= hi2 && far2 > lo2;
}

// Appends to the batch the images in the bucket at offset o from the cell's bucket bi with lo2 < d2 <= hi2 from its
// generator xi (nothing from a bucket that cannot hold one). Returns false when the batch outgrows the storage.
template <int D, class Cand>
LUNA_VC_HD bool gather_bucket(const double* xi, const int* bi, const int32_t* o, const double* pos, const double* side, const Grid& grid,
                              double lo2, double hi2, Cand& cand) {
    constexpr int kMax = sizeof(cand.j) / sizeof(cand.j[0]);
    if (!bucket_reaches<D>(xi, bi, o, grid, lo2, hi2)) return true;
    int64_t b = 0;
    uint32_t packed = 0;
    double shift[3] = {0, 0, 0};
    for (int a = 0; a < D; ++a) {
        int t = bi[a] + o[a], wraps = 0;  // t = wraps nb + tw with 0 <= tw < nb, without an integer division
        while (t < 0) {
            t += grid.nb[a];
            --wraps;
        }
        while (t >= grid.nb[a]) {
            t -= grid.nb[a];
            ++wraps;
        }
        shift[a] = static_cast<double>(wraps) * side[a];
        packed |= static_cast<uint32_t>(wraps + 128) << (8 * a);
        b = b * grid.nb[a] + t;
    }
    for (int64_t q = grid.start[b]; q < grid.start[b + 1]; ++q) {
        const int32_t j = grid.items[q];
        double d[3] = {0, 0, 0};
        double d2 = 0;
        for (int a = 0; a < D; ++a) {
            d[a] = pos[D * j + a] + shift[a] - xi[a];
            d2 += d[a] * d[a];
        }
        if (!(d2 > lo2 && d2 <= hi2)) continue;
        if (cand.n >= kMax) return false;
        const int e = cand.n++;
        cand.w[e] = packed;
        cand.d2[e] = d2;
        cand.j[e] = j;
    }
    return true;
}

// The far search of a cell much larger than the mean spacing (the evacuated middle of a blast on a moving mesh): every
// offset of the cube that can hold an image within hi2, by the grid's lower bound of its distance.
template <int D, class Cand>
LUNA_VC_HD bool gather_cube(const double* xi, const int* bi, const double* pos, const double* side, const Grid& grid, double lo2,
                            double hi2, Cand& cand) {
    int R[3] = {0, 0, 0};
    for (int a = 0; a < D; ++a) R[a] = static_cast<int>(floor(sqrt(hi2) / grid.w[a])) + 1;
    int32_t o[3] = {0, 0, 0};
    for (o[0] = -R[0]; o[0] <= R[0]; ++o[0])
        for (o[1] = -R[1]; o[1] <= R[1]; ++o[1])
            for (o[2] = -R[2]; o[2] <= R[2]; ++o[2]) {
                double lower = 0;
                for (int a = 0; a < D; ++a) {
                    const int gap = (o[a] < 0 ? -o[a] : o[a]) - 1;
                    const double g = (gap > 0 ? gap : 0) * grid.w[a];
                    lower += g * g;
                }
                if (lower > hi2) continue;
                if (!gather_bucket<D>(xi, bi, o, pos, side, grid, lo2, hi2, cand)) return false;
            }
    return true;
}

// Gathers the images of generators with lo2 < d2 <= hi2 from the cell's generator xi (every bucket whose lower bound is
// at most hi2: through the grid's sorted offsets while they reach, table2, else over the cube of offsets), then orders
// the batch by (d2, index). Returns false when the batch outgrows the storage.
template <int D, bool Far, class Cand>
LUNA_VC_HD bool gather(const double* xi, const int* bi, const double* pos, const double* side, const Grid& grid, double lo2, double hi2,
                       double table2, Cand& cand) {
    cand.n = 0;
    if (!Far || hi2 <= table2) {
        for (int k = 0; k < grid.n_offsets && grid.bound2[k] <= hi2; ++k)
            if (!gather_bucket<D>(xi, bi, grid.offsets + 3 * k, pos, side, grid, lo2, hi2, cand)) return false;
    } else if (!gather_cube<D>(xi, bi, pos, side, grid, lo2, hi2, cand)) {
        return false;
    }
    for (int k = 0; k < cand.n; ++k) {  // insertion sort by (d2, j), stable; the sorted d2 kept beside the order
        const double dk = cand.d2[k];
        const int32_t jk = cand.j[k];
        int m = k - 1;
        while (m >= 0 && (cand.key[m] > dk || (cand.key[m] == dk && cand.j[cand.order[m]] > jk))) {
            cand.key[m + 1] = cand.key[m];
            cand.order[m + 1] = cand.order[m];
            --m;
        }
        cand.key[m + 1] = dk;
        cand.order[m + 1] = k;
    }
    return true;
}

// The faces of a built 3D cell (vertex loops idx with offsets fo and neighbours tag): area vector, centroid relative to
// the generator, into out; the cell's volume and first moment summed into volume and cm (tetrahedra from the
// generator, face by face, each fanned from its first vertex). Returns kCellOk, or why the cell is not a gas cell.
template <class Faces>
LUNA_VC_HD int cell_faces3(int64_t i, const double (*v)[3], const int* idx, const int* fo, const int32_t* tag, int nf, Faces& out,
                           double& volume, double* cm) {
    for (int f = 0; f < nf; ++f) {
        const int a0 = fo[f], m = fo[f + 1] - a0;
        if (tag[f] < 0) return kReachesBox;
        if (tag[f] == i) return kTouchesSelf;
        const double* p0 = v[idx[a0]];
        double A[3] = {0, 0, 0};
        for (int k = 1; k + 1 < m; ++k) {
            const double* p1 = v[idx[a0 + k]];
            const double* p2 = v[idx[a0 + k + 1]];
            const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
            const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
            double t[3], x12[3];
            cross3(e1, e2, t);
            for (int a = 0; a < 3; ++a) A[a] += 0.5 * t[a];
            // tetrahedron (origin, p0, p1, p2): 6 V = p0 . (p1 x p2)
            cross3(p1, p2, x12);
            const double v6 = dot3(p0, x12);
            volume += v6 / 6.0;
            for (int a = 0; a < 3; ++a) cm[a] += v6 / 6.0 * (p0[a] + p1[a] + p2[a]) / 4.0;
        }
        // the face centroid: its triangles' centroids weighted by their areas along the face normal
        const double amag = sqrt(dot3(A, A));
        double C[3] = {0, 0, 0};
        double wsum = 0;
        for (int k = 1; k + 1 < m; ++k) {
            const double* p1 = v[idx[a0 + k]];
            const double* p2 = v[idx[a0 + k + 1]];
            const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
            const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
            double t[3];
            cross3(e1, e2, t);
            const double wgt = amag > 0 ? dot3(t, A) / amag : 0.0;
            for (int a = 0; a < 3; ++a) C[a] += wgt * ((p0[a] + p1[a] + p2[a]) / 3.0);
            wsum += wgt;
        }
        if (wsum > 0)
            for (int a = 0; a < 3; ++a) C[a] /= wsum;
        else
            for (int a = 0; a < 3; ++a) C[a] = p0[a];
        const int e = out.n++;
        out.j[e] = tag[f];
        for (int a = 0; a < 3; ++a) {
            out.a[e][a] = A[a];
            out.c[e][a] = C[a];
        }
    }
    return kCellOk;
}

// out.order: the faces by neighbour (insertion sort). Returns kDuplicatePair if two faces share a neighbour.
template <class Faces>
LUNA_VC_HD int order_faces(Faces& out) {
    for (int k = 0; k < out.n; ++k) {
        const int x = k;
        int j = k - 1;
        while (j >= 0 && out.j[out.order[j]] > out.j[x]) {
            out.order[j + 1] = out.order[j];
            --j;
        }
        out.order[j + 1] = x;
    }
    for (int k = 1; k < out.n; ++k)
        if (out.j[out.order[k]] == out.j[out.order[k - 1]]) return kDuplicatePair;
    return kCellOk;
}

// Cell i of the points pos [n][dim] (wrapped into [0, side)): clipped, then its faces (out.order by neighbour), volume
// and centroid relative to the generator. Returns kCellOk or why the cell could not be built.
//
// The cell is clipped by the generator images nearest first, in (distance, index) order, and is complete at the first
// image farther than twice its largest vertex radius: the images are gathered in batches, all of those within a radius
// at a time (first 2.1 bucket widths; then, while the cell still reaches past a batch, out to twice its reach, 1.5
// times the batch's radius or the search's limit, whichever is nearest; with Far, a batch too large for the candidate
// storage is gathered again as a thinner shell). The order, and so the cell, does not depend on where the batches
// end. Nearest first, a cell is cut about as often as it has faces. Without Far the search ends at the grid's sorted
// offsets (kOutOfOffsets) and at a full candidate store (kCandidates): the common cell's fast path, the cells it
// refuses built again with Far, which searches out to a box side and thins its batches.
template <int D, bool Far = true, class Poly, class Faces, class Cand>
LUNA_VC_HD int build_cell(int64_t i, const double* pos, const double* side, const Grid& grid, Poly& poly, Faces& out, Cand& cand,
                          double& volume, double* centroid) {
    const double* xi = pos + D * i;
    double half[3] = {0, 0, 0};
    double scale = 0, wmax = 0, wmin = 1e300;
    for (int a = 0; a < D; ++a) {
        half[a] = 0.5 * side[a];
        scale = side[a] > scale ? side[a] : scale;
        wmax = grid.w[a] > wmax ? grid.w[a] : wmax;
        wmin = grid.w[a] < wmin ? grid.w[a] : wmin;
    }
    poly.box(half);
    poly.eps = 1e-13 * scale;
    int bi[3] = {0, 0, 0};
    for (int a = 0; a < D; ++a) bi[a] = bucket_of(grid, xi, a);
    double rmax2 = poly.max_radius2();
    // the grid's offsets reach every bucket whose lower bound is below (K - 1)^2 w_min^2 (K: their reach per axis); the
    // far search stops at a box side from the generator
    const double reach = static_cast<double>(grid.reach - 1) * wmin;
    const double table2 = reach * reach;
    double far2 = 0;
    for (int a = 0; a < D; ++a) far2 = side[a] * side[a] > far2 ? side[a] * side[a] : far2;
    const double limit2 = Far ? far2 : table2;
    double lo2 = 0, hi2 = 4.41 * wmax * wmax;  // (d2 = 0: the generator itself)
    hi2 = hi2 < limit2 ? hi2 : limit2;
    for (;;) {
        if (!gather<D, Far>(xi, bi, pos, side, grid, lo2, hi2, table2, cand)) {  // too many for the storage
            if (!Far) return kCandidates;
            const double thinner = lo2 + 0.25 * (hi2 - lo2);
            if (!(thinner > lo2 && thinner < hi2)) return kCandidates;
            hi2 = thinner;
            continue;
        }
        bool done = false;
        for (int k = 0; k < cand.n; ++k) {
            const int e = cand.order[k];
            const double d2 = cand.key[k];
            if (d2 > 4.0 * rmax2) {
                done = true;
                break;
            }
            const double inv = 1.0 / sqrt(d2);
            double dv[3] = {0, 0, 0};
            const int32_t je = cand.j[e];
            for (int a = 0; a < D; ++a)
                dv[a] = pos[D * je + a] + static_cast<double>(static_cast<int>((cand.w[e] >> (8 * a)) & 0xff) - 128) * side[a] - xi[a];
            const double nrm[3] = {dv[0] * inv, dv[1] * inv, dv[2] * inv};
            if (poly.clip(nrm, 0.5 * d2 * inv, cand.j[e])) rmax2 = poly.max_radius2();
            if (poly.full) return kCapacity;
        }
        if (done || 4.0 * rmax2 <= hi2) break;  // every image within twice the reach has been clipped by
        if (hi2 >= limit2) return kOutOfOffsets;
        lo2 = hi2;
        hi2 = 4.0 * rmax2 < 2.25 * hi2 ? 4.0 * rmax2 : 2.25 * hi2;
        hi2 = hi2 < limit2 ? hi2 : limit2;
    }
    out.n = 0;
    volume = 0;
    double cm[3] = {0, 0, 0};
    if constexpr (D == 3) {
        const int c = poly.cur;
        const int code = cell_faces3(i, poly.v[c], poly.idx[c], poly.fo[c], poly.tag[c], poly.nf[c], out, volume, cm);
        if (code != kCellOk) return code;
    } else {
        const int c = poly.cur, m = poly.nv[c];
        for (int k = 0; k < m; ++k) {
            const double* p = poly.v[c][k];
            const double* q = poly.v[c][(k + 1) % m];
            const double cr = p[0] * q[1] - p[1] * q[0];
            volume += 0.5 * cr;
            cm[0] += cr * (p[0] + q[0]) / 6.0;
            cm[1] += cr * (p[1] + q[1]) / 6.0;
            if (poly.tag[c][k] < 0) return kReachesBox;
            if (poly.tag[c][k] == i) return kTouchesSelf;
            const int e = out.n++;
            out.j[e] = poly.tag[c][k];
            out.a[e][0] = q[1] - p[1];
            out.a[e][1] = -(q[0] - p[0]);
            out.a[e][2] = 0;
            out.c[e][0] = 0.5 * (p[0] + q[0]);
            out.c[e][1] = 0.5 * (p[1] + q[1]);
            out.c[e][2] = 0;
        }
    }
    for (int a = 0; a < D; ++a) centroid[a] = cm[a] / volume;
    return order_faces(out);
}

// A 3D cell kept as triangles of plane triples, the dual of its vertices (each vertex is where three planes meet; a
// triangle's cyclic order gives the vertex's orientation): a cut drops the triangles beyond the plane and fans the new
// plane over the boundary edges of the dropped region (edges whose reverse is not also dropped), instead of rebuilding
// every face loop. Room for kMaxPlanes planes (the starting box's six first) and kMaxTris vertices; vertex positions
// are kept beside their triangles. Its vertices are plane intersections, so its meshes agree with the face-loop
// cell's to round-off, not bit for bit; the host builder and the device remesher run the same code when they use it.
template <int kMaxPlanes, int kMaxTris>
struct DualT {
    double pn[kMaxPlanes][3], pc[kMaxPlanes];  // planes n.x <= c
    int32_t ptag[kMaxPlanes];
    int np;
    uint8_t tri[kMaxTris][3];
    double tv[kMaxTris][3];
    bool out[kMaxTris];
    uint16_t ek[3 * kMaxTris], eb[3 * kMaxTris];
    int nt;
    double eps;
    bool full;
    double rmax2;  // after a cut: the largest squared vertex radius (max_radius2())

    LUNA_VC_HD void vertex(int t) {  // the meeting point of the triangle's three planes (Cramer's rule)
        const double* a = pn[tri[t][0]];
        const double* b = pn[tri[t][1]];
        const double* c = pn[tri[t][2]];
        double bc[3], ca[3], ab[3];
        cross3(b, c, bc);
        cross3(c, a, ca);
        cross3(a, b, ab);
        const double det = dot3(a, bc);
        for (int k = 0; k < 3; ++k) tv[t][k] = (pc[tri[t][0]] * bc[k] + pc[tri[t][1]] * ca[k] + pc[tri[t][2]] * ab[k]) / det;
    }
    LUNA_VC_HD void box(const double* half) {
        full = false;
        np = 6;
        nt = 0;
        for (int k = 0; k < 6; ++k) {
            for (int a = 0; a < 3; ++a) pn[k][a] = a == k / 2 ? ((k & 1) ? 1.0 : -1.0) : 0.0;
            pc[k] = half[k / 2];
            ptag[k] = -1;
        }
        for (int x = 0; x < 2; ++x)
            for (int y = 0; y < 2; ++y)
                for (int z = 0; z < 2; ++z) {
                    int p0 = x, p1 = 2 + y, p2 = 4 + z;
                    double c01[3];
                    cross3(pn[p0], pn[p1], c01);
                    if (dot3(c01, pn[p2]) < 0) {  // oriented: (n0 x n1) . n2 > 0
                        const int sw = p1;
                        p1 = p2;
                        p2 = sw;
                    }
                    tri[nt][0] = static_cast<uint8_t>(p0);
                    tri[nt][1] = static_cast<uint8_t>(p1);
                    tri[nt][2] = static_cast<uint8_t>(p2);
                    vertex(nt);
                    ++nt;
                }
    }
    LUNA_VC_HD double max_radius2() const {
        double r = 0;
        for (int t = 0; t < nt; ++t) {
            const double d = dot3(tv[t], tv[t]);
            r = d > r ? d : r;
        }
        return r;
    }
    LUNA_VC_HD bool clip(const double* nrm, double c, int32_t tag) {
        bool any = false;
        for (int t = 0; t < nt; ++t) {
            out[t] = dot3(nrm, tv[t]) - c > eps;
            any = any || out[t];
        }
        if (!any) return false;
        if (np >= kMaxPlanes) {
            full = true;
            return false;
        }
        const int q = np++;
        for (int a = 0; a < 3; ++a) pn[q][a] = nrm[a];
        pc[q] = c;
        ptag[q] = tag;
        int ne = 0;  // the dropped triangles' edges, each as (from plane) << 8 | (to plane)
        for (int t = 0; t < nt; ++t)
            if (out[t])
                for (int k = 0; k < 3; ++k) ek[ne++] = static_cast<uint16_t>(tri[t][k] << 8 | tri[t][(k + 1) % 3]);
        int nb = 0;  // the boundary edges: those whose reverse is not a dropped triangle's edge, compacted in order
        for (int e = 0; e < ne; ++e) {
            const uint16_t rev = static_cast<uint16_t>((ek[e] & 0xff) << 8 | ek[e] >> 8);
            bool paired = false;
            for (int f = 0; f < ne && !paired; ++f) paired = ek[f] == rev;
            if (!paired) eb[nb++] = ek[e];
        }
        int w = 0;
        double r = 0;  // the largest squared vertex radius left, as max_radius2() gives it
        for (int t = 0; t < nt; ++t)
            if (!out[t]) {
                if (w != t) {
                    for (int k = 0; k < 3; ++k) tri[w][k] = tri[t][k];
                    for (int k = 0; k < 3; ++k) tv[w][k] = tv[t][k];
                }
                const double d = dot3(tv[w], tv[w]);
                r = d > r ? d : r;
                ++w;
            }
        nt = w;
        if (nt + nb > kMaxTris) {
            full = true;
            return false;
        }
        for (int e = 0; e < nb; ++e) {
            tri[nt][0] = static_cast<uint8_t>(eb[e] >> 8);
            tri[nt][1] = static_cast<uint8_t>(eb[e] & 0xff);
            tri[nt][2] = static_cast<uint8_t>(q);
            vertex(nt);
            const double d = dot3(tv[nt], tv[nt]);
            r = d > r ? d : r;
            ++nt;
        }
        rmax2 = r;
        return true;
    }
    // The faces (one per plane still holding vertices), volume and first moment, as cell_faces3: each face's vertices
    // in order around it (from its lowest triangle, each next triangle the one sharing the plane and the last vertex's
    // other plane), turned to run counter-clockwise seen from outside, fanned from the first.
    template <class Faces>
    LUNA_VC_HD int finish(int64_t i, Faces& faces, double& volume, double* cm) {
        int loop[kMaxTris];
        // each plane's triangles in increasing index (a counting sort of the corners): a face's walk looks only at the
        // triangles of its plane, in the order a scan over all triangles meets them, so it makes the same loop
        int start[kMaxPlanes + 1], at[kMaxPlanes];
        int16_t inc[3 * kMaxTris];
        for (int p = 0; p <= np; ++p) start[p] = 0;
        for (int t = 0; t < nt; ++t)
            for (int k = 0; k < 3; ++k) ++start[tri[t][k] + 1];
        for (int p = 0; p < np; ++p) {
            start[p + 1] += start[p];
            at[p] = start[p];
        }
        for (int t = 0; t < nt; ++t)
            for (int k = 0; k < 3; ++k) inc[at[tri[t][k]]++] = static_cast<int16_t>(t);
        for (int p = 0; p < np; ++p) {
            const int s0 = start[p], s1 = start[p + 1];
            if (s0 == s1) continue;
            const int t0 = inc[s0];
            int m = 0;
            if (ptag[p] < 0) return kReachesBox;
            if (ptag[p] == i) return kTouchesSelf;
            int cur = t0;
            int r = tri[cur][0] == p ? 0 : tri[cur][1] == p ? 1 : 2;
            int b = tri[cur][(r + 2) % 3];
            do {
                if (m >= kMaxTris) return kCapacity;
                loop[m++] = cur;
                int next = -1;  // the triangle with p followed by b
                for (int s = s0; s < s1 && next < 0; ++s)
                    for (int k = 0, t = inc[s]; k < 3; ++k)
                        if (tri[t][k] == p && tri[t][(k + 1) % 3] == b) {
                            next = t;
                            b = tri[t][(k + 2) % 3];
                            break;
                        }
                if (next < 0) return kCapacity;
                cur = next;
            } while (cur != t0);
            if (m < 3) continue;
            double A[3] = {0, 0, 0};
            for (int k = 1; k + 1 < m; ++k) {
                const double* p0 = tv[loop[0]];
                const double* p1 = tv[loop[k]];
                const double* p2 = tv[loop[k + 1]];
                const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
                const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
                double tt[3];
                cross3(e1, e2, tt);
                for (int a = 0; a < 3; ++a) A[a] += 0.5 * tt[a];
            }
            if (dot3(A, pn[p]) < 0)  // the other way round
                for (int k = 1, l = m - 1; k < l; ++k, --l) {
                    const int sw = loop[k];
                    loop[k] = loop[l];
                    loop[l] = sw;
                }
            if (faces.n >= static_cast<int>(sizeof(faces.j) / sizeof(faces.j[0]))) return kCapacity;
            int idx[kMaxTris + 1];
            for (int k = 0; k < m; ++k) idx[k] = loop[k];
            const int fo[2] = {0, m};
            const int32_t tag = ptag[p];
            const int code = cell_faces3(i, tv, idx, fo, &tag, 1, faces, volume, cm);
            if (code != kCellOk) return code;
        }
        return kCellOk;
    }
};

// Cell i as build_cell<3, Far> builds it, with the dual cell.
template <bool Far, class Dual, class Faces, class Cand>
LUNA_VC_HD int build_cell_dual(int64_t i, const double* pos, const double* side, const Grid& grid, Dual& poly, Faces& out, Cand& cand,
                               double& volume, double* centroid) {
    constexpr int D = 3;
    const double* xi = pos + D * i;
    double half[3] = {0, 0, 0};
    double scale = 0, wmax = 0, wmin = 1e300;
    for (int a = 0; a < D; ++a) {
        half[a] = 0.5 * side[a];
        scale = side[a] > scale ? side[a] : scale;
        wmax = grid.w[a] > wmax ? grid.w[a] : wmax;
        wmin = grid.w[a] < wmin ? grid.w[a] : wmin;
    }
    poly.box(half);
    poly.eps = 1e-13 * scale;
    int bi[3] = {0, 0, 0};
    for (int a = 0; a < D; ++a) bi[a] = bucket_of(grid, xi, a);
    double rmax2 = poly.max_radius2();
    const double reach = static_cast<double>(grid.reach - 1) * wmin;
    const double table2 = reach * reach;
    double far2 = 0;
    for (int a = 0; a < D; ++a) far2 = side[a] * side[a] > far2 ? side[a] * side[a] : far2;
    const double limit2 = Far ? far2 : table2;
    double lo2 = 0, hi2 = 4.41 * wmax * wmax;
    hi2 = hi2 < limit2 ? hi2 : limit2;
    for (;;) {
        if (!gather<D, Far>(xi, bi, pos, side, grid, lo2, hi2, table2, cand)) {
            if (!Far) return kCandidates;
            const double thinner = lo2 + 0.25 * (hi2 - lo2);
            if (!(thinner > lo2 && thinner < hi2)) return kCandidates;
            hi2 = thinner;
            continue;
        }
        bool done = false;
        for (int k = 0; k < cand.n; ++k) {
            const int e = cand.order[k];
            const double d2 = cand.key[k];
            if (d2 > 4.0 * rmax2) {
                done = true;
                break;
            }
            const double inv = 1.0 / sqrt(d2);
            double dv[3] = {0, 0, 0};
            const int32_t je = cand.j[e];
            for (int a = 0; a < D; ++a)
                dv[a] = pos[D * je + a] + static_cast<double>(static_cast<int>((cand.w[e] >> (8 * a)) & 0xff) - 128) * side[a] - xi[a];
            const double nrm[3] = {dv[0] * inv, dv[1] * inv, dv[2] * inv};
            if (poly.clip(nrm, 0.5 * d2 * inv, cand.j[e])) rmax2 = poly.rmax2;
            if (poly.full) return kCapacity;
        }
        if (done || 4.0 * rmax2 <= hi2) break;
        if (hi2 >= limit2) return kOutOfOffsets;
        lo2 = hi2;
        hi2 = 4.0 * rmax2 < 2.25 * hi2 ? 4.0 * rmax2 : 2.25 * hi2;
        hi2 = hi2 < limit2 ? hi2 : limit2;
    }
    out.n = 0;
    volume = 0;
    double cm[3] = {0, 0, 0};
    const int code = poly.finish(i, out, volume, cm);
    if (code != kCellOk) return code;
    for (int a = 0; a < D; ++a) centroid[a] = cm[a] / volume;
    return order_faces(out);
}

// The device remesher's storage (about 17 KB a thread in 3D, of which a gas cell touches a third) and the host
// builder's.
using Poly3 = Poly3T<96, 48, 384, 48>;
using Poly2 = Poly2T<64>;
using CellFaces = CellFacesT<48>;
using HostPoly3 = Poly3T<2048, 1024, 8192, 1024>;
using HostPoly2 = Poly2T<4096>;
using HostCellFaces = CellFacesT<4096>;
using Candidates = CandidatesT<160>;
using HostCandidates = CandidatesT<16384>;
using Dual = DualT<64, 128>;
using HostDual = DualT<256, 510>;

}  // namespace luna_voronoi
