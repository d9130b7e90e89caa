// One 3D cell per warp: the clipping of voronoi_cell.h restated in warp-wide phases, with the cell in shared memory.
//
// Every phase is a loop whose iterations are independent (one lane each, strided by 32), joined by warp reductions and
// prefix sums, and every quantity is computed in the order the one-thread clip computes it:
//   distances     lanes over vertices; the maximum is exact in any order;
//   kept vertices compacted in index order by a ballot prefix (the one-thread clip's remap);
//   crossings     lanes over faces count each face's kept entries and crossing edges; a prefix over faces puts the
//                 crossings in (face, position) order; each crossing finds the other occurrence of its edge; the
//                 first of the two numbers the new vertex (the one-thread clip's memo: first seen in face order) and
//                 gives its orientation, so the new vertex is p + t (q - p) from the same p and q;
//   new loops     a prefix over the faces that keep three entries places each face's loop;
//   new face      the cut vertices sorted, their mean, the diamond angles and the ordering on one lane.
// The finished cell's faces, volume and centroid are summed on one lane by the same code as the one-thread build
// (cell_faces3, order_faces). The mesh is the same, bit for bit.
#pragma once

#include "voronoi_cell.h"

namespace luna_voronoi {

constexpr int kWarpVerts = 96, kWarpFaces = 48, kWarpLoop = 384, kWarpCut = 48, kWarpOcc = 96, kWarpCand = 160;

// A warp's cell in shared memory (about 20 KB).
struct WarpCell {
    double v[2][kWarpVerts][3];
    int idx[2][kWarpLoop];
    int fo[2][kWarpFaces + 1];
    int32_t tag[2][kWarpFaces];
    double s[kWarpVerts];
    int remap[kWarpVerts];
    int face_kept[kWarpFaces], face_cross[kWarpFaces], face_occ0[kWarpFaces], face_out[kWarpFaces];
    int occ_f[kWarpOcc], occ_a[kWarpOcc], occ_b[kWarpOcc], occ_twin[kWarpOcc], occ_id[kWarpOcc];
    int cut[kWarpCut];
    double angle[kWarpCut];
    double cd[kWarpCand][3];
    double cd2[kWarpCand];
    int32_t cj[kWarpCand];
    int corder[kWarpCand];
    int nv[2], nf[2], cur, ncand;
    CellFacesT<kWarpFaces> faces;
};

#if defined(__CUDACC__)
__device__ __forceinline__ unsigned lanes_below() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int warp_exclusive_sum(int x, int lane, int* total) {
    int incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    *total = __shfl_sync(0xffffffffu, incl, 31);
    return incl - x;
}

__device__ __forceinline__ double warp_max(double x) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const double y = __shfl_xor_sync(0xffffffffu, x, d);
        x = y > x ? y : x;
    }
    return x;
}

__device__ __forceinline__ bool crossing(const double* s, int a, int b, double eps) {
    return (s[a] < -eps && s[b] > eps) || (s[a] > eps && s[b] < -eps);
}

// The largest squared vertex radius of the current polyhedron.
__device__ __forceinline__ double warp_radius2(const WarpCell& w, int lane) {
    double r = 0;
    const int c = w.cur;
    for (int k = lane; k < w.nv[c]; k += 32) {
        const double d = dot3(w.v[c][k], w.v[c][k]);
        r = d > r ? d : r;
    }
    return warp_max(r);
}

// Keeps {y : nrm.y <= c}, the new face tagged t. Returns 1 if cut, 0 if not, -1 if a capacity ran out (warp-uniform).
__device__ int warp_clip(WarpCell& w, const double* nrm, double c, int32_t t, double eps, int lane) {
    const int o = w.cur, n = o ^ 1;
    const int nvert = w.nv[o], nface = w.nf[o];
    double lmax = -1e300;
    for (int k = lane; k < nvert; k += 32) {
        w.s[k] = dot3(nrm, w.v[o][k]) - c;
        lmax = w.s[k] > lmax ? w.s[k] : lmax;
    }
    if (warp_max(lmax) <= eps) return 0;
    __syncwarp();
    int nkept = 0;
    for (int base = 0; base < nvert; base += 32) {
        const int k = base + lane;
        const bool keep = k < nvert && w.s[k] <= eps;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (k < nvert) w.remap[k] = keep ? nkept + __popc(m & lanes_below()) : -1;
        nkept += __popc(m);
    }
    __syncwarp();
    for (int k = lane; k < nvert; k += 32)
        if (w.remap[k] >= 0)
            for (int a = 0; a < 3; ++a) w.v[n][w.remap[k]][a] = w.v[o][k][a];
    for (int f = lane; f < nface; f += 32) {
        const int a0 = w.fo[o][f], m = w.fo[o][f + 1] - a0;
        int kept = 0, cross = 0;
        for (int k = 0; k < m; ++k) {
            const int a = w.idx[o][a0 + k], b = w.idx[o][a0 + (k + 1) % m];
            kept += w.s[a] <= eps;
            cross += crossing(w.s, a, b, eps);
        }
        w.face_kept[f] = kept;
        w.face_cross[f] = cross;
    }
    __syncwarp();
    int nocc = 0;
    for (int base = 0; base < nface; base += 32) {
        const int f = base + lane;
        int total;
        const int before = warp_exclusive_sum(f < nface ? w.face_cross[f] : 0, lane, &total);
        if (f < nface) w.face_occ0[f] = nocc + before;
        nocc += total;
    }
    if (nocc > kWarpOcc) return -1;
    __syncwarp();
    for (int f = lane; f < nface; f += 32) {
        const int a0 = w.fo[o][f], m = w.fo[o][f + 1] - a0;
        int q = w.face_occ0[f];
        for (int k = 0; k < m; ++k) {
            const int a = w.idx[o][a0 + k], b = w.idx[o][a0 + (k + 1) % m];
            if (crossing(w.s, a, b, eps)) {
                w.occ_f[q] = f;
                w.occ_a[q] = a;
                w.occ_b[q] = b;
                ++q;
            }
        }
    }
    __syncwarp();
    for (int q = lane; q < nocc; q += 32) {
        const int lo = min(w.occ_a[q], w.occ_b[q]), hi = max(w.occ_a[q], w.occ_b[q]);
        int twin = -1;  // the earliest other occurrence of the edge
        for (int r = 0; r < nocc && twin < 0; ++r)
            if (r != q && min(w.occ_a[r], w.occ_b[r]) == lo && max(w.occ_a[r], w.occ_b[r]) == hi) twin = r;
        w.occ_twin[q] = twin;
    }
    __syncwarp();
    int nnew = 0;
    for (int base = 0; base < nocc; base += 32) {
        const int q = base + lane;
        const bool first = q < nocc && (w.occ_twin[q] < 0 || q < w.occ_twin[q]);
        const unsigned m = __ballot_sync(0xffffffffu, first);
        if (first) w.occ_id[q] = nkept + nnew + __popc(m & lanes_below());
        nnew += __popc(m);
    }
    if (nkept + nnew > kWarpVerts || nnew > kWarpCut) return -1;
    __syncwarp();
    for (int q = lane; q < nocc; q += 32) {
        const int twin = w.occ_twin[q];
        if (twin >= 0 && twin < q) {
            w.occ_id[q] = w.occ_id[twin];
        } else {  // the first occurrence: the new vertex from its orientation
            const int a = w.occ_a[q], b = w.occ_b[q];
            const double tt = w.s[a] / (w.s[a] - w.s[b]);
            const double* p = w.v[o][a];
            const double* r = w.v[o][b];
            const int id = w.occ_id[q];
            w.v[n][id][0] = p[0] + tt * (r[0] - p[0]);
            w.v[n][id][1] = p[1] + tt * (r[1] - p[1]);
            w.v[n][id][2] = p[2] + tt * (r[2] - p[2]);
        }
    }
    __syncwarp();
    // the faces that keep three entries, in order, and their loops' offsets
    int fi = 0, li = 0;
    for (int base = 0; base < nface; base += 32) {
        const int f = base + lane;
        const int len = f < nface ? w.face_kept[f] + w.face_cross[f] : 0;
        const bool stays = f < nface && len >= 3;
        const unsigned m = __ballot_sync(0xffffffffu, stays);
        int total;
        const int before = warp_exclusive_sum(stays ? len : 0, lane, &total);
        if (f < nface) w.face_out[f] = stays ? fi + __popc(m & lanes_below()) : -1;
        if (stays) w.fo[n][fi + __popc(m & lanes_below())] = li + before;
        fi += __popc(m);
        li += total;
    }
    if (fi > kWarpFaces || li > kWarpLoop) return -1;
    __syncwarp();
    if (lane == 0) w.fo[n][fi] = li;
    for (int f = lane; f < nface; f += 32) {
        if (w.face_out[f] < 0) continue;
        const int a0 = w.fo[o][f], m = w.fo[o][f + 1] - a0;
        int at = w.fo[n][w.face_out[f]], q = w.face_occ0[f];
        for (int k = 0; k < m; ++k) {
            const int a = w.idx[o][a0 + k], b = w.idx[o][a0 + (k + 1) % m];
            if (w.s[a] <= eps) w.idx[n][at++] = w.remap[a];
            if (crossing(w.s, a, b, eps)) w.idx[n][at++] = w.occ_id[q++];
        }
        w.tag[n][w.face_out[f]] = w.tag[o][f];
    }
    __syncwarp();
    int status = 1;
    if (lane == 0) {  // the new face
        int ncut = 0;
        for (int k = 0; k < nvert; ++k)
            if (w.s[k] <= eps && w.s[k] >= -eps) {
                if (ncut >= kWarpCut) status = -1;
                else w.cut[ncut++] = w.remap[k];
            }
        for (int r = 0; r < nnew; ++r) {
            if (ncut >= kWarpCut) status = -1;
            else w.cut[ncut++] = nkept + r;
        }
        if (status < 0) ncut = 0;
        for (int k = 1; k < ncut; ++k) {  // sorted, once each
            const int x = w.cut[k];
            int j = k - 1;
            while (j >= 0 && w.cut[j] > x) {
                w.cut[j + 1] = w.cut[j];
                --j;
            }
            w.cut[j + 1] = x;
        }
        int unique = 0;
        for (int k = 0; k < ncut; ++k)
            if (unique == 0 || w.cut[unique - 1] != w.cut[k]) w.cut[unique++] = w.cut[k];
        ncut = unique;
        if (ncut >= 3) {
            double mean[3] = {0, 0, 0};
            for (int k = 0; k < ncut; ++k)
                for (int a = 0; a < 3; ++a) mean[a] += w.v[n][w.cut[k]][a];
            for (int a = 0; a < 3; ++a) mean[a] /= static_cast<double>(ncut);
            double u[3] = {0, 0, 0};
            u[fabs(nrm[0]) < 0.6 ? 0 : 1] = 1;
            const double un = dot3(u, nrm);
            for (int a = 0; a < 3; ++a) u[a] = u[a] - un * nrm[a];
            const double ul = sqrt(dot3(u, u));
            for (int a = 0; a < 3; ++a) u[a] = u[a] / ul;
            double wv[3];
            cross3(nrm, u, wv);
            for (int k = 0; k < ncut; ++k) {
                const double* p = w.v[n][w.cut[k]];
                const double d[3] = {p[0] - mean[0], p[1] - mean[1], p[2] - mean[2]};
                w.angle[k] = diamond_angle(dot3(d, u), dot3(d, wv));
            }
            for (int k = 1; k < ncut; ++k) {
                const int x = w.cut[k];
                const double ax = w.angle[k];
                int j = k - 1;
                while (j >= 0 && w.angle[j] > ax) {
                    w.cut[j + 1] = w.cut[j];
                    w.angle[j + 1] = w.angle[j];
                    --j;
                }
                w.cut[j + 1] = x;
                w.angle[j + 1] = ax;
            }
            if (fi >= kWarpFaces || li + ncut > kWarpLoop) {
                status = -1;
            } else {
                for (int k = 0; k < ncut; ++k) w.idx[n][li + k] = w.cut[k];
                w.tag[n][fi] = t;
                w.fo[n][fi + 1] = li + ncut;
                ++fi;
            }
        }
        w.nf[n] = fi;
        w.nv[n] = nkept + nnew;
        w.cur = n;
    }
    status = __shfl_sync(0xffffffffu, status, 0);
    __syncwarp();
    return status;
}

// The cell's images with lo2 < d2 <= hi2 through the grid's sorted offsets (lanes over offsets, in offset order), then
// ordered by (d2, index, gather position). Returns false when they outgrow the store (warp-uniform).
__device__ bool warp_gather(WarpCell& w, const double* xi, const int* bi, const double* pos, const double* side, const Grid& grid, double lo2,
                            double hi2, int lane) {
    int count = 0;
    for (int base = 0; base < grid.n_offsets; base += 32) {
        const int k = base + lane;
        const bool in = k < grid.n_offsets && grid.bound2[k] <= hi2;
        if (__ballot_sync(0xffffffffu, in) == 0) break;
        int64_t b = 0;
        double shift[3] = {0, 0, 0};
        int mine = 0;
        if (in) {
            const int32_t* o = grid.offsets + 3 * k;
            for (int a = 0; a < 3; ++a) {
                const int t = bi[a] + o[a];
                const int tw = ((t % grid.nb[a]) + grid.nb[a]) % grid.nb[a];
                shift[a] = static_cast<double>((t - tw) / grid.nb[a]) * side[a];
                b = b * grid.nb[a] + tw;
            }
            for (int64_t q = grid.start[b]; q < grid.start[b + 1]; ++q) {
                const int32_t j = grid.items[q];
                double d2 = 0;
                for (int a = 0; a < 3; ++a) {
                    const double d = pos[3 * j + a] + shift[a] - xi[a];
                    d2 += d * d;
                }
                mine += d2 > lo2 && d2 <= hi2;
            }
        }
        int total;
        int at = count + warp_exclusive_sum(mine, lane, &total);
        if (count + total > kWarpCand) return false;
        if (in) {
            for (int64_t q = grid.start[b]; q < grid.start[b + 1]; ++q) {
                const int32_t j = grid.items[q];
                double d[3];
                double d2 = 0;
                for (int a = 0; a < 3; ++a) {
                    d[a] = pos[3 * j + a] + shift[a] - xi[a];
                    d2 += d[a] * d[a];
                }
                if (!(d2 > lo2 && d2 <= hi2)) continue;
                for (int a = 0; a < 3; ++a) w.cd[at][a] = d[a];
                w.cd2[at] = d2;
                w.cj[at] = j;
                ++at;
            }
        }
        count += total;
    }
    __syncwarp();
    for (int q = lane; q < count; q += 32) {  // stable rank by (d2, j)
        int rank = 0;
        for (int r = 0; r < count; ++r)
            rank += w.cd2[r] < w.cd2[q] || (w.cd2[r] == w.cd2[q] && (w.cj[r] < w.cj[q] || (w.cj[r] == w.cj[q] && r < q)));
        w.corder[rank] = q;
    }
    if (lane == 0) w.ncand = count;
    __syncwarp();
    return true;
}

// Cell i on the fast path (the grid's sorted offsets, the candidate store): kCellOk, or why not (kOutOfOffsets and
// kCandidates send the cell to the far search). Warp-uniform.
__device__ int warp_build_cell(int64_t i, const double* pos, const double* side, const Grid& grid, WarpCell& w, double& volume,
                               double* centroid, int lane) {
    const double* xi = pos + 3 * i;
    double half[3], scale = 0, wmax = 0, wmin = 1e300;
    for (int a = 0; a < 3; ++a) {
        half[a] = 0.5 * side[a];
        scale = side[a] > scale ? side[a] : scale;
        wmax = grid.w[a] > wmax ? grid.w[a] : wmax;
        wmin = grid.w[a] < wmin ? grid.w[a] : wmin;
    }
    if (lane == 0) {
        w.cur = 0;
        w.nv[0] = 8;
        for (int k = 0; k < 8; ++k) {
            w.v[0][k][0] = (k & 1) ? half[0] : -half[0];
            w.v[0][k][1] = (k & 2) ? half[1] : -half[1];
            w.v[0][k][2] = (k & 4) ? half[2] : -half[2];
        }
        const int loops[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
        w.nf[0] = 6;
        w.fo[0][0] = 0;
        for (int f = 0; f < 6; ++f) {
            for (int k = 0; k < 4; ++k) w.idx[0][4 * f + k] = loops[f][k];
            w.fo[0][f + 1] = 4 * f + 4;
            w.tag[0][f] = -1;
        }
    }
    __syncwarp();
    const double eps = 1e-13 * scale;
    int bi[3];
    for (int a = 0; a < 3; ++a) bi[a] = bucket_of(grid, xi, a);
    double rmax2 = warp_radius2(w, lane);
    const double reach = static_cast<double>(grid.reach - 1) * wmin;
    const double table2 = reach * reach;
    double lo2 = 0, hi2 = 4.41 * wmax * wmax;
    hi2 = hi2 < table2 ? hi2 : table2;
    for (;;) {
        if (!warp_gather(w, xi, bi, pos, side, grid, lo2, hi2, lane)) return kCandidates;
        bool done = false;
        const int count = w.ncand;
        for (int k = 0; k < count; ++k) {
            const int e = w.corder[k];
            const double d2 = w.cd2[e];
            if (d2 > 4.0 * rmax2) {
                done = true;
                break;
            }
            const double inv = 1.0 / sqrt(d2);
            const double nrm[3] = {w.cd[e][0] * inv, w.cd[e][1] * inv, w.cd[e][2] * inv};
            const int cut = warp_clip(w, nrm, 0.5 * d2 * inv, w.cj[e], eps, lane);
            if (cut < 0) return kCapacity;
            if (cut > 0) rmax2 = warp_radius2(w, lane);
        }
        if (done || 4.0 * rmax2 <= hi2) break;
        if (hi2 >= table2) return kOutOfOffsets;
        lo2 = hi2;
        hi2 = 4.0 * rmax2 < 2.25 * hi2 ? 4.0 * rmax2 : 2.25 * hi2;
        hi2 = hi2 < table2 ? hi2 : table2;
    }
    int code = kCellOk;
    if (lane == 0) {
        double cm[3] = {0, 0, 0};
        volume = 0;
        w.faces.n = 0;
        const int c = w.cur;
        code = cell_faces3(i, w.v[c], w.idx[c], w.fo[c], w.tag[c], w.nf[c], w.faces, volume, cm);
        if (code == kCellOk) {
            for (int a = 0; a < 3; ++a) centroid[a] = cm[a] / volume;
            code = order_faces(w.faces);
        }
    }
    code = __shfl_sync(0xffffffffu, code, 0);
    __syncwarp();
    return code;
}
#endif

}  // namespace luna_voronoi
