// The mesh reordered for the step's kernels, once per mesh (a static mesh: once; a moving mesh: after each remesh).
//
// luna-cpp's sweep and flux kernels walk voronoi-cpp's lists and recompute the same geometry every step: each list entry
// costs three dependent loads (list -> face -> neighbour -> rows) plus the separation, the fit row X = [1, d + c_j - c_i]
// and the face offset. Everything there except the neighbours' primitive rows depends on the mesh only, so this pass
// computes it once, in the reference's arithmetic, into rows that the step streams in list order:
//   entry rows [2F]  per list entry: w X_p (the fit's weighted row, p = 0..D), the face offset x_f - c_i, the neighbour,
//                    whether the cell owns the face, the face, and whether the face is below 1e-6 of the cell's surface;
//   fit factors [N]  the Cholesky factor of the cell's normal matrix M = sum w X X^T (finite_volume.hpp:591-602);
//   dt rows [F]      the separation d of the face's generators and |d| (the CFL face terms, finite_volume.hpp:1074-1090);
//   face rows [F]    the unit normal A / |A|, |A|, both cells' face offsets and the two cells (FaceFlux, :1415-1434);
//   cell angle [N]   the largest AREPO face angle of the cell (the moving mesh's regularisation, :509, :526-537).
// The step then reads one streamed row per entry and gathers only the neighbour's primitive row: one dependent level.
#pragma once

#include <type_traits>

#include "kernels.cuh"

namespace luna {

// A list entry's row. wx[p] = w X_p with w = |A_f| (p = 0 .. D), off = face offset; bits: neighbour | owned << 31 in the
// low word, face | tiny << 31 in the high word (double rows); float rows keep the face word in a separate array.
struct alignas(64) EntryRow64 {
    double wx[4];
    double off[3];
    unsigned long long bits;
};
struct alignas(32) EntryRow32 {
    float wx[4];
    float off[3];
    unsigned int nbr_owned;
};
template <class G>
using EntryRow = typename std::conditional<sizeof(G) == sizeof(double), EntryRow64, EntryRow32>::type;

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

struct DtRow {
    double d[3];
    double dist;
};

template <int D>
constexpr int factor_width() {
    return (D + 1) * (D + 2) / 2;  // the lower triangle of the (D+1)^2 factor
}

template <int D, class G>
struct GeometryDev {
    EntryRow<G>* __restrict__ entries;
    unsigned int* __restrict__ face_tiny;  // float rows: face | tiny << 31 per entry
    G* __restrict__ factors;               // [N][factor_width]
    DtRow* __restrict__ dt_rows;           // [F]
    FaceRow<G>* __restrict__ faces;        // [F]
    double* __restrict__ max_angle;        // [N]
};

// One thread a cell: the cell's geometry in list order, as Sweep::operator() computes it (finite_volume.hpp:486-520),
// and the face rows of the faces it owns.
template <int D, class G>
__global__ void __launch_bounds__(128) k_geometry(MeshDev<D> m, GeometryDev<D, G> g) {
    constexpr int U = D + 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    double centroid[D];
#pragma unroll
    for (int a = 0; a < D; ++a) centroid[a] = m.cen[D * i + a];
    const int first = m.start[i], end = m.start[i + 1];
    double surface = 0, smallest = __longlong_as_double(0x7ff0000000000000ll), max_angle = 0;
    G M[U][U];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s < U; ++s) M[p][s] = G(0);
    for (int k = first; k < end; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e);
        const int j = e >= 0 ? m.neighbour[f] : m.owner[f];
        double d[D];
        m.separation(i, j, d);
        const double magnitude = m.mag[f];
        surface += magnitude;
        smallest = fmin(smallest, magnitude);
        const double d2 = dot<D>(d, d);
        max_angle = fmax(max_angle, face_angle<D>(magnitude) / (0.5 * sqrt(d2)));
        G X[U];
        X[0] = G(1);
#pragma unroll
        for (int p = 1; p < U; ++p) X[p] = static_cast<G>(d[p - 1] + m.cen[D * j + p - 1] - centroid[p - 1]);
        const G w = static_cast<G>(magnitude);
#pragma unroll
        for (int p = 0; p < U; ++p)
#pragma unroll
            for (int s = p; s < U; ++s) M[p][s] += w * X[p] * X[s];
        EntryRow<G>& row = g.entries[k];
#pragma unroll
        for (int p = 0; p < 4; ++p) row.wx[p] = p < U ? w * X[p] : G(0);
        if (e >= 0) {
            DtRow t;
#pragma unroll
            for (int a = 0; a < 3; ++a) t.d[a] = a < D ? d[a] : 0.0;
            t.dist = sqrt(d2);
            g.dt_rows[f] = t;
        }
    }
    const double tiny = 1e-6 * surface;
    const bool any_tiny = smallest < tiny;
    for (int k = first; k < end; ++k) {
        const int32_t e = m.list[k];
        const int f = list_face(e);
        const bool owned = e >= 0;
        const int j = owned ? m.neighbour[f] : m.owner[f];
        double off[D];
        m.face_offset(f, i, off);
        const bool tiny_face = any_tiny && m.mag[f] < tiny;
        EntryRow<G>& row = g.entries[k];
#pragma unroll
        for (int a = 0; a < 3; ++a) row.off[a] = a < D ? static_cast<G>(off[a]) : G(0);
        const unsigned int low = static_cast<unsigned int>(j) | (owned ? 0x80000000u : 0u);
        const unsigned int high = static_cast<unsigned int>(f) | (tiny_face ? 0x80000000u : 0u);
        if constexpr (sizeof(G) == sizeof(double)) {
            row.bits = static_cast<unsigned long long>(low) | (static_cast<unsigned long long>(high) << 32);
        } else {
            row.nbr_owned = low;
            g.face_tiny[k] = high;
        }
        if (owned) {  // the face row, written once by the owner
            double a[D];
#pragma unroll
            for (int q = 0; q < D; ++q) a[q] = m.area[D * f + q];
            const double magnitude = sqrt(dot<D>(a, a));
            double offj[D];
            m.face_offset(f, j, offj);
            FaceRow<G> r;
            const double inv = magnitude == 0 ? 0.0 : 1.0 / magnitude;
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
            r.mag = magnitude;
            r.o = i;
            r.j = j;
            if constexpr (sizeof(G) == sizeof(double)) r.pad = 0;
            g.faces[f] = r;
        }
    }
    // Sweep::solve's factorisation (finite_volume.hpp:591-602), the lower triangle row by row.
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
            for (int q = 0; q < s; ++q) sum -= L[p][q] * L[s][q];
            L[p][s] = p == s ? sqrt(sum) : sum / L[s][s];
        }
    G* out = g.factors + static_cast<int64_t>(factor_width<D>()) * i;
    int c = 0;
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int s = 0; s <= p; ++s) out[c++] = L[p][s];
    g.max_angle[i] = max_angle;
}

// The sweep over the reordered rows (Sweep<Moving, Grad>::operator(), finite_volume.hpp:463-569, same arithmetic):
// walk 1 sums b = sum w X (W_j - W_i) and the neighbours' range (tiny faces left out), and the owned faces' CFL terms;
// the fit is solved with the cell's stored factor; walk 2 clips at each face offset in list order. One streamed row and
// one gathered primitive row per entry.
template <int D, bool Moving, bool Grad, class G, bool Limit>
__global__ void __launch_bounds__(128) k_sweep_rows(MeshDev<D> m, GeometryDev<D, G> geo, const double* __restrict__ prims,
                                                    G* __restrict__ grad_out, double* __restrict__ w_out, double courant,
                                                    Counters* __restrict__ ctr) {
    constexpr int V = D + 2, U = D + 1, GS = grad_stride<D>();
    constexpr bool exact = sizeof(G) == sizeof(double);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double smallest_dt = 1.0e300;
    if (i < m.n) {
        const double* pi = prims + PS * i;
        double Wi[V];
#pragma unroll
        for (int v = 0; v < V; ++v) Wi[v] = pi[v];
        const double ci = pi[V], ri = pi[V + 1];
        G lo[V], hi[V], b[V][U];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            lo[v] = finite_max<G>();
            hi[v] = -finite_max<G>();
#pragma unroll
            for (int p = 0; p < U; ++p) b[v][p] = G(0);
        }
        const int first = m.start[i], end = m.start[i + 1];
        for (int k = first; k < end; ++k) {
            const EntryRow<G>& row = geo.entries[k];
            unsigned int low, high;
            if constexpr (exact) {
                const unsigned long long bits = row.bits;
                low = static_cast<unsigned int>(bits);
                high = static_cast<unsigned int>(bits >> 32);
            } else {
                low = row.nbr_owned;
                high = geo.face_tiny[k];
            }
            const int j = static_cast<int>(low & 0x7fffffffu);
            const bool owned = (low >> 31) != 0, tiny_face = (high >> 31) != 0;
            const double* pj = prims + PS * j;
            double Wj[V];
#pragma unroll
            for (int v = 0; v < V; ++v) Wj[v] = pj[v];
            if (owned) {  // FaceStep (finite_volume.hpp:1074-1090)
                const DtRow t = geo.dt_rows[high & 0x7fffffffu];
                double dv[D], d[D];
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    dv[a] = Wj[1 + a] - Wi[1 + a];
                    d[a] = t.d[a];
                }
                const double vsig = ci + pj[V] - dot<D>(dv, d) / t.dist;
                if (vsig > 0) {
                    smallest_dt = fmin(smallest_dt, courant * ((t.dist + ri) / vsig));
                    smallest_dt = fmin(smallest_dt, courant * ((t.dist + pj[V + 1]) / vsig));
                }
            }
            if constexpr (Grad) {
                G wx[U];
#pragma unroll
                for (int p = 0; p < U; ++p) wx[p] = row.wx[p];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const double dW = Wj[v] - Wi[v];
#pragma unroll
                    for (int p = 0; p < U; ++p) b[v][p] += wx[p] * static_cast<G>(dW);
                    if (!tiny_face) {
                        const G value = exact ? static_cast<G>(Wj[v]) : static_cast<G>(dW);
                        lo[v] = fmin(lo[v], value);
                        hi[v] = fmax(hi[v], value);
                    }
                }
            }
        }
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
            // Sweep::solve with the stored factor: forward and back substitution per variable.
            G L[U][U];
            const G* fr = geo.factors + static_cast<int64_t>(factor_width<D>()) * i;
            {
                int c = 0;
#pragma unroll
                for (int p = 0; p < U; ++p)
#pragma unroll
                    for (int s = 0; s <= p; ++s) L[p][s] = fr[c++];
            }
            G g[V * D];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                G z[U], x[U];
#pragma unroll
                for (int p = 0; p < U; ++p) {
                    G sum = b[v][p];
#pragma unroll
                    for (int q = 0; q < p; ++q) sum -= L[p][q] * z[q];
                    z[p] = sum / L[p][p];
                }
#pragma unroll
                for (int p = U - 1; p >= 0; --p) {
                    G sum = z[p];
#pragma unroll
                    for (int q = p + 1; q < U; ++q) sum -= L[q][p] * x[q];
                    x[p] = sum / L[p][p];
                }
#pragma unroll
                for (int a = 0; a < D; ++a) g[D * v + a] = x[1 + a];
            }
            if constexpr (Limit) {
                for (int k = first; k < end; ++k) {
                    const EntryRow<G>& row = geo.entries[k];
                    bool tiny_face;
                    if constexpr (exact)
                        tiny_face = (row.bits >> 63) != 0;
                    else
                        tiny_face = (geo.face_tiny[k] >> 31) != 0;
                    if (tiny_face) continue;
                    G rg[D];
#pragma unroll
                    for (int a = 0; a < D; ++a) rg[a] = row.off[a];
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        G* gv = g + D * v;
                        const G dp = dot<D>(gv, rg);
                        if constexpr (exact) {
                            if (dp > 0 && Wi[v] + dp > hi[v]) {
                                const G s = hi[v] > Wi[v] ? (hi[v] - Wi[v]) / dp : G(0);
#pragma unroll
                                for (int a = 0; a < D; ++a) gv[a] = gv[a] * s;
                            } else if (dp < 0 && Wi[v] + dp < lo[v]) {
                                const G s = lo[v] < Wi[v] ? (lo[v] - Wi[v]) / dp : G(0);
#pragma unroll
                                for (int a = 0; a < D; ++a) gv[a] = gv[a] * s;
                            }
                        } else {
                            if (dp > 0 && dp > hi[v]) {
                                const G s = hi[v] > 0 ? hi[v] / dp : G(0);
#pragma unroll
                                for (int a = 0; a < D; ++a) gv[a] = gv[a] * s;
                            } else if (dp < 0 && dp < lo[v]) {
                                const G s = lo[v] < 0 ? lo[v] / dp : G(0);
#pragma unroll
                                for (int a = 0; a < D; ++a) gv[a] = gv[a] * s;
                            }
                        }
                    }
                }
            }
            G* out = grad_out + static_cast<int64_t>(GS) * i;
#pragma unroll
            for (int c = 0; c < V * D; ++c) out[c] = g[c];
        }
    }
    block_min_to(smallest_dt, &ctr->dt_bits);
    if (i < m.n && !(smallest_dt == smallest_dt)) atomicOr(&ctr->error, 1ull);
}

// The static flux pass over the face rows (FaceFlux::operator(), finite_volume.hpp:1415-1434): one streamed row per
// face, then the two cells' primitive and gradient rows.
template <int D, int Order, class G, bool RF, int Riemann>
__global__ void __launch_bounds__(128) k_flux_rows(MeshDev<D> m, GeometryDev<D, G> geo, FluxArgs<D, G> x, double* __restrict__ flux,
                                                   unsigned long long* __restrict__ fallbacks) {
    constexpr int V = D + 2;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    int count = 0;
    if (f < m.f) {
        const FaceRow<G> r = geo.faces[f];
        double F[V];
        if (r.mag == 0) {
#pragma unroll
            for (int v = 0; v < V; ++v) F[v] = 0;
        } else {
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
                face_side<D, G>(x, r.o, ro, x.dt, L, count);
                face_side<D, G>(x, r.j, rj, x.dt, R, count);
            }
            riemann_solve<D, RF, Riemann>(L, R, n, wf, x.gas, F, false);
#pragma unroll
            for (int v = 0; v < V; ++v) F[v] *= r.mag;
        }
#pragma unroll
        for (int v = 0; v < V; ++v) flux[V * static_cast<int64_t>(f) + v] = F[v];
    }
    block_sum_to(static_cast<unsigned long long>(count), fallbacks);
}

}  // namespace luna
