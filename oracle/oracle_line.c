/* CPU oracle of luna-cpp's 1D solver on a static line, FiniteVolume<1> (src/hydro/finite_volume_1d.hpp): TEST
 * INFRASTRUCTURE ONLY — the checker of the CUDA line solver (luna_line_* in include/luna_b200.h).
 *
 * Pinned by LUNA's final states at N = 16 (src/test/luna_1d_values.hpp: Sod, Shu-Osher, Woodward-Colella; MC = the
 * face-centroid limiter on a uniform line, HLLC, CFL 0.8, LUNA's time-step rule), which the reference's own test holds
 * to 1e-12 (src/test/hydro1d_test.cpp:266-296).
 *
 * The line: generators at integer keys on a grid of `step` (voronoi-cpp's snapping grid, absent here), sorted; slot s is
 * the s-th generator along the line. Cell s reaches halfway to its neighbours; at a wall, to the wall (its ghost sits
 * at the mirror image of the end generator); a periodic line closes over the seam. Arithmetic in IEEE double in the
 * reference's operation order, compiled without multiply-add contraction.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "luna_oracle.h"

struct lo_line {
    int n, periodic, order, limiter, riemann;
    int walls[2];          /* LO_WALL_* left, right */
    double inflow[2][3];   /* primitives of an inflow wall */
    double step;           /* grid step */
    double *gap;           /* [n + 1]: gap[s + 1] = grid steps from slot s to slot s + 1; gap[0], gap[n]: over the ends */
    double *volume, *centroid;
    lo_gas gas;
    double* q;             /* Q [n][3], slot order */
    double* next;
};

/* Line::gap in grid steps (finite_volume_1d.hpp:105, load_inner :163-169): between neighbours the key difference; at a
 * wall twice the end generator's distance to it (the ghost at its mirror image); on a periodic line, across the seam. */
lo_line* lo_line_create(int n, const int64_t* keys, int64_t period, double step, int periodic, const int* walls, const double* inflow,
                        const lo_gas* gas, int order, int limiter, int riemann) {
    lo_line* ln = (lo_line*)calloc(1, sizeof(lo_line));
    ln->n = n;
    ln->periodic = periodic;
    ln->order = order;
    ln->limiter = limiter;
    ln->riemann = riemann;
    ln->walls[0] = walls ? walls[0] : LO_WALL_OUTFLOW;
    ln->walls[1] = walls ? walls[1] : LO_WALL_OUTFLOW;
    if (inflow) memcpy(ln->inflow, inflow, sizeof(ln->inflow));
    ln->step = step;
    ln->gas = *gas;
    ln->gap = (double*)malloc(sizeof(double) * (n + 1));
    ln->volume = (double*)malloc(sizeof(double) * n);
    ln->centroid = (double*)malloc(sizeof(double) * n);
    ln->q = (double*)calloc((size_t)n * 3, sizeof(double));
    ln->next = (double*)calloc((size_t)n * 3, sizeof(double));
    for (int s = 0; s + 1 < n; ++s) ln->gap[s + 1] = (double)(keys[s + 1] - keys[s]);
    if (periodic) {
        const double seam = (double)(keys[0] + period - keys[n - 1]);
        ln->gap[0] = seam;
        ln->gap[n] = seam;
    } else {
        ln->gap[0] = (double)(2 * keys[0]);
        ln->gap[n] = (double)(2 * (period - keys[n - 1]));
    }
    /* Line::volume, Line::centroid (load_inner :170-176): half of each gap, the centroid a quarter of their difference */
    for (int s = 0; s < n; ++s) {
        ln->volume[s] = (ln->gap[s] + ln->gap[s + 1]) * (0.5 * step);
        ln->centroid[s] = (ln->gap[s + 1] - ln->gap[s]) * (0.25 * step);
    }
    return ln;
}

void lo_line_destroy(lo_line* ln) {
    if (!ln) return;
    free(ln->gap);
    free(ln->volume);
    free(ln->centroid);
    free(ln->q);
    free(ln->next);
    free(ln);
}

double* lo_line_state(lo_line* ln) { return ln->q; }
const double* lo_line_volumes(const lo_line* ln) { return ln->volume; }
const double* lo_line_centroids(const lo_line* ln) { return ln->centroid; }

typedef struct {
    double W[3], c, V;
    int real;
} cell1;

static void primitive_of(const lo_line* ln, int s, double* W) {
    const double inv = 1.0 / ln->volume[s];
    double U[3];
    for (int v = 0; v < 3; ++v) U[v] = ln->q[3 * s + v] * inv;
    lo_primitive(1, U, &ln->gas, W);
}

/* Stencil::ghost (:117-122): the state behind a wall next to an end cell of state W. */
static void ghost(const lo_line* ln, const double* W, int left, double* out) {
    const int wall = ln->walls[left ? 0 : 1];
    if (wall == LO_WALL_REFLECTIVE) {
        out[0] = W[0];
        out[1] = -W[1];
        out[2] = W[2];
    } else if (wall == LO_WALL_INFLOW) {
        memcpy(out, ln->inflow[left ? 0 : 1], sizeof(double) * 3);
    } else {
        memcpy(out, W, sizeof(double) * 3);
    }
}
/* Stencil::ghost_face (:124-128): the ghost's face state: the mirror of the end cell's face state at a reflective wall,
 * else the ghost's own state. */
static void ghost_face(const lo_line* ln, const double* Wf, const double* W, int left, double* out) {
    if (ln->walls[left ? 0 : 1] == LO_WALL_REFLECTIVE) {
        out[0] = Wf[0];
        out[1] = -Wf[1];
        out[2] = Wf[2];
    } else {
        ghost(ln, W, left, out);
    }
}

/* The slot k steps from s, or -1 beyond a wall (Line::slot). */
static int slot_at(const lo_line* ln, int s, int k) {
    const int t = s + k;
    if (ln->periodic) return ((t % ln->n) + ln->n) % ln->n;
    return t >= 0 && t < ln->n ? t : -1;
}

/* Stencil::load<R> (:132-156) with R = 2: cells s - 2 .. s + 2 (ghosts behind walls: the state of ghost() next to the end
 * cell, the mirrored centroid) and the generator distances between them. */
static void load(const lo_line* ln, int s, cell1 cell[5], double gap[4]) {
    int slot[5];
    for (int k = 0; k < 5; ++k) {
        slot[k] = slot_at(ln, s, k - 2);
        memset(&cell[k], 0, sizeof(cell1));
        cell[k].real = 1;
        if (slot[k] >= 0) {
            primitive_of(ln, slot[k], cell[k].W);
            cell[k].c = ln->centroid[slot[k]];
            cell[k].V = ln->volume[slot[k]];
        }
    }
    for (int k = 0; k < 5; ++k) {
        if (slot[k] >= 0) continue;
        cell[k].real = 0;
        const int end = k < 2 ? k + 1 : k - 1;
        if (slot[end] < 0) continue;
        ghost(ln, cell[end].W, k < 2, cell[k].W);
        cell[k].c = -cell[end].c;
    }
    for (int k = 0; k < 4; ++k) {
        const int a = slot[k], b = slot[k + 1];
        /* length(a) = gap after slot a; length(-1) = the gap over the left end */
        gap[k] = a >= 0 ? ln->gap[a + 1] * ln->step : b >= 0 ? ln->gap[0] * ln->step : 0.0;
    }
}

/* Stencil::gradient (:183-207): the limited slope of variable v of cell[0] between cell[-1] and cell[1]. */
static double gradient(const lo_line* ln, const cell1* cell, double gapL, double gapR, int v) {
    const cell1* me = cell;
    const double dL = -gapL + cell[-1].c - me->c, dR = gapR + cell[1].c - me->c;
    const double Wi = me->W[v], left = cell[-1].W[v], right = cell[1].W[v];
    if (ln->limiter == LO_LIMITER_MINMOD || ln->limiter == LO_LIMITER_VAN_LEER) {
        const double sL = (left - Wi) / dL, sR = (right - Wi) / dR;
        if (!(sL * sR > 0)) return 0.0;
        if (ln->limiter == LO_LIMITER_VAN_LEER) return 2 * sL * sR / (sL + sR);
        return fabs(sL) < fabs(sR) ? sL : sR;
    }
    double g = ((right - Wi) - (left - Wi)) / (dR - dL);
    if (ln->limiter == LO_LIMITER_NONE) return g;
    const double r[2] = {-0.5 * gapL - me->c, 0.5 * gapR - me->c};
    const double lo = fmin(left, right), hi = fmax(left, right);
    for (int f = 0; f < 2; ++f) {
        const double dp = g * r[f];
        if (dp > 0 && Wi + dp > hi)
            g = g * (hi > Wi ? (hi - Wi) / dp : 0.0);
        else if (dp < 0 && Wi + dp < lo)
            g = g * (lo < Wi ? (lo - Wi) / dp : 0.0);
    }
    return g;
}

/* Kernel::face_state (:492-506): half a step on, then to the face at offset r; the cell's own W if rho or P would not
 * stay positive. */
static void face_state(const lo_line* ln, const double* W, const double* g, double r, double dt, double* out) {
    if (ln->order == 0) {
        memcpy(out, W, sizeof(double) * 3);
        return;
    }
    lo_half_step(1, W, g, dt, &ln->gas, out);
    for (int v = 0; v < 3; ++v) out[v] += g[v] * r;
    if (out[0] > 0 && out[2] > 0) return;
    memcpy(out, W, sizeof(double) * 3);
}

static void flux(const lo_line* ln, const double* L, const double* R, double* F) {
    const double n[1] = {1.0}, w[1] = {0.0};
    if (ln->riemann == 1)
        lo_hll_flux(1, L, R, n, w, &ln->gas, F);
    else
        lo_hllc_flux(1, L, R, n, w, &ln->gas, F);
}

/* Kernel::body, static (:555-660): per slot the gradients of s - 1, s, s + 1, the fluxes through its two faces, the
 * update into the next state. */
static void step_slot(lo_line* ln, int s, double dt) {
    cell1 cell[5];
    double gap[4], grad[5][3];
    load(ln, s, cell, gap);
    for (int k = 1; k <= 3; ++k) {
        for (int v = 0; v < 3; ++v) grad[k][v] = 0;
        if (!cell[k].real || ln->order != 1) continue;
        for (int v = 0; v < 3; ++v) grad[k][v] = gradient(ln, cell + k, gap[k - 1], gap[k], v);
    }
    double F[2][3];
    for (int f = 0; f < 2; ++f) {
        const int a = 1 + f, b = 2 + f;
        double L[3] = {0, 0, 0}, R[3] = {0, 0, 0};
        if (cell[a].real) face_state(ln, cell[a].W, grad[a], 0.5 * gap[a] - cell[a].c, dt, L);
        if (cell[b].real) face_state(ln, cell[b].W, grad[b], -0.5 * gap[a] - cell[b].c, dt, R);
        if (!cell[a].real) ghost_face(ln, R, cell[b].W, 1, L);
        if (!cell[b].real) ghost_face(ln, L, cell[a].W, 0, R);
        flux(ln, L, R, F[f]);
    }
    for (int v = 0; v < 3; ++v) ln->next[3 * s + v] = ln->q[3 * s + v] - dt * (F[1][v] - F[0][v]);
}

void lo_line_step(lo_line* ln, double dt) {
#pragma omp parallel for schedule(static)
    for (int s = 0; s < ln->n; ++s) step_slot(ln, s, dt);
    double* t = ln->q;
    ln->q = ln->next;
    ln->next = t;
}

/* time_step (:332-384), static: LUNA's rule (rule 1) courant V / (|v| + c); AREPO's (rule 0) courant times the smallest of
 * r / (c + |v|) and, per side, (distance + r) / vsig with vsig = c_i + c_j - (v_j - v_i) side > 0 (a ghost behind a wall). */
double lo_line_time_step(const lo_line* ln, double courant, int rule) {
    double smallest = INFINITY;
    for (int s = 0; s < ln->n; ++s) {
        double Wi[3];
        primitive_of(ln, s, Wi);
        const double ci = sqrt(ln->gas.gamma * Wi[2] / Wi[0]);
        const double volume = ln->volume[s], vi = fabs(Wi[1]);
        if (rule == 1) {
            smallest = fmin(smallest, courant * volume / (vi + ci));
            continue;
        }
        const double r = 0.5 * volume;
        double step = r / (ci + vi);
        for (int side = -1; side <= 1; side += 2) {
            const int t = slot_at(ln, s, side);
            double Wj[3];
            if (t >= 0)
                primitive_of(ln, t, Wj);
            else
                ghost(ln, Wi, side < 0, Wj);
            const double dist = (side < 0 ? ln->gap[s] : ln->gap[s + 1]) * ln->step;
            const double vsig = ci + sqrt(ln->gas.gamma * Wj[2] / Wj[0]) - (Wj[1] - Wi[1]) * side;
            if (vsig > 0) step = fmin(step, (dist + r) / vsig);
        }
        smallest = fmin(smallest, courant * step);
    }
    return smallest;
}
