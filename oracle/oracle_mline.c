/* CPU oracle of luna-cpp's 1D solver on a MOVING line, FiniteVolume<1> with Motion::moving
 * (src/hydro/finite_volume_1d.hpp): TEST INFRASTRUCTURE ONLY — the checker of the CUDA moving line (luna_mline_* in
 * include/luna_b200.h). Parity unpinned by reference-held numbers: the reference's moving-line tests are properties
 * (uniform states, conservation, the wall budget, Sod within LUNA's bounds, no crossings, mirrors), which the GPU tests
 * check on both this restatement's and the GPU's runs.
 *
 * The line as the reference keeps it: Q and the positions x per cell (cell order; cells supplied by a wall are
 * appended), and per slot (the generators sorted along the line) the grid key and the cell. voronoi-cpp's 1D mesh is
 * absent; its parts used here are restated: keys on a grid of step = length 2^-52 (period 2^52 steps: "2^30 grid steps are
 * too few in 1D", research_notes/stage1_1d_2026-11-04.md:35, :64-78), a point snaps to
 * the nearest grid point (ties to even), slots sort by (key, cell), a wall's ghost generator is the end generator's
 * mirror, and a cell inserted next to a wall takes the overlapped fraction of its old neighbour's Q. Arithmetic in
 * IEEE double in the reference's operation order (fma where it calls Kokkos::fma), compiled without contraction.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "luna_oracle.h"

typedef struct {
    double W[3], c, V;
    int real;
} mcell;

struct lo_mline {
    int n, cap, periodic, order, limiter, riemann, regularise;
    int walls[2];
    double inflow[2][3];
    double length, step;
    int64_t period;
    lo_gas gas;
    double *q, *next;          /* [cap][3], cell order */
    double *x, *x_next;        /* [cap], cell order */
    int64_t *keys, *keys_next; /* [cap], slot order */
    int* cell;                 /* [cap]: slot -> cell */
    double *gap, *volume, *centroid; /* [cap + 1], [cap], [cap]: slot order (gap[s + 1]: after slot s) */
    int supply[2], watching, looked, wants, until_look;
    double spacing;
    long long added, sorts, updates;
};

static const double shaping_speed = 0.5; /* FiniteVolume<1>::cell_shaping_speed (finite_volume_1d.hpp:26) */

static double sound(const lo_mline* ml, const double* W) { return sqrt(ml->gas.gamma * W[2] / W[0]); }

/* sorted_mesh::snap: the grid point nearest y (periodic: modulo the period). */
static int64_t snap(const lo_mline* ml, double y) {
    int64_t k = (int64_t)nearbyint(y / ml->step);
    if (ml->periodic) {
        k %= ml->period;
        if (k < 0) k += ml->period;
    } else {
        if (k < 0) k = 0;
        if (k > ml->period) k = ml->period;
    }
    return k;
}
/* sorted_mesh::before: the slot order, by key, then by cell. */
static int before(int64_t ka, int ia, int64_t kb, int ib) { return ka < kb || (ka == kb && ia < ib); }

/* Line::gap, volume, centroid (finite_volume_1d.hpp load_inner :163-176): between neighbours the key difference (a
 * periodic line's seam wraps); at a wall twice the end generator's distance to it. */
static void geometry(lo_mline* ml) {
    const int n = ml->n;
    for (int s = 0; s + 1 < n; ++s) {
        int64_t d = ml->keys[s + 1] - ml->keys[s];
        if (d < 0 && ml->periodic) d += ml->period;
        ml->gap[s + 1] = (double)d;
    }
    if (ml->periodic) {
        int64_t d = ml->keys[0] - ml->keys[n - 1];
        if (d < 0) d += ml->period;
        ml->gap[0] = ml->gap[n] = (double)d;
    } else {
        ml->gap[0] = (double)(2 * ml->keys[0]);
        ml->gap[n] = (double)(2 * (ml->period - ml->keys[n - 1]));
    }
    for (int s = 0; s < n; ++s) {
        ml->volume[s] = (ml->gap[s] + ml->gap[s + 1]) * (0.5 * ml->step);
        ml->centroid[s] = (ml->gap[s + 1] - ml->gap[s]) * (0.25 * ml->step);
    }
}

static const lo_mline* sort_line;
static int by_key(const void* a, const void* b) {
    const int sa = *(const int*)a, sb = *(const int*)b;
    const int64_t ka = sort_line->keys[sa], kb = sort_line->keys[sb];
    const int ia = sort_line->cell[sa], ib = sort_line->cell[sb];
    if (before(ka, ia, kb, ib)) return -1;
    if (before(kb, ib, ka, ia)) return 1;
    return 0;
}
/* mesh_->order(): the slots sorted by (key, cell). */
static void sort_slots(lo_mline* ml) {
    int* perm = (int*)malloc(sizeof(int) * ml->n);
    for (int s = 0; s < ml->n; ++s) perm[s] = s;
    sort_line = ml;
    qsort(perm, ml->n, sizeof(int), by_key);
    int64_t* k = (int64_t*)malloc(sizeof(int64_t) * ml->n);
    int* c = (int*)malloc(sizeof(int) * ml->n);
    for (int s = 0; s < ml->n; ++s) {
        k[s] = ml->keys[perm[s]];
        c[s] = ml->cell[perm[s]];
    }
    memcpy(ml->keys, k, sizeof(int64_t) * ml->n);
    memcpy(ml->cell, c, sizeof(int) * ml->n);
    free(k);
    free(c);
    free(perm);
}

static void reserve(lo_mline* ml, int count) {
    if (count <= ml->cap) return;
    int cap = ml->cap + ml->cap / 4;
    if (cap < count) cap = count;
    ml->q = (double*)realloc(ml->q, sizeof(double) * 3 * cap);
    ml->next = (double*)realloc(ml->next, sizeof(double) * 3 * cap);
    ml->x = (double*)realloc(ml->x, sizeof(double) * cap);
    ml->x_next = (double*)realloc(ml->x_next, sizeof(double) * cap);
    ml->keys = (int64_t*)realloc(ml->keys, sizeof(int64_t) * cap);
    ml->keys_next = (int64_t*)realloc(ml->keys_next, sizeof(int64_t) * cap);
    ml->cell = (int*)realloc(ml->cell, sizeof(int) * cap);
    ml->gap = (double*)realloc(ml->gap, sizeof(double) * (cap + 1));
    ml->volume = (double*)realloc(ml->volume, sizeof(double) * cap);
    ml->centroid = (double*)realloc(ml->centroid, sizeof(double) * cap);
    ml->cap = cap;
}

/* set_inflow_spacing (:61-66): a wall supplies cells on a moving, non-periodic line unless it reflects. */
void lo_mline_set_inflow_spacing(lo_mline* ml, double spacing) {
    for (int a = 0; a < 2; ++a) ml->supply[a] = !ml->periodic && ml->walls[a] != LO_WALL_REFLECTIVE && spacing > 0;
    ml->spacing = spacing;
}

lo_mline* lo_mline_create(int n, const double* positions, double length, int periodic, const int* walls, const double* inflow,
                          const lo_gas* gas, int order, int limiter, int riemann, int regularise) {
    lo_mline* ml = (lo_mline*)calloc(1, sizeof(lo_mline));
    ml->periodic = periodic;
    ml->order = order;
    ml->limiter = limiter;
    ml->riemann = riemann;
    ml->regularise = regularise;
    ml->walls[0] = walls ? walls[0] : LO_WALL_OUTFLOW;
    ml->walls[1] = walls ? walls[1] : LO_WALL_OUTFLOW;
    if (inflow) memcpy(ml->inflow, inflow, sizeof(ml->inflow));
    ml->length = length;
    ml->step = ldexp(length, -52);
    ml->period = (int64_t)1 << 52;
    ml->gas = *gas;
    reserve(ml, n);
    ml->n = n;
    memset(ml->q, 0, sizeof(double) * 3 * n);
    for (int i = 0; i < n; ++i) {
        ml->x[i] = positions[i];
        ml->cell[i] = i;
        ml->keys[i] = snap(ml, positions[i]);
    }
    sort_slots(ml);
    geometry(ml);
    lo_mline_set_inflow_spacing(ml, length / n);
    return ml;
}

void lo_mline_destroy(lo_mline* ml) {
    if (!ml) return;
    free(ml->q);
    free(ml->next);
    free(ml->x);
    free(ml->x_next);
    free(ml->keys);
    free(ml->keys_next);
    free(ml->cell);
    free(ml->gap);
    free(ml->volume);
    free(ml->centroid);
    free(ml);
}

int lo_mline_cells(const lo_mline* ml) { return ml->n; }
double* lo_mline_state(lo_mline* ml) { return ml->q; }
double* lo_mline_positions(lo_mline* ml) { return ml->x; }
void lo_mline_stats(const lo_mline* ml, long long* added, long long* sorts, long long* updates) {
    *added = ml->added;
    *sorts = ml->sorts;
    *updates = ml->updates;
}
/* Per cell (cell order): the generator's grid position, the cell's length and its centroid's offset. */
void lo_mline_geometry(const lo_mline* ml, double* generator, double* volume, double* centroid) {
    for (int s = 0; s < ml->n; ++s) {
        const int i = ml->cell[s];
        generator[i] = (double)ml->keys[s] * ml->step;
        volume[i] = ml->volume[s];
        centroid[i] = ml->centroid[s];
    }
}

static void primitive_at(const lo_mline* ml, int s, double* W) {
    const int i = ml->cell[s];
    const double inv = 1.0 / ml->volume[s];
    double U[3];
    for (int v = 0; v < 3; ++v) U[v] = ml->q[3 * i + v] * inv;
    lo_primitive(1, U, &ml->gas, W);
}
static void ghost(const lo_mline* ml, const double* W, int left, double* out) {
    const int wall = ml->walls[left ? 0 : 1];
    if (wall == LO_WALL_REFLECTIVE) {
        out[0] = W[0];
        out[1] = -W[1];
        out[2] = W[2];
    } else if (wall == LO_WALL_INFLOW) {
        memcpy(out, ml->inflow[left ? 0 : 1], sizeof(double) * 3);
    } else {
        memcpy(out, W, sizeof(double) * 3);
    }
}
static void ghost_face(const lo_mline* ml, const double* Wf, const double* W, int left, double* out) {
    if (ml->walls[left ? 0 : 1] == LO_WALL_REFLECTIVE) {
        out[0] = Wf[0];
        out[1] = -Wf[1];
        out[2] = Wf[2];
    } else {
        ghost(ml, W, left, out);
    }
}
static int slot_at(const lo_mline* ml, int s, int k) {
    const int t = s + k;
    if (ml->periodic) return ((t % ml->n) + ml->n) % ml->n;
    return t >= 0 && t < ml->n ? t : -1;
}
/* Stencil::load<R> (:132-156): cells s - R .. s + R into cell[], ghosts behind walls, the generator distances. */
static void load(const lo_mline* ml, int s, int R, mcell* cell, double* gap) {
    const int M = 2 * R + 1;
    int slot[5];
    for (int k = 0; k < M; ++k) {
        slot[k] = slot_at(ml, s, k - R);
        memset(&cell[k], 0, sizeof(mcell));
        cell[k].real = 1;
        if (slot[k] >= 0) {
            primitive_at(ml, slot[k], cell[k].W);
            cell[k].c = ml->centroid[slot[k]];
            cell[k].V = ml->volume[slot[k]];
        }
    }
    for (int k = 0; k < M; ++k) {
        if (slot[k] >= 0) continue;
        cell[k].real = 0;
        const int end = k < R ? k + 1 : k - 1;
        if (slot[end] < 0) continue;
        ghost(ml, cell[end].W, k < R, cell[k].W);
        cell[k].c = -cell[end].c;
    }
    for (int k = 0; k < M - 1; ++k) {
        const int a = slot[k], b = slot[k + 1];
        gap[k] = a >= 0 ? ml->gap[a + 1] * ml->step : b >= 0 ? ml->gap[0] * ml->step : 0.0;
    }
}
/* Stencil::gradient (:183-207). */
static double gradient(const lo_mline* ml, const mcell* cell, double gapL, double gapR, int v) {
    const mcell* me = cell;
    const double dL = -gapL + cell[-1].c - me->c, dR = gapR + cell[1].c - me->c;
    const double Wi = me->W[v], left = cell[-1].W[v], right = cell[1].W[v];
    if (ml->limiter == LO_LIMITER_MINMOD || ml->limiter == LO_LIMITER_VAN_LEER) {
        const double sL = (left - Wi) / dL, sR = (right - Wi) / dR;
        if (!(sL * sR > 0)) return 0.0;
        if (ml->limiter == LO_LIMITER_VAN_LEER) return 2 * sL * sR / (sL + sR);
        return fabs(sL) < fabs(sR) ? sL : sR;
    }
    double g = ((right - Wi) - (left - Wi)) / (dR - dL);
    if (ml->limiter == LO_LIMITER_NONE) return g;
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
/* Stencil::drift (:301-316): AREPO-ng's regularisation, the point velocity's difference from the fluid's. */
static double drift(const lo_mline* ml, const double* W, double g, double c, double volume) {
    const double r = 0.5 * volume;
    if (!ml->regularise || fabs(c) <= 0.5 * r) return 0.0;
    double offset = c;
    const double dgrad = fabs(g);
    if (dgrad > 0) {
        const double tmp = 3 * r + W[0] / dgrad;
        const double x = (tmp - sqrt(tmp * tmp - 8 * r * r)) / 4;
        if (x < 0.25 * r) offset += x / dgrad * g;
    }
    const double d = fabs(offset);
    if (d <= 0.75 * r) return 0.0;
    const double fraction = d > r ? shaping_speed : shaping_speed * (d - 0.75 * r) / (0.25 * r);
    return offset * (fraction * sound(ml, W) / d);
}
/* Stencil::point_velocity (:320-329): drift(), plus, for a generator beyond 0.75 r of its centroid, up to the fluid's
 * velocity at the generator, linear between the centroids of this cell and its neighbour there (luna-cpp #25). */
static double point_velocity(const lo_mline* ml, const mcell* cell, double gapL, double gapR, double g_rho, double volume) {
    const mcell* me = cell;
    const double r = 0.5 * volume, d = fabs(me->c), weight = fmin(1.0, (d - 0.75 * r) / (0.25 * r));
    const double drifting = drift(ml, me->W, g_rho, me->c, volume);
    if (!(weight > 0)) return drifting;
    const int side = me->c < 0 ? 1 : -1;
    const double between = side > 0 ? gapR + cell[1].c - me->c : gapL + me->c - cell[-1].c;
    return drifting + weight * (cell[side].W[1] - me->W[1]) * (d / between);
}
/* Stencil::room_at, wants_cell (:88-98): 0..2 cells an end slot asks its wall for. */
static int wants_cell(const lo_mline* ml, int s) {
    int wants = 0;
    const double spacing = ml->spacing;
    if (s == 0 && ml->supply[0]) {
        const int64_t d = ml->keys[0];
        wants += ml->volume[0] > 2 * spacing && (double)d * ml->step >= 1.5 * spacing;
    }
    if (s == ml->n - 1 && ml->supply[1]) {
        const int64_t d = ml->period - ml->keys[s];
        wants += ml->volume[s] > 2 * spacing && (double)d * ml->step >= 1.5 * spacing;
    }
    return wants;
}

static void flux(const lo_mline* ml, const double* L, const double* R, double w, double* F) {
    const double n[1] = {1.0}, wv[1] = {w};
    if (ml->riemann == 1)
        lo_hll_flux(1, L, R, n, wv, &ml->gas, F);
    else
        lo_hllc_flux(1, L, R, n, wv, &ml->gas, F);
}
/* Kernel::extrapolated (:507-523): W + g r, a whole step on (MUSCL-Hancock) when second; W if rho or P would not stay
 * positive. */
static void extrapolated(const lo_mline* ml, const double* W, const double* g, double r, int second, double dt, double* out) {
    if (ml->order == 0) {
        memcpy(out, W, sizeof(double) * 3);
        return;
    }
    if (second)
        lo_half_step(1, W, g, 2 * dt, &ml->gas, out);
    else
        memcpy(out, W, sizeof(double) * 3);
    for (int v = 0; v < 3; ++v) out[v] += g[v] * r;
    if (out[0] > 0 && out[2] > 0) return;
    memcpy(out, W, sizeof(double) * 3);
}
/* Kernel::moved (:546-550): where a point at x0 ends up after dt. */
static double moved(const lo_mline* ml, double x0, double velocity, double dt) {
    const double side = ml->length;
    const double y = fma(dt, velocity, x0);
    return ml->periodic ? y - side * floor(y / side) : fmin(fmax(y, 0.0), side);
}

/* Kernel::body, moving (:555-660) for slot s: gradients and point velocities of s - 1, s, s + 1, their new keys and moves
 * in grid steps, the fluxes through s's two faces on the meshes of t^n and t^n+1 (their mean at order 1), Q and x after
 * the step, the new key of s, and for the fused step the next dt of LUNA's rule and whether s and s + 1 are out of order. */
static void body(lo_mline* ml, int s, double dt, double courant, double* smallest, int* descents) {
    mcell cell[5];
    double gap[4], grad[5][3], point[5] = {0, 0, 0, 0, 0}, moves[5] = {0, 0, 0, 0, 0};
    int64_t key[5] = {0, 0, 0, 0, 0};
    load(ml, s, 2, cell, gap);
    for (int k = 1; k <= 3; ++k) {
        for (int v = 0; v < 3; ++v) grad[k][v] = 0;
        if (!cell[k].real) continue;
        if (ml->order == 1)
            for (int v = 0; v < 3; ++v) grad[k][v] = gradient(ml, cell + k, gap[k - 1], gap[k], v);
        point[k] = cell[k].W[1] + point_velocity(ml, cell + k, gap[k - 1], gap[k], grad[k][0], 0.5 * (gap[k - 1] + gap[k]));
    }
    for (int k = 1; k <= 3; ++k) {
        if (!cell[k].real) continue;
        const int t = slot_at(ml, s, k - 2);
        key[k] = snap(ml, moved(ml, ml->x[ml->cell[t]], point[k], dt));
        int64_t d = key[k] - ml->keys[t];
        if (ml->periodic) d = d > ml->period / 2 ? d - ml->period : d < -ml->period / 2 ? d + ml->period : d;
        moves[k] = (double)d;
    }
    double F[2][3];
    for (int f = 0; f < 2; ++f) {
        const int a = 1 + f, b = 2 + f;
        const int inside = cell[a].real && cell[b].real;
        const double travel = inside ? 0.5 * (moves[a] + moves[b]) * ml->step : 0.0;
        const double w = travel / dt;
        const double ra = 0.5 * gap[a] - cell[a].c, rb = -0.5 * gap[a] - cell[b].c;
        double pass[2][3];
        const int passes = ml->order == 1 ? 2 : 1;
        for (int second = 0; second < passes; ++second) {
            double L[3] = {0, 0, 0}, R[3] = {0, 0, 0};
            if (cell[a].real) extrapolated(ml, cell[a].W, grad[a], ra + second * travel, second, dt, L);
            if (cell[b].real) extrapolated(ml, cell[b].W, grad[b], rb + second * travel, second, dt, R);
            if (!cell[a].real) ghost_face(ml, R, cell[b].W, 1, L);
            if (!cell[b].real) ghost_face(ml, L, cell[a].W, 0, R);
            flux(ml, L, R, w, pass[second]);
        }
        for (int v = 0; v < 3; ++v) F[f][v] = ml->order == 1 ? 0.5 * (pass[0][v] + pass[1][v]) : pass[0][v];
    }
    const int i = ml->cell[s];
    double U[3];
    for (int v = 0; v < 3; ++v) {
        U[v] = ml->q[3 * i + v] - dt * (F[1][v] - F[0][v]);
        ml->next[3 * i + v] = U[v];
    }
    ml->x_next[i] = moved(ml, ml->x[i], point[2], dt);
    ml->keys_next[s] = key[2];
    double left, right;
    if (cell[1].real) {
        const int64_t d = key[2] - key[1];
        left = (double)(d < 0 && ml->periodic ? d + ml->period : d);
    } else {
        left = (double)(2 * key[2]);
    }
    if (cell[3].real) {
        const int t = slot_at(ml, s, 1);
        const int64_t d = key[3] - key[2];
        right = (double)(d < 0 && ml->periodic ? d + ml->period : d);
        *descents += !before(key[2], i, key[3], ml->cell[t]);
    } else {
        right = (double)(2 * (ml->period - key[2]));
    }
    if (smallest) {
        const double volume = (left + right) * (0.5 * ml->step), inv = 1.0 / volume;
        double Un[3], Wn[3];
        for (int v = 0; v < 3; ++v) Un[v] = U[v] * inv;
        lo_primitive(1, Un, &ml->gas, Wn);
        const double relative = fabs(point[2] - cell[2].W[1]);
        *smallest = fmin(*smallest, courant * volume / (relative + sound(ml, Wn)));
    }
}

/* due() (:957-964): look at the end cells after this step: while gas enters as the kernels asked, else every 64 steps. */
static int due(lo_mline* ml) {
    if (!ml->supply[0] && !ml->supply[1]) return 0;
    if (ml->watching) return !ml->looked || ml->wants > 0;
    if (--ml->until_look > 0) return 0;
    ml->until_look = 64;
    return 1;
}

/* supply_cells (:421-470): the cells the walls have room for, one at each wall at most, spacing from the end generator;
 * each takes the overlapped fraction of its old neighbour's Q. Returns the cells added. */
int lo_mline_supply_cells(lo_mline* ml) {
    const int last = ml->n - 1;
    double W0[3], Wl[3];
    primitive_at(ml, 0, W0);
    primitive_at(ml, last, Wl);
    const double end_left = (double)ml->keys[0] * ml->step, end_right = (double)(ml->period - ml->keys[last]) * ml->step;
    const int want_left = wants_cell(ml, 0), want_right = wants_cell(ml, last);
    const int entering = (ml->supply[0] && W0[1] > 0) || (ml->supply[1] && Wl[1] < 0);
    ml->watching = ml->watching || entering;
    double p[2];
    int side[2], requests = 0;
    if (want_left > 0) side[requests] = 0, p[requests++] = end_left - ml->spacing;
    if (want_right > 0) side[requests] = 1, p[requests++] = ml->length - (end_right - ml->spacing);
    if (requests == 0) return 0;
    const int n = ml->n;
    reserve(ml, n + requests);
    const int64_t P = ml->period;
    int done = 0, left_added = 0;
    int64_t new_key[2];
    for (int r = 0; r < requests; ++r) {
        const int64_t kp = snap(ml, p[r]);
        const int i = n + done;
        double fraction;
        int old;
        if (side[r] == 0) {
            const int64_t k0 = ml->keys[0], k1 = n > 1 ? ml->keys[1] : P;
            if (!(kp > 0 && kp < k0)) continue;
            old = ml->cell[0];
            fraction = ((double)(kp + k0) * (0.5 * ml->step)) / ((double)(k0 + k1) * (0.5 * ml->step));
            left_added = 1;
        } else {
            const int64_t kl = ml->keys[last], kb = n > 1 ? ml->keys[last - 1] : 0;
            if (!(kp > kl && kp < P)) continue;
            old = ml->cell[last];
            fraction = ((double)(2 * P - kl - kp) * (0.5 * ml->step)) / ((double)(2 * P - kb - kl) * (0.5 * ml->step));
        }
        for (int v = 0; v < 3; ++v) {
            const double part = fraction * ml->q[3 * old + v];
            ml->q[3 * old + v] -= part;
            ml->q[3 * i + v] = part;
        }
        ml->x[i] = p[r];
        new_key[side[r]] = kp;
        ++done;
    }
    /* the new slots: a left cell first, a right cell last */
    if (left_added) {
        memmove(ml->keys + 1, ml->keys, sizeof(int64_t) * n);
        memmove(ml->cell + 1, ml->cell, sizeof(int) * n);
        ml->keys[0] = new_key[0];
        ml->cell[0] = n;
    }
    if (done > left_added) {
        ml->keys[n + left_added] = new_key[1];
        ml->cell[n + left_added] = n + left_added;
    }
    ml->n = n + done;
    ml->added += done;
    geometry(ml);
    return done;
}

/* After a step's kernel: Q and x swap, the keys move, the slots re-sort when out of order, cells come from the walls. */
static int finish(lo_mline* ml, int descents) {
    double* t = ml->q;
    ml->q = ml->next;
    ml->next = t;
    t = ml->x;
    ml->x = ml->x_next;
    ml->x_next = t;
    int64_t* k = ml->keys;
    ml->keys = ml->keys_next;
    ml->keys_next = k;
    ml->updates += 1;
    int again = 0;
    if (descents != (ml->periodic ? 1 : 0)) {
        sort_slots(ml);
        ml->sorts += 1;
        again = 1;
    }
    geometry(ml);
    return again;
}

/* step(dt) (:389-410), moving. */
void lo_mline_step(lo_mline* ml, double dt) {
    int descents = 0;
    for (int s = 0; s < ml->n; ++s) body(ml, s, dt, 0.0, NULL, &descents);
    finish(ml, descents);
    if (due(ml)) lo_mline_supply_cells(ml);
    ml->looked = 0;
}

/* time_step(courant, rule) (:332-384), moving: the point velocity's |w - v| in place of |v|; with cells supplied, the
 * end slots' wishes too (while gas enters). */
double lo_mline_time_step(lo_mline* ml, double courant, int rule) {
    double smallest = INFINITY;
    int wants = 0;
    for (int s = 0; s < ml->n; ++s) {
        mcell cell[3];
        double gap[2] = {0, 0};
        load(ml, s, 1, cell, gap);
        const double* Wi = cell[1].W;
        const double ci = sound(ml, Wi);
        const double volume = ml->volume[s];
        const double g = ml->order == 1 ? gradient(ml, cell + 1, gap[0], gap[1], 0) : 0.0;
        const double vi = fabs(point_velocity(ml, cell + 1, gap[0], gap[1], g, volume));
        if (ml->watching) wants += wants_cell(ml, s);
        if (rule == 1) {
            smallest = fmin(smallest, courant * volume / (vi + ci));
            continue;
        }
        const double r = 0.5 * volume;
        double step = r / (ci + vi);
        for (int side = -1; side <= 1; side += 2) {
            const int t = slot_at(ml, s, side);
            double Wj[3];
            if (t >= 0)
                primitive_at(ml, t, Wj);
            else
                ghost(ml, Wi, side < 0, Wj);
            const double dist = (side < 0 ? ml->gap[s] : ml->gap[s + 1]) * ml->step;
            const double vsig = ci + sound(ml, Wj) - (Wj[1] - Wi[1]) * side;
            if (vsig > 0) step = fmin(step, (dist + r) / vsig);
        }
        smallest = fmin(smallest, courant * step);
    }
    if (ml->watching) {
        ml->wants = wants;
        ml->looked = 1;
    }
    return smallest;
}

/* step_and_time_step(dt, courant) (:412-418, run_fused :679-711): the step and the next dt of LUNA's rule in one pass;
 * when the slots re-sorted or cells were added, time_step(courant, luna) afresh. */
double lo_mline_step_and_time_step(lo_mline* ml, double dt, double courant) {
    double smallest = INFINITY;
    int descents = 0, wants = 0;
    for (int s = 0; s < ml->n; ++s) {
        body(ml, s, dt, courant, &smallest, &descents);
        if (ml->watching && (s == 0 || s == ml->n - 1)) wants += wants_cell(ml, s);
    }
    int again = finish(ml, descents);
    ml->wants = wants;
    ml->looked = ml->watching;
    if (due(ml)) again = lo_mline_supply_cells(ml) > 0 || again;
    ml->looked = 0;
    if (again) return lo_mline_time_step(ml, courant, 1);
    return smallest;
}
