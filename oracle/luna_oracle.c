/* CPU oracle of luna-cpp's hydro step: TEST INFRASTRUCTURE ONLY (the checker of the CUDA path and the timed CPU
 * baseline; nothing in the product links it). A plain C restatement of the reference's algorithm, in the reference's
 * operation order, compiled without multiply-add contraction (-ffp-contract=off). D = 2 or 3 at run time; states have
 * V = D + 2 entries, the least-squares fit U = D + 1 unknowns. Reference paths are relative to the luna-cpp tree. */

#define _GNU_SOURCE
#include "luna_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define VMAX 5
#define UMAX 4

/* ---------------------------------------------------------------------------------------------------------------------
 * euler.hpp
 * ------------------------------------------------------------------------------------------------------------------- */

/* Gas (euler.hpp:82-101): 1/(gamma-1) cached in double and in float, each rounded in its own type. */
void lo_gas_init(lo_gas* gas, double gamma) {
    gas->gamma = gamma;
    gas->smallr = 1e-10;
    gas->smallc = 1e-10;
    gas->inverse_gm1 = 1.0 / (gamma - 1.0);
    gas->inverse_gm1_float = 1.0f / ((float)gamma - 1.0f);
}

/* dot() written out left to right (euler.hpp:66-71). */
static double dotd(int D, const double* a, const double* b) {
    double s = a[0] * b[0];
    for (int k = 1; k < D; ++k) s = s + a[k] * b[k];
    return s;
}
static float dotf(int D, const float* a, const float* b) {
    float s = a[0] * b[0];
    for (int k = 1; k < D; ++k) s = s + a[k] * b[k];
    return s;
}

/* primitive(): U -> W with the RAMSES floors (euler.hpp:104-113). */
void lo_primitive(int D, const double* U, const lo_gas* gas, double* W) {
    const double rho = fmax(U[0], gas->smallr);
    const double inv_rho = 1.0 / rho;
    double v[3];
    for (int k = 0; k < D; ++k) v[k] = U[1 + k] * inv_rho;
    const double smalle = gas->smallc * gas->smallc / gas->gamma / (gas->gamma - 1.0);
    const double kinetic = 0.5 * rho * dotd(D, v, v);
    const double e = fmax(U[D + 1] - kinetic, smalle * rho);
    W[0] = rho;
    for (int k = 0; k < D; ++k) W[1 + k] = v[k];
    W[D + 1] = (gas->gamma - 1.0) * e;
}

/* conserved(): W -> U without floors (euler.hpp:165-172). */
void lo_conserved(int D, const double* W, const lo_gas* gas, double* U) {
    const double rho = W[0];
    const double kinetic = 0.5 * rho * dotd(D, W + 1, W + 1);
    U[0] = rho;
    for (int k = 0; k < D; ++k) U[1 + k] = rho * W[1 + k];
    U[D + 1] = W[D + 1] / (gas->gamma - 1.0) + kinetic;
}

/* half_step_rate(): sum_d A_d(W) dW/dx_d (euler.hpp:186-204); g is [V][D]. */
static void half_step_rate_d(int D, const double* W, const double* g, const lo_gas* gas, double* A) {
    const int P = D + 1;
    const double rho = W[0], inv_rho = 1.0 / W[0], rho_c2 = gas->gamma * W[P];
    for (int v = 0; v < D + 2; ++v) A[v] = 0;
    for (int d = 0; d < D; ++d) {
        const double vn = W[1 + d];
        A[0] += vn * g[0 * D + d] + rho * g[(1 + d) * D + d];
        for (int k = 0; k < D; ++k) {
            double row = vn * g[(1 + k) * D + d];
            if (k == d) row = row + inv_rho * g[P * D + d];
            A[1 + k] += row;
        }
        A[P] += rho_c2 * g[(1 + d) * D + d] + vn * g[P * D + d];
    }
}
static void half_step_rate_f(int D, const float* W, const float* g, const lo_gas* gas, float* A) {
    const int P = D + 1;
    const float rho = W[0], inv_rho = 1.0f / W[0], rho_c2 = (float)gas->gamma * W[P];
    for (int v = 0; v < D + 2; ++v) A[v] = 0;
    for (int d = 0; d < D; ++d) {
        const float vn = W[1 + d];
        A[0] += vn * g[0 * D + d] + rho * g[(1 + d) * D + d];
        for (int k = 0; k < D; ++k) {
            float row = vn * g[(1 + k) * D + d];
            if (k == d) row = row + inv_rho * g[P * D + d];
            A[1 + k] += row;
        }
        A[P] += rho_c2 * g[(1 + d) * D + d] + vn * g[P * D + d];
    }
}

/* half_step(): W - dt/2 A (euler.hpp:208-214). */
void lo_half_step(int D, const double* W, const double* g, double dt, const lo_gas* gas, double* out) {
    double A[VMAX];
    half_step_rate_d(D, W, g, gas, A);
    for (int v = 0; v < D + 2; ++v) out[v] = W[v] - 0.5 * dt * A[v];
}

/* detail::Side (euler.hpp:313-320) and side_with() (euler.hpp:324-336), in double and in float. */
typedef struct {
    double v[3], vn, c, E, F[VMAX], U[VMAX];
} side_d;
typedef struct {
    float v[3], vn, c, E, F[VMAX], U[VMAX];
} side_f;

static side_d side_with_d(int D, const double* W, const double* n, const double* w, const lo_gas* gas, double vn) {
    const int P = D + 1;
    side_d s;
    for (int k = 0; k < D; ++k) s.v[k] = W[1 + k] - w[k];
    s.vn = vn;
    s.c = 0;
    s.E = W[P] * gas->inverse_gm1 + W[0] * (0.5 * dotd(D, s.v, s.v));
    const double m = W[0] * s.vn;
    s.F[0] = m;
    for (int k = 0; k < D; ++k) s.F[1 + k] = m * s.v[k] + W[P] * n[k];
    s.F[P] = (s.E + W[P]) * s.vn;
    s.U[0] = W[0];
    for (int k = 0; k < D; ++k) s.U[1 + k] = W[0] * s.v[k];
    s.U[P] = s.E;
    return s;
}
static side_f side_with_f(int D, const float* W, const float* n, const lo_gas* gas, float vn) {
    const int P = D + 1;
    side_f s;
    for (int k = 0; k < D; ++k) s.v[k] = W[1 + k] - 0.0f;
    s.vn = vn;
    s.c = 0;
    s.E = W[P] * gas->inverse_gm1_float + W[0] * (0.5f * dotf(D, s.v, s.v));
    const float m = W[0] * s.vn;
    s.F[0] = m;
    for (int k = 0; k < D; ++k) s.F[1 + k] = m * s.v[k] + W[P] * n[k];
    s.F[P] = (s.E + W[P]) * s.vn;
    s.U[0] = W[0];
    for (int k = 0; k < D; ++k) s.U[1 + k] = W[0] * s.v[k];
    s.U[P] = s.E;
    return s;
}
/* side(): with the sound speed (euler.hpp:340-346). */
static side_d side_full_d(int D, const double* W, const double* n, const double* w, const lo_gas* gas) {
    const int P = D + 1;
    double rel[3];
    for (int k = 0; k < D; ++k) rel[k] = W[1 + k] - w[k];
    side_d s = side_with_d(D, W, n, w, gas, dotd(D, rel, n));
    const double c2 = gas->gamma * W[P] / W[0];
    s.c = c2 > 0 ? sqrt(c2) : 0.0;
    return s;
}

/* to_lab(): back to the lab frame (euler.hpp:350-356). */
static void to_lab_d(int D, double* F, const double* w) {
    const int P = D + 1;
    double e = w[0] * F[1];
    for (int k = 1; k < D; ++k) e = e + w[k] * F[1 + k];
    F[P] += e + 0.5 * dotd(D, w, w) * F[0];
    for (int k = 0; k < D; ++k) F[1 + k] += w[k] * F[0];
}

/* HLL::flux (euler.hpp:444-461). */
void lo_hll_flux(int D, const double* L, const double* R, const double* n, const double* w, const lo_gas* gas, double* F) {
    const side_d l = side_full_d(D, L, n, w, gas), r = side_full_d(D, R, n, w, gas);
    const double SL = fmin(l.vn - l.c, r.vn - r.c);
    const double SR = fmax(l.vn + l.c, r.vn + r.c);
    if (SL >= 0) {
        for (int v = 0; v < D + 2; ++v) F[v] = l.F[v];
    } else if (SR <= 0) {
        for (int v = 0; v < D + 2; ++v) F[v] = r.F[v];
    } else {
        const double inv_dS = 1.0 / (SR - SL);
        for (int v = 0; v < D + 2; ++v) F[v] = (SR * l.F[v] - SL * r.F[v] + SL * SR * (r.U[v] - l.U[v])) * inv_dS;
    }
    to_lab_d(D, F, w);
}

/* HLLC::nonzero (euler.hpp:546-550). */
static double nonzero_d(double d) {
    const double eps = 1e-20;
    return fabs(d) < eps ? (d < 0 ? -eps : eps) : d;
}
static float nonzero_f(float d) {
    const float eps = 1e-20f;
    return fabsf(d) < eps ? (d < 0 ? -eps : eps) : d;
}

/* HLLC::flux in double (euler.hpp:609-642). */
void lo_hllc_flux(int D, const double* L, const double* R, const double* n, const double* w, const lo_gas* gas, double* F) {
    const int P = D + 1;
    double rl[3], rr[3];
    for (int k = 0; k < D; ++k) {
        rl[k] = L[1 + k] - w[k];
        rr[k] = R[1 + k] - w[k];
    }
    const double vnL = dotd(D, rl, n), vnR = dotd(D, rr, n);
    const double inv_rhoL = 1.0 / L[0], inv_rhoR = 1.0 / R[0];
    const double c2L = gas->gamma * L[P] * inv_rhoL, c2R = gas->gamma * R[P] * inv_rhoR;
    const int ok = c2L >= 0 && c2R >= 0;
    const double cL = c2L > 0 ? sqrt(c2L) : 0.0, cR = c2R > 0 ? sqrt(c2R) : 0.0;
    const double SL = fmin(vnL - cL, vnR - cR);
    const double SR = fmax(vnL + cL, vnR + cR);
    const double denomL = L[0] * (SL - vnL), denomR = R[0] * (SR - vnR);
    const double SM = (R[P] - L[P] + denomL * vnL - denomR * vnR) / nonzero_d(denomL - denomR);
    const int left = ok && (SL >= 0 || SM >= 0);
    const int star = ok && SL < 0 && (SM >= 0 || SR > 0);
    double W[VMAX];
    for (int v = 0; v < D + 2; ++v) W[v] = left ? L[v] : R[v];
    const side_d s = side_with_d(D, W, n, w, gas, left ? vnL : vnR);
    if (!star) {
        for (int v = 0; v < D + 2; ++v) F[v] = s.F[v];
        to_lab_d(D, F, w);
        return;
    }
    const double S = left ? SL : SR, denom = left ? denomL : denomR;
    const double rho_star = denom / nonzero_d(S - SM);
    const double E_star = s.E * (left ? inv_rhoL : inv_rhoR) + (SM - s.vn) * (SM + W[P] * (1.0 / nonzero_d(denom)));
    double U_star[VMAX];
    U_star[0] = rho_star;
    for (int k = 0; k < D; ++k) U_star[1 + k] = rho_star * (s.v[k] + n[k] * (SM - s.vn));
    U_star[P] = rho_star * E_star;
    for (int v = 0; v < D + 2; ++v) F[v] = s.F[v] + S * (U_star[v] - s.U[v]);
    to_lab_d(D, F, w);
}

/* HLLC::flux with T = float and w = 0 (euler.hpp:609-642, as FaceFlux::solve calls it for a float Riemann policy). */
void lo_hllc_flux_float(int D, const float* L, const float* R, const float* n, const lo_gas* gas, float* F) {
    const int P = D + 1;
    float rl[3], rr[3];
    for (int k = 0; k < D; ++k) {
        rl[k] = L[1 + k] - 0.0f;
        rr[k] = R[1 + k] - 0.0f;
    }
    const float g = (float)gas->gamma;
    const float vnL = dotf(D, rl, n), vnR = dotf(D, rr, n);
    const float inv_rhoL = 1.0f / L[0], inv_rhoR = 1.0f / R[0];
    const float c2L = g * L[P] * inv_rhoL, c2R = g * R[P] * inv_rhoR;
    const int ok = c2L >= 0 && c2R >= 0;
    const float cL = c2L > 0 ? sqrtf(c2L) : 0.0f, cR = c2R > 0 ? sqrtf(c2R) : 0.0f;
    const float SL = fminf(vnL - cL, vnR - cR);
    const float SR = fmaxf(vnL + cL, vnR + cR);
    const float denomL = L[0] * (SL - vnL), denomR = R[0] * (SR - vnR);
    const float SM = (R[P] - L[P] + denomL * vnL - denomR * vnR) / nonzero_f(denomL - denomR);
    const int left = ok && (SL >= 0 || SM >= 0);
    const int star = ok && SL < 0 && (SM >= 0 || SR > 0);
    float W[VMAX];
    for (int v = 0; v < D + 2; ++v) W[v] = left ? L[v] : R[v];
    const side_f s = side_with_f(D, W, n, gas, left ? vnL : vnR);
    if (!star) {
        for (int v = 0; v < D + 2; ++v) F[v] = s.F[v];
        return;  /* to_lab with w = 0 in float adds zeros */
    }
    const float S = left ? SL : SR, denom = left ? denomL : denomR;
    const float rho_star = denom / nonzero_f(S - SM);
    const float E_star = s.E * (left ? inv_rhoL : inv_rhoR) + (SM - s.vn) * (SM + W[P] * (1.0f / nonzero_f(denom)));
    float U_star[VMAX];
    U_star[0] = rho_star;
    for (int k = 0; k < D; ++k) U_star[1 + k] = rho_star * (s.v[k] + n[k] * (SM - s.vn));
    U_star[P] = rho_star * E_star;
    for (int v = 0; v < D + 2; ++v) F[v] = s.F[v] + S * (U_star[v] - s.U[v]);
}

/* ---------------------------------------------------------------------------------------------------------------------
 * finite_volume.hpp
 * ------------------------------------------------------------------------------------------------------------------- */

struct lo_fv {
    lo_mesh mesh;
    lo_gas gas;
    int D, V, U, order, per_face, limiter_none, riemann, moving, grad_float, riemann_float, grad_half, flux_float;
    int64_t n, f;
    double box_inverse[3], step, per_step;
    int64_t period[3];
    double* q;        /* [N][V] */
    double* next;     /* order 0 per cell */
    double* prims;    /* [N][V + 2] */
    double* grad;     /* [N][V * D] (double, or the float rows widened exactly) */
    double* flux;     /* [F][V] */
    double* mag;      /* [F] */
    double* w;        /* [N][D] point velocities */
    double* x;        /* [N][D] positions (moving) */
    double* old_centroid;
    int32_t* steps;
    int prims_ready, swept;
    int64_t fallbacks[2];
    double pending_dt;
    /* owned copies of a moving mesh's arrays */
    void* mesh_store[16];
};

/* tet_mesh::wrap: the nearest periodic image of a separation (voronoi-cpp; restated as d - side * rint(d / side)). */
static double wrap(double d, double side, double inverse) { return d - side * rint(d * inverse); }

static int list_face(int32_t e) { return e >= 0 ? e : ~e; }

/* Geometry::separation (finite_volume.hpp:282-285): nearest image of generator j seen from generator i. */
static void separation(const lo_fv* fv, int64_t i, int64_t j, double* d) {
    const int D = fv->D;
    for (int a = 0; a < D; ++a)
        d[a] = wrap(fv->mesh.positions[D * j + a] - fv->mesh.positions[D * i + a], fv->mesh.box[a], fv->box_inverse[a]);
}
/* Geometry::face_offset (finite_volume.hpp:322-326): face centroid of f relative to the centroid of cell i. */
static void face_offset(const lo_fv* fv, int64_t f, int64_t i, double* out) {
    const int D = fv->D;
    const int64_t o = fv->mesh.owner[f];
    double rel[3];
    if (o == i) {
        for (int a = 0; a < D; ++a) rel[a] = fv->mesh.face_centroid[D * f + a];
    } else {
        double s[3];
        separation(fv, i, o, s);
        for (int a = 0; a < D; ++a) rel[a] = fv->mesh.face_centroid[D * f + a] + s[a];
    }
    for (int a = 0; a < D; ++a) out[a] = rel[a] - fv->mesh.centroid[D * i + a];
}
static double magnitude_of(const lo_fv* fv, int64_t f) {
    const int D = fv->D;
    return sqrt(dotd(D, fv->mesh.area + D * f, fv->mesh.area + D * f));
}

static double radius(int D, double v) {
    if (D == 3) return cbrt(v * (3.0 / (4.0 * M_PI)));
    return sqrt(v * (1.0 / M_PI));
}
static double face_angle(int D, double area) { return D == 3 ? sqrt(area / M_PI) : 0.5 * area; }

double lo_grid_step(int D, const double* box) {
    double longest = box[0];
    for (int a = 1; a < D; ++a) longest = fmax(longest, box[a]);
    return ldexp(longest, -30);
}

static void set_mesh(lo_fv* fv, const lo_mesh* mesh) {
    fv->mesh = *mesh;
    fv->f = mesh->f;
    for (int a = 0; a < fv->D; ++a) fv->box_inverse[a] = 1.0 / mesh->box[a];
    free(fv->flux);
    free(fv->mag);
    fv->flux = (double*)malloc(sizeof(double) * (size_t)(fv->f > 0 ? fv->f : 1) * fv->V);
    fv->mag = (double*)malloc(sizeof(double) * (size_t)(fv->f > 0 ? fv->f : 1));
    for (int64_t f = 0; f < fv->f; ++f) fv->mag[f] = magnitude_of(fv, f);
}

lo_fv* lo_fv_create(const lo_mesh* mesh, const lo_gas* gas, int order, int per_face, int limiter_none, int riemann,
                    int moving, int grad_float, int riemann_float) {
    lo_fv* fv = (lo_fv*)calloc(1, sizeof(lo_fv));
    fv->gas = *gas;
    fv->D = mesh->dim;
    fv->V = fv->D + 2;
    fv->U = fv->D + 1;
    fv->order = order;
    fv->per_face = per_face;
    fv->limiter_none = limiter_none;
    fv->riemann = riemann;
    fv->moving = moving;
    fv->grad_float = grad_float;
    fv->riemann_float = riemann_float;
    fv->n = mesh->n;
    const int64_t N = fv->n;
    fv->q = (double*)calloc((size_t)N * fv->V, sizeof(double));
    fv->next = (double*)calloc((size_t)N * fv->V, sizeof(double));
    fv->prims = (double*)calloc((size_t)N * (fv->V + 2), sizeof(double));
    fv->grad = (double*)calloc((size_t)N * fv->V * fv->D, sizeof(double));
    fv->w = (double*)calloc((size_t)N * fv->D, sizeof(double));
    fv->x = (double*)calloc((size_t)N * fv->D, sizeof(double));
    fv->old_centroid = (double*)calloc((size_t)N * fv->D, sizeof(double));
    fv->steps = (int32_t*)calloc((size_t)N * fv->D, sizeof(int32_t));
    set_mesh(fv, mesh);
    memcpy(fv->x, mesh->positions, sizeof(double) * (size_t)N * fv->D);
    fv->step = lo_grid_step(fv->D, mesh->box);
    fv->per_step = 1.0 / fv->step;
    for (int a = 0; a < fv->D; ++a) fv->period[a] = (int64_t)llround(mesh->box[a] / fv->step);
    return fv;
}

void lo_fv_destroy(lo_fv* fv) {
    if (!fv) return;
    free(fv->q);
    free(fv->next);
    free(fv->prims);
    free(fv->grad);
    free(fv->flux);
    free(fv->mag);
    free(fv->w);
    free(fv->x);
    free(fv->old_centroid);
    free(fv->steps);
    free(fv);
}

double* lo_fv_state(lo_fv* fv) {
    fv->prims_ready = 0;
    return fv->q;
}
void lo_fv_state_changed(lo_fv* fv) { fv->prims_ready = 0; }
const double* lo_fv_prims(const lo_fv* fv) { return fv->prims; }
const double* lo_fv_gradients(const lo_fv* fv) { return fv->grad; }
const double* lo_fv_point_velocities(const lo_fv* fv) { return fv->w; }
int64_t lo_fv_fallbacks(const lo_fv* fv) { return fv->fallbacks[0] + fv->fallbacks[1]; }

int lo_fv_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    return omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

/* primitives() (finite_volume.hpp:403-415): W = primitive(Q / V), c, r. */
static void primitives(lo_fv* fv) {
    const int D = fv->D, V = fv->V;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < fv->n; ++i) {
        const double inv = 1.0 / fv->mesh.volume[i];
        double U[VMAX], W[VMAX];
        for (int v = 0; v < V; ++v) U[v] = fv->q[V * i + v] * inv;
        lo_primitive(D, U, &fv->gas, W);
        double* p = fv->prims + (V + 2) * i;
        for (int v = 0; v < V; ++v) p[v] = W[v];
        p[V] = sqrt(fv->gas.gamma * W[D + 1] / W[0]);
        p[V + 1] = radius(D, fv->mesh.volume[i]);
    }
}

/* Sweep::solve (finite_volume.hpp:591-615): Cholesky of M once, then forward and back substitution per variable. */
static void solve_d(int U, int V, int D, double M[UMAX][UMAX], double b[VMAX][UMAX], double* grad) {
    double L[UMAX][UMAX];
    memset(L, 0, sizeof(L));
    for (int p = 0; p < U; ++p)
        for (int s = 0; s <= p; ++s) {
            double sum = M[s][p];
            for (int m = 0; m < s; ++m) sum -= L[p][m] * L[s][m];
            L[p][s] = p == s ? sqrt(sum) : sum / L[s][s];
        }
    for (int v = 0; v < V; ++v) {
        double z[UMAX], x[UMAX];
        for (int p = 0; p < U; ++p) {
            double sum = b[v][p];
            for (int m = 0; m < p; ++m) sum -= L[p][m] * z[m];
            z[p] = sum / L[p][p];
        }
        for (int p = U - 1; p >= 0; --p) {
            double sum = z[p];
            for (int m = p + 1; m < U; ++m) sum -= L[m][p] * x[m];
            x[p] = sum / L[p][p];
        }
        for (int a = 0; a < D; ++a) grad[D * v + a] = x[1 + a];
    }
}
static void solve_f(int U, int V, int D, float M[UMAX][UMAX], float b[VMAX][UMAX], float* grad) {
    float L[UMAX][UMAX];
    memset(L, 0, sizeof(L));
    for (int p = 0; p < U; ++p)
        for (int s = 0; s <= p; ++s) {
            float sum = M[s][p];
            for (int m = 0; m < s; ++m) sum -= L[p][m] * L[s][m];
            L[p][s] = p == s ? sqrtf(sum) : sum / L[s][s];
        }
    for (int v = 0; v < V; ++v) {
        float z[UMAX], x[UMAX];
        for (int p = 0; p < U; ++p) {
            float sum = b[v][p];
            for (int m = 0; m < p; ++m) sum -= L[p][m] * z[m];
            z[p] = sum / L[p][p];
        }
        for (int p = U - 1; p >= 0; --p) {
            float sum = z[p];
            for (int m = p + 1; m < U; ++m) sum -= L[m][p] * x[m];
            x[p] = sum / L[p][p];
        }
        for (int a = 0; a < D; ++a) grad[D * v + a] = x[1 + a];
    }
}

/* Sweep<Moving, Grad>::operator() (finite_volume.hpp:463-569) for one cell, double gradient policy. */
static void sweep_cell_d(lo_fv* fv, int64_t i, int grad_on) {
    const int D = fv->D, V = fv->V, U = fv->U;
    const double* Wi = fv->prims + (V + 2) * i;
    double surface = 0, smallest = INFINITY, max_angle = 0;
    double grad[VMAX * 3];
    double lo[VMAX], hi[VMAX];
    for (int v = 0; v < V; ++v) {
        for (int a = 0; a < D; ++a) grad[D * v + a] = 0;
        lo[v] = DBL_MAX;
        hi[v] = -DBL_MAX;
    }
    double M[UMAX][UMAX], b[VMAX][UMAX];
    memset(M, 0, sizeof(M));
    memset(b, 0, sizeof(b));
    const double* centroid = fv->mesh.centroid + D * i;
    const int32_t first = fv->mesh.start[i], end = fv->mesh.start[i + 1];
    for (int32_t k = first; k < end; ++k) {
        const int32_t e = fv->mesh.list[k];
        const int f = list_face(e);
        const int64_t j = e >= 0 ? fv->mesh.neighbour[f] : fv->mesh.owner[f];
        const double* Wj = fv->prims + (V + 2) * j;
        double d[3];
        separation(fv, i, j, d);
        const double magnitude = fv->mag[f];
        surface += magnitude;
        smallest = fmin(smallest, magnitude);
        if (fv->moving) max_angle = fmax(max_angle, face_angle(D, magnitude) / (0.5 * sqrt(dotd(D, d, d))));
        if (grad_on) {
            double X[UMAX];
            X[0] = 1;
            for (int p = 1; p < U; ++p) X[p] = d[p - 1] + fv->mesh.centroid[D * j + p - 1] - centroid[p - 1];
            const double w = magnitude;
            for (int p = 0; p < U; ++p)
                for (int s = p; s < U; ++s) M[p][s] += w * X[p] * X[s];
            for (int v = 0; v < V; ++v) {
                const double dW = Wj[v] - Wi[v];
                for (int p = 0; p < U; ++p) b[v][p] += w * X[p] * dW;
                lo[v] = fmin(lo[v], Wj[v]);
                hi[v] = fmax(hi[v], Wj[v]);
            }
        }
    }
    const double tiny = 1e-6 * surface;
    const int any_tiny = smallest < tiny;
    if (grad_on && any_tiny) { /* neighbour_range (finite_volume.hpp:572-588) */
        for (int v = 0; v < V; ++v) {
            lo[v] = DBL_MAX;
            hi[v] = -DBL_MAX;
        }
        for (int32_t k = first; k < end; ++k) {
            const int32_t e = fv->mesh.list[k];
            const int f = list_face(e);
            const int64_t j = e >= 0 ? fv->mesh.neighbour[f] : fv->mesh.owner[f];
            if (fv->mag[f] < tiny) continue;
            const double* Wj = fv->prims + (V + 2) * j;
            for (int v = 0; v < V; ++v) {
                lo[v] = fmin(lo[v], Wj[v]);
                hi[v] = fmax(hi[v], Wj[v]);
            }
        }
    }
    if (grad_on) solve_d(U, V, D, M, b, grad);
    if (fv->moving) { /* the point velocity (finite_volume.hpp:526-537) */
        const double factor = 2.25, speed = 0.5;
        double fraction = 0;
        if (max_angle > 0.75 * factor)
            fraction = max_angle > factor ? speed : speed * (max_angle - 0.75 * factor) / (0.25 * factor);
        double wi[3];
        for (int a = 0; a < D; ++a) wi[a] = Wi[1 + a];
        const double cd = sqrt(dotd(D, centroid, centroid));
        if (cd > 0 && fraction > 0) {
            const double s = fraction * Wi[V] / cd;
            for (int a = 0; a < D; ++a) wi[a] = wi[a] + centroid[a] * s;
        }
        for (int a = 0; a < D; ++a) fv->w[D * i + a] = wi[a];
    }
    if (!grad_on) return;
    if (!fv->limiter_none) /* the limiter walk (finite_volume.hpp:538-565) */
        for (int32_t k = first; k < end; ++k) {
            const int f = list_face(fv->mesh.list[k]);
            if (any_tiny && fv->mag[f] < tiny) continue;
            double offset[3];
            face_offset(fv, f, i, offset);
            for (int v = 0; v < V; ++v) {
                double* g = grad + D * v;
                const double dp = dotd(D, g, offset);
                if (dp > 0 && Wi[v] + dp > hi[v]) {
                    const double s = hi[v] > Wi[v] ? (hi[v] - Wi[v]) / dp : 0.0;
                    for (int a = 0; a < D; ++a) g[a] = g[a] * s;
                } else if (dp < 0 && Wi[v] + dp < lo[v]) {
                    const double s = lo[v] < Wi[v] ? (lo[v] - Wi[v]) / dp : 0.0;
                    for (int a = 0; a < D; ++a) g[a] = g[a] * s;
                }
            }
        }
    memcpy(fv->grad + V * D * i, grad, sizeof(double) * V * D);
}

/* The same sweep with the float gradient policy (Grad32: G = float; finite_volume.hpp:463-569 with exact = false). */
/* IEEE binary16 <-> binary32 with round to nearest, ties to even (the conversions of the Grad16 policy's rows). */
static uint16_t half_of(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u, field = (x >> 23) & 0xffu, mant = x & 0x7fffffu;
    if (field == 0xffu) return (uint16_t)(sign | 0x7c00u | (mant ? 0x200u : 0u));
    const int e = (int)field - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {                                  /* a subnormal half (or zero): units of 2^-24 */
        const int shift = 14 - e;
        if (shift > 24) return (uint16_t)sign;     /* below half of the smallest subnormal */
        const uint32_t full = mant | 0x800000u;
        uint32_t h = full >> shift;
        const uint32_t rest = full & ((1u << shift) - 1u), halfway = 1u << (shift - 1);
        if (rest > halfway || (rest == halfway && (h & 1u))) ++h;
        return (uint16_t)(sign | h);
    }
    uint32_t h = ((uint32_t)e << 10) | (mant >> 13);
    const uint32_t rest = mant & 0x1fffu;
    if (rest > 0x1000u || (rest == 0x1000u && (h & 1u))) ++h;  /* a carry moves into the exponent, to infinity at most */
    return (uint16_t)(sign | h);
}
static float float_of_half(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16, field = (h >> 10) & 0x1fu, mant = h & 0x3ffu;
    uint32_t x;
    if (field == 0x1fu) {
        x = sign | 0x7f800000u | (mant << 13);
    } else if (field == 0) {
        const float m = ldexpf((float)mant, -24);  /* exact */
        return sign ? -m : m;
    } else {
        x = sign | ((field - 15u + 127u) << 23) | (mant << 13);
    }
    float f;
    memcpy(&f, &x, 4);
    return f;
}
static float two_to(int k) { /* 2^k, k in [-126, 127] */
    const uint32_t x = (uint32_t)(k + 127) << 23;
    float f;
    memcpy(&f, &x, 4);
    return f;
}
/* Sweep::store and FaceFlux::gradient with P::half (finite_volume.hpp:616-641, :1289-1302; precision.hpp's half::): each
 * group (rho, the velocity, P) scaled by 2^k that puts its largest magnitude in [2^14, 2^15) (k = 0 for an all-zero
 * group, k within [-114, 126]), rounded to binary16, and read back times 2^-k. */
static void half_round_trip(int D, int V, float* g) {
    float largest[3] = {0, 0, 0};
    for (int c = 0; c < V * D; ++c) {
        const int group = c < D ? 0 : c < D + D * D ? 1 : 2;
        largest[group] = fmaxf(largest[group], fabsf(g[c]));
    }
    int k[3];
    for (int s = 0; s < 3; ++s) {
        if (!(largest[s] > 0)) {
            k[s] = 0;
            continue;
        }
        uint32_t bits;
        memcpy(&bits, &largest[s], 4);
        const int e = (int)((bits >> 23) & 0xffu) - 127;
        k[s] = 14 - e < -114 ? -114 : 14 - e > 126 ? 126 : 14 - e;
    }
    for (int c = 0; c < V * D; ++c) {
        const int group = c < D ? 0 : c < D + D * D ? 1 : 2;
        g[c] = float_of_half(half_of(g[c] * two_to(k[group]))) * two_to(-k[group]);
    }
}

static void sweep_cell_f(lo_fv* fv, int64_t i, int grad_on) {
    const int D = fv->D, V = fv->V, U = fv->U;
    const double* Wi = fv->prims + (V + 2) * i;
    double surface = 0, smallest = INFINITY, max_angle = 0;
    float grad[VMAX * 3];
    float lo[VMAX], hi[VMAX];
    for (int v = 0; v < V; ++v) {
        for (int a = 0; a < D; ++a) grad[D * v + a] = 0;
        lo[v] = FLT_MAX;
        hi[v] = -FLT_MAX;
    }
    float M[UMAX][UMAX], b[VMAX][UMAX];
    memset(M, 0, sizeof(M));
    memset(b, 0, sizeof(b));
    const double* centroid = fv->mesh.centroid + D * i;
    const int32_t first = fv->mesh.start[i], end = fv->mesh.start[i + 1];
    for (int32_t k = first; k < end; ++k) {
        const int32_t e = fv->mesh.list[k];
        const int f = list_face(e);
        const int64_t j = e >= 0 ? fv->mesh.neighbour[f] : fv->mesh.owner[f];
        const double* Wj = fv->prims + (V + 2) * j;
        double d[3];
        separation(fv, i, j, d);
        const double magnitude = fv->mag[f];
        surface += magnitude;
        smallest = fmin(smallest, magnitude);
        if (fv->moving) max_angle = fmax(max_angle, face_angle(D, magnitude) / (0.5 * sqrt(dotd(D, d, d))));
        if (grad_on) {
            float X[UMAX];
            X[0] = 1;
            for (int p = 1; p < U; ++p) X[p] = (float)(d[p - 1] + fv->mesh.centroid[D * j + p - 1] - centroid[p - 1]);
            const float w = (float)magnitude;
            for (int p = 0; p < U; ++p)
                for (int s = p; s < U; ++s) M[p][s] += w * X[p] * X[s];
            for (int v = 0; v < V; ++v) {
                const double dW = Wj[v] - Wi[v];
                for (int p = 0; p < U; ++p) b[v][p] += w * X[p] * (float)dW;
                const float value = (float)dW;
                lo[v] = fminf(lo[v], value);
                hi[v] = fmaxf(hi[v], value);
            }
        }
    }
    const double tiny = 1e-6 * surface;
    const int any_tiny = smallest < tiny;
    if (grad_on && any_tiny) {
        for (int v = 0; v < V; ++v) {
            lo[v] = FLT_MAX;
            hi[v] = -FLT_MAX;
        }
        for (int32_t k = first; k < end; ++k) {
            const int32_t e = fv->mesh.list[k];
            const int f = list_face(e);
            const int64_t j = e >= 0 ? fv->mesh.neighbour[f] : fv->mesh.owner[f];
            if (fv->mag[f] < tiny) continue;
            const double* Wj = fv->prims + (V + 2) * j;
            for (int v = 0; v < V; ++v) {
                const float value = (float)(Wj[v] - Wi[v]);
                lo[v] = fminf(lo[v], value);
                hi[v] = fmaxf(hi[v], value);
            }
        }
    }
    if (grad_on) solve_f(U, V, D, M, b, grad);
    if (fv->moving) {
        const double factor = 2.25, speed = 0.5;
        double fraction = 0;
        if (max_angle > 0.75 * factor)
            fraction = max_angle > factor ? speed : speed * (max_angle - 0.75 * factor) / (0.25 * factor);
        double wi[3];
        for (int a = 0; a < D; ++a) wi[a] = Wi[1 + a];
        const double cd = sqrt(dotd(D, centroid, centroid));
        if (cd > 0 && fraction > 0) {
            const double s = fraction * Wi[V] / cd;
            for (int a = 0; a < D; ++a) wi[a] = wi[a] + centroid[a] * s;
        }
        for (int a = 0; a < D; ++a) fv->w[D * i + a] = wi[a];
    }
    if (!grad_on) return;
    if (!fv->limiter_none)
        for (int32_t k = first; k < end; ++k) {
            const int f = list_face(fv->mesh.list[k]);
            if (any_tiny && fv->mag[f] < tiny) continue;
            double offset[3];
            face_offset(fv, f, i, offset);
            float rg[3];
            for (int a = 0; a < D; ++a) rg[a] = (float)offset[a];
            for (int v = 0; v < V; ++v) {
                float* g = grad + D * v;
                const float dp = dotf(D, g, rg);
                if (dp > 0 && dp > hi[v]) {
                    const float s = hi[v] > 0 ? hi[v] / dp : 0.0f;
                    for (int a = 0; a < D; ++a) g[a] = g[a] * s;
                } else if (dp < 0 && dp < lo[v]) {
                    const float s = lo[v] < 0 ? lo[v] / dp : 0.0f;
                    for (int a = 0; a < D; ++a) g[a] = g[a] * s;
                }
            }
        }
    if (fv->grad_half) half_round_trip(D, V, grad);
    for (int c = 0; c < V * D; ++c) fv->grad[V * D * i + c] = (double)grad[c];
}

void lo_fv_set_half_gradients(lo_fv* fv, int on) { fv->grad_half = on != 0; }
void lo_fv_set_float_fluxes(lo_fv* fv, int on) { fv->flux_float = on != 0; }

/* sweep() (finite_volume.hpp:1107-1149): Sweep, then the time-step reduction (TimeStep = FaceStep + CellStep,
 * finite_volume.hpp:1040-1104). */
static double sweep(lo_fv* fv, double courant) {
    const int D = fv->D, V = fv->V;
    const int grad_on = fv->order == 1;
    if (grad_on || fv->moving) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < fv->n; ++i) {
            if (fv->grad_float)
                sweep_cell_f(fv, i, grad_on);
            else
                sweep_cell_d(fv, i, grad_on);
        }
    }
    double smallest = DBL_MAX;
#pragma omp parallel for reduction(min : smallest) schedule(static)
    for (int64_t f = 0; f < fv->f; ++f) {
        const int64_t o = fv->mesh.owner[f], j = fv->mesh.neighbour[f];
        double d[3], dv[3];
        separation(fv, o, j, d);
        const double dist = sqrt(dotd(D, d, d));
        const double* po = fv->prims + (V + 2) * o;
        const double* pj = fv->prims + (V + 2) * j;
        for (int a = 0; a < D; ++a) dv[a] = pj[1 + a] - po[1 + a];
        const double vsig = po[V] + pj[V] - dotd(D, dv, d) / dist;
        if (vsig > 0) {
            smallest = fmin(smallest, courant * ((dist + po[V + 1]) / vsig));
            smallest = fmin(smallest, courant * ((dist + pj[V + 1]) / vsig));
        }
    }
#pragma omp parallel for reduction(min : smallest) schedule(static)
    for (int64_t i = 0; i < fv->n; ++i) {
        const double* p = fv->prims + (V + 2) * i;
        double rel[3];
        for (int a = 0; a < D; ++a) rel[a] = p[1 + a] - (fv->moving ? fv->w[D * i + a] : 0.0);
        const double step = p[V + 1] / (p[V] + sqrt(dotd(D, rel, rel)));
        smallest = fmin(smallest, courant * step);
    }
    return smallest;
}

/* time_step() (finite_volume.hpp:190-201). */
double lo_fv_time_step(lo_fv* fv, double courant) {
    if (!fv->prims_ready) primitives(fv);
    fv->prims_ready = 0;
    const double dt = sweep(fv, courant);
    fv->swept = 1;
    return dt;
}

/* FaceFlux::side at order 1 (finite_volume.hpp:1306-1329), double or float gradient policy. */
static void face_side(const lo_fv* fv, int64_t i, const double* r, double dt, double* Wf, int* fallbacks) {
    const int D = fv->D, V = fv->V;
    const double* W = fv->prims + (V + 2) * i;
    const double* g = fv->grad + V * D * i;
    if (!fv->grad_float) {
        lo_half_step(D, W, g, dt, &fv->gas, Wf);
        for (int v = 0; v < V; ++v) Wf[v] += dotd(D, g + D * v, r);
    } else {
        float Wg[VMAX], gf[VMAX * 3], rate[VMAX], rg[3];
        for (int v = 0; v < V; ++v) Wg[v] = (float)W[v];
        for (int c = 0; c < V * D; ++c) gf[c] = (float)g[c];
        half_step_rate_f(D, Wg, gf, &fv->gas, rate);
        for (int a = 0; a < D; ++a) rg[a] = (float)r[a];
        const float h = 0.5f * (float)dt;
        for (int v = 0; v < V; ++v) Wf[v] = W[v] + (double)(dotf(D, gf + D * v, rg) - h * rate[v]);
    }
    if (Wf[0] > 0 && Wf[D + 1] > 0) return;
    ++*fallbacks;
    for (int v = 0; v < V; ++v) Wf[v] = W[v];
}

/* MovingFlux<false>::pass_side (finite_volume.hpp:1451-1468): W + g . r, no half step. */
static void pass1_side(const lo_fv* fv, int64_t i, const double* r, double* Wf, int* fallbacks) {
    const int D = fv->D, V = fv->V;
    const double* W = fv->prims + (V + 2) * i;
    const double* g = fv->grad + V * D * i;
    if (!fv->grad_float) {
        for (int v = 0; v < V; ++v) Wf[v] = W[v] + dotd(D, g + D * v, r);
    } else {
        float gf[VMAX * 3], rg[3];
        for (int c = 0; c < V * D; ++c) gf[c] = (float)g[c];
        for (int a = 0; a < D; ++a) rg[a] = (float)r[a];
        for (int v = 0; v < V; ++v) Wf[v] = W[v] + (double)dotf(D, gf + D * v, rg);
    }
    if (Wf[0] > 0 && Wf[D + 1] > 0) return;
    ++*fallbacks;
    for (int v = 0; v < V; ++v) Wf[v] = W[v];
}

/* FaceFlux::solve (finite_volume.hpp:1400-1413): the Riemann solve along n, in float in the face's frame if asked. */
static void riemann_solve(const lo_fv* fv, const double* L, const double* R, const double* n, const double* wf, double* F) {
    const int D = fv->D, V = fv->V;
    if (!fv->riemann_float) {
        if (fv->riemann == 1)
            lo_hll_flux(D, L, R, n, wf, &fv->gas, F);
        else
            lo_hllc_flux(D, L, R, n, wf, &fv->gas, F);
        return;
    }
    float Lf[VMAX], Rf[VMAX], nf[3], Ff[VMAX];
    for (int v = 0; v < V; ++v) {
        Lf[v] = (float)(v >= 1 && v <= D ? L[v] - wf[v - 1] : L[v]);
        Rf[v] = (float)(v >= 1 && v <= D ? R[v] - wf[v - 1] : R[v]);
    }
    for (int a = 0; a < D; ++a) nf[a] = (float)n[a];
    lo_hllc_flux_float(D, Lf, Rf, nf, &fv->gas, Ff);
    for (int v = 0; v < V; ++v) F[v] = (double)Ff[v];
    to_lab_d(D, F, wf);
}

/* FaceFlux::face_velocity (finite_volume.hpp:1380-1397). */
static void face_velocity(const lo_fv* fv, int64_t f, int64_t o, int64_t j, const double* wL, const double* wR, double* out) {
    const int D = fv->D;
    double d[3], c[3], dw[3];
    separation(fv, o, j, d);
    const double dist = sqrt(dotd(D, d, d));
    const double inv_dist = 1.0 / dist;
    for (int a = 0; a < D; ++a) {
        c[a] = fv->mesh.face_centroid[D * f + a] - d[a] * 0.5;
        dw[a] = wL[a] - wR[a];
    }
    double facv = dotd(D, c, dw) * inv_dist;
    const double limit = 0.9 * dist, c2 = dotd(D, c, c);
    if (c2 > limit * limit) facv *= limit / sqrt(c2);
    const double s = facv * inv_dist;
    for (int a = 0; a < D; ++a) out[a] = (wL[a] + wR[a]) * 0.5 + d[a] * s;
}

/* The flux through face f times |A| (FaceFlux::operator(), finite_volume.hpp:1415-1434; MovingFlux::operator(),
 * :1469-1490 when pass >= 0). pass: -1 static, 0 moving pass 1 (t^n mesh), 1 moving pass 2 (t^n+1 mesh). */
static void face_flux(const lo_fv* fv, int64_t f, double dt, int pass, double* F, int* fb_o, int* fb_j) {
    const int D = fv->D, V = fv->V;
    const int64_t o = fv->mesh.owner[f], j = fv->mesh.neighbour[f];
    const double* a = fv->mesh.area + D * f;
    const double magnitude = sqrt(dotd(D, a, a));
    if (magnitude == 0) {
        for (int v = 0; v < V; ++v) F[v] = 0;
        return;
    }
    double L[VMAX], R[VMAX], n[3], wf[3] = {0, 0, 0};
    const double inv = 1.0 / magnitude;
    for (int k = 0; k < D; ++k) n[k] = a[k] * inv;
    if (pass < 0) {
        if (fv->order == 0) {
            double U[VMAX];
            const double io = 1.0 / fv->mesh.volume[o], ij = 1.0 / fv->mesh.volume[j];
            for (int v = 0; v < V; ++v) U[v] = fv->q[V * o + v] * io;
            lo_primitive(D, U, &fv->gas, L);
            for (int v = 0; v < V; ++v) U[v] = fv->q[V * j + v] * ij;
            lo_primitive(D, U, &fv->gas, R);
        } else {
            double ro[3], rj[3];
            face_offset(fv, f, o, ro);
            face_offset(fv, f, j, rj);
            face_side(fv, o, ro, dt, L, fb_o);
            face_side(fv, j, rj, dt, R, fb_j);
        }
    } else {
        const double unit = fv->step / fv->pending_dt;
        double wo[3], wj[3];
        for (int k = 0; k < D; ++k) {
            wo[k] = (double)fv->steps[D * o + k] * unit;
            wj[k] = (double)fv->steps[D * j + k] * unit;
        }
        face_velocity(fv, f, o, j, wo, wj, wf);
        double ro[3], rj[3];
        face_offset(fv, f, o, ro);
        face_offset(fv, f, j, rj);
        if (pass == 0) {
            pass1_side(fv, o, ro, L, fb_o);
            pass1_side(fv, j, rj, R, fb_j);
        } else {
            /* MovingFlux<true>::pass_side: r + c^{n+1} - c^n + w dt, FaceFlux::side with 2 dt (finite_volume.hpp:1452-1456) */
            const double mdt = 2 * fv->pending_dt;
            double r2[3];
            for (int k = 0; k < D; ++k)
                r2[k] = ro[k] + fv->mesh.centroid[D * o + k] - fv->old_centroid[D * o + k] + wo[k] * (0.5 * mdt);
            face_side(fv, o, r2, mdt, L, fb_o);
            for (int k = 0; k < D; ++k)
                r2[k] = rj[k] + fv->mesh.centroid[D * j + k] - fv->old_centroid[D * j + k] + wj[k] * (0.5 * mdt);
            face_side(fv, j, r2, mdt, R, fb_j);
        }
    }
    riemann_solve(fv, L, R, n, wf, F);
    for (int v = 0; v < V; ++v) F[v] *= magnitude;
}

/* apply() (finite_volume.hpp:1538-1631): per-face flux rows then a per-cell gather in list order, or the per-cell loop.
 * pass: as face_flux(); update with dt_update; pass 1 also writes the next primitives. */
static void apply(lo_fv* fv, double dt_flux, double dt_update, int pass) {
    const int D = fv->D, V = fv->V;
    int64_t count = 0;
    if (!fv->per_face) {
        double* next = fv->order == 0 ? fv->next : fv->q;
#pragma omp parallel for reduction(+ : count) schedule(static)
        for (int64_t i = 0; i < fv->n; ++i) {
            double sum[VMAX] = {0, 0, 0, 0, 0};
            for (int32_t k = fv->mesh.start[i]; k < fv->mesh.start[i + 1]; ++k) {
                const int32_t e = fv->mesh.list[k];
                const int f = list_face(e);
                int fo = 0, fj = 0;
                double F[VMAX];
                face_flux(fv, f, dt_flux, pass, F, &fo, &fj);
                const int owned = e >= 0;
                count += owned ? fo : fj;
                const double sign = owned ? 1.0 : -1.0;
                for (int v = 0; v < V; ++v) sum[v] += sign * F[v];
            }
            for (int v = 0; v < V; ++v) next[V * i + v] = fv->q[V * i + v] - dt_update * sum[v];
        }
        if (fv->order == 0) {
            double* t = fv->q;
            fv->q = fv->next;
            fv->next = t;
        }
        fv->fallbacks[pass < 0 ? 0 : pass] = count;
        return;
    }
#pragma omp parallel for reduction(+ : count) schedule(static)
    for (int64_t f = 0; f < fv->f; ++f) {
        int fb = 0;
        face_flux(fv, f, dt_flux, pass, fv->flux + V * f, &fb, &fb);
        /* Precision::flux = float: F(f, v) = static_cast<FluxStore>(value[v]) (finite_volume.hpp:1597), read back as double */
        if (fv->flux_float)
            for (int v = 0; v < V; ++v) fv->flux[V * f + v] = (double)(float)fv->flux[V * f + v];
        count += fb;
    }
    fv->fallbacks[pass < 0 ? 0 : pass] = count;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < fv->n; ++i) {
        double sum[VMAX] = {0, 0, 0, 0, 0};
        for (int32_t k = fv->mesh.start[i]; k < fv->mesh.start[i + 1]; ++k) {
            const int32_t e = fv->mesh.list[k];
            const int f = list_face(e);
            const double sign = e >= 0 ? 1.0 : -1.0;
            for (int v = 0; v < V; ++v) sum[v] += sign * fv->flux[V * f + v];
        }
        double next[VMAX];
        for (int v = 0; v < V; ++v) fv->q[V * i + v] = next[v] = fv->q[V * i + v] - dt_update * sum[v];
        if (pass == 1) {
            const double inv = 1.0 / fv->mesh.volume[i];
            double U[VMAX], W[VMAX];
            for (int v = 0; v < V; ++v) U[v] = next[v] * inv;
            lo_primitive(D, U, &fv->gas, W);
            double* p = fv->prims + (V + 2) * i;
            for (int v = 0; v < V; ++v) p[v] = W[v];
            p[V] = sqrt(fv->gas.gamma * W[D + 1] / W[0]);
            p[V + 1] = radius(D, fv->mesh.volume[i]);
        }
    }
}

/* step() (finite_volume.hpp:205-226) for a static mesh. */
void lo_fv_step(lo_fv* fv, double dt) {
    if (!fv->swept) {
        if (!fv->prims_ready) primitives(fv);
        fv->prims_ready = 0;
        sweep(fv, 1.0);
    }
    fv->swept = 0;
    fv->fallbacks[0] = fv->fallbacks[1] = 0;
    apply(fv, dt, dt, -1);
}

/* exact_predicates::snap / delta (voronoi-cpp): the grid key of a coordinate and the nearest periodic difference of two
 * keys; restated as rounding to the 2^-30 grid. */
static int64_t snap(const lo_fv* fv, double x, int a) {
    int64_t k = (int64_t)llround(x * fv->per_step);
    const int64_t p = fv->period[a];
    return ((k % p) + p) % p;
}
static int32_t delta(int64_t k0, int64_t k1, int64_t p) {
    int64_t d = k1 - k0;
    if (d > p / 2) d -= p;
    if (d < -(p / 2)) d += p;
    return (int32_t)d;
}

/* step_moving(), first half (finite_volume.hpp:1497-1515): keep_centroids, the t^n fluxes at half dt, the drift. */
void lo_fv_step_moving_begin(lo_fv* fv, double dt, double* positions_out) {
    const int D = fv->D;
    if (!fv->swept) {
        if (!fv->prims_ready) primitives(fv);
        fv->prims_ready = 0;
        sweep(fv, 1.0);
    }
    fv->swept = 0;
    fv->pending_dt = dt;
    for (int64_t i = 0; i < fv->n; ++i)
        for (int a = 0; a < D; ++a) {
            fv->old_centroid[D * i + a] = fv->mesh.centroid[D * i + a];
            const int64_t k0 = snap(fv, fv->x[D * i + a], a), k1 = snap(fv, fv->x[D * i + a] + dt * fv->w[D * i + a], a);
            fv->x[D * i + a] = (double)k0 * fv->step;
            fv->steps[D * i + a] = delta(k0, k1, fv->period[a]);
        }
    fv->fallbacks[0] = fv->fallbacks[1] = 0;
    apply(fv, 0.0, 0.5 * dt, 0);
    /* move(): the drift on the grid (finite_volume.hpp:1219-1231) */
    for (int64_t i = 0; i < fv->n; ++i)
        for (int a = 0; a < D; ++a) {
            const int64_t k = (int64_t)llround(fv->x[D * i + a] * fv->per_step) + fv->steps[D * i + a];
            const int64_t p = fv->period[a];
            fv->x[D * i + a] = (double)(((k % p) + p) % p) * fv->step;
        }
    memcpy(positions_out, fv->x, sizeof(double) * (size_t)fv->n * D);
}

/* step_moving(), second half (finite_volume.hpp:1516-1518): the fluxes of t^n+1 at half dt on the new mesh. */
void lo_fv_step_moving_end(lo_fv* fv, const lo_mesh* new_mesh) {
    set_mesh(fv, new_mesh);
    apply(fv, 0.0, 0.5 * fv->pending_dt, 1);
    fv->prims_ready = fv->per_face; /* the per-face update wrote the next primitives (finite_volume.hpp:1628) */
}

/* ---------------------------------------------------------------------------------------------------------------------
 * The adjoint of one static step (step_adjoint, finite_volume.hpp:2201-2231), double policy, order 1, per-face loop.
 * ------------------------------------------------------------------------------------------------------------------- */

/* primitive_adjoint (euler.hpp:143-162): Ubar = J^T Wbar, a floored density or energy takes its floor's derivative. */
static void primitive_adjoint(int D, const double* U, const double* Wbar, const lo_gas* gas, double* Ubar) {
    const int P = D + 1;
    const double rho = fmax(U[0], gas->smallr), inv_rho = 1.0 / rho;
    double v[3];
    for (int k = 0; k < D; ++k) v[k] = U[1 + k] * inv_rho;
    const double smalle = gas->smallc * gas->smallc / gas->gamma / (gas->gamma - 1.0);
    /* primitive_branches (euler.hpp:121-127) */
    double vb[3];
    for (int k = 0; k < D; ++k) vb[k] = U[1 + k] * (1.0 / rho);
    const int floors = (U[0] >= gas->smallr ? 0 : 1) | (U[P] - 0.5 * rho * dotd(D, vb, vb) >= smalle * rho ? 0 : 2);
    const double ebar = (gas->gamma - 1.0) * Wbar[P];
    double rhobar = Wbar[0], energybar = 0;
    double vbar[3];
    for (int k = 0; k < D; ++k) vbar[k] = Wbar[1 + k];
    if (floors & 2) {
        rhobar += smalle * ebar;
    } else {
        energybar = ebar;
        rhobar -= 0.5 * dotd(D, v, v) * ebar;
        const double s = rho * ebar;
        for (int k = 0; k < D; ++k) vbar[k] = vbar[k] - v[k] * s;
    }
    double mbar[3];
    for (int k = 0; k < D; ++k) mbar[k] = vbar[k] * inv_rho;
    rhobar -= dotd(D, v, vbar) * inv_rho;
    Ubar[0] = floors & 1 ? 0.0 : rhobar;
    for (int k = 0; k < D; ++k) Ubar[1 + k] = mbar[k];
    Ubar[P] = energybar;
}

/* half_step_adjoint (euler.hpp:241-272): adds J^T halfbar to Wbar and gbar. */
static void half_step_adjoint(int D, const double* W, const double* g, double dt, const lo_gas* gas, const double* halfbar, double* Wbar,
                              double* gbar) {
    const int P = D + 1;
    const double rho = W[0], inv_rho = 1.0 / W[0], rho_c2 = gas->gamma * W[P];
    double Abar[VMAX];
    for (int v = 0; v < D + 2; ++v) {
        Wbar[v] += halfbar[v];
        Abar[v] = -0.5 * dt * halfbar[v];
    }
    double inv_rhobar = 0, rho_c2bar = 0;
    for (int d = 0; d < D; ++d) {
        const double vn = W[1 + d];
        Wbar[1 + d] += Abar[0] * g[0 * D + d];
        gbar[0 * D + d] += Abar[0] * vn;
        Wbar[0] += Abar[0] * g[(1 + d) * D + d];
        gbar[(1 + d) * D + d] += Abar[0] * rho;
        for (int k = 0; k < D; ++k) {
            Wbar[1 + d] += Abar[1 + k] * g[(1 + k) * D + d];
            gbar[(1 + k) * D + d] += Abar[1 + k] * vn;
            if (k == d) {
                inv_rhobar += Abar[1 + k] * g[P * D + d];
                gbar[P * D + d] += Abar[1 + k] * inv_rho;
            }
        }
        rho_c2bar += Abar[P] * g[(1 + d) * D + d];
        gbar[(1 + d) * D + d] += Abar[P] * rho_c2;
        Wbar[1 + d] += Abar[P] * g[P * D + d];
        gbar[P * D + d] += Abar[P] * vn;
    }
    Wbar[0] -= inv_rho * inv_rho * inv_rhobar;
    Wbar[P] += gas->gamma * rho_c2bar;
}

/* detail::side_with_adjoint (euler.hpp:375-398): adds J^T to Wbar; returns vn's bar. vbar_in is taken by value. */
static double side_with_adjoint(int D, const double* W, const double* n, const lo_gas* gas, const side_d* s, const double* Fbar,
                                const double* Ubar, double Ebar, const double* vbar_in, double* Wbar) {
    const int P = D + 1;
    const double m = W[0] * s->vn;
    double vbar[3];
    for (int k = 0; k < D; ++k) vbar[k] = vbar_in ? vbar_in[k] : 0.0;
    Ebar += Fbar[P] * s->vn + Ubar[P];
    double Pbar = Fbar[P] * s->vn, vnbar = Fbar[P] * (s->E + W[P]), mbar = Fbar[0], rhobar = Ubar[0];
    for (int k = 0; k < D; ++k) {
        Pbar += Fbar[1 + k] * n[k];
        mbar += Fbar[1 + k] * s->v[k];
        vbar[k] += Fbar[1 + k] * m + Ubar[1 + k] * W[0];
        rhobar += Ubar[1 + k] * s->v[k];
    }
    rhobar += mbar * s->vn;
    vnbar += mbar * W[0];
    Pbar += Ebar * gas->inverse_gm1;
    rhobar += Ebar * (0.5 * dotd(D, s->v, s->v));
    const double e = Ebar * W[0];
    for (int k = 0; k < D; ++k) vbar[k] = vbar[k] + s->v[k] * e;
    Wbar[0] += rhobar;
    for (int k = 0; k < D; ++k) Wbar[1 + k] += vbar[k];
    Wbar[P] += Pbar;
    return vnbar;
}

/* detail::side_adjoint (euler.hpp:402-413). */
static void side_adjoint_full(int D, const double* W, const double* n, const lo_gas* gas, const side_d* s, const double* Fbar,
                              const double* Ubar, double vnbar, double cbar, double* Wbar) {
    const int P = D + 1;
    vnbar += side_with_adjoint(D, W, n, gas, s, Fbar, Ubar, 0.0, NULL, Wbar);
    for (int k = 0; k < D; ++k) Wbar[1 + k] += vnbar * n[k];
    const double c2 = gas->gamma * W[P] / W[0];
    if (c2 > 0) {
        const double c2bar = cbar / (2 * s->c);
        Wbar[P] += c2bar * gas->gamma / W[0];
        Wbar[0] -= c2bar * c2 / W[0];
    }
}

/* detail::to_lab_adjoint (euler.hpp:416-426). */
static void to_lab_adjoint(int D, const double* Fbar, const double* w, double* G) {
    const int P = D + 1;
    for (int v = 0; v < D + 2; ++v) G[v] = Fbar[v];
    G[0] += 0.5 * dotd(D, w, w) * Fbar[P];
    for (int k = 0; k < D; ++k) {
        G[0] += w[k] * Fbar[1 + k];
        G[1 + k] += w[k] * Fbar[P];
    }
}

/* HLL::flux_adjoint (euler.hpp:509-540) with HLL::branches (:468-477). */
static void hll_flux_adjoint(int D, const double* L, const double* R, const double* n, const double* w, const lo_gas* gas,
                             const double* Fbar_lab, double* Lbar, double* Rbar) {
    const int P = D + 1;
    const side_d l = side_full_d(D, L, n, w, gas), r = side_full_d(D, R, n, w, gas);
    const double a = l.vn - l.c, b = r.vn - r.c, A = l.vn + l.c, B = r.vn + r.c;
    const double SLm = fmin(a, b), SRm = fmax(A, B);
    const int wave = SLm >= 0 ? 1 : SRm <= 0 ? 2 : 0;
    const int pattern = (b < a ? 0 : 1) | (B > A ? 0 : 2);
    (void)P;
    const double SL = pattern & 1 ? l.vn - l.c : r.vn - r.c, SR = pattern & 2 ? l.vn + l.c : r.vn + r.c;
    double Fbar[VMAX];
    to_lab_adjoint(D, Fbar_lab, w, Fbar);
    double lF[VMAX] = {0}, rF[VMAX] = {0}, lU[VMAX] = {0}, rU[VMAX] = {0};
    double SLbar = 0, SRbar = 0;
    if (wave == 1) {
        for (int v = 0; v < D + 2; ++v) lF[v] = Fbar[v];
    } else if (wave == 2) {
        for (int v = 0; v < D + 2; ++v) rF[v] = Fbar[v];
    } else {
        const double inv_dS = 1.0 / (SR - SL);
        for (int v = 0; v < D + 2; ++v) {
            const double dU = r.U[v] - l.U[v], F = (SR * l.F[v] - SL * r.F[v] + SL * SR * dU) * inv_dS;
            const double N = Fbar[v] * inv_dS;
            SRbar += -Fbar[v] * F * inv_dS + N * (l.F[v] + SL * dU);
            SLbar += Fbar[v] * F * inv_dS + N * (-r.F[v] + SR * dU);
            lF[v] = SR * N;
            rF[v] = -SL * N;
            rU[v] = SL * SR * N;
            lU[v] = -SL * SR * N;
        }
    }
    double lvn = 0, lc = 0, rvn = 0, rc = 0;
    if (pattern & 1) {
        lvn += SLbar;
        lc -= SLbar;
    } else {
        rvn += SLbar;
        rc -= SLbar;
    }
    if (pattern & 2) {
        lvn += SRbar;
        lc += SRbar;
    } else {
        rvn += SRbar;
        rc += SRbar;
    }
    side_adjoint_full(D, L, n, gas, &l, lF, lU, lvn, lc, Lbar);
    side_adjoint_full(D, R, n, gas, &r, rF, rU, rvn, rc, Rbar);
}

/* HLLC::flux_adjoint (euler.hpp:738-832) with HLLC::waves (:651-680): only the case the forward took. */
static void hllc_flux_adjoint(int D, const double* L, const double* R, const double* n, const double* w, const lo_gas* gas,
                              const double* Fbar_lab, double* Lbar, double* Rbar) {
    const int P = D + 1;
    const double eps = 1e-20;
    double rl[3], rr[3];
    for (int k = 0; k < D; ++k) {
        rl[k] = L[1 + k] - w[k];
        rr[k] = R[1 + k] - w[k];
    }
    const double vnL = dotd(D, rl, n), vnR = dotd(D, rr, n);
    const double inv_rhoL = 1.0 / L[0], inv_rhoR = 1.0 / R[0];
    const double c2L = gas->gamma * L[P] * inv_rhoL, c2R = gas->gamma * R[P] * inv_rhoR;
    const int ok = c2L >= 0 && c2R >= 0;
    const double cL = c2L > 0 ? sqrt(c2L) : 0.0, cR = c2R > 0 ? sqrt(c2R) : 0.0;
    const double sl = vnL - cL, sr = vnR - cR, tl = vnL + cL, tr = vnR + cR;
    const double SL = fmin(sl, sr), SR = fmax(tl, tr);
    const double denomL = L[0] * (SL - vnL), denomR = R[0] * (SR - vnR);
    const double den_raw = denomL - denomR;
    const double SM = (R[P] - L[P] + denomL * vnL - denomR * vnR) / nonzero_d(den_raw);
    const int left = ok && (SL >= 0 || SM >= 0);
    const int star = ok && SL < 0 && (SM >= 0 || SR > 0);
    const double Sx = left ? SL : SR, denomx = left ? denomL : denomR;
    const int pattern = (sr < sl ? 0 : 1) | (tr > tl ? 0 : 2) | (fabs(den_raw) < eps) << 7 | (star && fabs(Sx - SM) < eps) << 8 |
                        (star && fabs(denomx) < eps) << 9;
    double Fbar[VMAX];
    to_lab_adjoint(D, Fbar_lab, w, Fbar);
    double W[VMAX];
    for (int v = 0; v < D + 2; ++v) W[v] = left ? L[v] : R[v];
    const double vn = left ? vnL : vnR;
    const side_d s = side_with_d(D, W, n, w, gas, vn);
    double Wbar[VMAX] = {0, 0, 0, 0, 0};
    double vnLbar = 0, vnRbar = 0;
    if (!star) {
        const double zero[VMAX] = {0, 0, 0, 0, 0};
        const double r = side_with_adjoint(D, W, n, gas, &s, Fbar, zero, 0.0, NULL, Wbar);
        if (left)
            vnLbar += r;
        else
            vnRbar += r;
    } else {
        const double S = left ? SL : SR, denom = left ? denomL : denomR, inv_side = left ? inv_rhoL : inv_rhoR;
        const double q = nonzero_d(S - SM), rho_star = denom / q, inv_denom = 1.0 / nonzero_d(denom);
        const double a2 = SM - s.vn, a3 = SM + W[P] * inv_denom, E_star = s.E * inv_side + a2 * a3;
        double v_star[3];
        for (int k = 0; k < D; ++k) v_star[k] = s.v[k] + n[k] * a2;
        double Sbar = 0, rho_starbar = 0, E_starbar = 0;
        double sUbar[VMAX], v_starbar[3] = {0, 0, 0};
        for (int v = 0; v < D + 2; ++v) {
            const double U_star = v == 0 ? rho_star : v == P ? rho_star * E_star : rho_star * v_star[v - 1];
            Sbar += Fbar[v] * (U_star - s.U[v]);
            sUbar[v] = -S * Fbar[v];
            const double U_starbar = S * Fbar[v];
            if (v == 0) {
                rho_starbar += U_starbar;
            } else if (v == P) {
                rho_starbar += U_starbar * E_star;
                E_starbar = U_starbar * rho_star;
            } else {
                rho_starbar += U_starbar * v_star[v - 1];
                v_starbar[v - 1] = U_starbar * rho_star;
            }
        }
        const double a2bar = dotd(D, v_starbar, n) + E_starbar * a3, a3bar = E_starbar * a2;
        double SMbar = a3bar + a2bar, vnbar = -a2bar;
        const double inv_denombar = a3bar * W[P];
        const double denombar = (pattern & 512 ? 0.0 : -inv_denom * inv_denom * inv_denombar) + rho_starbar / q;
        const double qbar = pattern & 256 ? 0.0 : -rho_starbar * rho_star / q;
        Sbar += qbar;
        SMbar -= qbar;
        const double sEbar = E_starbar * inv_side, inv_sidebar = E_starbar * s.E;
        vnbar += side_with_adjoint(D, W, n, gas, &s, Fbar, sUbar, sEbar, v_starbar, Wbar);
        Wbar[P] += a3bar * inv_denom;
        const double den = nonzero_d(den_raw), numbar = SMbar / den, denbar = pattern & 128 ? 0.0 : -SMbar * SM / den;
        double denomLbar = denbar + numbar * vnL, denomRbar = -denbar - numbar * vnR;
        if (left)
            denomLbar += denombar;
        else
            denomRbar += denombar;
        vnLbar += numbar * denomL;
        vnRbar -= numbar * denomR;
        Rbar[P] += numbar;
        Lbar[P] -= numbar;
        if (left)
            vnLbar += vnbar;
        else
            vnRbar += vnbar;
        double invLbar = 0, invRbar = 0;
        if (left)
            invLbar += inv_sidebar;
        else
            invRbar += inv_sidebar;
        double SLbar = denomLbar * L[0], SRbar = denomRbar * R[0];
        if (left)
            SLbar += Sbar;
        else
            SRbar += Sbar;
        Lbar[0] += denomLbar * (SL - vnL);
        vnLbar -= denomLbar * L[0];
        Rbar[0] += denomRbar * (SR - vnR);
        vnRbar -= denomRbar * R[0];
        double cLbar = 0, cRbar = 0;
        if (pattern & 1) {
            vnLbar += SLbar;
            cLbar -= SLbar;
        } else {
            vnRbar += SLbar;
            cRbar -= SLbar;
        }
        if (pattern & 2) {
            vnLbar += SRbar;
            cLbar += SRbar;
        } else {
            vnRbar += SRbar;
            cRbar += SRbar;
        }
        if (c2L > 0) {
            const double c2bar = cLbar / (2 * cL);
            Lbar[P] += c2bar * gas->gamma * inv_rhoL;
            invLbar += c2bar * gas->gamma * L[P];
        }
        if (c2R > 0) {
            const double c2bar = cRbar / (2 * cR);
            Rbar[P] += c2bar * gas->gamma * inv_rhoR;
            invRbar += c2bar * gas->gamma * R[P];
        }
        Lbar[0] -= inv_rhoL * inv_rhoL * invLbar;
        Rbar[0] -= inv_rhoR * inv_rhoR * invRbar;
    }
    for (int v = 0; v < D + 2; ++v) {
        Lbar[v] += left ? Wbar[v] : 0.0;
        Rbar[v] += left ? 0.0 : Wbar[v];
    }
    for (int k = 0; k < D; ++k) {
        Lbar[1 + k] += vnLbar * n[k];
        Rbar[1 + k] += vnRbar * n[k];
    }
}

/* The fit the sweep leaves for the adjoint (SweepFitHook<false>, finite_volume.hpp:1763-1926): M's Cholesky factor, M's
 * row 0, the unlimited gradient g0, per variable the last clip (offset, bound, flags) and the face its bound came through. */
typedef struct {
    double Lc[UMAX][UMAX], M0[UMAX], g0[VMAX * 3], offset[VMAX * 3], bound[VMAX];
    int clipped[VMAX], upper[VMAX], zero[VMAX], bound_face[VMAX];
} fit_t;

static void sweep_fit_cell(const lo_fv* fv, int64_t i, fit_t* fit) {
    const int D = fv->D, V = fv->V, U = fv->U;
    const double* Wi = fv->prims + (V + 2) * i;
    double surface = 0, smallest = INFINITY;
    double lo[VMAX], hi[VMAX];
    int lo_f[VMAX], hi_f[VMAX];
    for (int v = 0; v < V; ++v) {
        lo[v] = DBL_MAX;
        hi[v] = -DBL_MAX;
        lo_f[v] = hi_f[v] = -1;
    }
    double M[UMAX][UMAX], b[VMAX][UMAX];
    memset(M, 0, sizeof(M));
    memset(b, 0, sizeof(b));
    const double* centroid = fv->mesh.centroid + D * i;
    const int32_t first = fv->mesh.start[i], end = fv->mesh.start[i + 1];
    for (int32_t k = first; k < end; ++k) {
        const int32_t e = fv->mesh.list[k];
        const int f = list_face(e);
        const int64_t j = e >= 0 ? fv->mesh.neighbour[f] : fv->mesh.owner[f];
        const double* Wj = fv->prims + (V + 2) * j;
        double d[3];
        separation(fv, i, j, d);
        const double magnitude = fv->mag[f];
        surface += magnitude;
        smallest = fmin(smallest, magnitude);
        double X[UMAX];
        X[0] = 1;
        for (int p = 1; p < U; ++p) X[p] = d[p - 1] + fv->mesh.centroid[D * j + p - 1] - centroid[p - 1];
        const double w = magnitude;
        for (int p = 0; p < U; ++p)
            for (int s = p; s < U; ++s) M[p][s] += w * X[p] * X[s];
        for (int v = 0; v < V; ++v) {
            const double dW = Wj[v] - Wi[v];
            for (int p = 0; p < U; ++p) b[v][p] += w * X[p] * dW;
            if (Wj[v] < lo[v]) lo[v] = Wj[v], lo_f[v] = f;
            if (Wj[v] > hi[v]) hi[v] = Wj[v], hi_f[v] = f;
        }
    }
    const double tiny = 1e-6 * surface;
    const int any_tiny = smallest < tiny;
    if (any_tiny) {
        for (int v = 0; v < V; ++v) {
            lo[v] = DBL_MAX;
            hi[v] = -DBL_MAX;
        }
        for (int32_t k = first; k < end; ++k) {
            const int32_t e = fv->mesh.list[k];
            const int f = list_face(e);
            const int64_t j = e >= 0 ? fv->mesh.neighbour[f] : fv->mesh.owner[f];
            if (fv->mag[f] < tiny) continue;
            const double* Wj = fv->prims + (V + 2) * j;
            for (int v = 0; v < V; ++v) {
                if (Wj[v] < lo[v]) lo[v] = Wj[v], lo_f[v] = f;
                if (Wj[v] > hi[v]) hi[v] = Wj[v], hi_f[v] = f;
            }
        }
    }
    /* cholesky (finite_volume.hpp:677-687) */
    memset(fit, 0, sizeof(*fit));
    for (int p = 0; p < U; ++p)
        for (int s = 0; s <= p; ++s) {
            double sum = M[s][p];
            for (int m = 0; m < s; ++m) sum -= fit->Lc[p][m] * fit->Lc[s][m];
            fit->Lc[p][s] = p == s ? sqrt(sum) : sum / fit->Lc[s][s];
        }
    for (int p = 0; p < U; ++p) fit->M0[p] = M[0][p];
    double grad[VMAX * 3];
    solve_d(U, V, D, M, b, grad);
    memcpy(fit->g0, grad, sizeof(double) * V * D);
    int clip_f[VMAX];
    for (int v = 0; v < V; ++v) {
        fit->clipped[v] = fit->upper[v] = fit->zero[v] = 0;
        clip_f[v] = -1;
    }
    if (!fv->limiter_none)
        for (int32_t k = first; k < end; ++k) {
            const int f = list_face(fv->mesh.list[k]);
            if (any_tiny && fv->mag[f] < tiny) continue;
            double offset[3];
            face_offset(fv, f, i, offset);
            for (int v = 0; v < V; ++v) {
                double* g = grad + D * v;
                const double dp = dotd(D, g, offset);
                if (dp > 0 && Wi[v] + dp > hi[v]) {
                    const double s = hi[v] > Wi[v] ? (hi[v] - Wi[v]) / dp : 0.0;
                    for (int a = 0; a < D; ++a) g[a] = g[a] * s;
                    fit->clipped[v] = 1, fit->upper[v] = 1, fit->zero[v] = !(hi[v] > Wi[v]), clip_f[v] = f;
                } else if (dp < 0 && Wi[v] + dp < lo[v]) {
                    const double s = lo[v] < Wi[v] ? (lo[v] - Wi[v]) / dp : 0.0;
                    for (int a = 0; a < D; ++a) g[a] = g[a] * s;
                    fit->clipped[v] = 1, fit->upper[v] = 0, fit->zero[v] = !(lo[v] < Wi[v]), clip_f[v] = f;
                }
            }
        }
    for (int v = 0; v < V; ++v) {
        double offset[3] = {0, 0, 0};
        if (fit->clipped[v]) face_offset(fv, clip_f[v], i, offset);
        for (int a = 0; a < D; ++a) fit->offset[D * v + a] = offset[a];
        fit->bound[v] = fit->upper[v] ? hi[v] : lo[v];
        fit->bound_face[v] = fit->upper[v] ? hi_f[v] : lo_f[v];
    }
    memcpy(fv->grad + V * D * i, grad, sizeof(double) * V * D);
}

/* FaceFlux::side_value (finite_volume.hpp:1342-1347): the order-1 face state in double and whether it fell back. */
static int side_value(const lo_fv* fv, int64_t i, const double* r, double dt, double* Wf) {
    const int D = fv->D, V = fv->V;
    const double* W = fv->prims + (V + 2) * i;
    const double* g = fv->grad + V * D * i;
    lo_half_step(D, W, g, dt, &fv->gas, Wf);
    for (int v = 0; v < V; ++v) Wf[v] += dotd(D, g + D * v, r);
    const int fallback = !(Wf[0] > 0 && Wf[D + 1] > 0);
    if (fallback)
        for (int v = 0; v < V; ++v) Wf[v] = W[v];
    return fallback;
}

void lo_fv_step_adjoint(lo_fv* fv, double dt, double* qbar) {
    const int D = fv->D, V = fv->V, U = fv->U;
    const int64_t N = fv->n, F = fv->f;
    primitives(fv);
    fv->prims_ready = 1;
    fv->swept = 0;
    fit_t* fits = (fit_t*)malloc(sizeof(fit_t) * (size_t)N);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) sweep_fit_cell(fv, i, fits + i);
    /* AdjointFaces (finite_volume.hpp:2078-2102): the bars of both face states, one row per face */
    double* face_bar = (double*)calloc((size_t)F * 2 * V, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        const double* a = fv->mesh.area + D * f;
        const double magnitude = sqrt(dotd(D, a, a));
        double Lbar[VMAX] = {0, 0, 0, 0, 0}, Rbar[VMAX] = {0, 0, 0, 0, 0};
        if (magnitude != 0) {
            const int64_t o = fv->mesh.owner[f], j = fv->mesh.neighbour[f];
            double ro[3], rj[3], L[VMAX], R[VMAX], n[3], Fbar[VMAX], zero[3] = {0, 0, 0};
            face_offset(fv, f, o, ro);
            face_offset(fv, f, j, rj);
            side_value(fv, o, ro, dt, L);
            side_value(fv, j, rj, dt, R);
            for (int v = 0; v < V; ++v) Fbar[v] = magnitude * dt * (qbar[V * j + v] - qbar[V * o + v]);
            const double inv = 1.0 / magnitude;
            for (int k = 0; k < D; ++k) n[k] = a[k] * inv;
            if (fv->riemann == 1)
                hll_flux_adjoint(D, L, R, n, zero, &fv->gas, Fbar, Lbar, Rbar);
            else
                hllc_flux_adjoint(D, L, R, n, zero, &fv->gas, Fbar, Lbar, Rbar);
        }
        for (int v = 0; v < V; ++v) {
            face_bar[2 * V * f + v] = Lbar[v];
            face_bar[2 * V * f + V + v] = Rbar[v];
        }
    }
    /* AdjointCell (finite_volume.hpp:2107-2169) */
    double* wbar = (double*)calloc((size_t)N * V, sizeof(double));
    double* bbar = (double*)calloc((size_t)N * V * U, sizeof(double));
    double* boundbar = (double*)calloc((size_t)N * V, sizeof(double));
    int* bound_face = (int*)calloc((size_t)N * V, sizeof(int));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        const double* Wi = fv->prims + (V + 2) * i;
        const double* gi = fv->grad + V * D * i;
        double Wi_bar[VMAX] = {0, 0, 0, 0, 0}, gi_bar[VMAX * 3];
        memset(gi_bar, 0, sizeof(gi_bar));
        for (int32_t k = fv->mesh.start[i]; k < fv->mesh.start[i + 1]; ++k) {
            const int32_t e = fv->mesh.list[k];
            const int f = list_face(e);
            const double* a = fv->mesh.area + D * f;
            if (dotd(D, a, a) == 0) continue;
            const double* mine = face_bar + 2 * V * f + (e >= 0 ? 0 : V);
            double r[3], Wf[VMAX];
            face_offset(fv, f, i, r);
            const int fallback = side_value(fv, i, r, dt, Wf);
            if (fallback) {
                for (int v = 0; v < V; ++v) Wi_bar[v] += mine[v];
            } else {
                for (int v = 0; v < V; ++v)
                    for (int q = 0; q < D; ++q) gi_bar[D * v + q] = gi_bar[D * v + q] + r[q] * mine[v];
                half_step_adjoint(D, Wi, gi, dt, &fv->gas, mine, Wi_bar, gi_bar);
            }
        }
        const fit_t* ft = fits + i;
        double xbar[VMAX][UMAX], bsol[VMAX][UMAX], self[VMAX], bnd[VMAX];
        int face[VMAX];
        for (int v = 0; v < V; ++v) {
            const double* g0 = ft->g0 + D * v;
            double g0bar[3];
            for (int a = 0; a < D; ++a) g0bar[a] = gi_bar[D * v + a];
            self[v] = 0;
            bnd[v] = 0;
            face[v] = -1;
            if (ft->clipped[v] && ft->zero[v]) {
                for (int a = 0; a < D; ++a) g0bar[a] = 0;
            } else if (ft->clipped[v]) {
                const double* o = ft->offset + D * v;
                const double den = dotd(D, g0, o);
                const double s = (ft->bound[v] - Wi[v]) / den, t = dotd(D, gi_bar + D * v, g0) / den;
                for (int a = 0; a < D; ++a) g0bar[a] = gi_bar[D * v + a] * s - o[a] * (s * t);
                bnd[v] = t;
                face[v] = ft->bound_face[v];
                self[v] -= t;
            }
            xbar[v][0] = 0;
            for (int a = 0; a < D; ++a) xbar[v][1 + a] = g0bar[a];
        }
        /* solve_factored (finite_volume.hpp:688-702): b bar = M^-1 x bar */
        for (int v = 0; v < V; ++v) {
            double z[UMAX];
            for (int p = 0; p < U; ++p) {
                double sum = xbar[v][p];
                for (int m = 0; m < p; ++m) sum -= ft->Lc[p][m] * z[m];
                z[p] = sum / ft->Lc[p][p];
            }
            for (int p = U - 1; p >= 0; --p) {
                double sum = z[p];
                for (int m = p + 1; m < U; ++m) sum -= ft->Lc[m][p] * bsol[v][m];
                bsol[v][p] = sum / ft->Lc[p][p];
            }
        }
        for (int v = 0; v < V; ++v) {
            for (int p = 0; p < U; ++p) self[v] -= ft->M0[p] * bsol[v][p];
            wbar[V * i + v] = Wi_bar[v] + self[v];
            for (int p = 0; p < U; ++p) bbar[(size_t)(U * V) * i + U * v + p] = bsol[v][p];
            boundbar[V * i + v] = bnd[v];
            bound_face[V * i + v] = face[v];
        }
    }
    /* AdjointGather (finite_volume.hpp:2171-2195) */
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < N; ++j) {
        double W_bar[VMAX];
        for (int v = 0; v < V; ++v) W_bar[v] = wbar[V * j + v];
        const double* cj = fv->mesh.centroid + D * j;
        for (int32_t k = fv->mesh.start[j]; k < fv->mesh.start[j + 1]; ++k) {
            const int32_t e = fv->mesh.list[k];
            const int f = list_face(e);
            const int64_t i = e >= 0 ? fv->mesh.neighbour[f] : fv->mesh.owner[f];
            double sep[3], between[3];
            separation(fv, i, j, sep);
            for (int a = 0; a < D; ++a) between[a] = sep[a] + cj[a] - fv->mesh.centroid[D * i + a];
            const double w = fv->mag[f];
            for (int v = 0; v < V; ++v) {
                const double* bb = bbar + (size_t)(U * V) * i + U * v;
                double sum = bb[0];
                for (int p = 1; p < U; ++p) sum += between[p - 1] * bb[p];
                W_bar[v] += w * sum + (bound_face[V * i + v] == f ? boundbar[V * i + v] : 0.0);
            }
        }
        const double inv = 1.0 / fv->mesh.volume[j];
        double Uj[VMAX], U_bar[VMAX];
        for (int v = 0; v < V; ++v) Uj[v] = fv->q[V * j + v] * inv;
        primitive_adjoint(D, Uj, W_bar, &fv->gas, U_bar);
        for (int v = 0; v < V; ++v) qbar[V * j + v] += U_bar[v] * inv;
    }
    free(fits);
    free(face_bar);
    free(wbar);
    free(bbar);
    free(boundbar);
    free(bound_face);
}
