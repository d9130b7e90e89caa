/* CPU oracle of luna-cpp's per-step finite-volume hydro update: TEST INFRASTRUCTURE ONLY.
 *
 * A plain C restatement of the reference's algorithm (src/hydro/euler.hpp, src/hydro/finite_volume.hpp), used by the
 * tests as the checker of the CUDA path and by bench.py as the timed CPU baseline. Nothing in the product links it.
 * Each function cites the reference lines it follows. Arithmetic is IEEE double in the reference's operation order,
 * compiled without multiply-add contraction.
 *
 * Pinned by: LUNA's HLL/HLLC golden fluxes (src/test/hydro_test.cpp:48-80, to 1e-14), the flux invariants
 * (hydro_test.cpp:106-132), and the mesh invariants (uniform state, conservation, determinism; hydro_test.cpp:185-274).
 * The whole 3D step depends on voronoi-cpp's mesh, which is absent: its parity with the reference is pinned only through
 * those invariants (see the tests).
 */
#ifndef LUNA_ORACLE_H
#define LUNA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double gamma, smallr, smallc, inverse_gm1;
    float inverse_gm1_float;
} lo_gas;

/* voronoi-cpp's arrays (finite_volume.hpp:257-327), host pointers. */
typedef struct {
    int dim;
    int64_t n, f;
    const int32_t *owner, *neighbour, *start, *list;
    const double *area, *face_centroid, *centroid, *volume, *positions;
    double box[3];
} lo_mesh;

typedef struct lo_fv lo_fv;

void lo_gas_init(lo_gas* gas, double gamma);

/* euler.hpp: per-state functions (D = 2 or 3, states of D + 2 entries). */
void lo_primitive(int D, const double* U, const lo_gas* gas, double* W);
void lo_conserved(int D, const double* W, const lo_gas* gas, double* U);
void lo_half_step(int D, const double* W, const double* g /* [V][D] */, double dt, const lo_gas* gas, double* out);
void lo_hllc_flux(int D, const double* L, const double* R, const double* n, const double* w, const lo_gas* gas, double* F);
void lo_hll_flux(int D, const double* L, const double* R, const double* n, const double* w, const lo_gas* gas, double* F);
/* The float Riemann solve (T = float), as FaceFlux::solve runs it for a float policy (finite_volume.hpp:1400-1413). */
void lo_hllc_flux_float(int D, const float* L, const float* R, const float* n, const lo_gas* gas, float* F);

/* FiniteVolume<D> (static or moving mesh, order 0/1, per-face or per-cell update, face-centroid limiter or none,
 * HLLC (riemann 0) or HLL (1)). grad_float: the Grad32 policy (gradients, limiter, face-state change in float). */
lo_fv* lo_fv_create(const lo_mesh* mesh, const lo_gas* gas, int order, int per_face, int limiter_none, int riemann,
                    int moving, int grad_float, int riemann_float);
void lo_fv_destroy(lo_fv* fv);
double* lo_fv_state(lo_fv* fv); /* Q [N][V], extensive; writing it marks the primitives stale */
void lo_fv_state_changed(lo_fv* fv);
double lo_fv_time_step(lo_fv* fv, double courant);
/* The Grad16 policy (grad_float and on): the float gradients stored as binary16 with one power-of-two exponent per group
 * rho, v, P (finite_volume.hpp:616-641), so the flux reads them rounded. */
void lo_fv_set_half_gradients(lo_fv* fv, int on);
/* The flux rows of the per-face loop stored in float (Precision::flux = float, the reference's `single` preset). */
void lo_fv_set_float_fluxes(lo_fv* fv, int on);
void lo_fv_step(lo_fv* fv, double dt);
int64_t lo_fv_fallbacks(const lo_fv* fv);
int lo_fv_threads(int threads); /* sets the OpenMP thread count (<= 0: all); returns the count in use */
/* Rows of the last sweep: prims [N][V + 2] (W, c, r) and gradients [N][V * D] (double). */
const double* lo_fv_prims(const lo_fv* fv);
const double* lo_fv_gradients(const lo_fv* fv);
/* Moving mesh: point velocities of the last sweep [N][D]; positions [N][D]. */
const double* lo_fv_point_velocities(const lo_fv* fv);
/* Moving step in two halves around the caller's remesh (step_moving, finite_volume.hpp:1497-1519):
 * begin snaps the points, keeps the centroids, applies the t^n fluxes (half dt) and writes the new positions
 * [N][D] (on the grid) into positions_out; the caller builds the mesh of those positions and passes it to end. */
void lo_fv_step_moving_begin(lo_fv* fv, double dt, double* positions_out);
void lo_fv_step_moving_end(lo_fv* fv, const lo_mesh* new_mesh);
/* The adjoint of one static step at fixed dt (step_adjoint, finite_volume.hpp:2201-2231): qbar <- J^T qbar, with the
 * forward state Q^n in the object. */
void lo_fv_step_adjoint(lo_fv* fv, double dt, double* qbar);

/* The snapping grid of a box (voronoi-cpp's exact_predicates): step = 2^-30 of the longest side. */
double lo_grid_step(int D, const double* box);

/* FiniteVolume<1> on a static line (oracle_line.c; src/hydro/finite_volume_1d.hpp). keys: the generators' sorted grid
 * keys in [0, period]; walls: LO_WALL_* left, right (ignored when periodic); inflow: [2][3] primitives of inflow walls;
 * limiter: LO_LIMITER_*; riemann: 0 HLLC, 1 HLL. The state is Q [n][3] in slot (key) order. */
enum { LO_WALL_REFLECTIVE = 0, LO_WALL_OUTFLOW = 1, LO_WALL_INFLOW = 2 };
enum { LO_LIMITER_FACE_CENTROID = 0, LO_LIMITER_NONE = 1, LO_LIMITER_MINMOD = 2, LO_LIMITER_VAN_LEER = 3 };
typedef struct lo_line lo_line;
lo_line* lo_line_create(int n, const int64_t* keys, int64_t period, double step, int periodic, const int* walls, const double* inflow,
                        const lo_gas* gas, int order, int limiter, int riemann);
void lo_line_destroy(lo_line* ln);
double* lo_line_state(lo_line* ln);
const double* lo_line_volumes(const lo_line* ln);
const double* lo_line_centroids(const lo_line* ln);
double lo_line_time_step(const lo_line* ln, double courant, int rule /* 0 AREPO's, 1 LUNA's */);
void lo_line_step(lo_line* ln, double dt);

/* FiniteVolume<1> on a moving line (oracle_mline.c; finite_volume_1d.hpp with Motion::moving): n generators at
 * `positions` (cell order) on [0, length]; Q [cells][3] and x [cells] in cell order (cells supplied by a wall are
 * appended); regularise: AREPO-ng's point-velocity regularisation. lo_mline_state / lo_mline_positions point at arrays
 * that move with each step: fetch them again after one. */
typedef struct lo_mline lo_mline;
lo_mline* lo_mline_create(int n, const double* positions, double length, int periodic, const int* walls, const double* inflow,
                          const lo_gas* gas, int order, int limiter, int riemann, int regularise);
void lo_mline_destroy(lo_mline* ml);
int lo_mline_cells(const lo_mline* ml);
double* lo_mline_state(lo_mline* ml);
double* lo_mline_positions(lo_mline* ml);
void lo_mline_geometry(const lo_mline* ml, double* generator, double* volume, double* centroid);
void lo_mline_stats(const lo_mline* ml, long long* added, long long* sorts, long long* updates);
void lo_mline_set_inflow_spacing(lo_mline* ml, double spacing);
int lo_mline_supply_cells(lo_mline* ml);
double lo_mline_time_step(lo_mline* ml, double courant, int rule /* 0 AREPO's, 1 LUNA's */);
void lo_mline_step(lo_mline* ml, double dt);
double lo_mline_step_and_time_step(lo_mline* ml, double dt, double courant);

#ifdef __cplusplus
}
#endif

#endif
