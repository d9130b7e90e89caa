/* Periodic Voronoi mesh builder (host, C ABI).
 *
 * The hydro library consumes face lists in the layout voronoi-cpp's Mesh emits (owner/neighbour per face, a per-cell
 * CSR list of faces where a negative entry ~f marks a face the cell does not own, area vectors owner -> neighbour, face
 * centroids relative to the owner's generator, cell centroids relative to the cell's generator). voronoi-cpp is not part
 * of this project, so this builder produces that layout from generating points in a periodic box: each cell is the
 * periodic box around its generator clipped by the bisector planes (2D: lines) of nearby generators, found through a
 * bucket grid. It is infrastructure for tests, benchmarks and examples, not part of the hydro step.
 */
#ifndef LUNA_MESH_H
#define LUNA_MESH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct luna_mesh_build luna_mesh_build;

/* Arrays of a built mesh (owned by the builder; valid until luna_mesh_free). Row-major, D = dim. */
typedef struct {
    int dim;
    int64_t n_cells, n_faces;
    const int32_t* owner;           /* [F] */
    const int32_t* neighbour;       /* [F] */
    const int32_t* cell_face_start; /* [N + 1] */
    const int32_t* cell_face;       /* [2F]: f if the cell owns face f, ~f otherwise */
    const double* area;             /* [F][D] owner -> neighbour */
    const double* face_centroid;    /* [F][D] relative to the owner's generator */
    const double* centroid;         /* [N][D] relative to the cell's generator */
    const double* volume;           /* [N] */
    const double* positions;        /* [N][D] generators wrapped into [0, side) */
    double box[3];
    int64_t inconsistent;           /* faces seen from one side only (kept, from the side that saw them) */
} luna_mesh_arrays;

/* Builds the periodic Voronoi mesh of n points (row-major [n][dim]) in the box [0, side_a) per axis.
 * threads <= 0: all OpenMP threads. Returns 0 on success, non-zero on error (message in luna_mesh_error()). */
int luna_mesh_create(int dim, int64_t n, const double* points, const double* box, int threads, luna_mesh_build** out);
int luna_mesh_arrays_of(const luna_mesh_build* m, luna_mesh_arrays* out);
void luna_mesh_free(luna_mesh_build* m);
const char* luna_mesh_error(void);

/* The jittered lattice of problems_3d.hpp's jittered_points (mt19937_64 seeded `seed`, uniform(-jitter, jitter) spacings
 * per axis, lattice point (i + 1/2) h, wrapped into [0, side)), loops i, j (, k) with the last axis fastest.
 * cells: lattice size per axis (dim entries), side: box edges; out: [prod(cells)][dim]. */
int luna_jittered_points(int dim, const int* cells, const double* side, double jitter, uint64_t seed, double* out);

#ifdef __cplusplus
}
#endif

#endif
