/* The moving mesh's remesh on the device.
 *
 * luna-cpp's moving step drifts the generators and updates the Voronoi mesh between its two flux passes
 * (FiniteVolume::move(), src/hydro/finite_volume.hpp:1212-1250: mesh_->update(x_), mesh_->update_cells(), refresh()).
 * voronoi-cpp does that update on the device by repairing the previous tetrahedralisation (README.md:92-94). This
 * library rebuilds the mesh from the drifted generators on the device instead, each cell clipped by one thread with the
 * host builder's code, so the arrays equal luna_mesh_create's (libluna_mesh) bit for bit, in the layout
 * luna_fv_step_moving_end reads (faces by owner, then neighbour; lists by neighbour; ~f for a face the cell does not
 * own).
 */
#ifndef LUNA_REMESH_H
#define LUNA_REMESH_H

#include "luna_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct luna_remesh luna_remesh;

/* A remesher for dim 2 or 3 in the periodic box [0, box_a) per axis; its device buffers grow with the meshes it builds
 * and are kept between builds. */
LUNA_API luna_status luna_remesh_create(int dim, const double* box, luna_remesh** out);
LUNA_API luna_status luna_remesh_destroy(luna_remesh* r);
/* The stream its kernels run on (cudaStream_t; NULL = the legacy default stream). */
LUNA_API luna_status luna_remesh_set_stream(luna_remesh* r, void* stream);

/* A device buffer of n x dim doubles owned by r (kept until a larger one is asked for or r is destroyed) for the caller
 * to write generators into, e.g. luna_fv_step_moving_begin(fv, dt, *points, 1), then luna_remesh_build(r, n, *points,
 * 1, ...). */
LUNA_API luna_status luna_remesh_points(luna_remesh* r, int64_t n, double** points);

/* The periodic Voronoi mesh of n generators points [n][dim] (host or device memory; wrapped into the box). On return
 * *mesh holds device pointers owned by r (valid until the next build or luna_remesh_destroy) and *inconsistent the
 * faces seen from one side only (kept from the side that saw them, as luna_mesh_create keeps them). Synchronises on
 * r's stream (the face count is read back). Errors: LUNA_EINVAL for n out of [2, 2^30), a non-finite point or a cell
 * that cannot be built (box too small for the points, points too sparse for the bucket search, a cell of more than 48 faces).
 */
LUNA_API luna_status luna_remesh_build(luna_remesh* r, int64_t n, const double* points, int on_device, luna_mesh_desc* mesh,
                                       int64_t* inconsistent);

/* Device bytes r holds. */
LUNA_API luna_status luna_remesh_device_bytes(const luna_remesh* r, int64_t* out);

#ifdef __cplusplus
}
#endif

#endif
