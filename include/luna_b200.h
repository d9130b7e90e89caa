/* libluna_b200: luna-cpp's per-step finite-volume hydro update on a periodic Voronoi mesh, on one B200 (sm_100a).
 *
 * The C ABI a drop-in for luna-cpp's hydro::FiniteVolume<D, Exec, Riemann, Precision> (src/hydro/finite_volume.hpp):
 * the same call order (time_step(courant) -> dt, then step(dt); a moving mesh remeshes between the two flux passes of a
 * step), the same mesh arrays (voronoi-cpp's face lists as emitted), the same extensive conserved state Q[N][D + 2].
 * Plain pointers and sizes only; no exceptions cross the boundary: every call returns a luna_status and the message of
 * the last failure on this thread is in luna_last_error(). The library owns all device memory of a luna_fv; the caller's
 * mesh arrays may be freed after luna_fv_create / luna_fv_set_mesh. A luna_fv is thread-compatible, not thread-safe.
 * All kernels of a luna_fv run on its stream; the only host synchronisations are the reads of dt, of the fallback count
 * and of states copied to host memory.
 */
#ifndef LUNA_B200_H
#define LUNA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define LUNA_API __attribute__((visibility("default")))
#else
#define LUNA_API
#endif

typedef enum {
    LUNA_OK = 0,
    LUNA_EINVAL = 1,      /* bad argument (the reference throws std::invalid_argument / logic_error) */
    LUNA_ENOMEM = 2,      /* a device or host allocation failed */
    LUNA_ECUDA = 3,       /* a CUDA call failed (message in luna_last_error) */
    LUNA_ENONFINITE = 4,  /* a kernel found a non-finite dt, flux or state (error word set) */
    LUNA_ETIMEOUT = 5,    /* a bounded device-side wait gave up */
    LUNA_ESTATE = 6       /* call out of order (e.g. step_moving_end without begin) */
} luna_status;

enum { LUNA_UPDATE_PER_CELL = 0, LUNA_UPDATE_PER_FACE = 1 };            /* hydro::Update (finite_volume.hpp:25) */
enum { LUNA_LIMITER_FACE_CENTROID = 0, LUNA_LIMITER_NONE = 1 };         /* hydro::Limiter (finite_volume.hpp:29) */
enum { LUNA_LIMITER_MINMOD = 2, LUNA_LIMITER_VAN_LEER = 3 };            /* the 1D slopes (finite_volume_1d.hpp:187-192) */
enum { LUNA_WALL_REFLECTIVE = 0, LUNA_WALL_OUTFLOW = 1, LUNA_WALL_INFLOW = 2 }; /* hydro::Wall (finite_volume_1d.hpp:9) */
enum { LUNA_STATIC_MESH = 0, LUNA_MOVING = 1 };                         /* hydro::Motion (finite_volume.hpp:31) */
enum { LUNA_HLLC = 0, LUNA_HLL = 1 };                                   /* Riemann parameter (euler.hpp:444, :546) */
/* Precision policies (precision.hpp:26-54): LUNA_FP64 is Precision<> (double throughout); LUNA_FP32 is the reference's
 * `riemann32` preset Precision<double, float, double, float> (hydro_sedov.cpp:422): gradients, limiter, face-state change
 * and the Riemann solve in float in the face's frame; geometry, primitives (pressure recovery), flux rows and the
 * per-cell accumulation in double. LUNA_GRAD32 is the reference's Grad32 (precision.hpp:43): float gradients, limiter and
 * face-state change, a double Riemann solve (it keeps perturbations far below float's resolution of the state, which
 * a float Riemann solve cannot). The reduced policies take HLLC only, as the reference's presets. */
enum { LUNA_FP64 = 0, LUNA_FP32 = 1, LUNA_GRAD32 = 2, LUNA_GRAD16 = 3, LUNA_SINGLE = 4 };
/* LUNA_SINGLE is the reference's `single` preset Precision<double, float, float, float> (hydro_sedov.cpp:423): LUNA_FP32
 * with the per-face flux rows stored in float (each flux rounded once, summed per cell in double), 32 B a row in 3D
 * instead of 40; the per-cell loop stores no rows, so there it is LUNA_FP32. */
/* LUNA_GRAD16 is the reference's Grad16 (precision.hpp:47, its 3D default): Grad32 with the gradient rows stored as
 * binary16 (32 B a row) and one power-of-two exponent per group rho, v, P (4 B a cell). */

/* hydro::Gas (euler.hpp:82-101): gamma and the RAMSES floors. */
typedef struct {
    double gamma;
    double smallr; /* 1e-10 in the reference */
    double smallc; /* 1e-10 in the reference */
} luna_gas;

/* voronoi-cpp's mesh arrays as FiniteVolume::refresh() reads them (finite_volume.hpp:353-364), row-major, D = dim.
 * cell_face entries carry the owner bit: f if the cell owns face f, ~f otherwise (Geometry::owned_at, :318). */
typedef struct {
    int dim;                          /* 2 or 3 */
    int64_t n_cells, n_faces;
    const int32_t* owner;             /* [F] */
    const int32_t* neighbour;         /* [F] */
    const int32_t* cell_face_start;   /* [N + 1] */
    const int32_t* cell_face;         /* [2F] */
    const double* area;               /* [F][D], owner -> neighbour */
    const double* face_centroid;      /* [F][D], relative to the owner's generator */
    const double* centroid;           /* [N][D], relative to the cell's generator */
    const double* volume;             /* [N] */
    const double* positions;          /* [N][D], generators in [0, box) */
    double box[3];                    /* periodic box sides */
    int on_device;                    /* 1: the pointers are device pointers of the current device */
} luna_mesh_desc;

typedef struct luna_fv luna_fv;

/* FiniteVolume(exec, mesh, gas, order, update, limiter, motion) (finite_volume.hpp:79-107) with the Riemann and
 * Precision template parameters as arguments. order 0 or 1 (else LUNA_EINVAL, as the reference's invalid_argument).
 * A moving mesh requires the per-face update. */
LUNA_API luna_status luna_fv_create(const luna_mesh_desc* mesh, const luna_gas* gas, int order, int update, int limiter,
                                    int motion, int riemann, int precision, luna_fv** out);
LUNA_API luna_status luna_fv_destroy(luna_fv* fv);

/* The stream all kernels of fv run on (cudaStream_t; NULL = the legacy default stream). */
LUNA_API luna_status luna_fv_set_stream(luna_fv* fv, void* stream);

/* state() (finite_volume.hpp:145-148): the device array Q[N][D + 2]; the caller may write it, so the primitive rows are
 * recomputed by the next time_step(). */
LUNA_API luna_status luna_fv_state(luna_fv* fv, double** dev_q);
LUNA_API luna_status luna_fv_set_state(luna_fv* fv, const double* q, int on_device);
LUNA_API luna_status luna_fv_get_state(luna_fv* fv, double* q, int on_device);

/* time_step(courant) (finite_volume.hpp:190-201): primitives, the sweep (limited gradients, point velocities), the CFL
 * reduction; writes dt (AREPO's rule, finite_volume.hpp:1040-1104). Synchronises on the read of dt. */
LUNA_API luna_status luna_fv_time_step(luna_fv* fv, double courant, double* dt_out);
/* step(dt) (finite_volume.hpp:205-226) on a static mesh: face fluxes and the cell update. Asynchronous. */
LUNA_API luna_status luna_fv_step(luna_fv* fv, double dt);
/* fallbacks() (finite_volume.hpp:230-238): face sides of the last step that fell back to the cell's state. */
LUNA_API luna_status luna_fv_fallbacks(luna_fv* fv, int64_t* out);
/* The error word of the kernels since the last call (bit 0: non-finite dt term, bit 1: non-finite state after an update,
 * bit 2: a list entry out of range, bit 4: the learned limiter's tensor-core completion wait gave up); cleared by the
 * read. */
LUNA_API luna_status luna_fv_error_word(luna_fv* fv, uint32_t* out);

/* The moving step (step_moving, finite_volume.hpp:1497-1519), split around the caller's remesh because the mesh update
 * belongs to the mesh library: begin snaps the points to the mesh grid (2^-30 of the longest side), keeps the
 * centroids of t^n, applies the t^n fluxes at dt/2 and drifts the points; it writes the new generator positions
 * [N][D] (host or device memory) for the caller's remesh. end takes the t^n+1 mesh (same cells, same order) and
 * applies its fluxes at dt/2. Order 0 (step(): advance<0, true>() then move(), :205-226, :1212-1228): begin applies the
 * fluxes of the current mesh at dt (each side the cell's W, the face velocities from the point velocities) and drifts
 * the points off the grid (x + dt w, wrapped); end takes the new mesh. */
LUNA_API luna_status luna_fv_step_moving_begin(luna_fv* fv, double dt, double* positions_out, int on_device);
LUNA_API luna_status luna_fv_step_moving_end(luna_fv* fv, const luna_mesh_desc* new_mesh);
/* A static mesh replaced by another of the same cells (checkpoint restore; FiniteVolume::mesh_moved). */
LUNA_API luna_status luna_fv_set_mesh(luna_fv* fv, const luna_mesh_desc* mesh);
/* positions() / point_velocities() (finite_volume.hpp:150-158): [N][D], host or device memory. */
LUNA_API luna_status luna_fv_positions(luna_fv* fv, double* out, int on_device);
LUNA_API luna_status luna_fv_point_velocities(luna_fv* fv, double* out, int on_device);
/* The primitive rows [N][D + 4] (W, c, r) and the limited gradients [N][D + 2][D] (double) of the last sweep. */
LUNA_API luna_status luna_fv_prims(luna_fv* fv, double* out, int on_device);
LUNA_API luna_status luna_fv_gradients(luna_fv* fv, double* out, int on_device);

/* step_adjoint(dt, qbar) (finite_volume.hpp:2201-2231): qbar [N][D + 2] holds Qbar after the step on entry and
 * Qbar before it on return (J^T qbar at fixed dt; dt's dependence on Q is not differentiated). Q must be the state at
 * the start of the step (the caller restores it from a checkpoint); it is left unchanged. A static mesh, order 1, the
 * per-face loop and the FP64 policy (else LUNA_EINVAL, as the reference's logic_error, :1674-1679). No atomics: the
 * same bits every run. */
LUNA_API luna_status luna_fv_step_adjoint(luna_fv* fv, double dt, double* qbar, int on_device);
/* step_tangent(dt, dq) (finite_volume.hpp:2023-2062): the step of step(dt) and, beside it, dq [N][D + 2] <- J dq (the
 * tangent of Q, extensive) at fixed dt, linearised at the same point as luna_fv_step_adjoint (so the two are transposes:
 * <J dq, qbar> = <dq, J^T qbar>). Q advances as luna_fv_step(fv, dt) advances it. The same restrictions as the adjoint. */
LUNA_API luna_status luna_fv_step_tangent(luna_fv* fv, double dt, double* dq, int on_device);

/* The moving step's derivatives at fixed topology (step_moving_tangent / step_moving_adjoint, finite_volume.hpp:
 * 2431-3155): the state is (Q, x); a moving mesh, the per-face loop, the FP64 policy, dt fixed, outside a moving step. The geometry's own derivative in the generators (V, c, A, x_f) belongs to the mesh
 * library (GeometryDerivative, mesh_derivative.hpp:10-29): the tangent takes its tangents, the adjoint hands back its
 * bars. All arrays host or all device memory (on_device); Q's rows [N][D + 2], x's [N][D], V's [N], c's [N][D], A's and
 * x_f's [F][D].
 * tangent: dq, dx (of Q, x at the step's start) become those after the step; dV, dc, dA, dxf are GeometryDerivative::
 * tangent(dx) of the current mesh. Nothing steps: the caller then runs the step (begin, remesh, end).
 * adjoint: qbar, xbar (of Q, x after the step) become those at its start, but for the geometry's part: Vbar, cbar, Abar,
 * xfbar are written, and the caller adds GeometryDerivative::adjoint(Vbar, cbar, Abar, xfbar) to xbar. Q and the mesh
 * must be the step's start; nothing steps. No atomics: the same bits every run.
 * Order 1 (the two-pass MUSCL-Hancock step, step_moving_tangent_1 / step_moving_adjoint_1, :2767-3155; the grid steps'
 * quantisation taken as the identity) needs the mesh of t^n+1 between its passes, so each runs in parts around the
 * caller's step:
 *   tangent: luna_fv_step_moving_tangent (the first pass's tangent; dx becomes x^n+1's tangent), the step (begin,
 *   remesh, end), then luna_fv_step_moving_tangent_end with GeometryDerivative::tangent(dx) of the new mesh (the
 *   second pass's tangent, into dq).
 *   adjoint, at the step's start: luna_fv_step_moving_adjoint_begin; the step; luna_fv_step_moving_adjoint_new_mesh
 *   (qbar, xbar of Q, x after the step: xbar gains the second pass's bars, Abar and xfbar are the new mesh's for the
 *   caller's GeometryDerivative::adjoint, which the caller adds to xbar); the caller restores Q and the mesh of t^n;
 *   then luna_fv_step_moving_adjoint as for order 0 (qbar, xbar become those at the step's start, but for the
 *   geometry's part of t^n, handed back in Vbar, cbar, Abar, xfbar). */
LUNA_API luna_status luna_fv_step_moving_tangent(luna_fv* fv, double dt, double* dq, double* dx, const double* dV, const double* dc,
                                                 const double* dA, const double* dxf, int on_device);
/* The reference's steps_fixed argument of the order-1 derivatives: the grid steps of the moving points held (no
 * derivative through w-hat), as central differences small enough to change no step see it. Off by default. */
LUNA_API luna_status luna_fv_set_steps_fixed(luna_fv* fv, int held);
LUNA_API luna_status luna_fv_step_moving_tangent_end(luna_fv* fv, double dt, double* dq, const double* dx, const double* dV, const double* dc,
                                                     const double* dA, const double* dxf, int on_device);
LUNA_API luna_status luna_fv_step_moving_adjoint_begin(luna_fv* fv, double dt);
LUNA_API luna_status luna_fv_step_moving_adjoint_new_mesh(luna_fv* fv, double dt, const double* qbar, double* xbar, double* Abar,
                                                          double* xfbar, int on_device);
LUNA_API luna_status luna_fv_step_moving_adjoint(luna_fv* fv, double dt, double* qbar, double* xbar, double* Vbar, double* cbar, double* Abar,
                                                 double* xfbar, int on_device);

/* Per-phase device time (hydro::Timings, finite_volume.hpp:36-39, without its fences): with timing on, CUDA events on
 * fv's stream bracket every kernel; luna_fv_timings synchronises, adds the elapsed times since the last reset and counts
 * the launches per phase. Phases: 0 primitives, 1 sweep (gradients, limiter, point velocities, CFL reduction),
 * 2 fluxes, 3 update, 4 drift (the moving step's snapping and drift). */
typedef struct {
    double ms[5];
    int64_t launches[5];
} luna_timings;
LUNA_API luna_status luna_fv_set_timing(luna_fv* fv, int on);
LUNA_API luna_status luna_fv_timings(luna_fv* fv, luna_timings* out, int reset);

/* The learned slope limiter (no counterpart in the reference; the plain face-centroid limiter, Sweep's walk 2,
 * finite_volume.hpp:538-565, is its fallback and its judge). In the sweep each variable's admissible factor alpha (the
 * largest scaling of the unlimited gradient that keeps every face-centroid value within the neighbours' range, capped
 * at 2) and 32 features are computed; a 3-layer MLP (width 64, BF16 tensor-core MMA, FP32 accumulation) maps the
 * features to logits o; the gradient is scaled by alpha * sigmoid(o) in [0, alpha]: monotone by construction.
 * mode 0: the plain limiter; mode 1: the network with parameters `params` (device, luna_mlp_param_count() floats, kept
 * by the caller); mode 2: the factors min(alpha, 1), the plain limiter in min-factor form through the same path.
 * Order 1, the FP64 policy, the face-centroid limiter. */
LUNA_API luna_status luna_fv_set_limiter_mlp(luna_fv* fv, const float* params, int mode);
/* The limiter's inputs for the current state (device buffers): features [N][32] BF16, alpha [N][D + 2] (double, in rows
 * of 5), and the unlimited gradients [N][D + 2][D] (double). For building training data. */
LUNA_API luna_status luna_fv_limiter_inputs(luna_fv* fv, void* features, double* alpha, double* gradients);
/* The network's kernels on caller buffers (device): parameters FP32 [luna_mlp_param_count()]; features BF16 [n][32];
 * logits FP32 [n][16] (the first D + 2 used); features and logits 16-byte aligned. forward: on the 5th-generation tensor
 * cores (tcgen05, accumulators in tensor memory); it synchronises the stream to read its completion status
 * (LUNA_ETIMEOUT if a bounded wait gave up). train_step: the gradient of scale * sum w (sigmoid(o) - t)^2 over rows
 * (targets t and weights w FP32 [n][5]) into grad, the loss into *loss (device); workspace of
 * luna_mlp_train_workspace_floats(n) floats; deterministic. adam: one Adam update (step counts from 1). */
LUNA_API int64_t luna_mlp_param_count(void);
/* The polls a tensor-core completion wait of the learned limiter's forward makes before it gives up (LUNA_ETIMEOUT from
 * luna_mlp_forward and from the learned step's luna_fv_time_step), for every later launch in this process; < 0 restores
 * the default (2^22). After giving up, a CTA still waits for its MMA in flight with the default bound before it frees
 * tensor memory. Returns the previous limit. No counterpart in the reference (it has no learned limiter). */
LUNA_API int luna_mlp_set_wait_limit(int polls);
LUNA_API int64_t luna_mlp_train_workspace_floats(int64_t n);
LUNA_API luna_status luna_mlp_forward(const float* params, const void* features, int64_t n, float* logits, void* stream);
LUNA_API luna_status luna_mlp_train_step(const float* params, const void* features, const float* target, const float* weight, int64_t n,
                                         float scale, float* grad, float* loss, float* workspace, int64_t workspace_floats, void* stream);
LUNA_API luna_status luna_mlp_adam(float* params, const float* grad, float* m, float* v, float lr, float beta1, float beta2, float eps,
                                   int step, void* stream);

/* The flux-and-update pass of one static step (apply(), per-face loop) that allocates nothing, for callers that cannot
 * allocate device memory themselves: code that must run with a fixed device footprint, or under a runtime or memory
 * pool that owns every device allocation and hands the caller only finished buffers. It has no counterpart in the
 * reference (whose steps always borrow scratch from the mesh or allocate it).
 * The caller passes everything in device memory: the mesh arrays (mesh->on_device must be 1), Q [N][D + 2] (updated in
 * place: Q -= dt * sum of the face fluxes, in list order), and at order 1 the primitive rows [N][8] (W, c, r, then
 * padding) and the gradient rows (3D: [N][16], 2D: [N][8]; dW_v/dx_d at v * D + d, then padding) of the step's sweep.
 * The per-face flux rows go to one fixed device array of 32 MiB inside the library, so a mesh may have at most
 * 838,854 faces in 3D (1,048,568 in 2D); larger meshes are rejected with LUNA_EINVAL. Every GPU that loads the library
 * holds that array until the process exits. Every call shares it and it keeps the last call's contents; calls that
 * overlap on the GPU (other streams, other threads) race. The first call on a device looks up the array's device
 * address (once per device, with that device current); make that first call before any stream capture.
 * fallbacks_out (optional): the face sides that fell back to the cell's state. Giving it synchronises the stream and
 * also reads the pass's error word: a state that is not finite after the update returns LUNA_ENONFINITE (Q is then
 * already written). Without it the call does not synchronise and cannot report that.
 * The device mesh arrays are trusted: unlike luna_fv_create, this call does not check the lists, so an owner,
 * neighbour or cell_face entry out of range makes the kernels read out of bounds. */
LUNA_API luna_status luna_apply_static_noalloc(const luna_mesh_desc* mesh, const luna_gas* gas, int order, int riemann, const double* prims,
                                               const double* gradients, double* q, double dt, void* stream, int64_t* fallbacks_out);

/* The sweep's tiles for a mesh given in host memory: the layout luna_fv_create builds, computed on the host only (no
 * device work; no counterpart in the reference, a diagnostic of this library). Cells in Morton order of their
 * generators are cut into tiles of at most 128 cells; a tile's staged rows are its cells (in thread order) and then
 * the cells their lists reach, at most 416 of them (a cell needing more gets a tile of its own).
 * counts[6]: tiles, tiles within the 416-row budget, staged rows, entry slots, the most rows of a budget tile, the
 * most rows of a single-cell tile. The arrays may be null (sizes from a first call); else order [tiles * 128] (the
 * cell of each thread, -1 idle), slice_base [tiles * 4 + 1] (each warp's first entry slot / 32), stage_start
 * [tiles + 1], stage_cells [staged rows], local [entry slots] (each list entry's neighbour as a row of its tile's
 * staged cells, at slot (slice_base[t / 32] + k) * 32 + t % 32 for entry k of thread t). */
LUNA_API luna_status luna_mesh_tiles(const luna_mesh_desc* mesh, int64_t counts[6], int32_t* order, int32_t* slice_base, int32_t* stage_start,
                                     int32_t* stage_cells, uint32_t* local);

LUNA_API const char* luna_status_string(luna_status s);
LUNA_API const char* luna_last_error(void);
/* Device bytes held by fv (all its buffers). */
LUNA_API luna_status luna_fv_device_bytes(luna_fv* fv, int64_t* out);
/* Whether the static steps of fv run the fused flux-and-update pass (1; 0: flux rows then the update, or not yet
 * planned) and the faces between its tiles, solved by their own pass (no counterpart in the reference: a diagnostic).
 * The fused pass serves the FP64 per-face second-order step with the plain limiter when LUNA_FUSED_STEP=1 is in the
 * environment at the first step on a mesh: the same bits as the two-kernel pass in about 120 B a cell less device
 * memory, measured 5 % slower at 128^3 (the default is the two-kernel pass). */
LUNA_API luna_status luna_fv_fused_pass(luna_fv* fv, int* fused, int64_t* crossing_faces);

/* ---- The 1D solver: hydro::FiniteVolume<1, Exec, Riemann, Precision<>> on a static line (src/hydro/finite_volume_1d.hpp).
 * A batch of `lines` independent lines sharing one geometry: n_cells generators at `positions` (any order) on [0, length],
 * snapped to the 1D mesh's grid (step = length 2^-52), closed by two walls (LUNA_WALL_*, inflow: the primitives
 * rho, v, P of each inflow wall, [2][3]) or periodic. Q is [lines][n_cells][3] (rho, rho v, E, extensive) in the caller's
 * cell order. limiter: LUNA_LIMITER_FACE_CENTROID (LUNA's MC on a uniform line), NONE, MINMOD, VAN_LEER; riemann:
 * LUNA_HLLC or LUNA_HLL. The moving line is luna_mline_* below. */
typedef struct luna_line luna_line;
/* FiniteVolume(exec, mesh, gas, order, limiter, static_mesh, walls) (finite_volume_1d.hpp:41-56). */
LUNA_API luna_status luna_line_create(int64_t n_cells, int lines, const double* positions, double length, int periodic, const int* walls,
                                      const double* inflow, const luna_gas* gas, int order, int limiter, int riemann, luna_line** out);
LUNA_API luna_status luna_line_destroy(luna_line* ln);
LUNA_API luna_status luna_line_set_stream(luna_line* ln, void* stream);
/* Each cell's length and its centroid's offset from its generator (Line::volume, Line::centroid), caller order, host. */
LUNA_API luna_status luna_line_geometry(luna_line* ln, double* volume, double* centroid);
LUNA_API luna_status luna_line_set_state(luna_line* ln, const double* q, int on_device);
LUNA_API luna_status luna_line_get_state(luna_line* ln, double* q, int on_device);
/* time_step(courant, rule) (:332-384) of every line into dt_out [lines] (host); rule 0: AREPO's, 1: LUNA's. Synchronises. */
LUNA_API luna_status luna_line_time_step(luna_line* ln, double courant, int rule, double* dt_out);
/* step(dt) (:389-410): line k by dt[k] (host array [lines]). Asynchronous. */
LUNA_API luna_status luna_line_step(luna_line* ln, const double* dt);
/* step_and_time_step(dt, courant) (:412-418): the step and each line's next dt by LUNA's rule, one launch. Synchronises. */
LUNA_API luna_status luna_line_step_and_time_step(luna_line* ln, const double* dt, double courant, double* dt_next);
/* The step's derivatives at fixed dt (finite_volume_1d.hpp:852-898, FiniteVolume<1>::step_tangent / step_adjoint), each
 * line by dt[k]; x is [lines][n_cells][3] in the caller's cell order, in device memory (on_device != 0) or host memory.
 * step_tangent(dt, dq): dq <- J dq (J = d Q_after / d Q_before, extensive on both sides) and the state advances by the
 * step, as luna_line_step. step_adjoint(dt, qbar): qbar <- J^T qbar, the state unchanged (the step's start). A periodic
 * line needs 5 cells or more (the 5-cell stencil must not wrap onto itself). Synchronises when x is in host memory. */
LUNA_API luna_status luna_line_step_tangent(luna_line* ln, const double* dt, double* dq, int on_device);
LUNA_API luna_status luna_line_step_adjoint(luna_line* ln, const double* dt, double* qbar, int on_device);

/* ---- The 1D solver on a moving line: FiniteVolume<1> with Motion::moving (finite_volume_1d.hpp:41-56, the Moving
 * branches of Kernel::body :552-660, time_step :332-384, supply_cells :421-470, run_fused :679-711). One line of n_cells
 * generators at `positions` (the caller's cell order) on [0, length], snapped to the grid of step length 2^-52; the points
 * move with the gas (AREPO-ng's regularisation when `regularise`), each step by whole grid steps, and each face's flux is
 * the mean of those on the meshes of t^n and t^n+1 (order 1). Walls that do not reflect supply cells on a non-periodic
 * line (spacing length / n_cells by default; 0 turns it off): a cell inserted next to a wall takes the overlapped share of
 * its neighbour's Q, and is appended to the cell order (ids n_cells, n_cells + 1, ...). Q [cells][3] and x [cells] are in
 * cell order; luna_mline_cells gives the current count. The slots re-sort when points cross (the count in stats). */
typedef struct luna_mline luna_mline;
LUNA_API luna_status luna_mline_create(int64_t n_cells, const double* positions, double length, int periodic, const int* walls,
                                       const double* inflow, const luna_gas* gas, int order, int limiter, int riemann, int regularise,
                                       luna_mline** out);
LUNA_API luna_status luna_mline_destroy(luna_mline* ml);
LUNA_API luna_status luna_mline_set_stream(luna_mline* ml, void* stream);
LUNA_API luna_status luna_mline_cells(luna_mline* ml, int64_t* cells);
LUNA_API luna_status luna_mline_set_state(luna_mline* ml, const double* q, int on_device);
LUNA_API luna_status luna_mline_get_state(luna_mline* ml, double* q, int on_device);
/* The points' positions (FiniteVolume<1>::positions), cell order. */
LUNA_API luna_status luna_mline_positions(luna_mline* ml, double* x, int on_device);
/* Per cell (cell order, host): the generator's grid position, the cell's length, its centroid's offset from the generator. */
LUNA_API luna_status luna_mline_geometry(luna_mline* ml, double* generator, double* volume, double* centroid);
/* set_inflow_spacing (:61-66). */
LUNA_API luna_status luna_mline_set_inflow_spacing(luna_mline* ml, double spacing);
/* supply_cells (:421-470): the cells the walls have room for now; *added (may be null) the count. Synchronises. */
LUNA_API luna_status luna_mline_supply_cells(luna_mline* ml, int* added);
/* time_step(courant, rule) (:332-384): rule 0 AREPO's, 1 LUNA's, with the point velocity's |w - v|. Synchronises. */
LUNA_API luna_status luna_mline_time_step(luna_mline* ml, double courant, int rule, double* dt);
/* step(dt) (:389-410): the moving step, the slots' order, the walls' cells when due. Synchronises. */
LUNA_API luna_status luna_mline_step(luna_mline* ml, double dt);
/* step_and_time_step(dt, courant) (:412-418, :679-711): the step and the next dt of LUNA's rule in one launch (afresh by
 * time_step when the slots re-sorted or cells were added). Synchronises. */
LUNA_API luna_status luna_mline_step_and_time_step(luna_mline* ml, double dt, double courant, double* dt_next);
/* cells_added(), and the mesh's re-sorts and updates (MeshStats). Any pointer may be null. */
LUNA_API luna_status luna_mline_stats(luna_mline* ml, int64_t* cells_added, int64_t* sorts, int64_t* updates);

#ifdef __cplusplus
}
#endif

#endif
