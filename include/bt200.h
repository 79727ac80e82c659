/*
 * beamtracer-b200: the C ABI of the B200 (sm_100a) Vlasov-iteration path.
 *
 * Every entry point returns 0 on success or a negative BT_ERR_* code; bt_last_error()
 * gives the message of the calling thread's last failure.  Array arguments are plain
 * pointers: DEVICE pointers for the kernel-level entry points (the cunumpy kernel
 * interface of the reference, which runs its CUDA kernels on CuPy device arrays) and the
 * solver entry points that say so, HOST pointers where an entry point says "host".
 * Layouts are C order, the reference's: a (3, n) array is three rows of n values, an
 * (nx, ny) mesh array has y contiguous.  Integers are int64 where the reference passes
 * "int[:]" arrays (long long in its CUDA kernels).
 *
 * Work is queued on the context's CUDA stream; an entry point that must read a result
 * back (a count, a norm) synchronises that stream.  One context per host thread.
 */
#ifndef BT200_H
#define BT200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BT_OK 0
#define BT_ERR_ARG (-1)      /* an argument is invalid (null, negative size, bad shape) */
#define BT_ERR_CUDA (-2)     /* a CUDA call failed */
#define BT_ERR_CAPACITY (-3) /* an output buffer is too small; see bt_last_error */
#define BT_ERR_NOCONV (-4)   /* an iterative solve did not converge */
#define BT_ERR_TIMEOUT (-5)  /* a bounded device wait ran out */
#define BT_ERR_ALLOC (-6)    /* device memory could not be allocated */

typedef struct bt_ctx bt_ctx;

/* -- context ------------------------------------------------------------------------- */

/* A context on CUDA device `device` with its own non-blocking stream. */
int bt_ctx_create(int device, bt_ctx **out);
int bt_ctx_destroy(bt_ctx *ctx);
/* Queue the context's work on `stream` (a cudaStream_t; NULL is CUDA's default stream, as
 * for CuPy's and PyTorch's default streams).  A new context queues on its own non-blocking
 * stream until this is called; work on another stream is ordered with the context's only
 * by that stream's own rules (the default stream waits for blocking streams, not for
 * non-blocking ones). */
int bt_ctx_set_stream(bt_ctx *ctx, void *stream);
int bt_ctx_synchronize(bt_ctx *ctx);
/* Time the context's launches with CUDA events on its stream (off by default): the
 * kernels "trace_window", "deposit" (the sort and reduction of a flush of records),
 * "field_solve" (a whole bt_poisson_solve), "vcycle" (one multigrid V-cycle), "hierarchy"
 * (the coarse operators and the coarsest inverse of a new operator), "edge_field",
 * "vlasov_mix",
 * "staggered_field_2d".  bt_ctx_read_timer waits for the recorded launches and returns
 * their summed time [ms] and count since the last reset. */
int bt_ctx_set_timing(bt_ctx *ctx, int on);
int bt_ctx_read_timer(bt_ctx *ctx, const char *name, double *total_ms, int64_t *launches);
int bt_ctx_reset_timers(bt_ctx *ctx);
/* The deposit records (the runs of steps with a charge, the slots with none left out) that
 * the context's deposits have sorted and reduced while timing was on, since the last
 * bt_ctx_reset_timers (host out-param; waits for the context's stream).  For measurement:
 * the algorithmic bytes of the deposit are counted per record.  No counterpart in the
 * reference. */
int bt_ctx_deposit_records(bt_ctx *ctx, int64_t *records);
/* No counterpart in the reference.  The FP64 pipe's peak on the context's device
 * (TFLOP/s, a fused multiply-add two operations): independent FMA chains on every SM, the
 * fastest of three timed launches (CUDA events on the context's stream). */
int bt_measure_fp64_peak(bt_ctx *ctx, double *tflops);
/* The number of kernels the context has launched since its creation (host out-param). */
int bt_ctx_launch_count(bt_ctx *ctx, int64_t *count);
/* Copy the calling thread's last error message into buf (NUL-terminated); returns its length. */
size_t bt_last_error(char *buf, size_t len);
/* The library's version string. */
const char *bt_version(void);

/* -- the reference's kernel interface (device pointers) ------------------------------- */

/* kernels/staggered_field_2d/staggered_field_2d_pyccel.py:13-55 (CUDA: *_cuda.cu:18-37).
 * (E_x, E_y) at the n points (px, py): fx (nx + 1, ny) and fy (nx, ny + 1) interpolated
 * bilinearly with the cell clamped to the arrays. */
int bt_staggered_field_2d(bt_ctx *ctx, const double *px, const double *py, int64_t n,
                          const double *fx, const double *fy, int64_t nx, int64_t ny,
                          double origin_x, double origin_y, double h, double *ex,
                          double *ey);

/* kernels/deposit_trajectories_2d/deposit_trajectories_2d_pyccel.py:13-59 (CUDA:
 * *_cuda.cu:8-55).  Adds the n charges q at (px, py) to charge (nx, ny), area-weighted
 * (linear in r^2 radially when cylindrical != 0).  Deterministic: the contributions are
 * sorted by cell and summed per cell by warp segmented reductions in a fixed order, so
 * the result is the same bit for bit on every call.  Uses context-owned scratch. */
int bt_deposit_trajectories_2d(bt_ctx *ctx, const double *px, const double *py,
                               const double *q, int64_t n, double origin_x, double origin_y,
                               double h, int64_t cylindrical, double *charge, int64_t nx,
                               int64_t ny);

/* No counterpart in the reference.  The deposit of bt_deposit_trajectories_2d for callers
 * that may not allocate device memory -- whose device memory is budgeted up front by
 * another allocator, or that cannot take cudaMalloc's implicit synchronisation of the
 * device at the point where they deposit.  It allocates nothing: its scratch is a
 * file-scope __device__ array of about 5.4 MB that every GPU loading the library holds
 * until the process exits, sized for at most 65536 charges per call and a mesh of at most
 * 65536 nodes; larger calls fail with BT_ERR_ARG.  `stream` is a cudaStream_t (NULL: the
 * legacy default stream) on the calling thread's current device.  Every call looks up the
 * array's device address in the current device's context (cudaGetSymbolAddress, a host
 * call); the first call in a context may load the library's module there, so make that
 * first call before any stream capture.  All calls share the array and leave their scratch in
 * it: calls that overlap on the GPU race, so order them (one stream, or events). */
int bt_deposit_trajectories_2d_noalloc(void *stream, const double *px, const double *py,
                                       const double *q, int64_t n, double origin_x,
                                       double origin_y, double h, int64_t cylindrical,
                                       double *charge, int64_t nx, int64_t ny);

/* The arguments of kernels/trace_trajectories_2d/trace_trajectories_2d_pyccel.py:42-78,
 * all arrays on the device, with their shapes. */
typedef struct bt_trace_args {
    const int64_t *active; /* (n_active,) trajectory indices */
    int64_t n_active;
    double *x, *v; /* (3, n) positions, velocities (proper velocities if inv_c2 > 0) */
    int64_t n;
    const double *qm, *dq;                  /* (n,) charge/mass, signed current */
    int64_t *steps, *status, *electrode;    /* (n,) */
    const double *fxs, *fys;                /* the patches' edge fields, flattened */
    const int64_t *patch_int;               /* (n_patches, 6) */
    const double *patch_real;               /* (n_patches, 7) */
    int64_t n_patches;
    double origin_x, origin_y, h, upper_x, upper_y;
    int64_t cylindrical; /* 0 planar, 1 cylindrical, 2 planar with a symmetry plane */
    int64_t integrator;  /* 0 RK4, 1 Boris */
    double step_fraction;
    int64_t max_steps;
    const int64_t *cells;    /* (nx - 1, ny - 1) of the last patch */
    const int64_t *subcells; /* (cells, refine, refine) */
    int64_t refine;
    const double *planes; /* (n_planes,) */
    int64_t n_planes;
    double *hits; /* (n, n_planes, capacity, 8) */
    int64_t capacity;
    int64_t *counts;          /* (n, n_planes) */
    const int64_t *path_slot; /* (n,) */
    double *paths;            /* (slots, path_capacity, 2) */
    int64_t path_capacity;
    int64_t *path_count; /* (slots,) */
    int64_t num_threads; /* the reference's host threads: ignored on the GPU */
    double *charge;      /* (num_threads, n_nodes): the GPU adds into charge[0] */
    int64_t n_nodes;
    int64_t graded;
    const double *x_nodes; /* (n_x_nodes,) */
    int64_t n_x_nodes;
    double inv_c2;
} bt_trace_args;

/* kernels/trace_trajectories_2d/trace_trajectories_2d_pyccel.py:42-507 (CUDA:
 * *_cuda.cu:165-362).  Traces the active trajectories to their ends (status 0-4) or to a
 * sub-cell cut by an electrode surface (status -2), depositing dq dt at every step's
 * Hermite midpoint into charge[0] deterministically, recording plane crossings and kept
 * paths.  The trajectories advance in windows of `window` steps (0: the default), one
 * thread per trajectory; after each window the live ones are compacted and every
 * window's deposit records are sorted by cell and reduced in a fixed order. */
int bt_trace_trajectories_2d(bt_ctx *ctx, const bt_trace_args *args, int64_t window);

/* No counterpart in the reference.  bt_trace_trajectories_2d built with contracted
 * multiply-adds: the same step with every a * b + c one fused multiply-add rounded once,
 * so results agree with the exact build to rounding (not bit for bit) in fewer dependent
 * FP64 instructions.  bt_trace_trajectories_2d_magnetic_fast likewise. */
int bt_trace_trajectories_2d_fast(bt_ctx *ctx, const bt_trace_args *args, int64_t window);

/* An axisymmetric magnetic field from its on-axis profile (solver/fields.py:192-279,
 * AxisymmetricMagneticField): samples (DEVICE, n rows of order + 1) hold d^k B_z / dz^k,
 * k = 0..order, at z0 + hz i (fields.py:236-243); between samples they are interpolated
 * linearly and summed in the power series in r (fields.py:250-279).
 * mode 1: a cylindrical mesh, B = B_z x^ + B_r r^ at (x, r);
 * mode 2: a planar mesh with the solenoid's axis on y = axis_y: B = (B_z, sign(y - axis_y)
 * B_r, 0) at r = |y - axis_y|. */
typedef struct bt_magnetic {
    int32_t mode;
    int32_t order; /* 0..6 */
    int64_t n;     /* samples, at least 8 */
    double z0, hz, axis_y;
    const double *samples;
} bt_magnetic;

/* solver/tracer.py:851-1054 (BeamTracer._trace_numpy, the reference's only path with a
 * magnetic field) with _rk4 (:586-603) and _boris / _kick (:605-660): the arguments and
 * outputs of bt_trace_trajectories_2d, each step's acceleration q/m (E + v x B), Boris's
 * kick with the magnetic rotation, the spacing of mesh.py:197-202; every step ending in a
 * cell that touches an electrode pauses (status -2) for the caller's exact inside test
 * (tracer.py:1019-1024).  Non-relativistic (inv_c2 = 0), one patch, no symmetry plane. */
int bt_trace_trajectories_2d_magnetic(bt_ctx *ctx, const bt_trace_args *args,
                                      const bt_magnetic *magnetic, int64_t window);
int bt_trace_trajectories_2d_magnetic_fast(bt_ctx *ctx, const bt_trace_args *args,
                                           const bt_magnetic *magnetic, int64_t window);

/* The candidates of a batched trace: many independent meshes traced in one launch.  The
 * reference's design search traces its candidates one at a time
 * (optimization/einzel.py:389-403); this has no single-call counterpart there.
 * args->patch_int / patch_real hold one row per candidate (n_patches = n_candidates), as
 * the trace's one-patch rows: (nx, ny, offset into fxs, offset into fys, nodes, offset of
 * the first node) and (origin x, origin y, h, origin x, origin y, upper x, upper y), the
 * node offsets ascending and contiguous from 0 to args->n_nodes.  All DEVICE. */
typedef struct bt_trace_batch {
    int64_t n_candidates;
    const int32_t *candidate;  /* (n,) the candidate of every trajectory */
    const int64_t *cell_offset; /* (n_candidates,) where its cell table starts in cells */
    int64_t group;              /* windows between reads of the live count (0: chosen) */
    /* The candidates' electrodes as shapes (the bt_shapes tables of all candidates end to
     * end; candidate c's electrodes are shapes shape_first[c] .. shape_first[c + 1] - 1, in
     * its electrode order), or shape_first NULL.  With them a trajectory whose step ends in
     * a sub-cell an electrode surface cuts is tested against its candidate's shapes in the
     * kernel (at its mesh coordinates (x, r) or (x, y)) instead of pausing with status -2
     * for the caller's test. */
    const int64_t *shape_first;  /* (n_candidates + 1,) */
    const int32_t *shape_kind;
    const int64_t *shape_offset;
    const double *shape_params;
} bt_trace_batch;

/* No counterpart in the reference (see bt_trace_batch).  bt_trace_trajectories_2d over a
 * batch of candidate meshes: one window launch advances every candidate's live
 * trajectories, and one deposit sorts and reduces the records of all of them (keys are the
 * candidates' concatenated node indices).  Each trajectory's steps, crossings and end are
 * those it has traced alone; its charges are summed in the same record order, grouped
 * into deposits differently.  One patch per candidate, uniform axes, non-relativistic, no
 * magnetic field. */
int bt_trace_trajectories_2d_batch(bt_ctx *ctx, const bt_trace_args *args,
                                   const bt_trace_batch *batch, int64_t window);

/* No counterpart in the reference: bt_trace_trajectories_2d_batch built with contracted
 * multiply-adds (as bt_trace_trajectories_2d_fast). */
int bt_trace_trajectories_2d_batch_fast(bt_ctx *ctx, const bt_trace_args *args,
                                        const bt_trace_batch *batch, int64_t window);

/* The arguments of kernels/trace_trajectories_3d/trace_trajectories_3d_pyccel.py:19-61, all
 * arrays on the device: positions and velocities (3, n); patch_int (n_patches, 8): node
 * counts (nx, ny, nz), offsets of the three edge fields, node count, offset of the nodes in
 * charge; patch_real (n_patches, 10): origin (3), spacing, node box (x0, y0, z0, x1, y1, z1),
 * finest first and the base mesh last; bn (3, nx, ny, nz) of the base mesh when has_b;
 * cells (nx - 1, ny - 1, nz - 1); hits (n, n_planes, capacity, 8); paths (slots,
 * path_capacity, 3); charge (num_threads, nodes) and, with has_j, current (num_threads,
 * 3 nx ny nz): the GPU adds into row 0. */
typedef struct bt_trace3d_args {
    const int64_t *active;
    int64_t n_active;
    double *x, *v;
    int64_t n;
    const double *qm, *dq;
    int64_t *steps, *status, *electrode;
    const double *fxs, *fys, *fzs;
    const int64_t *patch_int;
    const double *patch_real;
    int64_t n_patches;
    const double *bn;
    int64_t has_b;
    double origin_x, origin_y, origin_z, h, upper_x, upper_y, upper_z;
    int64_t mirror_y, mirror_z, integrator;
    double step_fraction;
    int64_t max_steps;
    const int64_t *cells;
    const int64_t *subcells;
    int64_t refine;
    const double *planes;
    int64_t n_planes;
    double *hits;
    int64_t capacity;
    int64_t *counts;
    const int64_t *path_slot;
    double *paths;
    int64_t path_capacity;
    int64_t *path_count;
    int64_t num_threads; /* the reference's host threads: ignored on the GPU */
    double *charge;
    int64_t n_nodes;
    int64_t has_j;
    double *current;
    double inv_c2;
} bt_trace3d_args;

/* solver/fields3d.py:66-107 (StaggeredElectricField3D): the edge fields of a potential phi
 * (nx, ny, nz) along each axis by the 2D rule of bt_edge_field (solver/fields.py:18-67) on
 * every line of nodes: fx (nx + 1, ny, nz), fy (nx, ny + 1, nz), fz (nx, ny, nz + 1);
 * solid (nx, ny, nz) int32, near uint8, distance (6, nx, ny, nz) towards -x, +x, -y, +y,
 * -z, +z; extrapolation[6] per face (x min, x max, y min, ...): 1 symmetric, 0 linear. */
int bt_edge_field_3d(bt_ctx *ctx, const double *phi, const int32_t *solid, const uint8_t *near,
                     const double *distance, int64_t nx, int64_t ny, int64_t nz, double h,
                     const int32_t extrapolation[6], double *fx, double *fy, double *fz);

/* kernels/trace_trajectories_3d/trace_trajectories_3d_pyccel.py:19-657 (CUDA:
 * *_cuda.cu:120-399): every active trajectory to its end (status 0-4) or to a sub-cell an
 * electrode surface cuts (-2, for the caller's test), in windows of `window` steps (0: the
 * default), one thread per trajectory, the reference's step term by term in FP64 (RK4, or
 * Boris with the relativistic push of mpiparticles as published); the space charge (and,
 * with has_j, the current elements) deposited deterministically: every step's eight node
 * shares as (node, value) records, sorted by node and summed in record order. */
int bt_trace_trajectories_3d(bt_ctx *ctx, const bt_trace3d_args *args, int64_t window);

/* Counters of the last bt_trace_trajectories_2d call on this context (host out-params). */
int bt_trace_last_stats(bt_ctx *ctx, int64_t *windows, int64_t *records,
                        int64_t *deposit_flushes);

/* -- electrode shapes (device pointers) ------------------------------------------------ */

/* The configuration's electrode shapes (config.py ObjectParams.inside, the reference's
 * sections.py:636-784 objects): count shapes, shape s of kind[s] with its parameters at
 * params + offset[s]: 0 rectangle or line (mx, my, lx/2, ly/2), 1 circle (mx, my, r^2),
 * 2 polygon (n, then per edge x1, y1, x2, y2, boundary threshold, x_lo, x_hi, y_lo, y_hi),
 * 3 aperture (two such polygons: the shape and its mirror image).  The first holding a
 * point is its electrode. */
typedef struct bt_shapes {
    int64_t count;
    const int32_t *kind;
    const int64_t *offset;
    const double *params;
} bt_shapes;

/* solver/tracer.py:1092-1114 (BeamTracer._subcells): out (n_cells, refine, refine) int64,
 * the electrode of every sub-cell of the cells (ci, cj) holding its four corners and its
 * centre, -1 for none, -2 where they disagree.  x_nodes (n_x_nodes,) for a graded x axis,
 * else NULL. */
int bt_subcell_table(bt_ctx *ctx, const bt_shapes *shapes, const int64_t *ci,
                     const int64_t *cj, int64_t n_cells, double origin_x, double origin_y,
                     double h, const double *x_nodes, int64_t n_x_nodes, int64_t refine,
                     int64_t *out);

/* solver/mesh.py:127-201 (IonOpticsMesh._classify, _bracket): solid (nx, ny) int32, the
 * first electrode holding each node or -1; near (nx, ny) uint8, a free node with an
 * electrode neighbour; distance (4, nx, ny), towards -x, +x, -y, +y, the surface's place on
 * the edge to an electrode neighbour by eight bisections of that electrode's inside test
 * in 1/255 (1 without one).  x (nx,) the node positions, dx (nx - 1,) the edge lengths, the
 * nodes' y = origin_y + h j. */
int bt_classify_mesh(bt_ctx *ctx, const bt_shapes *shapes, int64_t nx, int64_t ny,
                     const double *x, const double *dx, double origin_y, double h,
                     int32_t *solid, uint8_t *near, double *distance);

/* -- the edge field (device pointers) --------------------------------------------------- */

/* solver/fields.py:18-67 and 116-152: the staggered edge fields of a potential.
 * phi (nx, ny); solid (nx, ny) int32 electrode index or -1; near (nx, ny) uint8;
 * distance (4, nx, ny) fractions of the edge towards -x, +x, -y, +y; dx (nx - 1,) the
 * edge lengths along x (graded) or NULL for a uniform h; extrapolation[4] 0 =
 * "extrapolate", 1 = "symmetric" for the faces x_min, x_max, y_min, y_max.
 * Writes fx (nx + 1, ny) and fy (nx, ny + 1). */
int bt_edge_field(bt_ctx *ctx, const double *phi, const int32_t *solid, const uint8_t *near,
                  const double *distance, const double *dx, int64_t nx, int64_t ny,
                  double h, const int32_t extrapolation[4], double *fx, double *fy);

/* solver/fields.py:324-377 (surface_field).  At every free node next to an electrode
 * (near (nx, ny) uint8), |E| (magnitude, (nx, ny)) from its two edge fields along each
 * axis -- the edge towards an electrode neighbour (the field at the surface), the larger of
 * the two with electrodes on both sides, else their mean -- and that electrode (electrode,
 * (nx, ny) int32: the first of the -x, +x, -y, +y neighbours that is solid); NaN and -1
 * elsewhere.  largest (n_electrodes, or NULL): each electrode's largest |E| (0 for one with
 * no free neighbour).  All arrays on the DEVICE. */
int bt_surface_field(bt_ctx *ctx, const double *fx, const double *fy, const int32_t *solid,
                     const uint8_t *near, int64_t nx, int64_t ny, int32_t n_electrodes,
                     double *magnitude, int32_t *electrode, double *largest);

/* The transpose of bt_edge_field (no counterpart in the reference; the differentiation
 * form): phi_bar (nx, ny) = D^T (fx_bar, fy_bar), D the linear map from the potential to
 * the edge fields that bt_edge_field applies on the same mesh arrays.  One thread a node,
 * its sum in a fixed order: the same bits on every call. */
int bt_edge_field_adjoint(bt_ctx *ctx, const double *fx_bar, const double *fy_bar,
                          const int32_t *solid, const uint8_t *near, const double *distance,
                          const double *dx, int64_t nx, int64_t ny, double h,
                          const int32_t extrapolation[4], double *phi_bar);

/* -- the per-iteration updates (device pointers) -------------------------------------- */

/* solver/vlasov.py:127-173 (AndersonMixer.update), on the device.  Anderson mixing of type
 * II of the iterate rho (DEVICE, nx * ny) with its new deposit G(rho) = charge / volumes
 * times column_factor[i] on node column i (volumes or column_factor NULL: left out):
 * the iterate and its residual are stored in row `head` of the ring buffers xs and fs
 * (DEVICE, (depth + 1) * nx * ny each; `count` rows, 1 to depth + 1, hold the last
 * iterates, the newest at `head`, the older ones before it cyclically) and rho is
 * overwritten with x + w f - (dX + w dF) gamma, gamma the least-squares solution of
 * dF gamma = f with singular values below 1e-10 of the largest left out (numpy.linalg.lstsq
 * with rcond 1e-10), through a QR of dF by Gram-Schmidt applied twice into q (DEVICE,
 * depth * nx * ny scratch).  depth 1 to 16.  stats (DEVICE, 2): max |new - old| and
 * max |new| (NaN if any entry is NaN). */
int bt_anderson_mix(bt_ctx *ctx, const double *charge, const double *volumes,
                    const double *column_factor, int64_t nx, int64_t ny, int32_t depth,
                    int32_t count, int32_t head, double relaxation, double *xs, double *fs,
                    double *q, double *rho, double *stats);

/* tracer.py:700-705, vlasov.py:176-184 and 389-397: the new density of an iteration.
 * deposit = charge / volumes (both (nx, ny)), times column_factor[i] (nx,) where given
 * (the space-charge compensation of node column i, NULL for none); then rho <- deposit
 * (first != 0) or (1 - relaxation) rho + relaxation deposit.  stats (device, 2 values):
 * max |rho_new - rho_old| and max |rho_new|. */
int bt_vlasov_mix(bt_ctx *ctx, const double *charge, const double *volumes,
                  const double *column_factor, int64_t nx, int64_t ny, double relaxation,
                  int32_t first, double *rho, double *stats);

/* vlasov.py:362-366: out (device, 1 value) = max |a - b| over n values. */
int bt_max_abs_diff(bt_ctx *ctx, const double *a, const double *b, int64_t n, double *out);

/* -- the field solve ----------------------------------------------------------------- */

typedef struct bt_poisson bt_poisson;

/* The mesh a field solve is built from (HOST pointers, copied on creation). */
typedef struct bt_mesh_desc {
    int64_t nx, ny;
    double h;                  /* the spacing along y (and along x on a uniform mesh) */
    const double *x;           /* (nx,) node positions along x */
    double origin_y;
    int32_t cylindrical;       /* 1: (x, r) with the axis at y = origin_y = 0 */
    const uint8_t *fixed;      /* (nx, ny) 1 for electrode and Dirichlet-face nodes */
    const double *fixed_value; /* (nx, ny) their potentials */
    const double *distance;    /* (4, nx, ny) surface distances towards -x, +x, -y, +y */
    const double *neumann;     /* (4,) outward normal derivative on x_min, x_max, y_min,
                                  y_max (ignored where the face's nodes are fixed), or NULL */
} bt_mesh_desc;

/* solver/poisson.py:536-933 (IonOpticsPoisson): build the finite-volume operator of the
 * mesh (patchwork's NodalPoisson as poisson.py:1-24, 491-534 documents it) and its
 * multigrid hierarchy on the device. */
int bt_poisson_create(bt_ctx *ctx, const bt_mesh_desc *mesh, bt_poisson **out);
int bt_poisson_destroy(bt_poisson *p);

/* Hold the nodes of `mask` (HOST (nx, ny) uint8, or NULL for none) that the mesh does not
 * fix at `value`: the initial plasma region of the first Vlasov iteration
 * (solver/vlasov.py:350-355, poisson.py:279-309). */
int bt_poisson_set_region(bt_poisson *p, const uint8_t *mask, double value);

/* The V-cycle's settings, the solver's tuning knobs (no counterpart in the reference, which
 * factorises with LU; defaults 2, 2, 1, 4096): red-black sweeps on the finest level and
 * four-colour sweeps on the coarse levels before and after each coarse correction (1-4),
 * smoothing staged through shared memory (1) or one launch per colour (0; the same values),
 * and the size above which a level is never part of the one-block tail. */
int bt_poisson_set_options(bt_poisson *p, int32_t fine_sweeps, int32_t coarse_sweeps,
                           int32_t staged, int64_t tail_nodes);

/* Move a solver to another context on the same device (after its queued work finishes):
 * its later work queues on that context's stream.  No counterpart in the reference. */
int bt_poisson_set_context(bt_poisson *p, bt_ctx *ctx);

/* -- the batched field solve (no counterpart in the reference, which solves each design
 * candidate's field on its own: optimization/einzel.py:389-403) ------------------------- */

typedef struct bt_poisson_batch bt_poisson_batch;

/* A batch of `count` solvers on one context (each candidate mesh's own bt_poisson, kept
 * alive and unchanged -- no bt_poisson_set_options -- while the batch lives), candidate c's
 * nodes at offset[c] (HOST) of the batch's concatenated potential and density.  Every
 * solver needs the staged smoother, at most 2 coarse sweeps and a hierarchy of at least two
 * levels with a one-block tail. */
int bt_poisson_batch_create(bt_ctx *ctx, bt_poisson *const *solvers, int64_t count,
                            const int64_t *offset, bt_poisson_batch **out);
int bt_poisson_batch_destroy(bt_poisson_batch *batch);

/* The linear field solve of every candidate c with members[c] != 0 (HOST flags), in place on
 * the DEVICE arrays phi and rho (rho NULL: no charge): the multigrid iteration
 * d <- d + V(r0 - A d) with one V-cycle over all members per step (a launch per level step
 * and kind, the coarse levels in one block per candidate), each member until its residual
 * is at most tol max(|b|, |r0|) -- the criterion of bt_poisson_solve -- or stops falling.
 * cycles and residual (HOST, count entries, may be NULL) get each member's V-cycles and
 * final residual norm.  BT_ERR_NOCONV if a member ends above 1e4 times its goal. */
int bt_poisson_batch_solve(bt_poisson_batch *batch, double *phi, const double *rho,
                           const uint8_t *members, double tol, int32_t max_cycles,
                           int32_t *cycles, double *residual);

/* The batched V-cycle's smoothing tiles (HOST tiling[6]): level 0's tile (x, y interior
 * nodes), the 9-point levels' tile, the launches a 9-point smoothing is split into (1 or 2)
 * and whether they were chosen (1) or are still to be tuned (0).  set == 0 reads them;
 * set != 0 fixes the first five (tiling[0] <= 0: tune again at the next solve).  By
 * default the first solve times a few tilings on the batch's own V-cycle and keeps the
 * fastest.  No counterpart in the reference. */
int bt_poisson_batch_tiling(bt_poisson_batch *batch, int32_t set, int32_t *tiling);

/* No counterpart in the reference (the differentiation form).  on != 0: the solver's
 * operator becomes the transpose of the free rows' block, A_ff^T (the neighbour
 * coefficients exchanged between each pair of free nodes, the diagonal kept), so
 * bt_poisson_solve solves A_ff^T z = rho / eps0 (+ its face and held terms: give the
 * transposed solver zero held values and zero Neumann values for a plain A_ff^T z = b).
 * It solves the similar system B y = W^-1 b, z = W y, B = W^-1 A^T W with W the control
 * volumes, which equals A wherever W A is symmetric, so the multigrid serves it as it
 * serves A.  Linear solves only (no Boltzmann species). */
int bt_poisson_set_transposed(bt_poisson *p, int32_t on);

/* No counterpart in the reference.  The held potentials' sensitivity: given phi_bar (the
 * sensitivity of a quantity to every node's potential) and z = A_ff^-T phi_bar (free
 * nodes), out (DEVICE, nx * ny) = phi_bar_d + sum over the free neighbours i of held
 * node d of A's coefficient from i to d times z_i, on held nodes; 0 on free nodes. */
int bt_poisson_fixed_adjoint(bt_poisson *p, const double *z, const double *phi_bar, double *out);

/* The residual r = rho / eps0 + c - A phi of the mesh's field equation on its free nodes (0
 * on the held ones), all DEVICE (nx, ny); rho may be NULL.  The composite solve of refined
 * boxes (solver/poisson.py:169-335 through patchwork, absent here) evaluates each node's
 * equation as its owner patch's row with it. */
int bt_poisson_residual(bt_poisson *p, const double *phi, const double *rho, double *r);

/* solver/refinement.py:201-231, 286-296, 330-377 (the composite nodes' maps:
 * Layout.on_base, deposit_total, PatchedElectricField's potentials of the patches,
 * fill_hanging): y[out_rows[r]] = (accumulate ? y[out_rows[r]] : constant[r]) +
 * sum over e in [row_ptr[r], row_ptr[r + 1]) of val[e] x[col[e]], in that order (no
 * atomics: the same bits on every run).  out_rows NULL: row r writes y[r]; constant NULL:
 * zero.  A row may read y's own entries only where no row writes them.  All DEVICE. */
int bt_csr_apply(bt_ctx *ctx, int64_t rows, const int64_t *out_rows, const int64_t *row_ptr,
                 const int64_t *col, const double *val, const double *constant,
                 int32_t accumulate, const double *x, double *y);

/* A linear solve of (A + diag(reaction)) phi = rho / eps0 + c on the free nodes, the held
 * ones at their values (phi DEVICE (nx, ny) in/out: first guess, solution; rho DEVICE or
 * NULL; reaction DEVICE (nx, ny)): one Newton step of solver/poisson.py:627-757 on a
 * patch of refined boxes, where the composite Newton iteration supplies the Jacobian's
 * reaction.  Relative residual tol; *cycles the V-cycles taken. */
int bt_poisson_solve_reaction(bt_poisson *p, double *phi, const double *rho,
                              const double *reaction, double tol, int32_t *cycles);

/* solver/poisson.py:76-141, 898-903 on the composite nodes of refined boxes: at the nodes
 * with own[k] != 0, e = amplitude exp(min(-sign (phi - up) / temperature, 50)) is added to
 * r as sign e and reaction[k] = e / temperature; elsewhere reaction[k] = 0.  All DEVICE
 * (n,). */
int bt_boltzmann_terms(bt_ctx *ctx, int64_t n, const uint8_t *own, const double *phi,
                       double amplitude, double temperature, double up, int32_t sign,
                       double *r, double *reaction);

/* One multigrid V-cycle from zero: z = M b (DEVICE (nx, ny); b a right-hand side of the
 * mesh's equation as the residual of bt_poisson_residual is one, zero on held nodes), the
 * operator's diagonal plus `reaction` (DEVICE, or NULL for none); the hierarchy is rebuilt
 * when `rebuild` is set, the reaction's presence changed or the held nodes did.  The
 * inexact local solve of each patch in the composite sweeps of refined boxes
 * (solver/poisson.py:169-335 through patchwork, absent here). */
int bt_poisson_vcycle(bt_poisson *p, const double *b, const double *reaction, int32_t rebuild,
                      double *z);

/* The residual of a composite Newton step's correction x (poisson.py:627-757 on refined
 * boxes): y = base + y - reaction x at the nodes with own[k] != 0 (y holding -K x there on
 * entry, base the step's residual), 0 elsewhere.  All DEVICE (n,). */
int bt_newton_residual(bt_ctx *ctx, int64_t n, const uint8_t *own, const double *base,
                       const double *reaction, const double *x, double *y);

/* poisson.py:809-933 (IonOpticsPoisson.solve).  phi (DEVICE (nx, ny), in/out): the first
 * guess on entry (its fixed nodes are set), the solution on return; rho (DEVICE (nx, ny),
 * C/m^3, or NULL).  With amplitude = 0 one linear solve: GMRES preconditioned by a
 * multigrid V-cycle to ||b - A phi|| <= tol max(||b||, ||b - A phi_0||).  With amplitude > 0
 * the Boltzmann species sign * amplitude exp(min(-sign (phi - up) / temperature, 50))
 * (amplitude = rho_0 / eps0) joins the source, and Newton's method runs: every step a
 * GMRES solve of that step's Jacobian (the multigrid rebuilt for it) to the relative
 * residual tol, until the largest update is below newton_tol or max_newton steps.
 * Host out-params (may be NULL): Newton steps, V-cycles. */
int bt_poisson_solve(bt_poisson *p, double *phi, const double *rho, double amplitude,
                     double temperature, double up, int32_t sign, double tol,
                     double newton_tol, int32_t max_newton, int32_t *newton_steps,
                     int32_t *cycles);

/* -- the adjoint of the trace (the differentiation form; no counterpart in the reference) -- */

/* A forward trace to reverse: RK4, one uniform patch, no magnetic field, not relativistic,
 * planar (0) or cylindrical (1).  All arrays on the DEVICE. */
typedef struct bt_adjoint_args {
    const double *x0, *v0;  /* (3, n) the trajectories' start states */
    const double *qm, *dq;  /* (n,) charge / mass, signed current */
    const int64_t *steps;   /* (n,) the steps each took in the forward trace */
    int64_t n;
    const double *fx, *fy;  /* the forward trace's edge fields (nx + 1, ny), (nx, ny + 1) */
    int64_t nx, ny;
    double origin_x, origin_y, h;
    int64_t cylindrical;
    double step_fraction;
    const double *planes;   /* (n_planes,), at most 8 */
    int64_t n_planes;
    const int64_t *counts;  /* (n, n_planes) the forward trace's crossing counts */
    int64_t capacity;       /* of the hit buffers the hit adjoint is laid out as */
    double *checkpoints;    /* (segments, 6, n): the states every 64 steps */
    int64_t segments;       /* at least ceil(max(steps) / 64) */
} bt_adjoint_args;

/* Replays every trajectory for its forward steps (trace.cu's step, the same bits) and
 * keeps its state every 64 steps in checkpoints; its end state (DEVICE (6, n): x then v)
 * in end_state unless NULL. */
int bt_adjoint_checkpoints(bt_ctx *ctx, const bt_adjoint_args *args, double *end_state);

/* The reverse sweep (after bt_adjoint_checkpoints): ADDS to fx_bar (nx + 1, ny) and fy_bar
 * (nx, ny + 1) the adjoint of the edge fields of a quantity whose adjoints of the trace's
 * outputs are charge_seed (nx, ny; the node charges the trace deposits) and hit_seed
 * (n, n_planes, capacity, 8; slots 1-5 the crossings' point y, z and velocity; the hits
 * buffer's layout); either may be NULL.  The scatter adds with atomics: reproducible to
 * rounding, not bit for bit. */
int bt_adjoint_sweep(bt_ctx *ctx, const bt_adjoint_args *args, const double *charge_seed,
                     const double *hit_seed, double *fx_bar, double *fy_bar);

#ifdef __cplusplus
}
#endif
#endif /* BT200_H */
