/*
 * gamera_op.h -- C ABI of the B200 implementation of GAMERA-OP's
 * single-domain MHD time step.
 *
 * The reference exposes its step as C globals plus `int solve(int nt)`
 * (src/solver.h:65, src/solver_solve.c:23-536) driven by `main`
 * (src/main.c:75).  These entry points are what a replacement `solve()`
 * binds to: the host keeps its config.yaml, problem hooks
 * (src/problem.h:5-12), boundary library (src/boundary_conditions.c) and
 * HDF5 output (src/hdf5_io.c:353-523); the state lives on the GPU between
 * output times.  Plain pointers and sizes only; every call returns 0 on
 * success or a negative GOP_E* code, and never aborts.
 *
 * Array layout at this boundary is the reference's own: field-major, then
 * i, j, k with k fastest, every axis ghost-extended to n + 2*4 + 1 points
 * (src/config.h:10, src/config.c:184-186, src/array.c:87-114).
 */
#ifndef GAMERA_OP_H
#define GAMERA_OP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GOP_ABI_VERSION 1

/* error codes */
#define GOP_OK 0
#define GOP_EINVAL (-22)   /* bad argument */
#define GOP_ENOMEM (-12)   /* device allocation failed */
#define GOP_ECUDA (-5)     /* CUDA runtime error (see gop_last_error) */
#define GOP_ENODEV (-19)   /* no usable sm_100 device */
#define GOP_ESTATE (-71)   /* call out of order (e.g. step before prepare) */
#define GOP_ENUMERIC (-34) /* non-finite or non-positive state detected */
#define GOP_EBUSY (-16)    /* admission refused: memory budget exceeded */

/* coordinate systems: COORD_TYPE of CMakeLists.txt:77-95 */
#define GOP_COORD_CARTESIAN 0
#define GOP_COORD_SPHERICAL 2

/* ghost-fill kinds per face, the library of src/boundary_conditions.c plus
 * the periodic halo of src/boundary_exchange.c */
#define GOP_BC_PERIODIC 'p'
#define GOP_BC_SYMMETRIC 's'
#define GOP_BC_REFLECTIVE 'r'
#define GOP_BC_FIXED 'f'
#define GOP_BC_EXTRAPOLATED 'e'
#define GOP_BC_NONE 'n'
#define GOP_BC_POLE 'o' /* spherical j faces on a pole (src/spherical/spherical_boundary.c):
                           mirror across the axis with a half turn in phi; needs
                           ring_average */

/* arithmetic of the reconstruction / Riemann flux / edge-EMF stages */
#define GOP_PREC_FP64 0  /* plain: everything in FP64 (reference parity) */
#define GOP_PREC_MIXED 1 /* FP32 stages, FP64 state, AB2 and p recovery */

typedef struct {
  int ni, nj, nk;     /* active cells (config.ni/nj/nk), each >= 4 */
  int coord;          /* GOP_COORD_* */
  const double *x1;   /* face coordinates incl. ghosts: ni+9 values, x1[i][0][0] */
  const double *x2;   /* nj+9 values, x2[0][j][0] */
  const double *x3;   /* nk+9 values, x3[0][0][k] */
  char bc[6];         /* faces i-lo,i-hi,j-lo,j-hi,k-lo,k-hi (GOP_BC_*) */
  char gem_bc[6];     /* ghost fill of the face field per face; 0 = same as bc
                         (gas_bc_* and gem_bc_* are separate hooks in the reference) */
  int precision;      /* GOP_PREC_* */
  /* physics constants of src/config.c:82-97 (0 selects the default) */
  double gamma;       /* 5/3 */
  double cfl;         /* 0.3 */
  double ca;          /* Boris speed of light CA, 10 */
  double rho_floor;   /* 0.00316227 */
  double p_floor;     /* 0.000316227 */
  /* doRingAverage (src/spherical/spherical_RingAverage.c): on a spherical grid
   * whose theta range starts at 0 and/or ends at pi, the cells of the rings
   * nearest each pole are averaged in phi after every update (block
   * averages of nchunk(j) blocks with a parabolic profile), the face field
   * by the equivalent flux correction, the E and B fields on the pole faces
   * are fixed, and the CFL length in phi of those rings is scaled up.  nk
   * must be 32, 64, 128 or 256 and cover the full phi circle with periodic k
   * faces, and nj must leave room for both pole bands. */
  int ring_average;
} gop_desc;

typedef struct {
  double time;       /* time_sim */
  double dt;         /* dt of the last step */
  double dt0;        /* dt0 (previous dt, AB2 history) */
  double divb_max;   /* divB_max of the current state (src/solver_func.c:324-343) */
  int64_t steps;     /* steps taken since prepare */
  int32_t flags;     /* 1: non-finite or non-positive state was seen;
                        2: a device-side pipeline wait timed out */
  int32_t reserved;
  size_t device_bytes; /* device memory held by this instance */
} gop_stats;

typedef struct gop_instance gop_instance;

/* Replaces allocate_solver + set_geometry_arrays + getweights
 * (src/solver_init.c:378-392,471-476; src/main.c:56): allocates device
 * state and builds geometry and PDM weight tables from the coordinates. */
int gop_create(const gop_desc *desc, gop_instance **out);
int gop_destroy(gop_instance *h);

/* Device bytes gop_create would allocate for desc (admission control). */
size_t gop_footprint(const gop_desc *desc);

/* Runs the instance's work on this CUDA stream (cudaStream_t as void*;
 * NULL = default stream). */
int gop_set_stream(gop_instance *h, void *stream);

/* Copies the primitive state into the instance.  gas: 6 fields
 * rho,v1,v2,v3,p,p_S ([6][NI][NJ][NK], the store slots gas[0][0..5]);
 * face_b: 3 fields mag_bi,mag_bj,mag_bk ([3][NI][NJ][NK], gem[0..2]).
 * For a restart also pass the AB2 history gas_p (gas[0][12..17]) and
 * face_b_p (gem[9..11]) with dt0 and time; otherwise NULL. */
int gop_upload(gop_instance *h, const double *gas, const double *face_b,
               const double *gas_p, const double *face_b_p, double time,
               double dt0);

/* The start of solve() before its loop (src/solver_solve.c:25-99): ghost
 * fill, derived variables, and for a fresh start (restart == 0) the AB2
 * history copy and the initial CFL dt0. */
int gop_prepare(gop_instance *h, int restart);

/* nsteps passes of the time loop (src/solver_solve.c:102-529).  Stops early
 * once time > time_stop (pass a huge value to disable).  Asynchronous with
 * respect to the host unless time_out is non-NULL, or unless time_stop is
 * finite and nsteps > 256: the call then looks at the stop flag every 256
 * steps (synchronising the stream) so it returns soon after time_stop.
 * Steps replay a CUDA graph of one step, captured at the first call (and
 * again after gop_prepare changes the kernels, gop_set_background or
 * gop_autotune); with gop_set_profiling on, or while the instance's stream
 * is being captured by the caller, they are launched one by one. */
int gop_step(gop_instance *h, int nsteps, double time_stop, double *time_out);

/* Copies the state back in the reference layout: any pointer may be NULL.
 * gas/face_b as in gop_upload; gas_h, gas_p (6 fields each) and
 * face_b_h, face_b_p, mags, mags_h, mags_p (3 fields each) complete the
 * 18-slot store arrays the per-step HDF5 dump writes
 * (src/hdf5_io.c:479-508). */
int gop_download(gop_instance *h, double *gas, double *face_b, double *gas_h,
                 double *gas_p, double *face_b_h, double *face_b_p,
                 double *mags, double *mags_h, double *mags_p);

int gop_get_stats(gop_instance *h, gop_stats *out);

/* Autotuner: times candidate thread-block shapes for each of the 11
 * tunable launches of a step on the instance's current state (after
 * gop_prepare; the state is not advanced) and keeps the fastest for the
 * following steps; then the order of the three flux launches and of the
 * three edge-EMF launches (each order a rotation of the axes; the launches
 * are independent, so no result changes), timing two whole steps per
 * rotation with the state restored after each.  reps: timed launches per
 * candidate (0 = 3); chosen (optional, 11 ints) receives the picked
 * candidate index per launch. */
#define GOP_NTUNE 11
#define GOP_TUNE_SWEEP 14 /* chosen[] value of a flux or EMF launch: the tile-staged sweep kernel */
int gop_autotune(gop_instance *h, int reps, int *chosen);
/* The launch orders the autotuner picked (axes, 3 ints each; may be NULL). */
int gop_get_launch_order(gop_instance *h, int *flux_order, int *emf_order);

/* Kernel choice for the face fluxes and edge EMFs: on (the default) runs
 * the tile-staged sweep kernels (shared-memory tiles filled by the Tensor
 * Memory Accelerator, persistent blocks) wherever they apply, off the
 * per-point kernels; both give the same results.  With the entropy channel
 * live the per-face flux kernels always run.  GOP_ENODEV if the sweep
 * kernels could not be set up for this instance. */
int gop_set_sweep(gop_instance *h, int on);

/* Diagnostics: time every kernel group of every step with CUDA events on
 * the instance's stream (off by default; switching resets the totals).
 * Groups: 0 begin, 1 ab2, 2 centre-to-edge, 3 edge EMF, 4 face flux,
 * 5 update, 6 ghost fill, 7 end.  ms[g] and count[g] (GOP_NGROUP entries)
 * are the summed milliseconds and the number of timed occurrences. */
#define GOP_NGROUP 8
int gop_set_profiling(gop_instance *h, int on);
int gop_get_profile(gop_instance *h, double *ms, int64_t *count);

/* Diagnostics: the device's FP64 arithmetic peak in TFLOP/s, measured by a
 * timed loop of independent fused multiply-adds on `stream` (the
 * denominator of the step's FP64 roofline).  No counterpart in the
 * reference. */
int gop_measure_fp64_peak(double *tflops, void *stream);

/* Last error message of the calling thread ("" if none). */
const char *gop_last_error(void);

/* Kernels launched by this library since load (for launch accounting). */
int64_t gop_kernel_launches(void);

/* ---- CFL dt of a caller-owned device state, allocating nothing -------- */

/* No counterpart in the reference: GAMERA-OP has no GPU and no allocation
 * constraints.  This is the one entry point for callers that must not
 * allocate device memory -- a serving loop whose device memory was
 * reserved at start-up and may not grow (cudaMalloc there can fail, and it
 * and cudaFree wait for work running on the device), or a host program that
 * owns every device buffer itself and hands the library only pointers.
 *
 * gas (6 fields) and face_b (3 fields) are DEVICE pointers in the layout of
 * gop_upload.  b0 (3 fields, B0 at the cell centroid) and b0_face (9
 * fields, field 3d+c = component c averaged over the faces normal to axis
 * d) describe a background field in the layout gop_set_background takes,
 * as DEVICE pointers; both NULL for none.  out is a device pointer to 2
 * doubles: the CFL time step over the active cells (CFL over the sum, over
 * the three axes, of the fast signal speed -- |v| plus the fast
 * magnetosonic speed with the Boris-limited Alfven speed of the cell's total
 * field -- divided by the cell's length along that axis) and the largest
 * |div B| of the cell-integrated total face field.  Asynchronous on `stream`
 * (cudaStream_t as void*); it calls no cudaMalloc/cudaFree.  Grids with
 * ring_average set are rejected with GOP_EINVAL.
 *
 * Its scratch is one file-scope device array of GOP_NOALLOC_SCRATCH_DOUBLES
 * doubles (64 KiB), held by every GPU that loads the library until exit, so
 * grids are limited to GOP_NOALLOC_MAX_N active cells per axis (larger ones
 * are rejected with GOP_EINVAL).  The first call on a device looks up that
 * array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  The coordinate arrays of desc are copied into it
 * from the host on `stream` at every call.  All calls share the array:
 * calls whose kernels overlap on the GPU race. */
#define GOP_NOALLOC_MAX_N 1024
#define GOP_NOALLOC_SCRATCH_DOUBLES 8192
int gop_cfl_dt_noalloc(const gop_desc *desc, const double *gas, const double *face_b,
                       const double *b0, const double *b0_face, double *out, void *stream);

/* ---- host-only problem setup (no device work) ------------------------ */

/* Face coordinates of the reference's default uniform grid
 * (src/solver_init.c:297-321 with one process): n+9 values into x. */
int gop_grid_uniform(int n, double xmin, double xmax, double *x);

#define GOP_PROBLEM_OT 1        /* src/problem_test_OT_cartesion.c */
#define GOP_PROBLEM_BLAST 2     /* src/problem_test_Blast_cartesion.c, any centre / field */
#define GOP_PROBLEM_LOOP_CART 3 /* src/problem_FieldLoop_cartesian.c */
#define GOP_PROBLEM_LOOP_SPH 4  /* field loop advected through a pole-free spherical shell */

typedef struct {
  int kind;          /* GOP_PROBLEM_* */
  double rho;        /* background density */
  double p_in;       /* blast: pressure inside radius */
  double p_out;      /* blast: ambient pressure; loops: pressure */
  double radius;     /* blast radius */
  double center[3];  /* blast centre */
  double b[3];       /* blast: uniform face field */
  double v[3];       /* loops: uniform Cartesian velocity */
  double loop[4];    /* loop_sph: axis x, axis y, radius R, amplitude A0 */
} gop_problem;

/* Fills p with the reference problem's values for kind. */
void gop_problem_defaults(int kind, gop_problem *p);

/* Writes the initial primitive state (6 fields) and face field (3 fields)
 * of problem p on desc's grid, in the layout of gop_upload.  Ghost cells are
 * left for gop_prepare to fill, exactly as problem_init leaves them
 * (src/main.c:57-61). */
int gop_problem_init(const gop_desc *desc, const gop_problem *p, double *gas, double *face_b);

/* The same initial state built on the device, directly in h's current state
 * (what gop_problem_init followed by gop_upload(h, gas, face_b, NULL, NULL,
 * 0, 0) leaves, to the last bits of the device's sin/cos/exp/acos/atan2):
 * cells, then for the potential problems AinitB's edge integrals
 * (src/solver_func.c:15-95, in the instance's work arrays as scratch) and
 * the face field.  gop_prepare follows as after gop_upload.  GOP_EINVAL if
 * the problem does not fit the instance's geometry.  The reference builds
 * its initial state on the host (problem_init). */
int gop_problem_init_device(gop_instance *h, const gop_problem *p);

/* ---- background magnetic field B0 ------------------------------------ */
/* The reference adds a time-independent background field B0 (the problem
 * sets its B10/B20/B30 hooks; set_background_field, src/solver_func.c:
 * 1851-2077, integrates it once) to the face fluxes, the magnetic stress,
 * the edge EMFs, the Alfven correction and the CFL dt.  Four groups of
 * arrays describe it, each field [i][j][k] like gop_upload's:
 *   b0       3 fields: B0 at the cell centroid (B0_b1..3)
 *   lorentz  3 fields: the Lorentz force of B0 (dmagsf_G_x1..3dir)
 *   b0_face  9 fields: field 3d+c = component c averaged over the faces
 *            normal to axis d (B0AfaceI/J/K_b1..3)
 *   b0_edge  9 fields: field 3d+c = component c averaged along the edges of
 *            axis d (B0AedgeI/J/K_b1..3; active range only)
 * gop_set_background installs them (all four, or all NULL to remove the
 * background); gop_prepare must follow, and a batch must be created after
 * it.  The instance then holds 24 more fields of doubles on the device than
 * gop_footprint counts. */
int gop_set_background(gop_instance *h, const double *b0, const double *lorentz,
                       const double *b0_face, const double *b0_edge);

#define GOP_BG_UNIFORM 1  /* constant b (src/common.c B10_uniform with b = 1/sqrt2) */
#define GOP_BG_DIPOLE 2   /* moment * (3xz, 3yz, 2z^2-x^2-y^2) / r^5 (src/common.c
                             B10_dipole with moment 1), evaluated on the grid's own
                             coordinates as the reference does */
typedef struct {
  int kind;          /* GOP_BG_* */
  double b[3];       /* uniform: the field */
  double moment;     /* dipole: scale of the reference's unit dipole */
} gop_background;

/* The same for one of the built-in backgrounds computed on the device,
 * straight into the instance's background block (the work of
 * gop_background_init, which takes seconds on the host for a large dipole
 * grid, without the host arrays or their upload); gop_prepare must follow.
 * The arrays agree with gop_background_init's to the last bits of the
 * device's pow, sin and cos. */
int gop_set_background_device(gop_instance *h, const gop_background *bg);

/* Copies the instance's background field back in gop_set_background's
 * layout (any pointer may be NULL); GOP_ESTATE without a background. */
int gop_get_background(gop_instance *h, double *b0, double *lorentz, double *b0_face,
                       double *b0_edge);

/* set_background_field on the host for one of the built-in backgrounds (no
 * volume source, as in every reference problem): the 12x12 Gauss face
 * averages with the metric scale factors, the 12-point edge averages and
 * the Lorentz force from the face stresses; arrays as gop_set_background
 * takes them. */
int gop_background_init(const gop_desc *desc, const gop_background *bg, double *b0,
                        double *lorentz, double *b0_face, double *b0_edge);

/* ---- batched stepping of many independent instances ---------------- */
typedef struct gop_batch gop_batch;

/* Groups instances (all already prepared, each at most once, at most 65535)
 * so one call advances each by its own number of steps.  One step of all
 * members is captured once in a CUDA graph: each member's own launch
 * sequence (its gop_step launches) on one of up to 16 parallel branches,
 * largest members placed first on the least-loaded branch, so the members
 * run side by side; the graph is replayed max(steps) times.  The members
 * may differ in size, geometry, boundary kinds and precision.  The members
 * must outlive the batch.  No counterpart in the reference, which runs one
 * domain per process. */
int gop_batch_create(gop_instance *const *members, int count, gop_batch **out);
int gop_batch_destroy(gop_batch *b);
/* steps[m] >= 0 per member (indexed as at creation); returns when all are
 * done.  Each member ends exactly as gop_step(member, steps[m], 1e300, ..)
 * would leave it; GOP_ENUMERIC if any member saw a non-finite state. */
int gop_batch_step(gop_batch *b, const int *steps);
/* gop_batch_step in two halves: launch enqueues the steps on the batch's
 * own non-blocking stream and returns; wait blocks until they are done and
 * checks the members' flags.  Between the two the host may create, upload
 * and prepare other instances (their set-up does not wait for the batch);
 * it must not touch the members or destroy any instance (cudaFree waits for
 * the whole device). */
int gop_batch_launch(gop_batch *b, const int *steps);
int gop_batch_wait(gop_batch *b);
/* Launches of the batch go to `stream` (cudaStream_t as void*; NULL: the
 * batch's own non-blocking stream). */
int gop_batch_set_stream(gop_batch *b, void *stream);
/* Chooses thread-block shapes for the members: gop_autotune on the first
 * member of each class of equal grid shape, geometry and precision, copied
 * to the rest of the class, then captures the batch graph again; then
 * times replays of the batch step with those picks and with every member
 * on the per-point flux and EMF kernels (the tile-staged sweeps, picked
 * with each grid alone, share the SMs with the other members' kernels in
 * a batch) and keeps the faster (skipped without device memory for a copy
 * of every member's state).  chosen[GOP_NTUNE] (may be NULL) receives the
 * candidate indices of the class with the most cells, as gop_autotune
 * picked them.  The state and scalars of every member are left as they
 * were. */
int gop_batch_autotune(gop_batch *b, int reps, int *chosen);

#ifdef __cplusplus
}
#endif
#endif
