/*
 * pppm_b200.h - C ABI of the B200-native PPPM-TDBEM time-step library (libpppm_b200.so).
 *
 * The reference (hellojxt/PPPM-TDBEM) exposes its hot path only as the C++ class
 * PPPMSolver (src/algorithm/pppm.h:11-165) driven by the demo loop
 * (experiments/demo/main.cu:170-275).  This header is the C boundary that replaces that
 * class for foreign callers (the C++ scene host in pppm-tdbem_b200/host, the Python
 * ctypes binding and torch.autograd.Function, test harnesses).  Each entry point cites the
 * reference member it replaces.
 *
 * Conventions
 *   - Every call returns an int status (PPPM_OK == 0) and never throws or exits.
 *   - Grids are res^3, cell (x, y, z) at linear index (x * res + y) * res + z (z fastest),
 *     the reference layout (src/core/array3D.h:76).
 *   - Vertices are float[3 * nv] (x, y, z interleaved); triangles int[3 * nt].
 *   - Time index t starts at -1; each step writes grid slot t + 1 then increments t
 *     (src/algorithm/fdtd.h:55,73-87).  Histories are rings of 32 slots per triangle
 *     (src/algorithm/bem.h:55).
 *   - A handle owns all its device memory and one CUDA stream.  Calls on one handle are not
 *     thread-safe; distinct handles may be used from distinct host threads.
 */
#ifndef PPPM_B200_H
#define PPPM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes ----- */
#define PPPM_OK 0
#define PPPM_ERR_ARG 1      /* bad argument (null pointer, index out of range, bad size)  */
#define PPPM_ERR_CUDA 2     /* a CUDA runtime call failed; see pppm_last_error_message()   */
#define PPPM_ERR_CAPACITY 3 /* a mesh exceeds a structural limit (see pppm_limits)         */
#define PPPM_ERR_NAN 4      /* a non-finite value reached the listener / state            */
#define PPPM_ERR_STATE 5    /* call out of order (e.g. step before set_mesh)              */
#define PPPM_ERR_TIMEOUT 6  /* a bounded device-side wait gave up                         */
#define PPPM_ERR_NOMEM 7    /* device allocation failed                                   */

/* ------------------------------------------------------------------ parameters ------- */
#define PPPM_PRECISION_FP32 0 /* FP32 grids/histories, fp16+scale weights (the reference's) */
#define PPPM_PRECISION_FP64 1 /* FP64 everywhere, unquantised weights: the error yardstick  */

#define PPPM_WEIGHTS_REF32 0 /* TDBEM weights in FP32 with the reference's arithmetic       */
#define PPPM_WEIGHTS_FP64 1  /* singular and near-singular face integrals in FP64           */

#define PPPM_METHOD_PPPM 0  /* FDTD + TDBEM near-field correction (PPPMSolver)              */
#define PPPM_METHOD_GHOST 1 /* FDTD + ghost cells (GhostCellSolver, ghost_cell.h:72-152);
                               FP32 handles, absorbing boundary                             */

typedef struct pppm_params {
    int res;               /* grid resolution (cells per axis), >= 8                      */
    float dl;              /* cell size h                                                 */
    float dt;              /* time step                                                   */
    float min_pos[3];      /* world position of the grid's lower corner                   */
    int pml_width;         /* PML layers; 0 = the reference's absorbing boundary (ABC)     */
    float reflect_coeff;   /* Dirichlet far-field factor, reference default 0.83          */
    float c;               /* speed of sound, reference hard-codes 340.3 (macro.h:82)     */
    float rho;             /* air density 1.225 (macro.h:83)                              */
    int precision;         /* PPPM_PRECISION_*                                            */
    int weights;           /* PPPM_WEIGHTS_*                                              */
    int device;            /* CUDA device ordinal                                         */
    void *stream;          /* cudaStream_t to use, or NULL to create one                  */
    int method;            /* PPPM_METHOD_*                                               */
    float ghost_threshold; /* ghost-cell method: condition number above which a ghost cell
                              falls back to first order (reference 25); 0 = first order
                              everywhere with thin-shell labels (ghost_cell.h:77, :95)     */
} pppm_params;

typedef struct pppm_handle pppm_handle;

/* Fill *p with the reference defaults (PPPMSolver constructor defaults, pppm.h:39-44). */
int pppm_params_default(pppm_params *p);

/* Replaces PPPMSolver::PPPMSolver(res, dl, dt, min_pos, pml_width, reflect_coeff)
 * (pppm.h:39-54).  Allocates the three grid time levels. */
int pppm_create(const pppm_params *p, pppm_handle **out);

/* Replaces PPPMSolver::clear() + delete (pppm.h:111-126). */
int pppm_destroy(pppm_handle *h);

/* Replaces PPPMSolver::set_mesh(verts, tris) (pppm.h:75-95): triangle geometry, per-cell
 * lists, 3^3 / 4^3 neighbour lists, GridCache and FaceCache weights, zeroed histories. */
int pppm_set_mesh(pppm_handle *h, const float *verts, int nv, const int *tris, int nt);

/* Replaces PPPMSolver::update_mesh(verts) (pppm.h:97-109): same topology, new vertex
 * positions; lists rebuilt, caches refreshed under the reference's recompute criteria
 * (pppm_cache.h:65-70, 123-128).  verts_on_device != 0: verts is a device pointer. */
int pppm_update_mesh(pppm_handle *h, const float *verts, int verts_on_device);

/* Replaces nsteps calls of PPPMSolver::update_grid_and_face(acc) (pppm.h:138-145).
 * acc holds nsteps rows of nt per-triangle normal accelerations (row s drives step s);
 * acc_on_device != 0: acc is a device pointer.  Listener values are recorded on the device
 * after every step (the demo's per-step read, experiments/demo/main.cu:266).  The call returns
 * once the steps are queued.  The step kernels raise a device status bit when a Dirichlet value
 * or a listener sample is not finite (the reference aborts on a NaN listener sample,
 * experiments/demo/main.cu:161-168); a copy of that word is queued behind the steps, and a later
 * pppm_step whose predecessors' copy has arrived returns PPPM_ERR_NAN without queuing anything,
 * until pppm_reset_fields or pppm_restore_state clears it. */
int pppm_step(pppm_handle *h, const float *acc, int acc_on_device, int nsteps);

/* No counterpart in the reference.  Waits for the handle's queued work and returns its step
 * status: PPPM_ERR_NAN once a non-finite Dirichlet value or listener sample appeared. */
int pppm_sync(pppm_handle *h);

/* Listener cells (experiments/demo/main.cu:148: int3(checkCoord * res)). */
int pppm_add_listener(pppm_handle *h, int x, int y, int z);
int pppm_clear_listeners(pppm_handle *h);
/* Number of recorded steps so far and listener count. */
int pppm_listener_count(pppm_handle *h, int *nsteps, int *nlisteners);
/* Copy recorded samples [first, first + count) x nlisteners into out (host). */
int pppm_read_listeners(pppm_handle *h, int first, int count, float *out);
/* No counterpart in the reference.  The same samples in the handle's element type (float for
 * FP32 handles, double for FP64), into a device buffer on the handle's stream (on_device != 0,
 * returns once queued) or a host buffer; non-finite samples are not checked. */
int pppm_read_listeners_raw(pppm_handle *h, int first, int count, void *out, int on_device);
int pppm_rewind_listeners(pppm_handle *h);

/* No counterpart in the reference.  The CUDA stream every call of the handle queues its work on
 * (the one given in pppm_params, or the handle's own), for ordering other work against it. */
int pppm_get_stream(pppm_handle *h, void **stream);

/* Current time index t (fdtd.t). */
int pppm_get_time(pppm_handle *h, int *t);
int pppm_set_time(pppm_handle *h, int t);

/* Replaces pg.fdtd.reset() + neumann.reset() + dirichlet.reset() (demo/main.cu:240-242):
 * zero grids and histories; t is kept (the demo restores it explicitly). */
int pppm_reset_fields(pppm_handle *h);

/* Whole solver state (grids, histories, PML fields, t) into / from a caller-owned host
 * buffer: cross-fade restart (demo/main.cu:215-244). */
int pppm_state_size(pppm_handle *h, size_t *bytes);
int pppm_save_state(pppm_handle *h, void *dst, size_t bytes);
int pppm_restore_state(pppm_handle *h, const void *src, size_t bytes);

/* ----------------------------------------------------------- read-out for parity ----- */
#define PPPM_DUMP_GRID_T 0        /* float/double res^3: grid slot t                     */
#define PPPM_DUMP_GRID_TM1 1      /* grid slot t-1                                       */
#define PPPM_DUMP_GRID_TM2 2      /* grid slot t-2                                       */
#define PPPM_DUMP_NEUMANN 3       /* nt x 32 ring                                        */
#define PPPM_DUMP_DIRICHLET 4     /* nt x 32 ring                                        */
#define PPPM_DUMP_TRI_GEOM 5      /* float nt x 7: centre xyz, normal xyz, area          */
#define PPPM_DUMP_TRI_CELLS 6     /* int nt x 6: grid coord xyz, base coord xyz          */
#define PPPM_DUMP_CELL_COUNTS 7   /* int res^3 triangles per cell                        */
#define PPPM_DUMP_N3_CELLS 8      /* int n3 x 4: x, y, z, 3^3 list length                */
#define PPPM_DUMP_N3_TRIS 9       /* int p3: concatenated 3^3 lists                      */
#define PPPM_DUMP_B4_CELLS 10     /* int b4 x 4: x, y, z, base-cell list length          */
#define PPPM_DUMP_B4_TRIS 11      /* int: concatenated base-cell lists                   */
#define PPPM_DUMP_N4_TRIS 12      /* int p4: concatenated 4^3 lists, one per base cell   */
#define PPPM_DUMP_GRID_CACHE 13   /* nt x 54 x 72 B LayerWeightHalf records (FP32 mode)  */
#define PPPM_DUMP_FACE_PAIRS 14   /* int pf x 2: (centre, neighbour) in hot-path order   */
#define PPPM_DUMP_FACE_CACHE 15   /* pf x 72 B weights in the same order (FP32 mode)     */
#define PPPM_DUMP_INTERP 16       /* float nt x 8 trilinear face weights                 */
#define PPPM_DUMP_CELL_TYPE 17    /* int res^3 labels AIR 0 SOLID 1 GHOST 2 UNKNOWN 3    */
#define PPPM_DUMP_CELL_NEAREST 18 /* int res^3 nearest triangle (-1 if none)             */
#define PPPM_DUMP_CELL_GHOST 19   /* int res^3 ghost index (-1 if not GHOST)             */
#define PPPM_DUMP_CELL_POINTS 20  /* float res^3 x 7: nearest xyz, reflect xyz, distance */
#define PPPM_DUMP_COUNTS 21       /* int[8]: n3, p3, b4, p4(pairs per centre), pf, nt, nv, ghost count */
#define PPPM_DUMP_GHOST_CELLS 22  /* ghost-cell method: int ghosts: linear cell index of each ghost */
#define PPPM_DUMP_GHOST_ORDER 23  /* int ghosts: 1 = first order, 0 = second order             */
#define PPPM_DUMP_GHOST_WEIGHTS 24 /* float ghosts x 8: reflection-point interpolation weights */
#define PPPM_DUMP_GHOST_ITERS 25  /* int: BiCGSTAB iterations of the last step's solve         */

int pppm_dump_size(pppm_handle *h, int what, size_t *bytes);
int pppm_dump(pppm_handle *h, int what, void *dst, size_t bytes);

/* Overwrite one grid slot (what = PPPM_DUMP_GRID_T/TM1/TM2) or one history ring
 * (PPPM_DUMP_NEUMANN / PPPM_DUMP_DIRICHLET) from host memory; used to set initial
 * conditions and by the parity harness.  Element type follows the handle's precision. */
int pppm_load(pppm_handle *h, int what, const void *src, size_t bytes);

/* Parity mode: replace the GridCache / FaceCache tables with tables read out of the
 * reference (same record layout as PPPM_DUMP_GRID_CACHE and PPPM_DUMP_FACE_CACHE).
 * face_pairs lists (centre, neighbour) for each face record.  FP32 handles only. */
int pppm_import_grid_cache(pppm_handle *h, const void *records, size_t bytes);
int pppm_import_face_cache(pppm_handle *h, const int *face_pairs, const void *records, int npairs);

/* ------------------------------------------------------------ cell labels ------------ */
/* Replaces fill_cell_data (ghost_cell_util.cu:214-230): nearest triangle within +-3 cells,
 * AIR / SOLID / GHOST / UNKNOWN labels, z-column sweep, ghost indices.  Reads the current
 * mesh.  *ghost_count receives the number of GHOST cells (may be NULL). */
int pppm_classify_cells(pppm_handle *h, int *ghost_count);

/* Replaces GhostCellSolver::fill_in_fresh_cell (ghost_cell.cu:207-218) for a moving mesh:
 * re-label after the last update_mesh and fill cells that turned from non-AIR to AIR in grid
 * slots t and t-1 by inverse-distance interpolation at the reflection point, minus
 * rho * a * |xf - xr|.  acc / acc_old: current and previous per-triangle accelerations
 * (host).  *fresh_count receives the number of fresh cells (may be NULL). */
int pppm_fill_fresh_cells(pppm_handle *h, const float *acc, const float *acc_old, int *fresh_count);

/* ------------------------------------------------------------ batched scenes --------- */
/* Many independent scenes advanced together by one persistent kernel per step under a
 * captured CUDA graph; no reference counterpart (the reference runs one scene per process).
 * Scenes are ordinary handles that already hold their mesh; nsteps[i] may differ. */
typedef struct pppm_batch pppm_batch;
int pppm_batch_create(pppm_handle **scenes, int nscenes, pppm_batch **out);
int pppm_batch_destroy(pppm_batch *b);
/* acc[i]: nsteps[i] x nt_i rows for scene i (device pointers when acc_on_device != 0). */
int pppm_batch_run(pppm_batch *b, const float *const *acc, const int *nsteps, int acc_on_device);

/* ------------------------------------------------------------ adjoint ---------------- */
/* No counterpart in the reference.  Gradient of L = sum_s sum_l dL_dsignal[s][l] * p_l(s)
 * over nsteps consecutive forward steps with respect to those steps' accelerations,
 * dL_dacc[s][tri], with the weight tables, lists and corrected cells the handle holds now
 * (the absorbing boundary or the PML, whichever the handle uses).  The listener samples are linear
 * in the accelerations, so the gradient does not depend on the forward state and no forward
 * state is stored: the transposed step runs backwards in time on adjoint state of the forward
 * state's size.  fresh != 0 starts a new reverse sweep (the nsteps steps are the last ones of
 * the differentiated run); fresh == 0 continues the sweep the previous call left, for the
 * nsteps steps just before the ones that call covered (a long run differentiated in chunks,
 * latest chunk first).  The adjoint state carries over a change of geometry between chunks:
 * a moving run is differentiated motion frame by motion frame, latest first, each call with
 * that frame's tables in the handle (pppm_save_cache_state / pppm_restore_cache_state and
 * pppm_update_mesh rebuild them exactly).  Element type: float for FP32 handles, double for
 * FP64 handles.  dL_dsignal: nsteps x nlisteners; dL_dacc: nsteps x nt; both device pointers
 * on the handle's stream when on_device != 0 (the call returns once the work is queued), else
 * host buffers (the call returns with dL_dacc written).  Listeners must lie in [1, res-2]^3. */
int pppm_adjoint(pppm_handle *h, const void *dL_dsignal, int nsteps, int on_device, int fresh, void *dL_dacc);

/* No counterpart in the reference.  The motion-frame state of the weight caches: the
 * grid-cache records with the triangle geometry they were computed for, the face-cache table
 * with its record pool, and the vertex positions.  A moving run's tables depend on its whole
 * motion so far: records are recomputed only when their geometry moved past the reference's
 * criteria (pppm_cache.h:65-70, 123-128).  Saving the state after a frame's pppm_set_mesh /
 * pppm_update_mesh and restoring it later, followed by pppm_update_mesh with that frame's
 * vertices (which then recomputes nothing) and with each later frame's vertices in turn,
 * rebuilds exactly the tables those frames had: the checkpoints of a frame-by-frame adjoint
 * (pppm_b200.autograd.moving_listener_signal).  The blob may sit in host memory or in device
 * memory (a checkpoint kept in HBM: copies go through unified addressing); both calls return
 * once the copies are done.  A restore leaves the handle's lists stale, and pppm_step /
 * pppm_adjoint return PPPM_ERR_STATE until pppm_update_mesh. */
int pppm_cache_state_size(pppm_handle *h, size_t *bytes);
int pppm_save_cache_state(pppm_handle *h, void *dst, size_t bytes);
int pppm_restore_cache_state(pppm_handle *h, const void *src, size_t bytes);

/* No counterpart in the reference.  Motion checkpoints for differentiating long moving runs,
 * kept by the handle in device memory: a checkpoint holds the vertex positions and the
 * grid-cache records of the current frame (a res-128 scene of 40960 triangles: about 160 MB)
 * and the size of the face-cache record pool; the pool itself stays in place, later refreshes
 * log the old records of the pool entries they rewrite.  pppm_checkpoint_push takes one after
 * the frame's pppm_set_mesh / pppm_update_mesh (*id: its index, 0 first); pppm_checkpoint_rewind
 * brings the caches back to checkpoint id and drops the later ones (a pppm_update_mesh with
 * that frame's vertices must follow before pppm_step / pppm_adjoint, which return
 * PPPM_ERR_STATE until then; further pppm_update_mesh calls replay the motion with the tables
 * the run had).  Checkpoints go on pppm_checkpoint_clear, pppm_set_mesh, a cache-state restore
 * or a weight import.  Their device memory is an arena kept for the next run of checkpoints
 * until pppm_checkpoint_clear with release != 0 (or pppm_set_mesh / pppm_destroy) frees it.
 * pppm_checkpoint_info: how many are held and the device bytes the arena and logs use. */
int pppm_checkpoint_push(pppm_handle *h, int *id);
int pppm_checkpoint_rewind(pppm_handle *h, int id);
int pppm_checkpoint_clear(pppm_handle *h, int release);
int pppm_checkpoint_info(pppm_handle *h, int *count, size_t *bytes);

/* ------------------------------------------------------------ weight diagnostics ----- */
/* TDBEM::init (bem.h:264-277) as this library evaluates it on the host: lambda and the 16
 * complex wave numbers (wave[2k] real, wave[2k+1] imaginary).  No device is touched. */
int pppm_tdbem_constants(float dt, float dl, float c, float *lambda, float *wave32);
/* TDBEM::laplace_weight (bem.h:306-330) of one pair evaluated on device `device` with the
 * FP32 weight arithmetic of the caches: src triangle (indices into verts) onto a point
 * (to_point != 0) or onto dst_face.  out32: 16 single-layer then 16 double-layer taps.  The
 * calling thread's current device is restored before the call returns. */
int pppm_pair_weights(int device, float dt, float dl, float c, const float *verts, int nv, const int *src,
                      int to_point, const int *dst_face, const float *dst_point, float *out32);
/* No counterpart in the reference.  pppm_pair_weights without any device allocation, for
 * callers that cannot allocate: a thread working beside a handle that is stepping on the same
 * device (cudaMalloc / cudaFree may synchronise the whole device and stall that handle's stream)
 * or a process whose device memory is already held by another allocator.  Same arguments and
 * result as pppm_pair_weights, plus the stream the copies and the kernel run on; returns after
 * out32 is written.  NULL means the legacy default stream, which waits for every blocking stream
 * on the device (a handle's stepping stream included, unless it was created non-blocking): pass a
 * stream created with cudaStreamNonBlocking to work beside queued steps.  A stream that is being
 * captured returns PPPM_ERR_STATE (the call synchronises its stream).  The calling thread's
 * current device is restored before the call returns.  The vertex rows are staged in a static
 * device array of PPPM_STATIC_MAX_VERTS rows (768 KiB) inside the library; nv above that limit
 * returns PPPM_ERR_CAPACITY.  Nothing in that array has to start at zero: each call copies its
 * rows in and the kernel writes all 32 taps.  The first call on a device does one-time setup
 * (it looks up the array's device address, which may load the library's device code); make that
 * call before capturing any stream on the device.  All calls on one device share the array, so
 * overlapping calls would race: calls from several host threads are serialised by a lock. */
#define PPPM_STATIC_MAX_VERTS 65536
int pppm_pair_weights_static(int device, void *stream, float dt, float dl, float c, const float *verts, int nv,
                             const int *src, int to_point, const int *dst_face, const float *dst_point, float *out32);

/* ------------------------------------------------------------ tuning ----------------- */
/* No counterpart in the reference.  Launch options of the recorded step graphs (pppm_step calls
 * of 4 or more steps with the absorbing boundary).  A change takes effect at the next such call,
 * which records new graphs. */
#define PPPM_OPT_CONV_PAIRS 0   /* 1 (default): the face-pair convolution streams the pairs' weights
                                   once for two consecutive steps; 0: once per step             */
#define PPPM_OPT_FACE_THREADS 1 /* threads per block of the face-stage kernels: 64, 128, 256    */
#define PPPM_OPT_TERMS_PAIRS 2  /* 1 (default): the triangles' grid-cache near-field terms are
                                   evaluated two steps per pass over their records; 0: per step */
#define PPPM_OPT_SPLIT_STENCIL 3 /* 1 (default): the stencil of the corrected cells stays on the
                                    graph's critical branch (the face and near stages read no other
                                    cell) and the rest of the grid runs on a branch beside them;
                                    0: one stencil launch before the face stage.  Same results.  */
#define PPPM_OPT_GRAPH_CHUNK 4  /* 32 (default): a call of more steps replays one recorded graph of
                                   this many steps as often as it fits, then a graph of the 1..32
                                   steps left, so frames of uneven length record a few short
                                   graphs instead of one long graph per length; 0: one graph per
                                   call; otherwise an even number in [2, 4096].  Same results. */
#define PPPM_OPT_STENCIL_VEC4 5 /* the FP32 interior stencil with res a multiple of 4: 1 four
                                   consecutive z cells per thread with 16-byte loads, 0 one cell per
                                   thread, -1 (default) four from res 96 up; pppm_autotune times both
                                   and keeps the faster.  Same results.                          */
int pppm_set_option(pppm_handle *h, int option, int value);
int pppm_get_option(pppm_handle *h, int option, int *value);
/* No counterpart in the reference.  Autotuner of the face stage, on the current mesh and state.
 * Phase 1 times kernels alone: two steps of the face-pair convolution in 6 configurations
 * (candidate i < 6: PPPM_OPT_CONV_PAIRS = i / 3, threads = {64, 128, 256}[i % 3]), then two steps
 * of the rest of the face stage with the near-field terms one pass per step (candidate 6) or two
 * steps per pass (candidate 7), reps launches of each kernel.  Phase 2 (absorbing boundary) times
 * 64 recorded steps (zero accelerations) of each of PPPM_TUNE_CONFIGS option sets (config j: conv_pairs = j / 6,
 * threads = {64, 128, 256}[(j / 2) % 3], terms_pairs = j % 2) from a device snapshot of the
 * fields and histories (a warm-up replay, then a timed one; best of min(reps, 3)) and sets the options to
 * the fastest (with a PML, phase 1 decides).  us_out (may be NULL; 2 * PPPM_TUNE_CANDIDATES +
 * PPPM_TUNE_CONFIGS floats): microseconds per launch of candidate i's first kernel (us_out[2 i])
 * and second kernel (us_out[2 i + 1]), then microseconds per step of each config; *best (may be
 * NULL): the config chosen (or, with a PML, the convolution candidate).  The fields, histories,
 * time and recorded listener samples are as before the call; it allocates a snapshot of the
 * fields and histories for its duration and records CUDA graphs, so it must not be called while
 * the handle's stream is being captured.  Needs a mesh and the PPPM method. */
#define PPPM_TUNE_CANDIDATES 8
#define PPPM_TUNE_CONFIGS 12
int pppm_autotune(pppm_handle *h, int reps, float *us_out, int *best);

/* ------------------------------------------------------------ diagnostics ------------ */
const char *pppm_status_string(int status);
const char *pppm_last_error_message(void);
/* Kernel launches issued by this handle since creation (for launch accounting). */
int pppm_launch_count(pppm_handle *h, long long *count);
/* Measurement mode: with timing enabled every step records CUDA events around each of its
 * kernels and synchronises; pppm_kernel_times returns the mean duration per kernel in
 * microseconds over the steps timed since pppm_enable_timing, and their number. */
int pppm_enable_timing(pppm_handle *h, int enable);
int pppm_kernel_times(pppm_handle *h, float *us_stencil, float *us_face, float *us_near, int *timed_steps);
/* No counterpart in the reference.  Measurement mode per kernel: where the recorded step graphs
 * run the split face stage (absorbing boundary, PPPM method, mesh set), steps in measurement mode
 * go in groups of four through a recorded graph of exactly those kernels (Neumann write, then per
 * step the face-pair convolution, the stencil, finish, near), serialised on the handle's stream
 * with an event between consecutive kernels; remaining steps and other handles time the fused
 * kernels.  Per kind: us_per_launch[k] = mean event-to-event time of its launches, launches[k]
 * their number (both arrays of nkinds entries, nkinds <= PPPM_KERNEL_KINDS). */
#define PPPM_KERNEL_STENCIL 0 /* FDTD / absorbing-boundary stencil (or the PML stencil)       */
#define PPPM_KERNEL_CONV 1    /* face-pair convolution, one step per pass                    */
#define PPPM_KERNEL_CONV2 2   /* face-pair convolution, two steps per pass                   */
#define PPPM_KERNEL_FIX 3     /* completion of the second step of a two-step pass            */
#define PPPM_KERNEL_FINISH 4  /* far field, Dirichlet update, near-field terms in one pass    */
#define PPPM_KERNEL_FINISH1 5 /* ... first step of a two-step pass over the grid-cache records */
#define PPPM_KERNEL_FINISH2 6 /* ... second step (completion of its terms)                    */
#define PPPM_KERNEL_NEAR 7    /* corrected cells: sums of the near-field terms                */
#define PPPM_KERNEL_NWRITE 8  /* Neumann history write of a call's first step                 */
#define PPPM_KERNEL_FACE 9    /* the fused face stage of direct launches                      */
#define PPPM_KERNEL_EMPTY 10  /* an empty one-block kernel between the Neumann write and the first
                                 convolution: the event-to-event floor of this measurement      */
#define PPPM_KERNEL_STENCIL_BULK 11 /* the split stencil: every cell but the corrected ones     */
#define PPPM_KERNEL_STENCIL_CORR 12 /* the split stencil: the corrected cells                   */
#define PPPM_KERNEL_KINDS 13
int pppm_kernel_profile(pppm_handle *h, int nkinds, float *us_per_launch, long long *launches);
/* No counterpart in the reference.  Duration of each step kernel kind on the current mesh and
 * state: reps back-to-back launches of the kind (those of the next step) recorded as one CUDA
 * graph, replayed once to warm up and once between two events; us_per_launch[k] = that time / reps
 * (the kernel plus the gap between dependent graph nodes; 0 for kinds not timed: NWRITE, EMPTY).
 * The launches write only the next step's grid slot, history slots and scratch, and the handle
 * rebuilds the state the next step reads afterwards, so stepping continues unchanged.  Absorbing
 * boundary, PPPM method, mesh set; not while the handle's stream is being captured. */
int pppm_time_kernels(pppm_handle *h, int reps, int nkinds, float *us_per_launch);

#ifdef __cplusplus
}
#endif

#endif /* PPPM_B200_H */
