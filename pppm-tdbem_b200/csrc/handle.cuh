// The solver handle: every device array of one scene, and the internal entry points the
// C ABI (capi.cu) strings together.
//
// HBM layout (one scene):
//   grid[3]        res^3 real each, x-major / z-contiguous (reference layout); ring by t.
//                  Between the near-field kernel of step t and the stencil kernel of step
//                  t+1 the dead slot t+1 carries, at corrected cells only, the FDTD-near
//                  correction of step t+1 (see step.cu).
//   pml[3]         res^3 x 6 real (PML only)
//   neumann/dirichlet  nt x 32 real rings in the reference layout (slot = t mod 32), kept
//                  current by every history write, for read-out and loading; the step reads
//                  hist, four shifted 16-slot copies (copy c holds time tau at (c - tau) mod 16)
//                  with both fields of a triangle in one row, so a lane's 4 Neumann and 4
//                  Dirichlet taps are one aligned load
//   cell CSR       cell_start[res^3 + 1] / cell_tris[nt] (sorted by triangle id per cell),
//                  same for base cells
//   3^3 pairs      n3 corrected cells: n3_cell, n3_start[n3 + 1]; p3 pairs: p3_tri, p3_woff
//                  (the pair's record offset in the triangle's grid-cache records)
//   near terms     terms[nt][54]: each triangle's 54 grid-cache records convolved with its own
//                  history in the current step (step.cu); a corrected cell sums its pairs' terms
//   face pairs     face_start[nt + 1] per centre triangle; pf pairs: face_nbr; dense
//                  weights face_half[pf][32] + face_scale[pf][2]; per centre: 8 corner cells,
//                  8 trilinear weights, denominator 0.5 * area - sum(factor)
//   caches         grid cache nt x 54 records (persistent, with the geometry snapshot of the
//                  last refresh); face cache per-centre open-addressing table
//                  (kFaceCacheSlots keys) into a growable record pool
#pragma once
#include <vector>
#include "common.cuh"
#include "tdbem.cuh"

namespace pb
{

// The per-call values of a pppm_step call live in device memory (one StepState per handle,
// written before the launches), so the kernels of a call can be recorded once as a CUDA graph
// and replayed for every later call with the same number of steps: kernel k of a call derives
// its time index, series row and acceleration row from the state and its own k (step.cu).
struct StepState
{
    int tnew0;         // time index produced by the call's first step
    int n3;            // corrected cells
    long long row0;    // listener-series row of the first step
    const float *acc;  // nsteps rows of nt accelerations, or null
    // batched runs: steps of time pair0, pair0 + 2, ... start a two-step pass over the face pairs
    // when their partner (the next time) is at most pair_end; pair_end < pair0: one pass per step
    int pair0 = 0, pair_end = -1;
    int conv_pairs = 0, terms_pairs = 0;  // which stages use the pairing (the handle's options)
    // listener series (R elements, row0 is its row of the first step), or null: read from here
    // rather than recorded into the graphs, so a series that grows keeps the recorded graphs valid
    void *series = nullptr;
};

// what step k of a call produces: its time index, listener-series row and acceleration row
struct StepDyn
{
    int tnew;
    long long row;
    const float *acc;
    void *series;
};

__device__ inline StepDyn bind_step(const StepState *st, int k, int nt)
{
    StepDyn d;
    d.tnew = st->tnew0 + k;
    d.row = st->row0 + k;
    d.acc = st->acc ? st->acc + (long long)k * nt : nullptr;
    d.series = st->series;
    return d;
}

// a recorded pppm_step call
struct StepGraph
{
    int nsteps = 0;
    bool open = false;               // a chunk of a longer call (more steps follow; see run_steps)
    std::vector<unsigned char> sig;  // the launch set it was recorded with
    cudaGraphExec_t exec = nullptr;
};
constexpr int kStepGraphs = 8;

struct Handle
{
    pppm_params prm{};
    bool fp64 = false;
    size_t real_size = 4;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t side = nullptr;                         // second branch of the recorded step graphs
    cudaStream_t side2 = nullptr;                        // third branch: the bulk of the split stencil
    cudaEvent_t ev_fin = nullptr, ev_conv = nullptr;     // fork / join points while recording
    cudaEvent_t ev_near = nullptr, ev_bulk = nullptr;
    cudaEvent_t ev_upd_fork = nullptr, ev_upd_join = nullptr;  // the grid-cache branch of a mesh update
    bool gc_launched = false;  // this update's grid-cache refresh runs on side2 (grid_cache_start)
    int res = 0;
    long long n_cells = 0;
    int t = -1;
    long long launches = 0;
    TdbemConsts tc{};

    void *grid[3] = {nullptr, nullptr, nullptr};  // ring slots, index (t + 3) % 3
    void *pml[3] = {nullptr, nullptr, nullptr};

    // ---- mesh
    bool mesh_set = false;
    int nv = 0, nt = 0;
    float *d_verts = nullptr;  // 3 nv
    int *d_tris = nullptr;     // 3 nt
    float *d_center = nullptr, *d_normal = nullptr, *d_area = nullptr;  // 3nt, 3nt, nt
    int *d_cellc = nullptr, *d_basec = nullptr;  // 3nt each: grid coord, base coord
    int *d_cell = nullptr, *d_base = nullptr;    // linear, -1 when outside the grid
    int *d_cell_count = nullptr, *d_cell_start = nullptr, *d_cell_tris = nullptr;
    int *d_base_count = nullptr, *d_base_start = nullptr, *d_base_tris = nullptr;
    int *d_cursor = nullptr;     // scratch res^3
    int *d_scan_tmp = nullptr;   // scan scratch
    size_t scan_tmp_elems = 0;
    int *d_flags = nullptr;      // res^3 scratch
    int *d_pair_work = nullptr;  // face-pair recompute scan + list, 2 (pf + 1) ints, grown
    long long pair_work_cap = 0;

    // ---- corrected cells and 3^3 pairs
    int n3 = 0;
    long long p3 = 0;
    int *d_n3_cell = nullptr, *d_n3_start = nullptr;
    int *d_p3_tri = nullptr;
    unsigned char *d_p3_woff = nullptr;
    long long p3_cap = 0;
    unsigned *d_corr_mask = nullptr;

    // ---- base cells and 4^3 lists
    int b4 = 0;
    long long p4 = 0;  // sum over base cells of 4^3 list lengths
    int *d_b4_cell = nullptr, *d_b4_start = nullptr, *d_n4_tris = nullptr;
    long long n4_cap = 0;

    // ---- face pairs (per centre triangle)
    long long pf = 0;
    int *d_face_start = nullptr, *d_face_nbr = nullptr, *d_face_pool = nullptr;
    void *d_face_w = nullptr;
    float2 *d_face_scale = nullptr;
    void *d_face_d1 = nullptr;  // pf: double-layer tap 1 of each pair, scale applied (step.cu: fix_kernel)
    long long pf_cap = 0;
    int *d_face_corner = nullptr;
    float *d_face_interp = nullptr;
    double *d_face_interp_d = nullptr;
    double *d_face_denom = nullptr;

    // ---- persistent caches
    bool gc_empty = true;
    void *d_gc_w = nullptr;        // FP32: __half2[nt][54][16]; FP64: double[nt][54][32]
    float2 *d_gc_scale = nullptr;  // FP32: [nt][54]
    void *d_gc_f = nullptr;        // [nt][54] factor of the new Dirichlet value per record (gc_factors)
    float *d_gc_snap = nullptr;    // nt x 7 centre, normal, area at last refresh
    int *d_gc_flag = nullptr;      // nt recompute flags
    int *d_fc_keys = nullptr;      // nt x kFaceCacheSlots neighbour ids, -1 = empty
    int *d_fc_slot = nullptr;      // nt x kFaceCacheSlots pool slots
    void *d_pool_w = nullptr;      // pool records (layout as face_w)
    float2 *d_pool_scale = nullptr;
    float2 *d_pool_meta = nullptr;  // (normal angle, distance) at last refresh
    int *d_pool_count = nullptr;    // device counter
    int2 *d_pool_key = nullptr;     // (centre, neighbour) of each pool slot
    long long pool_cap = 0;
    long long pool_used = 0;
    // motion checkpoints (cache.cu): rewrites of pool slots below the newest checkpoint's pool
    // size are logged with their old records, so a rewind undoes them
    float2 *d_pair_old_meta = nullptr;  // pf scratch: a rewritten pair's meta before the refresh
    long long pair_old_meta_cap = 0;
    int *d_log_count = nullptr;         // [0] rewrites to log (lookup), [1] log cursor
    struct Journal *journal = nullptr;
    int *d_pair_flag = nullptr;  // pf scratch: 1 = recompute
    int *d_status = nullptr;     // device-side status word (capacity / timeout)
    int *d_step_status = nullptr;  // step status word: non-finite values seen by the step kernels
    int *h_step_status = nullptr;  // pinned copy, written behind each pppm_step call
    cudaEvent_t ev_status = nullptr;  // recorded after that copy
    bool status_pending = false;   // a copy is queued and not yet looked at
    bool nonfinite = false;        // a non-finite value was seen (until the fields are reset)
    void *d_spec = nullptr;      // recompute scratch spectra
    size_t spec_bytes = 0;
    double *d_tw = nullptr;      // 8 radix-2 FFT twiddles (cos, sin)

    // ---- histories
    void *d_neumann = nullptr, *d_dirichlet = nullptr;  // reference layout: read-out and loading
    void *d_hist = nullptr;  // the step's copies: [4 copies][nt][kHistRow], both fields (step.cu)
    void *d_terms = nullptr;  // nt x 54 near-field terms of the current step (step.cu: near_terms)
    void *d_conv = nullptr;   // nt face-pair convolution sums of the pipelined step (step.cu)
    void *d_conv1 = nullptr;  // nt partial sums of the following step (step.cu: conv2_kernel)
    void *d_dlast = nullptr;  // nt Dirichlet values of the last finished step (step.cu: fix_kernel)
    void *d_terms1 = nullptr; // nt x 54 partial near-field terms of the following step (near_terms2)
    int conv_pairs = 1;       // recorded step graphs convolve the face pairs two steps per pass
    int face_threads = 256;   // threads per block of their face-stage kernels (step_autotune)
    bool terms_pairs = true;  // ... and the grid-cache near-field terms two steps per pass
    bool split_stencil = true;  // ... and the stencil split into corrected cells and the bulk
    bool corr_near_boundary = false;  // a corrected cell may neighbour the boundary layer (mesh_build)
    int stencil_vec4 = -1;      // interior stencil four cells per thread: 1 on, 0 off, -1 by grid size
    int graph_chunk = 32;       // steps per chunk graph of a long pppm_step call (0: one graph per call)

    // ---- listeners
    std::vector<int> listen_xyz;
    int *d_listen_cell = nullptr, *d_listen_n3 = nullptr;
    void *d_series = nullptr;
    long long series_cap = 0;  // steps
    long long series_count = 0;

    // ---- cell labels
    int *d_cell_type = nullptr, *d_cell_nearest = nullptr, *d_cell_ghost = nullptr;
    float *d_cell_points = nullptr;  // res^3 x 7
    int *d_cell_type_old = nullptr;
    int ghost_count = 0;

    // ---- timing
    bool timing = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    float us_stencil = 0, us_face = 0, us_near = 0;  // summed over timed_steps
    long long timed_steps = 0;
    // per kernel kind (PPPM_KERNEL_*): event time and launches summed in measurement mode
    double kind_us[PPPM_KERNEL_KINDS] = {};
    long long kind_n[PPPM_KERNEL_KINDS] = {};
    static constexpr int kProfileSteps = 4;
    // Neumann write, empty kernel, up to 5 kernels per step (convolution, bulk and corrected-cell
    // stencil, finish, near), end
    static constexpr int kProfileEvents = 3 + 5 * kProfileSteps;
    cudaEvent_t evk[kProfileEvents] = {};
    int evk_kind[kProfileEvents] = {};
    int evk_used = 0;  // event marks of the recorded profile graph
    StepGraph profile_graph;  // kProfileSteps split-stage steps with events between the kernels

    // ---- step launches
    StepState *d_state = nullptr;  // per-call values the step kernels read
    StepGraph graphs[kStepGraphs];
    StepGraph timing_graph;  // one step with event records between its kernels (measurement mode)
    int graph_next = 0;
    int near_blocks = 0;  // resident grid of the near kernel
    int batch_near_cells = 0;  // corrected cells the batch block map covers (grow-only, step.cu)

    // ---- ghost-cell method (ghost.cu)
    struct Ghost *ghost = nullptr;
    float *d_gneu = nullptr, *d_gneu_old = nullptr;  // this and the previous step's accelerations

    // ---- adjoint (adjoint.cu): transposed tables and adjoint state, built on first use
    long long mesh_version = 0;  // bumped whenever the lists or weight tables change
    bool tables_stale = false;   // a cache state was restored: no step until update_mesh
    struct Adjoint *adj = nullptr;

    // ---- pinned host words for batched reads of device counts (read_ints)
    int *h_pin = nullptr;

    // ---- scratch for accelerations
    float *d_acc = nullptr;
    long long acc_cap = 0;

    void *slot(int time) const { return grid[((time % 3) + 3) % 3]; }
    void *pml_slot(int time) const { return pml[((time % 3) + 3) % 3]; }
};

// ---------------------------------------------------------------- internal API -------
int dev_alloc(void **p, size_t bytes);
void dev_free(void *p);
template <typename T>
int dalloc(T **p, size_t count)
{
    return dev_alloc((void **)p, count * sizeof(T));
}
template <typename T>
int dgrow(T **p, long long &cap, long long need, cudaStream_t s)
{
    if (need <= cap)
        return PPPM_OK;
    long long nc = need + need / 2 + 64;
    dev_free(*p);
    *p = nullptr;
    int rc = dev_alloc((void **)p, (size_t)nc * sizeof(T));
    if (rc)
        return rc;
    cap = nc;
    (void)s;
    return PPPM_OK;
}

// mesh.cu
int mesh_build(Handle &h);                      // geometry + all lists from d_verts/d_tris
int exclusive_scan(Handle &h, const int *in, int *out, long long n);  // out[n] = total
// up to 4 independent exclusive scans in one set of launches
int exclusive_scan_set(Handle &h, const int *const *in, int *const *out, const long long *n, int count);
int read_int(Handle &h, const int *d, int *out);
constexpr int kPinnedInts = 16;
int read_ints(Handle &h, const int *const *src, int n, int *out);  // n device words, one synchronisation

// adjoint.cu
struct Adjoint;
int adjoint_run(Handle &h, const void *g, int nsteps, void *out, int fresh);  // device buffers
int adjoint_stage(Handle &h, size_t g_bytes, size_t out_bytes, void **g, void **out);
void adjoint_free(Handle &h);

// ghost.cu
struct Ghost;
int ghost_build(Handle &h);  // ghost list, interpolation weights, sparse rows, SOLID list
int ghost_read(Handle &h, int what, void *dst, size_t bytes);
void ghost_free(Handle &h);

// cache.cu
int cache_refresh(Handle &h);  // grid cache + face cache refresh, dense gathers, denominators
int grid_cache_start(Handle &h);  // the grid-cache refresh on side2, joined by cache_refresh
void join_grid_cache(Handle &h);  // the handle's stream waits for that branch (error paths)
int cache_free(Handle &h);
size_t cache_state_bytes(Handle &h);                               // pppm_cache_state_size
int cache_state_save(Handle &h, void *dst, size_t bytes);          // host or device buffer
int cache_state_restore(Handle &h, const void *src, size_t bytes);  // host or device buffer; tables stale
int journal_push(Handle &h, int *id);    // pppm_checkpoint_push
int journal_rewind(Handle &h, int id);   // pppm_checkpoint_rewind; tables stale
void journal_clear(Handle &h, bool release);  // pppm_checkpoint_clear (release: free the arena too)
size_t journal_bytes(const Handle &h);   // device bytes the checkpoints' arena and logs hold
int journal_count(const Handle &h);
int cache_regather(Handle &h);  // dense gathers + denominators from the persistent caches
int cache_import_grid(Handle &h, const void *records);                         // nt x 54 x 72 B
int cache_import_face(Handle &h, const int *pairs, const void *records, int n);  // n x 72 B

// step.cu
int step_prime(Handle &h);
int step_autotune(Handle &h, int reps, float *us, int *best);
int step_time_kernels(Handle &h, int reps, float *us);  // us: PPPM_KERNEL_KINDS entries
int gc_factors(Handle &h, cudaStream_t gs);
int step_run(Handle &h, const float *acc_dev, int nsteps);
int step_free(Handle &h);  // recorded graphs and the step state
// batched scenes (step.cu): one set of stage launches advances every scene
struct Batch;
int batch_create(Handle **hs, int n, Batch **out);
int batch_run(Batch *b, const float *const *dacc, const int *nsteps);  // dacc: device rows per scene
void batch_destroy(Batch *b);
int hist_import(Handle &h);  // reference-layout rings -> the step's history copies (the rings are
                             // kept current by every history write)

// cells.cu
int cells_classify(Handle &h, int *ghost_count);
int cells_fresh(Handle &h, const float *acc, const float *acc_old, int *fresh_count);  // host arrays
int cells_fresh_dev(Handle &h, const float *acc, const float *acc_old, int *fresh_count);  // device arrays

}  // namespace pb
