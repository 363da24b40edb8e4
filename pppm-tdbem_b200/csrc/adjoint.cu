// Adjoint of the PPPM time step (no counterpart in the reference).
//
// With the geometry, the cell labels and so every weight table held fixed, one step is a
// linear map of (grid slots, history rings, the step's accelerations), so the listener
// samples of a run are linear in the accelerations: series = A acc + B state0.  The gradient
// of L = sum_s sum_l g[s][l] series[s][l] with respect to acc is A^T g whatever the forward
// trajectory was.  The adjoint therefore runs the transposed step backwards in time on adjoint
// state of the forward state's size (three grid slots, 32-slot rings): it stores no forward
// states and recomputes no stretch of the run, and a long run can be differentiated in chunks
// (a call continues the adjoint state the previous call left, latest chunk first).
//
// The forward step at time t (step.cu), written as linear maps (a_k = -single-layer weight x
// scale, b_k = double-layer weight x scale of tap k; the FDTD-near row is stored shifted):
//   S  stencil   q = L(p^{t-1}, p^{t-2}) on [1, res-2]^3: interior leapfrog, and on the
//                boundary layer a 4x4 solve that also writes the ghosts of p^{t-1} and reads the
//                ghosts of p^{t-2}; p^t = q - C^t at corrected cells; N[t] = acc[t]
//   F  face      D[j][t] = (reflect sum_k iw_jk p^t[corner_jk] + sum_{pairs (j, i)} sum_k
//                a_k N[i][t-k] + b_k D[i][t-k] (k >= 1)) / denom_j
//   M  near      C^{t+1}[c] = sum_{pairs (c, tr)} sum_k af_k N[tr][t-k] + bf_k D[tr][t-k];
//                p^t[c] += 0.98 sum_{pairs (c, tr)} sum_k ab_k N[tr][t-k] + bb_k D[tr][t-k]
//   listeners read p^t after M.
//
// Adjoint variables: Lambda(tau) per grid slot (tau mod 3, ghosts included) and, per triangle,
// two accumulation rings over time (32 slots): accN[j][tau] and accD[j][tau] collect the adjoints
// of N[j][tau] and D[j][tau] from every later operation that read them.  Each reverse step pushes
// its operations' adjoints into those rings with the tables of its own step only, and nothing is
// kept per corrected cell from one step to the next, so the tables (lists, weights, corrected
// cells, corners) may change between steps: a moving run is differentiated frame by frame with
// each frame's tables loaded.  The reverse step at sigma runs seven kernels:
//   P1 listeners  Lambda(sigma)[listener cell] += dL/dseries[sigma]
//   P2 near BEM   per triangle j, over its near pairs (c, j): the BEM-near record (taps k) times
//                 0.98 Lambda(sigma)[c] into accN/accD[j][sigma - k]; then D[j][sigma] has all its
//                 readers: lamF[j] = accD[j][sigma] / denom_j (the adjoint of the face numerator)
//   P3 faces      per triangle j, over the centres i whose face list holds j: the face record
//                 (a_m, b_{m+1}) times lamF[i] into accN[j][sigma - m], accD[j][sigma - 1 - m];
//                 then N[j][sigma] has all its readers: dL/dacc[sigma][j] = accN[j][sigma]
//   P4 corners    Lambda(sigma)[cell] += reflect iw lamF[j] over the cells that are trilinear
//                 corners of some face
//   P5 near C     per triangle j, over its near pairs: the stored FDTD-near sum C^sigma (subtracted
//                 by the stencil at step sigma, computed from the histories of sigma - 1 with the
//                 tables of step sigma) gets -Lambda(sigma)[c]; its record (taps shifted by one)
//                 times that into accN/accD[j][sigma - 1 - k]
//   P6 boundary   per boundary-layer cell: lam_b = A^-T (adjoints of its ghost outputs, of
//                 its own output); the ghost adjoints of Lambda(sigma - 1) are consumed
//   P7 cells      transposed stencil as a gather over the 7 cells that read a cell:
//                 Lambda(sigma - 1) += S_cur^T; Lambda(sigma - 2) = S_prev^T (the first
//                 contribution to that slot's new time, so it overwrites the stale one)
// The gathers (P2, P3, P4, P5, P7) need no atomics: every sum belongs to one thread or warp.
#include <algorithm>
#include <vector>
#include "fdtd.cuh"
#include "handle.cuh"

namespace pb
{

struct Adjoint
{
    long long version = -1;  // Handle::mesh_version the tables were built for
    int nt = 0, n3 = 0, ncorner = 0;
    long long pfT = 0, p3T = 0;
    // transposed tables
    int *fT_start = nullptr, *fT_src = nullptr;  // per triangle j: the centres i whose face list holds j
    void *fT_w = nullptr;                         // [pfT][16] (a_m, b_{m+1}) weight pairs
    float2 *fT_scale = nullptr;                   // [pfT] (single, double) scales (FP32 weights)
    int *nT_start = nullptr, *nT_cell = nullptr, *nT_pair = nullptr;  // per triangle: (corrected index, pair)
    void *nT_w = nullptr;        // [p3T][2][16]: the pair's FDTD-near (shifted) and BEM-near records
    float2 *nT_scale = nullptr;  // [p3T][2] (FP32 weights)
    int *cT_cell = nullptr, *cT_start = nullptr, *cT_ref = nullptr;    // corner cells: (tri * 8 + k)
    // the transposes' scratch; every table array grows only (a moving sweep rebuilds the tables
    // every motion frame), with its capacity in cap[] (elements; bytes for the weights)
    int *d_count = nullptr, *d_cursor = nullptr;  // per key
    int *d_order = nullptr, *d_owner = nullptr;   // per value
    int *d_flag = nullptr;                        // res^3 + 1 corner-cell flags, then their scan
    long long cap[17] = {};
    // adjoint state
    void *lam[3] = {nullptr, nullptr, nullptr};
    void *lam_b = nullptr;  // 4 x res^3 (boundary layer only)
    void *psi[2] = {nullptr, nullptr};  // PML: 6 x res^3 each, adjoints of the auxiliary fields
    void *acc_n = nullptr, *acc_d = nullptr;  // [nt][kRing] accumulation rings (slot = tau mod 32)
    void *lam_f = nullptr;                    // [nt] adjoint of the face numerator at the current step
    int pos = 0;               // one past the next time the reverse sweep processes
    bool started = false;
    // host-call staging
    void *d_g = nullptr, *d_out = nullptr;
    long long g_cap = 0, out_cap = 0;
    // the call's reverse-step state on the device, and a recorded chunk of reverse steps with the
    // launch arguments it was recorded for
    void *d_step = nullptr;
    cudaGraphExec_t chunk = nullptr;
    std::vector<unsigned char> chunk_sig;
};

namespace
{

constexpr int kAdjTop = 1 << 29;  // time index where a fresh reverse sweep starts (any positive value)

template <typename T, int N>
struct alignas(16) AVec
{
    T v[N];
};

template <typename R>
struct AdjWRec;
template <>
struct AdjWRec<float>
{
    using T = __half2;
    using W4 = AVec<__half2, 4>;
    using H4 = AVec<float, 4>;
};
template <>
struct AdjWRec<double>
{
    using T = double2;
    using W4 = AVec<double2, 4>;
    using H4 = AVec<double, 4>;
};

// a_k and b_k of a weight record entry: the factors that multiply the Neumann and the
// Dirichlet history in the forward convolution
__device__ inline float wa(__half2 w, float2 s) { return -__low2float(w) * s.x; }
__device__ inline float wb(__half2 w, float2 s) { return __high2float(w) * s.y; }
__device__ inline double wa(double2 w, float2) { return -w.x; }
__device__ inline double wb(double2 w, float2) { return w.y; }

template <typename R>
struct AdjArgs
{
    using W = typename AdjWRec<R>::T;
    int res, nt, n3, nl, ncorner;
    long long ncells;
    int listen_cell[8];
    const int *n3_cell;
    const unsigned *corr_mask;  // corrected-cell bits
    const int *fT_start, *fT_src;
    const W *fT_w;
    const float2 *fT_scale;
    const int *nT_start, *nT_cell, *nT_pair;
    const W *nT_w;
    const float2 *nT_scale;
    const int *cT_cell, *cT_start, *cT_ref;
    const float *interp;
    const double *interp_d, *denom;
    float reflect;
    R *lam[3];
    R *lam_b;
    R *acc_n, *acc_d, *lam_f;
    double kappa;                 // (c dt / h)^2: interior leapfrog coefficient
    R coef, coef1, coef2, coef3;  // boundary solve coefficients (fdtd.cu:88-137)
    // the PML (pml_width > 0): adjoints of the six auxiliary fields per cell at two times
    // (slot = time mod 2) and the update's coefficients (fdtd.cu:179-232)
    R *psi[2];
    int pml_w;
    double pml_damp;                      // 2 / h inside the layer
    double pml_k, pml_ih2, pml_ih;        // (c dt)^2, 1 / h^2, 1 / h
    double pml_cdt, pml_i2h;              // c dt, 1 / (2 h)
    __device__ R *slot(int tau) const { return lam[((tau % 3) + 3) % 3]; }
};

// The reverse step a kernel launch covers: reverse step j of a pppm_adjoint call processes time
// sigma = top - 1 - j; its dL/dsignal row is g + (sigma - bottom) * nl and its dL/dacc row
// out + (sigma - bottom) * nt.  Read from device memory, so a recorded chunk of reverse steps
// replays for any stretch of a sweep (advance_adj_kernel moves top on after each chunk).
struct AdjStep
{
    int top, bottom;
    const void *g;
    void *out;
};

__device__ inline int adj_sigma(const AdjStep *st, int j) { return st->top - 1 - j; }

// P1: the listener samples' adjoints
template <typename R>
__global__ void adj_listen_kernel(const __grid_constant__ AdjArgs<R> a, const AdjStep *st, int jstep)
{
    if (threadIdx.x != 0)
        return;
    const int sigma = adj_sigma(st, jstep);
    const R *g = (const R *)st->g + (long long)(sigma - st->bottom) * a.nl;
    for (int l = 0; l < a.nl; l++)  // one thread: listeners may share a cell
        a.slot(sigma)[a.listen_cell[l]] += g[l];
}

template <typename R>
__device__ inline R warp_sum_adj(R v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// sums of the eight quads of a warp per lane position (lanes l, l ^ 4, ..., l ^ 28): lane q < 4 of
// quad 0 ends with the totals of taps 4q .. 4q + 3
template <typename R>
__device__ inline void quad_totals(R (&v)[4])
{
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int off = 4; off < 32; off <<= 1)
            v[i] += __shfl_xor_sync(0xffffffffu, v[i], off);
}

// the 16 taps of a near record (half = 0: FDTD-near, shifted by one tap; 1: BEM-near) of near pair p
// times v[pair], accumulated per lane over the pairs of triangle j (quad g takes pairs g, g + 8, ...;
// lane q taps 4q .. 4q + 3); cell_value(c) gives the factor of corrected cell c
template <typename R, typename F>
__device__ inline void near_push_sums(const AdjArgs<R> &a, int j, int half, int g, int q, F cell_value, R (&an)[4],
                                      R (&ad)[4])
{
    using W4 = typename AdjWRec<R>::W4;
#pragma unroll
    for (int i = 0; i < 4; i++)
        an[i] = ad[i] = 0;
    for (int p = a.nT_start[j] + g; p < a.nT_start[j + 1]; p += 8)
    {
        const R v = cell_value(a.n3_cell[a.nT_cell[p]]);
        const W4 w = *(const W4 *)(a.nT_w + ((long long)p * 2 + half) * kTaps + 4 * q);
        const float2 sc = a.nT_scale ? a.nT_scale[2 * p + half] : make_float2(1, 1);
#pragma unroll
        for (int i = 0; i < 4; i++)
        {
            an[i] += (R)wa(w.v[i], sc) * v;
            ad[i] += (R)wb(w.v[i], sc) * v;
        }
    }
    quad_totals<R>(an);
    quad_totals<R>(ad);
}

// add tap k of lane q's totals into ring slot (tau0 - k) of triangle j (lanes 0-3)
template <typename R>
__device__ inline void ring_add(R *ring, int j, int tau0, int q, const R (&v)[4])
{
    R *row = ring + (long long)j * kRing;
#pragma unroll
    for (int i = 0; i < 4; i++)
        row[(tau0 - 4 * q - i) & (kRing - 1)] += v[i];
}

// P2: near BEM push, then lamF of triangle j (one warp per triangle)
template <typename R>
__global__ void __launch_bounds__(256) adj_bem_kernel(const __grid_constant__ AdjArgs<R> a, const AdjStep *st,
                                                      int jstep)
{
    const int sigma = adj_sigma(st, jstep);
    const int j = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (j >= a.nt)
        return;
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const R *lam = a.slot(sigma);
    R an[4], ad[4];
    near_push_sums<R>(a, j, 1, g, q, [&](int c) { return (R)0.98 * lam[c]; }, an, ad);
    if (lane < 4)
    {
        ring_add<R>(a.acc_n, j, sigma, q, an);
        ring_add<R>(a.acc_d, j, sigma, q, ad);
    }
    __syncwarp();
    if (lane == 0)
    {
        R *slot = a.acc_d + (long long)j * kRing + (sigma & (kRing - 1));
        a.lam_f[j] = (R)(*slot / a.denom[j]);
        *slot = 0;  // the slot is reused for time sigma - 32
    }
}

// P3: face push (one warp per triangle j over the centres i whose face list holds j), then
// dL/dacc[sigma][j]
template <typename R>
__global__ void __launch_bounds__(256) adj_face_kernel(const __grid_constant__ AdjArgs<R> a, const AdjStep *st,
                                                       int jstep)
{
    const int sigma = adj_sigma(st, jstep);
    R *out_row = st->out ? (R *)st->out + (long long)(sigma - st->bottom) * a.nt : nullptr;
    using W4 = typename AdjWRec<R>::W4;
    const int j = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (j >= a.nt)
        return;
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    R an[4] = {0, 0, 0, 0}, ad[4] = {0, 0, 0, 0};
    for (int p = a.fT_start[j] + g; p < a.fT_start[j + 1]; p += 8)
    {
        const R lf = a.lam_f[a.fT_src[p]];
        const W4 w = *(const W4 *)(a.fT_w + (long long)p * kTaps + 4 * q);  // (a_m, b_{m+1})
        const float2 sc = a.fT_scale ? a.fT_scale[p] : make_float2(1, 1);
#pragma unroll
        for (int i = 0; i < 4; i++)
        {
            an[i] += (R)wa(w.v[i], sc) * lf;
            ad[i] += (R)wb(w.v[i], sc) * lf;
        }
    }
    quad_totals<R>(an);
    quad_totals<R>(ad);
    if (lane < 4)
    {
        ring_add<R>(a.acc_n, j, sigma, q, an);
        ring_add<R>(a.acc_d, j, sigma - 1, q, ad);
    }
    __syncwarp();
    if (lane == 0)
    {
        R *slot = a.acc_n + (long long)j * kRing + (sigma & (kRing - 1));
        if (out_row)
            out_row[j] = *slot;
        *slot = 0;
    }
}

// P5: the stored FDTD-near sums of step sigma (one warp per triangle)
template <typename R>
__global__ void __launch_bounds__(256) adj_fdtd_near_kernel(const __grid_constant__ AdjArgs<R> a, const AdjStep *st,
                                                            int jstep)
{
    const int sigma = adj_sigma(st, jstep);
    const int j = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (j >= a.nt)
        return;
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const R *lam = a.slot(sigma);
    R an[4], ad[4];
    near_push_sums<R>(a, j, 0, g, q, [&](int c) { return -lam[c]; }, an, ad);
    if (lane < 4)
    {
        ring_add<R>(a.acc_n, j, sigma - 1, q, an);
        ring_add<R>(a.acc_d, j, sigma - 1, q, ad);
    }
}

// P4: corner cells of the face interpolation
template <typename R>
__global__ void __launch_bounds__(256) adj_corner_kernel(const __grid_constant__ AdjArgs<R> a, const AdjStep *st,
                                                         int jstep)
{
    const int sigma = adj_sigma(st, jstep);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.ncorner)
        return;
    R v = 0;
    for (int r = a.cT_start[i]; r < a.cT_start[i + 1]; r++)
    {
        const int ref = a.cT_ref[r];
        const R iw = a.interp_d ? (R)a.interp_d[ref] : (R)a.interp[ref];
        v += iw * a.lam_f[ref >> 3];
    }
    a.slot(sigma)[a.cT_cell[i]] += (R)a.reflect * v;
}

__device__ inline int judge_of(int v, int res) { return -((int)(v == 1)) + ((int)(v == res - 2)); }

// P6: the boundary-layer solve transposed
template <typename R>
__global__ void __launch_bounds__(256) adj_boundary_kernel(const __grid_constant__ AdjArgs<R> a, const AdjStep *st,
                                                           int jstep)
{
    const int sigma = adj_sigma(st, jstep);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int res = a.res;
    if (i >= boundary_cells(res))
        return;
    int cc[3];
    boundary_cell(i, res, cc[0], cc[1], cc[2]);
    int judge[3];
#pragma unroll
    for (int d = 0; d < 3; d++)
        judge[d] = judge_of(cc[d], res);
    auto idx = [&](int x, int y, int z) { return ((long long)x * res + y) * res + z; };
    const long long ci = idx(cc[0], cc[1], cc[2]);
    R *cur = a.slot(sigma), *ghosts = a.slot(sigma - 1);
    long long gi[3] = {-1, -1, -1};
    R lo[4];
#pragma unroll
    for (int d = 0; d < 3; d++)
    {
        lo[d] = 0;
        if (judge[d] != 0)
        {
            int q[3] = {cc[0], cc[1], cc[2]};
            q[d] += judge[d];
            gi[d] = idx(q[0], q[1], q[2]);
            lo[d] = ghosts[gi[d]];
        }
    }
    lo[3] = cur[ci];
    // the forward matrix (same entries as the forward solve), transposed
    R m[4][4];
    m[3][3] = 1;
#pragma unroll
    for (int d = 0; d < 3; d++)
        m[3][d] = -a.coef * (judge[d] != 0);
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        const int ax = r, ay = (r + 1) % 3, az = (r + 2) % 3;
        m[r][3] = a.coef1;
        m[r][ax] = a.coef2;
        m[r][ay] = a.coef3 * (judge[ay] != 0);
        m[r][az] = a.coef3 * (judge[az] != 0);
    }
    R mt[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++)
            mt[r][c] = m[c][r];
    R lb[4];
    solve4<R>(mt, lo, lb);
#pragma unroll
    for (int k = 0; k < 4; k++)
        a.lam_b[k * a.ncells + ci] = lb[k];
#pragma unroll
    for (int d = 0; d < 3; d++)
        if (gi[d] >= 0)
            ghosts[gi[d]] = 0;
}

// P7: the transposed stencil, one thread per cell of the whole grid (ghost layer included)
template <typename R>
__global__ void __launch_bounds__(256) adj_stencil_kernel(const __grid_constant__ AdjArgs<R> a, const AdjStep *st,
                                                          int jstep)
{
    const int sigma = adj_sigma(st, jstep);
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.ncells)
        return;
    const int res = a.res;
    const int y[3] = {(int)(i / ((long long)res * res)), (int)((i / res) % res), (int)(i % res)};
    const R *lq = a.slot(sigma);
    const R *lb = a.lam_b;
    const long long nc = a.ncells;
    auto inside = [&](int x0, int x1, int x2) {
        return x0 >= 1 && x0 <= res - 2 && x1 >= 1 && x1 <= res - 2 && x2 >= 1 && x2 <= res - 2;
    };
    auto interior = [&](int x0, int x1, int x2) {
        return x0 >= 2 && x0 <= res - 3 && x1 >= 2 && x1 <= res - 3 && x2 >= 2 && x2 <= res - 3;
    };
    const double kappa = a.kappa;
    const double coef = a.coef, coef1 = a.coef1, coef2 = a.coef2, coef3 = a.coef3;
    double cur = 0, prev = 0;
    if (interior(y[0], y[1], y[2]))
    {
        const double l = lq[i];
        cur += (2 - 6 * kappa) * l;
        prev -= l;
    }
    else if (inside(y[0], y[1], y[2]))
    {
        const double b0 = lb[i], b1 = lb[nc + i], b2 = lb[2 * nc + i], b3 = lb[3 * nc + i];
        cur += b3 * (2 - 6 * coef) + (b0 + b1 + b2) * (2 * coef1 + 4 * coef3);
        prev += -b3 - coef1 * (b0 + b1 + b2);
    }
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
        for (int s = -1; s <= 1; s += 2)
        {
            int x[3] = {y[0], y[1], y[2]};
            x[d] += s;  // the reading cell; y = x - s e_d
            if (!inside(x[0], x[1], x[2]))
                continue;
            const long long xi = ((long long)x[0] * res + x[1]) * res + x[2];
            if (interior(x[0], x[1], x[2]))
            {
                cur += kappa * (double)lq[xi];
                continue;
            }
            const int jd = judge_of(x[d], res);
            const double bd = lb[(long long)d * nc + xi], b3 = lb[3 * nc + xi];
            const double bo = (double)lb[(long long)((d + 1) % 3) * nc + xi] + (double)lb[(long long)((d + 2) % 3) * nc + xi];
            if (s < 0)
            {
                // y = x + e_d
                cur += coef * (jd <= 0) * b3 + coef2 * (jd < 0) * bd - coef3 * (jd <= 0) * bo;
                prev += coef2 * jd * bd;
            }
            else
            {
                // y = x - e_d
                cur += coef * (jd >= 0) * b3 + coef2 * (jd > 0) * bd - coef3 * (jd >= 0) * bo;
                prev -= coef2 * jd * bd;
            }
        }
    R *lc = a.slot(sigma - 1), *lp = a.slot(sigma - 2);
    lc[i] = (R)((double)lc[i] + cur);
    lp[i] = (R)prev;
}


// P7 with the PML (pml_width > 0; no boundary solve, P6 does not run): the split-field update
// (fdtd.cu:179-232) transposed, one thread per cell of the whole grid.  Forward at a cell q of
// [1, res-2]^3, with K = (c dt)^2, sd = +1 above the grid's middle plane along d and -1 below,
// ps = q + sd e_d, ms = q - sd e_d, w(x) the damping at cell x (2/h inside the layer, else 0):
//   p^t[q] = 2 p^{t-1}[q] - p^{t-2}[q] + K sum_d [(p^{t-1}[q+e_d] - 2 p^{t-1}[q] + p^{t-1}[q-e_d]) / h^2
//            + (w(q) psi^{t-1}[ps]_{3+d} - w(ms) psi^{t-1}[ms]_d) / h]
// and, where w(q) != 0 (elsewhere the fields stay zero),
//   psi^t[q]_d     = psi^{t-1}[q]_d + c dt (-(w(ms) psi^{t-1}[ms]_d + w(q) psi^{t-1}[q]_d) / 2 - g_d)
//   psi^t[q]_{3+d} = psi^{t-1}[q]_{3+d} + c dt (-(w(ms) psi^{t-1}[q]_{3+d} + w(q) psi^{t-1}[ps]_{3+d}) / 2 - g_d)
// with g_d = (p^{t-1}[ps] - p^{t-1}[ms]) / (2 h).  The ghost layer holds zeros that nothing
// writes, so only cells of [1, res-2]^3 carry adjoints.  A cell j is read by itself and by its six
// neighbours q = j + s e_d; for such a q, j is ps of q when sd(q) = -s and ms of q when sd(q) = s.
__device__ inline bool in_pml(int x, int y, int z, int res, int w)
{
    return x < w || x >= res - w || y < w || y >= res - w || z < w || z >= res - w;
}

template <typename R>
__global__ void __launch_bounds__(256) adj_pml_kernel(const __grid_constant__ AdjArgs<R> a, const AdjStep *st,
                                                      int jstep)
{
    const int sigma = adj_sigma(st, jstep);
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.ncells)
        return;
    const int res = a.res, w = a.pml_w;
    const int y[3] = {(int)(i / ((long long)res * res)), (int)((i / res) % res), (int)(i % res)};
    const R *ln = a.slot(sigma);             // adjoint of p^sigma (the stencil's output)
    const R *pn = a.psi[sigma & 1];          // adjoint of psi^sigma
    R *lc = a.slot(sigma - 1), *lp = a.slot(sigma - 2);
    R *pc = a.psi[(sigma - 1) & 1];          // adjoint of psi^{sigma-1}, written here
    auto inside = [&](const int *x) {
        return x[0] >= 1 && x[0] <= res - 2 && x[1] >= 1 && x[1] <= res - 2 && x[2] >= 1 && x[2] <= res - 2;
    };
    auto damp = [&](const int *x) { return in_pml(x[0], x[1], x[2], res, w) ? a.pml_damp : 0.0; };
    if (!inside(y))
    {
        lp[i] = 0;
#pragma unroll
        for (int k = 0; k < 6; k++)
            pc[6 * i + k] = 0;
        return;
    }
    const double K = a.pml_k, ih2 = a.pml_ih2, ih = a.pml_ih, cdt = a.pml_cdt, i2h = a.pml_i2h;
    const double wj = damp(y);
    const double lj = ln[i];
    double cur = (2 - 6 * K * ih2) * lj;
    double ps[6] = {0, 0, 0, 0, 0, 0};
    if (wj != 0)
#pragma unroll
        for (int d = 0; d < 3; d++)
        {
            // psi^sigma[j] from psi^{sigma-1}[j]
            int m[3] = {y[0], y[1], y[2]};
            m[d] -= y[d] > res / 2 ? 1 : -1;
            ps[d] += (1 - cdt * wj / 2) * (double)pn[6 * i + d];
            ps[3 + d] += (1 - cdt * damp(m) / 2) * (double)pn[6 * i + 3 + d];
        }
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
        for (int s = -1; s <= 1; s += 2)
        {
            int x[3] = {y[0], y[1], y[2]};
            x[d] += s;  // the reading cell q
            if (!inside(x))
                continue;
            const long long xi = ((long long)x[0] * res + x[1]) * res + x[2];
            const double lq = ln[xi], wq = damp(x);
            cur += K * ih2 * lq;
            const int sq = x[d] > res / 2 ? 1 : -1;
            const double pd = wq != 0 ? (double)pn[6 * xi + d] : 0.0, pd3 = wq != 0 ? (double)pn[6 * xi + 3 + d] : 0.0;
            if (sq == -s)
            {
                // j = ps of q: p^sigma[q] reads psi_{3+d} of j; psi^sigma[q] reads p of j and psi_{3+d} of j
                ps[3 + d] += K * wq * ih * lq - cdt * wq / 2 * pd3;
                cur -= cdt * i2h * (pd + pd3);
            }
            else
            {
                // j = ms of q: p^sigma[q] reads psi_d of j (damped by w(j)); psi^sigma[q] reads p of j and psi_d of j
                ps[d] += -K * wj * ih * lq - cdt * wj / 2 * pd;
                cur += cdt * i2h * (pd + pd3);
            }
        }
    lc[i] = (R)((double)lc[i] + cur);
    lp[i] = (R)(-lj);
#pragma unroll
    for (int k = 0; k < 6; k++)
        pc[6 * i + k] = wj != 0 ? (R)ps[k] : (R)0;  // psi^{sigma-1}[j] is zero where j is undamped
}

// ---- tables
template <typename R>
__global__ void shift_face_kernel(const typename AdjWRec<R>::T *w, const float2 *scale, const int *pair, long long n,
                                  typename AdjWRec<R>::T *wt, float2 *scale_t)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * kTaps)
        return;
    const long long p2 = t / kTaps;
    const int m = (int)(t % kTaps);
    const long long p = pair[p2];
    const auto *src = w + p * kTaps;
    if constexpr (sizeof(R) == 4)
    {
        const __half lo = __low2half(src[m]);
        const __half hi = m + 1 < kTaps ? __high2half(src[m + 1]) : __float2half(0.0f);
        wt[t] = __halves2half2(lo, hi);
        if (m == 0 && scale)
            scale_t[p2] = scale[p];
    }
    else
        wt[t] = make_double2(src[m].x, m + 1 < kTaps ? src[m + 1].y : 0.0);
}

// near records of the transposed pairs: pair p2 (forward pair pair[p2] of triangle p3_tri and
// record offset p3_woff) gets its FDTD-near record shifted by one tap (row[k] = tap k + 1, the
// step pairs it with the next step's history) and its BEM-near record
template <typename R>
__global__ void near_records_kernel(const typename AdjWRec<R>::T *gc_w, const float2 *gc_scale, const int *p3_tri,
                                    const unsigned char *p3_woff, const int *pair, long long n,
                                    typename AdjWRec<R>::T *wt, float2 *scale_t)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * kTaps)
        return;
    const long long p2 = t / kTaps;
    const int k = (int)(t % kTaps);
    const long long pp = pair[p2];
    const long long rec = (long long)p3_tri[pp] * 54 + p3_woff[pp];
    const auto *f = gc_w + rec * kTaps, *b = gc_w + (rec + 27) * kTaps;
    typename AdjWRec<R>::T zero;
    memset(&zero, 0, sizeof(zero));
    wt[p2 * 2 * kTaps + k] = k + 1 < kTaps ? f[k + 1] : zero;
    wt[p2 * 2 * kTaps + kTaps + k] = b[k];
    if (k == 0 && gc_scale)
    {
        scale_t[2 * p2] = gc_scale[rec];
        scale_t[2 * p2 + 1] = gc_scale[rec + 27];
    }
}

// ---- transposed tables, built on the device (counting transposes, values ascending per key)

__global__ void key_count_kernel(const int *key, long long n, int *count)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        atomicAdd(&count[key[i]], 1);
}

__global__ void key_fill_kernel(const int *key, long long n, const int *start, int *cursor, int *order)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        order[start[key[i]] + atomicAdd(&cursor[key[i]], 1)] = (int)i;
}

// each key's values ascending: the fill's atomic order is arbitrary, the sweep's sums must not be
__global__ void key_sort_kernel(const int *start, int nkeys, int *order)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nkeys)
        return;
    const int b = start[k], e = start[k + 1];
    for (int i = b + 1; i < e; i++)
    {
        const int v = order[i];
        int j = i - 1;
        while (j >= b && order[j] > v)
        {
            order[j + 1] = order[j];
            j--;
        }
        order[j + 1] = v;
    }
}

// owner[p] = the segment of a CSR (start[nseg + 1]) that holds position p; one warp per segment
__global__ void owner_kernel(const int *start, int nseg, int *owner)
{
    const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (w >= nseg)
        return;
    for (int p = start[w] + lane; p < start[w + 1]; p += 32)
        owner[p] = w;
}

__global__ void gather_int_kernel(const int *src, const int *idx, long long n, int *out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = src[idx[i]];
}

// corner cells lie in the grid whenever the lists could be built (triangles at least two cells
// inside it); the bound keeps the writes in range regardless
__global__ void flag_cells_kernel(const int *cell, long long n, long long ncells, int *flag)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && cell[i] >= 0 && cell[i] < ncells)
        flag[cell[i]] = 1;
}

// the distinct corner cells in ascending order (pos: exclusive scan of the flags) and each
// corner's rank among them
__global__ void corner_rank_kernel(const int *cell, long long n, long long ncells, const int *pos, int *rank)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        rank[i] = cell[i] >= 0 && cell[i] < ncells ? pos[cell[i]] : 0;
}

__global__ void compact_cells_kernel(const int *flag, const int *pos, long long ncells, int *out)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < ncells && flag[c])
        out[pos[c]] = (int)c;
}

template <typename T>
int grow(T **p, long long &cap, long long need)
{
    need = std::max<long long>(need, 1);
    if (need <= cap)
        return PPPM_OK;
    dev_free(*p);
    *p = nullptr;
    const long long nc = need + need / 4 + 64;
    PB_TRY(dalloc(p, (size_t)nc));
    cap = nc;
    return PPPM_OK;
}

int grow_bytes(void **p, long long &cap, long long need)
{
    need = std::max<long long>(need, 1);
    if (need <= cap)
        return PPPM_OK;
    dev_free(*p);
    *p = nullptr;
    const long long nc = need + need / 4 + 256;
    PB_TRY(dev_alloc(p, (size_t)nc));
    cap = nc;
    return PPPM_OK;
}

// start[nkeys + 1], order[n]: the positions p of key[p] grouped by key, ascending inside a key
int transpose_dev(Handle &h, Adjoint &A, const int *key, long long n, int nkeys, int *start, int *order)
{
    cudaStream_t s = h.stream;
    const int T = 256;
    PB_TRY(grow(&A.d_count, A.cap[15], (long long)nkeys + 1));
    PB_TRY(grow(&A.d_cursor, A.cap[16], (long long)nkeys + 1));
    PB_CUDA(cudaMemsetAsync(A.d_count, 0, sizeof(int) * (size_t)(nkeys + 1), s));
    PB_CUDA(cudaMemsetAsync(A.d_cursor, 0, sizeof(int) * (size_t)(nkeys + 1), s));
    if (n > 0)
        key_count_kernel<<<div_up(n, T), T, 0, s>>>(key, n, A.d_count);
    PB_TRY(exclusive_scan(h, A.d_count, start, nkeys));
    if (n > 0)
    {
        key_fill_kernel<<<div_up(n, T), T, 0, s>>>(key, n, start, A.d_cursor, order);
        key_sort_kernel<<<div_up(nkeys, T), T, 0, s>>>(start, nkeys, order);
        h.launches += 3;
    }
    PB_CHECK_LAUNCH();
    return PPPM_OK;
}

void adj_free_tables(Adjoint &A)
{
    void **ptrs[] = {(void **)&A.fT_start, (void **)&A.fT_src,   &A.fT_w,   (void **)&A.fT_scale,
                     (void **)&A.nT_start, (void **)&A.nT_cell,  (void **)&A.nT_pair,  &A.nT_w,
                     (void **)&A.nT_scale, (void **)&A.cT_cell,  (void **)&A.cT_start, (void **)&A.cT_ref,
                     (void **)&A.d_count,  (void **)&A.d_cursor, (void **)&A.d_order,  (void **)&A.d_owner,
                     (void **)&A.d_flag};
    for (void **p : ptrs)
    {
        dev_free(*p);
        *p = nullptr;
    }
    for (long long &c : A.cap)
        c = 0;
}

void adj_free_state(Adjoint &A)
{
    void **ptrs[] = {&A.lam[0], &A.lam[1], &A.lam[2], &A.lam_b, &A.acc_n, &A.acc_d, &A.lam_f, &A.d_g, &A.d_out,
                     &A.psi[0], &A.psi[1], &A.d_step};
    if (A.chunk)
        cudaGraphExecDestroy(A.chunk);
    A.chunk = nullptr;
    A.chunk_sig.clear();
    for (void **p : ptrs)
    {
        dev_free(*p);
        *p = nullptr;
    }
    A.g_cap = A.out_cap = 0;
}

// The transposed tables of the current geometry: face pairs by neighbour (with the centre and
// the re-packed weights), 3^3 pairs by triangle (with the corrected cell and the near records),
// corner references by cell.  All on the device; one synchronisation reads the number of
// distinct corner cells.  Capacities only grow, so a sweep over many motion frames allocates
// once.
template <typename R>
int build_tables(Handle &h, Adjoint &A)
{
    using W = typename AdjWRec<R>::T;
    cudaStream_t s = h.stream;
    const int nt = h.nt, n3 = h.n3, T = 256;
    const long long pf = h.pf, p3 = h.p3, nc8 = (long long)nt * 8, ncells = h.n_cells;
    const long long wsz = (long long)sizeof(W);
    long long *c = A.cap;
    PB_TRY(grow(&A.d_order, c[0], std::max(std::max(pf, p3), nc8)));
    PB_TRY(grow(&A.d_owner, c[1], std::max(pf, p3)));
    PB_TRY(grow(&A.fT_start, c[2], nt + 1));
    PB_TRY(grow(&A.fT_src, c[3], pf));
    PB_TRY(grow_bytes(&A.fT_w, c[4], pf * kTaps * wsz));
    if (!h.fp64)
        PB_TRY(grow(&A.fT_scale, c[5], pf));
    PB_TRY(grow(&A.nT_start, c[6], nt + 1));
    PB_TRY(grow(&A.nT_cell, c[7], p3));
    PB_TRY(grow(&A.nT_pair, c[8], p3));
    PB_TRY(grow_bytes(&A.nT_w, c[9], p3 * 2 * kTaps * wsz));
    if (!h.fp64)
        PB_TRY(grow(&A.nT_scale, c[10], 2 * p3));
    PB_TRY(grow(&A.d_flag, c[11], 2 * (ncells + 1)));
    PB_TRY(grow(&A.cT_ref, c[12], nc8));
    int *order = A.d_order, *owner = A.d_owner;

    // face pairs by neighbour; fT_src = centre of each transposed pair
    PB_TRY(transpose_dev(h, A, h.d_face_nbr, pf, nt, A.fT_start, order));
    if (pf > 0)
    {
        owner_kernel<<<div_up((long long)nt * 32, T), T, 0, s>>>(h.d_face_start, nt, owner);
        gather_int_kernel<<<div_up(pf, T), T, 0, s>>>(owner, order, pf, A.fT_src);
        shift_face_kernel<R><<<div_up(pf * kTaps, T), T, 0, s>>>(
            (const W *)h.d_face_w, h.fp64 ? nullptr : h.d_face_scale, order, pf, (W *)A.fT_w, A.fT_scale);
        h.launches += 3;
    }
    A.pfT = pf;
    PB_CHECK_LAUNCH();

    // 3^3 pairs by triangle; nT_cell = corrected-cell index of each transposed pair
    PB_TRY(transpose_dev(h, A, h.d_p3_tri, p3, nt, A.nT_start, A.nT_pair));
    if (p3 > 0)
    {
        owner_kernel<<<div_up((long long)std::max(n3, 1) * 32, T), T, 0, s>>>(h.d_n3_start, n3, owner);
        gather_int_kernel<<<div_up(p3, T), T, 0, s>>>(owner, A.nT_pair, p3, A.nT_cell);
        near_records_kernel<R><<<div_up(p3 * kTaps, T), T, 0, s>>>(
            (const W *)h.d_gc_w, h.fp64 ? nullptr : h.d_gc_scale, h.d_p3_tri, h.d_p3_woff, A.nT_pair, p3,
            (W *)A.nT_w, A.nT_scale);
        h.launches += 3;
    }
    A.p3T = p3;
    PB_CHECK_LAUNCH();

    // corner references by cell: the distinct corner cells ascending, each corner's rank
    int *flag = A.d_flag, *pos = A.d_flag + (ncells + 1);
    PB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int) * (size_t)(ncells + 1), s));
    flag_cells_kernel<<<div_up(nc8, T), T, 0, s>>>(h.d_face_corner, nc8, ncells, flag);
    h.launches++;
    PB_TRY(exclusive_scan(h, flag, pos, ncells));
    int ncorner = 0;
    PB_TRY(read_int(h, pos + ncells, &ncorner));
    PB_TRY(grow(&A.cT_cell, c[13], ncorner));
    PB_TRY(grow(&A.cT_start, c[14], (long long)ncorner + 1));
    compact_cells_kernel<<<div_up(ncells, T), T, 0, s>>>(flag, pos, ncells, A.cT_cell);
    corner_rank_kernel<<<div_up(nc8, T), T, 0, s>>>(h.d_face_corner, nc8, ncells, pos, order);
    h.launches += 2;
    PB_TRY(transpose_dev(h, A, order, nc8, ncorner, A.cT_start, A.cT_ref));
    A.ncorner = ncorner;
    A.nt = nt;
    A.n3 = n3;
    A.version = h.mesh_version;
    return PPPM_OK;
}

template <typename R>
int alloc_state(Handle &h, Adjoint &A)
{
    const size_t rs = sizeof(R);
    for (int i = 0; i < 3; i++)
        if (!A.lam[i])
            PB_TRY(dev_alloc(&A.lam[i], (size_t)h.n_cells * rs));
    if (!A.lam_b)
        PB_TRY(dev_alloc(&A.lam_b, (size_t)4 * h.n_cells * rs));
    if (h.prm.pml_width > 0)
        for (int i = 0; i < 2; i++)
            if (!A.psi[i])
                PB_TRY(dev_alloc(&A.psi[i], (size_t)6 * h.n_cells * rs));
    // per triangle: the triangle count is fixed by the topology, so a sweep keeps these across
    // geometry changes
    if (!A.acc_n)
        PB_TRY(dev_alloc(&A.acc_n, (size_t)std::max(h.nt, 1) * kRing * rs));
    if (!A.acc_d)
        PB_TRY(dev_alloc(&A.acc_d, (size_t)std::max(h.nt, 1) * kRing * rs));
    if (!A.lam_f)
        PB_TRY(dev_alloc(&A.lam_f, (size_t)std::max(h.nt, 1) * rs));
    return PPPM_OK;
}

template <typename R>
int zero_state(Handle &h, Adjoint &A)
{
    const size_t rs = sizeof(R);
    for (int i = 0; i < 3; i++)
        PB_CUDA(cudaMemsetAsync(A.lam[i], 0, (size_t)h.n_cells * rs, h.stream));
    PB_CUDA(cudaMemsetAsync(A.acc_n, 0, (size_t)std::max(h.nt, 1) * kRing * rs, h.stream));
    PB_CUDA(cudaMemsetAsync(A.acc_d, 0, (size_t)std::max(h.nt, 1) * kRing * rs, h.stream));
    PB_CUDA(cudaMemsetAsync(A.lam_f, 0, (size_t)std::max(h.nt, 1) * rs, h.stream));
    for (int i = 0; i < 2; i++)
        if (A.psi[i])
            PB_CUDA(cudaMemsetAsync(A.psi[i], 0, (size_t)6 * h.n_cells * rs, h.stream));
    return PPPM_OK;
}

template <typename R>
AdjArgs<R> make_adj_args(Handle &h, Adjoint &A)
{
    using W = typename AdjWRec<R>::T;
    AdjArgs<R> a;
    memset(&a, 0, sizeof(a));
    a.res = h.res;
    a.nt = h.nt;
    a.n3 = h.n3;
    a.ncells = h.n_cells;
    a.nl = (int)h.listen_xyz.size() / 3;
    for (int l = 0; l < a.nl; l++)
    {
        a.listen_cell[l] = (h.listen_xyz[3 * l] * h.res + h.listen_xyz[3 * l + 1]) * h.res + h.listen_xyz[3 * l + 2];
    }
    a.ncorner = A.ncorner;
    a.n3_cell = h.d_n3_cell;
    a.corr_mask = h.d_corr_mask;
    a.fT_start = A.fT_start;
    a.fT_src = A.fT_src;
    a.fT_w = (const W *)A.fT_w;
    a.fT_scale = h.fp64 ? nullptr : A.fT_scale;
    a.nT_start = A.nT_start;
    a.nT_cell = A.nT_cell;
    a.nT_pair = A.nT_pair;
    a.nT_w = (const W *)A.nT_w;
    a.nT_scale = h.fp64 ? nullptr : A.nT_scale;
    a.cT_cell = A.cT_cell;
    a.cT_start = A.cT_start;
    a.cT_ref = A.cT_ref;
    a.interp = h.d_face_interp;
    a.interp_d = h.fp64 ? h.d_face_interp_d : nullptr;
    a.denom = h.d_face_denom;
    a.reflect = h.prm.reflect_coeff;
    for (int i = 0; i < 3; i++)
        a.lam[i] = (R *)A.lam[i];
    a.lam_b = (R *)A.lam_b;
    a.acc_n = (R *)A.acc_n;
    a.acc_d = (R *)A.acc_d;
    a.lam_f = (R *)A.lam_f;
    const double cd = h.prm.c, dtd = h.prm.dt, hd = h.prm.dl;
    a.kappa = cd * cd * dtd * dtd / (hd * hd);
    const R c = (R)h.prm.c, dt = (R)h.prm.dt, hh = (R)h.prm.dl;
    a.coef = c * c * dt * dt / (hh * hh);
    a.coef1 = 1 / (dt * dt);
    a.coef2 = c / (2 * hh * dt);
    a.coef3 = -(c * c) / (2 * hh * hh);
    for (int i = 0; i < 2; i++)
        a.psi[i] = (R *)A.psi[i];
    a.pml_w = h.prm.pml_width;
    // the forward's own coefficients (pml_kernel: c, dt, h as the step's floats)
    const double pc = (float)h.prm.c, pdt = (float)h.prm.dt, ph = (float)h.prm.dl;
    a.pml_damp = (double)(2.0f / h.prm.dl);
    a.pml_k = pc * pc * pdt * pdt;
    a.pml_ih2 = 1 / (ph * ph);
    a.pml_ih = 1 / ph;
    a.pml_cdt = pc * pdt;
    a.pml_i2h = 1 / (ph * 2);
    return a;
}

__global__ void set_adj_step_kernel(AdjStep *dst, AdjStep v) { *dst = v; }
__global__ void advance_adj_kernel(AdjStep *st, int g) { st->top -= g; }

// the kernels of reverse step j of the call (no error check: may run under stream capture)
template <typename R>
void adj_launch_step(const AdjArgs<R> &a, const AdjStep *st, int j, cudaStream_t s, long long nbd)
{
    const int T = 256, tw = div_up((long long)a.nt * 32, T);
    if (a.nl > 0)
        adj_listen_kernel<R><<<1, 32, 0, s>>>(a, st, j);
    adj_bem_kernel<R><<<tw, T, 0, s>>>(a, st, j);
    adj_face_kernel<R><<<tw, T, 0, s>>>(a, st, j);
    if (a.ncorner > 0)
        adj_corner_kernel<R><<<div_up(a.ncorner, T), T, 0, s>>>(a, st, j);
    adj_fdtd_near_kernel<R><<<tw, T, 0, s>>>(a, st, j);
    if (a.pml_w > 0)
        adj_pml_kernel<R><<<div_up(a.ncells, T), T, 0, s>>>(a, st, j);
    else
    {
        adj_boundary_kernel<R><<<div_up(nbd, T), T, 0, s>>>(a, st, j);
        adj_stencil_kernel<R><<<div_up(a.ncells, T), T, 0, s>>>(a, st, j);
    }
}

// A sweep's reverse steps cost five to seven launches each, so long sweeps with fixed tables
// replay a recorded chunk of kAdjChunk reverse steps (about 0.1 ms of host time per step to record,
// once per handle and launch arguments); the steps left over, short calls (a moving sweep's
// frames) and calls on a stream being captured launch the kernels directly.
constexpr int kAdjChunk = 32;

template <typename R>
int run_adjoint(Handle &h, const R *g, int nsteps, R *out, int fresh)
{
    if (!h.adj)
    {
        h.adj = new (std::nothrow) Adjoint();
        if (!h.adj)
            return PPPM_ERR_NOMEM;
    }
    Adjoint &A = *h.adj;
    if (A.version != h.mesh_version)
    {
        // the tables of the steps this call covers; the adjoint state (grid slots and per-triangle
        // rings) carries over, so a sweep may continue across a motion frame
        PB_TRY(build_tables<R>(h, A));
        PB_TRY(alloc_state<R>(h, A));
    }
    if (fresh || !A.started)
    {
        PB_TRY(zero_state<R>(h, A));
        A.pos = kAdjTop;
        A.started = true;
    }
    const AdjArgs<R> a = make_adj_args<R>(h, A);
    const int top = A.pos, bottom = A.pos - nsteps;
    const long long nbd = boundary_cells(h.res);
    cudaStream_t s = h.stream;
    if (!A.d_step)
        PB_TRY(dev_alloc(&A.d_step, sizeof(AdjStep)));
    AdjStep *dst = (AdjStep *)A.d_step;
    set_adj_step_kernel<<<1, 1, 0, s>>>(dst, AdjStep{top, bottom, g, out});
    PB_CHECK_LAUNCH();
    const long long per_step = 5 + (a.nl > 0) + (a.ncorner > 0) - (a.pml_w > 0);
    h.launches += 1;
    int done = 0;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PB_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusNone && nsteps >= 2 * kAdjChunk)
    {
        std::vector<unsigned char> sig((const unsigned char *)&a, (const unsigned char *)&a + sizeof(a));
        const bool have = A.chunk && A.chunk_sig == sig;
        if (!have && nsteps >= 4 * kAdjChunk)
        {
            if (A.chunk)
                cudaGraphExecDestroy(A.chunk);
            A.chunk = nullptr;
            A.chunk_sig.clear();
            cudaGraph_t graph = nullptr;
            PB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            for (int j = 0; j < kAdjChunk; j++)
                adj_launch_step<R>(a, dst, j, s, nbd);
            advance_adj_kernel<<<1, 1, 0, s>>>(dst, kAdjChunk);
            cudaError_t e = cudaStreamEndCapture(s, &graph);
            if (e == cudaSuccess)
                e = cudaGraphInstantiate(&A.chunk, graph, 0);
            if (graph)
                cudaGraphDestroy(graph);
            if (e != cudaSuccess)
            {
                A.chunk = nullptr;
                set_error("recording the adjoint chunk graph failed: %s", cudaGetErrorString(e));
                return PPPM_ERR_CUDA;
            }
            A.chunk_sig.swap(sig);
        }
        if (A.chunk && A.chunk_sig.size() == sizeof(a) && memcmp(A.chunk_sig.data(), &a, sizeof(a)) == 0)
        {
            const int chunks = nsteps / kAdjChunk;
            for (int c = 0; c < chunks; c++)
                PB_CUDA(cudaGraphLaunch(A.chunk, s));
            done = chunks * kAdjChunk;
            h.launches += (long long)chunks * (per_step * kAdjChunk + 1);
        }
    }
    for (int j = 0; j < nsteps - done; j++)  // relative to the state the chunks advanced
    {
        adj_launch_step<R>(a, dst, j, s, nbd);
        PB_CHECK_LAUNCH();
        h.launches += per_step;
    }
    A.pos = bottom;
    return PPPM_OK;
}

}  // namespace

int adjoint_run(Handle &h, const void *g, int nsteps, void *out, int fresh)
{
    if (h.fp64)
        return run_adjoint<double>(h, (const double *)g, nsteps, (double *)out, fresh);
    return run_adjoint<float>(h, (const float *)g, nsteps, (float *)out, fresh);
}

int adjoint_stage(Handle &h, size_t g_bytes, size_t out_bytes, void **g, void **out)
{
    if (!h.adj)
    {
        h.adj = new (std::nothrow) Adjoint();
        if (!h.adj)
            return PPPM_ERR_NOMEM;
    }
    Adjoint &A = *h.adj;
    if ((long long)g_bytes > A.g_cap)
    {
        dev_free(A.d_g);
        A.d_g = nullptr;
        PB_TRY(dev_alloc(&A.d_g, g_bytes));
        A.g_cap = (long long)g_bytes;
    }
    if ((long long)out_bytes > A.out_cap)
    {
        dev_free(A.d_out);
        A.d_out = nullptr;
        PB_TRY(dev_alloc(&A.d_out, out_bytes));
        A.out_cap = (long long)out_bytes;
    }
    *g = A.d_g;
    *out = A.d_out;
    return PPPM_OK;
}

void adjoint_free(Handle &h)
{
    if (!h.adj)
        return;
    adj_free_tables(*h.adj);
    adj_free_state(*h.adj);
    delete h.adj;
    h.adj = nullptr;
}

}  // namespace pb
