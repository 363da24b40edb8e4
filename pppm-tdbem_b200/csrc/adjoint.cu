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
// Adjoint variables: Lambda(tau) per grid slot (tau mod 3, ghosts included), and rings over
// time (4 shifted copies each, so a 16-tap window is 4 aligned 16-byte loads): lamF[j] (adjoint
// of the face numerator), lamP[c] (0.98 x adjoint of the near correction), lamC[c] (adjoint of
// the stored FDTD-near sum).  The reverse step at sigma runs five kernels:
//   A1 cells     add dL/dseries[sigma] at the listener cells; lamP[c][sigma] = 0.98
//                Lambda(sigma)[c]; lamC[c][sigma] = -Lambda(sigma + 1)[c]
//   A2 faces     per triangle j, gathers over the transposed pair lists:
//                lamF[j][sigma] = (sum_{face pairs (i, j)} sum_{k=1..15} b_k lamF[i][sigma+k]
//                  + sum_{near pairs (c, j)} sum_{k=0..15} bb_k lamP[c][sigma+k]
//                  + bf_k lamC[c][sigma+k]) / denom_j
//                dL/dacc[sigma+1][j] = sum_{face pairs} sum_{k=0..15} a_k lamF[i][sigma+1+k]
//                  + the near part of sigma + 1 (kept from the previous reverse step)
//   A3 corners   Lambda(sigma)[cell] += reflect iw lamF[j][sigma] over the cells that are
//                trilinear corners of some face
//   A4 boundary  per boundary-layer cell: lam_b = A^-T (adjoints of its ghost outputs, of
//                its own output); the ghost adjoints of Lambda(sigma - 1) are consumed
//   A5 cells     transposed stencil as a gather over the 7 cells that read a cell:
//                Lambda(sigma - 1) += S_cur^T; Lambda(sigma - 2) = S_prev^T (the first
//                contribution to that slot's new time, so it overwrites the stale one)
// After the last reverse step of a call, A2 in flush mode emits dL/dacc of the call's first
// step.  The gathers (A2, A3, A5) need no atomics: every sum belongs to one thread or warp.
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
    // adjoint state
    void *lam[3] = {nullptr, nullptr, nullptr};
    void *lam_b = nullptr;  // 4 x res^3 (boundary layer only)
    void *ring_f = nullptr, *ring_p = nullptr, *ring_c = nullptr;
    void *nearpart = nullptr;  // nt: near part of dL/dacc of the last reverse step's time
    int pos = 0;               // one past the next time the reverse sweep processes
    bool started = false;
    // host-call staging
    void *d_g = nullptr, *d_out = nullptr;
    long long g_cap = 0, out_cap = 0;
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
    R *ring_f, *ring_p, *ring_c;
    R *nearpart;
    double kappa;                 // (c dt / h)^2: interior leapfrog coefficient
    R coef, coef1, coef2, coef3;  // boundary solve coefficients (fdtd.cu:88-137)
    __device__ R *slot(int tau) const { return lam[((tau % 3) + 3) % 3]; }
};

// ring copy c holds time tau at index (tau + c) mod 32: a window starting at tau0 read from copy
// (-tau0) mod 4 starts on a multiple of 4
template <typename R>
__device__ inline void ring_put(R *ring, int rows, int row, int tau, R v)
{
#pragma unroll
    for (int c = 0; c < 4; c++)
        ring[((long long)c * rows + row) * kRing + ((tau + c) & (kRing - 1))] = v;
}

template <typename R>
__device__ inline const R *ring_window(const R *ring, int rows, int tau0, int q)
{
    const int c = (-tau0) & 3;
    return ring + (long long)c * rows * kRing + ((tau0 + c + 4 * q) & (kRing - 1));
}

// A1: corrected cells and listener injection
template <typename R>
__global__ void __launch_bounds__(256) adj_cells_kernel(const __grid_constant__ AdjArgs<R> a, int sigma,
                                                        const R *g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    R *cur = a.slot(sigma);
    if (i < a.n3)
    {
        const int c = a.n3_cell[i];
        R v = cur[c];
        for (int l = 0; l < a.nl; l++)
            if (a.listen_cell[l] == c)
                v += g[l];
        cur[c] = v;
        ring_put<R>(a.ring_p, a.n3, i, sigma, (R)0.98 * v);
        ring_put<R>(a.ring_c, a.n3, i, sigma, -a.slot(sigma + 1)[c]);
    }
    else if (i == a.n3)
        for (int l = 0; l < a.nl; l++)
        {
            const int c = a.listen_cell[l];
            if (!((a.corr_mask[c >> 5] >> (c & 31)) & 1u))  // corrected cells: done above
                cur[c] += g[l];
        }
}

template <typename R>
__device__ inline R warp_sum_adj(R v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// A2: one warp per triangle j; quad q of lane group g takes window positions 4q..4q+3 of pairs
// g, g + 8, ...  flush != 0: only dL/dacc of time sigma + 1 (the face part) plus the kept near part
template <typename R>
__global__ void __launch_bounds__(256) adj_face_kernel(const __grid_constant__ AdjArgs<R> a, int sigma, R *out_row,
                                                       int flush)
{
    using W4 = typename AdjWRec<R>::W4;
    using H4 = typename AdjWRec<R>::H4;
    const int j = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (j >= a.nt)
        return;
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    // face pairs: lamF window sigma + 1 .. sigma + 16, shifted records (a_m, b_{m+1})
    const R *wf = ring_window<R>(a.ring_f, a.nt, sigma + 1, q);
    R acc_n = 0, acc_d = 0;
    for (int p = a.fT_start[j] + g; p < a.fT_start[j + 1]; p += 8)
    {
        const W4 w = *(const W4 *)(a.fT_w + (long long)p * kTaps + 4 * q);
        const float2 s = a.fT_scale ? a.fT_scale[p] : make_float2(1, 1);
        const H4 h = *(const H4 *)(wf + (long long)a.fT_src[p] * kRing);
#pragma unroll
        for (int i = 0; i < 4; i++)
        {
            acc_n += (R)wa(w.v[i], s) * h.v[i];
            acc_d += (R)wb(w.v[i], s) * h.v[i];
        }
    }
    R near_n = 0, near_d = 0;
    if (!flush)
    {
        // near pairs: lamP / lamC windows sigma .. sigma + 15
        const R *wp = ring_window<R>(a.ring_p, a.n3, sigma, q), *wc = ring_window<R>(a.ring_c, a.n3, sigma, q);
        for (int p = a.nT_start[j] + g; p < a.nT_start[j + 1]; p += 8)
        {
            const int ci = a.nT_cell[p];
            const W4 rf = *(const W4 *)(a.nT_w + (long long)p * 2 * kTaps + 4 * q);
            const W4 rb = *(const W4 *)(a.nT_w + (long long)p * 2 * kTaps + kTaps + 4 * q);
            const float2 sf = a.nT_scale ? a.nT_scale[2 * p] : make_float2(1, 1);
            const float2 sb = a.nT_scale ? a.nT_scale[2 * p + 1] : make_float2(1, 1);
            const H4 hp = *(const H4 *)(wp + (long long)ci * kRing);
            const H4 hc = *(const H4 *)(wc + (long long)ci * kRing);
#pragma unroll
            for (int i = 0; i < 4; i++)
            {
                near_n += (R)wa(rb.v[i], sb) * hp.v[i] + (R)wa(rf.v[i], sf) * hc.v[i];
                near_d += (R)wb(rb.v[i], sb) * hp.v[i] + (R)wb(rf.v[i], sf) * hc.v[i];
            }
        }
    }
    acc_n = warp_sum_adj(acc_n);
    if (!flush)
    {
        acc_d = warp_sum_adj(acc_d);
        near_n = warp_sum_adj(near_n);
        near_d = warp_sum_adj(near_d);
        if (lane < 4)
        {
            const R lf = (R)((acc_d + near_d) / a.denom[j]);
            a.ring_f[((long long)lane * a.nt + j) * kRing + ((sigma + lane) & (kRing - 1))] = lf;
        }
    }
    if (lane == 0)
    {
        if (out_row)
            out_row[j] = acc_n + a.nearpart[j];
        if (!flush)
            a.nearpart[j] = near_n;
    }
}

// A3: corner cells of the face interpolation
template <typename R>
__global__ void __launch_bounds__(256) adj_corner_kernel(const __grid_constant__ AdjArgs<R> a, int sigma)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.ncorner)
        return;
    R v = 0;
    const int slot = sigma & (kRing - 1);  // copy 0 holds time sigma at index sigma mod 32
    for (int r = a.cT_start[i]; r < a.cT_start[i + 1]; r++)
    {
        const int ref = a.cT_ref[r];
        const R iw = a.interp_d ? (R)a.interp_d[ref] : (R)a.interp[ref];
        v += iw * a.ring_f[(long long)(ref >> 3) * kRing + slot];
    }
    a.slot(sigma)[a.cT_cell[i]] += (R)a.reflect * v;
}

__device__ inline int judge_of(int v, int res) { return -((int)(v == 1)) + ((int)(v == res - 2)); }

// A4: the boundary-layer solve transposed
template <typename R>
__global__ void __launch_bounds__(256) adj_boundary_kernel(const __grid_constant__ AdjArgs<R> a, int sigma)
{
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

// A5: the transposed stencil, one thread per cell of the whole grid (ghost layer included)
template <typename R>
__global__ void __launch_bounds__(256) adj_stencil_kernel(const __grid_constant__ AdjArgs<R> a, int sigma)
{
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

template <typename T>
int upload(Handle &h, T **d, const std::vector<T> &v)
{
    dev_free(*d);
    *d = nullptr;
    PB_TRY(dalloc(d, std::max<size_t>(v.size(), 1)));
    if (!v.empty())
        PB_CUDA(cudaMemcpyAsync(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h.stream));
    return PPPM_OK;
}

template <typename T>
int download(Handle &h, std::vector<T> &v, const T *d, size_t n)
{
    v.resize(n);
    if (n)
        PB_CUDA(cudaMemcpyAsync(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, h.stream));
    return PPPM_OK;
}

// CSR of (key -> values) from pairs given in value order, stable within a key
void transpose_csr(int nkeys, const std::vector<int> &keys, std::vector<int> &start, std::vector<int> &order)
{
    start.assign(nkeys + 1, 0);
    for (int k : keys)
        start[k + 1]++;
    for (int k = 0; k < nkeys; k++)
        start[k + 1] += start[k];
    std::vector<int> cursor(start.begin(), start.end() - 1);
    order.resize(keys.size());
    for (size_t p = 0; p < keys.size(); p++)
        order[cursor[keys[p]]++] = (int)p;
}

void adj_free_tables(Adjoint &A)
{
    void **ptrs[] = {(void **)&A.fT_start, (void **)&A.fT_src,   &A.fT_w,  (void **)&A.fT_scale,
                     (void **)&A.nT_start, (void **)&A.nT_cell,  (void **)&A.nT_pair, &A.nT_w,
                     (void **)&A.nT_scale, (void **)&A.cT_cell,  (void **)&A.cT_start, (void **)&A.cT_ref};
    for (void **p : ptrs)
    {
        dev_free(*p);
        *p = nullptr;
    }
}

void adj_free_state(Adjoint &A)
{
    void **ptrs[] = {&A.lam[0], &A.lam[1], &A.lam[2], &A.lam_b, &A.ring_f, &A.ring_p, &A.ring_c, &A.nearpart,
                     &A.d_g,    &A.d_out};
    for (void **p : ptrs)
    {
        dev_free(*p);
        *p = nullptr;
    }
    A.g_cap = A.out_cap = 0;
}

template <typename R>
int build_tables(Handle &h, Adjoint &A)
{
    using W = typename AdjWRec<R>::T;
    adj_free_tables(A);
    const int nt = h.nt, n3 = h.n3;
    std::vector<int> face_start, face_nbr, n3_start, p3_tri, corner, n3_cell;
    PB_TRY(download(h, face_start, h.d_face_start, (size_t)nt + 1));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    const long long pf = face_start[nt];
    PB_TRY(download(h, face_nbr, h.d_face_nbr, (size_t)pf));
    PB_TRY(download(h, n3_start, h.d_n3_start, (size_t)n3 + 1));
    PB_TRY(download(h, corner, h.d_face_corner, (size_t)nt * 8));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    const long long p3 = n3 ? n3_start[n3] : 0;
    PB_TRY(download(h, p3_tri, h.d_p3_tri, (size_t)p3));
    PB_CUDA(cudaStreamSynchronize(h.stream));

    // face pairs by neighbour
    std::vector<int> start, order;
    transpose_csr(nt, face_nbr, start, order);
    std::vector<int> src(pf), pair(pf);
    {
        std::vector<int> centre(pf);
        for (int i = 0; i < nt; i++)
            for (int p = face_start[i]; p < face_start[i + 1]; p++)
                centre[p] = i;
        for (long long k = 0; k < pf; k++)
        {
            pair[k] = order[k];
            src[k] = centre[order[k]];
        }
    }
    PB_TRY(upload(h, &A.fT_start, start));
    PB_TRY(upload(h, &A.fT_src, src));
    int *d_pair = nullptr;
    PB_TRY(upload(h, &d_pair, pair));
    PB_TRY(dev_alloc(&A.fT_w, (size_t)std::max<long long>(pf, 1) * kTaps * sizeof(W)));
    if (!h.fp64)
        PB_TRY(dalloc(&A.fT_scale, (size_t)std::max<long long>(pf, 1)));
    if (pf > 0)
        shift_face_kernel<R><<<div_up(pf * kTaps, 256), 256, 0, h.stream>>>(
            (const W *)h.d_face_w, h.fp64 ? nullptr : h.d_face_scale, d_pair, pf, (W *)A.fT_w, A.fT_scale);
    h.launches++;
    A.pfT = pf;

    // near pairs by triangle
    transpose_csr(nt, p3_tri, start, order);
    std::vector<int> cell(p3);
    {
        std::vector<int> owner(p3);
        for (int c = 0; c < n3; c++)
            for (int p = n3_start[c]; p < n3_start[c + 1]; p++)
                owner[p] = c;
        for (long long k = 0; k < p3; k++)
            cell[k] = owner[order[k]];
    }
    PB_TRY(upload(h, &A.nT_start, start));
    PB_TRY(upload(h, &A.nT_cell, cell));
    PB_TRY(upload(h, &A.nT_pair, order));
    PB_TRY(dev_alloc(&A.nT_w, (size_t)std::max<long long>(p3, 1) * 2 * kTaps * sizeof(W)));
    if (!h.fp64)
        PB_TRY(dalloc(&A.nT_scale, (size_t)std::max<long long>(p3, 1) * 2));
    if (p3 > 0)
        near_records_kernel<R><<<div_up(p3 * kTaps, 256), 256, 0, h.stream>>>(
            (const W *)h.d_gc_w, h.fp64 ? nullptr : h.d_gc_scale, h.d_p3_tri, h.d_p3_woff, A.nT_pair, p3,
            (W *)A.nT_w, A.nT_scale);
    h.launches++;
    A.p3T = p3;

    // corner cells
    std::vector<int> cells(corner.begin(), corner.end());
    std::sort(cells.begin(), cells.end());
    cells.erase(std::unique(cells.begin(), cells.end()), cells.end());
    std::vector<int> key(corner.size());
    for (size_t r = 0; r < corner.size(); r++)
        key[r] = (int)(std::lower_bound(cells.begin(), cells.end(), corner[r]) - cells.begin());
    transpose_csr((int)cells.size(), key, start, order);
    PB_TRY(upload(h, &A.cT_cell, cells));
    PB_TRY(upload(h, &A.cT_start, start));
    PB_TRY(upload(h, &A.cT_ref, order));
    A.ncorner = (int)cells.size();
    PB_CUDA(cudaStreamSynchronize(h.stream));
    dev_free(d_pair);
    PB_CHECK_LAUNCH();
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
    dev_free(A.ring_f);
    dev_free(A.ring_p);
    dev_free(A.ring_c);
    dev_free(A.nearpart);
    A.ring_f = A.ring_p = A.ring_c = A.nearpart = nullptr;
    PB_TRY(dev_alloc(&A.ring_f, (size_t)4 * std::max(A.nt, 1) * kRing * rs));
    PB_TRY(dev_alloc(&A.ring_p, (size_t)4 * std::max(A.n3, 1) * kRing * rs));
    PB_TRY(dev_alloc(&A.ring_c, (size_t)4 * std::max(A.n3, 1) * kRing * rs));
    PB_TRY(dev_alloc(&A.nearpart, (size_t)std::max(A.nt, 1) * rs));
    return PPPM_OK;
}

template <typename R>
int zero_state(Handle &h, Adjoint &A)
{
    const size_t rs = sizeof(R);
    for (int i = 0; i < 3; i++)
        PB_CUDA(cudaMemsetAsync(A.lam[i], 0, (size_t)h.n_cells * rs, h.stream));
    PB_CUDA(cudaMemsetAsync(A.ring_f, 0, (size_t)4 * std::max(A.nt, 1) * kRing * rs, h.stream));
    PB_CUDA(cudaMemsetAsync(A.ring_p, 0, (size_t)4 * std::max(A.n3, 1) * kRing * rs, h.stream));
    PB_CUDA(cudaMemsetAsync(A.ring_c, 0, (size_t)4 * std::max(A.n3, 1) * kRing * rs, h.stream));
    PB_CUDA(cudaMemsetAsync(A.nearpart, 0, (size_t)std::max(A.nt, 1) * rs, h.stream));
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
    a.ring_f = (R *)A.ring_f;
    a.ring_p = (R *)A.ring_p;
    a.ring_c = (R *)A.ring_c;
    a.nearpart = (R *)A.nearpart;
    const double cd = h.prm.c, dtd = h.prm.dt, hd = h.prm.dl;
    a.kappa = cd * cd * dtd * dtd / (hd * hd);
    const R c = (R)h.prm.c, dt = (R)h.prm.dt, hh = (R)h.prm.dl;
    a.coef = c * c * dt * dt / (hh * hh);
    a.coef1 = 1 / (dt * dt);
    a.coef2 = c / (2 * hh * dt);
    a.coef3 = -(c * c) / (2 * hh * hh);
    return a;
}

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
        if (A.started && !fresh)
        {
            set_error("the geometry changed since the adjoint sweep started: start a fresh sweep");
            return PPPM_ERR_STATE;
        }
        PB_TRY(build_tables<R>(h, A));
        PB_TRY(alloc_state<R>(h, A));
        A.started = false;
    }
    if (fresh || !A.started)
    {
        PB_TRY(zero_state<R>(h, A));
        A.pos = kAdjTop;
        A.started = true;
    }
    const AdjArgs<R> a = make_adj_args<R>(h, A);
    const int T = 256, top = A.pos, bottom = A.pos - nsteps;
    const long long nbd = boundary_cells(h.res);
    cudaStream_t s = h.stream;
    for (int sigma = top - 1; sigma >= bottom; sigma--)
    {
        adj_cells_kernel<R><<<div_up(a.n3 + 1, T), T, 0, s>>>(a, sigma, g + (long long)(sigma - bottom) * a.nl);
        R *row = sigma + 1 < top ? out + (long long)(sigma + 1 - bottom) * a.nt : nullptr;
        adj_face_kernel<R><<<div_up((long long)a.nt * 32, T), T, 0, s>>>(a, sigma, row, 0);
        if (a.ncorner > 0)
            adj_corner_kernel<R><<<div_up(a.ncorner, T), T, 0, s>>>(a, sigma);
        adj_boundary_kernel<R><<<div_up(nbd, T), T, 0, s>>>(a, sigma);
        adj_stencil_kernel<R><<<div_up(a.ncells, T), T, 0, s>>>(a, sigma);
        PB_CHECK_LAUNCH();
        h.launches += 4 + (a.ncorner > 0);
    }
    adj_face_kernel<R><<<div_up((long long)a.nt * 32, T), T, 0, s>>>(a, bottom - 1, out, 1);
    h.launches++;
    PB_CHECK_LAUNCH();
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
