// One PPPM time step as three kernels (the reference issues ~9 launches and ~10 device
// syncs per step, src/algorithm/pppm.h:138-145):
//
//   stencil   p^{t+1} = 2 p^t - p^{t-1} + (c dt)^2 lap p^t on [2, res-3]^3 (FP64 arithmetic
//             on FP32 storage, fdtd.cu:7-33), the absorbing boundary on layers 1 and res-2
//             (4x4 solve per cell that also writes the ghost layer of p^t, fdtd.cu:36-150) or
//             the split-field PML (fdtd.cu:162-232); at corrected cells subtract the FDTD-near
//             correction that the previous step's near kernel left in this very slot, which
//             turns p into the reference's far field (pppm.cu:8-50); write neumann[t+1] = acc
//             (pppm.cu:206-225).
//   face      per triangle (one warp): far field at the face by trilinear interpolation of
//             the 8 corner cells, the face-to-face convolution over its 4^3 list, and the
//             Dirichlet update (pppm.cu:116-193) - three reference kernels fused.
//   near      per corrected cell (one warp): p = far + 0.98 * sum(BEM-near weights . history)
//             (pppm.cu:53-113) and, in the same pass over the same pairs and history taps, the
//             FDTD-near sum of the NEXT step (its taps are t-14..t, all final now), stored in
//             the grid slot the next stencil writes.  One pass over the pair list per step
//             instead of two; no copy of the field into a separate far-field grid.
//
// Inside a convolution a warp handles two pairs at a time, one lane per tap, so weights
// (fp16 pairs) and history (16 consecutive ring slots) are read as coalesced 64-byte runs;
// partial sums stay in registers and are reduced once per triangle / cell.  No atomics.
#include <algorithm>
#include "fdtd.cuh"
#include "ghost.cuh"
#include "handle.cuh"

namespace pb
{

namespace
{

// Programmatic dependent launch on the step graph's main branch (corrected-cell stencil ->
// finish -> near -> next stencil): the dependent grid is scheduled while its predecessor's last
// blocks drain, and waits here, before its first read, until the predecessor has completed and
// its writes are visible.  Launched without the attribute, the wait returns at once.
__device__ inline void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
void launch_dependent(void (*kern)(KArgs...), int grid, int block, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, ((KArgs)args)...);
}

// The values of a scene that every step kernel reads (the per-step ones come from StepState)
struct StepArgs
{
    int res;
    double lap_coef;     // (c dt)^2 in double, reference arithmetic
    double hd;           // h in double
    double h2, rh2;      // h^2 in double and its correctly rounded reciprocal (leapfrog)
    float c, dt, h;
    int pml_width;
    float damp;
    int nt;
    int n_listen;
    int listen_cell[8];
    int *status;  // the handle's step status word: kStepNonFinite once a listener sample is not finite
};

// bit of the step status word: a non-finite Dirichlet value or listener sample appeared
constexpr int kStepNonFinite = 1;

template <typename R>
__device__ inline void flag_nonfinite(int *status, R v)
{
    if (status && !isfinite(v))
        atomicOr(status, kStepNonFinite);
}


// History rings in the step.  The reference keeps per triangle a ring of 32 values indexed by
// time mod 32 and reads the 16 taps t, t-1, ..., t-15 (bem.h:55).  Those rings (the canonical
// rings, reference layout) are kept current by every history write and serve read-out, loading
// and the Neumann value of a step without an acceleration row (the value 32 steps old, as the
// reference's ring holds it).  The taps are read from four copies of 16 slots instead: copy c
// holds time tau at slot (c - tau) mod 16, so taps 4q..4q+3 of time t sit at slots
// (c - t + 4q) .. +3 of copy c, ascending with the tap, and for c = t mod 4 they start on a
// multiple of 4.  A copy's row interleaves the two fields by 4-tap chunks: chunk j holds Neumann
// slots 4j..4j+3 then Dirichlet slots 4j..4j+3, so the Neumann and Dirichlet taps 4q..4q+3 of a
// triangle are one aligned 32-byte load (FP32) and a triangle's whole window is one 128-byte
// line.  A new value is written into all four copies and the canonical ring.
__host__ __device__ inline int hist_index(int copy, int time) { return (copy - time) & (kHist - 1); }

// the three grid time levels (and PML fields) by time index, the history copies
// [copy 0..3][nt][kHistRow] and the canonical rings [nt][kRing] of both fields
template <typename R>
struct Ring
{
    R *g[3];
    R *p[3];
    R *hist;
    R *canon[2];  // field 0 = Neumann, 1 = Dirichlet
    int nt;
    __device__ R *slot(int time) const { return g[((time % 3) + 3) % 3]; }
    __device__ R *pml(int time) const { return p[((time % 3) + 3) % 3]; }
    __device__ R *hrow(int copy, int tri) const { return hist + ((long long)copy * nt + tri) * kHistRow; }
    // position of slot s of a field inside a copy's row
    __device__ static int hpos(int field, int s) { return ((s >> 2) << 3) + (field << 2) + (s & 3); }
    __device__ R &hat(int field, int copy, int tri, int s) const { return hrow(copy, tri)[hpos(field, s)]; }
    __device__ R &canon_at(int field, int tri, int time) const
    {
        return canon[field][(long long)tri * kRing + (time & (kRing - 1))];
    }
    __device__ void hwrite(int field, int tri, int time, R v) const
    {
#pragma unroll
        for (int c = 0; c < 4; c++)
            hat(field, c, tri, hist_index(c, time)) = v;
        canon_at(field, tri, time) = v;
    }
    // N[time] of triangle tri: the acceleration row's value, or without one the value the
    // canonical ring holds for that slot (written 32 steps before, as the reference's ring)
    __device__ void nwrite(int tri, int time, const float *acc) const
    {
        hwrite(0, tri, time, acc ? (R)acc[tri] : canon_at(0, tri, time));
    }
    // N[time + 1] of triangle tri into the Dirichlet slot of `time` in copy time mod 4: that slot
    // is tap 0 of the Dirichlet window of `time` (the step's unknown, which no reader of the
    // window uses; finish of that step overwrites it with D[time]), so a two-step pass over the
    // face pairs at `time` receives N[time + 1] with the window (face_conv2).  acc_next: the
    // acceleration row of time + 1, or none.
    __device__ void stash_next(int tri, int time, const float *acc_next) const
    {
        hat(1, time & 3, tri, hist_index(time & 3, time)) = acc_next ? (R)acc_next[tri] : canon_at(0, tri, time + 1);
    }
};

template <typename Real>
__device__ inline Real ld(const Real *g, int res, int x, int y, int z)
{
    return g[((long long)x * res + y) * res + z];
}

// Absorbing boundary at a layer-1 / layer-(res-2) cell (fdtd.cu:88-137): unknowns are the
// ghost values on the outside of each boundary axis (time t) and p^{t+1} of the cell.
template <typename R>
__device__ inline R abc_cell(R *cur, const R *prev, int res, int x, int y, int z, R c, R dt, R h)
{
    int cc[3] = {x, y, z};
    int judge[3];
#pragma unroll
    for (int d = 0; d < 3; d++)
        judge[d] = -((int)(cc[d] == 1)) + ((int)(cc[d] == res - 2));
    auto at = [&](const R *g, int d, int s) {
        int q[3] = {x, y, z};
        q[d] += s;
        return g[((long long)q[0] * res + q[1]) * res + q[2]];
    };
    const R pc = cur[((long long)x * res + y) * res + z];
    const R pp = prev[((long long)x * res + y) * res + z];
    R a[4][4], b[4];
    R coef = c * c * dt * dt / (h * h);
    a[3][3] = 1;
#pragma unroll
    for (int d = 0; d < 3; d++)
        a[3][d] = -coef * (judge[d] != 0);
    b[3] = -pp + 2 * pc - coef * (6 * pc);
#pragma unroll
    for (int d = 0; d < 3; d++)
        b[3] += coef * at(cur, d, 1) * (judge[d] <= 0) + coef * at(cur, d, -1) * (judge[d] >= 0);
    R coef1 = 1 / (dt * dt), coef2 = c / (2 * h * dt), coef3 = -(c * c) / (2 * h * h);
#pragma unroll
    for (int idx = 0; idx < 3; idx++)
    {
        int ax = idx, ay = (idx + 1) % 3, az = (idx + 2) % 3;
        a[idx][3] = coef1;
        a[idx][ax] = coef2;
        a[idx][ay] = coef3 * (judge[ay] != 0);
        a[idx][az] = coef3 * (judge[az] != 0);
        b[idx] = -coef1 * (pp - 2 * pc) +
                 -coef2 * (at(cur, ax, 1) * (-(judge[ax] < 0)) + at(cur, ax, -1) * (-(judge[ax] > 0)) +
                           at(prev, ax, 1) * (-judge[ax]) + at(prev, ax, -1) * judge[ax]) +
                 -coef3 * (at(cur, ay, 1) * (judge[ay] <= 0) + at(cur, ay, -1) * (judge[ay] >= 0) +
                           at(cur, az, 1) * (judge[az] <= 0) + at(cur, az, -1) * (judge[az] >= 0) - 4 * pc);
    }
    R res4[4];
    solve4<R>(a, b, res4);
#pragma unroll
    for (int d = 0; d < 3; d++)
        if (judge[d] != 0)
        {
            int q[3] = {x, y, z};
            q[d] += judge[d];
            cur[((long long)q[0] * res + q[1]) * res + q[2]] = res4[d];
        }
    return res4[3];
}

// interior leapfrog (fdtd.cu:7-33): float storage, double arithmetic, "6 * p" in the
// storage precision; the neighbours summed in the reference's order (x-1, x+1, y-1, y+1, z-1, z+1).
// The division by h^2 is Markstein's correction of a product with the correctly rounded
// reciprocal (P. Markstein, IBM J. Res. Dev. 34(1), 1990: with r = RN(1/d), q = RN(a r) and the
// exact remainder a - d q from an FMA, RN(q + (a - d q) r) = RN(a / d)), so the quotient is the
// one the reference's division rounds to, without a division per cell.
template <typename R>
__device__ inline R leapfrog(R pc, R xm, R xp, R ym, R yp, R zm, R zp, R pprev, double coefd, double h2, double rh2)
{
    double sum = 0;
    sum += xm;
    sum += xp;
    sum += ym;
    sum += yp;
    sum += zm;
    sum += zp;
    sum -= 6 * pc;
    const double q = sum * rh2;
    const double lap = fma(fma(-q, h2, sum), rh2, q);
    double p = 2 * pc;
    p += coefd * lap;
    p += -pprev;
    return (R)p;
}

// Work split of the stencil launch into three block ranges so no warp mixes the short
// interior update with the long boundary solve; the boundary blocks come first, so they are
// scheduled first and their long solves overlap the interior blocks instead of trailing them:
//   [0, nb_bd)              boundary-layer cells (a coordinate equal to 1 or res-2), 256 per block
//   [nb_bd, nb_bd + nb_in)  interior cells [2, res-3]^3.  FP32 fields with res a multiple of 4
//                           (vec4): one thread per group of four consecutive z of an interior
//                           (x, y) row, 16-byte loads (stencil_interior4).  Otherwise by x plane: a
//                           block covers zlen (a power of two, at most 256) consecutive z of
//                           256 / zlen consecutive y rows, so threads find their cell without a
//                           division
//   the rest                Neumann ring write, one thread per triangle
// skip_corrected: the bulk of a split step (corrected cells are left to stencil_corr_kernel).
// The tiles of a plane are counted in powers of two (blocks past the last tile exit at once), so a
// block finds its plane and tile by shifts.
struct StencilSplit
{
    int nb_in, nb_bd, nb_nt;
    int zlog;              // log2 of the threads along z of an interior block
    int ytlog, ztlog;      // log2 of the interior blocks per x plane along y and along z
    int skip_corrected;
    int vec4;              // interior in groups of four z (FP32, res % 4 == 0): res / 4 groups per row
};

inline int ceil_log2(long long v)
{
    int l = 0;
    while ((1ll << l) < v)
        l++;
    return l;
}

// vec4: 1 four interior cells per thread where the layout allows it (FP32, res % 4 == 0), 0 one
// cell per thread, -1 four from res 96 up (measured: at res 64 the bulk launch is bound by the
// boundary layer's solves and the scalar interior finishes first; at res 128 the vector interior
// halves the bulk).  The autotuner times both.
inline StencilSplit stencil_split(int res, int nt, bool fp32, int vec4)
{
    long long mi = res - 4, m = res - 2;
    long long n_bd = 2 * m * m + 2 * (m - 2) * m + 2 * (m - 2) * (m - 2);
    StencilSplit sp{};
    sp.zlog = std::min(std::max(ceil_log2(mi), 5), 8);
    sp.ztlog = ceil_log2(div_up(mi, 1 << sp.zlog));
    sp.ytlog = ceil_log2(div_up(mi, 256 >> sp.zlog));
    sp.nb_in = (int)(mi << (sp.ytlog + sp.ztlog));
    if (fp32 && res % 4 == 0 && (vec4 > 0 || (vec4 < 0 && res >= 96)))
    {
        sp.vec4 = res / 4;
        sp.nb_in = (int)div_up(mi * mi * sp.vec4, 256);
    }
    sp.nb_bd = div_up(n_bd, 256);
    sp.nb_nt = div_up(nt, 256);
    sp.skip_corrected = 0;
    return sp;
}

__device__ inline bool is_corrected(const unsigned *corr_mask, long long c)
{
    return (corr_mask[c >> 5] >> (c & 31)) & 1u;
}

template <typename R>
__device__ inline void finish_cell(const StepArgs &a, long long row, long long c, R v, R *next, bool corrected,
                                   R *series)
{
    if (corrected)
    {
        R corr = next[c];
        v = v - corr;
    }
    next[c] = v;
    // a listener at a corrected cell is recorded by the near stage, after its correction
    if (!corrected)
        for (int l = 0; l < a.n_listen; l++)
            if (a.listen_cell[l] == (int)c)
            {
                series[row * a.n_listen + l] = v;
                flag_nonfinite(a.status, v);
            }
}

// the stencil at interior cell (x, y, z)
template <typename R>
__device__ inline R interior_cell(const StepArgs &a, const R *__restrict__ cur, const R *__restrict__ prev,
                                  long long c)
{
    const int res = a.res;
    const long long sx = (long long)res * res;
    return leapfrog<R>(cur[c], cur[c - sx], cur[c + sx], cur[c - res], cur[c + res], cur[c - 1], cur[c + 1], prev[c],
                       a.lap_coef, a.h2, a.rh2);
}

// Interior cells four at a time along z (FP32 fields, res a multiple of 4, so every group of four
// starts on a 16-byte boundary): thread t of the interior range takes z-group g = t mod (res/4) of
// interior row t div (res/4) (x, y in [2, res-3]).  It loads the group, its four x / y neighbour
// groups and p^{t-2} as 16-byte vectors and the two z halo values singly, and computes each interior
// cell of the group with the scalar leapfrog (same arithmetic: fields bit-identical).  A group of
// four interior cells with no corrected cell and no listener is stored as one vector; any other
// group goes cell by cell through finish_cell.
__device__ inline void stencil_interior4(const StepArgs &a, const float *__restrict__ cur,
                                         const float *__restrict__ prev, float *next, long long srow, int b,
                                         const StencilSplit &sp, const unsigned *corr_mask, float *series)
{
    const int res = a.res, mi = res - 4, G = sp.vec4;
    const long long t = (long long)b * 256 + threadIdx.x;
    const long long row = t / G;
    if (row >= (long long)mi * mi)
        return;
    const int g = (int)(t - row * G);
    const int x = 2 + (int)(row / mi), y = 2 + (int)(row % mi), z0 = 4 * g;
    const long long sx = (long long)res * res;
    const long long c0 = ((long long)x * res + y) * res + z0;
    const float4 cc = *(const float4 *)(cur + c0);
    const float4 xm = *(const float4 *)(cur + c0 - sx), xp = *(const float4 *)(cur + c0 + sx);
    const float4 ym = *(const float4 *)(cur + c0 - res), yp = *(const float4 *)(cur + c0 + res);
    const float4 pp = *(const float4 *)(prev + c0);
    // z - 1 of the group's first cell (read when that cell is interior: g >= 1) and z + 1 of its last
    // (read when interior: g <= res/4 - 2)
    const float zlo = g > 0 ? cur[c0 - 1] : 0.0f, zhi = g < G - 1 ? cur[c0 + 4] : 0.0f;
    const float c[6] = {zlo, cc.x, cc.y, cc.z, cc.w, zhi};
    const float vxm[4] = {xm.x, xm.y, xm.z, xm.w}, vxp[4] = {xp.x, xp.y, xp.z, xp.w};
    const float vym[4] = {ym.x, ym.y, ym.z, ym.w}, vyp[4] = {yp.x, yp.y, yp.z, yp.w};
    const float vp[4] = {pp.x, pp.y, pp.z, pp.w};
    const unsigned bits = (corr_mask[c0 >> 5] >> (c0 & 31)) & 0xfu;  // c0 % 4 == 0: one word
    bool listen = false;
    for (int l = 0; l < a.n_listen; l++)
        listen |= a.listen_cell[l] >= c0 && a.listen_cell[l] < c0 + 4;
    float v[4];
    int inside = 0;
#pragma unroll
    for (int u = 0; u < 4; u++)
    {
        v[u] = 0.0f;
        if (z0 + u >= 2 && z0 + u <= res - 3)
        {
            inside |= 1 << u;
            v[u] = leapfrog<float>(c[u + 1], vxm[u], vxp[u], vym[u], vyp[u], c[u], c[u + 2], vp[u], a.lap_coef, a.h2,
                                   a.rh2);
        }
    }
    if (inside == 0xf && !bits && !listen)
    {
        *(float4 *)(next + c0) = make_float4(v[0], v[1], v[2], v[3]);
        return;
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
        if ((inside >> u) & 1)
        {
            const bool corrected = (bits >> u) & 1u;
            if (sp.skip_corrected && corrected)
                continue;
            finish_cell<float>(a, srow, c0 + u, v[u], next, corrected, series);
        }
}

// the stencil work of block b of one scene's stencil grid (256 threads)
template <typename R>
__device__ inline void stencil_body(const StepArgs &a, const Ring<R> &ring, const StepDyn &dy, int b, StencilSplit sp,
                                    const unsigned *corr_mask)
{
    R *series = (R *)dy.series;
    R *cur = ring.slot(dy.tnew - 1), *next = ring.slot(dy.tnew);
    const R *prev = ring.slot(dy.tnew - 2);
    const int res = a.res;
    if (b < sp.nb_bd)
    {
        const int m = res - 2;
        int i = b * 256 + threadIdx.x;
        if (i >= 2 * m * m + 2 * (m - 2) * m + 2 * (m - 2) * (m - 2))
            return;
        int x, y, z;
        boundary_cell(i, res, x, y, z);
        const long long c = ((long long)x * res + y) * res + z;
        const bool corrected = is_corrected(corr_mask, c);
        if (sp.skip_corrected && corrected)
            return;
        R v = abc_cell<R>(cur, prev, res, x, y, z, (R)a.c, (R)a.dt, (R)a.h);
        finish_cell<R>(a, dy.row, c, v, next, corrected, series);
        return;
    }
    b -= sp.nb_bd;
    if (b < sp.nb_in)
    {
        if constexpr (sizeof(R) == 4)
            if (sp.vec4)
            {
                stencil_interior4(a, cur, prev, next, dy.row, b, sp, corr_mask, series);
                return;
            }
        const int mi = res - 4;
        const int plane = b >> (sp.ytlog + sp.ztlog), r = b & ((1 << (sp.ytlog + sp.ztlog)) - 1);
        const int yt = r >> sp.ztlog, zt = r & ((1 << sp.ztlog) - 1);
        const int z = 2 + (zt << sp.zlog) + (threadIdx.x & ((1 << sp.zlog) - 1));
        const int y = 2 + (yt << (8 - sp.zlog)) + (threadIdx.x >> sp.zlog);
        if (z >= 2 + mi || y >= 2 + mi)
            return;
        const long long c = ((long long)(2 + plane) * res + y) * res + z;
        const bool corrected = is_corrected(corr_mask, c);
        if (sp.skip_corrected && corrected)
            return;
        finish_cell<R>(a, dy.row, c, interior_cell<R>(a, cur, prev, c), next, corrected, series);
        return;
    }
    b -= sp.nb_in;
    int i = b * 256 + threadIdx.x;
    if (i < a.nt)
        ring.nwrite(i, dy.tnew, dy.acc);
}

template <typename R>
__global__ void __launch_bounds__(256) stencil_kernel(const __grid_constant__ StepArgs a0,
                                                       const __grid_constant__ Ring<R> ring, const StepState *st, int k,
                                                       StencilSplit sp, const unsigned *corr_mask)
{
    stencil_body<R>(a0, ring, bind_step(st, k, a0.nt), blockIdx.x, sp, corr_mask);
}

// The stencil at the corrected cells only (the split step's critical branch: the face stage reads
// the far field at the triangles' trilinear corners, which all lie in the 3^3 blocks of the
// triangles' cells, i.e. at corrected cells).  Threads stride over the corrected-cell list (its
// length is read from the step state); the arithmetic per cell is that of stencil_body.
template <typename R>
__device__ inline void stencil_corr_body(const StepArgs &a0, const Ring<R> &ring, const StepState *st, int k,
                                         const int *n3_cell, int first, int stride)
{
    const StepDyn dy = bind_step(st, k, a0.nt);
    R *cur = ring.slot(dy.tnew - 1), *next = ring.slot(dy.tnew);
    const R *prev = ring.slot(dy.tnew - 2);
    const int res = a0.res, n3 = st->n3;
    for (int ci = first; ci < n3; ci += stride)
    {
        const int c = n3_cell[ci];
        const int x = c / (res * res), y = (c / res) % res, z = c % res;
        R v;
        if (x == 1 || x == res - 2 || y == 1 || y == res - 2 || z == 1 || z == res - 2)
            v = abc_cell<R>(cur, prev, res, x, y, z, (R)a0.c, (R)a0.dt, (R)a0.h);
        else if (x >= 2 && x < res - 2 && y >= 2 && y < res - 2 && z >= 2 && z < res - 2)
            v = interior_cell<R>(a0, cur, prev, c);
        else
            continue;  // the ghost layer holds no unknown of the stencil
        next[c] = v - next[c];  // the FDTD-near correction the near stage left in this slot
    }
}

template <typename R>
__global__ void __launch_bounds__(256) stencil_corr_kernel(const __grid_constant__ StepArgs a0,
                                                            const __grid_constant__ Ring<R> ring, const StepState *st,
                                                            int k, const int *n3_cell)
{
    grid_dependency_wait();
    stencil_corr_body<R>(a0, ring, st, k, n3_cell, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// split-field PML (fdtd.cu:162-232) on [1, res-2]^3; pml slots hold 6 values per cell
template <typename R>
__device__ inline R pml_damp(int x, int y, int z, int res, int w, R damp)
{
    return (x < w || x >= res - w || y < w || y >= res - w || z < w || z >= res - w) ? damp : (R)0;
}

template <typename R>
__global__ void __launch_bounds__(256) pml_kernel(const __grid_constant__ StepArgs a0, const __grid_constant__ Ring<R> ring, const StepState *st, int k,
                                                   const unsigned *corr_mask)
{
    const StepArgs &a = a0;
    const StepDyn dy = bind_step(st, k, a0.nt);
    R *series = (R *)dy.series;
    const R *cur = ring.slot(dy.tnew - 1), *prev = ring.slot(dy.tnew - 2);
    R *next = ring.slot(dy.tnew);
    const R *pcur = ring.pml(dy.tnew - 1);
    R *pnext = ring.pml(dy.tnew);
    long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int res = a.res, m = res - 2, w = a.pml_width;
    if (gid < a.nt)
        ring.nwrite((int)gid, dy.tnew, dy.acc);
    if (gid >= (long long)m * m * m)
        return;
    int q[3] = {1 + (int)(gid / ((long long)m * m)), 1 + (int)((gid / m) % m), 1 + (int)(gid % m)};
    const R c = a.c, h = a.h, dt = a.dt, damp = a.damp;
    auto idx = [&](int x, int y, int z) { return ((long long)x * res + y) * res + z; };
    long long ci = idx(q[0], q[1], q[2]);
    int sgn[3];
#pragma unroll
    for (int d = 0; d < 3; d++)
        sgn[d] = q[d] > res / 2 ? 1 : -1;
    R cd = pml_damp<R>(q[0], q[1], q[2], res, w, damp);
    R rhs = 0;
#pragma unroll
    for (int d = 0; d < 3; d++)
    {
        int p1[3] = {q[0], q[1], q[2]}, m1[3] = {q[0], q[1], q[2]}, ps[3] = {q[0], q[1], q[2]}, ms[3] = {q[0], q[1], q[2]};
        p1[d] += 1;
        m1[d] -= 1;
        ps[d] += sgn[d];
        ms[d] -= sgn[d];
        rhs += 1 / (h * h) * (cur[idx(p1[0], p1[1], p1[2])] - 2 * cur[ci] + cur[idx(m1[0], m1[1], m1[2])]);
        rhs += 1 / h *
               (cd * pcur[6 * idx(ps[0], ps[1], ps[2]) + 3 + d] -
                pml_damp<R>(ms[0], ms[1], ms[2], res, w, damp) * pcur[6 * idx(ms[0], ms[1], ms[2]) + d]);
    }
    R v = cur[ci] * 2 - prev[ci] + c * c * dt * dt * rhs;
    if (cd != 0)
    {
#pragma unroll
        for (int d = 0; d < 3; d++)
        {
            int ps[3] = {q[0], q[1], q[2]}, ms[3] = {q[0], q[1], q[2]};
            ps[d] += sgn[d];
            ms[d] -= sgn[d];
            R dm = pml_damp<R>(ms[0], ms[1], ms[2], res, w, damp);
            R grad = cur[idx(ps[0], ps[1], ps[2])] - cur[idx(ms[0], ms[1], ms[2])];
            R r1 = 0;
            r1 += -1.0f / 2.0f * (dm * pcur[6 * idx(ms[0], ms[1], ms[2]) + d] + cd * pcur[6 * ci + d]);
            r1 += -1.0f / (h * 2.0f) * grad;
            pnext[6 * ci + d] = pcur[6 * ci + d] + c * dt * r1;
            R r2 = 0;
            r2 += -1.0f / 2.0f * (dm * pcur[6 * ci + 3 + d] + cd * pcur[6 * idx(ps[0], ps[1], ps[2]) + 3 + d]);
            r2 += -1.0f / (h * 2.0f) * grad;
            pnext[6 * ci + 3 + d] = pcur[6 * ci + 3 + d] + c * dt * r2;
        }
    }
    const bool corrected = (corr_mask[ci >> 5] >> (ci & 31)) & 1u;
    if (corrected)
        v = v - next[ci];
    next[ci] = v;
    if (!corrected)
        for (int l = 0; l < a.n_listen; l++)
            if (a.listen_cell[l] == (int)ci)
            {
                series[dy.row * a.n_listen + l] = v;
                flag_nonfinite(a.status, v);
            }
}

// ---- convolution helpers
// A pair is handled by a quad of 4 lanes: lane q takes taps 4q..4q+3 with one 16-byte load of
// the pair's weights (4 fp16 (single, double) tap pairs) and one load of the neighbour's Neumann
// and Dirichlet taps 4q..4q+3 from the history copy in which they are aligned at this time step
// (load_window); the 8 quads of a warp take pairs g, g + 8, ...  Each lane sums its
// taps in increasing pair and tap order; the warp reduces once per triangle / cell.
__device__ inline float conv_tap(__half2 w, float2 s, float n, float d)
{
    return -__low2float(w) * s.x * n + __high2float(w) * s.y * d;
}
__device__ inline double conv_tap(double2 w, float2, double n, double d) { return -w.x * n + w.y * d; }

template <typename T, int N>
struct alignas(16) Vec
{
    T v[N];
};

template <typename R>
struct WRec;
template <>
struct WRec<float>
{
    using T = __half2;
    using W4 = Vec<__half2, 4>;
    using H4 = Vec<float, 4>;
};
template <>
struct WRec<double>
{
    using T = double2;
    using W4 = Vec<double2, 4>;
    using H4 = Vec<double, 4>;
};

// Taps 4q..4q+3 of time t of both fields of one triangle: chunk (slot of tap 0) / 4 + q of copy
// t mod 4, which starts 8 values into the row per chunk.  FP32: one 32-byte load (PTX
// ld.global.v8.f32, sm_100), so a quad reads a triangle's two windows as one 128-byte line.  The
// asm is ordered against the kernel's own history writes (memory clobber).
__device__ inline int window_offset(int t, int q) { return (((hist_index(t & 3, t) >> 2) + q) & 3) << 3; }

__device__ inline void load_window(const float *p, Vec<float, 4> &n, Vec<float, 4> &d)
{
    asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(n.v[0]), "=f"(n.v[1]), "=f"(n.v[2]), "=f"(n.v[3]), "=f"(d.v[0]), "=f"(d.v[1]), "=f"(d.v[2]),
                   "=f"(d.v[3])
                 : "l"(p)
                 : "memory");
}
__device__ inline void load_window(const double *p, Vec<double, 4> &n, Vec<double, 4> &d)
{
    n = *(const Vec<double, 4> *)p;
    d = *(const Vec<double, 4> *)(p + 4);
}

constexpr unsigned kFull = 0xffffffffu;

template <typename R>
__device__ inline R warp_sum(R v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_xor_sync(kFull, v, off);
    return v;
}

// face stage: one warp per centre triangle.  The 8 far-field corner terms are fetched first
// (lanes 0-7) so their latency overlaps the convolution.
// the face-stage work of one scene's centre triangle tri (whole warp)
template <typename R>
struct FaceArgs
{
    const int *face_start, *face_nbr, *face_corner;
    const typename WRec<R>::T *face_w;
    const float2 *face_scale;
    const R *face_d1;  // per pair: double-layer tap 1 with its scale (fix_kernel)
    const int *order;  // centre triangles in base-cell order (the convolution kernels' warp order)
    R *dlast;          // per triangle: the Dirichlet value of the last finished step
    const float *interp;
    const double *interp_d, *denom;
    float reflect;
    // near-field terms of every triangle (see near_terms): its 54 grid-cache records
    const typename WRec<R>::T *gc_w;
    const float2 *gc_scale;
    R *terms;  // [nt][54]
    R *terms1;        // [nt][54] partial terms of the next step (near_terms2)
    const R *gc_f;    // [nt][54] factor of the next step's Dirichlet value per record (near_terms2)
    int *status;      // step status word (kStepNonFinite)
};

constexpr int kGcRecords = 54;  // per triangle: 27 FDTD-near then 27 BEM-near records (offsets in 3^3)

// The near-field terms of one triangle at time t (whole warp): for each of its 54 grid-cache
// records (27 offsets x {FDTD-near, BEM-near}) the record's convolution with the triangle's OWN
// history window, terms[tri][r].  A corrected cell's two sums are then plain sums of these terms
// over its 3^3 list (near_gather_body): each triangle's history is read once per step instead of
// once per corrected cell around it, and the records stream contiguously.  The FDTD-near terms
// belong to the next step: record tap k + 1 pairs with history tap k (taps t..t-14).  Lane q of
// quad g takes taps 4q..4q+3 of records g, g + 8, ...; d0 != 0 replaces Dirichlet tap 0 (time t)
// with dnew, the value this warp has just computed.
template <typename R>
__device__ inline void near_terms(const Ring<R> &ring, int t, const FaceArgs<R> &f, int tri, int lane, bool d0,
                                  R dnew)
{
    using W4 = typename WRec<R>::W4;
    using H4 = typename WRec<R>::H4;
    const int g = lane >> 2, q = lane & 3;
    H4 hn, hd;
    load_window(ring.hrow(t & 3, tri) + window_offset(t, q), hn, hd);
    if (d0 && q == 0)
        hd.v[0] = dnew;
    // history taps 4q-1 .. 4q+2 for the shifted FDTD-near records (tap -1 does not exist: 0)
    H4 sn, sd;
    const R pn = __shfl_up_sync(kFull, hn.v[3], 1), pd = __shfl_up_sync(kFull, hd.v[3], 1);
    sn.v[0] = q ? pn : (R)0;
    sd.v[0] = q ? pd : (R)0;
#pragma unroll
    for (int i = 1; i < 4; i++)
    {
        sn.v[i] = hn.v[i - 1];
        sd.v[i] = hd.v[i - 1];
    }
    const unsigned quad = 0xfu << (lane & ~3);
    const typename WRec<R>::T *rec = f.gc_w + (long long)tri * kGcRecords * kTaps;
    R *out = f.terms + (long long)tri * kGcRecords;
    for (int r = g; r < kGcRecords; r += 8)
    {
        const W4 w = *(const W4 *)(rec + (long long)r * kTaps + 4 * q);
        const float2 s = f.gc_scale ? f.gc_scale[(long long)tri * kGcRecords + r] : make_float2(1, 1);
        R v = 0;
        if (r < kGcRecords / 2)
        {
#pragma unroll
            for (int i = 0; i < 4; i++)
                v += conv_tap(w.v[i], s, sn.v[i], sd.v[i]);
        }
        else
        {
#pragma unroll
            for (int i = 0; i < 4; i++)
                v += conv_tap(w.v[i], s, hn.v[i], hd.v[i]);
        }
        v += __shfl_xor_sync(quad, v, 1);
        v += __shfl_xor_sync(quad, v, 2);
        if (q == 0)
            out[r] = v;
    }
}

// The near-field terms of time t (as near_terms with d0 set) and, from the same pass over the
// 54 records, the terms of time t+1 without the one product that needs D[t+1], which this step
// cannot know yet: BEM-near records pair record tap m with history tap m of time t+1 (tap 0 holds
// D[t+1]); FDTD-near records pair record tap m with history tap m-1 (record tap 1 meets D[t+1]).
// History tap j of time t+1 is tap j-1 of time t, so the time-(t+1) windows are the time-t window
// shifted by one and two taps (quad shuffles); tap -1 is N[t+1] = nnext (known: the acceleration
// row of the next step) and D[t+1] (left out).  face_finish of the next step adds
// gc_f[r] * D[t+1] to terms1[r] (gc_factors holds those factors).
template <typename R>
__device__ inline void near_terms2(const Ring<R> &ring, int t, const FaceArgs<R> &f, int tri, int lane, R dnew,
                                   R nnext)
{
    using W4 = typename WRec<R>::W4;
    using H4 = typename WRec<R>::H4;
    const int g = lane >> 2, q = lane & 3;
    H4 hn, hd;
    load_window(ring.hrow(t & 3, tri) + window_offset(t, q), hn, hd);
    if (q == 0)
        hd.v[0] = dnew;
    // time-t taps shifted by one (4q+i-1) and by two (4q+i-2)
    const R pn3 = __shfl_up_sync(kFull, hn.v[3], 1), pd3 = __shfl_up_sync(kFull, hd.v[3], 1);
    const R pn2 = __shfl_up_sync(kFull, hn.v[2], 1), pd2 = __shfl_up_sync(kFull, hd.v[2], 1);
    H4 sn, sd, bn, tn, td;
    sn.v[0] = q ? pn3 : (R)0;   // FDTD-near, time t: tap -1 does not exist
    bn.v[0] = q ? pn3 : nnext;  // BEM-near, time t+1: tap 0 of t+1 is N[t+1]
    sd.v[0] = q ? pd3 : (R)0;   // D: tap -1 is D[t+1], left out in both
#pragma unroll
    for (int i = 1; i < 4; i++)
    {
        sn.v[i] = hn.v[i - 1];
        bn.v[i] = hn.v[i - 1];
        sd.v[i] = hd.v[i - 1];
    }
    // FDTD-near, time t+1: record tap m pairs with time-t tap m-2; m = 0 has no term, m = 1 meets
    // time t+1 (N[t+1] included, D[t+1] left out)
    tn.v[0] = q ? pn2 : (R)0;
    td.v[0] = q ? pd2 : (R)0;
    tn.v[1] = q ? pn3 : nnext;
    td.v[1] = q ? pd3 : (R)0;
    tn.v[2] = hn.v[0];
    td.v[2] = hd.v[0];
    tn.v[3] = hn.v[1];
    td.v[3] = hd.v[1];
    const unsigned quad = 0xfu << (lane & ~3);
    const typename WRec<R>::T *rec = f.gc_w + (long long)tri * kGcRecords * kTaps;
    R *out = f.terms + (long long)tri * kGcRecords;
    R *out1 = f.terms1 + (long long)tri * kGcRecords;
    for (int r = g; r < kGcRecords; r += 8)
    {
        const W4 w = *(const W4 *)(rec + (long long)r * kTaps + 4 * q);
        const float2 s = f.gc_scale ? f.gc_scale[(long long)tri * kGcRecords + r] : make_float2(1, 1);
        R v = 0, v1 = 0;
        if (r < kGcRecords / 2)
        {
#pragma unroll
            for (int i = 0; i < 4; i++)
            {
                v += conv_tap(w.v[i], s, sn.v[i], sd.v[i]);
                v1 += conv_tap(w.v[i], s, tn.v[i], td.v[i]);
            }
        }
        else
        {
#pragma unroll
            for (int i = 0; i < 4; i++)
            {
                v += conv_tap(w.v[i], s, hn.v[i], hd.v[i]);
                v1 += conv_tap(w.v[i], s, bn.v[i], sd.v[i]);
            }
        }
        v += __shfl_xor_sync(quad, v, 1);
        v += __shfl_xor_sync(quad, v, 2);
        v1 += __shfl_xor_sync(quad, v1, 1);
        v1 += __shfl_xor_sync(quad, v1, 2);
        if (q == 0)
        {
            out[r] = v;
            out1[r] = v1;
        }
    }
}

// the second step of a two-step pass: its near-field terms from the partial terms and the new
// Dirichlet value
template <typename R>
__device__ inline void near_terms_complete(const FaceArgs<R> &f, int tri, int lane, R dnew)
{
    const long long o = (long long)tri * kGcRecords;
    for (int r = lane; r < kGcRecords; r += 32)
        f.terms[o + r] = f.terms1[o + r] + f.gc_f[o + r] * dnew;
}

// The face stage of centre triangle tri (whole warp) in two parts.  face_conv: the face-pair
// convolution over the triangle's 4^3 list -> its warp sum.  It reads only history that is final
// before the step begins (Neumann taps t..t-15 with N[t] = acc[t] already in the ring, Dirichlet
// taps t-1..t-15), so the pipelined step graph runs it beside the stencil.  face_finish: the far
// field at the 8 trilinear corners (from this step's stencil output), the Dirichlet update and the
// triangle's near-field terms.  Fused or split, the arithmetic and its order are the same.
template <typename R>
__device__ inline R face_conv(const Ring<R> &ring, int tnew, const FaceArgs<R> &f, int tri, int lane)
{
    using W4 = typename WRec<R>::W4;
    using H4 = typename WRec<R>::H4;
    const int g = lane >> 2, q = lane & 3;
    const R *base = ring.hrow(tnew & 3, 0) + window_offset(tnew, q);
    const int b = f.face_start[tri], e = f.face_start[tri + 1];
    R acc = 0;
    for (int p = b + g; p < e; p += 8)
    {
        const W4 w = *(const W4 *)(f.face_w + (long long)p * kTaps + 4 * q);
        const float2 s = f.face_scale ? f.face_scale[p] : make_float2(1, 1);
        const int nb = f.face_nbr[p];
        H4 hn, hd;
        load_window(base + (long long)nb * kHistRow, hn, hd);
#pragma unroll
        for (int i = 0; i < 4; i++)
        {
            // tap 0 of the Dirichlet history is this step's unknown: left out
            R di = (q == 0 && i == 0) ? (R)0 : hd.v[i];
            acc += conv_tap(w.v[i], s, hn.v[i], di);
        }
    }
    return warp_sum(acc);
}

// Two steps from one pass over the face pairs.  c0: step k's convolution, exactly as face_conv
// (same loads, same per-lane order).  c1: step k+1's convolution without its one term that needs
// a value of step k: Dirichlet tap 1 of time t+1 is D[t], which finish(k) computes; fix_kernel
// adds that term, sum_j d1_j D_j[t].  Everything else of step k+1 is final before step k:
// Neumann taps t+1..t-14 (N[t+1] = acc[k+1], read from the acceleration row since the ring
// receives it only in finish(k)) and Dirichlet taps t-1..t-14.  Tap 4q+i of time t+1 is tap
// 4q+i-1 of time t, so lane q's shifted window is its own taps 4q..4q+2 plus tap 4q-1 from the
// lane before it in the quad (tap -1: N[t+1]; for D, taps 0 and 1 of time t+1 are left out).
// The face weights, scales and neighbour indices are read once for both steps.
template <typename R>
__device__ inline void face_conv2(const Ring<R> &ring, int tnew, const FaceArgs<R> &f, int tri, int lane, R &c0,
                                  R &c1)
{
    using W4 = typename WRec<R>::W4;
    using H4 = typename WRec<R>::H4;
    const int g = lane >> 2, q = lane & 3;
    const R *base = ring.hrow(tnew & 3, 0) + window_offset(tnew, q);
    const unsigned quad = 0xfu << (lane & ~3);
    const int b = f.face_start[tri], e = f.face_start[tri + 1];
    R a0 = 0, a1 = 0;
    for (int p = b + g; p < e; p += 8)
    {
        const W4 w = *(const W4 *)(f.face_w + (long long)p * kTaps + 4 * q);
        const float2 s = f.face_scale ? f.face_scale[p] : make_float2(1, 1);
        const int nb = f.face_nbr[p];
        H4 hn, hd;
        load_window(base + (long long)nb * kHistRow, hn, hd);
        const R nnew = hd.v[0];  // lane q = 0: N[t+1], stashed in Dirichlet tap 0 (Ring::stash_next)
        const R un = __shfl_up_sync(quad, hn.v[3], 1, 4), ud = __shfl_up_sync(quad, hd.v[3], 1, 4);
#pragma unroll
        for (int i = 0; i < 4; i++)
        {
            R di = (q == 0 && i == 0) ? (R)0 : hd.v[i];
            a0 += conv_tap(w.v[i], s, hn.v[i], di);
        }
        H4 sn, sd;
        sn.v[0] = q ? un : nnew;
        sd.v[0] = q ? ud : (R)0;
        sd.v[1] = q ? hd.v[0] : (R)0;
#pragma unroll
        for (int i = 1; i < 4; i++)
            sn.v[i] = hn.v[i - 1];
        sd.v[2] = hd.v[1];
        sd.v[3] = hd.v[2];
#pragma unroll
        for (int i = 0; i < 4; i++)
            a1 += conv_tap(w.v[i], s, sn.v[i], sd.v[i]);
    }
    c0 = warp_sum(a0);
    c1 = warp_sum(a1);
}

// far-field corner values of triangle tri (lanes 0-7; the others 0)
template <typename R>
__device__ inline void face_corners(const Ring<R> &ring, int tnew, const FaceArgs<R> &f, int tri, int lane, R &iw,
                                    R &pv)
{
    iw = 0;
    pv = 0;
    if (lane < 8)
    {
        iw = f.interp_d ? (R)f.interp_d[8 * tri + lane] : (R)f.interp[8 * tri + lane];
        pv = ring.slot(tnew)[f.face_corner[8 * tri + lane]];
    }
}

// mode 0: one step; 1: first step of a two-step pass (nnext = N[t+1] of this triangle);
// 2: second step of a two-step pass.  commit = false: no history / Dirichlet writes (timing)
template <typename R>
__device__ inline void face_finish(const Ring<R> &ring, int tnew, const FaceArgs<R> &f, int tri, int lane, R iw, R pv,
                                   R conv, int mode = 0, R nnext = 0, bool commit = true)
{
    R far_sum = 0;  // corners in order 0..7
#pragma unroll
    for (int wi = 0; wi < 8; wi++)
        far_sum += __shfl_sync(kFull, iw, wi) * __shfl_sync(kFull, pv, wi);
    R num = far_sum * (R)f.reflect + conv;
    const R dnew = (R)(num / f.denom[tri]);
    if (commit && lane < 4)
        ring.hat(1, lane, tri, hist_index(lane, tnew)) = dnew;  // lane c: copy c
    else if (commit && lane == 4 && f.dlast)
        f.dlast[tri] = dnew;
    else if (commit && lane == 5)
        flag_nonfinite(f.status, dnew);  // a NaN acceleration or field reaches D within a step or two
    else if (commit && lane == 6)
        ring.canon_at(1, tri, tnew) = dnew;
    if (mode == 1)
        near_terms2<R>(ring, tnew, f, tri, lane, dnew, nnext);
    else if (mode == 2)
        near_terms_complete<R>(f, tri, lane, dnew);
    else
        near_terms<R>(ring, tnew, f, tri, lane, true, dnew);
}

// N[t+1] of triangle tri for a two-step pass: the next step's acceleration row, or, without one,
// the ring slot the step would read
template <typename R>
__device__ inline R next_neumann(const Ring<R> &ring, const StepDyn &dn, int tri)
{
    return dn.acc ? (R)dn.acc[tri] : ring.canon_at(0, tri, dn.tnew);
}

// the fused face stage (corner loads issued first so their latency overlaps the convolution)
template <typename R>
__device__ inline void face_body(const StepArgs &, const Ring<R> &ring, const StepDyn &dy, const FaceArgs<R> &f,
                                 int tri, int lane)
{
    R iw, pv;
    face_corners<R>(ring, dy.tnew, f, tri, lane, iw, pv);
    const R conv = face_conv<R>(ring, dy.tnew, f, tri, lane);
    face_finish<R>(ring, dy.tnew, f, tri, lane, iw, pv, conv);
}

// pipelined step: the face-pair convolution of step kstep into conv[tri]
// Warps take the centre triangles in base-cell order: centres that share a base cell have the
// same 4^3 neighbour list, so the warps of one block gather the same neighbours' history windows
// and mostly hit L1.  Each centre's sum is the same whatever warp computes it.
template <typename R>
__device__ inline int centre_of(const FaceArgs<R> &f, int w)
{
    return f.order ? f.order[w] : w;
}

template <typename R>
__global__ void __launch_bounds__(256) conv_kernel(const __grid_constant__ Ring<R> ring, const StepState *st,
                                                    int kstep, int nt, const __grid_constant__ FaceArgs<R> f, R *conv)
{
    const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (w >= nt)
        return;
    const int tri = centre_of(f, w);
    const R v = face_conv<R>(ring, st->tnew0 + kstep, f, tri, threadIdx.x & 31);
    if ((threadIdx.x & 31) == 0)
        conv[tri] = v;
}

// pipelined step pair: the face-pair convolution of step kstep into conv[tri] and the partial
// convolution of step kstep + 1 into conv1[tri] (face_conv2)
template <typename R>
__global__ void __launch_bounds__(256) conv2_kernel(const __grid_constant__ Ring<R> ring, const StepState *st,
                                                     int kstep, int nt, const __grid_constant__ FaceArgs<R> f, R *conv,
                                                     R *conv1)
{
    const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (w >= nt)
        return;
    const int tri = centre_of(f, w);
    R c0, c1;
    face_conv2<R>(ring, st->tnew0 + kstep, f, tri, threadIdx.x & 31, c0, c1);
    if ((threadIdx.x & 31) == 0)
    {
        conv[tri] = c0;
        conv1[tri] = c1;
    }
}

// second step of a pipelined pair: conv[tri] = conv1[tri] + sum_j d1_j D_j[t-1], with D[t-1] the
// Dirichlet values that finish of the step before has just written (compact per-triangle copy,
// small enough to stay in L1), lanes striding over the pairs
template <typename R>
__device__ inline void face_fix(const FaceArgs<R> &f, const R *conv1, R *conv, int tri, int lane)
{
    const int b = f.face_start[tri], e = f.face_start[tri + 1];
    R a = 0;
    for (int p = b + lane; p < e; p += 32)
        a += f.face_d1[p] * f.dlast[f.face_nbr[p]];
    a = warp_sum(a);
    if (lane == 0)
        conv[tri] = conv1[tri] + a;
}

template <typename R>
__global__ void __launch_bounds__(256) fix_kernel(int nt, const __grid_constant__ FaceArgs<R> f, const R *conv1, R *conv)
{
    const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (w >= nt)
        return;
    face_fix<R>(f, conv1, conv, centre_of(f, w), threadIdx.x & 31);
}

// pipelined step: the rest of the face stage of step kstep; next & 1: also the Neumann value of
// step kstep + 1 into the history (its slot is outside every window of this step), so the next
// step's convolution can start before that step's stencil; next & 2: step kstep + 1 starts a
// two-step pass over the face pairs, which receives N of step kstep + 2 with its history windows
// (Ring::stash_next)
// (one instantiation per mode: the two-step variants need more registers, which the one-step
// path should not carry)
template <typename R, int mode>
__global__ void __launch_bounds__(256) finish_kernel(const __grid_constant__ Ring<R> ring, const StepState *st,
                                                      int kstep, int nt, const __grid_constant__ FaceArgs<R> f,
                                                      const R *conv, int next)
{
    grid_dependency_wait();
    const int tri = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (tri >= nt)
        return;
    const int lane = threadIdx.x & 31;
    const StepDyn dy = bind_step(st, kstep, nt);
    const StepDyn dn = bind_step(st, kstep + 1, nt);
    R iw, pv;
    face_corners<R>(ring, dy.tnew, f, tri, lane, iw, pv);
    face_finish<R>(ring, dy.tnew, f, tri, lane, iw, pv, conv[tri], mode,
                   mode == 1 ? next_neumann<R>(ring, dn, tri) : (R)0);
    if ((next & 1) && lane == 0)
        ring.nwrite(tri, dn.tnew, dn.acc);
    else if ((next & 2) && lane == 1)
        ring.stash_next(tri, dn.tnew, bind_step(st, kstep + 2, nt).acc);
}

// the autotuner's finish: the same work without the history and Dirichlet writes, so that timing
// it changes no state (the near-field terms it writes are rebuilt by every step before they are
// read)
template <typename R, int mode>
__global__ void __launch_bounds__(256) finish_dry_kernel(const __grid_constant__ Ring<R> ring, const StepState *st,
                                                          int kstep, int nt, const __grid_constant__ FaceArgs<R> f,
                                                          const R *conv)
{
    const int tri = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (tri >= nt)
        return;
    const int lane = threadIdx.x & 31;
    const StepDyn dy = bind_step(st, kstep, nt);
    const StepDyn dn = bind_step(st, kstep + 1, nt);
    R iw, pv;
    face_corners<R>(ring, dy.tnew, f, tri, lane, iw, pv);
    face_finish<R>(ring, dy.tnew, f, tri, lane, iw, pv, conv[tri], mode,
                   mode == 1 ? next_neumann<R>(ring, dn, tri) : (R)0, false);
}

// the Neumann value of step kstep into the history (first step of a pipelined call); stash: the step
// starts a two-step pass over the face pairs (Ring::stash_next)
template <typename R>
__global__ void nwrite_kernel(const __grid_constant__ Ring<R> ring, const StepState *st, int kstep, int nt, int stash)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const StepDyn dy = bind_step(st, kstep, nt);
    if (i < nt)
    {
        ring.nwrite(i, dy.tnew, dy.acc);
        if (stash)
            ring.stash_next(i, dy.tnew, bind_step(st, kstep + 1, nt).acc);
    }
}

// the near-field terms of time t for every triangle without a face step (priming)
template <typename R>
__global__ void __launch_bounds__(256) terms_kernel(const __grid_constant__ Ring<R> ring, int nt, int t,
                                                     const __grid_constant__ FaceArgs<R> f)
{
    const int tri = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (tri < nt)
        near_terms<R>(ring, t, f, tri, threadIdx.x & 31, false, (R)0);
}

template <typename R>
__global__ void __launch_bounds__(256) face_kernel(const __grid_constant__ StepArgs a0,
                                                    const __grid_constant__ Ring<R> ring, const StepState *st, int kstep,
                                                    const __grid_constant__ FaceArgs<R> f)
{
    const int tri = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (tri < a0.nt)
        face_body<R>(a0, ring, bind_step(st, kstep, a0.nt), f, tri, threadIdx.x & 31);
}

// near stage: warps stride over the corrected cells (their number changes with the mesh, the
// grid does not).  A corrected cell's FDTD-near sum (for the next step) and BEM-near sum are the
// sums of its pairs' terms (near_terms), lanes striding over the pair list.  prime != 0: only the
// next step's FDTD-near sum.
template <typename R>
struct NearArgs
{
    const int *n3_cell, *n3_start, *p3_tri;
    const unsigned char *p3_woff;  // the pair's record offset in 3^3
    const R *terms;
};

// the near-stage work of corrected cells warp0, warp0 + nwarps, ... < n3 of one scene
template <typename R>
__device__ inline void near_body(const StepArgs &a, const Ring<R> &ring, const StepDyn &dy, const NearArgs<R> &na,
                                 int n3, int warp0, int nwarps, int lane, int prime)
{
    R *cur = ring.slot(dy.tnew), *nextslot = ring.slot(dy.tnew + 1);
    for (int ci = warp0; ci < n3; ci += nwarps)
    {
        // the cell and its far-field value are fetched before the pair sums, so their latency
        // overlaps the term gathers
        const int c = lane == 0 ? na.n3_cell[ci] : 0;
        const R far = lane == 0 && !prime ? cur[c] : (R)0;
        const int b = na.n3_start[ci], e = na.n3_start[ci + 1];
        R acc_f = 0, acc_b = 0;
        for (int p = b + lane; p < e; p += 32)
        {
            const R *t = na.terms + (long long)na.p3_tri[p] * kGcRecords + na.p3_woff[p];
            acc_f += t[0];
            if (!prime)
                acc_b += t[kGcRecords / 2];
        }
        acc_f = warp_sum(acc_f);
        if (!prime)
            acc_b = warp_sum(acc_b);
        if (lane == 0)
        {
            nextslot[c] = acc_f;
            if (!prime)
            {
                R v = (R)((double)far + (double)acc_b * 0.98);
                cur[c] = v;
                for (int l = 0; l < a.n_listen; l++)
                    if (a.listen_cell[l] == c)
                    {
                        ((R *)dy.series)[dy.row * a.n_listen + l] = v;
                        flag_nonfinite(a.status, v);
                    }
            }
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(256) near_kernel(const __grid_constant__ StepArgs a0,
                                                    const __grid_constant__ Ring<R> ring, const StepState *st, int kstep,
                                                    const __grid_constant__ NearArgs<R> na, int prime)
{
    grid_dependency_wait();
    near_body<R>(a0, ring, bind_step(st, kstep, a0.nt), na, st->n3,
                 (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5),
                 (int)(((long long)gridDim.x * blockDim.x) >> 5), threadIdx.x & 31, prime);
}

template <typename R>
StepArgs make_args(Handle &h)
{
    StepArgs a{};
    a.res = h.res;
    a.c = h.prm.c;
    a.dt = h.prm.dt;
    a.h = h.prm.dl;
    double cd = h.prm.c, dtd = h.prm.dt;
    a.lap_coef = cd * cd * dtd * dtd;
    a.hd = h.prm.dl;
    a.h2 = a.hd * a.hd;
    a.rh2 = 1.0 / a.h2;
    a.pml_width = h.prm.pml_width;
    a.damp = 2.0f / h.prm.dl;
    a.nt = h.mesh_set ? h.nt : 0;
    a.n_listen = (int)h.listen_xyz.size() / 3;
    a.status = h.d_step_status;
    return a;
}

template <typename R>
int fill_listeners(Handle &h, StepArgs &a)
{
    if (a.n_listen > 8)
    {
        set_error("at most 8 listeners");
        return PPPM_ERR_ARG;
    }
    for (int l = 0; l < a.n_listen; l++)
    {
        a.listen_cell[l] = (h.listen_xyz[3 * l] * h.res + h.listen_xyz[3 * l + 1]) * h.res + h.listen_xyz[3 * l + 2];
    }
    return PPPM_OK;
}

// Every argument the kernels of one step receive apart from the step index k.  Two calls with
// equal launch sets (same arrays, counts and listeners) record identical graphs.
template <typename R>
struct StepLaunch
{
    using W = typename WRec<R>::T;
    StepArgs a;  // the per-step fields stay zero: kernels bind them from the StepState
    Ring<R> ring;
    StencilSplit sp;
    const StepState *st;
    const unsigned *corr_mask;
    FaceArgs<R> fa;
    NearArgs<R> na;
    R *conv;   // per-triangle convolution sums of the pipelined step
    R *conv1;  // partial sums of the second step of a pipelined pair
    int pairs;         // pipelined graphs convolve the face pairs for two steps per pass (conv2 + fix)
    int face_threads;  // threads per block of the pipelined face-stage kernels
    int tpairs;        // the near-field terms two steps per pass (near_terms2)
    int split;         // recorded graphs: corrected-cell stencil on the main branch, the bulk beside it
    int corr_blocks;   // grid of stencil_corr_kernel (threads stride over the corrected cells)
    int mesh, pml, pml_blocks, stencil_blocks, face_blocks, near_blocks;
    int ghost;     // ghost-cell method: the ghost kernel after the stencil instead of face / near
    GhostStep gs;  // its arguments
};

__global__ void set_state_kernel(StepState *dst, StepState v) { *dst = v; }

template <typename R>
int make_launch(Handle &h, StepLaunch<R> &L)
{
    using W = typename WRec<R>::T;
    memset(&L, 0, sizeof(L));  // padding too: the launch set is compared byte by byte
    L.a = make_args<R>(h);
    PB_TRY(fill_listeners<R>(h, L.a));
    for (int i = 0; i < 3; i++)
    {
        L.ring.g[i] = (R *)h.grid[i];
        L.ring.p[i] = (R *)h.pml[i];
    }
    L.sp = stencil_split(h.res, L.a.nt, !h.fp64, h.stencil_vec4);
    L.st = h.d_state;
    L.corr_mask = h.d_corr_mask;
    L.ring.hist = (R *)h.d_hist;
    L.ring.canon[0] = (R *)h.d_neumann;
    L.ring.canon[1] = (R *)h.d_dirichlet;
    L.ring.nt = h.mesh_set ? h.nt : 0;
    L.mesh = h.mesh_set && h.prm.method == PPPM_METHOD_PPPM ? 1 : 0;
    L.pml = h.prm.pml_width > 0 ? 1 : 0;
    const int m = h.res - 2, T = 256;
    L.pml_blocks = (int)div_up(std::max<long long>((long long)m * m * m, L.a.nt), T);
    L.stencil_blocks = L.sp.nb_in + L.sp.nb_bd + L.sp.nb_nt;
    if (h.mesh_set && h.prm.method == PPPM_METHOD_GHOST)
    {
        if constexpr (sizeof(R) == 4)
        {
            L.ghost = 1;
            L.gs = ghost_args(h, L.a.n_listen, L.a.listen_cell);
        }
        return PPPM_OK;
    }
    if (h.mesh_set)
    {
        L.fa.face_start = h.d_face_start;
        L.fa.face_nbr = h.d_face_nbr;
        L.fa.face_corner = h.d_face_corner;
        L.fa.face_w = (const W *)h.d_face_w;
        L.fa.face_scale = h.fp64 ? nullptr : h.d_face_scale;
        L.fa.interp = h.d_face_interp;
        L.fa.interp_d = h.fp64 ? h.d_face_interp_d : nullptr;
        L.fa.denom = h.d_face_denom;
        L.fa.reflect = h.prm.reflect_coeff;
        L.fa.gc_w = (const W *)h.d_gc_w;
        L.fa.gc_scale = h.fp64 ? nullptr : h.d_gc_scale;
        L.fa.terms = (R *)h.d_terms;
        L.conv = (R *)h.d_conv;
        L.conv1 = (R *)h.d_conv1;
        L.pairs = h.conv_pairs;
        L.face_threads = h.face_threads;
        L.tpairs = h.terms_pairs ? 1 : 0;
        // the split step's bulk runs beside the near stage, which overwrites p^{t-1} at corrected
        // cells with the next step's sums: only when no corrected cell neighbours a boundary-layer
        // cell whose solve reads it (mesh_build's check)
        L.split = h.split_stencil && !h.corr_near_boundary ? 1 : 0;
        L.fa.face_d1 = (const R *)h.d_face_d1;
        L.fa.order = h.d_base_tris;
        L.fa.dlast = (R *)h.d_dlast;
        L.fa.terms1 = (R *)h.d_terms1;
        L.fa.gc_f = (const R *)h.d_gc_f;
        L.fa.status = h.d_step_status;
        L.na.n3_cell = h.d_n3_cell;
        L.na.n3_start = h.d_n3_start;
        L.na.p3_tri = h.d_p3_tri;
        L.na.p3_woff = h.d_p3_woff;
        L.na.terms = (const R *)h.d_terms;
        L.face_blocks = (int)div_up((long long)h.nt * 32, T);
        if (h.near_blocks <= 0)
        {
            // as many warps as stay resident: they stride over the corrected cells
            int per_sm = 0, sms = 0;
            PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, near_kernel<R>, T, 0));
            PB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h.prm.device));
            h.near_blocks = std::max(per_sm, 1) * std::max(sms, 1);
        }
        L.near_blocks = h.near_blocks;
        L.corr_blocks = std::max(1, h.near_blocks / 4);
    }
    return PPPM_OK;
}

// the kernels of step k of a call (no error check: may run under stream capture)
template <typename R>
void launch_step(const StepLaunch<R> &L, int k, cudaStream_t s, Handle *timed)
{
    const int T = 256;
    // timed: event records between the kernels (graph nodes when captured, see run_steps)
    auto mark = [&](int i) {
        if (timed)
            cudaEventRecordWithFlags(timed->ev[i], s, cudaEventRecordExternal);
    };
    mark(0);
    if (L.pml)
        pml_kernel<R><<<L.pml_blocks, T, 0, s>>>(L.a, L.ring, L.st, k, L.corr_mask);
    else
        stencil_kernel<R><<<L.stencil_blocks, T, 0, s>>>(L.a, L.ring, L.st, k, L.sp, L.corr_mask);
    mark(1);
    if constexpr (sizeof(R) == 4)
        if (L.ghost)
        {
            ghost_launch(L.gs, L.st, k, L.a.nt, s);
            mark(2);
        }
    if (L.mesh)
    {
        face_kernel<R><<<L.face_blocks, T, 0, s>>>(L.a, L.ring, L.st, k, L.fa);
        mark(2);
        near_kernel<R><<<L.near_blocks, T, 0, s>>>(L.a, L.ring, L.st, k, L.na, 0);
    }
    mark(3);
}

// The kernels of nsteps steps as a multi-branch graph (absorbing boundary with a mesh).  Per step:
//   side   conv(k)                       after finish(k-1): needs D[t-1] and N[t]
//   main   stencil(k) -> finish(k) -> near(k)   finish waits for conv(k) too
// so each step's face-pair convolution (the heavy part of the face stage) runs beside the
// previous step's near stage and this step's stencil; finish(k) also writes N[t+1] for conv(k+1).
// With pair set, steps go in pairs (k, k+1): conv2(k) streams the face pairs once for both steps
// and fix(k+1), after finish(k), adds the one term of step k+1 that needs D of step k.
// With the split stencil (L.split), the main branch computes only the corrected cells
// (stencil_corr_kernel: the face stage and the near stage read and write nothing else) and a
// third branch the rest of the grid:
//   bulk   stencil(k) without corrected cells   after near(k-1): p^t complete at corrected cells
//   main   corr(k) -> finish(k) -> near(k)       corr(k) after bulk(k-1): p^t complete elsewhere
// The bulk writes p^{t+1} at other cells than the main branch reads or writes in the meantime (the
// near stage's next-step sums go to corrected cells of slot t+2 = t-1, which the bulk reads only
// elsewhere), so it leaves the step's critical path.  Only used under stream capture: main =
// h.stream, side = h.side, bulk = h.side2, joined back before the end.
// after a chunk graph of g steps (run_steps): the call's state moves on by g steps
__global__ void advance_state_kernel(StepState *st, int g, int nt)
{
    st->tnew0 += g;
    st->row0 += g;
    if (st->acc)
        st->acc += (long long)g * nt;
}

// open: the nsteps steps are a chunk of a longer call (run_steps), so the last of them is no
// call's last step: it pairs, computes its terms and writes the next Neumann value as any other
// step does (nsteps is even then, so the pairs are those of the whole call); a kernel after the
// joins moves the call's state on by nsteps for the next chunk.
template <typename R>
void capture_pipelined(Handle &h, const StepLaunch<R> &L, int nsteps, bool pair, bool open)
{
    const int T = 256, FT = L.face_threads;
    const int nt = L.a.nt;
    const int wblocks = div_up((long long)nt * 32, FT);
    cudaStream_t s = h.stream, side = h.side, bulk = h.side2;
    const bool split = L.split && bulk;
    StencilSplit bsp = L.sp;
    bsp.skip_corrected = 1;
    // step j's convolution is a two-step pass (conv2_kernel)
    auto conv2_at = [&](int j) { return pair && !(j & 1) && j < nsteps && (open || j + 1 < nsteps); };
    nwrite_kernel<R><<<div_up(nt, T), T, 0, s>>>(L.ring, L.st, 0, nt, conv2_at(0) ? 1 : 0);
    cudaEventRecord(h.ev_fin, s);
    if (split)
        cudaEventRecord(h.ev_near, s);
    for (int k = 0; k < nsteps; k++)
    {
        const bool more = open || k + 1 < nsteps;  // a later step follows in this call
        cudaStreamWaitEvent(side, h.ev_fin, 0);
        if (pair && (k & 1))
            fix_kernel<R><<<wblocks, FT, 0, side>>>(nt, L.fa, L.conv1, L.conv);
        else if (pair && more)
            conv2_kernel<R><<<wblocks, FT, 0, side>>>(L.ring, L.st, k, nt, L.fa, L.conv, L.conv1);
        else
            conv_kernel<R><<<wblocks, FT, 0, side>>>(L.ring, L.st, k, nt, L.fa, L.conv);
        cudaEventRecord(h.ev_conv, side);
        if (split)
        {
            if (k > 0)
                cudaStreamWaitEvent(s, h.ev_bulk, 0);  // bulk(k-1)
            cudaStreamWaitEvent(bulk, h.ev_near, 0);   // near(k-1), or the call's start
            stencil_kernel<R><<<L.sp.nb_bd + L.sp.nb_in, T, 0, bulk>>>(L.a, L.ring, L.st, k, bsp, L.corr_mask);
            cudaEventRecord(h.ev_bulk, bulk);
            launch_dependent(stencil_corr_kernel<R>, L.corr_blocks, T, s, L.a, L.ring, L.st, k, L.na.n3_cell);
        }
        else
            // the stencil without its Neumann block range (finish / nwrite wrote N[t])
            stencil_kernel<R><<<L.sp.nb_bd + L.sp.nb_in, T, 0, s>>>(L.a, L.ring, L.st, k, L.sp, L.corr_mask);
        cudaStreamWaitEvent(s, h.ev_conv, 0);
        // the call's last step computes its terms in one pass (mode 0): the FDTD-near sums it
        // leaves for the next call are then exactly those that prime() rebuilds after a state
        // restore or a mesh update
        const int mode = L.tpairs && more ? ((k & 1) ? 2 : 1) : 0;
        const int nx = (more ? 1 : 0) | (conv2_at(k + 1) ? 2 : 0);
        const R *conv = L.conv;
        if (mode == 1)
            launch_dependent(finish_kernel<R, 1>, wblocks, FT, s, L.ring, L.st, k, nt, L.fa, conv, nx);
        else if (mode == 2)
            launch_dependent(finish_kernel<R, 2>, wblocks, FT, s, L.ring, L.st, k, nt, L.fa, conv, nx);
        else
            launch_dependent(finish_kernel<R, 0>, wblocks, FT, s, L.ring, L.st, k, nt, L.fa, conv, nx);
        cudaEventRecord(h.ev_fin, s);
        launch_dependent(near_kernel<R>, L.near_blocks, T, s, L.a, L.ring, L.st, k, L.na, 0);
        if (split)
            cudaEventRecord(h.ev_near, s);
    }
    if (split)
        cudaStreamWaitEvent(s, h.ev_bulk, 0);
    if (open)
        advance_state_kernel<<<1, 1, 0, s>>>(const_cast<StepState *>(L.st), nsteps, nt);
}


__global__ void empty_kernel() {}

// Measurement mode per kernel: the kernels of Handle::kProfileSteps steps exactly as
// capture_pipelined issues them for a call of that many steps, but serialised on the handle's
// stream with an event record between consecutive kernels; evk_kind[i] names the kind of the
// kernel between events i and i + 1.
template <typename R>
int profile_graph(Handle &h, const StepLaunch<R> &L, cudaGraphExec_t *out)
{
    const unsigned char *sig = (const unsigned char *)&L;
    StepGraph &g = h.profile_graph;
    if (g.exec && g.sig.size() == sizeof(L) && memcmp(g.sig.data(), sig, sizeof(L)) == 0)
    {
        *out = g.exec;
        return PPPM_OK;
    }
    if (g.exec)
        cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    const int T = 256, FT = L.face_threads, nt = L.a.nt, n = Handle::kProfileSteps;
    const int wblocks = div_up((long long)nt * 32, FT);
    const bool pair = L.pairs != 0;
    cudaStream_t s = h.stream;
    int e = 0;
    bool overflow = false;
    auto mark = [&](int kind) {
        if (e >= Handle::kProfileEvents)
        {
            overflow = true;
            return;
        }
        h.evk_kind[e] = kind;
        cudaEventRecordWithFlags(h.evk[e++], s, cudaEventRecordExternal);
    };
    cudaGraph_t graph = nullptr;
    PB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    auto conv2_at = [&](int j) { return pair && !(j & 1) && j + 1 < n; };
    mark(PPPM_KERNEL_NWRITE);
    nwrite_kernel<R><<<div_up(nt, T), T, 0, s>>>(L.ring, L.st, 0, nt, conv2_at(0) ? 1 : 0);
    mark(PPPM_KERNEL_EMPTY);
    empty_kernel<<<1, 32, 0, s>>>();
    for (int k = 0; k < n; k++)
    {
        if (pair && (k & 1))
        {
            mark(PPPM_KERNEL_FIX);
            fix_kernel<R><<<wblocks, FT, 0, s>>>(nt, L.fa, L.conv1, L.conv);
        }
        else if (pair && k + 1 < n)
        {
            mark(PPPM_KERNEL_CONV2);
            conv2_kernel<R><<<wblocks, FT, 0, s>>>(L.ring, L.st, k, nt, L.fa, L.conv, L.conv1);
        }
        else
        {
            mark(PPPM_KERNEL_CONV);
            conv_kernel<R><<<wblocks, FT, 0, s>>>(L.ring, L.st, k, nt, L.fa, L.conv);
        }
        if (L.split)
        {
            StencilSplit bsp = L.sp;
            bsp.skip_corrected = 1;
            mark(PPPM_KERNEL_STENCIL_BULK);
            stencil_kernel<R><<<L.sp.nb_bd + L.sp.nb_in, T, 0, s>>>(L.a, L.ring, L.st, k, bsp, L.corr_mask);
            mark(PPPM_KERNEL_STENCIL_CORR);
            stencil_corr_kernel<R><<<L.corr_blocks, T, 0, s>>>(L.a, L.ring, L.st, k, L.na.n3_cell);
        }
        else
        {
            mark(PPPM_KERNEL_STENCIL);
            stencil_kernel<R><<<L.sp.nb_bd + L.sp.nb_in, T, 0, s>>>(L.a, L.ring, L.st, k, L.sp, L.corr_mask);
        }
        const int mode = L.tpairs && k + 1 < n ? ((k & 1) ? 2 : 1) : 0;
        const int nx = (k + 1 < n ? 1 : 0) | (conv2_at(k + 1) ? 2 : 0);
        if (mode == 1)
        {
            mark(PPPM_KERNEL_FINISH1);
            finish_kernel<R, 1><<<wblocks, FT, 0, s>>>(L.ring, L.st, k, nt, L.fa, L.conv, nx);
        }
        else if (mode == 2)
        {
            mark(PPPM_KERNEL_FINISH2);
            finish_kernel<R, 2><<<wblocks, FT, 0, s>>>(L.ring, L.st, k, nt, L.fa, L.conv, nx);
        }
        else
        {
            mark(PPPM_KERNEL_FINISH);
            finish_kernel<R, 0><<<wblocks, FT, 0, s>>>(L.ring, L.st, k, nt, L.fa, L.conv, nx);
        }
        mark(PPPM_KERNEL_NEAR);
        near_kernel<R><<<L.near_blocks, T, 0, s>>>(L.a, L.ring, L.st, k, L.na, 0);
    }
    mark(-1);
    cudaError_t err = cudaStreamEndCapture(s, &graph);
    if (err == cudaSuccess && !overflow)
        err = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph)
        cudaGraphDestroy(graph);
    h.evk_used = overflow ? 0 : e;
    if (overflow)
    {
        g.exec = nullptr;
        set_error("profile graph: more event marks than its %d slots", Handle::kProfileEvents);
        return PPPM_ERR_STATE;
    }
    if (err != cudaSuccess)
    {
        g.exec = nullptr;
        set_error("recording the profile graph failed: %s", cudaGetErrorString(err));
        return PPPM_ERR_CUDA;
    }
    g.nsteps = n;
    g.sig.assign(sig, sig + sizeof(L));
    *out = g.exec;
    return PPPM_OK;
}

// Calls of at least kGraphSteps steps replay a CUDA graph of their kernels, recorded on the
// first call with that step count and launch set (the graph removes the host launch cost and
// most of the gap between dependent kernels); shorter calls, measurement mode and calls on a
// stream that the caller is capturing launch the kernels directly.
constexpr int kGraphSteps = 4;

template <typename R>
int graph_for(Handle &h, const StepLaunch<R> &L, int nsteps, cudaGraphExec_t *out, bool timed = false,
              bool open = false)
{
    const unsigned char *sig = (const unsigned char *)&L;
    StepGraph *slots = timed ? &h.timing_graph : h.graphs;
    const int nslots = timed ? 1 : kStepGraphs;
    for (int i = 0; i < nslots; i++)
    {
        StepGraph &g = slots[i];
        if (g.exec && g.nsteps == nsteps && g.open == open && g.sig.size() == sizeof(L) &&
            memcmp(g.sig.data(), sig, sizeof(L)) == 0)
        {
            *out = g.exec;
            return PPPM_OK;
        }
    }
    StepGraph &g = timed ? h.timing_graph : h.graphs[h.graph_next];
    if (!timed)
        h.graph_next = (h.graph_next + 1) % kStepGraphs;
    if (g.exec)
        cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    cudaGraph_t graph = nullptr;
    PB_CUDA(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal));
    if (!timed && L.mesh && !L.pml && h.side)
        capture_pipelined<R>(h, L, nsteps, L.pairs != 0, open);
    else
    {
        for (int k = 0; k < nsteps; k++)
            launch_step<R>(L, k, h.stream, timed ? &h : nullptr);
        if (open)
            advance_state_kernel<<<1, 1, 0, h.stream>>>(const_cast<StepState *>(L.st), nsteps, L.a.nt);
    }
    cudaError_t e = cudaStreamEndCapture(h.stream, &graph);
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph)
        cudaGraphDestroy(graph);
    if (e != cudaSuccess)
    {
        g.exec = nullptr;
        set_error("recording the step graph failed: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    g.nsteps = nsteps;
    g.open = open;
    g.sig.assign(sig, sig + sizeof(L));
    *out = g.exec;
    return PPPM_OK;
}

template <typename R>
int run_steps(Handle &h, const float *acc_dev, int nsteps)
{
    if (nsteps <= 0)
        return PPPM_OK;
    cudaStream_t s = h.stream;
    if (!h.d_state)
        PB_TRY(dalloc(&h.d_state, 1));
    StepState stt{h.t + 1, h.mesh_set ? h.n3 : 0, h.series_count, acc_dev};
    stt.series = h.d_series;
    set_state_kernel<<<1, 1, 0, s>>>(h.d_state, stt);
    h.launches++;
    PB_CHECK_LAUNCH();
    StepLaunch<R> L;
    PB_TRY(make_launch<R>(h, L));
    const long long per_step = 1 + (h.mesh_set ? 2 : 0);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PB_CUDA(cudaStreamIsCapturing(s, &cs));
    if (h.timing && cs == cudaStreamCaptureStatusNone)
    {
        // Measurement mode.  Where the recorded graphs run the split face stage, groups of
        // kProfileSteps steps replay the profile graph (those kernels serialised, events between
        // them); the other steps replay a one-step graph of the fused kernels with event records
        // between them.  Either way each kernel's duration is measured the way it runs inside a
        // recorded graph (no host launch gaps); the step state is rewritten per replay.
        int done = 0;
        if (L.mesh && !L.pml && h.side && nsteps >= Handle::kProfileSteps)
        {
            cudaGraphExec_t pexec = nullptr;
            PB_TRY(profile_graph<R>(h, L, &pexec));
            const int n = Handle::kProfileSteps;
            for (; done + n <= nsteps; done += n)
            {
                StepState sk{stt.tnew0 + done, stt.n3, stt.row0 + done,
                             acc_dev ? acc_dev + (long long)done * h.nt : nullptr};
                sk.series = h.d_series;
                set_state_kernel<<<1, 1, 0, s>>>(h.d_state, sk);
                PB_CHECK_LAUNCH();
                PB_CUDA(cudaGraphLaunch(pexec, s));
                PB_CUDA(cudaEventSynchronize(h.evk[h.evk_used - 1]));
                for (int i = 0; i + 1 < h.evk_used; i++)
                {
                    float ms = 0;
                    cudaEventElapsedTime(&ms, h.evk[i], h.evk[i + 1]);
                    const int kind = h.evk_kind[i];
                    h.kind_us[kind] += 1000.0 * ms;
                    h.kind_n[kind]++;
                    if (kind == PPPM_KERNEL_EMPTY)
                        continue;
                    if (kind == PPPM_KERNEL_STENCIL)
                        h.us_stencil += 1000 * ms;
                    else if (kind == PPPM_KERNEL_NEAR)
                        h.us_near += 1000 * ms;
                    else
                        h.us_face += 1000 * ms;
                }
                h.timed_steps += n;
                h.launches += 2 + (4 + L.split - per_step) * n;  // per_step * nsteps is added below
            }
        }
        cudaGraphExec_t exec = nullptr;
        if (done < nsteps)
            PB_TRY(graph_for<R>(h, L, 1, &exec, true));
        for (int k = done; k < nsteps; k++)
        {
            StepState sk{stt.tnew0 + k, stt.n3, stt.row0 + k,
                         acc_dev ? acc_dev + (long long)k * (h.mesh_set ? h.nt : 0) : nullptr};
            sk.series = h.d_series;
            set_state_kernel<<<1, 1, 0, s>>>(h.d_state, sk);
            PB_CHECK_LAUNCH();
            PB_CUDA(cudaGraphLaunch(exec, s));
            PB_CUDA(cudaEventSynchronize(h.ev[3]));
            float ta = 0, tb = 0, tc = 0;
            cudaEventElapsedTime(&ta, h.ev[0], h.ev[1]);
            if (h.mesh_set)
            {
                cudaEventElapsedTime(&tb, h.ev[1], h.ev[2]);
                cudaEventElapsedTime(&tc, h.ev[2], h.ev[3]);
            }
            h.us_stencil += 1000 * ta;
            h.us_face += 1000 * tb;
            h.us_near += 1000 * tc;
            h.timed_steps++;
            h.kind_us[PPPM_KERNEL_STENCIL] += 1000.0 * ta;
            h.kind_n[PPPM_KERNEL_STENCIL]++;
            if (h.mesh_set)
            {
                h.kind_us[PPPM_KERNEL_FACE] += 1000.0 * tb;
                h.kind_us[PPPM_KERNEL_NEAR] += 1000.0 * tc;
                h.kind_n[PPPM_KERNEL_FACE]++;
                h.kind_n[PPPM_KERNEL_NEAR]++;
            }
        }
    }
    else if (cs == cudaStreamCaptureStatusNone && nsteps >= kGraphSteps)
    {
        // Calls longer than G = h.graph_chunk steps (even) replay one recorded chunk of G steps
        // as often as it fits and then a graph of the remaining 1..G steps (with the call's
        // last-step work), so a run of frames of uneven length records a few short graphs
        // instead of one long graph per length (recording costs about 0.1 ms per step).  The
        // kernels, their order and their arguments are those of one graph of nsteps steps.
        const int G = h.graph_chunk;
        const int chunks = G > 0 && nsteps > G ? (nsteps - 1) / G : 0;
        const int rest = nsteps - chunks * G;
        const bool pipelined = L.mesh && !L.pml && h.side;
        if (chunks > 0)
        {
            cudaGraphExec_t cexec = nullptr;
            PB_TRY(graph_for<R>(h, L, G, &cexec, false, true));
            for (int c = 0; c < chunks; c++)
                PB_CUDA(cudaGraphLaunch(cexec, s));
        }
        cudaGraphExec_t exec = nullptr;
        PB_TRY(graph_for<R>(h, L, rest, &exec));
        PB_CUDA(cudaGraphLaunch(exec, s));
        // a pipelined graph launches the Neumann write, then per step the convolution, the
        // stencil (and its bulk), finish and near: counted here in place of per_step below; a
        // chunk also advances the state
        if (pipelined)
            h.launches += (chunks + 1) + (4 + L.split - per_step) * (long long)nsteps;
        h.launches += chunks;
    }
    else
        for (int k = 0; k < nsteps; k++)
        {
            launch_step<R>(L, k, s, nullptr);
            PB_CHECK_LAUNCH();
        }
    h.launches += per_step * nsteps;
    if (L.ghost)
    {
        // this and the previous step's accelerations, for the fresh cells of the next update
        h.launches += nsteps;
        const size_t row = sizeof(float) * h.nt;
        if (nsteps >= 2 && acc_dev)
            PB_CUDA(cudaMemcpyAsync(h.d_gneu_old, acc_dev + (long long)(nsteps - 2) * h.nt, row,
                                    cudaMemcpyDeviceToDevice, s));
        else
            PB_CUDA(cudaMemcpyAsync(h.d_gneu_old, h.d_gneu, row, cudaMemcpyDeviceToDevice, s));
        if (acc_dev)
            PB_CUDA(cudaMemcpyAsync(h.d_gneu, acc_dev + (long long)(nsteps - 1) * h.nt, row,
                                    cudaMemcpyDeviceToDevice, s));
        else
            PB_CUDA(cudaMemsetAsync(h.d_gneu, 0, row, s));
    }
    h.t += nsteps;
    h.series_count += nsteps;
    return PPPM_OK;
}

// Autotuner of the face stage: on the handle's current mesh and state, time the face-pair
// convolution of two consecutive steps in every candidate configuration - one pass per step
// (conv, conv) or one pass for both (conv2, fix) - at 64, 128 and 256 threads per block, each of
// the two launches reps times back to back on the handle's stream between CUDA events; then the
// rest of the face stage with the near-field terms one or two steps per pass.  The kernels write
// only scratch sums and derived terms, so no state of the scene changes.  us[2 i], us[2 i + 1]:
// microseconds per launch of the first and second kernel of candidate i, in the order
// (pairs 0, 64), (pairs 0, 128), (pairs 0, 256), (pairs 1, 64), ..., finish single, finish pairs.
constexpr int kTuneThreads[3] = {64, 128, 256};
constexpr int kTuneConfigs = 12;     // conv_pairs x face threads x terms_pairs (phase 2)
constexpr int kTuneGraphSteps = 64;  // recorded steps timed per configuration

template <typename R>
int autotune(Handle &h, int reps, float *us, int *best)
{
    if (!h.mesh_set || h.prm.method != PPPM_METHOD_PPPM || h.nt == 0)
    {
        set_error("autotune needs a mesh (PPPM method)");
        return PPPM_ERR_STATE;
    }
    if (!h.d_state)
        PB_TRY(dalloc(&h.d_state, 1));
    cudaStream_t s = h.stream;
    StepState stt{h.t + 1, h.n3, 0, nullptr};
    set_state_kernel<<<1, 1, 0, s>>>(h.d_state, stt);
    StepLaunch<R> L;
    PB_TRY(make_launch<R>(h, L));
    const int nt = h.nt;
    auto run = [&](int c, int which) {
        const int FT = kTuneThreads[c % 3], nb = div_up((long long)nt * 32, FT);
        if (c < 3)
            conv_kernel<R><<<nb, FT, 0, s>>>(L.ring, L.st, which, nt, L.fa, L.conv);
        else if (which == 1)
            fix_kernel<R><<<nb, FT, 0, s>>>(nt, L.fa, L.conv1, L.conv);
        else
            conv2_kernel<R><<<nb, FT, 0, s>>>(L.ring, L.st, 0, nt, L.fa, L.conv, L.conv1);
    };
    constexpr int kConv = 6;
    for (int c = 0; c < kConv; c++)
    {
        run(c, 0);
        run(c, 1);
    }
    PB_CHECK_LAUNCH();
    int bi = 0;
    float tot[kConv];
    for (int c = 0; c < kConv; c++)
    {
        PB_CUDA(cudaEventRecord(h.ev[0], s));
        for (int r = 0; r < reps; r++)
            run(c, 0);
        PB_CUDA(cudaEventRecord(h.ev[1], s));
        for (int r = 0; r < reps; r++)
            run(c, 1);
        PB_CUDA(cudaEventRecord(h.ev[2], s));
        PB_CUDA(cudaEventSynchronize(h.ev[2]));
        float ma = 0, mb = 0;
        PB_CUDA(cudaEventElapsedTime(&ma, h.ev[0], h.ev[1]));
        PB_CUDA(cudaEventElapsedTime(&mb, h.ev[1], h.ev[2]));
        us[2 * c] = 1000.0f * ma / reps;
        us[2 * c + 1] = 1000.0f * mb / reps;
        tot[c] = us[2 * c] + us[2 * c + 1];
        if (tot[c] < tot[bi])
            bi = c;
    }
    // the rest of the face stage (finish, the near-field terms): one pass per step, or two steps
    // per pass (candidates 9 and 10), at the chosen block size
    {
        const int FT = kTuneThreads[bi % 3], nb = div_up((long long)nt * 32, FT);
        for (int c = kConv; c < kConv + 2; c++)
        {
            const bool two = c != kConv;
            auto first = [&]() {
                if (two)
                    finish_dry_kernel<R, 1><<<nb, FT, 0, s>>>(L.ring, L.st, 0, nt, L.fa, L.conv);
                else
                    finish_dry_kernel<R, 0><<<nb, FT, 0, s>>>(L.ring, L.st, 0, nt, L.fa, L.conv);
            };
            auto second = [&]() {
                if (two)
                    finish_dry_kernel<R, 2><<<nb, FT, 0, s>>>(L.ring, L.st, 1, nt, L.fa, L.conv);
                else
                    finish_dry_kernel<R, 0><<<nb, FT, 0, s>>>(L.ring, L.st, 1, nt, L.fa, L.conv);
            };
            first();
            second();
            PB_CUDA(cudaEventRecord(h.ev[0], s));
            for (int r = 0; r < reps; r++)
                first();
            PB_CUDA(cudaEventRecord(h.ev[1], s));
            for (int r = 0; r < reps; r++)
                second();
            PB_CUDA(cudaEventRecord(h.ev[2], s));
            PB_CUDA(cudaEventSynchronize(h.ev[2]));
            PB_CHECK_LAUNCH();
            float ma = 0, mb = 0;
            PB_CUDA(cudaEventElapsedTime(&ma, h.ev[0], h.ev[1]));
            PB_CUDA(cudaEventElapsedTime(&mb, h.ev[1], h.ev[2]));
            us[2 * c] = 1000.0f * ma / reps;
            us[2 * c + 1] = 1000.0f * mb / reps;
        }
        h.launches += 4LL * reps + 4;
    }
    h.launches += 2LL * reps * kConv + 2 * kConv + 1;
    h.conv_pairs = bi / 3;
    h.face_threads = kTuneThreads[bi % 3];
    h.terms_pairs = us[2 * kConv + 2] + us[2 * kConv + 3] < us[2 * kConv] + us[2 * kConv + 1];
    *best = bi;
    if (!h.side || h.prm.pml_width > 0)
        return PPPM_OK;  // no two-branch step graphs: the kernel timings decide

    // Phase 2: the kernels compete inside the two-branch step graph (the convolution beside the
    // stencil and the near stage, the finish on the critical path), which isolated launches do not
    // show.  Time kTuneGraphSteps recorded steps (zero accelerations) of every configuration from
    // one device snapshot of the fields and histories: per candidate and rep, restore the snapshot,
    // replay the graph once (warm-up, weights into L2 as in a long run), replay it again timed; keep
    // the fastest of up to 3 reps.  us[2 * PPPM_TUNE_CANDIDATES + i]: microseconds per step of configuration i
    // (conv_pairs = i / 6, threads = {64, 128, 256}[(i / 2) % 3], terms_pairs = i % 2).  The steps
    // write listener rows past the recorded ones, which the next call overwrites; the fields and
    // histories are restored from the snapshot at the end; h.t and the series count do not move.
    // histories: the copies, then the two canonical rings
    const size_t gbytes = (size_t)h.n_cells * h.real_size, cbytes = (size_t)4 * nt * kHistRow * h.real_size,
                 rbytes = (size_t)nt * kRing * h.real_size, hbytes = cbytes + 2 * rbytes;
    const size_t abytes = (size_t)kTuneGraphSteps * nt * sizeof(float);
    void *snap = nullptr;
    PB_TRY(dev_alloc(&snap, 3 * gbytes + hbytes + abytes));
    // zero accelerations for the timed steps (the code paths of a call with accelerations)
    const float *zacc = (const float *)((char *)snap + 3 * gbytes + hbytes);
    PB_CUDA(cudaMemsetAsync((void *)zacc, 0, abytes, s));
    auto copy_state = [&](bool save) -> cudaError_t {
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < 3 && e == cudaSuccess; i++)
            e = save ? cudaMemcpyAsync((char *)snap + i * gbytes, h.grid[i], gbytes, cudaMemcpyDeviceToDevice, s)
                     : cudaMemcpyAsync(h.grid[i], (char *)snap + i * gbytes, gbytes, cudaMemcpyDeviceToDevice, s);
        void *hist[3] = {h.d_hist, h.d_neumann, h.d_dirichlet};
        const size_t hb[3] = {cbytes, rbytes, rbytes};
        char *at = (char *)snap + 3 * gbytes;
        for (int i = 0; i < 3 && e == cudaSuccess; at += hb[i], i++)
            e = save ? cudaMemcpyAsync(at, hist[i], hb[i], cudaMemcpyDeviceToDevice, s)
                     : cudaMemcpyAsync(hist[i], at, hb[i], cudaMemcpyDeviceToDevice, s);
        return e;
    };
    const int keep_pairs = h.conv_pairs, keep_threads = h.face_threads;
    const bool keep_terms = h.terms_pairs;
    int rc = PPPM_OK, gbest = -1;
    float *gus = us + 2 * PPPM_TUNE_CANDIDATES;
    cudaError_t e = copy_state(true);
    StepState sg{h.t + 1, h.n3, h.series_count, zacc};
    sg.series = h.d_series;  // the timed graphs write listener rows past the recorded ones
    // the interior stencil one or four cells per thread (FP32, res % 4 == 0): time the bulk launch
    // (no listeners; the snapshot restore below undoes its writes) both ways and keep the faster
    const int keep_vec4 = h.stencil_vec4;
    if (!h.fp64 && h.res % 4 == 0 && e == cudaSuccess)
    {
        float tv[2] = {0, 0};
        set_state_kernel<<<1, 1, 0, s>>>(h.d_state, sg);
        for (int v = 0; v < 2 && rc == PPPM_OK && e == cudaSuccess; v++)
        {
            h.stencil_vec4 = v;
            StepLaunch<R> S;
            rc = make_launch<R>(h, S);
            if (rc != PPPM_OK)
                break;
            S.a.n_listen = 0;
            StencilSplit bsp = S.sp;
            bsp.skip_corrected = 1;
            const int nb = S.sp.nb_bd + S.sp.nb_in;
            stencil_kernel<R><<<nb, 256, 0, s>>>(S.a, S.ring, S.st, 0, bsp, S.corr_mask);
            e = cudaEventRecord(h.ev[0], s);
            for (int r = 0; r < reps && e == cudaSuccess; r++)
                stencil_kernel<R><<<nb, 256, 0, s>>>(S.a, S.ring, S.st, 0, bsp, S.corr_mask);
            if (e == cudaSuccess)
                e = cudaEventRecord(h.ev[1], s);
            if (e == cudaSuccess)
                e = cudaEventSynchronize(h.ev[1]);
            if (e == cudaSuccess)
                e = cudaEventElapsedTime(&tv[v], h.ev[0], h.ev[1]);
            h.launches += reps + 1;
        }
        h.stencil_vec4 = rc == PPPM_OK && e == cudaSuccess ? (tv[1] < tv[0] ? 1 : 0) : keep_vec4;
    }
    for (int c = 0; c < kTuneConfigs && e == cudaSuccess && rc == PPPM_OK; c++)
    {
        h.conv_pairs = c / 6;
        h.face_threads = kTuneThreads[(c / 2) % 3];
        h.terms_pairs = (c & 1) != 0;
        StepLaunch<R> G;
        rc = make_launch<R>(h, G);
        cudaGraphExec_t exec = nullptr;
        if (rc == PPPM_OK)
            rc = graph_for<R>(h, G, kTuneGraphSteps, &exec);
        if (rc != PPPM_OK)
            break;
        float best_ms = 1e30f;
        for (int r = 0; r <= std::min(reps, 3) && e == cudaSuccess; r++)  // r = 0: warm-up
        {
            e = copy_state(false);
            set_state_kernel<<<1, 1, 0, s>>>(h.d_state, sg);
            if (e == cudaSuccess)
                e = cudaGraphLaunch(exec, s);
            set_state_kernel<<<1, 1, 0, s>>>(h.d_state, sg);
            if (e == cudaSuccess)
                e = cudaEventRecord(h.ev[0], s);
            if (e == cudaSuccess)
                e = cudaGraphLaunch(exec, s);
            if (e == cudaSuccess)
                e = cudaEventRecord(h.ev[1], s);
            if (e == cudaSuccess)
                e = cudaEventSynchronize(h.ev[1]);
            float ms = 0;
            if (e == cudaSuccess && r > 0 && cudaEventElapsedTime(&ms, h.ev[0], h.ev[1]) == cudaSuccess)
                best_ms = std::min(best_ms, ms);
        }
        h.launches += (long long)(std::min(reps, 3) + 1) * 2 * (kTuneGraphSteps * 4 + 1);
        gus[c] = 1000.0f * best_ms / kTuneGraphSteps;
        if (gbest < 0 || gus[c] < gus[gbest])
            gbest = c;
    }
    if (e == cudaSuccess)
        e = copy_state(false);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    dev_free(snap);
    if (rc == PPPM_OK && e != cudaSuccess)
    {
        set_error("autotune: %s", cudaGetErrorString(e));
        rc = PPPM_ERR_CUDA;
    }
    if (rc != PPPM_OK || gbest < 0)
    {
        h.conv_pairs = keep_pairs;
        h.face_threads = keep_threads;
        h.terms_pairs = keep_terms;
        h.stencil_vec4 = keep_vec4;
        return rc;
    }
    h.conv_pairs = gbest / 6;
    h.face_threads = kTuneThreads[(gbest / 2) % 3];
    h.terms_pairs = (gbest & 1) != 0;
    *best = gbest;
    return PPPM_OK;
}

template <typename R>
int prime(Handle &h)
{
    if (!h.mesh_set || h.n3 == 0)
        return PPPM_OK;
    if (!h.d_state)
        PB_TRY(dalloc(&h.d_state, 1));
    // taps t-k of the current time: the FDTD-near sum of step t + 1 into its slot
    StepState stt{h.t, h.n3, 0, nullptr};
    set_state_kernel<<<1, 1, 0, h.stream>>>(h.d_state, stt);

    StepLaunch<R> L;
    PB_TRY(make_launch<R>(h, L));
    L.a.n_listen = 0;
    terms_kernel<R><<<div_up((long long)h.nt * 32, 256), 256, 0, h.stream>>>(L.ring, h.nt, h.t, L.fa);
    near_kernel<R><<<L.near_blocks, 256, 0, h.stream>>>(L.a, L.ring, L.st, 0, L.na, 1);
    h.launches += 3;
    PB_CHECK_LAUNCH();
    return PPPM_OK;
}

// the canonical rings (index = time mod 32) -> the four history copies: the 16 times t-15..t
// that the taps of the next step and the near-field terms of time t reach (the canonical rings
// are current at all times, so nothing flows the other way)
template <typename R>
__global__ void hist_import_kernel(const R *canon_n, const R *canon_d, R *hist, int nt, int t)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long per = (long long)nt * kHist;
    if (i >= 2 * per)
        return;
    const int field = (int)(i / per);
    const long long r = i % per;
    const int tri = (int)(r / kHist), tau = t - (int)(r % kHist);
    const R v = (field ? canon_d : canon_n)[(long long)tri * kRing + (tau & (kRing - 1))];
#pragma unroll
    for (int c = 0; c < 4; c++)
        hist[((long long)c * nt + tri) * kHistRow + Ring<R>::hpos(field, hist_index(c, tau))] = v;
}

template <typename R>
int hist_copy(Handle &h)
{
    if (!h.mesh_set || !h.d_hist)
        return PPPM_OK;
    const long long n = 2ll * h.nt * kHist;
    hist_import_kernel<R><<<div_up(n, 256), 256, 0, h.stream>>>((const R *)h.d_neumann, (const R *)h.d_dirichlet,
                                                                 (R *)h.d_hist, h.nt, h.t);
    h.launches++;
    PB_CHECK_LAUNCH();
    return PPPM_OK;
}

// Per-kernel timing on the current mesh and state: for each step kernel kind, reps back-to-back
// launches recorded as one CUDA graph, replayed once to warm up and once between two events, so a
// launch is timed the way it runs inside the recorded step graphs (its duration plus the gap
// between dependent graph nodes) without event nodes between the kernels.  The launches are those
// of the step after the current time and write only that step's grid slot, history slots and
// scratch sums (listener recording off); prime() then rebuilds the correction that slot must hold,
// so stepping continues as if nothing had run.
template <typename R>
int time_kernels(Handle &h, int reps, float *us)
{
    if (!h.mesh_set || h.prm.method != PPPM_METHOD_PPPM || h.nt == 0 || h.prm.pml_width > 0)
    {
        set_error("kernel timing needs a mesh (PPPM method, absorbing boundary)");
        return PPPM_ERR_STATE;
    }
    if (reps < 1)
        return PPPM_ERR_ARG;
    if (!h.d_state)
        PB_TRY(dalloc(&h.d_state, 1));
    cudaStream_t s = h.stream;
    StepState stt{h.t + 1, h.n3, 0, nullptr};
    set_state_kernel<<<1, 1, 0, s>>>(h.d_state, stt);
    h.launches++;
    StepLaunch<R> L;
    PB_TRY(make_launch<R>(h, L));
    L.a.n_listen = 0;
    const int T = 256, FT = L.face_threads, nt = L.a.nt;
    const int wblocks = div_up((long long)nt * 32, FT);
    for (int k = 0; k < PPPM_KERNEL_KINDS; k++)
        us[k] = 0;
    auto launch = [&](int kind) {
        switch (kind)
        {
        case PPPM_KERNEL_STENCIL:
            stencil_kernel<R><<<L.sp.nb_bd + L.sp.nb_in, T, 0, s>>>(L.a, L.ring, L.st, 0, L.sp, L.corr_mask);
            break;
        case PPPM_KERNEL_CONV: conv_kernel<R><<<wblocks, FT, 0, s>>>(L.ring, L.st, 0, nt, L.fa, L.conv); break;
        case PPPM_KERNEL_CONV2:
            conv2_kernel<R><<<wblocks, FT, 0, s>>>(L.ring, L.st, 0, nt, L.fa, L.conv, L.conv1);
            break;
        case PPPM_KERNEL_FIX: fix_kernel<R><<<wblocks, FT, 0, s>>>(nt, L.fa, L.conv1, L.conv); break;
        case PPPM_KERNEL_FINISH:
            finish_kernel<R, 0><<<wblocks, FT, 0, s>>>(L.ring, L.st, 0, nt, L.fa, L.conv, 0);
            break;
        case PPPM_KERNEL_FINISH1:
            finish_kernel<R, 1><<<wblocks, FT, 0, s>>>(L.ring, L.st, 0, nt, L.fa, L.conv, 0);
            break;
        case PPPM_KERNEL_FINISH2:
            finish_kernel<R, 2><<<wblocks, FT, 0, s>>>(L.ring, L.st, 0, nt, L.fa, L.conv, 0);
            break;
        case PPPM_KERNEL_NEAR: near_kernel<R><<<L.near_blocks, T, 0, s>>>(L.a, L.ring, L.st, 0, L.na, 0); break;
        case PPPM_KERNEL_FACE: face_kernel<R><<<L.face_blocks, T, 0, s>>>(L.a, L.ring, L.st, 0, L.fa); break;
        case PPPM_KERNEL_STENCIL_BULK:
        {
            StencilSplit bsp = L.sp;
            bsp.skip_corrected = 1;
            stencil_kernel<R><<<L.sp.nb_bd + L.sp.nb_in, T, 0, s>>>(L.a, L.ring, L.st, 0, bsp, L.corr_mask);
            break;
        }
        case PPPM_KERNEL_STENCIL_CORR:
            stencil_corr_kernel<R><<<L.corr_blocks, T, 0, s>>>(L.a, L.ring, L.st, 0, L.na.n3_cell);
            break;
        default: break;
        }
    };
    const int kinds[] = {PPPM_KERNEL_STENCIL,      PPPM_KERNEL_CONV,         PPPM_KERNEL_CONV2,
                         PPPM_KERNEL_FIX,          PPPM_KERNEL_FINISH,       PPPM_KERNEL_FINISH1,
                         PPPM_KERNEL_FINISH2,      PPPM_KERNEL_NEAR,         PPPM_KERNEL_FACE,
                         PPPM_KERNEL_STENCIL_BULK, PPPM_KERNEL_STENCIL_CORR};
    // the near kernel also writes the FDTD-near sums of the step after next into the slot two
    // ahead, which is time t-1, a level the next step still reads: kept aside and put back
    const size_t slot_bytes = (size_t)h.n_cells * sizeof(R);
    void *keep = nullptr;
    PB_TRY(dev_alloc(&keep, slot_bytes));
    struct Free
    {
        void *p;
        ~Free() { dev_free(p); }
    } free_keep{keep};
    PB_CUDA(cudaMemcpyAsync(keep, h.slot(h.t - 1), slot_bytes, cudaMemcpyDeviceToDevice, s));
    for (int kind : kinds)
    {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        PB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int r = 0; r < reps; r++)
            launch(kind);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (e == cudaSuccess)
            e = cudaGraphInstantiate(&exec, graph, 0);
        if (graph)
            cudaGraphDestroy(graph);
        if (e == cudaSuccess)
            e = cudaGraphLaunch(exec, s);
        if (e == cudaSuccess)
            e = cudaEventRecord(h.ev[0], s);
        if (e == cudaSuccess)
            e = cudaGraphLaunch(exec, s);
        if (e == cudaSuccess)
            e = cudaEventRecord(h.ev[1], s);
        if (e == cudaSuccess)
            e = cudaEventSynchronize(h.ev[1]);
        float ms = 0;
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&ms, h.ev[0], h.ev[1]);
        if (exec)
            cudaGraphExecDestroy(exec);
        if (e != cudaSuccess)
        {
            set_error("kernel timing failed: %s", cudaGetErrorString(e));
            return PPPM_ERR_CUDA;
        }
        us[kind] = 1000.0f * ms / reps;
        h.launches += 2ll * reps;
    }
    PB_CUDA(cudaMemcpyAsync(h.slot(h.t - 1), keep, slot_bytes, cudaMemcpyDeviceToDevice, s));
    PB_TRY(prime<R>(h));
    PB_CUDA(cudaStreamSynchronize(s));  // the kept slot is freed on return
    return PPPM_OK;
}

}  // namespace

int step_time_kernels(Handle &h, int reps, float *us)
{
    return h.fp64 ? time_kernels<double>(h, reps, us) : time_kernels<float>(h, reps, us);
}

int hist_import(Handle &h) { return h.fp64 ? hist_copy<double>(h) : hist_copy<float>(h); }

int step_prime(Handle &h) { return h.fp64 ? prime<double>(h) : prime<float>(h); }

int step_autotune(Handle &h, int reps, float *us, int *best)
{
    return h.fp64 ? autotune<double>(h, reps, us, best) : autotune<float>(h, reps, us, best);
}

int step_run(Handle &h, const float *acc_dev, int nsteps)
{
    return h.fp64 ? run_steps<double>(h, acc_dev, nsteps) : run_steps<float>(h, acc_dev, nsteps);
}

int step_free(Handle &h)
{
    for (auto *g : {&h.graphs[0], &h.graphs[1], &h.graphs[2], &h.graphs[3], &h.timing_graph, &h.profile_graph})
    {
        if (g->exec)
            cudaGraphExecDestroy(g->exec);
        g->exec = nullptr;
        g->sig.clear();
    }
    dev_free(h.d_state);
    h.d_state = nullptr;
    return PPPM_OK;
}

}  // namespace pb

// ---------------------------------------------------------------- batched scenes -------
//
// Many scenes advance together: one launch of each stage kernel covers every active scene.
// A block finds its scene and its place in that scene's grid in a per-stage block map, then
// runs the same stage code as a single-scene launch on that scene's descriptor, so every
// scene's results are bit-identical to running it alone.  Scenes with fewer steps drop out:
// the run is split into phases with a fixed active set, and each phase replays a recorded
// CUDA graph of G steps (plus a kernel that advances every active scene's step state by G).
namespace pb
{
namespace
{

template <typename R>
struct BatchScene
{
    StepArgs a;
    Ring<R> ring;
    StencilSplit sp;
    const unsigned *corr_mask;
    FaceArgs<R> fa;
    NearArgs<R> na;
    StepState *st;
    R *conv;         // the scene's per-triangle convolution sums (pipelined graphs)
    R *conv1;        // partial sums of the second step of a pair (two steps per pass)
    int near_warps;  // warps of this scene's near grid
    int corr_threads;  // threads of this scene's corrected-cell stencil grid (they stride over the cells)
};

template <typename R>
__global__ void __launch_bounds__(256) batch_stencil_kernel(const BatchScene<R> *sc, const int2 *map, int k,
                                                             int skip_corrected)
{
    const int2 m = map[blockIdx.x];
    const BatchScene<R> &S = sc[m.x];
    StencilSplit sp = S.sp;
    sp.skip_corrected = skip_corrected;
    stencil_body<R>(S.a, S.ring, bind_step(S.st, k, S.a.nt), m.y, sp, S.corr_mask);
}

// the stencil at every active scene's corrected cells (stencil_corr_kernel per scene)
template <typename R>
__global__ void __launch_bounds__(256) batch_corr_kernel(const BatchScene<R> *sc, const int2 *map, int k)
{
    grid_dependency_wait();
    const int2 m = map[blockIdx.x];
    const BatchScene<R> &S = sc[m.x];
    stencil_corr_body<R>(S.a, S.ring, S.st, k, S.na.n3_cell, m.y * 256 + threadIdx.x, S.corr_threads);
}

template <typename R>
__global__ void __launch_bounds__(256) batch_face_kernel(const BatchScene<R> *sc, const int2 *map, int k)
{
    const int2 m = map[blockIdx.x];
    const BatchScene<R> &S = sc[m.x];
    const int tri = m.y * (int)(blockDim.x >> 5) + (int)(threadIdx.x >> 5);
    if (tri < S.a.nt)
        face_body<R>(S.a, S.ring, bind_step(S.st, k, S.a.nt), S.fa, tri, threadIdx.x & 31);
}

template <typename R>
__global__ void __launch_bounds__(256) batch_near_kernel(const BatchScene<R> *sc, const int2 *map, int k)
{
    grid_dependency_wait();
    const int2 m = map[blockIdx.x];
    const BatchScene<R> &S = sc[m.x];
    near_body<R>(S.a, S.ring, bind_step(S.st, k, S.a.nt), S.na, S.st->n3, m.y * 8 + (threadIdx.x >> 5), S.near_warps,
                 threadIdx.x & 31, 0);
}

// the pipelined batch step (see capture_pipelined): face-pair convolutions, the rest of the face
// stage, and the first step's Neumann values, over the same per-scene block maps
// The face-pair convolution of step k of every scene, one pass per step or two steps per pass
// (conv2_kernel / fix_kernel) as the scene's state says: a scene's steps pair up from the first
// step of its batched run (pair0), so the pairs, and the results, are those of the same steps
// run alone in one pppm_step call, wherever the batch's graphs and phases begin and end.
// a scene's step of time t starts a two-step pass over the face pairs (batch_conv_kernel)
__device__ inline bool batch_conv2_at(const StepState &st, int t)
{
    return st.pair_end >= st.pair0 && st.conv_pairs && !((t - st.pair0) & 1) && t + 1 <= st.pair_end;
}

template <typename R>
__global__ void __launch_bounds__(256) batch_conv_kernel(const BatchScene<R> *sc, const int2 *map, int k)
{
    const int2 m = map[blockIdx.x];
    const BatchScene<R> &S = sc[m.x];
    const int w = m.y * (int)(blockDim.x >> 5) + (int)(threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (w >= S.a.nt)
        return;
    const int tri = centre_of(S.fa, w);
    const int tnew = S.st->tnew0 + k, p0 = S.st->pair0, pe = S.st->pair_end;
    const bool paired = pe >= p0 && S.st->conv_pairs;
    if (paired && ((tnew - p0) & 1))
        face_fix<R>(S.fa, S.conv1, S.conv, tri, lane);  // second step of a pair
    else if (batch_conv2_at(*S.st, tnew))
    {
        R c0, c1;
        face_conv2<R>(S.ring, tnew, S.fa, tri, lane, c0, c1);
        if (lane == 0)
        {
            S.conv[tri] = c0;
            S.conv1[tri] = c1;
        }
    }
    else
    {
        const R v = face_conv<R>(S.ring, tnew, S.fa, tri, lane);
        if (lane == 0)
            S.conv[tri] = v;
    }
}

template <typename R>
__global__ void __launch_bounds__(256) batch_finish_kernel(const BatchScene<R> *sc, const int2 *map, int k, int next)
{
    grid_dependency_wait();
    const int2 m = map[blockIdx.x];
    const BatchScene<R> &S = sc[m.x];
    const int tri = m.y * (int)(blockDim.x >> 5) + (int)(threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (tri >= S.a.nt)
        return;
    const StepDyn dy = bind_step(S.st, k, S.a.nt);
    const StepDyn dn = bind_step(S.st, k + 1, S.a.nt);
    // the scene's pairing of steps (batch_conv_kernel)
    const int p0 = S.st->pair0, pe = S.st->pair_end;
    const int mode = pe >= p0 && S.st->terms_pairs && dy.tnew < pe ? (((dy.tnew - p0) & 1) ? 2 : 1) : 0;
    R iw, pv;
    face_corners<R>(S.ring, dy.tnew, S.fa, tri, lane, iw, pv);
    face_finish<R>(S.ring, dy.tnew, S.fa, tri, lane, iw, pv, S.conv[tri], mode,
                   mode == 1 ? next_neumann<R>(S.ring, dn, tri) : (R)0);
    if (next && lane == 0)
        S.ring.nwrite(tri, dn.tnew, dn.acc);
    else if (next && lane == 1 && batch_conv2_at(*S.st, dn.tnew))
        S.ring.stash_next(tri, dn.tnew, bind_step(S.st, k + 2, S.a.nt).acc);
}

template <typename R>
__global__ void batch_nwrite_kernel(const BatchScene<R> *sc, const int2 *map, int k)
{
    const int2 m = map[blockIdx.x];
    const BatchScene<R> &S = sc[m.x];
    const int i = m.y * blockDim.x + threadIdx.x;
    const StepDyn dy = bind_step(S.st, k, S.a.nt);
    if (i < S.a.nt)
    {
        S.ring.nwrite(i, dy.tnew, dy.acc);
        if (batch_conv2_at(*S.st, dy.tnew))
            S.ring.stash_next(i, dy.tnew, bind_step(S.st, k + 1, S.a.nt).acc);
    }
}

// after G steps: every active scene's state moves on by G steps
__global__ void batch_advance_kernel(StepState *const *states, const int *nt, int n, int g)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    StepState *st = states[i];
    st->tnew0 += g;
    st->row0 += g;
    if (st->acc)
        st->acc += (long long)g * nt[i];
}

}  // namespace
}  // namespace pb

namespace pb
{

struct BatchGraph
{
    std::vector<unsigned char> sig;
    cudaGraphExec_t exec = nullptr;
};

constexpr int kBatchGraphSteps = 16;  // steps per replayed graph
constexpr int kBatchGraphs = 16;      // recorded graphs kept per batch

struct Batch
{
    std::vector<Handle *> hs;
    bool fp64 = false;
    cudaStream_t stream = nullptr;  // the first scene's stream
    cudaEvent_t ev = nullptr;
    std::vector<unsigned char> host_scenes;
    // block maps: 0 stencil (with the Neumann range), 1 face (8 triangles per block), 2 near,
    // 3 stencil without the Neumann range, 4 Neumann values (256 triangles per block), 5 the
    // corrected-cell stencil
    std::vector<int2> host_map[6];
    int face_threads = 256;  // block size of the face-stage kernels (the first scene's launch option)
    std::vector<StepState *> host_states;
    std::vector<int> host_nt;
    void *d_scenes = nullptr;
    size_t scenes_cap = 0;
    int2 *d_map[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    size_t map_cap[6] = {0, 0, 0, 0, 0, 0};
    cudaStream_t side = nullptr;                      // second branch while recording
    cudaStream_t side2 = nullptr;                     // third branch: the bulk of the stencil
    cudaEvent_t ev_fin = nullptr, ev_conv = nullptr;  // fork / join points while recording
    cudaEvent_t ev_near = nullptr, ev_bulk = nullptr;
    bool split = true;  // every active scene's step may run split (make_launch's L.split)
    StepState **d_states = nullptr;
    int *d_nt = nullptr;
    size_t states_cap = 0, nt_cap = 0;
    BatchGraph graphs[kBatchGraphs];
    int graph_next = 0;
    long long launches = 0;
};

namespace
{

template <typename T>
int grow(T **p, size_t &cap, size_t need)
{
    if (need <= cap)
        return PPPM_OK;
    dev_free(*p);
    *p = nullptr;
    size_t nc = need + need / 2 + 16;
    PB_TRY(dev_alloc((void **)p, nc * sizeof(T)));
    cap = nc;
    return PPPM_OK;
}

// descriptors, block maps and state pointers of the active scenes, uploaded on b.stream
template <typename R>
int batch_tables(Batch &b, const std::vector<int> &active)
{
    const int T = 256;
    const size_t na = active.size();
    b.host_scenes.assign(na * sizeof(BatchScene<R>), 0);
    b.face_threads = b.hs[active.empty() ? 0 : active[0]]->face_threads;
    for (auto &m : b.host_map)
        m.clear();
    b.host_states.resize(na);
    b.host_nt.resize(na);
    b.split = true;
    for (size_t ai = 0; ai < na; ai++)
    {
        Handle &h = *b.hs[active[ai]];
        StepLaunch<R> L;
        PB_TRY(make_launch<R>(h, L));
        b.split = b.split && L.split;
        BatchScene<R> S;
        memset(&S, 0, sizeof(S));
        S.a = L.a;
        S.ring = L.ring;
        S.sp = L.sp;
        S.corr_mask = L.corr_mask;
        S.fa = L.fa;
        S.na = L.na;
        S.st = h.d_state;
        S.conv = L.conv;
        S.conv1 = L.conv1;
        // near-stage warps stride over the scene's corrected cells (their count is read on the
        // device), so the block map may exceed it: it grows with headroom and never shrinks, so a
        // moving scene, whose count changes at every update_mesh, keeps its recorded batch graphs
        if (h.n3 > h.batch_near_cells)
            h.batch_near_cells = h.n3 + h.n3 / 8 + 256;
        const int near_blocks = std::max(1, div_up((long long)h.batch_near_cells * 32, T));
        S.near_warps = near_blocks * (T / 32);
        const int corr_blocks = std::max(1, div_up((long long)h.batch_near_cells, T));
        S.corr_threads = corr_blocks * T;
        memcpy(b.host_scenes.data() + ai * sizeof(S), &S, sizeof(S));
        for (int k = 0; k < L.stencil_blocks; k++)
            b.host_map[0].push_back(make_int2((int)ai, k));
        for (int k = 0; k < div_up(h.nt, b.face_threads / 32); k++)
            b.host_map[1].push_back(make_int2((int)ai, k));
        for (int k = 0; k < near_blocks; k++)
            b.host_map[2].push_back(make_int2((int)ai, k));
        for (int k = 0; k < L.sp.nb_bd + L.sp.nb_in; k++)
            b.host_map[3].push_back(make_int2((int)ai, k));
        for (int k = 0; k < div_up(h.nt, T); k++)
            b.host_map[4].push_back(make_int2((int)ai, k));
        for (int k = 0; k < corr_blocks; k++)
            b.host_map[5].push_back(make_int2((int)ai, k));
        b.host_states[ai] = h.d_state;
        b.host_nt[ai] = h.nt;
    }
    void *ds = b.d_scenes;
    PB_TRY(grow((unsigned char **)&ds, b.scenes_cap, b.host_scenes.size()));
    b.d_scenes = ds;
    PB_CUDA(cudaMemcpyAsync(b.d_scenes, b.host_scenes.data(), b.host_scenes.size(), cudaMemcpyHostToDevice, b.stream));
    for (int i = 0; i < 6; i++)
    {
        PB_TRY(grow(&b.d_map[i], b.map_cap[i], b.host_map[i].size()));
        PB_CUDA(cudaMemcpyAsync(b.d_map[i], b.host_map[i].data(), b.host_map[i].size() * sizeof(int2),
                                cudaMemcpyHostToDevice, b.stream));
    }
    PB_TRY(grow(&b.d_states, b.states_cap, na));
    PB_TRY(grow(&b.d_nt, b.nt_cap, na));
    PB_CUDA(cudaMemcpyAsync(b.d_states, b.host_states.data(), na * sizeof(StepState *), cudaMemcpyHostToDevice,
                            b.stream));
    PB_CUDA(cudaMemcpyAsync(b.d_nt, b.host_nt.data(), na * sizeof(int), cudaMemcpyHostToDevice, b.stream));
    return PPPM_OK;
}

// the graph of g steps of the active set described by the current tables
template <typename R>
int batch_graph(Batch &b, int g, int nactive, cudaGraphExec_t *out)
{
    std::vector<unsigned char> sig(b.host_scenes);
    const void *ptrs[] = {b.d_scenes, b.d_map[0], b.d_map[1], b.d_map[2], b.d_map[3], b.d_map[4], b.d_map[5],
                          b.d_states, b.d_nt};
    const size_t sizes[] = {b.host_map[0].size(), b.host_map[1].size(), b.host_map[2].size(), b.host_map[3].size(),
                            b.host_map[4].size(), b.host_map[5].size(), (size_t)g, (size_t)nactive,
                            (size_t)b.face_threads, (size_t)b.split};
    sig.insert(sig.end(), (const unsigned char *)ptrs, (const unsigned char *)ptrs + sizeof(ptrs));
    sig.insert(sig.end(), (const unsigned char *)sizes, (const unsigned char *)sizes + sizeof(sizes));
    for (auto &gr : b.graphs)
        if (gr.exec && gr.sig == sig)
        {
            *out = gr.exec;
            return PPPM_OK;
        }
    BatchGraph &gr = b.graphs[b.graph_next];
    b.graph_next = (b.graph_next + 1) % kBatchGraphs;
    if (gr.exec)
        cudaGraphExecDestroy(gr.exec);
    gr.exec = nullptr;
    const BatchScene<R> *sc = (const BatchScene<R> *)b.d_scenes;
    const int n0 = (int)b.host_map[0].size(), n1 = (int)b.host_map[1].size(), n2 = (int)b.host_map[2].size();
    cudaGraph_t graph = nullptr;
    const int n3 = (int)b.host_map[3].size(), n4 = (int)b.host_map[4].size();
    const int FT = b.face_threads;
    PB_CUDA(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal));
    const int n5 = (int)b.host_map[5].size();
    if (n1 > 0 && n4 > 0 && b.side && b.side2)
    {
        // the branches of one scene's recorded steps (capture_pipelined): each step's face-pair
        // convolutions beside the previous near stage, and with the split stencil (every active
        // scene's L.split) the corrected cells' stencil on the main branch (corrected-cell stencil
        // -> finish -> near as dependent launches) and the rest of every grid on a third branch
        cudaStream_t s = b.stream, bulk = b.side2;
        const int2 *m1 = b.d_map[1], *m2 = b.d_map[2], *m5 = b.d_map[5];
        batch_nwrite_kernel<R><<<n4, 256, 0, s>>>(sc, b.d_map[4], 0);
        cudaEventRecord(b.ev_fin, s);
        cudaEventRecord(b.ev_near, s);
        for (int k = 0; k < g; k++)
        {
            cudaStreamWaitEvent(b.side, b.ev_fin, 0);
            batch_conv_kernel<R><<<n1, FT, 0, b.side>>>(sc, m1, k);
            cudaEventRecord(b.ev_conv, b.side);
            if (b.split)
            {
                if (k > 0)
                    cudaStreamWaitEvent(s, b.ev_bulk, 0);  // bulk(k-1)
                cudaStreamWaitEvent(bulk, b.ev_near, 0);   // near(k-1), or the graph's start
                batch_stencil_kernel<R><<<n3, 256, 0, bulk>>>(sc, b.d_map[3], k, 1);
                cudaEventRecord(b.ev_bulk, bulk);
                launch_dependent(batch_corr_kernel<R>, n5, 256, s, sc, m5, k);
            }
            else
                // the whole stencil but its Neumann block range (finish / nwrite wrote N[t])
                batch_stencil_kernel<R><<<n3, 256, 0, s>>>(sc, b.d_map[3], k, 0);
            cudaStreamWaitEvent(s, b.ev_conv, 0);
            launch_dependent(batch_finish_kernel<R>, n1, FT, s, sc, m1, k, k + 1 < g ? 1 : 0);
            cudaEventRecord(b.ev_fin, s);
            if (n2 > 0)
                launch_dependent(batch_near_kernel<R>, n2, 256, s, sc, m2, k);
            cudaEventRecord(b.ev_near, s);
        }
        if (b.split)
            cudaStreamWaitEvent(s, b.ev_bulk, 0);
    }
    else
        for (int k = 0; k < g; k++)
        {
            batch_stencil_kernel<R><<<n0, 256, 0, b.stream>>>(sc, b.d_map[0], k, 0);
            if (n1 > 0)
                batch_face_kernel<R><<<n1, FT, 0, b.stream>>>(sc, b.d_map[1], k);
            if (n2 > 0)
                batch_near_kernel<R><<<n2, 256, 0, b.stream>>>(sc, b.d_map[2], k);
        }
    batch_advance_kernel<<<div_up(nactive, 128), 128, 0, b.stream>>>(b.d_states, b.d_nt, nactive, g);
    cudaError_t e = cudaStreamEndCapture(b.stream, &graph);
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(&gr.exec, graph, 0);
    if (graph)
        cudaGraphDestroy(graph);
    if (e != cudaSuccess)
    {
        gr.exec = nullptr;
        set_error("recording the batch graph failed: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    gr.sig.swap(sig);
    *out = gr.exec;
    return PPPM_OK;
}

template <typename R>
int batch_run_t(Batch &b, const float *const *dacc, const int *nsteps)
{
    const int n = (int)b.hs.size();
    // work queued on the scenes' own streams comes first
    for (Handle *h : b.hs)
        if (h->stream != b.stream)
        {
            PB_CUDA(cudaEventRecord(b.ev, h->stream));
            PB_CUDA(cudaStreamWaitEvent(b.stream, b.ev, 0));
        }
    for (int i = 0; i < n; i++)
    {
        Handle &h = *b.hs[i];
        if (!h.d_state)
            PB_TRY(dalloc(&h.d_state, 1));
        StepState stt{h.t + 1, h.n3, h.series_count, dacc[i]};
        stt.series = h.d_series;
        // the scene's steps pair up as in one pppm_step call of nsteps[i] steps (recorded graphs:
        // at least kGraphSteps steps)
        stt.pair0 = h.t + 1;
        stt.pair_end = nsteps[i] >= kGraphSteps ? h.t + nsteps[i] : h.t;
        stt.conv_pairs = h.conv_pairs ? 1 : 0;
        stt.terms_pairs = h.terms_pairs ? 1 : 0;
        set_state_kernel<<<1, 1, 0, b.stream>>>(h.d_state, stt);
        b.launches++;
    }
    PB_CHECK_LAUNCH();
    std::vector<int> ends;
    for (int i = 0; i < n; i++)
        if (nsteps[i] > 0)
            ends.push_back(nsteps[i]);
    std::sort(ends.begin(), ends.end());
    ends.erase(std::unique(ends.begin(), ends.end()), ends.end());
    int done = 0;
    for (int end : ends)
    {
        std::vector<int> active;
        for (int i = 0; i < n; i++)
            if (nsteps[i] > done)
                active.push_back(i);
        PB_TRY(batch_tables<R>(b, active));
        int left = end - done;
        while (left > 0)
        {
            const int g = std::min(left, kBatchGraphSteps);
            cudaGraphExec_t exec = nullptr;
            PB_TRY(batch_graph<R>(b, g, (int)active.size(), &exec));
            PB_CUDA(cudaGraphLaunch(exec, b.stream));
            // pipelined graphs: conv, bulk stencil, corrected-cell stencil, finish and near per step,
            // plus the Neumann write and the state advance; otherwise stencil, face and near
            const bool piped = !b.host_map[1].empty() && !b.host_map[4].empty() && b.side && b.side2;
            b.launches += piped ? (b.split ? 5ll : 4ll) * g + 2 : 3ll * g + 1;
            left -= g;
        }
        done = end;
    }
    for (int i = 0; i < n; i++)
    {
        Handle &h = *b.hs[i];
        h.t += nsteps[i];
        h.series_count += nsteps[i];
        h.launches += 3ll * nsteps[i];
    }
    // later work on the scenes' streams waits for the batch
    PB_CUDA(cudaEventRecord(b.ev, b.stream));
    for (Handle *h : b.hs)
        if (h->stream != b.stream)
            PB_CUDA(cudaStreamWaitEvent(h->stream, b.ev, 0));
    return PPPM_OK;
}

}  // namespace

int batch_create(Handle **hs, int n, Batch **out)
{
    *out = nullptr;
    if (!hs || n <= 0)
        return PPPM_ERR_ARG;
    for (int i = 0; i < n; i++)
    {
        if (!hs[i] || !hs[i]->mesh_set)
        {
            set_error("batch scene %d has no mesh", i);
            return PPPM_ERR_STATE;
        }
        if (hs[i]->prm.pml_width > 0 || hs[i]->fp64 != hs[0]->fp64 || hs[i]->prm.device != hs[0]->prm.device ||
            hs[i]->prm.method != PPPM_METHOD_PPPM)
        {
            set_error("batch scenes must share device and precision and use the absorbing boundary and the "
                      "PPPM method (scene %d)", i);
            return PPPM_ERR_ARG;
        }
        for (int j = 0; j < i; j++)
            if (hs[j] == hs[i])
            {
                set_error("scene %d appears twice in the batch", i);
                return PPPM_ERR_ARG;
            }
    }
    Batch *b = new (std::nothrow) Batch();
    if (!b)
        return PPPM_ERR_NOMEM;
    b->hs.assign(hs, hs + n);
    b->fp64 = hs[0]->fp64;
    b->stream = hs[0]->stream;
    if (cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fin, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_conv, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_near, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_bulk, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->side2, cudaStreamNonBlocking) != cudaSuccess)
    {
        delete b;
        set_error("cudaEventCreate failed");
        return PPPM_ERR_CUDA;
    }
    *out = b;
    return PPPM_OK;
}

int batch_run(Batch *b, const float *const *dacc, const int *nsteps)
{
    cudaSetDevice(b->hs[0]->prm.device);
    return b->fp64 ? batch_run_t<double>(*b, dacc, nsteps) : batch_run_t<float>(*b, dacc, nsteps);
}

void batch_destroy(Batch *b)
{
    if (!b)
        return;
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    for (auto &g : b->graphs)
        if (g.exec)
            cudaGraphExecDestroy(g.exec);
    dev_free(b->d_scenes);
    for (auto *m : b->d_map)
        dev_free(m);
    dev_free(b->d_states);
    dev_free(b->d_nt);
    if (b->ev)
        cudaEventDestroy(b->ev);
    if (b->ev_fin)
        cudaEventDestroy(b->ev_fin);
    if (b->ev_conv)
        cudaEventDestroy(b->ev_conv);
    if (b->ev_near)
        cudaEventDestroy(b->ev_near);
    if (b->ev_bulk)
        cudaEventDestroy(b->ev_bulk);
    if (b->side)
        cudaStreamDestroy(b->side);
    if (b->side2)
        cudaStreamDestroy(b->side2);
    delete b;
}

}  // namespace pb
