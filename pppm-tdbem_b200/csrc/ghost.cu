// Ghost-cell method: the reference's GhostCellSolver (ghost_cell.cu:220-545, svd.cu, sparse.cu)
// as an alternative to the TDBEM correction.  Cells are labelled AIR / SOLID / GHOST (cells.cu);
// every step the FDTD update runs on the whole grid, then the pressure of each GHOST cell is set
// so that the surface's Neumann condition holds, and SOLID cells are zeroed.
//
// Per geometry (set_mesh / update_mesh), one thread per ghost cell:
//   * its interpolation box: the 8 cells around the reflection of the cell centre through the
//     surface (base = int((reflect - min) / h - 0.5)), in coordinates normalised to [-1, 1]^3;
//   * the 8 x 8 matrix Phi of the trilinear basis [xyz, xy, yz, xz, x, y, z, 1] at the 8 box
//     cells; the row of the ghost cell itself (when it is in its own box) holds the normal
//     derivative of the basis at the nearest surface point instead (ghost_cell.cu:257-303);
//   * Phi = U S V^T by a one-sided Jacobi SVD in FP64 (the reference: cuSOLVER gesvda in FP32);
//     condition number S_max / S_min above the threshold (25) -> first order, else the
//     reflection-point weights w = (Phi^+)^T phi(r) = U S^-1 V^T phi(r) (ghost_cell.cu:305-354);
//   * the row of the sparse system: 1 on the diagonal, -w_i for box cells that are ghosts.
// Per step, one block: the right-hand side from the new pressure and this step's accelerations
// (ghost_cell.cu:356-470), BiCGSTAB from the previous solution (the reference's settings: at most
// 100 iterations, residual 1e-6 of the initial one; no ILU0 preconditioner), the ghost pressures
// written into the grid, SOLID cells zeroed, the listener samples re-read.  Threshold 0 selects
// the first-order method everywhere: thin-shell labelling and no linear system.
#include "fdtd.cuh"
#include "ghost.cuh"

namespace pb
{

struct Ghost
{
    int count = 0, nsolid = 0;
    long long cap = 0, solid_cap = 0;
    int *d_cell = nullptr;    // [count] linear cell index
    int *d_order = nullptr;   // [count] 1 = first order
    float *d_w = nullptr;     // [count][8] reflection-point weights
    int *d_col = nullptr;     // [count][9] sparse row: columns (-1 = empty), diagonal last
    float *d_val = nullptr;   // [count][9]
    float *d_b = nullptr;     // right-hand side
    float *d_x = nullptr;     // solution, kept as the next step's initial guess
    float *d_work = nullptr;  // [6][count] BiCGSTAB vectors
    int *d_solid = nullptr;   // SOLID cells
    int *d_iters = nullptr;   // iterations of the last solve (diagnostics)
};

namespace
{
constexpr int kBox = 8;
constexpr int kRow = kBox + 1;

__device__ inline int3 box_offset(int i) { return make_int3(i % 2, (i / 2) % 2, i / 4); }

// one-sided Jacobi SVD of an 8 x 8 matrix (row-major a): a = U diag(s) V^T, U in a on return
__device__ void svd8(double a[kBox][kBox], double v[kBox][kBox], double s[kBox])
{
    for (int i = 0; i < kBox; i++)
        for (int j = 0; j < kBox; j++)
            v[i][j] = i == j;
    for (int sweep = 0; sweep < 40; sweep++)
    {
        double off = 0;
        for (int p = 0; p < kBox - 1; p++)
            for (int q = p + 1; q < kBox; q++)
            {
                double alpha = 0, beta = 0, gamma = 0;
                for (int i = 0; i < kBox; i++)
                {
                    alpha += a[i][p] * a[i][p];
                    beta += a[i][q] * a[i][q];
                    gamma += a[i][p] * a[i][q];
                }
                if (gamma == 0 || fabs(gamma) <= 1e-15 * sqrt(alpha * beta))
                    continue;
                off = fmax(off, fabs(gamma) / sqrt(alpha * beta));
                const double zeta = (beta - alpha) / (2 * gamma);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1 + zeta * zeta));
                const double c = 1 / sqrt(1 + t * t), sn = c * t;
                for (int i = 0; i < kBox; i++)
                {
                    const double ap = a[i][p], aq = a[i][q];
                    a[i][p] = c * ap - sn * aq;
                    a[i][q] = sn * ap + c * aq;
                    const double vp = v[i][p], vq = v[i][q];
                    v[i][p] = c * vp - sn * vq;
                    v[i][q] = sn * vp + c * vq;
                }
            }
        if (off < 1e-15)
            break;
    }
    for (int j = 0; j < kBox; j++)
    {
        double n = 0;
        for (int i = 0; i < kBox; i++)
            n += a[i][j] * a[i][j];
        s[j] = sqrt(n);
        if (s[j] > 0)
            for (int i = 0; i < kBox; i++)
                a[i][j] /= s[j];
    }
}


__device__ inline int3 reflect_base(const float *pt, const GhostGeo &g)
{
    // make_int3 of a float3 truncates toward zero (ghost_cell.cu:20-24)
    return make_int3((int)((pt[3] - g.mn.x) / g.h - 0.5f), (int)((pt[4] - g.mn.y) / g.h - 0.5f),
                     (int)((pt[5] - g.mn.z) / g.h - 0.5f));
}

// (p - centre(base)) / h * 2 - 1
__device__ inline f3 normalised(f3 p, int3 base, const GhostGeo &g)
{
    const f3 bc = cell_center(base.x, base.y, base.z, g.h, g.mn);
    return (p - bc) / g.h * 2.0f + mk(-1, -1, -1);
}

__global__ void ghost_list_kernel(long long n, const int *ghost_idx, int *cells)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && ghost_idx[i] >= 0)
        cells[ghost_idx[i]] = (int)i;
}

__global__ void solid_flag_kernel(long long n, const int *type, int *flag)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        flag[i] = type[i] == 1;  // SOLID
}

__global__ void solid_list_kernel(long long n, const int *flag, const int *pos, int *list)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && flag[i])
        list[pos[i]] = (int)i;
}

// the interpolation weights and the sparse row of every ghost cell
__global__ void ghost_matrix_kernel(GhostGeo g, int count, float threshold, const int *cells, const int *type,
                                    const int *ghost_idx, const float *points, int *order, float *w, int *col,
                                    float *val)
{
    const int gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= count)
        return;
    const int c = cells[gi];
    const int res = g.res;
    const int3 me = make_int3(c / (res * res), (c / res) % res, c % res);
    const float *pt = points + 7 * (long long)c;
    const f3 np = mk(pt[0], pt[1], pt[2]), rp = mk(pt[3], pt[4], pt[5]);
    const f3 nrm = normalize3(rp - np);
    const int3 base = reflect_base(pt, g);
    double phi[kBox][kBox];
    for (int i = 0; i < kBox; i++)
    {
        const int3 d = box_offset(i);
        const bool self = base.x + d.x == me.x && base.y + d.y == me.y && base.z + d.z == me.z;
        float r[kBox];
        if (self)
        {
            // normal derivative of the basis at the nearest surface point
            const f3 q = normalised(np, base, g);
            r[0] = dot3(nrm, mk(q.y * q.z, q.x * q.z, q.x * q.y));
            r[1] = dot3(nrm, mk(q.y, q.x, 0));
            r[2] = dot3(nrm, mk(0, q.z, q.y));
            r[3] = dot3(nrm, mk(q.z, 0, q.x));
            r[4] = dot3(nrm, mk(1, 0, 0));
            r[5] = dot3(nrm, mk(0, 1, 0));
            r[6] = dot3(nrm, mk(0, 0, 1));
            r[7] = 0;
        }
        else
        {
            const float x = (float)(d.x * 2 - 1), y = (float)(d.y * 2 - 1), z = (float)(d.z * 2 - 1);
            r[0] = x * y * z;
            r[1] = x * y;
            r[2] = y * z;
            r[3] = x * z;
            r[4] = x;
            r[5] = y;
            r[6] = z;
            r[7] = 1;
        }
        for (int k = 0; k < kBox; k++)
            phi[i][k] = r[k];
    }
    for (int k = 0; k < kRow; k++)
    {
        col[(long long)gi * kRow + k] = -1;
        val[(long long)gi * kRow + k] = 0;
    }
    col[(long long)gi * kRow + kBox] = gi;  // diagonal
    val[(long long)gi * kRow + kBox] = 1;
    double v[kBox][kBox], s[kBox];
    svd8(phi, v, s);
    double smax = 0, smin = 1e308;
    for (int k = 0; k < kBox; k++)
    {
        smax = fmax(smax, s[k]);
        smin = fmin(smin, s[k]);
    }
    // a box reaching outside the grid has no second-order stencil (the reference reads there)
    const bool inside = base.x >= 0 && base.y >= 0 && base.z >= 0 && base.x + 1 < res && base.y + 1 < res &&
                        base.z + 1 < res;
    bool first = !inside || !(smin > 0) || smax / smin > threshold;
    double wd[kBox];
    if (!first)
    {
        const f3 r = normalised(rp, base, g);
        const double pr[kBox] = {(double)(r.x * r.y * r.z), (double)(r.x * r.y), (double)(r.y * r.z),
                                 (double)(r.x * r.z),        (double)r.x,         (double)r.y,
                                 (double)r.z,                1.0};
        double vt[kBox];  // S^-1 V^T phi(r)
        for (int k = 0; k < kBox; k++)
        {
            double acc = 0;
            for (int j = 0; j < kBox; j++)
                acc += v[j][k] * pr[j];
            vt[k] = acc / s[k];
        }
        for (int i = 0; i < kBox; i++)
        {
            double acc = 0;
            for (int k = 0; k < kBox; k++)
                acc += phi[i][k] * vt[k];  // phi holds U now
            wd[i] = acc;
            if (!isfinite(acc))
                first = true;
        }
    }
    order[gi] = first ? 1 : 0;
    for (int i = 0; i < kBox; i++)
        w[(long long)gi * kBox + i] = first ? 0.0f : (float)wd[i];
    if (first)
        return;
    for (int i = 0; i < kBox; i++)
    {
        const int3 d = box_offset(i);
        const int nb = ((base.x + d.x) * res + (base.y + d.y)) * res + (base.z + d.z);
        if (type[nb] == 2 && ghost_idx[nb] != gi)  // another GHOST cell: a matrix entry
        {
            col[(long long)gi * kRow + i] = ghost_idx[nb];
            val[(long long)gi * kRow + i] = -(float)wd[i];
        }
    }
}


__device__ inline float block_sum(float v, float *red)
{
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();  // red is free
    if (lane == 0)
        red[warp] = v;
    __syncthreads();
    float t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++)
        t += red[i];
    return t;
}

__device__ inline void spmv(const GhostStep &a, const float *in, float *out)
{
    for (int r = threadIdx.x; r < a.count; r += blockDim.x)
    {
        float acc = 0;
        for (int k = 0; k < kRow; k++)
        {
            const int c = a.col[(long long)r * kRow + k];
            if (c >= 0)
                acc += a.val[(long long)r * kRow + k] * in[c];
        }
        out[r] = acc;
    }
    __syncthreads();
}

// one step of the ghost-cell method after the FDTD update (one block; tnew: the new time level)
__global__ void __launch_bounds__(1024) ghost_step_kernel(const __grid_constant__ GhostStep a, const StepState *st,
                                                          int kstep, int nt)
{
    __shared__ float red[32];
    const StepDyn dy = bind_step(st, kstep, nt);
    float *series = (float *)dy.series;
    float *p = a.grid[((dy.tnew % 3) + 3) % 3];
    const float *acc = dy.acc;
    const int G = a.count, res = a.g.res;
    const float hh = a.g.h;
    // right-hand side (ghost_cell.cu:356-470)
    for (int gi = threadIdx.x; gi < G; gi += blockDim.x)
    {
        const int c = a.cells[gi];
        const int near_tri = a.nearest[c];
        const float an = acc && near_tri >= 0 ? acc[near_tri] : 0.0f;
        const int3 me = make_int3(c / (res * res), (c / res) % res, c % res);
        float bv = 0;
        if (a.first_only || a.order[gi])
        {
            const int d6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
            int nn = 0;
            for (int k = 0; k < 6; k++)
            {
                const int nx = me.x + d6[k][0], ny = me.y + d6[k][1], nz = me.z + d6[k][2];
                if (nx < 0 || ny < 0 || nz < 0 || nx >= res || ny >= res || nz >= res)
                    continue;
                const int nb = (nx * res + ny) * res + nz;
                if (a.type[nb] == 0)  // AIR
                {
                    bv += -an * hh + p[nb];
                    nn++;
                }
            }
            bv /= nn;
        }
        else
        {
            const float *pt = a.points + 7 * (long long)c;
            const int3 base = reflect_base(pt, a.g);
            bv += -an * pt[6] * 2;
            for (int i = 0; i < kBox; i++)
            {
                const int3 d = box_offset(i);
                const int nb = ((base.x + d.x) * res + (base.y + d.y)) * res + (base.z + d.z);
                const float wi = a.w[(long long)gi * kBox + i];
                if (a.ghost_idx[nb] == gi)
                    bv += wi * (hh / 2 * an);
                else if (a.type[nb] != 2)
                    bv += wi * p[nb];
            }
        }
        a.b[gi] = bv;
    }
    __syncthreads();
    int it = 0;
    if (!a.first_only)
    {
        // BiCGSTAB (sparse.cu:140-300 without the ILU0 preconditioner), x from the previous step
        float *r0 = a.work, *r = a.work + G, *pv = a.work + 2 * G, *v = a.work + 3 * G, *s = a.work + 4 * G,
              *t = a.work + 5 * G;
        spmv(a, a.x, v);
        float part = 0;
        for (int i = threadIdx.x; i < G; i += blockDim.x)
        {
            const float ri = a.b[i] - v[i];
            r0[i] = ri;
            r[i] = ri;
            part += ri * ri;
        }
        float delta = block_sum(part, red), delta_prev = delta;
        const float threshold = 1e-6f * sqrtf(delta);
        float alpha = 0, omega = 1;
        if (delta > 0)
            for (it = 1; it <= 100; it++)
            {
                if (it > 1)
                {
                    part = 0;
                    for (int i = threadIdx.x; i < G; i += blockDim.x)
                        part += r0[i] * r[i];
                    delta = block_sum(part, red);
                    const float beta = (delta / delta_prev) * (alpha / omega);
                    delta_prev = delta;
                    for (int i = threadIdx.x; i < G; i += blockDim.x)
                        pv[i] = r[i] + beta * (pv[i] - omega * v[i]);
                }
                else
                    for (int i = threadIdx.x; i < G; i += blockDim.x)
                        pv[i] = r[i];
                __syncthreads();
                spmv(a, pv, v);
                part = 0;
                for (int i = threadIdx.x; i < G; i += blockDim.x)
                    part += r0[i] * v[i];
                alpha = delta / block_sum(part, red);
                if (!isfinite(alpha))  // breakdown: keep the current iterate
                    break;
                part = 0;
                for (int i = threadIdx.x; i < G; i += blockDim.x)
                {
                    a.x[i] += alpha * pv[i];
                    const float si = r[i] - alpha * v[i];
                    s[i] = si;
                    part += si * si;
                }
                const float nrm_s = sqrtf(block_sum(part, red));
                if (!(nrm_s >= threshold))  // converged (or no longer finite)
                    break;
                spmv(a, s, t);
                float pn = 0, pd = 0;
                for (int i = threadIdx.x; i < G; i += blockDim.x)
                {
                    pn += t[i] * s[i];
                    pd += t[i] * t[i];
                }
                const float on = block_sum(pn, red), od = block_sum(pd, red);
                omega = on / od;
                if (!isfinite(omega))
                    break;
                for (int i = threadIdx.x; i < G; i += blockDim.x)
                {
                    a.x[i] += omega * s[i];
                    r[i] = s[i] - omega * t[i];
                }
                __syncthreads();
            }
    }
    // ghost pressures into the grid, SOLID cells zeroed (ghost_cell.cu:472-561)
    const float *sol = a.first_only ? a.b : a.x;
    for (int gi = threadIdx.x; gi < G; gi += blockDim.x)
        p[a.cells[gi]] = sol[gi];
    for (int i = threadIdx.x; i < a.nsolid; i += blockDim.x)
        p[a.solid[i]] = 0;
    __syncthreads();
    if (threadIdx.x < a.n_listen && series)
        series[dy.row * a.n_listen + threadIdx.x] = p[a.listen_cell[threadIdx.x]];
    if (threadIdx.x == 0 && a.iters)
        *a.iters = it;
}

}  // namespace

int ghost_build(Handle &h)
{
    if (!h.ghost)
    {
        h.ghost = new (std::nothrow) Ghost();
        if (!h.ghost)
            return PPPM_ERR_NOMEM;
    }
    Ghost &G = *h.ghost;
    cudaStream_t s = h.stream;
    const long long n = h.n_cells;
    const int T = 256;
    const int count = h.ghost_count;
    if (count > G.cap)
    {
        void **ptrs[] = {(void **)&G.d_cell, (void **)&G.d_order, (void **)&G.d_w, (void **)&G.d_col,
                         (void **)&G.d_val,  (void **)&G.d_b,     (void **)&G.d_x, (void **)&G.d_work};
        for (void **q : ptrs)
        {
            dev_free(*q);
            *q = nullptr;
        }
        const long long cap = count + count / 2 + 64;
        PB_TRY(dalloc(&G.d_cell, (size_t)cap));
        PB_TRY(dalloc(&G.d_order, (size_t)cap));
        PB_TRY(dalloc(&G.d_w, (size_t)cap * kBox));
        PB_TRY(dalloc(&G.d_col, (size_t)cap * kRow));
        PB_TRY(dalloc(&G.d_val, (size_t)cap * kRow));
        PB_TRY(dalloc(&G.d_b, (size_t)cap));
        PB_TRY(dalloc(&G.d_x, (size_t)cap));
        PB_TRY(dalloc(&G.d_work, (size_t)cap * 6));
        PB_CUDA(cudaMemsetAsync(G.d_x, 0, sizeof(float) * cap, s));
        G.cap = cap;
    }
    if (!G.d_iters)
        PB_TRY(dalloc(&G.d_iters, 1));
    G.count = count;
    if (count > 0)
        PB_CUDA(cudaMemsetAsync(G.d_x, 0, sizeof(float) * count, s));
    if (count > 0)
    {
        ghost_list_kernel<<<div_up(n, T), T, 0, s>>>(n, h.d_cell_ghost, G.d_cell);
        h.launches++;
        const GhostGeo g{h.res, h.prm.dl, f3{h.prm.min_pos[0], h.prm.min_pos[1], h.prm.min_pos[2]}};
        ghost_matrix_kernel<<<div_up(count, 128), 128, 0, s>>>(g, count, h.prm.ghost_threshold, G.d_cell,
                                                               h.d_cell_type, h.d_cell_ghost, h.d_cell_points,
                                                               G.d_order, G.d_w, G.d_col, G.d_val);
        h.launches++;
        PB_CHECK_LAUNCH();
    }
    // SOLID cells, zeroed after every step
    int *flag = h.d_flags, *pos = h.d_flags + (n + 1);
    solid_flag_kernel<<<div_up(n, T), T, 0, s>>>(n, h.d_cell_type, flag);
    h.launches++;
    PB_TRY(exclusive_scan(h, flag, pos, n));
    int nsolid = 0;
    PB_TRY(read_int(h, pos + n, &nsolid));
    if (nsolid > G.solid_cap)
    {
        dev_free(G.d_solid);
        G.d_solid = nullptr;
        PB_TRY(dalloc(&G.d_solid, (size_t)nsolid + 64));
        G.solid_cap = nsolid + 64;
    }
    solid_list_kernel<<<div_up(n, T), T, 0, s>>>(n, flag, pos, G.d_solid);
    h.launches++;
    PB_CHECK_LAUNCH();
    G.nsolid = nsolid;
    return PPPM_OK;
}

// the arguments of the per-step ghost kernel (part of the step launch set)
GhostStep ghost_args(Handle &h, int n_listen, const int *listen_cell)
{
    Ghost &G = *h.ghost;
    GhostStep a;
    memset(&a, 0, sizeof(a));
    a.g = GhostGeo{h.res, h.prm.dl, f3{h.prm.min_pos[0], h.prm.min_pos[1], h.prm.min_pos[2]}};
    for (int i = 0; i < 3; i++)
        a.grid[i] = (float *)h.grid[i];
    a.count = G.count;
    a.nsolid = G.nsolid;
    a.first_only = h.prm.ghost_threshold <= 0 ? 1 : 0;
    a.n_listen = n_listen;
    for (int l = 0; l < n_listen && l < 8; l++)
        a.listen_cell[l] = listen_cell[l];
    a.cells = G.d_cell;
    a.order = G.d_order;
    a.col = G.d_col;
    a.type = h.d_cell_type;
    a.ghost_idx = h.d_cell_ghost;
    a.nearest = h.d_cell_nearest;
    a.solid = G.d_solid;
    a.w = G.d_w;
    a.val = G.d_val;
    a.points = h.d_cell_points;
    a.b = G.d_b;
    a.x = G.d_x;
    a.work = G.d_work;
    a.iters = G.d_iters;
    return a;
}

void ghost_launch(const GhostStep &a, const StepState *st, int kstep, int nt, cudaStream_t s)
{
    ghost_step_kernel<<<1, 1024, 0, s>>>(a, st, kstep, nt);
}

int ghost_read(Handle &h, int what, void *dst, size_t bytes)
{
    if (!h.ghost)
        return PPPM_ERR_STATE;
    Ghost &G = *h.ghost;
    const void *src = nullptr;
    size_t need = 0;
    switch (what)
    {
    case 0: src = G.d_cell; need = (size_t)G.count * sizeof(int); break;
    case 1: src = G.d_order; need = (size_t)G.count * sizeof(int); break;
    case 2: src = G.d_w; need = (size_t)G.count * kBox * sizeof(float); break;
    case 3: src = G.d_iters; need = sizeof(int); break;
    default: return PPPM_ERR_ARG;
    }
    if (!dst)
        return PPPM_ERR_ARG;
    if (bytes < need)
        return PPPM_ERR_ARG;
    if (need)
        PB_CUDA(cudaMemcpyAsync(dst, src, need, cudaMemcpyDeviceToHost, h.stream));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

void ghost_free(Handle &h)
{
    if (!h.ghost)
        return;
    Ghost &G = *h.ghost;
    void *ptrs[] = {G.d_cell, G.d_order, G.d_w, G.d_col, G.d_val, G.d_b, G.d_x, G.d_work, G.d_solid, G.d_iters};
    for (void *q : ptrs)
        dev_free(q);
    delete h.ghost;
    h.ghost = nullptr;
}

}  // namespace pb
