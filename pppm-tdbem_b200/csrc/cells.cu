// Cell classification and fresh-cell fill for moving rigid bodies.
//
// Reference semantics (src/algorithm/ghost_cell_util.cu, ghost_cell.cu):
//   nearest       for each cell, the nearest point over the triangles binned within +-3
//                 cells (first strict minimum in visiting order), its reflection through the
//                 surface, and the side from the angle-weighted vertex normal interpolated at
//                 the nearest point: SOLID if (normal . (centre - point)) <= 0, else AIR;
//                 UNKNOWN when no triangle is in range (ghost_cell_util.cu:7-118)
//   ghost         SOLID with an AIR 6-neighbour (labels before the sweep) -> GHOST (:120-155)
//   sweep         per (x, y) column along z: cells before the first labelled one take its
//                 label, later UNKNOWN cells take the last SOLID/AIR state (:157-189)
//   ghost index   inclusive scan of the pre-sweep GHOST flags, minus one, for cells GHOST
//                 after the sweep (:191-230)
//   fresh cells   old label != AIR and new label == AIR: pressure at t and t-1 from the
//                 inverse-square-distance mean of the 8 cells around the reflection point
//                 that are AIR in both labelings, minus rho * a * |xf - xr|; without such a
//                 cell, the nearest doubly-AIR cell of the 4^3 block (ghost_cell.cu:51-205)
// The nearest point on a triangle is Eberly's region-based closest-point algorithm
// ("Distance from a Point to a Triangle", Geometric Tools), in the same branch structure and
// arithmetic as the reference's helper (core/helper_math.h:1634-1786) so labels match bit for
// bit.  The fresh-cell pass reads only doubly-AIR neighbours, never another fresh cell, so
// it is race-free; cell lists are compacted with warp ballots.
#include "handle.cuh"

namespace pb
{

namespace
{
enum
{
    AIR = 0,
    SOLID = 1,
    GHOST = 2,
    UNKNOWN = 3
};

struct f2
{
    float x, y;
};

__device__ inline f2 min_edge02(float a11, float b1)
{
    int a = b1 < 0, b = a11 + b1 <= 0;
    return f2{0.0f, a * (b - (1 - b) * (b1 / a11))};
}

__device__ inline f2 min_edge12(float a01, float a11, float b1, float f10, float f01)
{
    float h0 = a01 + b1 - f10, h1 = a11 + b1 - f01;
    int a = h0 < 0, b = h1 <= 0;
    float y = a * (b + (1 - b) * h0 / (h0 - h1));
    return f2{1 - y, y};
}

__device__ inline f2 min_interior(f2 p0, float h0, f2 p1, float h1)
{
    float z = h0 / (h0 - h1);
    float omz = 1 - z;
    return f2{omz * p0.x + z * p1.x, omz * p0.y + z * p1.y};
}

// barycentric weights (w0, w1, w2) of the point of triangle v0 v1 v2 nearest to p
__device__ inline f3 nearest_coeff(f3 p, f3 v0, f3 v1, f3 v2)
{
    f3 diff = p - v0, e0 = v1 - v0, e1 = v2 - v0;
    float a00 = dot3(e0, e0), a01 = dot3(e0, e1), a11 = dot3(e1, e1), b0 = -dot3(diff, e0), b1 = -dot3(diff, e1);
    float f00 = b0, f10 = b0 + a00, f01 = b0 + a01;
    f2 p0{0, 0}, p1{0, 0}, q{0, 0};
    float dt1 = 0, h0 = 0, h1 = 0;
    if (f00 >= 0)
    {
        if (f01 >= 0)
            q = min_edge02(a11, b1);
        else
        {
            p0 = f2{0, f00 / (f00 - f01)};
            p1.x = f01 / (f01 - f10);
            p1.y = 1 - p1.x;
            dt1 = p1.y - p0.y;
            h0 = dt1 * (a11 * p0.y + b1);
            if (h0 >= 0)
                q = min_edge02(a11, b1);
            else
            {
                h1 = dt1 * (a01 * p1.x + a11 * p1.y + b1);
                q = h1 <= 0 ? min_edge12(a01, a11, b1, f10, f01) : min_interior(p0, h0, p1, h1);
            }
        }
    }
    else if (f01 <= 0)
    {
        if (f10 <= 0)
            q = min_edge12(a01, a11, b1, f10, f01);
        else
        {
            p0 = f2{f00 / (f00 - f10), 0.0f};
            p1.x = f01 / (f01 - f10);
            p1.y = 1 - p1.x;
            h0 = p1.y * (a01 * p0.x + b1);
            if (h0 >= 0)
                q = p0;
            else
            {
                h1 = p1.y * (a01 * p1.x + a11 * p1.y + b1);
                q = h1 <= 0 ? min_edge12(a01, a11, b1, f10, f01) : min_interior(p0, h0, p1, h1);
            }
        }
    }
    else if (f10 <= 0)
    {
        p0 = f2{0.0f, f00 / (f00 - f01)};
        p1.x = f01 / (f01 - f10);
        p1.y = 1 - p1.x;
        dt1 = p1.y - p0.y;
        h0 = dt1 * (a11 * p0.y + b1);
        if (h0 >= 0)
            q = min_edge02(a11, b1);
        else
        {
            h1 = dt1 * (a01 * p1.x + a11 * p1.y + b1);
            q = h1 <= 0 ? min_edge12(a01, a11, b1, f10, f01) : min_interior(p0, h0, p1, h1);
        }
    }
    else
    {
        p0 = f2{f00 / (f00 - f10), 0.0f};
        p1.x = 0.0f;
        p1.y = f00 / (f00 - f01);
        h0 = p1.y * (a01 * p0.x + b1);
        if (h0 >= 0)
            q = p0;
        else
        {
            h1 = p1.y * (a11 * p1.y + b1);
            q = h1 <= 0 ? min_edge02(a11, b1) : min_interior(p0, h0, p1, h1);
        }
    }
    return f3{1 - q.x - q.y, q.x, q.y};
}

// vertex -> incident faces CSR (faces ascending), built once per set_mesh
__global__ void vf_count_kernel(const int *tris, int nt, int *count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt)
        return;
    for (int k = 0; k < 3; k++)
        atomicAdd(&count[tris[3 * i + k]], 1);
}
__global__ void vf_fill_kernel(const int *tris, int nt, const int *start, int *cursor, int *list)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt)
        return;
    for (int k = 0; k < 3; k++)
    {
        int v = tris[3 * i + k];
        list[start[v] + atomicAdd(&cursor[v], 1)] = i;
    }
}
__global__ void vf_sort_kernel(const int *start, int nv, int *list)
{
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv)
        return;
    int b = start[v], e = start[v + 1];
    for (int i = b + 1; i < e; i++)
    {
        int x = list[i], j = i - 1;
        while (j >= b && list[j] > x)
        {
            list[j + 1] = list[j];
            j--;
        }
        list[j + 1] = x;
    }
}

__device__ inline f3 vertex_normal(int v, const float *verts, const int *tris, const float *normal, const int *vf_start,
                                   const int *vf_list)
{
    f3 acc{0, 0, 0};
    f3 pv = load3(verts, v);
    for (int j = vf_start[v]; j < vf_start[v + 1]; j++)
    {
        int f = vf_list[j];
        int vs[2], n = 0;
        for (int k = 0; k < 3; k++)
        {
            int u = tris[3 * f + k];
            if (u != v && n < 2)
                vs[n++] = u;
        }
        f3 e1 = load3(verts, vs[0]) - pv, e2 = load3(verts, vs[1]) - pv;
        float ang = acosf(dot3(e1, e2) / (len3(e1) * len3(e2)));
        acc = acc + load3(normal, f) * ang;
    }
    return normalize3(acc);
}

__global__ void nearest_kernel(int res, float h, f3 mn, const float *verts, const int *tris, const float *normal,
                               const int *cell_start, const int *cell_tris, const int *vf_start, const int *vf_list,
                               int thin, int *type, int *nearest, float *points)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)res * res * res;
    if (i >= n)
        return;
    int x = (int)(i / ((long long)res * res)), y = (int)((i / res) % res), z = (int)(i % res);
    f3 gc = cell_center(x, y, z, h, mn);
    float best = 3.402823466e+38F;
    int bi = -1;
    f3 bp{0, 0, 0}, bco{0, 0, 0};
    for (int dx = -3; dx <= 3; dx++)
        for (int dy = -3; dy <= 3; dy++)
            for (int dz = -3; dz <= 3; dz++)
            {
                int cx = x + dx, cy = y + dy, cz = z + dz;
                if (cx < 0 || cx >= res || cy < 0 || cy >= res || cz < 0 || cz >= res)
                    continue;
                int c = (cx * res + cy) * res + cz;
                for (int j = cell_start[c]; j < cell_start[c + 1]; j++)
                {
                    int f = cell_tris[j];
                    f3 v0 = load3(verts, tris[3 * f]), v1 = load3(verts, tris[3 * f + 1]),
                       v2 = load3(verts, tris[3 * f + 2]);
                    f3 co = nearest_coeff(gc, v0, v1, v2);
                    f3 np = co.x * v0 + co.y * v1 + co.z * v2;
                    float l = len3(gc - np);
                    if (l < best)
                    {
                        best = l;
                        bp = np;
                        bi = f;
                        bco = co;
                    }
                }
            }
    int ty = UNKNOWN;
    f3 refl{0, 0, 0};
    if (bi >= 0)
    {
        refl = 2 * bp - gc;
        f3 nv[3];
        for (int k = 0; k < 3; k++)
            nv[k] = vertex_normal(tris[3 * bi + k], verts, tris, normal, vf_start, vf_list);
        f3 nn = bco.x * nv[0] + bco.y * nv[1] + bco.z * nv[2];
        float dir = dot3(nn, gc - bp);
        // thin shell (first-order ghost cells): a centre within half a cell of its nearest point
        // on every axis is SOLID too (ghost_cell_util.cu:101-103)
        const f3 dv = bp - gc;
        const bool shell = thin && fabsf(dv.x) < h / 2 && fabsf(dv.y) < h / 2 && fabsf(dv.z) < h / 2;
        ty = (dir <= 0 || shell) ? SOLID : AIR;
    }
    type[i] = ty;
    nearest[i] = bi;
    float *pt = points + 7 * i;
    pt[0] = bp.x;
    pt[1] = bp.y;
    pt[2] = bp.z;
    pt[3] = refl.x;
    pt[4] = refl.y;
    pt[5] = refl.z;
    pt[6] = bi >= 0 ? best : 3.402823466e+38F;
}

__global__ void ghost_kernel(int res, const int *type_in, int *type_out, int *flag)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)res * res * res;
    if (i >= n)
        return;
    int x = (int)(i / ((long long)res * res)), y = (int)((i / res) % res), z = (int)(i % res);
    int ty = type_in[i];
    if (ty == SOLID)
    {
        int nb[6][3] = {{x + 1, y, z}, {x - 1, y, z}, {x, y + 1, z}, {x, y - 1, z}, {x, y, z + 1}, {x, y, z - 1}};
        for (int k = 0; k < 6; k++)
        {
            int a = nb[k][0], b = nb[k][1], c = nb[k][2];
            if (a < 0 || a >= res || b < 0 || b >= res || c < 0 || c >= res)
                continue;
            if (type_in[((long long)a * res + b) * res + c] == AIR)
                ty = GHOST;
        }
    }
    type_out[i] = ty;
    flag[i] = ty == GHOST;
}

__global__ void sweep_kernel(int res, int *type)
{
    int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= res * res)
        return;
    int *t = type + (long long)col * res;
    int cur = AIR;
    bool found = false;
    for (int z = 0; z < res; z++)
    {
        if (!found && t[z] != UNKNOWN)
        {
            found = true;
            cur = t[z];
            for (int k = 0; k < z; k++)
                t[k] = cur;
            continue;
        }
        int v = t[z];
        if (v == SOLID || v == GHOST)
            cur = SOLID;
        else if (v == AIR)
            cur = AIR;
        else
            t[z] = cur;
    }
}

// ghost index from the exclusive scan of the flags: inclusive(c) - 1 = excl(c) + flag(c) - 1
__global__ void ghost_index_kernel(long long n, const int *type, const int *flag, const int *excl, int *ghost)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    ghost[i] = type[i] == GHOST ? excl[i] + flag[i] - 1 : -1;
}

// fresh cells, compacted with warp ballots into a global list (order is irrelevant: each
// fresh cell writes only itself)
__global__ void fresh_list_kernel(long long n, const int *old_type, const int *new_type, int *list, int *count)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool fresh = i < n && old_type[i] != AIR && new_type[i] == AIR;
    unsigned m = __ballot_sync(0xffffffffu, fresh);
    int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0 && m)
        base = atomicAdd(count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (fresh)
        list[base + __popc(m & ((1u << lane) - 1))] = (int)i;
}

__global__ void fresh_fill_kernel(int res, float h, f3 mn, float rho, const int *list, const int *count,
                                  const int *old_type, const int *new_type, const int *nearest, const float *points,
                                  const float *acc, const float *acc_old, float *g_t, float *g_tm1)
{
    int li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= *count)
        return;
    int c = list[li];
    int x = c / (res * res), y = (c / res) % res, z = c % res;
    int nf = nearest[c];
    float accs[2] = {acc[nf], acc_old[nf]};
    float *gs[2] = {g_t, g_tm1};
    f3 xb{points[7 * c], points[7 * c + 1], points[7 * c + 2]};
    f3 xf = cell_center(x, y, z, h, mn);
    f3 xr = xb + 2 * (xf - xb);
    f3 rel = (xr - mn) / h;
    int gx = (int)rel.x, gy = (int)rel.y, gz = (int)rel.z;
    f3 d = xr - cell_center(gx, gy, gz, h, mn);
    int bx = gx - (d.x < 0), by = gy - (d.y < 0), bz = gz - (d.z < 0);
    auto inb = [&](int a, int b, int cc) { return a >= 0 && b >= 0 && cc >= 0 && a < res && b < res && cc < res; };
    auto both_air = [&](int a, int b, int cc) {
        long long q = ((long long)a * res + b) * res + cc;
        return old_type[q] == AIR && new_type[q] == AIR;
    };
    int nb[8];
    float co[8];
    bool found = false;
    for (int dx = 0; dx < 2; dx++)
        for (int dy = 0; dy < 2; dy++)
            for (int dz = 0; dz < 2; dz++)
            {
                int a = bx + dx, b = by + dy, cc = bz + dz, w = dx * 4 + dy * 2 + dz;
                nb[w] = inb(a, b, cc) ? (a * res + b) * res + cc : -1;
                if (nb[w] >= 0 && both_air(a, b, cc))
                {
                    float dist = len3(cell_center(a, b, cc, h, mn) - xr);
                    co[w] = 1.0 / (dist * dist + 1e-8f);
                    found = true;
                }
                else
                    co[w] = 0;
            }
    if (!found)
    {
        float md = 1e10, pr1 = 0, pr2 = 0;
        for (int dx = -1; dx < 3; dx++)
            for (int dy = -1; dy < 3; dy++)
                for (int dz = -1; dz < 3; dz++)
                {
                    int a = bx + dx, b = by + dy, cc = bz + dz;
                    if (!inb(a, b, cc) || !both_air(a, b, cc))
                        continue;
                    float dist = len3(cell_center(a, b, cc, h, mn) - xr);
                    if (dist < md)
                    {
                        md = dist;
                        long long q = ((long long)a * res + b) * res + cc;
                        pr1 = g_t[q];
                        pr2 = g_tm1[q];
                    }
                }
        g_t[c] = pr1;
        g_tm1[c] = pr2;
        return;
    }
    float sum = 0;
    for (int i = 0; i < 8; i++)
        sum += co[i];
    for (int i = 0; i < 8; i++)
        co[i] /= sum;
    for (int s = 0; s < 2; s++)
    {
        float pr = 0;
        for (int j = 0; j < 8; j++)
            if (nb[j] >= 0)
                pr += co[j] * gs[s][nb[j]];
        gs[s][c] = pr - rho * accs[s] * len3(xf - xr);
    }
}

}  // namespace

static int build_vertex_faces(Handle &h, int **start, int **list)
{
    cudaStream_t s = h.stream;
    int *count = nullptr, *cursor = nullptr;
    PB_TRY(dalloc(&count, (size_t)h.nv + 1));
    PB_TRY(dalloc(&cursor, (size_t)h.nv + 1));
    PB_TRY(dalloc(start, (size_t)h.nv + 1));
    PB_TRY(dalloc(list, 3 * (size_t)h.nt));
    PB_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (h.nv + 1), s));
    PB_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int) * (h.nv + 1), s));
    vf_count_kernel<<<div_up(h.nt, 256), 256, 0, s>>>(h.d_tris, h.nt, count);
    PB_TRY(exclusive_scan(h, count, *start, h.nv));
    vf_fill_kernel<<<div_up(h.nt, 256), 256, 0, s>>>(h.d_tris, h.nt, *start, cursor, *list);
    vf_sort_kernel<<<div_up(h.nv, 256), 256, 0, s>>>(*start, h.nv, *list);
    h.launches += 3;
    PB_CHECK_LAUNCH();
    PB_CUDA(cudaStreamSynchronize(s));
    dev_free(count);
    dev_free(cursor);
    return PPPM_OK;
}

int cells_classify(Handle &h, int *ghost_count)
{
    if (!h.mesh_set)
        return PPPM_ERR_STATE;
    if (h.fp64)
    {
        set_error("cell labels operate on FP32 handles");
        return PPPM_ERR_ARG;
    }
    cudaStream_t s = h.stream;
    const long long n = h.n_cells;
    const int T = 256;
    if (!h.d_cell_type)
    {
        PB_TRY(dalloc(&h.d_cell_type, (size_t)n));
        PB_TRY(dalloc(&h.d_cell_type_old, (size_t)n));
        PB_TRY(dalloc(&h.d_cell_nearest, (size_t)n));
        PB_TRY(dalloc(&h.d_cell_ghost, (size_t)n + 1));
        PB_TRY(dalloc(&h.d_cell_points, 7 * (size_t)n));
        PB_CUDA(cudaMemsetAsync(h.d_cell_type, 0, sizeof(int) * n, s));  // all AIR before the first labelling
    }
    int *vf_start = nullptr, *vf_list = nullptr;
    PB_TRY(build_vertex_faces(h, &vf_start, &vf_list));
    // keep the previous labels for the fresh-cell pass
    PB_CUDA(cudaMemcpyAsync(h.d_cell_type_old, h.d_cell_type, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    const f3 mn{h.prm.min_pos[0], h.prm.min_pos[1], h.prm.min_pos[2]};
    int *raw = h.d_flags, *flag = h.d_flags + (n + 1), *excl = h.d_flags + 2 * (n + 1);
    nearest_kernel<<<div_up(n, T), T, 0, s>>>(h.res, h.prm.dl, mn, h.d_verts, h.d_tris, h.d_normal, h.d_cell_start,
                                              h.d_cell_tris, vf_start, vf_list,
                                              h.prm.method == PPPM_METHOD_GHOST && h.prm.ghost_threshold <= 0, raw,
                                              h.d_cell_nearest, h.d_cell_points);
    ghost_kernel<<<div_up(n, T), T, 0, s>>>(h.res, raw, h.d_cell_type, flag);
    sweep_kernel<<<div_up((long long)h.res * h.res, T), T, 0, s>>>(h.res, h.d_cell_type);
    h.launches += 3;
    PB_CHECK_LAUNCH();
    PB_TRY(exclusive_scan(h, flag, excl, n));
    ghost_index_kernel<<<div_up(n, T), T, 0, s>>>(n, h.d_cell_type, flag, excl, h.d_cell_ghost);
    h.launches++;
    PB_CHECK_LAUNCH();
    int total = 0;
    PB_TRY(read_int(h, excl + n, &total));
    h.ghost_count = total;
    if (ghost_count)
        *ghost_count = total;
    dev_free(vf_start);
    dev_free(vf_list);
    return PPPM_OK;
}

int cells_fresh(Handle &h, const float *acc, const float *acc_old, int *fresh_count)
{
    if (!h.mesh_set || !h.d_cell_type)
        return PPPM_ERR_STATE;
    float *dacc = nullptr, *dold = nullptr;
    PB_TRY(dalloc(&dacc, (size_t)h.nt));
    PB_TRY(dalloc(&dold, (size_t)h.nt));
    PB_CUDA(cudaMemcpyAsync(dacc, acc, sizeof(float) * h.nt, cudaMemcpyHostToDevice, h.stream));
    PB_CUDA(cudaMemcpyAsync(dold, acc_old, sizeof(float) * h.nt, cudaMemcpyHostToDevice, h.stream));
    const int rc = cells_fresh_dev(h, dacc, dold, fresh_count);
    dev_free(dacc);
    dev_free(dold);
    return rc;
}

int cells_fresh_dev(Handle &h, const float *dacc, const float *dold, int *fresh_count)
{
    if (!h.mesh_set || !h.d_cell_type)
        return PPPM_ERR_STATE;
    cudaStream_t s = h.stream;
    const long long n = h.n_cells;
    int *list = h.d_flags, *count = h.d_flags + (n + 1);
    PB_CUDA(cudaMemsetAsync(count, 0, sizeof(int), s));
    fresh_list_kernel<<<div_up(n, 256), 256, 0, s>>>(n, h.d_cell_type_old, h.d_cell_type, list, count);
    const f3 mn{h.prm.min_pos[0], h.prm.min_pos[1], h.prm.min_pos[2]};
    fresh_fill_kernel<<<div_up(n, 256), 256, 0, s>>>(h.res, h.prm.dl, mn, h.prm.rho, list, count, h.d_cell_type_old,
                                                     h.d_cell_type, h.d_cell_nearest, h.d_cell_points, dacc, dold,
                                                     (float *)h.slot(h.t), (float *)h.slot(h.t - 1));
    h.launches += 2;
    PB_CHECK_LAUNCH();
    int cnt = 0;
    PB_TRY(read_int(h, count, &cnt));
    if (fresh_count)
        *fresh_count = cnt;
    return PPPM_OK;
}

}  // namespace pb
