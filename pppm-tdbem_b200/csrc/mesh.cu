// Mesh-side structures of one scene, rebuilt on every set_mesh / update_mesh:
// triangle geometry, per-cell and per-base-cell triangle lists (CSR, triangle ids ascending
// inside a cell, so the lists are deterministic), the corrected-cell set with its 3^3
// triangle pairs, the non-empty base cells with their 4^3 lists, and per-triangle face
// pair lists with interpolation corners.
//
// Reference semantics followed (src/algorithm/particle_grid.{h,cu}):
//   triangle record       particle_grid.cu:40-88 (centre = (v0+v1+v2)/3, normal =
//                         normalize(cross), area = |cross|/2, grid coord by truncation,
//                         base coord = coord - (centre < cell centre))
//   3^3 list of a cell    particle_grid.cu:139-182: cells in [1, res-2]^3 whose 27-cell block
//                         holds a triangle, sub-cells visited x fastest
//   4^3 list of a base    particle_grid.cu:184-223: base cells in [1, res-2]^3 with a
//                         non-empty base list, block (-1..2)^3, x fastest
// The reference fills lists by atomic append, so its in-cell order varies run to run; the
// sets are identical.
#include "handle.cuh"

namespace pb
{

namespace
{
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// up to kScanBatch independent scans in one launch (blockIdx.y selects the array)
constexpr int kScanBatch = 4;
struct ScanSet
{
    const int *in[kScanBatch];
    int *out[kScanBatch];
    int *sums[kScanBatch];  // per-tile totals, or null for single-tile arrays
    long long n_in[kScanBatch], n_out[kScanBatch];
};

__global__ void scan_tiles_kernel(const __grid_constant__ ScanSet set)
{
    const int a = blockIdx.y;
    const long long n_in = set.n_in[a], n_out = set.n_out[a];
    if ((long long)blockIdx.x * kScanTile >= n_out)
        return;  // block-uniform: this array has fewer tiles
    const int *in = set.in[a];
    int *out = set.out[a], *tile_sums = set.sums[a];
    __shared__ int warp_tot[kScanThreads / 32];
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++)
    {
        long long idx = base + i;
        v[i] = (idx < n_in) ? in[idx] : 0;
        sum += v[i];
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off)
            x += y;
    }
    if (lane == 31)
        warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        int w = (lane < kScanThreads / 32) ? warp_tot[lane] : 0;
        int s = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            int y = __shfl_up_sync(0xffffffffu, s, off);
            if (lane >= off)
                s += y;
        }
        if (lane < kScanThreads / 32)
            warp_tot[lane] = s - w;
        if (lane == kScanThreads / 32 - 1 && tile_sums)
            tile_sums[blockIdx.x] = s;
    }
    __syncthreads();
    int run = x - sum + warp_tot[warp];
#pragma unroll
    for (int i = 0; i < kScanItems; i++)
    {
        long long idx = base + i;
        if (idx < n_out)
            out[idx] = run;
        run += v[i];
    }
}

__global__ void scan_add_kernel(const __grid_constant__ ScanSet set)
{
    const int a = blockIdx.y;
    const long long n_out = set.n_out[a];
    if ((long long)blockIdx.x * kScanTile >= n_out || !set.sums[a])
        return;
    int *out = set.out[a];
    long long base = (long long)blockIdx.x * kScanTile;
    int add = set.in[a][blockIdx.x];  // scanned tile totals
    for (int i = threadIdx.x; i < kScanTile; i += blockDim.x)
    {
        long long idx = base + i;
        if (idx < n_out)
            out[idx] += add;
    }
}

__device__ inline void flag_error(int *status, int code) { atomicCAS(status, 0, code); }

// ---- triangle geometry (particle_grid.cu:40-88 without the incremental list moves)
__global__ void geometry_kernel(const float *verts, const int *tris, int nt, int res, float h, f3 mn, float *center,
                                float *normal, float *area, int *cellc, int *basec, int *cell, int *base, int *status)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt)
        return;
    f3 v0 = load3(verts, tris[3 * i]), v1 = load3(verts, tris[3 * i + 1]), v2 = load3(verts, tris[3 * i + 2]);
    f3 c = (v0 + v1 + v2) / 3.0f;
    f3 e = cross3(v1 - v0, v2 - v0);
    f3 n = normalize3(e);
    float a = len3(e) / 2.0f;
    f3 rel = (c - mn) / h;
    int gx = (int)rel.x, gy = (int)rel.y, gz = (int)rel.z;
    f3 cc = cell_center(gx, gy, gz, h, mn);
    f3 d = c - cc;
    int bx = gx - (d.x < 0), by = gy - (d.y < 0), bz = gz - (d.z < 0);
    store3(center, i, c);
    store3(normal, i, n);
    area[i] = a;
    cellc[3 * i] = gx;
    cellc[3 * i + 1] = gy;
    cellc[3 * i + 2] = gz;
    basec[3 * i] = bx;
    basec[3 * i + 1] = by;
    basec[3 * i + 2] = bz;
    // every structure below reads up to two cells around a triangle: keep triangles at
    // least two cells inside the grid (the reference reads those cells without checks)
    bool ok = gx >= 2 && gy >= 2 && gz >= 2 && gx <= res - 3 && gy <= res - 3 && gz <= res - 3 && bx >= 1 &&
              by >= 1 && bz >= 1 && bx <= res - 3 && by <= res - 3 && bz <= res - 3 && isfinite(c.x) &&
              isfinite(c.y) && isfinite(c.z);
    if (!ok)
    {
        flag_error(status, PPPM_ERR_ARG);
        cell[i] = -1;
        base[i] = -1;
        return;
    }
    cell[i] = (gx * res + gy) * res + gz;
    base[i] = (bx * res + by) * res + bz;
    // status[1]: a triangle within three cells of the grid's faces, so that a corrected cell (its
    // 3^3 block) may be the inward neighbour of a boundary-layer cell that is not corrected; that
    // cell's 4x4 solve reads p^{t-1} at the corrected cell, which the split step's near stage
    // overwrites beside it (make_launch records the step unsplit then)
    if (gx <= 3 || gy <= 3 || gz <= 3 || gx >= res - 4 || gy >= res - 4 || gz >= res - 4)
        atomicExch(status + 1, 1);
}

__global__ void count_kernel(const int *key, int n, int *count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && key[i] >= 0)
        atomicAdd(&count[key[i]], 1);
}

__global__ void fill_kernel(const int *key, int n, const int *start, int *cursor, int *list)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && key[i] >= 0)
        list[start[key[i]] + atomicAdd(&cursor[key[i]], 1)] = i;
}

// sort each cell's segment ascending (segments are short: a few to ~100 entries)
__global__ void sort_segments_kernel(const int *start, long long n_cells, int *list)
{
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells)
        return;
    int b = start[c], e = start[c + 1];
    for (int i = b + 1; i < e; i++)
    {
        int v = list[i], j = i - 1;
        while (j >= b && list[j] > v)
        {
            list[j + 1] = list[j];
            j--;
        }
        list[j + 1] = v;
    }
}

__device__ inline int cell_len(const int *start, int res, int x, int y, int z)
{
    if (x < 0 || y < 0 || z < 0 || x >= res || y >= res || z >= res)
        return 0;
    int c = (x * res + y) * res + z;
    return start[c + 1] - start[c];
}

// corrected-cell flags and 3^3 counts; base-cell flags and 4^3 counts
__global__ void block_counts_kernel(const int *cell_start, const int *base_start, int res, int *flag3, int *len3,
                                    int *flag4, int *len4)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)res * res * res;
    if (i >= n)
        return;
    int x = (int)(i / ((long long)res * res)), y = (int)((i / res) % res), z = (int)(i % res);
    bool inner = x >= 1 && y >= 1 && z >= 1 && x <= res - 2 && y <= res - 2 && z <= res - 2;
    int s3 = 0, s4 = 0;
    if (inner)
    {
        for (int dx = -1; dx <= 1; dx++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dz = -1; dz <= 1; dz++)
                    s3 += cell_len(cell_start, res, x + dx, y + dy, z + dz);
    }
    bool has_base = inner && (base_start[i + 1] - base_start[i]) > 0;
    if (has_base)
    {
        for (int dx = -1; dx <= 2; dx++)
            for (int dy = -1; dy <= 2; dy++)
                for (int dz = -1; dz <= 2; dz++)
                    s4 += cell_len(cell_start, res, x + dx, y + dy, z + dz);
    }
    flag3[i] = s3 > 0;
    len3[i] = s3;
    flag4[i] = has_base;
    len4[i] = s4;
}

// flagged cells i < n -> out_cell[pos[i]] = i, out_start[pos[i]] = start[i]; out_start[pos[n]] =
// start[n] closes the list (pos and start: exclusive scans over the n cells of the flags and of
// the list lengths, which are 0 for cells that are not flagged)
__global__ void compact_kernel(const int *flag, const int *pos, const int *start, long long n, int *out_cell,
                               int *out_start)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == n)
        out_start[pos[n]] = start[n];
    if (i >= n || !flag[i])
        return;
    out_cell[pos[i]] = (int)i;
    out_start[pos[i]] = start[i];
}

// 3^3 pairs of each corrected cell, sub-cells x fastest (particle_grid.cu:164-182);
// woff = GridCache weight index of (cell - triangle cell) (pppm_cache.h:38-42)
__global__ void fill_pairs3_kernel(const int *n3_cell, const int *n3_start, int n3, int res, const int *cell_start,
                                   const int *cell_tris, int *p3_tri, unsigned char *p3_woff, unsigned *mask)
{
    // one warp per corrected cell: lane l < 27 copies sub-cell l's list to its offset in the
    // cell's list (a warp prefix sum over the 27 lengths keeps the sub-cell order)
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= n3)
        return;
    const int i = (int)gw;
    const int c = n3_cell[i];
    const int x = c / (res * res), y = (c / res) % res, z = c % res;
    int b = 0, len = 0;
    unsigned char woff = 0;
    if (lane < 27)
    {
        const int dx = lane % 3 - 1, dy = lane / 3 % 3 - 1, dz = lane / 9 - 1;
        const int sc = ((x + dx) * res + (y + dy)) * res + (z + dz);
        woff = (unsigned char)((1 - dx) + 3 * (1 - dy) + 9 * (1 - dz));
        b = cell_start[sc];
        len = cell_start[sc + 1] - b;
    }
    int incl = len;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off)
            incl += v;
    }
    const int o = n3_start[i] + incl - len;
    for (int j = 0; j < len; j++)
    {
        p3_tri[o + j] = cell_tris[b + j];
        p3_woff[o + j] = woff;
    }
    if (lane == 0)
        atomicOr(&mask[c >> 5], 1u << (c & 31));
}

// 4^3 lists of the non-empty base cells (particle_grid.cu:198-223)
__global__ void fill_n4_kernel(const int *b4_cell, const int *b4_start, int b4, int res, const int *cell_start,
                               const int *cell_tris, int *n4_tris)
{
    // one warp per base cell: lane l copies sub-cells l and l + 32 (x fastest, then y, then z)
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= b4)
        return;
    const int i = (int)gw;
    const int c = b4_cell[i];
    const int x = c / (res * res), y = (c / res) % res, z = c % res;
    int b[2], len[2];
#pragma unroll
    for (int half = 0; half < 2; half++)
    {
        const int idx = lane + 32 * half;
        const int sx = x + idx % 4 - 1, sy = y + idx / 4 % 4 - 1, sz = z + idx / 16 - 1;
        b[half] = 0;
        len[half] = 0;
        if (sx >= 0 && sy >= 0 && sz >= 0 && sx < res && sy < res && sz < res)
        {
            const int sc = (sx * res + sy) * res + sz;
            b[half] = cell_start[sc];
            len[half] = cell_start[sc + 1] - b[half];
        }
    }
    int o = b4_start[i];
#pragma unroll
    for (int half = 0; half < 2; half++)
    {
        int incl = len[half];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const int v = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off)
                incl += v;
        }
        const int mine = o + incl - len[half];
        for (int j = 0; j < len[half]; j++)
            n4_tris[mine + j] = cell_tris[b[half] + j];
        o += __shfl_sync(0xffffffffu, incl, 31);
    }
}

// per centre triangle: length of its base cell's 4^3 list
__global__ void face_len_kernel(const int *base, int nt, const int *b4_pos, const int *b4_flag, const int *b4_start,
                                int *face_len)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt)
        return;
    int b = base[i];
    if (b < 0 || !b4_flag[b])
    {
        face_len[i] = 0;
        return;
    }
    int k = b4_pos[b];
    face_len[i] = b4_start[k + 1] - b4_start[k];
}

__global__ void face_fill_kernel(const int *base, const int *basec, int nt, int res, const int *b4_pos,
                                 const int *b4_flag, const int *b4_start, const int *n4_tris, const int *face_start,
                                 int *face_nbr, int *face_corner)
{
    // one warp per centre triangle: its 8 trilinear corner cells and a copy of its base cell's
    // 4^3 list (lanes stride over the list)
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= nt)
        return;
    const int i = (int)gw;
    const int b = base[i];
    if (lane < 8)
    {
        const int bx = basec[3 * i], by = basec[3 * i + 1], bz = basec[3 * i + 2];
        const int dx = lane >> 2, dy = (lane >> 1) & 1, dz = lane & 1;
        face_corner[8 * i + lane] = ((bx + dx) * res + (by + dy)) * res + (bz + dz);
    }
    if (b < 0 || !b4_flag[b])
        return;
    const int k = b4_pos[b];
    const int o = face_start[i], s0 = b4_start[k], n = b4_start[k + 1] - s0;
    for (int j = lane; j < n; j += 32)
        face_nbr[o + j] = n4_tris[s0 + j];
}

}  // namespace

int read_int(Handle &h, const int *d, int *out)
{
    PB_CUDA(cudaMemcpyAsync(out, d, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

int read_ints(Handle &h, const int *const *src, int n, int *out)
{
    if (n > kPinnedInts)
        return PPPM_ERR_ARG;
    for (int i = 0; i < n; i++)
        PB_CUDA(cudaMemcpyAsync(h.h_pin + i, src[i], sizeof(int), cudaMemcpyDeviceToHost, h.stream));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    for (int i = 0; i < n; i++)
        out[i] = h.h_pin[i];
    return PPPM_OK;
}

// Exclusive prefix sums of up to kScanBatch arrays at once: out_i[0..n_i] = scan of in_i[0..n_i),
// out_i[n_i] = total.  Three launches per level for the whole set (tiles, the tile totals
// recursively, tile offsets added).  Scratch: h.d_scan_tmp.
static int scan_level(Handle &h, ScanSet set, int count, int *scratch, long long scratch_left)
{
    ScanSet up{};  // the tile totals of every multi-tile array
    ScanSet add{};
    long long nb_max = 0;
    int multi = 0;
    for (int i = 0; i < count; i++)
    {
        const long long nb = (set.n_out[i] + kScanTile - 1) / kScanTile;
        nb_max = std::max(nb_max, nb);
        if (nb > 1)
        {
            if (scratch_left < 2 * (nb + 1))
            {
                set_error("scan scratch exhausted");
                return PPPM_ERR_CAPACITY;
            }
            int *sums = scratch, *offs = scratch + nb + 1;
            scratch += 2 * (nb + 1);
            scratch_left -= 2 * (nb + 1);
            set.sums[i] = sums;
            up.in[multi] = sums;
            up.out[multi] = offs;
            up.n_in[multi] = nb;
            up.n_out[multi] = nb + 1;
            add.in[multi] = offs;
            add.out[multi] = set.out[i];
            add.sums[multi] = sums;
            add.n_out[multi] = set.n_out[i];
            multi++;
        }
        else
            set.sums[i] = nullptr;
    }
    scan_tiles_kernel<<<dim3((unsigned)nb_max, count), kScanThreads, 0, h.stream>>>(set);
    h.launches++;
    PB_CHECK_LAUNCH();
    if (multi > 0)
    {
        PB_TRY(scan_level(h, up, multi, scratch, scratch_left));
        long long nb_add = 0;
        for (int i = 0; i < multi; i++)
            nb_add = std::max(nb_add, (add.n_out[i] + kScanTile - 1) / kScanTile);
        scan_add_kernel<<<dim3((unsigned)nb_add, multi), 256, 0, h.stream>>>(add);
        h.launches++;
        PB_CHECK_LAUNCH();
    }
    return PPPM_OK;
}

int exclusive_scan_set(Handle &h, const int *const *in, int *const *out, const long long *n, int count)
{
    if (count < 1 || count > kScanBatch)
        return PPPM_ERR_ARG;
    ScanSet set{};
    long long need = 64;
    for (int i = 0; i < count; i++)
    {
        set.in[i] = in[i];
        set.out[i] = out[i];
        set.n_in[i] = n[i];
        set.n_out[i] = n[i] + 1;
        need += 4 * (n[i] / kScanTile + 8);
    }
    if ((long long)h.scan_tmp_elems < need)
    {
        dev_free(h.d_scan_tmp);
        h.d_scan_tmp = nullptr;
        PB_TRY(dalloc(&h.d_scan_tmp, (size_t)need));
        h.scan_tmp_elems = (size_t)need;
    }
    return scan_level(h, set, count, h.d_scan_tmp, (long long)h.scan_tmp_elems);
}

int exclusive_scan(Handle &h, const int *in, int *out, long long n)
{
    return exclusive_scan_set(h, &in, &out, &n, 1);
}

int mesh_build(Handle &h)
{
    cudaStream_t s = h.stream;
    const int res = h.res, nt = h.nt;
    const long long nc = h.n_cells;
    const f3 mn{h.prm.min_pos[0], h.prm.min_pos[1], h.prm.min_pos[2]};
    const int T = 256;

    // per-mesh arrays sized by nt and res^3 (allocated once per set_mesh)
    if (!h.d_center)
    {
        PB_TRY(dalloc(&h.d_center, 3 * (size_t)nt));
        PB_TRY(dalloc(&h.d_normal, 3 * (size_t)nt));
        PB_TRY(dalloc(&h.d_area, (size_t)nt));
        PB_TRY(dalloc(&h.d_cellc, 3 * (size_t)nt));
        PB_TRY(dalloc(&h.d_basec, 3 * (size_t)nt));
        PB_TRY(dalloc(&h.d_cell, (size_t)nt));
        PB_TRY(dalloc(&h.d_base, (size_t)nt));
        PB_TRY(dalloc(&h.d_cell_tris, (size_t)nt));
        PB_TRY(dalloc(&h.d_base_tris, (size_t)nt));
        PB_TRY(dalloc(&h.d_cell_count, (size_t)nc));
        PB_TRY(dalloc(&h.d_base_count, (size_t)nc));
        PB_TRY(dalloc(&h.d_cell_start, (size_t)nc + 1));
        PB_TRY(dalloc(&h.d_base_start, (size_t)nc + 1));
        PB_TRY(dalloc(&h.d_cursor, (size_t)nc + 1));
        PB_TRY(dalloc(&h.d_flags, 6 * ((size_t)nc + 1)));
        // compact cell lists at their upper bounds: every corrected cell is within one cell of a
        // triangle's cell, every base cell holds a centre, so n3 <= 27 nt and b4 <= nt
        const long long n3_max = std::min<long long>(nc, 27ll * nt) + 1, b4_max = std::min<long long>(nc, nt) + 1;
        PB_TRY(dalloc(&h.d_n3_cell, (size_t)n3_max));
        PB_TRY(dalloc(&h.d_n3_start, (size_t)n3_max));
        PB_TRY(dalloc(&h.d_b4_cell, (size_t)b4_max));
        PB_TRY(dalloc(&h.d_b4_start, (size_t)b4_max));
        PB_TRY(dalloc(&h.d_face_start, (size_t)nt + 1));
        PB_TRY(dalloc(&h.d_face_corner, 8 * (size_t)nt));
        PB_TRY(dalloc(&h.d_status, 4));
    }
    PB_CUDA(cudaMemsetAsync(h.d_status, 0, 4 * sizeof(int), s));

    geometry_kernel<<<div_up(nt, T), T, 0, s>>>(h.d_verts, h.d_tris, nt, res, h.prm.dl, mn, h.d_center, h.d_normal,
                                                 h.d_area, h.d_cellc, h.d_basec, h.d_cell, h.d_base, h.d_status);
    h.launches++;
    PB_CHECK_LAUNCH();
    // the grid-cache refresh needs only this geometry: it runs on a side stream from here on
    if (h.prm.method == PPPM_METHOD_PPPM)
        PB_TRY(grid_cache_start(h));
    // (the status is read with the list sizes below: triangles outside the interior get no cell,
    // so the list builds in between stay in bounds)

    // ---- per-cell and per-base-cell CSR, ids ascending inside a cell
    PB_CUDA(cudaMemsetAsync(h.d_cell_count, 0, sizeof(int) * nc, s));
    PB_CUDA(cudaMemsetAsync(h.d_base_count, 0, sizeof(int) * nc, s));
    count_kernel<<<div_up(nt, T), T, 0, s>>>(h.d_cell, nt, h.d_cell_count);
    count_kernel<<<div_up(nt, T), T, 0, s>>>(h.d_base, nt, h.d_base_count);
    h.launches += 2;
    PB_CHECK_LAUNCH();
    {
        const int *in[2] = {h.d_cell_count, h.d_base_count};
        int *out[2] = {h.d_cell_start, h.d_base_start};
        const long long n[2] = {nc, nc};
        PB_TRY(exclusive_scan_set(h, in, out, n, 2));
    }
    for (int pass = 0; pass < 2; pass++)
    {
        const int *key = pass == 0 ? h.d_cell : h.d_base;
        int *start = pass == 0 ? h.d_cell_start : h.d_base_start;
        int *list = pass == 0 ? h.d_cell_tris : h.d_base_tris;
        PB_CUDA(cudaMemsetAsync(h.d_cursor, 0, sizeof(int) * nc, s));
        fill_kernel<<<div_up(nt, T), T, 0, s>>>(key, nt, start, h.d_cursor, list);
        h.launches++;
        sort_segments_kernel<<<div_up(nc, T), T, 0, s>>>(start, nc, list);
        h.launches++;
        PB_CHECK_LAUNCH();
    }

    if (h.prm.method == PPPM_METHOD_GHOST)
    {
        // the ghost-cell method labels cells from the per-cell lists; no correction lists
        int st = 0;
        PB_TRY(read_int(h, h.d_status, &st));
        if (st)
        {
            set_error("mesh leaves the grid interior: every triangle must lie at least two cells inside the grid");
            return st;
        }
        h.n3 = h.b4 = 0;
        h.p3 = h.p4 = h.pf = 0;
        return PPPM_OK;
    }

    // ---- corrected cells (3^3) and base cells (4^3)
    int *flag3 = h.d_flags, *len3 = h.d_flags + (nc + 1), *flag4 = h.d_flags + 2 * (nc + 1),
        *len4 = h.d_flags + 3 * (nc + 1);
    block_counts_kernel<<<div_up(nc, T), T, 0, s>>>(h.d_cell_start, h.d_base_start, res, flag3, len3, flag4, len4);
    h.launches++;
    PB_CHECK_LAUNCH();
    // Positions and list offsets of corrected cells and base cells from scans over the whole
    // grid, so no count is needed on the host before the compaction; one synchronisation then
    // reads the status and every size the host needs.
    int *pos3 = h.d_cursor;                           // nc + 1
    int *st3 = h.d_flags + 4 * (nc + 1);              // nc + 1
    int *st4 = h.d_flags + 5 * (nc + 1);              // nc + 1
    int *b4_pos = h.d_cell_count;                     // nc (flags of the last cell are 0: never inner)
    {
        const int *in[4] = {flag3, len3, flag4, len4};
        int *out[4] = {pos3, st3, b4_pos, st4};
        const long long n[4] = {nc, nc, nc - 1, nc};
        PB_TRY(exclusive_scan_set(h, in, out, n, 4));
    }
    compact_kernel<<<div_up(nc + 1, T), T, 0, s>>>(flag3, pos3, st3, nc, h.d_n3_cell, h.d_n3_start);
    h.launches++;
    compact_kernel<<<div_up(nc, T), T, 0, s>>>(flag4, b4_pos, st4, nc - 1, h.d_b4_cell, h.d_b4_start);
    h.launches++;
    PB_CHECK_LAUNCH();
    // face pairs per centre triangle: length of its base cell's 4^3 list
    int *face_len = len3;  // len3 was consumed by its scan
    face_len_kernel<<<div_up(nt, T), T, 0, s>>>(h.d_base, nt, b4_pos, flag4, h.d_b4_start, face_len);
    h.launches++;
    PB_CHECK_LAUNCH();
    PB_TRY(exclusive_scan(h, face_len, h.d_face_start, nt));
    int v[7];
    const int *src[7] = {h.d_status,       pos3 + nc, b4_pos + (nc - 1), st3 + nc, st4 + nc, h.d_face_start + nt,
                         h.d_status + 1};
    PB_TRY(read_ints(h, src, 7, v));
    h.corr_near_boundary = v[6] != 0;
    if (v[0])
    {
        set_error("mesh leaves the grid interior: every triangle must lie at least two cells inside the grid");
        return v[0];
    }
    const int n3 = v[1], b4 = v[2], p3 = v[3], p4 = v[4], pf = v[5];
    h.n3 = n3;
    h.b4 = b4;
    h.p3 = p3;
    h.p4 = p4;
    h.pf = pf;

    // ---- 3^3 pairs and corrected-cell mask
    if (p3 > h.p3_cap)
    {
        dev_free(h.d_p3_tri);
        dev_free(h.d_p3_woff);
        h.d_p3_tri = nullptr;
        h.d_p3_woff = nullptr;
        long long cap = p3 + p3 / 4 + 256;
        PB_TRY(dalloc(&h.d_p3_tri, (size_t)cap));
        PB_TRY(dalloc(&h.d_p3_woff, (size_t)cap));
        h.p3_cap = cap;
    }
    PB_CUDA(cudaMemsetAsync(h.d_corr_mask, 0, sizeof(unsigned) * ((nc + 31) / 32), s));
    fill_pairs3_kernel<<<div_up((long long)n3 * 32, T), T, 0, s>>>(h.d_n3_cell, h.d_n3_start, n3, res, h.d_cell_start, h.d_cell_tris,
                                                   h.d_p3_tri, h.d_p3_woff, h.d_corr_mask);
    h.launches++;
    PB_CHECK_LAUNCH();

    // ---- 4^3 lists
    if (p4 > h.n4_cap)
    {
        dev_free(h.d_n4_tris);
        h.d_n4_tris = nullptr;
        long long cap = p4 + p4 / 4 + 256;
        PB_TRY(dalloc(&h.d_n4_tris, (size_t)cap));
        h.n4_cap = cap;
    }
    fill_n4_kernel<<<div_up((long long)b4 * 32, T), T, 0, s>>>(h.d_b4_cell, h.d_b4_start, b4, res, h.d_cell_start, h.d_cell_tris,
                                               h.d_n4_tris);
    h.launches++;
    PB_CHECK_LAUNCH();

    // ---- face pairs per centre triangle
    if (pf > h.pf_cap)
    {
        dev_free(h.d_face_nbr);
        dev_free(h.d_face_pool);
        dev_free(h.d_face_w);
        dev_free(h.d_face_scale);
        dev_free(h.d_pair_flag);
        dev_free(h.d_face_d1);
        h.d_face_nbr = h.d_face_pool = h.d_pair_flag = nullptr;
        h.d_face_w = nullptr;
        h.d_face_scale = nullptr;
        h.d_face_d1 = nullptr;
        long long cap = pf + pf / 4 + 256;
        PB_TRY(dalloc(&h.d_face_nbr, (size_t)cap));
        PB_TRY(dalloc(&h.d_face_pool, (size_t)cap));
        PB_TRY(dalloc(&h.d_pair_flag, (size_t)cap + 1));
        PB_TRY(dev_alloc(&h.d_face_w, (size_t)cap * (h.fp64 ? 16 * sizeof(double2) : 16 * sizeof(__half2))));
        PB_TRY(dalloc(&h.d_face_scale, (size_t)cap));
        PB_TRY(dev_alloc(&h.d_face_d1, (size_t)cap * h.real_size));
        h.pf_cap = cap;
    }
    face_fill_kernel<<<div_up((long long)nt * 32, T), T, 0, s>>>(h.d_base, h.d_basec, nt, res, b4_pos, flag4, h.d_b4_start,
                                                 h.d_n4_tris, h.d_face_start, h.d_face_nbr, h.d_face_corner);
    h.launches++;
    PB_CHECK_LAUNCH();
    return PPPM_OK;
}

}  // namespace pb
