// GridCache / FaceCache: the TDBEM weight tables the per-step correction reads.
//
// Reference semantics kept (src/algorithm/pppm_cache.{h,cu}):
//   GridCache     one record pair per (triangle, 27 neighbour cells): the FDTD-near weights
//                 (8 stencil targets at scales {2, s, s, s, s, s, s, -6s}, s = (c dt / h)^2,
//                 shifted by one step, minus the BEM-near weights two steps back) and the
//                 BEM-near weights; targets inside the triangle's own cell are skipped
//                 (pppm_cache.cu:64-123).  Refreshed for a triangle when its centre moved
//                 > 1% h, its normal moved > 0.01 or its area changed > 1% (pppm_cache.h:65-70).
//   FaceCache     one record per (centre face, neighbour face) ever seen in the centre's 4^3
//                 block: the face-to-face integral minus the neighbour's point integrals at
//                 those of the centre's 8 interpolation corners farther than 1.5 h from the
//                 neighbour centre in some axis (pppm_cache.cu:234-271).  Records persist
//                 across mesh updates and are refreshed only when new or when the pair's
//                 normal dot product moved > 0.01 or its centre distance > 1%
//                 (pppm_cache.h:123-128, pppm_cache.cu:183-232).  Trilinear interpolation
//                 weights of every face are recomputed on every update (pppm_cache.cu:157-181).
// B200 layout: the persistent face records live in a pool addressed through a per-centre
// open-addressing table (kFaceCacheSlots keys per face, the reference's per-face bound);
// after each refresh the records the step needs are gathered into dense arrays in hot-path
// order, so the per-step kernels stream them.
#include "handle.cuh"

namespace pb
{

namespace
{

// ---- fp16 row packing (bem.h:171-191)
__device__ inline void pack_half(const float *s, const float *d, __half2 *out, float2 *scale)
{
    float ms = 0, md = 0;
    for (int i = 0; i < kTaps; i++)
    {
        ms = max(ms, abs(s[i]));
        md = max(md, abs(d[i]));
    }
    if (ms == 0)
        ms = 1;
    if (md == 0)
        md = 1;
    for (int i = 0; i < kTaps; i++)
    {
        float a = s[i] / ms, b = d[i] / md;
        out[i] = __halves2half2(__float2half_rn(a), __float2half_rn(b));
    }
    *scale = make_float2(ms, md);
}

__device__ inline void pack_double(const double *s, const double *d, double2 *out)
{
    for (int i = 0; i < kTaps; i++)
        out[i] = make_double2(s[i], d[i]);
}

struct DevConsts
{
    float lambda;
    float wave_re[kTaps], wave_im[kTaps];
    float threshold;
    double lambda_d;
    double wave_re_d[kTaps], wave_im_d[kTaps];
    float c, dt, h;
    f3 mn;
    int res;
    const double *tw;  // FFT twiddles, 8 x (cos, sin), filled on the device by twiddle_kernel
};

__global__ void twiddle_kernel(double *tw) { ref32::twiddle_fill(tw); }

__device__ inline void load_tri(const float *verts, const int *tris, int t, f3 *v, int *idx)
{
    idx[0] = tris[3 * t];
    idx[1] = tris[3 * t + 1];
    idx[2] = tris[3 * t + 2];
    v[0] = load3(verts, idx[0]);
    v[1] = load3(verts, idx[1]);
    v[2] = load3(verts, idx[2]);
}

// spectrum k <= 8 -> full 16 with conjugates, FFT, scaling (bem.h:306-321)
__device__ inline void spectrum_to_weights(cf *sp, float lambda, float *w, const double *tw)
{
    for (int k = kTaps / 2 + 1; k < kTaps; k++)
        sp[k] = cf{sp[kTaps - k].re, -sp[kTaps - k].im};
    ref32::scaled_fft(sp, lambda, w, tw);
}

__device__ inline void spectrum_to_weights_d(cd *sp, double lambda, double *w)
{
    for (int k = kTaps / 2 + 1; k < kTaps; k++)
        sp[k] = cd{sp[kTaps - k].re, -sp[kTaps - k].im};
    f64::scaled_fft(sp, lambda, w);
}

// ---------------------------------------------------------------- grid cache ---------
__global__ void gc_flag_kernel(const float *center, const float *normal, const float *area, const float *snap, int nt,
                               float h, int empty, int *flag)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt)
        return;
    if (empty)
    {
        flag[i] = 1;
        return;
    }
    f3 oc = f3{snap[7 * i], snap[7 * i + 1], snap[7 * i + 2]};
    f3 on = f3{snap[7 * i + 3], snap[7 * i + 4], snap[7 * i + 5]};
    float oa = snap[7 * i + 6];
    f3 c = load3(center, i), n = load3(normal, i);
    float a = area[i];
    flag[i] = (len3(oc - c) > 0.01 * h || len3(on - n) > 0.01 || abs(oa - a) > 0.01 * a) ? 1 : 0;
}

// Grid-cache refresh, one block per flagged triangle.  The FDTD-near rows of a triangle's 27
// records read the Green's function at the cell centres of 7-point stencils around its 27
// neighbour cells, and the BEM-near rows at those 27 centres: 81 distinct cells (offsets in
// [-2, 2]^3 with at most one coordinate of magnitude 2) instead of 243 point evaluations per
// wave number.  The block evaluates each (cell, wave number) once into shared memory (the
// unrounded terms of both_acc), then every (record, wave number) accumulates its points in the
// reference's order, then one FFT per thread, then packing: the records are bit-identical to a
// per-record evaluation.
constexpr int kGcPoints = 81;

// offset of distinct point p (0..80) from the triangle's cell
__device__ inline void gc_point_offset(int p, int &dx, int &dy, int &dz)
{
    if (p < 27)
    {
        dx = p % 3 - 1;
        dy = p / 3 % 3 - 1;
        dz = p / 9 - 1;
        return;
    }
    p -= 27;
    const int axis = p / 18, side = (p / 9) & 1, a = p % 3 - 1, b = p / 3 % 3 - 1;
    const int far = side ? 2 : -2;
    dx = axis == 0 ? far : a;
    dy = axis == 1 ? far : (axis == 0 ? a : b);
    dz = axis == 2 ? far : b;
}

__device__ inline void gc_block_body(int tri, const DevConsts &dc, const float *verts, const int *tris,
                                     const int *cellc, const float *center, const float *normal, const float *area,
                                     const int *flag, __half2 *gc_w, float2 *gc_scale, float *snap)
{
    if (!flag[tri])
        return;
    // The point terms of steps 1-2 and, once they are consumed, the 16-tap weights, the two
    // records' rows and their scales of steps 3-4 share one buffer (37 KB per block in all, so
    // four blocks fit an SM).
    constexpr int kWave = kTaps / 2 + 1;
    __shared__ __align__(16) unsigned char pool[kGcPoints * kWave * sizeof(ref32::PointTerms)];
    static_assert(2 * 27 * 4 * kTaps * sizeof(float) + 54 * 2 * sizeof(float) <=
                      kGcPoints * kWave * sizeof(ref32::PointTerms),
                  "weights, rows and scales fit in the point-term buffer");
    auto terms = reinterpret_cast<ref32::PointTerms(*)[kWave]>(pool);
    auto wts = reinterpret_cast<float(*)[4][kTaps]>(pool);  // per offset: ss, sd, qs, qd rows
    auto rows = reinterpret_cast<float(*)[2][kTaps]>(pool + 27 * 4 * kTaps * sizeof(float));  // 54 records
    auto rmax = reinterpret_cast<float(*)[2]>(pool + 2 * 27 * 4 * kTaps * sizeof(float));    // their scales
    __shared__ short point_of[125];            // 5^3 offset box -> distinct point
    __shared__ cf spec[27][kWave][4];          // ss, sd, qs, qd per record and wave number
    const int tid = threadIdx.x;
    f3 v[3];
    int idx[3];
    load_tri(verts, tris, tri, v, idx);
    const int tx = cellc[3 * tri], ty = cellc[3 * tri + 1], tz = cellc[3 * tri + 2];
    const float jac = ref32::jacobian(v);
    const f3 nrm = ref32::tri_normal(v);
    const float gx = (float)PB_TRI_X;
    const f3 q = ref32::local_to_global(gx, gx, v);
    // 1. the Green's function terms of every distinct cell centre and wave number
    for (int it = tid; it < kGcPoints * kWave; it += blockDim.x)
    {
        const int p = it / kWave, k = it % kWave;
        int dx, dy, dz;
        gc_point_offset(p, dx, dy, dz);
        if (k == 0)
            point_of[(dx + 2) * 25 + (dy + 2) * 5 + (dz + 2)] = (short)p;
        const f3 pt = cell_center(tx + dx, ty + dy, tz + dz, dc.h, dc.mn);
        terms[p][k] = ref32::point_terms(q, pt, nrm, cf{dc.wave_re[k], dc.wave_im[k]});
    }
    __syncthreads();
    // 2. spectra of each record: the 7-point stencil around its neighbour cell (FDTD-near) and
    // its centre (BEM-near), accumulated in the reference's order
    const float scale = dc.c * dc.c * dc.dt * dc.dt / (dc.h * dc.h);
    const double c = 0.5 * 1.0f * jac;
    for (int it = tid; it < 27 * kWave; it += blockDim.x)
    {
        const int woff = it / kWave, k = it % kWave;
        const int ox = woff % 3 - 1, oy = woff / 3 % 3 - 1, oz = woff / 9 - 1;
        const int sx[8] = {0, -1, 1, 0, 0, 0, 0, 0}, sy[8] = {0, 0, 0, -1, 1, 0, 0, 0},
                  sz[8] = {0, 0, 0, 0, 0, -1, 1, 0};
        const float dsc[8] = {2, scale, scale, scale, scale, scale, scale, -6 * scale};
        cf ls{0.0f, 0.0f}, ld{0.0f, 0.0f};
        for (int i = 0; i < 8; i++)
        {
            const int px = ox + sx[i], py = oy + sy[i], pz = oz + sz[i];
            if (px == 0 && py == 0 && pz == 0)
                continue;  // targets inside the triangle's own cell are skipped
            ref32::acc_terms(ls, ld, terms[point_of[(px + 2) * 25 + (py + 2) * 5 + (pz + 2)]][k], dsc[i], true);
        }
        spec[woff][k][0] = cf{(float)(0.0f + c * ls.re), (float)(0.0f + c * ls.im)};
        spec[woff][k][1] = cf{(float)(0.0f + c * ld.re), (float)(0.0f + c * ld.im)};
        cf bs{0.0f, 0.0f}, bd{0.0f, 0.0f};
        if (!(ox == 0 && oy == 0 && oz == 0))
            ref32::acc_terms(bs, bd, terms[point_of[(ox + 2) * 25 + (oy + 2) * 5 + (oz + 2)]][k], 1.0f, false);
        spec[woff][k][2] = cf{(float)(0.0f + c * bs.re), (float)(0.0f + c * bs.im)};
        spec[woff][k][3] = cf{(float)(0.0f + c * bd.re), (float)(0.0f + c * bd.im)};
    }
    __syncthreads();
    // 3. one 16-point transform per (record, layer row); the point terms are dead from here on
    for (int it = tid; it < 27 * 4; it += blockDim.x)
    {
        const int woff = it / 4, which = it % 4;
        cf sp[kTaps];
        for (int k = 0; k <= kTaps / 2; k++)
            sp[k] = spec[woff][k][which];
        spectrum_to_weights(sp, dc.lambda, wts[woff][which], dc.tw);
    }
    __syncthreads();
    // 4. per (offset, tap): the FDTD-near record (moved by one step, minus the BEM-near weights
    // two steps back) and the BEM-near record; the triangle's own cell has neither.  Records
    // 0..26 are the FDTD-near ones, 27..53 the BEM-near ones.
    for (int it = tid; it < 27 * kTaps; it += blockDim.x)
    {
        const int woff = it / kTaps, i = it % kTaps;
        const bool inside = woff == 13;
        float ws = 0, wd = 0;
        if (i >= 1)
        {
            ws = wts[woff][0][i - 1];
            wd = wts[woff][1][i - 1];
        }
        if (!inside && i >= 2)
        {
            ws += wts[woff][2][i - 2] * -1.0f;
            wd += wts[woff][3][i - 2] * -1.0f;
        }
        float bs = 0, bd = 0;
        if (!inside)
        {
            bs += wts[woff][2][i] * 1.0f;
            bd += wts[woff][3][i] * 1.0f;
        }
        rows[woff][0][i] = ws;
        rows[woff][1][i] = wd;
        rows[27 + woff][0][i] = bs;
        rows[27 + woff][1][i] = bd;
    }
    __syncthreads();
    // 5. fp16 packing (pack_half, bem.h:171-191): each row's max-abs scale, taps in order ...
    for (int it = tid; it < 54 * 2; it += blockDim.x)
    {
        const float *row = rows[it >> 1][it & 1];
        float m = 0;
        for (int i = 0; i < kTaps; i++)
            m = max(m, abs(row[i]));
        rmax[it >> 1][it & 1] = m == 0 ? 1.0f : m;
    }
    __syncthreads();
    // ... then every (record, tap) rounded to half, single and double layer in one half2
    for (int it = tid; it < 54 * kTaps; it += blockDim.x)
    {
        const int r = it / kTaps, i = it % kTaps;
        const float ms = rmax[r][0], md = rmax[r][1];
        const float a = rows[r][0][i] / ms, b = rows[r][1][i] / md;
        const size_t rec = (size_t)tri * 54 + r;
        gc_w[rec * kTaps + i] = __halves2half2(__float2half_rn(a), __float2half_rn(b));
        if (i == 0)
            gc_scale[rec] = make_float2(ms, md);
    }
    if (tid == 0)
    {
        f3 cc = load3(center, tri), nn = load3(normal, tri);
        snap[7 * tri] = cc.x;
        snap[7 * tri + 1] = cc.y;
        snap[7 * tri + 2] = cc.z;
        snap[7 * tri + 3] = nn.x;
        snap[7 * tri + 4] = nn.y;
        snap[7 * tri + 5] = nn.z;
        snap[7 * tri + 6] = area[tri];
    }
}

// Blocks take triangles tri = blockIdx.x, blockIdx.x + gridDim.x, ...: a grid of one block per
// triangle, or a smaller one that leaves room on the SMs for the kernels of the same mesh update
// running beside it (grid_cache_start)
__global__ void __launch_bounds__(256, 4) gc_block_kernel(DevConsts dc, const float *verts, const int *tris, int nt,
                                                          const int *cellc, const float *center, const float *normal,
                                                          const float *area, const int *flag, __half2 *gc_w,
                                                          float2 *gc_scale, float *snap)
{
    for (int tri = blockIdx.x; tri < nt; tri += gridDim.x)
    {
        gc_block_body(tri, dc, verts, tris, cellc, center, normal, area, flag, gc_w, gc_scale, snap);
        __syncthreads();  // the next triangle reuses the shared buffers
    }
}

// FP64 scheme: the same records entirely in double, unquantised
__global__ void gc_compute_kernel_d(DevConsts dc, const float *verts, const int *tris, const int *cellc,
                                    const float *center, const float *normal, const float *area, const int *flag,
                                    int nt, double2 *gc_w, float *snap)
{
    long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nt * 27)
        return;
    int tri = (int)(gid / 27), woff = (int)(gid % 27);
    if (!flag[tri])
        return;
    using namespace f64;
    f3 vf[3];
    int idx[3];
    load_tri(verts, tris, tri, vf, idx);
    d3 v[3] = {dd(vf[0]), dd(vf[1]), dd(vf[2])};
    int tx = cellc[3 * tri], ty = cellc[3 * tri + 1], tz = cellc[3 * tri + 2];
    int nx = tx + woff % 3 - 1, ny = ty + woff / 3 % 3 - 1, nz = tz + woff / 9 - 1;
    int dcx[8] = {nx, nx - 1, nx + 1, nx, nx, nx, nx, nx};
    int dcy[8] = {ny, ny, ny, ny - 1, ny + 1, ny, ny, ny};
    int dcz[8] = {nz, nz, nz, nz, nz, nz - 1, nz + 1, nz};
    double h = dc.h;
    double scale = (double)dc.c * dc.c * dc.dt * dc.dt / (h * h);
    double dsc[8] = {2, scale, scale, scale, scale, scale, scale, -6 * scale};
    d3 mn{dc.mn.x, dc.mn.y, dc.mn.z};
    auto ctr = [&](int i, int j, int k) { return d3{(i + 0.5) * h + mn.x, (j + 0.5) * h + mn.y, (k + 0.5) * h + mn.z}; };
    d3 pts[8];
    double sc[8];
    int n = 0;
    for (int i = 0; i < 8; i++)
        if (!(dcx[i] == tx && dcy[i] == ty && dcz[i] == tz))
        {
            pts[n] = ctr(dcx[i], dcy[i], dcz[i]);
            sc[n] = dsc[i];
            n++;
        }
    cd ss[kTaps], sd[kTaps];
    for (int k = 0; k <= kTaps / 2; k++)
    {
        cd kk{dc.wave_re_d[k], dc.wave_im_d[k]};
        ss[k] = face_to_points(v, pts, sc, n, kk, false);
        sd[k] = face_to_points(v, pts, sc, n, kk, true);
    }
    double ws[kTaps], wd[kTaps];
    spectrum_to_weights_d(ss, dc.lambda_d, ws);
    spectrum_to_weights_d(sd, dc.lambda_d, wd);
    for (int i = kTaps - 1; i >= 1; i--)
    {
        ws[i] = ws[i - 1];
        wd[i] = wd[i - 1];
    }
    ws[0] = 0;
    wd[0] = 0;
    bool inside = (nx == tx && ny == ty && nz == tz);
    double ps[kTaps] = {0}, pd[kTaps] = {0};
    if (!inside)
    {
        d3 p = ctr(nx, ny, nz);
        double one = 1.0;
        cd qs[kTaps], qd[kTaps];
        for (int k = 0; k <= kTaps / 2; k++)
        {
            cd kk{dc.wave_re_d[k], dc.wave_im_d[k]};
            qs[k] = face_to_points(v, &p, &one, 1, kk, false);
            qd[k] = face_to_points(v, &p, &one, 1, kk, true);
        }
        spectrum_to_weights_d(qs, dc.lambda_d, ps);
        spectrum_to_weights_d(qd, dc.lambda_d, pd);
        for (int i = 2; i < kTaps; i++)
        {
            ws[i] -= ps[i - 2];
            wd[i] -= pd[i - 2];
        }
    }
    size_t rec = (size_t)tri * 54 + woff;
    pack_double(ws, wd, gc_w + rec * kTaps);
    pack_double(ps, pd, gc_w + (rec + 27) * kTaps);
    if (woff == 0)
    {
        f3 c = load3(center, tri), nn = load3(normal, tri);
        snap[7 * tri] = c.x;
        snap[7 * tri + 1] = c.y;
        snap[7 * tri + 2] = c.z;
        snap[7 * tri + 3] = nn.x;
        snap[7 * tri + 4] = nn.y;
        snap[7 * tri + 5] = nn.z;
        snap[7 * tri + 6] = area[tri];
    }
}

// dense copy of the 3^3 pair records in hot-path order

// ---------------------------------------------------------------- face cache ---------
// trilinear weights of the 2x2x2 corner cells at the face's 1-point Gauss node
// (pppm_cache.cu:157-181)
__global__ void interp_kernel(const float *verts, const int *tris, const int *basec, int nt, float h, f3 mn,
                              float *interp, double *interp_d)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt)
        return;
    f3 v[3];
    int idx[3];
    load_tri(verts, tris, i, v, idx);
    float jac = ref32::jacobian(v);
    const float gx = (float)PB_TRI_X;
    f3 q = ref32::local_to_global(gx, gx, v);
    f3 base = cell_center(basec[3 * i], basec[3 * i + 1], basec[3 * i + 2], h, mn);
    f3 d = (q - base) / h;
    float wt[8];
    wt[0] = (1 - d.x) * (1 - d.y) * (1 - d.z);
    wt[1] = (1 - d.x) * (1 - d.y) * d.z;
    wt[2] = (1 - d.x) * d.y * (1 - d.z);
    wt[3] = (1 - d.x) * d.y * d.z;
    wt[4] = d.x * (1 - d.y) * (1 - d.z);
    wt[5] = d.x * (1 - d.y) * d.z;
    wt[6] = d.x * d.y * (1 - d.z);
    wt[7] = d.x * d.y * d.z;
    float s = 0.5 * 1.0f * jac;
    for (int k = 0; k < 8; k++)
    {
        float w = 0;
        w += s * wt[k];
        interp[8 * i + k] = w;
    }
    if (interp_d)
    {
        using namespace f64;
        d3 vd[3] = {dd(v[0]), dd(v[1]), dd(v[2])};
        double jd = jacobian(vd);
        d3 qd = ltg(1.0 / 3, 1.0 / 3, vd);
        double hh = h;
        double bx = (basec[3 * i] + 0.5) * hh + mn.x, by = (basec[3 * i + 1] + 0.5) * hh + mn.y,
               bz = (basec[3 * i + 2] + 0.5) * hh + mn.z;
        double ex = (qd.x - bx) / hh, ey = (qd.y - by) / hh, ez = (qd.z - bz) / hh;
        double wd8[8] = {(1 - ex) * (1 - ey) * (1 - ez), (1 - ex) * (1 - ey) * ez, (1 - ex) * ey * (1 - ez),
                         (1 - ex) * ey * ez,             ex * (1 - ey) * (1 - ez), ex * (1 - ey) * ez,
                         ex * ey * (1 - ez),             ex * ey * ez};
        for (int k = 0; k < 8; k++)
            interp_d[8 * i + k] = 0.5 * jd * wd8[k];
    }
}

__device__ inline unsigned hash_slot(int key) { return ((unsigned)key * 2654435761u) >> 22; }  // 10 bits

// one warp per centre face: find or insert each (centre, neighbour) pair in the centre's
// table, decide whether its record must be recomputed.
// A rewritten slot below log_floor (the newest motion checkpoint's pool size) gets its old meta
// kept in old_meta[p] and is counted in n_log; fresh slots record their key.
__global__ void fc_lookup_kernel(const int *face_start, const int *face_nbr, int nt, const float *center,
                                 const float *normal, int *keys, int *slots, int *pool_count, long long pool_cap,
                                 float2 *pool_meta, int2 *pool_key, long long log_floor, float2 *old_meta,
                                 int *n_log, int *face_pool, int *pair_flag, int *status)
{
    int warp = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    int lane = threadIdx.x & 31;
    if (warp >= nt)
        return;
    int ctr = warp;
    f3 cc = load3(center, ctr), cn = load3(normal, ctr);
    int *tk = keys + (size_t)ctr * kFaceCacheSlots;
    int *ts = slots + (size_t)ctr * kFaceCacheSlots;
    for (int p = face_start[ctr] + lane; p < face_start[ctr + 1]; p += 32)
    {
        int nbr = face_nbr[p];
        unsigned hsh = hash_slot(nbr);
        int slot = -1;
        bool fresh = false;
        for (int probe = 0; probe < kFaceCacheSlots; probe++)
        {
            unsigned pos = (hsh + probe) & (kFaceCacheSlots - 1);
            int cur = tk[pos];
            if (cur == nbr)
            {
                // inserted by an earlier refresh (this refresh inserts each pair once)
                slot = ts[pos];
                break;
            }
            if (cur == -1)
            {
                int prev = atomicCAS(&tk[pos], -1, nbr);
                if (prev == -1)
                {
                    slot = atomicAdd(pool_count, 1);
                    ts[pos] = slot;
                    fresh = true;
                    break;
                }
                if (prev == nbr)
                {
                    slot = ts[pos];
                    break;
                }
            }
        }
        if (slot < 0 || slot >= pool_cap)
        {
            atomicCAS(status, 0, PPPM_ERR_CAPACITY);
            face_pool[p] = 0;
            pair_flag[p] = 0;
            continue;
        }
        f3 nc = load3(center, nbr), nn = load3(normal, nbr);
        float angle = dot3(nn, cn);
        float dist = len3(nc - cc);
        int recompute = 0;
        if (fresh)
        {
            recompute = 1;
            pool_key[slot] = make_int2(ctr, nbr);
        }
        else
        {
            float2 m = pool_meta[slot];
            recompute = (abs(m.x - angle) > 0.01 || abs(m.y - dist) > 0.01 * dist) ? 1 : 0;
            if (recompute && slot < log_floor)
            {
                old_meta[p] = m;
                atomicAdd(n_log, 1);
            }
        }
        if (recompute)
            pool_meta[slot] = make_float2(angle, dist);
        face_pool[p] = slot;
        pair_flag[p] = recompute;
    }
}

__global__ void compact_pairs_kernel(const int *flag, const int *pos, long long n, int *out)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && flag[i])
        out[pos[i]] = (int)i;
}

// ---- motion checkpoints: undo log of pool rewrites, table rebuild

__device__ inline void copy_record(const int4 *src, int4 *dst, int words)
{
    for (int k = 0; k < words; k++)
        dst[k] = src[k];
}

// one thread per pair to recompute: a slot below the floor (written before the newest
// checkpoint) has its record, scale and old meta appended to the log before the refresh
// overwrites it
__global__ void log_rewrites_kernel(const int *work, int nwork, const int *face_pool, long long floor,
                                    const float2 *old_meta, const int4 *pool_w, const float2 *pool_scale,
                                    int rec_words, int cap, int *cursor, int *out_slot, int4 *out_rec,
                                    float2 *out_scale, float2 *out_meta)
{
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwork)
        return;
    const int p = work[w], slot = face_pool[p];
    if (slot >= floor)
        return;
    const int i = atomicAdd(cursor, 1);
    if (i >= cap)
        return;  // cannot happen: cap is the lookup's count of these pairs
    out_slot[i] = slot;
    copy_record(pool_w + (size_t)slot * rec_words, out_rec + (size_t)i * rec_words, rec_words);
    if (out_scale)
        out_scale[i] = pool_scale[slot];
    out_meta[i] = old_meta[p];
}

// a log batch written back (its slots are distinct: a refresh recomputes each pair once)
__global__ void apply_log_kernel(int n, const int *slot, const int4 *rec, const float2 *scale, const float2 *meta,
                                 int rec_words, int4 *pool_w, float2 *pool_scale, float2 *pool_meta)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int s = slot[i];
    copy_record(rec + (size_t)i * rec_words, pool_w + (size_t)s * rec_words, rec_words);
    if (scale)
        pool_scale[s] = scale[i];
    pool_meta[s] = meta[i];
}

// the per-centre tables from the pool keys of slots [0, used): the same (centre, neighbour) ->
// slot map as when those slots were inserted (probe positions may differ)
__global__ void fc_rebuild_kernel(const int2 *pool_key, long long used, int *keys, int *slots, int *status)
{
    long long sl = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= used)
        return;
    const int2 k = pool_key[sl];
    int *tk = keys + (size_t)k.x * kFaceCacheSlots;
    int *ts = slots + (size_t)k.x * kFaceCacheSlots;
    const unsigned hsh = hash_slot(k.y);
    for (int probe = 0; probe < kFaceCacheSlots; probe++)
    {
        const unsigned pos = (hsh + probe) & (kFaceCacheSlots - 1);
        if (atomicCAS(&tk[pos], -1, k.y) == -1)
        {
            ts[pos] = (int)sl;
            return;
        }
    }
    atomicCAS(status, 0, PPPM_ERR_CAPACITY);
}

__device__ inline int centre_of(const int *face_start, int nt, int p)
{
    int lo = 0, hi = nt;  // largest i with face_start[i] <= p
    while (hi - lo > 1)
    {
        int mid = (lo + hi) >> 1;
        if (face_start[mid] <= p)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Phase A: face-to-face spectra, one thread per (recomputed pair, k <= 8) evaluating both
// layers; spec[18 w + k] single layer, spec[18 w + 9 + k] double layer.
// mode: 0 = ref32 throughout, 1 = FP64 for panels sharing vertices (stored as float)
// The corner cells of centre ctr's interpolation that lie farther than 1.5 h from the neighbour's
// centre along some axis, with their scale (-interpolation weight) (pppm_cache.cu:234-271)
__device__ inline int far_corners(const DevConsts &dc, const int *basec, const float *interp, int ctr, f3 nbc,
                                  f3 *pts, float *sc)
{
    int n = 0;
    const int bx = basec[3 * ctr], by = basec[3 * ctr + 1], bz = basec[3 * ctr + 2];
    for (int dx = 0; dx < 2; dx++)
        for (int dy = 0; dy < 2; dy++)
            for (int dz = 0; dz < 2; dz++)
            {
                const int widx = dx * 4 + dy * 2 + dz;
                const f3 c = cell_center(bx + dx, by + dy, bz + dz, dc.h, dc.mn);
                if (abs(c.x - nbc.x) > dc.h * 1.5 || abs(c.y - nbc.y) > dc.h * 1.5 || abs(c.z - nbc.z) > dc.h * 1.5)
                {
                    pts[n] = c;
                    sc[n] = -interp[8 * ctr + widx];
                    n++;
                }
            }
    return n;
}

// Phase A, one thread per (pair, wave number): the face-to-face spectra of both layers plus the
// neighbour's point integrals at the centre's far interpolation corners, the pair's record spectra
__global__ void fc_spectra_kernel(DevConsts dc, const float *verts, const int *tris, const float *center,
                                  const int *basec, const float *interp, const int *face_start, int nt,
                                  const int *face_nbr, const int *work, int nwork, int mode, cf *spec)
{
    long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nwork * 9)
        return;
    int w = (int)(gid / 9), k = (int)(gid % 9);
    int p = work[w];
    int ctr = centre_of(face_start, nt, p), nbr = face_nbr[p];
    f3 sv[3], tv[3];
    int si[3], ti[3];
    load_tri(verts, tris, nbr, sv, si);
    load_tri(verts, tris, ctr, tv, ti);
    cf os, od;
    if (mode == 1 && ref32::common_vertices(si, ti) > 0)
    {
        using namespace f64;
        d3 s[3] = {dd(sv[0]), dd(sv[1]), dd(sv[2])}, t[3] = {dd(tv[0]), dd(tv[1]), dd(tv[2])};
        cd kk{dc.wave_re_d[k], dc.wave_im_d[k]};
        cd vs = face_to_face(s, si, t, ti, kk, dc.threshold, false);
        cd vd = face_to_face(s, si, t, ti, kk, dc.threshold, true);
        os = cf{(float)vs.re, (float)vs.im};
        od = cf{(float)vd.re, (float)vd.im};
    }
    else
        ref32::face_to_face2(sv, si, tv, ti, cf{dc.wave_re[k], dc.wave_im[k]}, dc.threshold, os, od);
    f3 pts[8];
    float sc[8];
    const int n = far_corners(dc, basec, interp, ctr, load3(center, nbr), pts, sc);
    cf ps, pd;
    ref32::face_to_points2(sv, pts, sc, n, true, cf{dc.wave_re[k], dc.wave_im[k]}, ps, pd);
    spec[(size_t)w * 18 + k] = cf{os.re + ps.re, os.im + ps.im};
    spec[(size_t)w * 18 + 9 + k] = cf{od.re + pd.re, od.im + pd.im};
}

__global__ void fc_spectra_kernel_d(DevConsts dc, const float *verts, const int *tris, const int *face_start, int nt,
                                    const int *face_nbr, const int *work, int nwork, cd *spec)
{
    long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nwork * 18)
        return;
    int w = (int)(gid / 18), r = (int)(gid % 18);
    int layer = r / 9, k = r % 9;
    int p = work[w];
    int ctr = centre_of(face_start, nt, p), nbr = face_nbr[p];
    f3 sv[3], tv[3];
    int si[3], ti[3];
    load_tri(verts, tris, nbr, sv, si);
    load_tri(verts, tris, ctr, tv, ti);
    using namespace f64;
    d3 s[3] = {dd(sv[0]), dd(sv[1]), dd(sv[2])}, t[3] = {dd(tv[0]), dd(tv[1]), dd(tv[2])};
    spec[(size_t)w * 18 + r] =
        face_to_face(s, si, t, ti, cd{dc.wave_re_d[k], dc.wave_im_d[k]}, (double)dc.h * 0.1, layer == 1);
}

// Phase B, one thread per pair: FFT of both record spectra, packing into the pool record
__global__ void fc_finish_kernel(DevConsts dc, const int *face_pool, const int *work, int nwork, const cf *spec,
                                 __half2 *pool_w, float2 *pool_scale)
{
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwork)
        return;
    int p = work[w];
    cf ss[kTaps], sd[kTaps];
    for (int k = 0; k <= kTaps / 2; k++)
    {
        ss[k] = spec[(size_t)w * 18 + k];
        sd[k] = spec[(size_t)w * 18 + 9 + k];
    }
    float ws[kTaps], wd[kTaps];
    spectrum_to_weights(ss, dc.lambda, ws, dc.tw);
    spectrum_to_weights(sd, dc.lambda, wd, dc.tw);
    int slot = face_pool[p];
    pack_half(ws, wd, pool_w + (size_t)slot * kTaps, pool_scale + slot);
}

__global__ void fc_finish_kernel_d(DevConsts dc, const float *verts, const int *tris, const float *center,
                                   const int *basec, const double *interp, const int *face_start, int nt,
                                   const int *face_nbr, const int *face_pool, const int *work, int nwork,
                                   const cd *spec, double2 *pool_w)
{
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwork)
        return;
    using namespace f64;
    int p = work[w];
    int ctr = centre_of(face_start, nt, p), nbr = face_nbr[p];
    f3 svf[3];
    int si[3];
    load_tri(verts, tris, nbr, svf, si);
    d3 sv[3] = {dd(svf[0]), dd(svf[1]), dd(svf[2])};
    d3 nbc = (1.0 / 3) * (sv[0] + sv[1] + sv[2]);
    double h = dc.h;
    d3 pts[8];
    double sc[8];
    int n = 0;
    int bx = basec[3 * ctr], by = basec[3 * ctr + 1], bz = basec[3 * ctr + 2];
    for (int dx = 0; dx < 2; dx++)
        for (int dy = 0; dy < 2; dy++)
            for (int dz = 0; dz < 2; dz++)
            {
                int widx = dx * 4 + dy * 2 + dz;
                d3 c{(bx + dx + 0.5) * h + dc.mn.x, (by + dy + 0.5) * h + dc.mn.y, (bz + dz + 0.5) * h + dc.mn.z};
                if (fabs(c.x - nbc.x) > h * 1.5 || fabs(c.y - nbc.y) > h * 1.5 || fabs(c.z - nbc.z) > h * 1.5)
                {
                    pts[n] = c;
                    sc[n] = -interp[8 * ctr + widx];
                    n++;
                }
            }
    cd ss[kTaps], sd[kTaps];
    for (int k = 0; k <= kTaps / 2; k++)
    {
        cd a = spec[(size_t)w * 18 + k], b = spec[(size_t)w * 18 + 9 + k];
        cd kk{dc.wave_re_d[k], dc.wave_im_d[k]};
        cd ps = face_to_points(sv, pts, sc, n, kk, false);
        cd pd = face_to_points(sv, pts, sc, n, kk, true);
        ss[k] = cd{a.re + ps.re, a.im + ps.im};
        sd[k] = cd{b.re + pd.re, b.im + pd.im};
    }
    double ws[kTaps], wd[kTaps];
    spectrum_to_weights_d(ss, dc.lambda_d, ws);
    spectrum_to_weights_d(sd, dc.lambda_d, wd);
    pack_double(ws, wd, pool_w + (size_t)face_pool[p] * kTaps);
}

// dense face weights in hot-path order from the pool: one thread per 16-byte chunk of a record
// (4 chunks per fp16 record, 16 per FP64 record)
template <typename Rec>
__global__ void gather_face_kernel(const int *face_pool, long long pf, const Rec *pool_w, const float2 *pool_scale,
                                   Rec *face_w, float2 *face_scale)
{
    constexpr int kChunks = (int)(kTaps * sizeof(Rec) / sizeof(uint4));
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= pf * kChunks)
        return;
    long long p = g / kChunks;
    int k = (int)(g % kChunks);
    int slot = face_pool[p];
    ((uint4 *)face_w)[p * kChunks + k] = ((const uint4 *)pool_w)[(size_t)slot * kChunks + k];
    if (k == 0 && pool_scale)
        face_scale[p] = pool_scale[slot];
}

template <typename Rec>
inline long long gather_face_threads(long long pf)
{
    return pf * (long long)(kTaps * sizeof(Rec) / sizeof(uint4));
}

// 0.5 * area - sum_j factor_j with factor_j = double-layer weight 0 of pair j, summed in
// list order in the working precision (pppm.cu:172-193)
// One warp per triangle: lanes fetch 32 factors at a time, every lane then adds them in list
// order, so the sum rounds exactly like a sequential loop.  Also writes each pair's
// double-layer tap 1 with its scale applied (the factor of D[t-1] in the convolution, as the
// step evaluates it) into d1 (float for FP32 handles, double for FP64), which the two-step
// convolution of the step reads (step.cu: fix_kernel).
__global__ void denom_kernel(const int *face_start, int nt, const float *area, const __half2 *face_w,
                             const float2 *face_scale, const double2 *face_wd, double *denom, void *d1)
{
    int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    int lane = threadIdx.x & 31;
    if (i >= nt)
        return;
    int b = face_start[i], e = face_start[i + 1];
    float sf = 0;
    double sd = 0;
    for (int base = b; base < e; base += 32)
    {
        int p = base + lane;
        float f = 0;
        double fd = 0;
        if (p < e)
        {
            if (face_wd)
            {
                fd = face_wd[(size_t)p * kTaps].y;
                if (d1)
                    ((double *)d1)[p] = face_wd[(size_t)p * kTaps + 1].y;
            }
            else
            {
                f = (float)__high2half(face_w[(size_t)p * kTaps]) * face_scale[p].y;
                if (d1)
                    ((float *)d1)[p] = __high2float(face_w[(size_t)p * kTaps + 1]) * face_scale[p].y;
            }
        }
        int cnt = min(32, e - base);
        for (int j = 0; j < cnt; j++)
        {
            if (face_wd)
                sd += __shfl_sync(0xffffffffu, fd, j);
            else
                sf += __shfl_sync(0xffffffffu, f, j);
        }
    }
    if (lane == 0)
        denom[i] = face_wd ? 0.5 * (double)area[i] - sd : 0.5 * area[i] - sf;
}

DevConsts make_consts(const Handle &h)
{
    DevConsts dc;
    dc.lambda = h.tc.lambda;
    dc.lambda_d = h.tc.lambda_d;
    for (int k = 0; k < kTaps; k++)
    {
        dc.wave_re[k] = h.tc.wave_re[k];
        dc.wave_im[k] = h.tc.wave_im[k];
        dc.wave_re_d[k] = h.tc.wave_re_d[k];
        dc.wave_im_d[k] = h.tc.wave_im_d[k];
    }
    dc.threshold = h.tc.threshold;
    dc.c = h.prm.c;
    dc.dt = h.prm.dt;
    dc.h = h.prm.dl;
    dc.mn = f3{h.prm.min_pos[0], h.prm.min_pos[1], h.prm.min_pos[2]};
    dc.res = h.res;
    dc.tw = h.d_tw;
    return dc;
}

// Per grid-cache record, the factor of the triangle's NEW Dirichlet value in the record's term
// one step later (the step's two-step near-field terms, step.cu: near_terms2): double-layer tap 1
// of the FDTD-near records (r < 27; they pair record tap j + 1 with history tap j) and tap 0 of the
// BEM-near records, with the record's scale applied as the step applies it.
__global__ void gc_factor_kernel(const __half2 *w, const float2 *scale, const double2 *wd, long long n, float *f,
                                 double *fd)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int tap = (i % 54) < 27 ? 1 : 0;
    if (wd)
        fd[i] = wd[i * kTaps + tap].y;
    else
        f[i] = __high2float(w[i * kTaps + tap]) * scale[i].y;
}

}  // namespace

// ---- motion checkpoints (pppm_checkpoint_*)
// A checkpoint keeps in device memory what a refresh overwrites wholesale - the vertex
// positions, the grid-cache records with their geometry snapshot - and the pool size.  The
// pool itself stays live: later refreshes only append to it, except for the in-place rewrites
// of pairs whose geometry moved, whose old records the newest checkpoint logs (log_rewrites_
// kernel).  A rewind writes the logs back, newest first, truncates the pool and rebuilds the
// per-centre tables from the pool keys.  Checkpoints form a stack: rewinding to one drops the
// later ones, and its own log restarts empty (the handle is back at its state).
struct LogBatch
{
    void *buf = nullptr;
    int n = 0;
};

struct MotionCheckpoint
{
    void *buf = nullptr;  // a chunk of the journal's arena
    size_t bytes = 0;
    long long used = 0;
    bool gc_empty = false;
    std::vector<LogBatch> log;
};

// Checkpoints live in an arena of slabs (slab i holds 8 * 2^i checkpoints of `chunk` bytes), so
// a run of many checkpoints costs a few allocations, and a cleared journal keeps its slabs for
// the next run unless released.
struct Journal
{
    std::vector<MotionCheckpoint> stack;
    std::vector<void *> slabs;
    size_t chunk = 0;
};

namespace
{
struct Span
{
    void *dev;
    size_t bytes;
};

std::vector<Span> checkpoint_parts(Handle &h)
{
    const size_t nt = (size_t)h.nt, rec = h.fp64 ? kTaps * sizeof(double2) : kTaps * sizeof(__half2);
    std::vector<Span> parts = {{h.d_verts, sizeof(float) * 3 * (size_t)h.nv}, {h.d_gc_w, nt * 54 * rec}};
    if (!h.fp64)
        parts.push_back({h.d_gc_scale, nt * 54 * sizeof(float2)});
    parts.push_back({h.d_gc_snap, nt * 7 * sizeof(float)});
    return parts;
}

size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// byte offsets of a log batch of n entries: slots, records, scales (FP32), metas
void log_layout(const Handle &h, int n, size_t off[4], size_t *total)
{
    const size_t rec = h.fp64 ? kTaps * sizeof(double2) : kTaps * sizeof(__half2);
    off[0] = 0;
    off[1] = align16(sizeof(int) * (size_t)n);
    off[2] = off[1] + rec * (size_t)n;
    off[3] = off[2] + (h.fp64 ? 0 : sizeof(float2) * (size_t)n);
    *total = off[3] + sizeof(float2) * (size_t)n;
}

void free_checkpoint(MotionCheckpoint &c)
{
    for (LogBatch &b : c.log)
        dev_free(b.buf);
    c.log.clear();
    c.buf = nullptr;  // its chunk stays in the arena
}

// the arena chunk of checkpoint k (slabs allocated as needed)
int arena_chunk(Journal &J, int k, size_t chunk, void **out)
{
    if (J.chunk != chunk)
    {
        for (void *p : J.slabs)
            dev_free(p);
        J.slabs.clear();
        J.chunk = chunk;
    }
    int base = 0;
    for (size_t i = 0;; i++)
    {
        const int n = 8 << i;
        if (i == J.slabs.size())
        {
            void *p = nullptr;
            PB_TRY(dev_alloc(&p, chunk * (size_t)n));
            J.slabs.push_back(p);
        }
        if (k < base + n)
        {
            *out = (char *)J.slabs[i] + chunk * (size_t)(k - base);
            return PPPM_OK;
        }
        base += n;
    }
}
}  // namespace

int journal_count(const Handle &h) { return h.journal ? (int)h.journal->stack.size() : 0; }

long long journal_floor(const Handle &h) { return journal_count(h) ? h.journal->stack.back().used : 0; }

size_t journal_bytes(const Handle &h)
{
    size_t b = 0;
    if (h.journal)
    {
        for (size_t i = 0; i < h.journal->slabs.size(); i++)
            b += h.journal->chunk * (size_t)(8 << i);
        for (const MotionCheckpoint &c : h.journal->stack)
            for (const LogBatch &l : c.log)
            {
                size_t off[4], total;
                log_layout(h, l.n, off, &total);
                b += total;
            }
    }
    return b;
}

void journal_clear(Handle &h, bool release)
{
    if (!h.journal)
        return;
    cudaStreamSynchronize(h.stream);
    for (MotionCheckpoint &c : h.journal->stack)
        free_checkpoint(c);
    h.journal->stack.clear();
    if (release)
    {
        for (void *p : h.journal->slabs)
            dev_free(p);
        delete h.journal;
        h.journal = nullptr;
    }
}

// the old records of the n slots below `floor` that this refresh recomputes, appended to the
// newest checkpoint's log (before the recompute kernels overwrite them)
int journal_log(Handle &h, const int *work, int nwork, long long floor, int n)
{
    const size_t rec = h.fp64 ? kTaps * sizeof(double2) : kTaps * sizeof(__half2);
    size_t off[4], total;
    log_layout(h, n, off, &total);
    LogBatch b;
    PB_TRY(dev_alloc(&b.buf, total));
    b.n = n;
    char *base = (char *)b.buf;
    log_rewrites_kernel<<<div_up(nwork, 256), 256, 0, h.stream>>>(
        work, nwork, h.d_face_pool, floor, h.d_pair_old_meta, (const int4 *)h.d_pool_w, h.d_pool_scale,
        (int)(rec / sizeof(int4)), n, h.d_log_count + 1, (int *)(base + off[0]), (int4 *)(base + off[1]),
        h.fp64 ? nullptr : (float2 *)(base + off[2]), (float2 *)(base + off[3]));
    h.launches++;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
    {
        dev_free(b.buf);
        set_error("CUDA error %s at %s:%d", cudaGetErrorString(e), __FILE__, __LINE__);
        return PPPM_ERR_CUDA;
    }
    h.journal->stack.back().log.push_back(b);
    return PPPM_OK;
}

int journal_push(Handle &h, int *id)
{
    if (!h.mesh_set || !h.d_gc_w || h.prm.method != PPPM_METHOD_PPPM)
    {
        set_error("checkpoint: needs a mesh (PPPM method)");
        return PPPM_ERR_STATE;
    }
    if (h.tables_stale)
    {
        set_error("checkpoint: call pppm_update_mesh after a rewind or restore first");
        return PPPM_ERR_STATE;
    }
    if (!h.journal)
    {
        h.journal = new (std::nothrow) Journal();
        if (!h.journal)
            return PPPM_ERR_NOMEM;
    }
    MotionCheckpoint c;
    for (const Span &p : checkpoint_parts(h))
        c.bytes += align16(p.bytes);
    PB_TRY(arena_chunk(*h.journal, (int)h.journal->stack.size(), (c.bytes + 255) & ~(size_t)255, &c.buf));
    char *o = (char *)c.buf;
    for (const Span &p : checkpoint_parts(h))
    {
        PB_CUDA(cudaMemcpyAsync(o, p.dev, p.bytes, cudaMemcpyDeviceToDevice, h.stream));
        o += align16(p.bytes);
    }
    c.used = h.pool_used;
    c.gc_empty = h.gc_empty;
    h.journal->stack.push_back(std::move(c));
    *id = (int)h.journal->stack.size() - 1;
    return PPPM_OK;
}

int journal_rewind(Handle &h, int id)
{
    if (id < 0 || id >= journal_count(h))
    {
        set_error("checkpoint %d: no such checkpoint (%d held)", id, journal_count(h));
        return PPPM_ERR_ARG;
    }
    cudaStream_t s = h.stream;
    const size_t rec = h.fp64 ? kTaps * sizeof(double2) : kTaps * sizeof(__half2);
    const int words = (int)(rec / sizeof(int4));
    std::vector<MotionCheckpoint> &st = h.journal->stack;
    // undo the logged rewrites, newest first
    for (int k = (int)st.size() - 1; k >= id; k--)
        for (int b = (int)st[k].log.size() - 1; b >= 0; b--)
        {
            const LogBatch &l = st[k].log[b];
            size_t off[4], total;
            log_layout(h, l.n, off, &total);
            const char *base = (const char *)l.buf;
            apply_log_kernel<<<div_up(l.n, 256), 256, 0, s>>>(
                l.n, (const int *)(base + off[0]), (const int4 *)(base + off[1]),
                h.fp64 ? nullptr : (const float2 *)(base + off[2]), (const float2 *)(base + off[3]), words,
                (int4 *)h.d_pool_w, h.d_pool_scale, h.d_pool_meta);
            h.launches++;
            PB_CHECK_LAUNCH();
        }
    // the checkpoint's grid cache and vertices, the pool truncated to its size, the tables
    const MotionCheckpoint &c = st[id];
    const char *o = (const char *)c.buf;
    for (const Span &p : checkpoint_parts(h))
    {
        PB_CUDA(cudaMemcpyAsync(p.dev, o, p.bytes, cudaMemcpyDeviceToDevice, s));
        o += align16(p.bytes);
    }
    const int u = (int)c.used;
    PB_CUDA(cudaMemcpyAsync(h.d_pool_count, &u, sizeof(int), cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemsetAsync(h.d_fc_keys, 0xff, sizeof(int) * (size_t)h.nt * kFaceCacheSlots, s));
    PB_CUDA(cudaMemsetAsync(h.d_status, 0, sizeof(int), s));
    if (c.used > 0)
    {
        fc_rebuild_kernel<<<div_up(c.used, 256), 256, 0, s>>>(h.d_pool_key, c.used, h.d_fc_keys, h.d_fc_slot,
                                                              h.d_status);
        h.launches++;
        PB_CHECK_LAUNCH();
    }
    int st_word = 0;
    PB_TRY(read_int(h, h.d_status, &st_word));  // also orders the frees below after the copies
    if (st_word)
    {
        set_error("checkpoint rewind: face-cache table overflow while rebuilding");
        return st_word;
    }
    for (LogBatch &l : st[id].log)
        dev_free(l.buf);
    st[id].log.clear();
    for (int k = (int)st.size() - 1; k > id; k--)
    {
        free_checkpoint(st[k]);
        st.pop_back();
    }
    h.pool_used = c.used;
    h.gc_empty = c.gc_empty;
    h.tables_stale = true;  // lists and dense tables still describe the geometry before the rewind
    h.mesh_version++;
    return PPPM_OK;
}

int gc_factors(Handle &h, cudaStream_t gs)
{
    const long long n = (long long)h.nt * 54;
    if (!h.d_gc_f || n == 0)
        return PPPM_OK;
    gc_factor_kernel<<<div_up(n, 256), 256, 0, gs>>>(
        h.fp64 ? nullptr : (const __half2 *)h.d_gc_w, h.d_gc_scale, h.fp64 ? (const double2 *)h.d_gc_w : nullptr, n,
        h.fp64 ? nullptr : (float *)h.d_gc_f, h.fp64 ? (double *)h.d_gc_f : nullptr);
    h.launches++;
    PB_CHECK_LAUNCH();
    return PPPM_OK;
}

// One-time allocations of the caches (the first set_mesh)
static int cache_alloc(Handle &h)
{
    if (h.d_gc_w)
        return PPPM_OK;
    cudaStream_t s = h.stream;
    const int nt = h.nt;
    const size_t rec_bytes = h.fp64 ? kTaps * sizeof(double2) : kTaps * sizeof(__half2);
    PB_TRY(dev_alloc(&h.d_gc_w, (size_t)nt * 54 * rec_bytes));
    PB_TRY(dev_alloc(&h.d_gc_f, (size_t)nt * 54 * h.real_size));
    if (!h.fp64)
        PB_TRY(dalloc(&h.d_gc_scale, (size_t)nt * 54));
    PB_TRY(dalloc(&h.d_gc_snap, (size_t)nt * 7));
    PB_TRY(dalloc(&h.d_gc_flag, (size_t)nt));
    PB_TRY(dalloc(&h.d_fc_keys, (size_t)nt * kFaceCacheSlots));
    PB_TRY(dalloc(&h.d_fc_slot, (size_t)nt * kFaceCacheSlots));
    PB_CUDA(cudaMemsetAsync(h.d_fc_keys, 0xff, sizeof(int) * (size_t)nt * kFaceCacheSlots, s));
    PB_TRY(dalloc(&h.d_pool_count, 1));
    PB_CUDA(cudaMemsetAsync(h.d_pool_count, 0, sizeof(int), s));
    PB_TRY(dalloc(&h.d_log_count, 2));
    PB_TRY(dalloc(&h.d_face_interp, (size_t)nt * 8));
    if (h.fp64)
        PB_TRY(dalloc(&h.d_face_interp_d, (size_t)nt * 8));
    PB_TRY(dalloc(&h.d_face_denom, (size_t)nt));
    PB_TRY(dalloc(&h.d_tw, (size_t)16));
    twiddle_kernel<<<1, 1, 0, s>>>(h.d_tw);
    h.launches++;
    PB_CHECK_LAUNCH();
    h.pool_used = 0;
    h.gc_empty = true;
    return PPPM_OK;
}

// The grid-cache refresh (recompute flags, records, the completion factors of the two-step terms)
// on stream gs
static int grid_cache_refresh(Handle &h, cudaStream_t gs)
{
    const int nt = h.nt, T = 256;
    DevConsts dc = make_consts(h);
    dc.tw = h.d_tw;
    gc_flag_kernel<<<div_up(nt, T), T, 0, gs>>>(h.d_center, h.d_normal, h.d_area, h.d_gc_snap, nt, h.prm.dl,
                                                h.gc_empty ? 1 : 0, h.d_gc_flag);
    h.launches++;
    PB_CHECK_LAUNCH();
    if (h.fp64)
        gc_compute_kernel_d<<<div_up((long long)nt * 27, 128), 128, 0, gs>>>(dc, h.d_verts, h.d_tris, h.d_cellc,
                                                                              h.d_center, h.d_normal, h.d_area,
                                                                              h.d_gc_flag, nt, (double2 *)h.d_gc_w,
                                                                              h.d_gc_snap);
    else
    {
        // four blocks of 37 KB shared memory per SM: ask for the largest shared-memory carve-out
        static bool carveout_set = false;
        if (!carveout_set)
        {
            PB_CUDA(cudaFuncSetAttribute(gc_block_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         cudaSharedmemCarveoutMaxShared));
            carveout_set = true;
        }
        // beside the rest of the update (side stream): two blocks per SM, half of what fits
        int blocks = nt;
        if (gs != h.stream)
        {
            int sms = 0;
            PB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h.prm.device));
            blocks = std::max(1, std::min(nt, 2 * sms));
        }
        gc_block_kernel<<<blocks, 256, 0, gs>>>(dc, h.d_verts, h.d_tris, nt, h.d_cellc, h.d_center, h.d_normal,
                                                h.d_area, h.d_gc_flag, (__half2 *)h.d_gc_w, h.d_gc_scale,
                                                h.d_gc_snap);
    }
    h.launches++;
    PB_CHECK_LAUNCH();
    h.gc_empty = false;
    return gc_factors(h, gs);
}

// The grid-cache refresh reads only the triangle geometry of this update (mesh_build's first
// kernel: centres, normals, areas, cells) and nothing else reads or writes its arrays until the
// step tables are primed, so update_mesh starts it on side2 right after the geometry kernel, where
// it runs (transcendental-bound) beside the list builds and the face-cache refresh (latency- and
// synchronisation-bound); cache_refresh joins it before returning.
int grid_cache_start(Handle &h)
{
    PB_TRY(cache_alloc(h));
    if (!h.side2 || !h.ev_upd_fork || !h.ev_upd_join)
        return PPPM_OK;  // cache_refresh then refreshes the grid cache on the handle's stream
    PB_CUDA(cudaEventRecord(h.ev_upd_fork, h.stream));
    PB_CUDA(cudaStreamWaitEvent(h.side2, h.ev_upd_fork, 0));
    PB_TRY(grid_cache_refresh(h, h.side2));
    PB_CUDA(cudaEventRecord(h.ev_upd_join, h.side2));
    h.gc_launched = true;
    return PPPM_OK;
}

void join_grid_cache(Handle &h)
{
    if (h.gc_launched)
        cudaStreamWaitEvent(h.stream, h.ev_upd_join, 0);
    h.gc_launched = false;
}

int cache_refresh(Handle &h)
{
    // whatever path this returns by, the handle's stream waits for the grid-cache branch
    struct Join
    {
        Handle &h;
        ~Join() { join_grid_cache(h); }
    } join{h};
    cudaStream_t s = h.stream;
    const int nt = h.nt, T = 256;
    const size_t rec_bytes = h.fp64 ? kTaps * sizeof(double2) : kTaps * sizeof(__half2);
    DevConsts dc = make_consts(h);
    PB_TRY(cache_alloc(h));
    dc.tw = h.d_tw;

    // ---- grid cache (already running on side2 when update_mesh started it with the geometry)
    if (!h.gc_launched)
        PB_TRY(grid_cache_refresh(h, s));

    // ---- face cache
    const f3 mn{h.prm.min_pos[0], h.prm.min_pos[1], h.prm.min_pos[2]};
    interp_kernel<<<div_up(nt, T), T, 0, s>>>(h.d_verts, h.d_tris, h.d_basec, nt, h.prm.dl, mn, h.d_face_interp,
                                               h.d_face_interp_d);
    h.launches++;
    PB_CHECK_LAUNCH();
    if (h.pf > 0)
    {
        // every pair may be new: make room for pf more records.  The first pool holds three
        // times that (the next update asks for pool_used + pf, about twice pf), so a moving scene
        // does not move its pool in its first frames; later growth is by half.
        long long need = h.pool_used + h.pf;
        if (need > h.pool_cap)
        {
            long long nc = (h.pool_cap == 0 ? 3 * need : need + need / 2) + 1024;
            void *nw = nullptr;
            float2 *nsc = nullptr, *nmeta = nullptr;
            int2 *nkey = nullptr;
            PB_TRY(dev_alloc(&nw, (size_t)nc * rec_bytes));
            if (!h.fp64)
                PB_TRY(dalloc(&nsc, (size_t)nc));
            PB_TRY(dalloc(&nmeta, (size_t)nc));
            PB_TRY(dalloc(&nkey, (size_t)nc));
            if (h.pool_used > 0)
            {
                PB_CUDA(cudaMemcpyAsync(nkey, h.d_pool_key, (size_t)h.pool_used * sizeof(int2),
                                        cudaMemcpyDeviceToDevice, s));
                PB_CUDA(cudaMemcpyAsync(nw, h.d_pool_w, (size_t)h.pool_used * rec_bytes, cudaMemcpyDeviceToDevice, s));
                if (!h.fp64)
                    PB_CUDA(cudaMemcpyAsync(nsc, h.d_pool_scale, (size_t)h.pool_used * sizeof(float2),
                                            cudaMemcpyDeviceToDevice, s));
                PB_CUDA(cudaMemcpyAsync(nmeta, h.d_pool_meta, (size_t)h.pool_used * sizeof(float2),
                                        cudaMemcpyDeviceToDevice, s));
            }
            PB_CUDA(cudaStreamSynchronize(s));
            dev_free(h.d_pool_w);
            dev_free(h.d_pool_scale);
            dev_free(h.d_pool_meta);
            dev_free(h.d_pool_key);
            h.d_pool_w = nw;
            h.d_pool_scale = nsc;
            h.d_pool_meta = nmeta;
            h.d_pool_key = nkey;
            h.pool_cap = nc;
        }
        // rewrites of slots that the newest motion checkpoint holds are logged (journal_rewind)
        const long long log_floor = journal_count(h) > 0 ? journal_floor(h) : 0;
        if (log_floor > 0)
            PB_TRY(dgrow(&h.d_pair_old_meta, h.pair_old_meta_cap, h.pf, s));
        PB_CUDA(cudaMemsetAsync(h.d_status, 0, sizeof(int), s));
        PB_CUDA(cudaMemsetAsync(h.d_log_count, 0, 2 * sizeof(int), s));
        fc_lookup_kernel<<<div_up((long long)nt * 32, T), T, 0, s>>>(
            h.d_face_start, h.d_face_nbr, nt, h.d_center, h.d_normal, h.d_fc_keys, h.d_fc_slot, h.d_pool_count,
            h.pool_cap, h.d_pool_meta, h.d_pool_key, log_floor, h.d_pair_old_meta, h.d_log_count, h.d_face_pool,
            h.d_pair_flag, h.d_status);
        h.launches++;
        PB_CHECK_LAUNCH();
        // compact the recompute list; one synchronisation reads the lookup status, the pool
        // size, the number of pairs to recompute and the number of logged rewrites
        PB_TRY(dgrow(&h.d_pair_work, h.pair_work_cap, 2 * (h.pf + 1), s));
        int *pos = h.d_pair_work;
        int *work = h.d_pair_work + (h.pf + 1);
        PB_TRY(exclusive_scan(h, h.d_pair_flag, pos, h.pf));
        int v[4];
        const int *src[4] = {h.d_status, h.d_pool_count, pos + h.pf, h.d_log_count};
        PB_TRY(read_ints(h, src, 4, v));
        if (v[0])
        {
            set_error("face cache: more than %d distinct neighbours seen by one face", kFaceCacheSlots);
            return v[0];
        }
        h.pool_used = v[1];
        const int nwork = v[2];
        if (nwork > 0)
        {
            compact_pairs_kernel<<<div_up(h.pf, T), T, 0, s>>>(h.d_pair_flag, pos, h.pf, work);
            h.launches++;
            if (v[3] > 0)
                PB_TRY(journal_log(h, work, nwork, log_floor, v[3]));
            size_t need_spec = (size_t)nwork * 18 * (h.fp64 ? sizeof(cd) : sizeof(cf));
            if (need_spec > h.spec_bytes)
            {
                dev_free(h.d_spec);
                h.d_spec = nullptr;
                PB_TRY(dev_alloc(&h.d_spec, need_spec + need_spec / 2));
                h.spec_bytes = need_spec + need_spec / 2;
            }
            if (h.fp64)
            {
                fc_spectra_kernel_d<<<div_up((long long)nwork * 18, 128), 128, 0, s>>>(
                    dc, h.d_verts, h.d_tris, h.d_face_start, nt, h.d_face_nbr, work, nwork, (cd *)h.d_spec);
                fc_finish_kernel_d<<<div_up(nwork, 128), 128, 0, s>>>(
                    dc, h.d_verts, h.d_tris, h.d_center, h.d_basec, h.d_face_interp_d, h.d_face_start, nt,
                    h.d_face_nbr, h.d_face_pool, work, nwork, (const cd *)h.d_spec, (double2 *)h.d_pool_w);
            }
            else
            {
                int mode = h.prm.weights == PPPM_WEIGHTS_FP64 ? 1 : 0;
                fc_spectra_kernel<<<div_up((long long)nwork * 9, 128), 128, 0, s>>>(
                    dc, h.d_verts, h.d_tris, h.d_center, h.d_basec, h.d_face_interp, h.d_face_start, nt,
                    h.d_face_nbr, work, nwork, mode, (cf *)h.d_spec);
                fc_finish_kernel<<<div_up(nwork, 128), 128, 0, s>>>(dc, h.d_face_pool, work, nwork,
                                                                     (const cf *)h.d_spec, (__half2 *)h.d_pool_w,
                                                                     h.d_pool_scale);
            }
            h.launches += 2;
            PB_CHECK_LAUNCH();
        }
        if (h.fp64)
            gather_face_kernel<double2><<<div_up(gather_face_threads<double2>(h.pf), T), T, 0, s>>>(
                h.d_face_pool, h.pf, (const double2 *)h.d_pool_w, nullptr, (double2 *)h.d_face_w, nullptr);
        else
            gather_face_kernel<__half2><<<div_up(gather_face_threads<__half2>(h.pf), T), T, 0, s>>>(
                h.d_face_pool, h.pf, (const __half2 *)h.d_pool_w, h.d_pool_scale, (__half2 *)h.d_face_w,
                h.d_face_scale);
        h.launches++;
        PB_CHECK_LAUNCH();
    }
    denom_kernel<<<div_up((long long)nt * 32, T), T, 0, s>>>(h.d_face_start, nt, h.d_area,
                                              h.fp64 ? nullptr : (const __half2 *)h.d_face_w, h.d_face_scale,
                                              h.fp64 ? (const double2 *)h.d_face_w : nullptr, h.d_face_denom,
                                              h.d_face_d1);
    h.launches++;
    PB_CHECK_LAUNCH();
    return PPPM_OK;
}

// ---- the motion-frame state of the caches (pppm_save_cache_state / pppm_restore_cache_state)
// Blob (host or device memory): int64 header[6] = {magic, nt, nv, record bytes, pool_used, gc_empty}, then the vertex
// positions, the grid-cache records (+ scales), their geometry snapshot, the face-cache key and
// slot tables, and the pool's first pool_used records (+ scales) with their geometry meta.
namespace
{
constexpr long long kCacheMagic = 0x7070706d63616368ll;

struct CachePart
{
    void *dev;
    size_t bytes;
};

std::vector<CachePart> cache_parts(Handle &h, long long pool_used)
{
    const size_t nt = (size_t)h.nt, rec = h.fp64 ? kTaps * sizeof(double2) : kTaps * sizeof(__half2);
    std::vector<CachePart> parts = {{h.d_verts, sizeof(float) * 3 * (size_t)h.nv}, {h.d_gc_w, nt * 54 * rec}};
    if (!h.fp64)
        parts.push_back({h.d_gc_scale, nt * 54 * sizeof(float2)});
    parts.push_back({h.d_gc_snap, nt * 7 * sizeof(float)});
    parts.push_back({h.d_fc_keys, nt * kFaceCacheSlots * sizeof(int)});
    parts.push_back({h.d_fc_slot, nt * kFaceCacheSlots * sizeof(int)});
    parts.push_back({h.d_pool_w, (size_t)pool_used * rec});
    if (!h.fp64)
        parts.push_back({h.d_pool_scale, (size_t)pool_used * sizeof(float2)});
    parts.push_back({h.d_pool_meta, (size_t)pool_used * sizeof(float2)});
    parts.push_back({h.d_pool_key, (size_t)pool_used * sizeof(int2)});
    return parts;
}
}  // namespace

size_t cache_state_bytes(Handle &h)
{
    size_t b = 6 * sizeof(long long);
    for (const CachePart &p : cache_parts(h, h.pool_used))
        b += p.bytes;
    return b;
}

int cache_state_save(Handle &h, void *dst, size_t bytes)
{
    if (!h.mesh_set || !h.d_gc_w || h.prm.method != PPPM_METHOD_PPPM)
    {
        set_error("cache state: needs a mesh (PPPM method)");
        return PPPM_ERR_STATE;
    }
    if (bytes < cache_state_bytes(h))
        return PPPM_ERR_ARG;
    const size_t rec = h.fp64 ? kTaps * sizeof(double2) : kTaps * sizeof(__half2);
    const long long hdr[6] = {kCacheMagic, h.nt, h.nv, (long long)rec, h.pool_used, h.gc_empty ? 1 : 0};
    // host or device memory alike (unified addressing): a checkpoint may stay in HBM
    PB_CUDA(cudaMemcpyAsync(dst, hdr, sizeof(hdr), cudaMemcpyDefault, h.stream));
    char *o = (char *)dst + sizeof(hdr);
    for (const CachePart &p : cache_parts(h, h.pool_used))
    {
        if (p.bytes)
            PB_CUDA(cudaMemcpyAsync(o, p.dev, p.bytes, cudaMemcpyDefault, h.stream));
        o += p.bytes;
    }
    PB_CUDA(cudaStreamSynchronize(h.stream));  // hdr is a stack array; the caller owns dst on return
    return PPPM_OK;
}

int cache_state_restore(Handle &h, const void *src, size_t bytes)
{
    if (!h.mesh_set || !h.d_gc_w || h.prm.method != PPPM_METHOD_PPPM)
    {
        set_error("cache state: needs a mesh (PPPM method)");
        return PPPM_ERR_STATE;
    }
    const size_t rec = h.fp64 ? kTaps * sizeof(double2) : kTaps * sizeof(__half2);
    long long hdr[6] = {0, 0, 0, 0, -1, 0};
    if (bytes >= sizeof(hdr))
    {
        PB_CUDA(cudaMemcpyAsync(hdr, src, sizeof(hdr), cudaMemcpyDefault, h.stream));
        PB_CUDA(cudaStreamSynchronize(h.stream));
    }
    if (bytes < sizeof(hdr) || hdr[0] != kCacheMagic || hdr[1] != h.nt || hdr[2] != h.nv ||
        hdr[3] != (long long)rec || hdr[4] < 0)
    {
        set_error("cache state: not a blob of this handle's mesh and precision");
        return PPPM_ERR_ARG;
    }
    const long long used = hdr[4];
    journal_clear(h, false);  // the blob replaces the pool the checkpoints' logs refer to
    size_t need = 6 * sizeof(long long);
    for (const CachePart &p : cache_parts(h, used))
        need += p.bytes;
    if (bytes < need)
        return PPPM_ERR_ARG;
    if (used > h.pool_cap)
    {
        // the blob's pool is larger than this handle's: grow (contents are replaced below)
        dev_free(h.d_pool_w);
        dev_free(h.d_pool_scale);
        dev_free(h.d_pool_meta);
        dev_free(h.d_pool_key);
        h.d_pool_w = nullptr;
        h.d_pool_scale = nullptr;
        h.d_pool_meta = nullptr;
        h.d_pool_key = nullptr;
        h.pool_cap = 0;
        const long long nc = used + used / 2 + 1024;
        PB_TRY(dev_alloc(&h.d_pool_w, (size_t)nc * rec));
        if (!h.fp64)
            PB_TRY(dalloc(&h.d_pool_scale, (size_t)nc));
        PB_TRY(dalloc(&h.d_pool_meta, (size_t)nc));
        PB_TRY(dalloc(&h.d_pool_key, (size_t)nc));
        h.pool_cap = nc;
    }
    const char *o = (const char *)src + sizeof(hdr);
    for (const CachePart &p : cache_parts(h, used))
    {
        if (p.bytes)
            PB_CUDA(cudaMemcpyAsync(p.dev, o, p.bytes, cudaMemcpyDefault, h.stream));
        o += p.bytes;
    }
    const int u = (int)used;
    PB_CUDA(cudaMemcpyAsync(h.d_pool_count, &u, sizeof(int), cudaMemcpyHostToDevice, h.stream));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    h.pool_used = used;
    h.gc_empty = hdr[5] != 0;
    h.tables_stale = true;  // the lists and dense tables still describe the geometry before the restore
    h.mesh_version++;
    return PPPM_OK;
}

int cache_free(Handle &h)
{
    journal_clear(h, true);
    dev_free(h.d_pool_key);
    dev_free(h.d_pair_old_meta);
    dev_free(h.d_log_count);
    h.d_pool_key = nullptr;
    h.d_pair_old_meta = nullptr;
    h.d_log_count = nullptr;
    h.pair_old_meta_cap = 0;
    dev_free(h.d_gc_f);
    h.d_gc_f = nullptr;
    void *ptrs[] = {h.d_gc_w,      h.d_gc_scale,  h.d_gc_snap,   h.d_gc_flag,    h.d_fc_keys,
                    h.d_fc_slot,   h.d_pool_w,    h.d_pool_scale, h.d_pool_meta, h.d_pool_count,
                    h.d_face_interp, h.d_face_interp_d, h.d_face_denom, h.d_spec, h.d_tw};
    for (void *p : ptrs)
        dev_free(p);
    h.d_gc_w = nullptr;
    h.d_gc_scale = nullptr;
    h.d_gc_snap = nullptr;
    h.d_gc_flag = nullptr;
    h.d_fc_keys = h.d_fc_slot = h.d_pool_count = nullptr;
    h.d_pool_w = nullptr;
    h.d_pool_scale = h.d_pool_meta = nullptr;
    h.d_face_interp = nullptr;
    h.d_face_interp_d = nullptr;
    h.d_face_denom = nullptr;
    h.d_spec = nullptr;
    h.d_tw = nullptr;
    h.pool_cap = h.pool_used = 0;
    h.spec_bytes = 0;
    return PPPM_OK;
}

}  // namespace pb

// ---------------------------------------------------------------- parity import -------
namespace pb
{

namespace
{
// reference LayerWeightHalf record: half s[16], float ms, half d[16], float md (72 bytes,
// bem.h:163-169)
struct RefRecord
{
    __half s[kTaps];
    float ms;
    __half d[kTaps];
    float md;
};
static_assert(sizeof(RefRecord) == 72, "reference record layout");

__global__ void import_records_kernel(const RefRecord *in, long long n, const long long *dst_index, __half2 *w,
                                      float2 *scale)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    long long r = dst_index ? dst_index[i] : i;
    RefRecord rec = in[i];
    for (int k = 0; k < kTaps; k++)
        w[r * kTaps + k] = __halves2half2(rec.s[k], rec.d[k]);
    scale[r] = make_float2(rec.ms, rec.md);
}

__global__ void snapshot_kernel(const float *center, const float *normal, const float *area, int nt, float *snap)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt)
        return;
    for (int k = 0; k < 3; k++)
    {
        snap[7 * i + k] = center[3 * i + k];
        snap[7 * i + 3 + k] = normal[3 * i + k];
    }
    snap[7 * i + 6] = area[i];
}
}  // namespace

int cache_regather(Handle &h)
{
    cudaStream_t s = h.stream;
    const int T = 256;
    if (h.pf > 0)
    {
        if (h.fp64)
            gather_face_kernel<double2><<<div_up(gather_face_threads<double2>(h.pf), T), T, 0, s>>>(
                h.d_face_pool, h.pf, (const double2 *)h.d_pool_w, nullptr, (double2 *)h.d_face_w, nullptr);
        else
            gather_face_kernel<__half2><<<div_up(gather_face_threads<__half2>(h.pf), T), T, 0, s>>>(
                h.d_face_pool, h.pf, (const __half2 *)h.d_pool_w, h.d_pool_scale, (__half2 *)h.d_face_w,
                h.d_face_scale);
        h.launches++;
    }
    denom_kernel<<<div_up((long long)h.nt * 32, T), T, 0, s>>>(h.d_face_start, h.nt, h.d_area,
                                                h.fp64 ? nullptr : (const __half2 *)h.d_face_w, h.d_face_scale,
                                                h.fp64 ? (const double2 *)h.d_face_w : nullptr, h.d_face_denom,
                                              h.d_face_d1);
    h.launches++;
    PB_CHECK_LAUNCH();
    return PPPM_OK;
}

int cache_import_grid(Handle &h, const void *records)
{
    if (h.fp64)
        return PPPM_ERR_ARG;
    journal_clear(h, false);  // imported records are not logged: the checkpoints would not undo them
    cudaStream_t s = h.stream;
    size_t n = (size_t)h.nt * 54;
    void *tmp = nullptr;
    PB_TRY(dev_alloc(&tmp, n * sizeof(RefRecord)));
    PB_CUDA(cudaMemcpyAsync(tmp, records, n * sizeof(RefRecord), cudaMemcpyHostToDevice, s));
    import_records_kernel<<<div_up((long long)n, 256), 256, 0, s>>>((const RefRecord *)tmp, (long long)n, nullptr,
                                                                      (__half2 *)h.d_gc_w, h.d_gc_scale);
    snapshot_kernel<<<div_up(h.nt, 256), 256, 0, s>>>(h.d_center, h.d_normal, h.d_area, h.nt, h.d_gc_snap);
    h.launches += 2;
    PB_CHECK_LAUNCH();
    PB_CUDA(cudaStreamSynchronize(s));
    dev_free(tmp);
    h.gc_empty = false;
    PB_TRY(gc_factors(h, h.stream));
    return cache_regather(h);
}

int cache_import_face(Handle &h, const int *pairs, const void *records, int n)
{
    if (h.fp64)
        return PPPM_ERR_ARG;
    journal_clear(h, false);  // imported records are not logged: the checkpoints would not undo them
    cudaStream_t s = h.stream;
    // (centre, neighbour) -> pool slot of the current face list
    std::vector<int> start(h.nt + 1), nbr(h.pf), pool(h.pf);
    PB_CUDA(cudaMemcpyAsync(start.data(), h.d_face_start, sizeof(int) * (h.nt + 1), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(nbr.data(), h.d_face_nbr, sizeof(int) * h.pf, cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(pool.data(), h.d_face_pool, sizeof(int) * h.pf, cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    std::vector<long long> dst(n);
    for (int i = 0; i < n; i++)
    {
        int c = pairs[2 * i], j = pairs[2 * i + 1];
        if (c < 0 || c >= h.nt)
            return PPPM_ERR_ARG;
        long long found = -1;
        for (int p = start[c]; p < start[c + 1]; p++)
            if (nbr[p] == j)
            {
                found = pool[p];
                break;
            }
        if (found < 0)
        {
            set_error("imported face pair (%d, %d) is not in the current 4^3 lists", c, j);
            return PPPM_ERR_ARG;
        }
        dst[i] = found;
    }
    void *tmp = nullptr;
    long long *ddst = nullptr;
    PB_TRY(dev_alloc(&tmp, (size_t)n * sizeof(RefRecord)));
    PB_TRY(dalloc(&ddst, (size_t)n));
    PB_CUDA(cudaMemcpyAsync(tmp, records, (size_t)n * sizeof(RefRecord), cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(ddst, dst.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, s));
    import_records_kernel<<<div_up(n, 256), 256, 0, s>>>((const RefRecord *)tmp, n, ddst, (__half2 *)h.d_pool_w,
                                                         h.d_pool_scale);
    h.launches++;
    PB_CHECK_LAUNCH();
    PB_CUDA(cudaStreamSynchronize(s));
    dev_free(tmp);
    dev_free(ddst);
    return cache_regather(h);
}

}  // namespace pb
