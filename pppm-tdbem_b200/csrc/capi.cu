// C ABI of libpppm_b200 (include/pppm_b200.h).  Every entry point validates its arguments,
// returns a status code and never throws; CUDA failures are reported as PPPM_ERR_CUDA with
// the message kept for pppm_last_error_message().
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>
#include "handle.cuh"

namespace pb
{

static thread_local std::string g_error;

void set_error(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
}

const char *last_error() { return g_error.c_str(); }

int dev_alloc(void **p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0)
        bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess)
    {
        *p = nullptr;
        set_error("cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PPPM_ERR_NOMEM : PPPM_ERR_CUDA;
    }
    return PPPM_OK;
}

void dev_free(void *p)
{
    if (p)
        cudaFree(p);
}

// TDBEM::init (bem.h:264-277) evaluated with the reference's host arithmetic: lambda from
// max((c dt)^{3/16}, EPS^{1/32}) in double, s_k = lambda e^{-2 pi i k / 16} rounded to
// complex<float>, BDF2 in float, division by c dt and multiplication by i in double.
void tdbem_init(TdbemConsts &out, float dt, float grid_size, float c)
{
    const double PI = PB_PI;
    float dtc = dt * c;
    double lam = std::max(std::pow((double)dtc, 3.0 / kTaps), std::pow((double)1e-8f, 1.0 / (2 * kTaps)));
    out.lambda = (float)lam;
    for (int k = 0; k < kTaps; k++)
    {
        double zre = (-2 * PI * 0.0f) / kTaps * k, zim = (-2 * PI * 1.0f) / kTaps * k;
        double er, ei;
        if (zim == 0)
        {
            er = std::exp(zre);
            ei = zim;
        }
        else
        {
            er = std::cos(zim);
            ei = std::sin(zim);
        }
        float sre = (float)(out.lambda * er), sim = (float)(out.lambda * ei);
        float qre = sre * sre - sim * sim, qim = sre * sim + sim * sre;  // s * s
        float tre = 4 * sre, tim = 4 * sim;                               // 4 * s
        float ure = qre - tre, uim = qim - tim;
        ure = ure + 3;
        double bre = 0.5 * ure, bim = 0.5 * uim;  // BDF2 = 0.5 (s^2 - 4 s + 3)
        bre = bre / dtc;
        bim = bim / dtc;
        double wre = bre * 0.0f - bim * 1.0f, wim = bre * 1.0f + bim * 0.0f;  // * i
        out.wave_re[k] = (float)wre;
        out.wave_im[k] = (float)wim;
    }
    out.threshold = (float)(grid_size * 0.1);
    // the same constants in double for the FP64 yardstick
    double dtcd = (double)dt * (double)c;
    out.lambda_d = std::max(std::pow(dtcd, 3.0 / kTaps), std::pow(1e-8, 1.0 / (2 * kTaps)));
    for (int k = 0; k < kTaps; k++)
    {
        double ang = -2 * M_PI * k / kTaps;
        double sre = out.lambda_d * std::cos(ang), sim = out.lambda_d * std::sin(ang);
        double ure = sre * sre - sim * sim - 4 * sre + 3, uim = 2 * sre * sim - 4 * sim;
        ure *= 0.5 / dtcd;
        uim *= 0.5 / dtcd;
        out.wave_re_d[k] = -uim;
        out.wave_im_d[k] = ure;
    }
}

}  // namespace pb

using namespace pb;

struct pppm_handle
{
    Handle h;
};

namespace
{

int check_handle(pppm_handle *p)
{
    if (!p)
    {
        set_error("null handle");
        return PPPM_ERR_ARG;
    }
    return PPPM_OK;
}

// release every array sized by the mesh (a failed set_mesh leaves the handle mesh-free)
void free_mesh(Handle &h)
{
    cudaStreamSynchronize(h.stream);
    adjoint_free(h);
    ghost_free(h);
    h.mesh_version++;
    cache_free(h);
    void **ptrs[] = {(void **)&h.d_verts,      (void **)&h.d_tris,        (void **)&h.d_center,
                     (void **)&h.d_normal,     (void **)&h.d_area,        (void **)&h.d_cellc,
                     (void **)&h.d_basec,      (void **)&h.d_cell,        (void **)&h.d_base,
                     (void **)&h.d_cell_count, (void **)&h.d_cell_start,  (void **)&h.d_cell_tris,
                     (void **)&h.d_base_count, (void **)&h.d_base_start,  (void **)&h.d_base_tris,
                     (void **)&h.d_cursor,     (void **)&h.d_flags,       (void **)&h.d_n3_cell,
                     (void **)&h.d_n3_start,   (void **)&h.d_p3_tri,      (void **)&h.d_p3_woff,
                     (void **)&h.d_b4_cell,
                     (void **)&h.d_b4_start,   (void **)&h.d_n4_tris,     (void **)&h.d_face_start,
                     (void **)&h.d_face_nbr,   (void **)&h.d_face_pool,   (void **)&h.d_face_w,
                     (void **)&h.d_face_scale, (void **)&h.d_face_corner, (void **)&h.d_pair_flag,
                     (void **)&h.d_status,     (void **)&h.d_neumann,     (void **)&h.d_dirichlet,
                     (void **)&h.d_hist,       (void **)&h.d_terms,       (void **)&h.d_conv,
                     (void **)&h.d_gneu,       (void **)&h.d_gneu_old,    (void **)&h.d_face_d1,
                     (void **)&h.d_conv1,      (void **)&h.d_dlast,       (void **)&h.d_terms1};
    for (void **q : ptrs)
    {
        dev_free(*q);
        *q = nullptr;
    }
    h.p3_cap = h.n4_cap = h.pf_cap = 0;
    h.n3 = h.b4 = 0;
    h.p3 = h.p4 = h.pf = 0;
    h.nv = h.nt = 0;
    h.gc_empty = true;
    cudaMemsetAsync(h.d_corr_mask, 0, sizeof(unsigned) * ((h.n_cells + 31) / 32), h.stream);
}

int ensure_series(Handle &h, long long extra)
{
    int nl = (int)h.listen_xyz.size() / 3;
    if (nl == 0)
        return PPPM_OK;
    long long need = h.series_count + extra;
    if (need <= h.series_cap)
        return PPPM_OK;
    long long cap = std::max<long long>(need + need / 2, 4096);
    void *nw = nullptr;
    PB_TRY(dev_alloc(&nw, (size_t)cap * nl * h.real_size));
    if (h.d_series && h.series_count > 0)
        PB_CUDA(cudaMemcpyAsync(nw, h.d_series, (size_t)h.series_count * nl * h.real_size, cudaMemcpyDeviceToDevice,
                                h.stream));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    dev_free(h.d_series);
    h.d_series = nw;
    h.series_cap = cap;
    return PPPM_OK;
}

// reference record for dumps
struct RefRecord
{
    __half s[kTaps];
    float ms;
    __half d[kTaps];
    float md;
};

void to_ref_records(const __half2 *w, const float2 *sc, size_t n, RefRecord *out)
{
    for (size_t r = 0; r < n; r++)
    {
        for (int k = 0; k < kTaps; k++)
        {
            out[r].s[k] = __low2half(w[r * kTaps + k]);
            out[r].d[k] = __high2half(w[r * kTaps + k]);
        }
        out[r].ms = sc[r].x;
        out[r].md = sc[r].y;
    }
}

template <typename T>
int d2h(Handle &h, std::vector<T> &v, const void *src, size_t n)
{
    v.resize(n);
    if (n == 0)
        return PPPM_OK;
    PB_CUDA(cudaMemcpyAsync(v.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, h.stream));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

}  // namespace

extern "C" {

// The step status of the calls whose copy has arrived: PPPM_ERR_NAN once a step kernel saw a
// non-finite Dirichlet value or listener sample.  wait: block until the last copy has arrived.
static int poll_step_status(Handle &h, bool wait)
{
    if (h.status_pending)
    {
        cudaError_t e = wait ? cudaEventSynchronize(h.ev_status) : cudaEventQuery(h.ev_status);
        if (e == cudaSuccess)
        {
            h.status_pending = false;
            if (*h.h_step_status & 1)
                h.nonfinite = true;
        }
        else if (e != cudaErrorNotReady)
            PB_CUDA(e);
    }
    if (h.nonfinite)
    {
        set_error("a non-finite Dirichlet value or listener sample appeared in an earlier step (reset the fields or "
                  "restore a saved state to go on)");
        return PPPM_ERR_NAN;
    }
    return PPPM_OK;
}

// queue a copy of the step status word behind the work on the handle's stream (not while the
// caller captures the stream: the copy would become part of the graph)
static int queue_step_status(Handle &h)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PB_CUDA(cudaStreamIsCapturing(h.stream, &cs));
    if (cs != cudaStreamCaptureStatusNone)
        return PPPM_OK;
    PB_CUDA(cudaMemcpyAsync(h.h_step_status, h.d_step_status, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
    PB_CUDA(cudaEventRecord(h.ev_status, h.stream));
    h.status_pending = true;
    return PPPM_OK;
}

// forget a non-finite flag: the fields it concerned are being replaced
static int clear_step_status(Handle &h)
{
    if (h.status_pending)
        PB_CUDA(cudaEventSynchronize(h.ev_status));
    h.status_pending = false;
    h.nonfinite = false;
    *h.h_step_status = 0;
    PB_CUDA(cudaMemsetAsync(h.d_step_status, 0, sizeof(int), h.stream));
    return PPPM_OK;
}

int pppm_params_default(pppm_params *p)
{
    if (!p)
        return PPPM_ERR_ARG;
    memset(p, 0, sizeof(*p));
    p->res = 32;
    p->dl = 0.005f;
    p->dt = 8e-6f;
    p->pml_width = 0;
    p->reflect_coeff = 0.83f;
    p->c = 340.3f;
    p->rho = 1.225f;
    p->precision = PPPM_PRECISION_FP32;
    p->weights = PPPM_WEIGHTS_REF32;
    p->device = 0;
    p->stream = nullptr;
    p->method = PPPM_METHOD_PPPM;
    p->ghost_threshold = 25.0f;
    return PPPM_OK;
}

int pppm_create(const pppm_params *p, pppm_handle **out)
{
    if (!p || !out)
        return PPPM_ERR_ARG;
    *out = nullptr;
    if (p->res < 8 || p->res > 1024 || !(p->dl > 0) || !(p->dt > 0) || !(p->c > 0) || p->pml_width < 0 ||
        p->pml_width * 2 >= p->res || (p->precision != PPPM_PRECISION_FP32 && p->precision != PPPM_PRECISION_FP64) ||
        (p->weights != PPPM_WEIGHTS_REF32 && p->weights != PPPM_WEIGHTS_FP64) ||
        (p->method != PPPM_METHOD_PPPM && p->method != PPPM_METHOD_GHOST) || !(p->ghost_threshold >= 0))
    {
        set_error("invalid parameters");
        return PPPM_ERR_ARG;
    }
    if (p->method == PPPM_METHOD_GHOST && (p->precision != PPPM_PRECISION_FP32 || p->pml_width > 0))
    {
        set_error("the ghost-cell method runs on FP32 handles with the absorbing boundary");
        return PPPM_ERR_ARG;
    }
    pppm_handle *ph = new (std::nothrow) pppm_handle();
    if (!ph)
        return PPPM_ERR_NOMEM;
    Handle &h = ph->h;
    h.prm = *p;
    h.fp64 = p->precision == PPPM_PRECISION_FP64;
    h.real_size = h.fp64 ? 8 : 4;
    h.res = p->res;
    h.n_cells = (long long)p->res * p->res * p->res;
    h.t = -1;
    auto fail = [&](int rc) {
        pppm_destroy(ph);
        return rc;
    };
    if (cudaSetDevice(p->device) != cudaSuccess)
    {
        set_error("cudaSetDevice(%d) failed", p->device);
        delete ph;
        return PPPM_ERR_CUDA;
    }
    if (p->stream)
        h.stream = (cudaStream_t)p->stream;
    else
    {
        if (cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking) != cudaSuccess)
        {
            set_error("cudaStreamCreate failed");
            delete ph;
            return PPPM_ERR_CUDA;
        }
        h.own_stream = true;
    }
    for (int i = 0; i < 3; i++)
    {
        int rc = dev_alloc(&h.grid[i], (size_t)h.n_cells * h.real_size);
        if (rc)
            return fail(rc);
        cudaMemsetAsync(h.grid[i], 0, (size_t)h.n_cells * h.real_size, h.stream);
        if (p->pml_width > 0)
        {
            rc = dev_alloc(&h.pml[i], (size_t)h.n_cells * 6 * h.real_size);
            if (rc)
                return fail(rc);
            cudaMemsetAsync(h.pml[i], 0, (size_t)h.n_cells * 6 * h.real_size, h.stream);
        }
    }
    {
        int rc = dalloc(&h.d_corr_mask, (size_t)(h.n_cells + 31) / 32);
        if (rc)
            return fail(rc);
        cudaMemsetAsync(h.d_corr_mask, 0, sizeof(unsigned) * ((h.n_cells + 31) / 32), h.stream);
    }
    for (int i = 0; i < 4; i++)
        cudaEventCreate(&h.ev[i]);
    for (auto &e : h.evk)
        cudaEventCreate(&e);
    {
        int rc = dalloc(&h.d_step_status, 1);
        if (rc)
            return fail(rc);
        cudaMemsetAsync(h.d_step_status, 0, sizeof(int), h.stream);
        if (cudaMallocHost((void **)&h.h_step_status, sizeof(int)) != cudaSuccess ||
            cudaEventCreateWithFlags(&h.ev_status, cudaEventDisableTiming) != cudaSuccess)
        {
            h.h_step_status = nullptr;
            set_error("cudaMallocHost / cudaEventCreate failed");
            return fail(PPPM_ERR_NOMEM);
        }
        *h.h_step_status = 0;
    }
    if (cudaStreamCreateWithFlags(&h.side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h.side2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h.ev_fin, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h.ev_conv, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h.ev_near, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h.ev_bulk, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h.ev_upd_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h.ev_upd_join, cudaEventDisableTiming) != cudaSuccess)
    {
        set_error("cudaStreamCreate / cudaEventCreate failed");
        return fail(PPPM_ERR_CUDA);
    }
    if (cudaMallocHost((void **)&h.h_pin, kPinnedInts * sizeof(int)) != cudaSuccess)
    {
        h.h_pin = nullptr;
        set_error("cudaMallocHost failed");
        return fail(PPPM_ERR_NOMEM);
    }
    tdbem_init(h.tc, p->dt, p->dl, p->c);
    if (cudaStreamSynchronize(h.stream) != cudaSuccess)
    {
        set_error("device initialisation failed");
        return fail(PPPM_ERR_CUDA);
    }
    *out = ph;
    return PPPM_OK;
}

int pppm_destroy(pppm_handle *ph)
{
    if (!ph)
        return PPPM_OK;
    Handle &h = ph->h;
    if (h.stream)
        cudaStreamSynchronize(h.stream);
    step_free(h);
    free_mesh(h);
    void *ptrs[] = {h.grid[0],        h.grid[1],         h.grid[2],        h.pml[0],          h.pml[1],
                    h.pml[2],         h.d_verts,         h.d_tris,         h.d_center,        h.d_normal,
                    h.d_area,         h.d_cellc,         h.d_basec,        h.d_cell,          h.d_base,
                    h.d_cell_count,   h.d_cell_start,    h.d_cell_tris,    h.d_base_count,    h.d_base_start,
                    h.d_base_tris,    h.d_cursor,        h.d_scan_tmp,     h.d_flags,         h.d_n3_cell,
                    h.d_n3_start,     h.d_p3_tri,        h.d_p3_woff,
                    h.d_corr_mask,    h.d_b4_cell,       h.d_b4_start,     h.d_n4_tris,       h.d_face_start,
                    h.d_face_nbr,     h.d_face_pool,     h.d_face_w,       h.d_face_scale,    h.d_face_corner,
                    h.d_pair_flag,    h.d_status,        h.d_neumann,      h.d_dirichlet,     h.d_listen_cell,
                    h.d_listen_n3,    h.d_series,        h.d_cell_type,    h.d_cell_nearest,  h.d_cell_ghost,
                    h.d_cell_points,  h.d_cell_type_old, h.d_acc,           h.d_pair_work};
    for (void *q : ptrs)
        dev_free(q);
    for (int i = 0; i < 4; i++)
        if (h.ev[i])
            cudaEventDestroy(h.ev[i]);
    for (auto &e : h.evk)
        if (e)
            cudaEventDestroy(e);
    dev_free(h.d_step_status);
    if (h.h_step_status)
        cudaFreeHost(h.h_step_status);
    if (h.ev_status)
        cudaEventDestroy(h.ev_status);
    if (h.h_pin)
        cudaFreeHost(h.h_pin);
    if (h.ev_fin)
        cudaEventDestroy(h.ev_fin);
    if (h.ev_conv)
        cudaEventDestroy(h.ev_conv);
    if (h.ev_near)
        cudaEventDestroy(h.ev_near);
    if (h.ev_bulk)
        cudaEventDestroy(h.ev_bulk);
    if (h.ev_upd_fork)
        cudaEventDestroy(h.ev_upd_fork);
    if (h.ev_upd_join)
        cudaEventDestroy(h.ev_upd_join);
    if (h.side)
        cudaStreamDestroy(h.side);
    if (h.side2)
        cudaStreamDestroy(h.side2);
    if (h.own_stream && h.stream)
        cudaStreamDestroy(h.stream);
    delete ph;
    return PPPM_OK;
}

int pppm_set_mesh(pppm_handle *ph, const float *verts, int nv, const int *tris, int nt)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (h.mesh_set)
    {
        set_error("set_mesh called twice; create a new handle for a new topology");
        return PPPM_ERR_STATE;
    }
    if (!verts || !tris || nv <= 0 || nt <= 0)
        return PPPM_ERR_ARG;
    for (long long i = 0; i < 3ll * nt; i++)
        if (tris[i] < 0 || tris[i] >= nv)
        {
            set_error("triangle index out of range");
            return PPPM_ERR_ARG;
        }
    for (long long i = 0; i < 3ll * nv; i++)
        if (!std::isfinite(verts[i]))
        {
            set_error("non-finite vertex");
            return PPPM_ERR_ARG;
        }
    cudaSetDevice(h.prm.device);
    free_mesh(h);
    h.nv = nv;
    h.nt = nt;
    PB_TRY(dalloc(&h.d_verts, 3 * (size_t)nv));
    PB_TRY(dalloc(&h.d_tris, 3 * (size_t)nt));
    PB_CUDA(cudaMemcpyAsync(h.d_verts, verts, sizeof(float) * 3 * nv, cudaMemcpyHostToDevice, h.stream));
    PB_CUDA(cudaMemcpyAsync(h.d_tris, tris, sizeof(int) * 3 * nt, cudaMemcpyHostToDevice, h.stream));
    PB_TRY(dev_alloc(&h.d_neumann, (size_t)nt * kRing * h.real_size));
    PB_TRY(dev_alloc(&h.d_dirichlet, (size_t)nt * kRing * h.real_size));
    PB_CUDA(cudaMemsetAsync(h.d_neumann, 0, (size_t)nt * kRing * h.real_size, h.stream));
    PB_CUDA(cudaMemsetAsync(h.d_dirichlet, 0, (size_t)nt * kRing * h.real_size, h.stream));
    PB_TRY(dev_alloc(&h.d_hist, (size_t)4 * nt * kHistRow * h.real_size));
    PB_TRY(dev_alloc(&h.d_terms, (size_t)54 * nt * h.real_size));
    PB_TRY(dev_alloc(&h.d_conv, (size_t)nt * h.real_size));
    PB_TRY(dev_alloc(&h.d_conv1, (size_t)nt * h.real_size));
    PB_TRY(dev_alloc(&h.d_dlast, (size_t)nt * h.real_size));
    PB_TRY(dev_alloc(&h.d_terms1, (size_t)54 * nt * h.real_size));
    PB_CUDA(cudaMemsetAsync(h.d_dlast, 0, (size_t)nt * h.real_size, h.stream));
    PB_CUDA(cudaMemsetAsync(h.d_hist, 0, (size_t)4 * nt * kHistRow * h.real_size, h.stream));
    int rc = mesh_build(h);
    if (rc != PPPM_OK)
        join_grid_cache(h);
    if (rc == PPPM_OK && h.prm.method == PPPM_METHOD_GHOST)
    {
        // GhostCellSolver::set_mesh (ghost_cell.h:84-99): labels, ghost system, zero accelerations
        rc = dalloc(&h.d_gneu, (size_t)nt);
        if (rc == PPPM_OK)
            rc = dalloc(&h.d_gneu_old, (size_t)nt);
        if (rc == PPPM_OK)
        {
            cudaMemsetAsync(h.d_gneu, 0, sizeof(float) * nt, h.stream);
            cudaMemsetAsync(h.d_gneu_old, 0, sizeof(float) * nt, h.stream);
            h.mesh_set = true;
            rc = cells_classify(h, nullptr);
            if (rc == PPPM_OK)
                rc = ghost_build(h);
        }
        if (rc != PPPM_OK)
        {
            h.mesh_set = false;
            free_mesh(h);
            return rc;
        }
        h.mesh_version++;
        PB_CUDA(cudaStreamSynchronize(h.stream));
        return PPPM_OK;
    }
    if (rc == PPPM_OK)
        rc = cache_refresh(h);
    if (rc != PPPM_OK)
    {
        free_mesh(h);
        return rc;
    }
    h.mesh_set = true;
    h.mesh_version++;
    PB_TRY(step_prime(h));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

int pppm_update_mesh(pppm_handle *ph, const float *verts, int verts_on_device)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (!h.mesh_set)
        return PPPM_ERR_STATE;
    if (!verts)
        return PPPM_ERR_ARG;
    cudaSetDevice(h.prm.device);
    PB_CUDA(cudaMemcpyAsync(h.d_verts, verts, sizeof(float) * 3 * h.nv,
                            verts_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h.stream));
    h.mesh_version++;
    h.tables_stale = false;
    {
        const int rc = mesh_build(h);
        if (rc != PPPM_OK)
        {
            join_grid_cache(h);
            return rc;
        }
    }
    if (h.prm.method == PPPM_METHOD_GHOST)
    {
        // GhostCellSolver::update_mesh (ghost_cell.h:101-117): new labels, fresh cells filled from
        // this and the previous step's accelerations, new ghost system
        PB_TRY(cells_classify(h, nullptr));
        PB_TRY(cells_fresh_dev(h, h.d_gneu, h.d_gneu_old, nullptr));
        PB_TRY(ghost_build(h));
        return PPPM_OK;
    }
    PB_TRY(cache_refresh(h));
    PB_TRY(step_prime(h));
    return PPPM_OK;
}

int pppm_step(pppm_handle *ph, const float *acc, int acc_on_device, int nsteps)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (nsteps < 0)
        return PPPM_ERR_ARG;
    if (nsteps == 0)
        return PPPM_OK;
    if (h.mesh_set && !acc)
    {
        set_error("accelerations required once a mesh is set");
        return PPPM_ERR_ARG;
    }
    cudaSetDevice(h.prm.device);
    if (h.tables_stale)
    {
        set_error("a cache state was restored: call pppm_update_mesh before stepping");
        return PPPM_ERR_STATE;
    }
    PB_TRY(poll_step_status(h, false));
    const float *dacc = nullptr;
    if (h.mesh_set)
    {
        if (acc_on_device)
            dacc = acc;
        else
        {
            long long need = (long long)nsteps * h.nt;
            if (need > h.acc_cap)
            {
                dev_free(h.d_acc);
                h.d_acc = nullptr;
                PB_TRY(dalloc(&h.d_acc, (size_t)need));
                h.acc_cap = need;
            }
            PB_CUDA(cudaMemcpyAsync(h.d_acc, acc, sizeof(float) * need, cudaMemcpyHostToDevice, h.stream));
            dacc = h.d_acc;
        }
    }
    PB_TRY(ensure_series(h, nsteps));
    PB_TRY(step_run(h, dacc, nsteps));
    return queue_step_status(h);
}

int pppm_sync(pppm_handle *ph)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    PB_CUDA(cudaStreamSynchronize(h.stream));
    PB_CUDA(cudaMemcpy(h.h_step_status, h.d_step_status, sizeof(int), cudaMemcpyDeviceToHost));
    h.status_pending = false;
    if (*h.h_step_status & 1)
        h.nonfinite = true;
    return poll_step_status(h, false);
}

struct pppm_batch
{
    std::vector<pppm_handle *> scenes;
    Batch *impl = nullptr;
};

int pppm_batch_create(pppm_handle **scenes, int nscenes, pppm_batch **out)
{
    if (!out)
        return PPPM_ERR_ARG;
    *out = nullptr;
    if (!scenes || nscenes <= 0)
        return PPPM_ERR_ARG;
    std::vector<Handle *> hs(nscenes);
    for (int i = 0; i < nscenes; i++)
    {
        PB_TRY(check_handle(scenes[i]));
        hs[i] = &scenes[i]->h;
    }
    pppm_batch *b = new (std::nothrow) pppm_batch();
    if (!b)
        return PPPM_ERR_NOMEM;
    b->scenes.assign(scenes, scenes + nscenes);
    int rc = batch_create(hs.data(), nscenes, &b->impl);
    if (rc)
    {
        delete b;
        return rc;
    }
    *out = b;
    return PPPM_OK;
}

int pppm_batch_destroy(pppm_batch *b)
{
    if (!b)
        return PPPM_OK;
    batch_destroy(b->impl);
    delete b;
    return PPPM_OK;
}

int pppm_batch_run(pppm_batch *b, const float *const *acc, const int *nsteps, int acc_on_device)
{
    if (!b || !b->impl || !acc || !nsteps)
        return PPPM_ERR_ARG;
    const int n = (int)b->scenes.size();
    std::vector<const float *> dacc(n, nullptr);
    for (int i = 0; i < n; i++)
    {
        Handle &h = b->scenes[i]->h;
        if (nsteps[i] < 0 || (nsteps[i] > 0 && !acc[i]))
            return PPPM_ERR_ARG;
        if (nsteps[i] == 0)
            continue;
        cudaSetDevice(h.prm.device);
        if (acc_on_device)
            dacc[i] = acc[i];
        else
        {
            long long need = (long long)nsteps[i] * h.nt;
            if (need > h.acc_cap)
            {
                dev_free(h.d_acc);
                h.d_acc = nullptr;
                PB_TRY(dalloc(&h.d_acc, (size_t)need));
                h.acc_cap = need;
            }
            PB_CUDA(cudaMemcpyAsync(h.d_acc, acc[i], sizeof(float) * need, cudaMemcpyHostToDevice, h.stream));
            dacc[i] = h.d_acc;
        }
        PB_TRY(ensure_series(h, nsteps[i]));
    }
    return batch_run(b->impl, dacc.data(), nsteps);
}

int pppm_adjoint(pppm_handle *ph, const void *dL_dsignal, int nsteps, int on_device, int fresh, void *dL_dacc)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (!h.mesh_set)
    {
        set_error("adjoint needs a mesh");
        return PPPM_ERR_STATE;
    }
    const int nl = (int)h.listen_xyz.size() / 3;
    for (int k = 0; k < 3 * nl; k++)
        if (h.listen_xyz[k] < 1 || h.listen_xyz[k] > h.res - 2)
        {
            set_error("adjoint: listener %d lies on the outer ghost layer", k / 3);
            return PPPM_ERR_ARG;
        }
    if (nsteps < 0 || (nsteps > 0 && ((!dL_dsignal && nl > 0) || !dL_dacc)))
        return PPPM_ERR_ARG;
    if (nsteps == 0)
        return PPPM_OK;
    if (h.tables_stale)
    {
        set_error("a cache state was restored: call pppm_update_mesh before the adjoint");
        return PPPM_ERR_STATE;
    }
    cudaSetDevice(h.prm.device);
    const size_t gb = (size_t)nsteps * nl * h.real_size, ob = (size_t)nsteps * h.nt * h.real_size;
    if (on_device)
        return adjoint_run(h, dL_dsignal, nsteps, dL_dacc, fresh);
    void *dg = nullptr, *dout = nullptr;
    PB_TRY(adjoint_stage(h, std::max<size_t>(gb, 16), ob, &dg, &dout));
    if (gb)
        PB_CUDA(cudaMemcpyAsync(dg, dL_dsignal, gb, cudaMemcpyHostToDevice, h.stream));
    PB_TRY(adjoint_run(h, dg, nsteps, dout, fresh));
    PB_CUDA(cudaMemcpyAsync(dL_dacc, dout, ob, cudaMemcpyDeviceToHost, h.stream));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

int pppm_add_listener(pppm_handle *ph, int x, int y, int z)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (x < 0 || y < 0 || z < 0 || x >= h.res || y >= h.res || z >= h.res)
        return PPPM_ERR_ARG;
    if (h.listen_xyz.size() / 3 >= 8)
    {
        set_error("at most 8 listeners");
        return PPPM_ERR_CAPACITY;
    }
    if (h.series_count > 0)
    {
        set_error("add listeners before the first step or after pppm_rewind_listeners");
        return PPPM_ERR_STATE;
    }
    h.listen_xyz.push_back(x);
    h.listen_xyz.push_back(y);
    h.listen_xyz.push_back(z);
    dev_free(h.d_series);
    h.d_series = nullptr;
    h.series_cap = 0;
    return PPPM_OK;
}

int pppm_clear_listeners(pppm_handle *ph)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    h.listen_xyz.clear();
    dev_free(h.d_series);
    h.d_series = nullptr;
    h.series_cap = 0;
    h.series_count = 0;
    return PPPM_OK;
}

int pppm_listener_count(pppm_handle *ph, int *nsteps, int *nlisteners)
{
    PB_TRY(check_handle(ph));
    if (nsteps)
        *nsteps = (int)ph->h.series_count;
    if (nlisteners)
        *nlisteners = (int)ph->h.listen_xyz.size() / 3;
    return PPPM_OK;
}

int pppm_read_listeners(pppm_handle *ph, int first, int count, float *out)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    int nl = (int)h.listen_xyz.size() / 3;
    if (!out || first < 0 || count < 0 || first + (long long)count > h.series_count)
        return PPPM_ERR_ARG;
    if (count == 0 || nl == 0)
        return PPPM_OK;
    size_t n = (size_t)count * nl;
    if (h.fp64)
    {
        std::vector<double> tmp(n);
        PB_CUDA(cudaMemcpyAsync(tmp.data(), (double *)h.d_series + (size_t)first * nl, n * sizeof(double),
                                cudaMemcpyDeviceToHost, h.stream));
        PB_CUDA(cudaStreamSynchronize(h.stream));
        for (size_t i = 0; i < n; i++)
            out[i] = (float)tmp[i];
    }
    else
    {
        PB_CUDA(cudaMemcpyAsync(out, (float *)h.d_series + (size_t)first * nl, n * sizeof(float),
                                cudaMemcpyDeviceToHost, h.stream));
        PB_CUDA(cudaStreamSynchronize(h.stream));
    }
    for (size_t i = 0; i < n; i++)
        if (!std::isfinite(out[i]))
        {
            set_error("non-finite listener sample at step %lld", (long long)first + (long long)(i / nl));
            return PPPM_ERR_NAN;
        }
    return PPPM_OK;
}

int pppm_read_listeners_raw(pppm_handle *ph, int first, int count, void *out, int on_device)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    const int nl = (int)h.listen_xyz.size() / 3;
    if (!out || first < 0 || count < 0 || first + (long long)count > h.series_count)
        return PPPM_ERR_ARG;
    if (count == 0 || nl == 0)
        return PPPM_OK;
    const size_t n = (size_t)count * nl * h.real_size;
    PB_CUDA(cudaMemcpyAsync(out, (const char *)h.d_series + (size_t)first * nl * h.real_size, n,
                            on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h.stream));
    if (!on_device)
        PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

int pppm_get_stream(pppm_handle *ph, void **stream)
{
    PB_TRY(check_handle(ph));
    if (!stream)
        return PPPM_ERR_ARG;
    *stream = (void *)ph->h.stream;
    return PPPM_OK;
}

int pppm_rewind_listeners(pppm_handle *ph)
{
    PB_TRY(check_handle(ph));
    ph->h.series_count = 0;
    return PPPM_OK;
}

int pppm_get_time(pppm_handle *ph, int *t)
{
    PB_TRY(check_handle(ph));
    if (!t)
        return PPPM_ERR_ARG;
    *t = ph->h.t;
    return PPPM_OK;
}

int pppm_set_time(pppm_handle *ph, int t)
{
    PB_TRY(check_handle(ph));
    if (t < -1)
        return PPPM_ERR_ARG;
    ph->h.t = t;
    return step_prime(ph->h);
}

int pppm_reset_fields(pppm_handle *ph)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    for (int i = 0; i < 3; i++)
    {
        PB_CUDA(cudaMemsetAsync(h.grid[i], 0, (size_t)h.n_cells * h.real_size, h.stream));
        if (h.pml[i])
            PB_CUDA(cudaMemsetAsync(h.pml[i], 0, (size_t)h.n_cells * 6 * h.real_size, h.stream));
    }
    if (h.mesh_set)
    {
        PB_CUDA(cudaMemsetAsync(h.d_neumann, 0, (size_t)h.nt * kRing * h.real_size, h.stream));
        PB_CUDA(cudaMemsetAsync(h.d_dirichlet, 0, (size_t)h.nt * kRing * h.real_size, h.stream));
        PB_CUDA(cudaMemsetAsync(h.d_hist, 0, (size_t)4 * h.nt * kHistRow * h.real_size, h.stream));
    }
    PB_TRY(step_prime(h));
    PB_TRY(clear_step_status(h));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

// state blob: int64 header[6] = {magic, t, res, nt, real_size, pml}, grids, pml, histories
static size_t state_bytes(const Handle &h)
{
    size_t g = (size_t)h.n_cells * h.real_size;
    size_t b = 6 * sizeof(long long) + 3 * g;
    if (h.prm.pml_width > 0)
        b += 3 * 6 * g;
    if (h.mesh_set)
        b += 2 * (size_t)h.nt * kRing * h.real_size;
    return b;
}

int pppm_state_size(pppm_handle *ph, size_t *bytes)
{
    PB_TRY(check_handle(ph));
    if (!bytes)
        return PPPM_ERR_ARG;
    *bytes = state_bytes(ph->h);
    return PPPM_OK;
}

int pppm_save_state(pppm_handle *ph, void *dst, size_t bytes)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (!dst || bytes < state_bytes(h))
        return PPPM_ERR_ARG;
    long long hdr[6] = {0x5050504d, h.t, h.res, h.mesh_set ? h.nt : 0, (long long)h.real_size, h.prm.pml_width};
    char *p = (char *)dst;
    memcpy(p, hdr, sizeof(hdr));
    p += sizeof(hdr);
    size_t g = (size_t)h.n_cells * h.real_size;
    for (int i = 0; i < 3; i++, p += g)
        PB_CUDA(cudaMemcpyAsync(p, h.slot(h.t - i), g, cudaMemcpyDeviceToHost, h.stream));
    if (h.prm.pml_width > 0)
        for (int i = 0; i < 3; i++, p += 6 * g)
            PB_CUDA(cudaMemcpyAsync(p, h.pml_slot(h.t - i), 6 * g, cudaMemcpyDeviceToHost, h.stream));
    if (h.mesh_set)
    {
        size_t hb = (size_t)h.nt * kRing * h.real_size;
        PB_CUDA(cudaMemcpyAsync(p, h.d_neumann, hb, cudaMemcpyDeviceToHost, h.stream));
        p += hb;
        PB_CUDA(cudaMemcpyAsync(p, h.d_dirichlet, hb, cudaMemcpyDeviceToHost, h.stream));
    }
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

int pppm_restore_state(pppm_handle *ph, const void *src, size_t bytes)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (!src || bytes < state_bytes(h))
        return PPPM_ERR_ARG;
    long long hdr[6];
    memcpy(hdr, src, sizeof(hdr));
    if (hdr[0] != 0x5050504d || hdr[2] != h.res || hdr[3] != (h.mesh_set ? h.nt : 0) ||
        hdr[4] != (long long)h.real_size || hdr[5] != h.prm.pml_width)
    {
        set_error("state blob does not match this handle");
        return PPPM_ERR_ARG;
    }
    h.t = (int)hdr[1];
    const char *p = (const char *)src + sizeof(hdr);
    size_t g = (size_t)h.n_cells * h.real_size;
    for (int i = 0; i < 3; i++, p += g)
        PB_CUDA(cudaMemcpyAsync(h.slot(h.t - i), p, g, cudaMemcpyHostToDevice, h.stream));
    if (h.prm.pml_width > 0)
        for (int i = 0; i < 3; i++, p += 6 * g)
            PB_CUDA(cudaMemcpyAsync(h.pml_slot(h.t - i), p, 6 * g, cudaMemcpyHostToDevice, h.stream));
    if (h.mesh_set)
    {
        size_t hb = (size_t)h.nt * kRing * h.real_size;
        PB_CUDA(cudaMemcpyAsync(h.d_neumann, p, hb, cudaMemcpyHostToDevice, h.stream));
        p += hb;
        PB_CUDA(cudaMemcpyAsync(h.d_dirichlet, p, hb, cudaMemcpyHostToDevice, h.stream));
        PB_TRY(hist_import(h));
    }
    PB_TRY(step_prime(h));
    PB_TRY(clear_step_status(h));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

int pppm_dump_size(pppm_handle *ph, int what, size_t *bytes)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (!bytes)
        return PPPM_ERR_ARG;
    size_t n = (size_t)h.n_cells;
    bool need_mesh = what >= PPPM_DUMP_NEUMANN && what <= PPPM_DUMP_INTERP;
    if (need_mesh && !h.mesh_set)
        return PPPM_ERR_STATE;
    bool need_cells = what >= PPPM_DUMP_CELL_TYPE && what <= PPPM_DUMP_CELL_POINTS;
    if (need_cells && !h.d_cell_type)
        return PPPM_ERR_STATE;
    switch (what)
    {
    case PPPM_DUMP_GRID_T:
    case PPPM_DUMP_GRID_TM1:
    case PPPM_DUMP_GRID_TM2: *bytes = n * h.real_size; break;
    case PPPM_DUMP_NEUMANN:
    case PPPM_DUMP_DIRICHLET: *bytes = (size_t)h.nt * kRing * h.real_size; break;
    case PPPM_DUMP_TRI_GEOM: *bytes = (size_t)h.nt * 7 * sizeof(float); break;
    case PPPM_DUMP_TRI_CELLS: *bytes = (size_t)h.nt * 6 * sizeof(int); break;
    case PPPM_DUMP_CELL_COUNTS: *bytes = n * sizeof(int); break;
    case PPPM_DUMP_N3_CELLS: *bytes = (size_t)h.n3 * 4 * sizeof(int); break;
    case PPPM_DUMP_N3_TRIS: *bytes = (size_t)h.p3 * sizeof(int); break;
    case PPPM_DUMP_B4_CELLS: *bytes = (size_t)h.b4 * 4 * sizeof(int); break;
    case PPPM_DUMP_B4_TRIS: *bytes = (size_t)h.nt * sizeof(int); break;
    case PPPM_DUMP_N4_TRIS: *bytes = (size_t)h.p4 * sizeof(int); break;
    case PPPM_DUMP_GRID_CACHE: *bytes = (size_t)h.nt * 54 * (h.fp64 ? 16 * sizeof(double2) : 72); break;
    case PPPM_DUMP_FACE_PAIRS: *bytes = (size_t)h.pf * 2 * sizeof(int); break;
    case PPPM_DUMP_FACE_CACHE: *bytes = (size_t)h.pf * (h.fp64 ? 16 * sizeof(double2) : 72); break;
    case PPPM_DUMP_INTERP: *bytes = (size_t)h.nt * 8 * sizeof(float); break;
    case PPPM_DUMP_CELL_TYPE:
    case PPPM_DUMP_CELL_NEAREST:
    case PPPM_DUMP_CELL_GHOST: *bytes = n * sizeof(int); break;
    case PPPM_DUMP_CELL_POINTS: *bytes = n * 7 * sizeof(float); break;
    case PPPM_DUMP_COUNTS: *bytes = 8 * sizeof(int); break;
    case PPPM_DUMP_GHOST_CELLS:
    case PPPM_DUMP_GHOST_ORDER: *bytes = h.ghost ? (size_t)h.ghost_count * sizeof(int) : 0; break;
    case PPPM_DUMP_GHOST_WEIGHTS: *bytes = h.ghost ? (size_t)h.ghost_count * 8 * sizeof(float) : 0; break;
    case PPPM_DUMP_GHOST_ITERS: *bytes = h.ghost ? sizeof(int) : 0; break;
    default: return PPPM_ERR_ARG;
    }
    return PPPM_OK;
}

int pppm_dump(pppm_handle *ph, int what, void *dst, size_t bytes)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    size_t need = 0;
    PB_TRY(pppm_dump_size(ph, what, &need));
    if (!dst || bytes < need)
        return PPPM_ERR_ARG;
    cudaStream_t s = h.stream;
    size_t n = (size_t)h.n_cells;
    auto copy = [&](const void *src, size_t b) -> int {
        if (b == 0)
            return PPPM_OK;
        PB_CUDA(cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        return PPPM_OK;
    };
    switch (what)
    {
    case PPPM_DUMP_GRID_T: return copy(h.slot(h.t), need);
    case PPPM_DUMP_GRID_TM1: return copy(h.slot(h.t - 1), need);
    case PPPM_DUMP_GRID_TM2: return copy(h.slot(h.t - 2), need);
    case PPPM_DUMP_NEUMANN: return copy(h.d_neumann, need);
    case PPPM_DUMP_DIRICHLET: return copy(h.d_dirichlet, need);
    case PPPM_DUMP_TRI_GEOM:
    {
        std::vector<float> c, nn, a;
        PB_TRY(d2h(h, c, h.d_center, 3 * (size_t)h.nt));
        PB_TRY(d2h(h, nn, h.d_normal, 3 * (size_t)h.nt));
        PB_TRY(d2h(h, a, h.d_area, (size_t)h.nt));
        float *o = (float *)dst;
        for (int i = 0; i < h.nt; i++)
        {
            for (int k = 0; k < 3; k++)
            {
                o[7 * i + k] = c[3 * i + k];
                o[7 * i + 3 + k] = nn[3 * i + k];
            }
            o[7 * i + 6] = a[i];
        }
        return PPPM_OK;
    }
    case PPPM_DUMP_TRI_CELLS:
    {
        std::vector<int> c, b;
        PB_TRY(d2h(h, c, h.d_cellc, 3 * (size_t)h.nt));
        PB_TRY(d2h(h, b, h.d_basec, 3 * (size_t)h.nt));
        int *o = (int *)dst;
        for (int i = 0; i < h.nt; i++)
            for (int k = 0; k < 3; k++)
            {
                o[6 * i + k] = c[3 * i + k];
                o[6 * i + 3 + k] = b[3 * i + k];
            }
        return PPPM_OK;
    }
    case PPPM_DUMP_CELL_COUNTS:
    {
        std::vector<int> st;
        int *o = (int *)dst;
        if (!h.mesh_set)
        {
            memset(o, 0, need);
            return PPPM_OK;
        }
        PB_TRY(d2h(h, st, h.d_cell_start, n + 1));
        for (size_t i = 0; i < n; i++)
            o[i] = st[i + 1] - st[i];
        return PPPM_OK;
    }
    case PPPM_DUMP_N3_CELLS:
    {
        std::vector<int> c, st;
        PB_TRY(d2h(h, c, h.d_n3_cell, (size_t)h.n3));
        PB_TRY(d2h(h, st, h.d_n3_start, (size_t)h.n3 + 1));
        int *o = (int *)dst;
        for (int i = 0; i < h.n3; i++)
        {
            o[4 * i] = c[i] / (h.res * h.res);
            o[4 * i + 1] = (c[i] / h.res) % h.res;
            o[4 * i + 2] = c[i] % h.res;
            o[4 * i + 3] = st[i + 1] - st[i];
        }
        return PPPM_OK;
    }
    case PPPM_DUMP_N3_TRIS: return copy(h.d_p3_tri, need);
    case PPPM_DUMP_B4_CELLS:
    {
        std::vector<int> c, bst;
        PB_TRY(d2h(h, c, h.d_b4_cell, (size_t)h.b4));
        PB_TRY(d2h(h, bst, h.d_base_start, n + 1));
        int *o = (int *)dst;
        for (int i = 0; i < h.b4; i++)
        {
            o[4 * i] = c[i] / (h.res * h.res);
            o[4 * i + 1] = (c[i] / h.res) % h.res;
            o[4 * i + 2] = c[i] % h.res;
            o[4 * i + 3] = bst[c[i] + 1] - bst[c[i]];
        }
        return PPPM_OK;
    }
    case PPPM_DUMP_B4_TRIS:
    {
        std::vector<int> c, bst, bl;
        PB_TRY(d2h(h, c, h.d_b4_cell, (size_t)h.b4));
        PB_TRY(d2h(h, bst, h.d_base_start, n + 1));
        PB_TRY(d2h(h, bl, h.d_base_tris, (size_t)h.nt));
        int *o = (int *)dst;
        size_t k = 0;
        for (int i = 0; i < h.b4; i++)
            for (int j = bst[c[i]]; j < bst[c[i] + 1]; j++)
                o[k++] = bl[j];
        for (; k < (size_t)h.nt; k++)
            o[k] = -1;
        return PPPM_OK;
    }
    case PPPM_DUMP_N4_TRIS: return copy(h.d_n4_tris, need);
    case PPPM_DUMP_GRID_CACHE:
    {
        size_t nrec = (size_t)h.nt * 54;
        if (h.fp64)
            return copy(h.d_gc_w, need);
        std::vector<__half2> w;
        std::vector<float2> sc;
        PB_TRY(d2h(h, w, h.d_gc_w, nrec * kTaps));
        PB_TRY(d2h(h, sc, h.d_gc_scale, nrec));
        to_ref_records(w.data(), sc.data(), nrec, (RefRecord *)dst);
        return PPPM_OK;
    }
    case PPPM_DUMP_FACE_PAIRS:
    {
        std::vector<int> st, nb;
        PB_TRY(d2h(h, st, h.d_face_start, (size_t)h.nt + 1));
        PB_TRY(d2h(h, nb, h.d_face_nbr, (size_t)h.pf));
        int *o = (int *)dst;
        for (int i = 0; i < h.nt; i++)
            for (int p = st[i]; p < st[i + 1]; p++)
            {
                o[2 * p] = i;
                o[2 * p + 1] = nb[p];
            }
        return PPPM_OK;
    }
    case PPPM_DUMP_FACE_CACHE:
    {
        if (h.fp64)
            return copy(h.d_face_w, need);
        std::vector<__half2> w;
        std::vector<float2> sc;
        PB_TRY(d2h(h, w, h.d_face_w, (size_t)h.pf * kTaps));
        PB_TRY(d2h(h, sc, h.d_face_scale, (size_t)h.pf));
        to_ref_records(w.data(), sc.data(), (size_t)h.pf, (RefRecord *)dst);
        return PPPM_OK;
    }
    case PPPM_DUMP_INTERP: return copy(h.d_face_interp, need);
    case PPPM_DUMP_CELL_TYPE: return copy(h.d_cell_type, need);
    case PPPM_DUMP_CELL_NEAREST: return copy(h.d_cell_nearest, need);
    case PPPM_DUMP_CELL_GHOST: return copy(h.d_cell_ghost, need);
    case PPPM_DUMP_CELL_POINTS: return copy(h.d_cell_points, need);
    case PPPM_DUMP_COUNTS:
    {
        int *o = (int *)dst;
        o[0] = h.n3;
        o[1] = (int)h.p3;
        o[2] = h.b4;
        o[3] = (int)h.p4;
        o[4] = (int)h.pf;
        o[5] = h.nt;
        o[6] = h.nv;
        o[7] = h.ghost_count;
        return PPPM_OK;
    }
    case PPPM_DUMP_GHOST_CELLS: return ghost_read(h, 0, dst, bytes);
    case PPPM_DUMP_GHOST_ORDER: return ghost_read(h, 1, dst, bytes);
    case PPPM_DUMP_GHOST_WEIGHTS: return ghost_read(h, 2, dst, bytes);
    case PPPM_DUMP_GHOST_ITERS: return ghost_read(h, 3, dst, bytes);
    default: return PPPM_ERR_ARG;
    }
}

int pppm_load(pppm_handle *ph, int what, const void *src, size_t bytes)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (!src)
        return PPPM_ERR_ARG;
    void *dst = nullptr;
    size_t need = 0;
    switch (what)
    {
    case PPPM_DUMP_GRID_T: dst = h.slot(h.t); need = (size_t)h.n_cells * h.real_size; break;
    case PPPM_DUMP_GRID_TM1: dst = h.slot(h.t - 1); need = (size_t)h.n_cells * h.real_size; break;
    case PPPM_DUMP_GRID_TM2: dst = h.slot(h.t - 2); need = (size_t)h.n_cells * h.real_size; break;
    case PPPM_DUMP_NEUMANN:
    case PPPM_DUMP_DIRICHLET:
        if (!h.mesh_set)
            return PPPM_ERR_STATE;
        dst = what == PPPM_DUMP_NEUMANN ? h.d_neumann : h.d_dirichlet;
        need = (size_t)h.nt * kRing * h.real_size;
        break;
    default: return PPPM_ERR_ARG;
    }
    if (bytes < need)
        return PPPM_ERR_ARG;
    const bool ring = what == PPPM_DUMP_NEUMANN || what == PPPM_DUMP_DIRICHLET;
    PB_CUDA(cudaMemcpyAsync(dst, src, need, cudaMemcpyHostToDevice, h.stream));
    if (ring)
        PB_TRY(hist_import(h));
    PB_TRY(step_prime(h));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

int pppm_import_grid_cache(pppm_handle *ph, const void *records, size_t bytes)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (!h.mesh_set || h.fp64)
        return PPPM_ERR_STATE;
    if (!records || bytes < (size_t)h.nt * 54 * 72)
        return PPPM_ERR_ARG;
    h.mesh_version++;
    PB_TRY(cache_import_grid(h, records));
    PB_TRY(step_prime(h));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

int pppm_import_face_cache(pppm_handle *ph, const int *face_pairs, const void *records, int npairs)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    if (!h.mesh_set || h.fp64)
        return PPPM_ERR_STATE;
    if (!face_pairs || !records || npairs < 0)
        return PPPM_ERR_ARG;
    h.mesh_version++;
    PB_TRY(cache_import_face(h, face_pairs, records, npairs));
    PB_TRY(step_prime(h));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    return PPPM_OK;
}

int pppm_classify_cells(pppm_handle *ph, int *ghost_count)
{
    PB_TRY(check_handle(ph));
    PB_TRY(cells_classify(ph->h, ghost_count));
    PB_CUDA(cudaStreamSynchronize(ph->h.stream));
    return PPPM_OK;
}

int pppm_fill_fresh_cells(pppm_handle *ph, const float *acc, const float *acc_old, int *fresh_count)
{
    PB_TRY(check_handle(ph));
    if (!acc || !acc_old)
        return PPPM_ERR_ARG;
    PB_TRY(cells_classify(ph->h, nullptr));
    PB_TRY(cells_fresh(ph->h, acc, acc_old, fresh_count));
    PB_CUDA(cudaStreamSynchronize(ph->h.stream));
    return PPPM_OK;
}

const char *pppm_status_string(int status)
{
    switch (status)
    {
    case PPPM_OK: return "ok";
    case PPPM_ERR_ARG: return "invalid argument";
    case PPPM_ERR_CUDA: return "CUDA error";
    case PPPM_ERR_CAPACITY: return "capacity exceeded";
    case PPPM_ERR_NAN: return "non-finite value";
    case PPPM_ERR_STATE: return "call out of order";
    case PPPM_ERR_TIMEOUT: return "device wait timed out";
    case PPPM_ERR_NOMEM: return "out of device memory";
    default: return "unknown status";
    }
}

const char *pppm_last_error_message(void) { return pb::last_error(); }

int pppm_launch_count(pppm_handle *ph, long long *count)
{
    PB_TRY(check_handle(ph));
    if (!count)
        return PPPM_ERR_ARG;
    *count = ph->h.launches;
    return PPPM_OK;
}

int pppm_set_option(pppm_handle *ph, int option, int value)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    switch (option)
    {
    case PPPM_OPT_CONV_PAIRS:
        if (value != 0 && value != 1)
            break;
        h.conv_pairs = value;
        return PPPM_OK;
    case PPPM_OPT_FACE_THREADS:
        if (value != 64 && value != 128 && value != 256)
            break;
        h.face_threads = value;
        return PPPM_OK;
    case PPPM_OPT_TERMS_PAIRS:
        if (value != 0 && value != 1)
            break;
        h.terms_pairs = value != 0;
        return PPPM_OK;
    case PPPM_OPT_SPLIT_STENCIL:
        if (value != 0 && value != 1)
            break;
        h.split_stencil = value != 0;
        return PPPM_OK;
    case PPPM_OPT_STENCIL_VEC4:
        if (value < -1 || value > 1)
            break;
        h.stencil_vec4 = value;
        return PPPM_OK;
    case PPPM_OPT_GRAPH_CHUNK:
        if (value != 0 && (value < 2 || value > 4096 || (value & 1)))
            break;
        h.graph_chunk = value;
        return PPPM_OK;
    default:
        set_error("unknown option %d", option);
        return PPPM_ERR_ARG;
    }
    set_error("option %d: value %d out of range", option, value);
    return PPPM_ERR_ARG;
}

int pppm_get_option(pppm_handle *ph, int option, int *value)
{
    PB_TRY(check_handle(ph));
    if (!value)
        return PPPM_ERR_ARG;
    Handle &h = ph->h;
    if (option == PPPM_OPT_CONV_PAIRS)
        *value = h.conv_pairs;
    else if (option == PPPM_OPT_FACE_THREADS)
        *value = h.face_threads;
    else if (option == PPPM_OPT_TERMS_PAIRS)
        *value = h.terms_pairs ? 1 : 0;
    else if (option == PPPM_OPT_SPLIT_STENCIL)
        *value = h.split_stencil ? 1 : 0;
    else if (option == PPPM_OPT_STENCIL_VEC4)
        *value = h.stencil_vec4;
    else if (option == PPPM_OPT_GRAPH_CHUNK)
        *value = h.graph_chunk;
    else
    {
        set_error("unknown option %d", option);
        return PPPM_ERR_ARG;
    }
    return PPPM_OK;
}

int pppm_autotune(pppm_handle *ph, int reps, float *us_out, int *best)
{
    PB_TRY(check_handle(ph));
    if (reps < 1 || reps > 10000)
    {
        set_error("autotune: reps must lie in [1, 10000]");
        return PPPM_ERR_ARG;
    }
    Handle &h = ph->h;
    cudaSetDevice(h.prm.device);
    float us[2 * PPPM_TUNE_CANDIDATES + PPPM_TUNE_CONFIGS] = {0};
    int b = 0;
    PB_TRY(ensure_series(h, 64));  // the timed step graphs write listener rows past the recorded ones
    PB_TRY(step_autotune(h, reps, us, &b));
    if (us_out)
        memcpy(us_out, us, sizeof(us));
    if (best)
        *best = b;
    return PPPM_OK;
}

int pppm_enable_timing(pppm_handle *ph, int enable)
{
    PB_TRY(check_handle(ph));
    ph->h.timing = enable != 0;
    ph->h.us_stencil = ph->h.us_face = ph->h.us_near = 0;
    ph->h.timed_steps = 0;
    for (int k = 0; k < PPPM_KERNEL_KINDS; k++)
    {
        ph->h.kind_us[k] = 0;
        ph->h.kind_n[k] = 0;
    }
    return PPPM_OK;
}

int pppm_time_kernels(pppm_handle *ph, int reps, int nkinds, float *us_per_launch)
{
    PB_TRY(check_handle(ph));
    if (nkinds < 0 || nkinds > PPPM_KERNEL_KINDS || (nkinds > 0 && !us_per_launch))
        return PPPM_ERR_ARG;
    Handle &h = ph->h;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PB_CUDA(cudaStreamIsCapturing(h.stream, &cs));
    if (cs != cudaStreamCaptureStatusNone)
        return PPPM_ERR_STATE;
    float us[PPPM_KERNEL_KINDS];
    PB_TRY(step_time_kernels(h, reps, us));
    PB_CUDA(cudaStreamSynchronize(h.stream));
    for (int k = 0; k < nkinds; k++)
        us_per_launch[k] = us[k];
    return PPPM_OK;
}

int pppm_cache_state_size(pppm_handle *ph, size_t *bytes)
{
    PB_TRY(check_handle(ph));
    if (!bytes)
        return PPPM_ERR_ARG;
    Handle &h = ph->h;
    if (!h.mesh_set || !h.d_gc_w || h.prm.method != PPPM_METHOD_PPPM)
        return PPPM_ERR_STATE;
    *bytes = cache_state_bytes(h);
    return PPPM_OK;
}

int pppm_save_cache_state(pppm_handle *ph, void *dst, size_t bytes)
{
    PB_TRY(check_handle(ph));
    if (!dst)
        return PPPM_ERR_ARG;
    cudaSetDevice(ph->h.prm.device);
    return cache_state_save(ph->h, dst, bytes);
}

int pppm_restore_cache_state(pppm_handle *ph, const void *src, size_t bytes)
{
    PB_TRY(check_handle(ph));
    if (!src)
        return PPPM_ERR_ARG;
    cudaSetDevice(ph->h.prm.device);
    return cache_state_restore(ph->h, src, bytes);
}

int pppm_checkpoint_push(pppm_handle *ph, int *id)
{
    PB_TRY(check_handle(ph));
    if (!id)
        return PPPM_ERR_ARG;
    cudaSetDevice(ph->h.prm.device);
    return journal_push(ph->h, id);
}

int pppm_checkpoint_rewind(pppm_handle *ph, int id)
{
    PB_TRY(check_handle(ph));
    cudaSetDevice(ph->h.prm.device);
    return journal_rewind(ph->h, id);
}

int pppm_checkpoint_clear(pppm_handle *ph, int release)
{
    PB_TRY(check_handle(ph));
    cudaSetDevice(ph->h.prm.device);
    journal_clear(ph->h, release != 0);
    return PPPM_OK;
}

int pppm_checkpoint_info(pppm_handle *ph, int *count, size_t *bytes)
{
    PB_TRY(check_handle(ph));
    if (count)
        *count = journal_count(ph->h);
    if (bytes)
        *bytes = journal_bytes(ph->h);
    return PPPM_OK;
}

int pppm_kernel_profile(pppm_handle *ph, int nkinds, float *us_per_launch, long long *launches)
{
    PB_TRY(check_handle(ph));
    if (nkinds < 0 || nkinds > PPPM_KERNEL_KINDS || (nkinds > 0 && (!us_per_launch || !launches)))
        return PPPM_ERR_ARG;
    const Handle &h = ph->h;
    for (int k = 0; k < nkinds; k++)
    {
        launches[k] = h.kind_n[k];
        us_per_launch[k] = h.kind_n[k] ? (float)(h.kind_us[k] / (double)h.kind_n[k]) : 0.0f;
    }
    return PPPM_OK;
}

int pppm_kernel_times(pppm_handle *ph, float *us_stencil, float *us_face, float *us_near, int *launches)
{
    PB_TRY(check_handle(ph));
    Handle &h = ph->h;
    double n = h.timed_steps > 0 ? (double)h.timed_steps : 1.0;
    if (us_stencil)
        *us_stencil = (float)(h.us_stencil / n);
    if (us_face)
        *us_face = (float)(h.us_face / n);
    if (us_near)
        *us_near = (float)(h.us_near / n);
    if (launches)
        *launches = (int)h.timed_steps;
    return PPPM_OK;
}

}  // extern "C"
