// Weight diagnostics of the C ABI: host TDBEM constants and single-pair weights on the device,
// used to pin the FP32 weight arithmetic against the reference's own values.
#include <mutex>
#include <vector>
#include "handle.cuh"

namespace
{
using namespace pb;

__global__ void pair_weight_kernel(TdbemConsts tc, const float *verts, int3 src, int to_point, int3 dst, f3 point,
                                   float *out)
{
    f3 sv[3] = {load3(verts, src.x), load3(verts, src.y), load3(verts, src.z)};
    int si[3] = {src.x, src.y, src.z};
    cf s[kTaps], d[kTaps];
    for (int k = 0; k <= kTaps / 2; k++)
    {
        cf kk{tc.wave_re[k], tc.wave_im[k]};
        if (to_point)
        {
            s[k] = ref32::face_to_points(sv, &point, nullptr, 1, false, kk, false);
            d[k] = ref32::face_to_points(sv, &point, nullptr, 1, false, kk, true);
        }
        else
        {
            f3 tv[3] = {load3(verts, dst.x), load3(verts, dst.y), load3(verts, dst.z)};
            int ti[3] = {dst.x, dst.y, dst.z};
            s[k] = ref32::face_to_face(sv, si, tv, ti, kk, tc.threshold, false);
            d[k] = ref32::face_to_face(sv, si, tv, ti, kk, tc.threshold, true);
        }
    }
    for (int k = kTaps / 2 + 1; k < kTaps; k++)
    {
        s[k] = cf{s[kTaps - k].re, -s[kTaps - k].im};
        d[k] = cf{d[kTaps - k].re, -d[kTaps - k].im};
    }
    ref32::scaled_fft(s, tc.lambda, out);
    ref32::scaled_fft(d, tc.lambda, out + kTaps);
}

// Makes `device` current for the scope of an entry point and gives the calling thread its
// previous current device back on every return path: these entry points may run on threads that
// drive other devices.
struct DeviceScope
{
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int device)
    {
        if (cudaGetDevice(&prev) != cudaSuccess)
            prev = -1;
        err = cudaSetDevice(device);
        if (err != cudaSuccess)
            cudaGetLastError();  // not left for the caller's next error check to find
    }
    ~DeviceScope()
    {
        if (prev >= 0)
            cudaSetDevice(prev);
    }
};
}  // namespace

extern "C" {

int pppm_tdbem_constants(float dt, float dl, float c, float *lambda, float *wave32)
{
    if (!lambda || !wave32 || !(dt > 0) || !(dl > 0) || !(c > 0))
        return PPPM_ERR_ARG;
    TdbemConsts tc;
    tdbem_init(tc, dt, dl, c);
    *lambda = tc.lambda;
    for (int k = 0; k < kTaps; k++)
    {
        wave32[2 * k] = tc.wave_re[k];
        wave32[2 * k + 1] = tc.wave_im[k];
    }
    return PPPM_OK;
}

int pppm_pair_weights(int device, float dt, float dl, float c, const float *verts, int nv, const int *src,
                      int to_point, const int *dst_face, const float *dst_point, float *out32)
{
    if (!verts || nv <= 0 || !src || !out32 || (to_point ? !dst_point : !dst_face))
        return PPPM_ERR_ARG;
    for (int k = 0; k < 3; k++)
        if (src[k] < 0 || src[k] >= nv || (!to_point && (dst_face[k] < 0 || dst_face[k] >= nv)))
            return PPPM_ERR_ARG;
    DeviceScope scope(device);
    PB_CUDA(scope.err);
    TdbemConsts tc;
    tdbem_init(tc, dt, dl, c);
    struct Buffers
    {
        float *dv = nullptr, *dout = nullptr;
        ~Buffers()
        {
            dev_free(dv);
            dev_free(dout);
        }
    } b;
    PB_TRY(dalloc(&b.dv, 3 * (size_t)nv));
    PB_TRY(dalloc(&b.dout, 2 * kTaps));
    PB_CUDA(cudaMemcpy(b.dv, verts, sizeof(float) * 3 * nv, cudaMemcpyHostToDevice));
    int3 s = make_int3(src[0], src[1], src[2]);
    int3 d = to_point ? make_int3(0, 0, 0) : make_int3(dst_face[0], dst_face[1], dst_face[2]);
    f3 p = to_point ? f3{dst_point[0], dst_point[1], dst_point[2]} : f3{0, 0, 0};
    pair_weight_kernel<<<1, 1>>>(tc, b.dv, s, to_point, d, p, b.dout);
    PB_CHECK_LAUNCH();
    PB_CUDA(cudaMemcpy(out32, b.dout, sizeof(float) * 2 * kTaps, cudaMemcpyDeviceToHost));
    return PPPM_OK;
}
}

// ---------------------------------------------------------------- no-allocation variant ---
// pppm_pair_weights_static: the same kernel on scratch that lives in this library's own device
// image instead of memory from cudaMalloc.  Callers that cannot allocate: a thread that runs
// beside a stepping handle on the same device (cudaMalloc / cudaFree may synchronise the whole
// device and stall that handle's stream for the length of its queued steps), and processes whose
// device memory is fully held by another allocator (a framework's caching pool), where a fresh
// cudaMalloc fails.  One scratch array per device and per process; calls that overlapped would
// race on it, so they are serialised by a process-wide lock.  The call leaves the calling
// thread's current device as it found it, refuses a stream that is being captured, and has
// finished with the scratch (its stream synchronised) on every return after the first copy was
// queued, so the next caller may overwrite it.

namespace
{
constexpr int kStaticMaxVerts = PPPM_STATIC_MAX_VERTS;

// vertex rows (3 floats each) followed by the 32 output taps
static __device__ __align__(256) float g_pair_scratch[3 * kStaticMaxVerts + 2 * kTaps];

constexpr int kMaxDevices = 64;
std::mutex g_static_lock;
float *g_scratch_ptr[kMaxDevices] = {};
}  // namespace

extern "C" {

int pppm_pair_weights_static(int device, void *stream, float dt, float dl, float c, const float *verts, int nv,
                             const int *src, int to_point, const int *dst_face, const float *dst_point, float *out32)
{
    if (!verts || nv <= 0 || !src || !out32 || (to_point ? !dst_point : !dst_face))
        return PPPM_ERR_ARG;
    if (nv > kStaticMaxVerts)
    {
        pb::set_error("pppm_pair_weights_static: %d vertices exceed the static scratch limit of %d "
                      "(PPPM_STATIC_MAX_VERTS); pass only the rows the pair uses or call pppm_pair_weights",
                      nv, kStaticMaxVerts);
        return PPPM_ERR_CAPACITY;
    }
    for (int k = 0; k < 3; k++)
        if (src[k] < 0 || src[k] >= nv || (!to_point && (dst_face[k] < 0 || dst_face[k] >= nv)))
            return PPPM_ERR_ARG;
    if (device < 0 || device >= kMaxDevices)
        return PPPM_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_static_lock);
    DeviceScope scope(device);
    PB_CUDA(scope.err);
    cudaStream_t s = (cudaStream_t)stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PB_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone)
    {
        pb::set_error("pppm_pair_weights_static: the stream is being captured; this call synchronises it");
        return PPPM_ERR_STATE;
    }
    if (!g_scratch_ptr[device])
    {
        // first call on this device: resolves the symbol (may load the module)
        float *p = nullptr;
        PB_CUDA(cudaGetSymbolAddress((void **)&p, g_pair_scratch));
        g_scratch_ptr[device] = p;
    }
    float *dv = g_scratch_ptr[device];
    float *dout = dv + 3 * kStaticMaxVerts;
    TdbemConsts tc;
    tdbem_init(tc, dt, dl, c);
    // from the first queued copy on, every return waits for the stream: the lock is released only
    // once this call's copies and kernel no longer touch the shared scratch
    struct Drain
    {
        cudaStream_t s;
        ~Drain() { cudaStreamSynchronize(s); }
    } drain{s};
    // nothing has to start at zero: the rows are copied in and the kernel writes all 32 taps
    PB_CUDA(cudaMemcpyAsync(dv, verts, sizeof(float) * 3 * nv, cudaMemcpyHostToDevice, s));
    int3 si = make_int3(src[0], src[1], src[2]);
    int3 di = to_point ? make_int3(0, 0, 0) : make_int3(dst_face[0], dst_face[1], dst_face[2]);
    f3 p = to_point ? f3{dst_point[0], dst_point[1], dst_point[2]} : f3{0, 0, 0};
    pair_weight_kernel<<<1, 1, 0, s>>>(tc, dv, si, to_point, di, p, dout);
    PB_CHECK_LAUNCH();
    PB_CUDA(cudaMemcpyAsync(out32, dout, sizeof(float) * 2 * kTaps, cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    return PPPM_OK;
}
}
