// Weight diagnostics of the C ABI: host TDBEM constants and single-pair weights on the device,
// used to pin the FP32 weight arithmetic against the reference's own values.
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
    PB_CUDA(cudaSetDevice(device));
    TdbemConsts tc;
    tdbem_init(tc, dt, dl, c);
    float *dv = nullptr, *dout = nullptr;
    PB_TRY(dalloc(&dv, 3 * (size_t)nv));
    PB_TRY(dalloc(&dout, 2 * kTaps));
    PB_CUDA(cudaMemcpy(dv, verts, sizeof(float) * 3 * nv, cudaMemcpyHostToDevice));
    int3 s = make_int3(src[0], src[1], src[2]);
    int3 d = to_point ? make_int3(0, 0, 0) : make_int3(dst_face[0], dst_face[1], dst_face[2]);
    f3 p = to_point ? f3{dst_point[0], dst_point[1], dst_point[2]} : f3{0, 0, 0};
    pair_weight_kernel<<<1, 1>>>(tc, dv, s, to_point, d, p, dout);
    PB_CHECK_LAUNCH();
    PB_CUDA(cudaMemcpy(out32, dout, sizeof(float) * 2 * kTaps, cudaMemcpyDeviceToHost));
    dev_free(dv);
    dev_free(dout);
    return PPPM_OK;
}
}
