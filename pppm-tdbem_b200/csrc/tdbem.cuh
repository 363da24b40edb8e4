// TDBEM weight evaluation: Laplace-domain boundary integrals on the BDF2 contour, a
// 16-point inverse FFT and the lambda^-n scaling that turn them into 16-tap time-domain
// convolution weights for the single and double layer.
//
// Algorithm (restated from the reference):
//   wave numbers      bem.h:264-277      s_k = lambda e^{-2 pi i k/16}, k_n = i BDF2(s_k)/(c dt)
//   point integral    integrand.h:193-220,254-267 (1-point triangle Gauss rule)
//   face integrals    integrand.h:175-191 (regular), 51-173 (identical / common-edge /
//                     common-vertex panels: the Duffy-type 4D rules of Sauter & Schwab,
//                     3-point Gauss-Legendre per dimension), 228-252 (dispatch)
//   kernels           potential.h:290-357 (e^{ikr}/(4 pi r) and its normal derivative)
//   FFT               bem.h:12-38 (recursive radix-2, positive exponent), 292-304 (scaling)
//   fp16 packing      bem.h:171-191 (max-abs scale per row, round-to-nearest-even)
//
// Two arithmetic flavours:
//   ref32  FP32 values with exactly the float/double promotions the reference's
//          thrust::complex<float> expressions produce (a double literal such as PI or 0.5
//          promotes a product to double; a complex<float> accumulator receives the double sum
//          rounded back to float).  Built with --use_fast_math like the reference, so expf,
//          sinf, cosf, sqrtf and float division compile to the same approximate instructions.
//          The aim is bit-identical fp16 weight tables.
//   f64    the same formulas entirely in double; used for the FP64 yardstick run and for the
//          singular panel integrals when PPPM_WEIGHTS_FP64 is selected.
#pragma once
#include "common.cuh"

namespace pb
{

// LINE_GAUSS_NUM = 3 Gauss-Legendre rule on [-1, 1] and the TRI_GAUSS_NUM = 1 triangle rule
// (centroid), the values the reference tables hold (helmholtz/gauss/line.h, triangle.h).
#define PB_LINE_X0 0.774596669241483
#define PB_LINE_W0 0.555555555555554
#define PB_LINE_W1 0.888888888888889
#define PB_TRI_X 0.3333333333333330
#define PB_PI 3.14159265359

struct cf
{
    float re, im;
};
struct cd
{
    double re, im;
};

// Host-side TDBEM constants (bem.h:264-277): lambda and the 16 complex wave numbers.
struct TdbemConsts
{
    float lambda;
    float wave_re[kTaps];
    float wave_im[kTaps];
    float threshold;  // face-to-face near-coincidence threshold, 0.1 * grid size
    double lambda_d;
    double wave_re_d[kTaps];
    double wave_im_d[kTaps];
};

void tdbem_init(TdbemConsts &out, float dt, float grid_size, float c);

// ----------------------------------------------------------------------- ref32 -------
namespace ref32
{

// thrust's cexpf for finite arguments (exp(x) (cos y, sin y), with the y == 0 and x == 0
// shortcuts tested on the bit patterns).
__device__ inline cf cexp(float x, float y)
{
    if ((__float_as_uint(y) & 0x7fffffffu) == 0)
        return cf{expf(x), y};
    if ((__float_as_uint(x) & 0x7fffffffu) == 0)
        return cf{cosf(y), sinf(y)};
    float e = expf(x);
    return cf{e * cosf(y), e * sinf(y)};
}

// i * r * k for complex k: (0*r, r) * k
__device__ inline cf ikr_of(float r, cf k)
{
    float a_re = 0.0f * r, a_im = r;
    return cf{a_re * k.re - a_im * k.im, a_re * k.im + a_im * k.re};
}

// single layer G = e^{ikr} / (4 pi r), target minus source
__device__ inline void single_acc(cf &acc, f3 src, f3 trg, cf k, float scale, bool scaled)
{
    f3 d = trg - src;
    float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
    if (r2 != 0)
    {
        float r = sqrtf(r2);
        cf e = cexp(ikr_of(r, k).re, ikr_of(r, k).im);
        double den = 4 * PB_PI * r;
        double qre = e.re / den, qim = e.im / den;
        if (scaled)
        {
            qre = qre * scale;
            qim = qim * scale;
        }
        acc.re = (float)(acc.re + qre);
        acc.im = (float)(acc.im + qim);
    }
}

// double layer dG/dn_src = -e^{ikr} (1 - ikr) (s - t).n / (4 pi r^3), source minus target
__device__ inline void double_acc(cf &acc, f3 src, f3 trg, f3 n, cf k, float scale, bool scaled)
{
    f3 d = src - trg;
    float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
    if (r2 != 0)
    {
        float r = sqrtf(r2);
        cf ikr = ikr_of(r, k);
        cf e = cexp(ikr.re, ikr.im);
        double den = 4 * PB_PI * r2 * r;
        double are = -e.re / den, aim = -e.im / den;
        float bre = 1.0f - ikr.re, bim = -ikr.im;
        double mre = are * bre - aim * bim;
        double mim = are * bim + aim * bre;
        float dn = dot3(d, n);
        mre = mre * dn;
        mim = mim * dn;
        if (scaled)
        {
            mre = mre * scale;
            mim = mim * scale;
        }
        acc.re = (float)(acc.re + mre);
        acc.im = (float)(acc.im + mim);
    }
}

// Both layers of one source/target pair with one exponential: r^2 of (t - s) and (s - t) are
// bitwise equal, so e^{ikr} is shared; each layer's own arithmetic is unchanged.
__device__ inline void both_acc(cf &as, cf &ad, f3 src, f3 trg, f3 n, cf k, float scale, bool scaled)
{
    f3 d = src - trg;
    float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
    if (r2 != 0)
    {
        float r = sqrtf(r2);
        cf ikr = ikr_of(r, k);
        cf e = cexp(ikr.re, ikr.im);
        double den1 = 4 * PB_PI * r;
        double qre = e.re / den1, qim = e.im / den1;
        double den = 4 * PB_PI * r2 * r;
        double are = -e.re / den, aim = -e.im / den;
        float bre = 1.0f - ikr.re, bim = -ikr.im;
        double mre = are * bre - aim * bim;
        double mim = are * bim + aim * bre;
        float dn = dot3(d, n);
        mre = mre * dn;
        mim = mim * dn;
        if (scaled)
        {
            qre = qre * scale;
            qim = qim * scale;
            mre = mre * scale;
            mim = mim * scale;
        }
        as.re = (float)(as.re + qre);
        as.im = (float)(as.im + qim);
        ad.re = (float)(ad.re + mre);
        ad.im = (float)(ad.im + mim);
    }
}

// both_acc split in two: the unrounded double-precision terms of one point (valid = r != 0),
// and their scaled accumulation.  point_terms + acc_terms perform exactly the operations of
// both_acc, so a point's terms can be computed once and accumulated into several sums.
struct PointTerms
{
    double qre, qim, mre, mim;
    int valid;
};

// a / b in double, rounded to nearest, from y = RN(1 / b): q = RN(a y), then one correction with
// the exact remainder a - b q (P. Markstein, IBM J. Res. Dev. 34(1), 1990), which gives the correctly
// rounded quotient for the normal operands met here; a zero numerator keeps its sign, as in the
// division.  Two quotients by the same b then cost one division instead of two.
__device__ inline double div_by(double a, double b, double y)
{
    const double q = __dmul_rn(a, y);
    const double r = __fma_rn(-b, q, a);
    return a == 0.0 ? a : __fma_rn(r, y, q);
}

__device__ inline PointTerms point_terms(f3 src, f3 trg, f3 n, cf k)
{
    PointTerms t{0, 0, 0, 0, 0};
    f3 d = src - trg;
    float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
    if (r2 != 0)
    {
        float r = sqrtf(r2);
        cf ikr = ikr_of(r, k);
        cf e = cexp(ikr.re, ikr.im);
        double den1 = 4 * PB_PI * r;
        const double y1 = 1.0 / den1;
        t.qre = div_by(e.re, den1, y1);
        t.qim = div_by(e.im, den1, y1);
        double den = 4 * PB_PI * r2 * r;
        const double y = 1.0 / den;
        double are = div_by(-e.re, den, y), aim = div_by(-e.im, den, y);
        float bre = 1.0f - ikr.re, bim = -ikr.im;
        double mre = are * bre - aim * bim;
        double mim = are * bim + aim * bre;
        float dn = dot3(d, n);
        t.mre = mre * dn;
        t.mim = mim * dn;
        t.valid = 1;
    }
    return t;
}

__device__ inline void acc_terms(cf &as, cf &ad, const PointTerms &t, float scale, bool scaled)
{
    if (!t.valid)
        return;
    double qre = t.qre, qim = t.qim, mre = t.mre, mim = t.mim;
    if (scaled)
    {
        qre = qre * scale;
        qim = qim * scale;
        mre = mre * scale;
        mim = mim * scale;
    }
    as.re = (float)(as.re + qre);
    as.im = (float)(as.im + qim);
    ad.re = (float)(ad.re + mre);
    ad.im = (float)(ad.im + mim);
}

__device__ inline cf layer_point(f3 src, f3 trg, f3 n, cf k, bool dbl)
{
    cf acc{0.0f, 0.0f};
    if (dbl)
        double_acc(acc, src, trg, n, k, 1.0f, false);
    else
        single_acc(acc, src, trg, k, 1.0f, false);
    return acc;
}

__device__ inline float jacobian(const f3 *v) { return len3(cross3(v[1] - v[0], v[2] - v[0])); }

__device__ inline f3 tri_normal(const f3 *v)
{
    f3 n = cross3(v[1] - v[0], v[2] - v[0]);
    return n / len3(n);
}

// unit triangle (0,0),(1,0),(0,1)
__device__ inline f3 local_to_global(float x1, float x2, const f3 *v)
{
    float s = 1 - x1 - x2;
    return f3{s * v[0].x + x1 * v[1].x + x2 * v[2].x, s * v[0].y + x1 * v[1].y + x2 * v[2].y,
              s * v[0].z + x1 * v[1].z + x2 * v[2].z};
}

// unit triangle (0,0),(1,0),(1,1)
__device__ inline f3 local_to_global2(float x1, float x2, const f3 *v)
{
    float a = 1 - x1, b = x1 - x2;
    return f3{a * v[0].x + b * v[1].x + x2 * v[2].x, a * v[0].y + b * v[1].y + x2 * v[2].y,
              a * v[0].z + b * v[1].z + x2 * v[2].z};
}

// Face-to-point integral over src with targets pts[0..n) weighted by scales (the reference
// accumulates the target sum in complex<float> first, then applies 0.5 * w * J in double).
__device__ inline cf face_to_points(const f3 *src_v, const f3 *pts, const float *scales, int n, bool scaled, cf k,
                                    bool dbl)
{
    float jac = jacobian(src_v);
    f3 nrm = tri_normal(src_v);
    const float gx = (float)PB_TRI_X;
    f3 q = local_to_global(gx, gx, src_v);
    cf lp{0.0f, 0.0f};
    for (int i = 0; i < n; i++)
    {
        if (dbl)
            double_acc(lp, q, pts[i], nrm, k, scaled ? scales[i] : 1.0f, scaled);
        else
            single_acc(lp, q, pts[i], k, scaled ? scales[i] : 1.0f, scaled);
    }
    double c = 0.5 * 1.0f * jac;
    cf out{0.0f, 0.0f};
    out.re = (float)(out.re + c * lp.re);
    out.im = (float)(out.im + c * lp.im);
    return out;
}

__device__ inline cf regular_face(const f3 *trial, const f3 *test, float trial_jac, float test_jac, cf k, bool dbl)
{
    f3 nrm = tri_normal(trial);
    const float gx = (float)PB_TRI_X;
    f3 a = local_to_global(gx, gx, trial);
    f3 b = local_to_global(gx, gx, test);
    double c = 0.25 * 1.0f * 1.0f * trial_jac * test_jac;
    cf lp = layer_point(a, b, nrm, k, dbl);
    cf out{0.0f, 0.0f};
    out.re = (float)(out.re + c * lp.re);
    out.im = (float)(out.im + c * lp.im);
    return out;
}

__device__ inline void add_lp(cf &acc, f3 a, f3 b, f3 n, cf k, bool dbl)
{
    cf lp = layer_point(a, b, n, k, dbl);
    acc.re += lp.re;
    acc.im += lp.im;
}

__device__ inline void add_lp_scaled(cf &acc, f3 a, f3 b, f3 n, cf k, bool dbl, float s)
{
    cf lp = layer_point(a, b, n, k, dbl);
    acc.re += lp.re * s;
    acc.im += lp.im * s;
}

// One 4D quadrature node of the singular rules (integrand.h:51-149).  Arguments computed
// as "xsi * (1.0 - ...)" are evaluated in double and rounded to float like the reference.
__device__ inline cf singular_node(float xsi, float e1, float e2, float e3, float weight, const f3 *tv, const f3 *sv,
                                   f3 n, int nn, cf k, bool dbl)
{
    cf r{0.0f, 0.0f};
    xsi = 0.5 * (xsi + 1);
    e1 = 0.5 * (e1 + 1);
    e2 = 0.5 * (e2 + 1);
    e3 = 0.5 * (e3 + 1);
    if (nn == 3)
    {
        float w = xsi * xsi * xsi * e1 * e1 * e2;
        float e12 = e1 * e2;
        float e123 = e1 * e2 * e3;
        add_lp(r, local_to_global2(xsi, xsi * (1.0 - e1 + e12), tv),
               local_to_global2(xsi * (1.0 - e123), xsi * (1.0 - e1), sv), n, k, dbl);
        add_lp(r, local_to_global2(xsi * (1.0 - e123), xsi * (1.0 - e1), tv),
               local_to_global2(xsi, xsi * (1.0 - e1 + e12), sv), n, k, dbl);
        add_lp(r, local_to_global2(xsi, xsi * (e1 - e12 + e123), tv),
               local_to_global2(xsi * (1.0 - e12), xsi * (e1 - e12), sv), n, k, dbl);
        add_lp(r, local_to_global2(xsi * (1.0 - e12), xsi * (e1 - e12), tv),
               local_to_global2(xsi, xsi * (e1 - e12 + e123), sv), n, k, dbl);
        add_lp(r, local_to_global2(xsi * (1.0 - e123), xsi * (e1 - e123), tv),
               local_to_global2(xsi, xsi * (e1 - e12), sv), n, k, dbl);
        add_lp(r, local_to_global2(xsi, xsi * (e1 - e12), tv),
               local_to_global2(xsi * (1.0 - e123), xsi * (e1 - e123), sv), n, k, dbl);
        r.re = r.re * w;
        r.im = r.im * w;
        r.re = r.re * weight;
        r.im = r.im * weight;
    }
    else if (nn == 2)
    {
        float w = xsi * xsi * xsi * e1 * e1;
        float e12 = e1 * e2;
        float e123 = e1 * e2 * e3;
        add_lp(r, local_to_global2(xsi, xsi * e1 * e3, tv), local_to_global2(xsi * (1.0 - e12), xsi * e1 * (1.0 - e2), sv),
               n, k, dbl);
        add_lp_scaled(r, local_to_global2(xsi, xsi * e1, tv),
                      local_to_global2(xsi * (1.0 - e123), xsi * e1 * e2 * (1 - e3), sv), n, k, dbl, e2);
        add_lp_scaled(r, local_to_global2(xsi * (1.0 - e12), xsi * e1 * (1.0 - e2), tv),
                      local_to_global2(xsi, xsi * e123, sv), n, k, dbl, e2);
        add_lp_scaled(r, local_to_global2(xsi * (1.0 - e123), xsi * e12 * (1.0 - e3), tv),
                      local_to_global2(xsi, xsi * e1, sv), n, k, dbl, e2);
        add_lp_scaled(r, local_to_global2(xsi * (1.0 - e123), xsi * e1 * (1.0 - e2 * e3), tv),
                      local_to_global2(xsi, xsi * e12, sv), n, k, dbl, e2);
        r.re = r.re * w;
        r.im = r.im * w;
        r.re = r.re * weight;
        r.im = r.im * weight;
    }
    else if (nn == 1)
    {
        float w = xsi * xsi * xsi * e2;
        add_lp(r, local_to_global2(xsi, xsi * e1, tv), local_to_global2(xsi * e2, xsi * e2 * e3, sv), n, k, dbl);
        add_lp(r, local_to_global2(xsi * e2, xsi * e2 * e3, tv), local_to_global2(xsi, xsi * e1, sv), n, k, dbl);
        r.re = r.re * w;
        r.im = r.im * w;
        r.re = r.re * weight;
        r.im = r.im * weight;
    }
    return r;
}

__device__ inline cf singular_face(const f3 *trial, const f3 *test, float trial_jac, float test_jac, cf k, int nn,
                                   bool dbl)
{
    const float gx[3] = {(float)PB_LINE_X0, 0.0f, (float)-PB_LINE_X0};
    const float gw[3] = {(float)PB_LINE_W0, (float)PB_LINE_W1, (float)PB_LINE_W0};
    f3 n = tri_normal(trial);
    cf acc{0.0f, 0.0f};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++)
                for (int d = 0; d < 3; d++)
                {
                    cf r = singular_node(gx[a], gx[b], gx[c], gx[d], gw[a] * gw[b] * gw[c] * gw[d], trial, test, n, nn,
                                         k, dbl);
                    acc.re += r.re;
                    acc.im += r.im;
                }
    acc.re = acc.re * trial_jac;
    acc.im = acc.im * trial_jac;
    acc.re = acc.re * test_jac;
    acc.im = acc.im * test_jac;
    acc.re = acc.re / 16;
    acc.im = acc.im / 16;
    return acc;
}

__device__ inline int common_vertices(const int *a, const int *b)
{
    int n = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            n += (a[i] == b[j]);
    return n;
}

// Face-to-face integral, src (trial) onto trg (test) (integrand.h:228-252).  The
// near-coincident branch evaluates the singular rule with zero shared vertices, which the
// rule defines as zero; the reference therefore returns 0 there and so does this.
__device__ inline cf face_to_face(const f3 *src, const int *si, const f3 *trg, const int *ti, cf k, float threshold,
                                  bool dbl)
{
    float sj = jacobian(src), tj = jacobian(trg);
    int nn = common_vertices(si, ti);
    f3 sc = (src[0] + src[1] + src[2]) / 3;
    f3 tc = (trg[0] + trg[1] + trg[2]) / 3;
    float dist = len3(sc - tc);
    if (dist < threshold && nn == 0)
        return cf{0.0f, 0.0f};
    if (nn == 0)
        return regular_face(src, trg, sj, tj, k, dbl);
    return singular_face(src, trg, sj, tj, k, nn, dbl);
}

// ---- two-layer variants: single and double layer of the same integral in one pass (each
// layer's arithmetic identical to the one-layer functions above)
__device__ inline void face_to_points2(const f3 *src_v, const f3 *pts, const float *scales, int n, bool scaled, cf k,
                                       cf &out_s, cf &out_d)
{
    float jac = jacobian(src_v);
    f3 nrm = tri_normal(src_v);
    const float gx = (float)PB_TRI_X;
    f3 q = local_to_global(gx, gx, src_v);
    cf ls{0.0f, 0.0f}, ld{0.0f, 0.0f};
    for (int i = 0; i < n; i++)
        both_acc(ls, ld, q, pts[i], nrm, k, scaled ? scales[i] : 1.0f, scaled);
    double c = 0.5 * 1.0f * jac;
    out_s = cf{(float)(0.0f + c * ls.re), (float)(0.0f + c * ls.im)};
    out_d = cf{(float)(0.0f + c * ld.re), (float)(0.0f + c * ld.im)};
}

__device__ inline void add_both(cf &rs, cf &rd, f3 a, f3 b, f3 n, cf k, bool scaled, float s)
{
    cf ls{0.0f, 0.0f}, ld{0.0f, 0.0f};
    both_acc(ls, ld, a, b, n, k, 1.0f, false);
    if (scaled)
    {
        rs.re += ls.re * s;
        rs.im += ls.im * s;
        rd.re += ld.re * s;
        rd.im += ld.im * s;
    }
    else
    {
        rs.re += ls.re;
        rs.im += ls.im;
        rd.re += ld.re;
        rd.im += ld.im;
    }
}

__device__ inline void singular_node2(float xsi, float e1, float e2, float e3, float weight, const f3 *tv,
                                      const f3 *sv, f3 n, int nn, cf k, cf &os, cf &od)
{
    cf rs{0.0f, 0.0f}, rd{0.0f, 0.0f};
    xsi = 0.5 * (xsi + 1);
    e1 = 0.5 * (e1 + 1);
    e2 = 0.5 * (e2 + 1);
    e3 = 0.5 * (e3 + 1);
    float w = 0;
    if (nn == 3)
    {
        w = xsi * xsi * xsi * e1 * e1 * e2;
        float e12 = e1 * e2;
        float e123 = e1 * e2 * e3;
        add_both(rs, rd, local_to_global2(xsi, xsi * (1.0 - e1 + e12), tv),
                 local_to_global2(xsi * (1.0 - e123), xsi * (1.0 - e1), sv), n, k, false, 0);
        add_both(rs, rd, local_to_global2(xsi * (1.0 - e123), xsi * (1.0 - e1), tv),
                 local_to_global2(xsi, xsi * (1.0 - e1 + e12), sv), n, k, false, 0);
        add_both(rs, rd, local_to_global2(xsi, xsi * (e1 - e12 + e123), tv),
                 local_to_global2(xsi * (1.0 - e12), xsi * (e1 - e12), sv), n, k, false, 0);
        add_both(rs, rd, local_to_global2(xsi * (1.0 - e12), xsi * (e1 - e12), tv),
                 local_to_global2(xsi, xsi * (e1 - e12 + e123), sv), n, k, false, 0);
        add_both(rs, rd, local_to_global2(xsi * (1.0 - e123), xsi * (e1 - e123), tv),
                 local_to_global2(xsi, xsi * (e1 - e12), sv), n, k, false, 0);
        add_both(rs, rd, local_to_global2(xsi, xsi * (e1 - e12), tv),
                 local_to_global2(xsi * (1.0 - e123), xsi * (e1 - e123), sv), n, k, false, 0);
    }
    else if (nn == 2)
    {
        w = xsi * xsi * xsi * e1 * e1;
        float e12 = e1 * e2;
        float e123 = e1 * e2 * e3;
        add_both(rs, rd, local_to_global2(xsi, xsi * e1 * e3, tv),
                 local_to_global2(xsi * (1.0 - e12), xsi * e1 * (1.0 - e2), sv), n, k, false, 0);
        add_both(rs, rd, local_to_global2(xsi, xsi * e1, tv),
                 local_to_global2(xsi * (1.0 - e123), xsi * e1 * e2 * (1 - e3), sv), n, k, true, e2);
        add_both(rs, rd, local_to_global2(xsi * (1.0 - e12), xsi * e1 * (1.0 - e2), tv),
                 local_to_global2(xsi, xsi * e123, sv), n, k, true, e2);
        add_both(rs, rd, local_to_global2(xsi * (1.0 - e123), xsi * e12 * (1.0 - e3), tv),
                 local_to_global2(xsi, xsi * e1, sv), n, k, true, e2);
        add_both(rs, rd, local_to_global2(xsi * (1.0 - e123), xsi * e1 * (1.0 - e2 * e3), tv),
                 local_to_global2(xsi, xsi * e12, sv), n, k, true, e2);
    }
    else if (nn == 1)
    {
        w = xsi * xsi * xsi * e2;
        add_both(rs, rd, local_to_global2(xsi, xsi * e1, tv), local_to_global2(xsi * e2, xsi * e2 * e3, sv), n, k,
                 false, 0);
        add_both(rs, rd, local_to_global2(xsi * e2, xsi * e2 * e3, tv), local_to_global2(xsi, xsi * e1, sv), n, k,
                 false, 0);
    }
    if (nn >= 1 && nn <= 3)
    {
        rs.re = rs.re * w;
        rs.im = rs.im * w;
        rs.re = rs.re * weight;
        rs.im = rs.im * weight;
        rd.re = rd.re * w;
        rd.im = rd.im * w;
        rd.re = rd.re * weight;
        rd.im = rd.im * weight;
    }
    os = rs;
    od = rd;
}

__device__ inline void face_to_face2(const f3 *src, const int *si, const f3 *trg, const int *ti, cf k, float threshold,
                                     cf &out_s, cf &out_d)
{
    float sj = jacobian(src), tj = jacobian(trg);
    int nn = common_vertices(si, ti);
    f3 sc = (src[0] + src[1] + src[2]) / 3;
    f3 tc = (trg[0] + trg[1] + trg[2]) / 3;
    float dist = len3(sc - tc);
    out_s = out_d = cf{0.0f, 0.0f};
    if (dist < threshold && nn == 0)
        return;
    if (nn == 0)
    {
        f3 nrm = tri_normal(src);
        const float gx = (float)PB_TRI_X;
        f3 a = local_to_global(gx, gx, src);
        f3 b = local_to_global(gx, gx, trg);
        double c = 0.25 * 1.0f * 1.0f * sj * tj;
        cf ls{0.0f, 0.0f}, ld{0.0f, 0.0f};
        both_acc(ls, ld, a, b, nrm, k, 1.0f, false);
        out_s = cf{(float)(0.0f + c * ls.re), (float)(0.0f + c * ls.im)};
        out_d = cf{(float)(0.0f + c * ld.re), (float)(0.0f + c * ld.im)};
        return;
    }
    const float gx[3] = {(float)PB_LINE_X0, 0.0f, (float)-PB_LINE_X0};
    const float gw[3] = {(float)PB_LINE_W0, (float)PB_LINE_W1, (float)PB_LINE_W0};
    f3 nrm = tri_normal(src);
    cf as{0.0f, 0.0f}, ad{0.0f, 0.0f};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++)
                for (int d = 0; d < 3; d++)
                {
                    cf rs, rd;
                    singular_node2(gx[a], gx[b], gx[c], gx[d], gw[a] * gw[b] * gw[c] * gw[d], src, trg, nrm, nn, k,
                                   rs, rd);
                    as.re += rs.re;
                    as.im += rs.im;
                    ad.re += rd.re;
                    ad.im += rd.im;
                }
    out_s = cf{as.re * sj, as.im * sj};
    out_s = cf{out_s.re * tj, out_s.im * tj};
    out_s = cf{out_s.re / 16, out_s.im / 16};
    out_d = cf{ad.re * sj, ad.im * sj};
    out_d = cf{out_d.re * tj, out_d.im * tj};
    out_d = cf{out_d.re / 16, out_d.im / 16};
}

// Recursive radix-2 transform of bem.h:12-38 (positive exponent), stage results rounded to
// float, twiddles applied in double.  in/out/buf: 16 entries; STEP is the current stride.
// Twiddle i of the transform, (cos, sin)(2 pi i / 16) with the reference's PI literal, from the
// device's own cos/sin: either computed here or read from a table filled by twiddle_fill.
__device__ inline void twiddle(int i, const double *tw, double &wr, double &wi)
{
    if (tw)
    {
        wr = tw[2 * i];
        wi = tw[2 * i + 1];
        return;
    }
    double ang = 2 * PB_PI * i / kTaps;
    wr = cos(ang);
    wi = sin(ang);
    if (ang == 0.0)
    {
        wr = 1.0;
        wi = 0.0;
    }
}

__device__ inline void twiddle_fill(double *tw)
{
    for (int i = 0; i < kTaps / 2; i++)
        twiddle(i, nullptr, tw[2 * i], tw[2 * i + 1]);
}

template <int STEP>
__device__ inline void fft_rec(const cf *in, cf *out, cf *buf, const double *tw)
{
    constexpr int N = kTaps;
    constexpr int NS = STEP * 2;
    fft_rec<NS>(in, out, buf, tw);
    fft_rec<NS>(in + STEP, out + STEP, buf + STEP, tw);
    for (int i = 0; i < N; i += NS)
    {
        buf[i / 2] = out[i];
        buf[(N + i) / 2] = out[i + STEP];
    }
    for (int i = 0; i < N / 2; i += STEP)
    {
        double wr, wi;
        twiddle(i, tw, wr, wi);
        cf b = buf[i + N / 2];
        double tre = wr * b.re - wi * b.im;
        double tim = wr * b.im + wi * b.re;
        cf a = buf[i];
        out[i] = cf{(float)(a.re + tre), (float)(a.im + tim)};
        out[i + N / 2] = cf{(float)(a.re - tre), (float)(a.im - tim)};
    }
}
template <>
__device__ inline void fft_rec<kTaps>(const cf *in, cf *out, cf *, const double *)
{
    out[0] = in[0];
}

// spectrum (16 values, k > 8 already conjugated) -> 16 real time-domain weights
__device__ inline void scaled_fft(const cf *spec, float lambda, float *out, const double *tw = nullptr)
{
    cf b1[kTaps], b2[kTaps];
    fft_rec<1>(spec, b1, b2, tw);
    float temp = 1.0f;
    for (int i = 0; i < kTaps; i++)
    {
        out[i] = b1[i].re / kTaps * temp;
        temp /= lambda;
    }
}

}  // namespace ref32

// ----------------------------------------------------------------------- f64 ---------
namespace f64
{
struct d3
{
    double x, y, z;
};
__device__ inline d3 dd(f3 a) { return d3{a.x, a.y, a.z}; }
__device__ inline d3 operator+(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ inline d3 operator-(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ inline d3 operator*(double s, d3 a) { return d3{s * a.x, s * a.y, s * a.z}; }
__device__ inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ inline d3 cross(d3 a, d3 b) { return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ inline double len(d3 a) { return sqrt(dot(a, a)); }

__device__ inline cd cexp(double x, double y)
{
    double e = exp(x), s, c;
    sincos(y, &s, &c);
    return cd{e * c, e * s};
}

__device__ inline void single_acc(cd &acc, d3 src, d3 trg, cd k, double scale)
{
    d3 d = trg - src;
    double r2 = dot(d, d);
    if (r2 != 0)
    {
        double r = sqrt(r2);
        cd e = cexp(-r * k.im, r * k.re);
        double den = 4 * M_PI * r;
        acc.re += e.re / den * scale;
        acc.im += e.im / den * scale;
    }
}

__device__ inline void double_acc(cd &acc, d3 src, d3 trg, d3 n, cd k, double scale)
{
    d3 d = src - trg;
    double r2 = dot(d, d);
    if (r2 != 0)
    {
        double r = sqrt(r2);
        double ire = -r * k.im, iim = r * k.re;
        cd e = cexp(ire, iim);
        double den = 4 * M_PI * r2 * r;
        double are = -e.re / den, aim = -e.im / den;
        double bre = 1.0 - ire, bim = -iim;
        double dn = dot(d, n) * scale;
        acc.re += (are * bre - aim * bim) * dn;
        acc.im += (are * bim + aim * bre) * dn;
    }
}

__device__ inline cd layer_point(d3 a, d3 b, d3 n, cd k, bool dbl)
{
    cd acc{0, 0};
    if (dbl)
        double_acc(acc, a, b, n, k, 1.0);
    else
        single_acc(acc, a, b, k, 1.0);
    return acc;
}

__device__ inline double jacobian(const d3 *v) { return len(cross(v[1] - v[0], v[2] - v[0])); }
__device__ inline d3 tri_normal(const d3 *v)
{
    d3 n = cross(v[1] - v[0], v[2] - v[0]);
    double l = len(n);
    return d3{n.x / l, n.y / l, n.z / l};
}
__device__ inline d3 ltg(double x1, double x2, const d3 *v) { return (1 - x1 - x2) * v[0] + x1 * v[1] + x2 * v[2]; }
__device__ inline d3 ltg2(double x1, double x2, const d3 *v) { return (1 - x1) * v[0] + (x1 - x2) * v[1] + x2 * v[2]; }

__device__ inline cd face_to_points(const d3 *src_v, const d3 *pts, const double *scales, int n, cd k, bool dbl)
{
    double jac = jacobian(src_v);
    d3 nrm = tri_normal(src_v);
    const double gx = 1.0 / 3.0;
    d3 q = ltg(gx, gx, src_v);
    cd lp{0, 0};
    for (int i = 0; i < n; i++)
    {
        if (dbl)
            double_acc(lp, q, pts[i], nrm, k, scales[i]);
        else
            single_acc(lp, q, pts[i], k, scales[i]);
    }
    return cd{0.5 * jac * lp.re, 0.5 * jac * lp.im};
}

__device__ inline void add_lp(cd &acc, d3 a, d3 b, d3 n, cd k, bool dbl, double s)
{
    cd lp = layer_point(a, b, n, k, dbl);
    acc.re += lp.re * s;
    acc.im += lp.im * s;
}

__device__ inline cd singular_face(const d3 *tv, const d3 *sv, double tj, double sj, cd k, int nn, bool dbl)
{
    const double gx[3] = {PB_LINE_X0, 0.0, -PB_LINE_X0};
    const double gw[3] = {PB_LINE_W0, PB_LINE_W1, PB_LINE_W0};
    d3 n = tri_normal(tv);
    cd acc{0, 0};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++)
                for (int d = 0; d < 3; d++)
                {
                    double xsi = 0.5 * (gx[a] + 1), e1 = 0.5 * (gx[b] + 1), e2 = 0.5 * (gx[c] + 1),
                           e3 = 0.5 * (gx[d] + 1);
                    double weight = gw[a] * gw[b] * gw[c] * gw[d];
                    cd r{0, 0};
                    if (nn == 3)
                    {
                        double w = xsi * xsi * xsi * e1 * e1 * e2, e12 = e1 * e2, e123 = e1 * e2 * e3;
                        add_lp(r, ltg2(xsi, xsi * (1 - e1 + e12), tv), ltg2(xsi * (1 - e123), xsi * (1 - e1), sv), n, k,
                               dbl, 1);
                        add_lp(r, ltg2(xsi * (1 - e123), xsi * (1 - e1), tv), ltg2(xsi, xsi * (1 - e1 + e12), sv), n, k,
                               dbl, 1);
                        add_lp(r, ltg2(xsi, xsi * (e1 - e12 + e123), tv), ltg2(xsi * (1 - e12), xsi * (e1 - e12), sv), n,
                               k, dbl, 1);
                        add_lp(r, ltg2(xsi * (1 - e12), xsi * (e1 - e12), tv), ltg2(xsi, xsi * (e1 - e12 + e123), sv), n,
                               k, dbl, 1);
                        add_lp(r, ltg2(xsi * (1 - e123), xsi * (e1 - e123), tv), ltg2(xsi, xsi * (e1 - e12), sv), n, k,
                               dbl, 1);
                        add_lp(r, ltg2(xsi, xsi * (e1 - e12), tv), ltg2(xsi * (1 - e123), xsi * (e1 - e123), sv), n, k,
                               dbl, 1);
                        r.re *= w * weight;
                        r.im *= w * weight;
                    }
                    else if (nn == 2)
                    {
                        double w = xsi * xsi * xsi * e1 * e1, e12 = e1 * e2, e123 = e1 * e2 * e3;
                        add_lp(r, ltg2(xsi, xsi * e1 * e3, tv), ltg2(xsi * (1 - e12), xsi * e1 * (1 - e2), sv), n, k,
                               dbl, 1);
                        add_lp(r, ltg2(xsi, xsi * e1, tv), ltg2(xsi * (1 - e123), xsi * e1 * e2 * (1 - e3), sv), n, k,
                               dbl, e2);
                        add_lp(r, ltg2(xsi * (1 - e12), xsi * e1 * (1 - e2), tv), ltg2(xsi, xsi * e123, sv), n, k, dbl,
                               e2);
                        add_lp(r, ltg2(xsi * (1 - e123), xsi * e12 * (1 - e3), tv), ltg2(xsi, xsi * e1, sv), n, k, dbl,
                               e2);
                        add_lp(r, ltg2(xsi * (1 - e123), xsi * e1 * (1 - e2 * e3), tv), ltg2(xsi, xsi * e12, sv), n, k,
                               dbl, e2);
                        r.re *= w * weight;
                        r.im *= w * weight;
                    }
                    else if (nn == 1)
                    {
                        double w = xsi * xsi * xsi * e2;
                        add_lp(r, ltg2(xsi, xsi * e1, tv), ltg2(xsi * e2, xsi * e2 * e3, sv), n, k, dbl, 1);
                        add_lp(r, ltg2(xsi * e2, xsi * e2 * e3, tv), ltg2(xsi, xsi * e1, sv), n, k, dbl, 1);
                        r.re *= w * weight;
                        r.im *= w * weight;
                    }
                    acc.re += r.re;
                    acc.im += r.im;
                }
    double s = tj * sj / 16;
    return cd{acc.re * s, acc.im * s};
}

__device__ inline cd face_to_face(const d3 *src, const int *si, const d3 *trg, const int *ti, cd k, double threshold,
                                  bool dbl)
{
    double sj = jacobian(src), tj = jacobian(trg);
    int nn = ref32::common_vertices(si, ti);
    d3 sc = (1.0 / 3) * (src[0] + src[1] + src[2]);
    d3 tc = (1.0 / 3) * (trg[0] + trg[1] + trg[2]);
    if (len(sc - tc) < threshold && nn == 0)
        return cd{0, 0};
    if (nn == 0)
    {
        d3 n = tri_normal(src);
        d3 a = ltg(1.0 / 3, 1.0 / 3, src), b = ltg(1.0 / 3, 1.0 / 3, trg);
        cd lp = layer_point(a, b, n, k, dbl);
        double c = 0.25 * sj * tj;
        return cd{c * lp.re, c * lp.im};
    }
    return singular_face(src, trg, sj, tj, k, nn, dbl);
}

// 16-point inverse DFT with lambda^-n scaling (the same transform as ref32::scaled_fft,
// evaluated directly in double)
__device__ inline void scaled_fft(const cd *spec, double lambda, double *out)
{
    for (int n = 0; n < kTaps; n++)
    {
        double acc = 0;
        for (int k = 0; k < kTaps; k++)
        {
            double ang = 2 * M_PI * (double)((n * k) % kTaps) / kTaps;
            acc += spec[k].re * cos(ang) - spec[k].im * sin(ang);
        }
        out[n] = acc / kTaps * pow(lambda, -(double)n);
    }
}

}  // namespace f64

}  // namespace pb
