/*
 * pppm_oracle.c - CPU restatement of the PPPM-TDBEM per-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity tests (tests/), __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load this library as the checker / baseline.  The product
 * (libpppm_b200.so) never links or calls it.
 *
 * It follows the reference's own order of operations per step (pppm.h:138-145): FDTD step,
 * far field = copy of the grid minus the FDTD-near sums, Neumann ring write, face far field,
 * face near field, Dirichlet update, near field add-back.  The GPU library fuses and
 * reorders these; agreement with this file is what the parity tests check.
 */
#define _GNU_SOURCE
#include "pppm_oracle.h"
#include <complex.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define TAPS 16
#define RING 32
#define FC_SLOTS 1024
#define PI_REF 3.14159265359

typedef _Float16 half_t;

typedef struct
{
    uint16_t s[TAPS];
    float ms;
    uint16_t d[TAPS];
    float md;
} rec72; /* bem.h:163-169 */

struct orc_scene
{
    int res, prec, pml;
    float dl, dt, c, reflect;
    float mn[3];
    long long ncell;
    int t;
    void *grid[3];
    void *pmlg[3];
    void *far;
    /* mesh */
    int mesh_set, nv, nt;
    float *V;
    int *F;
    float *center, *normal, *area;
    int *cellc, *basec, *cell, *base;
    int *cell_start, *cell_tris, *base_start, *base_tris;
    int n3;
    int *n3_cell, *n3_start, *p3_tri;
    unsigned char *p3_woff;
    int b4;
    int *b4_cell, *b4_start, *n4_tris, *b4_of_cell;
    long long pf;
    int *face_start, *face_nbr, *face_slot;
    int *corner;
    float *interp;
    double *interp_d;
    double *denom;
    /* grid cache: nt x 54 records */
    double *gc_w; /* nt x 54 x 32 unpacked (double) */
    rec72 *gc_r;
    float *gc_snap;
    int gc_empty;
    /* face cache pool */
    int *fc_keys, *fc_slots;
    long long pool_n, pool_cap;
    double *pool_w; /* pool x 32 */
    rec72 *pool_r;
    float *pool_meta; /* pool x 2 */
    /* histories */
    void *neumann, *dirichlet;
    /* TDBEM constants */
    double lambda;
    double complex wave[TAPS];
    double threshold;
    /* labels */
    int *type, *type_old, *nearest, *ghost;
    float *points;
};

/* ----------------------------------------------------------------- helpers --------- */
static void *xcalloc(size_t n, size_t sz)
{
    void *p = calloc(n ? n : 1, sz);
    return p;
}

static inline float h2f(uint16_t b)
{
    half_t h;
    memcpy(&h, &b, 2);
    return (float)h;
}
static inline uint16_t f2h(float f)
{
    half_t h = (half_t)f;
    uint16_t b;
    memcpy(&b, &h, 2);
    return b;
}

typedef struct
{
    double x, y, z;
} v3;
static inline v3 V3(double x, double y, double z)
{
    v3 r = {x, y, z};
    return r;
}
static inline v3 add(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(double s, v3 a) { return V3(s * a.x, s * a.y, s * a.z); }
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) { return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double norm(v3 a) { return sqrt(dot(a, a)); }

static inline v3 vert(const orc_scene *s, int i) { return V3(s->V[3 * i], s->V[3 * i + 1], s->V[3 * i + 2]); }
static inline long long lin(int res, int x, int y, int z) { return ((long long)x * res + y) * res + z; }
static inline int slot(int t) { return ((t % 3) + 3) % 3; }

/* cell centre (particle_grid.h:172-175) in float arithmetic */
static inline void cell_center_f(const orc_scene *s, int i, int j, int k, float *out)
{
    out[0] = (i + 0.5f) * s->dl + s->mn[0];
    out[1] = (j + 0.5f) * s->dl + s->mn[1];
    out[2] = (k + 0.5f) * s->dl + s->mn[2];
}

int orc_threads(void) { return omp_get_max_threads(); }

/* ----------------------------------------------------------------- TDBEM --------- */
/* TDBEM::init (bem.h:264-277) in double */
static void tdbem_init(orc_scene *s)
{
    double dtc = (double)s->dt * (double)s->c;
    double a = pow(dtc, 3.0 / TAPS), b = pow(1e-8, 1.0 / (2 * TAPS));
    s->lambda = a > b ? a : b;
    for (int k = 0; k < TAPS; k++)
    {
        double complex sk = s->lambda * cexp(-2.0 * M_PI * I * k / TAPS);
        double complex bdf2 = 0.5 * (sk * sk - 4.0 * sk + 3.0);
        s->wave[k] = bdf2 / dtc * I;
    }
    s->threshold = s->dl * 0.1;
}

/* potential.h:290-357: single layer e^{ikr}/(4 pi r) (target - source), double layer
 * -e^{ikr}(1 - ikr)((s - t).n)/(4 pi r^3) */
static double complex layer(v3 src, v3 trg, v3 n, double complex k, int dbl)
{
    if (!dbl)
    {
        v3 d = sub(trg, src);
        double r2 = dot(d, d);
        if (r2 == 0)
            return 0;
        double r = sqrt(r2);
        return cexp(I * r * k) / (4 * M_PI * r);
    }
    v3 d = sub(src, trg);
    double r2 = dot(d, d);
    if (r2 == 0)
        return 0;
    double r = sqrt(r2);
    double complex ikr = I * r * k;
    return -cexp(ikr) / (4 * M_PI * r2 * r) * (1.0 - ikr) * dot(d, n);
}

static v3 tri_normal(const v3 *v)
{
    v3 n = cross(sub(v[1], v[0]), sub(v[2], v[0]));
    return mul(1.0 / norm(n), n);
}
static double jacobian(const v3 *v) { return norm(cross(sub(v[1], v[0]), sub(v[2], v[0]))); }
static v3 ltg(double x1, double x2, const v3 *v)
{
    return add(add(mul(1 - x1 - x2, v[0]), mul(x1, v[1])), mul(x2, v[2]));
}
static v3 ltg2(double x1, double x2, const v3 *v) { return add(add(mul(1 - x1, v[0]), mul(x1 - x2, v[1])), mul(x2, v[2])); }

/* integrand.h:193-220: 1-point rule (centroid), weighted targets */
static double complex face_to_points(const v3 *sv, const v3 *pts, const double *sc, int n, double complex k, int dbl)
{
    double jac = jacobian(sv);
    v3 nrm = tri_normal(sv), q = ltg(1.0 / 3, 1.0 / 3, sv);
    double complex acc = 0;
    for (int i = 0; i < n; i++)
        acc += layer(q, pts[i], nrm, k, dbl) * sc[i];
    return 0.5 * jac * acc;
}

/* integrand.h:51-173: identical / common-edge / common-vertex panel rules (3-point
 * Gauss-Legendre per dimension), trial = src, test = trg, no vertex reordering */
static double complex singular_face(const v3 *tv, const v3 *sv, double tj, double sj, double complex k, int nn, int dbl)
{
    const double gx[3] = {0.774596669241483, 0.0, -0.774596669241483};
    const double gw[3] = {0.555555555555554, 0.888888888888889, 0.555555555555554};
    v3 n = tri_normal(tv);
    double complex acc = 0;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++)
                for (int d = 0; d < 3; d++)
                {
                    double xsi = 0.5 * (gx[a] + 1), e1 = 0.5 * (gx[b] + 1), e2 = 0.5 * (gx[c] + 1),
                           e3 = 0.5 * (gx[d] + 1);
                    double wgt = gw[a] * gw[b] * gw[c] * gw[d];
                    double complex r = 0;
                    if (nn == 3)
                    {
                        double w = xsi * xsi * xsi * e1 * e1 * e2, e12 = e1 * e2, e123 = e1 * e2 * e3;
                        r += layer(ltg2(xsi, xsi * (1 - e1 + e12), tv), ltg2(xsi * (1 - e123), xsi * (1 - e1), sv), n, k, dbl);
                        r += layer(ltg2(xsi * (1 - e123), xsi * (1 - e1), tv), ltg2(xsi, xsi * (1 - e1 + e12), sv), n, k, dbl);
                        r += layer(ltg2(xsi, xsi * (e1 - e12 + e123), tv), ltg2(xsi * (1 - e12), xsi * (e1 - e12), sv), n, k, dbl);
                        r += layer(ltg2(xsi * (1 - e12), xsi * (e1 - e12), tv), ltg2(xsi, xsi * (e1 - e12 + e123), sv), n, k, dbl);
                        r += layer(ltg2(xsi * (1 - e123), xsi * (e1 - e123), tv), ltg2(xsi, xsi * (e1 - e12), sv), n, k, dbl);
                        r += layer(ltg2(xsi, xsi * (e1 - e12), tv), ltg2(xsi * (1 - e123), xsi * (e1 - e123), sv), n, k, dbl);
                        r *= w * wgt;
                    }
                    else if (nn == 2)
                    {
                        double w = xsi * xsi * xsi * e1 * e1, e12 = e1 * e2, e123 = e1 * e2 * e3;
                        r += layer(ltg2(xsi, xsi * e1 * e3, tv), ltg2(xsi * (1 - e12), xsi * e1 * (1 - e2), sv), n, k, dbl);
                        r += layer(ltg2(xsi, xsi * e1, tv), ltg2(xsi * (1 - e123), xsi * e1 * e2 * (1 - e3), sv), n, k, dbl) * e2;
                        r += layer(ltg2(xsi * (1 - e12), xsi * e1 * (1 - e2), tv), ltg2(xsi, xsi * e123, sv), n, k, dbl) * e2;
                        r += layer(ltg2(xsi * (1 - e123), xsi * e12 * (1 - e3), tv), ltg2(xsi, xsi * e1, sv), n, k, dbl) * e2;
                        r += layer(ltg2(xsi * (1 - e123), xsi * e1 * (1 - e2 * e3), tv), ltg2(xsi, xsi * e12, sv), n, k, dbl) * e2;
                        r *= w * wgt;
                    }
                    else if (nn == 1)
                    {
                        double w = xsi * xsi * xsi * e2;
                        r += layer(ltg2(xsi, xsi * e1, tv), ltg2(xsi * e2, xsi * e2 * e3, sv), n, k, dbl);
                        r += layer(ltg2(xsi * e2, xsi * e2 * e3, tv), ltg2(xsi, xsi * e1, sv), n, k, dbl);
                        r *= w * wgt;
                    }
                    acc += r;
                }
    return acc * tj * sj / 16;
}

static int common_vertices(const int *a, const int *b)
{
    int n = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            n += a[i] == b[j];
    return n;
}

/* integrand.h:228-252 */
static double complex face_to_face(const v3 *sv, const int *si, const v3 *tv, const int *ti, double complex k, double thr,
                                   int dbl)
{
    double sj = jacobian(sv), tj = jacobian(tv);
    int nn = common_vertices(si, ti);
    v3 sc = mul(1.0 / 3, add(add(sv[0], sv[1]), sv[2])), tc = mul(1.0 / 3, add(add(tv[0], tv[1]), tv[2]));
    if (norm(sub(sc, tc)) < thr && nn == 0)
        return 0; /* the reference's near-coincident branch evaluates to zero */
    if (nn == 0)
    {
        v3 n = tri_normal(sv);
        return 0.25 * sj * tj * layer(ltg(1.0 / 3, 1.0 / 3, sv), ltg(1.0 / 3, 1.0 / 3, tv), n, k, dbl);
    }
    return singular_face(sv, tv, sj, tj, k, nn, dbl);
}

/* bem.h:292-321: spectrum at k <= 8 (conjugate-extended) -> 16 taps scaled by lambda^-n */
static void spectrum_to_taps(const double complex *sp9, double lambda, double *out)
{
    double complex sp[TAPS];
    for (int k = 0; k <= TAPS / 2; k++)
        sp[k] = sp9[k];
    for (int k = TAPS / 2 + 1; k < TAPS; k++)
        sp[k] = conj(sp[TAPS - k]);
    for (int n = 0; n < TAPS; n++)
    {
        double complex acc = 0;
        for (int k = 0; k < TAPS; k++)
            acc += sp[k] * cexp(2 * M_PI * I * (double)((n * k) % TAPS) / TAPS);
        out[n] = creal(acc) / TAPS * pow(lambda, -(double)n);
    }
}

static void load_tri(const orc_scene *s, int t, v3 *v, int *idx)
{
    for (int k = 0; k < 3; k++)
    {
        idx[k] = s->F[3 * t + k];
        v[k] = vert(s, idx[k]);
    }
}

static v3 center_d(const orc_scene *s, int i, int j, int k)
{
    return V3((i + 0.5) * s->dl + s->mn[0], (j + 0.5) * s->dl + s->mn[1], (k + 0.5) * s->dl + s->mn[2]);
}

/* pppm_cache.cu:64-123: FDTD-near and BEM-near weights of triangle tri at cell offset woff */
static void grid_weight(const orc_scene *s, int tri, int woff, double *fd, double *bm)
{
    v3 v[3];
    int idx[3];
    load_tri(s, tri, v, idx);
    int tx = s->cellc[3 * tri], ty = s->cellc[3 * tri + 1], tz = s->cellc[3 * tri + 2];
    int nx = tx + woff % 3 - 1, ny = ty + woff / 3 % 3 - 1, nz = tz + woff / 9 - 1;
    int dc[8][3] = {{nx, ny, nz}, {nx - 1, ny, nz}, {nx + 1, ny, nz}, {nx, ny - 1, nz},
                    {nx, ny + 1, nz}, {nx, ny, nz - 1}, {nx, ny, nz + 1}, {nx, ny, nz}};
    double sc = (double)s->c * s->c * s->dt * s->dt / ((double)s->dl * s->dl);
    double dsc[8] = {2, sc, sc, sc, sc, sc, sc, -6 * sc};
    v3 pts[8];
    double w[8];
    int n = 0;
    for (int i = 0; i < 8; i++)
        if (!(dc[i][0] == tx && dc[i][1] == ty && dc[i][2] == tz))
        {
            pts[n] = center_d(s, dc[i][0], dc[i][1], dc[i][2]);
            w[n] = dsc[i];
            n++;
        }
    double complex ss[TAPS / 2 + 1], sd[TAPS / 2 + 1];
    for (int k = 0; k <= TAPS / 2; k++)
    {
        ss[k] = face_to_points(v, pts, w, n, s->wave[k], 0);
        sd[k] = face_to_points(v, pts, w, n, s->wave[k], 1);
    }
    double ws[TAPS], wd[TAPS];
    spectrum_to_taps(ss, s->lambda, ws);
    spectrum_to_taps(sd, s->lambda, wd);
    for (int i = TAPS - 1; i >= 1; i--)
    {
        ws[i] = ws[i - 1];
        wd[i] = wd[i - 1];
    }
    ws[0] = wd[0] = 0;
    double ps[TAPS] = {0}, pd[TAPS] = {0};
    int inside = nx == tx && ny == ty && nz == tz;
    if (!inside)
    {
        v3 p = center_d(s, nx, ny, nz);
        double one = 1;
        double complex qs[TAPS / 2 + 1], qd[TAPS / 2 + 1];
        for (int k = 0; k <= TAPS / 2; k++)
        {
            qs[k] = face_to_points(v, &p, &one, 1, s->wave[k], 0);
            qd[k] = face_to_points(v, &p, &one, 1, s->wave[k], 1);
        }
        spectrum_to_taps(qs, s->lambda, ps);
        spectrum_to_taps(qd, s->lambda, pd);
        for (int i = 2; i < TAPS; i++)
        {
            ws[i] -= ps[i - 2];
            wd[i] -= pd[i - 2];
        }
    }
    for (int i = 0; i < TAPS; i++)
    {
        fd[i] = ws[i];
        fd[TAPS + i] = wd[i];
        bm[i] = ps[i];
        bm[TAPS + i] = pd[i];
    }
}

/* pppm_cache.cu:234-271: face pair weights (neighbour face onto centre face) */
static void face_weight(const orc_scene *s, int ctr, int nbr, double *out)
{
    v3 sv[3], tv[3];
    int si[3], ti[3];
    load_tri(s, nbr, sv, si);
    load_tri(s, ctr, tv, ti);
    double complex a[TAPS / 2 + 1], b[TAPS / 2 + 1];
    for (int k = 0; k <= TAPS / 2; k++)
    {
        a[k] = face_to_face(sv, si, tv, ti, s->wave[k], s->threshold, 0);
        b[k] = face_to_face(sv, si, tv, ti, s->wave[k], s->threshold, 1);
    }
    float nbc[3] = {s->center[3 * nbr], s->center[3 * nbr + 1], s->center[3 * nbr + 2]};
    v3 pts[8];
    double sc[8];
    int n = 0;
    int bx = s->basec[3 * ctr], by = s->basec[3 * ctr + 1], bz = s->basec[3 * ctr + 2];
    for (int dx = 0; dx < 2; dx++)
        for (int dy = 0; dy < 2; dy++)
            for (int dz = 0; dz < 2; dz++)
            {
                float c[3];
                cell_center_f(s, bx + dx, by + dy, bz + dz, c);
                double lim = s->dl * 1.5;
                if (fabsf(c[0] - nbc[0]) > lim || fabsf(c[1] - nbc[1]) > lim || fabsf(c[2] - nbc[2]) > lim)
                {
                    pts[n] = center_d(s, bx + dx, by + dy, bz + dz);
                    sc[n] = -s->interp_d[8 * ctr + dx * 4 + dy * 2 + dz];
                    n++;
                }
            }
    for (int k = 0; k <= TAPS / 2; k++)
    {
        a[k] += face_to_points(sv, pts, sc, n, s->wave[k], 0);
        b[k] += face_to_points(sv, pts, sc, n, s->wave[k], 1);
    }
    spectrum_to_taps(a, s->lambda, out);
    spectrum_to_taps(b, s->lambda, out + TAPS);
}

/* LayerWeightHalf::set (bem.h:171-191) from float taps */
static void pack(const double *w32, rec72 *r)
{
    float sv[TAPS], dv[TAPS], ms = 0, md = 0;
    for (int i = 0; i < TAPS; i++)
    {
        sv[i] = (float)w32[i];
        dv[i] = (float)w32[TAPS + i];
        ms = fmaxf(ms, fabsf(sv[i]));
        md = fmaxf(md, fabsf(dv[i]));
    }
    if (ms == 0)
        ms = 1;
    if (md == 0)
        md = 1;
    for (int i = 0; i < TAPS; i++)
    {
        r->s[i] = f2h(sv[i] / ms);
        r->d[i] = f2h(dv[i] / md);
    }
    r->ms = ms;
    r->md = md;
}

static void unpack(const rec72 *r, float *w32)
{
    for (int i = 0; i < TAPS; i++)
    {
        w32[i] = h2f(r->s[i]) * r->ms;
        w32[TAPS + i] = h2f(r->d[i]) * r->md;
    }
}

/* Frequency-domain pair integral at an arbitrary complex wave number (the reference's
 * TDBEM::helmholtz weights, bem.h:370-379): out4 = single (re, im), double (re, im). */
int orc_pair_integral(float dl, const float *V, const int *src, int to_point, const int *dst_face,
                      const float *dst_point, double k_re, double k_im, double *out4)
{
    v3 sv[3];
    for (int k = 0; k < 3; k++)
        sv[k] = V3(V[3 * src[k]], V[3 * src[k] + 1], V[3 * src[k] + 2]);
    double complex kk = k_re + I * k_im, a, b;
    if (to_point)
    {
        v3 p = V3(dst_point[0], dst_point[1], dst_point[2]);
        double one = 1;
        a = face_to_points(sv, &p, &one, 1, kk, 0);
        b = face_to_points(sv, &p, &one, 1, kk, 1);
    }
    else
    {
        v3 tv[3];
        for (int q = 0; q < 3; q++)
            tv[q] = V3(V[3 * dst_face[q]], V[3 * dst_face[q] + 1], V[3 * dst_face[q] + 2]);
        a = face_to_face(sv, src, tv, dst_face, kk, dl * 0.1, 0);
        b = face_to_face(sv, src, tv, dst_face, kk, dl * 0.1, 1);
    }
    out4[0] = creal(a);
    out4[1] = cimag(a);
    out4[2] = creal(b);
    out4[3] = cimag(b);
    return 0;
}

int orc_laplace_weight(float dt, float dl, float c, const float *V, const int *src, int to_point, const int *dst_face,
                       const float *dst_point, double *out32)
{
    orc_scene s;
    memset(&s, 0, sizeof(s));
    s.dt = dt;
    s.dl = dl;
    s.c = c;
    tdbem_init(&s);
    v3 sv[3];
    for (int k = 0; k < 3; k++)
        sv[k] = V3(V[3 * src[k]], V[3 * src[k] + 1], V[3 * src[k] + 2]);
    double complex a[TAPS / 2 + 1], b[TAPS / 2 + 1];
    for (int k = 0; k <= TAPS / 2; k++)
    {
        if (to_point)
        {
            v3 p = V3(dst_point[0], dst_point[1], dst_point[2]);
            double one = 1;
            a[k] = face_to_points(sv, &p, &one, 1, s.wave[k], 0);
            b[k] = face_to_points(sv, &p, &one, 1, s.wave[k], 1);
        }
        else
        {
            v3 tv[3];
            for (int q = 0; q < 3; q++)
                tv[q] = V3(V[3 * dst_face[q]], V[3 * dst_face[q] + 1], V[3 * dst_face[q] + 2]);
            a[k] = face_to_face(sv, src, tv, dst_face, s.wave[k], s.threshold, 0);
            b[k] = face_to_face(sv, src, tv, dst_face, s.wave[k], s.threshold, 1);
        }
    }
    spectrum_to_taps(a, s.lambda, out32);
    spectrum_to_taps(b, s.lambda, out32 + TAPS);
    return 0;
}

/* ----------------------------------------------------------------- scene --------- */
orc_scene *orc_create(int res, float dl, float dt, const float *min_pos, float reflect_coeff, float c, int pml_width,
                      int precision)
{
    if (res < 8 || dl <= 0 || dt <= 0)
        return NULL;
    orc_scene *s = (orc_scene *)xcalloc(1, sizeof(orc_scene));
    s->res = res;
    s->dl = dl;
    s->dt = dt;
    s->c = c;
    s->reflect = reflect_coeff;
    s->pml = pml_width;
    s->prec = precision;
    for (int k = 0; k < 3; k++)
        s->mn[k] = min_pos[k];
    s->ncell = (long long)res * res * res;
    s->t = -1;
    size_t rs = precision == ORC_F64 ? 8 : 4;
    for (int i = 0; i < 3; i++)
    {
        s->grid[i] = xcalloc(s->ncell, rs);
        if (pml_width > 0)
            s->pmlg[i] = xcalloc(s->ncell * 6, rs);
    }
    s->far = xcalloc(s->ncell, rs);
    tdbem_init(s);
    return s;
}

void orc_destroy(orc_scene *s)
{
    if (!s)
        return;
    void *p[] = {s->grid[0], s->grid[1], s->grid[2], s->pmlg[0], s->pmlg[1], s->pmlg[2], s->far, s->V, s->F,
                 s->center, s->normal, s->area, s->cellc, s->basec, s->cell, s->base, s->cell_start, s->cell_tris,
                 s->base_start, s->base_tris, s->n3_cell, s->n3_start, s->p3_tri, s->p3_woff, s->b4_cell,
                 s->b4_start, s->n4_tris, s->b4_of_cell, s->face_start, s->face_nbr, s->face_slot, s->corner,
                 s->interp, s->interp_d, s->denom, s->gc_w, s->gc_r, s->gc_snap, s->fc_keys, s->fc_slots, s->pool_w,
                 s->pool_r, s->pool_meta, s->neumann, s->dirichlet, s->type, s->type_old, s->nearest, s->ghost,
                 s->points};
    for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); i++)
        free(p[i]);
    free(s);
}

/* particle_grid.cu:40-88 (float arithmetic) */
static int geometry(orc_scene *s)
{
    int res = s->res;
    for (int i = 0; i < s->nt; i++)
    {
        float v[3][3];
        for (int k = 0; k < 3; k++)
            for (int q = 0; q < 3; q++)
                v[k][q] = s->V[3 * s->F[3 * i + k] + q];
        float e1[3], e2[3], c[3], cr[3];
        for (int q = 0; q < 3; q++)
        {
            c[q] = (v[0][q] + v[1][q] + v[2][q]) / 3.0f;
            e1[q] = v[1][q] - v[0][q];
            e2[q] = v[2][q] - v[0][q];
        }
        cr[0] = e1[1] * e2[2] - e1[2] * e2[1];
        cr[1] = e1[2] * e2[0] - e1[0] * e2[2];
        cr[2] = e1[0] * e2[1] - e1[1] * e2[0];
        float l = sqrtf(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        int g[3], b[3];
        for (int q = 0; q < 3; q++)
        {
            s->center[3 * i + q] = c[q];
            s->normal[3 * i + q] = cr[q] / l;
            g[q] = (int)((c[q] - s->mn[q]) / s->dl);
            float cc = (g[q] + 0.5f) * s->dl + s->mn[q];
            b[q] = g[q] - (c[q] - cc < 0);
            if (g[q] < 2 || g[q] > res - 3 || b[q] < 1 || b[q] > res - 3)
                return 1;
            s->cellc[3 * i + q] = g[q];
            s->basec[3 * i + q] = b[q];
        }
        s->area[i] = l / 2.0f;
        s->cell[i] = (int)lin(res, g[0], g[1], g[2]);
        s->base[i] = (int)lin(res, b[0], b[1], b[2]);
    }
    return 0;
}

/* CSR of keys with ids ascending inside a key */
static void csr(const int *key, int n, long long nkeys, int *start, int *list)
{
    memset(start, 0, sizeof(int) * (nkeys + 1));
    for (int i = 0; i < n; i++)
        start[key[i] + 1]++;
    for (long long c = 0; c < nkeys; c++)
        start[c + 1] += start[c];
    int *cur = (int *)xcalloc(nkeys, sizeof(int));
    for (int i = 0; i < n; i++) /* ascending i: lists come out sorted */
        list[start[key[i]] + cur[key[i]]++] = i;
    free(cur);
}

static inline int clen(const orc_scene *s, int x, int y, int z)
{
    if (x < 0 || y < 0 || z < 0 || x >= s->res || y >= s->res || z >= s->res)
        return 0;
    long long c = lin(s->res, x, y, z);
    return s->cell_start[c + 1] - s->cell_start[c];
}

/* particle_grid.cu:139-241: 3^3 lists of non-empty inner cells, 4^3 lists of non-empty base
 * cells, plus per-centre face pair lists */
static void lists(orc_scene *s)
{
    int res = s->res;
    long long nc = s->ncell;
    csr(s->cell, s->nt, nc, s->cell_start, s->cell_tris);
    csr(s->base, s->nt, nc, s->base_start, s->base_tris);
    free(s->n3_cell);
    free(s->n3_start);
    free(s->p3_tri);
    free(s->p3_woff);
    free(s->b4_cell);
    free(s->b4_start);
    free(s->n4_tris);
    int n3 = 0, b4 = 0;
    long long p3 = 0, p4 = 0;
    for (int x = 1; x <= res - 2; x++)
        for (int y = 1; y <= res - 2; y++)
            for (int z = 1; z <= res - 2; z++)
            {
                int s3 = 0;
                for (int dx = -1; dx <= 1; dx++)
                    for (int dy = -1; dy <= 1; dy++)
                        for (int dz = -1; dz <= 1; dz++)
                            s3 += clen(s, x + dx, y + dy, z + dz);
                if (s3)
                {
                    n3++;
                    p3 += s3;
                }
                long long c = lin(res, x, y, z);
                if (s->base_start[c + 1] > s->base_start[c])
                {
                    b4++;
                    for (int dx = -1; dx <= 2; dx++)
                        for (int dy = -1; dy <= 2; dy++)
                            for (int dz = -1; dz <= 2; dz++)
                                p4 += clen(s, x + dx, y + dy, z + dz);
                }
            }
    s->n3 = n3;
    s->b4 = b4;
    s->n3_cell = (int *)xcalloc(n3 + 1, sizeof(int));
    s->n3_start = (int *)xcalloc(n3 + 1, sizeof(int));
    s->p3_tri = (int *)xcalloc(p3 + 1, sizeof(int));
    s->p3_woff = (unsigned char *)xcalloc(p3 + 1, 1);
    s->b4_cell = (int *)xcalloc(b4 + 1, sizeof(int));
    s->b4_start = (int *)xcalloc(b4 + 1, sizeof(int));
    s->n4_tris = (int *)xcalloc(p4 + 1, sizeof(int));
    if (!s->b4_of_cell)
        s->b4_of_cell = (int *)xcalloc(nc, sizeof(int));
    for (long long c = 0; c < nc; c++)
        s->b4_of_cell[c] = -1;
    long long o3 = 0, o4 = 0;
    int i3 = 0, i4 = 0;
    for (int x = 1; x <= res - 2; x++)
        for (int y = 1; y <= res - 2; y++)
            for (int z = 1; z <= res - 2; z++)
            {
                long long c = lin(res, x, y, z);
                long long st = o3;
                for (int idx = 0; idx < 27; idx++)
                {
                    int dx = idx % 3 - 1, dy = idx / 3 % 3 - 1, dz = idx / 9 - 1;
                    long long sc = lin(res, x + dx, y + dy, z + dz);
                    for (int j = s->cell_start[sc]; j < s->cell_start[sc + 1]; j++)
                    {
                        s->p3_tri[o3] = s->cell_tris[j];
                        s->p3_woff[o3] = (unsigned char)((1 - dx) + 3 * (1 - dy) + 9 * (1 - dz));
                        o3++;
                    }
                }
                if (o3 > st)
                {
                    s->n3_cell[i3] = (int)c;
                    s->n3_start[i3] = (int)st;
                    i3++;
                }
                if (s->base_start[c + 1] > s->base_start[c])
                {
                    s->b4_cell[i4] = (int)c;
                    s->b4_start[i4] = (int)o4;
                    s->b4_of_cell[c] = i4;
                    i4++;
                    for (int idx = 0; idx < 64; idx++)
                    {
                        int sx = x + idx % 4 - 1, sy = y + idx / 4 % 4 - 1, sz = z + idx / 16 - 1;
                        if (sx < 0 || sy < 0 || sz < 0 || sx >= res || sy >= res || sz >= res)
                            continue;
                        long long sc = lin(res, sx, sy, sz);
                        for (int j = s->cell_start[sc]; j < s->cell_start[sc + 1]; j++)
                            s->n4_tris[o4++] = s->cell_tris[j];
                    }
                }
            }
    s->n3_start[n3] = (int)o3;
    s->b4_start[b4] = (int)o4;
    /* face pairs */
    long long pf = 0;
    for (int i = 0; i < s->nt; i++)
    {
        int k = s->b4_of_cell[s->base[i]];
        s->face_start[i] = (int)pf;
        if (k >= 0)
            pf += s->b4_start[k + 1] - s->b4_start[k];
    }
    s->face_start[s->nt] = (int)pf;
    s->pf = pf;
    free(s->face_nbr);
    free(s->face_slot);
    s->face_nbr = (int *)xcalloc(pf + 1, sizeof(int));
    s->face_slot = (int *)xcalloc(pf + 1, sizeof(int));
    for (int i = 0; i < s->nt; i++)
    {
        int k = s->b4_of_cell[s->base[i]];
        int o = s->face_start[i];
        if (k >= 0)
            for (int j = s->b4_start[k]; j < s->b4_start[k + 1]; j++)
                s->face_nbr[o++] = s->n4_tris[j];
        for (int w = 0; w < 8; w++)
            s->corner[8 * i + w] =
                (int)lin(res, s->basec[3 * i] + (w >> 2), s->basec[3 * i + 1] + ((w >> 1) & 1), s->basec[3 * i + 2] + (w & 1));
    }
}

/* pppm_cache.cu:157-181 */
static void interp_weights(orc_scene *s)
{
    for (int i = 0; i < s->nt; i++)
    {
        v3 v[3];
        int idx[3];
        load_tri(s, i, v, idx);
        double jac = jacobian(v);
        v3 q = ltg(1.0 / 3, 1.0 / 3, v);
        v3 b = center_d(s, s->basec[3 * i], s->basec[3 * i + 1], s->basec[3 * i + 2]);
        double dx = (q.x - b.x) / s->dl, dy = (q.y - b.y) / s->dl, dz = (q.z - b.z) / s->dl;
        double w[8] = {(1 - dx) * (1 - dy) * (1 - dz), (1 - dx) * (1 - dy) * dz, (1 - dx) * dy * (1 - dz),
                       (1 - dx) * dy * dz,             dx * (1 - dy) * (1 - dz), dx * (1 - dy) * dz,
                       dx * dy * (1 - dz),             dx * dy * dz};
        for (int k = 0; k < 8; k++)
        {
            s->interp_d[8 * i + k] = 0.5 * jac * w[k];
            s->interp[8 * i + k] = (float)s->interp_d[8 * i + k];
        }
    }
}

static unsigned hash_slot(int key) { return ((unsigned)key * 2654435761u) >> 22; }

/* refresh both caches under the reference's criteria (pppm_cache.h:65-70, 123-128) */
static int caches(orc_scene *s)
{
    int nt = s->nt;
    /* grid cache */
    int *flag = (int *)xcalloc(nt, sizeof(int));
    for (int i = 0; i < nt; i++)
    {
        if (s->gc_empty)
        {
            flag[i] = 1;
            continue;
        }
        float *o = s->gc_snap + 7 * i;
        float dc[3], dn[3];
        for (int q = 0; q < 3; q++)
        {
            dc[q] = o[q] - s->center[3 * i + q];
            dn[q] = o[3 + q] - s->normal[3 * i + q];
        }
        float lc = sqrtf(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]);
        float ln = sqrtf(dn[0] * dn[0] + dn[1] * dn[1] + dn[2] * dn[2]);
        flag[i] = lc > 0.01 * s->dl || ln > 0.01 || fabsf(o[6] - s->area[i]) > 0.01 * s->area[i];
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (long long g = 0; g < (long long)nt * 27; g++)
    {
        int i = (int)(g / 27), woff = (int)(g % 27);
        if (!flag[i])
            continue;
        double fd[2 * TAPS], bm[2 * TAPS];
        grid_weight(s, i, woff, fd, bm);
        memcpy(s->gc_w + ((size_t)i * 54 + woff) * 32, fd, sizeof(fd));
        memcpy(s->gc_w + ((size_t)i * 54 + 27 + woff) * 32, bm, sizeof(bm));
        pack(fd, &s->gc_r[(size_t)i * 54 + woff]);
        pack(bm, &s->gc_r[(size_t)i * 54 + 27 + woff]);
    }
    for (int i = 0; i < nt; i++)
        if (flag[i])
        {
            memcpy(s->gc_snap + 7 * i, s->center + 3 * i, 3 * sizeof(float));
            memcpy(s->gc_snap + 7 * i + 3, s->normal + 3 * i, 3 * sizeof(float));
            s->gc_snap[7 * i + 6] = s->area[i];
        }
    free(flag);
    s->gc_empty = 0;
    /* face cache */
    interp_weights(s);
    if (s->pool_n + s->pf > s->pool_cap)
    {
        long long cap = s->pool_n + s->pf + (s->pool_n + s->pf) / 2 + 1024;
        s->pool_w = (double *)realloc(s->pool_w, sizeof(double) * 32 * cap);
        s->pool_r = (rec72 *)realloc(s->pool_r, sizeof(rec72) * cap);
        s->pool_meta = (float *)realloc(s->pool_meta, sizeof(float) * 2 * cap);
        s->pool_cap = cap;
    }
    int *recompute = (int *)xcalloc(s->pf + 1, sizeof(int));
    for (int ctr = 0; ctr < nt; ctr++)
    {
        int *keys = s->fc_keys + (size_t)ctr * FC_SLOTS, *slots = s->fc_slots + (size_t)ctr * FC_SLOTS;
        for (int p = s->face_start[ctr]; p < s->face_start[ctr + 1]; p++)
        {
            int nbr = s->face_nbr[p], sl = -1, fresh = 0;
            unsigned h = hash_slot(nbr);
            for (int probe = 0; probe < FC_SLOTS; probe++)
            {
                unsigned pos = (h + probe) & (FC_SLOTS - 1);
                if (keys[pos] == nbr)
                {
                    sl = slots[pos];
                    break;
                }
                if (keys[pos] == -1)
                {
                    keys[pos] = nbr;
                    sl = slots[pos] = (int)s->pool_n++;
                    fresh = 1;
                    break;
                }
            }
            if (sl < 0)
            {
                free(recompute);
                return 3;
            }
            float ang = s->normal[3 * nbr] * s->normal[3 * ctr] + s->normal[3 * nbr + 1] * s->normal[3 * ctr + 1] +
                        s->normal[3 * nbr + 2] * s->normal[3 * ctr + 2];
            float d[3] = {s->center[3 * nbr] - s->center[3 * ctr], s->center[3 * nbr + 1] - s->center[3 * ctr + 1],
                          s->center[3 * nbr + 2] - s->center[3 * ctr + 2]};
            float dist = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            int rc = fresh || fabsf(s->pool_meta[2 * sl] - ang) > 0.01 || fabsf(s->pool_meta[2 * sl + 1] - dist) > 0.01 * dist;
            if (rc)
            {
                s->pool_meta[2 * sl] = ang;
                s->pool_meta[2 * sl + 1] = dist;
            }
            s->face_slot[p] = sl;
            recompute[p] = rc;
        }
    }
#pragma omp parallel for schedule(dynamic, 8)
    for (long long p = 0; p < s->pf; p++)
    {
        if (!recompute[p])
            continue;
        int lo = 0, hi = nt;
        while (hi - lo > 1)
        {
            int mid = (lo + hi) / 2;
            if (s->face_start[mid] <= p)
                lo = mid;
            else
                hi = mid;
        }
        double w[2 * TAPS];
        face_weight(s, lo, s->face_nbr[p], w);
        int sl = s->face_slot[p];
        memcpy(s->pool_w + (size_t)sl * 32, w, sizeof(w));
        pack(w, &s->pool_r[sl]);
    }
    free(recompute);
    return 0;
}

/* 0.5 * area - sum of double-layer weight 0 over the face's list (pppm.cu:172-193) */
static void denominators(orc_scene *s)
{
    for (int i = 0; i < s->nt; i++)
    {
        if (s->prec == ORC_F64)
        {
            double sum = 0;
            for (int p = s->face_start[i]; p < s->face_start[i + 1]; p++)
                sum += s->pool_w[(size_t)s->face_slot[p] * 32 + TAPS];
            s->denom[i] = 0.5 * s->area[i] - sum;
        }
        else
        {
            float sum = 0;
            for (int p = s->face_start[i]; p < s->face_start[i + 1]; p++)
            {
                const rec72 *r = &s->pool_r[s->face_slot[p]];
                sum += h2f(r->d[0]) * r->md;
            }
            s->denom[i] = 0.5 * s->area[i] - sum;
        }
    }
}

static int set_mesh_impl(orc_scene *s, const float *V, int nv, const int *F, int nt, const int *cells6);

int orc_set_mesh(orc_scene *s, const float *V, int nv, const int *F, int nt)
{
    return set_mesh_impl(s, V, nv, F, nt, NULL);
}

/* Same as orc_set_mesh with the triangles' grid and base cells given (nt x 6), e.g. the
 * reference's own assignment for centres that fall exactly on a cell face, where its
 * approximate device division and the oracle's IEEE division can round to different cells. */
int orc_set_mesh_cells(orc_scene *s, const float *V, int nv, const int *F, int nt, const int *cells6)
{
    return set_mesh_impl(s, V, nv, F, nt, cells6);
}

static int set_mesh_impl(orc_scene *s, const float *V, int nv, const int *F, int nt, const int *cells6)
{
    if (!s || s->mesh_set || nv <= 0 || nt <= 0)
        return 1;
    s->nv = nv;
    s->nt = nt;
    s->V = (float *)xcalloc(3 * nv, sizeof(float));
    s->F = (int *)xcalloc(3 * nt, sizeof(int));
    memcpy(s->V, V, sizeof(float) * 3 * nv);
    memcpy(s->F, F, sizeof(int) * 3 * nt);
    s->center = (float *)xcalloc(3 * nt, sizeof(float));
    s->normal = (float *)xcalloc(3 * nt, sizeof(float));
    s->area = (float *)xcalloc(nt, sizeof(float));
    s->cellc = (int *)xcalloc(3 * nt, sizeof(int));
    s->basec = (int *)xcalloc(3 * nt, sizeof(int));
    s->cell = (int *)xcalloc(nt, sizeof(int));
    s->base = (int *)xcalloc(nt, sizeof(int));
    s->cell_start = (int *)xcalloc(s->ncell + 1, sizeof(int));
    s->base_start = (int *)xcalloc(s->ncell + 1, sizeof(int));
    s->cell_tris = (int *)xcalloc(nt, sizeof(int));
    s->base_tris = (int *)xcalloc(nt, sizeof(int));
    s->face_start = (int *)xcalloc(nt + 1, sizeof(int));
    s->corner = (int *)xcalloc(8 * (size_t)nt, sizeof(int));
    s->interp = (float *)xcalloc(8 * (size_t)nt, sizeof(float));
    s->interp_d = (double *)xcalloc(8 * (size_t)nt, sizeof(double));
    s->denom = (double *)xcalloc(nt, sizeof(double));
    s->gc_w = (double *)xcalloc((size_t)nt * 54 * 32, sizeof(double));
    s->gc_r = (rec72 *)xcalloc((size_t)nt * 54, sizeof(rec72));
    s->gc_snap = (float *)xcalloc((size_t)nt * 7, sizeof(float));
    s->gc_empty = 1;
    s->fc_keys = (int *)malloc(sizeof(int) * (size_t)nt * FC_SLOTS);
    s->fc_slots = (int *)malloc(sizeof(int) * (size_t)nt * FC_SLOTS);
    memset(s->fc_keys, 0xff, sizeof(int) * (size_t)nt * FC_SLOTS);
    size_t rs = s->prec == ORC_F64 ? 8 : 4;
    s->neumann = xcalloc((size_t)nt * RING, rs);
    s->dirichlet = xcalloc((size_t)nt * RING, rs);
    if (geometry(s))
        return 1;
    if (cells6)
        for (int i = 0; i < nt; i++)
        {
            for (int q = 0; q < 3; q++)
            {
                s->cellc[3 * i + q] = cells6[6 * i + q];
                s->basec[3 * i + q] = cells6[6 * i + 3 + q];
            }
            s->cell[i] = (int)lin(s->res, cells6[6 * i], cells6[6 * i + 1], cells6[6 * i + 2]);
            s->base[i] = (int)lin(s->res, cells6[6 * i + 3], cells6[6 * i + 4], cells6[6 * i + 5]);
        }
    lists(s);
    if (caches(s))
        return 3;
    denominators(s);
    s->mesh_set = 1;
    return 0;
}

int orc_update_mesh(orc_scene *s, const float *V)
{
    if (!s || !s->mesh_set)
        return 5;
    memcpy(s->V, V, sizeof(float) * 3 * s->nv);
    if (geometry(s))
        return 1;
    lists(s);
    if (caches(s))
        return 3;
    denominators(s);
    return 0;
}

/* ----------------------------------------------------------------- step ---------- */
/* fdtd.cu:36-78 */
static void solve4(float a[4][4], float b[4], float r[4])
{
    float s0 = a[0][0] * a[1][1] - a[1][0] * a[0][1], s1 = a[0][0] * a[1][2] - a[1][0] * a[0][2];
    float s2 = a[0][0] * a[1][3] - a[1][0] * a[0][3], s3 = a[0][1] * a[1][2] - a[1][1] * a[0][2];
    float s4 = a[0][1] * a[1][3] - a[1][1] * a[0][3], s5 = a[0][2] * a[1][3] - a[1][2] * a[0][3];
    float c5 = a[2][2] * a[3][3] - a[3][2] * a[2][3], c4 = a[2][1] * a[3][3] - a[3][1] * a[2][3];
    float c3 = a[2][1] * a[3][2] - a[3][1] * a[2][2], c2 = a[2][0] * a[3][3] - a[3][0] * a[2][3];
    float c1 = a[2][0] * a[3][2] - a[3][0] * a[2][2], c0 = a[2][0] * a[3][1] - a[3][0] * a[2][1];
    float inv_det = 1.0 / (s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0);
    float m[4][4];
    m[0][0] = (a[1][1] * c5 - a[1][2] * c4 + a[1][3] * c3) * inv_det;
    m[0][1] = (-a[0][1] * c5 + a[0][2] * c4 - a[0][3] * c3) * inv_det;
    m[0][2] = (a[3][1] * s5 - a[3][2] * s4 + a[3][3] * s3) * inv_det;
    m[0][3] = (-a[2][1] * s5 + a[2][2] * s4 - a[2][3] * s3) * inv_det;
    m[1][0] = (-a[1][0] * c5 + a[1][2] * c2 - a[1][3] * c1) * inv_det;
    m[1][1] = (a[0][0] * c5 - a[0][2] * c2 + a[0][3] * c1) * inv_det;
    m[1][2] = (-a[3][0] * s5 + a[3][2] * s2 - a[3][3] * s1) * inv_det;
    m[1][3] = (a[2][0] * s5 - a[2][2] * s2 + a[2][3] * s1) * inv_det;
    m[2][0] = (a[1][0] * c4 - a[1][1] * c2 + a[1][3] * c0) * inv_det;
    m[2][1] = (-a[0][0] * c4 + a[0][1] * c2 - a[0][3] * c0) * inv_det;
    m[2][2] = (a[3][0] * s4 - a[3][1] * s2 + a[3][3] * s0) * inv_det;
    m[2][3] = (-a[2][0] * s4 + a[2][1] * s2 - a[2][3] * s0) * inv_det;
    m[3][0] = (-a[1][0] * c3 + a[1][1] * c1 - a[1][2] * c0) * inv_det;
    m[3][1] = (a[0][0] * c3 - a[0][1] * c1 + a[0][2] * c0) * inv_det;
    m[3][2] = (-a[3][0] * s3 + a[3][1] * s1 - a[3][2] * s0) * inv_det;
    m[3][3] = (a[2][0] * s3 - a[2][1] * s1 + a[2][2] * s0) * inv_det;
    for (int i = 0; i < 4; i++)
    {
        r[i] = 0;
        for (int j = 0; j < 4; j++)
            r[i] += m[i][j] * b[j];
    }
}

#define DEFINE_STEP(R, SUFFIX)                                                                                          \
    static void abc_##SUFFIX(const orc_scene *s, R *cur, const R *prev, R *next, int x, int y, int z)                  \
    {                                                                                                                    \
        int res = s->res, q[3] = {x, y, z}, judge[3];                                                                    \
        for (int d = 0; d < 3; d++)                                                                                      \
            judge[d] = -(q[d] == 1) + (q[d] == res - 2);                                                                 \
        R c = s->c, dt = s->dt, h = s->dl;                                                                               \
        long long ci = lin(res, x, y, z);                                                                                \
        R pc = cur[ci], pp = prev[ci];                                                                                   \
        long long st[3] = {(long long)res * res, res, 1};                                                                \
        R a[4][4], b[4], coef = c * c * dt * dt / (h * h);                                                              \
        a[3][3] = 1;                                                                                                     \
        for (int d = 0; d < 3; d++)                                                                                      \
            a[3][d] = -coef * (judge[d] != 0);                                                                           \
        b[3] = -pp + 2 * pc - coef * (6 * pc);                                                                           \
        for (int d = 0; d < 3; d++)                                                                                      \
            b[3] += coef * cur[ci + st[d]] * (judge[d] <= 0) + coef * cur[ci - st[d]] * (judge[d] >= 0);                \
        R c1 = 1 / (dt * dt), c2 = c / (2 * h * dt), c3 = -(c * c) / (2 * h * h);                                        \
        for (int i = 0; i < 3; i++)                                                                                      \
        {                                                                                                                \
            int ax = i, ay = (i + 1) % 3, az = (i + 2) % 3;                                                              \
            a[i][3] = c1;                                                                                                \
            a[i][ax] = c2;                                                                                               \
            a[i][ay] = c3 * (judge[ay] != 0);                                                                            \
            a[i][az] = c3 * (judge[az] != 0);                                                                            \
            b[i] = -c1 * (pp - 2 * pc) +                                                                                 \
                   -c2 * (cur[ci + st[ax]] * (-(judge[ax] < 0)) + cur[ci - st[ax]] * (-(judge[ax] > 0)) +               \
                          prev[ci + st[ax]] * (-judge[ax]) + prev[ci - st[ax]] * judge[ax]) +                            \
                   -c3 * (cur[ci + st[ay]] * (judge[ay] <= 0) + cur[ci - st[ay]] * (judge[ay] >= 0) +                   \
                          cur[ci + st[az]] * (judge[az] <= 0) + cur[ci - st[az]] * (judge[az] >= 0) - 4 * pc);          \
        }                                                                                                                \
        R r[4];                                                                                                          \
        solve4_##SUFFIX(a, b, r);                                                                                        \
        next[ci] = r[3];                                                                                                 \
        for (int d = 0; d < 3; d++)                                                                                      \
            if (judge[d])                                                                                                \
                cur[ci + judge[d] * st[d]] = r[d];                                                                       \
    }                                                                                                                    \
    static R conv_##SUFFIX(const R *w32, const R *n, const R *d, int t)                                                 \
    {                                                                                                                    \
        R acc = 0;                                                                                                       \
        for (int k = 0; k < TAPS; k++)                                                                                   \
        {                                                                                                                \
            int sl = ((t - k) % RING + RING) % RING;                                                                     \
            acc += -w32[k] * n[sl] + w32[TAPS + k] * d[sl];                                                              \
        }                                                                                                                \
        return acc;                                                                                                      \
    }                                                                                                                    \
    static void step_##SUFFIX(orc_scene *s, const float *acc, const R *wgc, const R *wface)                            \
    {                                                                                                                    \
        int res = s->res, t = s->t;                                                                                      \
        R *cur = (R *)s->grid[slot(t)], *prev = (R *)s->grid[slot(t - 1)], *next = (R *)s->grid[slot(t + 1)];           \
        double cd = s->c, dtd = s->dt, hd = s->dl, coefd = cd * cd * dtd * dtd;                                          \
        long long sx = (long long)res * res;                                                                             \
        if (s->pml > 0)                                                                                                  \
            pml_##SUFFIX(s, cur, prev, next);                                                                            \
        else                                                                                                             \
        {                                                                                                                \
            _Pragma("omp parallel for schedule(static)") for (int x = 2; x <= res - 3; x++) for (int y = 2;             \
                                                                                              y <= res - 3; y++)         \
                for (int z = 2; z <= res - 3; z++)                                                                       \
                {                                                                                                        \
                    long long i = lin(res, x, y, z);                                                                     \
                    R pc = cur[i];                                                                                       \
                    double sum = 0;                                                                                      \
                    sum += cur[i - sx];                                                                                  \
                    sum += cur[i + sx];                                                                                  \
                    sum += cur[i - res];                                                                                 \
                    sum += cur[i + res];                                                                                 \
                    sum += cur[i - 1];                                                                                   \
                    sum += cur[i + 1];                                                                                   \
                    sum -= 6 * pc;                                                                                       \
                    double lap = sum / (hd * hd);                                                                        \
                    double p = 2 * pc;                                                                                   \
                    p += coefd * lap;                                                                                    \
                    p += -prev[i];                                                                                       \
                    next[i] = (R)p;                                                                                      \
                }                                                                                                        \
            for (int x = 1; x <= res - 2; x++)                                                                           \
                for (int y = 1; y <= res - 2; y++)                                                                       \
                    for (int z = 1; z <= res - 2; z++)                                                                   \
                        if (x == 1 || y == 1 || z == 1 || x == res - 2 || y == res - 2 || z == res - 2)                  \
                            abc_##SUFFIX(s, cur, prev, next, x, y, z);                                                   \
        }                                                                                                                \
        s->t = ++t;                                                                                                      \
        if (!s->mesh_set)                                                                                                \
            return;                                                                                                      \
        R *p = next, *far = (R *)s->far, *N = (R *)s->neumann, *D = (R *)s->dirichlet;                                 \
        memcpy(far, p, sizeof(R) * s->ncell);                                                                            \
        _Pragma("omp parallel for schedule(dynamic, 64)") for (int i = 0; i < s->n3; i++)                               \
        {                                                                                                                \
            R sum = 0;                                                                                                   \
            for (int q = s->n3_start[i]; q < s->n3_start[i + 1]; q++)                                                   \
            {                                                                                                            \
                int tri = s->p3_tri[q];                                                                                  \
                sum += conv_##SUFFIX(wgc + ((size_t)tri * 54 + s->p3_woff[q]) * 32, N + (size_t)tri * RING,            \
                                     D + (size_t)tri * RING, t);                                                         \
            }                                                                                                            \
            far[s->n3_cell[i]] = p[s->n3_cell[i]] - sum;                                                                 \
        }                                                                                                                \
        int ts = ((t % RING) + RING) % RING;                                                                             \
        for (int i = 0; i < s->nt; i++)                                                                                  \
        {                                                                                                                \
            N[(size_t)i * RING + ts] = acc[i];                                                                           \
            D[(size_t)i * RING + ts] = 0;                                                                                \
        }                                                                                                                \
        R *newd = (R *)malloc(sizeof(R) * s->nt);                                                                        \
        _Pragma("omp parallel for schedule(dynamic, 64)") for (int i = 0; i < s->nt; i++)                               \
        {                                                                                                                \
            R far_sum = 0;                                                                                               \
            for (int w = 0; w < 8; w++)                                                                                  \
                far_sum += (s->prec == ORC_F64 ? (R)s->interp_d[8 * i + w] : (R)s->interp[8 * i + w]) *                 \
                           far[s->corner[8 * i + w]];                                                                    \
            R near_sum = 0;                                                                                              \
            for (int q = s->face_start[i]; q < s->face_start[i + 1]; q++)                                               \
            {                                                                                                            \
                int nb = s->face_nbr[q];                                                                                 \
                near_sum += conv_##SUFFIX(wface + (size_t)s->face_slot[q] * 32, N + (size_t)nb * RING,                  \
                                          D + (size_t)nb * RING, t);                                                     \
            }                                                                                                            \
            newd[i] = (R)((double)(far_sum * (R)s->reflect + near_sum) / s->denom[i]);                                  \
        }                                                                                                                \
        for (int i = 0; i < s->nt; i++)                                                                                  \
            D[(size_t)i * RING + ts] = newd[i];                                                                          \
        free(newd);                                                                                                      \
        _Pragma("omp parallel for schedule(dynamic, 64)") for (int i = 0; i < s->n3; i++)                               \
        {                                                                                                                \
            R sum = 0;                                                                                                   \
            for (int q = s->n3_start[i]; q < s->n3_start[i + 1]; q++)                                                   \
            {                                                                                                            \
                int tri = s->p3_tri[q];                                                                                  \
                sum += conv_##SUFFIX(wgc + ((size_t)tri * 54 + 27 + s->p3_woff[q]) * 32, N + (size_t)tri * RING,       \
                                     D + (size_t)tri * RING, t);                                                         \
            }                                                                                                            \
            int c = s->n3_cell[i];                                                                                       \
            p[c] = (R)((double)far[c] + (double)sum * 0.98);                                                             \
        }                                                                                                                \
    }

static void solve4_f(float a[4][4], float b[4], float r[4]) { solve4(a, b, r); }
static void solve4_d(double a[4][4], double b[4], double r[4])
{
    double s0 = a[0][0] * a[1][1] - a[1][0] * a[0][1], s1 = a[0][0] * a[1][2] - a[1][0] * a[0][2];
    double s2 = a[0][0] * a[1][3] - a[1][0] * a[0][3], s3 = a[0][1] * a[1][2] - a[1][1] * a[0][2];
    double s4 = a[0][1] * a[1][3] - a[1][1] * a[0][3], s5 = a[0][2] * a[1][3] - a[1][2] * a[0][3];
    double c5 = a[2][2] * a[3][3] - a[3][2] * a[2][3], c4 = a[2][1] * a[3][3] - a[3][1] * a[2][3];
    double c3 = a[2][1] * a[3][2] - a[3][1] * a[2][2], c2 = a[2][0] * a[3][3] - a[3][0] * a[2][3];
    double c1 = a[2][0] * a[3][2] - a[3][0] * a[2][2], c0 = a[2][0] * a[3][1] - a[3][0] * a[2][1];
    double id = 1.0 / (s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0);
    double m[4][4] = {{(a[1][1] * c5 - a[1][2] * c4 + a[1][3] * c3) * id, (-a[0][1] * c5 + a[0][2] * c4 - a[0][3] * c3) * id,
                       (a[3][1] * s5 - a[3][2] * s4 + a[3][3] * s3) * id, (-a[2][1] * s5 + a[2][2] * s4 - a[2][3] * s3) * id},
                      {(-a[1][0] * c5 + a[1][2] * c2 - a[1][3] * c1) * id, (a[0][0] * c5 - a[0][2] * c2 + a[0][3] * c1) * id,
                       (-a[3][0] * s5 + a[3][2] * s2 - a[3][3] * s1) * id, (a[2][0] * s5 - a[2][2] * s2 + a[2][3] * s1) * id},
                      {(a[1][0] * c4 - a[1][1] * c2 + a[1][3] * c0) * id, (-a[0][0] * c4 + a[0][1] * c2 - a[0][3] * c0) * id,
                       (a[3][0] * s4 - a[3][1] * s2 + a[3][3] * s0) * id, (-a[2][0] * s4 + a[2][1] * s2 - a[2][3] * s0) * id},
                      {(-a[1][0] * c3 + a[1][1] * c1 - a[1][2] * c0) * id, (a[0][0] * c3 - a[0][1] * c1 + a[0][2] * c0) * id,
                       (-a[3][0] * s3 + a[3][1] * s1 - a[3][2] * s0) * id, (a[2][0] * s3 - a[2][1] * s1 + a[2][2] * s0) * id}};
    for (int i = 0; i < 4; i++)
    {
        r[i] = 0;
        for (int j = 0; j < 4; j++)
            r[i] += m[i][j] * b[j];
    }
}

/* fdtd.cu:162-232 split-field PML */
#define DEFINE_PML(R, SUFFIX)                                                                                           \
    static R damp_##SUFFIX(const orc_scene *s, int x, int y, int z)                                                     \
    {                                                                                                                    \
        int w = s->pml, res = s->res;                                                                                    \
        return (x < w || x >= res - w || y < w || y >= res - w || z < w || z >= res - w) ? (R)(2.0f / s->dl) : (R)0;   \
    }                                                                                                                    \
    static void pml_##SUFFIX(orc_scene *s, const R *cur, const R *prev, R *next)                                        \
    {                                                                                                                    \
        int res = s->res, t = s->t;                                                                                      \
        const R *pc = (const R *)s->pmlg[slot(t)];                                                                       \
        R *pn = (R *)s->pmlg[slot(t + 1)];                                                                               \
        R c = s->c, h = s->dl, dt = s->dt;                                                                               \
        _Pragma("omp parallel for schedule(static)") for (int x = 1; x <= res - 2; x++) for (int y = 1; y <= res - 2;  \
                                                                                              y++) for (int z = 1;      \
                                                                                                        z <= res - 2;    \
                                                                                                        z++)             \
        {                                                                                                                \
            int q[3] = {x, y, z}, sg[3];                                                                                 \
            for (int d = 0; d < 3; d++)                                                                                  \
                sg[d] = q[d] > res / 2 ? 1 : -1;                                                                         \
            long long ci = lin(res, x, y, z);                                                                            \
            R cdmp = damp_##SUFFIX(s, x, y, z), rhs = 0;                                                                 \
            for (int d = 0; d < 3; d++)                                                                                  \
            {                                                                                                            \
                int p1[3] = {x, y, z}, m1[3] = {x, y, z}, ps[3] = {x, y, z}, ms[3] = {x, y, z};                           \
                p1[d]++;                                                                                                 \
                m1[d]--;                                                                                                 \
                ps[d] += sg[d];                                                                                          \
                ms[d] -= sg[d];                                                                                          \
                rhs += 1 / (h * h) * (cur[lin(res, p1[0], p1[1], p1[2])] - 2 * cur[ci] + cur[lin(res, m1[0], m1[1], m1[2])]); \
                rhs += 1 / h * (cdmp * pc[6 * lin(res, ps[0], ps[1], ps[2]) + 3 + d] -                                  \
                                damp_##SUFFIX(s, ms[0], ms[1], ms[2]) * pc[6 * lin(res, ms[0], ms[1], ms[2]) + d]);      \
            }                                                                                                            \
            next[ci] = cur[ci] * 2 - prev[ci] + c * c * dt * dt * rhs;                                                   \
            if (cdmp == 0)                                                                                               \
                continue;                                                                                                \
            for (int d = 0; d < 3; d++)                                                                                  \
            {                                                                                                            \
                int ps[3] = {x, y, z}, ms[3] = {x, y, z};                                                                \
                ps[d] += sg[d];                                                                                          \
                ms[d] -= sg[d];                                                                                          \
                long long pi = lin(res, ps[0], ps[1], ps[2]), mi = lin(res, ms[0], ms[1], ms[2]);                        \
                R dm = damp_##SUFFIX(s, ms[0], ms[1], ms[2]), grad = cur[pi] - cur[mi];                                  \
                R r1 = 0;                                                                                                \
                r1 += -1.0f / 2.0f * (dm * pc[6 * mi + d] + cdmp * pc[6 * ci + d]);                                      \
                r1 += -1.0f / (h * 2.0f) * grad;                                                                         \
                pn[6 * ci + d] = pc[6 * ci + d] + c * dt * r1;                                                           \
                R r2 = 0;                                                                                                \
                r2 += -1.0f / 2.0f * (dm * pc[6 * ci + 3 + d] + cdmp * pc[6 * pi + 3 + d]);                              \
                r2 += -1.0f / (h * 2.0f) * grad;                                                                         \
                pn[6 * ci + 3 + d] = pc[6 * ci + 3 + d] + c * dt * r2;                                                   \
            }                                                                                                            \
        }                                                                                                                \
    }

DEFINE_PML(float, f)
DEFINE_PML(double, d)
DEFINE_STEP(float, f)
DEFINE_STEP(double, d)

int orc_step(orc_scene *s, const float *acc, int nsteps, const int *listen_xyz, int nlisten, float *out)
{
    if (!s || nsteps < 0 || (s->mesh_set && !acc))
        return 1;
    float *wgc_f = NULL, *wface_f = NULL;
    if (s->mesh_set && s->prec == ORC_F32)
    {
        wgc_f = (float *)malloc(sizeof(float) * (size_t)s->nt * 54 * 32);
        wface_f = (float *)malloc(sizeof(float) * (size_t)(s->pool_n + 1) * 32);
        for (size_t r = 0; r < (size_t)s->nt * 54; r++)
            unpack(&s->gc_r[r], wgc_f + r * 32);
        for (long long r = 0; r < s->pool_n; r++)
            unpack(&s->pool_r[r], wface_f + r * 32);
    }
    for (int st = 0; st < nsteps; st++)
    {
        const float *a = s->mesh_set ? acc + (size_t)st * s->nt : NULL;
        if (s->prec == ORC_F64)
            step_d(s, a, s->gc_w, s->pool_w);
        else
            step_f(s, a, wgc_f, wface_f);
        for (int l = 0; l < nlisten; l++)
        {
            long long c = lin(s->res, listen_xyz[3 * l], listen_xyz[3 * l + 1], listen_xyz[3 * l + 2]);
            out[(size_t)st * nlisten + l] = s->prec == ORC_F64 ? (float)((double *)s->grid[slot(s->t)])[c]
                                                               : ((float *)s->grid[slot(s->t)])[c];
        }
    }
    free(wgc_f);
    free(wface_f);
    return 0;
}

int orc_time(orc_scene *s) { return s ? s->t : -1000; }
int orc_set_time(orc_scene *s, int t)
{
    if (!s)
        return 1;
    s->t = t;
    return 0;
}

int orc_read_grid(orc_scene *s, int rel, void *out)
{
    if (!s || rel > 0 || rel < -2)
        return 1;
    memcpy(out, s->grid[slot(s->t + rel)], s->ncell * (s->prec == ORC_F64 ? 8 : 4));
    return 0;
}
int orc_write_grid(orc_scene *s, int rel, const void *in)
{
    if (!s || rel > 0 || rel < -2)
        return 1;
    memcpy(s->grid[slot(s->t + rel)], in, s->ncell * (s->prec == ORC_F64 ? 8 : 4));
    return 0;
}
int orc_read_history(orc_scene *s, void *n, void *d)
{
    if (!s || !s->mesh_set)
        return 5;
    size_t b = (size_t)s->nt * RING * (s->prec == ORC_F64 ? 8 : 4);
    memcpy(n, s->neumann, b);
    memcpy(d, s->dirichlet, b);
    return 0;
}
int orc_write_history(orc_scene *s, const void *n, const void *d)
{
    if (!s || !s->mesh_set)
        return 5;
    size_t b = (size_t)s->nt * RING * (s->prec == ORC_F64 ? 8 : 4);
    memcpy(s->neumann, n, b);
    memcpy(s->dirichlet, d, b);
    return 0;
}

int orc_counts(orc_scene *s, int *o)
{
    if (!s || !s->mesh_set)
        return 5;
    o[0] = s->n3;
    o[1] = s->n3_start[s->n3];
    o[2] = s->b4;
    o[3] = s->b4_start[s->b4];
    o[4] = (int)s->pf;
    return 0;
}

int orc_lists(orc_scene *s, int *n3_cells, int *p3_tris, int *b4_cells, int *p4_tris, int *cell_counts)
{
    if (!s || !s->mesh_set)
        return 5;
    int res = s->res;
    for (int i = 0; i < s->n3; i++)
    {
        int c = s->n3_cell[i];
        n3_cells[4 * i] = c / (res * res);
        n3_cells[4 * i + 1] = (c / res) % res;
        n3_cells[4 * i + 2] = c % res;
        n3_cells[4 * i + 3] = s->n3_start[i + 1] - s->n3_start[i];
    }
    memcpy(p3_tris, s->p3_tri, sizeof(int) * s->n3_start[s->n3]);
    for (int i = 0; i < s->b4; i++)
    {
        int c = s->b4_cell[i];
        b4_cells[4 * i] = c / (res * res);
        b4_cells[4 * i + 1] = (c / res) % res;
        b4_cells[4 * i + 2] = c % res;
        b4_cells[4 * i + 3] = s->base_start[c + 1] - s->base_start[c];
    }
    memcpy(p4_tris, s->n4_tris, sizeof(int) * s->b4_start[s->b4]);
    for (long long c = 0; c < s->ncell; c++)
        cell_counts[c] = s->cell_start[c + 1] - s->cell_start[c];
    return 0;
}

int orc_face_pairs(orc_scene *s, int *pairs)
{
    if (!s || !s->mesh_set)
        return 5;
    for (int i = 0; i < s->nt; i++)
        for (int p = s->face_start[i]; p < s->face_start[i + 1]; p++)
        {
            pairs[2 * p] = i;
            pairs[2 * p + 1] = s->face_nbr[p];
        }
    return 0;
}

int orc_triangles(orc_scene *s, float *geom, int *cells)
{
    if (!s || !s->mesh_set)
        return 5;
    for (int i = 0; i < s->nt; i++)
    {
        for (int q = 0; q < 3; q++)
        {
            geom[7 * i + q] = s->center[3 * i + q];
            geom[7 * i + 3 + q] = s->normal[3 * i + q];
            cells[6 * i + q] = s->cellc[3 * i + q];
            cells[6 * i + 3 + q] = s->basec[3 * i + q];
        }
        geom[7 * i + 6] = s->area[i];
    }
    return 0;
}

int orc_interp(orc_scene *s, float *out)
{
    if (!s || !s->mesh_set)
        return 5;
    memcpy(out, s->interp, sizeof(float) * 8 * s->nt);
    return 0;
}

int orc_grid_weights(orc_scene *s, double *out)
{
    if (!s || !s->mesh_set)
        return 5;
    memcpy(out, s->gc_w, sizeof(double) * (size_t)s->nt * 54 * 32);
    return 0;
}

int orc_face_weights(orc_scene *s, double *out)
{
    if (!s || !s->mesh_set)
        return 5;
    for (long long p = 0; p < s->pf; p++)
        memcpy(out + p * 32, s->pool_w + (size_t)s->face_slot[p] * 32, sizeof(double) * 32);
    return 0;
}

int orc_grid_records(orc_scene *s, void *out)
{
    if (!s || !s->mesh_set)
        return 5;
    memcpy(out, s->gc_r, sizeof(rec72) * (size_t)s->nt * 54);
    return 0;
}

int orc_face_records(orc_scene *s, void *out)
{
    if (!s || !s->mesh_set)
        return 5;
    rec72 *o = (rec72 *)out;
    for (long long p = 0; p < s->pf; p++)
        o[p] = s->pool_r[s->face_slot[p]];
    return 0;
}

/* trilinear face weights (nt x 8) taken from elsewhere, e.g. the reference's own */
int orc_import_interp(orc_scene *s, const float *w)
{
    if (!s || !s->mesh_set)
        return 5;
    for (int i = 0; i < 8 * s->nt; i++)
    {
        s->interp[i] = w[i];
        s->interp_d[i] = w[i];
    }
    return 0;
}

int orc_import_grid_cache(orc_scene *s, const void *records)
{
    if (!s || !s->mesh_set || s->prec != ORC_F32)
        return 5;
    memcpy(s->gc_r, records, sizeof(rec72) * (size_t)s->nt * 54);
    return 0;
}

int orc_import_face_cache(orc_scene *s, const int *pairs, const void *records, int n)
{
    if (!s || !s->mesh_set || s->prec != ORC_F32)
        return 5;
    const rec72 *r = (const rec72 *)records;
    for (int i = 0; i < n; i++)
    {
        int c = pairs[2 * i], j = pairs[2 * i + 1], found = -1;
        for (int p = s->face_start[c]; p < s->face_start[c + 1]; p++)
            if (s->face_nbr[p] == j)
            {
                found = s->face_slot[p];
                break;
            }
        if (found < 0)
            return 1;
        s->pool_r[found] = r[i];
    }
    denominators(s);
    return 0;
}

/* ----------------------------------------------------------------- labels -------- */
/* Eberly's closest point on a triangle (Geometric Tools "Distance from a Point to a
 * Triangle"), same branch structure as core/helper_math.h:1634-1786 */
static void min_edge02(float a11, float b1, float *q)
{
    int a = b1 < 0, b = a11 + b1 <= 0;
    q[0] = 0.0f;
    q[1] = a * (b - (1 - b) * (b1 / a11));
}
static void min_edge12(float a01, float a11, float b1, float f10, float f01, float *q)
{
    float h0 = a01 + b1 - f10, h1 = a11 + b1 - f01;
    int a = h0 < 0, b = h1 <= 0;
    float y = a * (b + (1 - b) * h0 / (h0 - h1));
    q[0] = 1 - y;
    q[1] = y;
}
static void min_interior(const float *p0, float h0, const float *p1, float h1, float *q)
{
    float z = h0 / (h0 - h1), omz = 1 - z;
    q[0] = omz * p0[0] + z * p1[0];
    q[1] = omz * p0[1] + z * p1[1];
}
static void nearest_coeff(const float *p, const float *v0, const float *v1, const float *v2, float *co)
{
    float diff[3], e0[3], e1[3];
    for (int k = 0; k < 3; k++)
    {
        diff[k] = p[k] - v0[k];
        e0[k] = v1[k] - v0[k];
        e1[k] = v2[k] - v0[k];
    }
    float a00 = e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2], a01 = e0[0] * e1[0] + e0[1] * e1[1] + e0[2] * e1[2];
    float a11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
    float b0 = -(diff[0] * e0[0] + diff[1] * e0[1] + diff[2] * e0[2]);
    float b1 = -(diff[0] * e1[0] + diff[1] * e1[1] + diff[2] * e1[2]);
    float f00 = b0, f10 = b0 + a00, f01 = b0 + a01;
    float p0[2] = {0, 0}, p1[2] = {0, 0}, q[2] = {0, 0}, dt1, h0, h1;
    if (f00 >= 0)
    {
        if (f01 >= 0)
            min_edge02(a11, b1, q);
        else
        {
            p0[0] = 0;
            p0[1] = f00 / (f00 - f01);
            p1[0] = f01 / (f01 - f10);
            p1[1] = 1 - p1[0];
            dt1 = p1[1] - p0[1];
            h0 = dt1 * (a11 * p0[1] + b1);
            if (h0 >= 0)
                min_edge02(a11, b1, q);
            else
            {
                h1 = dt1 * (a01 * p1[0] + a11 * p1[1] + b1);
                if (h1 <= 0)
                    min_edge12(a01, a11, b1, f10, f01, q);
                else
                    min_interior(p0, h0, p1, h1, q);
            }
        }
    }
    else if (f01 <= 0)
    {
        if (f10 <= 0)
            min_edge12(a01, a11, b1, f10, f01, q);
        else
        {
            p0[0] = f00 / (f00 - f10);
            p0[1] = 0;
            p1[0] = f01 / (f01 - f10);
            p1[1] = 1 - p1[0];
            h0 = p1[1] * (a01 * p0[0] + b1);
            if (h0 >= 0)
            {
                q[0] = p0[0];
                q[1] = p0[1];
            }
            else
            {
                h1 = p1[1] * (a01 * p1[0] + a11 * p1[1] + b1);
                if (h1 <= 0)
                    min_edge12(a01, a11, b1, f10, f01, q);
                else
                    min_interior(p0, h0, p1, h1, q);
            }
        }
    }
    else if (f10 <= 0)
    {
        p0[0] = 0;
        p0[1] = f00 / (f00 - f01);
        p1[0] = f01 / (f01 - f10);
        p1[1] = 1 - p1[0];
        dt1 = p1[1] - p0[1];
        h0 = dt1 * (a11 * p0[1] + b1);
        if (h0 >= 0)
            min_edge02(a11, b1, q);
        else
        {
            h1 = dt1 * (a01 * p1[0] + a11 * p1[1] + b1);
            if (h1 <= 0)
                min_edge12(a01, a11, b1, f10, f01, q);
            else
                min_interior(p0, h0, p1, h1, q);
        }
    }
    else
    {
        p0[0] = f00 / (f00 - f10);
        p0[1] = 0;
        p1[0] = 0;
        p1[1] = f00 / (f00 - f01);
        h0 = p1[1] * (a01 * p0[0] + b1);
        if (h0 >= 0)
        {
            q[0] = p0[0];
            q[1] = p0[1];
        }
        else
        {
            h1 = p1[1] * (a11 * p1[1] + b1);
            if (h1 <= 0)
                min_edge02(a11, b1, q);
            else
                min_interior(p0, h0, p1, h1, q);
        }
    }
    co[0] = 1 - q[0] - q[1];
    co[1] = q[0];
    co[2] = q[1];
}

/* ghost_cell_util.cu:7-230 */
int orc_classify(orc_scene *s, int *type, int *nearest, int *ghost, float *points, int *ghost_count)
{
    if (!s || !s->mesh_set)
        return 5;
    int res = s->res;
    long long n = s->ncell;
    if (!s->type)
    {
        s->type = (int *)xcalloc(n, sizeof(int));
        s->type_old = (int *)xcalloc(n, sizeof(int));
        s->nearest = (int *)xcalloc(n, sizeof(int));
        s->ghost = (int *)xcalloc(n, sizeof(int));
        s->points = (float *)xcalloc(7 * n, sizeof(float));
    }
    memcpy(s->type_old, s->type, sizeof(int) * n);
    /* vertex -> faces, ascending */
    int *vs = (int *)xcalloc(s->nv + 1, sizeof(int)), *vl = (int *)xcalloc(3 * s->nt, sizeof(int));
    int *key = (int *)xcalloc(3 * s->nt, sizeof(int)), *fid = (int *)xcalloc(3 * s->nt, sizeof(int));
    for (int i = 0; i < s->nt; i++)
        for (int k = 0; k < 3; k++)
            vs[s->F[3 * i + k] + 1]++;
    for (int v = 0; v < s->nv; v++)
        vs[v + 1] += vs[v];
    int *cur = (int *)xcalloc(s->nv, sizeof(int));
    for (int i = 0; i < s->nt; i++)
        for (int k = 0; k < 3; k++)
        {
            int v = s->F[3 * i + k];
            vl[vs[v] + cur[v]++] = i;
        }
    free(cur);
    free(key);
    free(fid);
    int *raw = (int *)xcalloc(n, sizeof(int));
#pragma omp parallel for schedule(dynamic, 256)
    for (long long i = 0; i < n; i++)
    {
        int x = (int)(i / ((long long)res * res)), y = (int)((i / res) % res), z = (int)(i % res);
        float gc[3];
        cell_center_f(s, x, y, z, gc);
        float best = 3.402823466e+38F, bp[3] = {0, 0, 0}, bco[3] = {0, 0, 0};
        int bi = -1;
        for (int dx = -3; dx <= 3; dx++)
            for (int dy = -3; dy <= 3; dy++)
                for (int dz = -3; dz <= 3; dz++)
                {
                    int cx = x + dx, cy = y + dy, cz = z + dz;
                    if (cx < 0 || cy < 0 || cz < 0 || cx >= res || cy >= res || cz >= res)
                        continue;
                    long long c = lin(res, cx, cy, cz);
                    for (int j = s->cell_start[c]; j < s->cell_start[c + 1]; j++)
                    {
                        int f = s->cell_tris[j];
                        const float *v0 = s->V + 3 * s->F[3 * f], *v1 = s->V + 3 * s->F[3 * f + 1],
                                    *v2 = s->V + 3 * s->F[3 * f + 2];
                        float co[3], np[3];
                        nearest_coeff(gc, v0, v1, v2, co);
                        for (int q = 0; q < 3; q++)
                            np[q] = co[0] * v0[q] + co[1] * v1[q] + co[2] * v2[q];
                        float d0 = gc[0] - np[0], d1 = gc[1] - np[1], d2 = gc[2] - np[2];
                        float l = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
                        if (l < best)
                        {
                            best = l;
                            bi = f;
                            memcpy(bp, np, sizeof(bp));
                            memcpy(bco, co, sizeof(bco));
                        }
                    }
                }
        int ty = 3;
        float refl[3] = {0, 0, 0};
        if (bi >= 0)
        {
            float nn[3] = {0, 0, 0};
            for (int k = 0; k < 3; k++)
            {
                refl[k] = 2 * bp[k] - gc[k];
                int v = s->F[3 * bi + k];
                float acc[3] = {0, 0, 0};
                for (int j = vs[v]; j < vs[v + 1]; j++)
                {
                    int f = vl[j], o[2], m = 0;
                    for (int q = 0; q < 3; q++)
                        if (s->F[3 * f + q] != v && m < 2)
                            o[m++] = s->F[3 * f + q];
                    float e1[3], e2[3];
                    for (int q = 0; q < 3; q++)
                    {
                        e1[q] = s->V[3 * o[0] + q] - s->V[3 * v + q];
                        e2[q] = s->V[3 * o[1] + q] - s->V[3 * v + q];
                    }
                    float l1 = sqrtf(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
                    float l2 = sqrtf(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
                    float ang = acosf((e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2]) / (l1 * l2));
                    for (int q = 0; q < 3; q++)
                        acc[q] += s->normal[3 * f + q] * ang;
                }
                float l = sqrtf(acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2]);
                for (int q = 0; q < 3; q++)
                    nn[q] += bco[k] * (acc[q] / l);
            }
            float dir = nn[0] * (gc[0] - bp[0]) + nn[1] * (gc[1] - bp[1]) + nn[2] * (gc[2] - bp[2]);
            ty = dir <= 0 ? 1 : 0;
        }
        raw[i] = ty;
        s->nearest[i] = bi;
        float *pt = s->points + 7 * i;
        pt[0] = bp[0];
        pt[1] = bp[1];
        pt[2] = bp[2];
        pt[3] = refl[0];
        pt[4] = refl[1];
        pt[5] = refl[2];
        pt[6] = bi >= 0 ? best : 3.402823466e+38F;
    }
    free(vs);
    free(vl);
    int *flag = (int *)xcalloc(n, sizeof(int));
    for (long long i = 0; i < n; i++)
    {
        int x = (int)(i / ((long long)res * res)), y = (int)((i / res) % res), z = (int)(i % res);
        int ty = raw[i];
        if (ty == 1)
        {
            int nb[6][3] = {{x + 1, y, z}, {x - 1, y, z}, {x, y + 1, z}, {x, y - 1, z}, {x, y, z + 1}, {x, y, z - 1}};
            for (int k = 0; k < 6; k++)
            {
                if (nb[k][0] < 0 || nb[k][0] >= res || nb[k][1] < 0 || nb[k][1] >= res || nb[k][2] < 0 || nb[k][2] >= res)
                    continue;
                if (raw[lin(res, nb[k][0], nb[k][1], nb[k][2])] == 0)
                    ty = 2;
            }
        }
        s->type[i] = ty;
        flag[i] = ty == 2;
    }
    free(raw);
    for (int col = 0; col < res * res; col++)
    {
        int *t = s->type + (long long)col * res, curt = 0, found = 0;
        for (int z = 0; z < res; z++)
        {
            if (!found && t[z] != 3)
            {
                found = 1;
                curt = t[z];
                for (int k = 0; k < z; k++)
                    t[k] = curt;
                continue;
            }
            if (t[z] == 1 || t[z] == 2)
                curt = 1;
            else if (t[z] == 0)
                curt = 0;
            else
                t[z] = curt;
        }
    }
    int run = 0;
    for (long long i = 0; i < n; i++)
    {
        run += flag[i];
        s->ghost[i] = s->type[i] == 2 ? run - 1 : -1;
    }
    free(flag);
    if (ghost_count)
        *ghost_count = run;
    if (type)
        memcpy(type, s->type, sizeof(int) * n);
    if (nearest)
        memcpy(nearest, s->nearest, sizeof(int) * n);
    if (ghost)
        memcpy(ghost, s->ghost, sizeof(int) * n);
    if (points)
        memcpy(points, s->points, sizeof(float) * 7 * n);
    return 0;
}

/* ghost_cell.cu:51-205 on grid slots t and t-1 (FP32 scenes) */
int orc_fresh(orc_scene *s, const float *acc, const float *acc_old, int *fresh_count)
{
    if (!s || !s->type || s->prec != ORC_F32)
        return 5;
    int res = s->res, cnt = 0;
    float *gs[2] = {(float *)s->grid[slot(s->t)], (float *)s->grid[slot(s->t - 1)]};
    for (long long c = 0; c < s->ncell; c++)
    {
        if (!(s->type_old[c] != 0 && s->type[c] == 0))
            continue;
        cnt++;
        int x = (int)(c / ((long long)res * res)), y = (int)((c / res) % res), z = (int)(c % res);
        int nf = s->nearest[c];
        float accs[2] = {acc[nf], acc_old[nf]};
        float xb[3] = {s->points[7 * c], s->points[7 * c + 1], s->points[7 * c + 2]}, xf[3], xr[3];
        cell_center_f(s, x, y, z, xf);
        int b[3];
        for (int q = 0; q < 3; q++)
        {
            xr[q] = xb[q] + 2 * (xf[q] - xb[q]);
            int g = (int)((xr[q] - s->mn[q]) / s->dl);
            float cc = (g + 0.5f) * s->dl + s->mn[q];
            b[q] = g - (xr[q] - cc < 0);
        }
        long long nb[8];
        float co[8];
        int found = 0;
        for (int w = 0; w < 8; w++)
        {
            int a0 = b[0] + (w >> 2), a1 = b[1] + ((w >> 1) & 1), a2 = b[2] + (w & 1);
            nb[w] = -1;
            co[w] = 0;
            if (a0 < 0 || a1 < 0 || a2 < 0 || a0 >= res || a1 >= res || a2 >= res)
                continue;
            nb[w] = lin(res, a0, a1, a2);
            if (s->type_old[nb[w]] == 0 && s->type[nb[w]] == 0)
            {
                float cc[3];
                cell_center_f(s, a0, a1, a2, cc);
                float d0 = cc[0] - xr[0], d1 = cc[1] - xr[1], d2 = cc[2] - xr[2];
                float dist = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
                co[w] = (float)(1.0 / (dist * dist + 1e-8f));
                found = 1;
            }
        }
        float df[3] = {xf[0] - xr[0], xf[1] - xr[1], xf[2] - xr[2]};
        float lfr = sqrtf(df[0] * df[0] + df[1] * df[1] + df[2] * df[2]);
        if (!found)
        {
            float md = 1e10f, pr1 = 0, pr2 = 0;
            for (int dx = -1; dx < 3; dx++)
                for (int dy = -1; dy < 3; dy++)
                    for (int dz = -1; dz < 3; dz++)
                    {
                        int a0 = b[0] + dx, a1 = b[1] + dy, a2 = b[2] + dz;
                        if (a0 < 0 || a1 < 0 || a2 < 0 || a0 >= res || a1 >= res || a2 >= res)
                            continue;
                        long long q = lin(res, a0, a1, a2);
                        if (!(s->type_old[q] == 0 && s->type[q] == 0))
                            continue;
                        float cc[3];
                        cell_center_f(s, a0, a1, a2, cc);
                        float d0 = cc[0] - xr[0], d1 = cc[1] - xr[1], d2 = cc[2] - xr[2];
                        float dist = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
                        if (dist < md)
                        {
                            md = dist;
                            pr1 = gs[0][q];
                            pr2 = gs[1][q];
                        }
                    }
            gs[0][c] = pr1;
            gs[1][c] = pr2;
            continue;
        }
        float sum = 0;
        for (int w = 0; w < 8; w++)
            sum += co[w];
        for (int w = 0; w < 8; w++)
            co[w] /= sum;
        for (int k = 0; k < 2; k++)
        {
            float pr = 0;
            for (int w = 0; w < 8; w++)
                if (nb[w] >= 0)
                    pr += co[w] * gs[k][nb[w]];
            gs[k][c] = pr - 1.225f * accs[k] * lfr;
        }
    }
    if (fresh_count)
        *fresh_count = cnt;
    return 0;
}
