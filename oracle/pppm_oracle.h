/*
 * pppm_oracle.h - CPU restatement of the PPPM-TDBEM per-step hot path (TEST INFRASTRUCTURE).
 *
 * This library is the checker the parity tests compare libpppm_b200 against, and the timed
 * CPU baseline of bench.py.  It is never linked into the product.  Each function follows
 * the reference file:line cited at its definition in pppm_oracle.c.  Two precisions:
 *   ORC_F32  FP32 storage with the reference's arithmetic (double interior stencil, float
 *            boundary solve and convolutions, fp16+scale weight records)
 *   ORC_F64  the same scheme in double with unquantised weights
 * Weights are evaluated in double (integrals, FFT) and, for ORC_F32, packed to fp16 rows
 * with a max-abs scale like the reference; tables can also be imported (records of 72 bytes
 * in the reference layout).  The per-step loops are parallelised with OpenMP.
 */
#ifndef PPPM_ORACLE_H
#define PPPM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define ORC_F32 0
#define ORC_F64 1

typedef struct orc_scene orc_scene;

orc_scene *orc_create(int res, float dl, float dt, const float *min_pos, float reflect_coeff, float c, int pml_width,
                      int precision);
void orc_destroy(orc_scene *s);
int orc_set_mesh(orc_scene *s, const float *V, int nv, const int *F, int nt);
int orc_set_mesh_cells(orc_scene *s, const float *V, int nv, const int *F, int nt, const int *cells6);
int orc_update_mesh(orc_scene *s, const float *V);
int orc_step(orc_scene *s, const float *acc, int nsteps, const int *listen_xyz, int nlisten, float *out);
int orc_time(orc_scene *s);
int orc_set_time(orc_scene *s, int t);
/* grid slot t+rel (rel 0,-1,-2) as float or double (per precision) */
int orc_read_grid(orc_scene *s, int rel, void *out);
int orc_write_grid(orc_scene *s, int rel, const void *in);
int orc_read_history(orc_scene *s, void *neumann, void *dirichlet);
int orc_write_history(orc_scene *s, const void *neumann, const void *dirichlet);
/* counts: n3, p3, b4, p4, pf */
int orc_counts(orc_scene *s, int *out5);
int orc_lists(orc_scene *s, int *n3_cells, int *p3_tris, int *b4_cells, int *p4_tris, int *cell_counts);
int orc_face_pairs(orc_scene *s, int *pairs);
int orc_triangles(orc_scene *s, float *geom, int *cells);
int orc_interp(orc_scene *s, float *out);
/* weights in double before packing: grid nt x 54 x 32 (single 16, double 16); face pf x 32 */
int orc_grid_weights(orc_scene *s, double *out);
int orc_face_weights(orc_scene *s, double *out);
/* packed fp16 records (72 bytes, reference layout) */
int orc_grid_records(orc_scene *s, void *out);
int orc_face_records(orc_scene *s, void *out);
int orc_import_grid_cache(orc_scene *s, const void *records);
int orc_import_interp(orc_scene *s, const float *w);
int orc_import_face_cache(orc_scene *s, const int *pairs, const void *records, int n);
/* single pair weights (double): src triangle onto a point or a face */
int orc_laplace_weight(float dt, float dl, float c, const float *V, const int *src, int to_point, const int *dst_face,
                       const float *dst_point, double *out32);
/* frequency-domain pair integral at complex wave number k: single (re, im), double (re, im) */
int orc_pair_integral(float dl, const float *V, const int *src, int to_point, const int *dst_face,
                      const float *dst_point, double k_re, double k_im, double *out4);
/* cell labels: type, nearest, ghost index, points (nearest xyz, reflect xyz, distance) */
int orc_classify(orc_scene *s, int *type, int *nearest, int *ghost, float *points, int *ghost_count);
int orc_fresh(orc_scene *s, const float *acc, const float *acc_old, int *fresh_count);
int orc_threads(void);

#ifdef __cplusplus
}
#endif
#endif
