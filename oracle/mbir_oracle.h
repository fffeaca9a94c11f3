/*
 * CPU restatement of TIMBIR's 3D/4D MBIR ICD/NHICD hot path -- the ORACLE.
 *
 * Test infrastructure only.  This library is the checker that the CUDA path in
 * timbir_b200/ is compared against; it is never linked into, loaded by or
 * called from the product.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py use it.
 *
 * It restates, in plain single-threaded C, the reference's set-up, voxel
 * update, cost, ring-offset, variance, NHICD selection, random line order and
 * multi-resolution driver (reference: TIMBIR v0.0.2, src/MBIR_4D).  Each
 * function in mbir_oracle.c cites the reference lines it follows.  With
 * float arrays (liboracle.so) the operation order matches the reference
 * run single-threaded, so its results agree with the reference bit for bit
 * or to float rounding; with double arrays (liboracle64.so, -DORACLE_F64) it
 * is the FP64 oracle used for RMSE statements.
 *
 * Parity pin: tests/test_oracle_pin.py checks it against the reference library
 * built from its own sources (oracle/_ref, via oracle/Makefile) and against the
 * golden fixtures in tests/golden/, which were produced by that build; the
 * Park-Miller known-answer table of src/MBIR_4D/randlib.c:69-90 pins the RNG.
 */
#ifndef MBIR_ORACLE_H
#define MBIR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void *orc_create(const float *projections, const float *weights, const float *angles,
                 const float *proj_times, const float *recon_times, int proj_rows, int proj_cols,
                 int proj_num, int recon_num, float vox_wid, float rot_center, float sig_s,
                 float sig_t, float c_s, float c_t, float convg_thresh, int remove_rings,
                 int quad_convex, float huber_delta, float huber_T, int mult_xy, int mult_z,
                 int num_z_blocks);
void orc_destroy(void *h);
void orc_set_switches(void *h, int update_proj_offset, int update_var, double var_est);
int orc_prepare(void *h, const float *object, const float *offset);
int orc_iterate(void *h, int iter);
double orc_cost(void *h, double *forward, double *prior, double *errsino);
void orc_offset_update(void *h);
void orc_build_offset_windows(void *h);
int orc_get_offset_windows(void *h, float *out);
void orc_variance_update(void *h);
void orc_random_select(void *h);
void orc_vsc_select(void *h);
void orc_dims(void *h, int *d);
void orc_scalars(void *h, double *s);
void orc_view_map(void *h, int frame, int *num, int *idx);
void orc_get_object(void *h, float *out);
void orc_get_errorsino(void *h, float *out);
void orc_get_weight(void *h, float *out);
void orc_get_projselect(void *h, uint8_t *out);
void orc_get_offset(void *h, float *out);
void orc_get_magmap(void *h, float *out);
void orc_set_magmap(void *h, const float *in);
void orc_get_hr(void *h, float *out);
void orc_get_mask(void *h, uint8_t *out);
int orc_get_lines(void *h, int kind, int frame, int block, int *xs, int *ys);
void orc_set_lines(void *h, int frame, int block, int n, const int *xs, const int *ys);
int orc_amatrix(void *h, int row, int col, int view, int *idx, double *val, int cap);
double orc_functional_substitution(void *h, double V, double theta1, double theta2,
                                   const double *spatial27, const uint8_t *sflag27,
                                   const double *time2, const uint8_t *tflag2);
double orc_var_est(void *h);
int orc_num_z_blocks(void *h);
double orc_last_update_percentage(void *h);
long long orc_update_count(void *h);

void orc_srandom2(uint32_t seed);
double orc_random2(void);
double orc_randomized_select(float *a, uint32_t n, uint32_t i);
int orc_z_blocks_for_threads(int threads, int n_time, int n_z);



#ifdef __cplusplus
}
#endif
#endif
