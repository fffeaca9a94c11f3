/*
 * Flat C entry points into the reference library (TIMBIR v0.0.2,
 * src/MBIR_4D), compiled together with the unmodified reference sources into
 * oracle/_ref/libmbir4d_ref.so.  Test infrastructure only: it lets the tests
 * drive the reference one step at a time (set-up, one ICD iteration, one
 * offset update, ...) and read its state back, so the CPU restatement in
 * oracle/mbir_oracle.c and the CUDA path can be pinned against the reference
 * itself.  Nothing here re-implements the algorithm; every numeric step below
 * is a call into the reference.
 *
 * The set-up sequence mirrors the stage prologue of ICD_BackProject
 * (src/MBIR_4D/XT_ICD_update.c:1108-1170): mask, detector response, object
 * initialisation, error sinogram.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <math.h>
#include <omp.h>
#include "XT_Structures.h"
#include "XT_Constants.h"
#include "XT_Init.h"
#include "XT_Profile.h"
#include "XT_AMatrix.h"
#include "XT_NHICD.h"
#include "XT_ICD_update.h"
#include "XT_OffsetError.h"
#include "randlib.h"
#include "allocate.h"

/* Global functions of the reference that its headers do not declare. */
int32_t initObject(Sinogram *, ScannedObject *, TomoInputs *, Real_arr_t ****);
int32_t initErrorSinogam(Sinogram *, ScannedObject *, TomoInputs *, Real_arr_t **, Real_arr_t ***);
Real_t computeCost(Sinogram *, ScannedObject *, TomoInputs *, Real_arr_t ***);
int updateVoxelsTimeSlices(Sinogram *, ScannedObject *, TomoInputs *, Real_arr_t **, Real_arr_t ***, int32_t, Real_arr_t ****, uint8_t ***);
void update_Sinogram_Offset(Sinogram *, TomoInputs *, Real_arr_t ***);
void update_variance_parameter(Sinogram *, TomoInputs *, Real_arr_t ***);
void randomly_select_x_y(ScannedObject *, TomoInputs *, uint8_t ***);

typedef struct {
	Sinogram *S;
	ScannedObject *O;
	TomoInputs *T;
	Real_arr_t ****mag;   /* [N_time][num_z_blocks][N_y][N_x] */
	Real_arr_t **H_r;     /* [N_p][65] */
	Real_arr_t *H_t;
	Real_arr_t ***e;      /* [N_p][N_r][N_t] */
	uint8_t ***mask;      /* [N_time][N_y][N_x] */
	int prepared;
} ref_ctx;

/* Runs initStatStructures + initDynStructures for one stage whose voxel
 * scales are (mult_xy, mult_z).  The stage is treated as the first one
 * (mult_idx 0), so the object starts from zero and the inputs are taken from
 * the arrays given here.  `threads` fixes omp_get_max_threads(), which decides
 * num_z_blocks (src/MBIR_4D/XT_Init.c:389-398).  The caller's arrays are
 * copied: the reference keeps pointers to the angle/time arrays and frees the
 * projections itself. */
void *ref_create(const float *projections, const float *weights, const float *angles,
                 const float *proj_times, const float *recon_times, int proj_rows, int proj_cols,
                 int proj_num, int recon_num, float vox_wid, float rot_center, float sig_s,
                 float sig_t, float c_s, float c_t, float convg_thresh, int remove_rings,
                 int quad_convex, float huber_delta, float huber_T, int mult_xy, int mult_z,
                 int threads, FILE *log)
{
	ref_ctx *c = (ref_ctx *)calloc(1, sizeof(ref_ctx));
	int32_t mxy[1], mz[1];
	size_t nsino = (size_t)proj_num * proj_rows * proj_cols;
	float *pa = (float *)malloc(sizeof(float) * proj_num);
	float *pt = (float *)malloc(sizeof(float) * proj_num);
	float *rt = (float *)malloc(sizeof(float) * (recon_num + 1));
	float *pr = (float *)malloc(sizeof(float) * nsino);
	float *wt = (float *)malloc(sizeof(float) * nsino);
	memcpy(pa, angles, sizeof(float) * proj_num);
	memcpy(pt, proj_times, sizeof(float) * proj_num);
	memcpy(rt, recon_times, sizeof(float) * (recon_num + 1));
	memcpy(pr, projections, sizeof(float) * nsino);
	memcpy(wt, weights, sizeof(float) * nsino);
	c->S = (Sinogram *)calloc(1, sizeof(Sinogram));
	c->O = (ScannedObject *)calloc(1, sizeof(ScannedObject));
	c->T = (TomoInputs *)calloc(1, sizeof(TomoInputs));
	c->T->debug_file_ptr = log ? log : stdout;
	if (threads > 0)
		omp_set_num_threads(threads);
	srandom2(761521);
	if (initStatStructures(c->S, c->O, c->T, pa, pt, rt, proj_rows, proj_cols, proj_num, recon_num,
	                       vox_wid, rot_center, sig_s, sig_t, c_s, c_t, convg_thresh, remove_rings,
	                       quad_convex, huber_delta, huber_T))
		return NULL;
	mxy[0] = mult_xy;
	mz[0] = mult_z;
	if (initDynStructures(c->S, c->O, c->T, 0, mxy, mz, pr, wt, remove_rings, quad_convex))
		return NULL;
	free(pr);
	free(wt);
	return c;
}

/* Overrides the per-stage switches that initDynStructures derives from the
 * stage index (src/MBIR_4D/XT_Init.c:236-266) and the variance estimate. */
void ref_set_switches(void *h, int update_proj_offset, int update_var, double var_est)
{
	ref_ctx *c = (ref_ctx *)h;
	int64_t i, n = (int64_t)c->S->N_p * c->S->N_r * c->S->N_t;
	Real_arr_t *w = &(c->T->Weight[0][0][0]);
	c->T->updateProjOffset = (uint8_t)update_proj_offset;
	c->T->updateVar = (uint8_t)update_var;
	if (var_est > 0 && var_est != c->T->var_est) {
		for (i = 0; i < n; i++)
			w[i] = (Real_arr_t)(w[i] * c->T->var_est);
		c->T->var_est = var_est;
		for (i = 0; i < n; i++)
			w[i] /= var_est;
	}
}

/* Stage prologue of ICD_BackProject (XT_ICD_update.c:1134-1159).  If `object`
 * is given ([N_time][N_z][N_y][N_x]) it replaces the zero initial object
 * before the error sinogram is formed; if `offset` is given ([N_r][N_t]) it
 * replaces the zero ring offsets. */
int ref_prepare(void *h, const float *object, const float *offset)
{
	ref_ctx *c = (ref_ctx *)h;
	Sinogram *S = c->S;
	ScannedObject *O = c->O;
	TomoInputs *T = c->T;
	int32_t i, j, k;
	double x, y;
	c->mag = (Real_arr_t ****)multialloc(sizeof(Real_arr_t), 4, O->N_time, T->num_z_blocks, O->N_y, O->N_x);
	c->H_r = (Real_arr_t **)multialloc(sizeof(Real_arr_t), 2, S->N_p, DETECTOR_RESPONSE_BINS + 1);
	c->H_t = (Real_arr_t *)get_spc(DETECTOR_RESPONSE_BINS + 1, sizeof(Real_arr_t));
	c->e = (Real_arr_t ***)multialloc(sizeof(Real_arr_t), 3, S->N_p, S->N_r, S->N_t);
	c->mask = (uint8_t ***)multialloc(sizeof(uint8_t), 3, O->N_time, O->N_y, O->N_x);
	memset(&(c->mag[0][0][0][0]), 0, sizeof(Real_arr_t) * O->N_time * T->num_z_blocks * O->N_y * O->N_x);
	for (i = 0; i < O->N_time; i++)
		for (j = 0; j < O->N_y; j++)
			for (k = 0; k < O->N_x; k++) {
				x = O->x0 + ((Real_t)k + 0.5) * O->delta_xy;
				y = O->y0 + ((Real_t)j + 0.5) * O->delta_xy;
				c->mask[i][j][k] = (x * x + y * y < T->radius_obj * T->radius_obj) ? 1 : 0;
			}
	DetectorResponseProfile(c->H_r, c->H_t, S, O, T);
	if (initObject(S, O, T, c->mag))
		return -1;
	if (object) {
		for (i = 0; i < O->N_time; i++)
			memcpy(&(O->Object[i][1][0][0]), object + (size_t)i * O->N_z * O->N_y * O->N_x,
			       sizeof(float) * O->N_z * O->N_y * O->N_x);
	}
	if (offset)
		memcpy(&(S->ProjOffset[0][0]), offset, sizeof(float) * S->N_r * S->N_t);
	if (initErrorSinogam(S, O, T, c->H_r, c->e))
		return -1;
	c->prepared = 1;
	return 0;
}

int ref_iterate(void *h, int iter)
{
	ref_ctx *c = (ref_ctx *)h;
	return updateVoxelsTimeSlices(c->S, c->O, c->T, c->H_r, c->e, iter, c->mag, c->mask);
}

double ref_cost(void *h)
{
	ref_ctx *c = (ref_ctx *)h;
	return computeCost(c->S, c->O, c->T, c->e);
}

/* Forward / prior parts of the last computeCost call (XT_ICD_update.c:308-312). */
void ref_cost_parts(void *h, double *forward, double *prior, double *errsino)
{
	ref_ctx *c = (ref_ctx *)h;
	*forward = c->T->Forward_Cost;
	*prior = c->T->Prior_Cost;
	*errsino = c->T->ErrorSino_Cost;
}

void ref_offset_update(void *h)
{
	ref_ctx *c = (ref_ctx *)h;
	update_Sinogram_Offset(c->S, c->T, c->e);
}

void ref_variance_update(void *h)
{
	ref_ctx *c = (ref_ctx *)h;
	update_variance_parameter(c->S, c->T, c->e);
}

void ref_random_select(void *h)
{
	ref_ctx *c = (ref_ctx *)h;
	randomly_select_x_y(c->O, c->T, c->mask);
}

void ref_vsc_select(void *h)
{
	ref_ctx *c = (ref_ctx *)h;
	VSC_based_Voxel_Line_Select(c->O, c->T, c->mag);
}

/* Dimensions: N_p, N_r, N_t, N_x, N_y, N_z, N_time, num_z_blocks, z_overlap_num */
void ref_dims(void *h, int *d)
{
	ref_ctx *c = (ref_ctx *)h;
	d[0] = c->S->N_p; d[1] = c->S->N_r; d[2] = c->S->N_t;
	d[3] = c->O->N_x; d[4] = c->O->N_y; d[5] = c->O->N_z;
	d[6] = c->O->N_time; d[7] = c->T->num_z_blocks; d[8] = c->S->z_overlap_num;
}

/* Scalars: delta_r, R0, RMax, OffsetR, x0, y0, delta_xy, radius_obj, Sigma_S_Q,
 * Sigma_S_Q_P, Sigma_T_Q, Sigma_T_Q_P, C_S, C_T, Time_Filter[0], var_est,
 * ErrorSinoThresh, ErrorSinoDelta, delta_recon, alpha, Spatial_Filter[27] */
void ref_scalars(void *h, double *s)
{
	ref_ctx *c = (ref_ctx *)h;
	int i, j, k;
	s[0] = c->S->delta_r; s[1] = c->S->R0; s[2] = c->S->RMax; s[3] = c->S->OffsetR;
	s[4] = c->O->x0; s[5] = c->O->y0; s[6] = c->O->delta_xy; s[7] = c->T->radius_obj;
	s[8] = c->T->Sigma_S_Q; s[9] = c->T->Sigma_S_Q_P; s[10] = c->T->Sigma_T_Q; s[11] = c->T->Sigma_T_Q_P;
	s[12] = c->O->C_S; s[13] = c->O->C_T; s[14] = c->T->Time_Filter[0]; s[15] = c->T->var_est;
	s[16] = c->T->ErrorSinoThresh; s[17] = c->T->ErrorSinoDelta; s[18] = c->O->delta_recon; s[19] = c->T->alpha;
	for (i = 0; i < 3; i++)
		for (j = 0; j < 3; j++)
			for (k = 0; k < 3; k++)
				s[20 + 9 * i + 3 * j + k] = c->T->Spatial_Filter[i][j][k];
}

void ref_view_map(void *h, int frame, int *num, int *idx)
{
	ref_ctx *c = (ref_ctx *)h;
	int i;
	*num = c->O->ProjNum[frame];
	if (idx)
		for (i = 0; i < *num; i++)
			idx[i] = c->O->ProjIdxPtr[frame][i];
}

void ref_get_object(void *h, float *out)
{
	ref_ctx *c = (ref_ctx *)h;
	int i;
	size_t n = (size_t)c->O->N_z * c->O->N_y * c->O->N_x;
	for (i = 0; i < c->O->N_time; i++)
		memcpy(out + i * n, &(c->O->Object[i][1][0][0]), sizeof(float) * n);
}

void ref_get_errorsino(void *h, float *out)
{
	ref_ctx *c = (ref_ctx *)h;
	memcpy(out, &(c->e[0][0][0]), sizeof(float) * (size_t)c->S->N_p * c->S->N_r * c->S->N_t);
}

void ref_get_weight(void *h, float *out)
{
	ref_ctx *c = (ref_ctx *)h;
	memcpy(out, &(c->T->Weight[0][0][0]), sizeof(float) * (size_t)c->S->N_p * c->S->N_r * c->S->N_t);
}

void ref_get_projselect(void *h, uint8_t *out)
{
	ref_ctx *c = (ref_ctx *)h;
	size_t i, n = (size_t)c->S->N_p * c->S->N_r * c->S->N_t;
	bool *b = &(c->S->ProjSelect[0][0][0]);
	for (i = 0; i < n; i++)
		out[i] = b[i] ? 1 : 0;
}

void ref_get_offset(void *h, float *out)
{
	ref_ctx *c = (ref_ctx *)h;
	memcpy(out, &(c->S->ProjOffset[0][0]), sizeof(float) * (size_t)c->S->N_r * c->S->N_t);
}

void ref_get_magmap(void *h, float *out)
{
	ref_ctx *c = (ref_ctx *)h;
	memcpy(out, &(c->mag[0][0][0][0]),
	       sizeof(float) * (size_t)c->O->N_time * c->T->num_z_blocks * c->O->N_y * c->O->N_x);
}

void ref_set_magmap(void *h, const float *in)
{
	ref_ctx *c = (ref_ctx *)h;
	memcpy(&(c->mag[0][0][0][0]), in,
	       sizeof(float) * (size_t)c->O->N_time * c->T->num_z_blocks * c->O->N_y * c->O->N_x);
}

void ref_get_hr(void *h, float *out)
{
	ref_ctx *c = (ref_ctx *)h;
	memcpy(out, &(c->H_r[0][0]), sizeof(float) * (size_t)c->S->N_p * (DETECTOR_RESPONSE_BINS + 1));
}

void ref_get_mask(void *h, uint8_t *out)
{
	ref_ctx *c = (ref_ctx *)h;
	memcpy(out, &(c->mask[0][0][0]), (size_t)c->O->N_time * c->O->N_y * c->O->N_x);
}

/* Line lists of one (frame, block): kind 0 = random HICD order
 * (x_rand_select/y_rand_select), kind 1 = NHICD selection. */
int ref_get_lines(void *h, int kind, int frame, int block, int *xs, int *ys)
{
	ref_ctx *c = (ref_ctx *)h;
	int i, n;
	if (kind == 0) {
		n = c->T->UpdateSelectNum[frame][block];
		for (i = 0; i < n; i++) {
			xs[i] = c->T->x_rand_select[frame][block][i];
			ys[i] = c->T->y_rand_select[frame][block][i];
		}
	} else {
		n = c->T->NHICDSelectNum[frame][block];
		for (i = 0; i < n; i++) {
			xs[i] = c->T->x_NHICD_select[frame][block][i];
			ys[i] = c->T->y_NHICD_select[frame][block][i];
		}
	}
	return n;
}

/* One A-matrix column (src/MBIR_4D/XT_AMatrix.c:50-110).  Needs ref_prepare
 * (for H_r).  Returns the count; idx/val have room for `cap` entries. */
int ref_amatrix(void *h, int row, int col, int view, int *idx, double *val, int cap)
{
	ref_ctx *c = (ref_ctx *)h;
	AMatrixCol A;
	int i, n;
	int32_t ibuf[256];
	Real_t vbuf[256];
	A.index = ibuf;
	A.values = vbuf;
	calcAMatrixColumnforAngle(c->S, c->O, c->H_r, &A, row, col, view);
	n = A.count;
	for (i = 0; i < n && i < cap; i++) {
		idx[i] = A.index[i];
		val[i] = A.values[i];
	}
	return n;
}

double ref_functional_substitution(void *h, double V, double theta1, double theta2,
                                   const double *spatial27, const uint8_t *sflag27,
                                   const double *time2, const uint8_t *tflag2)
{
	ref_ctx *c = (ref_ctx *)h;
	Real_t sn[3][3][3], tn[2];
	bool sf[3][3][3], tf[2];
	int i, j, k;
	for (i = 0; i < 3; i++)
		for (j = 0; j < 3; j++)
			for (k = 0; k < 3; k++) {
				sn[i][j][k] = spatial27[9 * i + 3 * j + k];
				sf[i][j][k] = sflag27[9 * i + 3 * j + k] ? true : false;
			}
	for (i = 0; i < 2; i++) {
		tn[i] = time2[i];
		tf[i] = tflag2[i] ? true : false;
	}
	return CE_FunctionalSubstitution(V, theta1, theta2, c->O, c->T, sn, tn, sf, tf);
}

double ref_var_est(void *h) { return ((ref_ctx *)h)->T->var_est; }
int ref_num_z_blocks(void *h) { return ((ref_ctx *)h)->T->num_z_blocks; }

void ref_srandom2(uint32_t seed) { srandom2(seed); }
double ref_random2(void) { return random2(); }

double ref_randomized_select(float *a, uint32_t n, uint32_t i)
{
	return RandomizedSelect(a, 0, n - 1, i);
}

/* Builds the rectangular-patch constraint windows of the ring offsets with
 * the reference's own gen_offset_constraint_windows (XT_OffsetError.c:46-96),
 * which only its phantom set-up calls (XT_Init.c:772); afterwards offset mode
 * 3 solves the constrained problem (constrained_quad_opt). */
void ref_build_offset_windows(void *h)
{
	ref_ctx *c = (ref_ctx *)h;
	c->T->Write2Tiff = 0;
	gen_offset_constraint_windows(c->S, c->T);
}

/* The windows [M][N_r][N_t] into out (may be NULL); returns M. */
int ref_get_offset_windows(void *h, float *out)
{
	ref_ctx *c = (ref_ctx *)h;
	int M = c->S->off_constraint_num;
	size_t n = (size_t)M * c->S->N_r * c->S->N_t, q;
	if (out && M > 0)
		for (q = 0; q < n; q++)
			out[q] = (float)(&(c->S->off_constraint[0][0][0]))[q];
	return M;
}

/* The reference's x2 up-sampling of an object between resolution stages
 * (upsample_object_bilinear_2D / _3D, XT_ICD_update.c:359-498) on flat arrays:
 * in [n_z][n_y][n_x], out [n_z or 2 n_z][2 n_y][2 n_x].  The reference writes
 * into slices 1.. of a halo-padded object; the halo is dropped here. */
void upsample_object_bilinear_2D(Real_arr_t ***, Real_arr_t ***, int32_t, int32_t, int32_t);
void upsample_object_bilinear_3D(Real_arr_t ***, Real_arr_t ***, int32_t, int32_t, int32_t);
void ref_upsample(const float *in, float *out, int n_z, int n_y, int n_x, int z_too)
{
	const int oz = z_too ? 2 * n_z : n_z;
	Real_arr_t ***I = (Real_arr_t ***)multialloc(sizeof(Real_arr_t), 3, n_z, n_y, n_x);
	Real_arr_t ***O = (Real_arr_t ***)multialloc(sizeof(Real_arr_t), 3, oz + 2, 2 * n_y, 2 * n_x);
	size_t q, pl = (size_t)4 * n_y * n_x;
	for (q = 0; q < (size_t)n_z * n_y * n_x; q++)
		(&I[0][0][0])[q] = in[q];
	if (z_too)
		upsample_object_bilinear_3D(O, I, n_z, n_y, n_x);
	else
		upsample_object_bilinear_2D(O, I, n_z, n_y, n_x);
	for (q = 0; q < (size_t)oz * pl; q++)
		out[q] = (&O[1][0][0])[q];
	multifree(I, 3);
	multifree(O, 3);
}
