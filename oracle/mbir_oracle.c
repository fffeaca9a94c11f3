/*
 * CPU restatement of TIMBIR's MBIR ICD/NHICD hot path -- the ORACLE.
 * Test infrastructure only (see mbir_oracle.h); never part of the product.
 *
 * Reference: TIMBIR v0.0.2.  Paths below are relative to src/MBIR_4D.
 * Arrays follow the reference layouts: sinogram-shaped arrays are
 * [N_p][N_r][N_t] (t fastest), the object is [N_time][N_z+2][N_y][N_x] with
 * one halo slice on each side, the update-magnitude map is
 * [N_time][num_z_blocks][N_y][N_x].  Scalars are double, stored arrays are
 * `oarr_t` (float, or double with -DORACLE_F64).  The detector response table
 * is float in both builds because it defines the forward model.
 */
#include "mbir_oracle.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_F64
typedef double oarr_t;
#else
typedef float oarr_t;
#endif

#define P_MRF 1.2
#define Q_MRF 2.0
#define HALF_PI 1.57079632679489661923132169163975144
#define QUARTER_PI 0.785398163397448309615660845819875721
#define PI_D 3.14159265358979323846
#define PROFILE_RES 1536
#define BEAM_RES 512
#define RESP_BINS 64
#define MAX_ITERS 1000
#define MIN_XY_RES 64
#define MAX_STAGES 8

typedef struct {
	/* detector / sinogram (XT_Structures.h:63-97) */
	int N_p, N_r, N_t, z_overlap;
	double delta_r, delta_t, R0, RMax, T0, TMax, OffsetR, OffsetT;
	double *cosv, *sinv;
	float *angles, *ptimes, *rtimes;
	oarr_t *y, *w, *e, *d;
	uint8_t *sel;
	/* object (XT_Structures.h:99-137) */
	int N_x, N_y, N_z, N_time;
	double x0, y0, z0, delta_xy, delta_z, mult_xy, mult_z;
	double sig_s, sig_t, c_s, c_t, delta_recon;
	int *vnum, **vidx;
	oarr_t *obj;
	/* inputs (XT_Structures.h:146-190) */
	double stop_thresh, rot_center, radius_obj;
	double sSQ, sSQP, sTQ, sTQP, SF[3][3][3], TF, var_est, alpha, hT, hdelta;
	int upd_offset, offset_type, upd_var, nblk, K;
	int *xr, *yr, *nr, *xn, *yn, *nn; /* [N_time][nblk][N_y*N_x], [N_time][nblk] */
	oarr_t *mag;
	float *H_r;
	uint8_t *mask;
	double last_pct, fwd_cost, prior_cost, err_cost;
	long long updates;
	/* rectangular-patch constraint windows of the ring offsets, [nwin][N_r][N_t] */
	int nwin;
	oarr_t *win;
} orc_t;

#define SINO(c, p, r, t) ((((size_t)(p) * (c)->N_r) + (r)) * (c)->N_t + (t))
#define OBJ(c, i, z, yy, xx) (((((size_t)(i) * ((c)->N_z + 2)) + (z)) * (c)->N_y + (yy)) * (c)->N_x + (xx))
#define MAG(c, i, b, yy, xx) (((((size_t)(i) * (c)->nblk) + (b)) * (c)->N_y + (yy)) * (c)->N_x + (xx))
#define SEL(c, i, b) (((size_t)(i) * (c)->nblk + (b)) * (size_t)(c)->N_y * (c)->N_x)

/* ---------------------------------------------------------------- RNG ---- */
/* Park-Miller minimal standard generator, x' = 16807 x mod (2^31 - 1), value
 * x'/(2^31 - 1) in (0, 1] (randlib.c:119-141 random2, :168-174 srandom2). */
static uint32_t g_seed = 1;
void orc_srandom2(uint32_t seed) { g_seed = seed; }
double orc_random2(void)
{
	g_seed = (uint32_t)(((uint64_t)g_seed * 16807u) % 2147483647u);
	return (double)g_seed / 2147483647.0;
}

/* ------------------------------------------------------ order statistic -- */
/* Randomised quickselect, i-th smallest (1-based) of a[p..r], with the
 * reference's Lomuto partition and random pivot (XT_NHICD.c:63-126).  The
 * pivots consume RNG draws exactly as the reference does. */
static uint32_t orc_partition(float *A, uint32_t p, uint32_t r)
{
	float x = A[r], t;
	uint32_t i = p - 1, j;
	for (j = p; j < r; j++)
		if (A[j] <= x) {
			i++;
			t = A[i]; A[i] = A[j]; A[j] = t;
		}
	t = A[i + 1]; A[i + 1] = A[r]; A[r] = t;
	return i + 1;
}
static double orc_rselect(float *A, uint32_t p, uint32_t r, uint32_t i)
{
	for (;;) {
		uint32_t q, k, j, rnum;
		float t;
		if (p == r)
			return A[p];
		rnum = (uint32_t)floor(orc_random2() * (r - p + 1));
		rnum = (rnum == r - p + 1) ? r - p : rnum;
		j = p + rnum;
		t = A[r]; A[r] = A[j]; A[j] = t;
		q = orc_partition(A, p, r);
		k = q - p + 1;
		if (i == k)
			return A[q];
		else if (i < k)
			r = q - 1;
		else {
			p = q + 1;
			i = i - k;
		}
	}
}
double orc_randomized_select(float *a, uint32_t n, uint32_t i) { return orc_rselect(a, 0, n - 1, i); }

/* ----------------------------------------------------------- set-up ------ */
/* num_z_blocks from the thread count (XT_Init.c:389-398). */
int orc_z_blocks_for_threads(int threads, int n_time, int n_z)
{
	int nb = threads / n_time;
	if (nb < 2)
		nb = 2;
	else if (nb > n_z)
		nb = n_z;
	return (nb / 2) * 2;
}

/* View -> frame map, half-open windows [rt_i, rt_{i+1}) (XT_Init.c:69-96),
 * delta_recon = mean views per frame (:124-133). */
static void orc_view_frames(orc_t *c)
{
	int i, j, n, start = 0;
	double t, total = 0;
	int *buf = (int *)malloc(sizeof(int) * c->N_p);
	c->vnum = (int *)calloc(c->N_time, sizeof(int));
	c->vidx = (int **)calloc(c->N_time, sizeof(int *));
	for (i = 0; i < c->N_time; i++) {
		n = 0;
		for (j = start; j < c->N_p; j++) {
			t = c->ptimes[j];
			if (t >= c->rtimes[i] && t < c->rtimes[i + 1])
				buf[n++] = j;
			if (t >= c->rtimes[i + 1]) {
				start = j;
				break;
			}
		}
		c->vidx[i] = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
		memcpy(c->vidx[i], buf, sizeof(int) * n);
		c->vnum[i] = n;
		total += n;
	}
	c->delta_recon = total / c->N_time;
	free(buf);
}

static double orc_dist(int i, int j, int k, int l)
{
	return sqrt(pow((double)i - 1.0, 2.0) + pow((double)j - 1.0, 2.0) + pow((double)k - 1.0, 2.0) +
	            pow((double)l - 1.0, 2.0));
}

/* Prior weights proportional to 1/distance, normalised to sum
 * mult_xy^3 * delta_recon (XT_Init.c:144-190). */
static void orc_filter(orc_t *c)
{
	int i, j, k;
	double t, sum = 0, pc = c->mult_xy * c->mult_xy * c->mult_xy * c->delta_recon;
	c->TF = 1.0 / orc_dist(0, 1, 1, 1);
	sum += 2.0 * c->TF;
	for (i = 0; i < 3; i++)
		for (j = 0; j < 3; j++)
			for (k = 0; k < 3; k++) {
				if (i != 1 || j != 1 || k != 1) {
					t = 1.0 / orc_dist(1, i, j, k);
					c->SF[i][j][k] = t;
					sum = sum + t;
				} else
					c->SF[i][j][k] = 0;
			}
	for (i = 0; i < 3; i++)
		for (j = 0; j < 3; j++)
			for (k = 0; k < 3; k++)
				c->SF[i][j][k] = pc * c->SF[i][j][k] / sum;
	c->TF = pc * c->TF / sum;
}

/* initStatStructures (XT_Init.c:449-669) + initDynStructures at one stage
 * with the object starting from zero (XT_Init.c:211-445). */
void *orc_create(const float *projections, const float *weights, const float *angles,
                 const float *proj_times, const float *recon_times, int proj_rows, int proj_cols,
                 int proj_num, int recon_num, float vox_wid, float rot_center, float sig_s,
                 float sig_t, float c_s, float c_t, float convg_thresh, int remove_rings,
                 int quad_convex, float huber_delta, float huber_T, int mult_xy, int mult_z,
                 int num_z_blocks)
{
	orc_t *c = (orc_t *)calloc(1, sizeof(orc_t));
	int i, j, k;
	double len_r = (double)vox_wid * proj_cols, len_t = (double)vox_wid * proj_rows;
	size_t n;
	c->stop_thresh = convg_thresh;
	c->rot_center = rot_center;
	c->alpha = 1.5;
	c->N_time = recon_num;
	c->N_p = proj_num;
	c->N_r = proj_cols;
	c->radius_obj = (double)vox_wid * proj_cols / 2;
	c->N_t = proj_rows;
	c->offset_type = remove_rings;
	c->hT = quad_convex == 0 ? (double)huber_T : 100000;
	c->hdelta = quad_convex == 0 ? (double)huber_delta : 1;
	c->var_est = 1;
	c->sig_s = sig_s; c->sig_t = sig_t; c->c_s = c_s; c->c_t = c_t;
	c->delta_r = len_r / c->N_r;
	c->delta_t = len_t / c->N_t;
	c->R0 = -c->rot_center * c->delta_r;
	c->RMax = (c->N_r - c->rot_center) * c->delta_r;
	c->T0 = -len_t / 2.0;
	c->TMax = len_t / 2.0;
	c->x0 = c->R0;
	c->z0 = c->T0;
	c->y0 = -len_r / 2.0;
	c->K = 10;
	orc_srandom2(761521); /* XT_Engine.c:99 */
	c->angles = (float *)malloc(sizeof(float) * proj_num);
	c->ptimes = (float *)malloc(sizeof(float) * proj_num);
	c->rtimes = (float *)malloc(sizeof(float) * (recon_num + 1));
	memcpy(c->angles, angles, sizeof(float) * proj_num);
	memcpy(c->ptimes, proj_times, sizeof(float) * proj_num);
	memcpy(c->rtimes, recon_times, sizeof(float) * (recon_num + 1));
	orc_view_frames(c);
	c->cosv = (double *)malloc(sizeof(double) * proj_num);
	c->sinv = (double *)malloc(sizeof(double) * proj_num);
	for (i = 0; i < proj_num; i++) {
		c->cosv[i] = cos(c->angles[i]);
		c->sinv[i] = sin(c->angles[i]);
	}
	/* per-stage part (initDynStructures) */
	c->mult_xy = mult_xy;
	c->mult_z = mult_z;
	n = (size_t)c->N_p * c->N_r * c->N_t;
	c->y = (oarr_t *)malloc(sizeof(oarr_t) * n);
	c->w = (oarr_t *)malloc(sizeof(oarr_t) * n);
	c->e = (oarr_t *)calloc(n, sizeof(oarr_t));
	c->sel = (uint8_t *)malloc(n);
	c->d = (oarr_t *)calloc((size_t)c->N_r * c->N_t, sizeof(oarr_t));
	memset(c->sel, 1, n);
	for (i = 0; i < c->N_p; i++)
		for (j = 0; j < c->N_r; j++)
			for (k = 0; k < c->N_t; k++) {
				size_t src = (size_t)i * c->N_t * c->N_r + (size_t)k * c->N_r + j;
				c->y[SINO(c, i, j, k)] = projections[src];
				c->w[SINO(c, i, j, k)] = weights[src];
			}
	for (i = 0; i < (int)n; i++)
		c->w[i] /= c->var_est;
	c->N_x = (int)(c->N_r / c->mult_xy);
	c->N_y = (int)(c->N_r / c->mult_xy);
	c->N_z = (int)(c->N_t / c->mult_z);
	c->delta_xy = c->mult_xy * c->delta_r;
	c->delta_z = c->mult_z * c->delta_t;
	c->z_overlap = (int)c->mult_z;
	c->obj = (oarr_t *)calloc((size_t)c->N_time * (c->N_z + 2) * c->N_y * c->N_x, sizeof(oarr_t));
	c->OffsetR = (c->delta_xy / sqrt(2.0) + c->delta_r / 2.0) / RESP_BINS;
	c->OffsetT = ((c->delta_z / 2) + c->delta_t / 2) / RESP_BINS;
	c->nblk = num_z_blocks;
	n = (size_t)c->N_time * c->nblk * c->N_y * c->N_x;
	c->xr = (int *)calloc(n, sizeof(int));
	c->yr = (int *)calloc(n, sizeof(int));
	c->xn = (int *)calloc(n, sizeof(int));
	c->yn = (int *)calloc(n, sizeof(int));
	c->nr = (int *)calloc((size_t)c->N_time * c->nblk, sizeof(int));
	c->nn = (int *)calloc((size_t)c->N_time * c->nblk, sizeof(int));
	c->mag = (oarr_t *)calloc(n, sizeof(oarr_t));
	c->sSQ = pow(c->sig_s * c->mult_xy, Q_MRF);
	c->sSQP = pow(c->sig_s * c->mult_xy, Q_MRF - P_MRF);
	c->sTQ = pow(c->sig_t * c->delta_recon, Q_MRF);
	c->sTQP = pow(c->sig_t * c->delta_recon, Q_MRF - P_MRF);
	orc_filter(c);
	c->mask = (uint8_t *)calloc((size_t)c->N_time * c->N_y * c->N_x, 1);
	c->H_r = (float *)calloc((size_t)c->N_p * (RESP_BINS + 1), sizeof(float));
	return c;
}

void orc_destroy(void *h)
{
	orc_t *c = (orc_t *)h;
	int i;
	if (!c)
		return;
	for (i = 0; i < c->N_time; i++)
		free(c->vidx[i]);
	free(c->vidx); free(c->vnum); free(c->cosv); free(c->sinv);
	free(c->angles); free(c->ptimes); free(c->rtimes);
	free(c->y); free(c->w); free(c->e); free(c->d); free(c->sel); free(c->obj);
	free(c->xr); free(c->yr); free(c->xn); free(c->yn); free(c->nr); free(c->nn);
	free(c->mag); free(c->mask); free(c->H_r); free(c->win);
	free(c);
}

/* Stage switches that the multi-resolution driver derives per stage
 * (XT_Init.c:236-266); var_est rescales the weights as at XT_Init.c:327-330. */
void orc_set_switches(void *h, int update_proj_offset, int update_var, double var_est)
{
	orc_t *c = (orc_t *)h;
	size_t i, n = (size_t)c->N_p * c->N_r * c->N_t;
	c->upd_offset = update_proj_offset;
	c->upd_var = update_var;
	if (var_est > 0 && var_est != c->var_est) {
		for (i = 0; i < n; i++)
			c->w[i] = (oarr_t)(c->w[i] * c->var_est);
		c->var_est = var_est;
		for (i = 0; i < n; i++)
			c->w[i] /= var_est;
	}
}

/* ------------------------------------------------ detector response ------ */
/* Trapezoidal voxel profile per view sampled on PROFILE_RES points
 * (XT_Profile.c:47-108), convolved with a normalised 512-point Hamming beam
 * (XT_Profile.c:112-127), tabulated at 64 distances of step OffsetR plus a
 * trailing zero (XT_Profile.c:129-170). */
static void orc_detector_response(orc_t *c)
{
	int i, j, k, p, pi;
	double angle, maxv, tmp, d1, d2, lc, ln, rn, rc, t, sum, r, rmin, beam[BEAM_RES];
	double r0 = -c->delta_r / 2, step = c->delta_r / BEAM_RES, tc = PROFILE_RES / (2 * c->delta_xy);
	float *prof = (float *)malloc(sizeof(float) * PROFILE_RES);
	sum = 0;
	for (i = 0; i < BEAM_RES; i++) {
		beam[i] = 0.54 - 0.46 * cos((2 * PI_D / BEAM_RES) * i);
		sum = sum + beam[i];
	}
	for (i = 0; i < BEAM_RES; i++)
		beam[i] /= sum;
	for (k = 0; k < c->N_p; k++) {
		angle = c->angles[k];
		while (angle > HALF_PI)
			angle -= HALF_PI;
		while (angle < 0)
			angle += HALF_PI;
		if (angle <= QUARTER_PI)
			maxv = c->delta_xy / cos(angle);
		else
			maxv = c->delta_xy / cos(HALF_PI - angle);
		tmp = cos(QUARTER_PI);
		d1 = tmp * cos((QUARTER_PI - angle));
		d2 = tmp * fabs((cos((QUARTER_PI + angle))));
		lc = 1 - d1; ln = 1 - d2; rn = 1 + d2; rc = 1 + d1;
		for (j = 0; j < PROFILE_RES; j++) {
			t = 2.0 * j / PROFILE_RES;
			if (t <= lc || t >= rc)
				prof[j] = 0;
			else if (t > rn)
				prof[j] = maxv * (rc - t) / (rc - rn);
			else if (t >= ln)
				prof[j] = maxv;
			else
				prof[j] = maxv * (t - lc) / (ln - lc);
		}
		for (i = 0; i < RESP_BINS; i++) {
			rmin = i * c->OffsetR - c->delta_xy;
			sum = 0;
			for (p = 0; p < BEAM_RES; p++) {
				r = r0 + p * step;
				pi = (int)floor((r - rmin) * tc);
				if (pi >= 0 && pi <= PROFILE_RES - 1)
					sum += (prof[pi] * beam[p]);
			}
			c->H_r[(size_t)k * (RESP_BINS + 1) + i] = sum;
		}
		c->H_r[(size_t)k * (RESP_BINS + 1) + RESP_BINS] = 0.0;
	}
	free(prof);
}

/* -------------------------------------------------------- A-matrix ------- */
/* One column of A for voxel line (row, col) and view: the <= 2*mult_xy+1
 * detector bins whose centre lies within delta_xy of the voxel's projected
 * centre, weights by linear interpolation of H_r, kept if > 0
 * (XT_AMatrix.c:50-110). */
static int orc_acol(const orc_t *c, int row, int col, int view, int *idx, double *val)
{
	int j, imin, imax, id, n = 0;
	double x = c->x0 + ((double)col + 0.5) * c->delta_xy;
	double y = c->y0 + ((double)row + 0.5) * c->delta_xy;
	double r = x * c->cosv[view] - y * c->sinv[view];
	double rmin = r - c->delta_xy, rmax = r + c->delta_xy, rc, dr, w1, w2, f1;
	const float *H = c->H_r + (size_t)view * (RESP_BINS + 1);
	if (rmax < c->R0 || rmin > c->RMax)
		return 0;
	imin = (int)(floor(((rmin - c->R0) / c->delta_r)));
	imax = (int)(floor((rmax - c->R0) / c->delta_r));
	if (imax >= c->N_r)
		imax = c->N_r - 1;
	if (imin < 0)
		imin = 0;
	for (j = imin; j <= imax; j++) {
		rc = (c->R0 + (((double)j) + 0.5) * (c->delta_r));
		dr = fabs(r - rc);
		id = (int)(floor((dr / c->OffsetR)));
		if (id >= 0 && id < RESP_BINS) {
			w1 = dr - id * c->OffsetR;
			w2 = c->OffsetR - w1;
			f1 = (w2 * H[id] + w1 * H[id + 1]) / c->OffsetR;
			if (f1 > 0) {
				val[n] = f1;
				idx[n] = j;
				n++;
			}
		}
	}
	return n;
}

int orc_amatrix(void *h, int row, int col, int view, int *idx, double *val, int cap)
{
	int ib[512], n, i;
	double vb[512];
	n = orc_acol((orc_t *)h, row, col, view, ib, vb);
	for (i = 0; i < n && i < cap; i++) {
		idx[i] = ib[i];
		val[i] = vb[i];
	}
	return n;
}

static int orc_amax(const orc_t *c) { return (int)ceil(3 * c->delta_xy / c->delta_r) + 2; }

/* ------------------------------------------------ error sinogram --------- */
/* e = y - A x - d, then the zinger selection |e sqrt(w)| < T
 * (XT_ICD_update.c:655-716, forward projection XT_ForwardProject.c:8-25). */
static void orc_error_sino(orc_t *c)
{
	int i, j, k, p, s, m, n, view, cnt, amax = orc_amax(c);
	int *idx = (int *)malloc(sizeof(int) * amax);
	double *val = (double *)malloc(sizeof(double) * amax), pix;
	size_t q, ns = (size_t)c->N_p * c->N_r * c->N_t;
	memset(c->e, 0, sizeof(oarr_t) * ns);
	for (i = 0; i < c->N_time; i++)
		for (j = 0; j < c->N_y; j++)
			for (k = 0; k < c->N_x; k++)
				for (p = 0; p < c->vnum[i]; p++) {
					view = c->vidx[i][p];
					cnt = orc_acol(c, j, k, view, idx, val);
					for (s = 0; s < c->N_z; s++) {
						pix = c->obj[OBJ(c, i, s + 1, j, k)];
						for (m = 0; m < cnt; m++)
							for (n = 0; n < c->z_overlap; n++)
								c->e[SINO(c, view, idx[m], s * c->z_overlap + n)] += pix * val[m];
					}
				}
	for (p = 0; p < c->N_p; p++)
		for (j = 0; j < c->N_r; j++)
			for (k = 0; k < c->N_t; k++) {
				q = SINO(c, p, j, k);
				c->e[q] = c->y[q] - c->e[q] - c->d[(size_t)j * c->N_t + k];
				c->sel[q] = fabs(c->e[q] * sqrt(c->w[q])) < c->hT;
			}
	free(idx);
	free(val);
}

/* ------------------------------------------------------------ prior ------ */
/* qGGMRF potential rho(D) = (|D|^q/s^q) / (c + |D|^(q-p)/s^(q-p)) and its
 * derivative (XT_ICD_update.c:83-128). */
static double orc_rho(double d, double sQ, double sQP, double cc)
{
	return ((pow(fabs(d), Q_MRF) / sQ) / (cc + pow(fabs(d), Q_MRF - P_MRF) / sQP));
}
static double orc_drho(double d, double sQ, double sQP, double cc)
{
	double t1 = pow(fabs(d), Q_MRF - P_MRF) / (sQP);
	double t2 = pow(fabs(d), Q_MRF - 1);
	double t3 = cc + t1;
	if (d < 0)
		return ((-1 * t2 / (t3 * sQ)) * (Q_MRF - ((Q_MRF - P_MRF) * t1) / (t3)));
	return ((t2 / (t3 * sQ)) * (Q_MRF - ((Q_MRF - P_MRF) * t1) / (t3)));
}

/* Surrogate (majorizer) step for one voxel, then over-relaxation by alpha
 * (XT_ICD_update.c:134-183): b_j = f_j rho'(D_j)/D_j (rho''(0) f_j at D_j=0),
 * u = (sum b_j x_j + theta2 V - theta1) / (sum b_j + theta2). */
static double orc_substitute(const orc_t *c, double V, double th1, double th2, double sn[3][3][3],
                             const uint8_t sf[3][3][3], const double tn[2], const uint8_t tf[2])
{
	double u, t1 = 0, t2 = 0, tcst, ref = V, d0, prm;
	int i, j, k;
	for (i = 0; i < 3; i++)
		for (j = 0; j < 3; j++)
			for (k = 0; k < 3; k++) {
				if (sf[i][j][k] && (i != 1 || j != 1 || k != 1)) {
					d0 = (ref - sn[i][j][k]);
					if (d0 != 0)
						prm = orc_drho(d0, c->sSQ, c->sSQP, c->c_s) / (d0);
					else
						prm = Q_MRF / (c->sSQ * c->c_s);
					tcst = c->SF[i][j][k] * prm;
					t1 += tcst * sn[i][j][k];
					t2 += tcst;
				}
			}
	for (i = 0; i < 2; i++) {
		if (tf[i]) {
			d0 = (ref - tn[i]);
			if (d0 != 0)
				prm = orc_drho(d0, c->sTQ, c->sTQP, c->c_t) / (d0);
			else
				prm = Q_MRF / (c->sTQ * c->c_t);
			tcst = c->TF * prm;
			t1 += tcst * tn[i];
			t2 += tcst;
		}
	}
	u = (t1 + (th2 * V) - th1) / (t2 + th2);
	ref = ref + c->alpha * (u - ref);
	return ref;
}

double orc_functional_substitution(void *h, double V, double theta1, double theta2,
                                   const double *spatial27, const uint8_t *sflag27,
                                   const double *time2, const uint8_t *tflag2)
{
	double sn[3][3][3], tn[2];
	uint8_t sf[3][3][3], tf[2];
	int i;
	for (i = 0; i < 27; i++) {
		sn[i / 9][(i / 3) % 3][i % 3] = spatial27[i];
		sf[i / 9][(i / 3) % 3][i % 3] = sflag27[i];
	}
	tn[0] = time2[0]; tn[1] = time2[1];
	tf[0] = tflag2[0]; tf[1] = tflag2[1];
	return orc_substitute((orc_t *)h, V, theta1, theta2, sn, sf, tn, tf);
}

/* --------------------------------------------------- voxel update -------- */
/* theta1/theta2 with the generalized-Huber weights, surrogate step, then the
 * error-sinogram and selection refresh (XT_VoxUpdate.c:43-115). */
static void orc_voxel(orc_t *c, int *cnt, int *idx, double *val, int amax, double sn[3][3][3],
                      uint8_t sf[3][3][3], double tn[2], uint8_t tf[2], int i, int s, int j, int k)
{
	int p, q, r, view, ir, it;
	double V = c->obj[OBJ(c, i, s + 1, j, k)], th1 = 0.0, th2 = 0.0, a, tmp, dx, nv;
	size_t o;
	for (p = 0; p < c->vnum[i]; p++) {
		view = c->vidx[i][p];
		for (q = 0; q < cnt[p]; q++) {
			ir = idx[p * amax + q];
			a = val[p * amax + q];
			for (r = 0; r < c->z_overlap; r++) {
				it = s * c->z_overlap + r;
				o = SINO(c, view, ir, it);
				if (c->sel[o]) {
					th2 += (a * a * c->w[o]);
					th1 += -(c->e[o] * a * c->w[o]);
				} else {
					tmp = c->hT * c->hdelta * sqrt(c->w[o]) / fabs(c->e[o]);
					th2 += (a * a * tmp);
					th1 += -(c->e[o] * a * tmp);
				}
			}
		}
	}
	nv = orc_substitute(c, V, th1, th2, sn, sf, tn, tf);
	c->obj[OBJ(c, i, s + 1, j, k)] = (oarr_t)nv;
	dx = c->obj[OBJ(c, i, s + 1, j, k)] - V;
	for (p = 0; p < c->vnum[i]; p++) {
		view = c->vidx[i][p];
		for (q = 0; q < cnt[p]; q++) {
			ir = idx[p * amax + q];
			a = val[p * amax + q];
			for (r = 0; r < c->z_overlap; r++) {
				it = s * c->z_overlap + r;
				o = SINO(c, view, ir, it);
				c->e[o] -= (a * dx);
				c->sel[o] = fabs(c->e[o] * sqrt(c->w[o])) < c->hT;
			}
		}
	}
	c->updates++;
}

/* One task: voxel lines xy_begin..xy_end of a line list, slices
 * slice_begin..slice_end of frame i (XT_VoxUpdate.c:117-281).  Gathers the
 * 26-neighbourhood (z halo rule of :126-131 at a single rank) and the two
 * temporal neighbours, applies zero skipping (:236-259), updates, and keeps
 * the per-line magnitude map.  Returns the sum of |x'| over updated voxels. */
static double orc_update_lines(orc_t *c, int i, int z0, int z1, int b0, int b1, const int *xs,
                               const int *ys, int iter, oarr_t *mag)
{
	int amax = orc_amax(c), nv = c->vnum[i] > 0 ? c->vnum[i] : 1;
	int *cnt = (int *)malloc(sizeof(int) * nv);
	int *idx = (int *)malloc(sizeof(int) * (size_t)nv * amax);
	double *val = (double *)malloc(sizeof(double) * (size_t)nv * amax);
	double sn[3][3][3], tn[2], V, tot = 0.0;
	uint8_t sf[3][3][3], tf[2], zs;
	int li, j, k, p, q, r, s, ip, iq, ir, zmin = 1, zmax = c->N_z;
	for (li = b0; li <= b1; li++) {
		k = xs[li];
		j = ys[li];
		mag[(size_t)j * c->N_x + k] = 0;
		for (p = 0; p < c->vnum[i]; p++)
			cnt[p] = orc_acol(c, j, k, c->vidx[i][p], idx + (size_t)p * amax, val + (size_t)p * amax);
		for (s = z0; s <= z1; s++) {
			if (c->mask[((size_t)i * c->N_y + j) * c->N_x + k] != 1)
				continue;
			if (i - 1 >= 0) {
				tn[0] = c->obj[OBJ(c, i - 1, s + 1, j, k)];
				tf[0] = 1;
			} else {
				tn[0] = 0.0;
				tf[0] = 0;
			}
			if (i + 1 < c->N_time) {
				tn[1] = c->obj[OBJ(c, i + 1, s + 1, j, k)];
				tf[1] = 1;
			} else {
				tn[1] = 0.0;
				tf[1] = 0;
			}
			for (p = 0; p < 3; p++) {
				ip = s + p;
				for (q = 0; q < 3; q++) {
					iq = j + q - 1;
					for (r = 0; r < 3; r++) {
						ir = k + r - 1;
						if (ip >= zmin && ip <= zmax && iq >= 0 && iq < c->N_y && ir >= 0 && ir < c->N_x) {
							sn[p][q][r] = c->obj[OBJ(c, i, ip, iq, ir)];
							sf[p][q][r] = 1;
						} else {
							sn[p][q][r] = 0.0;
							sf[p][q][r] = 0;
						}
					}
				}
			}
			sn[1][1][1] = 0.0;
			V = c->obj[OBJ(c, i, s + 1, j, k)];
			zs = 1;
			if (V == 0.0 && iter > 1) {
				if (tn[0] > 0.0 || tn[1] > 0.0)
					zs = 0;
				for (p = 0; p < 27; p++)
					if (sn[p / 9][(p / 3) % 3][p % 3] > 0.0)
						zs = 0;
			} else
				zs = 0;
			if (!zs) {
				orc_voxel(c, cnt, idx, val, amax, sn, sf, tn, tf, i, s, j, k);
				mag[(size_t)j * c->N_x + k] += fabs(c->obj[OBJ(c, i, s + 1, j, k)] - V);
				tot += fabs(c->obj[OBJ(c, i, s + 1, j, k)]);
			}
		}
	}
	free(cnt);
	free(idx);
	free(val);
	return tot;
}

/* ----------------------------------------------------- line orders ------- */
/* Random permutation of the in-mask lines per (frame, block), one RNG draw
 * per element (XT_ICD_update.c:500-532). */
void orc_random_select(void *h)
{
	orc_t *c = (orc_t *)h;
	int i, b, j, n, idx, col, row, sz, per = c->N_z / c->nblk;
	int *ctr = (int *)malloc(sizeof(int) * c->N_y * c->N_x);
	for (i = 0; i < c->N_time; i++)
		for (b = 0; b < c->nblk; b++) {
			int *xs = c->xr + SEL(c, i, b), *ys = c->yr + SEL(c, i, b), *num = c->nr + (size_t)i * c->nblk + b;
			sz = c->N_y * c->N_x;
			for (idx = 0; idx < sz; idx++)
				ctr[idx] = idx;
			*num = 0;
			for (j = 0; j < c->N_x * c->N_y; j++) {
				idx = (int)floor(orc_random2() * sz);
				idx = (idx == sz) ? sz - 1 : idx;
				col = ctr[idx] % c->N_x;
				row = ctr[idx] / c->N_x;
				for (n = b * per; n < (b + 1) * per; n++)
					if (c->mask[((size_t)i * c->N_y + row) * c->N_x + col] == 1) {
						xs[*num] = col;
						ys[*num] = row;
						(*num)++;
						break;
					}
				ctr[idx] = ctr[sz - 1];
				sz--;
			}
		}
	free(ctr);
}

/* NHICD selection: 5x5 Hamming-filtered magnitude map, threshold at the
 * order statistic that keeps floor(N_sel/10) lines, lines strictly above it
 * in raster order (XT_NHICD.c:128-216). */
void orc_vsc_select(void *h)
{
	static const double HW[5][5] = {{0.0064, 0.0432, 0.0800, 0.0432, 0.0064},
	                                {0.0432, 0.2916, 0.5400, 0.2916, 0.0432},
	                                {0.0800, 0.5400, 1.0000, 0.5400, 0.0800},
	                                {0.0432, 0.2916, 0.5400, 0.2916, 0.0432},
	                                {0.0064, 0.0432, 0.0800, 0.0432, 0.0064}};
	orc_t *c = (orc_t *)h;
	int i, b, j, k, p, q, n, cnt;
	size_t N = (size_t)c->N_y * c->N_x;
	float *f = (float *)malloc(sizeof(float) * N), *fc = (float *)malloc(sizeof(float) * N);
	double acc, th;
	for (i = 0; i < c->N_time; i++)
		for (b = 0; b < c->nblk; b++) {
			const oarr_t *m = c->mag + MAG(c, i, b, 0, 0);
			int *xs = c->xn + SEL(c, i, b), *ys = c->yn + SEL(c, i, b);
			n = c->nr[(size_t)i * c->nblk + b] / c->K;
			for (j = 0; j < c->N_y; j++)
				for (k = 0; k < c->N_x; k++) {
					acc = 0;
					for (p = -2; p <= 2; p++)
						for (q = -2; q <= 2; q++)
							if (j + p >= 0 && j + p < c->N_y && k + q >= 0 && k + q < c->N_x)
								acc += HW[p + 2][q + 2] * m[(size_t)(j + p) * c->N_x + k + q];
					f[(size_t)j * c->N_x + k] = acc;
					fc[(size_t)j * c->N_x + k] = acc;
				}
			th = orc_rselect(f, 0, (uint32_t)N - 1, (uint32_t)(N - n));
			cnt = 0;
			for (j = 0; j < c->N_y; j++)
				for (k = 0; k < c->N_x; k++)
					if (fc[(size_t)j * c->N_x + k] > th) {
						xs[cnt] = k;
						ys[cnt] = j;
						cnt++;
					}
			c->nn[(size_t)i * c->nblk + b] = cnt;
		}
	free(f);
	free(fc);
}

/* ----------------------------------------------------- ring offsets ------ */
/* Per detector element (r,t): num = sum_p w e (selected) or T delta sqrt(w) sgn(e),
 * den = sum_p w or T delta sqrt(w)/|e| (XT_ICD_update.c:820-840, 876-893). */
static void orc_offset_terms(orc_t *c, double *num, double *den)
{
	int i, j, k;
	double tmp, sg;
	size_t o;
	for (i = 0; i < c->N_r; i++)
		for (j = 0; j < c->N_t; j++) {
			double nm = 0, dn = 0;
			for (k = 0; k < c->N_p; k++) {
				o = SINO(c, k, i, j);
				tmp = c->hT * c->hdelta * sqrt(c->w[o]);
				if (c->sel[o]) {
					nm += c->e[o] * c->w[o];
					dn += c->w[o];
				} else {
					sg = (c->e[o] > 0) - (c->e[o] < 0);
					nm += tmp * sg;
					dn += tmp / fabs(c->e[o]);
				}
			}
			num[(size_t)i * c->N_t + j] = nm;
			den[(size_t)i * c->N_t + j] = dn;
		}
}

static void orc_apply_shift(orc_t *c, int i, int j, double shift)
{
	int k;
	size_t o;
	for (k = 0; k < c->N_p; k++) {
		o = SINO(c, k, i, j);
		c->e[o] -= shift;
		c->sel[o] = fabs(c->e[o] * sqrt(c->w[o])) < c->hT;
	}
}

/* remove_rings 1: d += num/den (XT_ICD_update.c:870-917).
 * remove_rings 2: d += (num - gamma)/den with gamma making the update keep
 * sum d fixed at zero mean (XT_ICD_update.c:817-867).
 * remove_rings 3: the rectangular-patch constrained solve
 * (XT_ICD_update.c:753-814, XT_OffsetError.c:99-168); on the reconstruct path
 * the constraint windows are never built, so the solve has M = 0 constraints
 * and reduces to x = b/Lambda with b = sum (e + d) w-terms. */
/* ------------------------------------------- offset constraint windows -- */
/* Overlapping rectangular windows over the detector (gen_offset_constraint_windows,
 * XT_OffsetError.c:46-96): sides r_size = 2 N_r / round(sqrt(N_r)) and
 * t_size = 2 N_t / round(sqrt(N_t)), origins every half side, wrapping
 * around the detector edges, separable tent weights. */
void orc_build_offset_windows(void *h)
{
	orc_t *c = (orc_t *)h;
	int rs = 2 * c->N_r / (int)(sqrt(c->N_r) + 0.5), ts = 2 * c->N_t / (int)(sqrt(c->N_t) + 0.5);
	int i, j, k, l, m = 0;
	for (i = 0; i <= c->N_r - rs / 2; i += rs / 2)
		for (j = 0; j <= c->N_t - ts / 2; j += ts / 2)
			m++;
	free(c->win);
	c->nwin = m;
	c->win = (oarr_t *)calloc((size_t)m * c->N_r * c->N_t, sizeof(oarr_t));
	m = 0;
	for (i = 0; i <= c->N_r - rs / 2; i += rs / 2)
		for (j = 0; j <= c->N_t - ts / 2; j += ts / 2) {
			for (k = i; k < i + rs; k++)
				for (l = j; l < j + ts; l++) {
					double a = (k - i) < rs / 2 ? (k - i + 1) : rs - (k - i);
					a *= (l - j) < ts / 2 ? (l - j + 1) : ts - (l - j);
					c->win[((size_t)m * c->N_r + k % c->N_r) * c->N_t + l % c->N_t] = (oarr_t)a;
				}
			m++;
		}
}

int orc_get_offset_windows(void *h, float *out)
{
	orc_t *c = (orc_t *)h;
	size_t q, n = (size_t)c->nwin * c->N_r * c->N_t;
	if (out)
		for (q = 0; q < n; q++)
			out[q] = (float)c->win[q];
	return c->nwin;
}

/* In-place inverse of the n x n matrix a (row-major) by LU decomposition with
 * partial pivoting (rows scaled by their largest entry for the pivot choice)
 * and forward / back substitution of each unit vector, as invert2 does
 * (invert.c:110-140). */
static void lu_inverse(double *a, int n)
{
	int i, j, k, imax = 0, *piv = (int *)malloc(sizeof(int) * n);
	double *scale = (double *)malloc(sizeof(double) * n), *col = (double *)malloc(sizeof(double) * n);
	double *y = (double *)malloc(sizeof(double) * n * n);
	for (i = 0; i < n; i++) {
		double big = 0;
		for (j = 0; j < n; j++)
			if (fabs(a[i * n + j]) > big)
				big = fabs(a[i * n + j]);
		scale[i] = big > 0 ? 1.0 / big : 0.0;
	}
	for (j = 0; j < n; j++) {
		double big = 0;
		for (i = 0; i < j; i++) {
			double sum = a[i * n + j];
			for (k = 0; k < i; k++)
				sum -= a[i * n + k] * a[k * n + j];
			a[i * n + j] = sum;
		}
		for (i = j; i < n; i++) {
			double sum = a[i * n + j];
			for (k = 0; k < j; k++)
				sum -= a[i * n + k] * a[k * n + j];
			a[i * n + j] = sum;
			if (scale[i] * fabs(sum) >= big) {
				big = scale[i] * fabs(sum);
				imax = i;
			}
		}
		if (j != imax) {
			for (k = 0; k < n; k++) {
				double t = a[imax * n + k];
				a[imax * n + k] = a[j * n + k];
				a[j * n + k] = t;
			}
			scale[imax] = scale[j];
		}
		piv[j] = imax;
		if (a[j * n + j] == 0.0)
			a[j * n + j] = 1e-20;
		for (i = j + 1; i < n; i++)
			a[i * n + j] /= a[j * n + j];
	}
	for (j = 0; j < n; j++) {
		int first = -1;
		for (i = 0; i < n; i++)
			col[i] = i == j ? 1.0 : 0.0;
		for (i = 0; i < n; i++) {
			double sum = col[piv[i]];
			col[piv[i]] = col[i];
			if (first >= 0)
				for (k = first; k < i; k++)
					sum -= a[i * n + k] * col[k];
			else if (sum != 0.0)
				first = i;
			col[i] = sum;
		}
		for (i = n - 1; i >= 0; i--) {
			double sum = col[i];
			for (k = i + 1; k < n; k++)
				sum -= a[i * n + k] * col[k];
			col[i] = sum / a[i * n + i];
		}
		for (i = 0; i < n; i++)
			y[i * n + j] = col[i];
	}
	memcpy(a, y, sizeof(double) * n * n);
	free(piv); free(scale); free(col); free(y);
}

/* Offsets x minimising sum Lambda (x - b / Lambda)^2 subject to A x = 0 for
 * the constraint windows A (constrained_quad_opt, XT_OffsetError.c:99-168):
 * D = A Lambda^-1 A^T, t = D^-1 A (b / Lambda), x = (b - A^T t) / Lambda. */
static void orc_constrained_offsets(orc_t *c, const double *b, const double *L, oarr_t *x)
{
	const int M = c->nwin, Nr = c->N_r, Nt = c->N_t;
	const size_t ne = (size_t)Nr * Nt;
	double *D = (double *)calloc((size_t)M * M, sizeof(double));
	double *t2 = (double *)calloc(M, sizeof(double)), *t = (double *)calloc(M, sizeof(double));
	int i, j;
	size_t q;
	for (i = 0; i < M; i++)
		for (j = 0; j < M; j++)
			for (q = 0; q < ne; q++)
				D[i * M + j] += (double)c->win[i * ne + q] * (double)c->win[j * ne + q] / L[q];
	lu_inverse(D, M);
	for (i = 0; i < M; i++)
		for (q = 0; q < ne; q++)
			t2[i] += (double)c->win[i * ne + q] * b[q] / L[q];
	for (i = 0; i < M; i++)
		for (j = 0; j < M; j++)
			t[i] += D[i * M + j] * t2[j];
	for (q = 0; q < ne; q++) {
		oarr_t v = 0;
		for (i = 0; i < M; i++)
			v += (double)c->win[i * ne + q] * t[i];
		x[q] = (oarr_t)((b[q] - v) / L[q]);
	}
	free(D); free(t2); free(t);
}

void orc_offset_update(void *h)
{
	orc_t *c = (orc_t *)h;
	size_t n = (size_t)c->N_r * c->N_t, q;
	double *num = (double *)malloc(sizeof(double) * n), *den = (double *)malloc(sizeof(double) * n);
	double ns = 0, ds = 0, g = 0;
	int i, j, k;
	if (c->offset_type == 3) {
		double tmp, sg;
		size_t o;
		for (i = 0; i < c->N_r; i++)
			for (j = 0; j < c->N_t; j++) {
				double b = 0, L = 0;
				q = (size_t)i * c->N_t + j;
				for (k = 0; k < c->N_p; k++) {
					o = SINO(c, k, i, j);
					tmp = c->hT * c->hdelta * sqrt(c->w[o]);
					if (c->sel[o]) {
						L += c->w[o];
						b += (c->e[o] + c->d[q]) * c->w[o];
					} else {
						sg = (c->e[o] > 0) - (c->e[o] < 0);
						(void)sg;
						L += tmp / fabs(c->e[o]);
						b += (c->e[o] + c->d[q]) * tmp / fabs(c->e[o]);
					}
				}
				num[q] = b;
				den[q] = L;
			}
		{
			/* without windows (the reference's reconstruct path: none are
			 * built) the constraint is empty and x = b / Lambda */
			oarr_t *xs = (oarr_t *)malloc(sizeof(oarr_t) * n);
			if (c->nwin > 0)
				orc_constrained_offsets(c, num, den, xs);
			else
				for (q = 0; q < n; q++)
					xs[q] = (oarr_t)((num[q] - 0.0) / den[q]);
			for (k = 0; k < c->N_p; k++)
				for (i = 0; i < c->N_r; i++)
					for (j = 0; j < c->N_t; j++) {
						q = (size_t)i * c->N_t + j;
						o = SINO(c, k, i, j);
						c->e[o] += c->d[q] - xs[q];
						c->sel[o] = fabs(c->e[o] * sqrt(c->w[o])) < c->hT;
					}
			for (q = 0; q < n; q++)
				c->d[q] = xs[q];
			free(xs);
		}
		free(num);
		free(den);
		return;
	}
	orc_offset_terms(c, num, den);
	if (c->offset_type == 2) {
		for (q = 0; q < n; q++) {
			ns += c->d[q] + (num[q] / den[q]);
			ds += 1.0 / den[q];
		}
		g = ns / ds;
	}
	if (c->offset_type == 1 || c->offset_type == 2) {
		for (i = 0; i < c->N_r; i++)
			for (j = 0; j < c->N_t; j++) {
				q = (size_t)i * c->N_t + j;
				c->d[q] = c->d[q] + (num[q] - g) / den[q];
				orc_apply_shift(c, i, j, (num[q] - g) / den[q]);
			}
	}
	free(num);
	free(den);
}

/* ----------------------------------------------------------- variance ---- */
/* sigma^2 = mean(selected: e^2 w_orig ; else |e| delta T sqrt(w_orig sigma^2_old)),
 * then w = w_orig / sigma^2 and the selection refresh (XT_ICD_update.c:720-751). */
void orc_variance_update(void *h)
{
	orc_t *c = (orc_t *)h;
	size_t k, n = (size_t)c->N_p * c->N_r * c->N_t;
	double acc = 0, t;
	for (k = 0; k < n; k++) {
		c->w[k] = c->w[k] * c->var_est;
		if (c->sel[k])
			t = c->e[k] * c->e[k] * c->w[k];
		else
			t = fabs(c->e[k]) * c->hdelta * c->hT * sqrt(c->w[k] * c->var_est);
		acc += t;
	}
	c->var_est = acc / ((double)1 * (double)c->N_p * (double)c->N_r * (double)c->N_t);
	for (k = 0; k < n; k++) {
		c->w[k] /= c->var_est;
		c->sel[k] = fabs(c->e[k] * sqrt(c->w[k])) < c->hT;
	}
}

/* --------------------------------------------------------------- cost ---- */
/* MAP cost: generalized-Huber data term, N log(sigma^2)/2, and the prior over
 * the 13 causal spatial pairs plus the forward temporal pair
 * (XT_ICD_update.c:186-319). */
double orc_cost(void *h, double *forward, double *prior, double *errsino)
{
	orc_t *c = (orc_t *)h;
	size_t o, n = (size_t)c->N_p * c->N_r * c->N_t;
	double cost = 0, t, tp = 0, dl, fw;
	int i, p, j, k, Nz = c->N_z + 1, jm, km, pp, ip, jp, kp;
	const double sQ = c->sSQ, sQP = c->sSQP, cs = c->c_s;
	for (o = 0; o < n; o++) {
		t = c->e[o] * sqrt(c->w[o]);
		if (c->sel[o])
			t = t * t;
		else
			t = 2.0 * c->hdelta * c->hT * fabs(t) + c->hT * c->hT * (1.0 - 2.0 * c->hdelta);
		cost += t;
	}
	cost /= 2.0;
#define X(a, b, cc, d) (c->obj[OBJ(c, a, b, cc, d)])
#define SP(f, dd) tp += c->SF f * orc_rho(dd, sQ, sQP, cs)
	for (i = 0; i < c->N_time; i++)
		for (p = 1; p < c->N_z + 1; p++)
			for (j = 0; j < c->N_y; j++)
				for (k = 0; k < c->N_x; k++) {
					jm = j - 1 >= 0; km = k - 1 >= 0;
					pp = p + 1 < Nz; ip = i + 1 < c->N_time; jp = j + 1 < c->N_y; kp = k + 1 < c->N_x;
					if (kp) { dl = X(i, p, j, k) - X(i, p, j, k + 1); SP([1][1][2], dl); }
					if (jp) {
						if (km) { dl = X(i, p, j, k) - X(i, p, j + 1, k - 1); SP([1][2][0], dl); }
						dl = X(i, p, j, k) - X(i, p, j + 1, k); SP([1][2][1], dl);
						if (kp) { dl = X(i, p, j, k) - X(i, p, j + 1, k + 1); SP([1][2][2], dl); }
					}
					if (pp) {
						if (jm) { dl = X(i, p, j, k) - X(i, p + 1, j - 1, k); SP([2][0][1], dl); }
						dl = X(i, p, j, k) - X(i, p + 1, j, k); SP([2][1][1], dl);
						if (jp) { dl = X(i, p, j, k) - X(i, p + 1, j + 1, k); SP([2][2][1], dl); }
						if (jm) {
							if (km) { dl = X(i, p, j, k) - X(i, p + 1, j - 1, k - 1); SP([2][0][0], dl); }
							if (kp) { dl = X(i, p, j, k) - X(i, p + 1, j - 1, k + 1); SP([2][0][2], dl); }
						}
						if (km) { dl = X(i, p, j, k) - X(i, p + 1, j, k - 1); SP([2][1][0], dl); }
						if (jp) {
							if (km) { dl = X(i, p, j, k) - X(i, p + 1, j + 1, k - 1); SP([2][2][0], dl); }
							if (kp) { dl = X(i, p, j, k) - X(i, p + 1, j + 1, k + 1); SP([2][2][2], dl); }
						}
						if (kp) { dl = X(i, p, j, k) - X(i, p + 1, j, k + 1); SP([2][1][2], dl); }
					}
					if (ip) {
						dl = X(i, p, j, k) - X(i + 1, p, j, k);
						tp += c->TF * orc_rho(dl, c->sTQ, c->sTQP, c->c_t);
					}
				}
#undef X
#undef SP
	c->err_cost = cost;
	fw = cost + (double)1 * (double)c->N_p * (double)c->N_r * (double)c->N_t * log(c->var_est) / 2;
	c->fwd_cost = fw;
	c->prior_cost = tp;
	if (forward) *forward = fw;
	if (prior) *prior = tp;
	if (errsino) *errsino = cost;
	return fw + tp;
}

/* ------------------------------------------------------- stage set-up ---- */
/* Mask, detector response and error sinogram of a stage
 * (XT_ICD_update.c:1140-1159). */
int orc_prepare(void *h, const float *object, const float *offset)
{
	orc_t *c = (orc_t *)h;
	int i, j, k, s;
	double x, y;
	for (i = 0; i < c->N_time; i++)
		for (j = 0; j < c->N_y; j++)
			for (k = 0; k < c->N_x; k++) {
				x = c->x0 + ((double)k + 0.5) * c->delta_xy;
				y = c->y0 + ((double)j + 0.5) * c->delta_xy;
				c->mask[((size_t)i * c->N_y + j) * c->N_x + k] = (x * x + y * y < c->radius_obj * c->radius_obj);
			}
	orc_detector_response(c);
	if (object)
		for (i = 0; i < c->N_time; i++)
			for (s = 0; s < c->N_z; s++)
				for (j = 0; j < c->N_y; j++)
					for (k = 0; k < c->N_x; k++)
						c->obj[OBJ(c, i, s + 1, j, k)] =
						    object[(((size_t)i * c->N_z + s) * c->N_y + j) * c->N_x + k];
	if (offset)
		for (i = 0; i < c->N_r * c->N_t; i++)
			c->d[i] = offset[i];
	orc_error_sino(c);
	return 0;
}

/* --------------------------------------------------------- iteration ----- */
static double orc_half(orc_t *c, int j, int second, int nhicd, int iter)
{
	int i, b, idx, zs, ze, per = (int)floor(c->N_z / c->nblk), b0, b1, num;
	double tot = 0;
	for (i = 0; i < c->N_time; i++)
		for (b = 0; b < c->nblk; b += 2) {
			if (!second)
				idx = (i % 2 == 0) ? b : b + 1;
			else
				idx = (i % 2 == 0) ? b + 1 : b;
			zs = idx * per;
			ze = (idx + 1) * per - 1;
			ze = (idx >= c->nblk - 1) ? c->N_z - 1 : ze;
			if (!nhicd) {
				num = c->nr[(size_t)i * c->nblk + idx];
				b0 = j * (num / c->K);
				b1 = (j + 1) * (num / c->K) - 1;
				b1 = (j == c->K - 1) ? num - 1 : b1;
				tot += orc_update_lines(c, i, zs, ze, b0, b1, c->xr + SEL(c, i, idx), c->yr + SEL(c, i, idx),
				                        iter, c->mag + MAG(c, i, idx, 0, 0));
			} else {
				num = c->nn[(size_t)i * c->nblk + idx];
				orc_update_lines(c, i, zs, ze, 0, num - 1, c->xn + SEL(c, i, idx), c->yn + SEL(c, i, idx),
				                 iter, c->mag + MAG(c, i, idx, 0, 0));
			}
		}
	return tot;
}

/* One outer ICD iteration: K = 10 sub-iterations, each two checkerboard HICD
 * half-sweeps over (frame, z-block), ring-offset updates after every
 * half-sweep, NHICD selection and (from the second iteration) two NHICD
 * half-sweeps; then the variance update and the convergence test
 * (XT_ICD_update.c:936-1105).  Returns 1 when converged. */
int orc_iterate(void *h, int iter)
{
	orc_t *c = (orc_t *)h;
	int i, b, j;
	double vox = 0, avg = 0;
	orc_random_select(c);
	for (j = 0; j < c->K; j++) {
		vox = 0.0;
		vox += orc_half(c, j, 0, 0, iter);
		if (c->upd_offset > 1)
			orc_offset_update(c);
		vox += orc_half(c, j, 1, 0, iter);
		if (c->upd_offset > 1)
			orc_offset_update(c);
		orc_vsc_select(c);
		if (iter > 1) {
			orc_half(c, j, 0, 1, iter);
			if (c->upd_offset > 1)
				orc_offset_update(c);
			orc_half(c, j, 1, 1, iter);
			if (c->upd_offset > 1)
				orc_offset_update(c);
		}
	}
	if (c->upd_var == 1)
		orc_variance_update(c);
	for (i = 0; i < c->N_time; i++)
		for (b = 0; b < c->nblk; b++) {
			int n = c->nr[(size_t)i * c->nblk + b];
			const int *xs = c->xr + SEL(c, i, b), *ys = c->yr + SEL(c, i, b);
			for (j = 0; j < n; j++)
				avg += c->mag[MAG(c, i, b, ys[j], xs[j])];
		}
	c->last_pct = 100 * avg / vox;
	return c->last_pct < c->stop_thresh ? 1 : 0;
}

/* ----------------------------------------------------------- accessors --- */
void orc_dims(void *h, int *d)
{
	orc_t *c = (orc_t *)h;
	d[0] = c->N_p; d[1] = c->N_r; d[2] = c->N_t; d[3] = c->N_x; d[4] = c->N_y; d[5] = c->N_z;
	d[6] = c->N_time; d[7] = c->nblk; d[8] = c->z_overlap;
}
void orc_scalars(void *h, double *s)
{
	orc_t *c = (orc_t *)h;
	int i, j, k;
	s[0] = c->delta_r; s[1] = c->R0; s[2] = c->RMax; s[3] = c->OffsetR;
	s[4] = c->x0; s[5] = c->y0; s[6] = c->delta_xy; s[7] = c->radius_obj;
	s[8] = c->sSQ; s[9] = c->sSQP; s[10] = c->sTQ; s[11] = c->sTQP;
	s[12] = c->c_s; s[13] = c->c_t; s[14] = c->TF; s[15] = c->var_est;
	s[16] = c->hT; s[17] = c->hdelta; s[18] = c->delta_recon; s[19] = c->alpha;
	for (i = 0; i < 3; i++)
		for (j = 0; j < 3; j++)
			for (k = 0; k < 3; k++)
				s[20 + 9 * i + 3 * j + k] = c->SF[i][j][k];
}
void orc_view_map(void *h, int frame, int *num, int *idx)
{
	orc_t *c = (orc_t *)h;
	*num = c->vnum[frame];
	if (idx)
		memcpy(idx, c->vidx[frame], sizeof(int) * c->vnum[frame]);
}
void orc_get_object(void *h, float *out)
{
	orc_t *c = (orc_t *)h;
	int i, s;
	size_t j, n = (size_t)c->N_y * c->N_x;
	for (i = 0; i < c->N_time; i++)
		for (s = 0; s < c->N_z; s++)
			for (j = 0; j < n; j++)
				out[((size_t)i * c->N_z + s) * n + j] = (float)c->obj[OBJ(c, i, s + 1, 0, 0) + j];
}
void orc_get_errorsino(void *h, float *out)
{
	orc_t *c = (orc_t *)h;
	size_t i, n = (size_t)c->N_p * c->N_r * c->N_t;
	for (i = 0; i < n; i++)
		out[i] = (float)c->e[i];
}
void orc_get_weight(void *h, float *out)
{
	orc_t *c = (orc_t *)h;
	size_t i, n = (size_t)c->N_p * c->N_r * c->N_t;
	for (i = 0; i < n; i++)
		out[i] = (float)c->w[i];
}
void orc_get_projselect(void *h, uint8_t *out)
{
	orc_t *c = (orc_t *)h;
	memcpy(out, c->sel, (size_t)c->N_p * c->N_r * c->N_t);
}
void orc_get_offset(void *h, float *out)
{
	orc_t *c = (orc_t *)h;
	size_t i;
	for (i = 0; i < (size_t)c->N_r * c->N_t; i++)
		out[i] = (float)c->d[i];
}
void orc_get_magmap(void *h, float *out)
{
	orc_t *c = (orc_t *)h;
	size_t i, n = (size_t)c->N_time * c->nblk * c->N_y * c->N_x;
	for (i = 0; i < n; i++)
		out[i] = (float)c->mag[i];
}
void orc_set_magmap(void *h, const float *in)
{
	orc_t *c = (orc_t *)h;
	size_t i, n = (size_t)c->N_time * c->nblk * c->N_y * c->N_x;
	for (i = 0; i < n; i++)
		c->mag[i] = in[i];
}
void orc_get_hr(void *h, float *out)
{
	orc_t *c = (orc_t *)h;
	memcpy(out, c->H_r, sizeof(float) * (size_t)c->N_p * (RESP_BINS + 1));
}
void orc_get_mask(void *h, uint8_t *out)
{
	orc_t *c = (orc_t *)h;
	memcpy(out, c->mask, (size_t)c->N_time * c->N_y * c->N_x);
}
int orc_get_lines(void *h, int kind, int frame, int block, int *xs, int *ys)
{
	orc_t *c = (orc_t *)h;
	int n = kind == 0 ? c->nr[(size_t)frame * c->nblk + block] : c->nn[(size_t)frame * c->nblk + block];
	const int *sx = (kind == 0 ? c->xr : c->xn) + SEL(c, frame, block);
	const int *sy = (kind == 0 ? c->yr : c->yn) + SEL(c, frame, block);
	memcpy(xs, sx, sizeof(int) * n);
	memcpy(ys, sy, sizeof(int) * n);
	return n;
}
void orc_set_lines(void *h, int frame, int block, int n, const int *xs, const int *ys)
{
	orc_t *c = (orc_t *)h;
	c->nr[(size_t)frame * c->nblk + block] = n;
	memcpy(c->xr + SEL(c, frame, block), xs, sizeof(int) * n);
	memcpy(c->yr + SEL(c, frame, block), ys, sizeof(int) * n);
}
double orc_var_est(void *h) { return ((orc_t *)h)->var_est; }
int orc_num_z_blocks(void *h) { return ((orc_t *)h)->nblk; }
double orc_last_update_percentage(void *h) { return ((orc_t *)h)->last_pct; }
long long orc_update_count(void *h) { return ((orc_t *)h)->updates; }
