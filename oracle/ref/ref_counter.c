/*
 * Call counter and iteration clock for the reference driver binary
 * (oracle/_ref/XT_Main_ref).  The reference sources are compiled unmodified;
 * XT_VoxUpdate.c and XT_ICD_update.c are compiled with -finstrument-functions
 * so that every entry/exit of their functions calls the two hooks below.
 *
 *  - compute_voxel_update_Atten (src/MBIR_4D/XT_VoxUpdate.c:43) is called
 *    exactly once per voxel update that is not zero-skipped, so its entry count
 *    is the voxel-update count of the metric;
 *  - updateVoxelsTimeSlices (src/MBIR_4D/XT_ICD_update.c:936) is one outer ICD
 *    iteration; its exit time stamps the iteration.
 *
 * On each iteration exit one line goes to stderr:
 *   ORACLE_ITER <n> <seconds in this iteration> <voxel updates in this iteration>
 * If ORACLE_MAX_ITERS is set, the process exits (status 0) after that many
 * iterations, which bounds the CPU-baseline sample.  Test infrastructure only.
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include <time.h>
#include <unistd.h>

#define NOINST __attribute__((no_instrument_function))

void compute_voxel_update_Atten(void);
int updateVoxelsTimeSlices(void);

static long long g_updates = 0, g_updates_at_start = 0;
static int g_iter = 0, g_max_iters = -1, g_init = 0;
static double g_t_start = 0.0;

static NOINST double now_s(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

NOINST void __cyg_profile_func_enter(void *fn, void *site)
{
	(void)site;
	if (fn == (void *)compute_voxel_update_Atten) {
		__atomic_fetch_add(&g_updates, 1, __ATOMIC_RELAXED);
	} else if (fn == (void *)updateVoxelsTimeSlices) {
		if (!g_init) {
			const char *m = getenv("ORACLE_MAX_ITERS");
			g_max_iters = m ? atoi(m) : -1;
			g_init = 1;
		}
		g_updates_at_start = __atomic_load_n(&g_updates, __ATOMIC_RELAXED);
		g_t_start = now_s();
	}
}

NOINST void __cyg_profile_func_exit(void *fn, void *site)
{
	(void)site;
	if (fn == (void *)updateVoxelsTimeSlices) {
		double dt = now_s() - g_t_start;
		long long n = __atomic_load_n(&g_updates, __ATOMIC_RELAXED) - g_updates_at_start;
		g_iter++;
		fprintf(stderr, "ORACLE_ITER %d %.6f %lld\n", g_iter, dt, n);
		fflush(stderr);
		if (g_max_iters > 0 && g_iter >= g_max_iters) {
			fflush(stdout);
			_exit(0);
		}
	}
}
