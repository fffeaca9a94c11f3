/*
 * Drop-in replacement for the reference library's public call.
 *
 * reconstruct() replaces TIMBIR v0.0.2 src/include/mbir4d.h:35
 * (implemented at src/MBIR_4D/XT_Engine.c:81).  Same signature, same
 * argument meaning, same preconditions (XT_Engine.c:101-104), same outputs in
 * the current working directory (object_time_<t>.bin, proj_offset.bin,
 * variance_estimate.bin, mag_update.bin, status.bin, projs_runtime.bin,
 * weights_runtime.bin), same ownership: it free()s projections, weights,
 * proj_angles, proj_times and recon_times, and does not write *object.
 * Returns 0 on success and -1 on failure, with an "[ERROR]" line written to
 * debug_msg_ptr.  The work runs on the current CUDA device.
 *
 * Unlike the reference's header, this one includes what it needs.
 */
#ifndef MBIR4D_H_
#define MBIR4D_H_
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

int reconstruct(float **object, float *projections, float *weights, float *proj_angles,
                float *proj_times, float *recon_times, int32_t proj_rows, int32_t proj_cols,
                int32_t proj_num, int32_t recon_num, float vox_wid, float rot_center, float sig_s,
                float sig_t, float c_s, float c_t, float convg_thresh, int32_t remove_rings,
                int32_t quad_convex, float huber_delta, float huber_T, uint8_t restart,
                FILE *debug_msg_ptr);

#ifdef __cplusplus
}
#endif
#endif
