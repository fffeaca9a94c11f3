// Host-side set-up arithmetic of one reconstruction stage (FP64), and the
// Park-Miller generator that orders voxel lines.  Declarations shared by
// mbir_setup.cpp, mbir_stage.cu and mbir_reconstruct.cpp.
#pragma once
#include <cstdint>
#include <vector>

namespace mbir {

// Park-Miller minimal standard generator: x' = 16807 x mod (2^31 - 1),
// returned as x' / (2^31 - 1) in (0, 1] (TIMBIR randlib.c:119-141).  One
// stream runs through a whole reconstruct() call, seeded with 761521
// (XT_Engine.c:99).
struct ParkMiller {
    uint32_t state = 761521u;
    double next()
    {
        state = (uint32_t)(((uint64_t)state * 16807u) % 2147483647u);
        return (double)state / 2147483647.0;
    }
};

// Static geometry of a scan (initStatStructures, XT_Init.c:449-669).
struct ScanGeom {
    int N_p, N_r, N_t, N_time;
    double delta_r, delta_t, R0, RMax, T0, rot_center, radius_obj, y0;
    std::vector<float> angles, ptimes, rtimes;
    std::vector<double> cosv, sinv;
    std::vector<std::vector<int>> views;  // views of each frame
    std::vector<int> frame_of_view;       // -1 for a view in no frame
    double delta_recon;
};

// Per-stage geometry and prior constants (initDynStructures, XT_Init.c:211-445).
struct StageGeom {
    double mult_xy, mult_z, delta_xy, delta_z, OffsetR, x0;
    int N_x, N_y, N_z, m_z;
    double sSQ, sSQP, sTQ, sTQP, SF[27], TF;
};

int scan_geom(ScanGeom &sg, const float *angles, const float *ptimes, const float *rtimes,
              int proj_rows, int proj_cols, int proj_num, int recon_num, float vox_wid,
              float rot_center, char *err, int errlen);
void stage_geom(const ScanGeom &sg, StageGeom &st, int mult_xy, int mult_z, double sig_s,
                double sig_t);
void detector_response_params(const ScanGeom &sg, const StageGeom &st, std::vector<double> &trap,
                              std::vector<double> &beam, double &r0, double &step, double &tc);
void object_mask(const ScanGeom &sg, const StageGeom &st, std::vector<uint8_t> &mask);
int z_blocks_for_threads(int threads, int n_time, int n_z);

// Random permutation of the in-mask lines of one (frame, z-block), one draw
// per element (XT_ICD_update.c:500-532).  Returns the number of lines.
int random_lines(ParkMiller &rng, const uint8_t *mask, int N_y, int N_x, int slices_in_block,
                 int *xs, int *ys);
// i-th smallest (1-based) of a[0..n-1] by randomised quickselect with the
// reference's partition and pivot draws (XT_NHICD.c:63-126).  Reorders a.
double order_statistic(ParkMiller &rng, float *a, uint32_t n, uint32_t i);

// Bilinear x2 up-sampling used between resolution stages
// (XT_ICD_update.c:323-498).  Shapes are [n_z][n_y][n_x] of the input.
void upsample_xy(const float *in, float *out, int n_z, int n_y, int n_x);
void upsample_xyz(const float *in, float *out, int n_z, int n_y, int n_x);

}  // namespace mbir

// The prologue of a stage that follows `prev` in one multi-resolution run,
// with the start object and magnitude map up-sampled from prev's on the
// device (mbir_stage.cu); *mag_carried = 1 when the magnitude map was carried.
struct MbirStage;
int mbir_icd_prepare_from(MbirStage *S, MbirStage *prev, int initICD, const float *offset, int *mag_carried);
