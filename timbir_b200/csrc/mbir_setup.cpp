// Host set-up arithmetic of the MBIR stages, in FP64 with the host C
// library's cos/sin/pow/sqrt so that the tables the kernels consume (view
// cosines, detector response, prior weights) carry the same bits as the
// reference's.  Reference: TIMBIR v0.0.2, src/MBIR_4D.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "mbir_host.h"

namespace mbir {

static const double kP = 1.2, kQ = 2.0;
static const double kHalfPi = 1.57079632679489661923132169163975144;
static const double kQuarterPi = 0.785398163397448309615660845819875721;
static const double kPi = 3.14159265358979323846;
static const int kProfileRes = 1536, kBeamRes = 512, kRespBins = 64;

// initStatStructures + initRandomAngles + calculateSinCos
// (XT_Init.c:449-669, 100-137, 69-96, 193-206).
int scan_geom(ScanGeom &sg, const float *angles, const float *ptimes, const float *rtimes,
              int proj_rows, int proj_cols, int proj_num, int recon_num, float vox_wid,
              float rot_center, char *err, int errlen)
{
    const double len_r = (double)vox_wid * proj_cols, len_t = (double)vox_wid * proj_rows;
    sg.N_p = proj_num;
    sg.N_r = proj_cols;
    sg.N_t = proj_rows;
    sg.N_time = recon_num;
    sg.rot_center = rot_center;
    sg.radius_obj = (double)vox_wid * proj_cols / 2;
    sg.delta_r = len_r / sg.N_r;
    sg.delta_t = len_t / sg.N_t;
    sg.R0 = -sg.rot_center * sg.delta_r;
    sg.RMax = (sg.N_r - sg.rot_center) * sg.delta_r;
    sg.T0 = -len_t / 2.0;
    sg.y0 = -len_r / 2.0;
    sg.angles.assign(angles, angles + proj_num);
    sg.ptimes.assign(ptimes, ptimes + proj_num);
    sg.rtimes.assign(rtimes, rtimes + recon_num + 1);
    for (int i = 0; i + 1 < proj_num; i++)
        if (ptimes[i + 1] < ptimes[i]) {
            snprintf(err, errlen, "Projection acquisition time decreased for increasing index.");
            return -1;
        }
    for (int i = 0; i < recon_num; i++)
        if (rtimes[i + 1] < rtimes[i]) {
            snprintf(err, errlen, "Reconstruction times decreased for increasing index.");
            return -1;
        }
    // half-open windows [rt_i, rt_{i+1}); the scan for frame i resumes at the
    // first view that ended frame i-1
    sg.views.assign(recon_num, {});
    sg.frame_of_view.assign(proj_num, -1);
    int start = 0;
    double total = 0;
    for (int i = 0; i < recon_num; i++) {
        for (int j = start; j < proj_num; j++) {
            const double t = ptimes[j];
            if (t >= rtimes[i] && t < rtimes[i + 1]) {
                sg.views[i].push_back(j);
                sg.frame_of_view[j] = i;
            }
            if (t >= rtimes[i + 1]) {
                start = j;
                break;
            }
        }
        total += (double)sg.views[i].size();
    }
    sg.delta_recon = total / recon_num;
    sg.cosv.resize(proj_num);
    sg.sinv.resize(proj_num);
    for (int i = 0; i < proj_num; i++) {
        sg.cosv[i] = cos((double)angles[i]);
        sg.sinv[i] = sin((double)angles[i]);
    }
    return 0;
}

static double node_distance(int i, int j, int k, int l)
{
    return sqrt(pow((double)i - 1.0, 2.0) + pow((double)j - 1.0, 2.0) + pow((double)k - 1.0, 2.0) +
                pow((double)l - 1.0, 2.0));
}

// initDynStructures' geometry, sigma scaling and initFilter
// (XT_Init.c:339-345, 383-387, 431-435, 144-190).
void stage_geom(const ScanGeom &sg, StageGeom &st, int mult_xy, int mult_z, double sig_s, double sig_t)
{
    st.mult_xy = mult_xy;
    st.mult_z = mult_z;
    st.N_x = (int)(sg.N_r / st.mult_xy);
    st.N_y = (int)(sg.N_r / st.mult_xy);
    st.N_z = (int)(sg.N_t / st.mult_z);
    st.delta_xy = st.mult_xy * sg.delta_r;
    st.delta_z = st.mult_z * sg.delta_t;
    st.m_z = mult_z;
    st.x0 = sg.R0;
    st.OffsetR = (st.delta_xy / sqrt(2.0) + sg.delta_r / 2.0) / kRespBins;
    st.sSQ = pow(sig_s * st.mult_xy, kQ);
    st.sSQP = pow(sig_s * st.mult_xy, kQ - kP);
    st.sTQ = pow(sig_t * sg.delta_recon, kQ);
    st.sTQP = pow(sig_t * sg.delta_recon, kQ - kP);
    const double pc = st.mult_xy * st.mult_xy * st.mult_xy * sg.delta_recon;
    double sum = 0;
    st.TF = 1.0 / node_distance(0, 1, 1, 1);
    sum += 2.0 * st.TF;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++) {
                const int n = 9 * a + 3 * b + c;
                if (n != 13) {
                    st.SF[n] = 1.0 / node_distance(1, a, b, c);
                    sum = sum + st.SF[n];
                } else
                    st.SF[n] = 0;
            }
    for (int n = 0; n < 27; n++) st.SF[n] = pc * st.SF[n] / sum;
    st.TF = pc * st.TF / sum;
}

// Host half of the detector response H_r[view][0..64] (XT_Profile.c:47-170):
// the quantities that need the host C library's cos -- per view the
// trapezoid's height and corners (maxv, lc, ln, rn, rc), and the normalised
// 512-point Hamming beam -- so that the GPU half (k_detector_response), which
// samples the trapezoid and convolves it with the beam in the reference's
// operation order, produces the reference's bits.
void detector_response_params(const ScanGeom &sg, const StageGeom &st, std::vector<double> &trap,
                              std::vector<double> &beam, double &r0, double &step, double &tc)
{
    beam.assign(kBeamRes, 0.0);
    double sum = 0;
    for (int i = 0; i < kBeamRes; i++) {
        beam[i] = 0.54 - 0.46 * cos((2 * kPi / kBeamRes) * i);
        sum = sum + beam[i];
    }
    for (int i = 0; i < kBeamRes; i++) beam[i] /= sum;
    r0 = -sg.delta_r / 2;
    step = sg.delta_r / kBeamRes;
    tc = kProfileRes / (2 * st.delta_xy);
    trap.assign((size_t)sg.N_p * 5, 0.0);
    for (int k = 0; k < sg.N_p; k++) {
        double angle = sg.angles[k], maxv;
        while (angle > kHalfPi) angle -= kHalfPi;
        while (angle < 0) angle += kHalfPi;
        if (angle <= kQuarterPi)
            maxv = st.delta_xy / cos(angle);
        else
            maxv = st.delta_xy / cos(kHalfPi - angle);
        const double c45 = cos(kQuarterPi);
        const double d1 = c45 * cos((kQuarterPi - angle));
        const double d2 = c45 * fabs((cos((kQuarterPi + angle))));
        double *t = &trap[(size_t)k * 5];
        t[0] = maxv;
        t[1] = 1 - d1;  // left corner
        t[2] = 1 - d2;  // left near
        t[3] = 1 + d2;  // right near
        t[4] = 1 + d1;  // right corner
    }
}

// Voxel lines whose centre lies inside the detector's field of view
// (XT_ICD_update.c:1140-1149).
void object_mask(const ScanGeom &sg, const StageGeom &st, std::vector<uint8_t> &mask)
{
    mask.assign((size_t)st.N_y * st.N_x, 0);
    for (int j = 0; j < st.N_y; j++)
        for (int k = 0; k < st.N_x; k++) {
            const double x = st.x0 + ((double)k + 0.5) * st.delta_xy;
            const double y = sg.y0 + ((double)j + 0.5) * st.delta_xy;
            mask[(size_t)j * st.N_x + k] = (x * x + y * y < sg.radius_obj * sg.radius_obj) ? 1 : 0;
        }
}

// XT_Init.c:389-398.
int z_blocks_for_threads(int threads, int n_time, int n_z)
{
    int nb = threads / n_time;
    if (nb < 2)
        nb = 2;
    else if (nb > n_z)
        nb = n_z;
    return (nb / 2) * 2;
}

int random_lines(ParkMiller &rng, const uint8_t *mask, int N_y, int N_x, int slices_in_block, int *xs,
                 int *ys)
{
    const int total = N_y * N_x;
    std::vector<int> pool(total);
    for (int i = 0; i < total; i++) pool[i] = i;
    int size = total, n = 0;
    for (int j = 0; j < total; j++) {
        int idx = (int)floor(rng.next() * size);
        idx = (idx == size) ? size - 1 : idx;
        const int col = pool[idx] % N_x, row = pool[idx] / N_x;
        if (slices_in_block > 0 && mask[(size_t)row * N_x + col] == 1) {
            xs[n] = col;
            ys[n] = row;
            n++;
        }
        pool[idx] = pool[size - 1];
        size--;
    }
    return n;
}

double order_statistic(ParkMiller &rng, float *A, uint32_t n, uint32_t i)
{
    uint32_t p = 0, r = n - 1;
    for (;;) {
        if (p == r) return A[p];
        uint32_t rnum = (uint32_t)floor(rng.next() * (r - p + 1));
        rnum = (rnum == r - p + 1) ? r - p : rnum;
        std::swap(A[r], A[p + rnum]);
        const float x = A[r];
        uint32_t s = p - 1;
        for (uint32_t j = p; j < r; j++)
            if (A[j] <= x) {
                s++;
                std::swap(A[s], A[j]);
            }
        std::swap(A[s + 1], A[r]);
        const uint32_t q = s + 1, k = q - p + 1;
        if (i == k) return A[q];
        if (i < k)
            r = q - 1;
        else {
            p = q + 1;
            i -= k;
        }
    }
}

// x-y doubling of one slice into a float row buffer, then y doubling
// (upsample_object_bilinear_2D, XT_ICD_update.c:358-389).
void upsample_xy(const float *in, float *out, int n_z, int n_y, int n_x)
{
    const int ox = 2 * n_x, oy = 2 * n_y;
    std::vector<float> b((size_t)n_y * ox);
    for (int s = 0; s < n_z; s++) {
        const float *I = in + (size_t)s * n_y * n_x;
        float *O = out + (size_t)s * oy * ox;
        for (int j = 0; j < n_y; j++) {
            const float *r = I + (size_t)j * n_x;
            float *B = &b[(size_t)j * ox];
            B[0] = r[0];
            B[1] = (3.0 * r[0] + r[1]) / 4.0;
            B[ox - 1] = r[n_x - 1];
            B[ox - 2] = (r[n_x - 2] + 3.0 * r[n_x - 1]) / 4.0;
            for (int k = 1; k < n_x - 1; k++) {
                B[2 * k] = (r[k - 1] + 3.0 * r[k]) / 4.0;
                B[2 * k + 1] = (3.0 * r[k] + r[k + 1]) / 4.0;
            }
        }
        for (int k = 0; k < ox; k++) {
            O[k] = b[k];
            O[ox + k] = (3.0 * b[k] + b[ox + k]) / 4.0;
            O[(size_t)(oy - 1) * ox + k] = b[(size_t)(n_y - 1) * ox + k];
            O[(size_t)(oy - 2) * ox + k] = (b[(size_t)(n_y - 2) * ox + k] + 3.0 * b[(size_t)(n_y - 1) * ox + k]) / 4.0;
        }
        for (int j = 1; j < n_y - 1; j++)
            for (int k = 0; k < ox; k++) {
                const float bm = b[(size_t)(j - 1) * ox + k], b0 = b[(size_t)j * ox + k], bp = b[(size_t)(j + 1) * ox + k];
                O[(size_t)(2 * j) * ox + k] = (bm + 3.0 * b0) / 4.0;
                O[(size_t)(2 * j + 1) * ox + k] = (3 * b0 + bp) / 4.0;  // float arithmetic, as the reference
            }
    }
}

// x, y and z doubling with FP64 intermediate buffers
// (upsample_object_bilinear_3D, XT_ICD_update.c:437-498).
void upsample_xyz(const float *in, float *out, int n_z, int n_y, int n_x)
{
    const int ox = 2 * n_x, oy = 2 * n_y;
    std::vector<double> b2((size_t)n_z * n_y * ox), b3((size_t)n_z * oy * ox);
    for (int s = 0; s < n_z; s++) {
        for (int j = 0; j < n_y; j++) {
            const float *r = in + ((size_t)s * n_y + j) * n_x;
            double *B = &b2[((size_t)s * n_y + j) * ox];
            B[0] = r[0];
            B[1] = (3.0 * r[0] + r[1]) / 4.0;
            B[ox - 1] = r[n_x - 1];
            B[ox - 2] = (r[n_x - 2] + 3.0 * r[n_x - 1]) / 4.0;
            for (int k = 1; k < n_x - 1; k++) {
                B[2 * k] = (r[k - 1] + 3.0 * r[k]) / 4.0;
                B[2 * k + 1] = (3.0 * r[k] + r[k + 1]) / 4.0;
            }
        }
        const double *B = &b2[(size_t)s * n_y * ox];
        double *C = &b3[(size_t)s * oy * ox];
        for (int k = 0; k < ox; k++) {
            C[k] = B[k];
            C[ox + k] = (3.0 * B[k] + B[ox + k]) / 4.0;
            C[(size_t)(oy - 1) * ox + k] = B[(size_t)(n_y - 1) * ox + k];
            C[(size_t)(oy - 2) * ox + k] = (B[(size_t)(n_y - 2) * ox + k] + 3.0 * B[(size_t)(n_y - 1) * ox + k]) / 4.0;
        }
        for (int j = 1; j < n_y - 1; j++)
            for (int k = 0; k < ox; k++) {
                C[(size_t)(2 * j) * ox + k] = (B[(size_t)(j - 1) * ox + k] + 3.0 * B[(size_t)j * ox + k]) / 4.0;
                C[(size_t)(2 * j + 1) * ox + k] = (3 * B[(size_t)j * ox + k] + B[(size_t)(j + 1) * ox + k]) / 4.0;
            }
    }
    const size_t pl = (size_t)oy * ox;
    for (size_t q = 0; q < pl; q++) {
        out[q] = b3[q];
        out[pl + q] = (3.0 * b3[q] + b3[pl + q]) / 4.0;
        out[(size_t)(2 * n_z - 1) * pl + q] = b3[(size_t)(n_z - 1) * pl + q];
        out[(size_t)(2 * n_z - 2) * pl + q] = (3.0 * b3[(size_t)(n_z - 1) * pl + q] + b3[(size_t)(n_z - 2) * pl + q]) / 4.0;
    }
    for (int s = 1; s < n_z - 1; s++)
        for (size_t q = 0; q < pl; q++) {
            out[(size_t)(2 * s) * pl + q] = (b3[(size_t)(s - 1) * pl + q] + 3.0 * b3[(size_t)s * pl + q]) / 4.0;
            out[(size_t)(2 * s + 1) * pl + q] = (3.0 * b3[(size_t)s * pl + q] + b3[(size_t)(s + 1) * pl + q]) / 4.0;
        }
}

}  // namespace mbir
