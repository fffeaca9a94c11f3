// reconstruct(): the drop-in library call (TIMBIR v0.0.2 src/include/mbir4d.h:35,
// src/MBIR_4D/XT_Engine.c:81-203) running every stage on the GPU.
//
// The multi-resolution schedule, the per-stage switches, the restart files
// and the output files follow the reference; each stage's ICD runs through
// the stage-level C ABI (include/timbir_b200.h).
//
// Environment knobs (none needed for drop-in use):
//   TIMBIR_COMPUTE_COST=1     evaluate the MAP cost each iteration, append it
//                             to cost.bin and stop with an error if it rises,
//                             as the reference does when built without
//                             -DNO_COST_CALCULATE (its shipped build omits it).
//   TIMBIR_MAX_ITERS=n        cap on ICD iterations per stage (default 1000,
//                             MAX_NUM_ITERATIONS of XT_Constants.h:86).
//   TIMBIR_Z_BLOCK_THREADS=n  thread count fed to the reference's z-block rule
//                             (XT_Init.c:389-398); default: as many z-blocks as
//                             the stage allows (reference schedule only).
//   TIMBIR_SCHEDULE=reference the reference's voxel-update schedule on the GPU
//                             (checkerboard z-block tasks, random line order,
//                             exactly updateVoxelsTimeSlices); default: the
//                             super-voxel schedule, which reaches the same MAP
//                             estimate far faster.
//   TIMBIR_SV_SIDE=n          super-voxel side (default: largest that fits).
//   TIMBIR_SV_ACACHE=m        A-matrix column cache of the super-voxel
//                             schedule: -1 when it fits (default), 0 never,
//                             1 always.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <memory>
#include <vector>

#include "../../include/mbir4d.h"
#include "../../include/timbir_b200.h"
#include "mbir_host.h"

using namespace mbir;

#define LOG_INFO(fp, ...)                                                                      \
    do {                                                                                       \
        if (fp) {                                                                              \
            fprintf(fp, "[INFO] (%s:%d) ", __FILE__, __LINE__);                               \
            fprintf(fp, __VA_ARGS__);                                                          \
        }                                                                                      \
    } while (0)
#define LOG_ERR(fp, ...)                                                                       \
    do {                                                                                       \
        if (fp) {                                                                              \
            fprintf(fp, "[ERROR] (%s:%d) ", __FILE__, __LINE__);                              \
            fprintf(fp, __VA_ARGS__);                                                          \
            fflush(fp);                                                                        \
        }                                                                                      \
    } while (0)

static int write_bin(const char *name, const void *data, size_t elsize, size_t n)
{
    char file[256];
    snprintf(file, sizeof(file), "%s.bin", name);
    FILE *f = fopen(file, "wb");
    if (!f) return -1;
    const size_t w = fwrite(data, elsize, n, f);
    fclose(f);
    return w == n ? 0 : -1;
}

static int append_bin(const char *name, const void *data, size_t elsize, size_t n)
{
    char file[256];
    snprintf(file, sizeof(file), "%s.bin", name);
    FILE *f = fopen(file, "ab");
    if (!f) return -1;
    const size_t w = fwrite(data, elsize, n, f);
    fclose(f);
    return w == n ? 0 : -1;
}

static int read_bin(const char *name, void *data, size_t elsize, size_t n)
{
    char file[256];
    snprintf(file, sizeof(file), "%s.bin", name);
    FILE *f = fopen(file, "rb");
    if (!f) return -1;
    const size_t r = fread(data, elsize, n, f);
    fclose(f);
    return r == n ? 0 : -1;
}

static int env_int(const char *name, int dflt)
{
    const char *v = getenv(name);
    return (v && *v) ? atoi(v) : dflt;
}

namespace {
struct Inputs {
    float *projections, *weights, *angles, *ptimes, *rtimes;
    void release()
    {
        free(projections);
        free(weights);
        projections = weights = nullptr;
    }
    void release_all()
    {
        release();
        free(angles);
        free(ptimes);
        free(rtimes);
        angles = ptimes = rtimes = nullptr;
    }
};
}  // namespace

extern "C" int reconstruct(float **object, float *projections, float *weights, float *proj_angles,
                           float *proj_times, float *recon_times, int32_t proj_rows, int32_t proj_cols,
                           int32_t proj_num, int32_t recon_num, float vox_wid, float rot_center,
                           float sig_s, float sig_t, float c_s, float c_t, float convg_thresh,
                           int32_t remove_rings, int32_t quad_convex, float huber_delta, float huber_T,
                           uint8_t restart, FILE *debug_msg_ptr)
{
    (void)object;  // the reference never writes *object (XT_Engine.c:178-179)
    FILE *log = debug_msg_ptr;
    Inputs in{projections, weights, proj_angles, proj_times, recon_times};
    const time_t start = time(nullptr);
    const int nodes = 1;
    LOG_INFO(log, "Reconstructing the data ....\n");
    // preconditions (XT_Engine.c:101-104)
    if (proj_rows % nodes != 0 || proj_rows < 4 || proj_cols % 2 != 0 ||
        (proj_rows / nodes) % 2 != 0 || proj_rows / nodes < 2) {
        LOG_ERR(log, "Invalid dimensions: proj_rows must be even and >= 4, proj_cols must be even.\n");
        return -1;
    }
    if (proj_num <= 0 || recon_num <= 0 || remove_rings < 0 || remove_rings > 3 || quad_convex < 0 ||
        quad_convex > 1) {
        LOG_ERR(log, "Invalid arguments.\n");
        return -1;
    }
    // multi-resolution schedule (XT_Engine.c:111-141)
    int multres = (int)(std::log(((float)proj_cols) / 64) / std::log(2.0) + 1);
    if (multres > 8) multres = 8;
    if (multres < 2) multres = 2;
    int mxy[8], mz[8];
    mxy[0] = 1;
    mz[0] = 1;
    for (int i = 1; i < multres; i++) {
        if (proj_cols % (mxy[i - 1] * 2) == 0) {
            mxy[i] = mxy[i - 1] * 2;
            if (proj_rows / nodes % (mz[i - 1] * 2) == 0 && proj_rows / nodes / (mz[i - 1] * 2) >= 2)
                mz[i] = mz[i - 1] * 2;
            else
                mz[i] = mz[i - 1];
        } else {
            multres = i;
            break;
        }
    }
    int sxy[8], sz[8];
    for (int i = 0; i < multres; i++) {
        sxy[i] = mxy[multres - 1 - i];
        sz[i] = mz[multres - 1 - i];
    }
    int last = 0;
    if (restart == 1 && read_bin("status", &last, sizeof(int32_t), 1)) {
        LOG_ERR(log, "Error in reading file status.bin.\n");
        return -1;
    }
    LOG_INFO(log, "Number of multi-resolution stages is %d.\n", multres);
    const int max_iters = env_int("TIMBIR_MAX_ITERS", 1000);
    const int want_cost = env_int("TIMBIR_COMPUTE_COST", 0);
    const int zthreads = env_int("TIMBIR_Z_BLOCK_THREADS", 1 << 20);
    const char *sched_env = getenv("TIMBIR_SCHEDULE");
    const int use_sv = !(sched_env && strcmp(sched_env, "reference") == 0);
    const int sv_side = env_int("TIMBIR_SV_SIDE", 0);
    const int sv_acache = env_int("TIMBIR_SV_ACACHE", -1);
    int prev_sv_blocks = -1;  // magnitude-map planes per frame of the previous stage (this call)
    uint32_t rng_state = 761521u;
    std::vector<float> carried_offset;  // ring offsets kept in memory between stages
    const size_t nsino = (size_t)proj_num * proj_rows * proj_cols;
    // the previous stage of this call, kept on the device until the next
    // stage has taken its object and magnitude map (freed on every exit)
    std::unique_ptr<MbirStage, void (*)(MbirStage *)> prev_stage(nullptr, mbir_free_stage);

    for (int i = last; i < multres; i++) {
        LOG_INFO(log, "Running multi-resolution stage %d with x-y voxel scale = %d and z voxel scale = %d.\n",
                 i, sxy[i], sz[i]);
        const int N_x = proj_cols / sxy[i], N_z = proj_rows / sz[i];
        // stage switches (XT_Init.c:230-266)
        int initICD = 0;
        if (i > 0) {
            if (sz[i] == sz[i - 1])
                initICD = 2;
            else if (sz[i - 1] / sz[i] == 2)
                initICD = 3;
        }
        int upd_offset = (i == 0) ? 0 : (i == 1 ? 2 : 3);
        if (remove_rings == 0) upd_offset = 0;
        const int upd_var = (i > 0 && quad_convex == 0) ? 1 : 0;
        const int init_mag = i > 0;
        double var_est = 1.0;
        if (i != 0 && read_bin("variance_estimate", &var_est, sizeof(double), 1)) {
            LOG_ERR(log, "Error in reading file variance_estimate.bin.\n");
            in.release_all();
            return -1;
        }
        // inputs: the caller's arrays for the stages of this call; a restarted
        // call's first stage reads the runtime copies (reference layout
        // [view][col][row], XT_Init.c:296-315) as the reference does
        std::vector<float> pr_in, wt_in;
        const float *P = projections, *W = weights;
        if (i != 0 && i == last) {
            std::vector<float> a(nsino), b(nsino);
            if (read_bin("projs_runtime", a.data(), sizeof(float), nsino) ||
                read_bin("weights_runtime", b.data(), sizeof(float), nsino)) {
                LOG_ERR(log, "Error in reading the runtime projection/weight files.\n");
                in.release_all();
                return -1;
            }
            pr_in.resize(nsino);
            wt_in.resize(nsino);
            for (int p = 0; p < proj_num; p++)
                for (int r = 0; r < proj_cols; r++)
                    for (int t = 0; t < proj_rows; t++) {
                        pr_in[((size_t)p * proj_rows + t) * proj_cols + r] = a[((size_t)p * proj_cols + r) * proj_rows + t];
                        wt_in[((size_t)p * proj_rows + t) * proj_cols + r] = b[((size_t)p * proj_cols + r) * proj_rows + t];
                    }
            P = pr_in.data();
            W = wt_in.data();
        } else if (i == 0) {
            std::vector<float> a(nsino), b(nsino);
            for (int p = 0; p < proj_num; p++)
                for (int t = 0; t < proj_rows; t++)
                    for (int r = 0; r < proj_cols; r++) {
                        a[((size_t)p * proj_cols + r) * proj_rows + t] = projections[((size_t)p * proj_rows + t) * proj_cols + r];
                        b[((size_t)p * proj_cols + r) * proj_rows + t] = weights[((size_t)p * proj_rows + t) * proj_cols + r];
                    }
            if (write_bin("weights_runtime", b.data(), sizeof(float), nsino) ||
                write_bin("projs_runtime", a.data(), sizeof(float), nsino)) {
                LOG_ERR(log, "Error in writing the runtime projection/weight files.\n");
                in.release_all();
                return -1;
            }
        }
        const int nblk = z_blocks_for_threads(zthreads, recon_num, N_z);
        int prev = zthreads / recon_num;
        if (prev < 2)
            prev = 2;
        else {
            if (initICD == 3 && prev > N_z / 2)
                prev = N_z / 2;
            else if (prev > N_z)
                prev = N_z;
        }
        prev = (prev / 2) * 2;
        MbirStage *S = nullptr;
        if (mbir_init_stage(&S, P, W, proj_angles, proj_times, recon_times, proj_rows, proj_cols, proj_num,
                            recon_num, vox_wid, rot_center, sig_s, sig_t, c_s, c_t, convg_thresh,
                            remove_rings, quad_convex, huber_delta, huber_T, sxy[i], sz[i], nblk)) {
            LOG_ERR(log, "Stage set-up failed: %s\n", mbir_last_error());
            in.release_all();
            return -1;
        }
        mbir_set_rng_state(S, rng_state);
        int nblk_stage = nblk;
        if (use_sv) {
            if (mbir_set_acache(S, sv_acache) || mbir_set_schedule(S, 1, sv_side, 0)) {
                LOG_ERR(log, "Super-voxel schedule set-up failed: %s\n", mbir_last_error());
                mbir_free_stage(S);
                in.release_all();
                return -1;
            }
            const char *nh = getenv("TIMBIR_SV_NHICD");
            if (nh && *nh && mbir_set_sv_nhicd(S, atof(nh))) {
                LOG_ERR(log, "NHICD fraction: %s\n", mbir_last_error());
                mbir_free_stage(S);
                in.release_all();
                return -1;
            }
            int32_t d[9];
            mbir_stage_dims(S, d);
            nblk_stage = d[7];
            // the previous stage's map planes are known only within this call
            prev = prev_sv_blocks > 0 ? prev_sv_blocks : -1;
        }
        mbir_set_stage_switches(S, upd_offset, upd_var, var_est);
        // ring offsets: read back at stages that re-read them (XT_Init.c:343-351)
        std::vector<float> off((size_t)proj_cols * proj_rows, 0.0f);
        const float *offp = nullptr;
        if (upd_offset == 1 || upd_offset == 3) {
            if (read_bin("proj_offset", off.data(), sizeof(float), off.size()))
                LOG_ERR(log, "Error in reading file proj_offset.bin.\n");
            offp = off.data();
        } else if (!carried_offset.empty()) {
            offp = carried_offset.data();
        }
        // initial object and magnitude map (initObject, XT_ICD_update.c:540-651)
        const int N_y = N_x;
        const size_t nvox = (size_t)recon_num * N_z * N_y * N_x, nxy = (size_t)N_y * N_x;
        std::vector<float> obj(nvox, 0.0f), mag((size_t)recon_num * nblk_stage * nxy, 0.0f);
        bool have_mag = false;
        const bool on_device = prev_stage && (initICD == 2 || initICD == 3);
        if (on_device) {
            // the previous stage of this call is still on the device: its object
            // and magnitude map are up-sampled there, nothing is read back
            int carried = 0;
            if (mbir_icd_prepare_from(S, prev_stage.get(), initICD, offp, &carried)) {
                LOG_ERR(log, "Stage prologue failed: %s\n", mbir_last_error());
                mbir_free_stage(S);
                in.release_all();
                return -1;
            }
            if (!carried)
                LOG_INFO(log, "Number of axial blocks is incompatible with previous stage; "
                              "initializing the multi-resolution map to zeros.\n");
            prev_stage.reset();
        } else if (initICD == 2 || initICD == 3) {
            const int cz = initICD == 3 ? N_z / 2 : N_z;
            std::vector<float> coarse((size_t)cz * (N_y / 2) * (N_x / 2));
            for (int f = 0; f < recon_num; f++) {
                char name[64];
                snprintf(name, sizeof(name), "object_time_%d", f);
                if (read_bin(name, coarse.data(), sizeof(float), coarse.size())) {
                    LOG_ERR(log, "Error in reading file %s.bin.\n", name);
                    mbir_free_stage(S);
                    in.release_all();
                    return -1;
                }
                float *dst = obj.data() + (size_t)f * N_z * nxy;
                if (initICD == 3)
                    upsample_xyz(coarse.data(), dst, cz, N_y / 2, N_x / 2);
                else
                    upsample_xy(coarse.data(), dst, cz, N_y / 2, N_x / 2);
            }
            if (init_mag) {
                if (prev > 0 && (prev == nblk_stage || prev == nblk_stage / 2)) {
                    const int pb = prev;
                    std::vector<float> cm((size_t)recon_num * pb * (nxy / 4));
                    if (read_bin("mag_update", cm.data(), sizeof(float), cm.size()) == 0) {
                        for (int f = 0; f < recon_num; f++) {
                            const float *src = cm.data() + (size_t)f * pb * (nxy / 4);
                            float *dst = mag.data() + (size_t)f * nblk_stage * nxy;
                            if (pb == nblk_stage)
                                upsample_xy(src, dst, pb, N_y / 2, N_x / 2);
                            else
                                upsample_xyz(src, dst, pb, N_y / 2, N_x / 2);
                        }
                        have_mag = true;
                    }
                } else {
                    LOG_INFO(log, "Number of axial blocks is incompatible with previous stage; "
                                  "initializing the multi-resolution map to zeros.\n");
                }
            }
        }
        if (!on_device && mbir_icd_prepare(S, obj.data(), offp, have_mag ? mag.data() : nullptr)) {
            LOG_ERR(log, "Stage prologue failed: %s\n", mbir_last_error());
            mbir_free_stage(S);
            in.release_all();
            return -1;
        }
        // ICD iterations (ICD_BackProject, XT_ICD_update.c:1172-1203)
        double cost = 0, cost_last = 0;
        if (want_cost) {
            mbir_compute_cost(S, &cost, nullptr, nullptr);
            cost_last = cost;
            LOG_INFO(log, "------------- Iteration 0, Cost = %f------------\n", cost);
            write_bin("cost", &cost, sizeof(double), 1);
        }
        const time_t icd_start = time(nullptr);
        int failed = 0;
        for (int it = 1; it <= max_iters; it++) {
            int32_t conv = 0;
            if (mbir_update_voxels_time_slices(S, it, &conv)) {
                LOG_ERR(log, "ICD iteration failed: %s\n", mbir_last_error());
                failed = 1;
                break;
            }
            LOG_INFO(log, "Percentage average magnitude of voxel updates is %f.\n", mbir_get_update_percentage(S));
            if (want_cost) {
                mbir_compute_cost(S, &cost, nullptr, nullptr);
                LOG_INFO(log, "------------- Iteration = %d, Cost = %f, Time since start of ICD = %fmins ------------\n",
                         it, cost, difftime(time(nullptr), icd_start) / 60.0);
                append_bin("cost", &cost, sizeof(double), 1);
                if (cost > cost_last) {
                    LOG_ERR(log, "Cost value increased.\n");
                    failed = 1;
                    break;
                }
                cost_last = cost;
            } else {
                LOG_INFO(log, "-------------ICD_BackProject: ICD Iter = %d, time since start of ICD = %fmins------------.\n",
                         it, difftime(time(nullptr), icd_start) / 60.0);
            }
            if (conv != 0 && it > 1) {
                LOG_INFO(log, "Convergence criteria is met.\n");
                break;
            }
        }
        if (!failed) {
            var_est = mbir_get_var_est(S);
            write_bin("variance_estimate", &var_est, sizeof(double), 1);
            mbir_get_magmap(S, mag.data());
            write_bin("mag_update", mag.data(), sizeof(float), mag.size());
            mbir_get_object(S, obj.data());
            for (int f = 0; f < recon_num; f++) {
                char name[64];
                snprintf(name, sizeof(name), "object_time_%d", f);
                write_bin(name, obj.data() + (size_t)f * N_z * nxy, sizeof(float), (size_t)N_z * nxy);
            }
            carried_offset.assign((size_t)proj_cols * proj_rows, 0.0f);
            mbir_get_offset(S, carried_offset.data());
            write_bin("proj_offset", carried_offset.data(), sizeof(float), carried_offset.size());
            int32_t st = i;
            write_bin("status", &st, sizeof(int32_t), 1);
            prev_sv_blocks = nblk_stage;
            rng_state = mbir_get_rng_state(S);
        }
        LOG_INFO(log, "Time elapsed is %f minutes.\n", difftime(time(nullptr), start) / 60.0);
        if (failed)
            mbir_free_stage(S);
        else
            prev_stage.reset(S);
        if (failed) {
            LOG_ERR(log, "Reconstruction failed!\n");
            in.release_all();
            return -1;
        }
        LOG_INFO(log, "Completed multi-resolution stage %d.\n", i);
    }
    in.release_all();
    LOG_INFO(log, "Exiting MBIR 4D\n");
    return 0;
}
