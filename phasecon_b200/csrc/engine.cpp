// Drop-in reconstruct() (replaces MBIR_4D/XT_Engine.c:81-194): the
// multi-resolution stage loop around GPU sessions, object initialisation by
// bilinear upsampling between stages (XT_ICD_update.c:358-496, 540-647), the
// per-stage ICD loop with the reference's convergence test and cost log
// (XT_ICD_update.c:1148-1189), and the reference's side-effect files.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mbirgpu.h"
#include "session.h"

namespace mbirgpu {
namespace {

void log_info(FILE *fp, const char *fmt, ...)
{
    if (!fp) return;
    va_list ap;
    va_start(ap, fmt);
    std::fprintf(fp, "[INFO] (mbirgpu) ");
    std::vfprintf(fp, fmt, ap);
    va_end(ap);
    std::fflush(fp);
}

bool write_bin(const std::string &name, const void *data, size_t bytes, bool append = false)
{
    FILE *fp = std::fopen((name + ".bin").c_str(), append ? "ab" : "wb");
    if (!fp) return false;
    const bool ok = std::fwrite(data, 1, bytes, fp) == bytes;
    std::fclose(fp);
    return ok;
}

bool read_bin(const std::string &name, void *data, size_t bytes)
{
    FILE *fp = std::fopen((name + ".bin").c_str(), "rb");
    if (!fp) return false;
    const bool ok = std::fread(data, 1, bytes, fp) == bytes;
    std::fclose(fp);
    return ok;
}

// 2x bilinear upsampling in x-y of one [nz][ny][nx] volume into
// [nz][2ny][2nx] (upsample_object_bilinear_2D, XT_ICD_update.c:358-390).
void upsample_xy(const float *in, float *out, int nz, int ny, int nx)
{
    std::vector<float> buf((size_t)ny * 2 * nx);
    for (int s = 0; s < nz; s++) {
        const float *I = in + (size_t)s * ny * nx;
        float *O = out + (size_t)s * 4 * ny * nx;
        for (int j = 0; j < ny; j++) {
            float *b = &buf[(size_t)j * 2 * nx];
            const float *r = I + (size_t)j * nx;
            b[0] = r[0];
            b[1] = (3.0 * r[0] + r[1]) / 4.0;
            b[2 * nx - 1] = r[nx - 1];
            b[2 * nx - 2] = (r[nx - 2] + 3.0 * r[nx - 1]) / 4.0;
            for (int k = 1; k < nx - 1; k++) {
                b[2 * k] = (r[k - 1] + 3.0 * r[k]) / 4.0;
                b[2 * k + 1] = (3.0 * r[k] + r[k + 1]) / 4.0;
            }
        }
        const int W = 2 * nx;
        for (int k = 0; k < W; k++) {
            O[k] = buf[k];
            O[W + k] = (3.0 * buf[k] + buf[W + k]) / 4.0;
            O[(size_t)(2 * ny - 1) * W + k] = buf[(size_t)(ny - 1) * W + k];
            O[(size_t)(2 * ny - 2) * W + k] = (buf[(size_t)(ny - 2) * W + k] + 3.0 * buf[(size_t)(ny - 1) * W + k]) / 4.0;
        }
        for (int j = 1; j < ny - 1; j++)
            for (int k = 0; k < W; k++) {
                O[(size_t)(2 * j) * W + k] = (buf[(size_t)(j - 1) * W + k] + 3.0 * buf[(size_t)j * W + k]) / 4.0;
                O[(size_t)(2 * j + 1) * W + k] = (3 * buf[(size_t)j * W + k] + buf[(size_t)(j + 1) * W + k]) / 4.0;
            }
    }
}

// 2x upsampling in x, y and z (upsample_object_bilinear_3D,
// XT_ICD_update.c:448-496): x-y first, then z with the same 1/4-3/4 weights.
// The reference keeps its intermediate buffers in double; here they are
// float, which changes only the initial value of the next stage.
void upsample_xyz(const float *in, float *out, int nz, int ny, int nx)
{
    std::vector<float> xy((size_t)nz * 4 * ny * nx);
    upsample_xy(in, xy.data(), nz, ny, nx);
    const size_t plane = (size_t)4 * ny * nx;
    for (size_t p = 0; p < plane; p++) {
        out[p] = xy[p];
        out[plane + p] = (3.0 * xy[p] + xy[plane + p]) / 4.0;
        out[(size_t)(2 * nz - 1) * plane + p] = xy[(size_t)(nz - 1) * plane + p];
        out[(size_t)(2 * nz - 2) * plane + p] = (3.0 * xy[(size_t)(nz - 1) * plane + p] + xy[(size_t)(nz - 2) * plane + p]) / 4.0;
    }
    for (int s = 1; s < nz - 1; s++)
        for (size_t p = 0; p < plane; p++) {
            out[(size_t)(2 * s) * plane + p] = (xy[(size_t)(s - 1) * plane + p] + 3.0 * xy[(size_t)s * plane + p]) / 4.0;
            out[(size_t)(2 * s + 1) * plane + p] = (3.0 * xy[(size_t)s * plane + p] + xy[(size_t)(s + 1) * plane + p]) / 4.0;
        }
}

}  // namespace
}  // namespace mbirgpu

using namespace mbirgpu;

extern "C" int reconstruct(float **object, float *projections, float *weights, float *proj_angles,
                           float *proj_times, float *recon_times, int32_t proj_rows, int32_t proj_cols,
                           int32_t proj_num, int32_t recon_num, float vox_wid, float rot_center, float sig_s,
                           float sig_t, float c_s, float c_t, float convg_thresh, int32_t remove_rings,
                           int32_t quad_convex, float huber_delta, float huber_T, uint8_t restart,
                           FILE *debug_msg_ptr)
{
    FILE *dbg = debug_msg_ptr;
    if (!object) return fail("object pointer is NULL");
    *object = nullptr;
    if (remove_rings < 0 || remove_rings > 3) return fail("remove_rings must be 0, 1, 2 or 3 (got %d)", remove_rings);
    const mbirgpu_options opt = current_options();
    log_info(dbg, "Reconstructing the data ....\n");

    // multi-resolution plan, XT_Engine.c:111-141 (one rank)
    const int MAX_MULTRES = 8, MIN_XY = 64;
    int multres_num = (int)(std::log(((float)proj_cols) / MIN_XY) / std::log(2.0) + 1);
    if (multres_num > MAX_MULTRES) multres_num = MAX_MULTRES;
    if (multres_num < 2) multres_num = 2;
    int mxy[MAX_MULTRES], mz[MAX_MULTRES];
    mxy[0] = 1;
    mz[0] = 1;
    for (int i = 1; i < multres_num; i++) {
        if (proj_cols % (mxy[i - 1] * 2) == 0) {
            mxy[i] = mxy[i - 1] * 2;
            mz[i] = (proj_rows % (mz[i - 1] * 2) == 0 && proj_rows / (mz[i - 1] * 2) >= 2) ? mz[i - 1] * 2 : mz[i - 1];
        } else {
            multres_num = i;
            break;
        }
    }
    // coarse to fine; optionally keep only the finest opt.num_stages stages
    std::vector<int> stage_xy, stage_z;
    for (int i = 0; i < multres_num; i++) {
        stage_xy.push_back(mxy[multres_num - 1 - i]);
        stage_z.push_back(mz[multres_num - 1 - i]);
    }
    if (opt.num_stages > 0 && opt.num_stages < (int)stage_xy.size()) {
        stage_xy.erase(stage_xy.begin(), stage_xy.end() - opt.num_stages);
        stage_z.erase(stage_z.begin(), stage_z.end() - opt.num_stages);
    }
    const int nstages = (int)stage_xy.size();
    int first_stage = 0;
    if (restart == 1) {
        int32_t st = 0;
        if (!read_bin("status", &st, sizeof(st))) return fail("restart requested but status.bin is unreadable");
        first_stage = st;
    }
    if (first_stage < 0 || first_stage >= nstages) return fail("status.bin names stage %d of %d", first_stage, nstages);
    log_info(dbg, "Number of multi-resolution stages is %d.\n", nstages);

    mbirgpu_problem pb{};
    pb.projections = projections;
    pb.weights = weights;
    pb.proj_angles = proj_angles;
    pb.proj_times = proj_times;
    pb.recon_times = recon_times;
    pb.proj_rows = proj_rows;
    pb.proj_cols = proj_cols;
    pb.proj_num = proj_num;
    pb.recon_num = recon_num;
    pb.vox_wid = vox_wid;
    pb.rot_center = rot_center;
    pb.sig_s = sig_s;
    pb.sig_t = sig_t;
    pb.c_s = c_s;
    pb.c_t = c_t;
    pb.convg_thresh = convg_thresh;
    pb.quad_convex = quad_convex;
    pb.huber_delta = huber_delta;
    pb.huber_T = huber_T;

    std::vector<float> prev;  // previous stage's object, [T][Z][Y][X]
    std::vector<float> offset((size_t)proj_cols * proj_rows, 0.0f);  // ring-correction offset d [N_r][N_t]
    bool have_offset = false;
    int prev_nz = 0, prev_ny = 0, prev_nx = 0;
    std::vector<float> cur;
    int nz = 0, ny = 0, nx = 0;
    for (int si = first_stage; si < nstages; si++) {
        log_info(dbg, "Running multi-resolution stage %d with x-y voxel scale = %d and z voxel scale = %d.\n", si,
                 stage_xy[si], stage_z[si]);
        mbirgpu_session *sp = nullptr;
        if (mbirgpu_session_create(&sp, &pb, &opt, stage_xy[si], stage_z[si], nullptr)) return -1;
        Session *s = reinterpret_cast<Session *>(sp);
        const Geom &g = s->hs.g;
        nz = g.N_z;
        ny = g.N_y;
        nx = g.N_x;
        cur.assign((size_t)recon_num * nz * ny * nx, 0.0f);
        if (si > first_stage || (si > 0 && restart == 1)) {
            // initObject (XT_ICD_update.c:540-647): previous stage, upsampled
            if (prev.empty()) {
                prev_nz = (stage_z[si - 1] == stage_z[si]) ? nz : nz / 2;
                prev_ny = ny / 2;
                prev_nx = nx / 2;
                prev.assign((size_t)recon_num * prev_nz * prev_ny * prev_nx, 0.0f);
                const size_t n = (size_t)prev_nz * prev_ny * prev_nx;
                for (int t = 0; t < recon_num; t++)
                    if (!read_bin("object_time_" + std::to_string(t), prev.data() + t * n, n * sizeof(float))) {
                        mbirgpu_session_destroy(sp);
                        return fail("cannot read object_time_%d.bin to initialise stage %d", t, si);
                    }
            }
            const size_t pn = (size_t)prev_nz * prev_ny * prev_nx, cn = (size_t)nz * ny * nx;
            for (int t = 0; t < recon_num; t++) {
                if (prev_nz == nz) upsample_xy(prev.data() + t * pn, cur.data() + t * cn, nz, prev_ny, prev_nx);
                else upsample_xyz(prev.data() + t * pn, cur.data() + t * cn, prev_nz, prev_ny, prev_nx);
            }
            if (mbirgpu_session_set_object(sp, cur.data())) {
                mbirgpu_session_destroy(sp);
                return -1;
            }
        }
        // ring correction: none in the first stage, estimated from zero in the
        // second, from the previous stage's offset (proj_offset.bin) after that
        // (updateProjOffset, XT_Init.c:246-255, 345-349)
        if (remove_rings && si >= 1) {
            if (si >= 2 && !have_offset) {
                if (!read_bin("proj_offset", offset.data(), offset.size() * sizeof(float))) {
                    mbirgpu_session_destroy(sp);
                    return fail("cannot read proj_offset.bin to initialise stage %d", si);
                }
                have_offset = true;
            }
            if (mbirgpu_session_set_ring_correction(sp, remove_rings, si >= 2 ? offset.data() : nullptr)) {
                mbirgpu_session_destroy(sp);
                return -1;
            }
        }
        // noise-variance re-estimation with the generalised-Huber data term after
        // the first stage (updateVar, XT_Init.c:270-278)
        if (!quad_convex && si >= 1 && mbirgpu_session_set_variance_estimation(sp, 1)) {
            mbirgpu_session_destroy(sp);
            return -1;
        }
        // ICD loop with cost log, XT_ICD_update.c:1148-1189
        std::vector<double> costs(opt.max_iterations + 1, 0.0);
        int iters = 0;
        mbirgpu_iter_stats tot;
        if (s->run(opt.max_iterations, costs.data(), &iters, &tot)) {
            mbirgpu_session_destroy(sp);
            return -1;
        }
        if (opt.compute_cost) {
            for (int it = 1; it <= iters; it++)
                if (costs[it] > costs[it - 1])
                    log_info(dbg, "Cost value increased at iteration %d (%.10g -> %.10g).\n", it, costs[it - 1],
                             costs[it]);
            log_info(dbg, "Stage %d: %d iterations, final cost %.10g, %lld voxel updates.\n", si, iters, costs[iters],
                     (long long)tot.voxel_updates);
        }
        if (s->get_object(cur.data())) {
            mbirgpu_session_destroy(sp);
            return -1;
        }
        if (remove_rings && si >= 1) {
            if (mbirgpu_session_get_offset(sp, offset.data())) {
                mbirgpu_session_destroy(sp);
                return -1;
            }
            have_offset = true;
        }
        if (opt.write_files) {
            bool ok = true;
            if (opt.compute_cost) ok &= write_bin("cost", costs.data(), (size_t)(iters + 1) * sizeof(double));
            const size_t n = (size_t)nz * ny * nx;
            for (int t = 0; t < recon_num && ok; t++)
                ok &= write_bin("object_time_" + std::to_string(t), cur.data() + t * n, n * sizeof(float));
            ok &= write_bin("proj_offset", offset.data(), offset.size() * sizeof(float));
            double var_est = 1.0;
            mbirgpu_session_get_variance(sp, &var_est);
            ok &= write_bin("variance_estimate", &var_est, sizeof(var_est));
            std::vector<float> mag((size_t)recon_num * ny * nx);
            if (cudaMemcpy(mag.data(), s->d_mag, mag.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
                ok = false;
            ok &= write_bin("mag_update", mag.data(), mag.size() * sizeof(float));
            const int32_t status = first_stage;  // the reference records its starting stage, XT_Engine.c:168
            ok &= write_bin("status", &status, sizeof(status));
            if (!ok) {
                mbirgpu_session_destroy(sp);
                return fail("writing the stage %d output files failed", si);
            }
        }
        mbirgpu_session_destroy(sp);
        prev.swap(cur);
        prev_nz = nz;
        prev_ny = ny;
        prev_nx = nx;
        log_info(dbg, "Completed multi-resolution stage %d.\n", si);
    }
    // output with one zero halo slice above and below each frame, XT_Init.c:362-363
    const size_t plane = (size_t)prev_ny * prev_nx, vol = (size_t)(prev_nz + 2) * plane;
    float *outp = (float *)std::calloc((size_t)recon_num * vol, sizeof(float));
    if (!outp) return fail("out of host memory for the output object");
    for (int t = 0; t < recon_num; t++)
        std::memcpy(outp + t * vol + plane, prev.data() + (size_t)t * prev_nz * plane, (size_t)prev_nz * plane * sizeof(float));
    *object = outp;
    log_info(dbg, "Exiting MBIR 4D\n");
    return 0;
}
