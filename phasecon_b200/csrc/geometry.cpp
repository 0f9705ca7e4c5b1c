// Host-side stage setup of libmbirgpu: detector/object geometry, the view to
// time-frame map, qGGMRF constants and the per-view detector response H_r.
// Restates MBIR_4D/XT_Init.c:211-432 and MBIR_4D/XT_Profile.c:47-218 for one
// rank. The double-precision arithmetic is kept operation for operation (and
// compiled without multiply-add contraction) so that H_r, and therefore every
// A-matrix value built from it on the device, equals the reference's bit for
// bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>
#include "mbir_internal.h"

namespace mbirgpu {

namespace {

constexpr int kProfileRes = 1536;  // PROFILE_RESOLUTION, MBIR_4D/XT_Constants.h:77
constexpr int kBeamRes = 512;      // BEAM_RESOLUTION, XT_Constants.h:78
constexpr double kHalfPi = 1.57079632679489661923132169163975144;
constexpr double kQuarterPi = 0.785398163397448309615660845819875721;

// Euclidean distance to a neighbour of the 4-D (t,z,y,x) prior grid,
// MBIR_4D/XT_Init.c:138-141.
double grid_distance(int a, int b, int c, int d)
{
    return std::sqrt(std::pow(a - 1.0, 2.0) + std::pow(b - 1.0, 2.0) + std::pow(c - 1.0, 2.0) +
                     std::pow(d - 1.0, 2.0));
}

// Detector response H_r[view][0..64] (XT_Profile.c:129-218): the voxel's
// trapezoidal line-integral profile at the view's angle (XT_Profile.c:47-104,
// stored as the reference's Real_arr_t: float in MBIR_4D, double in
// PCMBIR_3D) convolved with a normalised Hamming beam (XT_Profile.c:108-124),
// sampled every OffsetR. Views are independent: they are split over host
// threads (each view's arithmetic is the same whichever thread runs it).
template <typename T>
void detector_response_views(const Geom &g, const float *angles, T *H_r, int bins, int beam_res,
                             const std::vector<double> &beam, int v_begin, int v_end)
{
    std::vector<T> prof(kProfileRes);
    const double r0 = -(g.delta_r) / 2, step = (g.delta_r) / beam_res;
    const double to_bin = (kProfileRes) / (2 * g.delta_xy);
    for (int v = v_begin; v < v_end; v++) {
        double ang = angles[v];
        while (ang > kHalfPi) ang -= kHalfPi;
        while (ang < 0) ang += kHalfPi;
        const double peak = ang <= kQuarterPi ? g.delta_xy / std::cos(ang) : g.delta_xy / std::cos(kHalfPi - ang);
        const double c45 = std::cos(kQuarterPi);
        const double d1 = c45 * std::cos((kQuarterPi - ang));
        const double d2 = c45 * std::fabs((std::cos((kQuarterPi + ang))));
        const double left_corner = 1 - d1, left_near = 1 - d2, right_near = 1 + d2, right_corner = 1 + d1;
        for (int j = 0; j < kProfileRes; j++) {
            const double t = 2.0 * j / kProfileRes;
            T val;
            if (t <= left_corner || t >= right_corner) val = 0;
            else if (t > right_near) val = (T)(peak * (right_corner - t) / (right_corner - right_near));
            else if (t >= left_near) val = (T)peak;
            else val = (T)(peak * (t - left_corner) / (left_near - left_corner));
            prof[j] = val;
        }
        T *h = H_r + (size_t)v * (bins + 1);
        for (int i = 0; i < bins; i++) {
            const double center = i * g.OffsetR, rmin = center - g.delta_xy;
            double acc = 0;
            for (int p = 0; p < beam_res; p++) {
                const double r = r0 + p * step;
                const int idx = (int)std::floor((r - rmin) * to_bin);
                if (idx >= 0 && idx <= kProfileRes - 1) acc += (prof[idx] * beam[p]);
            }
            h[i] = (T)acc;
        }
        h[bins] = 0;
    }
}

template <typename T>
void detector_response_t(const Geom &g, const float *angles, T *H_r, int bins, int beam_res)
{
    std::vector<double> beam(beam_res);
    double total = 0;
    for (int i = 0; i < beam_res; i++) {
        beam[i] = 0.54 - 0.46 * std::cos((2 * 3.14159265358979323846 / beam_res) * i);
        total = total + beam[i];
    }
    for (int i = 0; i < beam_res; i++) beam[i] /= total;
    // about 32 k beam-sample steps per view: threads pay off from a few dozen views
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::max(1, std::min({hw, 32, g.N_p / 16}));
    if (nt == 1) {
        detector_response_views<T>(g, angles, H_r, bins, beam_res, beam, 0, g.N_p);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; t++) {
        const int a = (int)((long long)g.N_p * t / nt), b = (int)((long long)g.N_p * (t + 1) / nt);
        pool.emplace_back(detector_response_views<T>, std::cref(g), angles, H_r, bins, beam_res, std::cref(beam), a, b);
    }
    for (auto &th : pool) th.join();
}

}  // namespace

void detector_response(const Geom &g, const float *angles, float *H_r)
{
    detector_response_t<float>(g, angles, H_r, kRespBins, kBeamRes);
}
void detector_response_f64(const Geom &g, const float *angles, double *H_r, int bins, int beam_res)
{
    detector_response_t<double>(g, angles, H_r, bins, beam_res);
}

std::string build_setup(HostSetup &hs, const ProblemDesc &pd, const float *angles, const float *proj_times,
                        const float *recon_times, int mult_xy, int mult_z)
{
    Geom &g = hs.g;
    std::memset(&g, 0, sizeof(g));
    // argument checks of XT_Engine.c:101-104 (one rank) and XT_Init.c:427-428
    if (pd.proj_rows < 4) return "The minimum number of projection rows should be 4.";
    if (pd.proj_cols % 2 != 0) return "The number of projection columns should be even.";
    if (pd.proj_rows % 2 != 0) return "The number of projection rows should be an even number.";
    if (pd.proj_num < 1 || pd.recon_num < 1) return "proj_num and recon_num must be positive.";
    if (mult_xy < 1 || mult_z < 1 || pd.proj_cols % mult_xy != 0 || pd.proj_rows % mult_z != 0)
        return "Voxel scale does not divide the detector size.";
    if (2 * mult_xy + 1 > kMaxKmax) return "Voxel scale above 4 is not supported.";

    g.p = pd.mrf_p;
    g.q = pd.mrf_q;
    g.alpha = pd.alpha;
    g.c_s = pd.c_s;
    g.c_t = pd.c_t;
    g.mult_xy = mult_xy;
    g.mult_z = mult_z;
    const double vox = pd.vox_wid, rot = pd.rot_center;
    const double length_R = vox * pd.proj_cols, length_T = vox * pd.proj_rows;
    g.N_time = pd.recon_num;
    g.N_p = pd.proj_num;
    g.N_r = pd.proj_cols;
    g.N_t = pd.proj_rows;
    g.radius_obj = vox * pd.proj_cols / 2;
    g.delta_r = length_R / g.N_r;
    g.delta_t = length_T / g.N_t;
    g.R0 = -rot * g.delta_r;
    g.RMax = (g.N_r - rot) * g.delta_r;
    g.T0 = -length_T / 2.0;
    g.TMax = length_T / 2.0;
    g.N_x = (int)(g.N_r / (double)mult_xy);
    g.N_y = g.N_x;
    g.N_z = (int)(g.N_t / (double)mult_z);
    g.delta_xy = mult_xy * g.delta_r;
    g.delta_z = mult_z * g.delta_t;
    g.z_overlap = mult_z;
    g.x0 = g.R0;
    g.z0 = g.T0;
    g.y0 = -length_R / 2.0;
    g.OffsetR = (g.delta_xy / std::sqrt(2.0) + g.delta_r / 2.0) / kRespBins;
    g.OffsetT = ((g.delta_z / 2) + g.delta_t / 2) / kRespBins;
    if (pd.quad_convex) {
        g.huber = 0;
        g.huber_T = 100000;  // ZINGER_DISABLE_PARAM_T, XT_Constants.h:97
        g.huber_delta = 1;   // ZINGER_DISABLE_PARAM_DELTA, XT_Constants.h:98
    } else {
        g.huber = 1;
        g.huber_T = pd.huber_T;
        g.huber_delta = pd.huber_delta;
    }
    if ((long long)g.N_p * g.N_r >= (1LL << 24)) return "proj_num * proj_cols must stay below 2^24.";
    if ((long long)g.N_p * g.N_r * g.N_t >= (1LL << 32)) return "proj_num * proj_cols * proj_rows must stay below 2^32.";

    // view -> frame map (initRandomAngles / initSparseAnglesOfObject, XT_Init.c:69-131)
    for (int i = 0; i + 1 < g.N_p; i++)
        if (proj_times[i + 1] < proj_times[i])
            return "Projection acquisition time decreased for increasing index. Check input files.";
    for (int i = 0; i < g.N_time; i++)
        if (recon_times[i + 1] < recon_times[i])
            return "Reconstruction times decreased for increasing index. Check input files.";
    hs.view_first.assign(g.N_time + 1, 0);
    hs.views.clear();
    int start = 0;
    double total = 0;
    g.max_views = 0;
    for (int i = 0; i < g.N_time; i++) {
        int n = 0;
        for (int j = start; j < g.N_p; j++) {
            const double t = proj_times[j];
            if (t >= recon_times[i] && t < recon_times[i + 1]) {
                hs.views.push_back(j);
                n++;
            }
            if (t >= recon_times[i + 1]) {
                start = j;
                break;
            }
        }
        hs.view_first[i + 1] = hs.view_first[i] + n;
        if (n > g.max_views) g.max_views = n;
        total += n;
    }
    g.delta_recon = total / g.N_time;

    // qGGMRF scale powers (XT_Init.c:418-421) and neighbour filters (initFilter, XT_Init.c:144-190)
    const double sig_s = pd.sig_s, sig_t = pd.sig_t;
    g.sigma_s_q = std::pow(sig_s * mult_xy, g.q);
    g.sigma_s_q_p = std::pow(sig_s * mult_xy, g.q - g.p);
    g.sigma_t_q = std::pow(sig_t * g.delta_recon, g.q);
    g.sigma_t_q_p = std::pow(sig_t * g.delta_recon, g.q - g.p);
    const double prior_const = (double)mult_xy * (double)mult_xy * (double)mult_xy * g.delta_recon;
    const double tf = 1.0 / grid_distance(0, 1, 1, 1);
    double norm = 2.0 * tf;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++) {
                double v = 0;
                if (a != 1 || b != 1 || c != 1) {
                    v = 1.0 / grid_distance(1, a, b, c);
                    norm = norm + v;
                }
                g.spatial_filter[(a * 3 + b) * 3 + c] = v;
            }
    for (int a = 0; a < 27; a++) g.spatial_filter[a] = prior_const * g.spatial_filter[a] / norm;
    g.time_filter = prior_const * tf / norm;

    g.kmax = 2 * mult_xy + 1;
    g.rec_words = ((1 + g.kmax) + 3) / 4 * 4;

    hs.cosv.resize(g.N_p);
    hs.sinv.resize(g.N_p);
    for (int i = 0; i < g.N_p; i++) {  // calculateSinCos, XT_Init.c:193-206
        hs.cosv[i] = std::cos((double)angles[i]);
        hs.sinv[i] = std::sin((double)angles[i]);
    }
    hs.H_r.assign((size_t)g.N_p * (kRespBins + 1), 0.0f);
    detector_response(g, angles, hs.H_r.data());

    // reconstruction circle of ICD_BackProject (XT_ICD_update.c:1127-1136)
    hs.mask.assign((size_t)g.N_y * g.N_x, 0);
    for (int j = 0; j < g.N_y; j++)
        for (int k = 0; k < g.N_x; k++) {
            const double x = g.x0 + ((double)k + 0.5) * g.delta_xy;
            const double y = g.y0 + ((double)j + 0.5) * g.delta_xy;
            hs.mask[(size_t)j * g.N_x + k] = (x * x + y * y < g.radius_obj * g.radius_obj) ? 1 : 0;
        }
    return "";
}

}  // namespace mbirgpu
