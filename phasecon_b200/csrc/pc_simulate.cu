// Phase-contrast data simulator: the drop-in phcontomo_forward_project
// (PCMBIR_3D/XT_Engine.c:199-253) and the in-memory mbirgpu_pc_simulate.
//
// ForwardProject (PCMBIR_3D/XT_genSinogram.c:59-343) on the geometry of
// initPhantomStructures (PCMBIR_3D/XT_Init.c:611-684), per view i:
//   P_mag[i][t][r]   = sum_{col, slice} mag[slice][col] A(col, i, r) Z(slice, t)
//   P_phase[i][t][r] = the same with the phase phantom
// (A = calcAMatrixColumnforAngle x wavenumber, PCMBIR_3D/XT_AMatrix.c:50-110;
// Z = the voxel-line response of storeVoxelLineResponse,
// PCMBIR_3D/XT_Profile.c:229-297), the exit field
// sqrt(count) e^{-P_mag} (cos, sin)(-P_phase), its windowed Fresnel
// transform (compute_FresnelTran, window sigma 1/sqrt(lambda z / 2),
// XT_Init.c:677-681), |.|^2 averaged over the phantom pixels of each detector
// pixel and noise m <- |m + sqrt|m| n| with n = randlib's normal()
// (PCMBIR_3D/randlib.c:208-225) after srandom2(761521) (XT_Engine.c:212).
//
// GPU plan. Z has at most two entries per slice, so the projection factors
// into the per-column z response p[col][t] = sum_slice obj[slice][col] Z(slice, t)
// followed by a 2-D parallel-beam projection of those N_t-long lines: one warp
// per voxel column, lanes over detector rows t, each lane computing the FP64 A
// entries of one view for the warp (shuffled to all lanes) and every entry
// adding a p into FP64 projection images with red.global.add.f64 (order
// differs from the reference's sequential sums at the 1e-16 level). The field
// is formed in FP64 and transformed by the library's batched FP32 Fresnel
// kernels; the detector pass (one thread per detector pixel) reads the
// transform's output, accumulates |.|^2 like the reference (a float sum of
// FP64 terms) and draws its normal by skipping the Park-Miller generator
// (x <- 16807 x mod 2^31 - 1) ahead to its own position, so no sequential
// pass over the draws is needed. This file is compiled without multiply-add
// contraction so the FP64 geometry rounds like the reference's.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mbirgpu.h"
#include "mbir_internal.h"
#include "pc_internal.h"

namespace mbirgpu {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kPlanck = 4.135668e-19;      // PLANCKS_CONSTANT, keV s (PCMBIR_3D/XT_Constants.h:84)
constexpr double kLightSpeed = 299792458e+6;  // LIGHT_SPEED, um/s (XT_Constants.h:85)
constexpr int kMinRows = 4;                   // MIN_PROJECTION_ROWS (XT_Constants.h:186)
constexpr int kMinRowsPerNode = 2;            // MIN_ROWS_PER_NODE (XT_Constants.h:185)
constexpr uint32_t kNoiseSeed = 761521;       // srandom2 seed of phcontomo_forward_project (XT_Engine.c:212)
constexpr uint64_t kPmModulus = 2147483647ull;  // MAXPRIME of randlib.c:42
constexpr uint64_t kPmMultiplier = 16807ull;
constexpr int kSimBins = 256;     // DETECTOR_RESPONSE_BINS of PCMBIR_3D/XT_Constants.h:163
constexpr int kSimBeamRes = 256;  // BEAM_RESOLUTION, XT_Constants.h:162
constexpr int kSimChannels = 3;  // AvgNumXElements = ceil(3 delta_xy / delta_r) with delta_xy = delta_r
constexpr int kZEntries = 4;     // voxel-line response entries per detector row (at most 2 arise)

std::mutex g_sim_mu;
bool g_sim_init = false;
mbirgpu_pc_sim_options g_sim_opt;

struct SimGeom {
    int N_p, N_r, N_t, N_x, N_y, N_z;
    double delta_r, delta_t, R0, RMax, T0, TMax, OffsetR, OffsetT;
    double x0, y0, z0, delta_xy, delta_z;
    double wavelength, wavenumber, distance, window_sigma;
};

// initPhantomStructures (XT_Init.c:611-684) for one rank.
SimGeom phantom_geometry(int P_xy, int P_z, int proj_rows, int proj_cols, int proj_num, double vox_wid,
                         double rot_center, double obj2det_dist, double light_energy)
{
    SimGeom s{};
    const double length_R = vox_wid * proj_cols, length_T = vox_wid * proj_rows;
    const double rot = rot_center * (P_xy / proj_cols);  // integer quotient, as the reference
    s.wavelength = kPlanck * kLightSpeed / light_energy;
    s.wavenumber = 2 * kPi / s.wavelength;
    s.distance = obj2det_dist;
    s.N_p = proj_num;
    s.N_r = P_xy;
    s.N_t = P_z;
    s.delta_r = length_R / s.N_r;
    s.delta_t = length_T / s.N_t;
    s.R0 = -rot * s.delta_r;
    s.RMax = (s.N_r - rot) * s.delta_r;
    s.T0 = -length_T / 2.0;
    s.TMax = length_T / 2.0;
    s.N_x = s.N_y = P_xy;
    s.N_z = P_z;
    s.delta_xy = s.delta_r;
    s.delta_z = s.delta_t;
    s.x0 = s.R0;
    s.z0 = s.T0;
    s.y0 = -length_R / 2.0;
    s.OffsetR = (s.delta_xy / std::sqrt(2.0) + s.delta_r / 2.0) / kSimBins;
    s.OffsetT = ((s.delta_z / 2) + s.delta_t / 2) / kSimBins;
    s.window_sigma = 1.0 / (std::sqrt(0.5 * s.wavelength * s.distance));
    return s;
}

// ZLineResponseProfile + storeVoxelLineResponse (PCMBIR_3D/XT_Profile.c:182-297),
// transposed to per-detector-row lists: for row t, the slices s with Z(s, t) != 0.
void zline_response(const SimGeom &s, std::vector<int> &zc, std::vector<int> &zs, std::vector<double> &zv,
                    bool *overflow)
{
    std::vector<double> Ht(kSimBins + 1);
    for (int i = 0; i < kSimBins; i++) {
        const double center = i * s.OffsetT;
        double h;
        if (s.delta_z >= s.delta_t) {
            if (center <= ((s.delta_z / 2) - (s.delta_t / 2))) h = s.delta_t;
            else h = -center + (s.delta_z / 2) + s.delta_t / 2;
        } else {
            if (center <= s.delta_t / 2 - s.delta_z / 2) h = s.delta_z;
            else h = -center + (s.delta_z / 2) + s.delta_t / 2;
        }
        if (h < 0) h = 0;
        Ht[i] = h / s.delta_t;
    }
    Ht[kSimBins] = 0;
    zc.assign(s.N_t, 0);
    zs.assign((size_t)s.N_t * kZEntries, 0);
    zv.assign((size_t)s.N_t * kZEntries, 0.0);
    *overflow = false;
    for (int i = 0; i < s.N_z; i++) {
        const double t = ((double)i + 0.5) * s.delta_z + s.z0;
        const double tmin = (t - s.delta_z / 2) > s.T0 ? t - s.delta_z / 2 : s.T0;
        const double tmax = (t + s.delta_z / 2) <= s.TMax ? t + s.delta_z / 2 : s.TMax;
        int lo = (int)(std::floor((tmin - s.T0) / s.delta_t));
        int hi = (int)(std::floor((tmax - s.T0) / s.delta_t));
        if (lo < 0) lo = 0;
        if (hi >= s.N_t) hi = s.N_t - 1;
        for (int it = lo; it <= hi; it++) {
            const double center = ((double)it + 0.5) * s.delta_t + s.T0;
            const double d = std::fabs(center - t);
            const int idx = (int)(std::floor(d / s.OffsetT));
            double thick = 0;
            if (idx < kSimBins) {
                const double w3 = d - (double)(idx)*s.OffsetT;
                const double w4 = ((double)idx + 1) * s.OffsetT - d;
                thick = (w4 / s.OffsetT) * Ht[idx] + (w3 / s.OffsetT) * Ht[idx + 1];
            }
            if (thick != 0) {
                if (zc[it] >= kZEntries) {
                    *overflow = true;
                    continue;
                }
                zs[(size_t)it * kZEntries + zc[it]] = i;
                zv[(size_t)it * kZEntries + zc[it]] = thick;
                zc[it]++;
            }
        }
    }
}

// frequency of DFT index i with the wrap at n/2 (XT_FresnelTran.c:32-40, XT_Init.c:218-226)
double freq(int i, int n, double delta) { return i >= n / 2 ? -(double)(n - i) / (n * delta) : (double)i / (n * delta); }

bool pow2(int n) { return n >= 2 && (n & (n - 1)) == 0; }

// ---- device side --------------------------------------------------------------

// One warp per voxel column; lane owns detector rows lane + 32 k, k < KT.
template <int KT>
__global__ void __launch_bounds__(256) sim_project_kernel(SimGeom s, const double *__restrict__ H,
                                                          const double *__restrict__ cosv,
                                                          const double *__restrict__ sinv,
                                                          const float *__restrict__ mag,
                                                          const float *__restrict__ phase,
                                                          const int *__restrict__ zc, const int *__restrict__ zs,
                                                          const double *__restrict__ zv, double *__restrict__ pm,
                                                          double *__restrict__ pp, int *__restrict__ err)
{
    const int nxy = s.N_x * s.N_y;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= nxy) return;  // warp-uniform
    const int c = (int)gw, row = c / s.N_x, col = c - row * s.N_x;

    // z response of this column's lines: p[t] = sum_slice obj[slice][c] Z(slice, t)
    double am[KT], ap[KT];
    bool any = false;
#pragma unroll
    for (int k = 0; k < KT; k++) {
        am[k] = ap[k] = 0.0;
        const int t = lane + 32 * k;
        if (t < s.N_t) {
            for (int e = 0; e < zc[t]; e++) {
                const size_t src = (size_t)zs[t * kZEntries + e] * nxy + c;
                const double w = zv[t * kZEntries + e];
                am[k] += (double)__ldg(mag + src) * w;
                ap[k] += (double)__ldg(phase + src) * w;
            }
        }
        any |= am[k] != 0.0 || ap[k] != 0.0;
    }
    if (!__any_sync(0xffffffffu, any)) return;

    const double x = s.x0 + ((double)col + 0.5) * s.delta_xy;
    const double y = s.y0 + ((double)row + 0.5) * s.delta_xy;
    for (int vb = 0; vb < s.N_p; vb += 32) {
        // lane computes the A column of view vb + lane (calcAMatrixColumnforAngle)
        int cnt = 0, jj[kSimChannels] = {0, 0, 0};
        double aa[kSimChannels] = {0.0, 0.0, 0.0};
        const int v = vb + lane;
        if (v < s.N_p) {
            const double r = x * cosv[v] - y * sinv[v];
            const double rmin = r - s.delta_xy, rmax = r + s.delta_xy;
            if (!(rmax < s.R0 || rmin > s.RMax)) {
                int imin = (int)(floor(((rmin - s.R0) / s.delta_r)));
                int imax = (int)(floor((rmax - s.R0) / s.delta_r));
                if (imax >= s.N_r) imax = s.N_r - 1;
                if (imin < 0) imin = 0;
                const double *h = H + (size_t)v * (kSimBins + 1);
                for (int j = imin; j <= imax; j++) {
                    const double center = (s.R0 + (((double)j) + 0.5) * (s.delta_r));
                    const double d = fabs(r - center);
                    const int bin = (int)(floor((d / s.OffsetR)));
                    if (bin >= 0 && bin < kSimBins) {
                        const double w1 = d - bin * s.OffsetR;
                        const double w2 = s.OffsetR - w1;
                        const double f1 = (w2 * h[bin] + w1 * h[bin + 1]) / s.OffsetR;
                        if (f1 > 0) {
                            if (cnt < kSimChannels) {
#pragma unroll
                                for (int q = 0; q < kSimChannels; q++)
                                    if (q == cnt) {
                                        aa[q] = f1 * s.wavenumber;
                                        jj[q] = j;
                                    }
                                cnt++;
                            } else {
                                atomicOr(err, 1);  // more channels than a column can reach
                            }
                        }
                    }
                }
            }
        }
        const int nvb = min(32, s.N_p - vb);
        for (int u = 0; u < nvb; u++) {
            const int cu = __shfl_sync(0xffffffffu, cnt, u);
#pragma unroll
            for (int q = 0; q < kSimChannels; q++) {
                const double a = __shfl_sync(0xffffffffu, aa[q], u);
                const int j = __shfl_sync(0xffffffffu, jj[q], u);
                if (q < cu) {
                    const size_t base = ((size_t)(vb + u) * s.N_r + j) * s.N_t;
#pragma unroll
                    for (int k = 0; k < KT; k++) {
                        const int t = lane + 32 * k;
                        if (t < s.N_t) {
                            if (am[k] != 0.0) atomicAdd(pm + base + t, a * am[k]);
                            if (ap[k] != 0.0) atomicAdd(pp + base + t, a * ap[k]);
                        }
                    }
                }
            }
        }
    }
}

// exit field sqrt(count) e^{-P_mag} (cos, sin)(-P_phase) (XT_genSinogram.c:214-225), [V][R][C]
__global__ void sim_field_kernel(size_t n, const double *__restrict__ pm, const double *__restrict__ pp,
                                 double amp, float2 *__restrict__ field)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double e = exp(-pm[i]);
        const double re = e * cos(-pp[i]), im = e * sin(-pp[i]);
        field[i] = make_float2((float)(re * amp - im * 0.0), (float)(re * 0.0 + im * amp));
    }
}

__device__ __forceinline__ uint64_t pm_mulmod(uint64_t a, uint64_t b) { return (a * b) % kPmModulus; }

// value of the n-th random2() call (n >= 1) after srandom2(seed): seed 16807^n mod (2^31 - 1)
__device__ uint64_t pm_state(uint64_t seed, uint64_t n)
{
    uint64_t r = 1, b = kPmMultiplier;
    while (n) {
        if (n & 1) r = pm_mulmod(r, b);
        b = pm_mulmod(b, b);
        n >>= 1;
    }
    return pm_mulmod(seed % kPmModulus, r);
}

// The idx-th value (0-based) of randlib's normal() after srandom2(seed): pair
// idx / 2 draws theta = 2 pi random2() and r = sqrt(-2 log random2()) and
// returns r cos(theta), then r sin(theta) (randlib.c:208-225).
__device__ double pm_normal(uint64_t seed, uint64_t idx)
{
    const uint64_t p = idx >> 1;
    const uint64_t x1 = pm_state(seed, 2 * p + 1);
    const uint64_t x2 = pm_mulmod(x1, kPmMultiplier);
    const double theta = 2 * kPi * ((double)x1 / (double)kPmModulus);
    const double r = sqrt(-2 * log((double)x2 / (double)kPmModulus));
    return (idx & 1) ? r * sin(theta) : r * cos(theta);
}

// detector pixel (v, row, col): mean |F|^2 over its phantom pixels, then noise
// (XT_genSinogram.c:239-262); F is [V][R][C].
__global__ void sim_measure_kernel(int V, int rows, int cols, int R, int C, int ts, int rs,
                                   const float2 *__restrict__ F, float *__restrict__ meas)
{
    const size_t n = (size_t)V * rows * cols;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int v = (int)(idx / ((size_t)rows * cols));
        const int rem = (int)(idx - (size_t)v * rows * cols);
        const int row = rem / cols, col = rem - row * cols;
        float m = 0.0f;
        for (int ti = 0; ti < ts; ti++)
            for (int ri = 0; ri < rs; ri++) {
                const int to = row * ts + ti, ro = col * rs + ri;
                const float2 z = F[((size_t)v * R + ro) * C + to];
                const double b = (double)z.x * (double)z.x + (double)z.y * (double)z.y;
                m = (float)((double)m + b);
            }
        m = m / (float)(ts * rs);
        const double nrm = pm_normal(kNoiseSeed, idx);
        meas[idx] = (float)fabs((double)m + sqrt(fabs((double)m)) * nrm);
    }
}

// [V][R][C] -> [V][C][R] (the reference's projs[i][t][r])
__global__ void sim_transpose_kernel(int V, int R, int C, const double *__restrict__ in, double *__restrict__ out)
{
    const size_t n = (size_t)V * R * C;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int v = (int)(i / ((size_t)R * C));
        const int rem = (int)(i - (size_t)v * R * C);
        const int t = rem / R, r = rem - t * R;
        out[i] = in[((size_t)v * R + r) * C + t];
    }
}

#define SCK(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail("%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

struct DevBufs {
    std::vector<void *> p;
    ~DevBufs()
    {
        for (void *q : p) cudaFree(q);
    }
    template <typename T>
    int alloc(T **out, size_t n)
    {
        *out = nullptr;
        cudaError_t e = cudaMalloc((void **)out, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) return fail("cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
        p.push_back(*out);
        return 0;
    }
};

bool write_doubles_file(const char *name, const std::vector<double> &v)
{
    FILE *fp = std::fopen((std::string(name) + ".bin").c_str(), "wb");
    if (!fp) return false;
    const bool ok = std::fwrite(v.data(), sizeof(double), v.size(), fp) == v.size();
    std::fclose(fp);
    return ok;
}

const mbirgpu_pc_sim_options &sim_options()
{
    std::lock_guard<std::mutex> lk(g_sim_mu);
    if (!g_sim_init) {
        mbirgpu_pc_sim_default_options(&g_sim_opt);
        g_sim_init = true;
    }
    return g_sim_opt;
}

// argument checks of phcontomo_forward_project (XT_Engine.c:214-217, one rank)
// plus the sizes this implementation handles
int check_sim_args(const mbirgpu_pc_sim_options &o, int rows, int cols, int V)
{
    const int P_xy = o.phantom_xy, P_z = o.phantom_z;
    if (rows < kMinRows) return fail("The minimum number of projection rows should be %d.", kMinRows);
    if (cols % 2 != 0) return fail("The number of projection columns should be even.");
    if (rows % 2 != 0 || rows < kMinRowsPerNode)
        return fail("The number of projection rows divided by the number of nodes should be an even number greater "
                    "than or equal to %d.", kMinRowsPerNode);
    if (V < 1) return fail("proj_num must be positive");
    if (!pow2(P_xy) || !pow2(P_z) || P_xy > 1024 || P_z > 256)
        return fail("phantom sizes must be powers of two, xy <= 1024 and z <= 256 (got %d x %d)", P_xy, P_z);
    const int rs = P_xy / cols, ts = P_z / rows;
    if (rs < 1 || ts < 1) return fail("the detector (%d x %d) is finer than the phantom (%d x %d)", rows, cols, P_z, P_xy);
    if (o.expected_count <= 0) return fail("expected_count must be positive");
    return 0;
}

int simulate(const float *mag, const float *phase, const mbirgpu_pc_sim_options &o, float *meas, float *brights,
             const float *angles, int rows, int cols, int V, float vox_wid, float rot_center, float dist,
             float energy, double *out_mag, double *out_phase, double *out_avg)
{
    if (!mag || !phase || !meas || !brights || !angles) return fail("phantom, output and angle pointers must be set");
    if (check_sim_args(o, rows, cols, V)) return -1;
    const int P_xy = o.phantom_xy, P_z = o.phantom_z;
    const int rs = P_xy / cols, ts = P_z / rows;
    const SimGeom s = phantom_geometry(P_xy, P_z, rows, cols, V, vox_wid, rot_center, dist, energy);
    std::vector<int> zc, zs;
    std::vector<double> zv;
    bool overflow = false;
    zline_response(s, zc, zs, zv, &overflow);
    if (overflow) return fail("voxel-line response with more than %d entries per detector row", kZEntries);
    Geom g{};
    g.N_p = V;
    g.N_r = s.N_r;
    g.delta_r = s.delta_r;
    g.delta_xy = s.delta_xy;
    g.OffsetR = s.OffsetR;
    std::vector<double> H((size_t)V * (kSimBins + 1)), cosv(V), sinv(V);
    detector_response_f64(g, angles, H.data(), kSimBins, kSimBeamRes);
    for (int i = 0; i < V; i++) {
        const double a = angles[i];
        cosv[i] = std::cos(a);
        sinv[i] = std::sin(a);
    }
    // transfer table of compute_FresnelTran with the phantom window
    const int R = s.N_r, Cn = s.N_t;
    std::vector<float2> Hf((size_t)R * Cn);
    for (int i = 0; i < R; i++)
        for (int j = 0; j < Cn; j++) {
            const double u = freq(i, R, s.delta_r), v = freq(j, Cn, s.delta_t);
            const double win = std::exp(-(u * u + v * v) / (2 * s.window_sigma * s.window_sigma));
            const double ph = -(u * u + v * v) * kPi * s.wavelength * s.distance;
            Hf[(size_t)i * Cn + j] = make_float2((float)(std::cos(ph) * win), (float)(std::sin(ph) * win));
        }
    PcDims d{};
    size_t smem_rows = 0, smem_cols = 0;
    if (pc_transform_dims(d, V, R, Cn, &smem_rows, &smem_cols)) return -1;
    const std::vector<float2> tw = pc_twiddles(d.nmax);

    const size_t nvox = (size_t)P_z * P_xy * P_xy, nproj = (size_t)V * R * Cn, nmeas = (size_t)V * rows * cols;
    DevBufs B;
    float *d_mag, *d_phase, *d_meas;
    double *d_H, *d_cos, *d_sin, *d_zv, *d_pm, *d_pp;
    int *d_zc, *d_zs, *d_err;
    float2 *d_field, *d_work, *d_tw, *d_Hf;
    if (B.alloc(&d_mag, nvox) || B.alloc(&d_phase, nvox) || B.alloc(&d_meas, nmeas) || B.alloc(&d_H, H.size()) ||
        B.alloc(&d_cos, V) || B.alloc(&d_sin, V) || B.alloc(&d_zv, zv.size()) || B.alloc(&d_zc, zc.size()) ||
        B.alloc(&d_zs, zs.size()) || B.alloc(&d_err, 1) || B.alloc(&d_pm, nproj) || B.alloc(&d_pp, nproj) ||
        B.alloc(&d_field, nproj) || B.alloc(&d_work, nproj) || B.alloc(&d_tw, tw.size()) ||
        B.alloc(&d_Hf, Hf.size()))
        return -1;
    cudaStream_t st = nullptr;
    SCK(cudaMemcpyAsync(d_mag, mag, nvox * sizeof(float), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_phase, phase, nvox * sizeof(float), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_H, H.data(), H.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_cos, cosv.data(), V * sizeof(double), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_sin, sinv.data(), V * sizeof(double), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_zv, zv.data(), zv.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_zc, zc.data(), zc.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_zs, zs.data(), zs.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_Hf, Hf.data(), Hf.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
    SCK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    SCK(cudaMemsetAsync(d_pm, 0, nproj * sizeof(double), st));
    SCK(cudaMemsetAsync(d_pp, 0, nproj * sizeof(double), st));

    const long long threads = (long long)P_xy * P_xy * 32;
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    if (P_z <= 32) sim_project_kernel<1><<<blocks, 256, 0, st>>>(s, d_H, d_cos, d_sin, d_mag, d_phase, d_zc, d_zs, d_zv, d_pm, d_pp, d_err);
    else if (P_z <= 64) sim_project_kernel<2><<<blocks, 256, 0, st>>>(s, d_H, d_cos, d_sin, d_mag, d_phase, d_zc, d_zs, d_zv, d_pm, d_pp, d_err);
    else if (P_z <= 128) sim_project_kernel<4><<<blocks, 256, 0, st>>>(s, d_H, d_cos, d_sin, d_mag, d_phase, d_zc, d_zs, d_zv, d_pm, d_pp, d_err);
    else sim_project_kernel<8><<<blocks, 256, 0, st>>>(s, d_H, d_cos, d_sin, d_mag, d_phase, d_zc, d_zs, d_zv, d_pm, d_pp, d_err);
    SCK(cudaGetLastError());
    sim_field_kernel<<<148 * 8, 256, 0, st>>>(nproj, d_pm, d_pp, std::sqrt((double)o.expected_count), d_field);
    PcArgs A{};
    A.tw = d_tw;
    A.work = d_work;
    pc_transform(d, A, smem_rows, smem_cols, PC_IN_PLAIN, d_field, d_Hf, PC_OUT_PLAIN, d_field, 0, st);
    sim_measure_kernel<<<148 * 8, 256, 0, st>>>(V, rows, cols, R, Cn, ts, rs, d_field, d_meas);
    SCK(cudaGetLastError());
    int err = 0;
    SCK(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(meas, d_meas, nmeas * sizeof(float), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    if (err) return fail("a voxel column reached more than %d detector channels in one view", kSimChannels);
    for (size_t i = 0; i < (size_t)rows * cols; i++) brights[i] = o.expected_count;
    double avg = 0;
    for (size_t i = 0; i < nmeas; i++) avg += meas[i];
    avg /= (double)nmeas;
    if (out_avg) *out_avg = avg;

    // projections in the reference's [N_p][N_t][N_r] layout (the field buffer is free now)
    const bool files = o.write_files != 0;
    if (out_mag || out_phase || files) {
        double *d_tr = reinterpret_cast<double *>(d_work);  // nproj complex floats = nproj doubles
        std::vector<double> hbuf;
        double *pr[2] = {d_pm, d_pp};
        double *outs[2] = {out_mag, out_phase};
        const char *names[2] = {"SimMagProjs", "SimPhaseProjs"};
        for (int k = 0; k < 2; k++) {
            if (!outs[k] && !files) continue;
            sim_transpose_kernel<<<148 * 8, 256, 0, st>>>(V, R, Cn, pr[k], d_tr);
            double *dst = outs[k];
            if (!dst) {
                hbuf.resize(nproj);
                dst = hbuf.data();
            }
            SCK(cudaMemcpyAsync(dst, d_tr, nproj * sizeof(double), cudaMemcpyDeviceToHost, st));
            SCK(cudaStreamSynchronize(st));
            if (files) {
                std::vector<double> v(dst, dst + nproj);
                if (!write_doubles_file(names[k], v)) return fail("writing %s.bin failed", names[k]);
            }
        }
    }
    if (files) {
        std::vector<double> v(nvox);
        for (size_t i = 0; i < nvox; i++) v[i] = mag[i];
        if (!write_doubles_file("mag_phantom", v)) return fail("writing mag_phantom.bin failed");
        for (size_t i = 0; i < nvox; i++) v[i] = phase[i];
        if (!write_doubles_file("phase_phantom", v)) return fail("writing phase_phantom.bin failed");
    }
    return 0;
}

bool read_phantom(const char *path, std::vector<float> &v)
{
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return false;
    const bool ok = std::fread(v.data(), sizeof(float), v.size(), fp) == v.size();
    std::fclose(fp);
    return ok;
}

}  // namespace

}  // namespace mbirgpu

using namespace mbirgpu;

extern "C" {

void mbirgpu_pc_sim_default_options(mbirgpu_pc_sim_options *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    std::snprintf(o->mag_phantom_path, sizeof(o->mag_phantom_path), "%s",
                  "/scratch/rice/m/mohank/Sim_Datasets/Absorp_Latex_Phantom.bin");
    std::snprintf(o->phase_phantom_path, sizeof(o->phase_phantom_path), "%s",
                  "/scratch/rice/m/mohank/Sim_Datasets/RefIndex_Latex_Phantom.bin");
    o->phantom_xy = 512;
    o->phantom_z = 128;
    o->expected_count = 2500.0f;
    o->write_files = 1;
}

int mbirgpu_pc_sim_set_options(const mbirgpu_pc_sim_options *o)
{
    if (!o) return fail("options pointer is NULL");
    if (o->expected_count <= 0) return fail("expected_count must be positive");
    sim_options();
    std::lock_guard<std::mutex> lk(g_sim_mu);
    g_sim_opt = *o;
    g_sim_opt.mag_phantom_path[sizeof(g_sim_opt.mag_phantom_path) - 1] = 0;
    g_sim_opt.phase_phantom_path[sizeof(g_sim_opt.phase_phantom_path) - 1] = 0;
    return 0;
}

int mbirgpu_pc_sim_get_options(mbirgpu_pc_sim_options *o)
{
    if (!o) return fail("options pointer is NULL");
    const mbirgpu_pc_sim_options cur = sim_options();
    *o = cur;
    return 0;
}

int mbirgpu_pc_simulate(const float *mag_phantom, const float *phase_phantom, const mbirgpu_pc_sim_options *opt,
                        float *measurements, float *brights, const float *proj_angles, int32_t proj_rows,
                        int32_t proj_cols, int32_t proj_num, float vox_wid, float rot_center, float obj2det_dist,
                        float light_energy, double *sim_mag_projs, double *sim_phase_projs, double *measurement_avg)
{
    const mbirgpu_pc_sim_options o = opt ? *opt : sim_options();
    return simulate(mag_phantom, phase_phantom, o, measurements, brights, proj_angles, proj_rows, proj_cols, proj_num,
                    vox_wid, rot_center, obj2det_dist, light_energy, sim_mag_projs, sim_phase_projs, measurement_avg);
}

int phcontomo_forward_project(float **measurements, float **brights, float *proj_angles, int32_t proj_rows,
                              int32_t proj_cols, int32_t proj_num, float vox_wid, float rot_center,
                              float obj2det_dist, float light_energy, float pag_regparam, FILE *debug_msg_ptr)
{
    (void)pag_regparam;  // initPhantomStructures stores delta/beta, the simulator never reads it
    if (!measurements || !brights || !*measurements || !*brights)
        return fail("measurements and brights must point to caller-allocated arrays");
    const mbirgpu_pc_sim_options o = sim_options();
    if (debug_msg_ptr) std::fprintf(debug_msg_ptr, "[INFO] (mbirgpu) Forward projecting the object ....\n");
    if (check_sim_args(o, proj_rows, proj_cols, proj_num)) return -1;
    const size_t nvox = (size_t)o.phantom_z * o.phantom_xy * o.phantom_xy;
    std::vector<float> mag(nvox), phase(nvox);
    if (!read_phantom(o.mag_phantom_path, mag)) return fail("Error in reading file %s", o.mag_phantom_path);
    if (!read_phantom(o.phase_phantom_path, phase)) return fail("Error in reading file %s", o.phase_phantom_path);
    double avg = 0;
    const int rc = simulate(mag.data(), phase.data(), o, *measurements, *brights, proj_angles, proj_rows, proj_cols,
                            proj_num, vox_wid, rot_center, obj2det_dist, light_energy, nullptr, nullptr, &avg);
    if (rc) {
        if (debug_msg_ptr) std::fprintf(debug_msg_ptr, "[ERROR] (mbirgpu) Forward projection failed: %s\n",
                                        mbirgpu_last_error());
        return -1;
    }
    if (debug_msg_ptr)
        std::fprintf(debug_msg_ptr,
                     "[INFO] (mbirgpu) The expected count is %g; the average of all measurement data is %f\n",
                     (double)o.expected_count, avg);
    return 0;
}

}  // extern "C"
