// Phase-contrast (PCMBIR_3D) host side of libmbirgpu: session state, the
// steepest-descent / phase-retrieval ADMM driver over batched kernels, and
// the drop-in phcontomo_reconstruct.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/mbirgpu.h"
#include "pc_internal.h"
#include "session.h"

namespace mbirgpu {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kPlanck = 4.135668e-19;       // PLANCKS_CONSTANT, keV s (PCMBIR_3D/XT_Constants.h:84)
constexpr double kLightSpeed = 299792458e+6;   // LIGHT_SPEED, um/s (XT_Constants.h:85)

bool pow2(int n) { return n >= 2 && (n & (n - 1)) == 0; }
int ilog2(int n)
{
    int l = 0;
    while ((1 << l) < n) l++;
    return l;
}

// frequency index i of an n-point DFT with the wrap at n/2 of XT_FresnelTran.c:32-40
double freq(int i, int n, double delta) { return i >= n / 2 ? -(double)(n - i) / (n * delta) : (double)i / (n * delta); }

}  // namespace

int pc_transform_dims(PcDims &d, int V, int R, int C, size_t *smem_rows, size_t *smem_cols, int fft_radix)
{
    d.V = V;
    d.R = R;
    d.C = C;
    d.N = R * C;
    d.logR = ilog2(R);
    d.logC = ilog2(C);
    d.nmax = std::max(R, C);
    d.fft_radix = fft_radix > 0 ? fft_radix : kPcDefaultFftRadix;
    if (d.fft_radix != 2 && d.fft_radix != 4 && d.fft_radix != 8 && d.fft_radix != 16)
        return fail("fft_radix must be 2, 4, 8 or 16 (got %d)", fft_radix);
    // sequences per CTA: up to 4,096 points in each of the two padded buffers,
    // no more sequences than there are (rows: R sequences of length C;
    // columns: C sequences of length R)
    d.rows_per_cta = std::max(1, std::min(R, 4096 / C));
    d.cols_per_cta = std::max(1, std::min(C, 4096 / R));
    // the full twiddle circle (nmax) and the two buffers
    *smem_rows = (size_t)(d.nmax + 2 * d.rows_per_cta * fft_seq_stride(C)) * sizeof(float2);
    *smem_cols = (size_t)(d.nmax + 2 * d.cols_per_cta * fft_seq_stride(R)) * sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(pc_rows_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem_rows);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pc_rows_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem_rows);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pc_cols_filter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem_cols);
    return e == cudaSuccess ? 0 : fail("cudaFuncSetAttribute failed: %s", cudaGetErrorString(e));
}

std::vector<float2> pc_twiddles(int nmax)
{
    std::vector<float2> tw(nmax / 2);
    for (int m = 0; m < nmax / 2; m++) {
        const double a = -2.0 * kPi * m / nmax;
        tw[m] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    return tw;
}

void pc_transform(const PcDims &d, PcArgs A, size_t smem_rows, size_t smem_cols, int prologue, const float2 *in,
                  const float2 *table, int epilogue, float2 *out, int acc_slot, cudaStream_t st)
{
    A.in = in;
    A.out = out;
    A.acc_slot = acc_slot;
    dim3 grows((d.R + d.rows_per_cta - 1) / d.rows_per_cta, d.V), gcols(d.C / d.cols_per_cta, d.V);
    // 256-point sequences with radix-16 stages: the register-resident passes
    // (16 sequences per CTA; the twiddle table and one padded buffer, 37 KB)
    const bool rows256 = d.C == 256 && d.R % 16 == 0 && d.fft_radix == 16;
    const bool cols256 = d.R == 256 && d.C % 16 == 0 && d.fft_radix == 16;
    const size_t smem256 = (size_t)(d.nmax + 16 * fft_seq_stride(256)) * sizeof(float2);
    if (rows256) pc_rows_forward_256<<<dim3(d.R / 16, d.V), 256, smem256, st>>>(d, A, prologue);
    else pc_rows_forward<<<grows, 256, smem_rows, st>>>(d, A, prologue);
    if (cols256) pc_cols_filter_256<<<dim3(d.C / 16, d.V), 256, smem256, st>>>(d, A, table);
    else pc_cols_filter<<<gcols, 256, smem_cols, st>>>(d, A, table);
    if (rows256) pc_rows_inverse_256<<<dim3(d.R / 16, d.V), 256, smem256, st>>>(d, A, epilogue);
    else pc_rows_inverse<<<grows, 256, smem_rows, st>>>(d, A, epilogue);
}

#define PCK(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail("%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

struct PcSession {
    PcDims d{};
    mbirgpu_pc_options opt{};
    cudaStream_t st = nullptr;
    double wavelength = 0, wavenumber = 0, distance = 0, dob = 0, delta = 1;
    PcPrior prior{};
    size_t smem_rows = 0, smem_cols = 0;
    std::vector<void *> allocs;

    float2 *d_tw = nullptr, *d_Hf = nullptr, *d_Hh = nullptr, *d_Hp = nullptr;
    float *d_D = nullptr, *d_y = nullptr, *d_zr = nullptr, *d_zi = nullptr;
    float2 *d_work = nullptr, *d_T1 = nullptr, *d_w = nullptr, *d_wold = nullptr, *d_g = nullptr, *d_buf = nullptr,
           *d_v = nullptr, *d_om = nullptr;
    double *d_acc = nullptr, *d_costs = nullptr, *d_dual = nullptr, *d_primal = nullptr;
    int *d_act_pret = nullptr, *d_act_sd = nullptr, *d_sd_steps = nullptr, *d_pret_iters = nullptr;
    float *d_thr = nullptr;

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    ~PcSession()
    {
        for (void *p : allocs) cudaFree(p);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }

    template <typename T>
    int alloc(T **p, size_t n)
    {
        *p = nullptr;
        cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) return fail("cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
        allocs.push_back(*p);
        return 0;
    }

    PcArgs args(int *active) const
    {
        PcArgs A{};
        A.tw = d_tw;
        A.work = d_work;
        A.D = d_D;
        A.y = d_y;
        A.lam = nullptr;  // Weight = 1 (XT_Init.c:366)
        A.omega = d_om;
        A.w = d_w;
        A.wold = d_wold;
        A.g = d_g;
        A.buf = d_buf;
        A.vdual = d_v;
        A.zr = d_zr;
        A.zi = d_zi;
        A.acc = d_acc;
        A.active = active;
        A.sd_thresh_out = d_thr;
        A.sd_steps = d_sd_steps;
        A.pret_iters = d_pret_iters;
        A.dual_res = d_dual;
        A.primal_res = d_primal;
        return A;
    }

    // one Fresnel-type transform: prologue (rows FFT), transfer (cols), epilogue (inverse rows)
    void transform(PcArgs A, int prologue, const float2 *in, const float2 *table, int epilogue, float2 *out,
                   int acc_slot)
    {
        pc_transform(d, A, smem_rows, smem_cols, prologue, in, table, epilogue, out, acc_slot, st);
        launches += 3;
    }

    int64_t launches = 0;  // kernels this session has launched
    int nms_lanes = kPcDefaultNmsLanes, nms_ctas = kPcDefaultNmsCtas;  // proximal sweep layout

    dim3 pointwise_grid() const { return dim3(std::max(1, std::min(64, d.N / 1024)), d.V); }

    int init(const mbirgpu_pc_problem *pb, const mbirgpu_pc_options *o, void *stream);
    void sd_step(int *active, int step);
    int omega_from_w(int *active);
    void pret_cost(int *active);
    int run(double *costs, int32_t *iters, mbirgpu_pc_stats *stats);
    int any_active(const int *flags, bool *any);

    // one proximal sweep over every pixel of the active views
    void nms_sweep(const PcArgs &A)
    {
        launches += launch_nms_sweep(d, A, prior, opt.nms_order, nms_lanes, nms_ctas, opt.nms_max_iter,
                                     (float)opt.nms_threshold, pointwise_grid(), st);
    }
};

int PcSession::init(const mbirgpu_pc_problem *pb, const mbirgpu_pc_options *o, void *stream)
{
    if (o) opt = *o;
    else mbirgpu_pc_default_options(&opt);
    st = (cudaStream_t)stream;
    const int R = pb->proj_cols, C = pb->proj_rows, V = pb->proj_num;
    if (!pow2(R) || !pow2(C) || R > 1024 || C > 1024)
        return fail("phase retrieval needs power-of-two detector sizes up to 1024 (got %d x %d)", C, R);
    if (V < 1) return fail("proj_num must be positive");
    if (opt.nms_order != 0 && opt.nms_order != 1) return fail("nms_order must be 0 (raster) or 1 (colour classes)");
    nms_lanes = opt.nms_lanes > 0 ? opt.nms_lanes : kPcDefaultNmsLanes;
    nms_ctas = opt.nms_ctas_per_view > 0 ? opt.nms_ctas_per_view : kPcDefaultNmsCtas;
    if (nms_lanes != 1 && nms_lanes != 2 && nms_lanes != 4 && nms_lanes != 8)
        return fail("nms_lanes must be 1, 2, 4 or 8 (got %d)", opt.nms_lanes);
    if (nms_ctas != 1 && nms_ctas != 2 && nms_ctas != 4)
        return fail("nms_ctas_per_view must be 1, 2 or 4 (got %d)", opt.nms_ctas_per_view);
    if (pc_transform_dims(d, V, R, C, &smem_rows, &smem_cols, opt.fft_radix)) return -1;
    d.nu = (float)opt.nu;
    dob = pb->pag_regparam;
    d.delta_over_beta = (float)dob;

    // physics constants (XT_Init.c:256-260, 530)
    wavelength = kPlanck * kLightSpeed / (double)pb->light_energy;
    wavenumber = 2 * kPi / wavelength;
    distance = pb->obj2det_dist;
    delta = pb->vox_wid;
    const double sigma = 2.0 / std::sqrt(wavelength * distance);

    const size_t NV = (size_t)V * d.N;
    if (alloc(&d_tw, d.nmax / 2) || alloc(&d_Hf, d.N) || alloc(&d_Hh, d.N) || alloc(&d_Hp, d.N) ||
        alloc(&d_D, d.N) || alloc(&d_y, NV) || alloc(&d_zr, NV) || alloc(&d_zi, NV) || alloc(&d_work, NV) ||
        alloc(&d_T1, NV) || alloc(&d_w, NV) || alloc(&d_wold, NV) || alloc(&d_g, NV) || alloc(&d_buf, NV) ||
        alloc(&d_v, NV) || alloc(&d_om, NV) || alloc(&d_acc, (size_t)V * kPcAccSlots) ||
        alloc(&d_dual, V) || alloc(&d_primal, V) || alloc(&d_act_pret, V) || alloc(&d_act_sd, V) ||
        alloc(&d_sd_steps, V) || alloc(&d_pret_iters, V) || alloc(&d_thr, V))
        return -1;

    // twiddles and transfer tables in double, rounded once to float
    const std::vector<float2> tw = pc_twiddles(d.nmax);
    std::vector<float2> Hf(d.N), Hh(d.N), Hp(d.N);
    const double kover2R = kPi / (distance * wavelength);
    const double reg = dob / (2 * wavenumber);
    for (int i = 0; i < R; i++)
        for (int j = 0; j < C; j++) {
            const double u = freq(i, R, delta), v = freq(j, C, delta);
            const double win = std::exp(-(u * u + v * v) / (2 * sigma * sigma));  // XT_Init.c:210-232
            const double ph = -(u * u + v * v) * kPi * wavelength * distance;     // XT_FresnelTran.c:41-43
            Hf[(size_t)i * C + j] = make_float2((float)(std::cos(ph) * win), (float)(std::sin(ph) * win));
            const double uu = u * 2 * kPi, vv = v * 2 * kPi;                       // XT_FresnelTran.c:101-112
            const double phh = (uu * uu + vv * vv) / (4 * kover2R);
            Hh[(size_t)i * C + j] = make_float2((float)std::cos(phh), (float)std::sin(phh));
            const double tran = distance * reg * (u * u + v * v) * 4 * kPi * kPi + 1;  // XT_Paganin.c:109
            Hp[(size_t)i * C + j] = make_float2((float)(1.0 / tran), 0.0f);
        }
    // measurements -> sqrt(I) / sqrt(mean bright), D = sqrt(bright) / sqrt(mean bright) (XT_Init.c:353-389)
    double bavg = 0;
    for (int k = 0; k < C; k++)
        for (int j = 0; j < R; j++) bavg += pb->brights[(size_t)k * R + j];
    bavg /= (double)C * R;
    bavg = std::sqrt(bavg);
    std::vector<float> D(d.N), y(NV);
    for (int j = 0; j < R; j++)
        for (int k = 0; k < C; k++) D[(size_t)j * C + k] = (float)(std::sqrt((double)pb->brights[(size_t)k * R + j]) / bavg);
    for (int i = 0; i < V; i++)
        for (int j = 0; j < R; j++)
            for (int k = 0; k < C; k++)
                y[((size_t)i * R + j) * C + k] =
                    (float)(std::sqrt((double)pb->measurements[((size_t)i * C + k) * R + j]) / bavg);
    PCK(cudaMemcpyAsync(d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
    PCK(cudaMemcpyAsync(d_Hf, Hf.data(), Hf.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
    PCK(cudaMemcpyAsync(d_Hh, Hh.data(), Hh.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
    PCK(cudaMemcpyAsync(d_Hp, Hp.data(), Hp.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
    PCK(cudaMemcpyAsync(d_D, D.data(), D.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    PCK(cudaMemcpyAsync(d_y, y.data(), y.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    PCK(cudaMemsetAsync(d_acc, 0, (size_t)V * kPcAccSlots * sizeof(double), st));
    PCK(cudaMemsetAsync(d_zr, 0, NV * sizeof(float), st));
    PCK(cudaMemsetAsync(d_zi, 0, NV * sizeof(float), st));
    PCK(cudaMemsetAsync(d_v, 0, NV * sizeof(float2), st));

    // prior: PCMBIR's in-plane filter (initFilter, XT_Init.c:144-190, prior constant 1,
    // no temporal weight), decorrelating transform (:234-247), qGGMRF scale powers (:482-491)
    double f3[27], tot = 0;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++) {
                double v = 0;
                if (a != 1 || b != 1 || c != 1) {
                    v = 1.0 / std::sqrt(std::pow(a - 1.0, 2.0) + std::pow(b - 1.0, 2.0) + std::pow(c - 1.0, 2.0));
                    tot += v;
                }
                f3[(a * 3 + b) * 3 + c] = v;
            }
    for (int a = 0; a < 9; a++) prior.f[a] = f3[9 + a] / tot;
    prior.T00 = 1;
    prior.T01 = dob;
    prior.T10 = 1;
    prior.T11 = -dob;
    const double q = opt.mrf_q, p = opt.mrf_p;
    prior.ph_sq = std::pow(pb->phase_sig_s, q);
    prior.ph_sqp = std::pow(pb->phase_sig_s, q - p);
    prior.ph_c = pb->phase_c_s;
    prior.mg_sq = std::pow(pb->mag_sig_s, q);
    prior.mg_sqp = std::pow(pb->mag_sig_s, q - p);
    prior.mg_c = pb->mag_c_s;
    prior.qmp = q - p;
    prior.ph_isq_f = (float)(1.0 / prior.ph_sq);
    prior.ph_isqp_f = (float)(1.0 / prior.ph_sqp);
    prior.ph_c_f = (float)prior.ph_c;
    prior.mg_isq_f = (float)(1.0 / prior.mg_sq);
    prior.mg_isqp_f = (float)(1.0 / prior.mg_sqp);
    prior.mg_c_f = (float)prior.mg_c;
    prior.qmp_f = (float)prior.qmp;
    for (int a = 0; a < 9; a++) prior.f_f[a] = (float)prior.f[a];
    prior.T00_f = (float)prior.T00;
    prior.T01_f = (float)prior.T01;
    prior.T10_f = (float)prior.T10;
    prior.T11_f = (float)prior.T11;
    PCK(cudaStreamSynchronize(st));
    return 0;
}

// One steepest-descent step of all active views (steepest_descent_iter,
// PCMBIR_3D/XT_PhaseRet.c:205-270). The two Hermitian transforms of the
// gradient (:102, :111) act on operands that differ only by the measured
// term, so one transform of conj(Omega) Lambda (Omega H D w - y) gives the
// same gradient (the transform is linear); the cost evaluated at :214 is not
// used by the reference outside debug builds and is not computed.
void PcSession::sd_step(int *active, int step)
{
    PcArgs A = args(active);
    transform(A, PC_IN_DW, d_w, d_Hf, PC_OUT_GRES, d_T1, 0);
    transform(A, PC_IN_PLAIN, d_T1, d_Hh, PC_OUT_GRAD, nullptr, PC_ACC_GG);
    transform(A, PC_IN_DW, d_g, d_Hf, PC_OUT_SFWD, d_T1, 0);
    transform(A, PC_IN_PLAIN, d_T1, d_Hh, PC_OUT_SDEN, nullptr, PC_ACC_DEN);
    pc_sd_update<<<pointwise_grid(), 256, 0, st>>>(d, A);
    transform(A, PC_IN_DW, d_w, d_Hf, PC_OUT_OMEGA, nullptr, 0);
    pc_sd_finish<<<(d.V + 127) / 128, 128, 0, st>>>(d, A, step, (float)opt.sd_threshold);
    launches += 2;
}

int PcSession::omega_from_w(int *active)
{
    transform(args(active), PC_IN_DW, d_w, d_Hf, PC_OUT_OMEGA, nullptr, 0);
    PCK(cudaGetLastError());
    return 0;
}

void PcSession::pret_cost(int *active)
{
    PcArgs A = args(active);
    transform(A, PC_IN_DEZ, nullptr, d_Hf, PC_OUT_PCOST, nullptr, PC_ACC_PCOST);
    pc_prior_cost<<<pointwise_grid(), 256, 0, st>>>(d, A, prior);
    launches += 1;
}

int PcSession::any_active(const int *flags, bool *any)
{
    std::vector<int> h(d.V);
    PCK(cudaMemcpyAsync(h.data(), flags, d.V * sizeof(int), cudaMemcpyDeviceToHost, st));
    PCK(cudaStreamSynchronize(st));
    *any = std::any_of(h.begin(), h.end(), [](int x) { return x != 0; });
    return 0;
}

// The per-view phase-retrieval ADMM of estimate_complex_projection
// (PCMBIR_3D/XT_CmplxProjEst.c:91-229) for all views at once; each view
// keeps its own stopping decisions through the per-view flags.
int PcSession::run(double *costs, int32_t *iters, mbirgpu_pc_stats *stats)
{
    const int V = d.V, P = opt.pret_max_iter;
    const int64_t launches0 = launches;
    if (!ev0) PCK(cudaEventCreate(&ev0));
    if (!ev1) PCK(cudaEventCreate(&ev1));
    PCK(cudaEventRecord(ev0, st));
    if (!d_costs && alloc(&d_costs, (size_t)(P + 1) * V)) return -1;
    {
        std::vector<double> nan((size_t)(P + 1) * V, std::numeric_limits<double>::quiet_NaN());
        PCK(cudaMemcpyAsync(d_costs, nan.data(), nan.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    std::vector<int> ones(V, 1);
    PCK(cudaMemcpyAsync(d_act_pret, ones.data(), V * sizeof(int), cudaMemcpyHostToDevice, st));
    PCK(cudaMemsetAsync(d_sd_steps, 0, V * sizeof(int), st));
    PCK(cudaMemsetAsync(d_acc, 0, (size_t)V * kPcAccSlots * sizeof(double), st));
    PCK(cudaMemsetAsync(d_v, 0, (size_t)V * d.N * sizeof(float2), st));  // XT_CmplxProjEst.c:108-109
    // cost before the first iteration (:111)
    pret_cost(d_act_pret);
    pc_pret_finish<<<(V + 127) / 128, 128, 0, st>>>(d, args(d_act_pret), -1, (float)opt.pret_threshold, d_costs);
    launches += 1;
    PCK(cudaGetLastError());
    int it = 0;
    for (; it < P; it++) {
        PcArgs A = args(d_act_pret);
        nms_sweep(A);
        pc_pret_prepare<<<pointwise_grid(), 256, 0, st>>>(d, A);
        launches += 1;
        PCK(cudaMemcpyAsync(d_act_sd, d_act_pret, V * sizeof(int), cudaMemcpyDeviceToDevice, st));
        for (int j = 0; j < opt.sd_max_iter; j++) {
            sd_step(d_act_sd, j);
            if ((j & 7) == 7 || j + 1 == opt.sd_max_iter) {
                PCK(cudaGetLastError());
                bool any = false;
                if (any_active(d_act_sd, &any)) return -1;
                if (!any) break;
            }
        }
        pc_pret_dual<<<pointwise_grid(), 256, 0, st>>>(d, A);
        launches += 1;
        pret_cost(d_act_pret);
        pc_pret_finish<<<(V + 127) / 128, 128, 0, st>>>(d, A, it, (float)opt.pret_threshold,
                                                         d_costs + (size_t)(it + 1) * V);
        launches += 1;
        PCK(cudaGetLastError());
        bool any = false;
        if (any_active(d_act_pret, &any)) return -1;
        if (!any) {
            it++;
            break;
        }
    }
    PCK(cudaEventRecord(ev1, st));
    PCK(cudaStreamSynchronize(st));
    float ms = 0;
    PCK(cudaEventElapsedTime(&ms, ev0, ev1));
    std::vector<int> steps(V), pit(V);
    PCK(cudaMemcpy(steps.data(), d_sd_steps, V * sizeof(int), cudaMemcpyDeviceToHost));
    PCK(cudaMemcpy(pit.data(), d_pret_iters, V * sizeof(int), cudaMemcpyDeviceToHost));
    if (costs) {
        std::vector<double> h((size_t)(P + 1) * V);
        PCK(cudaMemcpy(h.data(), d_costs, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int v = 0; v < V; v++)
            for (int k = 0; k <= P; k++) costs[(size_t)v * (P + 1) + k] = h[(size_t)k * V + v];
    }
    if (iters) std::copy(pit.begin(), pit.end(), iters);
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        for (int v = 0; v < V; v++) {
            stats->sd_steps += steps[v];
            stats->fresnel_transforms += 5LL * steps[v] + pit[v] + 1;
        }
        stats->kernel_ms = ms;
        stats->kernel_launches = launches - launches0;
    }
    return 0;
}

}  // namespace mbirgpu

using mbirgpu::fail;
using mbirgpu::PcSession;

namespace {

template <typename T>
int upload(PcSession *s, T *dst, const T *src, size_t n)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? 0 : fail("upload failed: %s", cudaGetErrorString(e));
}

template <typename T>
int download(PcSession *s, T *dst, const T *src, size_t n)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? 0 : fail("download failed: %s", cudaGetErrorString(e));
}

bool write_doubles(const std::string &name, const std::vector<double> &v)
{
    FILE *fp = std::fopen((name + ".bin").c_str(), "wb");
    if (!fp) return false;
    const bool ok = std::fwrite(v.data(), sizeof(double), v.size(), fp) == v.size();
    std::fclose(fp);
    return ok;
}

bool read_doubles(const std::string &name, std::vector<double> &v)
{
    FILE *fp = std::fopen((name + ".bin").c_str(), "rb");
    if (!fp) return false;
    const bool ok = std::fread(v.data(), sizeof(double), v.size(), fp) == v.size();
    std::fclose(fp);
    return ok;
}

}  // namespace

#define PCSESSION(sp)                                  \
    if (!(sp)) return fail("session pointer is NULL"); \
    PcSession *s = reinterpret_cast<PcSession *>(sp)

extern "C" {

void mbirgpu_pc_default_options(mbirgpu_pc_options *o)
{
    std::memset(o, 0, sizeof(*o));
    o->pret_max_iter = 100;
    o->sd_max_iter = 100;
    o->nms_max_iter = 50;
    o->pret_threshold = 0.0000001;
    o->sd_threshold = 0.0005;
    o->nms_threshold = 0.005;
    o->mu = 0.5;
    o->nu = 0.5;
    o->mrf_p = 1.2;
    o->mrf_q = 2.0;
    o->nms_order = 0;
    o->fft_radix = 0;
}

int mbirgpu_pc_session_create(mbirgpu_pc_session **out, const mbirgpu_pc_problem *pb, const mbirgpu_pc_options *opt,
                              void *stream)
{
    if (!out || !pb || !pb->measurements || !pb->brights) return fail("NULL argument");
    *out = nullptr;
    PcSession *s = new (std::nothrow) PcSession();
    if (!s) return fail("out of host memory");
    if (s->init(pb, opt, stream)) {
        std::string keep = mbirgpu_last_error();
        delete s;
        fail("%s", keep.c_str());
        return -1;
    }
    *out = reinterpret_cast<mbirgpu_pc_session *>(s);
    return 0;
}

int mbirgpu_pc_session_destroy(mbirgpu_pc_session *sp)
{
    delete reinterpret_cast<PcSession *>(sp);
    return 0;
}

int mbirgpu_pc_fresnel(mbirgpu_pc_session *sp, const float *in, float *out, int32_t herm)
{
    PCSESSION(sp);
    if (!in || !out) return fail("NULL argument");
    const size_t NV = (size_t)s->d.V * s->d.N;
    if (upload(s, s->d_T1, reinterpret_cast<const float2 *>(in), NV)) return -1;
    s->transform(s->args(nullptr), mbirgpu::PC_IN_PLAIN, s->d_T1, herm ? s->d_Hh : s->d_Hf, mbirgpu::PC_OUT_PLAIN,
                 s->d_buf, 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail("Fresnel transform launch failed: %s", cudaGetErrorString(e));
    return download(s, reinterpret_cast<float2 *>(out), s->d_buf, NV);
}

int mbirgpu_pc_time_fresnel(mbirgpu_pc_session *sp, int32_t n, int32_t herm, double *ms)
{
    PCSESSION(sp);
    if (!ms || n < 1) return fail("need n >= 1 and a result pointer");
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
        if (a) cudaEventDestroy(a);
        return fail("cudaEventCreate failed");
    }
    cudaEventRecord(a, s->st);
    for (int i = 0; i < n; i++)
        s->transform(s->args(nullptr), mbirgpu::PC_IN_PLAIN, s->d_T1, herm ? s->d_Hh : s->d_Hf,
                     mbirgpu::PC_OUT_PLAIN, s->d_buf, 0);
    cudaEventRecord(b, s->st);
    cudaError_t e = cudaEventSynchronize(b);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return fail("timing the Fresnel transforms failed: %s", cudaGetErrorString(e));
    *ms = t;
    return 0;
}

int mbirgpu_pc_paganin(mbirgpu_pc_session *sp, float *zr, float *zi)
{
    PCSESSION(sp);
    s->transform(s->args(nullptr), mbirgpu::PC_IN_PAG, nullptr, s->d_Hp, mbirgpu::PC_OUT_PAG, nullptr, 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail("Paganin launch failed: %s", cudaGetErrorString(e));
    const size_t NV = (size_t)s->d.V * s->d.N;
    if (zr && download(s, zr, s->d_zr, NV)) return -1;
    if (zi && download(s, zi, s->d_zi, NV)) return -1;
    return 0;
}

int mbirgpu_pc_set_z(mbirgpu_pc_session *sp, const float *zr, const float *zi)
{
    PCSESSION(sp);
    if (!zr || !zi) return fail("NULL argument");
    const size_t NV = (size_t)s->d.V * s->d.N;
    return upload(s, s->d_zr, zr, NV) || upload(s, s->d_zi, zi, NV) ? -1 : 0;
}

int mbirgpu_pc_init_admm(mbirgpu_pc_session *sp)
{
    PCSESSION(sp);
    const size_t NV = (size_t)s->d.V * s->d.N;
    // w = e^{-z}: the prepare kernel writes buf = e^{-z} + v with v = 0
    cudaError_t e = cudaMemsetAsync(s->d_v, 0, NV * sizeof(float2), s->st);
    if (e != cudaSuccess) return fail("memset failed: %s", cudaGetErrorString(e));
    mbirgpu::pc_pret_prepare<<<s->pointwise_grid(), 256, 0, s->st>>>(s->d, s->args(nullptr));
    e = cudaMemcpyAsync(s->d_w, s->d_buf, NV * sizeof(float2), cudaMemcpyDeviceToDevice, s->st);
    if (e != cudaSuccess) return fail("copy failed: %s", cudaGetErrorString(e));
    if (s->omega_from_w(nullptr)) return -1;
    e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? 0 : fail("init failed: %s", cudaGetErrorString(e));
}

int mbirgpu_pc_set_state(mbirgpu_pc_session *sp, const float *w, const float *v, const float *omega)
{
    PCSESSION(sp);
    const size_t NV = (size_t)s->d.V * s->d.N;
    if (w && upload(s, s->d_w, reinterpret_cast<const float2 *>(w), NV)) return -1;
    if (v && upload(s, s->d_v, reinterpret_cast<const float2 *>(v), NV)) return -1;
    if (omega && upload(s, s->d_om, reinterpret_cast<const float2 *>(omega), NV)) return -1;
    return 0;
}

int mbirgpu_pc_get_state(mbirgpu_pc_session *sp, float *zr, float *zi, float *w, float *v, float *omega)
{
    PCSESSION(sp);
    const size_t NV = (size_t)s->d.V * s->d.N;
    if (zr && download(s, zr, s->d_zr, NV)) return -1;
    if (zi && download(s, zi, s->d_zi, NV)) return -1;
    if (w && download(s, reinterpret_cast<float2 *>(w), s->d_w, NV)) return -1;
    if (v && download(s, reinterpret_cast<float2 *>(v), s->d_v, NV)) return -1;
    if (omega && download(s, reinterpret_cast<float2 *>(omega), s->d_om, NV)) return -1;
    return 0;
}

int mbirgpu_pc_sd_step(mbirgpu_pc_session *sp, const float *buf, float *thresh)
{
    PCSESSION(sp);
    const size_t NV = (size_t)s->d.V * s->d.N;
    if (buf && upload(s, s->d_buf, reinterpret_cast<const float2 *>(buf), NV)) return -1;
    std::vector<int> ones(s->d.V, 1);
    if (upload(s, s->d_act_sd, ones.data(), ones.size())) return -1;
    cudaError_t e = cudaMemsetAsync(s->d_acc, 0, (size_t)s->d.V * mbirgpu::kPcAccSlots * sizeof(double), s->st);
    if (e != cudaSuccess) return fail("memset failed: %s", cudaGetErrorString(e));
    s->sd_step(s->d_act_sd, 0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail("steepest-descent launch failed: %s", cudaGetErrorString(e));
    if (thresh) return download(s, thresh, s->d_thr, s->d.V);
    e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? 0 : fail("steepest-descent step failed: %s", cudaGetErrorString(e));
}

int mbirgpu_pc_nms_sweep(mbirgpu_pc_session *sp)
{
    PCSESSION(sp);
    s->nms_sweep(s->args(nullptr));
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? 0 : fail("Nelder-Mead sweep failed: %s", cudaGetErrorString(e));
}

int mbirgpu_pc_run(mbirgpu_pc_session *sp, double *costs, int32_t *iters, mbirgpu_pc_stats *stats)
{
    PCSESSION(sp);
    return s->run(costs, iters, stats);
}

int phcontomo_reconstruct(float **magobject, float **phaseobject, float *measurements, float *brights,
                          float *proj_angles, float *proj_times, float *recon_times, int32_t proj_rows,
                          int32_t proj_cols, int32_t proj_num, int32_t recon_num, float vox_wid, float rot_center,
                          float mag_sig_s, float mag_sig_t, float mag_c_s, float mag_c_t, float phase_sig_s,
                          float phase_sig_t, float phase_c_s, float phase_c_t, float convg_thresh,
                          float obj2det_dist, float light_energy, float pag_regparam, uint8_t restart,
                          uint8_t recon_type, FILE *debug_msg_ptr)
{
    (void)proj_angles; (void)proj_times; (void)recon_times; (void)recon_num; (void)rot_center; (void)mag_sig_t;
    (void)mag_c_t; (void)phase_sig_t; (void)phase_c_t; (void)convg_thresh; (void)restart;
    if (magobject) *magobject = nullptr;
    if (phaseobject) *phaseobject = nullptr;
    if (recon_type != 1 && recon_type != 2)
        return fail("recon_type %d: only 1 (Paganin) and 2 (phase-retrieval ADMM) are supported", recon_type);
    // argument checks of PCMBIR_3D/XT_Engine.c:95-98 (one rank)
    if (proj_rows < 4) return fail("The minimum number of projection rows should be 4.");
    if (proj_cols % 2 != 0) return fail("The number of projection columns should be even.");
    if (proj_rows % 2 != 0) return fail("The number of projection rows should be an even number.");
    mbirgpu_pc_problem pb{};
    pb.measurements = measurements;
    pb.brights = brights;
    pb.proj_rows = proj_rows;
    pb.proj_cols = proj_cols;
    pb.proj_num = proj_num;
    pb.vox_wid = vox_wid;
    pb.mag_sig_s = mag_sig_s;
    pb.mag_c_s = mag_c_s;
    pb.phase_sig_s = phase_sig_s;
    pb.phase_c_s = phase_c_s;
    pb.obj2det_dist = obj2det_dist;
    pb.light_energy = light_energy;
    pb.pag_regparam = pag_regparam;
    mbirgpu_pc_options opt;
    mbirgpu_pc_default_options(&opt);
    mbirgpu_pc_session *sp = nullptr;
    if (mbirgpu_pc_session_create(&sp, &pb, &opt, nullptr)) return -1;
    const size_t NV = (size_t)proj_num * proj_rows * proj_cols;
    std::vector<float> zr(NV), zi(NV);
    std::vector<double> buf(NV);
    int rc = 0;
    if (debug_msg_ptr) std::fprintf(debug_msg_ptr, "[INFO] (mbirgpu) Phase-contrast reconstruction, type %d\n", recon_type);
    if (recon_type == 1) {
        rc = mbirgpu_pc_paganin(sp, zr.data(), zi.data());
        if (!rc) {
            for (size_t i = 0; i < NV; i++) buf[i] = zr[i];
            bool ok = write_doubles("pag_mag_ret", buf);
            for (size_t i = 0; i < NV; i++) buf[i] = zi[i];
            ok &= write_doubles("pag_phase_ret", buf);
            if (!ok) rc = fail("writing pag_mag_ret.bin / pag_phase_ret.bin failed");
        }
    } else {
        std::vector<double> a(NV), b(NV);
        if (!read_doubles("pag_mag_ret", a) || !read_doubles("pag_phase_ret", b))
            rc = fail("recon_type 2 needs pag_mag_ret.bin and pag_phase_ret.bin (run recon_type 1 first)");
        for (size_t i = 0; !rc && i < NV; i++) {
            zr[i] = (float)a[i];
            zi[i] = (float)b[i];
        }
        if (!rc) rc = mbirgpu_pc_set_z(sp, zr.data(), zi.data());
        if (!rc) rc = mbirgpu_pc_init_admm(sp);
        std::vector<double> costs((size_t)proj_num * (opt.pret_max_iter + 1));
        std::vector<int32_t> iters(proj_num);
        mbirgpu_pc_stats stats;
        if (!rc) rc = mbirgpu_pc_run(sp, costs.data(), iters.data(), &stats);
        std::vector<float> w(2 * NV), v(2 * NV), om(2 * NV);
        if (!rc) rc = mbirgpu_pc_get_state(sp, zr.data(), zi.data(), w.data(), v.data(), om.data());
        if (!rc) {
            bool ok = true;
            std::vector<double> aux(4 * NV);
            for (size_t i = 0; i < NV; i++) aux[4 * i] = aux[4 * i + 1] = aux[4 * i + 2] = aux[4 * i + 3] = zr[i];
            ok &= write_doubles("mag_tomo_aux", aux);
            for (size_t i = 0; i < NV; i++) aux[4 * i] = aux[4 * i + 1] = aux[4 * i + 2] = aux[4 * i + 3] = zi[i];
            ok &= write_doubles("phase_tomo_aux", aux);
            auto part = [&](const std::vector<float> &c, int k) {
                for (size_t i = 0; i < NV; i++) buf[i] = c[2 * i + k];
                return buf;
            };
            ok &= write_doubles("mag_pret_aux", part(w, 0)) && write_doubles("phase_pret_aux", part(w, 1));
            ok &= write_doubles("mag_pret_dual", part(v, 0)) && write_doubles("phase_pret_dual", part(v, 1));
            ok &= write_doubles("omega_real", part(om, 0)) && write_doubles("omega_imag", part(om, 1));
            for (int p = 0; p < proj_num && ok; p++) {
                std::vector<double> hist;
                for (int k = 0; k <= opt.pret_max_iter; k++) {
                    const double c = costs[(size_t)p * (opt.pret_max_iter + 1) + k];
                    if (std::isnan(c)) break;
                    hist.push_back(c);
                }
                ok &= write_doubles("pret_cost_proj_" + std::to_string(p), hist);
            }
            if (!ok) rc = fail("writing the phase-retrieval output files failed");
            if (debug_msg_ptr)
                std::fprintf(debug_msg_ptr, "[INFO] (mbirgpu) %lld steepest-descent steps, %.1f ms\n",
                             (long long)stats.sd_steps, stats.kernel_ms);
        }
    }
    mbirgpu_pc_session_destroy(sp);
    return rc;
}

}  // extern "C"
