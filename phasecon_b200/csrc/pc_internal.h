// Internal declarations of the phase-contrast (PCMBIR) part of libmbirgpu.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

namespace mbirgpu {

// Per-view FP64 accumulator slots.
enum PcAcc {
    PC_ACC_GG = 0,      // sum |g|^2 (step-size numerator)
    PC_ACC_DEN = 1,     // sum Re(conj g D^H H'^H Omega^H Lambda Omega H D g)
    PC_ACC_UP = 2,      // sum |alpha g|
    PC_ACC_VAL = 3,     // sum |w|
    PC_ACC_PRIMAL = 4,  // sum |e^{-z} - w|^2
    PC_ACC_DUALW = 5,   // sum |w - w_old|^2
    PC_ACC_VSUM = 6,    // sum |v|^2
    PC_ACC_PCOST = 7,   // data term of the phase-retrieval cost
    PC_ACC_PRIOR = 8,   // prior term of the phase-retrieval cost
};
constexpr int kPcAccSlots = 16;

enum PcPrologue { PC_IN_PLAIN = 0, PC_IN_DW = 1, PC_IN_DEZ = 2, PC_IN_PAG = 3 };
enum PcEpilogue {
    PC_OUT_PLAIN = 0,
    PC_OUT_GRES = 1,
    PC_OUT_GRAD = 2,
    PC_OUT_SFWD = 3,
    PC_OUT_SDEN = 4,
    PC_OUT_OMEGA = 5,
    PC_OUT_PCOST = 6,
    PC_OUT_PAG = 7,
};

struct PcDims {
    int V, R, C, N, logR, logC, nmax;
    int rows_per_cta, cols_per_cta;
    float nu, delta_over_beta;
    int fft_radix;  // largest radix of an FFT stage (2, 4, 8, 16)
};

// Device pointers (any may be null when the op does not use it).
struct PcArgs {
    const float2 *tw;                 // twiddles exp(-2 pi i m / nmax), m < nmax/2
    float2 *work;                     // [V][R][C] spectrum scratch
    const float2 *in;                 // prologue input
    float2 *out;                      // epilogue output
    const float *D;                   // [R][C] sqrt(bright) / sqrt(mean bright)
    const float *y;                   // [V][R][C] sqrt(intensity) / sqrt(mean bright)
    const float *lam;                 // [V][R][C] weights (null: all ones)
    float2 *omega, *w, *wold, *g, *buf, *vdual;
    float *zr, *zi;
    double *acc;                      // [V][kPcAccSlots]
    int acc_slot;
    int *active;                      // per-view loop flag (null: all views)
    float *sd_thresh_out;
    int *sd_steps, *pret_iters;
    double *dual_res, *primal_res;
};

struct PcPrior {
    double f[9];                           // in-plane neighbour weights [dy][dx]
    double T00, T01, T10, T11;             // decorrelating transform
    double ph_sq, ph_sqp, ph_c, mg_sq, mg_sqp, mg_c, qmp;
    float ph_isq_f, ph_isqp_f, ph_c_f, mg_isq_f, mg_isqp_f, mg_c_f, qmp_f;
    float f_f[9], T00_f, T01_f, T10_f, T11_f;  // FP32 copies for the per-pixel search
};

__global__ void pc_rows_forward(PcDims d, PcArgs A, int prologue);
__global__ void pc_cols_filter(PcDims d, PcArgs A, const float2 *transfer);
__global__ void pc_rows_inverse(PcDims d, PcArgs A, int epilogue);
// the same passes for 256-point sequences with radix-16 stages, the points in
// registers (16 sequences per 256-thread CTA)
__global__ void pc_rows_forward_256(PcDims d, PcArgs A, int prologue);
__global__ void pc_cols_filter_256(PcDims d, PcArgs A, const float2 *transfer);
__global__ void pc_rows_inverse_256(PcDims d, PcArgs A, int epilogue);
__global__ void pc_sd_update(PcDims d, PcArgs A);
__global__ void pc_sd_finish(PcDims d, PcArgs A, int step, float sd_thresh);
__global__ void pc_pret_prepare(PcDims d, PcArgs A);
__global__ void pc_pret_dual(PcDims d, PcArgs A);
__global__ void pc_prior_cost(PcDims d, PcArgs A, const __grid_constant__ PcPrior P);
__global__ void pc_pret_finish(PcDims d, PcArgs A, int iter, float pret_thresh, double *costs_out);
// One Nelder-Mead proximal sweep over the active views: order 0 the raster
// order by anti-diagonal wavefronts (one launch, clusters of ctas CTAs per
// view), 1 the four colour classes (four launches of the pointwise grid);
// lanes (1, 2, 4, 8) share one pixel's search. Returns the kernels launched.
int launch_nms_sweep(const PcDims &d, const PcArgs &A, const PcPrior &P, int order, int lanes, int ctas,
                     int max_iter, float threshold, dim3 pointwise, cudaStream_t st);
// lanes per pixel and CTAs per view of the proximal sweep when none are asked for
constexpr int kPcDefaultNmsLanes = 4;
constexpr int kPcDefaultNmsCtas = 4;

// Launch geometry of the three-pass transform for V views of R x C (powers of
// two): fills d's sizes and per-CTA tiles, the dynamic shared memory of the
// row and column passes, and raises the kernels' shared-memory limits.
int pc_transform_dims(PcDims &d, int V, int R, int C, size_t *smem_rows, size_t *smem_cols, int fft_radix = 0);
// the FFT stage radix used when none is asked for
constexpr int kPcDefaultFftRadix = 16;
// float2 slots one FFT sequence of length n takes in shared memory: n plus
// one padding slot per 16, rounded up to an odd count
__host__ __device__ inline int fft_seq_stride(int n) { return (n + n / 16) | 1; }
// exp(-2 pi i m / nmax), m < nmax / 2, computed in double and rounded once
std::vector<float2> pc_twiddles(int nmax);
// One Fresnel-type transform of every view: prologue + FFT along C, FFT along
// R x transfer table x inverse FFT along R, inverse FFT along C / N + epilogue.
void pc_transform(const PcDims &d, PcArgs A, size_t smem_rows, size_t smem_cols, int prologue, const float2 *in,
                  const float2 *table, int epilogue, float2 *out, int acc_slot, cudaStream_t st);
int fail(const char *fmt, ...);

}  // namespace mbirgpu
