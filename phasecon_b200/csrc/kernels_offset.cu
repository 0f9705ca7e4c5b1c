// Nuisance parameters of the data term: the ring-correction offset d of the
// reference's update_Sinogram_Offset (MBIR_4D/XT_ICD_update.c:749-923) with
// its constraint windows (MBIR_4D/XT_OffsetError.c:46-165), and the noise
// variance of update_variance_parameter (XT_ICD_update.c:716-747).
//
// The data term is 1/2 sum w (y - Ax - d)^2 (or its generalised Huber form)
// with one offset d[r][t] per detector pixel shared by all views; the error
// sinogram holds e = y - Ax - d. An update minimises the data term over d with
// x fixed, through the surrogate weights of the Huber branch:
//   lambda_p = sum_views (select ? w : T delta sqrt(w) / |e|)
//   mode 1 (unconstrained):  d += num / lambda,      num = sum (select ? e w : T delta sqrt(w) sign e)
//   mode 2 (zero mean):      d += (num - gamma) / lambda,  gamma = sum (d + num / lambda) / sum 1 / lambda
//   mode 3 (patches):        d = argmin sum lambda (d - b / lambda)^2 subject to C d = 0,
//                            b = sum (e + d) (select ? w : T delta sqrt(w) / |e|),
// and e moves by the change of d in every view. "select" is the reference's
// ProjSelect, |e sqrt(w)| < T, evaluated on the current e. In mode 3 the
// constraint matrix C would hold overlapping rectangular windows, but the
// reference's reconstruct never builds them (gen_offset_constraint_windows is
// called only by initPhantomStructures, MBIR_4D/XT_Init.c:528; initStructures
// leaves off_constraint empty), so constrained_quad_opt runs with zero
// constraints and returns d = b / lambda. This build does exactly that.
//
// GPU layout: one thread per detector pixel p = r N_t + t walks the views
// (e[v][p], reads coalesced across threads), FP64 sums; mode 2's two global
// sums are one deterministic single-CTA reduction.
#include <algorithm>
#include <cmath>

#include "mbir_internal.h"

namespace mbirgpu {

namespace {

// per pixel: num (or b) and lambda over all views
__global__ void offset_sums_kernel(int N_p, int nrt, int mode, const float *__restrict__ e, const float *__restrict__ w,
                                   const float *__restrict__ d, double T, double delta, double *__restrict__ num,
                                   double *__restrict__ lam)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nrt; p += gridDim.x * blockDim.x) {
        double a = 0.0, l = 0.0;
        const double dp = d[p];
        for (int v = 0; v < N_p; v++) {
            const size_t i = (size_t)v * nrt + p;
            const double ev = e[i], wv = w[i];
            const double sw = sqrt(wv);
            const bool select = fabs(ev * sw) < T;
            const double wt = select ? wv : T * delta * sw / fabs(ev);
            l += wt;
            if (mode == 3) a += (ev + dp) * wt;
            else a += select ? ev * wv : T * delta * sw * (double)((ev > 0) - (ev < 0));
        }
        num[p] = a;
        lam[p] = l;
    }
}

// mode 2: gamma = sum (d + num / lambda) / sum 1 / lambda, one CTA, fixed order
__global__ void offset_gamma_kernel(int nrt, const float *__restrict__ d, const double *__restrict__ num,
                                    const double *__restrict__ lam, double *__restrict__ gamma)
{
    __shared__ double s_a[256], s_b[256];
    double a = 0.0, b = 0.0;
    for (int p = threadIdx.x; p < nrt; p += blockDim.x) {
        a += (double)d[p] + num[p] / lam[p];
        b += 1.0 / lam[p];
    }
    s_a[threadIdx.x] = a;
    s_b[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s_a[threadIdx.x] += s_a[threadIdx.x + s];
            s_b[threadIdx.x] += s_b[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *gamma = s_a[0] / s_b[0];
}

// modes 1 and 2: step = (num - gamma) / lambda; d += step; e -= step in every view
__global__ void offset_step_kernel(int N_p, int nrt, const double *__restrict__ num, const double *__restrict__ lam,
                                   const double *__restrict__ gamma, float *__restrict__ d, float *__restrict__ e)
{
    const size_t n = (size_t)N_p * nrt;
    const double g = gamma ? *gamma : 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int p = (int)(i % nrt);
        const double step = (num[p] - g) / lam[p];
        e[i] = (float)((double)e[i] - step);
        if (i < (size_t)nrt) d[p] = (float)((double)d[p] + step);
    }
}

// mode 3 with no constraints (constrained_quad_opt with M = 0,
// XT_OffsetError.c:100-165): x = b / lambda (stored in float like the
// reference's x); e += d - x in every view, then d = x (XT_ICD_update.c:789-805)
__global__ void offset_solve_kernel(int nrt, const double *__restrict__ b, const double *__restrict__ lam,
                                    float *__restrict__ x)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nrt; p += gridDim.x * blockDim.x)
        x[p] = (float)(b[p] / lam[p]);
}

__global__ void offset_replace_kernel(int N_p, int nrt, const float *__restrict__ x, const float *__restrict__ d,
                                      float *__restrict__ e)
{
    const size_t n = (size_t)N_p * nrt;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int p = (int)(i % nrt);
        e[i] += d[p] - x[p];
    }
}

__global__ void offset_copy_kernel(int n, const float *__restrict__ a, float *__restrict__ b)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// update_variance_parameter (XT_ICD_update.c:716-747), first half: the
// weights are scaled by the old variance (W1 = W v_old, stored in float) and
// each CTA sums select ? e^2 W1 : |e| delta T sqrt(W1 v_old) over its range
// ("select" = |e sqrt(W)| < T with the weights before the scaling, the
// reference's stored ProjSelect).
__global__ void variance_partial_kernel(size_t n, const float *__restrict__ e, float *__restrict__ w, double v_old,
                                        double T, double delta, double *__restrict__ partial)
{
    __shared__ double s_acc[256];
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float ev = e[i], w0 = w[i];
        const bool select = fabs((double)ev * sqrt((double)w0)) < T;
        const float w1 = (float)((double)w0 * v_old);
        w[i] = w1;
        acc += select ? (double)(ev * ev * w1) : fabs((double)ev) * delta * T * sqrt((double)w1 * v_old);
    }
    s_acc[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) s_acc[threadIdx.x] += s_acc[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s_acc[0];
}

// second half: v_new = sum / n (fixed-order sum of the partials), W = W1 / v_new
__global__ void variance_finish_kernel(int nparts, const double *__restrict__ partial, double n, double *__restrict__ v)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < nparts; i++) s += partial[i];
        *v = s / n;
    }
}

__global__ void variance_scale_kernel(size_t n, float *__restrict__ w, const double *__restrict__ v)
{
    const double vn = *v;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        w[i] = (float)((double)w[i] / vn);
}

}  // namespace

constexpr int kVarParts = 148 * 4;

size_t variance_scratch_doubles() { return kVarParts + 1; }

int variance_update(const Geom &g, int N_p, const float *d_err, float *d_w, double *var_est, double *d_scratch,
                    cudaStream_t st)
{
    const size_t n = (size_t)N_p * g.N_r * g.N_t;
    variance_partial_kernel<<<kVarParts, 256, 0, st>>>(n, d_err, d_w, *var_est, g.huber_T, g.huber_delta, d_scratch);
    variance_finish_kernel<<<1, 32, 0, st>>>(kVarParts, d_scratch, (double)n, d_scratch + kVarParts);
    variance_scale_kernel<<<148 * 8, 256, 0, st>>>(n, d_w, d_scratch + kVarParts);
    if (cudaMemcpyAsync(var_est, d_scratch + kVarParts, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return -1;
    if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int offset_update(const Geom &g, int mode, int N_p, float *d_err, const float *d_w, float *d_off, double *d_num,
                  double *d_lam, double *d_gamma, float *d_x, cudaStream_t st)
{
    const int nrt = g.N_r * g.N_t;
    const int blocks = std::max(1, std::min(148 * 4, (nrt + 127) / 128));
    offset_sums_kernel<<<blocks, 128, 0, st>>>(N_p, nrt, mode, d_err, d_w, d_off, g.huber_T, g.huber_delta, d_num,
                                               d_lam);
    const size_t n = (size_t)N_p * nrt;
    const unsigned eb = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
    if (mode == 1 || mode == 2) {
        if (mode == 2) offset_gamma_kernel<<<1, 256, 0, st>>>(nrt, d_off, d_num, d_lam, d_gamma);
        offset_step_kernel<<<eb, 256, 0, st>>>(N_p, nrt, d_num, d_lam, mode == 2 ? d_gamma : nullptr, d_off, d_err);
    } else {
        offset_solve_kernel<<<blocks, 128, 0, st>>>(nrt, d_num, d_lam, d_x);
        offset_replace_kernel<<<eb, 256, 0, st>>>(N_p, nrt, d_x, d_off, d_err);
        offset_copy_kernel<<<blocks, 128, 0, st>>>(nrt, d_x, d_off);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace mbirgpu
