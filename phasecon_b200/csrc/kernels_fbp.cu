// Filtered back-projection (FBP) of the measured sinogram, the classical
// initial image (and the input of the learned warm start).
//
// Parallel beam: f(x) ~ (pi / n_views) sum_views q_v(x . theta_v), with
// q_v = delta_r (y_v * h) along the detector channels and h the Ram-Lak ramp
// filter sampled at the channel pitch (h[0] = 1 / (4 delta_r^2),
// h[odd n] = -1 / (pi n delta_r)^2, h[even n != 0] = 0). The sum over views is
// the adjoint of the session's A matrix (each voxel's footprint integrates to
// its width per view), taken per frame over that frame's views.
#include "mbir_internal.h"

namespace mbirgpu {

namespace {

constexpr double kPi = 3.14159265358979323846;

// One CTA per view: the view's [N_r][N_t] block in shared memory, every
// (channel, row) output a direct convolution over the channels (FP32 sums of
// an exactly tabulated filter). The filter is zero at even nonzero offsets,
// so the sum runs over the centre tap and the odd offsets only.
__global__ void ramp_filter_kernel(int N_r, int N_t, double delta_r, const float *__restrict__ y,
                                   float *__restrict__ q)
{
    extern __shared__ float s[];
    float *sy = s, *h = s + (size_t)N_r * N_t;  // h[n + N_r - 1], n in (-N_r, N_r)
    const size_t base = (size_t)blockIdx.x * N_r * N_t;
    for (int i = threadIdx.x; i < N_r * N_t; i += blockDim.x) sy[i] = y[base + i];
    for (int i = threadIdx.x; i < 2 * N_r - 1; i += blockDim.x) {
        const int n = i - (N_r - 1);
        double v = 0.0;
        if (n == 0) v = 1.0 / (4.0 * delta_r * delta_r);
        else if (n & 1) v = -1.0 / (kPi * kPi * (double)n * (double)n * delta_r * delta_r);
        h[i] = (float)(v * delta_r);
    }
    __syncthreads();
    for (int o = threadIdx.x; o < N_r * N_t; o += blockDim.x) {
        const int r = o / N_t, t = o - r * N_t;
        float acc = sy[r * N_t + t] * h[N_r - 1];
        // channels k = r - n for odd n: k runs over the parity opposite to r's
        for (int k = (r & 1) ^ 1; k < N_r; k += 2) acc += sy[k * N_t + t] * h[r - k + N_r - 1];
        q[base + o] = acc;
    }
}

// x[f][..] *= pi / (views of frame f)
__global__ void fbp_scale_kernel(int n_frames, size_t per_frame, const int32_t *__restrict__ view_first,
                                 float *__restrict__ x)
{
    const size_t n = (size_t)n_frames * per_frame;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int f = (int)(i / per_frame);
        const int nv = view_first[f + 1] - view_first[f];
        x[i] = nv > 0 ? (float)(kPi / nv) * x[i] : 0.0f;
    }
}

// x[f][c][..] = 0 for columns c outside the reconstruction circle
__global__ void mask_object_kernel(int n_frames, int nxy, int N_z, const uint8_t *__restrict__ mask,
                                   float *__restrict__ x)
{
    const size_t n = (size_t)n_frames * nxy * N_z;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (!mask[(i / N_z) % nxy]) x[i] = 0.0f;
}

}  // namespace

void launch_mask_object(const Geom &g, const uint8_t *d_mask, float *d_x, cudaStream_t st)
{
    mask_object_kernel<<<148 * 8, 256, 0, st>>>(g.N_time, g.N_x * g.N_y, g.N_z, d_mask, d_x);
}

void launch_fbp(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first, const int32_t *d_views,
                const float *d_y, float *d_q, float *d_x, cudaStream_t st)
{
    const size_t smem = ((size_t)g.N_r * g.N_t + 2 * (size_t)g.N_r) * sizeof(float);
    cudaFuncSetAttribute(ramp_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ramp_filter_kernel<<<g.N_p, 256, smem, st>>>(g.N_r, g.N_t, g.delta_r, d_y, d_q);
    launch_back_project(g, d_table, d_view_first, d_views, d_q, d_x, st);
    const size_t per_frame = (size_t)g.N_x * g.N_y * g.N_z;
    fbp_scale_kernel<<<148 * 8, 256, 0, st>>>(g.N_time, per_frame, d_view_first, d_x);
}

}  // namespace mbirgpu
