// Non-homogeneous ICD voxel-line selection on the GPU.
//
// Replaces VSC_based_Voxel_Line_Select and ComputeVSC (MBIR_4D/XT_NHICD.c:
// 128-216). Per frame: the per-column update magnitude of the latest visit
// (sum over z of |x_new - x_old|, MagUpdateMap, XT_VoxUpdate.c:158,265) is
// filtered with the reference's 5x5 Hamming window (FP64 sum, stored as
// float like filtMagUpdateMap); the threshold is the (N - k)-th smallest
// filtered value over all N = N_y N_x columns (RandomizedSelect's order
// statistic), found here by an exact 4-digit radix select on the float bit
// patterns (non-negative floats order like their bits); the selected columns
// are those strictly above it -- the k largest -- that lie inside the mask
// (the reference also picks unmasked columns near the edge but its update
// skips them, XT_VoxUpdate.c:168).
#include <algorithm>

#include "mbir_internal.h"

namespace mbirgpu {

namespace {

__constant__ double c_hamming[5][5] = {{0.0064, 0.0432, 0.0800, 0.0432, 0.0064},
                                       {0.0432, 0.2916, 0.5400, 0.2916, 0.0432},
                                       {0.0800, 0.5400, 1.0000, 0.5400, 0.0800},
                                       {0.0432, 0.2916, 0.5400, 0.2916, 0.0432},
                                       {0.0064, 0.0432, 0.0800, 0.0432, 0.0064}};

__global__ void vsc_filter_kernel(int n_frames, int NY, int NX, const float *__restrict__ mag,
                                  float *__restrict__ filt)
{
    const int nxy = NX * NY;
    const long long n = (long long)n_frames * nxy;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(i / nxy), c = (int)(i - (long long)f * nxy);
        const int j = c / NX, k = c - j * NX;
        const float *m = mag + (size_t)f * nxy;
        double acc = 0.0;
        for (int p = -2; p <= 2; p++) {
            const int jj = j + p;
            if (jj < 0 || jj >= NY) continue;
            for (int q = -2; q <= 2; q++) {
                const int kk = k + q;
                if (kk < 0 || kk >= NX) continue;
                acc = __dadd_rn(acc, __dmul_rn(c_hamming[p + 2][q + 2], (double)m[jj * NX + kk]));  // no contraction, as the host
            }
        }
        filt[i] = (float)acc;
    }
}

// One CTA per frame: T = the (k+1)-th largest key (the (N-k)-th smallest), then
// sel = mask && key > T.
__global__ void __launch_bounds__(1024) nh_select_kernel(int nxy, int k, const float *__restrict__ filt,
                                                         const uint8_t *__restrict__ mask, uint8_t *__restrict__ sel)
{
    __shared__ unsigned int hist[256];
    __shared__ unsigned int s_prefix;
    __shared__ int s_rank;
    const int f = blockIdx.x;
    const unsigned int *key = reinterpret_cast<const unsigned int *>(filt + (size_t)f * nxy);
    uint8_t *out = sel + (size_t)f * nxy;
    if (k <= 0) {  // nothing to select: the threshold is the maximum
        for (int i = threadIdx.x; i < nxy; i += blockDim.x) out[i] = 0;
        return;
    }
    unsigned int prefix = 0, pmask = 0;
    int rank = k + 1;  // 1-based rank from the top
    bool found = true;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < nxy; i += blockDim.x) {
            const unsigned int u = key[i];
            if ((u & pmask) == prefix) atomicAdd(&hist[(u >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int cum = 0, b = 255;
            for (; b >= 0; b--) {
                if (cum + (int)hist[b] >= rank) break;
                cum += (int)hist[b];
            }
            if (b < 0) {  // fewer than k + 1 keys: every key is above the threshold
                s_rank = -1;
            } else {
                s_prefix = prefix | ((unsigned int)b << shift);
                s_rank = rank - cum;
            }
        }
        __syncthreads();
        if (s_rank < 0) {
            found = false;
            break;
        }
        prefix = s_prefix;
        rank = s_rank;
        pmask |= 0xFFu << shift;
        __syncthreads();
    }
    for (int i = threadIdx.x; i < nxy; i += blockDim.x)
        out[i] = (uint8_t)(mask[i] && (!found || key[i] > prefix));
}

}  // namespace

void launch_nh_select(int n_frames, int N_y, int N_x, const float *d_mag, const uint8_t *d_mask, int k,
                      float *d_filt, uint8_t *d_sel, cudaStream_t st)
{
    const long long n = (long long)n_frames * N_y * N_x;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    vsc_filter_kernel<<<blocks, 256, 0, st>>>(n_frames, N_y, N_x, d_mag, d_filt);
    nh_select_kernel<<<n_frames, 1024, 0, st>>>(N_y * N_x, k, d_filt, d_mask, d_sel);
}

}  // namespace mbirgpu
