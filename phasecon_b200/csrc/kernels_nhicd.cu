// Non-homogeneous ICD voxel-line selection on the GPU.
//
// Replaces VSC_based_Voxel_Line_Select and ComputeVSC (MBIR_4D/XT_NHICD.c:
// 128-216). Per frame: the per-column update magnitude of the latest visit
// (sum over z of |x_new - x_old|, MagUpdateMap, XT_VoxUpdate.c:158,265) is
// filtered with the reference's 5x5 Hamming window (FP64 sum, stored as
// float like filtMagUpdateMap); the threshold is the (N - k)-th smallest
// filtered value over all N = N_y N_x columns (RandomizedSelect's order
// statistic), found here by an exact 4-digit radix select on the float bit
// patterns (non-negative floats order like their bits) spread over many CTAs
// per frame; the selected columns
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

// number of selected columns of every (frame, SV); histogram per (phase, count)
__global__ void nh_count_kernel(int n_frames, int NY, int NX, int sv, int K, const uint8_t *__restrict__ sel,
                                int *__restrict__ svcount, int *__restrict__ hist)
{
    const int nsx = (NX + sv - 1) / sv, nsy = (NY + sv - 1) / sv, maxc = sv * sv;
    const long long n = (long long)n_frames * nsx * nsy;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(i / ((long long)nsx * nsy));
        const int r = (int)(i - (long long)f * nsx * nsy), sy = r / nsx, sx = r - sy * nsx;
        const uint8_t *s = sel + (size_t)f * NX * NY;
        int cnt = 0;
        for (int a = 0; a < sv; a++) {
            const int j = sy * sv + a;
            if (j >= NY) break;
            for (int b = 0; b < sv; b++) {
                const int k = sx * sv + b;
                if (k < NX) cnt += s[j * NX + k] != 0;
            }
        }
        svcount[i] = cnt;
        if (cnt) {
            const int color = (sy % K) * K + sx % K;
            const int phase = ((color - f) % (K * K) + K * K) % (K * K);
            atomicAdd(&hist[phase * (maxc + 1) + cnt], 1);
        }
    }
}

// per phase: bucket offsets, counts descending; the phase's total
__global__ void nh_offsets_kernel(int phases, int maxc, const int *__restrict__ hist, int *__restrict__ off,
                                  int *__restrict__ n_items)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= phases) return;
    int o = 0;
    for (int c = maxc; c >= 1; c--) {
        off[p * (maxc + 1) + c] = o;
        o += hist[p * (maxc + 1) + c];
    }
    n_items[p] = o;
}

// walk each phase's SVs in the sweep's own queue order (frames fastest, spread
// slots) and append the non-empty ones to their count's bucket
__global__ void nh_scatter_kernel(int n_frames, int NY, int NX, int sv, int K, int perm, int per_phase,
                                  const int *__restrict__ svcount, const int *__restrict__ off,
                                  int *__restrict__ cursor, uint32_t *__restrict__ items)
{
    const int nsx = (NX + sv - 1) / sv, nsy = (NY + sv - 1) / sv, maxc = sv * sv, KK = K * K;
    const int hx = (nsx + K - 1) / K, slots = hx * ((nsy + K - 1) / K);
    const long long n = (long long)KK * n_frames * slots;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(i / ((long long)n_frames * slots));
        const int q = (int)(i - (long long)p * n_frames * slots);
        const int f = q % n_frames;
        const int rem = (int)((long long)(q / n_frames) * perm % slots);
        const int color = (p + f) % KK;
        const int sx = K * (rem % hx) + color % K, sy = K * (rem / hx) + color / K;
        if (sx >= nsx || sy >= nsy) continue;
        const int cnt = svcount[((size_t)f * nsy + sy) * nsx + sx];
        if (!cnt) continue;
        const int pos = atomicAdd(&cursor[p * (maxc + 1) + cnt], 1);
        items[(size_t)p * per_phase + off[p * (maxc + 1) + cnt] + pos] =
            ((uint32_t)f << 22) | ((uint32_t)sy << 11) | (uint32_t)sx;
    }
}

// The order statistic by radix select over the float bit patterns, spread
// over many CTAs per frame: per 8-bit digit (most significant first) a
// histogram kernel over all keys that match the prefix so far, then a
// one-warp-per-frame kernel that picks the digit holding the rank (the
// (k+1)-th largest key, the threshold); state[f] = {prefix, prefix mask,
// remaining rank, found}. sel = mask && key > threshold: the k largest.
struct NhSelState {
    unsigned int prefix, pmask;
    int rank, found;
};

__global__ void nh_sel_init_kernel(int n_frames, int k, NhSelState *__restrict__ state, unsigned int *__restrict__ ghist)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_frames) state[i] = NhSelState{0u, 0u, k + 1, 1};
    for (int b = i; b < n_frames * 256; b += gridDim.x * blockDim.x) ghist[b] = 0u;
}

__global__ void nh_sel_hist_kernel(int nxy, int shift, const float *__restrict__ filt,
                                   const NhSelState *__restrict__ state, unsigned int *__restrict__ ghist)
{
    __shared__ unsigned int hist[256];
    const int f = blockIdx.y;
    const NhSelState st = state[f];
    if (!st.found) return;  // uniform: this frame's selection is settled
    for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0u;
    __syncthreads();
    const unsigned int *key = reinterpret_cast<const unsigned int *>(filt + (size_t)f * nxy);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nxy; i += gridDim.x * blockDim.x) {
        const unsigned int u = key[i];
        if ((u & st.pmask) == st.prefix) atomicAdd(&hist[(u >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x)
        if (hist[b]) atomicAdd(&ghist[f * 256 + b], hist[b]);
}

// one warp per frame: the digit whose cumulative count from the top reaches
// the rank; clears the histogram for the next digit
__global__ void nh_sel_pick_kernel(int shift, NhSelState *__restrict__ state, unsigned int *__restrict__ ghist)
{
    const int f = blockIdx.x, lane = threadIdx.x;
    NhSelState st = state[f];
    unsigned int *h = ghist + f * 256;
    if (st.found && lane == 0) {
        int cum = 0, b = 255;
        for (; b >= 0; b--) {
            if (cum + (int)h[b] >= st.rank) break;
            cum += (int)h[b];
        }
        if (b < 0) {  // fewer than k + 1 keys: every key is above the threshold
            st.found = 0;
        } else {
            st.prefix |= (unsigned int)b << shift;
            st.pmask |= 0xFFu << shift;
            st.rank -= cum;
        }
        state[f] = st;
    }
    __syncwarp();
    for (int b = lane; b < 256; b += 32) h[b] = 0u;
}

__global__ void nh_sel_final_kernel(int n_frames, int nxy, int k, const float *__restrict__ filt,
                                    const uint8_t *__restrict__ mask, const NhSelState *__restrict__ state,
                                    uint8_t *__restrict__ sel)
{
    const long long n = (long long)n_frames * nxy;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(i / nxy), c = (int)(i - (long long)f * nxy);
        const unsigned int u = reinterpret_cast<const unsigned int *>(filt)[i];
        const NhSelState st = state[f];
        sel[i] = (uint8_t)(k > 0 && mask[c] && (!st.found || u > st.prefix));
    }
}

}  // namespace

int nh_items_per_phase(int n_frames, int N_y, int N_x, int sv, int K)
{
    return n_frames * sv_slots(N_x, N_y, sv, K);
}

size_t nh_items_scratch_ints(int n_frames, int N_y, int N_x, int sv, int K)
{
    const size_t nsv = (size_t)((N_x + sv - 1) / sv) * ((N_y + sv - 1) / sv);
    return (size_t)n_frames * nsv + 3 * (size_t)K * K * (sv * sv + 1);
}

bool nh_items_supported(int n_frames, int N_y, int N_x, int sv)
{
    return n_frames <= 1024 && (N_x + sv - 1) / sv <= 2048 && (N_y + sv - 1) / sv <= 2048;
}

void launch_nh_items(int n_frames, int N_y, int N_x, int sv, int K, const uint8_t *d_sel, uint32_t *d_items,
                     int *d_n_items, int *d_scratch, cudaStream_t st)
{
    const int nsx = (N_x + sv - 1) / sv, nsy = (N_y + sv - 1) / sv, maxc = sv * sv, KK = K * K;
    const size_t nsv = (size_t)n_frames * nsx * nsy, hsz = (size_t)KK * (maxc + 1);
    int *svcount = d_scratch, *hist = d_scratch + nsv, *off = hist + hsz, *cursor = off + hsz;
    cudaMemsetAsync(hist, 0, hsz * sizeof(int), st);
    cudaMemsetAsync(cursor, 0, hsz * sizeof(int), st);
    const int blocks = (int)std::min<size_t>((nsv + 255) / 256, 148 * 8);
    nh_count_kernel<<<blocks, 256, 0, st>>>(n_frames, N_y, N_x, sv, K, d_sel, svcount, hist);
    nh_offsets_kernel<<<1, 32, 0, st>>>(KK, maxc, hist, off, d_n_items);
    const int per_phase = nh_items_per_phase(n_frames, N_y, N_x, sv, K);
    const long long n = (long long)KK * per_phase;
    const int sblocks = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
    nh_scatter_kernel<<<sblocks, 256, 0, st>>>(n_frames, N_y, N_x, sv, K,
                                               spread_multiplier(sv_slots(N_x, N_y, sv, K)), per_phase, svcount, off,
                                               cursor, d_items);
}

void launch_nh_select(int n_frames, int N_y, int N_x, const float *d_mag, const uint8_t *d_mask, int k,
                      float *d_filt, uint8_t *d_sel, cudaStream_t st, void *d_sel_scratch)
{
    const int nxy = N_y * N_x;
    const long long n = (long long)n_frames * nxy;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    vsc_filter_kernel<<<blocks, 256, 0, st>>>(n_frames, N_y, N_x, d_mag, d_filt);
    NhSelState *state = reinterpret_cast<NhSelState *>(d_sel_scratch);
    unsigned int *ghist = reinterpret_cast<unsigned int *>(state + n_frames);
    nh_sel_init_kernel<<<(n_frames * 256 + 255) / 256, 256, 0, st>>>(n_frames, k, state, ghist);
    // about 4 keys per thread: enough CTAs per frame to spread the reads over the GPU
    const int per_frame = std::max(1, std::min(64, (nxy + 1023) / 1024));
    for (int shift = 24; shift >= 0; shift -= 8) {
        nh_sel_hist_kernel<<<dim3(per_frame, n_frames), 256, 0, st>>>(nxy, shift, d_filt, state, ghist);
        nh_sel_pick_kernel<<<n_frames, 32, 0, st>>>(shift, state, ghist);
    }
    nh_sel_final_kernel<<<blocks, 256, 0, st>>>(n_frames, nxy, k, d_filt, d_mask, state, d_sel);
}

size_t nh_select_scratch_bytes(int n_frames)
{
    return (size_t)n_frames * (sizeof(NhSelState) + 256 * sizeof(unsigned int));
}

}  // namespace mbirgpu
