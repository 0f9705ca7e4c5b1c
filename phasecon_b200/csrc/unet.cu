// Learned warm start: a 3-D U-Net trained and run by this library's own
// kernels, mapping a filtered back-projection frame to a converged MBIR frame.
//
// Network (base width c, default 16): four levels of c, 2c, 4c, 8c channels;
// each encoder level two 3x3x3 convolutions with ReLU, 2x2x2 max-pooling
// between levels; each decoder level nearest 2x upsampling, a 3x3x3
// convolution to the level's width, concatenation with the encoder skip, and
// two 3x3x3 convolutions; a 1x1x1 head to one channel added to the input
// (the network predicts the correction to the FBP image). Activations and
// weights are BF16 ([voxel][channel], channels fastest), accumulation FP32,
// master weights and Adam state FP32.
//
// Convolutions are implicit GEMMs on the tensor cores (mma.sync m16n8k16
// BF16 -> FP32):
//   forward   out[v][co] = sum_{tap, ci} in[v + off(tap)][ci] w[tap][ci][co]
//             (M = voxels, N = co, K = 27 ci; zero padding), a CTA per
//             2 x 8 x 16 output tile whose input halo (4 x 10 x 18 voxels, 16
//             channels at a time) and weights sit in shared memory for all
//             27 taps; the one-channel first layer folds the taps into K;
//   data grad the same kernel on the output gradient with the weights
//             flipped in space and transposed in channels;
//   weight grad dw[tap][ci][co] = sum_v in[v + off(tap)][ci] g[v][co]
//             (M = ci, N = co, K = voxels) over the same tiles, all 27 taps
//             from one staged halo, FP32 atomics once per CTA.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <map>
#include <utility>
#include <vector>

#include "../../include/mbirgpu.h"
#include "mbir_internal.h"

namespace mbirgpu {

int fail(const char *fmt, ...);
int conv_tc_launch(const __nv_bfloat16 *in, int Kin, const __nv_bfloat16 *wt, __nv_bfloat16 *wtc, const float *bias,
                   __nv_bfloat16 *out, int Nout, int d, int h, int w, int df, int relu, cudaStream_t st);
int conv_tc_status(cudaStream_t st);

namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t ld_pair(const bf16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

// Four 8x8 b16 matrices from shared memory in one instruction
// (ldmatrix.x4): lane l supplies the address of row l % 8 of matrix l / 8, and
// receives its fragment of each matrix in r[0..3].
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const bf16 *p)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

constexpr int kPadK = 24;  // shared-memory row stride (16 + 8) in bf16: conflict-free fragment loads

// Output tile of the forward convolution CTA: FZ x FY x FX voxels (256 = 8
// warps x two m16 rows of 16 voxels along x); its input halo tile holds
// (FZ+2)(FY+2)(FX+2) voxels x 16 channels, staged once per 16-channel chunk
// and read by all 27 taps from shared memory.
constexpr int FZ = 2, FY = 8, FX = 16;
constexpr int FHZ = FZ + 2, FHY = FY + 2, FHX = FX + 2;
constexpr int kFHalo = FHZ * FHY * FHX;
constexpr int kFThreads = 32 * FZ * FY / 2;  // 256

template <int NT>
constexpr size_t conv_smem() { return (size_t)(kFHalo + 27 * NT) * kPadK * sizeof(bf16); }

// The weight-gradient tile: TZ x TY x TX = 128 voxels, halo (TZ+2)(TY+2)(TX+2).
constexpr int TZ = 2, TY = 4, TX = 16;
constexpr int HZ = TZ + 2, HY = TY + 2, HX = TX + 2;
constexpr int kHalo = HZ * HY * HX;

// out[v][n] = act(sum_{tap, k} in[v + off(tap)][k] wt[tap][n][k] + b[n]) with
// wt in [27][Nout][Kin] layout (the forward weights transposed per tap, or the
// data-gradient weights flipped in space); NT output channels per CTA. The
// grid is D slices deep, a stack of frames Df slices each (Df a multiple of
// FZ, so no tile straddles two frames); zero padding is per frame.
template <int NT>
__global__ void __launch_bounds__(kFThreads) conv_tile_kernel(const bf16 *__restrict__ in, int Kin,
                                                        const bf16 *__restrict__ wt, const float *__restrict__ bias,
                                                        bf16 *__restrict__ out, int Nout, int D, int H, int W,
                                                        int relu, int Df)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bf16 *Hs = reinterpret_cast<bf16 *>(smem_raw);  // [kFHalo][kPadK]
    bf16 *Ws = Hs + kFHalo * kPadK;                   // [27][NT][kPadK]
    const int tiles_x = (W + FX - 1) / FX, tiles_y = (H + FY - 1) / FY;
    int b = blockIdx.x;
    const int x0 = (b % tiles_x) * FX;
    b /= tiles_x;
    const int y0 = (b % tiles_y) * FY, z0 = (b / tiles_y) * FZ;
    const int zf0 = (z0 / Df) * Df, zf1 = min(zf0 + Df, D);  // this tile's frame
    const int n0 = blockIdx.y * NT;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    float acc[2][NT / 8][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < NT / 8; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0f;
    for (int c0 = 0; c0 < Kin; c0 += 16) {
        const bool full = c0 + 16 <= Kin;
        for (int hv = threadIdx.x; hv < kFHalo; hv += blockDim.x) {
            const int hz = hv / (FHY * FHX), r = hv - hz * (FHY * FHX), hy = r / FHX, hx = r - hy * FHX;
            const int z = z0 + hz - 1, y = y0 + hy - 1, x = x0 + hx - 1;
            bf16 *dst = Hs + hv * kPadK;
            const bool inside = z >= zf0 && z < zf1 && y >= 0 && y < H && x >= 0 && x < W;
            const long long v = ((long long)z * H + y) * W + x;
            if (inside && full) {
                const uint4 *p = reinterpret_cast<const uint4 *>(in + v * Kin + c0);
                reinterpret_cast<uint4 *>(dst)[0] = p[0];
                reinterpret_cast<uint4 *>(dst)[1] = p[1];
            } else {
                for (int k = 0; k < 16; k++)
                    dst[k] = (inside && c0 + k < Kin) ? in[v * Kin + c0 + k] : __float2bfloat16(0.0f);
            }
        }
        for (int e = threadIdx.x; e < 27 * NT; e += blockDim.x) {
            const int tap = e / NT, n = e - tap * NT;
            bf16 *dst = Ws + e * kPadK;
            const bool ok = n0 + n < Nout;
            const size_t src = ((size_t)tap * Nout + n0 + n) * Kin + c0;
            if (ok && full) {
                const uint4 *p = reinterpret_cast<const uint4 *>(wt + src);
                reinterpret_cast<uint4 *>(dst)[0] = p[0];
                reinterpret_cast<uint4 *>(dst)[1] = p[1];
            } else {
                for (int k = 0; k < 16; k++) dst[k] = (ok && c0 + k < Kin) ? wt[src + k] : __float2bfloat16(0.0f);
            }
        }
        __syncthreads();
        // ldmatrix lane roles: A (16 voxels x 16 channels) matrices are
        // (voxels 0-7 | 8-15) x (channels 0-7 | 8-15) in the mma fragment order;
        // B (16 output channels x 16 k) matrices are (outputs 0-7 | 8-15) x (k 0-7 | 8-15)
        const int lm = lane >> 3, lr = lane & 7;
        const int a_row = (lm & 1) * 8 + lr, a_k = (lm >> 1) * 8;
        const int b_row = (lm >> 1) * 8 + lr, b_k = (lm & 1) * 8;
#pragma unroll 1
        for (int tap = 0; tap < 27; tap++) {
            const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;  // halo offsets 0..2
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int row = warp * 2 + i, tz = row / FY, ty = row % FY;
                const bf16 *hrow = Hs + (((tz + dz) * FHY + ty + dy) * FHX + dx) * kPadK;
                uint32_t a[4];
                ldsm_x4(a, hrow + a_row * kPadK + a_k);
#pragma unroll
                for (int j = 0; j < NT / 8; j += 2) {
                    uint32_t b4[4];  // b4[0..1]: outputs j*8.., b4[2..3]: outputs (j+1)*8..
                    ldsm_x4(b4, Ws + (tap * NT + j * 8 + b_row) * kPadK + b_k);
                    const uint32_t b0[2] = {b4[0], b4[1]}, b1[2] = {b4[2], b4[3]};
                    mma_bf16(acc[i][j], a, b0);
                    mma_bf16(acc[i][j + 1], a, b1);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int row = warp * 2 + i, z = z0 + row / FY, y = y0 + row % FY;
        if (z >= D || y >= H) continue;
#pragma unroll
        for (int j = 0; j < NT / 8; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int x = x0 + g + h * 8;
                if (x >= W) continue;
                const long long v = ((long long)z * H + y) * W + x;
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const int n = n0 + j * 8 + tig * 2 + q;
                    if (n >= Nout) continue;
                    float val = acc[i][j][h * 2 + q] + (bias ? bias[n] : 0.0f);
                    if (relu) val = fmaxf(val, 0.0f);
                    out[v * Nout + n] = __float2bfloat16(val);
                }
            }
    }
}

// The first convolution (one input channel): the 27 taps are the GEMM's K
// (padded to 32) instead of 27 separate one-channel products. Same output tile
// as conv_tile_kernel; wt in [27][Nout][1] layout.
constexpr int kPadK32 = 40;

template <int NT>
__global__ void __launch_bounds__(kFThreads) conv_first_kernel(const bf16 *__restrict__ in,
                                                               const bf16 *__restrict__ wt,
                                                               const float *__restrict__ bias, bf16 *__restrict__ out,
                                                               int Nout, int D, int H, int W, int relu, int Df)
{
    __shared__ __align__(16) bf16 As[FZ * FY * FX][kPadK32];
    __shared__ __align__(16) bf16 Bs[NT][kPadK32];
    const int tiles_x = (W + FX - 1) / FX, tiles_y = (H + FY - 1) / FY;
    int b = blockIdx.x;
    const int x0 = (b % tiles_x) * FX;
    b /= tiles_x;
    const int y0 = (b % tiles_y) * FY, z0 = (b / tiles_y) * FZ;
    const int n0 = blockIdx.y * NT;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    {
        const int tv = threadIdx.x;  // one output voxel per thread
        const int tz = tv / (FY * FX), r = tv - tz * (FY * FX), ty = r / FX, tx = r - ty * FX;
        const int z = z0 + tz, y = y0 + ty, x = x0 + tx;
        const int zf0 = (z / Df) * Df, zf1 = min(zf0 + Df, D);  // this voxel's frame
        for (int k = 0; k < 32; k++) {
            float v = 0.0f;
            if (k < 27) {
                const int zz = z + k / 9 - 1, yy = y + (k / 3) % 3 - 1, xx = x + k % 3 - 1;
                if (zz >= zf0 && zz < zf1 && yy >= 0 && yy < H && xx >= 0 && xx < W)
                    v = __bfloat162float(in[((long long)zz * H + yy) * W + xx]);
            }
            As[tv][k] = __float2bfloat16(v);
        }
    }
    for (int e = threadIdx.x; e < NT * 32; e += blockDim.x) {
        const int n = e / 32, k = e % 32;
        Bs[n][k] = (k < 27 && n0 + n < Nout) ? wt[(size_t)k * Nout + n0 + n] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    float acc[2][NT / 8][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < NT / 8; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0f;
#pragma unroll
    for (int kk = 0; kk < 32; kk += 16)
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const bf16 *arow = &As[(warp * 2 + i) * 16][kk];
            const uint32_t a[4] = {ld_pair(arow + g * kPadK32 + tig * 2), ld_pair(arow + (g + 8) * kPadK32 + tig * 2),
                                   ld_pair(arow + g * kPadK32 + tig * 2 + 8),
                                   ld_pair(arow + (g + 8) * kPadK32 + tig * 2 + 8)};
#pragma unroll
            for (int j = 0; j < NT / 8; j++) {
                const uint32_t bb[2] = {ld_pair(&Bs[j * 8 + g][kk + tig * 2]), ld_pair(&Bs[j * 8 + g][kk + tig * 2 + 8])};
                mma_bf16(acc[i][j], a, bb);
            }
        }
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int row = warp * 2 + i, z = z0 + row / FY, y = y0 + row % FY;
        if (z >= D || y >= H) continue;
#pragma unroll
        for (int j = 0; j < NT / 8; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int x = x0 + g + h * 8;
                if (x >= W) continue;
                const long long v = ((long long)z * H + y) * W + x;
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const int n = n0 + j * 8 + tig * 2 + q;
                    if (n >= Nout) continue;
                    float val = acc[i][j][h * 2 + q] + (bias ? bias[n] : 0.0f);
                    if (relu) val = fmaxf(val, 0.0f);
                    out[v * Nout + n] = __float2bfloat16(val);
                }
            }
    }
}

// Tile-kernel weights from w[27][Cin][Cout]: forward wt[tap][co][ci] (per-tap
// transpose); data gradient wt[tap][ci][co] = w[26 - tap][ci][co] (spatial flip).
__global__ void tile_weights_kernel(const bf16 *__restrict__ w, int Cin, int Cout, int flip, bf16 *__restrict__ wt)
{
    const long long n = 27LL * Cin * Cout;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int co = (int)(i % Cout), ci = (int)((i / Cout) % Cin), tap = (int)(i / ((long long)Cout * Cin));
        if (flip) wt[((size_t)(26 - tap) * Cin + ci) * Cout + co] = w[i];
        else wt[((size_t)tap * Cout + co) * Cin + ci] = w[i];
    }
}

// Weight gradient dw[tap][ci][co] += sum_v in[v + off(tap)][ci] g[v][co]
// (M = 16 input channels, N = NT output channels, K = voxels). A CTA of 8 warps
// walks output tiles (the forward kernel's 2 x 4 x 16); per tile it stages the
// input halo transposed ([ci][halo voxel]) and the output gradient transposed
// ([co][voxel]) in shared memory, and warp w accumulates the taps w, w + 8,
// w + 16, w + 24 over all its tiles in registers before one FP32 atomic add
// per weight.
constexpr int kHaloPad = kHalo + 8;   // row stride of the transposed halo
constexpr int kTileVox = TZ * TY * TX;  // 128
constexpr int kTilePad = kTileVox + 8;

template <int NT>
__global__ void __launch_bounds__(256) conv_wgrad_tile_kernel(const bf16 *__restrict__ in, int Cin,
                                                              const bf16 *__restrict__ gout, int Cout,
                                                              float *__restrict__ dw, int D, int H, int W)
{
    __shared__ __align__(16) bf16 Ah[16][kHaloPad];
    __shared__ __align__(16) bf16 Bg[NT][kTilePad];
    const int tiles_x = (W + TX - 1) / TX, tiles_y = (H + TY - 1) / TY;
    const int n_tiles = tiles_x * tiles_y * ((D + TZ - 1) / TZ);
    const int c0 = blockIdx.y * 16, n0 = blockIdx.z * NT;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    float acc[4][NT / 8][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int j = 0; j < NT / 8; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[a][j][q] = 0.0f;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        int b = t;
        const int x0 = (b % tiles_x) * TX;
        b /= tiles_x;
        const int y0 = (b % tiles_y) * TY, z0 = (b / tiles_y) * TZ;
        for (int e = threadIdx.x; e < kHalo * 16; e += blockDim.x) {
            const int hv = e >> 4, ci = e & 15;
            const int hz = hv / (HY * HX), r = hv - hz * (HY * HX), hy = r / HX, hx = r - hy * HX;
            const int z = z0 + hz - 1, y = y0 + hy - 1, x = x0 + hx - 1;
            const bool inside = z >= 0 && z < D && y >= 0 && y < H && x >= 0 && x < W && c0 + ci < Cin;
            Ah[ci][hv] = inside ? in[(((long long)z * H + y) * W + x) * Cin + c0 + ci] : __float2bfloat16(0.0f);
        }
        for (int e = threadIdx.x; e < kTileVox * NT; e += blockDim.x) {
            const int tv = e / NT, n = e - tv * NT;
            const int tz = tv / (TY * TX), r = tv - tz * (TY * TX), ty = r / TX, tx = r - ty * TX;
            const int z = z0 + tz, y = y0 + ty, x = x0 + tx;
            const bool inside = z < D && y < H && x < W && n0 + n < Cout;
            Bg[n][tv] = inside ? gout[(((long long)z * H + y) * W + x) * Cout + n0 + n] : __float2bfloat16(0.0f);
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const int tap = warp + 8 * a;
            if (tap >= 27) break;
            const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
#pragma unroll 2
            for (int ks = 0; ks < TZ * TY; ks++) {  // one tile row of 16 voxels per k-step
                const int tz = ks / TY, ty = ks % TY;
                const int h0 = ((tz + dz) * HY + ty + dy) * HX + dx;
                auto pack = [&](int ci, int x) {
                    const uint32_t lo = __bfloat16_as_ushort(Ah[ci][h0 + x]);
                    const uint32_t hi = __bfloat16_as_ushort(Ah[ci][h0 + x + 1]);
                    return lo | (hi << 16);
                };
                const uint32_t av[4] = {pack(g, tig * 2), pack(g + 8, tig * 2), pack(g, tig * 2 + 8),
                                        pack(g + 8, tig * 2 + 8)};
#pragma unroll
                for (int j = 0; j < NT / 8; j++) {
                    const bf16 *brow = &Bg[j * 8 + g][ks * 16];
                    const uint32_t bb[2] = {ld_pair(brow + tig * 2), ld_pair(brow + tig * 2 + 8)};
                    mma_bf16(acc[a][j], av, bb);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; a++) {
        const int tap = warp + 8 * a;
        if (tap >= 27) break;
#pragma unroll
        for (int j = 0; j < NT / 8; j++)
#pragma unroll
            for (int h = 0; h < 2; h++)
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const int ci = c0 + g + h * 8, co = n0 + j * 8 + tig * 2 + q;
                    if (ci < Cin && co < Cout) atomicAdd(&dw[((size_t)tap * Cin + ci) * Cout + co], acc[a][j][h * 2 + q]);
                }
    }
}

// db[co] += sum_v g[v][co]
__global__ void bias_grad_kernel(const bf16 *__restrict__ g, long long V, int C, float *__restrict__ db)
{
    const int c = threadIdx.x % C, lanes = blockDim.x / C;
    float s = 0.0f;
    for (long long v = blockIdx.x * (long long)lanes + threadIdx.x / C; v < V && threadIdx.x < lanes * C;
         v += (long long)gridDim.x * lanes)
        s += __bfloat162float(g[v * C + c]);
    if (threadIdx.x < lanes * C) atomicAdd(&db[c], s);
}

__global__ void relu_grad_kernel(bf16 *__restrict__ g, const bf16 *__restrict__ act, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (!(__bfloat162float(act[i]) > 0.0f)) g[i] = __float2bfloat16(0.0f);
}

// 2x2x2 max-pooling of a D x H x W grid (even sizes)
__global__ void maxpool_kernel(const bf16 *__restrict__ in, int C, int D, int H, int W, bf16 *__restrict__ out)
{
    const int d = D / 2, h = H / 2, w = W / 2;
    const long long n = (long long)d * h * w * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long vo = i / C;
        const int x = (int)(vo % w), y = (int)((vo / w) % h), z = (int)(vo / ((long long)w * h));
        float m = -INFINITY;
        for (int q = 0; q < 8; q++) {
            const long long vi = ((long long)(2 * z + (q >> 2)) * H + 2 * y + ((q >> 1) & 1)) * W + 2 * x + (q & 1);
            m = fmaxf(m, __bfloat162float(in[vi * C + c]));
        }
        out[i] = __float2bfloat16(m);
    }
}

// the gradient goes to the first input of each 2x2x2 block that holds the max
__global__ void maxpool_grad_kernel(const bf16 *__restrict__ in, const bf16 *__restrict__ out,
                                    const bf16 *__restrict__ gout, int C, int D, int H, int W, bf16 *__restrict__ gin,
                                    int accumulate)
{
    const int d = D / 2, h = H / 2, w = W / 2;
    const long long n = (long long)d * h * w * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long vo = i / C;
        const int x = (int)(vo % w), y = (int)((vo / w) % h), z = (int)(vo / ((long long)w * h));
        const float m = __bfloat162float(out[i]), gv = __bfloat162float(gout[i]);
        bool done = false;
        for (int q = 0; q < 8; q++) {
            const long long vi = ((long long)(2 * z + (q >> 2)) * H + 2 * y + ((q >> 1) & 1)) * W + 2 * x + (q & 1);
            const bool hit = !done && __bfloat162float(in[vi * C + c]) == m;
            done |= hit;
            const float add = hit ? gv : 0.0f;
            gin[vi * C + c] = __float2bfloat16(accumulate ? __bfloat162float(gin[vi * C + c]) + add : add);
        }
    }
}

// nearest 2x upsampling of a d x h x w grid to 2d x 2h x 2w
__global__ void upsample_kernel(const bf16 *__restrict__ in, int C, int d, int h, int w, bf16 *__restrict__ out)
{
    const int D = 2 * d, H = 2 * h, W = 2 * w;
    const long long n = (long long)D * H * W * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long v = i / C;
        const int x = (int)(v % W), y = (int)((v / W) % H), z = (int)(v / ((long long)W * H));
        out[i] = in[(((long long)(z / 2) * h + y / 2) * w + x / 2) * C + c];
    }
}

// the same with 16-byte pieces (C a multiple of 8): thread i copies channels
// 8 (i mod C/8) .. + 7 of output voxel i / (C/8)
__global__ void upsample8_kernel(const bf16 *__restrict__ in, int C, int d, int h, int w, bf16 *__restrict__ out)
{
    const int H = 2 * h, W = 2 * w, P = C / 8;
    const long long n = (long long)2 * d * H * W * P;
    const uint4 *src = reinterpret_cast<const uint4 *>(in);
    uint4 *dst = reinterpret_cast<uint4 *>(out);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(i % P);
        const long long v = i / P;
        const int x = (int)(v % W);
        const long long r = v / W;
        const int y = (int)(r % H), z = (int)(r / H);
        dst[i] = src[(((long long)(z >> 1) * h + (y >> 1)) * w + (x >> 1)) * P + p];
    }
}

__global__ void upsample_grad_kernel(const bf16 *__restrict__ gout, int C, int d, int h, int w, bf16 *__restrict__ gin)
{
    const int H = 2 * h, W = 2 * w;
    const long long n = (long long)d * h * w * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long v = i / C;
        const int x = (int)(v % w), y = (int)((v / w) % h), z = (int)(v / ((long long)w * h));
        float s = 0.0f;
        for (int q = 0; q < 8; q++)
            s += __bfloat162float(
                gout[(((long long)(2 * z + (q >> 2)) * H + 2 * y + ((q >> 1) & 1)) * W + 2 * x + (q & 1)) * C + c]);
        gin[i] = __float2bfloat16(s);
    }
}

// cat[v] = [a[v] (Ca channels), b[v] (Cb channels)]
__global__ void concat_kernel(const bf16 *__restrict__ a, int Ca, const bf16 *__restrict__ b, int Cb, long long V,
                              bf16 *__restrict__ cat)
{
    const int C = Ca + Cb;
    const long long n = V * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long v = i / C;
        cat[i] = c < Ca ? a[v * Ca + c] : b[v * Cb + c - Ca];
    }
}

// the same with 16-byte pieces (Ca, Cb multiples of 8)
__global__ void concat8_kernel(const bf16 *__restrict__ a, int Ca, const bf16 *__restrict__ b, int Cb, long long V,
                               bf16 *__restrict__ cat)
{
    const int Pa = Ca / 8, P = (Ca + Cb) / 8, Pb = P - Pa;
    const long long n = V * P;
    const uint4 *sa = reinterpret_cast<const uint4 *>(a), *sb = reinterpret_cast<const uint4 *>(b);
    uint4 *dst = reinterpret_cast<uint4 *>(cat);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(i % P);
        const long long v = i / P;
        dst[i] = p < Pa ? sa[v * Pa + p] : sb[v * Pb + p - Pa];
    }
}

// ga = gcat[:, :Ca]; gb += gcat[:, Ca:]
__global__ void split_grad_kernel(const bf16 *__restrict__ gcat, int Ca, int Cb, long long V, bf16 *__restrict__ ga,
                                  bf16 *__restrict__ gb)
{
    const int C = Ca + Cb;
    const long long n = V * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long v = i / C;
        if (c < Ca) ga[v * Ca + c] = gcat[i];
        else gb[v * Cb + c - Ca] = __float2bfloat16(__bfloat162float(gb[v * Cb + c - Ca]) + __bfloat162float(gcat[i]));
    }
}

// y = bf16(s x): the network sees the input scaled to values of order one
__global__ void to_bf16_kernel(const float *__restrict__ x, long long n, float s, bf16 *__restrict__ y)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(s * x[i]);
}

// out[v] = in[v] + (b + sum_c w[c] x[v][c]) / s  (1x1x1 head, FP32 output, residual over the input)
__global__ void head_kernel(const bf16 *__restrict__ x, int C, const float *__restrict__ w, const float *__restrict__ b,
                            const float *__restrict__ in, long long V, float inv_s, float *__restrict__ out)
{
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        float s = b[0];
        for (int c = 0; c < C; c++) s += w[c] * __bfloat162float(x[v * C + c]);
        out[v] = in[v] + s * inv_s;
    }
}

// loss = mean (out - t)^2 (FP64 sum), g = 2 (out - t) / V; head grads: gx[v][c] = g w[c] / s,
// dw[c] += sum_v g x[v][c] / s, db += sum_v g / s.
__global__ void loss_head_grad_kernel(const float *__restrict__ out, const float *__restrict__ t, long long V,
                                      const bf16 *__restrict__ x, int C, const float *__restrict__ w, float inv_s,
                                      bf16 *__restrict__ gx, float *__restrict__ dw, float *__restrict__ db,
                                      double *__restrict__ loss)
{
    __shared__ float s_dw[128];
    __shared__ float s_db;
    __shared__ double s_loss;
    for (int c = threadIdx.x; c < C; c += blockDim.x) s_dw[c] = 0.0f;
    if (threadIdx.x == 0) {
        s_db = 0.0f;
        s_loss = 0.0;
    }
    __syncthreads();
    double l = 0.0;
    float lb = 0.0f;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
        const float d = out[v] - t[v];
        l += (double)d * d;
        const float g = 2.0f * d / (float)V * inv_s;
        lb += g;
        for (int c = 0; c < C; c++) {
            const float xv = __bfloat162float(x[v * C + c]);
            gx[v * C + c] = __float2bfloat16(g * w[c]);
            atomicAdd(&s_dw[c], g * xv);
        }
    }
    atomicAdd(&s_db, lb);
    atomicAdd(&s_loss, l / (double)V);
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&dw[c], s_dw[c]);
    if (threadIdx.x == 0) {
        atomicAdd(db, s_db);
        atomicAdd(loss, s_loss);
    }
}

// Adam on FP32 master weights; refreshes the BF16 copy.
__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2, bf16 *__restrict__ pb)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        pb[i] = __float2bfloat16(pi);
    }
}

__global__ void copy_to_bf16_kernel(const float *__restrict__ p, long long n, bf16 *__restrict__ pb)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        pb[i] = __float2bfloat16(p[i]);
}

inline unsigned grid_for(long long n, int threads = 256)
{
    return (unsigned)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 32));
}

}  // namespace

// --------------------------------------------------------------------------------------------------------------
struct UNet {
    int c = 16;
    struct Conv {
        int cin, cout;
        size_t w, b;  // offsets into the parameter arrays (FP32 master / BF16 copy)
    };
    std::vector<Conv> convs;  // 17 convolutions in forward order
    size_t head_w = 0, head_b = 0, n_params = 0;
    float *d_p = nullptr, *d_g = nullptr, *d_m = nullptr, *d_v = nullptr;
    bf16 *d_pb = nullptr, *d_wt = nullptr;  // BF16 copy; flipped weights scratch
    bf16 *d_wtc = nullptr;                   // weights re-laid for the tcgen05 kernel
    bool tensor_path = true;                 // tcgen05 convolutions where the shape allows
    bool conv_err = false;                   // a tcgen05 launch failed
    long long steps = 0;
    float scale = 1.0f;  // input scale: the network sees scale x input
    cudaStream_t st = nullptr;

    // activations (and, for training, gradients) for one grid size: D slices
    // = a stack of D / Df frames of Df slices each
    int D = 0, H = 0, W = 0, Df = 0;
    bool has_grads = false;
    std::vector<std::pair<void *, size_t>> bufs;     // activation blocks in use (pointer, bytes)
    std::multimap<size_t, void *> spare;              // released blocks kept for reuse, by size
    bf16 *x0 = nullptr;
    bf16 *act[4][2] = {};  // encoder level l: conv a, conv b (= skip)
    bf16 *pool[3] = {};    // pooled encoder output of level l (input of level l+1)
    bf16 *up[3] = {}, *u[3] = {}, *cat[3] = {}, *dec[3][2] = {};
    bf16 *gact[4][2] = {}, *gpool[3] = {}, *gup[3] = {}, *gu[3] = {}, *gcat[3] = {}, *gdec[3][2] = {};
    float *out = nullptr;
    double *d_loss = nullptr;

    ~UNet()
    {
        free_acts();
        for (auto &b : spare) cudaFree(b.second);
        for (void *p : {(void *)d_p, (void *)d_g, (void *)d_m, (void *)d_v, (void *)d_pb, (void *)d_wt,
                        (void *)d_wtc, (void *)d_loss})
            if (p) cudaFree(p);
    }
    // Activation blocks go back to a size-keyed pool instead of to the driver:
    // switching between the training grid and the stacked inference grid then
    // allocates only the first time each block size is needed.
    void free_acts()
    {
        for (auto &b : bufs) spare.emplace(b.second, b.first);
        bufs.clear();
        D = H = W = Df = 0;
        has_grads = false;
    }
    int init(int base, uint64_t seed);
    int ensure(int d, int h, int w, int frames = 1, bool grads = true);
    long long vox(int l) const { return (long long)(D >> l) * (H >> l) * (W >> l); }
    void conv(int i, const bf16 *in, bf16 *o, int l, bool relu);
    void conv_tiles(const bf16 *in, int Kin, const float *bias, bf16 *o, int Nout, int l, bool relu);
    void conv_back(int i, const bf16 *in, const bf16 *o, bf16 *go, bf16 *gin, int l);
    int forward(const float *d_in);
    int backward(const float *d_target, double *loss);
    int step(float lr);
};

int UNet::init(int base, uint64_t seed)
{
    if (base < 4 || base > 16 || base % 4) return fail("U-Net base width must be 4, 8, 12 or 16 (got %d)", base);
    c = base;
    size_t off = 0;
    auto add = [&](int cin, int cout) {
        Conv k{cin, cout, off, 0};
        off += (size_t)27 * cin * cout;
        k.b = off;
        off += cout;
        convs.push_back(k);
    };
    const int C[4] = {c, 2 * c, 4 * c, 8 * c};
    for (int l = 0; l < 4; l++) {
        add(l == 0 ? 1 : C[l - 1], C[l]);
        add(C[l], C[l]);
    }
    for (int l = 2; l >= 0; l--) {
        add(C[l + 1], C[l]);
        add(2 * C[l], C[l]);
        add(C[l], C[l]);
    }
    head_w = off;
    off += c;
    head_b = off;
    off += 1;
    n_params = off;
    // He-normal initialisation (seeded), zero biases; a small head keeps the
    // initial output close to the input
    std::vector<float> h(n_params, 0.0f);
    std::mt19937_64 rng(seed);
    for (auto &k : convs) {
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (27.0f * k.cin)));
        for (size_t i = 0; i < (size_t)27 * k.cin * k.cout; i++) h[k.w + i] = nd(rng);
    }
    std::normal_distribution<float> nh(0.0f, 1e-3f);
    for (int i = 0; i < c; i++) h[head_w + i] = nh(rng);
    cudaError_t e = cudaSuccess;
    for (float **p : {&d_p, &d_g, &d_m, &d_v})
        if (e == cudaSuccess) e = cudaMalloc((void **)p, n_params * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_pb, n_params * sizeof(bf16));
    size_t wt = 0;
    for (auto &k : convs) wt = std::max(wt, (size_t)27 * k.cin * k.cout);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_wt, wt * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_wtc, wt * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_loss, sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(d_p, h.data(), n_params * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_m, 0, n_params * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(d_v, 0, n_params * sizeof(float));
    if (e != cudaSuccess) return fail("U-Net allocation failed: %s", cudaGetErrorString(e));
    copy_to_bf16_kernel<<<grid_for((long long)n_params), 256, 0, st>>>(d_p, (long long)n_params, d_pb);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(conv_tile_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)conv_smem<64>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(conv_tile_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)conv_smem<32>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(conv_tile_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)conv_smem<16>());
    return e == cudaSuccess ? 0 : fail("U-Net init failed: %s", cudaGetErrorString(e));
}

int UNet::ensure(int d, int h, int w, int frames, bool grads)
{
    if (d * frames == D && d == Df && h == H && w == W && (has_grads || !grads)) return 0;
    if (d % 8 || h % 8 || w % 8 || d < 8 || h < 8 || w < 8)
        return fail("U-Net grid sizes must be multiples of 8 (got %d x %d x %d)", d, h, w);
    if (frames > 1 && d % 16)
        return fail("stacked frames need a depth that is a multiple of 16 (got %d)", d);
    free_acts();
    D = d * frames;
    Df = d;
    H = h;
    W = w;
    has_grads = grads;
    const int C[4] = {c, 2 * c, 4 * c, 8 * c};
    cudaError_t e = cudaSuccess;
    auto block = [&](void **p, size_t bytes) {
        if (e != cudaSuccess) return;
        auto it = spare.find(bytes);
        if (it != spare.end()) {
            *p = it->second;
            spare.erase(it);
        } else {
            e = cudaMalloc(p, bytes);
            if (e != cudaSuccess) return;
        }
        bufs.emplace_back(*p, bytes);
    };
    auto alloc = [&](bf16 **p, long long n) { block((void **)p, (size_t)n * sizeof(bf16)); };
    auto galloc = [&](bf16 **p, long long n) {  // gradient buffers: training only
        if (grads) alloc(p, n);
        else *p = nullptr;
    };
    alloc(&x0, vox(0));
    for (int l = 0; l < 4; l++)
        for (int k = 0; k < 2; k++) {
            alloc(&act[l][k], vox(l) * C[l]);
            galloc(&gact[l][k], vox(l) * C[l]);
        }
    for (int l = 0; l < 3; l++) {
        alloc(&pool[l], vox(l + 1) * C[l]);
        galloc(&gpool[l], vox(l + 1) * C[l]);
        alloc(&up[l], vox(l) * C[l + 1]);
        galloc(&gup[l], vox(l) * C[l + 1]);
        alloc(&u[l], vox(l) * C[l]);
        galloc(&gu[l], vox(l) * C[l]);
        alloc(&cat[l], vox(l) * 2 * C[l]);
        galloc(&gcat[l], vox(l) * 2 * C[l]);
        for (int k = 0; k < 2; k++) {
            alloc(&dec[l][k], vox(l) * C[l]);
            galloc(&gdec[l][k], vox(l) * C[l]);
        }
    }
    block((void **)&out, (size_t)vox(0) * sizeof(float));
    if (e != cudaSuccess) {
        free_acts();
        return fail("U-Net activation allocation failed: %s", cudaGetErrorString(e));
    }
    return 0;
}

// out = act(conv(in)) with weights in the tile layout (d_wt); Nout output channels.
void UNet::conv_tiles(const bf16 *in, int Kin, const float *bias, bf16 *o, int Nout, int l, bool relu)
{
    const int d = D >> l, h = H >> l, w = W >> l, df = Df >> l;
    const unsigned tiles = (unsigned)(((d + FZ - 1) / FZ) * ((h + FY - 1) / FY) * ((w + FX - 1) / FX));
    const int r = relu ? 1 : 0;
    if (tensor_path) {
        const int done = conv_tc_launch(in, Kin, d_wt, d_wtc, bias, o, Nout, d, h, w, df, r, st);
        if (done < 0) conv_err = true;
        if (done) return;
    }
    if (Kin == 1) {
        dim3 grid(tiles, (unsigned)((Nout + 15) / 16));
        conv_first_kernel<16><<<grid, kFThreads, 0, st>>>(in, d_wt, bias, o, Nout, d, h, w, r, df);
    } else if (Nout > 32) {
        dim3 grid(tiles, (unsigned)((Nout + 63) / 64));
        conv_tile_kernel<64><<<grid, kFThreads, conv_smem<64>(), st>>>(in, Kin, d_wt, bias, o, Nout, d, h, w, r, df);
    } else if (Nout > 16) {
        conv_tile_kernel<32><<<dim3(tiles, 1), kFThreads, conv_smem<32>(), st>>>(in, Kin, d_wt, bias, o, Nout, d, h,
                                                                                w, r, df);
    } else {
        conv_tile_kernel<16><<<dim3(tiles, 1), kFThreads, conv_smem<16>(), st>>>(in, Kin, d_wt, bias, o, Nout, d, h,
                                                                                w, r, df);
    }
}

void UNet::conv(int i, const bf16 *in, bf16 *o, int l, bool relu)
{
    const Conv &k = convs[i];
    tile_weights_kernel<<<grid_for(27LL * k.cin * k.cout), 256, 0, st>>>(d_pb + k.w, k.cin, k.cout, 0, d_wt);
    conv_tiles(in, k.cin, d_p + k.b, o, k.cout, l, relu);
}

// o = relu(conv(in)); go: gradient w.r.t. o (overwritten by the ReLU mask);
// gin (may be null): gradient w.r.t. in.
void UNet::conv_back(int i, const bf16 *in, const bf16 *o, bf16 *go, bf16 *gin, int l)
{
    const Conv &k = convs[i];
    const long long V = vox(l);
    relu_grad_kernel<<<grid_for(V * k.cout), 256, 0, st>>>(go, o, V * k.cout);
    {
        const int d = D >> l, h = H >> l, w = W >> l;
        const int tiles = ((d + TZ - 1) / TZ) * ((h + TY - 1) / TY) * ((w + TX - 1) / TX);
        const int nci = (k.cin + 15) / 16;
        const unsigned gx = (unsigned)std::max(1, std::min(tiles, 4 * 148 / std::max(1, nci)));
        if (k.cout > 32) {
            dim3 grid(gx, (unsigned)nci, (unsigned)((k.cout + 63) / 64));
            conv_wgrad_tile_kernel<64><<<grid, 256, 0, st>>>(in, k.cin, go, k.cout, d_g + k.w, d, h, w);
        } else if (k.cout > 16) {
            conv_wgrad_tile_kernel<32><<<dim3(gx, nci, 1), 256, 0, st>>>(in, k.cin, go, k.cout, d_g + k.w, d, h, w);
        } else {
            conv_wgrad_tile_kernel<16><<<dim3(gx, nci, 1), 256, 0, st>>>(in, k.cin, go, k.cout, d_g + k.w, d, h, w);
        }
    }
    const int lanes = std::max(1, 256 / k.cout);
    bias_grad_kernel<<<grid_for(V, lanes), lanes * k.cout, 0, st>>>(go, V, k.cout, d_g + k.b);
    if (gin) {
        tile_weights_kernel<<<grid_for(27LL * k.cin * k.cout), 256, 0, st>>>(d_pb + k.w, k.cin, k.cout, 1, d_wt);
        conv_tiles(go, k.cout, nullptr, gin, k.cin, l, false);
    }
}

int UNet::forward(const float *d_in)
{
    const int C[4] = {c, 2 * c, 4 * c, 8 * c};
    to_bf16_kernel<<<grid_for(vox(0)), 256, 0, st>>>(d_in, vox(0), scale, x0);
    int ci = 0;
    const bf16 *x = x0;
    for (int l = 0; l < 4; l++) {
        conv(ci++, x, act[l][0], l, true);
        conv(ci++, act[l][0], act[l][1], l, true);
        if (l < 3) {
            maxpool_kernel<<<grid_for(vox(l + 1) * C[l]), 256, 0, st>>>(act[l][1], C[l], D >> l, H >> l, W >> l,
                                                                        pool[l]);
            x = pool[l];
        }
    }
    const bf16 *y = act[3][1];
    for (int l = 2; l >= 0; l--) {
        if (C[l + 1] % 8 == 0)
            upsample8_kernel<<<grid_for(vox(l) * C[l + 1] / 8), 256, 0, st>>>(y, C[l + 1], D >> (l + 1),
                                                                             H >> (l + 1), W >> (l + 1), up[l]);
        else
            upsample_kernel<<<grid_for(vox(l) * C[l + 1]), 256, 0, st>>>(y, C[l + 1], D >> (l + 1), H >> (l + 1),
                                                                         W >> (l + 1), up[l]);
        conv(ci++, up[l], u[l], l, true);
        if (C[l] % 8 == 0)
            concat8_kernel<<<grid_for(vox(l) * 2 * C[l] / 8), 256, 0, st>>>(u[l], C[l], act[l][1], C[l], vox(l),
                                                                           cat[l]);
        else
            concat_kernel<<<grid_for(vox(l) * 2 * C[l]), 256, 0, st>>>(u[l], C[l], act[l][1], C[l], vox(l), cat[l]);
        conv(ci++, cat[l], dec[l][0], l, true);
        conv(ci++, dec[l][0], dec[l][1], l, true);
        y = dec[l][1];
    }
    head_kernel<<<grid_for(vox(0)), 256, 0, st>>>(y, c, d_p + head_w, d_p + head_b, d_in, vox(0), 1.0f / scale, out);
    cudaError_t e = cudaGetLastError();
    if (conv_err) {
        conv_err = false;
        return -1;
    }
    return e == cudaSuccess ? 0 : fail("U-Net forward failed: %s", cudaGetErrorString(e));
}

// Gradients of mean((out - target)^2) after forward(); the reverse of forward's order.
int UNet::backward(const float *d_target, double *loss)
{
    if (!has_grads || D != Df) return fail("U-Net backward needs a single-frame grid with gradient buffers");
    const int C[4] = {c, 2 * c, 4 * c, 8 * c};
    cudaError_t e = cudaMemsetAsync(d_g, 0, n_params * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_loss, 0, sizeof(double), st);
    if (e != cudaSuccess) return fail("U-Net backward failed: %s", cudaGetErrorString(e));
    loss_head_grad_kernel<<<grid_for(vox(0)), 256, 0, st>>>(out, d_target, vox(0), dec[0][1], c, d_p + head_w,
                                                            1.0f / scale, gdec[0][1], d_g + head_w, d_g + head_b,
                                                            d_loss);
    int ci = (int)convs.size() - 1;
    // decoder, finest level first
    for (int l = 0; l <= 2; l++) {
        const int i2 = ci--, i1 = ci--, iu = ci--;
        conv_back(i2, dec[l][0], dec[l][1], gdec[l][1], gdec[l][0], l);
        conv_back(i1, cat[l], dec[l][0], gdec[l][0], gcat[l], l);
        // split: the upsampled branch's gradient; the skip's gradient starts here
        cudaMemsetAsync(gact[l][1], 0, (size_t)vox(l) * C[l] * sizeof(bf16), st);
        split_grad_kernel<<<grid_for(vox(l) * 2 * C[l]), 256, 0, st>>>(gcat[l], C[l], C[l], vox(l), gu[l],
                                                                       gact[l][1]);
        conv_back(iu, up[l], u[l], gu[l], gup[l], l);
        bf16 *gy = (l == 2) ? gact[3][1] : gdec[l + 1][1];
        upsample_grad_kernel<<<grid_for(vox(l + 1) * C[l + 1]), 256, 0, st>>>(gup[l], C[l + 1], D >> (l + 1),
                                                                              H >> (l + 1), W >> (l + 1), gy);
    }
    // encoder, deepest level first
    for (int l = 3; l >= 0; l--) {
        const int ib = ci--, ia = ci--;
        if (l < 3)  // the pooled output's gradient adds to the skip's
            maxpool_grad_kernel<<<grid_for(vox(l + 1) * C[l]), 256, 0, st>>>(act[l][1], pool[l], gpool[l], C[l],
                                                                             D >> l, H >> l, W >> l, gact[l][1], 1);
        conv_back(ib, act[l][0], act[l][1], gact[l][1], gact[l][0], l);
        bf16 *gx = l > 0 ? gpool[l - 1] : nullptr;
        conv_back(ia, l > 0 ? pool[l - 1] : x0, act[l][0], gact[l][0], gx, l);
    }
    e = cudaGetLastError();
    if (conv_err) {
        conv_err = false;
        return -1;
    }
    if (e == cudaSuccess && loss) e = cudaMemcpyAsync(loss, d_loss, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && loss) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && loss && tensor_path && conv_tc_status(st))
        return fail("U-Net backward: a tensor-core convolution gave up waiting");
    return e == cudaSuccess ? 0 : fail("U-Net backward failed: %s", cudaGetErrorString(e));
}

int UNet::step(float lr)
{
    steps++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)steps), c2 = 1.0f - std::pow(b2, (float)steps);
    adam_kernel<<<grid_for((long long)n_params), 256, 0, st>>>(d_p, d_g, d_m, d_v, (long long)n_params, lr, b1, b2,
                                                               1e-8f, c1, c2, d_pb);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail("U-Net update failed: %s", cudaGetErrorString(e));
}

// The network applied to every frame of a volume [N_time][N_z][N_y][N_x]
// (FP32, device), in place; completes before returning.
int unet_apply_frames(UNet *u, float *d_vol, int N_time, int N_z, int N_y, int N_x)
{
    const size_t frame = (size_t)N_z * N_y * N_x;
    if (N_time > 1 && N_z % 16 == 0) {
        // all frames in one pass: the convolutions see a stack of frames (zero
        // padding per frame), so the coarse levels get N_time times the tiles
        if (u->ensure(N_z, N_y, N_x, N_time, false) || u->forward(d_vol)) return -1;
        cudaError_t e = cudaMemcpyAsync(d_vol, u->out, N_time * frame * sizeof(float), cudaMemcpyDeviceToDevice,
                                        u->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(u->st);
        if (e == cudaSuccess && u->tensor_path && conv_tc_status(u->st))
            return fail("U-Net inference: a tensor-core convolution gave up waiting");
        return e == cudaSuccess ? 0 : fail("U-Net inference failed: %s", cudaGetErrorString(e));
    }
    if (u->ensure(N_z, N_y, N_x)) return -1;
    for (int f = 0; f < N_time; f++) {
        if (u->forward(d_vol + f * frame)) return -1;
        cudaError_t e = cudaMemcpyAsync(d_vol + f * frame, u->out, frame * sizeof(float), cudaMemcpyDeviceToDevice,
                                        u->st);
        if (e != cudaSuccess) return fail("copy failed: %s", cudaGetErrorString(e));
    }
    cudaError_t e = cudaStreamSynchronize(u->st);
    if (e == cudaSuccess && u->tensor_path && conv_tc_status(u->st))
        return fail("U-Net inference: a tensor-core convolution gave up waiting");
    return e == cudaSuccess ? 0 : fail("U-Net inference failed: %s", cudaGetErrorString(e));
}

}  // namespace mbirgpu

using mbirgpu::fail;
using mbirgpu::UNet;

#define UNETP(up)                                    \
    if (!(up)) return fail("U-Net pointer is NULL"); \
    UNet *u = reinterpret_cast<UNet *>(up)

extern "C" {

int mbirgpu_unet_create(mbirgpu_unet **out, int32_t base_channels, uint64_t seed, void *stream)
{
    if (!out) return fail("NULL argument");
    *out = nullptr;
    UNet *u = new (std::nothrow) UNet();
    if (!u) return fail("out of host memory");
    u->st = (cudaStream_t)stream;
    if (u->init(base_channels, seed)) {
        std::string why = mbirgpu_last_error();
        delete u;
        fail("%s", why.c_str());
        return -1;
    }
    *out = reinterpret_cast<mbirgpu_unet *>(u);
    return 0;
}

int mbirgpu_unet_destroy(mbirgpu_unet *up)
{
    delete reinterpret_cast<UNet *>(up);
    return 0;
}

int64_t mbirgpu_unet_num_params(const mbirgpu_unet *up)
{
    return up ? (int64_t)reinterpret_cast<const UNet *>(up)->n_params : 0;
}

int mbirgpu_unet_set_input_scale(mbirgpu_unet *up, float scale)
{
    UNETP(up);
    if (!(scale > 0.0f)) return fail("the input scale must be positive");
    u->scale = scale;
    return 0;
}

float mbirgpu_unet_get_input_scale(const mbirgpu_unet *up)
{
    return up ? reinterpret_cast<const UNet *>(up)->scale : 0.0f;
}

int mbirgpu_unet_get_params(mbirgpu_unet *up, float *params)
{
    UNETP(up);
    if (!params) return fail("NULL argument");
    cudaError_t e = cudaMemcpy(params, u->d_p, u->n_params * sizeof(float), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : fail("copy failed: %s", cudaGetErrorString(e));
}

int mbirgpu_unet_set_params(mbirgpu_unet *up, const float *params)
{
    UNETP(up);
    if (!params) return fail("NULL argument");
    cudaError_t e = cudaMemcpy(u->d_p, params, u->n_params * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail("copy failed: %s", cudaGetErrorString(e));
    mbirgpu::copy_to_bf16_kernel<<<mbirgpu::grid_for((long long)u->n_params), 256, 0, u->st>>>(
        u->d_p, (long long)u->n_params, u->d_pb);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(u->st);
    return e == cudaSuccess ? 0 : fail("U-Net parameter upload failed: %s", cudaGetErrorString(e));
}

int mbirgpu_unet_forward(mbirgpu_unet *up, const float *d_input, float *d_output, int32_t D, int32_t H, int32_t W)
{
    UNETP(up);
    if (!d_input || !d_output) return fail("NULL argument");
    if (u->ensure(D, H, W, 1, false) || u->forward(d_input)) return -1;
    cudaError_t e = cudaMemcpyAsync(d_output, u->out, (size_t)D * H * W * sizeof(float), cudaMemcpyDeviceToDevice,
                                    u->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(u->st);
    if (e == cudaSuccess && u->tensor_path && mbirgpu::conv_tc_status(u->st))
        return fail("U-Net forward: a tensor-core convolution gave up waiting");
    return e == cudaSuccess ? 0 : fail("U-Net forward failed: %s", cudaGetErrorString(e));
}

int mbirgpu_unet_set_tensor_path(mbirgpu_unet *up, int32_t path)
{
    UNETP(up);
    if (path != 0 && path != 1) return fail("tensor path must be 0 (mma.sync) or 1 (tcgen05)");
    u->tensor_path = path == 1;
    return 0;
}

int32_t mbirgpu_unet_get_tensor_path(const mbirgpu_unet *up)
{
    return up && reinterpret_cast<const UNet *>(up)->tensor_path ? 1 : 0;
}

int mbirgpu_unet_gradients(mbirgpu_unet *up, const float *d_input, const float *d_target, int32_t D, int32_t H,
                           int32_t W, double *loss, float *grads)
{
    UNETP(up);
    if (!d_input || !d_target) return fail("NULL argument");
    if (u->ensure(D, H, W) || u->forward(d_input) || u->backward(d_target, loss)) return -1;
    if (grads) {
        cudaError_t e = cudaStreamSynchronize(u->st);
        if (e == cudaSuccess) e = cudaMemcpy(grads, u->d_g, u->n_params * sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return fail("copy failed: %s", cudaGetErrorString(e));
    }
    return 0;
}

int mbirgpu_unet_train_step(mbirgpu_unet *up, const float *d_input, const float *d_target, int32_t D, int32_t H,
                            int32_t W, float lr, double *loss)
{
    UNETP(up);
    if (!d_input || !d_target) return fail("NULL argument");
    if (u->ensure(D, H, W) || u->forward(d_input) || u->backward(d_target, loss)) return -1;
    return u->step(lr);
}

}  // extern "C"
