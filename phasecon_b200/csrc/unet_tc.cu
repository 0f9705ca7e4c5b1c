// The U-Net's 3x3x3 convolutions on the fifth-generation tensor cores:
// tcgen05.mma with the accumulators in tensor memory (TMEM), operands in
// shared memory.
//
//   out[v][n] = act(sum_{tap, k} in[v + off(tap)][k] wt[tap][n][k] + b[n])
//
// is an implicit GEMM with M = output voxels, N = output channels, K = 27 taps
// x input channels. A CTA owns TZ x 16 x 8 output voxels (z, y, x) and NT
// output channels. For each 16-channel chunk of the input, producer warps
// stage the (TZ+2) x 18 x 10 halo in shared memory as two 8-channel halves,
// each [halo voxel][8 channels] (16 bytes a voxel, zeros outside the grid,
// which is the convolution's zero padding), and a TMA bulk copy brings the
// chunk's weights. The halo needs no im2col: in the canonical K-major layout
// without swizzle a tcgen05 operand is 8-row core matrices of 16-byte rows,
// rows 16 bytes apart, core matrices SBO bytes apart along M and LBO bytes
// apart along K. Eight consecutive x voxels of one halo row are such a core
// matrix; sixteen output rows y are sixteen core matrices one halo row (160
// bytes) apart; the two channel halves are LBO = one half-halo apart. The A
// operand of tap (dz, dy, dx) and output plane zt is therefore the same
// shared-memory tile with its start address moved by
// ((zt + dz) * 18 + dy) * 10 + dx voxels: 27 x TZ MMAs (M = 128, N = NT,
// K = 16) per chunk read the staged halo in place.
//
// The halo is staged by threads rather than by a TMA tile load: a tile load
// whose box rows are 16 bytes (8 channels of one voxel, the row of a core
// matrix) moved about 8 bytes per cycle per SM, which bound the kernel; 128
// producer threads issue 16-byte asynchronous copies (cp.async, zero-filled
// outside the grid) whose completion arrives on the stage's mbarrier, so the
// producers run ahead over all stages without holding the data in
// registers; the MMA issuer orders the copies before the tensor cores' reads
// (fence.proxy.async) once the stage is full.
//
// Persistent, warp-specialised CTA (one per SM), 9 warps:
//   warps 0-3       producers: per (tile, chunk) item, wait for a free stage;
//                   thread 0 posts the weight bytes on the stage's "full"
//                   mbarrier and issues their bulk copy; all 128 threads copy
//                   the halo (16-byte pieces, coalesced) and arrive when their
//                   copies land;
//   warps 4-7       epilogue: tcgen05.ld of the accumulator (warp w reads the
//                   TMEM lanes of its quadrant w % 4 = output rows), bias,
//                   ReLU, BF16, 32-byte stores; then free the accumulator;
//   warp 8 lane 0   MMA issuer: waits for a full stage and for a free TMEM
//                   accumulator, issues the tile's MMAs, and commits them to
//                   the stage's "empty" mbarrier (the stage is reused once the
//                   MMAs that read it are done) and, after a tile's last
//                   chunk, to the accumulator's "full" mbarrier.
// Every CTA serves one N slice (its weights never change) and walks tiles
// with a stride of the CTAs per slice. TMEM holds two accumulators (2 x TZ x
// NT FP32 columns), so the epilogue of one tile overlaps the MMAs of the
// next. Every wait is bounded: a wait that runs out records an error code
// that the host reads, and the CTA stops its loops, waits (bounded) for its
// own MMAs, frees its TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "mbir_internal.h"

namespace mbirgpu {

int fail(const char *fmt, ...);

namespace {

using bf16 = __nv_bfloat16;

constexpr int TZ = 2, TYY = 16, TXX = 8;                      // output tile (z, y, x): 256 voxels, 2 MMAs of M = 128
constexpr int HZ = TZ + 2, HY = TYY + 2, HX = TXX + 2;        // halo 4 x 18 x 10
constexpr int kHalo = HZ * HY * HX;                           // 720 voxels
constexpr int kHalfBytes = kHalo * 16;                        // one 8-channel half: 11,520 bytes
constexpr int kProducers = 128;                               // warps 0-3
constexpr int kThreads = 288;                                 // producers, 4 epilogue warps, MMA warp
constexpr int kHaloItems = 2 * kHalo;                         // 16-byte halo pieces per chunk
constexpr int kPerProducer = (kHaloItems + kProducers - 1) / kProducers;  // 12
constexpr long long kWaitCycles = 4000000000LL;               // about 2 s at the boost clock

__device__ int g_conv_tc_error = 0;

template <int NT>
struct Cfg {
    static constexpr int kWBytes = 27 * NT * 32;               // one chunk's weights: 27 taps x NT x 16 bf16
    static constexpr int kStage = 2 * kHalfBytes + kWBytes;   // multiple of 128 bytes
    static constexpr int kStages = NT == 64 ? 2 : NT == 32 ? 3 : 4;
    static constexpr int kAcc = TZ * NT;                      // FP32 columns of one accumulator
    static constexpr int kTmemCols = 2 * kAcc;                // 64, 128, 256: a power of two >= 32
    static constexpr size_t kSmem = (size_t)kStages * kStage + 1024;
    static_assert(kStage % 128 == 0, "stage size");
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity. Returns false (and
// records `code`) when it runs out or when another role of the CTA gave up.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort, int code, unsigned sleep_ns = 0)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (sleep_ns) __nanosleep(sleep_ns);  // leave the issue slots to the warps doing work
        if (*abort) return false;
        if (clock64() - t0 > kWaitCycles) {
            *abort = 1;
            atomicCAS(&g_conv_tc_error, 0, code);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void mbar_expect_tx_only(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Shared-memory matrix descriptor: canonical K-major layout, no swizzle
// (start, LBO, SBO in 16-byte units; bits 46-47 = 1 for this architecture).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_ss(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 FP32 columns of this warp's 32 TMEM lanes into v[0..15]. The load and
// its wait are one asm statement, so no instruction can read the destination
// registers before the asynchronous load has written them.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

struct Grid {
    int d, h, w, df;         // stacked depth, height, width, frame depth
    int tiles_x, tiles_y, tiles, nsplit, nchunks;
};

__device__ __forceinline__ void tile_coords(const Grid &g, int t, int &x0, int &y0, int &z0)
{
    x0 = (t % g.tiles_x) * TXX;
    t /= g.tiles_x;
    y0 = (t % g.tiles_y) * TYY;
    z0 = (t / g.tiles_y) * TZ;
}

template <int NT>
__global__ void __launch_bounds__(kThreads, 1)
    conv_tc_kernel(const bf16 *__restrict__ in, int Kin, const bf16 *__restrict__ wtc,
                   const float *__restrict__ bias, bf16 *__restrict__ out, int Nout, Grid g, int relu)
{
    using C = Cfg<NT>;
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar_full[C::kStages], bar_empty[C::kStages];
    __shared__ __align__(8) uint64_t bar_acc_full[2], bar_acc_empty[2], bar_done;
    __shared__ uint32_t tmem_base_s;
    __shared__ int abort_s;
    __shared__ float bias_s[NT];
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // this CTA's N slice and its tiles: tile = slot, slot + stride, ...
    const int ns = blockIdx.x % g.nsplit, slot = blockIdx.x / g.nsplit, stride = gridDim.x / g.nsplit;
    const int n0 = ns * NT;

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::kStages; s++) {
            mbar_init(smem_u32(&bar_full[s]), kProducers);
            mbar_init(smem_u32(&bar_empty[s]), 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(smem_u32(&bar_acc_full[a]), 1);
            mbar_init(smem_u32(&bar_acc_empty[a]), 4);
        }
        mbar_init(smem_u32(&bar_done), 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < NT) bias_s[threadIdx.x] = bias ? bias[n0 + threadIdx.x] : 0.0f;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(C::kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    volatile int *abort = &abort_s;

    if (warp < 4) {
        // ---- producers: halo by 128 threads, weights by one bulk copy ----
        int it = 0;
        const int tid = threadIdx.x;
        for (int t = slot; t < g.tiles && !*abort; t += stride) {
            int x0, y0, z0;
            tile_coords(g, t, x0, y0, z0);
            const int zf0 = (z0 / g.df) * g.df, zf1 = zf0 + g.df;  // this tile's frame
            bool ok = true;
            for (int c = 0; c < g.nchunks; c++, it++) {
                const int s = it % C::kStages;
                const uint32_t ph = (uint32_t)(it / C::kStages) & 1u;
                int wok = 0;
                if (lane == 0) wok = mbar_wait(smem_u32(&bar_empty[s]), ph ^ 1u, abort, 1, 64) ? 1 : 0;
                if (!__shfl_sync(0xffffffffu, wok, 0)) {
                    ok = false;
                    break;
                }
                const uint32_t st = base + (uint32_t)s * C::kStage, fb = smem_u32(&bar_full[s]);
                if (tid == 0) {
                    mbar_expect_tx_only(fb, (uint32_t)C::kWBytes);
                    bulk_load(st + 2 * kHalfBytes, wtc + ((size_t)ns * g.nchunks + c) * (C::kWBytes / 2),
                              (uint32_t)C::kWBytes, fb);
                }
                // the halo by asynchronous 16-byte copies (zero-filled outside
                // the frame: the convolution's padding) that hold no registers
                // while in flight, so the producers go on to the next free
                // stage at once; the stage's mbarrier sees each thread's arrival
                // when its copies have landed
#pragma unroll
                for (int r = 0; r < kPerProducer; r++) {
                    const int e = tid + r * kProducers;  // piece e: halo voxel e / 2, channel half e % 2
                    if (e < kHaloItems) {
                        const int hv = e >> 1, hz = hv / (HY * HX), rr = hv - hz * (HY * HX), hy = rr / HX,
                                  hx = rr - hy * HX;
                        const int z = z0 + hz - 1, y = y0 + hy - 1, x = x0 + hx - 1;
                        const bool inb = z >= zf0 && z < zf1 && z < g.d && y >= 0 && y < g.h && x >= 0 && x < g.w;
                        const bf16 *src =
                            inb ? in + (((long long)z * g.h + y) * g.w + x) * Kin + c * 16 + (e & 1) * 8 : in;
                        const uint32_t dst = st + (uint32_t)((e & 1) * kHalfBytes + (e >> 1) * 16);
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
                                     "r"(inb ? 16 : 0)
                                     : "memory");
                    }
                }
                asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(fb) : "memory");
            }
            if (!ok) break;
        }
        // no copy of this thread may land after the CTA has gone
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp < 8) {
        // ---- epilogue ----
        const int q = warp & 3;             // TMEM lane quadrant = output rows 32q .. 32q + 31
        const int m = q * 32 + lane;        // row of the M = 128 tile
        const int yl = m >> 3, xl = m & 7;
        int ut = 0;
        for (int t = slot; t < g.tiles; t += stride, ut++) {
            const int a = ut & 1;
            const uint32_t aph = (uint32_t)(ut >> 1) & 1u;
            // lane 0 waits and tells the warp, so the warp stays converged for
            // the warp-wide tcgen05.ld whatever the wait's outcome
            int wok = 0;
            if (lane == 0) wok = mbar_wait(smem_u32(&bar_acc_full[a]), aph, abort, 4, 64) ? 1 : 0;
            if (!__shfl_sync(0xffffffffu, wok, 0)) break;
            tc_fence_after();
            int x0, y0, z0;
            tile_coords(g, t, x0, y0, z0);
            const int zl = z0 % g.df, y = y0 + yl, x = x0 + xl;
#pragma unroll
            for (int zt = 0; zt < TZ; zt++) {
                const bool inside = zl + zt < g.df && z0 + zt < g.d && y < g.h && x < g.w;
                const long long v = (((long long)(z0 + zt) * g.h + y) * g.w + x);
                float acc[NT];
#pragma unroll
                for (int j = 0; j < NT / 16; j++)
                    tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * C::kAcc + zt * NT + j * 16),
                              acc + j * 16);
                if (inside) {
#pragma unroll
                    for (int j = 0; j < NT / 16; j++) {
                        alignas(16) bf16 o[16];
#pragma unroll
                        for (int i = 0; i < 16; i++) {
                            float val = acc[j * 16 + i] + bias_s[j * 16 + i];
                            if (relu) val = fmaxf(val, 0.0f);
                            o[i] = __float2bfloat16(val);
                        }
                        uint4 *dst = reinterpret_cast<uint4 *>(out + v * Nout + n0 + j * 16);
                        dst[0] = reinterpret_cast<const uint4 *>(o)[0];
                        dst[1] = reinterpret_cast<const uint4 *>(o)[1];
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar_acc_empty[a]));
        }
    } else if (lane == 0) {
        // ---- MMA issuer ----
        constexpr uint32_t idesc = idesc_bf16(NT);
        int it = 0, ut = 0;
        bool ok = true;
        for (int t = slot; t < g.tiles && ok; t += stride, ut++) {
            const int a = ut & 1;
            const uint32_t aph = (uint32_t)(ut >> 1) & 1u;
            if (!(ok = mbar_wait(smem_u32(&bar_acc_empty[a]), aph ^ 1u, abort, 2))) break;
            tc_fence_after();
            const uint32_t d0 = tmem + (uint32_t)(a * C::kAcc);
            for (int c = 0; c < g.nchunks; c++, it++) {
                const int s = it % C::kStages;
                const uint32_t ph = (uint32_t)(it / C::kStages) & 1u;
                if (!(ok = mbar_wait(smem_u32(&bar_full[s]), ph, abort, 3))) break;
                tc_fence_after();
                // the halo was written by the producers' copies (generic proxy)
                // and is read by the tensor cores (async proxy)
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                const uint32_t st = base + (uint32_t)s * C::kStage;
                // descriptors of tap 0; a tap moves the start address (16-byte
                // units in the low bits, which cannot carry: the stage lies
                // below 256 KB) by a compile-time offset
                const uint64_t a0 = sdesc(st, kHalfBytes, HX * 16);
                const uint64_t b0 = sdesc(st + 2 * kHalfBytes, 128, 256);
#pragma unroll
                for (int tap = 0; tap < 27; tap++) {
                    const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
#pragma unroll
                    for (int zt = 0; zt < TZ; zt++) {
                        const uint32_t aoff = (uint32_t)((((zt + dz) * HY + dy) * HX + dx) * 16);
                        mma_bf16_ss(d0 + (uint32_t)(zt * NT), a0 + (aoff >> 4), b0 + (uint32_t)(tap * NT * 2), idesc,
                                    (c > 0 || tap > 0) ? 1u : 0u);
                    }
                }
                mma_commit(smem_u32(&bar_empty[s]));
            }
            if (ok) mma_commit(smem_u32(&bar_acc_full[a]));
        }
        // all MMAs issued by this thread are complete before TMEM is released
        mma_commit(smem_u32(&bar_done));
        const long long t0 = clock64();
        while (!mbar_try_wait(smem_u32(&bar_done), 0u) && clock64() - t0 < kWaitCycles) {
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::kTmemCols)
                     : "memory");
    }
}

// wtc[ns][c][tap][g][half][r][k] = wt[tap][ns NT + 8 g + r][16 c + 8 half + k]:
// each (ns, chunk) block is the shared-memory image of the chunk's B operands
// (27 taps of NT x 16, K-major core matrices: 8 rows x 16 bytes, the two
// 8-channel halves 128 bytes apart, row groups 256 bytes apart).
__global__ void tc_weights_kernel(const bf16 *__restrict__ wt, int Kin, int Nout, int NT, bf16 *__restrict__ wtc)
{
    const long long n = 27LL * Nout * Kin;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long r = i;
        const int k = (int)(r % 8); r /= 8;
        const int row = (int)(r % 8); r /= 8;
        const int half = (int)(r % 2); r /= 2;
        const int grp = (int)(r % (NT / 8)); r /= NT / 8;
        const int tap = (int)(r % 27); r /= 27;
        const int c = (int)(r % (Kin / 16));
        const int ns = (int)(r / (Kin / 16));
        const int co = ns * NT + grp * 8 + row, ci = c * 16 + half * 8 + k;
        wtc[i] = wt[((size_t)tap * Nout + co) * Kin + ci];
    }
}

int sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
                                                      cudaSuccess)
            n = 148;
    }
    return n;
}

template <int NT>
int launch(const bf16 *in, int Kin, const bf16 *wtc, const float *bias, bf16 *out, int Nout, const Grid &g, int relu,
           cudaStream_t st)
{
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(conv_tc_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg<NT>::kSmem) != cudaSuccess)
            return fail("tensor-core convolution: shared-memory attribute refused");
        attr = true;
    }
    // CTAs per N slice: one per SM in all, at most one per tile
    const int per_slice = std::max(1, std::min(g.tiles, sm_count() / g.nsplit));
    conv_tc_kernel<NT><<<(unsigned)(per_slice * g.nsplit), kThreads, Cfg<NT>::kSmem, st>>>(in, Kin, wtc, bias, out,
                                                                                          Nout, g, relu);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 1 : fail("tensor-core convolution launch failed: %s", cudaGetErrorString(e));
}

}  // namespace

// Output channels per CTA for a convolution with Nout outputs (0: the shape is
// not served by the tensor-core kernel).
int conv_tc_split(int Kin, int Nout)
{
    if (Kin < 16 || Kin % 16 || Nout % 16) return 0;
    return Nout % 64 == 0 ? 64 : Nout % 32 == 0 ? 32 : 16;
}

// out = act(conv(in)) on a grid of d slices (a stack of d / df frames of df
// slices, zero padding per frame) with weights wt in [27][Nout][Kin]; wtc is
// scratch of 27 Nout Kin bf16 for the re-laid weights. Returns 1 when
// launched, 0 when the shape is not served (the caller runs its other
// kernel), -1 on an error.
int conv_tc_launch(const __nv_bfloat16 *in, int Kin, const __nv_bfloat16 *wt, __nv_bfloat16 *wtc, const float *bias,
                   __nv_bfloat16 *out, int Nout, int d, int h, int w, int df, int relu, cudaStream_t st)
{
    const int NT = conv_tc_split(Kin, Nout);
    if (!NT || (d != df && df % TZ) || d % df) return 0;
    Grid g;
    g.d = d;
    g.h = h;
    g.w = w;
    g.df = df;
    g.tiles_x = (w + TXX - 1) / TXX;
    g.tiles_y = (h + TYY - 1) / TYY;
    const long long tiles = (long long)g.tiles_x * g.tiles_y * ((d + TZ - 1) / TZ);
    if (tiles > (1LL << 30)) return 0;
    g.tiles = (int)tiles;
    g.nsplit = Nout / NT;
    g.nchunks = Kin / 16;
    tc_weights_kernel<<<(unsigned)std::min<long long>((27LL * Nout * Kin + 255) / 256, 4096), 256, 0, st>>>(wt, Kin,
                                                                                                           Nout, NT,
                                                                                                           wtc);
    switch (NT) {
    case 64: return launch<64>(in, Kin, wtc, bias, out, Nout, g, relu, st);
    case 32: return launch<32>(in, Kin, wtc, bias, out, Nout, g, relu, st);
    default: return launch<16>(in, Kin, wtc, bias, out, Nout, g, relu, st);
    }
}

// 0 when no tensor-core convolution has given up on a wait since the last
// call; otherwise the code of the first wait that ran out (1 stage free,
// 2 accumulator free, 3 stage full, 4 accumulator full), which is cleared.
int conv_tc_status(cudaStream_t st)
{
    int code = 0;
    if (cudaMemcpyFromSymbolAsync(&code, g_conv_tc_error, sizeof(int), 0, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return -1;
    if (code) {
        const int zero = 0;
        cudaMemcpyToSymbolAsync(g_conv_tc_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st);
        cudaStreamSynchronize(st);
    }
    return code;
}

}  // namespace mbirgpu
