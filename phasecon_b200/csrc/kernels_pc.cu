// Phase-contrast (PCMBIR) kernels: batched Fresnel transforms and the
// per-view phase-retrieval ADMM pieces, all views of a scan in each launch.
//
// Fresnel transform of one view (replaces compute_FresnelTran /
// compute_HermFresnelTran, PCMBIR_3D/XT_FresnelTran.c:12-137):
//   pass 1  rows:  prologue op forms the input, FFT along t (length N_t)
//   pass 2  cols:  FFT along r (length N_r), multiply by the transfer table,
//                  inverse FFT along r
//   pass 3  rows:  inverse FFT along t, scale by 1/(N_r N_t), epilogue op
// so every pass reads and writes the view once. FFTs are Stockham autosort
// stages of radix up to 16 (the R points of a butterfly in registers,
// ping-pong between two shared-memory buffers; for 256-point sequences the
// points stay in registers with one shared-memory exchange per transform)
// with twiddles exp(-2 pi i m / n_max) precomputed in double and rounded once
// to float.
// Per-view sums needed by the steepest-descent step size and the stopping
// tests are block-reduced and added in FP64. Views whose loop has stopped
// (per-view flags) skip every launch.
#include <cfloat>
#include "pc_internal.h"

namespace mbirgpu {

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }

// Shared-memory layout of the FFT buffers: element i of sequence q sits at
// q * sstride + i + i / 16 (one float2 of padding after every 16, and a
// sequence stride fft_seq_stride(n) = (n + n / 16) | 1, odd in float2
// units), so both the contiguous accesses of a stage and the strided ones of
// the column pass's transposed staging spread over the banks.
__device__ __forceinline__ int fpos(int q, int i, int sstride) { return q * sstride + i + (i >> 4); }

// exp(-+ 2 pi i m / nmax), 0 <= m < nmax, from the full-circle table the
// kernels keep in shared memory (load_twiddles).
__device__ __forceinline__ float2 twid(const float2 *tw, int m, int nmax, bool inverse)
{
    float2 w = tw[m];
    if (inverse) w.y = -w.y;
    return w;
}

__host__ __device__ constexpr int bit_reverse(int i, int bits)
{
    int r = 0;
    for (int b = 0; b < bits; b++)
        if (i & (1 << b)) r |= 1 << (bits - 1 - b);
    return r;
}

__host__ __device__ constexpr int log2_const(int n) { return n <= 1 ? 0 : 1 + log2_const(n >> 1); }

// R-point DFT of x in registers, natural order in and out (radix-2
// decimation in time over a bit-reversed copy; every index is a constant).
template <int R>
__device__ __forceinline__ void dft_regs(float2 (&x)[R], const float2 *tw, int nmax, bool inverse)
{
    constexpr int bits = log2_const(R);
    float2 y[R];
#pragma unroll
    for (int i = 0; i < R; i++) y[bit_reverse(i, bits)] = x[i];
#pragma unroll
    for (int len = 2; len <= R; len <<= 1) {
#pragma unroll
        for (int i = 0; i < R; i += len)
#pragma unroll
            for (int k = 0; k < len / 2; k++) {
                const float2 t = cmul(twid(tw, k * (nmax / len), nmax, inverse), y[i + k + len / 2]);
                y[i + k + len / 2] = csub(y[i + k], t);
                y[i + k] = cadd(y[i + k], t);
            }
    }
#pragma unroll
    for (int i = 0; i < R; i++) x[i] = y[i];
}

// One radix-R stage of a Stockham autosort FFT over nseq sequences of length
// n whose sub-transforms have length L so far: butterfly j of a sequence
// takes x_p = a[j + p n / R], p < R, multiplies x_p by w_{RL}^{p (j mod L)},
// transforms the R points in registers and writes them to b at
// (j - j mod L) R + j mod L + p L.
template <int R>
__device__ __forceinline__ void stockham_stage(const float2 *a, float2 *b, int n, int log2n, int L, int nseq,
                                               int sstride, const float2 *tw, int nmax, bool inverse)
{
    constexpr int lr = log2_const(R);
    const int lm = log2n - lr;  // butterflies per sequence: n / R = 2^lm
    const int m = 1 << lm;
    const int tscale = nmax / (R * L);
    for (int idx = threadIdx.x; idx < (nseq << lm); idx += blockDim.x) {
        const int q = idx >> lm, j = idx & (m - 1);
        const int k = j & (L - 1);
        float2 x[R];
#pragma unroll
        for (int p = 0; p < R; p++) x[p] = a[fpos(q, j + p * m, sstride)];
        if (L > 1) {
#pragma unroll
            for (int p = 1; p < R; p++) x[p] = cmul(twid(tw, k * p * tscale, nmax, inverse), x[p]);
        }
        dft_regs<R>(x, tw, nmax, inverse);
        const int o = ((j - k) << lr) + k;
#pragma unroll
        for (int p = 0; p < R; p++) b[fpos(q, o + p * L, sstride)] = x[p];
    }
}

// nseq sequences of length n (power of two) in the padded layout of `a`;
// stages of radix max_radix (16, 8, 4 or 2; smaller for the rest) ping-pong
// between a and b.
// Returns the buffer holding the result.
__device__ float2 *fft_smem(float2 *a, float2 *b, int n, int log2n, int nseq, int sstride, const float2 *tw,
                            int nmax, bool inverse, int max_radix)
{
    for (int L = 1; L < n;) {
        const int rem = n / L < max_radix ? n / L : max_radix;
        if (rem >= 16) {
            stockham_stage<16>(a, b, n, log2n, L, nseq, sstride, tw, nmax, inverse);
            L <<= 4;
        } else if (rem >= 8) {
            stockham_stage<8>(a, b, n, log2n, L, nseq, sstride, tw, nmax, inverse);
            L <<= 3;
        } else if (rem >= 4) {
            stockham_stage<4>(a, b, n, log2n, L, nseq, sstride, tw, nmax, inverse);
            L <<= 2;
        } else {
            stockham_stage<2>(a, b, n, log2n, L, nseq, sstride, tw, nmax, inverse);
            L <<= 1;
        }
        __syncthreads();
        float2 *tmp = a;
        a = b;
        b = tmp;
    }
    return a;
}

// The full circle exp(-2 pi i m / nmax), m < nmax, from the half-circle
// table tw (m < nmax / 2; the other half is -tw).
__device__ __forceinline__ void load_twiddles(float2 *s_tw, const float2 *tw, int nmax)
{
    const int h = nmax / 2;
    for (int i = threadIdx.x; i < h; i += blockDim.x) {
        const float2 w = tw[i];
        s_tw[i] = w;
        s_tw[i + h] = make_float2(-w.x, -w.y);
    }
}

// FP64 block sum of per-thread values, one atomicAdd per CTA.
__device__ void block_add(double v, double *dst, double *sh)
{
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += sh[i];
        atomicAdd(dst, s);
    }
    __syncthreads();
}

// e^{-z} for z = zr + i zi
__device__ __forceinline__ float2 expz(float zr, float zi)
{
    const float e = expf(-zr);
    float s, c;
    sincosf(-zi, &s, &c);
    return make_float2(e * c, e * s);
}

// the same with the hardware approximations, for the Nelder-Mead search whose
// stop rule (a 0.005 % relative vertex movement) is far above their error
__device__ __forceinline__ float2 expz_fast(float zr, float zi)
{
    const float e = __expf(-zr);
    float s, c;
    __sincosf(-zi, &s, &c);
    return make_float2(e * c, e * s);
}

}  // namespace

// Global <-> shared staging of the passes: each thread takes kStage elements
// a blockDim.x apart per round and issues all their global loads before any
// of its shared-memory stores, so that a round keeps kStage loads in flight
// per thread instead of one.
constexpr int kStage = 8;

namespace {
// prologue input of element i (pixel p of the view)
__device__ __forceinline__ float2 prologue_in(const PcArgs &A, int prologue, size_t i, size_t p)
{
    switch (prologue) {
    case PC_IN_DW: return cscale(__ldg(A.in + i), __ldg(A.D + p));
    case PC_IN_DEZ: return cscale(expz(__ldg(A.zr + i), __ldg(A.zi + i)), __ldg(A.D + p));
    case PC_IN_PAG: {
        const float m = __ldg(A.y + i), dp = __ldg(A.D + p);
        return make_float2(m * m / (dp * dp), 0.f);
    }
    default: return __ldg(A.in + i);
    }
}

// the operands an epilogue reads besides the transform's value t
struct EpiIn {
    float2 a, b;
    float s0, s1;
};

__device__ __forceinline__ EpiIn epilogue_in(const PcArgs &A, int epilogue, size_t i, size_t p)
{
    EpiIn r = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), 1.f, 0.f};
    switch (epilogue) {
    case PC_OUT_GRES:
        r.a = A.omega[i];
        r.s0 = A.lam ? __ldg(A.lam + i) : 1.0f;
        r.s1 = __ldg(A.y + i);
        break;
    case PC_OUT_GRAD:
        r.a = A.w[i];
        r.b = A.buf[i];
        r.s0 = __ldg(A.D + p);
        break;
    case PC_OUT_SFWD:
        r.a = A.omega[i];
        r.s0 = A.lam ? __ldg(A.lam + i) : 1.0f;
        break;
    case PC_OUT_SDEN:
        r.a = A.g[i];
        r.s0 = __ldg(A.D + p);
        break;
    case PC_OUT_OMEGA: r.s1 = __ldg(A.y + i); break;
    case PC_OUT_PCOST:
        r.s0 = A.lam ? __ldg(A.lam + i) : 1.0f;
        r.s1 = __ldg(A.y + i);
        break;
    default: break;
    }
    return r;
}

// writes element i's epilogue result; returns its term of the per-view sum
__device__ __forceinline__ double epilogue_out(const PcDims &d, const PcArgs &A, int epilogue, size_t i, float2 t,
                                               const EpiIn &in)
{
    switch (epilogue) {
    case PC_OUT_GRES: {  // conj(Omega) Lambda (Omega t - y)
        const float2 r = csub(cmul(in.a, t), make_float2(in.s1, 0.f));
        A.out[i] = cmul(cconj(in.a), cscale(r, in.s0));
        return 0.0;
    }
    case PC_OUT_GRAD: {  // g = D t + nu (w - buf); sum |g|^2
        const float2 g = cadd(cscale(t, in.s0), cscale(csub(in.a, in.b), d.nu));
        A.g[i] = g;
        return (double)cabs2(g);
    }
    case PC_OUT_SFWD:  // conj(Omega) Lambda Omega t
        A.out[i] = cmul(cconj(in.a), cscale(cmul(in.a, t), in.s0));
        return 0.0;
    case PC_OUT_SDEN: {  // sum Re(conj(g) D t)
        const float2 dt = cscale(t, in.s0);
        return (double)in.a.x * (double)dt.x + (double)in.a.y * (double)dt.y;
    }
    case PC_OUT_OMEGA: {  // Omega = (y / t) / |y / t|
        const float den = cabs2(t) + FLT_MIN;
        const float2 q = make_float2(in.s1 * t.x / den, -in.s1 * t.y / den);
        const float m = sqrtf(cabs2(q)) + FLT_MIN;
        A.omega[i] = make_float2(q.x / m, q.y / m);
        return 0.0;
    }
    case PC_OUT_PCOST: {  // sum Lambda (y - |t|)^2 / 2
        const double rr = (double)in.s1 - sqrt((double)cabs2(t));
        return rr * rr * in.s0 / 2.0;
    }
    case PC_OUT_PAG: {  // Paganin: thickness -log|Re t|
        const float th = -logf(fabsf(t.x));
        A.zr[i] = th / 2.0f;
        A.zi[i] = th * d.delta_over_beta / 2.0f;
        return 0.0;
    }
    default: A.out[i] = t; return 0.0;
    }
}

__device__ __forceinline__ int ilog2_pow2(int n) { return 31 - __clz(n); }
}  // namespace

// ---------------------------------------------------------------------------- pass 1
__global__ void pc_rows_forward(PcDims d, PcArgs A, int prologue)
{
    extern __shared__ float2 smem[];
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    const int C = d.C, lc = d.logC, rpc = d.rows_per_cta, S = fft_seq_stride(C);
    float2 *s_tw = smem, *a = smem + d.nmax, *b = a + rpc * S;
    load_twiddles(s_tw, A.tw, d.nmax);
    const int r0 = blockIdx.x * rpc;
    const int nrows = min(rpc, d.R - r0);
    const int total = nrows * C;
    const size_t vb = (size_t)v * d.N, pb = (size_t)r0 * C;
    for (int e0 = threadIdx.x; e0 < total; e0 += kStage * blockDim.x) {
        float2 x[kStage];
#pragma unroll
        for (int u = 0; u < kStage; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total) x[u] = prologue_in(A, prologue, vb + pb + e, pb + e);
        }
#pragma unroll
        for (int u = 0; u < kStage; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total) a[fpos(e >> lc, e & (C - 1), S)] = x[u];
        }
    }
    __syncthreads();
    float2 *res = fft_smem(a, b, C, lc, nrows, S, s_tw, d.nmax, false, d.fft_radix);
    for (int e = threadIdx.x; e < total; e += blockDim.x) A.work[vb + pb + e] = res[fpos(e >> lc, e & (C - 1), S)];
}

// ---------------------------------------------------------------------------- pass 2
__global__ void pc_cols_filter(PcDims d, PcArgs A, const float2 *__restrict__ transfer)
{
    extern __shared__ float2 smem[];
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    const int R = d.R, C = d.C, cb = d.cols_per_cta, lcb = ilog2_pow2(cb), S = fft_seq_stride(R);
    float2 *s_tw = smem, *a = smem + d.nmax, *b = a + cb * S;
    load_twiddles(s_tw, A.tw, d.nmax);
    const int c0 = blockIdx.x * cb;
    const int total = cb * R;
    const size_t vb = (size_t)v * d.N;
    for (int e0 = threadIdx.x; e0 < total; e0 += kStage * blockDim.x) {
        float2 x[kStage];
#pragma unroll
        for (int u = 0; u < kStage; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total) x[u] = A.work[vb + (size_t)(e >> lcb) * C + c0 + (e & (cb - 1))];
        }
#pragma unroll
        for (int u = 0; u < kStage; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total) a[fpos(e & (cb - 1), e >> lcb, S)] = x[u];
        }
    }
    __syncthreads();
    float2 *res = fft_smem(a, b, R, d.logR, cb, S, s_tw, d.nmax, false, d.fft_radix);
    float2 *other = res == a ? b : a;
    for (int e0 = threadIdx.x; e0 < total; e0 += kStage * blockDim.x) {
        float2 h[kStage];
#pragma unroll
        for (int u = 0; u < kStage; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total) h[u] = __ldg(transfer + (size_t)(e >> lcb) * C + c0 + (e & (cb - 1)));
        }
#pragma unroll
        for (int u = 0; u < kStage; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total) {
                const int i = fpos(e & (cb - 1), e >> lcb, S);
                res[i] = cmul(res[i], h[u]);
            }
        }
    }
    __syncthreads();
    res = fft_smem(res, other, R, d.logR, cb, S, s_tw, d.nmax, true, d.fft_radix);
    for (int e = threadIdx.x; e < total; e += blockDim.x)
        A.work[vb + (size_t)(e >> lcb) * C + c0 + (e & (cb - 1))] = res[fpos(e & (cb - 1), e >> lcb, S)];
}

// ---------------------------------------------------------------------------- pass 3
__global__ void pc_rows_inverse(PcDims d, PcArgs A, int epilogue)
{
    extern __shared__ float2 smem[];
    __shared__ double s_red[32];
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    const int C = d.C, lc = d.logC, rpc = d.rows_per_cta, S = fft_seq_stride(C);
    float2 *s_tw = smem, *a = smem + d.nmax, *b = a + rpc * S;
    load_twiddles(s_tw, A.tw, d.nmax);
    const int r0 = blockIdx.x * rpc;
    const int nrows = min(rpc, d.R - r0);
    const int total = nrows * C;
    const size_t vb = (size_t)v * d.N, pb = (size_t)r0 * C;
    for (int e0 = threadIdx.x; e0 < total; e0 += kStage * blockDim.x) {
        float2 x[kStage];
#pragma unroll
        for (int u = 0; u < kStage; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total) x[u] = A.work[vb + pb + e];
        }
#pragma unroll
        for (int u = 0; u < kStage; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total) a[fpos(e >> lc, e & (C - 1), S)] = x[u];
        }
    }
    __syncthreads();
    float2 *res = fft_smem(a, b, C, lc, nrows, S, s_tw, d.nmax, true, d.fft_radix);
    const float inv_n = 1.0f / (float)d.N;
    double acc = 0.0;
    constexpr int kEpi = kStage / 2;  // the epilogues read up to two complex operands per element
    for (int e0 = threadIdx.x; e0 < total; e0 += kEpi * blockDim.x) {
        EpiIn in[kEpi];
#pragma unroll
        for (int u = 0; u < kEpi; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total) in[u] = epilogue_in(A, epilogue, vb + pb + e, pb + e);
        }
#pragma unroll
        for (int u = 0; u < kEpi; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < total)
                acc += epilogue_out(d, A, epilogue, vb + pb + e, cscale(res[fpos(e >> lc, e & (C - 1), S)], inv_n),
                                    in[u]);
        }
    }
    if (epilogue == PC_OUT_GRAD || epilogue == PC_OUT_SDEN || epilogue == PC_OUT_PCOST)
        block_add(acc, A.acc + (size_t)v * kPcAccSlots + A.acc_slot, s_red);
}

// ---------------------------------------------------------------------------- 256-point passes
// Length-256 transforms (radix 16 x 16) with the data in registers: a thread
// owns butterfly j (0..15) of one sequence and loads its 16 points x[j + 16p]
// straight from global memory (the prologue applied on the way), transforms
// them (stage 1), writes them through shared memory once, reads the stage-2
// points x[j + 16p] back, twiddles and transforms them, and holds the outputs
// X[j + 16p] for the epilogue or the global store. The arithmetic is that of
// the generic passes' two radix-16 stages; one shared-memory exchange per
// transform instead of four, and one barrier instead of four. A CTA holds 16
// sequences (256 threads).
namespace {
constexpr int kF = 16;  // sequences per CTA and points per thread

// stage 2 of a 256-point transform on this thread's points x[p] = a[j + 16p]:
// twiddles w_256^(p j) (twiddle index scaled to the table's nmax), then the
// 16-point DFT; outputs X[j + 16p] in x[p]
__device__ __forceinline__ void stage2_256(float2 (&x)[kF], int j, const float2 *tw, int nmax, bool inverse)
{
    const int sc = nmax >> 8;
#pragma unroll
    for (int p = 1; p < kF; p++) x[p] = cmul(twid(tw, p * j * sc, nmax, inverse), x[p]);
    dft_regs<kF>(x, tw, nmax, inverse);
}
}  // namespace

__global__ void __launch_bounds__(256) pc_rows_forward_256(PcDims d, PcArgs A, int prologue)
{
    extern __shared__ float2 smem[];
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    const int S = fft_seq_stride(256);
    float2 *s_tw = smem, *a = smem + d.nmax;
    load_twiddles(s_tw, A.tw, d.nmax);
    const int q = threadIdx.x >> 4, j = threadIdx.x & 15;  // sequence (row) of the CTA, butterfly
    const int r = blockIdx.x * kF + q;
    const size_t pb = (size_t)r * 256, vb = (size_t)v * d.N;
    float2 x[kF];
#pragma unroll
    for (int p = 0; p < kF; p++) x[p] = prologue_in(A, prologue, vb + pb + j + 16 * p, pb + j + 16 * p);
    __syncthreads();  // the twiddle table
    dft_regs<kF>(x, s_tw, d.nmax, false);  // stage 1 (L = 1): outputs at 16 j + p
#pragma unroll
    for (int p = 0; p < kF; p++) a[fpos(q, 16 * j + p, S)] = x[p];
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kF; p++) x[p] = a[fpos(q, j + 16 * p, S)];
    stage2_256(x, j, s_tw, d.nmax, false);
#pragma unroll
    for (int p = 0; p < kF; p++) A.work[vb + pb + j + 16 * p] = x[p];
}

__global__ void __launch_bounds__(256, 2) pc_cols_filter_256(PcDims d, PcArgs A, const float2 *__restrict__ transfer)
{
    extern __shared__ float2 smem[];
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    const int C = d.C, S = fft_seq_stride(256);
    float2 *s_tw = smem, *a = smem + d.nmax;
    load_twiddles(s_tw, A.tw, d.nmax);
    const int q = threadIdx.x & 15, j = threadIdx.x >> 4;  // column of the CTA (fastest: coalesced), butterfly
    const int c = blockIdx.x * kF + q;
    const size_t vb = (size_t)v * d.N;
    float2 x[kF];
#pragma unroll
    for (int p = 0; p < kF; p++) x[p] = A.work[vb + (size_t)(j + 16 * p) * C + c];
    __syncthreads();  // the twiddle table
    dft_regs<kF>(x, s_tw, d.nmax, false);
#pragma unroll
    for (int p = 0; p < kF; p++) a[fpos(q, 16 * j + p, S)] = x[p];
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kF; p++) x[p] = a[fpos(q, j + 16 * p, S)];
    stage2_256(x, j, s_tw, d.nmax, false);
    // the forward outputs X[j + 16p] are the inverse's stage-1 inputs of the
    // same butterfly j: multiply by the transfer table and go on in registers
#pragma unroll
    for (int p = 0; p < kF; p++) x[p] = cmul(x[p], __ldg(transfer + (size_t)(j + 16 * p) * C + c));
    dft_regs<kF>(x, s_tw, d.nmax, true);
    __syncthreads();  // every thread has read its stage-2 points
#pragma unroll
    for (int p = 0; p < kF; p++) a[fpos(q, 16 * j + p, S)] = x[p];
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kF; p++) x[p] = a[fpos(q, j + 16 * p, S)];
    stage2_256(x, j, s_tw, d.nmax, true);
#pragma unroll
    for (int p = 0; p < kF; p++) A.work[vb + (size_t)(j + 16 * p) * C + c] = x[p];
}

__global__ void __launch_bounds__(256, 3) pc_rows_inverse_256(PcDims d, PcArgs A, int epilogue)
{
    extern __shared__ float2 smem[];
    __shared__ double s_red[32];
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    const int S = fft_seq_stride(256);
    float2 *s_tw = smem, *a = smem + d.nmax;
    load_twiddles(s_tw, A.tw, d.nmax);
    const int q = threadIdx.x >> 4, j = threadIdx.x & 15;
    const int r = blockIdx.x * kF + q;
    const size_t pb = (size_t)r * 256, vb = (size_t)v * d.N;
    float2 x[kF];
#pragma unroll
    for (int p = 0; p < kF; p++) x[p] = A.work[vb + pb + j + 16 * p];
    __syncthreads();
    dft_regs<kF>(x, s_tw, d.nmax, true);
#pragma unroll
    for (int p = 0; p < kF; p++) a[fpos(q, 16 * j + p, S)] = x[p];
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kF; p++) x[p] = a[fpos(q, j + 16 * p, S)];
    stage2_256(x, j, s_tw, d.nmax, true);
    const float inv_n = 1.0f / (float)d.N;
    double acc = 0.0;
    constexpr int kEpi = 4;  // operands of four elements in flight
#pragma unroll
    for (int p0 = 0; p0 < kF; p0 += kEpi) {
        EpiIn in[kEpi];
#pragma unroll
        for (int u = 0; u < kEpi; u++) {
            const size_t e = pb + j + 16 * (p0 + u);
            in[u] = epilogue_in(A, epilogue, vb + e, e);
        }
#pragma unroll
        for (int u = 0; u < kEpi; u++) {
            const size_t e = pb + j + 16 * (p0 + u);
            acc += epilogue_out(d, A, epilogue, vb + e, cscale(x[p0 + u], inv_n), in[u]);
        }
    }
    if (epilogue == PC_OUT_GRAD || epilogue == PC_OUT_SDEN || epilogue == PC_OUT_PCOST)
        block_add(acc, A.acc + (size_t)v * kPcAccSlots + A.acc_slot, s_red);
}

// ---------------------------------------------------------------------------- pointwise steps
// w -= alpha g with alpha = sum|g|^2 / (sum Re(conj g D^H H'^H ..) + nu sum|g|^2 + eps)
// (compute_stepsize, PCMBIR_3D/XT_PhaseRet.c:126-165); sums |alpha g| and |w|.
__global__ void pc_sd_update(PcDims d, PcArgs A)
{
    __shared__ double s_red[32];
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    double *acc = A.acc + (size_t)v * kPcAccSlots;
    const double num = acc[PC_ACC_GG], den = acc[PC_ACC_DEN] + d.nu * num;
    const double alpha = num / (den + DBL_MIN);
    const float af = (float)alpha;
    double up = 0, val = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < d.N; e += gridDim.x * blockDim.x) {
        const size_t i = (size_t)v * d.N + e;
        const float2 g = A.g[i];
        const float2 w = csub(A.w[i], cscale(g, af));
        A.w[i] = w;
        up += fabs(alpha) * sqrt((double)cabs2(g));
        val += sqrt((double)cabs2(w));
    }
    block_add(up, acc + PC_ACC_UP, s_red);
    block_add(val, acc + PC_ACC_VAL, s_red);
}

// per view: threshold 100 sum|alpha g| / sum|w|; stop after step j > 1 when below
// the steepest-descent threshold (XT_CmplxProjEst.c:179-183)
__global__ void pc_sd_finish(PcDims d, PcArgs A, int step, float sd_thresh)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= d.V) return;
    if (A.active && !A.active[v]) return;
    double *acc = A.acc + (size_t)v * kPcAccSlots;
    const double th = 100.0 * acc[PC_ACC_UP] / acc[PC_ACC_VAL];
    A.sd_thresh_out[v] = (float)th;
    A.sd_steps[v] = step + 1;
    if (th < sd_thresh && step > 1) A.active[v] = 0;
    for (int s = 0; s < PC_ACC_PRIMAL; s++) acc[s] = 0.0;
}

// wold = w; buf = e^{-z} + v (XT_CmplxProjEst.c:170-177)
__global__ void pc_pret_prepare(PcDims d, PcArgs A)
{
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < d.N; e += gridDim.x * blockDim.x) {
        const size_t i = (size_t)v * d.N + e;
        A.wold[i] = A.w[i];
        A.buf[i] = cadd(expz(A.zr[i], A.zi[i]), A.vdual[i]);
    }
}

// v += e^{-z} - w; sums for the primal / dual residuals (XT_CmplxProjEst.c:186-199)
__global__ void pc_pret_dual(PcDims d, PcArgs A)
{
    __shared__ double s_red[32];
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    double pr = 0, du = 0, sm = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < d.N; e += gridDim.x * blockDim.x) {
        const size_t i = (size_t)v * d.N + e;
        const float2 w = A.w[i];
        const float2 dd = csub(expz(A.zr[i], A.zi[i]), w);
        const float2 nv = cadd(A.vdual[i], dd);
        A.vdual[i] = nv;
        const float2 dw = csub(w, A.wold[i]);
        pr += (double)cabs2(dd);
        du += (double)cabs2(dw);
        sm += (double)cabs2(nv);
    }
    double *acc = A.acc + (size_t)v * kPcAccSlots;
    block_add(pr, acc + PC_ACC_PRIMAL, s_red);
    block_add(du, acc + PC_ACC_DUALW, s_red);
    block_add(sm, acc + PC_ACC_VSUM, s_red);
}

// the decorrelated qGGMRF prior over the causal pixel pairs (+col, +row,
// +row+col, +row-col) of compute_pretcost (XT_CmplxProjEst.c:43-83), FP64
__global__ void pc_prior_cost(PcDims d, PcArgs A, const __grid_constant__ PcPrior P)
{
    __shared__ double s_red[32];
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    double acc = 0;
    const int R = d.R, C = d.C;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < d.N; e += gridDim.x * blockDim.x) {
        const int j = e / C, k = e % C;
        const size_t i = (size_t)v * d.N + e;
        const double zr = A.zr[i], zi = A.zi[i];
        const int dj[4] = {0, 1, 1, 1}, dk[4] = {1, 0, 1, -1};
        for (int m = 0; m < 4; m++) {
            const int jj = j + dj[m], kk = k + dk[m];
            if (jj >= R || kk < 0 || kk >= C) continue;
            const size_t n = (size_t)v * d.N + (size_t)jj * C + kk;
            const double db = zr - (double)A.zr[n], dd = zi - (double)A.zi[n];
            const double dph = P.T00 * dd + P.T01 * db, dmg = P.T10 * dd + P.T11 * db;
            const double fw = P.f[(dj[m] + 1) * 3 + (dk[m] + 1)];
            const double aph = fabs(dph), amg = fabs(dmg);
            if (aph > 0)
                acc += fw * (aph * aph / P.ph_sq) / (P.ph_c + exp(P.qmp * log(aph)) / P.ph_sqp);
            if (amg > 0)
                acc += fw * (amg * amg / P.mg_sq) / (P.mg_c + exp(P.qmp * log(amg)) / P.mg_sqp);
        }
    }
    block_add(acc, A.acc + (size_t)v * kPcAccSlots + PC_ACC_PRIOR, s_red);
}

// per view: dual residual sqrt(sum|w - wold|^2 / sum|v|^2); stop when below the
// phase-retrieval threshold after iteration 1 (XT_CmplxProjEst.c:198-214)
__global__ void pc_pret_finish(PcDims d, PcArgs A, int iter, float pret_thresh, double *costs_out)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= d.V) return;
    if (A.active && !A.active[v]) return;
    double *acc = A.acc + (size_t)v * kPcAccSlots;
    const double dual = sqrt(acc[PC_ACC_DUALW] / acc[PC_ACC_VSUM]);
    const double primal = sqrt(acc[PC_ACC_PRIMAL] / (double)d.N);
    A.dual_res[v] = dual;
    A.primal_res[v] = primal;
    if (costs_out) costs_out[v] = acc[PC_ACC_PCOST] + acc[PC_ACC_PRIOR];
    A.pret_iters[v] = iter + 1;
    if (dual < pret_thresh && iter > 1) A.active[v] = 0;
    for (int s = 0; s < kPcAccSlots; s++) acc[s] = 0.0;
}

// ---------------------------------------------------------------------------- Nelder-Mead proximal
// Per-pixel 2-D Nelder-Mead on z = (zr, zi) minimising nu/2 |e^{-z} - b|^2 +
// decorrelated qGGMRF over the 3x3 neighbourhood (Cost_NMS and
// Nelder_Mead_Simplex_2DSearch, PCMBIR_3D/XT_Search.c:8-215), b = w - v. The
// reference sweeps pixels in raster order (XT_CmplxProjEst.c:117-160);
// pc_nms_wavefront keeps that order exactly, pc_nms updates colour classes.
//
// One pixel's search runs on a group of G adjacent lanes (G = 1, 2, 4 or 8).
// The eight neighbour slots s = 0..7 (3x3 position s < 4 ? s : s + 1) are dealt
// round-robin over the group's lanes; lane 0 adds the data term; a butterfly of
// xor shuffles sums the partial costs, which leaves the same sum (the same
// pairwise additions) in every lane, so the group takes every branch together.
namespace {
template <int G>
struct NmsLane {
    static constexpr int kN = 8 / G;  // neighbour slots per lane
    float br, bi, half_nu;
    float nr[kN], ni[kN], fw[kN];
    unsigned flags;  // bit m: slot g + G m lies inside the image
    unsigned mask;   // the group's lanes within the warp
    bool data;       // this lane adds the data term
};

// a^e for a > 0 with the hardware base-2 logarithm and exponential (the
// search's stop rule, a 0.005 % relative vertex movement, is far above their
// error)
__device__ __forceinline__ float pow_fast(float a, float e)
{
    float l, r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(a));
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e * l));
    return r;
}

template <int G>
__device__ __forceinline__ float nms_cost(const NmsLane<G> &c, const PcPrior &P, float zr, float zi)
{
    float cost = 0.f;
    if (c.data) {
        const float2 ez = expz_fast(zr, zi);
        cost = ((ez.x - c.br) * (ez.x - c.br) + (ez.y - c.bi) * (ez.y - c.bi)) * c.half_nu;
    }
#pragma unroll
    for (int m = 0; m < NmsLane<G>::kN; m++) {
        if (c.flags & (1u << m)) {
            const float db = zr - c.nr[m], dd = zi - c.ni[m];
            const float dph = P.T00_f * dd + P.T01_f * db, dmg = P.T10_f * dd + P.T11_f * db;
            const float aph = fabsf(dph), amg = fabsf(dmg);
            // rho(x) = x^2 / sig^2 / (c + |x|^(q-p) / sig^(q-p)) for both channels,
            // the two quotients over one reciprocal: x1/y1 + x2/y2 = (x1 y2 + x2 y1) / (y1 y2)
            const float pph = aph > 0.f ? pow_fast(aph, P.qmp_f) : 0.f;
            const float pmg = amg > 0.f ? pow_fast(amg, P.qmp_f) : 0.f;
            const float x1 = aph * aph * P.ph_isq_f, y1 = P.ph_c_f + pph * P.ph_isqp_f;
            const float x2 = amg * amg * P.mg_isq_f, y2 = P.mg_c_f + pmg * P.mg_isqp_f;
            cost += c.fw[m] * __fdividef(x1 * y2 + x2 * y1, y1 * y2);
        }
    }
#pragma unroll
    for (int o = 1; o < G; o <<= 1) cost += __shfl_xor_sync(c.mask, cost, o);
    return cost;
}

// The search of Nelder_Mead_Simplex_2DSearch for pixel (j, k) of view v,
// written back to z by the group's lane 0. Neighbours are read from z as it
// stands (Gauss-Seidel). Each iteration evaluates the reflected point, then
// at most one second point (expansion, outside or inside contraction; which
// one follows the reference's case analysis), then the shrink's two points:
// the cost is called from one place per kind, so lanes of a warp that take
// different cases share the calls instead of running them one case at a time.
template <int G>
__device__ void nms_pixel(const PcDims &d, const PcArgs &A, const PcPrior &P, int v, int j, int k, int max_iter,
                          float threshold, int g, unsigned mask)
{
    const int R = d.R, C = d.C;
    const size_t i = (size_t)v * d.N + (size_t)j * C + k;
    NmsLane<G> c;
    const float2 b = csub(A.w[i], A.vdual[i]);
    c.br = b.x;
    c.bi = b.y;
    c.half_nu = d.nu / 2;
    c.mask = mask;
    c.data = g == 0;
    c.flags = 0;
#pragma unroll
    for (int m = 0; m < NmsLane<G>::kN; m++) {
        const int s = g + G * m, a = s < 4 ? s : s + 1;
        const int jj = j + a / 3 - 1, kk = k + a % 3 - 1;
        c.nr[m] = c.ni[m] = 0.f;
        c.fw[m] = P.f_f[a];
        if (jj >= 0 && jj < R && kk >= 0 && kk < C) {
            const size_t n = (size_t)v * d.N + (size_t)jj * C + kk;
            c.nr[m] = __ldcg(A.zr + n);
            c.ni[m] = __ldcg(A.zi + n);
            c.flags |= 1u << m;
        }
    }
    const float z0r = __ldcg(A.zr + i), z0i = __ldcg(A.zi + i);
    float pr[3] = {z0r, 2 * z0r, z0r}, pi[3] = {z0i, z0i, 2 * z0i};
    float cc[3];
#pragma unroll
    for (int q = 0; q < 3; q++) cc[q] = nms_cost<G>(c, P, pr[q], pi[q]);
    auto swap_pts = [&](int a2, int b2) {
        float t = pr[a2]; pr[a2] = pr[b2]; pr[b2] = t;
        t = pi[a2]; pi[a2] = pi[b2]; pi[b2] = t;
        t = cc[a2]; cc[a2] = cc[b2]; cc[b2] = t;
    };
    auto sort3 = [&]() {
        if (cc[2] < cc[1]) swap_pts(1, 2);
        if (cc[1] < cc[0]) swap_pts(0, 1);
        if (cc[2] < cc[1]) swap_pts(1, 2);
    };
    sort3();
    float cr0 = (pr[0] + pr[1]) / 2.0f, ci0 = (pi[0] + pi[1]) / 2.0f;
    for (int it = 0; it < max_iter; it++) {
        const float o_r[4] = {cr0, pr[0], pr[1], pr[2]}, o_i[4] = {ci0, pi[0], pi[1], pi[2]};
        const float rr = cr0 + (cr0 - pr[2]), ri = ci0 + (ci0 - pi[2]);
        const float crf = nms_cost<G>(c, P, rr, ri);
        // 0: accept the reflection; 1: expansion; 2: outside contraction;
        // 3: inside contraction; -1: no case holds (a NaN cost), nothing moves
        const int kind = (crf < cc[1] && crf >= cc[0]) ? 0
                         : crf < cc[0]                 ? 1
                         : (crf >= cc[1] && crf < cc[2]) ? 2
                         : crf >= cc[2]                ? 3
                                                       : -1;
        float sr = rr, si = ri;
        if (kind == 1) { sr = cr0 + 2.0f * (rr - cr0); si = ci0 + 2.0f * (ri - ci0); }
        if (kind == 2) { sr = cr0 + 0.5f * (rr - cr0); si = ci0 + 0.5f * (ri - ci0); }
        if (kind == 3) { sr = cr0 - 0.5f * (cr0 - pr[2]); si = ci0 - 0.5f * (ci0 - pi[2]); }
        float cs = crf;
        if (kind > 0) cs = nms_cost<G>(c, P, sr, si);
        bool take_s = kind == 1 ? cs < crf : kind == 2 ? cs <= crf : kind == 3 ? cs < cc[2] : false;
        const bool take_r = kind == 0 || (kind == 1 && !take_s);
        const bool shrink = (kind == 2 || kind == 3) && !take_s;
        if (take_r || take_s) {
            pr[2] = take_s ? sr : rr;
            pi[2] = take_s ? si : ri;
            cc[2] = take_s ? cs : crf;
            if (cc[2] < cc[1]) swap_pts(1, 2);
            if (cc[1] < cc[0]) swap_pts(0, 1);
        }
        if (shrink) {
#pragma unroll
            for (int q = 1; q < 3; q++) {
                pr[q] = pr[0] + 0.5f * (pr[q] - pr[0]);
                pi[q] = pi[0] + 0.5f * (pi[q] - pi[0]);
                cc[q] = nms_cost<G>(c, P, pr[q], pi[q]);
            }
            sort3();
        }
        cr0 = (pr[0] + pr[1]) / 2.0f;
        ci0 = (pi[0] + pi[1]) / 2.0f;
        const float n_r[4] = {cr0, pr[0], pr[1], pr[2]}, n_i[4] = {ci0, pi[0], pi[1], pi[2]};
        float num = 0.f, den = 0.f;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            num += fabsf(o_r[q] - n_r[q]) + fabsf(o_i[q] - n_i[q]);
            den += fabsf(o_r[q]) + fabsf(o_i[q]);
        }
        if (num / den * 100.0f < threshold && it > 1) break;
    }
    if (g == 0) {
        A.zr[i] = pr[0];
        A.zi[i] = pi[0];
    }
}

// lanes of the G-lane group that thread t belongs to
template <int G>
__device__ __forceinline__ unsigned group_mask(int t)
{
    return G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((t & 31) & ~(G - 1)));
}

__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// every thread of the cluster, with release/acquire at cluster scope so that
// the z written before it is seen by the cluster's CTAs after it
__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
}  // namespace

// Colour-class sweep: pixels of one (row parity, column parity) class
// together -- no two 8-neighbours share a class -- over four launches.
template <int G>
__global__ void pc_nms(PcDims d, PcArgs A, const __grid_constant__ PcPrior P, int color, int max_iter,
                       float threshold)
{
    const int v = blockIdx.y;
    if (A.active && !A.active[v]) return;
    const int cj = color >> 1, ck = color & 1;
    const int hr = (d.R - cj + 1) / 2, hc = (d.C - ck + 1) / 2;
    const int g = threadIdx.x % G, groups = gridDim.x * blockDim.x / G;
    const unsigned mask = group_mask<G>(threadIdx.x);
    for (int e = (blockIdx.x * blockDim.x + threadIdx.x) / G; e < hr * hc; e += groups)
        nms_pixel<G>(d, A, P, v, 2 * (e / hc) + cj, 2 * (e % hc) + ck, max_iter, threshold, g, mask);
}

// The reference's raster order, exactly: pixel (j, k) reads the updated
// (j-1, k-1..k+1) and (j, k-1) and the not yet updated (j, k+1) and row j+1,
// so every pixel of the anti-diagonal 2j + k = t depends only on pixels of
// smaller t and none of larger t reads it first. The CTAs of one cluster share
// a view (the cluster size is the number of CTAs per view) and walk its
// 2(R-1) + C wavefronts, the pixels of each dealt over all their lane groups,
// with a barrier between wavefronts: the block barrier for one CTA per view,
// the cluster barrier (release/acquire at cluster scope) for more.
template <int G>
__global__ void pc_nms_wavefront(PcDims d, PcArgs A, const __grid_constant__ PcPrior P, int max_iter,
                                 float threshold, int ctas_per_view)
{
    const int v = blockIdx.x / ctas_per_view;
    const int part = ctas_per_view > 1 ? (int)cluster_rank() : 0;
    // a view's CTAs all return here or none does
    if (A.active && !A.active[v]) return;
    const int R = d.R, C = d.C;
    const int T = 2 * (R - 1) + C;
    const int g = threadIdx.x % G, groups = blockDim.x / G;
    // groups interleaved over the cluster's CTAs, so that short anti-diagonals
    // still spread over all of them
    const int grp = ((int)threadIdx.x / G) * ctas_per_view + part, all_groups = groups * ctas_per_view;
    const unsigned mask = group_mask<G>(threadIdx.x);
    for (int t = 0; t < T; t++) {
        const int j_lo = t >= C ? (t - C + 2) / 2 : 0;  // smallest j with t - 2j <= C - 1
        const int j_hi = min(R - 1, t / 2);
        for (int j = j_lo + grp; j <= j_hi; j += all_groups)
            nms_pixel<G>(d, A, P, v, j, t - 2 * j, max_iter, threshold, g, mask);
        if (ctas_per_view > 1) cluster_sync_all();
        else __syncthreads();
    }
}

namespace {
template <int G>
int nms_sweep(const PcDims &d, const PcArgs &A, const PcPrior &P, int order, int ctas, int max_iter, float thr,
              dim3 pointwise, cudaStream_t st)
{
    if (order == 0) {
        // 128 lane groups per view: the most pixels an anti-diagonal of a
        // 256-wide view holds, dealt over the view's CTAs
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(d.V * ctas);
        cfg.blockDim = dim3(max(32, 128 * G / ctas));
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, pc_nms_wavefront<G>, d, A, P, max_iter, thr, ctas);
        return 1;
    }
    for (int color = 0; color < 4; color++) pc_nms<G><<<pointwise, 256, 0, st>>>(d, A, P, color, max_iter, thr);
    return 4;
}
}  // namespace

int launch_nms_sweep(const PcDims &d, const PcArgs &A, const PcPrior &P, int order, int lanes, int ctas,
                     int max_iter, float threshold, dim3 pointwise, cudaStream_t st)
{
    switch (lanes) {
    case 1: return nms_sweep<1>(d, A, P, order, ctas, max_iter, threshold, pointwise, st);
    case 2: return nms_sweep<2>(d, A, P, order, ctas, max_iter, threshold, pointwise, st);
    case 4: return nms_sweep<4>(d, A, P, order, ctas, max_iter, threshold, pointwise, st);
    default: return nms_sweep<8>(d, A, P, order, ctas, max_iter, threshold, pointwise, st);
    }
}

}  // namespace mbirgpu
