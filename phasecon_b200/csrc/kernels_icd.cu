// Super-voxel parallel ICD sweep (one colour phase per launch).
//
// Replaces the voxel loop of updateVoxelsTimeSlices / updateVoxels_Atten /
// compute_voxel_update_Atten (MBIR_4D/XT_ICD_update.c:932-1092,
// XT_VoxUpdate.c:45-283) and the surrogate solve CE_FunctionalSubstitution
// (XT_ICD_update.c:133-182).
//
// Schedule. The image plane is tiled into super-voxels (SVs) of sv x sv voxel
// columns; with K x K colours (K = 2 or 4) an SV's colour is
// (sv_y mod K) K + (sv_x mod K). Phase p updates, in frame f, the SVs of
// colour (p + f) mod K^2: no two SVs updated at once share a prior neighbour,
// and a voxel and its temporal neighbours (same column, frames f +- 1) are
// never updated at once -- the GPU counterpart of the reference's z-block /
// frame checkerboard (XT_ICD_update.c:964-1046). Frames use disjoint views,
// so different frames never share sinogram entries; concurrent SVs of one
// frame can share entries along a ray, and their error sinogram updates are
// atomic adds (how many may run at once is bounded by sv_max_concurrent).
//
// A grid of persistent CTAs (as many as fit on the GPU) drains a queue of the
// phase's SVs, frames fastest and SV slots in a spread order (queue index x
// perm mod slots), so the SVs in flight are far apart; a CTA owns one SV at a
// time and visits its voxel columns one
// after another in a seeded random order (the counterpart of
// randomly_select_x_y, XT_ICD_update.c:499-531). For one column all warps
// cooperate, with three CTA barriers per column:
//   1. neighbourhood: the 8 in-plane neighbour columns and the 2 temporal
//      neighbours are split over the warps; each lane owns one slice z and
//      accumulates the qGGMRF surrogate terms b = w rho'(d)/d of those
//      neighbours (XT_ICD_update.c:140-172); a block-wide OR decides whether
//      any slice escapes zero skipping (XT_VoxUpdate.c:238-261);
//   2. theta: the column's views are split over warps; a lane owns one
//      detector row t and accumulates theta1 = -sum a w e and theta2 =
//      sum a^2 w over the column's A entries (a = A value x delta_t,
//      XT_VoxUpdate.c:56-85) -- reads of e[view][r][0..N_t) are coalesced,
//      and four views' records and entries are in flight at once;
//   3. solve: warp 0 sums the partials, then updates even slices and odd
//      slices in turn (their only mutual coupling is the in-column z +- 1
//      prior pair), x <- V + alpha (u - V);
//   4. apply: e[view][r][t] -= a dx(slice of t) with atomic adds.
// All arithmetic is FP32; the host refreshes e in FP64 periodically.
#include <mutex>
#include <vector>

#include "mbir_internal.h"

namespace mbirgpu {

namespace {

constexpr int kMaxWarps = 8;
constexpr int kMaxSvCols = 256;  // sv <= 16

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Surrogate weight rho'(d)/d of the qGGMRF potential
// |d|^(q-p) ... (derivative per XT_ICD_update.c:92-118; value at d = 0 per
// :119-128): |d|^(q-2) (q - (q-p) t1 / t3) / (t3 sq), t1 = |d|^(q-p) / sqp,
// t3 = c + t1. Takes isq = 1 / sq and isqp = 1 / sqp. The weight is
// evaluated ~28 times per voxel update, so it uses the hardware base-2
// logarithm / exponential (one logarithm for both powers) and reciprocal:
// FP32 arithmetic whose rounding the FP64 MAP cost, by which the method's
// result is measured, does not see.
__device__ __forceinline__ float lg2_hw(float x)
{
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ex2_hw(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rcp_hw(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float qg_weight(float d, float q, float qmp, float isq, float isqp, float c, float b0)
{
    if (d == 0.0f) return b0;
    const float l = lg2_hw(fabsf(d));
    const float t1 = ex2_hw(qmp * l) * isqp;
    const float rt3 = rcp_hw(c + t1);
    float r = (q - qmp * t1 * rt3) * rt3 * isq;
    if (q != 2.0f) r *= ex2_hw((q - 2.0f) * l);
    return r;
}

template <int KW>
struct Rec {
    uint4 w[KW];
};

template <int KW>
__device__ __forceinline__ Rec<KW> load_rec(const uint32_t *p)
{
    Rec<KW> r;
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
#pragma unroll
    for (int i = 0; i < KW; i++) r.w[i] = __ldg(q + i);
    return r;
}

template <int KW>
__device__ __forceinline__ Rec<KW> load_rec_smem(const uint32_t *p)
{
    Rec<KW> r;
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
#pragma unroll
    for (int i = 0; i < KW; i++) r.w[i] = q[i];
    return r;
}

// Copy a column's A records (nwords 32-bit words, a multiple of 4, 16-byte
// aligned on both sides) into shared memory with one TMA bulk copy, issued by
// thread 0, that completes on the buffer's mbarrier; the copy lands while the
// CTA works on the current column.
__device__ __forceinline__ void stage_records(uint32_t *dst, const uint32_t *src, int nwords,
                                              unsigned long long *bar)
{
    if (threadIdx.x != 0) return;
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar), d = (unsigned)__cvta_generic_to_shared(dst);
    const unsigned bytes = 4u * (unsigned)nwords;
    if (bytes == 0) {  // a frame without views: complete the phase with no transfer
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(b) : "memory");
        return;
    }
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
                 "l"(src), "r"(bytes), "r"(b)
                 : "memory");
}

// Bounded wait (about 2 s of clock64) for phase `parity` of mbarrier `bar`;
// returns false if it ran out.
__device__ __forceinline__ bool wait_parity_bounded(unsigned long long *bar, uint32_t parity)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, P;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > 4000000000LL) return false;
    }
}

// Every thread waits for buffer b's copy: the n-th copy into a buffer
// completes the mbarrier's phase n, so the parity of the wait is the count of
// earlier waits on that buffer (bit b of `phases`, identical in every thread).
// The wait is bounded; a copy that never lands is counted (the host turns the
// count into an error) and raises the CTA's abort flag: the caller stops
// updating and staging after the next barrier, and the kernel waits for the
// late copy once more before it exits (abort_bar / abort_parity).
// Returns whether this thread's wait saw the copy land.
__device__ __forceinline__ bool wait_staged(unsigned long long *bar, uint32_t &phases, int b, unsigned &timeouts,
                                            int &abort, int &abort_bar, uint32_t &abort_parity)
{
    const uint32_t parity = (phases >> b) & 1u;
    const bool ok = wait_parity_bounded(bar, parity);
    if (!ok) {
        timeouts++;
        abort = 1;  // every writer stores the same values
        abort_bar = b;
        abort_parity = parity;
    }
    phases ^= 1u << b;
    return ok;
}

template <int KW>
__device__ __forceinline__ float rec_val(const Rec<KW> &r, int q)
{
    // word 1 + q of the record
    const int wi = 1 + q;
    const uint4 &u = r.w[wi >> 2];
    const uint32_t bits = (wi & 3) == 0 ? u.x : (wi & 3) == 1 ? u.y : (wi & 3) == 2 ? u.z : u.w;
    return __uint_as_float(bits);
}

template <int VEC>
struct VecF;
template <>
struct VecF<4> {
    using T = float4;
    __device__ static void get(const T &v, float *o) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
};
template <>
struct VecF<2> {
    using T = float2;
    __device__ static void get(const T &v, float *o) { o[0] = v.x; o[1] = v.y; }
};

// Vector reduction into global memory (red.global.add.v{2,4}.f32, sm_90+).
__device__ __forceinline__ void red_add(float *p, const float (&d)[4])
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(d[0]), "f"(d[1]), "f"(d[2]), "f"(d[3])
                 : "memory");
}
__device__ __forceinline__ void red_add(float *p, const float (&d)[2])
{
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(d[0]), "f"(d[1]) : "memory");
}


struct IcdSmem {
    unsigned long long stage_bar[2];  // completion of the two record buffers' bulk copies
    float num[kMaxWarps][32], den[kMaxWarps][32];
    float th1[kMaxWarps][32], th2[kMaxWarps][32];
    int pos[kMaxWarps][32];
    float dx[32];
    int order[kMaxSvCols];
    int ncols, item;
    int abort;              // a record copy did not land in time: stop updating
    int abort_bar;          // the buffer whose copy was late, and the wait's parity
    uint32_t abort_parity;
};

struct IcdCount {
    unsigned long long upd, skip;
    float sum_dx, sum_x;
    unsigned timeouts;     // record copies that did not land in time
    uint32_t phases;       // parity of the next wait on each record buffer
};

// Warp 0 adds the CTA's counters to the problem's statistics and clears them.
__device__ __forceinline__ void flush_counts(IcdCount &cnt, IcdStats *stats)
{
    if ((threadIdx.x >> 5) == 0) {
        for (int off = 16; off > 0; off >>= 1) {
            cnt.upd += __shfl_xor_sync(0xffffffffu, cnt.upd, off);
            cnt.skip += __shfl_xor_sync(0xffffffffu, cnt.skip, off);
            cnt.sum_dx += __shfl_xor_sync(0xffffffffu, cnt.sum_dx, off);
            cnt.sum_x += __shfl_xor_sync(0xffffffffu, cnt.sum_x, off);
        }
        if ((threadIdx.x & 31) == 0 && (cnt.upd || cnt.skip)) {
            atomicAdd(&stats->updates, cnt.upd);
            atomicAdd(&stats->skipped, cnt.skip);
            atomicAdd(&stats->sum_abs_dx, (double)cnt.sum_dx);
            atomicAdd(&stats->sum_abs_x, (double)cnt.sum_x);
        }
    }
    if (cnt.timeouts && (threadIdx.x & 31) == 0) atomicAdd(&stats->stage_timeouts, cnt.timeouts);
    const uint32_t phases = cnt.phases;
    cnt = IcdCount{};
    cnt.phases = phases;
}

// theta1 / theta2 partial sums of one lane (VEC detector rows starting at
// sinogram row offset `row0` within each A entry's row, views gfirst,
// gfirst + gstride, ... of the column): theta1 = -sum a w e,
// theta2 = sum a^2 w with a = A value x delta_t (XT_VoxUpdate.c:56-85).
template <int KW, int kUnroll, int VEC, bool kStaged, int kHuber>
__device__ __forceinline__ void theta_pass(const IcdConst &K, const uint32_t *col_rec, const float *__restrict__ err,
                                           const float *__restrict__ wgt, int gfirst, int gstride, int nv, int RW,
                                           int NT, int row0, float (&th1)[VEC], float (&th2)[VEC])
{
    using VT = typename VecF<VEC>::T;
    for (int v0 = gfirst; v0 < nv; v0 += kUnroll * gstride) {
        Rec<KW> R[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const int v = v0 + u * gstride;
            if (v < nv) R[u] = kStaged ? load_rec_smem<KW>(col_rec + (size_t)v * RW) : load_rec<KW>(col_rec + (size_t)v * RW);
            else R[u].w[0].x = 0u;
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const uint32_t hdr = R[u].w[0].x;
            const int cnt_q = hdr >> 24;
            // sinogram rows stay below 2^24 and N_t rows each: 32-bit offsets
            const unsigned sb = (hdr & 0xFFFFFFu) * (unsigned)NT + (unsigned)row0;
#pragma unroll
            for (int q = 0; q < 4 * KW - 1; q++) {
                if (q < cnt_q) {
                    float ev[VEC], wv[VEC];
                    VecF<VEC>::get(__ldcg(reinterpret_cast<const VT *>(err + (sb + (unsigned)(q * NT)))), ev);
                    VecF<VEC>::get(__ldg(reinterpret_cast<const VT *>(wgt + (sb + (unsigned)(q * NT)))), wv);
                    const float a = rec_val<KW>(R[u], q) * K.dt;
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        float ww = wv[i];
                        if (kHuber == 1 || (kHuber == 2 && K.huber)) {
                            const float sw = sqrtf(ww);
                            if (!(fabsf(ev[i] * sw) < K.huber_T)) ww = K.huber_T * K.huber_delta * sw / fabsf(ev[i]);
                        }
                        const float aw = a * ww;
                        th2[i] += a * aw;
                        th1[i] -= ev[i] * aw;
                    }
                }
            }
        }
    }
}

// One column's theta: every lane's partial sums (theta_pass, when `run`),
// folded over the view groups of the warp and stored by group 0 into the
// warp's row of S.th1 / S.th2.
template <int KW, int kUnroll, int VEC, bool kStaged, int kHuber>
__device__ __forceinline__ void theta_column(const IcdConst &K, const uint32_t *col_rec, const float *__restrict__ err,
                                             const float *__restrict__ wgt, int gfirst, int gstride, int nv, int RW,
                                             int NT, int row0, bool run, int lprp, int grp, int t0, int warp,
                                             IcdSmem &S)
{
    float th1[VEC], th2[VEC];
#pragma unroll
    for (int i = 0; i < VEC; i++) th1[i] = th2[i] = 0.0f;
    if (run) theta_pass<KW, kUnroll, VEC, kStaged, kHuber>(K, col_rec, err, wgt, gfirst, gstride, nv, RW, NT, row0, th1, th2);
    for (int off = lprp; off < 32; off <<= 1) {
#pragma unroll
        for (int i = 0; i < VEC; i++) {
            th1[i] += __shfl_xor_sync(0xffffffffu, th1[i], off);
            th2[i] += __shfl_xor_sync(0xffffffffu, th2[i], off);
        }
    }
    if (grp == 0 && run) {
#pragma unroll
        for (int i = 0; i < VEC; i++) {
            S.th1[warp][t0 + i] = th1[i];
            S.th2[warp][t0 + i] = th2[i];
        }
    }
}

// Update the voxel columns of super-voxel (sx, sy) of frame f; the whole CTA
// cooperates (see the file comment for the four passes per column).
// KW: 16-byte words per A record (1, 2, 3 for voxel scale 1, 2, 4);
// kUnroll: views whose records and sinogram entries are in flight together;
// VEC: consecutive detector rows one lane owns (4 when N_t % 4 == 0, else 2);
// kStaged: the column's records are read from shared memory (srec: two
// buffers of stage_words words), the next column's copied in by a TMA bulk copy
// while the current one is updated, so the theta pass waits on one global
// round trip per view group instead of two and the apply pass on none.
// kHuber: 0 the quadratic data term, 1 the generalised Huber one
// (XT_VoxUpdate.c:68-82), 2 decided per problem at run time (K.huber).
template <int KW, int kUnroll, int VEC, bool kStaged, int kHuber>
__device__ __forceinline__ void icd_update_sv(const Geom &g, const IcdLaunch &L, const IcdConst &K,
                                              const uint32_t *__restrict__ table,
                                              const int32_t *__restrict__ view_first,
                                              const uint8_t *__restrict__ mask, float *__restrict__ x,
                                              float *__restrict__ err, const float *__restrict__ wgt,
                                              float *__restrict__ mag, int f, int sx, int sy, IcdSmem &S,
                                              IcdCount &cnt, uint32_t *srec, int stage_words)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, W = blockDim.x >> 5;
    const int NX = g.N_x, NY = g.N_y, NZ = g.N_z, NT = g.N_t, MZ = g.z_overlap;
    const int nxy = NX * NY;
    const int RW = g.rec_words;
    // A voxel column is updated in chunks of at most 32 detector rows (32 / MZ
    // voxel slices, one per lane of warp 0); chunk k covers rows [32k, 32k + 32)
    // and slices [k CZ, k CZ + CZ). Columns of up to 32 rows are one chunk.
    const int CT = NT < 32 ? NT : 32, CZ = CT / MZ;
    const int n_chunks = (NT + 31) / 32;

    // lane -> (view group, run of VEC detector rows) for the theta / apply passes
    using VT = typename VecF<VEC>::T;
    const int lpr = CT / VEC;  // lanes per sinogram row of a full chunk
    int lprp = 1;
    while (lprp < lpr) lprp <<= 1;
    const int G = 32 / lprp;  // view groups per warp
    const int grp = lane / lprp, tq = lane % lprp;
    const int t0 = tq * VEC;  // first detector row of this lane within the chunk
    const int gstride = W * G;
    const int gfirst = warp * G + grp;
    const int fv0 = view_first[f], nv = view_first[f + 1] - fv0;
    const int iter = L.iter_dev ? *L.iter_dev : L.iter;  // 1-based iteration number

    // ---- the SV's columns inside the reconstruction circle, shuffled ----------
    if (warp == 0) {
        const int ncand = L.sv * L.sv;
        int n = 0;
        for (int base = 0; base < ncand; base += 32) {
            const int i = base + lane;
            int ok = 0, c = 0;
            if (i < ncand) {
                const int j = sy * L.sv + i / L.sv, k = sx * L.sv + i % L.sv;
                if (j < NY && k < NX) {
                    c = j * NX + k;
                    ok = mask[c] && (!L.sel || L.sel[(size_t)f * nxy + c]);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) S.order[n + __popc(m & ((1u << lane) - 1))] = c;
            n += __popc(m);
        }
        __syncwarp();
        if (lane == 0) {
            uint64_t h = mix64(L.seed ^ mix64(((uint64_t)iter << 40) ^ ((uint64_t)f << 20) ^
                                             (uint64_t)(sy * L.n_sv_x + sx)));
            for (int i = n - 1; i > 0; i--) {  // Fisher-Yates
                h = mix64(h);
                const int r = (int)(h % (uint64_t)(i + 1));
                const int t = S.order[i];
                S.order[i] = S.order[r];
                S.order[r] = t;
            }
            S.ncols = n;
        }
    }
    __syncthreads();
    const int ncols = S.ncols;
    const size_t rec_frame = (size_t)fv0 * nxy;
    if (kStaged && ncols > 0)
        stage_records(srec, table + (rec_frame + (size_t)S.order[0] * nv) * RW, nv * RW, &S.stage_bar[0]);

    for (int ci = 0; ci < ncols; ci++) {
        const int c = S.order[ci];
        const int j = c / NX, k = c - j * NX;
        const size_t col_off = ((size_t)f * nxy + c) * NZ;
        const uint32_t *col_rec = kStaged ? srec + (ci & 1) * stage_words : table + (rec_frame + (size_t)c * nv) * RW;

        for (int ch = 0; ch < n_chunks; ch++) {
            const int z0 = ch * CZ;                                  // first slice of the chunk
            const int cz = NZ - z0 < CZ ? NZ - z0 : CZ;              // slices in the chunk
            const int ct = cz * MZ;                                  // detector rows in the chunk
            const int rbase = ch * 32;                               // first detector row of the chunk
            const bool zl = lane < cz;
            const int z = z0 + lane;                                 // this lane's slice
            const bool row_ok = tq < ct / VEC;

            // ---- 1. neighbourhood (sources split over warps) + column activity ------
            int active_pred;
            const float V = zl ? x[col_off + z] : 0.0f;  // the column itself (warp 0 reuses it in the solve)
            {
                float num = 0.0f, den = 0.0f;
                int pos = 0;
                for (int s = warp; s < 10; s += W) {
                    if (s < 8) {
                        const int o = s < 4 ? s : s + 1;  // skip the centre of the 3x3
                        const int dy = o / 3 - 1, dx = o % 3 - 1;
                        const int jj = j + dy, kk = k + dx;
                        const bool valid = jj >= 0 && jj < NY && kk >= 0 && kk < NX;
                        const size_t noff = ((size_t)f * nxy + jj * NX + kk) * NZ;
                        const float nz0 = (valid && zl) ? x[noff + z] : 0.0f;
                        float nzm = __shfl_up_sync(0xffffffffu, nz0, 1);
                        float nzp = __shfl_down_sync(0xffffffffu, nz0, 1);
                        // across chunk edges the z +- 1 neighbours are outside the warp
                        if (lane == 0 && z > 0 && valid) nzm = x[noff + z - 1];
                        if (lane == cz - 1 && z + 1 < NZ && valid) nzp = x[noff + z + 1];
                        if (valid && zl) {
                            const float nb[3] = {nzm, nz0, nzp};
#pragma unroll
                            for (int dz = -1; dz <= 1; dz++) {
                                const int zz = z + dz;
                                if (zz < 0 || zz >= NZ) continue;
                                const float n = nb[dz + 1];
                                const float b = qg_weight(V - n, K.q, K.qmp, K.issq, K.issqp, K.cs, K.bs0);
                                const float cf = K.sf[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] * b;
                                num += cf * n;
                                den += cf;
                                pos |= n > 0.0f;
                            }
                        }
                    } else {
                        const int ff = f + (s == 8 ? -1 : 1);
                        if (ff >= 0 && ff < g.N_time && zl) {
                            const float n = x[((size_t)ff * nxy + c) * NZ + z];
                            const float b = qg_weight(V - n, K.q, K.qmp, K.istq, K.istqp, K.ct, K.bt0);
                            const float cf = K.tf * b;
                            num += cf * n;
                            den += cf;
                            pos |= n > 0.0f;
                        }
                    }
                }
                S.num[warp][lane] = num;
                S.den[warp][lane] = den;
                S.pos[warp][lane] = pos;
                // a column is skipped only if every slice is zero with no positive
                // neighbour (in-column neighbours are the column's own values)
                active_pred = !L.zero_skipping || iter <= 1 || (zl && V != 0.0f) || pos;
            }
            // ---- 2. theta over the column's views. When the column is surely
            //         active (zero skipping off or in its first iteration, or a
            //         nonzero slice: the same test in every warp, as every warp
            //         read the column), theta runs before the barrier that also
            //         publishes the neighbourhood sums, so its loads go out without
            //         waiting for the other warps; otherwise after it, and only
            //         for an active column -------------------------------------------
            bool recs_ok = true;
            if (kStaged && ch == 0)  // issued one column earlier
                recs_ok = wait_staged(&S.stage_bar[ci & 1], cnt.phases, ci & 1, cnt.timeouts, S.abort, S.abort_bar,
                                      S.abort_parity);
            const bool sure = !L.zero_skipping || iter <= 1 || __any_sync(0xffffffffu, zl && V != 0.0f);
            // a thread whose wait gave up reads no record (their headers address
            // the sinogram); the CTA leaves after the barrier
            if (sure)
                theta_column<KW, kUnroll, VEC, kStaged, kHuber>(K, col_rec, err, wgt, gfirst, gstride, nv, RW, NT,
                                                               rbase + t0, row_ok && recs_ok, lprp, grp, t0, warp, S);
            const int any_active = __syncthreads_or(active_pred);
            if (ch == 0) {
                // a late copy leaves this column's records undefined: no update, no
                // further copies (S.abort is read after the barrier, so uniformly)
                if (kStaged && S.abort) return;
                // every thread is past the previous column's apply pass: its record
                // buffer may be refilled with the next column's
                if (kStaged && ci + 1 < ncols)
                    stage_records(srec + ((ci + 1) & 1) * stage_words,
                                  table + (rec_frame + (size_t)S.order[ci + 1] * nv) * RW, nv * RW,
                                  &S.stage_bar[(ci + 1) & 1]);
            }
            if (!any_active) {
                if (warp == 0 && zl) cnt.skip++;
                if (warp == 0 && lane == 0 && ch == 0) mag[(size_t)f * nxy + c] = 0.0f;
                continue;  // uniform across the CTA
            }
            if (!sure) {  // uniform across the CTA
                theta_column<KW, kUnroll, VEC, kStaged, kHuber>(K, col_rec, err, wgt, gfirst, gstride, nv, RW, NT,
                                                               rbase + t0, row_ok && recs_ok, lprp, grp, t0, warp, S);
                __syncthreads();
            }

            // ---- 3. zero-skipping and solve (warp 0, lane = slice of the chunk) ------
            if (warp == 0) {
                const float V0 = V;
                float numA = 0.0f, denA = 0.0f, t1 = 0.0f, t2 = 0.0f;
                int pos = 0;
                for (int w = 0; w < W; w++) {
                    numA += S.num[w][lane];
                    denA += S.den[w][lane];
                    pos |= S.pos[w][lane];
                    if (lane < ct) {
                        t1 += S.th1[w][lane];
                        t2 += S.th2[w][lane];
                    }
                }
                // in-column z - 1 / z + 1: the chunk below is already updated
                // (Gauss-Seidel over the chunks), the chunk above not yet
                const float edge_m = (z0 > 0) ? x[col_off + z0 - 1] : 0.0f;
                const float edge_p = (z0 + cz < NZ) ? x[col_off + z0 + cz] : 0.0f;
                {
                    float vm = __shfl_up_sync(0xffffffffu, V0, 1);
                    float vp = __shfl_down_sync(0xffffffffu, V0, 1);
                    if (lane == 0) vm = edge_m;
                    if (lane == cz - 1) vp = edge_p;
                    if (z >= 1 && vm > 0.0f) pos = 1;
                    if (z + 1 < NZ && vp > 0.0f) pos = 1;
                }
                const bool skip = !zl || (L.zero_skipping && iter > 1 && V0 == 0.0f && !pos);
                __syncwarp();
                S.th1[0][lane] = t1;
                S.th2[0][lane] = t2;
                __syncwarp();
                float th1 = 0.0f, th2 = 0.0f;
                if (zl)
                    for (int r = 0; r < MZ; r++) {
                        th1 += S.th1[0][lane * MZ + r];
                        th2 += S.th2[0][lane * MZ + r];
                    }
                float cur = V0;
#pragma unroll
                for (int parity = 0; parity < 2; parity++) {
                    float vm = __shfl_up_sync(0xffffffffu, cur, 1);
                    float vp = __shfl_down_sync(0xffffffffu, cur, 1);
                    if (lane == 0) vm = edge_m;
                    if (lane == cz - 1) vp = edge_p;
                    if (!skip && (z & 1) == parity) {
                        float num = numA, den = denA;
                        if (z >= 1) {
                            const float cf = K.sf[0 * 9 + 4] * qg_weight(V0 - vm, K.q, K.qmp, K.issq, K.issqp, K.cs, K.bs0);
                            num += cf * vm;
                            den += cf;
                        }
                        if (z + 1 < NZ) {
                            const float cf = K.sf[2 * 9 + 4] * qg_weight(V0 - vp, K.q, K.qmp, K.issq, K.issqp, K.cs, K.bs0);
                            num += cf * vp;
                            den += cf;
                        }
                        const float u = (num + th2 * V0 - th1) / (den + th2);
                        cur = V0 + K.alpha * (u - V0);
                    }
                }
                const float dx = skip ? 0.0f : cur - V0;
                S.dx[lane] = dx;
                if (zl) {
                    if (!skip) {
                        x[col_off + z] = cur;
                        cnt.upd++;
                        cnt.sum_dx += fabsf(dx);
                        cnt.sum_x += fabsf(cur);
                    } else {
                        cnt.skip++;
                    }
                }
                float m = fabsf(dx);
                for (int off = 16; off > 0; off >>= 1) m += __shfl_xor_sync(0xffffffffu, m, off);
                if (lane == 0) {
                    float *mp = mag + (size_t)f * nxy + c;
                    *mp = ch == 0 ? m : *mp + m;
                }
            }
            __syncthreads();

            // ---- 4. apply e -= a dx (the next chunk's or column's barrier orders
            //         these reductions before its theta loads) ---------------------------
            {
                float dxv[VEC];
                bool any = false;
#pragma unroll
                for (int i = 0; i < VEC; i++) {
                    dxv[i] = row_ok ? S.dx[(t0 + i) / MZ] : 0.0f;
                    any |= dxv[i] != 0.0f;
                }
                if (any) {
                    for (int v0 = gfirst; v0 < nv; v0 += kUnroll * gstride) {
                        Rec<KW> R[kUnroll];
#pragma unroll
                        for (int u = 0; u < kUnroll; u++) {
                            const int v = v0 + u * gstride;
                            if (v < nv) R[u] = kStaged ? load_rec_smem<KW>(col_rec + (size_t)v * RW)
                                                   : load_rec<KW>(col_rec + (size_t)v * RW);
                            else R[u].w[0].x = 0u;
                        }
#pragma unroll
                        for (int u = 0; u < kUnroll; u++) {
                            const uint32_t hdr = R[u].w[0].x;
                            const int cnt_q = hdr >> 24;
                            const unsigned sb = (hdr & 0xFFFFFFu) * (unsigned)NT + (unsigned)(rbase + t0);
#pragma unroll
                            for (int q = 0; q < 4 * KW - 1; q++) {
                                if (q < cnt_q) {
                                    const float a = -(rec_val<KW>(R[u], q) * K.dt);
                                    float d[VEC];
#pragma unroll
                                    for (int i = 0; i < VEC; i++) d[i] = a * dxv[i];
                                    red_add(err + (sb + (unsigned)(q * NT)), d);
                                }
                            }
                        }
                    }
                }
            }
        }
    }
}

}  // namespace

// One colour phase of one problem: persistent CTAs drain the phase's SV queue.
// With kStaged, the dynamic shared memory holds two record buffers of
// stage_words words each (the current and the next column's A records).
template <int KW, int kUnroll, int VEC, bool kStaged, int kHuber>
__global__ void __launch_bounds__(kMaxWarps * 32, 4) icd_phase_kernel(
    Geom g, IcdLaunch L, IcdConst K, const uint32_t *__restrict__ table, const int32_t *__restrict__ view_first,
    const uint8_t *__restrict__ mask, float *__restrict__ x, float *__restrict__ err, const float *__restrict__ wgt,
    float *__restrict__ mag, IcdStats *__restrict__ stats, unsigned int *__restrict__ queue, int stage_words)
{
    __shared__ IcdSmem S;
    extern __shared__ __align__(16) uint32_t s_rec[];
    const int KC = L.colors_k;
    const int hx = (L.n_sv_x + KC - 1) / KC, slots = hx * ((L.n_sv_y + KC - 1) / KC);
    const int n_items = L.items ? *L.n_items : g.N_time * slots;
    IcdCount cnt{};
    if (threadIdx.x == 0) S.abort = 0;
    if (kStaged && threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((unsigned)__cvta_generic_to_shared(&S.stage_bar[0]))
                     : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((unsigned)__cvta_generic_to_shared(&S.stage_bar[1]))
                     : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (;;) {
        __syncthreads();  // S.item / S.order of the previous SV are no longer read
        if (kStaged && S.abort) break;  // uniform: written before the barrier
        if (threadIdx.x == 0) S.item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int item = S.item;
        if (item >= n_items) break;
        int f, sx, sy;
        if (L.items) {  // explicit work list (its SVs hold columns to update)
            const uint32_t code = L.items[item];
            f = (int)(code >> 22);
            sy = (int)((code >> 11) & 2047u);
            sx = (int)(code & 2047u);
        } else {
            f = item % g.N_time;  // frames fastest: concurrent SVs spread over the frames
            const int rem = (int)((long long)(item / g.N_time) * L.perm % slots);
            const int color = (L.phase + f) % (KC * KC);  // frame f +- 1 is never on the same colour
            sx = KC * (rem % hx) + color % KC;
            sy = KC * (rem / hx) + color / KC;
        }
        if (sx >= L.n_sv_x || sy >= L.n_sv_y) continue;  // uniform
        icd_update_sv<KW, kUnroll, VEC, kStaged, kHuber>(g, L, K, table, view_first, mask, x, err, wgt, mag, f, sx, sy,
                                                         S,
                                                 cnt, s_rec, stage_words);
    }
    // after an abort, the late copy may still write into this CTA's shared
    // memory: give it one more bounded wait before the CTA exits
    if (kStaged && S.abort && threadIdx.x == 0) wait_parity_bounded(&S.stage_bar[S.abort_bar], S.abort_parity);
    flush_counts(cnt, stats);
}

// Record staging needs two buffers of (most views in a frame) x record words;
// above this size the sweep reads records from global memory instead.
constexpr int kMaxStageBytes = 16 * 1024;

template <int KW, int U, int VEC, bool kStaged, int kHuber>
static void launch_staged(const Geom &g, const IcdLaunch &L, const IcdConst &K, const uint32_t *d_table,
                          const int32_t *d_view_first, const uint8_t *d_mask, float *d_x, float *d_err,
                          const float *d_w, float *d_mag, IcdStats *d_stats, unsigned int *d_queue, int stage_words,
                          cudaStream_t st)
{
    const int threads = L.warps * 32;
    const size_t smem = kStaged ? 2 * (size_t)stage_words * sizeof(uint32_t) : 0;
    // resident CTAs per SM, cached per (device, block size, shared memory) so a
    // launch being captured into a CUDA graph makes no occupancy query
    struct Occ {
        int dev, threads, sms, per_sm;
        size_t smem;
    };
    static std::mutex mu;
    static std::vector<Occ> cache;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(mu);
        bool hit = false;
        for (const Occ &o : cache)
            if (o.dev == dev && o.threads == threads && o.smem == smem) {
                sms = o.sms;
                per_sm = o.per_sm;
                hit = true;
                break;
            }
        if (!hit) {
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, icd_phase_kernel<KW, U, VEC, kStaged, kHuber>, threads, smem);
            cache.push_back({dev, threads, sms, per_sm, smem});
        }
    }
    const long long items = (long long)g.N_time * sv_slots(g.N_x, g.N_y, L.sv, L.colors_k);
    long long grid = (long long)sms * (per_sm > 0 ? per_sm : 1);
    if (grid > items) grid = items;
    if (L.max_ctas > 0 && grid > L.max_ctas) grid = L.max_ctas;
    icd_phase_kernel<KW, U, VEC, kStaged, kHuber><<<(unsigned)grid, threads, smem, st>>>(
        g, L, K, d_table, d_view_first, d_mask, d_x, d_err, d_w, d_mag, d_stats, d_queue, stage_words);
}

template <int KW, int U, int VEC>
static void launch_kw(const Geom &g, const IcdLaunch &L, const IcdConst &K, const uint32_t *d_table,
                      const int32_t *d_view_first, const uint8_t *d_mask, float *d_x, float *d_err, const float *d_w,
                      float *d_mag, IcdStats *d_stats, unsigned int *d_queue, cudaStream_t st)
{
    const int stage_words = g.max_views * g.rec_words;  // a multiple of 4 words: 16-byte aligned buffers
    const bool staged = L.stage_records && 2 * (size_t)stage_words * sizeof(uint32_t) <= (size_t)kMaxStageBytes;
#define MBIR_STAGED(S, H)                                                                                         \
    launch_staged<KW, U, VEC, S, H>(g, L, K, d_table, d_view_first, d_mask, d_x, d_err, d_w, d_mag, d_stats, d_queue, \
                                    S ? stage_words : 0, st)
    if (staged) {
        if (K.huber) MBIR_STAGED(true, 1);
        else MBIR_STAGED(true, 0);
    } else {
        if (K.huber) MBIR_STAGED(false, 1);
        else MBIR_STAGED(false, 0);
    }
#undef MBIR_STAGED
}

IcdConst make_icd_const(const Geom &g)
{
    IcdConst K;
    for (int i = 0; i < 27; i++) K.sf[i] = (float)g.spatial_filter[i];
    K.tf = (float)g.time_filter;
    K.q = (float)g.q;
    K.qmp = (float)(g.q - g.p);
    K.ssq = (float)g.sigma_s_q;
    K.ssqp = (float)g.sigma_s_q_p;
    K.stq = (float)g.sigma_t_q;
    K.stqp = (float)g.sigma_t_q_p;
    K.issq = (float)(1.0 / g.sigma_s_q);
    K.issqp = (float)(1.0 / g.sigma_s_q_p);
    K.istq = (float)(1.0 / g.sigma_t_q);
    K.istqp = (float)(1.0 / g.sigma_t_q_p);
    K.cs = (float)g.c_s;
    K.ct = (float)g.c_t;
    K.bs0 = (float)(g.q / (g.sigma_s_q * g.c_s));
    K.bt0 = (float)(g.q / (g.sigma_t_q * g.c_t));
    K.alpha = (float)g.alpha;
    K.dt = (float)g.delta_t;
    K.huber_T = (float)g.huber_T;
    K.huber_delta = (float)g.huber_delta;
    K.huber = g.huber;
    return K;
}

void launch_icd_phase(const Geom &g, const IcdLaunch &L, const uint32_t *d_table, const int32_t *d_view_first,
                      const uint8_t *d_mask, float *d_x, float *d_err, const float *d_w, float *d_mag,
                      IcdStats *d_stats, unsigned int *d_queue, cudaStream_t st)
{
    const IcdConst K = make_icd_const(g);
#define MBIR_LAUNCH(KW, U, VEC) \
    launch_kw<KW, U, VEC>(g, L, K, d_table, d_view_first, d_mask, d_x, d_err, d_w, d_mag, d_stats, d_queue, st)
    const int kw = g.rec_words / 4;
    const bool v4 = g.N_t % 4 == 0;
    if (kw == 1) {
        if (L.unroll >= 2) {
            if (v4) MBIR_LAUNCH(1, 2, 4);
            else MBIR_LAUNCH(1, 2, 2);
        } else {
            if (v4) MBIR_LAUNCH(1, 1, 4);
            else MBIR_LAUNCH(1, 1, 2);
        }
    } else if (kw == 2) {
        if (v4) MBIR_LAUNCH(2, 1, 4);
        else MBIR_LAUNCH(2, 1, 2);
    } else {
        if (v4) MBIR_LAUNCH(3, 1, 4);
        else MBIR_LAUNCH(3, 1, 2);
    }
#undef MBIR_LAUNCH
}

// ---------------------------------------------------------------------------------------------
// Many independent problems in one persistent launch per colour phase. The
// queue runs over the SV items of every problem of the launch, interleaved in
// proportion to each problem's item count (item_map[] gives the problem and
// its item), so the CTAs working at any moment spread over the problems; a
// CTA keeps the descriptor of its current problem in shared memory and
// reloads it when its next item belongs to another problem. Problems of one
// launch share the record width and the detector-row vector width (template
// parameters).
template <int KW, int kUnroll, int VEC>
__global__ void __launch_bounds__(kMaxWarps * 32, 4) icd_batch_kernel(const BatchDesc *__restrict__ descs,
                                                                      const int2 *__restrict__ item_map, int total,
                                                                      int phase, unsigned int *__restrict__ queue)
{
    __shared__ IcdSmem S;
    __shared__ __align__(16) BatchDesc P;
    int cur = -1;
    IcdCount cnt{};
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) S.item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int item = S.item;
        if (item >= total) break;
        const int2 pm = item_map[item];  // (problem, item of that problem)
        if (pm.x != cur) {                // uniform
            if (cur >= 0) flush_counts(cnt, P.stats);
            __syncthreads();
            const int4 *src = reinterpret_cast<const int4 *>(descs + pm.x);
            int4 *dst = reinterpret_cast<int4 *>(&P);
            for (int i = threadIdx.x; i < (int)(sizeof(BatchDesc) / sizeof(int4)); i += blockDim.x) dst[i] = src[i];
            __syncthreads();
            cur = pm.x;
        }
        if (!P.active) continue;
        const int K = P.L.colors_k;
        const int hx = (P.L.n_sv_x + K - 1) / K, slots = hx * ((P.L.n_sv_y + K - 1) / K);
        const int f = pm.y % P.g.N_time;
        const int rem = (int)((long long)(pm.y / P.g.N_time) * P.L.perm % slots);
        const int color = (phase + f) % (K * K);
        const int sx = K * (rem % hx) + color % K;
        const int sy = K * (rem / hx) + color / K;
        if (sx >= P.L.n_sv_x || sy >= P.L.n_sv_y) continue;
        icd_update_sv<KW, kUnroll, VEC, false, 2>(P.g, P.L, P.K, P.table, P.view_first, P.mask, P.x, P.err, P.w, P.mag,
                                               f, sx, sy, S, cnt, nullptr, 0);
    }
    if (cur >= 0) flush_counts(cnt, P.stats);
}

// Before an iteration: advance every problem's iteration number and clear its counters.
__global__ void batch_begin_iteration(BatchDesc *descs, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    descs[i].L.iter += 1;
    *descs[i].stats = IcdStats{};
}

// After an iteration: accumulate the updates and stop problems whose
// convergence statistic 100 sum|dx| / sum|x| fell below their threshold after
// the first iteration (XT_ICD_update.c:1083-1090).
__global__ void batch_end_iteration(BatchDesc *descs, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !descs[i].active) return;
    const IcdStats s = *descs[i].stats;
    descs[i].total_updates += s.updates;
    descs[i].iters_done = descs[i].L.iter;
    const double pct = s.sum_abs_x > 0 ? 100.0 * s.sum_abs_dx / s.sum_abs_x : 0.0;
    descs[i].last_pct = pct;
    if (descs[i].L.iter > 1 && pct < descs[i].convg_thresh) descs[i].active = 0;
}

int batch_grid(int vec, int warps)
{
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (vec == 4) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, icd_batch_kernel<1, 2, 4>, warps * 32, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, icd_batch_kernel<1, 2, 2>, warps * 32, 0);
    return sms * (per_sm > 0 ? per_sm : 1);
}

void launch_icd_batch(int vec, int warps, int grid, const BatchDesc *d_descs, const int2 *d_item_map, int total,
                      int phase, unsigned int *d_queue, cudaStream_t st)
{
    if (vec == 4) icd_batch_kernel<1, 2, 4><<<grid, warps * 32, 0, st>>>(d_descs, d_item_map, total, phase, d_queue);
    else icd_batch_kernel<1, 2, 2><<<grid, warps * 32, 0, st>>>(d_descs, d_item_map, total, phase, d_queue);
}

int icd_grid(int warps)
{
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, icd_phase_kernel<1, 2, 4, false, 0>, warps * 32, 0);
    return sms * (per_sm > 0 ? per_sm : 1);
}

void launch_batch_begin(BatchDesc *d_descs, int n, cudaStream_t st)
{
    batch_begin_iteration<<<(n + 127) / 128, 128, 0, st>>>(d_descs, n);
}

void launch_batch_end(BatchDesc *d_descs, int n, cudaStream_t st)
{
    batch_end_iteration<<<(n + 127) / 128, 128, 0, st>>>(d_descs, n);
}

}  // namespace mbirgpu
