// Super-voxel parallel ICD sweep (one colour phase per launch).
//
// Replaces the voxel loop of updateVoxelsTimeSlices / updateVoxels_Atten /
// compute_voxel_update_Atten (MBIR_4D/XT_ICD_update.c:932-1092,
// XT_VoxUpdate.c:45-283) and the surrogate solve CE_FunctionalSubstitution
// (XT_ICD_update.c:133-182).
//
// Schedule. The image plane is tiled into super-voxels (SVs) of sv x sv voxel
// columns; an SV's colour is (sv_y & 1, sv_x & 1). Phase p updates, in frame
// f, the SVs of colour p ^ (f & 1): no two SVs updated at once share a prior
// neighbour, and a voxel and its temporal neighbours (same column, frames
// f +- 1) are never updated at once -- the GPU counterpart of the
// reference's z-block / frame checkerboard (XT_ICD_update.c:964-1046). Frames
// use disjoint views, so different frames never share sinogram entries;
// concurrent SVs of one frame can share entries along a ray, and their error
// sinogram updates are atomic adds.
//
// One CTA owns one SV and visits its voxel columns one after another in a
// seeded random order (the counterpart of randomly_select_x_y,
// XT_ICD_update.c:499-531). For one column all warps cooperate:
//   1. neighbourhood: the 8 in-plane neighbour columns and the 2 temporal
//      neighbours are split over the warps; each lane owns one slice z and
//      accumulates the qGGMRF surrogate terms b = w rho'(d)/d of those
//      neighbours (XT_ICD_update.c:140-172) and the zero-skipping test
//      (XT_VoxUpdate.c:238-261);
//   2. theta: the column's views are split over warps; a lane owns one
//      detector row t and accumulates theta1 = -sum a w e and theta2 =
//      sum a^2 w over the column's A entries (a = A value x delta_t,
//      XT_VoxUpdate.c:56-85) -- reads of e[view][r][0..N_t) are coalesced;
//   3. solve: warp 0 sums the partials, then updates even slices and odd
//      slices in turn (their only mutual coupling is the in-column z +- 1
//      prior pair), x <- V + alpha (u - V);
//   4. apply: e[view][r][t] -= a dx(slice of t) with atomic adds.
// All arithmetic is FP32; the host refreshes e in FP64 periodically.
#include "mbir_internal.h"

namespace mbirgpu {

namespace {

constexpr int kMaxWarps = 8;
constexpr int kMaxSvCols = 256;  // sv <= 16

struct IcdConst {
    float sf[27];
    float tf;
    float q, qmp, ssq, ssqp, stq, stqp, cs, ct, bs0, bt0, alpha, dt;
    float huber_T, huber_delta;
    int huber;
};

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Surrogate weight rho'(d)/d of the qGGMRF potential
// |d|^q / sq / (c + |d|^(q-p) / sqp) (derivative per XT_ICD_update.c:92-118;
// value at d = 0 per :119-128): |d|^(q-2) (q - (q-p) t1 / t3) / (t3 sq),
// t1 = |d|^(q-p) / sqp, t3 = c + t1.
__device__ __forceinline__ float qg_weight(float d, float q, float qmp, float sq, float sqp, float c, float b0)
{
    if (d == 0.0f) return b0;
    const float ad = fabsf(d);
    const float t1 = __expf(qmp * __logf(ad)) / sqp;
    const float t3 = c + t1;
    float r = (q - qmp * t1 / t3) / (t3 * sq);
    if (q != 2.0f) r *= __expf((q - 2.0f) * __logf(ad));
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
__device__ __forceinline__ float rec_val(const Rec<KW> &r, int q)
{
    // word 1 + q of the record
    const int wi = 1 + q;
    const uint4 &u = r.w[wi >> 2];
    const uint32_t bits = (wi & 3) == 0 ? u.x : (wi & 3) == 1 ? u.y : (wi & 3) == 2 ? u.z : u.w;
    return __uint_as_float(bits);
}

}  // namespace

template <int KW>
__global__ void __launch_bounds__(kMaxWarps * 32) icd_phase_kernel(
    Geom g, IcdLaunch L, IcdConst K, const uint32_t *__restrict__ table, const int32_t *__restrict__ view_first,
    const int32_t *__restrict__ views, const uint8_t *__restrict__ mask, float *__restrict__ x,
    float *__restrict__ err, const float *__restrict__ wgt, float *__restrict__ mag, IcdStats *__restrict__ stats)
{
    __shared__ float s_num[kMaxWarps][32], s_den[kMaxWarps][32];
    __shared__ float s_th1[kMaxWarps][32], s_th2[kMaxWarps][32];
    __shared__ int s_pos[kMaxWarps][32];
    __shared__ float s_dx[32];
    __shared__ int s_order[kMaxSvCols];
    __shared__ int s_ncols, s_active;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, W = blockDim.x >> 5;
    const int f = blockIdx.y;
    const int color = L.phase ^ (f & 1);
    const int half_x = (L.n_sv_x + 1) / 2;
    const int sx = 2 * (blockIdx.x % half_x) + (color & 1);
    const int sy = 2 * (blockIdx.x / half_x) + (color >> 1);
    if (sx >= L.n_sv_x || sy >= L.n_sv_y) return;

    const int NX = g.N_x, NY = g.N_y, NZ = g.N_z, NT = g.N_t, NR = g.N_r, MZ = g.z_overlap;
    const int nxy = NX * NY;
    const int fv0 = view_first[f], nv = view_first[f + 1] - fv0;
    const int RW = g.rec_words;

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
                    ok = mask[c];
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) s_order[n + __popc(m & ((1u << lane) - 1))] = c;
            n += __popc(m);
        }
        __syncwarp();
        if (lane == 0) {
            uint64_t h = mix64(L.seed ^ mix64(((uint64_t)L.iter << 40) ^ ((uint64_t)f << 20) ^
                                             (uint64_t)(sy * L.n_sv_x + sx)));
            for (int i = n - 1; i > 0; i--) {  // Fisher-Yates
                h = mix64(h);
                const int r = (int)(h % (uint64_t)(i + 1));
                const int t = s_order[i];
                s_order[i] = s_order[r];
                s_order[r] = t;
            }
            s_ncols = n;
        }
    }
    __syncthreads();
    const int ncols = s_ncols;

    // lane -> (view group, detector row) for the theta / apply passes
    int ntp = 4;
    while (ntp < NT) ntp <<= 1;
    const int G = 32 / ntp;  // view groups per warp
    const int grp = lane / ntp, trow = lane % ntp;
    const bool row_ok = trow < NT;
    const int gstride = W * G;
    const int gfirst = warp * G + grp;
    const int zrow = trow / MZ;  // voxel slice of this detector row

    unsigned long long n_upd = 0, n_skip = 0;
    float sum_dx = 0.0f, sum_x = 0.0f;

    for (int ci = 0; ci < ncols; ci++) {
        const int c = s_order[ci];
        const int j = c / NX, k = c - j * NX;
        const size_t col_off = ((size_t)f * nxy + c) * NZ;
        const bool zl = lane < NZ;

        // ---- 1. neighbourhood (sources split over warps) -------------------------
        {
            const float V = zl ? x[col_off + lane] : 0.0f;
            float num = 0.0f, den = 0.0f;
            int pos = 0;
            for (int s = warp; s < 10; s += W) {
                if (s < 8) {
                    const int o = s < 4 ? s : s + 1;  // skip the centre of the 3x3
                    const int dy = o / 3 - 1, dx = o % 3 - 1;
                    const int jj = j + dy, kk = k + dx;
                    const bool valid = jj >= 0 && jj < NY && kk >= 0 && kk < NX;
                    const float nz0 = (valid && zl) ? x[((size_t)f * nxy + jj * NX + kk) * NZ + lane] : 0.0f;
                    const float nzm = __shfl_up_sync(0xffffffffu, nz0, 1);
                    const float nzp = __shfl_down_sync(0xffffffffu, nz0, 1);
                    if (valid && zl) {
                        const float nb[3] = {nzm, nz0, nzp};
#pragma unroll
                        for (int dz = -1; dz <= 1; dz++) {
                            const int zz = lane + dz;
                            if (zz < 0 || zz >= NZ) continue;
                            const float n = nb[dz + 1];
                            const float b = qg_weight(V - n, K.q, K.qmp, K.ssq, K.ssqp, K.cs, K.bs0);
                            const float cf = K.sf[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] * b;
                            num += cf * n;
                            den += cf;
                            pos |= n > 0.0f;
                        }
                    }
                } else {
                    const int ff = f + (s == 8 ? -1 : 1);
                    if (ff >= 0 && ff < g.N_time && zl) {
                        const float n = x[((size_t)ff * nxy + c) * NZ + lane];
                        const float b = qg_weight(V - n, K.q, K.qmp, K.stq, K.stqp, K.ct, K.bt0);
                        const float cf = K.tf * b;
                        num += cf * n;
                        den += cf;
                        pos |= n > 0.0f;
                    }
                }
            }
            s_num[warp][lane] = num;
            s_den[warp][lane] = den;
            s_pos[warp][lane] = pos;
        }
        __syncthreads();

        // ---- zero-skipping decision (warp 0) ---------------------------------------
        float V0 = 0.0f, numA = 0.0f, denA = 0.0f;
        bool skip = true;
        if (warp == 0) {
            V0 = zl ? x[col_off + lane] : 0.0f;
            int pos = 0;
            for (int w = 0; w < W; w++) {
                numA += s_num[w][lane];
                denA += s_den[w][lane];
                pos |= s_pos[w][lane];
            }
            const float vm = __shfl_up_sync(0xffffffffu, V0, 1);
            const float vp = __shfl_down_sync(0xffffffffu, V0, 1);
            if (lane >= 1 && vm > 0.0f) pos = 1;
            if (lane + 1 < NZ && vp > 0.0f) pos = 1;
            skip = !zl || (L.zero_skipping && L.iter > 1 && V0 == 0.0f && !pos);
            const unsigned act = __ballot_sync(0xffffffffu, !skip);
            if (lane == 0) s_active = act != 0u;
        }
        __syncthreads();
        if (!s_active) {
            if (warp == 0 && zl) n_skip++;
            if (warp == 0 && lane == 0) mag[(size_t)f * nxy + c] = 0.0f;
            continue;  // uniform across the CTA
        }

        // ---- 2. theta over the column's views ---------------------------------------
        const uint32_t *col_rec = table + ((size_t)fv0 * nxy + (size_t)c * nv) * RW;
        {
            float th1 = 0.0f, th2 = 0.0f;
            if (row_ok) {
                for (int v = gfirst; v < nv; v += gstride) {
                    const Rec<KW> R = load_rec<KW>(col_rec + (size_t)v * RW);
                    const uint32_t hdr = R.w[0].x;
                    const int cnt = hdr >> 16, first = hdr & 0xFFFF;
                    const size_t sbase = ((size_t)views[fv0 + v] * NR + first) * NT + trow;
#pragma unroll
                    for (int q = 0; q < 4 * KW - 1; q++) {
                        if (q < cnt) {
                            const float a = rec_val<KW>(R, q) * K.dt;
                            const float e = __ldcg(err + sbase + (size_t)q * NT);
                            const float wv = __ldg(wgt + sbase + (size_t)q * NT);
                            float ww = wv;
                            if (K.huber) {
                                const float se = fabsf(e * sqrtf(wv));
                                if (!(se < K.huber_T)) ww = K.huber_T * K.huber_delta * sqrtf(wv) / fabsf(e);
                            }
                            th2 += a * a * ww;
                            th1 -= e * a * ww;
                        }
                    }
                }
            }
            // fold the view groups of the warp onto group 0
            for (int off = ntp; off < 32; off <<= 1) {
                th1 += __shfl_xor_sync(0xffffffffu, th1, off);
                th2 += __shfl_xor_sync(0xffffffffu, th2, off);
            }
            s_th1[warp][lane] = th1;
            s_th2[warp][lane] = th2;
        }
        __syncthreads();

        // ---- 3. solve (warp 0, lane = slice) ----------------------------------------
        if (warp == 0) {
            // sum over warps per detector row, then over the rows of each slice
            float t1 = 0.0f, t2 = 0.0f;
            for (int w = 0; w < W; w++) {
                t1 += s_th1[w][lane];
                t2 += s_th2[w][lane];
            }
            __syncwarp();
            s_th1[0][lane] = t1;
            s_th2[0][lane] = t2;
            __syncwarp();
            float th1 = 0.0f, th2 = 0.0f;
            if (zl)
                for (int r = 0; r < MZ; r++) {
                    th1 += s_th1[0][lane * MZ + r];
                    th2 += s_th2[0][lane * MZ + r];
                }
            float cur = V0;
#pragma unroll
            for (int parity = 0; parity < 2; parity++) {
                const float vm = __shfl_up_sync(0xffffffffu, cur, 1);
                const float vp = __shfl_down_sync(0xffffffffu, cur, 1);
                if (!skip && (lane & 1) == parity) {
                    float num = numA, den = denA;
                    if (lane >= 1) {
                        const float cf = K.sf[0 * 9 + 4] * qg_weight(V0 - vm, K.q, K.qmp, K.ssq, K.ssqp, K.cs, K.bs0);
                        num += cf * vm;
                        den += cf;
                    }
                    if (lane + 1 < NZ) {
                        const float cf = K.sf[2 * 9 + 4] * qg_weight(V0 - vp, K.q, K.qmp, K.ssq, K.ssqp, K.cs, K.bs0);
                        num += cf * vp;
                        den += cf;
                    }
                    const float u = (num + th2 * V0 - th1) / (den + th2);
                    cur = V0 + K.alpha * (u - V0);
                }
            }
            const float dx = skip ? 0.0f : cur - V0;
            if (zl) {
                if (!skip) x[col_off + lane] = cur;
                s_dx[lane] = dx;
                if (skip) n_skip++;
                else {
                    n_upd++;
                    sum_dx += fabsf(dx);
                    sum_x += fabsf(cur);
                }
            } else {
                s_dx[lane] = 0.0f;
            }
            float m = fabsf(dx);
            for (int off = 16; off > 0; off >>= 1) m += __shfl_xor_sync(0xffffffffu, m, off);
            if (lane == 0) mag[(size_t)f * nxy + c] = m;
        }
        __syncthreads();

        // ---- 4. apply e -= a dx ------------------------------------------------------
        {
            const float dx = row_ok ? s_dx[zrow] : 0.0f;
            if (dx != 0.0f) {
                for (int v = gfirst; v < nv; v += gstride) {
                    const Rec<KW> R = load_rec<KW>(col_rec + (size_t)v * RW);
                    const uint32_t hdr = R.w[0].x;
                    const int cnt = hdr >> 16, first = hdr & 0xFFFF;
                    const size_t sbase = ((size_t)views[fv0 + v] * NR + first) * NT + trow;
#pragma unroll
                    for (int q = 0; q < 4 * KW - 1; q++)
                        if (q < cnt) atomicAdd(err + sbase + (size_t)q * NT, -(rec_val<KW>(R, q) * K.dt) * dx);
                }
            }
        }
        // the next column's neighbourhood pass reads x written above and its
        // theta pass reads e updated above; both are ordered by the barrier
        // after the next neighbourhood pass.
    }

    // ---- per-CTA statistics -------------------------------------------------------------
    if (warp == 0) {
        for (int off = 16; off > 0; off >>= 1) {
            n_upd += __shfl_xor_sync(0xffffffffu, n_upd, off);
            n_skip += __shfl_xor_sync(0xffffffffu, n_skip, off);
            sum_dx += __shfl_xor_sync(0xffffffffu, sum_dx, off);
            sum_x += __shfl_xor_sync(0xffffffffu, sum_x, off);
        }
        if (lane == 0) {
            atomicAdd(&stats->updates, n_upd);
            atomicAdd(&stats->skipped, n_skip);
            atomicAdd(&stats->sum_abs_dx, (double)sum_dx);
            atomicAdd(&stats->sum_abs_x, (double)sum_x);
        }
    }
}

void launch_icd_phase(const Geom &g, const IcdLaunch &L, const uint32_t *d_table, const int32_t *d_view_first,
                      const int32_t *d_views, const uint8_t *d_mask, float *d_x, float *d_err, const float *d_w,
                      float *d_mag, IcdStats *d_stats, cudaStream_t st)
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
    K.cs = (float)g.c_s;
    K.ct = (float)g.c_t;
    K.bs0 = (float)(g.q / (g.sigma_s_q * g.c_s));
    K.bt0 = (float)(g.q / (g.sigma_t_q * g.c_t));
    K.alpha = (float)g.alpha;
    K.dt = (float)g.delta_t;
    K.huber_T = (float)g.huber_T;
    K.huber_delta = (float)g.huber_delta;
    K.huber = g.huber;
    const int half_x = (L.n_sv_x + 1) / 2, half_y = (L.n_sv_y + 1) / 2;
    dim3 grid(half_x * half_y, g.N_time);
    const int threads = L.warps * 32;
    switch (g.rec_words / 4) {
    case 1:
        icd_phase_kernel<1><<<grid, threads, 0, st>>>(g, L, K, d_table, d_view_first, d_views, d_mask, d_x, d_err, d_w,
                                                      d_mag, d_stats);
        break;
    case 2:
        icd_phase_kernel<2><<<grid, threads, 0, st>>>(g, L, K, d_table, d_view_first, d_views, d_mask, d_x, d_err, d_w,
                                                      d_mag, d_stats);
        break;
    default:
        icd_phase_kernel<3><<<grid, threads, 0, st>>>(g, L, K, d_table, d_view_first, d_views, d_mask, d_x, d_err, d_w,
                                                      d_mag, d_stats);
        break;
    }
}

}  // namespace mbirgpu
