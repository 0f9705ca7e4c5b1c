// Layout conversions and the sparse forward / back projectors.
//
// Forward projection (replaces initErrorSinogam, MBIR_4D/XT_ICD_update.c:651-712,
// and forward_project_voxel_AMat1D, XT_ForwardProject.c:44-61): column-driven,
// FP64 accumulation in an L2-resident FP64 image of the sinogram, rounded to
// float once: e = y - A x (or A x when no y is given). The A value is used
// unscaled, as the reference does here (the voxel update scales it by
// delta_t, XT_VoxUpdate.c:61).
//
// Back projection (the adjoint, A^T s): one warp per (frame, voxel column),
// lanes over detector rows, FP64 accumulation over the frame's views (of FP32
// sums over groups of four views where the records are one 16-byte word),
// then a sum over the z_overlap rows of each voxel slice.
#include "mbir_internal.h"

namespace mbirgpu {

// [N_p][N_t][N_r] (the ABI's [view][row][col]) -> [N_p][N_r][N_t]
__global__ void transpose_rows_cols(const float *__restrict__ in, float *__restrict__ out, int N_t, int N_r)
{
    __shared__ float tile[32][33];
    const size_t base = (size_t)blockIdx.z * N_t * N_r;
    const int r0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int t = t0 + i, r = r0 + threadIdx.x;
        if (t < N_t && r < N_r) tile[i][threadIdx.x] = in[base + (size_t)t * N_r + r];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, t = t0 + threadIdx.x;
        if (t < N_t && r < N_r) out[base + (size_t)r * N_t + t] = tile[threadIdx.x][i];
    }
}

void launch_transpose_sino(const float *in, float *out, int N_p, int N_t, int N_r, cudaStream_t st)
{
    dim3 grid((N_r + 31) / 32, (N_t + 31) / 32, N_p), block(32, 8);
    transpose_rows_cols<<<grid, block, 0, st>>>(in, out, N_t, N_r);
}

void launch_untranspose_sino(const float *in, float *out, int N_p, int N_r, int N_t, cudaStream_t st)
{
    // [N_p][N_r][N_t] -> [N_p][N_t][N_r] is the same transpose with the roles swapped
    dim3 grid((N_t + 31) / 32, (N_r + 31) / 32, N_p), block(32, 8);
    transpose_rows_cols<<<grid, block, 0, st>>>(in, out, N_r, N_t);
}

// [T][Z][Y*X] <-> [T][Y*X][Z]
void launch_vol_to_zfast(const float *in, float *out, int N_time, int N_z, int N_y, int N_x, cudaStream_t st)
{
    const int nxy = N_y * N_x;
    dim3 grid((nxy + 31) / 32, (N_z + 31) / 32, N_time), block(32, 8);
    transpose_rows_cols<<<grid, block, 0, st>>>(in, out, N_z, nxy);
}

void launch_zfast_to_vol(const float *in, float *out, int N_time, int N_z, int N_y, int N_x, cudaStream_t st)
{
    const int nxy = N_y * N_x;
    dim3 grid((N_z + 31) / 32, (nxy + 31) / 32, N_time), block(32, 8);
    transpose_rows_cols<<<grid, block, 0, st>>>(in, out, nxy, N_z);
}

// Tile-accumulated form: a CTA owns a tile of kFpTy x kFpTx voxel columns of
// one frame (and one 32-row chunk); warp w takes the frame's views w, w + 8,
// ... For one view the tile's A entries fall on a narrow band of detector
// channels (at most kFpTx |cos| + kFpTy |sin| + 3 wide), so the warp sums
// every column's a * x into its own FP64 band of kFpBand channels x 32 rows
// in shared memory (lane = detector row: no two lanes share an element, no
// atomics), then adds the band to the FP64 sinogram image with one global
// reduction per nonzero element -- about a seventh of the reductions of one
// per A entry. Entries outside the band (none for these tile sizes) reduce
// straight into the image. Columns whose voxels are all zero are skipped.
constexpr int kFpTx = 8, kFpTy = 4, kFpCols = kFpTx * kFpTy;  // 32 columns: one per lane in the band search
constexpr int kFpBand = 16;                                   // channels of a warp's band
constexpr int kFpWarps = 8;

// KW: 16-byte words per A record (1, 2, 3 for voxel scale 1, 2, 4), so the
// value loop has its compile-time bound 4 KW - 1.
template <int KW>
__global__ void __launch_bounds__(kFpWarps * 32) forward_project_kernel(Geom g, const uint32_t *__restrict__ table,
                                                                       const int32_t *__restrict__ view_first,
                                                                       const float *__restrict__ x,
                                                                       double *__restrict__ acc)
{
    __shared__ double s_band[kFpWarps][kFpBand][32];
    __shared__ double s_x[kFpCols][32];
    const int nxy = g.N_x * g.N_y;
    const int n_chunks = (g.N_t + kRowChunk - 1) / kRowChunk;
    const int tiles_x = (g.N_x + kFpTx - 1) / kFpTx, tiles_y = (g.N_y + kFpTy - 1) / kFpTy;
    long long b = blockIdx.x;
    const int ch = (int)(b % n_chunks);
    b /= n_chunks;
    const int tx = (int)(b % tiles_x);
    b /= tiles_x;
    const int ty = (int)(b % tiles_y);
    const int f = (int)(b / tiles_y);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = ch * kRowChunk + lane;  // this lane's detector row
    const bool row_ok = t < g.N_t;
    // the tile's voxel values, column i = (i / kFpTx, i % kFpTx), as doubles
    int active = 0;  // bit i: column i is in the grid and has a nonzero voxel
    for (int i = warp; i < kFpCols; i += kFpWarps) {
        const int j = ty * kFpTy + i / kFpTx, k = tx * kFpTx + i % kFpTx;
        const bool in = j < g.N_y && k < g.N_x;
        const double xv =
            (in && row_ok) ? (double)__ldg(x + ((size_t)f * nxy + (size_t)j * g.N_x + k) * g.N_z + t / g.z_overlap) : 0.0;
        s_x[i][lane] = xv;
    }
    for (int o = lane; o < kFpBand * 32; o += 32) s_band[warp][o / 32][o % 32] = 0.0;
    __syncthreads();
    for (int i = 0; i < kFpCols; i++) active |= (__any_sync(0xffffffffu, s_x[i][lane] != 0.0) ? 1 : 0) << i;
    if (!active) return;  // uniform: every warp computed the same mask
    const int fv0 = view_first[f], nv = view_first[f + 1] - fv0;
    // lane l: column l of the tile
    const int lj = ty * kFpTy + lane / kFpTx, lk = tx * kFpTx + lane % kFpTx;
    const bool lane_col = ((active >> lane) & 1) != 0;
    const uint32_t *lane_rec = lane_col ? table + ((size_t)fv0 * nxy + ((size_t)lj * g.N_x + lk) * nv) * g.rec_words : nullptr;
    double *band = &s_band[warp][0][0];
    double *my_band = band + lane;
    for (int v = warp; v < nv; v += kFpWarps) {
        // lane l holds column l's record for this view; the band starts at the
        // smallest first sinogram row of the view's entries
        uint4 rw[KW];
#pragma unroll
        for (int k = 0; k < KW; k++) rw[k] = make_uint4(0u, 0u, 0u, 0u);
        if (lane_col) {
            const uint4 *r4 = reinterpret_cast<const uint4 *>(lane_rec + (size_t)v * g.rec_words);
#pragma unroll
            for (int k = 0; k < KW; k++) rw[k] = __ldg(r4 + k);
        }
        const uint32_t hdr = rw[0].x;
        int lo = (hdr >> 24) ? (int)(hdr & 0xFFFFFFu) : 0x7FFFFFFF;
        for (int off = 16; off > 0; off >>= 1) lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, off));
        if (lo == 0x7FFFFFFF) continue;  // no entry of this view in the tile
        int used = 0;                    // band channels touched, as a bit set
        for (int i = 0; i < kFpCols; i++) {
            const uint32_t hi = __shfl_sync(0xffffffffu, hdr, i);
            const int cnt = hi >> 24;
            if (!cnt) continue;  // also the inactive columns (header 0); uniform over the warp
            const int row = (int)(hi & 0xFFFFFFu);
            const double xv = s_x[i][lane];
            const int o0 = row - lo;
#pragma unroll
            for (int q = 0; q < 4 * KW - 1; q++) {  // value q is word 1 + q of column i's record
                if (q < cnt) {
                    const uint4 &u = rw[(1 + q) >> 2];
                    const uint32_t mine = ((1 + q) & 3) == 0 ? u.x : ((1 + q) & 3) == 1 ? u.y : ((1 + q) & 3) == 2 ? u.z : u.w;
                    const double val = xv * (double)__uint_as_float(__shfl_sync(0xffffffffu, mine, i));
                    const int o = o0 + q;
                    if (o < kFpBand) {
                        my_band[o * 32] += val;
                        used |= 1 << o;
                    } else if (row_ok) {
                        atomicAdd(acc + (size_t)(row + q) * g.N_t + t, val);
                    }
                }
            }
        }
        while (used) {
            const int o = __ffs(used) - 1;
            used &= used - 1;
            const double s = my_band[o * 32];
            my_band[o * 32] = 0.0;
            if (row_ok && s != 0.0) atomicAdd(acc + (size_t)(lo + o) * g.N_t + t, s);
        }
    }
}

__global__ void finish_projection_kernel(size_t n, const double *__restrict__ acc, const float *__restrict__ y,
                                         float *__restrict__ out, const float *__restrict__ off, int nrt)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!y) {
            out[i] = (float)acc[i];
        } else {
            const float e = (float)((double)y[i] - acc[i]);
            out[i] = off ? e - off[i % nrt] : e;  // initErrorSinogam, XT_ICD_update.c:689
        }
    }
}

void launch_forward_project(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first,
                            const float *d_x, const float *d_y, double *d_acc, float *d_out, cudaStream_t st,
                            const float *d_off)
{
    const size_t n = (size_t)g.N_p * g.N_r * g.N_t;
    cudaMemsetAsync(d_acc, 0, n * sizeof(double), st);
    const long long blocks = (long long)g.N_time * ((g.N_y + kFpTy - 1) / kFpTy) * ((g.N_x + kFpTx - 1) / kFpTx) *
                             ((g.N_t + kRowChunk - 1) / kRowChunk);
    if (g.rec_words == 4)
        forward_project_kernel<1><<<(unsigned)blocks, kFpWarps * 32, 0, st>>>(g, d_table, d_view_first, d_x, d_acc);
    else if (g.rec_words == 8)
        forward_project_kernel<2><<<(unsigned)blocks, kFpWarps * 32, 0, st>>>(g, d_table, d_view_first, d_x, d_acc);
    else
        forward_project_kernel<3><<<(unsigned)blocks, kFpWarps * 32, 0, st>>>(g, d_table, d_view_first, d_x, d_acc);
    finish_projection_kernel<<<148 * 8, 256, 0, st>>>(n, d_acc, d_y, d_out, d_off, g.N_r * g.N_t);
}

// One warp per (frame, column, chunk of 32 detector rows); out is
// [N_time][N_y][N_x][N_z].
__global__ void back_project_kernel(Geom g, const uint32_t *__restrict__ table,
                                    const int32_t *__restrict__ view_first, const int32_t *__restrict__ views,
                                    const float *__restrict__ sino, float *__restrict__ out)
{
    const int nxy = g.N_x * g.N_y;
    const int n_chunks = (g.N_t + kRowChunk - 1) / kRowChunk;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= (long long)g.N_time * nxy * n_chunks) return;
    const int ch = (int)(gw % n_chunks);
    const long long fc = gw / n_chunks;
    const int f = (int)(fc / nxy), c = (int)(fc - (long long)f * nxy);
    const int t = ch * kRowChunk + lane;  // this lane's detector row
    const int fv0 = view_first[f], nv = view_first[f + 1] - fv0;
    const uint32_t *rec = table + ((size_t)fv0 * nxy + (size_t)c * nv) * g.rec_words;
    double acc = 0.0;
    if (t < g.N_t && g.rec_words == 4) {
        // records of one 16-byte word (header + up to 3 weights): four views'
        // records, then their sinogram entries, in flight at once
        constexpr int U = 4;
        const uint4 *r4 = reinterpret_cast<const uint4 *>(rec);
        for (int v0 = 0; v0 < nv; v0 += U) {
            uint4 R[U];
#pragma unroll
            for (int u = 0; u < U; u++) R[u] = v0 + u < nv ? __ldg(r4 + v0 + u) : make_uint4(0, 0, 0, 0);
            float s[U][3];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int cnt = R[u].x >> 24;
                const float *p = sino + (size_t)(R[u].x & 0xFFFFFFu) * g.N_t + t;
#pragma unroll
                for (int q = 0; q < 3; q++) s[u][q] = q < cnt ? __ldg(p + (size_t)q * g.N_t) : 0.0f;
            }
            // the group's twelve products summed in FP32, the groups in FP64
            // (one conversion per four views instead of six per view)
            float part = 0.0f;
#pragma unroll
            for (int u = 0; u < U; u++)
                part += __uint_as_float(R[u].y) * s[u][0] + __uint_as_float(R[u].z) * s[u][1] +
                        __uint_as_float(R[u].w) * s[u][2];
            acc += (double)part;
        }
    } else if (t < g.N_t) {
        for (int v = 0; v < nv; v++, rec += g.rec_words) {
            const uint32_t hdr = __ldg(rec);
            const int cnt = hdr >> 24, row = hdr & 0xFFFFFF;
            for (int q = 0; q < cnt; q++) {
                const double a = (double)__uint_as_float(__ldg(rec + 1 + q));
                acc += a * (double)__ldg(sino + ((size_t)row + q) * g.N_t + t);
            }
        }
    }
    // rows of one voxel slice are z_overlap consecutive lanes (32 is a multiple of z_overlap)
    for (int off = 1; off < g.z_overlap; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (t < g.N_t && t % g.z_overlap == 0)
        out[((size_t)f * nxy + c) * g.N_z + t / g.z_overlap] = (float)acc;
}

void launch_back_project(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first,
                         const int32_t *d_views, const float *d_sino, float *d_x, cudaStream_t st)
{
    const long long warps = (long long)g.N_time * g.N_x * g.N_y * ((g.N_t + kRowChunk - 1) / kRowChunk);
    const int threads = 256;
    const long long blocks = (warps * 32 + threads - 1) / threads;
    back_project_kernel<<<(unsigned)blocks, threads, 0, st>>>(g, d_table, d_view_first, d_views, d_sino, d_x);
}

}  // namespace mbirgpu
