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
// lanes over detector rows, FP64 accumulation over the frame's views, then a
// sum over the z_overlap rows of each voxel slice.
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

// One warp per (frame, voxel column, chunk of 32 detector rows), lane =
// detector row: every A entry of the column adds a * x into an FP64
// accumulator image of the sinogram with a global FP64 reduction
// (red.global.add.f64, performed in L2). Columns whose voxels are all zero are
// skipped.
__global__ void __launch_bounds__(256) forward_project_kernel(Geom g, const uint32_t *__restrict__ table,
                                                             const int32_t *__restrict__ view_first,
                                                             const float *__restrict__ x, double *__restrict__ acc)
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
    const bool row_ok = t < g.N_t;
    const double xv = row_ok ? (double)__ldg(x + ((size_t)f * nxy + c) * g.N_z + t / g.z_overlap) : 0.0;
    if (__all_sync(0xffffffffu, xv == 0.0)) return;
    const int fv0 = view_first[f], nv = view_first[f + 1] - fv0;
    const uint32_t *rec = table + ((size_t)fv0 * nxy + (size_t)c * nv) * g.rec_words;
    if (!row_ok) return;
    constexpr int U = 4;
    for (int v0 = 0; v0 < nv; v0 += U) {
        uint32_t hdr[U];
#pragma unroll
        for (int u = 0; u < U; u++) hdr[u] = v0 + u < nv ? __ldg(rec + (size_t)(v0 + u) * g.rec_words) : 0u;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int cnt = hdr[u] >> 24, row = hdr[u] & 0xFFFFFF;
            const uint32_t *r = rec + (size_t)(v0 + u) * g.rec_words + 1;
            for (int q = 0; q < cnt; q++)
                atomicAdd(acc + (size_t)(row + q) * g.N_t + t, xv * (double)__uint_as_float(__ldg(r + q)));
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
    const long long warps = (long long)g.N_time * g.N_x * g.N_y * ((g.N_t + kRowChunk - 1) / kRowChunk);
    const long long blocks = (warps * 32 + 255) / 256;
    forward_project_kernel<<<(unsigned)blocks, 256, 0, st>>>(g, d_table, d_view_first, d_x, d_acc);
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
#pragma unroll
            for (int u = 0; u < U; u++)
                acc += (double)__uint_as_float(R[u].y) * (double)s[u][0] +
                       (double)__uint_as_float(R[u].z) * (double)s[u][1] +
                       (double)__uint_as_float(R[u].w) * (double)s[u][2];
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
