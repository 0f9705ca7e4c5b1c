// Layout conversions and the sparse forward / back projectors.
//
// Forward projection (replaces initErrorSinogam, MBIR_4D/XT_ICD_update.c:651-712,
// and forward_project_voxel_AMat1D, XT_ForwardProject.c:44-61): one CTA per
// (view, detector-channel chunk) keeps an FP64 accumulator for its chunk of the
// view's sinogram row block in shared memory, streams every voxel column of
// the view's frame (one warp per column, one lane per detector row), and adds
// x * a into the channels the column's A record names. The A value is used
// unscaled, as the reference does here (the voxel update scales it by
// delta_t, XT_VoxUpdate.c:61). The result is rounded to float once:
// e = y - A x (or A x when no y is given).
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

namespace {
constexpr int kFwdThreads = 256;
constexpr int kFwdSmemBytes = 96 * 1024;
}  // namespace

// grid: (channel chunks, N_p); dynamic smem: chunk * N_t doubles
__global__ void __launch_bounds__(kFwdThreads) forward_project_kernel(
    Geom g, const uint32_t *__restrict__ table, const int32_t *__restrict__ view_first,
    const int32_t *__restrict__ views, const int32_t *__restrict__ view_frame, const float *__restrict__ x,
    const float *__restrict__ y, float *__restrict__ out, int chunk)
{
    extern __shared__ double acc[];
    const int vi = blockIdx.y;  // position in views[]
    const int f = view_frame[vi];
    const int fv0 = view_first[f], nv = view_first[f + 1] - fv0, v = vi - fv0;
    const int view = views[vi];
    const int r0 = blockIdx.x * chunk, r1 = min(r0 + chunk, g.N_r);
    const int NT = g.N_t, nxy = g.N_x * g.N_y;
    for (int i = threadIdx.x; i < (r1 - r0) * NT; i += blockDim.x) acc[i] = 0.0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int z = lane / g.z_overlap;
    const uint32_t *rec0 = table + ((size_t)fv0 * nxy + v) * g.rec_words;
    const float *xf = x + (size_t)f * nxy * g.N_z;
    for (int c = warp; c < nxy; c += nw) {
        const uint32_t *rec = rec0 + (size_t)c * nv * g.rec_words;
        const uint32_t hdr = __ldg(rec);
        const int cnt = hdr >> 16, first = hdr & 0xFFFF;
        if (cnt == 0 || first + cnt <= r0 || first >= r1) continue;
        if (lane >= NT) continue;
        const double xv = (double)__ldg(xf + (size_t)c * g.N_z + z);
        if (xv == 0.0) continue;
        for (int q = 0; q < cnt; q++) {
            const int r = first + q;
            if (r < r0 || r >= r1) continue;
            const double a = (double)__uint_as_float(__ldg(rec + 1 + q));
            atomicAdd(&acc[(r - r0) * NT + lane], xv * a);
        }
    }
    __syncthreads();
    const size_t obase = ((size_t)view * g.N_r + r0) * NT;
    for (int i = threadIdx.x; i < (r1 - r0) * NT; i += blockDim.x) {
        const double s = acc[i];
        out[obase + i] = y ? (float)((double)y[obase + i] - s) : (float)s;
    }
}

void launch_forward_project(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first,
                            const int32_t *d_views, const int32_t * /*d_view_local*/, const int32_t *d_view_frame,
                            const float *d_x, const float *d_y, float *d_out, cudaStream_t st)
{
    int chunk = kFwdSmemBytes / (int)(sizeof(double) * g.N_t);
    if (chunk > g.N_r) chunk = g.N_r;
    const int nchunks = (g.N_r + chunk - 1) / chunk;
    const size_t smem = (size_t)chunk * g.N_t * sizeof(double);
    cudaFuncSetAttribute(forward_project_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmemBytes);
    dim3 grid(nchunks, g.N_p);
    forward_project_kernel<<<grid, kFwdThreads, smem, st>>>(g, d_table, d_view_first, d_views, d_view_frame, d_x,
                                                             d_y, d_out, chunk);
}

// One warp per (frame, column); out is [N_time][N_y][N_x][N_z].
__global__ void back_project_kernel(Geom g, const uint32_t *__restrict__ table,
                                    const int32_t *__restrict__ view_first, const int32_t *__restrict__ views,
                                    const float *__restrict__ sino, float *__restrict__ out)
{
    const int nxy = g.N_x * g.N_y;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= (long long)g.N_time * nxy) return;
    const int f = (int)(gw / nxy), c = (int)(gw - (long long)f * nxy);
    const int fv0 = view_first[f], nv = view_first[f + 1] - fv0;
    const uint32_t *rec = table + ((size_t)fv0 * nxy + (size_t)c * nv) * g.rec_words;
    double acc = 0.0;
    if (lane < g.N_t) {
        for (int v = 0; v < nv; v++, rec += g.rec_words) {
            const uint32_t hdr = __ldg(rec);
            const int cnt = hdr >> 16, first = hdr & 0xFFFF;
            const int view = views[fv0 + v];
            for (int q = 0; q < cnt; q++) {
                const double a = (double)__uint_as_float(__ldg(rec + 1 + q));
                acc += a * (double)__ldg(sino + ((size_t)view * g.N_r + first + q) * g.N_t + lane);
            }
        }
    }
    for (int off = 1; off < g.z_overlap; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane < g.N_t && lane % g.z_overlap == 0)
        out[((size_t)f * nxy + c) * g.N_z + lane / g.z_overlap] = (float)acc;
}

void launch_back_project(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first,
                         const int32_t *d_views, const float *d_sino, float *d_x, cudaStream_t st)
{
    const long long warps = (long long)g.N_time * g.N_x * g.N_y;
    const int threads = 256;
    const long long blocks = (warps * 32 + threads - 1) / threads;
    back_project_kernel<<<(unsigned)blocks, threads, 0, st>>>(g, d_table, d_view_first, d_views, d_sino, d_x);
}

}  // namespace mbirgpu
