// Compressed A-matrix table. One record per (view, voxel column): the first
// detector channel the column projects onto at that view, how many channels
// follow, and their FP32 weights. The weights restate
// calcAMatrixColumnforAngle (MBIR_4D/XT_AMatrix.c:50-110) in double precision.
// This file is compiled with -fmad=false so no multiply-add is fused, which
// keeps every value equal to the reference's (rounded once to float).
//
// Layout: for frame f with views view_first[f] .. view_first[f+1]-1 (nv of
// them), the records of column c are contiguous:
//   record (f, c, v) at  view_first[f]*NXY + c*nv + v      (v = view in frame)
// so the ICD kernel reads one column's views with unit stride.
// Record = rec_words 32-bit words: word 0 = row | count << 24, where row =
// view * N_r + first channel is the record's first sinogram row (so kernels
// need no view lookup), then kmax float weights, zero padded.
#include "mbir_internal.h"

namespace mbirgpu {

__global__ void build_amatrix_kernel(Geom g, const float *__restrict__ Hr, const double *__restrict__ cosv,
                                     const double *__restrict__ sinv, const int32_t *__restrict__ views,
                                     const int32_t *__restrict__ view_first, const int32_t *__restrict__ view_frame,
                                     uint32_t *__restrict__ table, int *__restrict__ err)
{
    const int nxy = g.N_x * g.N_y;
    const long long total = (long long)g.N_p * nxy;
    for (long long rec = blockIdx.x * (long long)blockDim.x + threadIdx.x; rec < total;
         rec += (long long)gridDim.x * blockDim.x) {
        // frame f owns records [view_first[f]*nxy, view_first[f+1]*nxy)
        const int f = view_frame[rec / nxy];
        const int fv0 = view_first[f], nv = view_first[f + 1] - fv0;
        const long long local = rec - (long long)fv0 * nxy;
        const int c = (int)(local / nv);
        const int v = (int)(local - (long long)c * nv);
        const int view = views[fv0 + v];
        const int row = c / g.N_x, col = c - row * g.N_x;
        uint32_t *out = table + rec * g.rec_words;

        const float *h = Hr + (size_t)view * (kRespBins + 1);
        const double x = g.x0 + ((double)col + 0.5) * g.delta_xy;
        const double y = g.y0 + ((double)row + 0.5) * g.delta_xy;
        const double r = x * cosv[view] - y * sinv[view];
        const double rmin = r - g.delta_xy, rmax = r + g.delta_xy;
        int count = 0, first = 0, last = -2;
        float vals[kMaxKmax];
        if (!(rmax < g.R0 || rmin > g.RMax)) {
            int imin = (int)(floor(((rmin - g.R0) / g.delta_r)));
            int imax = (int)(floor((rmax - g.R0) / g.delta_r));
            if (imax >= g.N_r) imax = g.N_r - 1;
            if (imin < 0) imin = 0;
            for (int j = imin; j <= imax; j++) {
                const double center = (g.R0 + (((double)j) + 0.5) * (g.delta_r));
                const double d = fabs(r - center);
                const int bin = (int)(floor((d / g.OffsetR)));
                if (bin >= 0 && bin < kRespBins) {
                    const double w1 = d - bin * g.OffsetR;
                    const double w2 = g.OffsetR - w1;
                    const double f1 = (w2 * (double)h[bin] + w1 * (double)h[bin + 1]) / g.OffsetR;
                    if (f1 > 0) {
                        if (count == 0) first = j;
                        else if (j != last + 1) atomicOr(err, 1);  // non-contiguous channels
                        if (count < g.kmax) vals[count] = (float)f1;
                        else atomicOr(err, 2);  // more channels than the record holds
                        last = j;
                        count++;
                    }
                }
            }
        }
        if (count > g.kmax) count = g.kmax;
        out[0] = (uint32_t)(view * g.N_r + first) | ((uint32_t)count << 24);
        for (int q = 0; q < g.rec_words - 1; q++) out[1 + q] = q < count ? __float_as_uint(vals[q]) : 0u;
    }
}

void launch_build_amatrix(const Geom &g, const float *d_Hr, const double *d_cos, const double *d_sin,
                          const int32_t *d_views, const int32_t *d_view_first, const int32_t *d_view_frame,
                          uint32_t *d_table, int *d_err, cudaStream_t st)
{
    const long long total = (long long)g.N_p * g.N_x * g.N_y;
    const int threads = 256;
    long long blocks = (total + threads - 1) / threads;
    if (blocks > 148LL * 64) blocks = 148LL * 64;
    build_amatrix_kernel<<<(unsigned)blocks, threads, 0, st>>>(g, d_Hr, d_cos, d_sin, d_views, d_view_first,
                                                               d_view_frame, d_table, d_err);
}

// Sum of record counts over voxel columns inside the reconstruction circle:
// the A-matrix nonzeros one sweep visits per voxel slice (before the
// z_overlap factor).
__global__ void count_masked_nnz_kernel(int n_records, int nxy, int rec_words, const int32_t *__restrict__ view_first,
                                        const int32_t *__restrict__ view_frame, const uint8_t *__restrict__ mask,
                                        const uint32_t *__restrict__ table, unsigned long long *__restrict__ out)
{
    unsigned long long acc = 0;
    for (long long rec = blockIdx.x * (long long)blockDim.x + threadIdx.x; rec < (long long)n_records * nxy;
         rec += (long long)gridDim.x * blockDim.x) {
        const int f = view_frame[rec / nxy];
        const int fv0 = view_first[f], nv = view_first[f + 1] - fv0;
        const int c = (int)((rec - (long long)fv0 * nxy) / nv);
        if (mask[c]) acc += table[rec * rec_words] >> 24;
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

void launch_count_masked_nnz(const Geom &g, int n_assigned, const int32_t *d_view_first, const int32_t *d_view_frame,
                             const uint8_t *d_mask, const uint32_t *d_table, unsigned long long *d_out,
                             cudaStream_t st)
{
    const long long total = (long long)n_assigned * g.N_x * g.N_y;
    long long blocks = (total + 255) / 256;
    if (blocks > 148LL * 32) blocks = 148LL * 32;
    if (blocks < 1) blocks = 1;
    count_masked_nnz_kernel<<<(unsigned)blocks, 256, 0, st>>>(n_assigned, g.N_x * g.N_y, g.rec_words, d_view_first,
                                                              d_view_frame, d_mask, d_table, d_out);
}

}  // namespace mbirgpu
