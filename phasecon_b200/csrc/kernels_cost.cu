// FP64 MAP cost (replaces computeCost, MBIR_4D/XT_ICD_update.c:185-318).
//
// Data term: 1/2 sum w e^2 where |e sqrt(w)| < T, else the generalised-Huber
// branch 2 delta T |e sqrt(w)| + T^2 (1 - 2 delta) (XT_ICD_update.c:192-204);
// the test is made as e^2 w < T^2.
// Prior term: for every voxel the 13 causal spatial pairs (+x; the three +y
// pairs of its slice; the nine pairs of the next slice) and the +t pair, each
// filter weight times the qGGMRF potential |d|^q / sigma^q / (c + |d|^(q-p) /
// sigma^(q-p)) (XT_ICD_update.c:82-90, 206-298). Neighbour differences are
// taken in float as the reference's float - float. The log-variance term is
// zero (variance estimate 1).
//
// Deterministic: every block writes its partial sums, then one block adds the
// partials in a fixed order.
#include "mbir_internal.h"

namespace mbirgpu {

namespace {
constexpr int kCostThreads = 256;
constexpr int kCostBlocks = 148 * 8;
}

int cost_partials_needed(const Geom &) { return 2 * kCostBlocks; }

// qGGMRF potential |d|^q / sq / (c + |d|^(q-p) / sqp) in FP64, with the
// reciprocals of the scale powers precomputed. |d|^(q-p) is exp((q-p) log|d|)
// (relative error a few ulp of double); zero differences cost nothing.
__device__ inline double qg_potential(float d, double q, double qmp, double inv_sq, double inv_sqp, double c)
{
    if (d == 0.0f) return 0.0;
    const double ad = fabs((double)d);
    const double lg = log(ad);
    const double num = (q == 2.0 ? ad * ad : exp(q * lg)) * inv_sq;
    return num / (c + exp(qmp * lg) * inv_sqp);
}

__device__ inline double block_sum(double v, double *sh)
{
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double s = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += sh[i];
    return s;  // valid in thread 0
}

// x is [N_time][N_y][N_x][N_z]
__global__ void __launch_bounds__(kCostThreads) cost_partials_kernel(Geom g, const float *__restrict__ err,
                                                                    const float *__restrict__ w,
                                                                    const float *__restrict__ x,
                                                                    double *__restrict__ partials)
{
    __shared__ double sh[kCostThreads / 32];
    const long long nsino = (long long)g.N_p * g.N_r * g.N_t;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double data = 0;
    const double T2 = g.huber_T * g.huber_T;
    for (long long i = tid; i < nsino; i += stride) {
        // |e sqrt(w)| < T  <=>  e^2 w < T^2; the square root is only needed on the Huber branch
        const double e = (double)err[i], ww = (double)w[i];
        const double t2 = e * e * ww;
        if (t2 < T2) data += t2;
        else data += 2.0 * g.huber_delta * g.huber_T * sqrt(t2) + T2 * (1.0 - 2.0 * g.huber_delta);
    }
    const double qmp = g.q - g.p;
    const double inv_ssq = 1.0 / g.sigma_s_q, inv_ssqp = 1.0 / g.sigma_s_q_p;
    const double inv_stq = 1.0 / g.sigma_t_q, inv_stqp = 1.0 / g.sigma_t_q_p;
    const int NX = g.N_x, NY = g.N_y, NZ = g.N_z, NT = g.N_time;
    const long long nvox = (long long)NT * NY * NX * NZ;
    double prior = 0;
    for (long long i = tid; i < nvox; i += stride) {
        const int z = (int)(i % NZ);
        long long rest = i / NZ;
        const int k = (int)(rest % NX);
        rest /= NX;
        const int j = (int)(rest % NY);
        const int f = (int)(rest / NY);
        const float c = x[i];
        auto X = [&](int ff, int jj, int kk, int zz) -> float {
            return x[(((size_t)ff * NY + jj) * NX + kk) * NZ + zz];
        };
        auto sf = [&](int dz, int dy, int dx) -> double { return g.spatial_filter[dz * 9 + dy * 3 + dx]; };
        auto S = [&](float d) -> double { return qg_potential(d, g.q, qmp, inv_ssq, inv_ssqp, g.c_s); };
        const bool jm = j - 1 >= 0, km = k - 1 >= 0, jp = j + 1 < NY, kp = k + 1 < NX, zp = z + 1 < NZ;
        double acc = 0;
        if (kp) acc += sf(1, 1, 2) * S(c - X(f, j, k + 1, z));
        if (jp) {
            if (km) acc += sf(1, 2, 0) * S(c - X(f, j + 1, k - 1, z));
            acc += sf(1, 2, 1) * S(c - X(f, j + 1, k, z));
            if (kp) acc += sf(1, 2, 2) * S(c - X(f, j + 1, k + 1, z));
        }
        if (zp) {
            for (int dy = -1; dy <= 1; dy++) {
                if ((dy < 0 && !jm) || (dy > 0 && !jp)) continue;
                for (int dx = -1; dx <= 1; dx++) {
                    if ((dx < 0 && !km) || (dx > 0 && !kp)) continue;
                    acc += sf(2, dy + 1, dx + 1) * S(c - X(f, j + dy, k + dx, z + 1));
                }
            }
        }
        if (f + 1 < NT)
            acc += g.time_filter * qg_potential(c - X(f + 1, j, k, z), g.q, qmp, inv_stq, inv_stqp, g.c_t);
        prior += acc;
    }
    const double ds = block_sum(data, sh);
    const double ps = block_sum(prior, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = ds;
        partials[gridDim.x + blockIdx.x] = ps;
    }
}

__global__ void cost_finish_kernel(const double *__restrict__ partials, int nblocks, double *__restrict__ out)
{
    if (threadIdx.x == 0) {
        double d = 0, p = 0;
        for (int i = 0; i < nblocks; i++) {
            d += partials[i];
            p += partials[nblocks + i];
        }
        out[0] = d / 2.0;
        out[1] = p;
    }
}

void launch_cost(const Geom &g, const float *d_err, const float *d_w, const float *d_x, double *d_partials,
                 int n_partials, double *d_out, cudaStream_t st)
{
    const int blocks = n_partials / 2;
    cost_partials_kernel<<<blocks, kCostThreads, 0, st>>>(g, d_err, d_w, d_x, d_partials);
    cost_finish_kernel<<<1, 32, 0, st>>>(d_partials, blocks, d_out);
}

}  // namespace mbirgpu
