// Forward projection that allocates nothing: the FP64 sinogram accumulator
// lives in a fixed-size array in the library's own device memory instead of
// a buffer taken from cudaMalloc.
//
// Who needs it: a caller whose device memory is owned by someone else -- a
// framework whose caching allocator has already reserved the free HBM, or a
// service that budgets every byte at start-up -- and a caller inside a
// latency-critical loop that must not let cudaMalloc / cudaFree synchronise
// the device. The other projection entry points take their scratch from
// cudaMalloc (per session or per call), which those callers cannot allow.
//
// Limits and rules of use:
// * the scratch holds kNoallocMaxSinoEntries doubles (16 MiB), so a session
//   qualifies when N_p * N_r * N_t is at most that (180 views x 128 columns x
//   16 rows is 368,640); larger sessions are rejected with an error;
// * the call runs on the device the session was created on: it makes that
//   device current for its duration and restores the caller's current
//   device before it returns, so a caller that has another GPU current still
//   gets this session's scratch, table and stream;
// * the scratch's device address is looked up (cudaGetSymbolAddress, with
//   the session's device current) on the first call on a device, and looked
//   up again on every later call whose stream is not capturing, so a module
//   reloaded after cudaDeviceReset is picked up; a call whose stream is
//   capturing uses the address found by an earlier call on that device and
//   fails if there was none: make the first call before any stream capture;
// * the scratch must be zero where the projection accumulates; every call
//   clears the part it uses on the session's stream before the projection
//   kernel runs, so callers do nothing for it; the output is fully written;
// * there is one scratch per device: two calls in flight at once on the same
//   device (different streams or threads) would add into the same array and
//   corrupt each other's results; order them (same stream, or an event).
#include <mutex>

#include "../../include/mbirgpu.h"
#include "session.h"

namespace mbirgpu {

namespace {

constexpr size_t kNoallocMaxSinoEntries = size_t(1) << 21;  // 2,097,152 doubles = 16 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_acc[kNoallocMaxSinoEntries];

std::mutex g_scratch_mu;
double *g_scratch_ptr[kMaxDevices] = {};

// The forward projector with the object read in the ABI's volume layout
// [N_time][N_z][N_y][N_x] (no conversion pass, so no staging buffer): one warp
// per (frame, voxel column, chunk of 32 detector rows), lane = detector row,
// FP64 reductions into acc.
__global__ void __launch_bounds__(256) forward_project_vol_kernel(Geom g, const uint32_t *__restrict__ table,
                                                                 const int32_t *__restrict__ view_first,
                                                                 const float *__restrict__ vol,
                                                                 double *__restrict__ acc)
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
    const double xv =
        row_ok ? (double)__ldg(vol + ((size_t)f * g.N_z + t / g.z_overlap) * nxy + c) : 0.0;
    if (__all_sync(0xffffffffu, xv == 0.0)) return;
    const int fv0 = view_first[f], nv = view_first[f + 1] - fv0;
    const uint32_t *rec = table + ((size_t)fv0 * nxy + (size_t)c * nv) * g.rec_words;
    if (!row_ok) return;
    for (int v = 0; v < nv; v++, rec += g.rec_words) {
        const uint32_t hdr = __ldg(rec);
        const int cnt = hdr >> 24, row = hdr & 0xFFFFFF;
        for (int q = 0; q < cnt; q++)
            atomicAdd(acc + (size_t)(row + q) * g.N_t + t, xv * (double)__uint_as_float(__ldg(rec + 1 + q)));
    }
}

__global__ void round_accumulator_kernel(size_t n, const double *__restrict__ acc, float *__restrict__ out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (float)acc[i];
}

// Address of device dev's scratch (dev is current). Looked up whenever the
// stream is not capturing -- the module behind the symbol may have been
// reloaded (cudaDeviceReset) since the last call -- and taken from the cache
// of the last lookup while it is.
int scratch_for_device(int dev, cudaStream_t stream, double **out)
{
    if (dev < 0 || dev >= kMaxDevices) return fail("device %d is beyond the %d devices supported", dev, kMaxDevices);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(stream, &cs);
    if (e != cudaSuccess) return fail("cudaStreamIsCapturing failed: %s", cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (cs == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_acc);
        if (e != cudaSuccess)
            return fail("cudaGetSymbolAddress of the projection scratch failed on device %d: %s", dev,
                        cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double *>(p);
    } else if (!g_scratch_ptr[dev]) {
        return fail("forward_project_noalloc: the first call on device %d was made while its stream was capturing; "
                    "make one call before capturing so the scratch address is known",
                    dev);
    }
    *out = g_scratch_ptr[dev];
    return 0;
}

// Makes the session's device current for one call and restores the
// caller's device afterwards.
struct DeviceScope {
    int prev = -1;
    bool switched = false;
    int enter(int dev)
    {
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) return fail("cudaGetDevice failed: %s", cudaGetErrorString(e));
        if (prev != dev) {
            e = cudaSetDevice(dev);
            if (e != cudaSuccess) return fail("cudaSetDevice(%d) failed: %s", dev, cudaGetErrorString(e));
            switched = true;
        }
        return 0;
    }
    ~DeviceScope()
    {
        if (switched) cudaSetDevice(prev);
    }
};

int forward_project_noalloc(Session *s, const float *object_dev, float *sino_dev)
{
    const Geom &g = s->hs.g;
    const size_t n = (size_t)g.N_p * g.N_r * g.N_t;
    if (n > kNoallocMaxSinoEntries)
        return fail("forward_project_noalloc: the sinogram has %zu entries (%d views x %d columns x %d rows); "
                    "the fixed scratch holds at most %zu",
                    n, g.N_p, g.N_r, g.N_t, kNoallocMaxSinoEntries);
    double *acc = nullptr;
    if (scratch_for_device(s->device, s->st, &acc)) return -1;
    cudaError_t e = cudaMemsetAsync(acc, 0, n * sizeof(double), s->st);
    if (e != cudaSuccess) return fail("clearing the projection scratch failed: %s", cudaGetErrorString(e));
    const long long warps = (long long)g.N_time * g.N_x * g.N_y * ((g.N_t + kRowChunk - 1) / kRowChunk);
    const long long blocks = (warps * 32 + 255) / 256;
    forward_project_vol_kernel<<<(unsigned)blocks, 256, 0, s->st>>>(g, s->d_table, s->d_view_first, object_dev, acc);
    round_accumulator_kernel<<<148 * 8, 256, 0, s->st>>>(n, acc, sino_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail("forward_project_noalloc launch failed: %s", cudaGetErrorString(e));
    return 0;
}

}  // namespace

}  // namespace mbirgpu

extern "C" int mbirgpu_session_forward_project_noalloc(mbirgpu_session *sp, const float *object_dev, float *sino_dev)
{
    using namespace mbirgpu;
    if (!sp) return fail("session pointer is NULL");
    if (!object_dev || !sino_dev) return fail("NULL argument");
    Session *s = reinterpret_cast<Session *>(sp);
    DeviceScope scope;
    if (scope.enter(s->device)) return -1;
    return forward_project_noalloc(s, object_dev, sino_dev);
}
