// Batched reconstruction of many independent MBIR problems.
//
// The problems stay resident side by side (one Session each: y, w, e, x and
// the A table); an ICD iteration of all of them is one colour phase after
// another, each phase ONE persistent launch per record class whose CTAs
// drain a queue over the super-voxels of every problem, interleaved in
// proportion to each problem's size (icd_batch_kernel). Problems whose detector-row count is a multiple of 4
// and the others run as two launches of the same phase on two streams, so
// they overlap. Device-side bookkeeping kernels advance the iteration number
// and stop converged problems, so one iteration is a fixed launch sequence:
// it is captured once as a CUDA graph (and a second graph with the periodic
// FP64 refresh of every error sinogram), and a run is a loop of graph
// launches. The super-voxel size and CTA width come from the batch
// autotuner: one measured batched sweep per candidate, scaled by the
// candidate's relative iteration count to convergence.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <memory>
#include <numeric>
#include <vector>

#include "../../include/mbirgpu.h"
#include "session.h"

namespace mbirgpu {

#define BCK(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail("%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

struct Batch {
    std::vector<std::unique_ptr<Session>> m;
    mbirgpu_options opt{};
    cudaStream_t st = nullptr, st2 = nullptr;
    bool own_st = false;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    int sv = 8, warps = 4, colors = 2;
    struct Class {
        int vec = 4;
        std::vector<int> idx;
        BatchDesc *d_desc = nullptr;
        int2 *d_map = nullptr;  // interleaved (problem, item) per queue position
        int map_cap = 0, total = 0;
        int n = 0, grid = 0;
    } cls[2];
    static constexpr int kPhases = 16;  // K x K colours, K <= 4
    unsigned int *d_queue = nullptr;  // [class][phase]
    long long grid_cap(const Class &c, int sv_, int k_);
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // plain iteration, iteration + FP64 refresh
    int iters_run = 0;
    long long graph_launches = 0;
    std::vector<Session::TuneEntry> tune_log;

    ~Batch()
    {
        for (auto &g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto &c : cls) {
            if (c.d_desc) cudaFree(c.d_desc);
            if (c.d_map) cudaFree(c.d_map);
        }
        if (d_queue) cudaFree(d_queue);
        for (cudaEvent_t e : {ev_fork, ev_join, ev_t0, ev_t1})
            if (e) cudaEventDestroy(e);
        m.clear();
        if (st2) cudaStreamDestroy(st2);
        if (own_st && st) cudaStreamDestroy(st);
    }

    int init(const mbirgpu_problem *pbs, int n, const mbirgpu_options *o, void *stream);
    int build_descs();

    void enqueue_iteration(bool refresh);
    int capture();
    int autotune();
    int run(int iterations, mbirgpu_batch_stats *stats);
};

int Batch::init(const mbirgpu_problem *pbs, int n, const mbirgpu_options *o, void *stream)
{
    if (n < 1 || n > kMaxBatch) return fail("a batch holds 1..%d problems (got %d)", kMaxBatch, n);
    opt = o ? *o : current_options();
    if (stream) {
        st = (cudaStream_t)stream;
    } else {
        BCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));  // graphs cannot capture the legacy stream
        own_st = true;
    }
    BCK(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
    BCK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    BCK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    BCK(cudaEventCreate(&ev_t0));
    BCK(cudaEventCreate(&ev_t1));
    mbirgpu_options mo = opt;
    mo.sv_size = 8;  // members skip their own autotuner; the batch tunes once
    mo.cta_warps = 4;
    mo.nhicd_passes = 0;
    for (int i = 0; i < n; i++) {
        std::unique_ptr<Session> s(new (std::nothrow) Session());
        if (!s) return fail("out of host memory");
        if (s->init(&pbs[i], &mo, 1, 1, st)) {
            const std::string why = mbirgpu_last_error();
            return fail("problem %d: %s", i, why.c_str());
        }
        if (s->hs.g.rec_words != 4) return fail("problem %d: batched problems need voxel scale 1", i);
        s->opt = opt;
        m.push_back(std::move(s));
    }
    // record classes: detector rows a multiple of 4 (16-byte lanes) or not
    for (int i = 0; i < n; i++) cls[m[i]->hs.g.N_t % 4 == 0 ? 0 : 1].idx.push_back(i);
    cls[0].vec = 4;
    cls[1].vec = 2;
    for (auto &c : cls) {
        c.n = (int)c.idx.size();
        // longest items first: cost of one SV item ~ views per frame x detector rows
        std::sort(c.idx.begin(), c.idx.end(), [&](int a, int b) {
            const Geom &ga = m[a]->hs.g, &gb = m[b]->hs.g;
            return (long long)ga.max_views * ga.N_t > (long long)gb.max_views * gb.N_t;
        });
        if (c.n) BCK(cudaMalloc((void **)&c.d_desc, c.n * sizeof(BatchDesc)));
    }
    BCK(cudaMalloc((void **)&d_queue, 2 * kPhases * sizeof(unsigned int)));
    sv = opt.sv_size > 0 ? opt.sv_size : 8;
    warps = opt.cta_warps > 0 ? opt.cta_warps : 4;
    colors = opt.sv_colors > 0 ? opt.sv_colors : 2;
    if (autotune()) return -1;
    if (build_descs()) return -1;
    return capture();
}

// Items of one colour phase of each problem (every SV slot of the colour, all frames).
static int phase_items(const Geom &g, int sv, int K) { return g.N_time * sv_slots(g.N_x, g.N_y, sv, K); }

// Descriptors for the current (sv, warps), iteration counters at iters_run,
// all active, and the queue order: each problem's items spread evenly over
// the queue (item k of problem p at position key (k + 0.5) / items_p), so the
// CTAs at work at any moment cover every problem in proportion to its size.
int Batch::build_descs()
{
    for (auto &c : cls) {
        if (!c.n) continue;
        std::vector<BatchDesc> h(c.n);
        std::vector<int> items(c.n);
        for (int a = 0; a < c.n; a++) {
            Session &s = *m[c.idx[a]];
            BatchDesc &d = h[a];
            std::memset(&d, 0, sizeof(d));
            d.g = s.hs.g;
            d.g.N_p = s.n_assigned;
            d.L.sv = sv;
            d.L.n_sv_x = (d.g.N_x + sv - 1) / sv;
            d.L.n_sv_y = (d.g.N_y + sv - 1) / sv;
            d.L.warps = warps;
            d.L.iter = iters_run;
            d.L.zero_skipping = opt.zero_skipping;
            d.L.unroll = 2;
            d.L.seed = opt.seed;
            d.L.colors_k = colors;
            d.L.perm = spread_multiplier(sv_slots(d.g.N_x, d.g.N_y, sv, colors));
            d.K = make_icd_const(s.hs.g);
            d.table = s.d_table;
            d.view_first = s.d_view_first;
            d.mask = s.d_mask;
            d.x = s.d_x;
            d.err = s.d_err;
            d.w = s.d_w;
            d.mag = s.d_mag;
            d.stats = s.d_stats;
            d.convg_thresh = s.convg_thresh;
            d.active = 1;
            items[a] = phase_items(d.g, sv, colors);
        }
        struct Key {
            double key;
            int p, k;
        };
        std::vector<Key> keys;
        for (int a = 0; a < c.n; a++)
            for (int k = 0; k < items[a]; k++) keys.push_back({(k + 0.5) / items[a], a, k});
        std::stable_sort(keys.begin(), keys.end(), [](const Key &x, const Key &y) { return x.key < y.key; });
        std::vector<int2> map(keys.size());
        for (size_t i = 0; i < keys.size(); i++) map[i] = make_int2(keys[i].p, keys[i].k);
        c.total = (int)map.size();
        if (c.total > c.map_cap) {
            if (c.d_map) cudaFree(c.d_map);
            c.d_map = nullptr;
            BCK(cudaMalloc((void **)&c.d_map, c.total * sizeof(int2)));
            c.map_cap = c.total;
        }
        BCK(cudaMemcpyAsync(c.d_desc, h.data(), c.n * sizeof(BatchDesc), cudaMemcpyHostToDevice, st));
        BCK(cudaMemcpyAsync(c.d_map, map.data(), c.total * sizeof(int2), cudaMemcpyHostToDevice, st));
        c.grid = (int)std::min<long long>(batch_grid(c.vec, warps), grid_cap(c, sv, colors));
    }
    BCK(cudaStreamSynchronize(st));
    return 0;
}

// Largest grid for which every problem of a class stays within its
// concurrent-update bound (sv_max_concurrent): a problem's share of the CTAs
// at work follows its share of the work -- items are interleaved in
// proportion to their count, and an item's duration grows with views x
// detector rows.
long long Batch::grid_cap(const Class &c, int sv_, int k_)
{
    double total = 0;
    for (int a = 0; a < c.n; a++) {
        const Geom &g = m[c.idx[a]]->hs.g;
        total += (double)phase_items(g, sv_, k_) * g.max_views * g.N_t;
    }
    double cap = 1e18;
    for (int a = 0; a < c.n; a++) {
        const Geom &g = m[c.idx[a]]->hs.g;
        const double share = (double)phase_items(g, sv_, k_) * g.max_views * g.N_t / std::max(1.0, total);
        cap = std::min(cap, (double)sv_max_concurrent(g.N_x, g.N_y, g.N_time, sv_, k_) / std::max(share, 1e-12));
    }
    return std::max(1LL, (long long)cap);
}

// One iteration of every active problem: begin, K^2 colour phases (the two
// classes of a phase on two streams), end, and optionally the FP64 refresh.
void Batch::enqueue_iteration(bool refresh)
{
    for (auto &c : cls)
        if (c.n) launch_batch_begin(c.d_desc, c.n, st);
    cudaMemsetAsync(d_queue, 0, 2 * kPhases * sizeof(unsigned int), st);
    for (int ph = 0; ph < colors * colors; ph++) {
        const bool both = cls[0].n && cls[1].n;
        if (both) {
            cudaEventRecord(ev_fork, st);
            cudaStreamWaitEvent(st2, ev_fork, 0);
        }
        if (cls[0].n)
            launch_icd_batch(4, warps, cls[0].grid, cls[0].d_desc, cls[0].d_map, cls[0].total, ph, d_queue + ph, st);
        if (cls[1].n)
            launch_icd_batch(2, warps, cls[1].grid, cls[1].d_desc, cls[1].d_map, cls[1].total, ph,
                             d_queue + kPhases + ph, both ? st2 : st);
        if (both) {
            cudaEventRecord(ev_join, st2);
            cudaStreamWaitEvent(st, ev_join, 0);
        }
    }
    for (auto &c : cls)
        if (c.n) launch_batch_end(c.d_desc, c.n, st);
    if (refresh)
        for (auto &s : m) launch_forward_project(s->hs.g, s->d_table, s->d_view_first, s->d_x, s->d_y, s->d_acc,
                                                 s->d_err, st);
}

int Batch::capture()
{
    for (int r = 0; r < 2; r++) {
        if (graph[r]) {
            cudaGraphExecDestroy(graph[r]);
            graph[r] = nullptr;
        }
        cudaGraph_t g = nullptr;
        BCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        enqueue_iteration(r == 1);
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess) return fail("capturing the batch iteration failed: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&graph[r], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail("instantiating the batch graph failed: %s", cudaGetErrorString(e));
    }
    return 0;
}

// Candidates (sv, K) in {(4, 2), (4, 4), (8, 2), (8, 4), (16, 2)} x warps in
// {2, 4}, each with its grid capped (grid_cap): one timed batched sweep each on
// the current state (snapshotted and restored), scaled by the relative iterations
// to convergence of the candidate's same-colour spacing. User-fixed sv_size /
// cta_warps / sv_colors restrict the search.
int Batch::autotune()
{
    if (opt.sv_size > 0 && opt.cta_warps > 0 && opt.sv_colors > 0) return 0;
    for (auto &s : m) {
        BCK(cudaMemcpyAsync(s->d_tmp, s->d_x, s->n_vox * sizeof(float), cudaMemcpyDeviceToDevice, st));
        BCK(cudaMemcpyAsync(s->d_acc, s->d_err, s->n_sino * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    const int cand[5][2] = {{4, 2}, {4, 4}, {8, 2}, {8, 4}, {16, 2}};
    const int ws[2] = {2, 4};
    auto allowed = [&](int a, int b) {
        return !(opt.sv_size > 0 && cand[a][0] != opt.sv_size) && !(opt.sv_colors > 0 && cand[a][1] != opt.sv_colors) &&
               !(opt.cta_warps > 0 && ws[b] != opt.cta_warps);
    };
    double best = 1e300;
    int best_sv = sv, best_w = warps, best_k = colors;
    for (int a = 0; a < 5; a++) {
        for (int b = 0; b < 2; b++) {
            if (!allowed(a, b)) continue;
            sv = cand[a][0];
            colors = cand[a][1];
            warps = ws[b];
            if (build_descs()) return -1;
            BCK(cudaEventRecord(ev_t0, st));
            enqueue_iteration(false);
            BCK(cudaEventRecord(ev_t1, st));
            BCK(cudaGetLastError());
            BCK(cudaEventSynchronize(ev_t1));
            float ms = 0;
            BCK(cudaEventElapsedTime(&ms, ev_t0, ev_t1));
            tune_log.push_back({sv, warps, ms});
            const double est = ms * sv_convergence_factor(sv, colors);
            if (est < best) {
                best = est;
                best_sv = sv;
                best_w = warps;
                best_k = colors;
            }
            for (auto &s : m) {
                BCK(cudaMemcpyAsync(s->d_x, s->d_tmp, s->n_vox * sizeof(float), cudaMemcpyDeviceToDevice, st));
                BCK(cudaMemcpyAsync(s->d_err, s->d_acc, s->n_sino * sizeof(float), cudaMemcpyDeviceToDevice, st));
            }
        }
    }
    sv = best_sv;
    warps = best_w;
    colors = best_k;
    for (auto &s : m) {
        const Geom &g = s->hs.g;
        BCK(cudaMemsetAsync(s->d_mag, 0, (size_t)g.N_time * g.N_x * g.N_y * sizeof(float), st));
    }
    BCK(cudaStreamSynchronize(st));
    return 0;
}

int Batch::run(int iterations, mbirgpu_batch_stats *stats)
{
    BCK(cudaEventRecord(ev_t0, st));
    int launched = 0;
    for (int it = 0; it < iterations; it++) {
        const int k = iters_run + it + 1;
        const bool refresh = opt.refresh_every > 0 && k % opt.refresh_every == 0;
        BCK(cudaGraphLaunch(graph[refresh ? 1 : 0], st));
        launched++;
    }
    BCK(cudaEventRecord(ev_t1, st));
    BCK(cudaEventSynchronize(ev_t1));
    iters_run += iterations;
    graph_launches += launched;
    float ms = 0;
    BCK(cudaEventElapsedTime(&ms, ev_t0, ev_t1));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        long long upd = 0;
        int conv = 0;
        for (auto &c : cls) {
            if (!c.n) continue;
            std::vector<BatchDesc> h(c.n);
            BCK(cudaMemcpy(h.data(), c.d_desc, c.n * sizeof(BatchDesc), cudaMemcpyDeviceToHost));
            for (auto &d : h) {
                upd += (long long)d.total_updates;
                conv += !d.active;
            }
        }
        stats->voxel_updates = upd;
        stats->device_ms = ms;
        stats->graph_launches = launched;
        stats->kernel_launches_per_iteration =
            (cls[0].n ? 2 : 0) + (cls[1].n ? 2 : 0) + colors * colors * ((cls[0].n ? 1 : 0) + (cls[1].n ? 1 : 0));
        stats->problems_converged = conv;
        stats->sv_size = sv;
        stats->cta_warps = warps;
        stats->sv_colors = colors;
    }
    return 0;
}

}  // namespace mbirgpu

using mbirgpu::Batch;
using mbirgpu::fail;

#define BATCH(bp)                                    \
    if (!(bp)) return fail("batch pointer is NULL"); \
    Batch *b = reinterpret_cast<Batch *>(bp)

extern "C" {

int mbirgpu_batch_create(mbirgpu_batch **out, const mbirgpu_problem *problems, int32_t n,
                         const mbirgpu_options *opt, void *stream)
{
    if (!out || !problems) return fail("NULL argument");
    *out = nullptr;
    Batch *b = new (std::nothrow) Batch();
    if (!b) return fail("out of host memory");
    if (b->init(problems, n, opt, stream)) {
        std::string keep = mbirgpu_last_error();
        delete b;
        fail("%s", keep.c_str());
        return -1;
    }
    *out = reinterpret_cast<mbirgpu_batch *>(b);
    return 0;
}

int mbirgpu_batch_destroy(mbirgpu_batch *bp)
{
    delete reinterpret_cast<Batch *>(bp);
    return 0;
}

int mbirgpu_batch_run(mbirgpu_batch *bp, int32_t iterations, mbirgpu_batch_stats *stats)
{
    BATCH(bp);
    if (iterations < 0) return fail("iterations must be >= 0");
    return b->run(iterations, stats);
}

int mbirgpu_batch_problem_info(mbirgpu_batch *bp, int32_t i, mbirgpu_session_info *info, int32_t *iterations,
                               int32_t *converged)
{
    BATCH(bp);
    if (i < 0 || i >= (int)b->m.size()) return fail("problem index %d out of range", i);
    if (info && mbirgpu_session_info_get(reinterpret_cast<mbirgpu_session *>(b->m[i].get()), info)) return -1;
    if (iterations || converged) {
        for (auto &c : b->cls)
            for (int a = 0; a < c.n; a++)
                if (c.idx[a] == i) {
                    mbirgpu::BatchDesc d;
                    cudaError_t e = cudaMemcpy(&d, c.d_desc + a, sizeof(d), cudaMemcpyDeviceToHost);
                    if (e != cudaSuccess) return fail("reading the batch state failed: %s", cudaGetErrorString(e));
                    if (iterations) *iterations = d.iters_done;
                    if (converged) *converged = !d.active;
                }
    }
    return 0;
}

int mbirgpu_batch_get_object(mbirgpu_batch *bp, int32_t i, float *object)
{
    BATCH(bp);
    if (i < 0 || i >= (int)b->m.size()) return fail("problem index %d out of range", i);
    if (!object) return fail("NULL object");
    return b->m[i]->get_object(object);
}

int mbirgpu_batch_cost(mbirgpu_batch *bp, int32_t i, double *total)
{
    BATCH(bp);
    if (i < 0 || i >= (int)b->m.size()) return fail("problem index %d out of range", i);
    return b->m[i]->cost(total, nullptr, nullptr);
}

int mbirgpu_reconstruct_batch(float **objects, const mbirgpu_problem *problems, int32_t n, int32_t iterations)
{
    if (!objects || !problems) return fail("NULL argument");
    for (int i = 0; i < n; i++) objects[i] = nullptr;
    mbirgpu_batch *bp = nullptr;
    if (mbirgpu_batch_create(&bp, problems, n, nullptr, nullptr)) return -1;
    Batch *b = reinterpret_cast<Batch *>(bp);
    int rc = b->run(iterations, nullptr);
    for (int i = 0; i < n && !rc; i++) {
        const mbirgpu::Geom &g = b->m[i]->hs.g;
        const size_t slab = (size_t)g.N_y * g.N_x;
        std::vector<float> vol((size_t)g.N_time * g.N_z * slab);
        rc = b->m[i]->get_object(vol.data());
        if (rc) break;
        // the reference's layout: [N_time][N_z + 2][N_y][N_x] with zero halo slices
        float *out = (float *)std::calloc((size_t)g.N_time * (g.N_z + 2) * slab, sizeof(float));
        if (!out) {
            rc = fail("out of host memory");
            break;
        }
        for (int t = 0; t < g.N_time; t++)
            std::memcpy(out + ((size_t)t * (g.N_z + 2) + 1) * slab, vol.data() + (size_t)t * g.N_z * slab,
                        (size_t)g.N_z * slab * sizeof(float));
        objects[i] = out;
    }
    if (rc)
        for (int i = 0; i < n; i++) {
            std::free(objects[i]);
            objects[i] = nullptr;
        }
    mbirgpu_batch_destroy(bp);
    return rc;
}

}  // extern "C"
