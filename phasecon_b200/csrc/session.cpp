// Session layer of libmbirgpu: one stage of one problem resident in GPU
// memory, and the C ABI functions declared in include/mbirgpu.h that act on it.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mbirgpu.h"
#include "mbir_internal.h"
#include "session.h"

namespace mbirgpu {

thread_local std::string g_last_error;

int fail(const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return -1;
}

namespace {
std::mutex g_opt_mu;
mbirgpu_options g_opt;
bool g_opt_init = false;
}  // namespace

mbirgpu_options current_options()
{
    std::lock_guard<std::mutex> lk(g_opt_mu);
    if (!g_opt_init) {
        mbirgpu_default_options(&g_opt);
        g_opt_init = true;
    }
    return g_opt;
}

#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail("%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
static int dalloc(T **p, size_t n, size_t *acc)
{
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) return fail("cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
    *acc += n * sizeof(T);
    return 0;
}

Session::~Session()
{
    void *ptrs[] = {d_y, d_w, d_err, d_x, d_tmp, d_table, d_Hr, d_cos, d_sin, d_views, d_view_first, d_view_frame,
                    d_mask, d_mag, d_stats, d_cost_partials, d_cost_out, d_flag, d_acc, d_queue, d_filt, d_sel,
                    d_nh_items, d_nh_n, d_nh_scratch, d_nh_selstate, d_off, d_offx, d_onum, d_olam, d_ogamma,
                    d_var};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (auto &ev : ev_pairs) {
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    drop_graphs();
    if (d_iter) cudaFree(d_iter);
}

void Session::drop_graphs()
{
    for (auto &row : graphs)
        for (auto &ge : row)
            if (ge) {
                cudaGraphExecDestroy(ge);
                ge = nullptr;
            }
    for (auto &row : graph_seen)
        for (int &n : row) n = 0;
}

// An iteration is replayed from a CUDA graph when its launches depend on
// nothing the host decides during the iteration: a stream of the session's
// own (the legacy default stream cannot be captured), no ring correction (its
// offset updates interleave with the phases; kept on direct launches), no
// variance re-estimation (it reads a value back to the host), and no
// schedule measurement in progress.
bool Session::graph_ok() const
{
    return opt.graph_iterations && st != nullptr && !rings && !update_var && !tuning;
}

int Session::init(const mbirgpu_problem *pb, const mbirgpu_options *o, int mult_xy, int mult_z, void *stream)
{
    opt = o ? *o : current_options();
    st = (cudaStream_t)stream;
    CK(cudaGetDevice(&device));
    ProblemDesc pd{};
    pd.proj_rows = pb->proj_rows;
    pd.proj_cols = pb->proj_cols;
    pd.proj_num = pb->proj_num;
    pd.recon_num = pb->recon_num;
    pd.vox_wid = pb->vox_wid;
    pd.rot_center = pb->rot_center;
    pd.sig_s = pb->sig_s;
    pd.sig_t = pb->sig_t;
    pd.c_s = pb->c_s;
    pd.c_t = pb->c_t;
    pd.quad_convex = pb->quad_convex;
    pd.huber_delta = pb->huber_delta;
    pd.huber_T = pb->huber_T;
    pd.mrf_p = opt.mrf_p;
    pd.mrf_q = opt.mrf_q;
    pd.alpha = opt.alpha;
    convg_thresh = pb->convg_thresh;
    std::string msg = build_setup(hs, pd, pb->proj_angles, pb->proj_times, pb->recon_times, mult_xy, mult_z);
    if (!msg.empty()) return fail("%s", msg.c_str());
    const Geom &g = hs.g;
    for (int f = 0; f < g.N_time; f++)
        if (hs.view_first[f + 1] == hs.view_first[f])
            return fail("Time frame %d has no projection views.", f);

    n_sino = (size_t)g.N_p * g.N_r * g.N_t;
    n_vox = (size_t)g.N_time * g.N_y * g.N_x * g.N_z;
    const size_t nxy = (size_t)g.N_x * g.N_y;
    const size_t table_words = (size_t)g.N_p * nxy * g.rec_words;
    size_t &acc = device_bytes;
    if (dalloc(&d_y, n_sino, &acc) || dalloc(&d_w, n_sino, &acc) || dalloc(&d_err, n_sino, &acc) ||
        dalloc(&d_x, n_vox, &acc) || dalloc(&d_tmp, std::max(n_sino, n_vox), &acc) ||
        dalloc(&d_table, table_words, &acc) || dalloc(&d_Hr, hs.H_r.size(), &acc) ||
        dalloc(&d_cos, (size_t)g.N_p, &acc) || dalloc(&d_sin, (size_t)g.N_p, &acc) ||
        dalloc(&d_views, (size_t)g.N_p, &acc) || dalloc(&d_view_first, (size_t)g.N_time + 1, &acc) ||
        dalloc(&d_view_frame, (size_t)g.N_p, &acc) || dalloc(&d_mask, nxy, &acc) ||
        dalloc(&d_mag, (size_t)g.N_time * nxy, &acc) || dalloc(&d_stats, 1, &acc) ||
        dalloc(&d_cost_partials, (size_t)cost_partials_needed(g), &acc) || dalloc(&d_cost_out, 2, &acc) ||
        dalloc(&d_flag, 1, &acc) || dalloc(&d_acc, n_sino, &acc) || dalloc(&d_queue, kQueueCounters, &acc))
        return -1;
    if (opt.nhicd_passes > 0 &&
        (dalloc(&d_filt, (size_t)g.N_time * nxy, &acc) || dalloc(&d_sel, (size_t)g.N_time * nxy, &acc)))
        return -1;
    if (opt.nhicd_passes > 0) {
        // work lists for any NH schedule: the smallest super-voxels need the most
        for (int K : {2, 4}) {
            nh_items_cap = std::max(nh_items_cap, (size_t)K * K * nh_items_per_phase(g.N_time, g.N_y, g.N_x, 1, K));
            for (int sv = 1; sv <= 16; sv *= 2)
                nh_scratch_cap = std::max(nh_scratch_cap, nh_items_scratch_ints(g.N_time, g.N_y, g.N_x, sv, K));
        }
        if (dalloc(&d_nh_items, nh_items_cap, &acc) || dalloc(&d_nh_n, (size_t)kMaxPhases, &acc) ||
            dalloc(&d_nh_scratch, nh_scratch_cap, &acc) ||
            dalloc(&d_nh_selstate, (nh_select_scratch_bytes(g.N_time) + 7) / 8, &acc))
            return -1;
    }

    // views not assigned to any frame keep no A records; frame map for the builder
    std::vector<int32_t> view_frame(g.N_p, 0);
    for (int f = 0; f < g.N_time; f++)
        for (int i = hs.view_first[f]; i < hs.view_first[f + 1]; i++) view_frame[i] = f;
    n_assigned = hs.view_first[g.N_time];

    CK(cudaMemcpyAsync(d_Hr, hs.H_r.data(), hs.H_r.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_cos, hs.cosv.data(), g.N_p * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_sin, hs.sinv.data(), g.N_p * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d_views, 0, g.N_p * sizeof(int32_t), st));
    if (n_assigned)
        CK(cudaMemcpyAsync(d_views, hs.views.data(), n_assigned * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_view_first, hs.view_first.data(), (g.N_time + 1) * sizeof(int32_t), cudaMemcpyHostToDevice,
                       st));
    CK(cudaMemcpyAsync(d_view_frame, view_frame.data(), g.N_p * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_mask, hs.mask.data(), nxy, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d_flag, 0, sizeof(int), st));
    CK(cudaMemsetAsync(d_table, 0, table_words * sizeof(uint32_t), st));

    // measurements: [view][row][col] -> [view][col][row]
    CK(cudaMemcpyAsync(d_tmp, pb->projections, n_sino * sizeof(float), cudaMemcpyHostToDevice, st));
    launch_transpose_sino(d_tmp, d_y, g.N_p, g.N_t, g.N_r, st);
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpyAsync(d_tmp, pb->weights, n_sino * sizeof(float), cudaMemcpyHostToDevice, st));
    launch_transpose_sino(d_tmp, d_w, g.N_p, g.N_t, g.N_r, st);

    // A table over the assigned views (records of view position i in views[])
    Geom gb = g;
    gb.N_p = n_assigned;
    if (n_assigned) launch_build_amatrix(gb, d_Hr, d_cos, d_sin, d_views, d_view_first, d_view_frame, d_table, d_flag, st);
    CK(cudaGetLastError());
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (flag) return fail("A-matrix build: a voxel column hit %s detector channels.",
                          (flag & 2) ? "more than the record holds" : "non-contiguous");

    // A nonzeros over the columns a sweep visits (for the roofline's byte count)
    CK(cudaMemsetAsync(d_stats, 0, sizeof(IcdStats), st));
    if (n_assigned)
        launch_count_masked_nnz(g, n_assigned, d_view_first, d_view_frame, d_mask, d_table, &d_stats->updates, st);
    unsigned long long nnz = 0;
    CK(cudaMemcpyAsync(&nnz, &d_stats->updates, sizeof(nnz), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    masked_nnz = (int64_t)nnz;
    CK(cudaMemsetAsync(d_x, 0, n_vox * sizeof(float), st));
    CK(cudaMemsetAsync(d_mag, 0, (size_t)g.N_time * nxy * sizeof(float), st));
    masked_columns = 0;
    for (uint8_t m : hs.mask) masked_columns += m;
    masked_columns *= g.N_time;
    choose_schedule();
    if (refresh_error()) return -1;
    return autotune();
}
// Default schedule, a function of the problem's shape only (autotune = 0):
// 4 x 4 super-voxels in K = 2 colours (the 4-D workload's measured best,
// and the concurrency cap sv_max_concurrent keeps it convergent on any
// frame size), 4 warps per column when a frame has at least 64 views to
// split over them, else 2. Fields the user fixed are kept.
void Session::choose_schedule()
{
    const Geom &g = hs.g;
    sv = opt.sv_size > 0 ? std::min(opt.sv_size, 16) : 4;
    colors = opt.sv_colors > 0 ? opt.sv_colors : 2;
    warps = opt.cta_warps > 0 ? std::min(opt.cta_warps, 8) : (g.max_views >= 64 ? 4 : 2);
    sync_nh_schedule();
}

// Schedule autotuner (opt-in, autotune = 1). Candidates: (super-voxel edge sv, colours K) in
// {(4, 2), (4, 4), (8, 2), (8, 4), (16, 2)} and warps per CTA in {2, 4}, each
// with its grid capped at sv_max_concurrent CTAs. Each candidate runs one
// iteration as the run will (the second one when non-homogeneous passes are
// on) on the current state (snapshotted and restored afterwards);
// its time is scaled by the relative number of iterations its same-colour
// spacing needs to converge (sv_convergence_factor). The smallest estimated
// time to convergence wins. User-fixed sv_size / cta_warps / sv_colors
// restrict the search; with all three fixed there is none. The result
// depends on measured times, so two runs on the same inputs can pick
// different schedules and end on (equally converged) different images.

// Schedule of the non-homogeneous passes: the user's, else the full sweep's
// super-voxels and colours with twice its warps per column (up to 8). Those
// passes are bound by chains of column updates inside the few super-voxels
// that hold many selected columns, so a shorter time per column pays more
// than the occupancy the wider CTAs cost (4-D workload: 18.6 ms per
// iteration with 8 warps against 20.6 ms with 4).
void Session::sync_nh_schedule()
{
    nh_sv = opt.nh_sv_size > 0 ? std::min(opt.nh_sv_size, 16) : sv;
    nh_colors = opt.nh_sv_colors > 0 ? opt.nh_sv_colors : colors;
    nh_warps = opt.nh_cta_warps > 0 ? std::min(opt.nh_cta_warps, 8) : std::min(8, 2 * warps);
}

int Session::autotune()
{
    if (!opt.autotune) return 0;
    if (opt.sv_size > 0 && opt.cta_warps > 0 && opt.sv_colors > 0) return 0;
    const Geom &g = hs.g;
    // snapshot x and e into the scratch buffers (d_tmp holds a volume, d_acc a sinogram)
    CK(cudaMemcpyAsync(d_tmp, d_x, n_vox * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(d_acc, d_err, n_sino * sizeof(float), cudaMemcpyDeviceToDevice, st));
    const bool save_timing = timing;
    timing = true;
    tuning = true;
    const int cand[5][2] = {{4, 2}, {4, 4}, {8, 2}, {8, 4}, {16, 2}};
    const int ws[2] = {2, 4};
    auto allowed = [&](int a, int b) {
        if (opt.sv_size > 0 && cand[a][0] != opt.sv_size) return false;
        if (opt.sv_colors > 0 && cand[a][1] != opt.sv_colors) return false;
        if (opt.cta_warps > 0 && ws[b] != opt.cta_warps) return false;
        return cand[a][0] <= std::max(g.N_x, g.N_y);
    };
    double best = 1e300;
    int best_sv = sv, best_w = warps, best_k = colors;
    for (int a = 0; a < 5; a++) {
        for (int b = 0; b < 2; b++) {
            if (!allowed(a, b)) continue;
            sv = cand[a][0];
            colors = cand[a][1];
            warps = ws[b];
            sync_nh_schedule();
            // time a full iteration as the run will do it: with non-homogeneous
            // passes that is iteration 2 (they start there), after iteration 1
            mbirgpu_iter_stats st_;
            const int saved_refresh = opt.refresh_every;
            opt.refresh_every = 0;
            int rc = icd_iteration(1, &st_);
            if (!rc && opt.nhicd_passes > 0 && d_sel) rc = icd_iteration(2, &st_);
            opt.refresh_every = saved_refresh;
            if (rc) return -1;
            const double est = st_.kernel_ms * sv_convergence_factor(sv, colors);
            tune_log.push_back({sv, warps, st_.kernel_ms});
            if (est < best) {
                best = est;
                best_sv = sv;
                best_w = warps;
                best_k = colors;
            }
            CK(cudaMemcpyAsync(d_x, d_tmp, n_vox * sizeof(float), cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(d_err, d_acc, n_sino * sizeof(float), cudaMemcpyDeviceToDevice, st));
        }
    }
    timing = save_timing;
    tuning = false;
    drop_graphs();
    sv = best_sv;
    warps = best_w;
    colors = best_k;
    sync_nh_schedule();
    CK(cudaMemsetAsync(d_mag, 0, (size_t)g.N_time * g.N_x * g.N_y * sizeof(float), st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

int Session::refresh_error()
{
    // views outside every frame keep e = y (they never enter the problem)
    launch_forward_project(hs.g, d_table, d_view_first, d_x, d_y, d_acc, d_err, st, rings ? d_off : nullptr);
    CK(cudaGetLastError());
    return 0;
}

int Session::set_object(const float *obj)
{
    const Geom &g = hs.g;
    CK(cudaMemcpyAsync(d_tmp, obj, n_vox * sizeof(float), cudaMemcpyHostToDevice, st));
    launch_vol_to_zfast(d_tmp, d_x, g.N_time, g.N_z, g.N_y, g.N_x, st);
    CK(cudaGetLastError());
    return refresh_error();
}

int Session::get_object(float *obj)
{
    const Geom &g = hs.g;
    launch_zfast_to_vol(d_x, d_tmp, g.N_time, g.N_z, g.N_y, g.N_x, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(obj, d_tmp, n_vox * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

int Session::cost(double *total, double *data, double *prior)
{
    const Geom &g = hs.g;
    launch_cost(g, d_err, d_w, d_x, d_cost_partials, cost_partials_needed(g), d_cost_out, st);
    CK(cudaGetLastError());
    double h[2];
    CK(cudaMemcpyAsync(h, d_cost_out, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // the variance's normalisation N log(var) / 2 (XT_ICD_update.c:307); 0 while var = 1
    const double lognorm = (double)g.N_p * g.N_r * g.N_t * std::log(var_est) / 2;
    if (data) *data = h[0] + lognorm;
    if (prior) *prior = h[1];
    if (total) *total = h[0] + lognorm + h[1];
    return 0;
}

// Every launch of one ICD iteration on the session's stream (memsets, the
// full-sweep colour phases, the non-homogeneous passes, the periodic FP64
// refresh). graph_mode: the kernels read the iteration number from d_iter and
// the timing events are recorded as graph nodes.
int Session::enqueue_iteration(int iter, bool graph_mode, int *launches_out)
{
    const Geom &g = hs.g;
    CK(cudaMemsetAsync(d_stats, 0, sizeof(IcdStats), st));
    CK(cudaMemsetAsync(d_queue, 0, kQueueCounters * sizeof(unsigned int), st));
    IcdLaunch L{};
    L.sv = sv;
    L.n_sv_x = (g.N_x + sv - 1) / sv;
    L.n_sv_y = (g.N_y + sv - 1) / sv;
    L.warps = warps;
    L.iter = iter;
    L.iter_dev = graph_mode ? d_iter : nullptr;
    L.zero_skipping = opt.zero_skipping;
    L.unroll = opt.icd_unroll > 0 ? opt.icd_unroll : 4;
    L.seed = opt.seed;
    L.colors_k = colors;
    L.perm = spread_multiplier(sv_slots(g.N_x, g.N_y, sv, colors));
    L.max_ctas = sv_max_concurrent(g.N_x, g.N_y, g.N_time, sv, colors);
    L.stage_records = opt.stage_records;
    const int phases = colors * colors;
    Geom gb = g;
    gb.N_p = n_assigned;
    auto record = [&](cudaEvent_t e) -> cudaError_t {
        return graph_mode ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal) : cudaEventRecord(e, st);
    };
    if (timing) CK(record(ev_pairs[0].first));
    for (int ph = 0; ph < phases; ph++) {
        L.phase = ph;
        launch_icd_phase(gb, L, d_table, d_view_first, d_mask, d_x, d_err, d_w, d_mag, d_stats, d_queue + ph, st);
        if (rings && update_offset()) return -1;
    }
    if (timing) CK(record(ev_pairs[0].second));
    int launches = phases;
    // non-homogeneous passes (the reference's NH-ICD, from iteration 2): each
    // re-updates the k columns per frame with the largest filtered update
    // magnitude, k = masked columns / NHICD_Iterations (XT_NHICD.c:176)
    const int nh = (d_sel && iter > 1) ? std::min(opt.nhicd_passes, kMaxNhPasses) : 0;
    if (nh > 0 && timing) CK(record(ev_pairs[1].first));
    for (int pass = 0; pass < nh; pass++) {
        const int k = (int)(masked_columns / std::max(1, g.N_time)) / kNhicdIterations;
        launch_nh_select(g.N_time, g.N_y, g.N_x, d_mag, d_mask, k, d_filt, d_sel, st, d_nh_selstate);
        IcdLaunch Ln = L;
        Ln.sel = d_sel;
        Ln.seed = L.seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(pass + 1));
        Ln.sv = nh_sv;
        Ln.n_sv_x = (g.N_x + nh_sv - 1) / nh_sv;
        Ln.n_sv_y = (g.N_y + nh_sv - 1) / nh_sv;
        Ln.colors_k = nh_colors;
        Ln.warps = nh_warps;
        Ln.perm = spread_multiplier(sv_slots(g.N_x, g.N_y, nh_sv, nh_colors));
        Ln.max_ctas = sv_max_concurrent(g.N_x, g.N_y, g.N_time, nh_sv, nh_colors);
        const int nh_phases = nh_colors * nh_colors;
        const int per_phase = nh_items_per_phase(g.N_time, g.N_y, g.N_x, nh_sv, nh_colors);
        const bool lists = opt.nh_work_lists && nh_items_supported(g.N_time, g.N_y, g.N_x, nh_sv) &&
                           (size_t)nh_phases * per_phase <= nh_items_cap &&
                           nh_items_scratch_ints(g.N_time, g.N_y, g.N_x, nh_sv, nh_colors) <= nh_scratch_cap;
        if (lists) launch_nh_items(g.N_time, g.N_y, g.N_x, nh_sv, nh_colors, d_sel, d_nh_items, d_nh_n, d_nh_scratch, st);
        for (int ph = 0; ph < nh_phases; ph++) {
            Ln.phase = ph;
            Ln.items = lists ? d_nh_items + (size_t)ph * per_phase : nullptr;
            Ln.n_items = lists ? d_nh_n + ph : nullptr;
            launch_icd_phase(gb, Ln, d_table, d_view_first, d_mask, d_x, d_err, d_w, d_mag, d_stats,
                             d_queue + kMaxPhases * (pass + 1) + ph, st);
        }
        if (rings && update_offset()) return -1;
        launches += nh_phases + 11 + (lists ? 3 : 0);  // filter + 10 select launches, 3 list launches
    }
    if (nh > 0 && timing) CK(record(ev_pairs[1].second));
    CK(cudaGetLastError());
    // the noise-variance re-estimation reads its sums back to the host, so an
    // iteration that has it is never captured
    if (!graph_mode && update_var && variance_update(g, g.N_p, d_err, d_w, &var_est, d_var, st))
        return fail("variance update failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (opt.refresh_every > 0 && iter % opt.refresh_every == 0) {
        if (refresh_error()) return -1;
        launches += 1;
    }
    *launches_out = launches;
    return 0;
}

int Session::icd_iteration(int iter, mbirgpu_iter_stats *out)
{
    const Geom &g = hs.g;
    if (timing && ev_pairs.size() < 2) {
        while (ev_pairs.size() < 2) {
            cudaEvent_t a, b;
            CK(cudaEventCreate(&a));
            CK(cudaEventCreate(&b));
            ev_pairs.push_back({a, b});
        }
    }
    const int nh = (d_sel && iter > 1) ? std::min(opt.nhicd_passes, kMaxNhPasses) : 0;
    int launches = 0;
    const bool refresh_it = opt.refresh_every > 0 && iter % opt.refresh_every == 0;
    // the first iteration of each kind launches directly (it sets the kernel
    // attributes and occupancy figures the captured launches reuse); later
    // ones replay a graph
    if (graph_ok() && graph_seen[nh > 0][refresh_it] == 0) {
        if (enqueue_iteration(iter, false, &launches)) return -1;
        graph_seen[nh > 0][refresh_it] = 1;
    } else if (graph_ok()) {
        // one graph per (NH passes or not, FP64 refresh or not); the kernels
        // read this iteration's number from d_iter
        if (graphs_timed != timing) {
            drop_graphs();
            graphs_timed = timing;
        }
        if (!d_iter) {
            cudaError_t e = cudaMalloc((void **)&d_iter, sizeof(int));
            if (e != cudaSuccess) return fail("cudaMalloc of the iteration counter failed: %s", cudaGetErrorString(e));
        }
        const bool refresh = refresh_it;
        cudaGraphExec_t &ge = graphs[nh > 0][refresh];
        h_iter = iter;
        CK(cudaMemcpyAsync(d_iter, &h_iter, sizeof(int), cudaMemcpyHostToDevice, st));
        if (!ge) {
            cudaGraph_t gr = nullptr;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            const int rc = enqueue_iteration(iter, true, &launches);
            cudaError_t e = cudaStreamEndCapture(st, &gr);
            if (rc) {
                if (gr) cudaGraphDestroy(gr);
                return -1;
            }
            if (e != cudaSuccess) return fail("capturing the ICD iteration failed: %s", cudaGetErrorString(e));
            e = cudaGraphInstantiate(&ge, gr, 0);
            cudaGraphDestroy(gr);
            if (e != cudaSuccess) return fail("instantiating the ICD iteration graph failed: %s", cudaGetErrorString(e));
        }
        graph_launches_[nh > 0][refresh] = launches ? launches : graph_launches_[nh > 0][refresh];
        launches = graph_launches_[nh > 0][refresh];
        CK(cudaGraphLaunch(ge, st));
    } else {
        if (enqueue_iteration(iter, false, &launches)) return -1;
    }
    IcdStats hst;
    CK(cudaMemcpyAsync(&hst, d_stats, sizeof(hst), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hst.stage_timeouts)
        return fail("ICD iteration %d: %u staged A-record copies did not complete", iter, hst.stage_timeouts);
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->voxel_updates = (int64_t)hst.updates;
        out->zero_skipped = (int64_t)hst.skipped;
        out->sum_abs_update = hst.sum_abs_dx;
        out->sum_abs_value = hst.sum_abs_x;
        out->kernel_launches = launches;
        if (timing) {
            float m = 0;
            CK(cudaEventElapsedTime(&m, ev_pairs[0].first, ev_pairs[0].second));
            double ms = m;
            if (nh > 0) {
                CK(cudaEventElapsedTime(&m, ev_pairs[1].first, ev_pairs[1].second));
                ms += m;
            }
            out->kernel_ms = ms;
        }
    }
    return 0;
}

int Session::run(int max_iter, double *costs, int *iters, mbirgpu_iter_stats *total)
{
    double c_prev = 0, c = 0;
    if (opt.compute_cost) {
        if (cost(&c, nullptr, nullptr)) return -1;
        if (costs) costs[0] = c;
        c_prev = c;
    }
    if (total) std::memset(total, 0, sizeof(*total));
    int it = 1;
    for (; it <= max_iter; it++) {
        mbirgpu_iter_stats s;
        if (icd_iteration(it, &s)) return -1;
        if (total) {
            total->voxel_updates += s.voxel_updates;
            total->zero_skipped += s.zero_skipped;
            total->sum_abs_update += s.sum_abs_update;
            total->sum_abs_value += s.sum_abs_value;
            total->kernel_ms += s.kernel_ms;
            total->kernel_launches += s.kernel_launches;
        }
        bool stop = false;
        // the reference's test, XT_ICD_update.c:1083-1090 and :1174
        const double pct = s.sum_abs_value > 0 ? 100.0 * s.sum_abs_update / s.sum_abs_value : 0.0;
        if (it > 1 && pct < convg_thresh) stop = true;
        if (opt.compute_cost) {
            if (cost(&c, nullptr, nullptr)) return -1;
            if (costs) costs[it] = c;
            if (opt.cost_rel_tol > 0 && it > 1 && std::fabs(c_prev - c) < opt.cost_rel_tol * std::fabs(c)) stop = true;
            c_prev = c;
        }
        if (stop) break;
    }
    if (iters) *iters = std::min(it, max_iter);
    return 0;
}

int Session::amatrix(int32_t *first, int32_t *count, float *values)
{
    const Geom &g = hs.g;
    const size_t nxy = (size_t)g.N_x * g.N_y;
    std::vector<uint32_t> tab((size_t)n_assigned * nxy * g.rec_words);
    if (!tab.empty())
        CK(cudaMemcpyAsync(tab.data(), d_table, tab.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::fill(first, first + (size_t)g.N_p * nxy, 0);
    std::fill(count, count + (size_t)g.N_p * nxy, 0);
    std::fill(values, values + (size_t)g.N_p * nxy * g.kmax, 0.0f);
    for (int f = 0; f < g.N_time; f++) {
        const int fv0 = hs.view_first[f], nv = hs.view_first[f + 1] - fv0;
        for (size_t c = 0; c < nxy; c++)
            for (int v = 0; v < nv; v++) {
                const uint32_t *rec = tab.data() + (((size_t)fv0 * nxy) + c * nv + v) * g.rec_words;
                const int view = hs.views[fv0 + v];
                const size_t o = (size_t)view * nxy + c;
                first[o] = (int32_t)(rec[0] & 0xFFFFFF) - view * g.N_r;
                count[o] = rec[0] >> 24;
                for (int q = 0; q < g.kmax; q++) std::memcpy(&values[o * g.kmax + q], &rec[1 + q], 4);
            }
    }
    return 0;
}

int Session::forward_project(const float *obj, float *sino)
{
    const Geom &g = hs.g;
    float *d_obj = nullptr, *d_out = nullptr;
    size_t acc = 0;
    if (dalloc(&d_obj, n_vox, &acc) || dalloc(&d_out, n_sino, &acc)) {
        if (d_obj) cudaFree(d_obj);
        return -1;
    }
    cudaError_t e = cudaMemcpyAsync(d_tmp, obj, n_vox * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        launch_vol_to_zfast(d_tmp, d_obj, g.N_time, g.N_z, g.N_y, g.N_x, st);
        launch_forward_project(g, d_table, d_view_first, d_obj, nullptr, d_acc, d_out, st);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(sino, d_out, n_sino * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_obj);
    cudaFree(d_out);
    if (e != cudaSuccess) return fail("forward projection failed: %s", cudaGetErrorString(e));
    return 0;
}

int Session::back_project(const float *sino, float *obj)
{
    const Geom &g = hs.g;
    float *d_s = nullptr, *d_o = nullptr;
    size_t acc = 0;
    if (dalloc(&d_s, n_sino, &acc) || dalloc(&d_o, n_vox, &acc)) {
        if (d_s) cudaFree(d_s);
        return -1;
    }
    cudaError_t e = cudaMemcpyAsync(d_s, sino, n_sino * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) launch_back_project(g, d_table, d_view_first, d_views, d_s, d_o, st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) {
        launch_zfast_to_vol(d_o, d_tmp, g.N_time, g.N_z, g.N_y, g.N_x, st);
        e = cudaMemcpyAsync(obj, d_tmp, n_vox * sizeof(float), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_s);
    cudaFree(d_o);
    if (e != cudaSuccess) return fail("back projection failed: %s", cudaGetErrorString(e));
    return 0;
}

int Session::fbp(float *obj)
{
    const Geom &g = hs.g;
    if (!fbp_supported(g)) return fail("FBP: %d channels x %d rows per view exceed the filter's shared memory", g.N_r, g.N_t);
    float *d_o = nullptr;
    size_t acc = 0;
    if (dalloc(&d_o, n_vox, &acc)) return -1;
    launch_fbp(g, d_table, d_view_first, d_views, d_y, d_tmp, d_o, st);
    launch_zfast_to_vol(d_o, d_tmp, g.N_time, g.N_z, g.N_y, g.N_x, st);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(obj, d_tmp, n_vox * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_o);
    if (e != cudaSuccess) return fail("filtered back-projection failed: %s", cudaGetErrorString(e));
    return 0;
}

int Session::set_object_fbp()
{
    const Geom &g = hs.g;
    if (!fbp_supported(g)) return fail("FBP: %d channels x %d rows per view exceed the filter's shared memory", g.N_r, g.N_t);
    launch_fbp(g, d_table, d_view_first, d_views, d_y, d_tmp, d_x, st);
    launch_mask_object(g, d_mask, d_x, st);
    CK(cudaGetLastError());
    return refresh_error();
}

int unet_apply_frames(UNet *u, float *d_vol, int N_time, int N_z, int N_y, int N_x);

// Ring correction of reconstruct (remove_rings 1..3): the offset d enters
// e = y - Ax - d and is re-estimated after every full-sweep phase and every
// NH pass (the reference re-estimates after each of its z-block phases,
// XT_ICD_update.c:983-1043). offset: the starting d (host, [N_r][N_t]), null = 0.
int Session::set_ring_correction(int mode, const float *offset)
{
    const Geom &g = hs.g;
    if (mode < 0 || mode > 3) return fail("remove_rings must be 0, 1, 2 or 3 (got %d)", mode);
    const size_t nrt = (size_t)g.N_r * g.N_t;
    size_t &acc = device_bytes;
    if (!d_off && (dalloc(&d_off, nrt, &acc) || dalloc(&d_offx, nrt, &acc) || dalloc(&d_onum, nrt, &acc) ||
                   dalloc(&d_olam, nrt, &acc) || dalloc(&d_ogamma, 1, &acc)))
        return -1;
    if (offset) CK(cudaMemcpyAsync(d_off, offset, nrt * sizeof(float), cudaMemcpyHostToDevice, st));
    else CK(cudaMemsetAsync(d_off, 0, nrt * sizeof(float), st));
    rings = mode;
    if (refresh_error()) return -1;
    CK(cudaStreamSynchronize(st));
    return 0;
}

// Noise-variance re-estimation of reconstruct with the generalised-Huber data
// term (quad_convex = 0) after the first multires stage (updateVar,
// XT_Init.c:270-278): var starts at 1 and is re-estimated at the end of every
// iteration, the weights rescaled with it.
int Session::set_variance_estimation(int on)
{
    if (on && !d_var) {
        size_t &acc = device_bytes;
        if (dalloc(&d_var, variance_scratch_doubles(), &acc)) return -1;
    }
    update_var = on ? 1 : 0;
    return 0;
}

int Session::update_offset()
{
    if (offset_update(hs.g, rings, hs.g.N_p, d_err, d_w, d_off, d_onum, d_olam, d_ogamma, d_offx, st))
        return fail("ring correction update failed: %s", cudaGetErrorString(cudaGetLastError()));
    return 0;
}

int Session::set_object_unet(UNet *u)
{
    const Geom &g = hs.g;
    if (!fbp_supported(g)) return fail("FBP: %d channels x %d rows per view exceed the filter's shared memory", g.N_r, g.N_t);
    // d_tmp (max(sinogram, volume) floats) holds the filtered sinogram during
    // the FBP, then the volume in the network's [T][Z][Y][X] layout
    launch_fbp(g, d_table, d_view_first, d_views, d_y, d_tmp, d_x, st);
    launch_zfast_to_vol(d_x, d_tmp, g.N_time, g.N_z, g.N_y, g.N_x, st);
    cudaError_t e = cudaStreamSynchronize(st);  // the network runs on its own stream
    int rc = e == cudaSuccess ? unet_apply_frames(u, d_tmp, g.N_time, g.N_z, g.N_y, g.N_x) : -1;
    if (!rc) {
        launch_vol_to_zfast(d_tmp, d_x, g.N_time, g.N_z, g.N_y, g.N_x, st);
        launch_mask_object(g, d_mask, d_x, st);
        rc = refresh_error();
        e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) return fail("warm start failed: %s", cudaGetErrorString(e));
    return rc;
}

}  // namespace mbirgpu

using mbirgpu::fail;
using mbirgpu::Session;

extern "C" {

void mbirgpu_default_options(mbirgpu_options *o)
{
    std::memset(o, 0, sizeof(*o));
    o->mrf_p = 1.2;
    o->mrf_q = 2.0;
    o->alpha = 1.5;
    o->max_iterations = 1000;
    o->num_stages = 0;
    o->cost_rel_tol = 0.0;
    o->zero_skipping = 1;
    o->write_files = 1;
    o->compute_cost = 1;
    o->refresh_every = 8;
    o->sv_size = 0;
    o->cta_warps = 0;
    o->icd_unroll = 0;
    o->seed = 761521;  // the reference's srandom2 seed, XT_Engine.c:99
    o->nhicd_passes = mbirgpu::kNhicdIterations;  // the reference runs NH-ICD by default (NO_NHICD 0)
    o->sv_colors = 0;
    o->stage_records = 1;
    o->nh_sv_size = 0;
    o->nh_sv_colors = 0;
    o->nh_cta_warps = 0;
    o->nh_work_lists = 1;
    o->autotune = 0;
    o->graph_iterations = 1;
}

int mbirgpu_set_options(const mbirgpu_options *o)
{
    if (!o) return fail("options pointer is NULL");
    if (!(o->mrf_p >= 1.0 && o->mrf_p <= o->mrf_q)) return fail("need 1 <= mrf_p <= mrf_q");
    if (o->max_iterations < 1) return fail("max_iterations must be positive");
    if (o->sv_size < 0 || o->sv_size > 16) return fail("sv_size must be 0 (auto) or 1..16");
    if (o->cta_warps < 0 || o->cta_warps > 8) return fail("cta_warps must be 0 (auto) or 1..8");
    if (o->icd_unroll < 0 || o->icd_unroll > 4) return fail("icd_unroll must be 0 (auto) or 1..4");
    if (o->nhicd_passes < 0 || o->nhicd_passes > mbirgpu::kMaxNhPasses)
        return fail("nhicd_passes must be 0 (off) .. %d", mbirgpu::kMaxNhPasses);
    if (o->sv_colors != 0 && o->sv_colors != 2 && o->sv_colors != 4) return fail("sv_colors must be 0 (auto), 2 or 4");
    if (o->nh_sv_size < 0 || o->nh_sv_size > 16) return fail("nh_sv_size must be 0 (auto) or 1..16");
    if (o->nh_sv_colors != 0 && o->nh_sv_colors != 2 && o->nh_sv_colors != 4)
        return fail("nh_sv_colors must be 0 (auto), 2 or 4");
    if (o->nh_cta_warps < 0 || o->nh_cta_warps > 8) return fail("nh_cta_warps must be 0 (auto) or 1..8");
    if (o->autotune != 0 && o->autotune != 1) return fail("autotune must be 0 (schedule by rule) or 1 (measured)");
    if (o->graph_iterations != 0 && o->graph_iterations != 1) return fail("graph_iterations must be 0 or 1");
    mbirgpu_options cur = mbirgpu::current_options();
    (void)cur;
    std::lock_guard<std::mutex> lk(mbirgpu::g_opt_mu);
    mbirgpu::g_opt = *o;
    mbirgpu::g_opt_init = true;
    return 0;
}

int mbirgpu_get_options(mbirgpu_options *o)
{
    if (!o) return fail("options pointer is NULL");
    *o = mbirgpu::current_options();
    return 0;
}

const char *mbirgpu_last_error(void) { return mbirgpu::g_last_error.c_str(); }

int mbirgpu_session_create(mbirgpu_session **out, const mbirgpu_problem *pb, const mbirgpu_options *opt,
                           int32_t mult_xy, int32_t mult_z, void *stream)
{
    if (!out || !pb) return fail("NULL argument");
    *out = nullptr;
    if (!pb->projections || !pb->weights || !pb->proj_angles || !pb->proj_times || !pb->recon_times)
        return fail("NULL input array");
    Session *s = new (std::nothrow) Session();
    if (!s) return fail("out of host memory");
    if (s->init(pb, opt, mult_xy, mult_z, stream)) {
        std::string keep = mbirgpu::g_last_error;
        delete s;
        mbirgpu::g_last_error = keep;
        return -1;
    }
    *out = reinterpret_cast<mbirgpu_session *>(s);
    return 0;
}

int mbirgpu_session_destroy(mbirgpu_session *s)
{
    delete reinterpret_cast<Session *>(s);
    return 0;
}

int mbirgpu_session_info_get(const mbirgpu_session *sp, mbirgpu_session_info *info)
{
    if (!sp || !info) return fail("NULL argument");
    const Session *s = reinterpret_cast<const Session *>(sp);
    const mbirgpu::Geom &g = s->hs.g;
    std::memset(info, 0, sizeof(*info));
    info->N_r = g.N_r;
    info->N_t = g.N_t;
    info->N_p = g.N_p;
    info->N_time = g.N_time;
    info->N_x = g.N_x;
    info->N_y = g.N_y;
    info->N_z = g.N_z;
    info->mult_xy = g.mult_xy;
    info->mult_z = g.mult_z;
    info->max_views = g.max_views;
    info->kmax = g.kmax;
    info->sv_size = s->sv;
    info->cta_warps = s->warps;
    info->sv_colors = s->colors;
    info->masked_columns = s->masked_columns;
    info->nnz = s->masked_nnz;
    info->delta_t = g.delta_t;
    info->device_bytes = s->device_bytes;
    return 0;
}

#define SESSION(sp)                                       \
    if (!(sp)) return fail("session pointer is NULL");    \
    Session *s = reinterpret_cast<Session *>(sp)

int mbirgpu_session_set_stream(mbirgpu_session *sp, void *stream)
{
    SESSION(sp);
    s->st = (cudaStream_t)stream;
    return 0;
}

int mbirgpu_session_set_timing(mbirgpu_session *sp, int32_t enable)
{
    SESSION(sp);
    s->timing = enable != 0;
    return 0;
}

int mbirgpu_session_set_object(mbirgpu_session *sp, const float *object)
{
    SESSION(sp);
    if (!object) return fail("NULL object");
    return s->set_object(object);
}

int mbirgpu_session_get_object(mbirgpu_session *sp, float *object)
{
    SESSION(sp);
    if (!object) return fail("NULL object");
    return s->get_object(object);
}

int mbirgpu_session_object_device(mbirgpu_session *sp, float **d_object)
{
    SESSION(sp);
    if (!d_object) return fail("NULL argument");
    *d_object = s->d_x;
    return 0;
}

int mbirgpu_session_refresh_error(mbirgpu_session *sp)
{
    SESSION(sp);
    return s->refresh_error();
}

int mbirgpu_session_get_error(mbirgpu_session *sp, float *err)
{
    SESSION(sp);
    if (!err) return fail("NULL argument");
    cudaError_t e = cudaMemcpyAsync(err, s->d_err, s->n_sino * sizeof(float), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return fail("copy of the error sinogram failed: %s", cudaGetErrorString(e));
    return 0;
}

int mbirgpu_session_cost(mbirgpu_session *sp, double *total, double *data_term, double *prior_term)
{
    SESSION(sp);
    return s->cost(total, data_term, prior_term);
}

int mbirgpu_session_icd_iteration(mbirgpu_session *sp, int32_t iter, mbirgpu_iter_stats *stats)
{
    SESSION(sp);
    if (iter < 1) return fail("iterations are numbered from 1");
    return s->icd_iteration(iter, stats);
}

int mbirgpu_session_fbp(mbirgpu_session *sp, float *object)
{
    SESSION(sp);
    if (!object) return fail("NULL object");
    return s->fbp(object);
}

int mbirgpu_session_set_object_fbp(mbirgpu_session *sp)
{
    SESSION(sp);
    return s->set_object_fbp();
}

int mbirgpu_session_set_object_zero(mbirgpu_session *sp)
{
    SESSION(sp);
    cudaError_t e = cudaMemsetAsync(s->d_x, 0, s->n_vox * sizeof(float), s->st);
    if (e != cudaSuccess) return fail("clearing the object failed: %s", cudaGetErrorString(e));
    return s->refresh_error();
}

int mbirgpu_session_set_ring_correction(mbirgpu_session *sp, int32_t remove_rings, const float *offset)
{
    SESSION(sp);
    return s->set_ring_correction(remove_rings, offset);
}

int mbirgpu_session_set_variance_estimation(mbirgpu_session *sp, int32_t on)
{
    SESSION(sp);
    return s->set_variance_estimation(on);
}

int mbirgpu_session_get_variance(mbirgpu_session *sp, double *var_est)
{
    SESSION(sp);
    if (!var_est) return fail("NULL argument");
    *var_est = s->var_est;
    return 0;
}

int mbirgpu_session_update_variance(mbirgpu_session *sp)
{
    SESSION(sp);
    if (!s->d_var) {  // allocate the scratch without switching the per-iteration update on
        const int on = s->update_var;
        if (s->set_variance_estimation(1)) return -1;
        s->update_var = on;
    }
    const mbirgpu::Geom &g = s->hs.g;
    if (mbirgpu::variance_update(g, g.N_p, s->d_err, s->d_w, &s->var_est, s->d_var, s->st))
        return fail("variance update failed: %s", cudaGetErrorString(cudaGetLastError()));
    return 0;
}

int mbirgpu_session_update_offset(mbirgpu_session *sp)
{
    SESSION(sp);
    if (!s->rings) return fail("ring correction is off (mbirgpu_session_set_ring_correction)");
    if (s->update_offset()) return -1;
    cudaError_t e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? 0 : fail("offset update failed: %s", cudaGetErrorString(e));
}

int mbirgpu_session_get_offset(mbirgpu_session *sp, float *offset)
{
    SESSION(sp);
    if (!offset) return fail("NULL offset");
    const mbirgpu::Geom &g = s->hs.g;
    const size_t nrt = (size_t)g.N_r * g.N_t;
    if (!s->d_off) {
        std::memset(offset, 0, nrt * sizeof(float));
        return 0;
    }
    cudaError_t e = cudaMemcpyAsync(offset, s->d_off, nrt * sizeof(float), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? 0 : fail("offset download failed: %s", cudaGetErrorString(e));
}

int mbirgpu_session_set_object_unet(mbirgpu_session *sp, mbirgpu_unet *u)
{
    SESSION(sp);
    if (!u) return fail("U-Net pointer is NULL");
    return s->set_object_unet(reinterpret_cast<mbirgpu::UNet *>(u));
}

int mbirgpu_session_nh_select(mbirgpu_session *sp, const float *mag, uint8_t *sel)
{
    SESSION(sp);
    if (!mag || !sel) return fail("NULL argument");
    const mbirgpu::Geom &g = s->hs.g;
    const size_t n = (size_t)g.N_time * g.N_y * g.N_x;
    float *d_m = nullptr, *d_f = nullptr;
    uint8_t *d_s = nullptr;
    void *d_scr = nullptr;
    cudaError_t e = cudaMalloc((void **)&d_m, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_f, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_s, n);
    if (e == cudaSuccess) e = cudaMalloc(&d_scr, mbirgpu::nh_select_scratch_bytes(g.N_time));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_m, mag, n * sizeof(float), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) {
        const int k = (int)(s->masked_columns / std::max(1, g.N_time)) / mbirgpu::kNhicdIterations;
        mbirgpu::launch_nh_select(g.N_time, g.N_y, g.N_x, d_m, s->d_mask, k, d_f, d_s, s->st, d_scr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(sel, d_s, n, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    cudaFree(d_m);
    cudaFree(d_f);
    cudaFree(d_s);
    cudaFree(d_scr);
    if (e != cudaSuccess) return fail("NH-ICD selection failed: %s", cudaGetErrorString(e));
    return 0;
}

int mbirgpu_session_forward_project(mbirgpu_session *sp, const float *object, float *sino)
{
    SESSION(sp);
    if (!object || !sino) return fail("NULL argument");
    return s->forward_project(object, sino);
}

int mbirgpu_session_back_project(mbirgpu_session *sp, const float *sino, float *object)
{
    SESSION(sp);
    if (!object || !sino) return fail("NULL argument");
    return s->back_project(sino, object);
}

int mbirgpu_session_get_amatrix(mbirgpu_session *sp, int32_t *first, int32_t *count, float *values)
{
    SESSION(sp);
    if (!first || !count || !values) return fail("NULL argument");
    return s->amatrix(first, count, values);
}

int mbirgpu_session_get_detector_response(mbirgpu_session *sp, float *H_r)
{
    SESSION(sp);
    if (!H_r) return fail("NULL argument");
    std::memcpy(H_r, s->hs.H_r.data(), s->hs.H_r.size() * sizeof(float));
    return 0;
}

int mbirgpu_session_run(mbirgpu_session *sp, int32_t max_iter, double *costs, int32_t *iters,
                        mbirgpu_iter_stats *total)
{
    SESSION(sp);
    if (max_iter < 1) return fail("max_iter must be positive");
    int it = 0;
    int rc = s->run(max_iter, costs, &it, total);
    if (iters) *iters = it;
    return rc;
}

}  // extern "C"
