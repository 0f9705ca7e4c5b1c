"""Benchmark: plain GPU super-voxel ICD on the 4-D time-interlaced MBIR workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one ICD iteration over the whole 4-D problem (every voxel inside the
reconstruction circle of all 8 frames updated once). The workload is seeded
synthetic data with the shapes of the 4-D configuration: a Cahn-Hilliard
two-phase microstructure on 256x256x32 voxels x 8 frames, 1,024 interlaced
parallel-beam views (K=8 sub-frames, 4 rotations), a 256x32 detector,
Poisson I0 = 2e4, qGGMRF p = 1.2 (see phasecon_b200/workloads.py).

One JSON line on rank 0 carries:
  value       voxel-updates/s over K timed iterations, inputs resident in HBM
              (device time, CUDA events on the session's stream, max over ranks);
  e2e         the same metric through the public API with host buffers: session
              creation from host arrays (H2D of y, w, geometry; A-matrix build;
              initial projection), K iterations, and the D2H read of the object;
  time_to_converged_s  plain GPU ICD from zero to relative cost change < 1e-4;
  roofline    the ICD sweep kernel's algorithmic bytes (12 nnz_v + 8 per voxel
              update) over its measured launch time, against MEASURED_PEAKS.json;
  cpu_baseline the reference C (oracle/_ref, built from source) on a bounded
              sample of the workload on this host's cores;
  warm_start  the learned warm start: the U-Net trained from --ws-seeds seeds
              on seeded Cahn-Hilliard scans and ellipsoid phantoms, and the
              wall time of plain ICD to the plain method's converged cost
              from zero, from FBP and from each network (speedup_vs_zero_init
              is the smallest over the seeds), with its clock record.
With --gpus N > 1 (torchrun) every rank runs an independent replica (the path
does not shard on one problem); value is the sum over ranks / max time.
--workload pc|batch|warmstart print the phase-contrast, batched and warm-start
lines instead.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-converged cost (rel 1e-4), voxel-updates/s; warm-start vs plain GPU ICD"
UNIT = "voxel-updates/s"
WORKLOAD = "4d_cahn_hilliard_256x256x32_8frames_1024views"
SAMPLE_ROWS = 4  # detector rows of the CPU-baseline sample (4 of the 32 voxel slices)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-converge", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--max-converge-iters", type=int, default=400)
    ap.add_argument("--schedule", default="",
                    help="4-D workload: fix the sweep schedule as SV,WARPS,COLORS (super-voxel edge, warps per "
                         "column, K of the K x K colouring) instead of the library's shape rule")
    ap.add_argument("--workload", default="4d", choices=["4d", "batch", "warmstart", "pc"],
                    help="4d: the 4-D benchmark (default); batch: 48 uneven 3-D problems, batched vs sequential; "
                         "warmstart: the learned warm start on the 4-D workload; pc: the phase-contrast scan "
                         "(180 views of 256 x 256), phase-retrieval ADMM iterations")
    ap.add_argument("--nms-order", type=int, default=-1,
                    help="pc workload: Nelder-Mead sweep order, 0 raster (the reference's), 1 colour classes; "
                         "-1: the library default")
    ap.add_argument("--pc-cpu-views", type=int, default=0,
                    help="pc workload: views of the reference CPU sample (0: one per host thread, at most 32)")
    ap.add_argument("--train-scans", type=int, default=16, help="seeded 4-D training scans (8 frame pairs each)")
    ap.add_argument("--train-ellipsoids", type=int, default=32,
                    help="seeded single-frame ellipsoid-phantom training pairs added to the Cahn-Hilliard scans")
    ap.add_argument("--ws-seeds", type=int, default=3, help="warm start: independent trainings (network seeds)")
    ap.add_argument("--no-warmstart", action="store_true", help="4-D workload: skip the learned warm start")
    ap.add_argument("--train-steps", type=int, default=6000)
    ap.add_argument("--average-from", type=float, default=0.7,
                    help="warm start: average the network weights from this fraction of the training steps on (1 = off)")
    return ap.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, v: float) -> float:
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, v: float) -> float:
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per ICD sweep launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "icd_phase_kernel_4d.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch_full_size:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# --------------------------------------------------------------------------- CPU sample (reference C)


def cpu_sample_problem(seed: int = 0):
    """A bounded sample of the 4-D workload for the CPU reference: the same
    Cahn-Hilliard frames, views and detector columns, restricted to the first
    SAMPLE_ROWS detector rows / voxel slices. Measurements are formed with the
    oracle's restated reference projector, so no GPU kernel of this project is
    involved."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    from phasecon_b200 import phantoms as P
    angles, times = P.interlaced_views(8, 256, 1024)
    rt = np.linspace(0.0, 1024.0, 9).astype(np.float32)
    vol = P.cahn_hilliard_frames(256, 32, 8, steps=5000, seed=seed)[:, :SAMPLE_ROWS]
    pb = O.Problem(np.zeros((1024, SAMPLE_ROWS, 256), np.float32), np.ones((1024, SAMPLE_ROWS, 256), np.float32),
                   angles, times, rt, SAMPLE_ROWS, 256, 1024, 8, rot_center=128.0, sig_s=0.01, sig_t=0.01, c_s=1.0,
                   c_t=1.0, mrf_p=1.2, convg_thresh=0.0)
    orc = O.Oracle(pb)
    ax = orc.forward(np.ascontiguousarray(vol))
    y, w = P.poisson_measurements(ax, 2e4, seed)
    pb.projections = np.ascontiguousarray(y.transpose(0, 2, 1))
    pb.weights = np.ascontiguousarray(w.transpose(0, 2, 1))
    return pb


def reference_parallelism(threads: int, n_time: int, n_z: int) -> int:
    """Voxel-line updates the reference runs at once: its OpenMP loops go over
    (frame, every other z block) with num_z_blocks = threads / N_time, at least
    2, at most N_z, rounded down to even (MBIR_4D/XT_Init.c:379-384,
    XT_ICD_update.c:964-1046)."""
    nzb = threads // n_time
    nzb = 2 if nzb < 2 else min(nzb, n_z)
    nzb = (nzb // 2) * 2
    return min(threads, n_time * nzb // 2)


def reference_rate(pb, warmup: int, steps: int):
    """Reference C as it ships (the build with -DNO_COST_CALCULATE -DNO_DEBUG of
    MBIR_4D/Makefile:3: no cost pass, no cost-increase abort), single stage,
    all host threads: voxel-updates/s over `steps` ICD iterations after
    `warmup`, from two runs (warmup and warmup+steps iterations) so set-up time
    cancels."""
    import oracle as O
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    _, _, u1 = O.ref_reconstruct(pb, tempfile.mkdtemp(), max_iter=max(warmup, 1), num_stages=1, threads=threads,
                                 timing=True)
    t1 = time.perf_counter()
    _, _, u2 = O.ref_reconstruct(pb, tempfile.mkdtemp(), max_iter=max(warmup, 1) + steps, num_stages=1,
                                 threads=threads, timing=True)
    t2 = time.perf_counter()
    dt = (t2 - t1) - (t1 - t0)
    upd = u2 - u1
    return upd / dt if dt > 0 else float("nan"), dt, upd, threads


def reference_sample_text(threads: int, steps: int, warmup: int, upd: int, dt: float) -> str:
    busy = reference_parallelism(threads, 8, SAMPLE_ROWS)
    return (f"reference C MBIR_4D built from source as it ships (-DNO_COST_CALCULATE -DNO_DEBUG), single stage, "
            f"{SAMPLE_ROWS} of 32 detector rows of the same 4-D workload, {steps} ICD iterations after {warmup} "
            f"(two runs, set-up cancelled; {upd} voxel updates, {dt:.1f} s); {threads} OpenMP threads, of which the "
            f"reference keeps {busy} busy: it runs (frame, z block) items with num_z_blocks = threads / frames "
            f"(XT_Init.c:379-384), the same on the full 32-row workload")


def run_reference_arm(args, rank):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_available(timing=True):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_mbir4d_timing.so was not built"}))
        return
    pb = cpu_sample_problem()
    rate, dt, upd, threads = reference_rate(pb, args.warmup, args.steps)
    sample = reference_sample_text(threads, args.steps, args.warmup, upd, dt)
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_rows": SAMPLE_ROWS}, "impl": "reference",
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample,
                             "busy_threads": reference_parallelism(threads, 8, SAMPLE_ROWS)},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "voxel_updates": upd}
    print(json.dumps(line))


# --------------------------------------------------------------------------- our arm


def run_ours(args, world, rank, local, pg):
    import torch

    import phasecon_b200 as pc
    from phasecon_b200 import workloads as W

    torch.cuda.set_device(local)
    # a stream of the benchmark's own: the library replays ICD iterations from
    # CUDA graphs on any stream but the legacy default one
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    pb, _, p = W.config_4d(seed=0)
    opt = pc.get_options()
    opt.mrf_p = p
    if args.schedule:
        opt.sv_size, opt.cta_warps, opt.sv_colors = (int(v) for v in args.schedule.split(","))
    s = pc.Session(pb, options=opt, stream=stream.cuda_stream)
    s.set_timing(True)
    info = s.info
    refresh = opt.refresh_every

    # warm-up, then K timed iterations (device events on the session stream)
    for it in range(1, args.warmup + 1):
        s.icd_iteration(it)
    barrier(pg)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kernel_ms, updates, launches = 0.0, 0, 0
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for it in range(args.warmup + 1, args.warmup + args.steps + 1):
            st = s.icd_iteration(it)
            kernel_ms += st.kernel_ms
            updates += st.voxel_updates
            launches += st.kernel_launches
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(pg)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(pg, ms)
    total_updates = sum_over_ranks(pg, float(updates))
    value = total_updates / (ms_max / 1e3)

    # roofline of the ICD sweep kernel: every ICD launch of the timed iterations
    # (K^2 colour phases of the full sweep + K^2 per non-homogeneous pass from
    # iteration 2), algorithmic bytes 12 nnz_v + 8 per voxel update
    nh = opt.nhicd_passes
    phases = info.sv_colors ** 2
    icd_launches = sum(phases * (1 + (nh if it > 1 else 0))
                       for it in range(args.warmup + 1, args.warmup + args.steps + 1))
    entries = info.nnz * info.N_t  # (e, w) entries one full sweep reads: nnz_v summed over voxel slices
    full = info.masked_columns * info.N_z
    bytes_per_update = (12.0 * entries + 8.0 * full) / full
    bytes_total = bytes_per_update * updates
    avg_launch_s = kernel_ms / icd_launches / 1e3
    peak, peak_kind = measured_peaks()
    achieved = bytes_total / (kernel_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": profiled_traffic(), "peak_source": peak_kind, "kernel": "icd_phase_kernel",
                "algorithmic_bytes_per_launch": bytes_total / icd_launches, "avg_launch_ms": avg_launch_s * 1e3,
                "bytes_per_voxel_update": bytes_per_update, "icd_launches": icd_launches,
                # the captured launch behind `traffic` is one full-sweep colour
                # phase; its algorithmic bytes are a K-squared-th of a full sweep's
                "traffic_launch": "one full-sweep colour phase (profiles/icd_phase_kernel_4d.txt)",
                "algorithmic_bytes_full_phase": (12.0 * entries + 8.0 * full) / phases}

    # time to converged cost from zero (plain GPU ICD), FP64 cost every iteration
    conv = {}
    if not args.no_converge:
        s.set_object_zero()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        costs = [s.cost()[0]]
        it = 0
        while it < args.max_converge_iters:
            it += 1
            s.icd_iteration(it)
            costs.append(s.cost()[0])
            if it > 1 and abs(costs[-2] - costs[-1]) < 1e-4 * abs(costs[-1]):
                break
        torch.cuda.synchronize()
        tconv = time.perf_counter() - t0
        conv = {"time_to_converged_s": tconv, "iterations_to_converged": it, "converged_cost": costs[-1],
                "initial_cost": costs[0], "converged": it < args.max_converge_iters}
        # FP64 cost of the final state against the CPU oracle on the same (e, x)
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O
            s.refresh_error()
            x = s.get_object()
            e = s.get_error()
            gpu_cost = s.cost()[0]
            orc_pb = O.Problem(pb.projections, pb.weights, pb.proj_angles, pb.proj_times, pb.recon_times,
                               pb.proj_rows, pb.proj_cols, pb.proj_num, pb.recon_num, rot_center=pb.rot_center,
                               sig_s=pb.sig_s, sig_t=pb.sig_t, c_s=pb.c_s, c_t=pb.c_t, mrf_p=p)
            orc_cost = O.Oracle(orc_pb).cost(e, x)[0]
            conv["cost_rel_err_vs_fp64_oracle"] = abs(gpu_cost - orc_cost) / abs(orc_cost)
        except Exception as ex:  # the oracle is the checker only; its absence does not stop the bench
            conv["cost_rel_err_vs_fp64_oracle"] = f"unavailable: {ex}"
    obj_shape = tuple(s.shape)
    s.close()

    # end to end through the public API with host buffers: the measured
    # sinogram and weights in pinned host memory (copied there before the
    # timed region), the object read back into a pinned buffer
    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
        t.numpy()[...] = a
        return t

    keep = [pinned(pb.projections), pinned(pb.weights)]
    pb_host = dataclasses.replace(pb, projections=keep[0].numpy(), weights=keep[1].numpy())
    h_arrays = pb_host.arrays()
    h2d = sum(a.nbytes for a in h_arrays)
    obj_t = torch.empty(obj_shape, dtype=torch.float32, pin_memory=True)
    torch.cuda.synchronize()
    barrier(pg)
    t0 = time.perf_counter()
    s2 = pc.Session(pb_host, options=opt, stream=stream.cuda_stream)
    e2e_upd = 0
    for it in range(1, args.steps + 1):
        e2e_upd += s2.icd_iteration(it).voxel_updates
    obj = s2.get_object(out=obj_t.numpy())
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(pg, time.perf_counter() - t0)
    s2.close()
    d2h = obj.nbytes
    e2e = {"value": sum_over_ranks(pg, float(e2e_upd)) / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
           "steps_per_call": args.steps,
           "note": "one session from pinned host arrays (H2D of y, w, angles, times), A-matrix build, K "
                   "iterations, D2H of the object into pinned memory; bytes per step = bytes per call / K"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle
            if oracle.ref_available(timing=True):
                spb = cpu_sample_problem()
                rate, dt, upd, threads = reference_rate(spb, 1, 2)
                cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                       "busy_threads": reference_parallelism(threads, 8, SAMPLE_ROWS),
                       "sample": reference_sample_text(threads, 2, 1, upd, dt)}
            else:
                cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                       "sample": "oracle/_ref not built on this host"}
        except Exception as ex:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {ex}"}

    ws = None
    if not args.no_warmstart and not args.no_converge:
        try:
            ws = warmstart_section(args, rank, local, pb, p)
        except Exception as ex:  # the ICD line above stands on its own
            ws = {"speedup_vs_zero_init": None, "error": f"{type(ex).__name__}: {ex}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "voxels": [info.N_time, info.N_z, info.N_y, info.N_x],
                           "views": info.N_p, "detector": [info.N_t, info.N_r], "sv_size": info.sv_size,
                           "cta_warps": info.cta_warps, "sv_colors": info.sv_colors,
                           "nhicd_passes": opt.nhicd_passes,
                           "parallelism": f"replicas{world}",
                           "l2": "inputs larger than L2: A table %.2f GB, y/w/e %.0f MB, x %.0f MB" % (
                               info.device_bytes / 1e9, 3 * info.N_p * info.N_r * info.N_t * 4 / 1e6,
                               info.N_time * info.N_z * info.N_y * info.N_x * 4 / 1e6)},
                "voxel_updates_per_step": updates / args.steps, "roofline": roofline, "cpu_baseline": cpu,
                "e2e": e2e, "clocks": clk.summary(), "gpu_launches": launches}
        line.update(conv)
        if ws is not None:
            line["warm_start"] = ws
            line["speedup_vs_zero_init"] = ws["speedup_vs_zero_init"]
        print(json.dumps(line))


def run_batch(args, world, rank, local, pg):
    """48 independent uneven 3-D problems: K iterations of the batched persistent
    launch (CUDA graph per iteration) against K iterations of each problem in
    its own session, one after another; plain SV-ICD in both (no NH passes)."""
    import torch

    import phasecon_b200 as pc
    from phasecon_b200 import workloads as W

    torch.cuda.set_device(local)
    probs = W.config_batch(seed=rank)
    opt = pc.get_options()
    opt.nhicd_passes = 0
    # batched: creation (H2D, A tables, autotune, graph capture), warm-up, timed run
    t0 = time.perf_counter()
    b = pc.Batch(probs, options=opt)
    t_create = time.perf_counter() - t0
    b.run(args.warmup)
    before = b.run(0).voxel_updates
    with ClockSampler(local) as clk:
        st = b.run(args.steps)
    upd = st.voxel_updates - before
    ms = max_over_ranks(pg, st.device_ms)
    value = sum_over_ranks(pg, float(upd)) / (ms / 1e3)
    costs = [b.cost(i) for i in range(len(probs))]
    b.close()
    # sequential: each problem alone (its own autotuned session), same iterations
    seq_ms, seq_upd = 0.0, 0
    for p in probs:
        s = pc.Session(p, options=opt)
        s.set_timing(True)
        for it in range(1, args.warmup + 1):
            s.icd_iteration(it)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for it in range(args.warmup + 1, args.warmup + args.steps + 1):
            seq_upd += s.icd_iteration(it).voxel_updates
        e1.record()
        torch.cuda.synchronize()
        seq_ms += e0.elapsed_time(e1)
        s.close()
    seq_value = sum_over_ranks(pg, float(seq_upd)) / (max_over_ranks(pg, seq_ms) / 1e3)
    if rank == 0:
        print(json.dumps({
            "metric": "aggregate voxel-updates/s, batched persistent launch vs sequential per-problem solves",
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batch_48_uneven_3d", "problems": len(probs),
                       "edges": sorted({p.proj_cols for p in probs}), "depths": [min(p.proj_rows for p in probs),
                                                                                 max(p.proj_rows for p in probs)],
                       "views": [min(p.proj_num for p in probs), max(p.proj_num for p in probs)],
                       "sv_size": st.sv_size, "cta_warps": st.cta_warps, "sv_colors": st.sv_colors,
                       "kernel_launches_per_iteration": st.kernel_launches_per_iteration,
                       "graph_launches": st.graph_launches, "parallelism": f"replicas{world}"},
            "sequential": {"value": seq_value, "unit": UNIT, "ms_per_step": seq_ms / args.steps},
            "speedup_vs_sequential": value / seq_value if seq_value else None,
            "batch_create_s": t_create, "mean_final_cost": float(np.mean(costs)),
            "clocks": clk.summary()}))


def warmstart_section(args, rank: int, local: int, pb, p: float) -> dict:
    """The learned warm start on the 4-D workload `pb`: one training set (the
    8 frame pairs of each of `--train-scans` seeded 4-D Cahn-Hilliard scans and
    `--train-ellipsoids` seeded single-frame ellipsoid phantoms scanned with one
    frame's views; input = the GPU FBP, target = plain GPU ICD to rel 1e-4;
    seeds other than the benchmark's), `--ws-seeds` networks trained on it from
    different seeds (each ending on the checkpoint whose warm start leaves the
    lowest MAP cost on a held-out 4-D scan; a training that learned next to
    nothing by that measure is repeated once from another initialisation),
    then plain ICD on the benchmark scan timed to the plain
    method's converged cost (x (1 + 1e-4)) from zero, from FBP and from each
    network's output; each time includes its initialisation (FBP, network,
    error sinogram) and follows one untimed run of the same start."""
    import torch

    import phasecon_b200 as pc
    from phasecon_b200 import warmstart as WS

    t0 = time.perf_counter()
    pairs = []
    for i in range(args.train_scans):
        pairs += WS.training_pairs_4d(1000 + rank * 100000 + i)
    n_ch = len(pairs)
    for i in range(args.train_ellipsoids):
        x, t, _ = WS.training_pair(5000 + rank * 100000 + i, kind="ellipsoids")
        pairs.append((x, t))
    t_data = time.perf_counter() - t0
    opt = pc.get_options()
    opt.mrf_p = p
    # a held-out 4-D scan (never trained on) picks each training's checkpoint
    # by the MAP cost its warm start leaves there
    from phasecon_b200 import workloads as W
    pb_val, _, _ = W.config_4d(seed=9000 + rank * 100000)
    s_val = pc.Session(pb_val, options=opt, stream=torch.cuda.current_stream().cuda_stream)
    s = pc.Session(pb, options=opt, stream=torch.cuda.current_stream().cuda_stream)
    s.set_object_zero()
    _, c_conv = WS.converge(s, rel=1e-7, max_iter=400)
    target = c_conv[-1] * (1 + 1e-4)

    def timed_start(start):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        start()
        torch.cuda.synchronize()
        t_init = time.perf_counter() - t0
        it, costs = WS.iterations_to_cost(s, target, max_iter=400)
        torch.cuda.synchronize()
        return {"time_to_converged_cost_s": time.perf_counter() - t0, "init_s": t_init, "iterations": it,
                "initial_cost": costs[0], "final_cost": costs[-1]}

    starts = {"zero": s.set_object_zero, "fbp": s.set_object_fbp}
    res, seeds, train_s, losses, held_out = {}, [], [], [], []
    with ClockSampler(local) as clk:
        for name, fn in starts.items():
            timed_start(fn)  # untimed: module loading, the FBP's allocations
            res[name] = timed_start(fn)
    clocks = [clk.summary()]
    # the held-out scan's cost from the FBP start: a training whose best
    # warm start is not at least a tenth below it has learned next to nothing
    # (a run stuck near the identity map happens now and then) and is
    # repeated once from another initialisation
    s_val.set_object_fbp()
    fbp_val_cost = float(s_val.cost()[0])
    for k in range(args.ws_seeds):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tries = []
        for attempt in range(2):
            init_seed = rank * 1000 + k + 100 * attempt
            cand = WS.UNet(16, seed=init_seed)
            sc = []
            hist = WS.train(cand, pairs, args.train_steps, lr=1e-3, seed=init_seed, average_from=args.average_from,
                            val_session=s_val, scores=sc, warmup=args.train_steps // 20)
            picked = sc[sc[-1]] if sc and sc[-1] is not None else None
            tries.append((picked[2] if picked else float("inf"), cand, hist, {
                "init_seed": init_seed, "candidates": len(sc) - 1, "chosen_step": picked[0] if picked else None,
                "chosen_averaged": picked[1] if picked else None, "chosen_cost": picked[2] if picked else None,
                "worst_cost": max(c[2] for c in sc[:-1]) if len(sc) > 1 else None}))
            if tries[-1][0] <= 0.9 * fbp_val_cost:
                break
        best = min(range(len(tries)), key=lambda i: tries[i][0])
        for i, t in enumerate(tries):
            if i != best:
                t[1].close()
        _, net, hist, info = tries[best]
        info["trainings"] = len(tries)
        info["fbp_start_cost"] = fbp_val_cost
        held_out.append(info)
        torch.cuda.synchronize()
        train_s.append(time.perf_counter() - t0)
        losses.append([float(np.mean(hist[:20])), float(np.mean(hist[-20:]))])
        with ClockSampler(local) as clk:
            timed_start(lambda: WS.warm_start(s, net))  # untimed: the stacked grid's activation blocks
            r = timed_start(lambda: WS.warm_start(s, net))
        clocks.append(clk.summary())
        r["seed"] = rank * 1000 + k
        seeds.append(r)
        net.close()
    s.close()
    s_val.close()
    tz, tf = res["zero"]["time_to_converged_cost_s"], res["fbp"]["time_to_converged_cost_s"]
    sp = [tz / r["time_to_converged_cost_s"] for r in seeds]
    return {"speedup_vs_zero_init": min(sp) if sp else None, "speedup_vs_zero_init_per_seed": sp,
            "speedup_vs_zero_init_median": float(np.median(sp)) if sp else None,
            "speedup_vs_fbp_init_per_seed": [tf / r["time_to_converged_cost_s"] for r in seeds],
            "target_cost": target, "starts": res, "unet_starts": seeds,
            "train": {"pairs": len(pairs), "cahn_hilliard_pairs": n_ch, "ellipsoid_pairs": len(pairs) - n_ch,
                      "checkpoint_selection": "lowest MAP cost the warm start leaves on a held-out 4-D scan "
                                              "(seed 9000), candidates every 250 steps from a quarter of the run; "
                                              "a training whose best is not 10 % below the held-out FBP start's "
                                              "cost is repeated once from another initialisation",
                      "lr_warmup_steps": args.train_steps // 20,
                      "held_out_selection": held_out,
                      "steps": args.train_steps, "seeds": args.ws_seeds, "data_s": t_data, "train_s": train_s,
                      "loss_first_last": losses},
            "unet": "4 levels 16/32/64/128, 3x3x3, BF16 weights and activations, FP32 accumulation",
            "timing": "wall time per start (init + ICD to the target cost), each after one untimed run of the "
                      "same start; speedup_vs_zero_init is the smallest over the seeds",
            "clocks": clocks}


def run_warmstart(args, world, rank, local, pg):
    """The learned warm start alone (the same section the default 4-D line
    carries), as its own JSON line."""
    import torch

    from phasecon_b200 import workloads as W

    torch.cuda.set_device(local)
    pb, _, p = W.config_4d(seed=0)
    ws = warmstart_section(args, rank, local, pb, p)
    if rank == 0:
        tu = max(r["time_to_converged_cost_s"] for r in ws["unet_starts"]) if ws["unet_starts"] else None
        print(json.dumps({
            "metric": "warm start: wall time to the plain method's converged cost (rel 1e-4), 4-D workload",
            "value": tu, "unit": "s", "n_gpus": world, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 network / f32 ICD", "data": "synthetic",
            "config": {"workload": WORKLOAD}, **ws}))


def pc_reference_rate(pb, views: int, threads: int, workdir: str):
    """The reference's phcontomo_reconstruct (PCMBIR_3D, built from source with
    the FP64 FFT shim, all host threads, OpenMP over views) on the first
    `views` views of the scan: Paganin (recon_type 1), then recon_type 2 with
    1 and with 2 phase-retrieval iterations; the difference of the two times is
    one PRet iteration of every sampled view. Returns view-PRet-iterations/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    meas = np.ascontiguousarray(pb.measurements[:views])
    V, rows, cols = meas.shape
    args = dict(measurements=meas, brights=pb.brights, proj_angles=np.zeros(V, np.float32),
                proj_times=np.arange(V, dtype=np.float32), recon_times=np.array([0, V], np.float32),
                proj_rows=rows, proj_cols=cols, proj_num=V, recon_num=1, vox_wid=pb.vox_wid, rot_center=cols / 2,
                mag_sig_s=pb.mag_sig_s, mag_sig_t=1.0, mag_c_s=pb.mag_c_s, mag_c_t=1.0, phase_sig_s=pb.phase_sig_s,
                phase_sig_t=1.0, phase_c_s=pb.phase_c_s, phase_c_t=1.0, convg_thresh=0.0,
                obj2det_dist=pb.obj2det_dist, light_energy=pb.light_energy, pag_regparam=pb.pag_regparam)
    O.ref_pc_reconstruct(workdir, **args, recon_type=1, threads=threads)
    t = []
    for n in (1, 2):
        t0 = time.perf_counter()
        O.ref_pc_reconstruct(workdir, **args, recon_type=2, pret_max_iter=n, threads=threads)
        t.append(time.perf_counter() - t0)
    dt = t[1] - t[0]
    return V / dt if dt > 0 else float("nan"), dt, V


def run_pc(args, world, rank, local, pg):
    """Phase-contrast configuration: 40 random spheres in a 256 um cube, 180
    views of 256 x 256 at 20 keV and 50 mm (phasecon_b200/workloads.py
    config_pc). A step is one phase-retrieval ADMM iteration (Nelder-Mead
    proximal sweep, steepest descent on the exit wave to its stop rule, dual
    update, cost) of every view, batched over the views; the state starts from
    Paganin retrieval. Warm-up runs W iterations in a session of its own; the
    timed session runs K iterations (CUDA events on its stream)."""
    import torch

    from phasecon_b200 import pcmbir as PC
    from phasecon_b200 import workloads as W

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    pb, _ = W.config_pc(seed=rank)
    V, rows, cols = pb.dims
    N = rows * cols
    kw = {} if args.nms_order < 0 else {"nms_order": args.nms_order}
    warm = PC.PcSession(pb, PC.default_options(pret_max_iter=max(args.warmup, 1), **kw),
                        stream=stream.cuda_stream)
    warm.paganin()
    warm.init_admm()
    warm.run()
    warm.close()
    opts = PC.default_options(pret_max_iter=args.steps, **kw)
    s = PC.PcSession(pb, opts, stream=stream.cuda_stream)
    s.paganin()
    s.init_admm()
    barrier(pg)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        costs, iters, st = s.run()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(pg)
    ms = max_over_ranks(pg, ev0.elapsed_time(ev1))
    view_iters = int(iters.sum())
    value = sum_over_ranks(pg, float(view_iters)) / (ms / 1e3)
    # dominant memory-side kernel family: the Fresnel-type transform (3 launches
    # per transform of all views), 16 B per pixel (read + write complex FP32)
    n_tr = 20
    s.time_fresnel(2)
    tr_ms = s.time_fresnel(n_tr)
    alg_bytes = 16.0 * V * N
    achieved = alg_bytes / (tr_ms / n_tr / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "peak_source": peak_kind, "kernel": "pc_rows_fft + pc_cols_filter + pc_rows_fft",
                "algorithmic_bytes_per_launch": alg_bytes, "avg_transform_ms": tr_ms / n_tr,
                "transforms_per_step": st.fresnel_transforms / max(args.steps, 1)}
    zr, zi, _, _, _ = s.get_state()
    s.close()
    # end to end through the session API with host buffers: session from host
    # measurements (H2D), Paganin, K iterations, D2H of the retrieved z
    torch.cuda.synchronize()
    barrier(pg)
    t0 = time.perf_counter()
    s2 = PC.PcSession(pb, opts, stream=stream.cuda_stream)
    s2.paganin()
    s2.init_admm()
    _, it2, _ = s2.run()
    out = s2.get_state()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(pg, time.perf_counter() - t0)
    s2.close()
    e2e = {"value": sum_over_ranks(pg, float(it2.sum())) / t_e2e, "unit": "view-iterations/s",
           "h2d_bytes_per_step": (pb.measurements.nbytes + pb.brights.nbytes) / args.steps,
           "d2h_bytes_per_step": sum(a.nbytes for a in out[:2]) / args.steps, "steps_per_call": args.steps,
           "note": "session from host arrays, Paganin start, K iterations, D2H of the retrieved z (r, i)"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle
            if oracle.ref_pc_available():
                threads = os.cpu_count() or 1
                nv = args.pc_cpu_views or min(threads, 32)
                rate, dt, nv = pc_reference_rate(pb, nv, threads, tempfile.mkdtemp())
                cpu = {"value": rate, "unit": "view-iterations/s", "cores": threads, "kind": "reference",
                       "sample": f"reference PCMBIR_3D phcontomo_reconstruct built from source (FFTW replaced by an "
                                 f"FP64 radix-2 FFT with tabulated twiddles), recon_type 2 on the first {nv} views "
                                 f"of the same scan, one phase-retrieval iteration each (1- and 2-iteration runs "
                                 f"differenced, {dt:.1f} s), OpenMP over views"}
        except Exception as ex:
            cpu = {"value": None, "unit": "view-iterations/s", "cores": 0, "kind": "reference",
                   "sample": f"failed: {ex}"}
    if rank == 0:
        print(json.dumps({
            "metric": "phase-retrieval ADMM iterations x views per second (config 3 phase contrast)",
            "value": value, "unit": "view-iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 per-view sums)", "data": "synthetic",
            "config": {"workload": "pc_spheres_256cube_180views_256x256", "views": V, "detector": [rows, cols],
                       "nms_order": int(opts.nms_order), "sd_max_iter": int(opts.sd_max_iter),
                       "nms_max_iter": int(opts.nms_max_iter), "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2: 14 per-view complex/real FP32 arrays of 180 x 256^2 (~1 GB)"},
            "sd_steps_per_view_iteration": st.sd_steps / max(view_iters, 1),
            "final_cost_mean": float(np.nanmean([c[np.isfinite(c)][-1] for c in costs])),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
            "gpu_launches": int(st.kernel_launches)}))


def main():
    args = parse()
    world, rank, local, pg = dist_setup()
    try:
        if args.impl == "reference":
            run_reference_arm(args, rank)
        elif args.workload == "batch":
            run_batch(args, world, rank, local, pg)
        elif args.workload == "warmstart":
            run_warmstart(args, world, rank, local, pg)
        elif args.workload == "pc":
            run_pc(args, world, rank, local, pg)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
