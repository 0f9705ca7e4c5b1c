"""Run a few iterations of a synthetic workload (for profiling and quick checks).

    python -m phasecon_b200.run_workload [--workload 4d|3d] [--iters N] [--sv S] [--warps W]
                                         [--refresh] [--cost] [--ch-steps K]
    python -m phasecon_b200.run_workload --workload pc [--iters N] [--views V] [--nms-order 0|1]
    python -m phasecon_b200.run_workload --workload unet [--iters N]

Builds the seeded workload (phasecon_b200/workloads.py). For 4d / 3d: one
session with the given schedule (autotuned when --sv/--warps are 0), N ICD
iterations from zero, then optionally one FP64 error-sinogram refresh and one
FP64 cost evaluation; --ch-steps shortens the phantom simulation (same array
sizes) to keep the number of unrelated kernel launches small under a
profiler. For pc: the phase-contrast scan, Paganin retrieval, the ADMM start
and N phase-retrieval iterations of every view. For unet: N training steps and
one inference of the warm-start network on a seeded 32 x 256 x 256 frame.
"""
from __future__ import annotations

import argparse
import time

from . import Session, get_options
from . import workloads as W


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="4d", choices=["4d", "3d", "pc", "unet"])
    ap.add_argument("--views", type=int, default=180)
    ap.add_argument("--nms-order", type=int, default=0)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--sv", type=int, default=0)
    ap.add_argument("--warps", type=int, default=0)
    ap.add_argument("--refresh", action="store_true")
    ap.add_argument("--cost", action="store_true")
    ap.add_argument("--ch-steps", type=int, default=5000)
    a = ap.parse_args(argv)
    if a.workload == "pc":
        return run_pc(a)
    if a.workload == "unet":
        return run_unet(a)
    if a.workload == "4d":
        pb, _, p = W.config_4d(ch_steps=a.ch_steps)
    else:
        pb, _, p = W.config_3d()
    o = get_options()
    o.mrf_p, o.refresh_every, o.sv_size, o.cta_warps = p, 0, a.sv, a.warps
    s = Session(pb, options=o)
    t0 = time.perf_counter()
    for it in range(1, a.iters + 1):
        st = s.icd_iteration(it)
    if a.refresh:
        s.refresh_error()
    c = s.cost() if a.cost else None
    print(f"workload {a.workload}: sv {s.info.sv_size} warps {s.info.cta_warps} iters {a.iters} "
          f"updates/iter {st.voxel_updates} wall {time.perf_counter() - t0:.3f}s cost {c}")


def run_pc(a):
    from .pcmbir import PcSession, default_options
    pb, _ = W.config_pc(views=a.views)
    s = PcSession(pb, default_options(pret_max_iter=a.iters, nms_order=a.nms_order))
    s.paganin()
    s.init_admm()
    t0 = time.perf_counter()
    costs, iters, st = s.run()
    print(f"workload pc: views {a.views} iters {a.iters} sd_steps {st.sd_steps} transforms "
          f"{st.fresnel_transforms} device {st.kernel_ms:.1f} ms wall {time.perf_counter() - t0:.3f}s "
          f"cost[0] {costs[0, :a.iters + 1]}")


def run_unet(a):
    import numpy as np
    import torch

    from .warmstart import UNet
    rng = np.random.default_rng(0)
    x = torch.from_numpy((0.01 + 0.01 * rng.random((32, 256, 256))).astype(np.float32)).cuda()
    t = x * 1.1
    net = UNet(16)
    net.input_scale = 50.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.iters):
        loss = net.train_step(x, t, 1e-3)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    net.forward(x)
    torch.cuda.synchronize()
    print(f"workload unet: {a.iters} training steps {1e3 * (t1 - t0) / max(a.iters, 1):.1f} ms/step, "
          f"inference {1e3 * (time.perf_counter() - t1):.1f} ms, loss {loss:.4g}")


if __name__ == "__main__":
    main()
