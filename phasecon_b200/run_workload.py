"""Run a few iterations of a synthetic workload (for profiling and quick checks).

    python -m phasecon_b200.run_workload [--workload 4d|3d] [--iters N] [--sv S] [--warps W] [--colors K]
                                         [--refresh] [--cost] [--ch-steps K]
    python -m phasecon_b200.run_workload --workload pc [--iters N] [--views V] [--nms-order 0|1]
    python -m phasecon_b200.run_workload --workload unet [--iters N]
    python -m phasecon_b200.run_workload --workload pcsim [--views V]

Builds the seeded workload (phasecon_b200/workloads.py). For 4d / 3d: one
session with the given schedule (autotuned unless --sv, --warps and --colors are all set), N ICD
iterations from zero, then optionally one FP64 error-sinogram refresh and one
FP64 cost evaluation; --ch-steps shortens the phantom simulation (same array
sizes) to keep the number of unrelated kernel launches small under a
profiler. For pc: the phase-contrast scan, Paganin retrieval, the ADMM start
and N phase-retrieval iterations of every view. For unet: N training steps and
one inference of the warm-start network on a seeded 32 x 256 x 256 frame. For
pcsim: the phase-contrast data simulator on a seeded 40-sphere phantom of
512 x 512 x 256 voxels, V views onto a 256 x 256 detector (2 x 1 phantom
pixels per detector pixel).
"""
from __future__ import annotations

import argparse
import time

from . import Session, get_options
from . import workloads as W


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="4d", choices=["4d", "3d", "pc", "unet", "pcsim"])
    ap.add_argument("--views", type=int, default=180)
    ap.add_argument("--nms-order", type=int, default=0)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--sv", type=int, default=0)
    ap.add_argument("--warps", type=int, default=0)
    ap.add_argument("--colors", type=int, default=0)
    ap.add_argument("--refresh", action="store_true")
    ap.add_argument("--cost", action="store_true")
    ap.add_argument("--ch-steps", type=int, default=5000)
    a = ap.parse_args(argv)
    if a.workload == "pc":
        return run_pc(a)
    if a.workload == "unet":
        return run_unet(a)
    if a.workload == "pcsim":
        return run_pcsim(a)
    if a.workload == "4d":
        pb, _, p = W.config_4d(ch_steps=a.ch_steps)
    else:
        pb, _, p = W.config_3d()
    o = get_options()
    o.mrf_p, o.refresh_every, o.sv_size, o.cta_warps, o.sv_colors = p, 0, a.sv, a.warps, a.colors
    s = Session(pb, options=o)
    t0 = time.perf_counter()
    for it in range(1, a.iters + 1):
        st = s.icd_iteration(it)
    if a.refresh:
        s.refresh_error()
    c = s.cost() if a.cost else None
    print(f"workload {a.workload}: sv {s.info.sv_size} warps {s.info.cta_warps} colours {s.info.sv_colors} "
          f"iters {a.iters} "
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
    # warm inference of one 32 x 256 x 256 frame on each tensor-core path
    # (wall time around one synchronous call, median of 5)
    C = [16, 32, 64, 128]
    flops = 0.0  # the 3x3x3 convolutions: encoder two per level, decoder three per level
    for l in range(4):
        vox = x.numel() / 8 ** l
        flops += 2 * 27 * vox * ((1 if l == 0 else C[l - 1]) * C[l] + C[l] * C[l])
        if l < 3:
            flops += 2 * 27 * vox * (C[l + 1] * C[l] + 2 * C[l] * C[l] + C[l] * C[l])
    for path in (1, 0):
        net.tensor_path = path
        net.forward(x)
        ts = []
        for _ in range(5):
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            net.forward(x)
            ts.append(time.perf_counter() - t2)
        ms = 1e3 * sorted(ts)[2]
        print(f"  inference, {'tcgen05' if path else 'mma.sync'} convolutions: {ms:.2f} ms per frame, "
              f"{flops / ms / 1e9:.1f} TFLOP/s ({flops / 1e12:.3f} TFLOP)")
    net.tensor_path = 1


def run_pcsim(a):
    import numpy as np

    from . import pcmbir as PC
    rng = np.random.default_rng(0)
    o = PC.sim_options(write_files=0, phantom_xy=512, phantom_z=256)
    Pz, Pxy = o.phantom_z, o.phantom_xy
    z, y, x = np.meshgrid(np.arange(Pz) + 0.5, np.arange(Pxy) + 0.5, np.arange(Pxy) + 0.5, indexing="ij",
                          sparse=True)
    mag = np.zeros((Pz, Pxy, Pxy), np.float32)
    ph = np.zeros_like(mag)
    for _ in range(40):
        c = rng.uniform([0.2 * Pz, 0.2 * Pxy, 0.2 * Pxy], [0.8 * Pz, 0.8 * Pxy, 0.8 * Pxy])
        r = rng.uniform(0.02, 0.08) * Pxy
        inside = (z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2 < r * r
        d = rng.uniform(1e-7, 5e-7)
        ph[inside] += d
        mag[inside] += d / 100
    ang = np.linspace(0, np.pi, a.views, endpoint=False).astype(np.float32)
    PC.simulate(mag, ph, ang, 256, 256, 1.0, 128.0, 5e4, 20.0, options=o)  # warm-up (module load, allocations)
    t0 = time.perf_counter()
    meas, br, avg = PC.simulate(mag, ph, ang, 256, 256, 1.0, 128.0, 5e4, 20.0, options=o)
    print(f"workload pcsim: phantom {Pz}x{Pxy}x{Pxy}, {a.views} views onto 256x256: wall "
          f"{time.perf_counter() - t0:.3f}s (incl. host<->device copies), mean measurement {avg:.2f}")


if __name__ == "__main__":
    main()
