"""The benchmark workloads, as seeded synthetic problems.

``config_4d`` is the 4-D time-interlaced problem: a Cahn-Hilliard two-phase
microstructure (256x256x32 voxels at 1 mm, 8 frames, attenuation 0.005/0.02
per mm), 1,024 parallel-beam views interlaced over K=8 sub-frames across 4
rotations (gen_interlaced_views_0_to_Inf, 256 views per rotation), a 256x32
detector, Poisson counts at I0 = 2e4, spatial + temporal qGGMRF with p = 1.2.
``config_3d`` is the 3-D Shepp-Logan-type problem (128x128x16, 180 views,
I0 = 1e4, p = 1.1). Measurements are y = -log(N/I0), w = N, N ~ Poisson(I0
e^{-Ax}) with A the reference's own system matrix (applied by the GPU forward
projector, whose parity with the reference is tested).
"""
from __future__ import annotations

import numpy as np

from . import phantoms as P
from .mbir import Problem, Session, get_options


def _measure(pb: Problem, obj: np.ndarray, I0: float, seed: int) -> Problem:
    o = get_options()
    s = Session(pb, options=o)
    ax = s.forward_project(obj)  # [view][col][row]
    s.close()
    y, w = P.poisson_measurements(ax, I0, seed)
    pb.projections = np.ascontiguousarray(y.transpose(0, 2, 1))
    pb.weights = np.ascontiguousarray(w.transpose(0, 2, 1))
    return pb


def config_4d(seed: int = 0, n_xy: int = 256, n_z: int = 32, frames: int = 8, views: int = 1024,
              ch_steps: int = 5000):
    angles, times = P.interlaced_views(8, 256, views)
    recon_times = np.linspace(0.0, float(views), frames + 1).astype(np.float32)
    obj = P.cahn_hilliard_frames(n_xy, n_z, frames, steps=ch_steps, seed=seed)
    zeros = np.zeros((views, n_z, n_xy), np.float32)
    pb = Problem(zeros, np.ones_like(zeros), angles, times, recon_times, n_z, n_xy, views, frames, vox_wid=1.0,
                 rot_center=n_xy / 2, sig_s=0.01, sig_t=0.01, c_s=1.0, c_t=1.0, convg_thresh=0.0)
    return _measure(pb, obj, 2e4, seed), obj, 1.2


def config_3d(seed: int = 0, n_xy: int = 128, n_z: int = 16, views: int = 180):
    angles, times, recon_times = P.uniform_views(views)
    obj = P.ellipsoid_phantom(n_xy, n_z, seed)[None]
    zeros = np.zeros((views, n_z, n_xy), np.float32)
    pb = Problem(zeros, np.ones_like(zeros), angles, times, recon_times, n_z, n_xy, views, 1, vox_wid=1.0,
                 rot_center=n_xy / 2, sig_s=0.01, sig_t=1.0, c_s=1.0, c_t=1.0, convg_thresh=0.0)
    return _measure(pb, obj, 1e4, seed), obj, 1.1
