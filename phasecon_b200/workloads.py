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
``config_batch`` is the batch of independent uneven 3-D problems: edges from
{64, 96, 128, 192, 256}, slab depths 8-32 (even), 90-360 views, seeded random
ellipsoid sets (0-0.02 per mm), Poisson I0 in [5e3, 5e4].
``config_pc`` is the phase-contrast scan: 40 random spheres (radius 5-40 um,
refractive decrement delta in [1e-7, 5e-7], beta = delta / 100) in a 256 um
cube at 1 um, 180 parallel-beam views over 180 deg on a 256x256 detector at
20 keV, Fresnel propagation over 50 mm, intensities with Gaussian noise at a
per-pixel SNR of 100.
"""
from __future__ import annotations

import numpy as np

from . import phantoms as P
from .mbir import Problem, Session, get_options


def _measure(pb: Problem, obj: np.ndarray, I0: float, seed: int) -> Problem:
    o = get_options()
    # a projection-only session: a fixed schedule skips the ICD autotuner
    o.sv_size, o.cta_warps, o.sv_colors, o.nhicd_passes = 8, 4, 2, 0
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


def config_batch(seed: int = 0, n: int = 48, edges=(64, 96, 128, 192, 256), depth=(8, 32), views=(90, 360)):
    """n independent 3-D problems of uneven size. Returns a list of Problem."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        n_xy = int(rng.choice(edges))
        n_z = int(rng.integers(depth[0] // 2, depth[1] // 2 + 1)) * 2
        nv = int(rng.integers(views[0], views[1] + 1))
        I0 = float(rng.uniform(5e3, 5e4))
        angles, times, recon_times = P.uniform_views(nv)
        obj = P.random_ellipsoids(n_xy, n_z, seed * 1000 + i)[None]
        zeros = np.zeros((nv, n_z, n_xy), np.float32)
        pb = Problem(zeros, np.ones_like(zeros), angles, times, recon_times, n_z, n_xy, nv, 1, vox_wid=1.0,
                     rot_center=n_xy / 2, sig_s=0.01, sig_t=1.0, c_s=1.0, c_t=1.0, convg_thresh=0.0)
        out.append(_measure(pb, obj, I0, seed * 1000 + i))
    return out


def config_pc(seed: int = 0, n: int = 256, views: int = 180, spheres: int = 40, energy_kev: float = 20.0,
              distance_um: float = 5e4, snr: float = 100.0):
    """Phase-contrast scan of random spheres. Returns (PcProblem, (zr, zi)
    true [views][n][n] in the session layout [view][N_r][N_t])."""
    from .pcmbir import PcProblem
    rng = np.random.default_rng(seed)
    lam = 4.135668e-19 * 299792458e+6 / energy_kev  # um
    k = 2 * np.pi / lam
    rad = rng.uniform(5.0, 40.0, spheres)
    ctr = rng.uniform(-n / 2 + rad[:, None], n / 2 - rad[:, None], (spheres, 3))
    delta = rng.uniform(1e-7, 5e-7, spheres)
    beta = delta / 100.0
    coords = np.arange(n) - n / 2 + 0.5
    theta = np.arange(views) * np.pi / views
    zr = np.zeros((views, n, n))
    zi = np.zeros((views, n, n))
    tt = coords[None, :]
    for s in range(spheres):
        r0 = ctr[s, 0] * np.cos(theta) + ctr[s, 1] * np.sin(theta)  # [views]
        d2 = (coords[None, :, None] - r0[:, None, None]) ** 2 + (tt[:, None, :] * 0 + (coords[None, None, :] - ctr[s, 2]) ** 2)
        th = 2 * np.sqrt(np.maximum(rad[s] ** 2 - d2, 0.0))
        zr += k * beta[s] * th
        zi += k * delta[s] * th
    u = np.fft.fftfreq(n, 1.0)
    H = np.exp(-1j * np.pi * lam * distance_um * (u[:, None] ** 2 + u[None, :] ** 2))
    bright = np.full((n, n), 1.0e4, np.float32)
    w = np.exp(-zr) * np.exp(-1j * zi)
    inten = np.abs(np.fft.ifft2(np.fft.fft2(w, axes=(1, 2)) * H, axes=(1, 2))) ** 2 * 1.0e4
    inten = inten + rng.normal(size=inten.shape) * inten / snr
    meas = np.ascontiguousarray(np.maximum(inten, 1e-3).transpose(0, 2, 1), np.float32)
    pb = PcProblem(measurements=meas, brights=bright, vox_wid=1.0, mag_sig_s=0.05, mag_c_s=1.0, phase_sig_s=0.05,
                   phase_c_s=1.0, obj2det_dist=distance_um, light_energy=energy_kev, pag_regparam=100.0)
    return pb, (zr, zi)
