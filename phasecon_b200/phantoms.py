"""Seeded synthetic workloads for the MBIR hot path.

No measurement data ships with phasecon (its examples list projections.bin and
weights.bin as missing), so every workload here is synthetic and seeded:

* ``ellipsoid_phantom`` -- a 10-ellipsoid head-like phantom of the Shepp-Logan
  type (outer shell, inner region, eight interior features) whose parameters
  are drawn from a seed, scaled to attenuation 0 .. mu_max per unit length;
* ``random_ellipsoids`` -- seeded random ellipsoid sets (batched workloads);
* ``cahn_hilliard_frames`` -- a periodic Cahn-Hilliard spinodal simulation
  thresholded to a two-phase attenuation map, one volume per time frame;
* ``uniform_views`` / ``interlaced_views`` -- view angle and time schedules,
  the latter restating gen_interlaced_views_0_to_Inf
  (reconstruct/real_data/APS_Data_Format/XT_Views.c:7-46);
* ``poisson_measurements`` -- y = -log(N/I0), w = N with N ~ Poisson(I0 e^{-Ax}).
"""
from __future__ import annotations

import math

import numpy as np


def _ellipsoid_mask(shape, center, axes, phi):
    nz, ny, nx = shape
    z = (np.arange(nz) + 0.5) / nz * 2 - 1
    y = (np.arange(ny) + 0.5) / ny * 2 - 1
    x = (np.arange(nx) + 0.5) / nx * 2 - 1
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    c, s = math.cos(phi), math.sin(phi)
    xr = (X - center[2]) * c + (Y - center[1]) * s
    yr = -(X - center[2]) * s + (Y - center[1]) * c
    zr = Z - center[0]
    return (xr / axes[2]) ** 2 + (yr / axes[1]) ** 2 + (zr / axes[0]) ** 2 <= 1.0


def ellipsoid_phantom(n_xy: int, n_z: int, seed: int = 0, mu_max: float = 0.02) -> np.ndarray:
    """A seeded 10-ellipsoid head-like phantom, [n_z][n_xy][n_xy] float32.

    Layout: an outer shell (ellipsoid 1, densest), an inner region that
    subtracts most of it (ellipsoid 2), and eight small interior features of
    varying sign. The volume spans [-1,1]^3 in normalised coordinates; values
    are clipped to [0, mu_max].
    """
    rng = np.random.default_rng(seed)
    shape = (n_z, n_xy, n_xy)
    vol = np.zeros(shape, np.float64)
    a0 = (1.6, 0.69 * (0.95 + 0.1 * rng.random()), 0.92 * (0.95 + 0.1 * rng.random()))
    vol[_ellipsoid_mask(shape, (0, 0, 0), (a0[0], a0[2], a0[1]), 0.0)] += 1.0
    a1 = (1.5, a0[2] * 0.95, a0[1] * 0.93)
    vol[_ellipsoid_mask(shape, (0, -0.018, 0), a1, 0.0)] -= 0.8
    for _ in range(8):
        center = (rng.uniform(-0.5, 0.5), rng.uniform(-0.55, 0.55), rng.uniform(-0.45, 0.45))
        axes = (rng.uniform(0.2, 1.0), rng.uniform(0.04, 0.25), rng.uniform(0.04, 0.25))
        amp = rng.choice([-0.2, -0.1, 0.1, 0.2, 0.3])
        vol[_ellipsoid_mask(shape, center, axes, rng.uniform(0, math.pi))] += amp
    vol = np.clip(vol, 0.0, None)
    vol = vol / max(vol.max(), 1e-12) * mu_max
    return vol.astype(np.float32)


def random_ellipsoids(n_xy: int, n_z: int, seed: int, count: int = 12, mu_max: float = 0.02) -> np.ndarray:
    """Seeded random ellipsoid set inside the field of view, [n_z][n_xy][n_xy]."""
    rng = np.random.default_rng(seed)
    shape = (n_z, n_xy, n_xy)
    vol = np.zeros(shape, np.float64)
    for _ in range(count):
        r = rng.uniform(0, 0.6)
        th = rng.uniform(0, 2 * math.pi)
        center = (rng.uniform(-0.6, 0.6), r * math.sin(th), r * math.cos(th))
        axes = (rng.uniform(0.2, 1.2), rng.uniform(0.05, 0.3), rng.uniform(0.05, 0.3))
        vol[_ellipsoid_mask(shape, center, axes, rng.uniform(0, math.pi))] += rng.uniform(0.2, 1.0)
    vol = vol / max(vol.max(), 1e-12) * mu_max
    return vol.astype(np.float32)


def cahn_hilliard_frames(n_xy: int, n_z: int, n_frames: int, steps: int = 5000, seed: int = 0,
                         mobility: float = 1.0, kappa: float = 0.5, dt: float = 0.02,
                         mu_lo: float = 0.005, mu_hi: float = 0.02, device: str | None = None) -> np.ndarray:
    """Two-phase microstructure evolving over ``n_frames`` time frames.

    Explicit Euler on c_t = M lap(c^3 - c - kappa lap c) on a periodic
    [n_z][n_xy][n_xy] grid with unit spacing, started from seeded uniform noise
    in [-0.05, 0.05]; ``steps`` steps are split evenly across the frames and
    each frame is the field after its share, thresholded at 0 to mu_lo/mu_hi.
    Runs with torch on ``device`` (CUDA when available) for speed.
    Returns [n_frames][n_z][n_xy][n_xy] float32.
    """
    import torch

    dev = device or ("cuda" if torch.cuda.is_available() else "cpu")
    g = np.random.default_rng(seed)
    c = torch.tensor(g.uniform(-0.05, 0.05, size=(n_z, n_xy, n_xy)), dtype=torch.float32, device=dev)

    def lap(u):
        return (torch.roll(u, 1, 0) + torch.roll(u, -1, 0) + torch.roll(u, 1, 1) + torch.roll(u, -1, 1)
                + torch.roll(u, 1, 2) + torch.roll(u, -1, 2) - 6.0 * u)

    per = max(1, steps // n_frames)
    frames = []
    for _ in range(n_frames):
        for _ in range(per):
            c = c + dt * mobility * lap(c * c * c - c - kappa * lap(c))
        frames.append(torch.where(c > 0, mu_hi, mu_lo).to(torch.float32).cpu().numpy())
    return np.stack(frames).astype(np.float32)


def uniform_views(n_views: int, span: float = math.pi):
    """Angles uniform on [0, span), times 0..n-1, one frame covering all.

    Angles are formed in double and rounded once to float32, which reproduces
    the shipped sidecar Examples/shepp-logan-3D/proj_angles.bin (256 views).
    """
    angles = (np.arange(n_views, dtype=np.float64) * (span / n_views)).astype(np.float32)
    times = np.arange(n_views, dtype=np.float32)
    recon_times = np.array([0.0, float(n_views)], np.float32)
    return angles, times, recon_times


def interlaced_views(K: int, n_theta: int, n_p: int, proj_start: int = 0, float_arith: bool = False):
    """Bit-reversed interlaced view schedule over repeated rotations.

    Restates gen_interlaced_views_0_to_Inf with min_acq_time = 0
    (reconstruct/real_data/APS_Data_Format/XT_Views.c:7-46): view i gets angle
    (i K + bitrev_K(floor(i/L) mod K)) pi/n_theta and time (i K + bitrev)/K,
    L = n_theta/K. By default the angle is formed in double precision and
    rounded once to float32, which reproduces the shipped sidecar
    Examples/cahn-hilliard-4D/proj_angles.bin bit for bit; ``float_arith``
    instead follows XT_Views.c:11,31 literally (float pi/n_theta times a float
    count), which differs from the sidecar by one ulp on about a third of views.
    """
    L = n_theta // K
    maxbits = int(math.floor(math.log(K) / math.log(2.0) + 0.5))
    dtheta32 = np.float32(math.pi / n_theta)
    angles = np.zeros(n_p + proj_start, np.float32)
    times = np.zeros(n_p + proj_start, np.float32)
    for i in range(n_p + proj_start):
        temp = (i // L) % K
        br = 0
        for j in range(maxbits):
            if temp & (1 << j):
                br |= 1 << ((maxbits - 1) - j)
        a = np.float32(i * K + br)
        times[i] = np.float32(a / np.float32(K))
        angles[i] = np.float32(a * dtheta32) if float_arith else np.float32((i * K + br) * (math.pi / n_theta))
    return angles[proj_start:], times[proj_start:]


def poisson_measurements(ax: np.ndarray, I0: float, seed: int):
    """y = -log(N/I0), w = N with N ~ Poisson(I0 exp(-Ax)), counts clipped to >= 1."""
    rng = np.random.default_rng(seed)
    lam = I0 * np.exp(-np.asarray(ax, np.float64))
    counts = np.maximum(rng.poisson(lam), 1).astype(np.float64)
    y = (-np.log(counts / I0)).astype(np.float32)
    return y, counts.astype(np.float32)
