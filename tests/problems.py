"""Small seeded MBIR problems for the parity tests (built with the oracle's projector)."""
from __future__ import annotations

import numpy as np

import oracle as O
from phasecon_b200 import phantoms as P


def make_problem(ncol=32, nrow=8, nview=40, nframe=1, seed=0, p=1.2, I0=1e4, sig_s=0.01, sig_t=0.01,
                 c_s=1.0, c_t=1.0, quad_convex=1, huber_delta=0.5, huber_T=4.0, moving=False):
    """A seeded ellipsoid phantom, parallel beam over [0, pi), Poisson data.

    Returns (oracle Problem, true object [nframe][nrow][ncol][ncol]). With
    ``moving`` each frame's phantom differs (seed + frame).
    """
    ang, t, rt = P.uniform_views(nview)
    if nframe > 1:
        rt = np.linspace(0, nview, nframe + 1).astype(np.float32)
    pb = O.Problem(np.zeros((nview, nrow, ncol), np.float32), np.ones((nview, nrow, ncol), np.float32), ang, t, rt,
                   nrow, ncol, nview, nframe, rot_center=ncol / 2, sig_s=sig_s, sig_t=sig_t, c_s=c_s, c_t=c_t,
                   mrf_p=p, quad_convex=quad_convex, huber_delta=huber_delta, huber_T=huber_T)
    orc = O.Oracle(pb)
    vols = [P.ellipsoid_phantom(ncol, nrow, seed + (f if moving else 0)) for f in range(nframe)]
    obj = np.stack(vols).astype(np.float32)
    ax = orc.forward(obj)
    y, w = P.poisson_measurements(ax, I0, seed)
    pb.projections = np.ascontiguousarray(y.transpose(0, 2, 1))
    pb.weights = np.ascontiguousarray(w.transpose(0, 2, 1))
    return pb, obj


def to_gpu_problem(pb):
    from phasecon_b200 import Problem
    return Problem(pb.projections, pb.weights, pb.proj_angles, pb.proj_times, pb.recon_times, pb.proj_rows,
                   pb.proj_cols, pb.proj_num, pb.recon_num, pb.vox_wid, pb.rot_center, pb.sig_s, pb.sig_t, pb.c_s,
                   pb.c_t, pb.convg_thresh, pb.quad_convex, pb.huber_delta, pb.huber_T)
