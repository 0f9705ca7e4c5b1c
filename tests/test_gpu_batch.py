"""The batched persistent ICD (mbirgpu_batch_*) against one-problem sessions.

Each member of a batch runs the same super-voxel algorithm (same schedule,
same seeds) as a session with the same super-voxel size and CTA width. Which
super-voxels run at the same moment differs (and varies from run to run in
both), so the trajectories differ slightly; after 40 iterations both are
converged: final FP64 cost within 2e-4 relative, object RMSE within 0.5 % of
its dynamic range (the ICD tolerance used against the reference).
"""
import numpy as np
import pytest

import phasecon_b200 as pc
from phasecon_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small_batch():
    return W.config_batch(seed=3, n=5, edges=(32, 48, 64), depth=(6, 12), views=(40, 90))


def test_batch_matches_single_sessions():
    probs = small_batch()
    assert {p.proj_rows % 4 == 0 for p in probs} == {True, False}  # both record classes
    o = pc.get_options()
    o.sv_size, o.cta_warps, o.sv_colors, o.nhicd_passes, o.refresh_every = 8, 4, 2, 0, 4
    b = pc.Batch(probs, options=o)
    n_it = 40
    st = b.run(n_it)
    assert st.graph_launches == n_it and st.sv_size == 8 and st.cta_warps == 4
    for i, p in enumerate(probs):
        s = pc.Session(p, options=o)
        for it in range(1, n_it + 1):
            s.icd_iteration(it)
        c_single = s.cost()[0]
        c_batch = b.cost(i)
        assert abs(c_batch - c_single) <= 2e-4 * abs(c_single), (i, c_batch, c_single)
        xs, xb = s.get_object(), b.get_object(i)
        assert np.sqrt(np.mean((xs - xb) ** 2)) <= 0.005 * max(xs.max() - xs.min(), 1e-12)
        _, iters, conv = b.info(i)
        assert iters == n_it and not conv
    assert st.voxel_updates > 0


def test_batch_autotuner_and_per_problem_convergence():
    probs = small_batch()
    probs[1].convg_thresh = 1000.0  # 100 sum|dx| / sum|x| is below that after any iteration: stops after the 2nd
    b = pc.Batch(probs)
    st = b.run(6)
    assert st.sv_size in (4, 8, 16) and st.cta_warps in (2, 4)
    _, iters, conv = b.info(1)
    assert conv and iters == 2
    _, iters0, conv0 = b.info(0)
    assert iters0 == 6 and not conv0
    st2 = b.run(2)  # continues where it stopped
    assert st2.voxel_updates > st.voxel_updates
    assert b.info(0)[1] == 8 and b.info(1)[1] == 2


def test_reconstruct_batch_layout():
    import ctypes
    probs = small_batch()[:3]
    saved = pc.get_options()
    try:
        pc.set_options(sv_size=8, cta_warps=4, sv_colors=2)  # the same schedule in both runs below
        outs = pc.reconstruct_batch(probs, 20)
        b = pc.Batch(probs)
        b.run(20)
    finally:
        pc.lib().mbirgpu_set_options(ctypes.byref(saved))
    for i, (p, o) in enumerate(zip(probs, outs)):
        assert o.shape == (1, p.proj_rows + 2, p.proj_cols, p.proj_cols)
        assert np.all(o[:, 0] == 0) and np.all(o[:, -1] == 0)
        x = b.get_object(i)  # runs differ only by which SVs run at the same moment
        assert np.sqrt(np.mean((o[:, 1:-1] - x) ** 2)) <= 0.005 * max(x.max() - x.min(), 1e-12)
