"""Noise-variance re-estimation of the generalised-Huber data term on the GPU
against the reference C (update_variance_parameter, MBIR_4D/XT_ICD_update.c:716-747).

Two successive re-estimations on the same error sinogram (the second one on the
weights the first one rescaled): each variance within 1e-6 relative of the
reference's (FP64 sums in another order; the reference forms some products in
float). The drop-in reconstruct with quad_convex = 0 (the variance is
re-estimated in every iteration after the first multires stage) against the
reference's own reconstruct: final cost within 2e-3 at the reference's stop,
and the written variance_estimate within 2e-2 relative with both runs taken
to a tight stop (the estimate drifts while the image converges; see the test).
"""
import os

import numpy as np
import pytest

import oracle as O
import phasecon_b200 as pc
from problems import make_problem, to_gpu_problem

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_variance_update_matches_reference():
    pb, obj = make_problem(ncol=64, nrow=8, nview=60, nframe=1, seed=5, quad_convex=0, huber_T=2.0, huber_delta=0.2)
    o = pc.get_options()
    o.mrf_p = pb.mrf_p
    s = pc.Session(to_gpu_problem(pb), options=o)
    s.set_object((0.8 * obj).astype(np.float32))
    e0 = s.get_error()
    w0 = np.ascontiguousarray(pb.weights.transpose(0, 2, 1))
    assert s.variance == 1.0
    v1 = s.update_variance()
    w1r, v1r = O.ref_variance_update(pb, e0, w0, 1.0)
    assert v1 == pytest.approx(v1r, rel=1e-6)
    assert v1 != pytest.approx(1.0, rel=1e-3)
    v2 = s.update_variance()
    _, v2r = O.ref_variance_update(pb, e0, w1r, v1r)
    assert v2 == pytest.approx(v2r, rel=1e-6)
    s.close()


def gpu_reconstruct(pb, tmp_path, convg_thresh, max_iterations):
    args = (pb.projections, pb.weights, pb.proj_angles, pb.proj_times, pb.recon_times, pb.proj_rows,
            pb.proj_cols, pb.proj_num, pb.recon_num, pb.vox_wid, pb.rot_center, pb.sig_s, pb.sig_t, pb.c_s, pb.c_t)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    saved = pc.get_options()
    try:
        pc.set_options(mrf_p=pb.mrf_p, max_iterations=max_iterations, cost_rel_tol=0.0)
        pc.reconstruct(*args, convg_thresh=convg_thresh, remove_rings=0, quad_convex=0, huber_delta=0.2, huber_T=2.0)
        cost = np.fromfile("cost.bin", np.float64)
        var = np.fromfile("variance_estimate.bin", np.float64)[0]
    finally:
        os.chdir(cwd)
        import ctypes
        pc.lib().mbirgpu_set_options(ctypes.byref(saved))
    return cost, var


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_reconstruct_huber_with_variance_matches_reference(tmp_path):
    """Final cost at the reference's loose stop (convg_thresh 0.05 %, the build
    with the cost pass) within 2e-3; the variance estimate with both runs
    taken further (convg_thresh 0.002 %, the reference as it ships, without
    the cost pass whose rounding-level 'cost increased' check stops it early)
    within 2e-2. The estimate is re-taken from the residual in every
    iteration, so it drifts slowly while the image converges: measured, the
    reference's own estimate moves by 0.6 % between stops at 0.05 %, 0.01 %
    and 0.002 % (0.5854, 0.5817, 0.5834), the GPU's by up to 0.5 % run to run
    at one stop (0.5867-0.5893, the order of its concurrent updates), and the
    two lie 0.5-1.0 % apart."""
    pb, _ = make_problem(ncol=64, nrow=8, nview=60, nframe=1, seed=5, quad_convex=0, huber_T=2.0, huber_delta=0.2)
    pb.convg_thresh = 0.05
    (tmp_path / "loose").mkdir()
    cost, _ = gpu_reconstruct(pb, tmp_path / "loose", 0.05, 60)
    _, ref_cost, _ = O.ref_reconstruct(pb, str(tmp_path / "ref_loose"), max_iter=60)
    assert abs(cost[-1] - ref_cost[-1]) / abs(ref_cost[-1]) < 2e-3, (cost[-1], ref_cost[-1])

    pb.convg_thresh = 0.002
    (tmp_path / "tight").mkdir()
    _, var = gpu_reconstruct(pb, tmp_path / "tight", 0.002, 400)
    wd = str(tmp_path / "ref_tight")
    O.ref_reconstruct(pb, wd, max_iter=400, timing=True)
    ref_var = np.fromfile(os.path.join(wd, "variance_estimate.bin"), np.float64)[0]
    assert ref_var != pytest.approx(1.0, rel=1e-3)
    assert var == pytest.approx(ref_var, rel=2e-2)
