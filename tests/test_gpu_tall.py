"""Problems with more than 32 detector rows (thick slabs).

The reference takes any even number of rows per process
(MBIR_4D/XT_Init.c:289); the CUDA path updates a voxel column in chunks of 32
detector rows (one warp lane per row), so these tests cover the chunk
boundaries: voxel slices whose z +- 1 prior neighbour lies in the next or the
previous chunk, projections and back projections over several chunks, and the
drop-in reconstruct() against the reference's on 64 and 128 rows.

Tolerances: projections max |diff| <= 1e-6 x max |ref| (FP64 accumulation on
both sides), adjoint 1e-6 relative, reconstruct() the method's (converged cost
within 1e-4, image RMSE within 0.5 % of the range).
"""
import os

import numpy as np
import pytest

import oracle as O
import phasecon_b200 as pc
from problems import make_problem, to_gpu_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nrow,m", [(64, 1), (96, 1), (64, 2), (128, 2)])
def test_tall_forward_projection_matches_oracle(nrow, m):
    pb, _ = make_problem(ncol=32, nrow=nrow, nview=24, nframe=2, seed=nrow + m, moving=True)
    orc = O.Oracle(pb, m, m)
    x = np.random.default_rng(m).uniform(0, 0.02, orc.shape).astype(np.float32)
    o = pc.get_options()
    o.mrf_p = pb.mrf_p
    s = pc.Session(to_gpu_problem(pb), mult_xy=m, mult_z=m, options=o)
    ax = s.forward_project(x)
    ref = orc.forward(x)
    assert np.abs(ax - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("nrow", [64, 80])
def test_tall_back_projection_is_adjoint(nrow):
    pb, _ = make_problem(ncol=32, nrow=nrow, nview=30, nframe=2, seed=nrow)
    s = pc.Session(to_gpu_problem(pb))
    rng = np.random.default_rng(1)
    x = rng.uniform(0, 1, s.shape).astype(np.float32)
    y = rng.normal(0, 1, s.sino_shape).astype(np.float32)
    lhs = np.dot(s.forward_project(x).astype(np.float64).ravel(), y.astype(np.float64).ravel())
    rhs = np.dot(x.astype(np.float64).ravel(), s.back_project(y).astype(np.float64).ravel())
    assert lhs == pytest.approx(rhs, rel=1e-6)


def test_tall_icd_cost_falls_monotonically_across_chunks():
    """ICD on a 96-row, 2-frame problem: three row chunks per column; the FP64
    cost falls at every iteration (up to FP32 atomic noise) and the GPU's cost
    of its state agrees with the oracle's."""
    pb, _ = make_problem(ncol=32, nrow=96, nview=40, nframe=2, seed=9, moving=True)
    o = pc.get_options()
    o.mrf_p = pb.mrf_p
    s = pc.Session(to_gpu_problem(pb), options=o)
    costs = [s.cost()[0]]
    for it in range(1, 9):
        s.icd_iteration(it)
        costs.append(s.cost()[0])
    assert np.all(np.diff(costs) <= 1e-6 * np.array(costs[:-1])), costs
    x = s.get_object()
    orc = O.Oracle(pb)
    c_orc = orc.cost(orc.error_sino(x), x)[0]
    assert abs(costs[-1] - c_orc) / c_orc < 1e-5


@pytest.mark.skipif(not (O.ref_available() and O.ref_available(timing=True)), reason="reference build not present")
@pytest.mark.parametrize("nrow,ncol,nview", [(64, 64, 60), (128, 32, 40)])
def test_tall_reconstruct_dropin_matches_reference(tmp_path, nrow, ncol, nview):
    """reconstruct() with 64 and 128 detector rows against the reference's
    reconstruct() (its multi-resolution plan; both stop on the reference's test
    100 sum|dx| / sum|x| < 0.005)."""
    pb, _ = make_problem(ncol=ncol, nrow=nrow, nview=nview, nframe=1, seed=nrow)
    pb.convg_thresh = 0.005
    args = (pb.projections, pb.weights, pb.proj_angles, pb.proj_times, pb.recon_times, pb.proj_rows,
            pb.proj_cols, pb.proj_num, pb.recon_num, pb.vox_wid, pb.rot_center, pb.sig_s, pb.sig_t, pb.c_s,
            pb.c_t)
    cwd = os.getcwd()
    os.makedirs(tmp_path / "gpu")
    os.chdir(tmp_path / "gpu")
    saved = pc.get_options()
    try:
        pc.set_options(mrf_p=pb.mrf_p, max_iterations=200, cost_rel_tol=0.0)
        out = pc.reconstruct(*args, convg_thresh=pb.convg_thresh, remove_rings=0, quad_convex=1)
        cost = np.fromfile("cost.bin", np.float64)
    finally:
        os.chdir(cwd)
        import ctypes
        pc.lib().mbirgpu_set_options(ctypes.byref(saved))
    assert out.shape == (1, nrow + 2, ncol, ncol)
    xr, ref_cost, _ = O.ref_reconstruct_and_cost(pb, str(tmp_path / "ref"), 200, num_stages=0,
                                                 threads=os.cpu_count() or 1)
    x = out[:, 1:-1]
    assert np.sqrt(np.mean((x - xr) ** 2)) <= 0.005 * (xr.max() - xr.min())
    assert abs(cost[-1] - ref_cost) / ref_cost < 1e-4, (cost[-3:], ref_cost)
