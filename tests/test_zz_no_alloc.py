"""The allocation-free forward projection agrees with the session's forward projection.

Collected last on purpose: the library's fixed device scratch is then reused
after every other GPU test of the run, and the test must pass alone as well.
Tolerance: both paths accumulate in FP64 with atomic reductions (order
varies), then round to float once: max |diff| <= 1e-6 x max |A x|.
"""
import numpy as np
import pytest

import phasecon_b200 as pc
from problems import make_problem, to_gpu_problem

pytestmark = pytest.mark.gpu


def _device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def test_forward_project_noalloc_matches_session_projection_twice_in_a_row():
    import torch
    pb, obj = make_problem(ncol=32, nrow=8, nview=40, nframe=2, moving=True, seed=3)
    s = pc.Session(to_gpu_problem(pb))
    rng = np.random.default_rng(5)
    objects = [obj, (obj * rng.uniform(0.5, 1.5, obj.shape)).astype(np.float32)]
    for o in objects:
        ref = s.forward_project(o)
        x = _device(o)
        out = torch.full(s.sino_shape, float("nan"), device="cuda")
        torch.cuda.synchronize()
        s.forward_project_noalloc(x.data_ptr(), out.data_ptr())
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_forward_project_noalloc_rejects_sessions_beyond_the_scratch():
    import torch
    V, rows, cols = 1100, 32, 64  # 2,252,800 sinogram entries > 2,097,152
    ang = np.linspace(0, np.pi, V, endpoint=False).astype(np.float32)
    prob = pc.Problem(np.zeros((V, rows, cols), np.float32), np.ones((V, rows, cols), np.float32), ang,
                      np.arange(V, dtype=np.float32), np.array([0, V], np.float32), rows, cols, V, 1,
                      rot_center=cols / 2)
    s = pc.Session(prob)
    x = torch.zeros(s.shape, device="cuda")
    out = torch.zeros(s.sino_shape, device="cuda")
    with pytest.raises(pc.MbirError, match="fixed scratch holds at most 2097152"):
        s.forward_project_noalloc(x.data_ptr(), out.data_ptr())
