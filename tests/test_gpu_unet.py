"""The learned warm start: FBP, the U-Net's BF16 tensor-core kernels against the
FP64 oracle, training, and what the trained network gains.

Tolerances: loss within 1e-3 relative of the oracle's; every layer's weight
and bias gradient within 5e-2 relative L2 error and cosine similarity >= 0.995
(the oracle rounds to BF16 where the GPU stores BF16, so the remaining
difference is FP32 accumulation order plus the rare BF16 rounding flip it
causes); FBP of a uniform cylinder within 5 % of the true value inside.
"""
import numpy as np
import pytest

import unet_oracle as UO
import phasecon_b200 as pc
from phasecon_b200 import phantoms as P
from phasecon_b200 import warmstart as WS
from phasecon_b200.workloads import _measure

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()


@pytest.mark.parametrize("c,shape", [(4, (8, 8, 8)), (8, (16, 16, 8)), (16, (16, 24, 40))])
def test_unet_gradients_match_fp64_oracle(c, shape):
    """c = 4 and 8 run the mma.sync convolutions; c = 16 runs every 3x3x3
    convolution but the first (one input channel) on the tcgen05 kernels,
    forward and data gradient, on a grid whose y and x are not multiples of
    the tile at any level."""
    rng = np.random.default_rng(c)
    net = WS.UNet(c, seed=3)
    net.input_scale = 50.0
    params = net.get_params()
    params[-c - 1:-1] = rng.normal(0, 0.3, c)  # a head with real weight: every layer's gradient matters
    params[-1] = 0.01
    net.set_params(params)
    x = (0.01 + 0.01 * rng.random(shape)).astype(np.float32)
    t = (x + 0.003 * rng.normal(size=shape)).astype(np.float32)
    loss, g = net.gradients(_dev(x), _dev(t))
    lo, go = UO.forward_backward(net.get_params(), c, x, t, bf16=True, scale=50.0)
    assert loss == pytest.approx(lo, rel=1e-3)
    off = 0
    for k, (cin, cout) in enumerate(UO.layer_shapes(c) + [(c, 1)]):
        sizes = (27 * cin * cout, cout) if k < 17 else (c, 1)
        for m in sizes:
            a, b = g[off:off + m].astype(np.float64), go[off:off + m]
            off += m
            if np.abs(b).max() == 0:
                assert np.abs(a).max() == 0
                continue
            rel = np.linalg.norm(a - b) / np.linalg.norm(b)
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
            assert rel < 5e-2 and cos >= 0.995, (k, m, rel, cos)
    assert off == net.num_params


def test_unet_training_reduces_the_loss():
    rng = np.random.default_rng(1)
    shape = (8, 32, 32)
    net = WS.UNet(4, seed=1)
    _, yy, xx = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    t = (0.02 * ((yy - 16) ** 2 + (xx - 16) ** 2 < 100)).astype(np.float32)
    x = (t + 0.004 * rng.normal(size=shape)).astype(np.float32)
    hist = WS.train(net, [(x, t)], steps=120, lr=2e-3)
    assert np.mean(hist[-10:]) < 0.5 * np.mean(hist[:3]), (hist[:3], hist[-10:])


def test_fbp_of_a_uniform_cylinder():
    n, nz, nv = 64, 8, 180
    angles, times, rt = P.uniform_views(nv)
    jj, kk = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    r2 = (jj - n / 2 + 0.5) ** 2 + (kk - n / 2 + 0.5) ** 2
    obj = np.repeat(((r2 < (0.3 * n) ** 2) * 0.02).astype(np.float32)[None], nz, 0)[None]
    z = np.zeros((nv, nz, n), np.float32)
    pb = pc.Problem(z, np.ones_like(z), angles, times, rt, nz, n, nv, 1, rot_center=n / 2)
    sino = pc.Session(pb).forward_project(obj)  # [view][col][row]
    pb.projections = np.ascontiguousarray(sino.transpose(0, 2, 1))
    f = pc.Session(pb).fbp()[0]
    assert abs(f[:, r2 < (0.2 * n) ** 2].mean() - 0.02) < 0.05 * 0.02
    assert np.abs(f[:, r2 > (0.4 * n) ** 2]).mean() < 0.1 * 0.02


def _small_problem(seed, n=64, nz=8):
    a, t, rt = WS.frame_views(seed % 8)
    nv = a.size
    z = np.zeros((nv, nz, n), np.float32)
    pb = pc.Problem(z, np.ones_like(z), a, t, rt, nz, n, nv, 1, rot_center=n / 2, sig_s=0.01, sig_t=1.0, c_s=1.0,
                    c_t=1.0)
    return _measure(pb, P.random_ellipsoids(n, nz, seed)[None], 2e4, seed)


def test_trained_warm_start_needs_fewer_iterations():
    """ICD from the trained network's output reaches the plain method's
    converged cost (within 1e-4 relative) in fewer iterations than from zero."""
    o = pc.get_options()
    o.nhicd_passes = 0
    pairs = []
    for seed in range(6):
        s = pc.Session(_small_problem(seed), options=o)
        fbp = s.fbp()[0]
        s.set_object(np.zeros(s.shape, np.float32))
        WS.converge(s, rel=1e-5)
        pairs.append((fbp, s.get_object()[0]))
        s.close()
    net = WS.UNet(8, seed=0)
    WS.train(net, pairs, steps=400, lr=1e-3)
    s = pc.Session(_small_problem(100), options=o)
    s.set_object(np.zeros(s.shape, np.float32))
    _, c_conv = WS.converge(s, rel=1e-7, max_iter=300)  # the converged cost of the plain method
    target = c_conv[-1] * (1 + 1e-4)
    s.set_object(np.zeros(s.shape, np.float32))
    it_zero, c_zero = WS.iterations_to_cost(s, target)
    s.set_object_fbp()
    it_fbp, _ = WS.iterations_to_cost(s, target)
    WS.warm_start(s, net)
    it_net, c_net = WS.iterations_to_cost(s, target)
    print(f"iterations to the plain method's converged cost: zero {it_zero}, FBP {it_fbp}, U-Net {it_net}")
    assert it_zero is not None and it_net is not None and it_net < it_zero, (it_net, it_fbp, it_zero)
    assert c_net[0] < c_zero[0]


@pytest.mark.parametrize("c", [8, 16])
def test_stacked_frame_inference_equals_per_frame(c):
    """The warm start runs the network on all frames of a 4-D problem in one
    stacked pass (zero padding per frame); every voxel must equal the
    one-frame-at-a-time network output bit for bit (same tiles, same sums).
    c = 16 runs the tcgen05 convolutions, whose TMA halo loads zero-fill per
    frame."""
    import torch
    n, nz, frames = 32, 16, 3
    angles, times, rt = P.uniform_views(60)
    times = np.linspace(0, frames, angles.size, endpoint=False).astype(np.float32)
    rt = np.linspace(0, frames, frames + 1).astype(np.float32)
    z = np.zeros((angles.size, nz, n), np.float32)
    pb = pc.Problem(z, np.ones_like(z), angles, times, rt, nz, n, angles.size, frames, rot_center=n / 2)
    obj = np.stack([P.random_ellipsoids(n, nz, s) for s in range(frames)])
    pb = _measure(pb, obj, 2e4, 0)
    s = pc.Session(pb)
    fbp = s.fbp()
    net = WS.UNet(c, seed=2)
    params = net.get_params()
    params[-c - 1:-1] = np.random.default_rng(0).normal(0, 0.3, c)  # a head with weight: the network matters
    net.set_params(params)
    net.input_scale = 40.0
    WS.warm_start(s, net)
    got = s.get_object()
    inside = got != 0
    assert inside.mean() > 0.4
    for f in range(frames):
        exp = net.forward(torch.from_numpy(np.ascontiguousarray(fbp[f])).cuda()).cpu().numpy()
        np.testing.assert_array_equal(got[f][inside[f]], exp[inside[f]])
    s.close()


@pytest.mark.parametrize("shape", [(16, 24, 40), (32, 64, 64)])
def test_tensor_path_matches_mma_sync(shape):
    """The tcgen05 convolutions (TMEM accumulators, TMA-staged halo and
    weights) against the mma.sync kernels on the same BF16 weights and input:
    both accumulate BF16 products in FP32, in different orders, and round each
    layer's activations to BF16, so the networks' corrections agree to 1e-2
    relative L2 (an occasional BF16 rounding flip per layer), and the
    tcgen05 path is deterministic run to run."""
    import torch
    rng = np.random.default_rng(7)
    net = WS.UNet(16, seed=5)
    params = net.get_params()
    params[-17:-1] = rng.normal(0, 0.3, 16)
    net.set_params(params)
    net.input_scale = 50.0
    x = torch.from_numpy((0.01 + 0.01 * rng.random(shape)).astype(np.float32)).cuda()
    assert net.tensor_path == 1
    a = net.forward(x).cpu().numpy() - x.cpu().numpy()
    a2 = net.forward(x).cpu().numpy() - x.cpu().numpy()
    net.tensor_path = 0
    b = net.forward(x).cpu().numpy() - x.cpu().numpy()
    net.tensor_path = 1
    np.testing.assert_array_equal(a, a2)
    assert np.abs(b).max() > 0
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel < 1e-2, rel

