"""Learned warm start: training pairs, the U-Net wrapper and the training loop.

The network (phasecon_b200/csrc/unet.cu, run by the library's own BF16
tensor-core kernels) maps a filtered back-projection frame to the converged
MBIR frame of the same scan. Training pairs come from seeded phantoms: the
scan is simulated with the reference's system matrix (GPU forward
projector), the input is its FBP and the target is plain GPU ICD run to the
relative-cost-change test. At use, ICD runs from the network's output to the
same convergence test, so the network only moves the starting point.
Device buffers are torch CUDA tensors (plumbing only; every operation on them
is a libmbirgpu kernel).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import phantoms as P
from .mbir import MbirError, Problem, Session, _check, get_options, lib as _mbir_lib
from .workloads import _measure

_bound = False


def lib() -> C.CDLL:
    global _bound
    L = _mbir_lib()
    if not _bound:
        vp = C.c_void_p
        L.mbirgpu_unet_create.argtypes = [C.POINTER(vp), C.c_int32, C.c_uint64, vp]
        L.mbirgpu_unet_destroy.argtypes = [vp]
        L.mbirgpu_unet_num_params.argtypes = [vp]
        L.mbirgpu_unet_num_params.restype = C.c_int64
        L.mbirgpu_unet_set_input_scale.argtypes = [vp, C.c_float]
        L.mbirgpu_unet_get_input_scale.argtypes = [vp]
        L.mbirgpu_unet_get_input_scale.restype = C.c_float
        L.mbirgpu_unet_get_params.argtypes = [vp, vp]
        L.mbirgpu_unet_set_params.argtypes = [vp, vp]
        L.mbirgpu_unet_forward.argtypes = [vp, vp, vp, C.c_int32, C.c_int32, C.c_int32]
        L.mbirgpu_unet_gradients.argtypes = [vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double), vp]
        L.mbirgpu_unet_set_tensor_path.argtypes = [vp, C.c_int32]
        L.mbirgpu_unet_get_tensor_path.argtypes = [vp]
        L.mbirgpu_unet_get_tensor_path.restype = C.c_int32
        L.mbirgpu_unet_train_step.argtypes = [vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                              C.POINTER(C.c_double)]
        L.mbirgpu_session_set_object_unet.argtypes = [vp, vp]
        _bound = True
    return L


class UNet:
    """The warm-start network (mbirgpu_unet_*)."""

    def __init__(self, base_channels: int = 16, seed: int = 0):
        self.c = base_channels
        self.h = C.c_void_p()
        _check(lib().mbirgpu_unet_create(C.byref(self.h), base_channels, seed, None))

    def close(self):
        if self.h:
            lib().mbirgpu_unet_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_params(self) -> int:
        return int(lib().mbirgpu_unet_num_params(self.h))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params, np.float32)
        _check(lib().mbirgpu_unet_get_params(self.h, p.ctypes.data))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.num_params:
            raise MbirError(f"expected {self.num_params} parameters, got {p.size}")
        _check(lib().mbirgpu_unet_set_params(self.h, p.ctypes.data))

    @property
    def input_scale(self) -> float:
        return float(lib().mbirgpu_unet_get_input_scale(self.h))

    @input_scale.setter
    def input_scale(self, s: float) -> None:
        _check(lib().mbirgpu_unet_set_input_scale(self.h, s))

    @property
    def tensor_path(self) -> int:
        """1: the 3x3x3 convolutions run on the tcgen05 kernels wherever the
        channel counts are multiples of 16 (the default); 0: on the mma.sync
        kernels everywhere."""
        return int(lib().mbirgpu_unet_get_tensor_path(self.h))

    @tensor_path.setter
    def tensor_path(self, path: int) -> None:
        _check(lib().mbirgpu_unet_set_tensor_path(self.h, int(path)))

    def save(self, path: str) -> None:
        np.savez_compressed(path, params=self.get_params(), base=self.c, scale=self.input_scale)

    @classmethod
    def load(cls, path: str) -> "UNet":
        d = np.load(path)
        u = cls(int(d["base"]))
        u.set_params(d["params"])
        u.input_scale = float(d["scale"])
        return u

    def forward(self, x):
        """x: torch CUDA float32 [D][H][W] -> network output (new tensor)."""
        import torch
        x = x.contiguous()
        out = torch.empty_like(x)
        D, H, W = x.shape
        _check(lib().mbirgpu_unet_forward(self.h, x.data_ptr(), out.data_ptr(), D, H, W))
        return out

    def gradients(self, x, t):
        """(loss, flat FP32 gradient) for one pair of torch CUDA tensors."""
        D, H, W = x.shape
        g = np.zeros(self.num_params, np.float32)
        loss = C.c_double()
        _check(lib().mbirgpu_unet_gradients(self.h, x.contiguous().data_ptr(), t.contiguous().data_ptr(), D, H, W,
                                            C.byref(loss), g.ctypes.data))
        return loss.value, g

    def train_step(self, x, t, lr: float) -> float:
        D, H, W = x.shape
        loss = C.c_double()
        _check(lib().mbirgpu_unet_train_step(self.h, x.data_ptr(), t.data_ptr(), D, H, W, lr, C.byref(loss)))
        return loss.value


def warm_start(session: Session, net: UNet) -> None:
    """The session's object becomes net(FBP) per frame (e = y - A x recomputed)."""
    _check(lib().mbirgpu_session_set_object_unet(session.h, net.h))


def converge(session: Session, max_iter: int = 200, rel: float = 1e-4, start_iter: int = 1):
    """Plain ICD until the relative FP64 cost change is below `rel`; returns
    (iterations, cost history)."""
    costs = [session.cost()[0]]
    it = 0
    while it < max_iter:
        it += 1
        session.icd_iteration(start_iter + it - 1)
        costs.append(session.cost()[0])
        if it > 1 and abs(costs[-2] - costs[-1]) < rel * abs(costs[-1]):
            break
    return it, costs


def iterations_to_cost(session: Session, target: float, max_iter: int = 300):
    """Plain ICD iterations until the FP64 cost is at most `target` (for a
    warm start: the plain method's converged cost times 1 + 1e-4); returns
    (iterations, cost history) or (None, history) if it never does."""
    costs = [session.cost()[0]]
    if costs[0] <= target:
        return 0, costs
    for it in range(1, max_iter + 1):
        session.icd_iteration(it)
        costs.append(session.cost()[0])
        if costs[-1] <= target:
            return it, costs
    return None, costs


def frame_views(frame: int = 0, K: int = 8, n_theta: int = 256, n_p: int = 1024, frames: int = 8):
    """The views of one frame of the 4-D schedule (interlaced, 128 per frame)."""
    angles, times = P.interlaced_views(K, n_theta, n_p)
    edges = np.linspace(0.0, float(n_p), frames + 1)
    sel = (times >= edges[frame]) & (times < edges[frame + 1])
    a = np.ascontiguousarray(angles[sel])
    t = np.ascontiguousarray(times[sel] - edges[frame]).astype(np.float32)
    return a, t, np.array([0.0, float(edges[frame + 1] - edges[frame])], np.float32)


def training_pair(seed: int, n_xy: int = 256, n_z: int = 32, kind: str = "mixed", I0: float = 2e4,
                  p: float = 1.2, icd_rel: float = 1e-4):
    """(FBP input, converged ICD target, phantom), each [n_z][n_xy][n_xy] float32,
    for one seeded phantom scanned with one frame's views of the 4-D schedule."""
    rng = np.random.default_rng(seed)
    k = kind if kind != "mixed" else ("ch" if rng.random() < 0.5 else "ellipsoids")
    if k == "ch":
        obj = P.cahn_hilliard_frames(n_xy, n_z, 1, steps=int(rng.integers(300, 1200)), seed=seed)[0]
    else:
        obj = P.random_ellipsoids(n_xy, n_z, seed)
    a, t, rt = frame_views(int(rng.integers(0, 8)))
    nv = a.size
    z = np.zeros((nv, n_z, n_xy), np.float32)
    pb = Problem(z, np.ones_like(z), a, t, rt, n_z, n_xy, nv, 1, rot_center=n_xy / 2, sig_s=0.01, sig_t=1.0,
                 c_s=1.0, c_t=1.0)
    pb = _measure(pb, obj[None], I0, seed)
    o = get_options()
    o.mrf_p = p
    s = Session(pb, options=o)
    fbp = s.fbp()[0]
    s.set_object_zero()
    converge(s, rel=icd_rel)
    target = s.get_object()[0]
    s.close()
    return fbp.astype(np.float32), target.astype(np.float32), obj.astype(np.float32)


def training_pairs_4d(seed: int, ch_steps: int | None = None, rel: float = 1e-4):
    """The 8 (FBP frame, converged frame) pairs of one seeded 4-D scan with the
    4-D workload's geometry and schedule (Cahn-Hilliard evolution, 1,024
    interlaced views, Poisson I0 = 2e4): targets from plain GPU ICD on the
    whole 4-D problem, temporal prior included."""
    from .workloads import config_4d
    rng = np.random.default_rng(seed)
    steps = ch_steps if ch_steps is not None else int(rng.integers(2000, 8001))
    pb, _, p = config_4d(seed=seed, ch_steps=steps)
    o = get_options()
    o.mrf_p = p
    s = Session(pb, options=o)
    fbp = s.fbp()
    s.set_object_zero()
    converge(s, rel=rel)
    target = s.get_object()
    s.close()
    return [(fbp[f], target[f]) for f in range(fbp.shape[0])]


def warm_start_score(session: Session, net: UNet, icd_iterations: int = 0) -> float:
    """The MAP cost a warm start leaves on a held-out scan: the session's object
    becomes net(FBP), then `icd_iterations` plain ICD iterations run (none by
    default: two ICD iterations already level the candidates' costs to within
    0.2 %, while the starting costs differ by 10 % and more and set how many
    iterations the start needs); returns the FP64 cost (lower is better): the
    MAP cost function is the measure of the network's error."""
    warm_start(session, net)
    for it in range(1, icd_iterations + 1):
        session.icd_iteration(it)
    return float(session.cost()[0])


def train(net: UNet, pairs, steps: int, lr: float = 1e-3, seed: int = 0, log_every: int = 0,
          average_from: float = 1.0, average_every: int = 50, val_pairs=None, val_every: int = 250,
          val_session: Session | None = None, scores: list | None = None, warmup: int = 0):
    """Adam steps over randomly drawn (input, target) pairs of host arrays;
    returns the loss history. The network's input scale is set so that it
    sees values of order one. Learning rate: a cosine schedule from `lr` down
    to lr / 100 over all steps; with average_from < 1, the cosine runs down to
    lr / 10 over the first average_from of the steps, the rest run at lr / 10
    and the network ends as the average of its weights taken every
    `average_every` steps over that tail (stochastic weight averaging). The
    first `warmup` steps ramp the rate up linearly from lr / warmup.

    With `val_session` (a session on a held-out scan, never trained on) or
    `val_pairs` (held-out pairs) the network ends as the candidate with the
    lowest score, the candidates being the weights every `val_every` steps
    from a quarter of the run on, the running weight average at the same
    points of the tail, and the final weights: single-sample Adam steps
    occasionally land on a worse point late in a run. The score is the MAP
    cost the warm start leaves on the held-out scan (warm_start_score) when a
    session is given, else the mean loss on the held-out pairs. `scores`, when given, receives (step, averaged, score)
    for every candidate and the index of the chosen one last."""
    import torch
    rng = np.random.default_rng(seed)
    net.input_scale = 1.0 / max(float(np.mean([np.abs(t).max() for _, t in pairs])), 1e-12)

    def to_dev(ps):
        return [(torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda(),
                 torch.from_numpy(np.ascontiguousarray(t, np.float32)).cuda()) for x, t in ps]

    dev = to_dev(pairs)
    val = to_dev(val_pairs) if (val_pairs and val_session is None) else []
    best = [np.inf, None]

    chosen = [None]

    def consider(params, step=-1, averaged=False):
        keep = net.get_params()
        net.set_params(params.astype(np.float32))
        if val_session is not None:
            score = warm_start_score(val_session, net)
        else:
            score = float(np.mean([net.gradients(x, t)[0] for x, t in val]))
        net.set_params(keep)
        if scores is not None:
            scores.append((step, averaged, score))
        if score < best[0]:
            best[0], best[1] = score, params.astype(np.float32).copy()
            chosen[0] = len(scores) - 1 if scores is not None else None

    hist = []
    tail = int(average_from * steps) if average_from < 1.0 else steps
    avg, navg = None, 0
    for s in range(steps):
        x, t = dev[int(rng.integers(0, len(dev)))]
        if tail < steps:
            lr_s = lr * 0.1 if s >= tail else lr * (0.1 + 0.9 * 0.5 * (1.0 + np.cos(np.pi * s / max(1, tail))))
        else:
            lr_s = lr * (0.01 + 0.99 * 0.5 * (1.0 + np.cos(np.pi * s / max(1, steps))))
        if s < warmup:
            lr_s *= (s + 1) / warmup
        hist.append(net.train_step(x, t, float(lr_s)))
        if s >= tail and (s - tail) % average_every == average_every - 1:
            p = net.get_params().astype(np.float64)
            avg = p if avg is None else avg + p
            navg += 1
        if (val or val_session is not None) and s >= steps // 4 and (s + 1) % val_every == 0:
            consider(net.get_params(), s + 1)
            if navg:
                consider(avg / navg, s + 1, True)
        if log_every and (s + 1) % log_every == 0:
            print(f"step {s + 1}: loss {np.mean(hist[-log_every:]):.4g}", flush=True)
    if navg:
        net.set_params((avg / navg).astype(np.float32))
    if val or val_session is not None:
        consider(net.get_params(), steps, navg > 0)
        net.set_params(best[1])
        if scores is not None:
            scores.append(chosen[0])
    return hist
