"""FP64 numpy reference of the warm-start U-Net (forward and backward).

TEST INFRASTRUCTURE ONLY: the checker for the GPU network kernels (BF16
tensor-core convolutions) in phasecon_b200/csrc/unet.cu. The network has no
counterpart in phasecon; it is restated here from its definition: four levels
of c, 2c, 4c, 8c channels, two 3x3x3 convolutions + ReLU per encoder level,
2x2x2 max-pooling, nearest 2x upsampling + 3x3x3 convolution + ReLU,
concatenation [upsampled, skip], two 3x3x3 convolutions + ReLU per decoder
level, a 1x1x1 head added to the input; loss mean((out - target)^2). Its
gradient is pinned by central finite differences (tests/test_oracle_unet.py).

With ``bf16=True`` the values the GPU stores in BF16 (weights, activations,
activation gradients) are rounded to BF16 at the same points, so the
remaining differences are FP32-vs-FP64 accumulation only.
Parameter layout (flat, layer order): per convolution w[27][cin][cout] then
b[cout]; head w[c], head b[1].
"""
from __future__ import annotations

import numpy as np


def to_bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layer_shapes(c: int):
    C = [c, 2 * c, 4 * c, 8 * c]
    convs = []
    for l in range(4):
        convs.append((1 if l == 0 else C[l - 1], C[l]))
        convs.append((C[l], C[l]))
    for l in (2, 1, 0):
        convs += [(C[l + 1], C[l]), (2 * C[l], C[l]), (C[l], C[l])]
    return convs


def unpack(params, c):
    out, off = [], 0
    for cin, cout in layer_shapes(c):
        w = params[off:off + 27 * cin * cout].reshape(27, cin, cout)
        off += 27 * cin * cout
        b = params[off:off + cout]
        off += cout
        out.append((w, b))
    hw = params[off:off + c]
    hb = params[off + c]
    return out, hw, hb


def _shift(x, tap):
    """x[z+dz, y+dy, x+dx] with zero padding; x is [D, H, W, C]."""
    dz, dy, dx = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
    D, H, W = x.shape[:3]
    out = np.zeros_like(x)
    zs, ys, xs = (slice(max(0, -dz), D - max(0, dz)), slice(max(0, -dy), H - max(0, dy)),
                  slice(max(0, -dx), W - max(0, dx)))
    zd, yd, xd = (slice(max(0, dz), D - max(0, -dz)), slice(max(0, dy), H - max(0, -dy)),
                  slice(max(0, dx), W - max(0, -dx)))
    out[zs, ys, xs] = x[zd, yd, xd]
    return out


def conv(x, w, b):
    out = np.zeros(x.shape[:3] + (w.shape[2],))
    for t in range(27):
        out += _shift(x, t) @ w[t]
    return out + b


def conv_back(x, w, g):
    """(dx, dw, db) of out = conv(x, w, b) given g = d loss / d out."""
    dw = np.zeros_like(w)
    dx = np.zeros_like(x)
    for t in range(27):
        dw[t] = np.einsum("zyxi,zyxo->io", _shift(x, t), g)
        # out[v] += x[v + off] w  =>  dx[u] += g[u - off] w^T
        dx += _shift(g @ w[t].T, 26 - t)
    return dx, dw, g.sum(axis=(0, 1, 2))


def pool(x):
    D, H, W, C = x.shape
    return x.reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).max(axis=(1, 3, 5))


def pool_back(x, p, g):
    """Gradient to the first (z, y, x order) input of each block holding the max."""
    out = np.zeros_like(x)
    done = np.zeros(p.shape, bool)
    for q in range(8):
        a, b, c = q >> 2, (q >> 1) & 1, q & 1
        hit = (~done) & (x[a::2, b::2, c::2] == p)
        out[a::2, b::2, c::2] = np.where(hit, g, 0.0)
        done |= hit
    return out


def up(x):
    return x.repeat(2, 0).repeat(2, 1).repeat(2, 2)


def up_back(g):
    D, H, W, C = g.shape
    return g.reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(1, 3, 5))


def forward_backward(params, c, inp, target, bf16=True, scale=1.0):
    """Loss and flat gradient for one input [D][H][W] (FP64). The network sees
    scale x input and the head's correction is divided by scale."""
    R = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    layers, hw, hb = unpack(np.asarray(params, np.float64), c)
    Wq = [(R(w), b) for w, b in layers]
    C = [c, 2 * c, 4 * c, 8 * c]
    x0 = R(np.float32(scale) * np.asarray(inp, np.float32)[..., None])
    acts, i = {}, 0

    def cr(x, k):
        w, b = Wq[k]
        return R(np.maximum(conv(x, w, b), 0.0))

    x = x0
    for l in range(4):
        a = cr(x, i)
        i += 1
        s = cr(a, i)
        i += 1
        acts[("enc", l)] = (x, a, s)
        if l < 3:
            x = R(pool(s))
            acts[("pool", l)] = x
    y = acts[("enc", 3)][2]
    for l in (2, 1, 0):
        u_in = R(up(y))
        u = cr(u_in, i)
        i += 1
        cat = np.concatenate([u, acts[("enc", l)][2]], axis=-1)
        d1 = cr(cat, i)
        i += 1
        d2 = cr(d1, i)
        i += 1
        acts[("dec", l)] = (u_in, u, cat, d1, d2)
        y = d2
    out = np.asarray(inp, np.float64) + (hb + y @ hw) / scale
    diff = out - np.asarray(target, np.float64)
    V = diff.size
    loss = float(np.mean(diff ** 2))
    gout = 2.0 * diff / V / scale
    grads = [None] * len(Wq)
    ghw = np.einsum("zyxc,zyx->c", y, gout)
    ghb = gout.sum()
    gy = R(gout[..., None] * hw)

    def cb(k, xin, o, go, need_dx=True):
        go = np.where(o > 0, go, 0.0)
        dx, dw, db = conv_back(xin, Wq[k][0], go)
        grads[k] = (dw, db)
        return R(dx) if need_dx else None

    i = len(Wq) - 1
    gskip = {}
    for l in (0, 1, 2):
        u_in, u, cat, d1, d2 = acts[("dec", l)]
        g1 = cb(i, d1, d2, gy)
        i -= 1
        gcat = cb(i, cat, d1, g1)
        i -= 1
        gskip[l] = gcat[..., C[l]:]
        gup = cb(i, u_in, u, gcat[..., :C[l]])
        i -= 1
        gy = R(up_back(gup))
    g, gpool = gy, None  # gradient of the bottleneck output
    for l in (3, 2, 1, 0):
        xin, a, s = acts[("enc", l)]
        if l < 3:
            g = R(gskip[l] + pool_back(s, acts[("pool", l)], gpool))
        ga = cb(i, a, s, g)
        i -= 1
        gpool = cb(i, xin, a, ga, need_dx=l > 0)
        i -= 1
    flat = []
    for dw, db in grads:
        flat += [dw.ravel(), db.ravel()]
    flat += [ghw.ravel(), np.array([ghb])]
    return loss, np.concatenate(flat)
