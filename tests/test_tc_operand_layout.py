"""The shared-memory operand layout of the tcgen05 convolution kernel
(phasecon_b200/csrc/unet_tc.cu), checked on the CPU.

The kernel never builds an im2col matrix: per 16-channel chunk it stages the
(TZ+2) x 18 x 10 input halo as two 8-channel halves [halo voxel][8 channels]
and points the A operand of each of the 27 taps at that tile with a shifted
start address, reading it through the canonical K-major, no-swizzle matrix
descriptor (8-row core matrices of 16-byte rows; SBO between row groups along
M, LBO between the two 16-byte halves along K). The B operands are the
re-laid weights wtc[ns][chunk][tap][row group][half][row][8]. This test
models exactly those addresses -- the staging, the weight re-layout of
tc_weights_kernel and every descriptor the MMA thread issues -- and checks
that the modelled MMAs give the direct convolution (zero padding per frame,
partial tiles at the edges) and that no address leaves its stage.
"""
import numpy as np
import pytest

TZ, TYY, TXX = 2, 16, 8
HZ, HY, HX = TZ + 2, TYY + 2, TXX + 2
HALO = HZ * HY * HX
HALF = HALO * 16  # bytes of one 8-channel half


def operand(stage, start, lbo, sbo, rows):
    """rows x 16 BF16 operand read through a K-major no-swizzle descriptor."""
    r = np.arange(rows)[:, None]
    k = np.arange(16)[None, :]
    addr = start + (r // 8) * sbo + (r % 8) * 16 + (k // 8) * lbo + (k % 8) * 2
    assert addr.min() >= 0 and addr.max() + 2 <= 2 * stage.size
    return stage[addr // 2]


def conv_direct(x, wt, bias, d, h, w, df):
    Kin, Nout = x.shape[1], wt.shape[1]
    X = x.reshape(d, h, w, Kin)
    out = np.zeros((d, h, w, Nout))
    for z in range(d):
        f0 = (z // df) * df
        for tap in range(27):
            dz, dy, dx = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
            zz = z + dz
            if zz < f0 or zz >= f0 + df:
                continue
            for y in range(h):
                yy = y + dy
                if 0 <= yy < h:
                    xs = np.arange(w) + dx
                    ok = (xs >= 0) & (xs < w)
                    out[z, y, ok] += X[zz, yy, xs[ok]] @ wt[tap].T
    return np.maximum(out + bias, 0).reshape(d * h * w, Nout)


def conv_modelled(x, wt, bias, d, h, w, df, NT):
    Kin, Nout = x.shape[1], wt.shape[1]
    nsplit, nchunks = Nout // NT, Kin // 16
    # tc_weights_kernel: wtc[ns][c][tap][grp][half][row][k]
    wtc = (wt.reshape(27, nsplit, NT // 8, 8, nchunks, 2, 8)       # tap, ns, grp, row, c, half, k
           .transpose(1, 4, 0, 2, 5, 3, 6).reshape(-1))
    wbytes = 27 * NT * 32
    X = x.reshape(d, h, w, Kin)
    out = np.zeros((d * h * w, Nout))
    tiles_x, tiles_y = -(-w // TXX), -(-h // TYY)
    n_tiles = tiles_x * tiles_y * -(-d // TZ)
    hz, hy, hx = np.meshgrid(np.arange(HZ), np.arange(HY), np.arange(HX), indexing="ij")
    hz, hy, hx = hz.ravel(), hy.ravel(), hx.ravel()  # halo voxel hv = (hz * HY + hy) * HX + hx
    for ns in range(nsplit):
        for t in range(n_tiles):
            x0 = (t % tiles_x) * TXX
            y0 = ((t // tiles_x) % tiles_y) * TYY
            z0 = (t // (tiles_x * tiles_y)) * TZ
            zf0 = (z0 // df) * df
            acc = np.zeros((TZ, 128, NT))
            for c in range(nchunks):
                stage = np.zeros((2 * HALF + wbytes) // 2)
                # producers: piece e = (halo voxel e // 2, half e % 2), zeros outside the frame / grid
                z, y, xx = z0 + hz - 1, y0 + hy - 1, x0 + hx - 1
                ok = (z >= zf0) & (z < zf0 + df) & (z < d) & (y >= 0) & (y < h) & (xx >= 0) & (xx < w)
                for half in range(2):
                    vals = np.zeros((HALO, 8))
                    vals[ok] = X[z[ok], y[ok], xx[ok], c * 16 + half * 8:c * 16 + half * 8 + 8]
                    stage[(half * HALF) // 2:(half * HALF + HALO * 16) // 2] = vals.ravel()
                off = (ns * nchunks + c) * (wbytes // 2)
                stage[HALF:] = wtc[off:off + wbytes // 2]
                for tap in range(27):
                    dz, dy, dx = tap // 9, (tap // 3) % 3, tap % 3
                    B = operand(stage, 2 * HALF + tap * NT * 32, 128, 256, NT)
                    for zt in range(TZ):
                        A = operand(stage, (((zt + dz) * HY + dy) * HX + dx) * 16, HALF, HX * 16, 128)
                        acc[zt] += A @ B.T
            # epilogue: TMEM lane m = output row (y0 + m // 8, x0 + m % 8)
            m = np.arange(128)
            for zt in range(TZ):
                y, xx = y0 + m // 8, x0 + m % 8
                inside = (z0 + zt - zf0 < df) & (z0 + zt < d) & (y < h) & (xx < w)
                v = ((z0 + zt) * h + y[inside]) * w + xx[inside]
                out[v, ns * NT:(ns + 1) * NT] = np.maximum(acc[zt][inside] + bias[ns * NT:(ns + 1) * NT], 0)
    return out


@pytest.mark.parametrize("d,h,w,df,Kin,Nout,NT", [
    (4, 20, 12, 4, 32, 32, 32),   # two chunks, partial y and x tiles
    (4, 16, 8, 2, 16, 48, 16),    # stacked frames of depth 2, three N slices
    (2, 18, 9, 2, 16, 64, 64),    # odd width
])
def test_modelled_operands_give_the_convolution(d, h, w, df, Kin, Nout, NT):
    rng = np.random.default_rng(d * 100 + h)
    x = rng.normal(size=(d * h * w, Kin))
    wt = rng.normal(size=(27, Nout, Kin))
    b = rng.normal(size=Nout)
    ref = conv_direct(x, wt, b, d, h, w, df)
    got = conv_modelled(x, wt, b, d, h, w, df, NT)
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-9)
