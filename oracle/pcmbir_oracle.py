"""FP64 numpy restatement of phasecon's phase-contrast (PCMBIR_3D) hot path.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA phase-retrieval kernels.
Pinned against the reference C built from source with an FP64 FFTW-API shim
(oracle/Makefile target ``ref_pc``; tests/test_oracle_pc.py). Every function
cites the reference file:line it restates (paths relative to the phasecon
project root). Images are [rows][cols] = [N_r][N_t] per view; FFTW's sign
convention (forward e^{-2 pi i jk/n}) matches numpy.fft.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

EPS = np.finfo(np.float64).tiny  # EPSILON_ERROR = DBL_MIN, PCMBIR_3D/XT_Constants.h:48
PLANCK_KEV_S = 4.135668e-19       # PLANCKS_CONSTANT, XT_Constants.h:84
LIGHT_SPEED_UM_S = 299792458e+6   # LIGHT_SPEED, XT_Constants.h:85


@dataclass
class PcGeom:
    rows: int
    cols: int
    delta_rows: float = 1.0
    delta_cols: float = 1.0
    energy_kev: float = 20.0
    distance: float = 5e4
    mag_sig_s: float = 1.0
    mag_c_s: float = 1.0
    phase_sig_s: float = 1.0
    phase_c_s: float = 1.0
    delta_over_beta: float = 100.0
    mrf_p: float = 1.2
    mrf_q: float = 2.0
    mu: float = 0.5  # ADMM_mu, XT_Init.c:496
    nu: float = 0.5  # ADMM_nu, XT_Init.c:497

    @property
    def wavelength(self) -> float:  # XT_Init.c:258
        return PLANCK_KEV_S * LIGHT_SPEED_UM_S / self.energy_kev

    @property
    def wavenumber(self) -> float:
        return 2 * math.pi / self.wavelength

    @property
    def window_sigma(self) -> float:  # XT_Init.c:530
        return 2.0 / math.sqrt(self.wavelength * self.distance)

    def freqs(self, scale: float = 1.0):
        """Frequency grids u[i], v[j] with wrap at n/2 (XT_FresnelTran.c:32-40)."""
        i = np.arange(self.rows, dtype=np.float64)
        j = np.arange(self.cols, dtype=np.float64)
        u = np.where(i >= self.rows // 2, -(self.rows - i), i) * scale / (self.rows * self.delta_rows)
        v = np.where(j >= self.cols // 2, -(self.cols - j), j) * scale / (self.cols * self.delta_cols)
        return u[:, None], v[None, :]

    def window(self) -> np.ndarray:
        """Gaussian frequency window (create_FresnelTranWindow, XT_Init.c:210-232)."""
        u, v = self.freqs()
        s = self.window_sigma
        return np.exp(-(u * u + v * v) / (2 * s * s))

    def transfer(self, herm: bool) -> np.ndarray:
        """Frequency response of compute_FresnelTran (XT_FresnelTran.c:12-78):
        exp(-i pi lambda z (u^2+v^2)) x window; of compute_HermFresnelTran
        (:82-137): exp(+i (u'^2+v'^2) / (4 pi / (lambda z))) with u' in rad,
        no window."""
        lam, z = self.wavelength, self.distance
        if herm:
            u, v = self.freqs(2 * math.pi)
            ph = (u * u + v * v) / (4 * (math.pi / (z * lam)))
            return np.cos(ph) + 1j * np.sin(ph)
        u, v = self.freqs()
        ph = -(u * u + v * v) * math.pi * lam * z
        w = self.window()
        return np.cos(ph) * w + 1j * np.sin(ph) * w

    def filter(self) -> np.ndarray:
        """In-plane neighbour weights Spatial_Filter[1][.][.] of PCMBIR's
        initFilter (XT_Init.c:144-190: prior constant 1, no temporal term)."""
        d = np.zeros((3, 3, 3))
        tot = 0.0
        for a in range(3):
            for b in range(3):
                for c in range(3):
                    if a != 1 or b != 1 or c != 1:
                        d[a, b, c] = 1.0 / math.sqrt((a - 1) ** 2 + (b - 1) ** 2 + (c - 1) ** 2)
                        tot += d[a, b, c]
        return (d / tot)[1]

    def decorr(self) -> np.ndarray:
        """[[1, delta/beta], [1, -delta/beta]] (compute_DecorrObjTransform, XT_Init.c:234-247)."""
        return np.array([[1.0, self.delta_over_beta], [1.0, -self.delta_over_beta]])


def fresnel(g: PcGeom, x: np.ndarray, herm: bool = False) -> np.ndarray:
    """y = H x: FFT, multiply by the transfer function, inverse FFT / N."""
    return np.fft.ifft2(np.fft.fft2(x) * g.transfer(herm))


def phase_projection(g: PcGeom, y, D, w) -> np.ndarray:
    """Omega = (y / H(D w)) / |.| (compute_phase_projection, XT_PhaseRet.c:10-33;
    cmplx_div adds EPS to the squared magnitude, XT_CmplxArith.c:11-20)."""
    t = fresnel(g, D * w)
    q = y * np.conj(t) / (np.abs(t) ** 2 + EPS)
    return q / (np.abs(q) + EPS)


def sd_iter(g: PcGeom, y, om, D, w, lam, buf):
    """One steepest-descent step on w (steepest_descent_iter, XT_PhaseRet.c:205-270):
    gradient D^H H'^H Omega^H Lambda (Omega H D w) - D^H H'^H Omega^H Lambda y
    + nu (w - buf) (:76-124), exact step along it for the quadratic with the
    reference's transform pair (:126-165), then the Omega update (:257).
    H' is the window-less Hermitian transform. Returns (w, Omega, threshold)."""
    nu = g.nu

    def A(x):  # Omega H D x
        return fresnel(g, D * x) * om

    def AH(x):  # D^H H'^H Omega^H x
        return fresnel(g, np.conj(om) * x, herm=True) * np.conj(D)

    grad = AH(lam * A(w)) - AH(lam * y) + nu * (w - buf)
    num = np.sum(np.abs(grad) ** 2)
    den = np.sum(np.real(np.conj(grad) * AH(lam * A(grad)))) + nu * num
    alpha = num / (den + EPS)
    w = w - alpha * grad
    up = np.sum(np.sqrt(alpha * alpha * np.abs(grad) ** 2))
    val = np.sum(np.abs(w))
    om = phase_projection(g, y, D, w)
    return w, om, 100.0 * up / val


def qg_value(d, sq, sqp, c, p, q):
    """qGGMRF potential (Mag/Phase_QGGMRF_Spatial_Value, XT_Prior.c:7-25)."""
    ad = abs(d)
    return (ad ** q / sq) / (c + ad ** (q - p) / sqp)


class NmsCost:
    """Per-pixel proximal cost nu/2 |e^{-z} - b|^2 + decorrelated qGGMRF over
    the 3x3 neighbourhood (Cost_NMS, XT_Search.c:8-39, macro-off branch)."""

    def __init__(self, g: PcGeom):
        self.g = g
        self.f = g.filter()
        self.T = g.decorr()
        p, q = g.mrf_p, g.mrf_q
        self.m = (g.mag_sig_s ** q, g.mag_sig_s ** (q - p), g.mag_c_s)
        self.ph = (g.phase_sig_s ** q, g.phase_sig_s ** (q - p), g.phase_c_s)

    def __call__(self, zr, zi, br, bi, nr, ni, flag):
        g = self.g
        ev = math.exp(-zr)
        c, s = ev * math.cos(-zi), ev * math.sin(-zi)
        cost = ((c - br) ** 2 + (s - bi) ** 2) * g.nu / 2
        T = self.T
        for a in range(3):
            for b in range(3):
                if flag[a][b]:
                    db, dd = zr - nr[a][b], zi - ni[a][b]
                    cost += self.f[a, b] * qg_value(T[0, 0] * dd + T[0, 1] * db, *self.ph, g.mrf_p, g.mrf_q)
                    cost += self.f[a, b] * qg_value(T[1, 0] * dd + T[1, 1] * db, *self.m, g.mrf_p, g.mrf_q)
        return cost


def nelder_mead(cost, zr1, zi1, br, bi, nr, ni, flag, max_iter=50, threshold=0.005,
                rho=1.0, chi=2.0, gamma=0.5, sigma=0.5):
    """2-D Nelder-Mead over z = (zr, zi) from the simplex {z, (2zr, zi), (zr, 2zi)}
    (Nelder_Mead_Simplex_2DSearch, XT_Search.c:112-215): vertices kept sorted by
    cost, reflection / expansion / outside and inside contraction / shrink, stop
    when the summed relative vertex movement is below `threshold` percent after
    the second iteration. Returns (zr, zi, iterations)."""
    def f(a, b):
        return cost(a, b, br, bi, nr, ni, flag)

    P = [[zr1, zi1], [2 * zr1, zi1], [zr1, 2 * zi1]]
    C = [f(*P[0]), f(*P[1]), f(*P[2])]

    def sort3():  # two-pass bubble on (1,2), (0,1), (1,2) (NMS_Sort, :65-89)
        for a, b in ((1, 2), (0, 1), (1, 2)):
            if C[b] < C[a]:
                P[a], P[b] = P[b], P[a]
                C[a], C[b] = C[b], C[a]

    def accept(pt, c):  # replace the worst and bubble up (NMS_Accept, :42-63)
        P[2], C[2] = list(pt), c
        for a, b in ((1, 2), (0, 1)):
            if C[b] < C[a]:
                P[a], P[b] = P[b], P[a]
                C[a], C[b] = C[b], C[a]

    def shrink():  # NMS_Shrink, :91-102
        for k in (1, 2):
            P[k] = [P[0][0] + sigma * (P[k][0] - P[0][0]), P[0][1] + sigma * (P[k][1] - P[0][1])]
            C[k] = f(*P[k])
        sort3()

    sort3()
    cen = [(P[0][0] + P[1][0]) / 2.0, (P[0][1] + P[1][1]) / 2.0]
    it = 0
    for it in range(max_iter):
        old = [list(cen)] + [list(p) for p in P]
        ref = [cen[0] + rho * (cen[0] - P[2][0]), cen[1] + rho * (cen[1] - P[2][1])]
        cr = f(*ref)
        if C[0] <= cr < C[1]:
            accept(ref, cr)
        elif cr < C[0]:
            ex = [cen[0] + chi * (ref[0] - cen[0]), cen[1] + chi * (ref[1] - cen[1])]
            ce = f(*ex)
            accept(ex, ce) if ce < cr else accept(ref, cr)
        elif C[1] <= cr < C[2]:
            oc = [cen[0] + gamma * (ref[0] - cen[0]), cen[1] + gamma * (ref[1] - cen[1])]
            co = f(*oc)
            accept(oc, co) if co <= cr else shrink()
        elif cr >= C[2]:
            ic = [cen[0] - gamma * (cen[0] - P[2][0]), cen[1] - gamma * (cen[1] - P[2][1])]
            ci = f(*ic)
            accept(ic, ci) if ci < C[2] else shrink()
        cen = [(P[0][0] + P[1][0]) / 2.0, (P[0][1] + P[1][1]) / 2.0]
        new = [cen] + P
        num = sum(abs(o[0] - n[0]) + abs(o[1] - n[1]) for o, n in zip(old, new))
        den = sum(abs(o[0]) + abs(o[1]) for o in old)
        if num / den * 100 < threshold and it > 1:
            break
    return P[0][0], P[0][1], it


def neighbourhood(zr, zi, j, k):
    """3x3 neighbourhood with boundary flags (XT_CmplxProjEst.c:124-157)."""
    R, Cc = zr.shape
    nr = [[0.0] * 3 for _ in range(3)]
    ni = [[0.0] * 3 for _ in range(3)]
    fl = [[False] * 3 for _ in range(3)]
    for a in range(3):
        for b in range(3):
            jj, kk = j + a - 1, k + b - 1
            if 0 <= jj < R and 0 <= kk < Cc:
                nr[a][b], ni[a][b], fl[a][b] = zr[jj, kk], zi[jj, kk], True
    return nr, ni, fl


def pret_cost(g: PcGeom, y, D, zr, zi, lam):
    """compute_pretcost (XT_CmplxProjEst.c:15-89, macro-off prior): data term
    sum Lambda (y - |H(D e^{-z})|)^2 / 2 plus the decorrelated prior over the
    causal pairs (+col, +row, +row+col, +row-col)."""
    t = fresnel(g, np.exp(-zr) * (np.cos(-zi) + 1j * np.sin(-zi)) * D)
    cost = np.sum((y - np.abs(t)) ** 2 * lam / 2)
    T, f = g.decorr(), g.filter()
    p, q = g.mrf_p, g.mrf_q
    ph = (g.phase_sig_s ** q, g.phase_sig_s ** (q - p), g.phase_c_s)
    mg = (g.mag_sig_s ** q, g.mag_sig_s ** (q - p), g.mag_c_s)

    def pot(d, s):
        ad = np.abs(d)
        return (ad ** q / s[0]) / (s[2] + ad ** (q - p) / s[1])

    for (dj, dk, w) in ((0, 1, f[1, 2]), (1, 0, f[2, 1]), (1, 1, f[2, 2]), (1, -1, f[2, 0])):
        R, Cc = zr.shape
        j0, j1 = 0, R - dj
        k0, k1 = max(0, -dk), Cc - max(0, dk)
        db = zr[j0:j1, k0:k1] - zr[j0 + dj:j1 + dj, k0 + dk:k1 + dk]
        dd = zi[j0:j1, k0:k1] - zi[j0 + dj:j1 + dj, k0 + dk:k1 + dk]
        cost += w * np.sum(pot(T[0, 0] * dd + T[0, 1] * db, ph)) + w * np.sum(pot(T[1, 0] * dd + T[1, 1] * db, mg))
    return float(cost)


def paganin(g: PcGeom, meas, D):
    """Single-material Paganin retrieval (paganins_1mat_phase_retrieval,
    XT_Paganin.c:77-134): thickness -log|F^-1[F(I/I0) / (1 + z (delta/beta)/(2k)
    4 pi^2 (u^2+v^2))]|, z_r = t/2, z_i = t (delta/beta)/2."""
    I0 = np.abs(D) ** 2
    u, v = g.freqs()
    reg = g.delta_over_beta / (2 * g.wavenumber)
    filt = 1.0 / (g.distance * reg * (u * u + v * v) * 4 * math.pi * math.pi + 1)
    t = -np.log(np.abs(np.real(np.fft.ifft2(np.fft.fft2(meas * meas / I0) * filt))))
    return t / 2, t * g.delta_over_beta / 2


def pixel_order(R, Cc, order="raster"):
    """Pixel visiting order of one proximal sweep: the reference's raster order
    (XT_CmplxProjEst.c:117-160), or "color": the four (row parity, column
    parity) classes one after the other, raster order inside each -- no two
    8-neighbours share a class, so a class may be updated in parallel."""
    if order == "raster":
        return [(j, k) for j in range(R) for k in range(Cc)]
    return [(j, k) for c in range(4) for j in range(c >> 1, R, 2) for k in range(c & 1, Cc, 2)]


def nms_sweep(g: PcGeom, zr, zi, b, nms_iters=50, nms_thresh=0.005, order="raster"):
    """One Nelder-Mead proximal sweep over every pixel of one view, in place."""
    cost_fn = NmsCost(g)
    for j, k in pixel_order(*zr.shape, order):
        nr, ni, fl = neighbourhood(zr, zi, j, k)
        zr[j, k], zi[j, k], _ = nelder_mead(cost_fn, zr[j, k], zi[j, k], b[j, k].real, b[j, k].imag,
                                            nr, ni, fl, nms_iters, nms_thresh)


def estimate_projection(g: PcGeom, y, om, D, zr, zi, lam, w, pret_iters=100, sd_iters=100, nms_iters=50,
                        pret_thresh=1e-7, sd_thresh=5e-4, nms_thresh=0.005, order="raster"):
    """Per-view phase-retrieval ADMM (estimate_complex_projection,
    XT_CmplxProjEst.c:91-229, macro-off): per iteration a Nelder-Mead
    proximal update of every pixel's z against b = w - v (raster order as the
    reference, or colour classes, see pixel_order), up to sd_iters
    steepest-descent steps on w towards e^{-z} + v, the dual update
    v += e^{-z} - w, and a stop on the dual residual. The dual starts at zero
    (:108-109). Returns (zr, zi, w, v, Omega, cost history)."""
    zr, zi, w, om = zr.copy(), zi.copy(), w.copy(), om.copy()
    v = np.zeros_like(w)
    costs = [pret_cost(g, y, D, zr, zi, lam)]
    for it in range(pret_iters):
        nms_sweep(g, zr, zi, w - v, nms_iters, nms_thresh, order)
        wold = w.copy()
        ez = np.exp(-zr) * (np.cos(-zi) + 1j * np.sin(-zi))
        buf = ez + v
        for s in range(sd_iters):
            w, om, th = sd_iter(g, y, om, D, w, lam, buf)
            if th < sd_thresh and s > 1:
                break
        d = ez - w
        v = v + d
        dual = math.sqrt(np.sum(np.abs(w - wold) ** 2) / np.sum(np.abs(v) ** 2))
        costs.append(pret_cost(g, y, D, zr, zi, lam))
        if dual < pret_thresh and it > 1:
            break
    return zr, zi, w, v, om, costs
