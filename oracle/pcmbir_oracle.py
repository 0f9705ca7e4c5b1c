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
    sim_window: bool = False  # the data simulator's window (initPhantomStructures, XT_Init.c:677)

    @property
    def wavelength(self) -> float:  # XT_Init.c:258
        return PLANCK_KEV_S * LIGHT_SPEED_UM_S / self.energy_kev

    @property
    def wavenumber(self) -> float:
        return 2 * math.pi / self.wavelength

    @property
    def window_sigma(self) -> float:  # XT_Init.c:530; the simulator's XT_Init.c:677
        if self.sim_window:
            return 1.0 / math.sqrt(0.5 * self.wavelength * self.distance)
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


# ---- data simulator (phcontomo_forward_project) -----------------------------------------------

PM_MODULUS = 2147483647  # MAXPRIME, PCMBIR_3D/randlib.c:42
PM_MULTIPLIER = 16807
SIM_NOISE_SEED = 761521  # srandom2 seed of phcontomo_forward_project, PCMBIR_3D/XT_Engine.c:212


def random2_states(seed: int, n: int) -> np.ndarray:
    """States x_1..x_n of randlib's random2() after srandom2(seed)
    (PCMBIR_3D/randlib.c:119-141, 168-174): x_k = seed 16807^k mod (2^31 - 1);
    random2() returns x_k / (2^31 - 1). Computed in blocks: the first B
    states one by one, then each block from the previous one times 16807^B."""
    B = 4096
    first = np.empty(min(n, B), np.uint64)
    x = seed % PM_MODULUS
    for i in range(first.size):
        x = (x * PM_MULTIPLIER) % PM_MODULUS
        first[i] = x
    if n <= B:
        return first
    out = np.empty(n, np.uint64)
    out[:B] = first
    step = np.uint64(pow(PM_MULTIPLIER, B, PM_MODULUS))
    for s in range(B, n, B):
        e = min(n, s + B)
        out[s:e] = (out[s - B:e - B] * step) % np.uint64(PM_MODULUS)
    return out


def randlib_normals(n: int, seed: int = SIM_NOISE_SEED) -> np.ndarray:
    """The first n values of randlib's normal() (PCMBIR_3D/randlib.c:208-225)
    after srandom2(seed), from a fresh process: pair p draws theta = 2 pi u and
    r = sqrt(-2 log u') from two consecutive random2() values and returns
    r cos(theta), then r sin(theta)."""
    pairs = (n + 1) // 2
    x = random2_states(seed, 2 * pairs).astype(np.float64) / PM_MODULUS
    theta = 2 * 3.14159265358979323846 * x[0::2]
    r = np.sqrt(-2 * np.log(x[1::2]))
    out = np.empty(2 * pairs)
    out[0::2] = r * np.cos(theta)
    out[1::2] = r * np.sin(theta)
    return out[:n]


def sim_detector(intensity: np.ndarray, proj_rows: int, proj_cols: int, seed: int = SIM_NOISE_SEED) -> np.ndarray:
    """The detector stage of ForwardProject (PCMBIR_3D/XT_genSinogram.c:239-262):
    intensity |F|^2 [V][N_r][N_t] (phantom resolution) averaged over the
    (N_t / proj_rows) x (N_r / proj_cols) pixels of each detector pixel (a
    float32 running sum of FP64 terms, t outer, r inner), then
    m <- |m + sqrt|m| n| with n the normal() sequence in (view, row, col) order."""
    V, R, Cn = intensity.shape
    rs, ts = R // proj_cols, Cn // proj_rows
    m = np.zeros((V, proj_rows, proj_cols), np.float32)
    for ti in range(ts):
        for ri in range(rs):
            blk = intensity[:, ri:rs * proj_cols:rs, ti:ts * proj_rows:ts]  # [V][col][row]
            m = (m.astype(np.float64) + blk.transpose(0, 2, 1)).astype(np.float32)
    m = (m / np.float32(ts * rs)).astype(np.float32)
    n = randlib_normals(m.size, seed).reshape(m.shape)
    md = m.astype(np.float64)
    return np.abs(md + np.sqrt(np.abs(md)) * n).astype(np.float32)


def sim_geometry(P_xy: int, P_z: int, proj_rows: int, proj_cols: int, vox_wid: float, energy_kev: float,
                 distance: float) -> PcGeom:
    """Transform geometry of the simulator (initPhantomStructures, XT_Init.c:611-684):
    N_r = P_xy rows of pitch vox_wid proj_cols / P_xy, N_t = P_z columns of
    pitch vox_wid proj_rows / P_z, window sigma 1 / sqrt(lambda z / 2)."""
    return PcGeom(rows=P_xy, cols=P_z, delta_rows=float(np.float32(vox_wid)) * proj_cols / P_xy,
                  delta_cols=float(np.float32(vox_wid)) * proj_rows / P_z, energy_kev=float(np.float32(energy_kev)),
                  distance=float(np.float32(distance)), sim_window=True)


def sim_from_projections(pm: np.ndarray, pp: np.ndarray, g: PcGeom, proj_rows: int, proj_cols: int,
                         count: float = 2500.0) -> np.ndarray:
    """Measurements of ForwardProject (XT_genSinogram.c:212-262) from the FP64
    projections P_mag, P_phase [V][N_t][N_r] (the reference's SimMagProjs /
    SimPhaseProjs): field sqrt(count) e^{-P_mag} (cos, sin)(-P_phase) per view
    ([N_r][N_t]), the windowed Fresnel transform, |.|^2, then sim_detector."""
    e = np.exp(-pm)
    a_r, a_i = e * np.cos(-pp), e * np.sin(-pp)
    s = math.sqrt(count)
    field = (a_r * s - a_i * 0.0) + 1j * (a_r * 0.0 + a_i * s)
    field = field.transpose(0, 2, 1)  # [V][N_r][N_t]
    F = np.fft.ifft2(np.fft.fft2(field, axes=(1, 2)) * g.transfer(False)[None], axes=(1, 2))
    inten = F.real * F.real + F.imag * F.imag
    return sim_detector(inten, proj_rows, proj_cols)


SIM_BINS = 256      # DETECTOR_RESPONSE_BINS of PCMBIR_3D/XT_Constants.h:163
SIM_BEAM_RES = 256  # BEAM_RESOLUTION, XT_Constants.h:162
SIM_PROFILE_RES = 1536  # PROFILE_RESOLUTION, XT_Constants.h:161


def sim_project(mag: np.ndarray, phase: np.ndarray, angles, proj_rows: int, proj_cols: int, vox_wid: float,
                rot_center: float, light_energy: float):
    """FP64 projections P_mag, P_phase [V][N_t][N_r] of ForwardProject
    (PCMBIR_3D/XT_genSinogram.c:141-181) on the geometry of
    initPhantomStructures (XT_Init.c:611-684): A columns of
    calcAMatrixColumnforAngle x wavenumber (XT_AMatrix.c:50-110) from the
    detector response of DetectorResponseProfile (XT_Profile.c:47-180) and the
    voxel-line response of storeVoxelLineResponse (XT_Profile.c:182-297).
    Sums run in another order than the reference's (agreement ~1e-15)."""
    P_z, P_xy, _ = mag.shape
    vox, rot = float(np.float32(vox_wid)), float(np.float32(rot_center))
    lam = PLANCK_KEV_S * LIGHT_SPEED_UM_S / float(np.float32(light_energy))
    k = 2 * math.pi / lam
    LR, LT = vox * proj_cols, vox * proj_rows
    RC = rot * (P_xy // proj_cols)
    dr, dt = LR / P_xy, LT / P_z
    R0, RMax, T0, TMax = -RC * dr, (P_xy - RC) * dr, -LT / 2.0, LT / 2.0
    dxy, dz = dr, dt
    x0, y0, z0 = R0, -LR / 2.0, T0
    off_r = (dxy / math.sqrt(2.0) + dr / 2.0) / SIM_BINS
    off_t = ((dz / 2) + dt / 2) / SIM_BINS
    # voxel-line response Z[slice][t]
    ht = np.zeros(SIM_BINS + 1)
    for i in range(SIM_BINS):
        c = i * off_t
        h = dt if c <= (dz / 2 - dt / 2) else -c + dz / 2 + dt / 2
        if dz < dt:
            h = dz if c <= dt / 2 - dz / 2 else -c + dz / 2 + dt / 2
        ht[i] = max(h, 0.0) / dt
    Z = np.zeros((P_z, P_z))
    for i in range(P_z):
        t = (i + 0.5) * dz + z0
        tmin = t - dz / 2 if (t - dz / 2) > T0 else T0
        tmax = t + dz / 2 if (t + dz / 2) <= TMax else TMax
        lo, hi = max(int(math.floor((tmin - T0) / dt)), 0), min(int(math.floor((tmax - T0) / dt)), P_z - 1)
        for it in range(lo, hi + 1):
            d = abs(((it + 0.5) * dt + T0) - t)
            idx = int(math.floor(d / off_t))
            if idx < SIM_BINS:
                Z[i, it] = ((idx + 1) * off_t - d) / off_t * ht[idx] + (d - idx * off_t) / off_t * ht[idx + 1]
    # z response of every column: p[t][col]
    pm = np.einsum("st,sc->tc", Z, mag.reshape(P_z, -1).astype(np.float64))
    pp = np.einsum("st,sc->tc", Z, phase.reshape(P_z, -1).astype(np.float64))
    beam = 0.54 - 0.46 * np.cos((2 * math.pi / SIM_BEAM_RES) * np.arange(SIM_BEAM_RES))
    beam = beam / beam.sum()
    rows_, cols_ = np.meshgrid(np.arange(P_xy), np.arange(P_xy), indexing="ij")
    x = (x0 + (cols_.ravel() + 0.5) * dxy)
    y = (y0 + (rows_.ravel() + 0.5) * dxy)
    V = len(angles)
    out_m = np.zeros((V, P_z, P_xy))
    out_p = np.zeros((V, P_z, P_xy))
    jprof = 2.0 * np.arange(SIM_PROFILE_RES) / SIM_PROFILE_RES
    for v in range(V):
        a = float(np.float32(angles[v]))
        cs, sn = math.cos(a), math.sin(a)
        ang = a
        while ang > math.pi / 2:
            ang -= math.pi / 2
        while ang < 0:
            ang += math.pi / 2
        peak = dxy / math.cos(ang) if ang <= math.pi / 4 else dxy / math.cos(math.pi / 2 - ang)
        t45 = math.cos(math.pi / 4)
        d1, d2 = t45 * math.cos(math.pi / 4 - ang), t45 * abs(math.cos(math.pi / 4 + ang))
        lc, ln, rn, rc = 1 - d1, 1 - d2, 1 + d2, 1 + d1
        prof = np.where((jprof <= lc) | (jprof >= rc), 0.0,
                        np.where(jprof > rn, peak * (rc - jprof) / (rc - rn),
                                 np.where(jprof >= ln, peak, peak * (jprof - lc) / (ln - lc))))
        r_beam = -dr / 2 + np.arange(SIM_BEAM_RES) * (dr / SIM_BEAM_RES)
        rmin_b = np.arange(SIM_BINS)[:, None] * off_r - dxy
        pidx = np.floor((r_beam[None, :] - rmin_b) * (SIM_PROFILE_RES / (2 * dxy))).astype(np.int64)
        ok = (pidx >= 0) & (pidx <= SIM_PROFILE_RES - 1)
        H = np.zeros(SIM_BINS + 1)
        H[:SIM_BINS] = np.where(ok, prof[np.clip(pidx, 0, SIM_PROFILE_RES - 1)] * beam[None, :], 0.0).sum(1)
        r = x * cs - y * sn
        live = ~((r + dxy < R0) | (r - dxy > RMax))
        imin = np.maximum(np.floor((r - dxy - R0) / dr).astype(np.int64), 0)
        imax = np.minimum(np.floor((r + dxy - R0) / dr).astype(np.int64), P_xy - 1)
        for o in range(3):
            j = imin + o
            sel = live & (j <= imax)
            dd = np.abs(r - (R0 + (j + 0.5) * dr))
            b = np.floor(dd / off_r).astype(np.int64)
            sel &= (b >= 0) & (b < SIM_BINS)
            bb = np.clip(b, 0, SIM_BINS - 1)
            w1 = dd - bb * off_r
            f1 = ((off_r - w1) * H[bb] + w1 * H[bb + 1]) / off_r
            sel &= f1 > 0
            cidx = np.nonzero(sel)[0]
            aval = f1[cidx] * k
            np.add.at(out_m[v].T, j[cidx], aval[:, None] * pm[:, cidx].T)
            np.add.at(out_p[v].T, j[cidx], aval[:, None] * pp[:, cidx].T)
    return out_m, out_p


def simulate(mag, phase, angles, proj_rows, proj_cols, vox_wid, rot_center, obj2det_dist, light_energy,
             count: float = 2500.0):
    """The whole simulator (phcontomo_forward_project): (measurements, P_mag, P_phase)."""
    pm, pp = sim_project(mag, phase, angles, proj_rows, proj_cols, vox_wid, rot_center, light_energy)
    g = sim_geometry(mag.shape[1], mag.shape[0], proj_rows, proj_cols, vox_wid, light_energy, obj2det_dist)
    return sim_from_projections(pm, pp, g, proj_rows, proj_cols, count), pm, pp
