"""Python mirror of phasecon's PCMBIR_3D (phase-contrast) interface over libmbirgpu.

``phcontomo_reconstruct`` takes the reference's arguments (PCMBIR_3D/XT_Engine.c:82,
include/pcmbir4d.h:35) and, like it, leaves its results in files of the working
directory. ``PcSession`` keeps every view of a scan resident on the GPU and
exposes the pieces of the per-view phase-retrieval ADMM (Fresnel transforms,
Paganin retrieval, steepest descent, the Nelder-Mead proximal sweep, the full
loop) for tests, benchmarks and callers that drive the loop themselves.

Images are [proj_num][N_r][N_t] = [proj_num][proj_cols][proj_rows] on the
session side (the reference's per-view [j][k] arrays); measurements and
brights come in the reference's input layout [proj_num][proj_rows][proj_cols]
and [proj_rows][proj_cols]. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from .mbir import MbirError, _check, lib as _mbir_lib


class PcProblemStruct(C.Structure):
    _fields_ = [
        ("measurements", C.c_void_p), ("brights", C.c_void_p), ("proj_rows", C.c_int32), ("proj_cols", C.c_int32),
        ("proj_num", C.c_int32), ("vox_wid", C.c_float), ("mag_sig_s", C.c_float), ("mag_c_s", C.c_float),
        ("phase_sig_s", C.c_float), ("phase_c_s", C.c_float), ("obj2det_dist", C.c_float),
        ("light_energy", C.c_float), ("pag_regparam", C.c_float),
    ]


class PcOptions(C.Structure):
    _fields_ = [
        ("pret_max_iter", C.c_int32), ("sd_max_iter", C.c_int32), ("nms_max_iter", C.c_int32),
        ("pret_threshold", C.c_double), ("sd_threshold", C.c_double), ("nms_threshold", C.c_double),
        ("mu", C.c_double), ("nu", C.c_double), ("mrf_p", C.c_double), ("mrf_q", C.c_double),
        ("nms_order", C.c_int32), ("fft_radix", C.c_int32),
        ("nms_lanes", C.c_int32), ("nms_ctas_per_view", C.c_int32),
    ]


class PcStats(C.Structure):
    _fields_ = [("sd_steps", C.c_int64), ("fresnel_transforms", C.c_int64), ("kernel_ms", C.c_double),
                ("kernel_launches", C.c_int64)]


class SimOptions(C.Structure):
    """mbirgpu_pc_sim_options: the simulator's constants of PCMBIR_3D/XT_Constants.h."""
    _fields_ = [
        ("mag_phantom_path", C.c_char * 1024), ("phase_phantom_path", C.c_char * 1024), ("phantom_xy", C.c_int32),
        ("phantom_z", C.c_int32), ("expected_count", C.c_float), ("write_files", C.c_int32),
    ]


_bound = False


def lib() -> C.CDLL:
    """libmbirgpu.so with the phase-contrast signatures declared."""
    global _bound
    L = _mbir_lib()
    if not _bound:
        vp, fp = C.c_void_p, C.POINTER(C.c_float)
        L.phcontomo_reconstruct.argtypes = [C.POINTER(fp), C.POINTER(fp)] + [vp] * 5 + [C.c_int32] * 4 + \
            [C.c_float] * 14 + [C.c_uint8, C.c_uint8, vp]
        L.mbirgpu_pc_default_options.argtypes = [C.POINTER(PcOptions)]
        L.mbirgpu_pc_default_options.restype = None
        L.mbirgpu_pc_session_create.argtypes = [C.POINTER(vp), C.POINTER(PcProblemStruct), C.POINTER(PcOptions), vp]
        L.mbirgpu_pc_session_destroy.argtypes = [vp]
        L.mbirgpu_pc_fresnel.argtypes = [vp, vp, vp, C.c_int32]
        L.mbirgpu_pc_paganin.argtypes = [vp, vp, vp]
        L.mbirgpu_pc_time_fresnel.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
        L.mbirgpu_pc_set_z.argtypes = [vp, vp, vp]
        L.mbirgpu_pc_init_admm.argtypes = [vp]
        L.mbirgpu_pc_set_state.argtypes = [vp, vp, vp, vp]
        L.mbirgpu_pc_get_state.argtypes = [vp, vp, vp, vp, vp, vp]
        L.mbirgpu_pc_sd_step.argtypes = [vp, vp, vp]
        L.mbirgpu_pc_nms_sweep.argtypes = [vp]
        L.mbirgpu_pc_run.argtypes = [vp, vp, vp, C.POINTER(PcStats)]
        L.phcontomo_forward_project.argtypes = [C.POINTER(fp), C.POINTER(fp), vp, C.c_int32, C.c_int32, C.c_int32] + \
            [C.c_float] * 5 + [vp]
        L.mbirgpu_pc_sim_default_options.argtypes = [C.POINTER(SimOptions)]
        L.mbirgpu_pc_sim_default_options.restype = None
        L.mbirgpu_pc_sim_set_options.argtypes = [C.POINTER(SimOptions)]
        L.mbirgpu_pc_sim_get_options.argtypes = [C.POINTER(SimOptions)]
        L.mbirgpu_pc_simulate.argtypes = [vp, vp, C.POINTER(SimOptions), vp, vp, vp, C.c_int32, C.c_int32, C.c_int32] + \
            [C.c_float] * 4 + [vp, vp, C.POINTER(C.c_double)]
        _bound = True
    return L


def default_options(**kw) -> PcOptions:
    o = PcOptions()
    lib().mbirgpu_pc_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


@dataclass
class PcProblem:
    """Scan description of phcontomo_reconstruct (PCMBIR_3D/XT_Engine.c:82-90)."""
    measurements: np.ndarray  # [proj_num][proj_rows][proj_cols] intensities
    brights: np.ndarray       # [proj_rows][proj_cols]
    vox_wid: float = 1.0
    mag_sig_s: float = 1.0
    mag_c_s: float = 1.0
    phase_sig_s: float = 1.0
    phase_c_s: float = 1.0
    obj2det_dist: float = 5e4
    light_energy: float = 20.0
    pag_regparam: float = 100.0

    @property
    def dims(self):
        V, rows, cols = self.measurements.shape
        return V, rows, cols


def _c2f(a: np.ndarray) -> np.ndarray:
    """complex [V][R][C] -> interleaved float32 [V][R][C][2]."""
    a = np.asarray(a)
    out = np.empty(a.shape + (2,), np.float32)
    out[..., 0] = a.real
    out[..., 1] = a.imag
    return out


def _f2c(a: np.ndarray) -> np.ndarray:
    return a[..., 0].astype(np.float64) + 1j * a[..., 1].astype(np.float64)


class PcSession:
    """Every view of one phase-contrast scan resident on the GPU."""

    def __init__(self, pb: PcProblem, options: PcOptions | None = None, stream: int | None = None):
        self._meas = np.ascontiguousarray(pb.measurements, np.float32)
        self._brights = np.ascontiguousarray(pb.brights, np.float32)
        V, rows, cols = self._meas.shape
        if self._brights.shape != (rows, cols):
            raise MbirError(f"brights must be [{rows}][{cols}]")
        ps = PcProblemStruct(self._meas.ctypes.data, self._brights.ctypes.data, rows, cols, V, pb.vox_wid,
                             pb.mag_sig_s, pb.mag_c_s, pb.phase_sig_s, pb.phase_c_s, pb.obj2det_dist,
                             pb.light_energy, pb.pag_regparam)
        self.options = options if options is not None else default_options()
        self.h = C.c_void_p()
        _check(lib().mbirgpu_pc_session_create(C.byref(self.h), C.byref(ps), C.byref(self.options),
                                               C.c_void_p(stream or 0)))
        self.shape = (V, cols, rows)  # [N_p][N_r][N_t]

    def close(self):
        if self.h:
            lib().mbirgpu_pc_session_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def fresnel(self, x: np.ndarray, herm: bool = False) -> np.ndarray:
        a = _c2f(np.reshape(x, self.shape))
        out = np.zeros_like(a)
        _check(lib().mbirgpu_pc_fresnel(self.h, a.ctypes.data, out.ctypes.data, 1 if herm else 0))
        return _f2c(out)

    def time_fresnel(self, n: int, herm: bool = False) -> float:
        """Device milliseconds of n back-to-back transforms of every view."""
        ms = C.c_double()
        _check(lib().mbirgpu_pc_time_fresnel(self.h, n, 1 if herm else 0, C.byref(ms)))
        return ms.value

    def paganin(self):
        zr = np.zeros(self.shape, np.float32)
        zi = np.zeros(self.shape, np.float32)
        _check(lib().mbirgpu_pc_paganin(self.h, zr.ctypes.data, zi.ctypes.data))
        return zr, zi

    def set_z(self, zr: np.ndarray, zi: np.ndarray) -> None:
        a = np.ascontiguousarray(np.reshape(zr, self.shape), np.float32)
        b = np.ascontiguousarray(np.reshape(zi, self.shape), np.float32)
        _check(lib().mbirgpu_pc_set_z(self.h, a.ctypes.data, b.ctypes.data))

    def init_admm(self) -> None:
        _check(lib().mbirgpu_pc_init_admm(self.h))

    def set_state(self, w=None, v=None, omega=None) -> None:
        arrs = [None if x is None else _c2f(np.reshape(x, self.shape)) for x in (w, v, omega)]
        _check(lib().mbirgpu_pc_set_state(self.h, *(None if a is None else a.ctypes.data for a in arrs)))

    def get_state(self):
        """(zr, zi, w, v, omega) with the complex ones as complex128."""
        zr = np.zeros(self.shape, np.float32)
        zi = np.zeros(self.shape, np.float32)
        c = [np.zeros(self.shape + (2,), np.float32) for _ in range(3)]
        _check(lib().mbirgpu_pc_get_state(self.h, zr.ctypes.data, zi.ctypes.data, *(a.ctypes.data for a in c)))
        return (zr, zi) + tuple(_f2c(a) for a in c)

    def sd_step(self, buf: np.ndarray | None = None) -> np.ndarray:
        b = None if buf is None else _c2f(np.reshape(buf, self.shape))
        th = np.zeros(self.shape[0], np.float32)
        _check(lib().mbirgpu_pc_sd_step(self.h, None if b is None else b.ctypes.data, th.ctypes.data))
        return th

    def nms_sweep(self) -> None:
        _check(lib().mbirgpu_pc_nms_sweep(self.h))

    def run(self):
        """The per-view ADMM; returns (costs [V][P+1] with NaN after a view stopped,
        iterations [V], PcStats)."""
        V = self.shape[0]
        P = self.options.pret_max_iter
        costs = np.zeros((V, P + 1), np.float64)
        iters = np.zeros(V, np.int32)
        st = PcStats()
        _check(lib().mbirgpu_pc_run(self.h, costs.ctypes.data, iters.ctypes.data, C.byref(st)))
        return costs, iters, st


def phcontomo_reconstruct(measurements, brights, proj_angles, proj_times, recon_times, proj_rows, proj_cols,
                          proj_num, recon_num, vox_wid, rot_center, mag_sig_s, mag_sig_t, mag_c_s, mag_c_t,
                          phase_sig_s, phase_sig_t, phase_c_s, phase_c_t, convg_thresh, obj2det_dist,
                          light_energy, pag_regparam, restart=0, recon_type=1, workdir: str | None = None) -> None:
    """The reference's phcontomo_reconstruct run on the GPU. Results go to files
    of `workdir` (default: the current directory) as in the reference; raises
    MbirError where the reference returns -1."""
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in
            (measurements, brights, proj_angles, proj_times, recon_times)]
    fp = C.POINTER(C.c_float)
    mag, ph = fp(), fp()
    cwd = os.getcwd()
    if workdir is not None:
        os.chdir(workdir)
    try:
        rc = lib().phcontomo_reconstruct(C.byref(mag), C.byref(ph), *(a.ctypes.data for a in arrs), proj_rows,
                                         proj_cols, proj_num, recon_num, vox_wid, rot_center, mag_sig_s, mag_sig_t,
                                         mag_c_s, mag_c_t, phase_sig_s, phase_sig_t, phase_c_s, phase_c_t,
                                         convg_thresh, obj2det_dist, light_energy, pag_regparam, restart,
                                         recon_type, None)
    finally:
        os.chdir(cwd)
    _check(rc)


def sim_options(**kw) -> SimOptions:
    """The current simulator settings, with fields overridden by keyword."""
    o = SimOptions()
    _check(lib().mbirgpu_pc_sim_get_options(C.byref(o)))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise MbirError(f"unknown simulator option {k}")
        setattr(o, k, v.encode() if isinstance(v, str) else v)
    return o


def set_sim_options(o: SimOptions) -> None:
    _check(lib().mbirgpu_pc_sim_set_options(C.byref(o)))


def simulate(mag, phase, proj_angles, proj_rows: int, proj_cols: int, vox_wid: float, rot_center: float,
             obj2det_dist: float, light_energy: float, options: SimOptions | None = None,
             projections: bool = False):
    """mbirgpu_pc_simulate on phantoms [P_z][P_xy][P_xy]: returns (measurements
    [proj_num][proj_rows][proj_cols], brights, average) and, with projections,
    also the FP64 projections (SimMagProjs, SimPhaseProjs) [proj_num][P_z][P_xy]."""
    mag = np.ascontiguousarray(mag, np.float32)
    phase = np.ascontiguousarray(phase, np.float32)
    ang = np.ascontiguousarray(proj_angles, np.float32)
    o = options if options is not None else sim_options(write_files=0)
    if mag.shape != (o.phantom_z, o.phantom_xy, o.phantom_xy) or phase.shape != mag.shape:
        raise MbirError(f"phantoms must be [{o.phantom_z}][{o.phantom_xy}][{o.phantom_xy}]")
    V = ang.size
    meas = np.zeros((V, proj_rows, proj_cols), np.float32)
    br = np.zeros((proj_rows, proj_cols), np.float32)
    pm = np.zeros((V, o.phantom_z, o.phantom_xy)) if projections else None
    pp = np.zeros_like(pm) if projections else None
    avg = C.c_double()
    _check(lib().mbirgpu_pc_simulate(mag.ctypes.data, phase.ctypes.data, C.byref(o), meas.ctypes.data,
                                     br.ctypes.data, ang.ctypes.data, proj_rows, proj_cols, V, vox_wid, rot_center,
                                     obj2det_dist, light_energy, pm.ctypes.data if projections else None,
                                     pp.ctypes.data if projections else None, C.byref(avg)))
    if projections:
        return meas, br, avg.value, pm, pp
    return meas, br, avg.value


def phcontomo_forward_project(measurements: np.ndarray, brights: np.ndarray, proj_angles, proj_rows: int,
                              proj_cols: int, proj_num: int, vox_wid: float, rot_center: float, obj2det_dist: float,
                              light_energy: float, pag_regparam: float, workdir: str | None = None) -> None:
    """The reference's phcontomo_forward_project: fills the caller's float32
    arrays measurements [proj_num][proj_rows][proj_cols] and brights
    [proj_rows][proj_cols] from the phantom files named by the simulator
    settings; output files go to `workdir` (default: the current directory)."""
    for a in (measurements, brights):
        if a.dtype != np.float32 or not a.flags.c_contiguous:
            raise MbirError("measurements and brights must be C-contiguous float32 arrays")
    if measurements.size != proj_num * proj_rows * proj_cols or brights.size != proj_rows * proj_cols:
        raise MbirError("measurements / brights sizes do not match the detector")
    ang = np.ascontiguousarray(proj_angles, np.float32)
    fp = C.POINTER(C.c_float)
    pm, pb = measurements.ctypes.data_as(fp), brights.ctypes.data_as(fp)
    cwd = os.getcwd()
    if workdir is not None:
        os.chdir(workdir)
    try:
        rc = lib().phcontomo_forward_project(C.byref(pm), C.byref(pb), ang.ctypes.data, proj_rows, proj_cols,
                                             proj_num, vox_wid, rot_center, obj2det_dist, light_energy,
                                             pag_regparam, None)
    finally:
        os.chdir(cwd)
    _check(rc)
