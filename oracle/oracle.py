"""ctypes front end to the CPU oracle (TEST INFRASTRUCTURE ONLY).

Two libraries sit under ``oracle/_ref/`` after ``make -C oracle all ref``:

* ``libmbir_oracle.so`` -- the C restatement of the phasecon MBIR_4D hot path
  (oracle/mbir_oracle.c, each function citing the reference file:line it
  restates);
* ``libref_mbir4d.so`` -- the reference C itself, built from its own sources
  with a single-rank MPI shim (oracle/Makefile, oracle/ref_harness.c).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module, as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
RESP_BINS = 64

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


class OrcGeom(C.Structure):
    _fields_ = [
        ("N_r", C.c_int32), ("N_t", C.c_int32), ("N_p", C.c_int32), ("z_overlap", C.c_int32),
        ("delta_r", C.c_double), ("delta_t", C.c_double), ("R0", C.c_double), ("RMax", C.c_double),
        ("T0", C.c_double), ("TMax", C.c_double), ("OffsetR", C.c_double), ("OffsetT", C.c_double),
        ("N_time", C.c_int32), ("N_x", C.c_int32), ("N_y", C.c_int32), ("N_z", C.c_int32),
        ("mult_xy", C.c_int32), ("mult_z", C.c_int32),
        ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("delta_xy", C.c_double),
        ("delta_z", C.c_double), ("delta_recon", C.c_double), ("radius_obj", C.c_double),
        ("p", C.c_double), ("q", C.c_double), ("alpha", C.c_double), ("c_s", C.c_double), ("c_t", C.c_double),
        ("sigma_s_q", C.c_double), ("sigma_s_q_p", C.c_double), ("sigma_t_q", C.c_double),
        ("sigma_t_q_p", C.c_double),
        ("spatial_filter", C.c_double * 27), ("time_filter", C.c_double),
        ("huber_T", C.c_double), ("huber_delta", C.c_double),
        ("num_z_blocks", C.c_int32),
    ]


class RefProblem(C.Structure):
    """Mirror of RefProblem in oracle/ref_harness.c."""
    _fields_ = [
        ("projections", C.c_void_p), ("weights", C.c_void_p), ("proj_angles", C.c_void_p),
        ("proj_times", C.c_void_p), ("recon_times", C.c_void_p),
        ("proj_rows", C.c_int32), ("proj_cols", C.c_int32), ("proj_num", C.c_int32), ("recon_num", C.c_int32),
        ("vox_wid", C.c_float), ("rot_center", C.c_float), ("sig_s", C.c_float), ("sig_t", C.c_float),
        ("c_s", C.c_float), ("c_t", C.c_float), ("convg_thresh", C.c_float),
        ("quad_convex", C.c_int32), ("huber_delta", C.c_float), ("huber_T", C.c_float),
        ("mult_xy", C.c_int32), ("mult_z", C.c_int32),
    ]


@dataclass
class Problem:
    """One reconstruction problem in the reference's ABI layout.

    projections/weights are [proj_num][proj_rows][proj_cols] (col fastest), as
    passed to ``reconstruct`` (MBIR_4D/XT_Engine.c:81).
    """
    projections: np.ndarray
    weights: np.ndarray
    proj_angles: np.ndarray
    proj_times: np.ndarray
    recon_times: np.ndarray
    proj_rows: int
    proj_cols: int
    proj_num: int
    recon_num: int
    vox_wid: float = 1.0
    rot_center: float = 0.0
    sig_s: float = 0.01
    sig_t: float = 1.0
    c_s: float = 1.0
    c_t: float = 1.0
    convg_thresh: float = 0.0
    quad_convex: int = 1
    huber_delta: float = 0.5
    huber_T: float = 4.0
    mrf_p: float = 1.2
    _keep: list = field(default_factory=list, repr=False)

    def ref_struct(self, mult_xy: int = 1, mult_z: int = 1) -> RefProblem:
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in
                (self.projections, self.weights, self.proj_angles, self.proj_times, self.recon_times)]
        self._keep = arrs
        return RefProblem(*(a.ctypes.data for a in arrs), self.proj_rows, self.proj_cols, self.proj_num,
                          self.recon_num, self.vox_wid, self.rot_center, self.sig_s, self.sig_t, self.c_s,
                          self.c_t, self.convg_thresh, self.quad_convex, self.huber_delta, self.huber_T,
                          mult_xy, mult_z)


def reference_root() -> str | None:
    """The phasecon checkout the reference builds read (environment variable
    PHASECON_REFERENCE_ROOT), or None when it is unset or holds no sources."""
    root = os.environ.get("PHASECON_REFERENCE_ROOT", "")
    return root if root and os.path.isdir(os.path.join(root, "Source_Code", "MBIR_4D")) else None


def build(with_reference: bool | None = None) -> None:
    """Build the oracle libraries; the reference builds only where its sources
    are reachable (PHASECON_REFERENCE_ROOT), else the prebuilt ones under
    _ref/ are kept as they are."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if with_reference is None:
        with_reference = reference_root() is not None
    if with_reference:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)
        subprocess.run(["make", "-s", "-C", HERE, "ref_pc"], check=True)


_orc = None
_ref = {}


def orc_lib() -> C.CDLL:
    global _orc
    if _orc is None:
        path = os.path.join(REF_DIR, "libmbir_oracle.so")
        if not os.path.exists(path):
            build(with_reference=False)
        lib = C.CDLL(path)
        P = C.POINTER(OrcGeom)
        lib.orc_init_geometry.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                          C.c_double, C.c_int32, C.c_double, C.c_double, C.c_int32, _f32p, _f32p,
                                          _i32p, _i32p]
        lib.orc_init_geometry.restype = C.c_int
        lib.orc_detector_response.argtypes = [P, _f32p, _f32p]
        lib.orc_amatrix_column.argtypes = [P, _f32p, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                                           _i32p, _f64p]
        lib.orc_amatrix_column.restype = C.c_int32
        lib.orc_forward_project.argtypes = [P, _f32p, _f32p, _i32p, _i32p, _f32p, _f64p]
        lib.orc_cost.argtypes = [P, _f32p, _f32p, _f32p, _f64p]
        lib.orc_cost.restype = C.c_double
        lib.orc_functional_substitution.argtypes = [P, C.c_double, C.c_double, C.c_double, _f64p, _u8p, _f64p,
                                                    _u8p]
        lib.orc_functional_substitution.restype = C.c_double
        lib.orc_random2_sequence.argtypes = [C.c_uint32, C.c_int32, _f64p]
        lib.orc_icd_pass.argtypes = [P, _f32p, _f32p, _i32p, _i32p, _u8p, _i32p, C.c_int32, C.c_int32, _f32p,
                                     _f32p, _f32p]
        lib.orc_icd_pass.restype = C.c_int64
        _orc = lib
    return _orc


def _ref_name(timing: bool) -> str:
    return "libref_mbir4d_timing.so" if timing else "libref_mbir4d.so"


def ref_available(timing: bool = False) -> bool:
    return os.path.exists(os.path.join(REF_DIR, _ref_name(timing)))


def ref_lib(timing: bool = False) -> C.CDLL:
    """The reference MBIR_4D built from source: the cost-on build (cost.bin per
    iteration, the "Cost value increased" abort of XT_ICD_update.c:1171), or
    with timing=True the build with the reference Makefile's own
    -DNO_COST_CALCULATE -DNO_DEBUG (MBIR_4D/Makefile:3), which has neither."""
    if timing not in _ref:
        lib = C.CDLL(os.path.join(REF_DIR, _ref_name(timing)))
        P = C.POINTER(RefProblem)
        lib.ref_set_options.argtypes = [C.c_double, C.c_int, C.c_int]
        lib.ref_geometry.argtypes = [P, _f64p, _f64p, _f32p, _f32p, _i32p, _i32p]
        lib.ref_amatrix.argtypes = [P, C.c_int32, _u8p, _i32p, _f64p]
        lib.ref_error_sino_and_cost.argtypes = [P, _f32p, _f32p, _u8p, C.POINTER(C.c_double)]
        lib.ref_functional_substitution.argtypes = [P, C.c_int32, _f64p, _f64p, _f64p, _f64p, _u8p, _f64p, _u8p,
                                                    _f64p]
        lib.ref_random2_sequence.argtypes = [C.c_uint32, C.c_int32, _f64p]
        lib.ref_vsc_select.argtypes = [C.c_int32, C.c_int32, _f32p, C.c_int32, _u8p]
        lib.ref_vsc_select.restype = C.c_int32
        lib.ref_reconstruct.argtypes = [P, C.c_int32, C.c_int32, C.POINTER(C.POINTER(C.c_float))]
        lib.ref_offset_update.argtypes = [P, C.c_int32, _f32p, _f32p]
        lib.ref_variance_update.argtypes = [P, _f32p, _f32p, C.POINTER(C.c_double)]
        lib.ref_reconstruct.restype = C.c_int
        lib.ref_free.argtypes = [C.c_void_p]
        lib.ref_vox_updates.restype = C.c_longlong
        _ref[timing] = lib
    return _ref[timing]


# --------------------------------------------------------------------------- restatement


class Oracle:
    """Geometry plus the restated kernels for one problem at one voxel scale."""

    def __init__(self, pb: Problem, mult_xy: int = 1, mult_z: int = 1, num_threads: int = 2):
        lib = orc_lib()
        self.pb = pb
        self.g = OrcGeom()
        self.proj_idx = np.zeros(pb.proj_num, np.int32)
        self.proj_cnt = np.zeros(pb.recon_num, np.int32)
        f = lambda v: float(np.float32(v))  # the ABI passes these as float (MBIR_4D/XT_Engine.c:81)
        rc = lib.orc_init_geometry(C.byref(self.g), pb.proj_rows, pb.proj_cols, pb.proj_num, pb.recon_num,
                                   f(pb.vox_wid), f(pb.rot_center), f(pb.sig_s), f(pb.sig_t), f(pb.c_s), f(pb.c_t),
                                   mult_xy, mult_z, pb.mrf_p, pb.quad_convex, f(pb.huber_delta), f(pb.huber_T),
                                   num_threads,
                                   np.ascontiguousarray(pb.proj_times, np.float32),
                                   np.ascontiguousarray(pb.recon_times, np.float32), self.proj_idx, self.proj_cnt)
        if rc != 0:
            raise ValueError("oracle geometry rejected the problem")
        self.angles = np.ascontiguousarray(pb.proj_angles, np.float32)
        self.H_r = np.zeros((pb.proj_num, RESP_BINS + 1), np.float32)
        lib.orc_detector_response(C.byref(self.g), self.angles, self.H_r)
        # internal [view][col][row] sinogram layout (MBIR_4D/XT_Init.c:292-301)
        self.y = np.ascontiguousarray(pb.projections.reshape(pb.proj_num, pb.proj_rows, pb.proj_cols)
                                      .transpose(0, 2, 1), np.float32)
        self.w = np.ascontiguousarray(pb.weights.reshape(pb.proj_num, pb.proj_rows, pb.proj_cols)
                                      .transpose(0, 2, 1), np.float32)

    @property
    def shape(self):
        g = self.g
        return (g.N_time, g.N_z, g.N_y, g.N_x)

    def amatrix_column(self, view: int, row: int, col: int):
        idx = np.zeros(64, np.int32)
        val = np.zeros(64, np.float64)
        a = float(self.angles[view])
        n = orc_lib().orc_amatrix_column(C.byref(self.g), self.H_r, np.cos(np.float64(a)), np.sin(np.float64(a)),
                                         view, row, col, idx, val)
        return idx[:n].copy(), val[:n].copy()

    def forward(self, obj: np.ndarray) -> np.ndarray:
        ax = np.zeros((self.pb.proj_num, self.pb.proj_cols, self.pb.proj_rows), np.float64)
        orc_lib().orc_forward_project(C.byref(self.g), self.H_r, self.angles, self.proj_idx, self.proj_cnt,
                                      np.ascontiguousarray(obj, np.float32), ax)
        return ax

    def error_sino(self, obj: np.ndarray) -> np.ndarray:
        return (self.y.astype(np.float64) - self.forward(obj)).astype(np.float32)

    def cost(self, err: np.ndarray, obj: np.ndarray) -> tuple[float, float, float]:
        parts = np.zeros(2, np.float64)
        c = orc_lib().orc_cost(C.byref(self.g), np.ascontiguousarray(err, np.float32), self.w,
                               np.ascontiguousarray(obj, np.float32), parts)
        return c, parts[0], parts[1]

    def mask(self) -> np.ndarray:
        """Circular field-of-view mask of ICD_BackProject (XT_ICD_update.c:1127-1136)."""
        g = self.g
        k = np.arange(g.N_x, dtype=np.float64)
        j = np.arange(g.N_y, dtype=np.float64)
        x = g.x0 + (k + 0.5) * g.delta_xy
        y = g.y0 + (j + 0.5) * g.delta_xy
        return ((x[None, :] ** 2 + y[:, None] ** 2) < g.radius_obj * g.radius_obj).astype(np.uint8)

    def icd_pass(self, obj: np.ndarray, err: np.ndarray, order: np.ndarray, it: int) -> int:
        return int(orc_lib().orc_icd_pass(C.byref(self.g), self.H_r, self.angles, self.proj_idx, self.proj_cnt,
                                          np.ascontiguousarray(self.mask()), np.ascontiguousarray(order, np.int32),
                                          len(order), it, obj, err, self.w))

    def functional_substitution(self, V, th1, th2, nhood, nflag, tnhood, tflag) -> float:
        return orc_lib().orc_functional_substitution(C.byref(self.g), V, th1, th2,
                                                     np.ascontiguousarray(nhood, np.float64),
                                                     np.ascontiguousarray(nflag, np.uint8),
                                                     np.ascontiguousarray(tnhood, np.float64),
                                                     np.ascontiguousarray(tflag, np.uint8))


HAMMING_5X5 = np.array([[0.0064, 0.0432, 0.0800, 0.0432, 0.0064],
                        [0.0432, 0.2916, 0.5400, 0.2916, 0.0432],
                        [0.0800, 0.5400, 1.0000, 0.5400, 0.0800],
                        [0.0432, 0.2916, 0.5400, 0.2916, 0.0432],
                        [0.0064, 0.0432, 0.0800, 0.0432, 0.0064]])  # XT_NHICD.c:132-136
NHICD_ITERATIONS = 10  # XT_Init.c:406


def vsc_select(mag: np.ndarray, n_lines: int, nhicd_iterations: int = NHICD_ITERATIONS) -> np.ndarray:
    """NH-ICD voxel-line selection of one frame / z block
    (VSC_based_Voxel_Line_Select, XT_NHICD.c:164-216): the update-magnitude map
    filtered by the 5x5 Hamming window in FP64 in the reference's (p, q) order,
    stored as float (ComputeVSC, :128-161); threshold = the (N - k)-th smallest
    filtered value, N = ny nx, k = floor(n_lines / NHICD_Iterations)
    (RandomizedSelect's order statistic, :177-178); selected = filtered > threshold.
    Returns a bool [ny][nx] map (unmasked lines included, as the reference)."""
    mag = np.asarray(mag, np.float32)
    ny, nx = mag.shape
    acc = np.zeros((ny, nx), np.float64)
    pad = np.zeros((ny + 4, nx + 4), np.float64)
    pad[2:-2, 2:-2] = mag
    for p in range(5):
        for q in range(5):
            acc = acc + HAMMING_5X5[p, q] * pad[p:p + ny, q:q + nx]
    filt = acc.astype(np.float32)
    k = n_lines // nhicd_iterations
    N = ny * nx
    thresh = np.sort(filt.ravel())[N - k - 1]
    return filt > thresh


def ref_vsc_select(mag: np.ndarray, n_lines: int) -> np.ndarray:
    """The reference's own VSC_based_Voxel_Line_Select on one frame (oracle/_ref)."""
    mag = np.ascontiguousarray(mag, np.float32)
    out = np.zeros(mag.shape, np.uint8)
    ref_lib().ref_vsc_select(mag.shape[0], mag.shape[1], mag, n_lines, out)
    return out.astype(bool)


def random2_sequence(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float64)
    orc_lib().orc_random2_sequence(seed, n, out)
    return out


# --------------------------------------------------------------------------- reference (built from source)


def ref_geometry(pb: Problem, mult_xy: int = 1, mult_z: int = 1):
    lib = ref_lib()
    lib.ref_set_options(pb.mrf_p, 1000, 0)
    s = pb.ref_struct(mult_xy, mult_z)
    scal = np.zeros(32, np.float64)
    filt = np.zeros(27, np.float64)
    H_r = np.zeros((pb.proj_num, RESP_BINS + 1), np.float32)
    H_t = np.zeros(RESP_BINS + 1, np.float32)
    idx = np.zeros(pb.proj_num, np.int32)
    cnt = np.zeros(pb.recon_num, np.int32)
    if lib.ref_geometry(C.byref(s), scal, filt, H_r, H_t, idx, cnt) != 0:
        raise RuntimeError("reference initStructures failed")
    return dict(scal=scal, filt=filt, H_r=H_r, H_t=H_t, proj_idx=idx, proj_cnt=cnt)


def ref_amatrix(pb: Problem, mult_xy: int = 1, mult_z: int = 1):
    lib = ref_lib()
    lib.ref_set_options(pb.mrf_p, 1000, 0)
    s = pb.ref_struct(mult_xy, mult_z)
    n = pb.proj_cols // mult_xy
    kmax = 2 * mult_xy + 1
    count = np.zeros((pb.proj_num, n, n), np.uint8)
    index = np.zeros((pb.proj_num, n, n, kmax), np.int32)
    value = np.zeros((pb.proj_num, n, n, kmax), np.float64)
    if lib.ref_amatrix(C.byref(s), kmax, count, index, value) != 0:
        raise RuntimeError("reference A-matrix failed")
    return count, index, value


def ref_error_sino_and_cost(pb: Problem, obj: np.ndarray, mult_xy: int = 1, mult_z: int = 1):
    lib = ref_lib()
    lib.ref_set_options(pb.mrf_p, 1000, 0)
    s = pb.ref_struct(mult_xy, mult_z)
    err = np.zeros((pb.proj_num, pb.proj_cols, pb.proj_rows), np.float32)
    sel = np.zeros(err.shape, np.uint8)
    cost = C.c_double(0)
    if lib.ref_error_sino_and_cost(C.byref(s), np.ascontiguousarray(obj, np.float32), err, sel,
                                   C.byref(cost)) != 0:
        raise RuntimeError("reference error sinogram failed")
    return err, sel, cost.value


def ref_functional_substitution(pb: Problem, V, th1, th2, nhood, nflag, tnhood, tflag):
    lib = ref_lib()
    lib.ref_set_options(pb.mrf_p, 1000, 0)
    s = pb.ref_struct()
    n = len(V)
    out = np.zeros(n, np.float64)
    lib.ref_functional_substitution(C.byref(s), n, np.ascontiguousarray(V, np.float64),
                                    np.ascontiguousarray(th1, np.float64), np.ascontiguousarray(th2, np.float64),
                                    np.ascontiguousarray(nhood, np.float64), np.ascontiguousarray(nflag, np.uint8),
                                    np.ascontiguousarray(tnhood, np.float64), np.ascontiguousarray(tflag, np.uint8),
                                    out)
    return out


def ref_random2_sequence(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float64)
    ref_lib().ref_random2_sequence(seed, n, out)
    return out


def ref_offset_update(pb: Problem, mode: int, err: np.ndarray, d: np.ndarray):
    """The reference's update_Sinogram_Offset (MBIR_4D/XT_ICD_update.c:749-923)
    on err [N_p][N_r][N_t] and offset d [N_r][N_t]; returns the updated copies."""
    e2 = np.ascontiguousarray(err, np.float32).copy()
    d2 = np.ascontiguousarray(d, np.float32).copy()
    s = pb.ref_struct()
    if ref_lib().ref_offset_update(C.byref(s), mode, e2, d2) != 0:
        raise RuntimeError("reference offset update failed")
    return e2, d2


def ref_variance_update(pb: Problem, err: np.ndarray, w: np.ndarray, var_est: float):
    """The reference's update_variance_parameter (MBIR_4D/XT_ICD_update.c:716-747)
    on err and weights w ([N_p][N_r][N_t]) with the current variance; returns
    (new weights, new variance)."""
    w2 = np.ascontiguousarray(w, np.float32).copy()
    v = C.c_double(var_est)
    if ref_lib().ref_variance_update(C.byref(pb.ref_struct()), np.ascontiguousarray(err, np.float32), w2,
                                     C.byref(v)) != 0:
        raise RuntimeError("reference variance update failed")
    return w2, v.value


def ref_reconstruct(pb: Problem, workdir: str, max_iter: int = 1000, num_stages: int = 0, threads: int = 0,
                    remove_rings: int = 0, timing: bool = False):
    """Run the reference's ``reconstruct`` in ``workdir`` (remove_rings: its
    ring-correction mode, 0 = off; timing: the build without the cost pass).

    Returns (object with halo [N_time][N_z+2][N_y][N_x] as the reference
    returns it, FP64 cost per iteration from cost.bin -- None for the timing
    build, which writes none -- and the voxel updates counted).
    """
    lib = ref_lib(timing)
    lib.ref_set_options(pb.mrf_p, max_iter, num_stages)
    lib.ref_reset_vox_updates()
    s = pb.ref_struct()
    out = C.POINTER(C.c_float)()
    cwd = os.getcwd()
    os.makedirs(workdir, exist_ok=True)
    os.chdir(workdir)
    try:
        rc = lib.ref_reconstruct(C.byref(s), threads, remove_rings, C.byref(out))
    finally:
        os.chdir(cwd)
    if rc != 0:
        raise RuntimeError(f"reference reconstruct returned {rc}")
    n = pb.recon_num * (pb.proj_rows + 2) * pb.proj_cols * pb.proj_cols
    obj = np.ctypeslib.as_array(out, shape=(n,)).copy().reshape(pb.recon_num, pb.proj_rows + 2, pb.proj_cols,
                                                                  pb.proj_cols)
    lib.ref_free(out)
    cpath = os.path.join(workdir, "cost.bin")
    cost = None if timing else np.fromfile(cpath, dtype=np.float64)
    return obj, cost, int(lib.ref_vox_updates())


def ref_reconstruct_and_cost(pb: Problem, workdir: str, max_iter: int, num_stages: int = 1, threads: int = 0):
    """The reference's ``reconstruct`` as it ships (the build without the cost
    pass, so no rounding-level cost increase can abort it) for max_iter
    iterations, then the reference's own MAP cost (computeCost,
    XT_ICD_update.c:185-318) of the object it returned, evaluated on a fresh
    error sinogram (initErrorSinogam) by the cost-on build.

    Returns (object without halo [N_time][N_z][N_y][N_x], that cost, voxel
    updates)."""
    obj, _, upd = ref_reconstruct(pb, workdir, max_iter=max_iter, num_stages=num_stages, threads=threads,
                                  timing=True)
    x = np.ascontiguousarray(obj[:, 1:-1])
    _, _, cost = ref_error_sino_and_cost(pb, x)
    return x, cost, upd


# --------------------------------------------------------------------------- PCMBIR reference (built from source)


class PcParams(C.Structure):
    """Mirror of PcParams in oracle/ref_pc_harness.c."""
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("delta_rows", C.c_double), ("delta_cols", C.c_double),
                ("wavelength", C.c_double), ("distance", C.c_double), ("window_sigma", C.c_double),
                ("mag_sig_s", C.c_double), ("mag_c_s", C.c_double), ("phase_sig_s", C.c_double),
                ("phase_c_s", C.c_double), ("delta_over_beta", C.c_double), ("mrf_p", C.c_double)]


_ref_pc = None


def ref_pc_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_pcmbir.so"))


def ref_pc_lib() -> C.CDLL:
    global _ref_pc
    if _ref_pc is None:
        lib = C.CDLL(os.path.join(REF_DIR, "libref_pcmbir.so"))
        P = C.POINTER(PcParams)
        lib.ref_pc_fresnel.argtypes = [P, _f64p, _f64p, C.c_int]
        lib.ref_pc_sd_iter.argtypes = [P] + [_f64p] * 11 + [C.c_double]
        lib.ref_pc_sd_iter.restype = C.c_double
        lib.ref_pc_phase_projection.argtypes = [P] + [_f64p] * 8
        lib.ref_pc_nms.argtypes = [P, C.c_int32, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, _u8p, C.c_double,
                                   C.c_int32, C.c_double, _i32p]
        lib.ref_pc_estimate.argtypes = [P] + [_f64p] * 15 + [C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                                              C.c_double]
        lib.ref_pc_paganin.argtypes = [P, _f64p, _f64p, _f64p, C.c_double, _f64p, _f64p]
        lib.ref_pc_filter.argtypes = [P, _f64p, _f64p]
        _ref_pc = lib
    return _ref_pc


def pc_params(g) -> PcParams:
    return PcParams(g.rows, g.cols, g.delta_rows, g.delta_cols, g.wavelength, g.distance, g.window_sigma,
                    g.mag_sig_s, g.mag_c_s, g.phase_sig_s, g.phase_c_s, g.delta_over_beta, g.mrf_p)


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ref_pc_fresnel(g, x, herm=False):
    xi = np.ascontiguousarray(np.stack([x.real, x.imag], -1), np.float64)
    out = np.zeros_like(xi)
    ref_pc_lib().ref_pc_fresnel(C.byref(pc_params(g)), xi, out, 1 if herm else 0)
    return out[..., 0] + 1j * out[..., 1]


def ref_pc_sd_iter(g, y, om, D, w, lam, buf):
    arrs = [_c(y.real), _c(np.zeros_like(y.real)), _c(om.real), _c(om.imag), _c(D.real), _c(D.imag), _c(w.real),
            _c(w.imag), _c(lam), _c(buf.real), _c(buf.imag)]
    t = ref_pc_lib().ref_pc_sd_iter(C.byref(pc_params(g)), arrs[0], arrs[1], arrs[2], arrs[3], arrs[4], arrs[5],
                                    arrs[6], arrs[7], arrs[8], arrs[9], arrs[10], g.nu)
    return arrs[6] + 1j * arrs[7], arrs[2] + 1j * arrs[3], t


def ref_pc_phase_projection(g, y, D, w):
    om_r, om_i = np.zeros(y.shape), np.zeros(y.shape)
    ref_pc_lib().ref_pc_phase_projection(C.byref(pc_params(g)), _c(y.real), _c(np.zeros(y.shape)), _c(D.real),
                                         _c(D.imag), _c(w.real), _c(w.imag), om_r, om_i)
    return om_r + 1j * om_i


def ref_pc_nms(g, zr1, zi1, br, bi, nbr_r, nbr_i, flag, max_iter=50, thresh=0.005):
    n = len(zr1)
    zr = np.zeros((n, 4))
    zi = np.zeros((n, 4))
    zr[:, 1], zi[:, 1] = zr1, zi1
    iters = np.zeros(n, np.int32)
    ref_pc_lib().ref_pc_nms(C.byref(pc_params(g)), n, zr, zi, _c(br), _c(bi), _c(nbr_r), _c(nbr_i),
                            np.ascontiguousarray(flag, np.uint8), g.nu, max_iter, thresh, iters)
    return zr[:, 1].copy(), zi[:, 1].copy(), iters


def ref_pc_estimate(g, y, om, D, zr, zi, lam, w, workdir, pret_iters=100, sd_iters=100, nms_iters=50):
    R, Cc = y.shape
    z_r = np.zeros((R, Cc, 4))
    z_i = np.zeros((R, Cc, 4))
    z_r[..., 1], z_i[..., 1] = zr, zi
    om_r, om_i = _c(om.real), _c(om.imag)
    w_r, w_i = _c(w.real), _c(w.imag)
    v_r, v_i = np.zeros((R, Cc)), np.zeros((R, Cc))
    cwd = os.getcwd()
    os.makedirs(workdir, exist_ok=True)
    os.chdir(workdir)
    try:
        ref_pc_lib().ref_pc_estimate(C.byref(pc_params(g)), _c(y.real), _c(np.zeros((R, Cc))), om_r, om_i, _c(D.real),
                                     _c(D.imag), z_r, z_i, _c(lam), _c(zr), _c(zi), w_r, w_i, v_r, v_i, nms_iters,
                                     sd_iters, pret_iters, g.mu, g.nu)
        cost = np.fromfile("pret_cost_proj_0.bin", np.float64) if os.path.exists(
            "pret_cost_proj_0.bin") else None
    finally:
        os.chdir(cwd)
    return z_r[..., 1].copy(), z_i[..., 1].copy(), w_r + 1j * w_i, v_r + 1j * v_i, om_r + 1j * om_i, cost


def ref_pc_reconstruct(workdir: str, measurements, brights, proj_angles, proj_times, recon_times, proj_rows,
                       proj_cols, proj_num, recon_num, vox_wid, rot_center, mag_sig_s, mag_sig_t, mag_c_s, mag_c_t,
                       phase_sig_s, phase_sig_t, phase_c_s, phase_c_t, convg_thresh, obj2det_dist, light_energy,
                       pag_regparam, restart=0, recon_type=1, pret_max_iter: int = 100, mrf_p: float = 1.2,
                       threads: int = 0) -> None:
    """The reference's own phcontomo_reconstruct (PCMBIR_3D/XT_Engine.c:82-197)
    run in `workdir`, where it leaves its output files (pag_*_ret.bin for
    recon_type 1; *_pret_aux, *_pret_dual, omega_*, pret_cost_proj_<i> ... for
    recon_type 2). pret_max_iter sets PRet_MaxIter (XT_Init.c:516, 100 as
    shipped); threads sets the OpenMP thread count (0: the default)."""
    lib = ref_pc_lib()
    C.c_int.in_dll(lib, "oracle_ref_pret_max_iter").value = int(pret_max_iter)
    C.c_double.in_dll(lib, "oracle_ref_pc_mrf_p").value = float(mrf_p)
    fp = C.POINTER(C.c_float)
    lib.phcontomo_reconstruct.argtypes = [C.POINTER(fp), C.POINTER(fp)] + [C.c_void_p] * 5 + [C.c_int32] * 4 + \
        [C.c_float] * 14 + [C.c_uint8, C.c_uint8, C.c_void_p]
    lib.phcontomo_reconstruct.restype = C.c_int
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in
            (measurements, brights, proj_angles, proj_times, recon_times)]
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    if threads > 0:
        try:
            omp = C.CDLL("libgomp.so.1")
            omp.omp_set_num_threads(int(threads))
        except OSError:
            pass
    mag, ph = fp(), fp()
    cwd = os.getcwd()
    os.makedirs(workdir, exist_ok=True)
    os.chdir(workdir)
    dbg = libc.fopen(b"debug.txt", b"a")
    try:
        rc = lib.phcontomo_reconstruct(C.byref(mag), C.byref(ph), *(a.ctypes.data for a in arrs), proj_rows, proj_cols,
                                       proj_num, recon_num, vox_wid, rot_center, mag_sig_s, mag_sig_t, mag_c_s, mag_c_t,
                                       phase_sig_s, phase_sig_t, phase_c_s, phase_c_t, convg_thresh, obj2det_dist,
                                       light_energy, pag_regparam, restart, recon_type, dbg)
    finally:
        libc.fclose(dbg)
        os.chdir(cwd)
    if rc != 0:
        raise RuntimeError(f"reference phcontomo_reconstruct returned {rc}")


def ref_pc_paganin(g, meas, D):
    zr, zi = np.zeros(meas.shape), np.zeros(meas.shape)
    ref_pc_lib().ref_pc_paganin(C.byref(pc_params(g)), _c(meas), _c(D.real), _c(D.imag), g.wavenumber, zr, zi)
    return zr, zi


def ref_pc_filter(g):
    f, d = np.zeros(27), np.zeros(4)
    ref_pc_lib().ref_pc_filter(C.byref(pc_params(g)), f, d)
    return f.reshape(3, 3, 3), d.reshape(2, 2)


def ref_pc_forward_project(mag, phase, angles, proj_rows, proj_cols, vox_wid, rot_center, obj2det_dist,
                           light_energy, pag_regparam, workdir):
    """The reference's own phcontomo_forward_project (PCMBIR_3D/XT_Engine.c:199-253,
    XT_genSinogram.c:59-343) on phantoms mag / phase [P_z][P_xy][P_xy]: the
    phantoms are written where the patched build reads them
    (oracle_mag_phantom_input.bin / oracle_phase_phantom_input.bin in
    `workdir`), the phantom-size globals are set, and the reference runs in
    `workdir`. Returns (measurements [proj_num][proj_rows][proj_cols], brights,
    SimMagProjs, SimPhaseProjs [proj_num][P_z][P_xy] FP64, mag_phantom,
    phase_phantom FP64)."""
    mag = np.ascontiguousarray(mag, np.float32)
    phase = np.ascontiguousarray(phase, np.float32)
    P_z, P_xy, _ = mag.shape
    lib = ref_pc_lib()
    C.c_int.in_dll(lib, "oracle_ref_phantom_xy").value = P_xy
    C.c_int.in_dll(lib, "oracle_ref_phantom_z").value = P_z
    fp = C.POINTER(C.c_float)
    lib.phcontomo_forward_project.argtypes = [C.POINTER(fp), C.POINTER(fp), _f32p, C.c_int32, C.c_int32, C.c_int32,
                                              C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p]
    lib.phcontomo_forward_project.restype = C.c_int
    V = len(angles)
    meas = np.zeros(V * proj_rows * proj_cols, np.float32)
    br = np.zeros(proj_rows * proj_cols, np.float32)
    pm, pb = meas.ctypes.data_as(fp), br.ctypes.data_as(fp)
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    cwd = os.getcwd()
    os.makedirs(workdir, exist_ok=True)
    os.chdir(workdir)
    dbg = libc.fopen(b"debug.txt", b"w")
    try:
        mag.tofile("oracle_mag_phantom_input.bin")
        phase.tofile("oracle_phase_phantom_input.bin")
        rc = lib.phcontomo_forward_project(C.byref(pm), C.byref(pb), np.ascontiguousarray(angles, np.float32),
                                           proj_rows, proj_cols, V, vox_wid, rot_center, obj2det_dist, light_energy,
                                           pag_regparam, dbg)
        libc.fclose(dbg)
        if rc != 0:
            raise RuntimeError("reference phcontomo_forward_project failed")
        n = V * P_z * P_xy
        out = (meas.reshape(V, proj_rows, proj_cols), br.reshape(proj_rows, proj_cols),
               np.fromfile("SimMagProjs.bin", np.float64, n).reshape(V, P_z, P_xy),
               np.fromfile("SimPhaseProjs.bin", np.float64, n).reshape(V, P_z, P_xy),
               np.fromfile("mag_phantom.bin", np.float64).reshape(P_z, P_xy, P_xy),
               np.fromfile("phase_phantom.bin", np.float64).reshape(P_z, P_xy, P_xy))
    finally:
        os.chdir(cwd)
    return out
