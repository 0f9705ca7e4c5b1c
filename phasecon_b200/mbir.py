"""Python mirror of phasecon's MBIR_4D interface over libmbirgpu's C ABI.

``reconstruct`` takes the same arguments, in the same order and with the same
meaning, as the reference's C entry point (MBIR_4D/XT_Engine.c:81) and returns
the same object layout ([recon_num][proj_rows+2][proj_cols][proj_cols], one
zero halo slice above and below each frame's volume). ``Session`` exposes one
resident stage for tests, benchmarks and callers that drive iterations
themselves. Everything runs in libmbirgpu.so on the GPU; there is no CPU
fallback: if the library is missing or no CUDA device is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libmbirgpu.so")

#: every symbol include/mbirgpu.h declares
EXPORTS = (
    "reconstruct", "mbirgpu_default_options", "mbirgpu_set_options", "mbirgpu_get_options", "mbirgpu_last_error",
    "mbirgpu_session_create", "mbirgpu_session_destroy", "mbirgpu_session_info_get", "mbirgpu_session_set_stream",
    "mbirgpu_session_set_timing", "mbirgpu_session_set_object", "mbirgpu_session_get_object",
    "mbirgpu_session_object_device", "mbirgpu_session_refresh_error", "mbirgpu_session_get_error",
    "mbirgpu_session_cost", "mbirgpu_session_icd_iteration", "mbirgpu_session_forward_project",
    "mbirgpu_session_back_project", "mbirgpu_session_get_amatrix", "mbirgpu_session_get_detector_response",
    "mbirgpu_session_run", "mbirgpu_session_forward_project_noalloc", "mbirgpu_session_nh_select",
    "mbirgpu_session_fbp", "mbirgpu_session_set_object_fbp", "mbirgpu_session_set_object_zero",
    "mbirgpu_session_set_ring_correction",
    "mbirgpu_session_get_offset", "mbirgpu_session_update_offset", "mbirgpu_session_set_variance_estimation",
    "mbirgpu_session_update_variance", "mbirgpu_session_get_variance",
    "mbirgpu_unet_create", "mbirgpu_unet_destroy", "mbirgpu_unet_num_params", "mbirgpu_unet_set_input_scale",
    "mbirgpu_unet_get_input_scale", "mbirgpu_unet_get_params", "mbirgpu_unet_set_params", "mbirgpu_unet_forward",
    "mbirgpu_unet_gradients", "mbirgpu_unet_train_step", "mbirgpu_session_set_object_unet",
    "mbirgpu_unet_set_tensor_path", "mbirgpu_unet_get_tensor_path",
    "mbirgpu_batch_create", "mbirgpu_batch_destroy", "mbirgpu_batch_run", "mbirgpu_batch_problem_info",
    "mbirgpu_batch_get_object", "mbirgpu_batch_cost", "mbirgpu_reconstruct_batch",
    "phcontomo_reconstruct", "mbirgpu_pc_default_options", "mbirgpu_pc_session_create", "mbirgpu_pc_session_destroy",
    "mbirgpu_pc_fresnel", "mbirgpu_pc_time_fresnel", "mbirgpu_pc_paganin", "mbirgpu_pc_set_z", "mbirgpu_pc_init_admm", "mbirgpu_pc_set_state",
    "mbirgpu_pc_get_state", "mbirgpu_pc_sd_step", "mbirgpu_pc_nms_sweep", "mbirgpu_pc_run",
    "phcontomo_forward_project", "mbirgpu_pc_sim_default_options", "mbirgpu_pc_sim_set_options",
    "mbirgpu_pc_sim_get_options", "mbirgpu_pc_simulate",
)


class MbirError(RuntimeError):
    pass


class Options(C.Structure):
    _fields_ = [
        ("mrf_p", C.c_double), ("mrf_q", C.c_double), ("alpha", C.c_double), ("max_iterations", C.c_int32),
        ("num_stages", C.c_int32), ("cost_rel_tol", C.c_double), ("zero_skipping", C.c_int32),
        ("write_files", C.c_int32), ("compute_cost", C.c_int32), ("refresh_every", C.c_int32),
        ("sv_size", C.c_int32), ("cta_warps", C.c_int32), ("icd_unroll", C.c_int32), ("seed", C.c_uint64),
        ("nhicd_passes", C.c_int32), ("sv_colors", C.c_int32), ("stage_records", C.c_int32),
        ("nh_sv_size", C.c_int32), ("nh_sv_colors", C.c_int32), ("nh_cta_warps", C.c_int32),
        ("nh_work_lists", C.c_int32), ("autotune", C.c_int32),
        ("graph_iterations", C.c_int32),
    ]


class ProblemStruct(C.Structure):
    _fields_ = [
        ("projections", C.c_void_p), ("weights", C.c_void_p), ("proj_angles", C.c_void_p),
        ("proj_times", C.c_void_p), ("recon_times", C.c_void_p),
        ("proj_rows", C.c_int32), ("proj_cols", C.c_int32), ("proj_num", C.c_int32), ("recon_num", C.c_int32),
        ("vox_wid", C.c_float), ("rot_center", C.c_float), ("sig_s", C.c_float), ("sig_t", C.c_float),
        ("c_s", C.c_float), ("c_t", C.c_float), ("convg_thresh", C.c_float), ("quad_convex", C.c_int32),
        ("huber_delta", C.c_float), ("huber_T", C.c_float),
    ]


class SessionInfo(C.Structure):
    _fields_ = [
        ("N_r", C.c_int32), ("N_t", C.c_int32), ("N_p", C.c_int32), ("N_time", C.c_int32), ("N_x", C.c_int32),
        ("N_y", C.c_int32), ("N_z", C.c_int32), ("mult_xy", C.c_int32), ("mult_z", C.c_int32),
        ("max_views", C.c_int32), ("kmax", C.c_int32), ("sv_size", C.c_int32), ("cta_warps", C.c_int32),
        ("masked_columns", C.c_int64), ("nnz", C.c_int64), ("delta_t", C.c_double), ("device_bytes", C.c_size_t),
        ("sv_colors", C.c_int32),
    ]


class IterStats(C.Structure):
    _fields_ = [
        ("voxel_updates", C.c_int64), ("zero_skipped", C.c_int64), ("sum_abs_update", C.c_double),
        ("sum_abs_value", C.c_double), ("kernel_ms", C.c_double), ("kernel_launches", C.c_int32),
    ]


class BatchStats(C.Structure):
    _fields_ = [
        ("voxel_updates", C.c_int64), ("device_ms", C.c_double), ("graph_launches", C.c_int32),
        ("kernel_launches_per_iteration", C.c_int32), ("problems_converged", C.c_int32), ("sv_size", C.c_int32),
        ("cta_warps", C.c_int32), ("sv_colors", C.c_int32),
    ]


_lib = None


def lib() -> C.CDLL:
    """Load libmbirgpu.so; raise if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MbirError(f"{LIB_PATH} is missing: build it with `python -m phasecon_b200.build`")
        L = C.CDLL(LIB_PATH)
        fp = C.POINTER(C.c_float)
        L.reconstruct.argtypes = [C.POINTER(fp), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_float,
                                  C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32, C.c_int32, C.c_float,
                                  C.c_float, C.c_uint8, C.c_void_p]
        L.reconstruct.restype = C.c_int
        L.mbirgpu_default_options.argtypes = [C.POINTER(Options)]
        L.mbirgpu_default_options.restype = None
        L.mbirgpu_set_options.argtypes = [C.POINTER(Options)]
        L.mbirgpu_get_options.argtypes = [C.POINTER(Options)]
        L.mbirgpu_last_error.restype = C.c_char_p
        L.mbirgpu_session_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(ProblemStruct), C.POINTER(Options),
                                             C.c_int32, C.c_int32, C.c_void_p]
        L.mbirgpu_session_destroy.argtypes = [C.c_void_p]
        L.mbirgpu_session_info_get.argtypes = [C.c_void_p, C.POINTER(SessionInfo)]
        L.mbirgpu_session_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        L.mbirgpu_session_set_timing.argtypes = [C.c_void_p, C.c_int32]
        L.mbirgpu_session_set_object.argtypes = [C.c_void_p, C.c_void_p]
        L.mbirgpu_session_get_object.argtypes = [C.c_void_p, C.c_void_p]
        L.mbirgpu_session_object_device.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.mbirgpu_session_refresh_error.argtypes = [C.c_void_p]
        L.mbirgpu_session_get_error.argtypes = [C.c_void_p, C.c_void_p]
        L.mbirgpu_session_cost.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                           C.POINTER(C.c_double)]
        L.mbirgpu_session_icd_iteration.argtypes = [C.c_void_p, C.c_int32, C.POINTER(IterStats)]
        L.mbirgpu_session_forward_project.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.mbirgpu_session_back_project.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.mbirgpu_session_forward_project_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.mbirgpu_session_nh_select.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.mbirgpu_session_fbp.argtypes = [C.c_void_p, C.c_void_p]
        L.mbirgpu_session_set_object_fbp.argtypes = [C.c_void_p]
        L.mbirgpu_session_set_object_zero.argtypes = [C.c_void_p]
        L.mbirgpu_session_set_ring_correction.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.mbirgpu_session_update_offset.argtypes = [C.c_void_p]
        L.mbirgpu_session_get_offset.argtypes = [C.c_void_p, C.c_void_p]
        L.mbirgpu_session_set_variance_estimation.argtypes = [C.c_void_p, C.c_int32]
        L.mbirgpu_session_update_variance.argtypes = [C.c_void_p]
        L.mbirgpu_session_get_variance.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.mbirgpu_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_void_p, C.c_int32, C.POINTER(Options),
                                           C.c_void_p]
        L.mbirgpu_batch_destroy.argtypes = [C.c_void_p]
        L.mbirgpu_batch_run.argtypes = [C.c_void_p, C.c_int32, C.POINTER(BatchStats)]
        L.mbirgpu_batch_problem_info.argtypes = [C.c_void_p, C.c_int32, C.POINTER(SessionInfo),
                                                 C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.mbirgpu_batch_get_object.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.mbirgpu_batch_cost.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]
        L.mbirgpu_reconstruct_batch.argtypes = [C.POINTER(C.POINTER(C.c_float)), C.c_void_p, C.c_int32, C.c_int32]
        L.mbirgpu_session_get_amatrix.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.mbirgpu_session_get_detector_response.argtypes = [C.c_void_p, C.c_void_p]
        L.mbirgpu_session_run.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_int32),
                                          C.POINTER(IterStats)]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise MbirError(lib().mbirgpu_last_error().decode(errors="replace"))


def default_options() -> Options:
    o = Options()
    lib().mbirgpu_default_options(C.byref(o))
    return o


def set_options(**kw) -> Options:
    """Update the process-wide options (former compile-time constants)."""
    o = Options()
    _check(lib().mbirgpu_get_options(C.byref(o)))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    _check(lib().mbirgpu_set_options(C.byref(o)))
    return o


def get_options() -> Options:
    o = Options()
    _check(lib().mbirgpu_get_options(C.byref(o)))
    return o


@dataclass
class Problem:
    """Arguments of reconstruct() (MBIR_4D/XT_Engine.c:50-80), ABI layouts."""
    projections: np.ndarray   # [proj_num][proj_rows][proj_cols]
    weights: np.ndarray       # [proj_num][proj_rows][proj_cols]
    proj_angles: np.ndarray   # [proj_num]
    proj_times: np.ndarray    # [proj_num]
    recon_times: np.ndarray   # [recon_num + 1]
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

    def arrays(self):
        return [np.ascontiguousarray(a, dtype=np.float32) for a in
                (self.projections, self.weights, self.proj_angles, self.proj_times, self.recon_times)]


def reconstruct(projections, weights, proj_angles, proj_times, recon_times, proj_rows, proj_cols, proj_num,
                recon_num, vox_wid, rot_center, sig_s, sig_t, c_s, c_t, convg_thresh, remove_rings=0,
                quad_convex=1, huber_delta=0.5, huber_T=4.0, restart=0, debug_file=None) -> np.ndarray:
    """The reference's reconstruct(), run on the GPU.

    Returns the object as the reference returns it:
    [recon_num][proj_rows+2][proj_cols][proj_cols] float32 with zero halo slices.
    Raises MbirError where the reference returns -1.
    """
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in
            (projections, weights, proj_angles, proj_times, recon_times)]
    out = C.POINTER(C.c_float)()
    fp = None
    if debug_file is not None:
        libc = C.CDLL(None)
        libc.fopen.restype = C.c_void_p
        libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
        libc.fclose.argtypes = [C.c_void_p]
        fp = libc.fopen(str(debug_file).encode(), b"w")
    try:
        rc = lib().reconstruct(C.byref(out), *(a.ctypes.data for a in arrs), proj_rows, proj_cols, proj_num,
                               recon_num, vox_wid, rot_center, sig_s, sig_t, c_s, c_t, convg_thresh, remove_rings,
                               quad_convex, huber_delta, huber_T, restart, fp)
    finally:
        if fp:
            libc.fclose(fp)
    _check(rc)
    n = recon_num * (proj_rows + 2) * proj_cols * proj_cols
    obj = np.ctypeslib.as_array(out, shape=(n,)).copy()
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    libc.free(C.cast(out, C.c_void_p))
    return obj.reshape(recon_num, proj_rows + 2, proj_cols, proj_cols)


class Session:
    """One multi-resolution stage of one problem resident on the GPU."""

    def __init__(self, pb: Problem, mult_xy: int = 1, mult_z: int = 1, options: Options | None = None,
                 stream: int | None = None):
        self._arrs = pb.arrays()
        ps = ProblemStruct(*(a.ctypes.data for a in self._arrs), pb.proj_rows, pb.proj_cols, pb.proj_num,
                           pb.recon_num, pb.vox_wid, pb.rot_center, pb.sig_s, pb.sig_t, pb.c_s, pb.c_t,
                           pb.convg_thresh, pb.quad_convex, pb.huber_delta, pb.huber_T)
        self.h = C.c_void_p()
        opt = options if options is not None else get_options()
        _check(lib().mbirgpu_session_create(C.byref(self.h), C.byref(ps), C.byref(opt), mult_xy, mult_z,
                                            C.c_void_p(stream or 0)))
        self.pb = pb
        info = SessionInfo()
        _check(lib().mbirgpu_session_info_get(self.h, C.byref(info)))
        self.info = info

    def close(self):
        if self.h:
            lib().mbirgpu_session_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        i = self.info
        return (i.N_time, i.N_z, i.N_y, i.N_x)

    @property
    def sino_shape(self):
        i = self.info
        return (i.N_p, i.N_r, i.N_t)

    def set_stream(self, stream: int) -> None:
        _check(lib().mbirgpu_session_set_stream(self.h, C.c_void_p(stream)))

    def set_timing(self, on: bool) -> None:
        _check(lib().mbirgpu_session_set_timing(self.h, 1 if on else 0))

    def set_object(self, obj: np.ndarray) -> None:
        a = np.ascontiguousarray(obj, np.float32).reshape(self.shape)
        _check(lib().mbirgpu_session_set_object(self.h, a.ctypes.data))

    def get_object(self, out: np.ndarray | None = None) -> np.ndarray:
        """The object [N_time][N_z][N_y][N_x]; into `out` (a C-contiguous float32
        array of that shape, e.g. in pinned memory) when given."""
        if out is None:
            out = np.zeros(self.shape, np.float32)
        elif out.dtype != np.float32 or out.shape != tuple(self.shape) or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float32 array of shape {tuple(self.shape)}")
        _check(lib().mbirgpu_session_get_object(self.h, out.ctypes.data))
        return out

    def refresh_error(self) -> None:
        _check(lib().mbirgpu_session_refresh_error(self.h))

    def get_error(self) -> np.ndarray:
        a = np.zeros(self.sino_shape, np.float32)
        _check(lib().mbirgpu_session_get_error(self.h, a.ctypes.data))
        return a

    def cost(self):
        t, d, p = C.c_double(), C.c_double(), C.c_double()
        _check(lib().mbirgpu_session_cost(self.h, C.byref(t), C.byref(d), C.byref(p)))
        return t.value, d.value, p.value

    def icd_iteration(self, it: int) -> IterStats:
        s = IterStats()
        _check(lib().mbirgpu_session_icd_iteration(self.h, it, C.byref(s)))
        return s

    def run(self, max_iter: int):
        costs = np.zeros(max_iter + 1, np.float64)
        n = C.c_int32()
        s = IterStats()
        _check(lib().mbirgpu_session_run(self.h, max_iter, costs.ctypes.data, C.byref(n), C.byref(s)))
        return costs[:n.value + 1], s

    def forward_project(self, obj: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(obj, np.float32).reshape(self.shape)
        out = np.zeros(self.sino_shape, np.float32)
        _check(lib().mbirgpu_session_forward_project(self.h, a.ctypes.data, out.ctypes.data))
        return out

    def forward_project_noalloc(self, object_dev: int, sino_dev: int) -> None:
        """A x from a device object [N_time][N_z][N_y][N_x] into a device
        sinogram [N_p][N_r][N_t] (raw device addresses), allocating nothing;
        enqueued on the session's stream, not waited for."""
        _check(lib().mbirgpu_session_forward_project_noalloc(self.h, C.c_void_p(object_dev), C.c_void_p(sino_dev)))

    def fbp(self) -> np.ndarray:
        """Filtered back-projection of the measurements, [N_time][N_z][N_y][N_x]."""
        a = np.zeros(self.shape, np.float32)
        _check(lib().mbirgpu_session_fbp(self.h, a.ctypes.data))
        return a

    def set_object_fbp(self) -> None:
        _check(lib().mbirgpu_session_set_object_fbp(self.h))

    def set_object_zero(self) -> None:
        """x = 0 on the device, then e = y - A x (no host copy)."""
        _check(lib().mbirgpu_session_set_object_zero(self.h))

    def set_ring_correction(self, remove_rings: int, offset: np.ndarray | None = None) -> None:
        """Estimate a per-detector-pixel offset d (remove_rings 1, 2, 3; 0 off),
        starting from offset [proj_cols][proj_rows] (None = zero)."""
        ptr = None
        if offset is not None:
            self._offset_in = np.ascontiguousarray(offset, np.float32)
            ptr = self._offset_in.ctypes.data
        _check(lib().mbirgpu_session_set_ring_correction(self.h, remove_rings, ptr))

    def update_offset(self) -> None:
        _check(lib().mbirgpu_session_update_offset(self.h))

    def set_variance_estimation(self, on: bool) -> None:
        _check(lib().mbirgpu_session_set_variance_estimation(self.h, 1 if on else 0))

    def update_variance(self) -> float:
        _check(lib().mbirgpu_session_update_variance(self.h))
        return self.variance

    @property
    def variance(self) -> float:
        v = C.c_double()
        _check(lib().mbirgpu_session_get_variance(self.h, C.byref(v)))
        return v.value

    def get_offset(self) -> np.ndarray:
        """The offset d, [proj_cols][proj_rows]."""
        a = np.zeros(self.sino_shape[1:], np.float32)
        _check(lib().mbirgpu_session_get_offset(self.h, a.ctypes.data))
        return a

    def nh_select(self, mag: np.ndarray) -> np.ndarray:
        """NH-ICD voxel-line selection [N_time][N_y][N_x] (uint8) for an
        update-magnitude map [N_time][N_y][N_x]."""
        i = self.info
        m = np.ascontiguousarray(mag, np.float32).reshape(i.N_time, i.N_y, i.N_x)
        out = np.zeros((i.N_time, i.N_y, i.N_x), np.uint8)
        _check(lib().mbirgpu_session_nh_select(self.h, m.ctypes.data, out.ctypes.data))
        return out

    def back_project(self, sino: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(sino, np.float32).reshape(self.sino_shape)
        out = np.zeros(self.shape, np.float32)
        _check(lib().mbirgpu_session_back_project(self.h, a.ctypes.data, out.ctypes.data))
        return out

    def amatrix(self):
        i = self.info
        first = np.zeros((i.N_p, i.N_y, i.N_x), np.int32)
        count = np.zeros((i.N_p, i.N_y, i.N_x), np.int32)
        vals = np.zeros((i.N_p, i.N_y, i.N_x, i.kmax), np.float32)
        _check(lib().mbirgpu_session_get_amatrix(self.h, first.ctypes.data, count.ctypes.data, vals.ctypes.data))
        return first, count, vals

    def detector_response(self) -> np.ndarray:
        out = np.zeros((self.info.N_p, 65), np.float32)
        _check(lib().mbirgpu_session_get_detector_response(self.h, out.ctypes.data))
        return out


def _problem_structs(problems):
    keep = [pb.arrays() for pb in problems]
    arr = (ProblemStruct * len(problems))()
    for i, (pb, a) in enumerate(zip(problems, keep)):
        arr[i] = ProblemStruct(*(x.ctypes.data for x in a), pb.proj_rows, pb.proj_cols, pb.proj_num, pb.recon_num,
                               pb.vox_wid, pb.rot_center, pb.sig_s, pb.sig_t, pb.c_s, pb.c_t, pb.convg_thresh,
                               pb.quad_convex, pb.huber_delta, pb.huber_T)
    return arr, keep


class Batch:
    """Many independent problems resident together, iterated by one persistent
    launch per colour phase captured as a CUDA graph (mbirgpu_batch_*)."""

    def __init__(self, problems, options: Options | None = None, stream: int | None = None):
        self._arr, self._keep = _problem_structs(problems)
        self.problems = list(problems)
        self.h = C.c_void_p()
        opt = options if options is not None else get_options()
        _check(lib().mbirgpu_batch_create(C.byref(self.h), C.cast(self._arr, C.c_void_p), len(problems),
                                          C.byref(opt), C.c_void_p(stream or 0)))

    def close(self):
        if self.h:
            lib().mbirgpu_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, iterations: int) -> BatchStats:
        st = BatchStats()
        _check(lib().mbirgpu_batch_run(self.h, iterations, C.byref(st)))
        return st

    def info(self, i: int):
        inf = SessionInfo()
        it, conv = C.c_int32(), C.c_int32()
        _check(lib().mbirgpu_batch_problem_info(self.h, i, C.byref(inf), C.byref(it), C.byref(conv)))
        return inf, it.value, bool(conv.value)

    def get_object(self, i: int) -> np.ndarray:
        inf, _, _ = self.info(i)
        a = np.zeros((inf.N_time, inf.N_z, inf.N_y, inf.N_x), np.float32)
        _check(lib().mbirgpu_batch_get_object(self.h, i, a.ctypes.data))
        return a

    def cost(self, i: int) -> float:
        c = C.c_double()
        _check(lib().mbirgpu_batch_cost(self.h, i, C.byref(c)))
        return c.value


def reconstruct_batch(problems, iterations: int):
    """mbirgpu_reconstruct_batch: every object in reconstruct()'s layout
    [recon_num][proj_rows+2][proj_cols][proj_cols]."""
    arr, keep = _problem_structs(problems)
    outs = (C.POINTER(C.c_float) * len(problems))()
    _check(lib().mbirgpu_reconstruct_batch(outs, C.cast(arr, C.c_void_p), len(problems), iterations))
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    res = []
    for pb, o in zip(problems, outs):
        n = pb.recon_num * (pb.proj_rows + 2) * pb.proj_cols * pb.proj_cols
        res.append(np.ctypeslib.as_array(o, shape=(n,)).copy().reshape(pb.recon_num, pb.proj_rows + 2, pb.proj_cols,
                                                                        pb.proj_cols))
        libc.free(C.cast(o, C.c_void_p))
    return res
