"""ctypes binding of libmemphys_cuda.so (the C ABI in include/memphys.h).

This is the Python side of the drop-in boundary: every call goes through the
``extern "C"`` entry points, exactly as a cgo / JNI / C++ caller would bind
them.  The library is loaded lazily; if it has not been built this module
raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmemphys_cuda.so")

MP_OK, MP_NOT_CONVERGED, MP_BREAKDOWN, MP_NAN_DETECTED, MP_SINGULAR_STENCIL, MP_BAD_ARG, \
    MP_CUDA_ERROR, MP_NO_DEVICE, MP_TIMEOUT, MP_KNN_FAILED = range(10)
MP_FP64, MP_FP32, MP_MG32 = 0, 1, 2
MP_GRAD_X, MP_GRAD_Y, MP_GRAD_Z, MP_LAPLACIAN = range(4)
MP_ROWS_ALL, MP_ROWS_INTERNAL, MP_ROWS_BOUNDARY = range(3)
MP_PRECOND_NONE, MP_PRECOND_JACOBI, MP_PRECOND_AMG, MP_PRECOND_SOR = range(4)
MP_GUESS_PREVIOUS, MP_GUESS_ZERO, MP_GUESS_LEARNED, MP_GUESS_EXTRAPOLATE, MP_GUESS_PROJECT = range(5)
MP_LOG_FIELDS = 8

STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", 2: "BREAKDOWN", 3: "NAN_DETECTED",
                4: "SINGULAR_STENCIL", 5: "BAD_ARG", 6: "CUDA_ERROR", 7: "NO_DEVICE",
                8: "TIMEOUT", 9: "KNN_FAILED"}

# every entry point declared in include/memphys.h
EXPORTS = [
    "mp_last_error", "mp_version", "mp_device_info", "mp_set_device", "mp_malloc", "mp_free", "mp_malloc_host",
    "mp_free_host", "mp_memcpy", "mp_memset", "mp_stream_create", "mp_stream_destroy",
    "mp_stream_sync", "mp_timer_start", "mp_timer_stop", "mp_profiler", "mp_launch_count", "mp_num_poly_terms",
    "mp_cloud_size", "mp_poly_exponents", "mp_knn_stencils", "mp_knn_stencils_noalloc",
    "mp_interp_matrix", "mp_knn_probe", "mp_order_rcm", "mp_order_morton", "mp_permute_stencils", "mp_permute_rows",
    "mp_sis_create", "mp_sis_system_size", "mp_sis_set_graph", "mp_sis_set_tolerance",
    "mp_sis_single_timestep",
    "mp_sis_destroy", "mp_ist_create", "mp_ist_set_graph", "mp_ist_single_timestep",
    "mp_ist_destroy", "mp_fsf_create", "mp_fsf_set_graph", "mp_fsf_set_layout",
    "mp_fsf_single_timestep",
    "mp_fsf_destroy",
    "mp_stencil_weights",
    "mp_stencil_weights_batched", "mp_stencil_plan_create", "mp_stencil_plan_run",
    "mp_stencil_plan_singular", "mp_stencil_plan_info", "mp_stencil_plan_destroy", "mp_cloud_create", "mp_cloud_create_stencils", "mp_cloud_info",
    "mp_cloud_get", "mp_cloud_destroy", "mp_op_create_ell", "mp_op_from_cloud", "mp_op_apply",
    "mp_op_apply_multi", "mp_op_info", "mp_op_largest_eig", "mp_op_destroy", "mp_solver_cfg_default", "mp_ppe_create",
    "mp_ppe_system_size", "mp_ppe_solve", "mp_ppe_destroy", "mp_fs1_create",
    "mp_fs1_system_size", "mp_fs1_set_state", "mp_fs1_get_state", "mp_fs1_step",
    "mp_fs1_single_timestep", "mp_fs1_last_stats", "mp_fs1_log", "mp_fs1_kernel_counts",
    "mp_fs1_destroy", "mp_mlp_create", "mp_mlp_num_params", "mp_mlp_get_params",
    "mp_mlp_set_params", "mp_mlp_forward", "mp_mlp_gradient", "mp_mlp_train", "mp_mlp_set_spin_limit", "mp_mlp_destroy",
    "mp_fs1_attach_mlp", "mp_fs1_train_mlp", "mp_fs1_set_guess", "mp_fs1_samples",
]


class MemphysError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class SisCfg(C.Structure):
    _fields_ = [("rho", C.c_double), ("mu", C.c_double), ("dt", C.c_double),
                ("n_outer_iter", C.c_int), ("iterative_tolerance", C.c_double),
                ("precond_freq_it", C.c_int)]


class SolverCfg(C.Structure):
    _fields_ = [("tol", C.c_double), ("maxit", C.c_int), ("precond", C.c_int),
                ("precision", C.c_int), ("guess", C.c_int), ("inner_tol", C.c_double),
                ("amg_max_levels", C.c_int), ("amg_coarse_size", C.c_int),
                ("smoother_sweeps", C.c_int), ("cheb_lower", C.c_double),
                ("guess_vectors", C.c_int), ("sor_omega", C.c_double)]


class Fs1Cfg(C.Structure):
    _fields_ = [("rho", C.c_double), ("mu", C.c_double), ("dt", C.c_double),
                ("temporal_order", C.c_int)]


_lib = None


def lib() -> C.CDLL:
    """Load libmemphys_cuda.so; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built: run `python -m memphys_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i, d, sz = C.c_void_p, C.c_int, C.c_double, C.c_size_t
        sig = {
            "mp_last_error": [C.c_char_p, sz], "mp_version": [],
            "mp_device_info": [C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(sz)],
            "mp_set_device": [i], "mp_malloc": [C.POINTER(vp), sz], "mp_free": [vp],
            "mp_malloc_host": [C.POINTER(vp), sz], "mp_free_host": [vp],
            "mp_memcpy": [vp, vp, sz, vp], "mp_memset": [vp, i, sz, vp],
            "mp_stream_create": [C.POINTER(vp)], "mp_stream_destroy": [vp],
            "mp_stream_sync": [vp], "mp_timer_start": [vp, C.POINTER(vp)],
            "mp_timer_stop": [vp, vp, C.POINTER(d)],
            "mp_profiler": [i], "mp_launch_count": [C.POINTER(C.c_int64), i],
            "mp_num_poly_terms": [i, i], "mp_cloud_size": [i, i, d], "mp_poly_exponents": [i, i, vp],
            "mp_knn_stencils": [vp, vp, i, i, i, vp, vp],
            "mp_knn_stencils_noalloc": [vp, vp, i, i, i, vp, vp],
            "mp_interp_matrix": [vp, i, i, vp, i, i, i, i, vp, vp, vp],
            "mp_knn_probe": [vp, i, i, vp, i, i, vp, vp],
            "mp_order_rcm": [vp, i, i, vp], "mp_order_morton": [vp, i, i, vp, vp],
            "mp_permute_stencils": [vp, i, i, vp, vp, vp],
            "mp_permute_rows": [vp, vp, i, i, vp, vp],
            "mp_sis_create": [vp, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(vp)],
            "mp_sis_system_size": [vp, C.POINTER(i)], "mp_sis_set_graph": [vp, i],
            "mp_sis_set_tolerance": [vp, C.c_double],
            "mp_sis_single_timestep": [vp, vp, vp, vp, vp, i, C.POINTER(i), C.POINTER(d),
                                       C.POINTER(d), vp],
            "mp_sis_destroy": [vp],
            "mp_ist_create": [vp, vp, vp, vp, i, d, d, d, vp, C.POINTER(vp)],
            "mp_ist_set_graph": [vp, i],
            "mp_ist_single_timestep": [vp, vp, vp, vp, vp, i, C.POINTER(i), C.POINTER(d), vp],
            "mp_ist_destroy": [vp],
            "mp_fsf_create": [vp, vp, vp, vp, vp, vp, vp, d, i, i, d, d, d, vp, C.POINTER(vp)],
            "mp_fsf_set_graph": [vp, i], "mp_fsf_set_layout": [vp, i],
            "mp_fsf_single_timestep": [vp, vp, vp, vp, vp, i, vp], "mp_fsf_destroy": [vp],
            "mp_stencil_weights": [vp, i, i, vp, i, i, i, vp, vp, vp, vp, vp, vp],
            "mp_stencil_weights_batched": [i, vp, vp, vp, i, i, i, vp, vp, vp],
            "mp_stencil_plan_create": [i, vp, vp, i, i, C.POINTER(vp)],
            "mp_stencil_plan_run": [vp, vp, i, vp, vp, vp],
            "mp_stencil_plan_singular": [vp, C.POINTER(i), vp],
            "mp_stencil_plan_info": [vp, vp, vp], "mp_stencil_plan_destroy": [vp],
            "mp_cloud_create": [vp, vp, i, i, i, i, d, i, vp, C.POINTER(vp)],
            "mp_cloud_create_stencils": [vp, vp, i, i, vp, i, i, i, i, vp, C.POINTER(vp)],
            "mp_cloud_info": [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)],
            "mp_cloud_get": [vp, vp, vp, vp, vp, vp, vp, vp], "mp_cloud_destroy": [vp],
            "mp_op_create_ell": [i, i, i, vp, vp, i, C.POINTER(vp)],
            "mp_op_from_cloud": [vp, i, i, i, C.POINTER(vp)],
            "mp_op_apply": [vp, vp, vp, d, d, vp], "mp_op_apply_multi": [i, vp, vp, vp, vp],
            "mp_op_info": [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i)],
            "mp_op_largest_eig": [vp, i, d, i, C.c_uint64, C.POINTER(d), C.POINTER(d),
                                  C.POINTER(i), vp],
            "mp_op_destroy": [vp], "mp_solver_cfg_default": [C.POINTER(SolverCfg)],
            "mp_ppe_create": [vp, vp, vp, vp, d, d, d, C.POINTER(SolverCfg), C.POINTER(vp)],
            "mp_ppe_system_size": [vp],
            "mp_ppe_solve": [vp, vp, vp, C.POINTER(i), C.POINTER(d), C.POINTER(d), vp],
            "mp_ppe_destroy": [vp],
            "mp_fs1_create": [vp, vp, vp, vp, vp, vp, vp, C.POINTER(Fs1Cfg), C.POINTER(SolverCfg),
                              C.POINTER(vp)],
            "mp_fs1_system_size": [vp], "mp_fs1_set_state": [vp, vp, vp, i, vp],
            "mp_fs1_get_state": [vp, vp, vp, vp], "mp_fs1_step": [vp, i, i, vp],
            "mp_fs1_single_timestep": [vp, vp, vp, vp, vp, i, vp],
            "mp_fs1_last_stats": [vp, C.POINTER(i), C.POINTER(d), C.POINTER(d), C.POINTER(d)],
            "mp_fs1_log": [vp, i, i, vp],
            "mp_fs1_kernel_counts": [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)],
            "mp_fs1_destroy": [vp],
            "mp_mlp_create": [C.c_uint64, C.POINTER(vp)], "mp_mlp_num_params": [],
            "mp_mlp_get_params": [vp, vp], "mp_mlp_set_params": [vp, vp],
            "mp_mlp_forward": [vp, vp, i, vp],
            "mp_mlp_gradient": [vp, vp, vp, i, C.POINTER(d), vp],
            "mp_mlp_train": [vp, vp, vp, i, i, i, d, C.c_uint64, C.POINTER(d)],
            "mp_mlp_set_spin_limit": [vp, C.c_longlong], "mp_mlp_destroy": [vp],
            "mp_fs1_attach_mlp": [vp, vp, i, i, i],
            "mp_fs1_train_mlp": [vp, i, i, d, C.c_uint64, C.POINTER(d)],
            "mp_fs1_set_guess": [vp, i],
            "mp_fs1_samples": [vp, vp, vp, vp, i, C.POINTER(i)],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().mp_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str = "") -> int:
    if rc != MP_OK:
        raise MemphysError(rc, f"{what}: {last_error()}" if what else last_error())
    return rc


def ptr(a) -> C.c_void_p | None:
    """Address of a numpy array, a DeviceArray, or any object with data_ptr() (torch).
    The caller must keep the object referenced until the C call returns."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous, "arrays passed to the C ABI must be C-contiguous"
        return C.c_void_p(a.ctypes.data)
    if isinstance(a, DeviceArray):
        return C.c_void_p(a.ptr)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    if isinstance(a, int):
        return C.c_void_p(a)
    raise TypeError(f"cannot pass {type(a)} to the C ABI")


def device_info():
    sm, ma, mi, mem = C.c_int(), C.c_int(), C.c_int(), C.c_size_t()
    check(lib().mp_device_info(C.byref(sm), C.byref(ma), C.byref(mi), C.byref(mem)),
          "mp_device_info")
    return {"sm_count": sm.value, "cc": (ma.value, mi.value), "total_mem": mem.value}


class DeviceArray:
    """A device buffer allocated through the C ABI (mp_malloc), with a numpy view of
    its shape and dtype for copies."""

    def __init__(self, shape, dtype=np.float64):
        self.shape = tuple(np.atleast_1d(shape)) if not isinstance(shape, tuple) else shape
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        p = C.c_void_p()
        check(lib().mp_malloc(C.byref(p), max(self.nbytes, 1)), "mp_malloc")
        self.ptr = p.value

    @classmethod
    def from_host(cls, a: np.ndarray, stream=None) -> "DeviceArray":
        a = np.ascontiguousarray(a)
        d = cls(a.shape, a.dtype)
        d.upload(a, stream)
        return d

    def upload(self, a: np.ndarray, stream=None):
        a = np.ascontiguousarray(a, self.dtype)
        check(lib().mp_memcpy(C.c_void_p(self.ptr), ptr(a), self.nbytes, stream), "mp_memcpy")
        check(lib().mp_stream_sync(stream), "mp_stream_sync")

    def to_host(self, stream=None) -> np.ndarray:
        out = np.empty(self.shape, self.dtype)
        check(lib().mp_memcpy(ptr(out), C.c_void_p(self.ptr), self.nbytes, stream), "mp_memcpy")
        check(lib().mp_stream_sync(stream), "mp_stream_sync")
        return out

    def zero(self, stream=None):
        check(lib().mp_memset(C.c_void_p(self.ptr), 0, self.nbytes, stream), "mp_memset")

    def free(self):
        if getattr(self, "ptr", None):
            lib().mp_free(C.c_void_p(self.ptr))
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PinnedArray:
    """Page-locked host buffer (mp_malloc_host) exposed as a numpy array."""

    def __init__(self, shape, dtype=np.float64):
        dtype = np.dtype(dtype)
        n = int(np.prod(shape))
        p = C.c_void_p()
        check(lib().mp_malloc_host(C.byref(p), max(n * dtype.itemsize, 1)), "mp_malloc_host")
        self.ptr = p.value
        buf = (C.c_char * (n * dtype.itemsize)).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=dtype, count=n).reshape(shape)

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                self.array = None
                lib().mp_free_host(C.c_void_p(self.ptr))
                self.ptr = None
        except Exception:
            pass


def launch_count(reset: bool = False) -> int:
    c = C.c_int64()
    check(lib().mp_launch_count(C.byref(c), int(reset)), "mp_launch_count")
    return c.value


def solver_cfg(**kw) -> SolverCfg:
    cfg = SolverCfg()
    check(lib().mp_solver_cfg_default(C.byref(cfg)), "mp_solver_cfg_default")
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


class Stream:
    def __init__(self):
        s = C.c_void_p()
        check(lib().mp_stream_create(C.byref(s)), "mp_stream_create")
        self.handle = s

    def sync(self):
        check(lib().mp_stream_sync(self.handle), "mp_stream_sync")

    def __del__(self):
        try:
            lib().mp_stream_destroy(self.handle)
        except Exception:
            pass


class Timer:
    """CUDA-event timing on a stream (events recorded on that stream)."""

    def __init__(self, stream=None):
        self.stream = stream
        self.t = C.c_void_p()

    def __enter__(self):
        check(lib().mp_timer_start(self.stream, C.byref(self.t)), "mp_timer_start")
        return self

    def __exit__(self, *exc):
        ms = C.c_double()
        check(lib().mp_timer_stop(self.t, self.stream, C.byref(ms)), "mp_timer_stop")
        self.ms = ms.value
        return False
