"""ctypes binding of libgvc.so (the C ABI declared in include/gvc.h).

Shared by the two drop-in packages in this directory (bvh_diff_gaussian_rasterization,
gpu_mesh_sampling).  There is no CPU fallback: if libgvc.so is missing or cannot be
loaded, every call raises.
"""
import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgvc.so")

GVC_OK = 0
GVC_ERR_TRAVERSAL = 4
GVC_ERR_TIMEOUT = 7
STATUS_NAMES = {
    0: "GVC_OK", 1: "GVC_ERR_ARG", 2: "GVC_ERR_CUDA", 3: "GVC_ERR_CAPACITY",
    4: "GVC_ERR_TRAVERSAL", 5: "GVC_ERR_UNSUPPORTED", 6: "GVC_ERR_STATE", 7: "GVC_ERR_TIMEOUT",
}
OPT_COV_GRAD, OPT_BWD_MODE, OPT_EVAL_PATH, OPT_COUNT_PAIRS, OPT_TIME_KERNELS, OPT_TRAVERSAL = 1, 2, 3, 4, 5, 6
OPT_CAND_LOG = 7
DTYPE_CODES = {"float64": 0, "float32": 1, "uint16": 2, "uint8": 3}

_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_f32 = ctypes.c_float

# name -> argtypes (restype is int unless listed in _RESTYPES)
_SIGNATURES = {
    "gvc_ctx_create": [ctypes.POINTER(_vp)],
    "gvc_launch_count": [],
    "gvc_ctx_destroy": [_vp],
    "gvc_last_error": [_vp],
    "gvc_set_option": [_vp, _int, _int],
    "gvc_get_stats": [_vp, _vp, _vp],
    "gvc_sync_status": [_vp, _vp],
    "gvc_build_bvh": [_vp, _vp, _i64, _int, _int, _vp],
    "gvc_rasterize_gaussians": [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _f32, _vp, _f32, _int, _int,
                                _vp, _vp, _vp, _vp],
    "gvc_rasterize_gaussians_backward": [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f32, _vp,
                                         _f32, _vp, _vp, _int, _int, _vp, _vp, _vp, _vp, _vp, _vp],
    "gvc_sample_uniform": [_vp, _vp, _vp, _vp, _vp, _int, _i64, _vp, _vp, _vp],
    "gvc_sample_tets": [_vp, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _vp, _vp],
    "gvc_sample_cells": [_vp, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp],
    "gvc_knn3_mean_dist2": [_vp, _i64, _vp, _vp, _vp],
    "gvc_training_samples": [_vp, _i64, _vp, _i64, _vp, _vp, _i64, _i64, ctypes.c_uint64, _vp, _vp, _vp],
    "gvc_debug_lbvh": [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "gvc_debug_lbvh_escape": [_vp, _vp, _vp],
    "gvc_debug_preprocess": [_vp, _i64, _vp, _vp, _vp, _vp, _f32, _vp, _vp, _vp],
    "gvc_debug_sample_order": [_vp, _vp, _vp, _vp],
    "gvc_debug_tc_gemm": [_vp, _vp, _vp, _int, _vp, _vp],
    "gvc_debug_wait_timeout": [_vp, _vp],
    "gvc_sample_tets_static": [_i64, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _i64],
}
_RESTYPES = {"gvc_ctx_destroy": None, "gvc_last_error": ctypes.c_char_p, "gvc_launch_count": ctypes.c_int64}


class GvcStats(ctypes.Structure):
    _fields_ = [("fwd_candidates", ctypes.c_int64), ("fwd_contributing", ctypes.c_int64),
                ("bwd_contributing", ctypes.c_int64), ("max_stack_fwd", ctypes.c_int32),
                ("max_stack_bwd", ctypes.c_int32), ("fwd_kernel_ms", ctypes.c_double),
                ("bwd_kernel_ms", ctypes.c_double), ("fwd_kernel_calls", ctypes.c_int64),
                ("bwd_kernel_calls", ctypes.c_int64), ("fwd_leaf_hits", ctypes.c_int64),
                ("fwd_node_visits", ctypes.c_int64), ("bwd_leaf_hits", ctypes.c_int64),
                ("bwd_node_visits", ctypes.c_int64), ("fwd_lane_evals", ctypes.c_int64),
                ("bwd_rows", ctypes.c_int64)]


_lib = None
_lib_lock = threading.Lock()


def lib():
    """Loads libgvc.so once; raises if it is absent (no fallback path exists)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    "libgvc.so not found at %s: build it with "
                    "`python gaussian-volume-compression_b200/build.py`" % LIB_PATH)
            handle = ctypes.CDLL(LIB_PATH)
            for name, args in _SIGNATURES.items():
                fn = getattr(handle, name)
                fn.argtypes = args
                fn.restype = _RESTYPES.get(name, ctypes.c_int)
            _lib = handle
        return _lib


def launch_count():
    """Kernel launches issued by libgvc.so in this process so far."""
    return int(lib().gvc_launch_count())


def exported_symbols():
    return list(_SIGNATURES)


class GvcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%s)" % (msg, STATUS_NAMES.get(code, code)))
        self.code = code


class Context:
    """Owns one gvc_ctx (created on the current CUDA device)."""

    def __init__(self):
        L = lib()
        p = _vp()
        rc = L.gvc_ctx_create(ctypes.byref(p))
        if rc != GVC_OK:
            raise GvcError(rc, "gvc_ctx_create failed")
        self._p = p
        self._L = L

    @property
    def handle(self):
        return self._p

    def check(self, rc):
        if rc != GVC_OK:
            msg = self._L.gvc_last_error(self._p)
            raise GvcError(rc, msg.decode() if msg else "libgvc error")

    def call(self, name, *args):
        self.check(getattr(self._L, name)(self._p, *args))

    def set_option(self, opt, value):
        self.call("gvc_set_option", int(opt), int(value))

    def sync_status(self, stream):
        self.check(self._L.gvc_sync_status(self._p, _vp(stream)))

    def stats(self, stream):
        s = GvcStats()
        self.check(self._L.gvc_get_stats(self._p, ctypes.byref(s), _vp(stream)))
        return {k: getattr(s, k) for k, _ in GvcStats._fields_}

    def __del__(self):
        try:
            if getattr(self, "_p", None):
                self._L.gvc_ctx_destroy(self._p)
                self._p = None
        except Exception:
            pass


def ptr(t):
    """Device (or host) address of a tensor / numpy array as a c_void_p (None if empty)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return _vp(t.data_ptr()) if t.numel() > 0 else None
    return _vp(t.ctypes.data) if t.size > 0 else None
