"""ctypes wrappers of oracle/_ref/libgvc_ref.so, the reference's own rasterizer kernels
compiled for the host CPU by oracle/build_ref.py.  TEST INFRASTRUCTURE ONLY: the tests
use it to pin the C restatement (gvc_oracle.c) and the GPU kernels against the
reference's own arithmetic; bench.py's reference arm times it.

available() is False when the library was not built (the reference sources were not
present where it was built); callers skip then.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_libs = {}


def path(fma=False):
    return os.path.join(REF_DIR, "libgvc_ref_fma.so" if fma else "libgvc_ref.so")


def available(fma=False):
    return os.path.exists(path(fma))


def reference_root():
    """Where the reference tree is: $GVC_REFERENCE_ROOT, else the root the recipe built
    from (oracle/_ref/REFERENCE_ROOT), if that directory still exists; else None."""
    cands = [os.environ.get("GVC_REFERENCE_ROOT")]
    rec = os.path.join(REF_DIR, "REFERENCE_ROOT")
    if os.path.exists(rec):
        cands.append(open(rec).read().strip())
    for c in cands:
        if c and os.path.isdir(c):
            return c
    return None


def lib(fma=False):
    if fma not in _libs:
        if not available(fma):
            raise FileNotFoundError(path(fma) + " is not built (python oracle/build_ref.py)")
        L = ctypes.CDLL(path(fma))
        vp, i32, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.gvc_ref_openmp.restype = i32
        L.gvc_ref_config.argtypes = [i32, i32]
        L.gvc_ref_preprocess.argtypes = [i32, vp, vp, f32, vp, vp, vp, vp]
        L.gvc_ref_forward.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32]
        L.gvc_ref_backward.argtypes = [i32, i32, vp, vp, f32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                       vp, vp, vp, i32]
        _libs[fma] = L
    return _libs[fma]


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size > 0 else None


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def config(nthreads=0, serial=False, fma=False):
    lib(fma).gvc_ref_config(int(nthreads), int(bool(serial)))


def preprocess(means, scales, rots, weights, scale_modifier=1.0, fma=False):
    """Returns (conics [P,6] f32, aabbs [P,6] f32) as forward.cu:10-114 computes them."""
    means, scales, rots, weights = _f(means), _f(scales), _f(rots), _f(weights).reshape(-1)
    P = means.shape[0]
    conics = np.zeros((P, 6), np.float32)
    aabbs = np.zeros((P, 6), np.float32)
    lib(fma).gvc_ref_preprocess(P, _p(means), _p(scales), scale_modifier, _p(rots), _p(weights), _p(conics),
                                _p(aabbs))
    return conics, aabbs


def forward(means, values, weights, samples, conics, aabbs, fma=False, use_gaussian_bvh=True):
    """Forward: (out [S], outw [S], counts).  use_gaussian_bvh: thread per sample
    (forward.cu:185-259; counts per sample); otherwise warp per Gaussian with atomic sums
    into the samples (forward.cu:116-182, 261-274; counts per Gaussian)."""
    means, values, weights, samples = _f(means), _f(values).reshape(-1), _f(weights).reshape(-1), _f(samples)
    conics, aabbs = _f(conics), _f(aabbs)
    P, S = means.shape[0], samples.shape[0]
    out = np.zeros(S, np.float32)
    outw = np.zeros(S, np.float32)
    cnt = np.zeros(S if use_gaussian_bvh else P, np.int32)
    lib(fma).gvc_ref_forward(P, S, _p(means), _p(values), _p(weights), _p(samples), _p(conics), _p(aabbs),
                             _p(out), _p(outw), _p(cnt), int(bool(use_gaussian_bvh)))
    return out, outw, cnt


def backward(means, scales, rots, conics, values, weights, aabbs, samples, out, outw, gout, gw,
             scale_modifier=1.0, fma=False, use_gaussian_bvh=True):
    """Backward: use_gaussian_bvh: thread per sample with atomic sums into the Gaussians
    (backward.cu:339-559); otherwise warp per Gaussian with warp reductions
    (backward.cu:127-337); then the covariance adjoint (:9-125).  Returns a dict of
    dmeans [P,3], dvalues [P], dweights [P], dscales [P,3], drots [P,4], dconics [P,6]."""
    means, scales, rots, conics = _f(means), _f(scales), _f(rots), _f(conics)
    values, weights, aabbs, samples = _f(values).reshape(-1), _f(weights).reshape(-1), _f(aabbs), _f(samples)
    out, outw, gout, gw = _f(out), _f(outw), _f(gout), _f(gw)
    P, S = means.shape[0], samples.shape[0]
    r = {"dmeans": np.zeros((P, 3), np.float32), "dvalues": np.zeros(P, np.float32),
         "dweights": np.zeros(P, np.float32), "dscales": np.zeros((P, 3), np.float32),
         "drots": np.zeros((P, 4), np.float32), "dconics": np.zeros((P, 6), np.float32)}
    lib(fma).gvc_ref_backward(P, S, _p(means), _p(scales), scale_modifier, _p(rots), _p(conics), _p(values),
                              _p(weights), _p(aabbs), _p(samples), _p(out), _p(outw), _p(gout), _p(gw),
                              _p(r["dmeans"]), _p(r["dvalues"]), _p(r["dweights"]), _p(r["dscales"]),
                              _p(r["drots"]), _p(r["dconics"]), int(bool(use_gaussian_bvh)))
    return r
