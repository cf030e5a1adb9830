"""distCUDA2 backed by libgvc.so (gvc_knn3_mean_dist2).

The reference's training code calls `distCUDA2(points)` (scene/gaussian_model.py:16,
:175-179 to initialise scales, :729-733 when densifying) with a [P, 3] float32 CUDA
tensor and uses the returned [P] float32 tensor: per point, the mean of the squared
distances to its three nearest other points.  The result is exact (not an
approximation): the three smallest float32 squared distances, summed in ascending order
and divided by 3; with fewer than four points the missing neighbours count as FLT_MAX.
"""
import ctypes
import importlib.util
import os
import sys
import threading

import torch


def _load_native():
    mod = sys.modules.get("gvc_native")
    if mod is None:
        path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gvc_native.py")
        spec = importlib.util.spec_from_file_location("gvc_native", path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules["gvc_native"] = mod
        spec.loader.exec_module(mod)
    return mod


_n = _load_native()
_lock = threading.Lock()
_contexts = {}


def _ctx(dev):
    with _lock:
        c = _contexts.get(dev)
        if c is None:
            with torch.cuda.device(dev):
                c = _n.Context()
            _contexts[dev] = c
        return c


def distCUDA2(points):
    """[P, 3] float32 CUDA tensor -> [P] float32 mean squared 3-NN distance (same device)."""
    if not isinstance(points, torch.Tensor):
        raise RuntimeError("points must be a tensor")
    if points.device.type != "cuda":
        raise RuntimeError("points must be a CUDA tensor")
    if points.dtype != torch.float32:
        raise RuntimeError("points: expected scalar type Float but found %s" % points.dtype)
    if points.dim() != 2 or points.shape[1] != 3:
        raise RuntimeError("points must have shape [P, 3], got %s" % (tuple(points.shape),))
    pts = points.contiguous()
    dev = pts.device.index if pts.device.index is not None else torch.cuda.current_device()
    out = torch.empty(pts.shape[0], dtype=torch.float32, device=pts.device)
    if pts.shape[0] == 0:
        return out
    with torch.cuda.device(dev):
        c = _ctx(dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        c.call("gvc_knn3_mean_dist2", int(pts.shape[0]), _n.ptr(pts), _n.ptr(out), ctypes.c_void_p(st))
    return out
