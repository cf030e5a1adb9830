"""Native ops of bvh_diff_gaussian_rasterization, backed by libgvc.so.

Same three entry points, argument order and return arity as the reference's pybind
module (diff-gaussian-rasterization/ext.cu:150-154):

    build_bvh(samples, debug, use_gaussian_bvh) -> None
    rasterize_gaussians(means3D, scales, rotations, values, weights, scale_modifier,
                        min_x, min_y, min_z, max_x, max_y, max_z, background,
                        use_gaussian_bvh, debug) -> (out_cells[S], out_weights[S], conics[6P])
    rasterize_gaussians_backward(means3D, scales, rotations, conics, values, weights,
                        out_cells, out_weights, scale_modifier, min/max xyz, background,
                        dL_dout_cells, dL_dout_weights, use_gaussian_bvh, debug)
        -> (dL_dmeans3D[P,3], dL_dscales[P,3], dL_drotations[P,4], dL_dvalues[P,1], dL_dweights[P,1])

Like the reference (ext.cu:8-10), the sample set and its BVH are module state: the
last build_bvh call's samples are used by every following forward and backward on the
same device.  The state lives in one libgvc context per CUDA device.
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

_state_lock = threading.Lock()
_contexts = {}   # device index -> gvc_native.Context
_samples = {}    # device index -> contiguous samples tensor (kept alive for the context)


def _device_index(t):
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise RuntimeError("expected a CUDA tensor")
    return t.device.index if t.device.index is not None else torch.cuda.current_device()


def _ctx(dev):
    with _state_lock:
        c = _contexts.get(dev)
        if c is None:
            with torch.cuda.device(dev):
                c = _n.Context()
            _contexts[dev] = c
        return c


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def _f32(t, name, numel=None):
    if not isinstance(t, torch.Tensor):
        raise RuntimeError("%s must be a tensor" % name)
    if t.dtype != torch.float32:
        raise RuntimeError("%s: expected scalar type Float but found %s" % (name, t.dtype))
    if t.device.type != "cuda":
        raise RuntimeError("%s must be a CUDA tensor" % name)
    t = t.contiguous()
    if numel is not None and t.numel() != numel:
        raise RuntimeError("%s has %d elements, expected %d" % (name, t.numel(), numel))
    return t


def build_bvh(samples, debug, use_gaussian_bvh):
    """ext.cu:28-65: stores the samples and builds the spatial index used by the next
    forward and backward."""
    samples = _f32(samples, "samples")
    if samples.dim() != 2 or samples.size(1) != 3:
        raise RuntimeError("samples must have dimensions (num_samples, 3)")
    dev = _device_index(samples)
    c = _ctx(dev)
    with torch.cuda.device(dev):
        c.call("gvc_build_bvh", _n.ptr(samples), int(samples.size(0)), int(bool(debug)),
               int(bool(use_gaussian_bvh)), ctypes.c_void_p(_stream(dev)))
    _samples[dev] = samples


def _stored(dev):
    s = _samples.get(dev)
    if s is None:
        raise RuntimeError("build_bvh must be called before rasterize_gaussians")
    return s


def _bounds(vals):
    return (ctypes.c_float * 6)(*[float(v) for v in vals])


def rasterize_gaussians(means3D, scales, rotations, values, weights, scale_modifier,
                        min_x, min_y, min_z, max_x, max_y, max_z, background,
                        use_gaussian_bvh, debug):
    """ext.cu:67-105 / rasterize_points.cu:17-73."""
    if means3D.dim() != 2 or means3D.size(1) != 3:
        raise RuntimeError("means3D must have dimensions (num_points, 3)")
    P = means3D.size(0)
    means3D = _f32(means3D, "means3D")
    dev = _device_index(means3D)
    samples = _stored(dev)
    S = samples.size(0)
    opts = dict(dtype=torch.float32, device=means3D.device)
    out_cells = torch.zeros(S, **opts)
    out_weights = torch.zeros(S, **opts)
    conics = torch.zeros(P * 6, **opts)
    if P == 0:
        return out_cells, out_weights, conics
    scales = _f32(scales, "scales", 3 * P)
    rotations = _f32(rotations, "rotations", 4 * P)
    values = _f32(values, "values", P)
    weights = _f32(weights, "weights", P)
    c = _ctx(dev)
    with torch.cuda.device(dev):
        c.call("gvc_rasterize_gaussians", P, _n.ptr(means3D), _n.ptr(scales), _n.ptr(rotations),
               _n.ptr(values), _n.ptr(weights), float(scale_modifier),
               _bounds((min_x, min_y, min_z, max_x, max_y, max_z)), float(background),
               int(bool(use_gaussian_bvh)), int(bool(debug)), _n.ptr(out_cells), _n.ptr(out_weights),
               _n.ptr(conics), ctypes.c_void_p(_stream(dev)))
    return out_cells, out_weights, conics


def rasterize_gaussians_backward(means3D, scales, rotations, conics, values, weights, out_cells,
                                 out_weights, scale_modifier, min_x, min_y, min_z, max_x, max_y,
                                 max_z, background, dL_dout_cells, dL_dout_weights,
                                 use_gaussian_bvh, debug):
    """ext.cu:107-147 / rasterize_points.cu:75-137."""
    P = means3D.size(0)
    means3D = _f32(means3D, "means3D", 3 * P)
    dev = _device_index(means3D)
    samples = _stored(dev)
    S = samples.size(0)
    opts = dict(dtype=torch.float32, device=means3D.device)
    dmeans = torch.zeros(P, 3, **opts)
    dscales = torch.zeros(P, 3, **opts)
    drots = torch.zeros(P, 4, **opts)
    dvalues = torch.zeros(P, 1, **opts)
    dweights = torch.zeros(P, 1, **opts)
    if P == 0:
        return dmeans, dscales, drots, dvalues, dweights
    scales = _f32(scales, "scales", 3 * P)
    rotations = _f32(rotations, "rotations", 4 * P)
    conics = _f32(conics, "conics", 6 * P)
    values = _f32(values, "values", P)
    weights = _f32(weights, "weights", P)
    out_cells = _f32(out_cells, "out_cells", S)
    out_weights = _f32(out_weights, "out_weights", S)
    dL_dout_cells = _f32(dL_dout_cells, "dL_dout_cells", S)
    dL_dout_weights = _f32(dL_dout_weights, "dL_dout_weights", S)
    c = _ctx(dev)
    with torch.cuda.device(dev):
        c.call("gvc_rasterize_gaussians_backward", P, _n.ptr(means3D), _n.ptr(scales),
               _n.ptr(rotations), _n.ptr(conics), _n.ptr(values), _n.ptr(weights),
               _n.ptr(out_cells), _n.ptr(out_weights), float(scale_modifier),
               _bounds((min_x, min_y, min_z, max_x, max_y, max_z)), float(background),
               _n.ptr(dL_dout_cells), _n.ptr(dL_dout_weights), int(bool(use_gaussian_bvh)),
               int(bool(debug)), _n.ptr(dmeans), _n.ptr(dscales), _n.ptr(drots), _n.ptr(dvalues),
               _n.ptr(dweights), ctypes.c_void_p(_stream(dev)))
    return dmeans, dscales, drots, dvalues, dweights


# ---- extensions beyond the reference's three ops (options, status, statistics) ----

def set_option(opt, value, device=None):
    dev = torch.cuda.current_device() if device is None else device
    _ctx(dev).set_option(opt, value)


def set_cov_grad_mode(mode, device=None):
    """'true' (default): exact gradient of the forward; 'ref_compat': the reference's
    formula of diff-gaussian-rasterization/cuda_rasterizer/backward.cu:50-124."""
    set_option(_n.OPT_COV_GRAD, {"true": 0, "ref_compat": 1}[mode], device)


def set_backward_mode(mode, device=None):
    """'auto' (follow use_gaussian_bvh; the tensor-core reduction on the tensor-core eval
    path), 'deterministic', 'atomic' (sample-tile traversal) or 'tensor_core'."""
    set_option(_n.OPT_BWD_MODE, {"auto": 0, "deterministic": 1, "atomic": 2, "tensor_core": 3}[mode], device)


def set_eval_path(path, device=None):
    """Forward kernel: 'plain' (default: FP32, CTA per 128 samples), 'tensor_core'
    (tcgen05 BF16 split exponent, same pipeline) or 'plain_tile' (FP32, warp per 32 samples)."""
    set_option(_n.OPT_EVAL_PATH, {"plain": 0, "tensor_core": 1, "plain_tile": 2}[path], device)


def set_traversal(kind, device=None):
    """Gaussian-LBVH traversal of the block-group forwards and the tensor-core backward:
    'stack' (default: warp-cooperative, shared-memory node stack) or 'stackless' (escape
    edges, one subtree per lane below the levels that fit the warp).  Same candidates."""
    set_option(_n.OPT_TRAVERSAL, {"stack": 0, "stackless": 1}[kind], device)


def set_candidate_log(on, device=None):
    """With the tensor-core backward selected, the forward records each block's candidate
    Gaussians and the backward reads them back instead of walking the tree again (on by
    default; off: the backward walks the tree on its own, finer block groups)."""
    set_option(_n.OPT_CAND_LOG, 1 if on else 0, device)


def set_count_pairs(on, device=None):
    set_option(_n.OPT_COUNT_PAIRS, 1 if on else 0, device)


def check_status(device=None):
    """Waits for the current stream and raises if a kernel recorded a failure."""
    dev = torch.cuda.current_device() if device is None else device
    _ctx(dev).sync_status(_stream(dev))


def stats(device=None):
    dev = torch.cuda.current_device() if device is None else device
    return _ctx(dev).stats(_stream(dev))


def context(device=None):
    dev = torch.cuda.current_device() if device is None else device
    return _ctx(dev)


def set_time_kernels(on, device=None):
    """Times the forward / backward evaluation kernels with CUDA events (see stats())."""
    set_option(_n.OPT_TIME_KERNELS, 1 if on else 0, device)
