"""Python side of the oracle -- TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the checker;
never by the product path (the product raises when libgvc.so is missing).

Contents:
  * ctypes wrappers of the C restatement in gvc_oracle.c (see that file's header for
    the parity status: kernel semantics restated from source, Python-side orderings
    pinned by fixtures generated from the reference's own Python code);
  * numpy/torch FP64 restatements of the reference's Python layers:
      - activations: scene/gaussian_model.py:71-77 (_apply_cap), :114-132 (getters);
      - 21-bit Morton order: gaussian_renderer/__init__.py:45-58 and train.py:292-315;
  * an FP64 autograd forward over a frozen pair list (for finite differences);
  * the synthetic workloads of the benchmark configurations (seeded).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "gvc_oracle.c")
LIB = os.path.join(HERE, "libgvc_oracle.so")

_lib = None


def build(force=False):
    """Compiles gvc_oracle.c with OpenMP and without FP contraction."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-o", LIB, SRC, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, i64, i32, f32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_float
        sig = {
            "orc_preprocess": [i64, vp, vp, vp, vp, f32, vp, vp, vp, i32],
            "orc_forward": [i64, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32],
            "orc_pair_counts": [i64, i64, vp, vp, vp, vp, vp, vp, i32],
            "orc_pair_list": [i64, i64, vp, vp, vp, vp, vp, i64, vp, vp],
            "orc_backward": [i64, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32],
            "orc_cov_backward": [i64, vp, vp, vp, f32, vp, i32, vp, vp, i32],
            "orc_centroid_bounds": [i64, vp, vp, vp],
            "orc_morton_keys": [i64, vp, vp, vp, vp],
            "orc_sort_keys": [i64, vp, vp, vp],
            "orc_lbvh_build": [i64, vp, vp, vp, vp, vp, vp],
            "orc_sample_uniform": [vp, vp, vp, vp, i64, vp, vp, vp, i32],
            "orc_sample_tets": [i64, vp, i64, vp, vp, i64, vp, vp, vp, i32],
            "orc_tet_boxes": [i64, vp, vp, vp],
            "orc_sample_cells": [i64, vp, i64, vp, vp, vp, vp, i64, vp, vp, vp, i32],
            "orc_knn3_mean_dist2": [i64, vp, vp, i32],
            "orc_philox4x32_10": [vp, vp, vp],
            "orc_tet_points": [i64, ctypes.c_uint64, vp, vp, i64, vp, i32],
            "orc_openmp_enabled": [],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int64 if name == "orc_pair_list" else (
                ctypes.c_int if name == "orc_openmp_enabled" else None)
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size > 0 else None


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


# --------------------------------------------------------------------------------------
# Rasterizer path
# --------------------------------------------------------------------------------------
def preprocess(means, scales, rots, weights, scale_modifier=1.0, nthreads=0):
    """Returns (conics32 [P,6] as the product writes them, conics64 [P,6], aabbs [P,6])."""
    means, scales, rots, weights = (_c(means, np.float32), _c(scales, np.float32), _c(rots, np.float32),
                                    _c(weights, np.float32).reshape(-1))
    P = means.shape[0]
    c32 = np.zeros((P, 6), np.float32)
    c64 = np.zeros((P, 6), np.float64)
    bb = np.zeros((P, 6), np.float32)
    lib().orc_preprocess(P, _p(means), _p(scales), _p(rots), _p(weights), scale_modifier, _p(c32), _p(c64),
                         _p(bb), nthreads)
    return c32, c64, bb


def forward(means, values, weights, conics, aabbs, samples, nthreads=0, with_counts=False):
    """FP64 forward over the declared candidate set; returns (out, outw[, counts])."""
    means, values, weights = _c(means, np.float32), _c(values, np.float32).reshape(-1), _c(weights, np.float32).reshape(-1)
    conics, aabbs, samples = _c(conics, np.float64), _c(aabbs, np.float32), _c(samples, np.float32)
    P, S = means.shape[0], samples.shape[0]
    out = np.zeros(S, np.float64)
    outw = np.zeros(S, np.float64)
    cnt = np.zeros(S, np.int64) if with_counts else None
    lib().orc_forward(P, S, _p(means), _p(values), _p(weights), _p(conics), _p(aabbs), _p(samples), _p(out),
                      _p(outw), _p(cnt), nthreads)
    return (out, outw, cnt) if with_counts else (out, outw)


def pair_counts(means, conics, aabbs, samples, nthreads=0):
    means, conics, aabbs, samples = _c(means, np.float32), _c(conics, np.float64), _c(aabbs, np.float32), _c(samples, np.float32)
    a, b = ctypes.c_int64(0), ctypes.c_int64(0)
    lib().orc_pair_counts(means.shape[0], samples.shape[0], _p(means), _p(conics), _p(aabbs), _p(samples),
                          ctypes.byref(a), ctypes.byref(b), nthreads)
    return a.value, b.value


def pair_list(means, conics, aabbs, samples, outw=None, cap=None):
    means, conics, aabbs, samples = _c(means, np.float32), _c(conics, np.float64), _c(aabbs, np.float32), _c(samples, np.float32)
    ow = _c(outw, np.float64) if outw is not None else None
    P, S = means.shape[0], samples.shape[0]
    if cap is None:
        n = lib().orc_pair_list(P, S, _p(means), _p(conics), _p(aabbs), _p(samples), _p(ow), 0, None, None)
        cap = n
    ps = np.zeros(max(cap, 1), np.int64)
    pg = np.zeros(max(cap, 1), np.int64)
    n = lib().orc_pair_list(P, S, _p(means), _p(conics), _p(aabbs), _p(samples), _p(ow), cap, _p(ps), _p(pg))
    return ps[:min(n, cap)], pg[:min(n, cap)]


def backward(means, values, weights, conics, aabbs, samples, out_cells, out_weights, gout, gw, nthreads=0):
    """FP64 per-pair adjoint (Gaussian-owned).  Returns dict of dmeans, dvalues, dweights, dconics."""
    means, values, weights = _c(means, np.float32), _c(values, np.float32).reshape(-1), _c(weights, np.float32).reshape(-1)
    conics, aabbs, samples = _c(conics, np.float64), _c(aabbs, np.float32), _c(samples, np.float32)
    out_cells, out_weights = _c(out_cells, np.float32), _c(out_weights, np.float32)
    gout, gw = _c(gout, np.float32), _c(gw, np.float32)
    P, S = means.shape[0], samples.shape[0]
    dm = np.zeros((P, 3)); dv = np.zeros(P); dw = np.zeros(P); dc = np.zeros((P, 6))
    lib().orc_backward(P, S, _p(means), _p(values), _p(weights), _p(conics), _p(aabbs), _p(samples),
                       _p(out_cells), _p(out_weights), _p(gout), _p(gw), _p(dm), _p(dv), _p(dw), _p(dc), nthreads)
    return {"dmeans": dm, "dvalues": dv, "dweights": dw, "dconics": dc}


def cov_backward(scales, rots, conics32, dconics, scale_modifier=1.0, ref_compat=False, nthreads=0):
    scales, rots, conics32, dconics = _c(scales, np.float32), _c(rots, np.float32), _c(conics32, np.float32), _c(dconics, np.float64)
    P = scales.shape[0]
    ds = np.zeros((P, 3)); dq = np.zeros((P, 4))
    lib().orc_cov_backward(P, _p(scales), _p(rots), _p(conics32), scale_modifier, _p(dconics), int(ref_compat),
                           _p(ds), _p(dq), nthreads)
    return ds, dq


# --------------------------------------------------------------------------------------
# LBVH specification
# --------------------------------------------------------------------------------------
def lbvh_build(boxes):
    """boxes [n,6] float32 -> (sorted keys u32, perm i32, left i32, right i32, node_boxes [n-1,6])."""
    boxes = _c(boxes, np.float32)
    n = boxes.shape[0]
    keys = np.zeros(n, np.uint32)
    perm = np.zeros(n, np.int32)
    left = np.zeros(max(n - 1, 1), np.int32)
    right = np.zeros(max(n - 1, 1), np.int32)
    nb = np.zeros((max(n - 1, 1), 6), np.float32)
    lib().orc_lbvh_build(n, _p(boxes), _p(keys), _p(perm), _p(left), _p(right), _p(nb))
    return keys, perm, left[:n - 1], right[:n - 1], nb[:n - 1]


def morton30_points(pts):
    """Declared 30-bit Morton keys of points over their own bounds, and the stable order."""
    pts = _c(pts, np.float32)
    boxes = np.concatenate([pts, pts], axis=1)
    lo = np.zeros(3, np.float32); hi = np.zeros(3, np.float32)
    lib().orc_centroid_bounds(pts.shape[0], _p(boxes), _p(lo), _p(hi))
    keys = np.zeros(pts.shape[0], np.uint32)
    lib().orc_morton_keys(pts.shape[0], _p(boxes), _p(lo), _p(hi), _p(keys))
    skeys = np.zeros_like(keys)
    perm = np.zeros(pts.shape[0], np.int32)
    lib().orc_sort_keys(pts.shape[0], _p(keys), _p(skeys), _p(perm))
    return keys, skeys, perm


# --------------------------------------------------------------------------------------
# Mesh sampler
# --------------------------------------------------------------------------------------
def sample_uniform(dims, origin, spacing, values, samples, nthreads=0):
    """Returns (value as float64, valid mask) per the declared uniform-grid semantics."""
    dims = _c(dims, np.int64).reshape(3)
    origin = _c(origin, np.float32).reshape(3)
    spacing = _c(spacing, np.float32).reshape(3)
    vals = _c(np.asarray(values).reshape(-1), np.float64)
    samples = _c(samples, np.float32).reshape(-1, 3)
    out = np.zeros(samples.shape[0]); valid = np.zeros(samples.shape[0], np.int8)
    lib().orc_sample_uniform(_p(dims), _p(origin), _p(spacing), _p(vals), samples.shape[0], _p(samples),
                             _p(out), _p(valid), nthreads)
    return out, valid.astype(bool)


def cast_sampled(out, valid, dtype):
    """The product's dtype conversion of sampled values (round half up, saturate; -1 wraps)."""
    dtype = np.dtype(dtype)
    if dtype.kind == "f":
        r = out.astype(dtype)
        r[~valid] = -1
        return r
    info = np.iinfo(dtype)
    r = np.clip(np.floor(out + 0.5), 0, info.max).astype(dtype)
    r[~valid] = info.max
    return r


def sample_tets(pts, conn4, values, samples, nthreads=0):
    pts = _c(pts, np.float32).reshape(-1, 3)
    conn4 = _c(conn4, np.int64).reshape(-1, 4)
    values = _c(values, np.float64).reshape(-1)
    samples = _c(samples, np.float32).reshape(-1, 3)
    n = samples.shape[0]
    out = np.zeros(n); cell = np.zeros(n, np.int64)
    lib().orc_sample_tets(pts.shape[0], _p(pts), conn4.shape[0], _p(conn4), _p(values), n, _p(samples), _p(out),
                          _p(cell), nthreads)
    return out, cell


def sample_cells(pts, types, offsets, conn, values, samples, nthreads=0):
    """Mixed explicit cells (VTK 10/12/13/14 located, 1/3/5/9 never contain a point);
    returns (values f64 or -1, lowest containing cell id or -1)."""
    pts = _c(pts, np.float32).reshape(-1, 3)
    types = _c(types, np.uint8).reshape(-1)
    offsets = _c(offsets, np.int64).reshape(-1)
    conn = _c(conn, np.int32).reshape(-1)
    values = _c(values, np.float64).reshape(-1)
    samples = _c(samples, np.float32).reshape(-1, 3)
    n = samples.shape[0]
    out = np.zeros(n); cell = np.zeros(n, np.int64)
    lib().orc_sample_cells(pts.shape[0], _p(pts), types.shape[0], _p(types), _p(offsets), _p(conn), _p(values), n,
                           _p(samples), _p(out), _p(cell), nthreads)
    return out, cell


def knn3_mean_dist2(pts, nthreads=0):
    """Mean squared distance to the three nearest other points, float32 (the initial
    scale rule of scene/gaussian_model.py:175-179, :729-733; simple-knn distCUDA2)."""
    pts = _c(pts, np.float32).reshape(-1, 3)
    out = np.zeros(pts.shape[0], np.float32)
    lib().orc_knn3_mean_dist2(pts.shape[0], _p(pts), _p(out), nthreads)
    return out


def philox4x32_10(ctr, key):
    """Philox4x32-10 of one counter block (four uint32) under a key (two uint32)."""
    c = _c(ctr, np.uint32)
    k = _c(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(_p(c), _p(k), _p(out))
    return out


def training_samples(pts, tets, values, num_batches, batch_size, seed=0, nthreads=0):
    """Training batches of train.py:34-61 + :273-315 with the declared Philox generator:
    points in random tetrahedra, per-batch stable sort by the clamped 21-bit Morton code
    (morton21, pinned to the reference's own code), ground truth by the tetrahedral
    locator at the sorted points, converted to float32.  Returns ([B,S,3], [B,S])."""
    pts = _c(pts, np.float32).reshape(-1, 3)
    tets = _c(tets, np.int64).reshape(-1, 4)
    N = num_batches * batch_size
    raw = np.zeros((N, 3), np.float32)
    lib().orc_tet_points(N, int(seed), _p(pts), _p(tets), tets.shape[0], _p(raw), nthreads)
    keys = morton21(raw, clamp=True).reshape(num_batches, batch_size)
    order = np.argsort(keys, axis=1, kind="stable")
    samples = np.take_along_axis(raw.reshape(num_batches, batch_size, 3), order[:, :, None], axis=1)
    gt = None
    if values is not None:
        v, _ = sample_tets(pts, tets, values, samples.reshape(-1, 3), nthreads)
        gt = v.astype(np.float32).reshape(num_batches, batch_size)
    return samples, gt


# --------------------------------------------------------------------------------------
# Reference Python layers (FP64 restatements)
# --------------------------------------------------------------------------------------
def activations(xyz, log_scales, rot_raw, weight_raw, value_raw, max_scale=0.02, xp=np):
    """scene/gaussian_model.py:71-77 (exp + tanh soft cap) and :114-132 (getters)."""
    if xp is np:
        s = np.exp(log_scales)
        r = np.linalg.norm(s, axis=1, keepdims=True) + 1e-8
        s = s * ((max_scale * np.tanh(r / max_scale)) / r)
        q = rot_raw / np.maximum(np.linalg.norm(rot_raw, axis=1, keepdims=True), 1e-12)
        w = 1.0 / (1.0 + np.exp(-weight_raw))
        v = 1.0 / (1.0 + np.exp(-value_raw))
        return xyz, s, q, w, v
    import torch
    s = torch.exp(log_scales)
    r = torch.linalg.norm(s, dim=1, keepdim=True) + 1e-8
    s = s * ((max_scale * torch.tanh(r / max_scale)) / r)
    q = torch.nn.functional.normalize(rot_raw)
    return xyz, s, q, torch.sigmoid(weight_raw), torch.sigmoid(value_raw)


def _part1by2(n):
    n = n & 0x1fffff
    n = (n | (n << 32)) & 0x1f00000000ffff
    n = (n | (n << 16)) & 0x1f0000ff0000ff
    n = (n | (n << 8)) & 0x100f00f00f00f00f
    n = (n | (n << 4)) & 0x10c30c30c30c30c3
    n = (n | (n << 2)) & 0x1249249249249249
    return n


def morton21(xyz, clamp=False):
    """63-bit Morton codes of gaussian_renderer/__init__.py:45-58 (no clamp, values wrap
    through the 21-bit mask) or train.py:292-315 (clamp to [0,1])."""
    import torch
    t = torch.as_tensor(xyz, dtype=torch.float32)
    if clamp:
        t = torch.clamp(t, 0.0, 1.0)
    q = (t * ((1 << 21) - 1)).to(torch.int64)
    return (_part1by2(q[:, 0]) | (_part1by2(q[:, 1]) << 1) | (_part1by2(q[:, 2]) << 2)).numpy()


def torch_forward_pairs(ps, pg, samples, means, scales, rots, values, weights, scale_modifier=1.0, S=None):
    """FP64 autograd forward over a frozen pair list (AABB and window decisions fixed).
    Inputs are float64 torch tensors (activated parameters); returns (out, outw) for
    samples in `ps` (others: out = -1, outw = 0 are constants)."""
    import torch
    r, x, y, z = rots[:, 0], rots[:, 1], rots[:, 2], rots[:, 3]
    R = torch.stack([
        torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - r * z), 2 * (x * z + r * y)], -1),
        torch.stack([2 * (x * y + r * z), 1 - 2 * (x * x + z * z), 2 * (y * z - r * x)], -1),
        torch.stack([2 * (x * z - r * y), 2 * (y * z + r * x), 1 - 2 * (x * x + y * y)], -1)], -2)
    sv = scale_modifier * scales
    Sigma = R @ torch.diag_embed(sv * sv) @ R.transpose(1, 2)
    d = torch.diagonal(Sigma, dim1=1, dim2=2)
    eps = torch.max(torch.abs(d), dim=1).values * 1e-5
    A = Sigma + eps[:, None, None] * torch.eye(3, dtype=Sigma.dtype)
    C = torch.linalg.inv(A)
    ps_t = torch.as_tensor(ps)
    pg_t = torch.as_tensor(pg)
    dlt = samples[ps_t] - means[pg_t]
    q = torch.einsum("ni,nij,nj->n", dlt, C[pg_t], dlt)
    e = torch.exp(-0.5 * q)
    wt = weights.reshape(-1)[pg_t] * e
    S = int(S if S is not None else samples.shape[0])
    W = torch.zeros(S, dtype=samples.dtype).index_add(0, ps_t, wt)
    V = torch.zeros(S, dtype=samples.dtype).index_add(0, ps_t, wt * values.reshape(-1)[pg_t])
    return W, V


# --------------------------------------------------------------------------------------
# Synthetic workloads: defined in the package (gvc_workloads.py) so that the benchmark's
# GPU leg does not import the oracle; re-exported here for the tests.
# --------------------------------------------------------------------------------------
import sys as _sys

_PKG = os.path.join(os.path.dirname(HERE), "gaussian-volume-compression_b200")
if _PKG not in _sys.path:
    _sys.path.insert(0, _PKG)
from gvc_workloads import (mixture_small, grid_centres, blob_target, mixture_large,  # noqa: E402,F401
                           jittered_tet_mesh, mixed_cell_mesh, blob_field)
