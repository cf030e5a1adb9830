"""sample_mesh / sample_meshu with the argument conversions, checks and errors of the
reference's pybind functions (gpu_sampling/sample_mesh.cu:26-240 and :242-414), running
the locate + interpolate kernels of libgvc.so."""
import ctypes
import importlib.util
import os
import sys
import threading

import numpy as np
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

VTK_TETRA = 10
# VTK cell types the reference maps to Viskores shapes (sample_mesh.cu:300-336)
VTK_KNOWN = {1, 3, 5, 9, 10, 12, 13, 14}


def _ctx():
    dev = torch.cuda.current_device()
    with _lock:
        c = _contexts.get(dev)
        if c is None:
            c = _n.Context()
            _contexts[dev] = c
        return dev, c


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _dev(a, dtype):
    dev = torch.cuda.current_device()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).to(device="cuda:%d" % dev)


def sample_mesh(dims_arr, origin_arr, spacing_arr, val_arr, samp_arr):
    """Uniform point field (x fastest) sampled by trilinear interpolation; outside -> -1
    in the values' dtype.  Output dtype follows the values (sample_mesh.cu:76-115)."""
    dims = np.ascontiguousarray(dims_arr, dtype=np.int64).reshape(-1)
    origin = np.ascontiguousarray(origin_arr, dtype=np.float32).reshape(-1)
    spacing = np.ascontiguousarray(spacing_arr, dtype=np.float32).reshape(-1)
    vals = np.ascontiguousarray(val_arr)
    if dims.size < 3 or origin.size < 3 or spacing.size < 3:
        raise RuntimeError("dims, origin and spacing need three entries")
    total = int(dims[0]) * int(dims[1]) * int(dims[2])
    if vals.size != total:
        raise RuntimeError("Values array size does not match dims.")
    code = _n.DTYPE_CODES.get(vals.dtype.name) if vals.dtype.byteorder in "=|" else None
    if code is None:
        raise RuntimeError("Unsupported values dtype. Expected float64, float32, uint16, or uint8.")
    samples = np.ascontiguousarray(samp_arr, dtype=np.float32)
    n = samples.shape[0] if samples.ndim > 0 else 0
    samples = samples.reshape(n, 3) if n else samples.reshape(0, 3)
    out = np.empty(n, dtype=vals.dtype)
    if n == 0:
        return out
    dev, c = _ctx()
    d_vals = torch.from_numpy(vals.reshape(-1).view(np.uint8)).to("cuda:%d" % dev)
    d_samp = _dev(samples, np.float32)
    d_out = torch.empty(n * vals.dtype.itemsize, dtype=torch.uint8, device="cuda:%d" % dev)
    # host arrays must stay referenced until the call returns
    h_dims, h_origin, h_spacing = dims[:3].copy(), origin[:3].copy(), spacing[:3].copy()
    c.call("gvc_sample_uniform", _n.ptr(h_dims), _n.ptr(h_origin), _n.ptr(h_spacing), _n.ptr(d_vals), code, n,
           _n.ptr(d_samp), _n.ptr(d_out), _stream(dev))
    out[:] = d_out.cpu().numpy().view(vals.dtype)
    return out


# points per cell for each VTK type the reference maps (sample_mesh.cu:300-336)
VTK_NPTS = {1: 1, 3: 2, 5: 3, 9: 4, 10: 4, 12: 8, 13: 6, 14: 5}


def _check_cells(conn, cell_types, cell_offsets):
    """Validates the cells as sample_mesh.cu:300-336 does; returns (conn int32, types uint8,
    offsets int64).  A cell's point count is the distance to the next offset (the last cell
    ends at the connectivity size) and must equal its type's node count."""
    conn = np.ascontiguousarray(conn, dtype=np.int64).reshape(-1)
    types = np.ascontiguousarray(cell_types, dtype=np.int64).reshape(-1)
    offs = np.ascontiguousarray(cell_offsets, dtype=np.int64).reshape(-1)
    C = types.size
    if C == 0:
        return conn.astype(np.int32), types.astype(np.uint8), offs[:0].copy()
    if offs.size < C:
        raise RuntimeError("cell_offsets has fewer entries than cell_types")
    unknown = types[~np.isin(types, list(VTK_KNOWN))]
    if unknown.size:
        raise RuntimeError("Unsupported VTK cell type: " + str(int(unknown[0])))
    start = offs[:C]
    end = np.empty(C, dtype=np.int64)
    end[:-1] = offs[1:C]
    end[-1] = conn.size
    want = np.vectorize(VTK_NPTS.get, otypes=[np.int64])(types)
    if np.any(end - start != want) or np.any(start < 0) or np.any(end > conn.size):
        raise RuntimeError("cell point count does not match its VTK cell type")
    return conn.astype(np.int32), types.astype(np.uint8), start.copy()


def _tets_from_cells(conn, types, offs):
    """[C,4] int32 vertex ids of an all-tetrahedra mesh (already validated)."""
    idx = offs[:, None] + np.arange(4, dtype=np.int64)[None, :]
    return conn[idx].astype(np.int32)


def sample_meshu_cells(pts_arr, conn4, val_arr, samp_arr):
    """Samples a tetrahedral mesh given as [C,4] vertex ids; returns (values f64, cell ids)."""
    pts = np.ascontiguousarray(pts_arr, dtype=np.float32).reshape(-1, 3)
    vals = np.ascontiguousarray(val_arr, dtype=np.float64).reshape(-1)
    samples = np.ascontiguousarray(samp_arr, dtype=np.float32).reshape(-1, 3)
    conn4 = np.ascontiguousarray(conn4, dtype=np.int32).reshape(-1, 4)
    n, C = samples.shape[0], conn4.shape[0]
    out = np.full(n, -1.0, dtype=np.float64)
    cells = np.full(n, -1, dtype=np.int64)
    if n == 0:
        return out, cells
    if C and (conn4.min() < 0 or conn4.max() >= pts.shape[0]):
        raise RuntimeError("connectivity refers to a point outside the point array")
    if vals.size < pts.shape[0]:
        raise RuntimeError("values must hold one entry per point")
    dev, c = _ctx()
    d_pts = _dev(pts, np.float32)
    d_conn = _dev(conn4, np.int32)
    d_vals = _dev(vals, np.float64)
    d_samp = _dev(samples, np.float32)
    d_out = torch.empty(n, dtype=torch.float64, device="cuda:%d" % dev)
    d_cell = torch.empty(n, dtype=torch.int64, device="cuda:%d" % dev)
    c.call("gvc_sample_tets", pts.shape[0], _n.ptr(d_pts), C, _n.ptr(d_conn), _n.ptr(d_vals), n,
           _n.ptr(d_samp), _n.ptr(d_out), _n.ptr(d_cell), _stream(dev))
    c.sync_status(torch.cuda.current_stream(dev).cuda_stream)
    return d_out.cpu().numpy(), d_cell.cpu().numpy()


def sample_meshu_mixed(pts_arr, conn_arr, cell_types_arr, cell_offsets_arr, val_arr, samp_arr):
    """Samples an explicit mesh of mixed VTK cells; returns (values f64, lowest containing
    cell id or -1)."""
    conn, types, offs = _check_cells(conn_arr, cell_types_arr, cell_offsets_arr)
    pts = np.ascontiguousarray(pts_arr, dtype=np.float32).reshape(-1, 3)
    vals = np.ascontiguousarray(val_arr, dtype=np.float64).reshape(-1)
    samples = np.ascontiguousarray(samp_arr, dtype=np.float32).reshape(-1, 3)
    n, C = samples.shape[0], types.size
    out = np.full(n, -1.0, dtype=np.float64)
    cells = np.full(n, -1, dtype=np.int64)
    if n == 0:
        return out, cells
    if conn.size and (conn.min() < 0 or conn.max() >= pts.shape[0]):
        raise RuntimeError("connectivity refers to a point outside the point array")
    if vals.size < pts.shape[0]:
        raise RuntimeError("values must hold one entry per point")
    dev, c = _ctx()
    d_pts = _dev(pts, np.float32)
    d_conn = _dev(conn if conn.size else np.zeros(1, np.int32), np.int32)
    d_types = _dev(types if C else np.zeros(1, np.uint8), np.uint8)
    d_offs = _dev(offs if C else np.zeros(1, np.int64), np.int64)
    d_vals = _dev(vals if vals.size else np.zeros(1), np.float64)
    d_samp = _dev(samples, np.float32)
    d_out = torch.empty(n, dtype=torch.float64, device="cuda:%d" % dev)
    d_cell = torch.empty(n, dtype=torch.int64, device="cuda:%d" % dev)
    c.call("gvc_sample_cells", pts.shape[0], _n.ptr(d_pts), C, _n.ptr(d_types), _n.ptr(d_offs), _n.ptr(d_conn),
           _n.ptr(d_vals), n, _n.ptr(d_samp), _n.ptr(d_out), _n.ptr(d_cell), _stream(dev))
    c.sync_status(torch.cuda.current_stream(dev).cuda_stream)
    return d_out.cpu().numpy(), d_cell.cpu().numpy()


def sample_meshu(pts_arr, conn_arr, cell_types_arr, cell_offsets_arr, val_arr, samp_arr):
    """Explicit mesh point field sampled at points; outside every cell -> -1 (float64).
    All-tetrahedra meshes take the tetrahedral kernel; mixed meshes the general one."""
    conn, types, offs = _check_cells(conn_arr, cell_types_arr, cell_offsets_arr)
    if types.size and np.all(types == VTK_TETRA):
        out, _ = sample_meshu_cells(pts_arr, _tets_from_cells(conn, types, offs), val_arr, samp_arr)
        return out
    out, _ = sample_meshu_mixed(pts_arr, conn_arr, cell_types_arr, cell_offsets_arr, val_arr, samp_arr)
    return out


def sample_training_batches(pts_arr, tets_arr, val_arr, num_batches, batch_size, seed=0, gt_cells=None):
    """Training batches built on the device (train.py:34-61 sample_mesh_points, :273-282
    ground truth through gpu_sampleu, :286-315 per-batch Morton sort).

    pts [Np,3] and val [Np] are the mesh's points and point field; tets [C,4] the vertex
    ids of its tetrahedra (the reference's `mesh.triangulate()`).  Points are drawn
    uniformly over cells and inside each by sorted-uniform barycentric weights (Philox
    keyed by `seed`), sorted per batch by their clamped 21-bit Morton code, and sampled for
    the ground truth.  gt_cells = (conn, cell_types, cell_offsets) takes the ground truth
    from that (untriangulated) cell mesh instead, as the reference does when it samples
    the original mesh.  Returns CUDA tensors (samples [B,S,3] float32, gt [B,S] float32);
    nothing goes through host memory after the mesh upload.  The call's workspace (about
    48 bytes per sample) belongs to a context of its own, released before returning.
    """
    pts = np.ascontiguousarray(pts_arr, dtype=np.float32).reshape(-1, 3)
    tets = np.ascontiguousarray(tets_arr, dtype=np.int64).reshape(-1, 4)
    vals = np.ascontiguousarray(val_arr, dtype=np.float64).reshape(-1)
    B, S = int(num_batches), int(batch_size)
    if B < 0 or S < 0:
        raise RuntimeError("num_batches and batch_size must be non-negative")
    if tets.shape[0] == 0 or pts.shape[0] == 0:
        raise RuntimeError("the mesh has no cells or no points")
    if tets.min() < 0 or tets.max() >= pts.shape[0]:
        raise RuntimeError("connectivity refers to a point outside the point array")
    if vals.size < pts.shape[0]:
        raise RuntimeError("values must hold one entry per point")
    dev = torch.cuda.current_device()
    c = _n.Context()   # one-off workspace, freed with the context at the end of the call
    d = "cuda:%d" % dev
    samples = torch.empty((B, S, 3), dtype=torch.float32, device=d)
    gt = torch.empty((B, S), dtype=torch.float32, device=d)
    if B * S == 0:
        return samples, gt
    d_pts = _dev(pts, np.float32)
    d_tets = _dev(tets, np.int32)
    d_vals = _dev(vals, np.float64)
    c.call("gvc_training_samples", pts.shape[0], _n.ptr(d_pts), tets.shape[0], _n.ptr(d_tets), _n.ptr(d_vals),
           B, S, ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), _n.ptr(samples),
           None if gt_cells is not None else _n.ptr(gt), _stream(dev))
    if gt_cells is not None:
        conn, types, offs = _check_cells(*gt_cells)
        if conn.size and (conn.min() < 0 or conn.max() >= pts.shape[0]):
            raise RuntimeError("connectivity refers to a point outside the point array")
        C = types.size
        d_conn = _dev(conn if conn.size else np.zeros(1, np.int32), np.int32)
        d_types = _dev(types if C else np.zeros(1, np.uint8), np.uint8)
        d_offs = _dev(offs if C else np.zeros(1, np.int64), np.int64)
        g64 = torch.empty(B * S, dtype=torch.float64, device=d)
        c.call("gvc_sample_cells", pts.shape[0], _n.ptr(d_pts), C, _n.ptr(d_types), _n.ptr(d_offs), _n.ptr(d_conn),
               _n.ptr(d_vals), B * S, _n.ptr(samples), _n.ptr(g64), None, _stream(dev))
        gt.copy_(g64.view(B, S))
    c.sync_status(torch.cuda.current_stream(dev).cuda_stream)
    return samples, gt
