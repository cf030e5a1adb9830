"""The allocation-free tetrahedral sampler (gvc_sample_tets_static) against the regular
entry point (gvc_sample_tets), through the C ABI, on two calls in a row.

This entry point exists for callers that cannot allocate device memory when they sample
(their device memory belongs to another allocator, or cudaMalloc's device-wide
synchronisation is unacceptable where they call); its scratch is a static device array
that limits meshes to 32768 cells.  The file is collected last on purpose."""
import ctypes

import numpy as np
import pytest
import torch

import gvc_native

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _regular(pts, tets, vals, q):
    ctx = gvc_native.Context()
    out = torch.empty(q.shape[0], dtype=torch.float64, device="cuda")
    cell = torch.empty(q.shape[0], dtype=torch.int64, device="cuda")
    d = [_dev(pts, np.float32), _dev(tets, np.int32), _dev(vals, np.float64), _dev(q, np.float32)]
    stream = torch.cuda.current_stream().cuda_stream
    ctx.call("gvc_sample_tets", pts.shape[0], gvc_native.ptr(d[0]), tets.shape[0], gvc_native.ptr(d[1]),
             gvc_native.ptr(d[2]), q.shape[0], gvc_native.ptr(d[3]), gvc_native.ptr(out), gvc_native.ptr(cell),
             ctypes.c_void_p(stream))
    ctx.sync_status(stream)
    return out.cpu().numpy(), cell.cpu().numpy()


def _static(pts, tets, vals, q):
    lib = gvc_native.lib()
    out = torch.full((q.shape[0],), 7.0, dtype=torch.float64, device="cuda")
    cell = torch.full((q.shape[0],), 7, dtype=torch.int64, device="cuda")
    d = [_dev(pts, np.float32), _dev(tets, np.int32), _dev(vals, np.float64), _dev(q, np.float32)]
    err = ctypes.create_string_buffer(256)
    rc = lib.gvc_sample_tets_static(pts.shape[0], gvc_native.ptr(d[0]), tets.shape[0], gvc_native.ptr(d[1]),
                                    gvc_native.ptr(d[2]), q.shape[0], gvc_native.ptr(d[3]), gvc_native.ptr(out),
                                    gvc_native.ptr(cell), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                    err, 256)
    return rc, err.value.decode(), out.cpu().numpy(), cell.cpu().numpy()


def test_static_sampler_matches_regular_entry_point(cuda, orc):
    # two different meshes in a row: the shared scratch must not leak between calls
    for n, seed, ns in ((16, 1, 200000), (12, 2, 150000)):
        pts, tets = orc.jittered_tet_mesh(n=n, seed=seed)
        assert tets.shape[0] <= 32768
        vals = orc.blob_field(pts).astype(np.float64)
        q = (np.random.default_rng(seed).random((ns, 3)) * 1.02 - 0.01).astype(np.float32)
        q[:500] = pts[:500]
        rc, msg, out, cell = _static(pts, tets, vals, q)
        assert rc == 0, msg
        ref_out, ref_cell = _regular(pts, tets, vals, q)
        np.testing.assert_array_equal(cell, ref_cell)
        np.testing.assert_array_equal(out, ref_out)
        assert (cell >= 0).mean() > 0.9


def test_static_sampler_rejects_large_meshes(cuda, orc):
    pts, tets = orc.jittered_tet_mesh(n=18, seed=0)   # 34992 tets > 32768
    rc, msg, _, _ = _static(pts, tets, np.zeros(pts.shape[0]), np.zeros((4, 3), np.float32))
    assert rc == 3  # GVC_ERR_CAPACITY
    assert "exceed the static maximum of 32768" in msg
