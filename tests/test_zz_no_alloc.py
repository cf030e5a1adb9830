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


def _static_call(d, out, cell, npts, C, N):
    """One call of the entry point on device buffers that already exist."""
    lib = gvc_native.lib()
    err = ctypes.create_string_buffer(256)
    rc = lib.gvc_sample_tets_static(npts, gvc_native.ptr(d[0]), C, gvc_native.ptr(d[1]), gvc_native.ptr(d[2]), N,
                                    gvc_native.ptr(d[3]), gvc_native.ptr(out), gvc_native.ptr(cell),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), err, 256)
    return rc, err.value.decode()


def _static(pts, tets, vals, q):
    out = torch.full((q.shape[0],), 7.0, dtype=torch.float64, device="cuda")
    cell = torch.full((q.shape[0],), 7, dtype=torch.int64, device="cuda")
    d = [_dev(pts, np.float32), _dev(tets, np.int32), _dev(vals, np.float64), _dev(q, np.float32)]
    rc, msg = _static_call(d, out, cell, pts.shape[0], tets.shape[0], q.shape[0])
    return rc, msg, out.cpu().numpy(), cell.cpu().numpy()


def test_static_sampler_matches_regular_entry_point(cuda, orc):
    # set-up only (N = 0): resolves the scratch array on this device
    z = torch.zeros(1, device="cuda")
    rc, msg = _static_call([z, z, z, z], z, z, 0, 0, 0)
    assert rc == 0, msg
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


@pytest.mark.parametrize("C", [32767, 32768])
def test_static_sampler_at_the_cell_limit(cuda, orc, C):
    # the first C tetrahedra of an 18^3 mesh (34992 tets): the layout is tightest here
    pts, tets = orc.jittered_tet_mesh(n=18, seed=3)
    tets = np.ascontiguousarray(tets[:C])
    vals = orc.blob_field(pts).astype(np.float64)
    q = (np.random.default_rng(C).random((120000, 3)) * 1.02 - 0.01).astype(np.float32)
    rc, msg, out, cell = _static(pts, tets, vals, q)
    assert rc == 0, msg
    ref_out, ref_cell = _regular(pts, tets, vals, q)
    np.testing.assert_array_equal(cell, ref_cell)
    np.testing.assert_array_equal(out, ref_out)
    assert (cell >= 0).mean() > 0.8


def test_static_sampler_allocates_nothing(cuda, orc):
    pts, tets = orc.jittered_tet_mesh(n=16, seed=4)
    vals = orc.blob_field(pts).astype(np.float64)
    q = (np.random.default_rng(4).random((100000, 3))).astype(np.float32)
    d = [_dev(pts, np.float32), _dev(tets, np.int32), _dev(vals, np.float64), _dev(q, np.float32)]
    out = torch.empty(q.shape[0], dtype=torch.float64, device="cuda")
    cell = torch.empty(q.shape[0], dtype=torch.int64, device="cuda")
    args = (d, out, cell, pts.shape[0], tets.shape[0], q.shape[0])
    assert _static_call(*args)[0] == 0  # warm-up: set-up and every kernel loaded
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        rc, msg = _static_call(*args)
        assert rc == 0, msg
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_static_sampler_rejects_large_meshes(cuda, orc):
    pts, tets = orc.jittered_tet_mesh(n=18, seed=0)   # 34992 tets > 32768
    rc, msg, _, _ = _static(pts, tets, np.zeros(pts.shape[0]), np.zeros((4, 3), np.float32))
    assert rc == 3  # GVC_ERR_CAPACITY
    assert "exceed the static maximum of 32768" in msg
    rc, msg, _, _ = _static(pts, tets[:32769], np.zeros(pts.shape[0]), np.zeros((4, 3), np.float32))
    assert rc == 3 and "32769 cells" in msg
