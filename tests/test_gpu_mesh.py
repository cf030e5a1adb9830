"""GPU parity of the mesh samplers against the oracle: bit-exact values (every dtype) for
the uniform grid; bit-exact cell ids and values for tetrahedra."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.uint16, np.uint8])
def test_uniform_bit_exact(cuda, orc, dtype):
    from gpu_mesh_sampling import gpu_sample
    rng = np.random.default_rng(0)
    dims = np.array([33, 17, 25])
    origin = np.array([-0.5, 0.0, 0.25], np.float32)
    spacing = np.array([1 / 32, 1 / 16, 1 / 24], np.float32)
    if np.dtype(dtype).kind == "f":
        vals = rng.normal(size=dims.prod()).astype(dtype)
    else:
        vals = rng.integers(0, np.iinfo(dtype).max, dims.prod()).astype(dtype)
    hi = origin + (dims - 1) * spacing
    pts = (origin - 0.05 + rng.random((100000, 3)) * (hi - origin + 0.1)).astype(np.float32)
    pts[:10] = origin
    pts[10:20] = hi
    out = gpu_sample(dims, origin, spacing, vals, pts)
    assert out.dtype == dtype
    ref, valid = orc.sample_uniform(dims, origin, spacing, vals, pts)
    np.testing.assert_array_equal(out, orc.cast_sampled(ref, valid, dtype))
    assert valid.mean() > 0.5 and not valid.all()


@pytest.mark.parametrize("n,ns", [(12, 100000), (48, 1000000), (128, 1000000)])
def test_tets_bit_exact(cuda, orc, n, ns):
    from gpu_mesh_sampling._gpu_mesh_sampling import sample_meshu_cells
    pts, tets = orc.jittered_tet_mesh(n=n, seed=n)
    vals = orc.blob_field(pts).astype(np.float64)
    rng = np.random.default_rng(n)
    q = (rng.random((ns, 3)) * 1.02 - 0.01).astype(np.float32)
    q[:1000] = pts[rng.integers(0, pts.shape[0], 1000)]          # exactly on vertices (shared by many tets)
    a, b = tets[rng.integers(0, tets.shape[0], 1000), :2].T
    q[1000:2000] = ((pts[a].astype(np.float64) + pts[b]) * 0.5).astype(np.float32)  # on edges
    out, cell = sample_meshu_cells(pts, tets, vals, q)
    ref, rcell = orc.sample_tets(pts, tets, vals, q)
    np.testing.assert_array_equal(cell, rcell)
    np.testing.assert_array_equal(out, ref)
    assert (cell >= 0).mean() > 0.9


def test_sampleu_vtk_arrays(cuda, orc):
    from gpu_mesh_sampling import gpu_sampleu
    pts, tets = orc.jittered_tet_mesh(n=8, seed=2)
    vals = orc.blob_field(pts).astype(np.float64)
    C = tets.shape[0]
    conn = tets.reshape(-1).astype(np.int64)
    types = np.full(C, 10, np.int64)
    offsets = np.arange(C + 1, dtype=np.int64) * 4   # VTK offsets with the trailing entry
    q = np.random.default_rng(3).random((20000, 3)).astype(np.float32)
    out = gpu_sampleu(pts, conn, types, offsets, vals, q)
    ref, _ = orc.sample_tets(pts, tets, vals, q)
    assert out.dtype == np.float64
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("kinds,n,ns", [((12,), 6, 50000), ((13,), 6, 50000), ((14,), 6, 50000),
                                        ((12, 13, 14), 16, 400000), ((12, 13, 14, 10), 12, 200000)])
def test_mixed_cells_bit_exact(cuda, orc, kinds, n, ns):
    from gpu_mesh_sampling._gpu_mesh_sampling import sample_meshu_mixed
    pts, conn, types, offs = orc.mixed_cell_mesh(n=n, seed=n, kinds=kinds)
    vals = orc.blob_field(pts).astype(np.float64)
    rng = np.random.default_rng(n)
    lo, hi = pts.min(0), pts.max(0)
    q = (lo - 0.01 + rng.random((ns, 3)) * (hi - lo + 0.02)).astype(np.float32)
    q[:1000] = pts[conn[rng.integers(0, conn.size, 1000)]]       # on vertices shared by several cells
    out, cell = sample_meshu_mixed(pts, conn, types, offs, vals, q)
    ref, rcell = orc.sample_cells(pts, types, offs[:-1], conn, vals, q)
    np.testing.assert_array_equal(cell, rcell)
    np.testing.assert_array_equal(out, ref)
    # the affinely mapped grid (with tetrahedra) fills about half of its bounding box
    assert (cell >= 0).mean() > (0.3 if 10 in kinds else 0.5)


def test_sampleu_mixed_vtk_arrays(cuda, orc):
    from gpu_mesh_sampling import gpu_sampleu
    pts, conn, types, offs = orc.mixed_cell_mesh(n=8, seed=4, kinds=(12, 13, 14))
    vals = orc.blob_field(pts).astype(np.float64)
    q = np.random.default_rng(3).random((20000, 3)).astype(np.float32)
    out = gpu_sampleu(pts, conn, types, offs, vals, q)
    ref, _ = orc.sample_cells(pts, types, offs[:-1], conn, vals, q)
    assert out.dtype == np.float64
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("n", [2, 4])
def test_tets_shared_faces_bit_exact(cuda, orc, n):
    """Points exactly on faces shared by several tetrahedra: the lowest containing cell
    wins on the GPU as in the oracle."""
    from gpu_mesh_sampling._gpu_mesh_sampling import sample_meshu_cells
    from test_mesh_oracle import face_points
    pts, tets = orc.jittered_tet_mesh(n=n, seed=0, jitter=0.0)
    vals = orc.blob_field(pts).astype(np.float64)
    q = face_points(n)
    out, cell = sample_meshu_cells(pts, tets, vals, q)
    ref, rcell = orc.sample_tets(pts, tets, vals, q)
    np.testing.assert_array_equal(cell, rcell)
    np.testing.assert_array_equal(out, ref)
    assert (cell >= 0).all()
