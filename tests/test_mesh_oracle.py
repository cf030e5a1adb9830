"""CPU checks of the mesh-sampling oracle: exactness on linear / trilinear fields, no
gaps between tets, the lowest-id tie-break, the invalid value."""
import numpy as np


def test_uniform_reproduces_trilinear_field(orc):
    rng = np.random.default_rng(0)
    dims = np.array([7, 5, 9])
    origin = np.array([-0.5, 0.25, 0.0], np.float32)
    spacing = np.array([0.25, 0.5, 0.125], np.float32)
    i, j, k = np.meshgrid(np.arange(7), np.arange(5), np.arange(9), indexing="ij")
    X = origin[0] + i * spacing[0]
    Y = origin[1] + j * spacing[1]
    Z = origin[2] + k * spacing[2]
    f = lambda x, y, z: 1.0 + 2 * x - 3 * y + 0.5 * z + 0.25 * x * y * z
    vals = np.transpose(f(X, Y, Z), (2, 1, 0)).reshape(-1)  # x fastest
    hi = origin + (dims - 1) * spacing
    pts = (origin + rng.random((2000, 3)) * (hi - origin)).astype(np.float32)
    pts = np.concatenate([pts, [hi.astype(np.float32), origin, hi + 0.01, origin - 0.01]]).astype(np.float32)
    out, valid = orc.sample_uniform(dims, origin, spacing, vals, pts)
    p = pts.astype(np.float64)
    assert valid[:-2].all() and not valid[-2:].any()
    np.testing.assert_allclose(out[:-2], f(p[:-2, 0], p[:-2, 1], p[:-2, 2]), rtol=1e-12, atol=1e-12)


def test_tets_interpolate_linear_field_without_gaps(orc):
    pts, tets = orc.jittered_tet_mesh(n=6, seed=1)
    a = np.array([0.3, -1.2, 2.0])
    vals = pts.astype(np.float64) @ a + 0.7
    rng = np.random.default_rng(2)
    q = rng.random((5000, 3)).astype(np.float32)
    out, cell = orc.sample_tets(pts, tets, vals, q)
    assert (cell >= 0).all()
    np.testing.assert_allclose(out, q.astype(np.float64) @ a + 0.7, rtol=0, atol=1e-9)
    out2, cell2 = orc.sample_tets(pts, tets, vals, np.array([[1.5, 0.5, 0.5], [-0.1, 0.2, 0.3]], np.float32))
    assert (cell2 == -1).all() and (out2 == -1.0).all()


def test_tets_lowest_id_on_shared_vertex(orc):
    pts, tets = orc.jittered_tet_mesh(n=3, seed=0, jitter=0.0)
    # a grid vertex is shared by many tets: the lowest containing id wins
    v = np.array([[1 / 3, 1 / 3, 1 / 3]], np.float32)
    out, cell = orc.sample_tets(pts, tets, np.arange(pts.shape[0], dtype=np.float64), v)
    owners = [c for c in range(tets.shape[0]) if (np.abs(pts[tets[c]] - v).sum(1) < 1e-7).any()]
    assert cell[0] == min(owners)


def test_tet_grid_search_matches_brute_force(orc):
    pts, tets = orc.jittered_tet_mesh(n=4, seed=3)
    rng = np.random.default_rng(4)
    q = rng.random((300, 3)).astype(np.float32)
    out, cell = orc.sample_tets(pts, tets, np.zeros(pts.shape[0]), q)
    for s in range(q.shape[0]):
        best = -1
        for c in range(tets.shape[0]):
            _, cc = orc.sample_tets(pts, tets[c:c + 1], np.zeros(pts.shape[0]), q[s:s + 1])
            if cc[0] == 0:
                best = c
                break
        assert best == cell[s]


def _unit_cube_points(pts, n, q01):
    """Maps points of [0,1]^3 into the (affinely mapped) grid of mixed_cell_mesh."""
    N1 = n + 1
    g0 = pts[0].astype(np.float64)
    e = np.stack([pts[n], pts[n * N1], pts[n * N1 * N1]]).astype(np.float64) - g0
    return (g0 + q01 @ e).astype(np.float32)


def _linear(pts, a=(0.3, -1.2, 2.0), b=0.7):
    return pts.astype(np.float64) @ np.asarray(a) + b


def test_cells_reproduce_linear_field(orc):
    """Every isoparametric cell reproduces a linear field (partition of unity) and the
    conforming mixed mesh leaves no gaps."""
    rng = np.random.default_rng(5)
    for kinds in ((12,), (13,), (14,), (12, 13, 14), (12, 13, 14, 10)):
        n = 5
        pts, conn, types, offs = orc.mixed_cell_mesh(n=n, seed=len(kinds), kinds=kinds)
        q01 = 0.01 + 0.98 * rng.random((8000, 3))
        q = _unit_cube_points(pts, n, q01) if 10 in kinds else q01.astype(np.float32)
        out, cell = orc.sample_cells(pts, types, offs[:-1], conn, _linear(pts), q)
        assert (cell >= 0).all(), kinds
        assert set(np.unique(types[cell])) <= set(kinds)
        np.testing.assert_allclose(out, _linear(q), rtol=0, atol=1e-9)
        far = np.array([[2.0, 2.0, 2.0], [-1.0, 0.5, 0.5]], np.float32)
        out2, cell2 = orc.sample_cells(pts, types, offs[:-1], conn, _linear(pts), far)
        assert (cell2 == -1).all() and (out2 == -1.0).all()


def test_cells_trilinear_hex_and_lowest_id(orc):
    """A single-hex field that is trilinear in the hex's own parameters comes back exactly
    at mapped points; a vertex shared by several cells resolves to the lowest cell id."""
    pts, conn, types, offs = orc.mixed_cell_mesh(n=3, seed=7, kinds=(12,), jitter=0.0, extras=False)
    f = lambda p: 1.0 + p[:, 0] - 2 * p[:, 1] + 0.5 * p[:, 2] + 3 * p[:, 0] * p[:, 1] * p[:, 2]
    vals = f(pts.astype(np.float64))
    q = (np.random.default_rng(0).random((2000, 3))).astype(np.float32)
    out, cell = orc.sample_cells(pts, types, offs[:-1], conn, vals, q)
    assert (cell >= 0).all()
    np.testing.assert_allclose(out, f(q.astype(np.float64)), rtol=0, atol=1e-9)
    v = np.array([[1 / 3, 1 / 3, 1 / 3]], np.float32)          # grid vertex shared by 8 hexes
    _, c = orc.sample_cells(pts, types, offs[:-1], conn, vals, v)
    owners = [k for k in range(types.size)
              if (np.abs(pts[conn[offs[k]:offs[k + 1]]] - v).sum(1) < 1e-7).any()]
    assert c[0] == min(owners)


def test_cells_zero_volume_types_and_tet_agreement(orc):
    """VTK vertex/line/triangle/quad cells never contain a point; an all-tet mesh gives the
    tetrahedral sampler's answer bit for bit."""
    pts, tets = orc.jittered_tet_mesh(n=4, seed=3)
    vals = orc.blob_field(pts).astype(np.float64)
    q = np.random.default_rng(1).random((3000, 3)).astype(np.float32)
    C = tets.shape[0]
    ref, rcell = orc.sample_tets(pts, tets, vals, q)
    out, cell = orc.sample_cells(pts, np.full(C, 10), np.arange(C) * 4, tets.reshape(-1), vals, q)
    np.testing.assert_array_equal(cell, rcell)
    np.testing.assert_array_equal(out, ref)
    conn = np.array([0, 1, 2, 0, 1, 5, 7, 9, 11], np.int32)
    types = np.array([1, 3, 5], np.uint8)
    out, cell = orc.sample_cells(pts, types, np.array([0, 1, 3]), conn, vals, pts[:50])
    assert (cell == -1).all() and (out == -1.0).all()


def face_points(n=2):
    """Points exactly on faces shared by two or more tetrahedra of an unjittered n^3 Kuhn
    grid: on the grid planes between hexahedra and on the diagonal planes inside each
    hexahedron (dyadic coordinates, so every orientation test is exact)."""
    h = 1.0 / n
    pts = []
    for a in range(1, n):
        for y in (0.25, 0.375, 0.625):
            for z in (0.125, 0.3125, 0.875):
                pts.append([a * h, y, z])
                pts.append([y, a * h, z])
                pts.append([z, y, a * h])
    for v in (0.125, 0.25, 0.375):
        pts.append([v, v, 0.0625])       # on x = y inside the first hexahedron
        pts.append([v, 0.03125, v])      # on x = z
        pts.append([0.03125, v, v])      # on y = z
    return np.array(pts, np.float32)


def test_tets_lowest_id_on_shared_face(orc):
    pts, tets = orc.jittered_tet_mesh(n=2, seed=0, jitter=0.0)
    vals = np.arange(pts.shape[0], dtype=np.float64)
    q = face_points(2)
    out, cell = orc.sample_tets(pts, tets, vals, q)
    for i in range(q.shape[0]):
        owners = [c for c in range(tets.shape[0])
                  if orc.sample_tets(pts, tets[c:c + 1], vals, q[i:i + 1])[1][0] == 0]
        assert len(owners) >= 2, (i, q[i], owners)   # the point is on a shared face
        assert cell[i] == min(owners)
