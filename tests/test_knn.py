"""Three-nearest-neighbour mean squared distance (distCUDA2 drop-in).

The reference's training code initialises and densifies Gaussian scales with
simple-knn's distCUDA2 (scene/gaussian_model.py:175-179, :729-733).  The oracle's C
restatement is pinned against scipy's KD-tree in float64; the CUDA kernel must match the
oracle bit for bit.
"""
import numpy as np
import pytest


def _clustered(n, seed, dup=0):
    rng = np.random.default_rng(seed)
    c = rng.random((64, 3))
    p = (c[rng.integers(0, 64, n)] + rng.normal(0.0, 0.004, (n, 3))).astype(np.float32)
    if dup:
        p[:dup] = p[dup:2 * dup]
    return p


def _lattice(k):
    g = (np.arange(k, dtype=np.float32) / k)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], 1).astype(np.float32)


def _scipy_ref(p):
    from scipy.spatial import cKDTree
    q = p.astype(np.float64)
    d, _ = cKDTree(q).query(q, k=4)
    return (d[:, 1:] ** 2).mean(1)


@pytest.mark.parametrize("kind", ["uniform", "clustered", "duplicates", "lattice"])
def test_oracle_matches_kdtree(orc, kind):
    rng = np.random.default_rng(3)
    p = {"uniform": lambda: rng.random((20000, 3), dtype=np.float32),
         "clustered": lambda: _clustered(20000, 4),
         "duplicates": lambda: _clustered(20000, 5, dup=500),
         "lattice": lambda: _lattice(24)}[kind]()
    got = orc.knn3_mean_dist2(p).astype(np.float64)
    ref = _scipy_ref(p)
    # float32 squared distances and sum: a few ulps of the float64 value
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-12)


def test_oracle_small_counts(orc):
    big = np.float32(3.4028235e38)
    p = np.array([[0, 0, 0], [1, 0, 0], [0, 2, 0]], np.float32)
    assert np.isinf(orc.knn3_mean_dist2(p[:1])).all()
    assert np.isinf(orc.knn3_mean_dist2(p[:2])).all()
    three = orc.knn3_mean_dist2(p)
    # (d0 + d1) + FLT_MAX rounds to FLT_MAX for small distances
    assert np.all(three == np.float32(big / np.float32(3.0)))
    four = orc.knn3_mean_dist2(np.vstack([p, [[0, 0, 3]]]).astype(np.float32))
    assert four[0] == np.float32((np.float32(1.0) + np.float32(4.0) + np.float32(9.0)) / np.float32(3.0))


def test_distcuda2_rejects_bad_input():
    torch = pytest.importorskip("torch")
    from simple_knn._C import distCUDA2
    with pytest.raises(RuntimeError):
        distCUDA2(torch.zeros(4, 3))               # not on a GPU
    with pytest.raises(RuntimeError):
        distCUDA2(np.zeros((4, 3), np.float32))    # not a tensor


def _gpu(p):
    import torch
    from simple_knn._C import distCUDA2
    t = torch.from_numpy(p).cuda()
    out = distCUDA2(t)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 33, 1000])
def test_gpu_knn_small(cuda, orc, n):
    p = np.random.default_rng(n).random((n, 3), dtype=np.float32)
    got = _gpu(p)
    ref = orc.knn3_mean_dist2(p)
    assert got.dtype == np.float32 and got.shape == (n,)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["uniform", "clustered", "duplicates", "lattice", "plane"])
def test_gpu_knn_bit_exact(cuda, orc, kind):
    rng = np.random.default_rng(11)
    if kind == "uniform":
        p = rng.random((200000, 3), dtype=np.float32)
    elif kind == "clustered":
        p = _clustered(200000, 12)
    elif kind == "duplicates":
        p = _clustered(100000, 13, dup=5000)
    elif kind == "lattice":
        p = _lattice(40)            # many exactly equal distances
    else:
        p = rng.random((100000, 3), dtype=np.float32)
        p[:, 2] = 0.5               # all on one plane: degenerate extent
    got = _gpu(p)
    ref = orc.knn3_mean_dist2(p)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.gpu
def test_gpu_knn_densify_call(cuda, orc):
    """The densify call site: existing points concatenated with new ones, scaled by 0.1
    and clamped (scene/gaussian_model.py:727-734); the new points' slice is taken."""
    import torch
    from simple_knn._C import distCUDA2
    old = torch.from_numpy(_clustered(150000, 21)).cuda()
    new = torch.rand(30000, 3, device="cuda")
    allp = torch.cat([old, new], 0)
    d2 = torch.clamp_min(distCUDA2(allp) * 0.1, 0.0000001)[old.shape[0]:]
    ref = orc.knn3_mean_dist2(allp.cpu().numpy())[old.shape[0]:]
    ref = np.maximum(ref * np.float32(0.1), np.float32(0.0000001))
    np.testing.assert_array_equal(d2.cpu().numpy(), ref)


@pytest.mark.gpu
def test_gpu_knn_large(cuda, orc):
    """2M points (the headline Gaussian count), half uniform, half clustered."""
    rng = np.random.default_rng(31)
    p = np.vstack([rng.random((1000000, 3), dtype=np.float32), _clustered(1000000, 32)])
    got = _gpu(p)
    ref = orc.knn3_mean_dist2(p)
    np.testing.assert_array_equal(got, ref)
