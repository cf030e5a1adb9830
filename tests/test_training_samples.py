"""Training sample batches on the device (train.py:34-61, :273-282, :286-315).

The generator is Philox4x32-10, pinned here by the published known-answer vectors of its
authors' Random123 distribution; the per-batch Morton order is the oracle's morton21,
pinned by fixtures made from the reference's own code (tests/golden).  The GPU batches
(points, order and float32 ground truth) must match the oracle bit for bit.
"""
import numpy as np
import pytest

import gvc_workloads as wl

# Philox4x32-10 known answers: (counter, key) -> output
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(orc, ctr, key, want):
    assert tuple(int(x) for x in orc.philox4x32_10(ctr, key)) == want


def test_oracle_batches_properties(orc):
    pts, tets = wl.jittered_tet_mesh(n=8, seed=2)
    vals = wl.blob_field(pts).astype(np.float64)
    B, S = 3, 20000
    samples, gt = orc.training_samples(pts, tets, vals, B, S, seed=9)
    assert samples.shape == (B, S, 3) and gt.shape == (B, S) and gt.dtype == np.float32
    for b in range(B):
        keys = orc.morton21(samples[b], clamp=True)
        assert np.all(np.diff(keys.astype(np.uint64)) >= 0)
    # every point lies in the mesh (up to rounding on its boundary) and has a value
    assert samples.min() >= -1e-6 and samples.max() <= 1 + 1e-6
    assert (gt != -1).mean() > 0.999
    # uniform over cells: the mean of a fixed fine grid of the unit cube is 1/2
    assert np.abs(samples.reshape(-1, 3).mean(0) - 0.5).max() < 0.01
    # another seed gives other points; the same seed the same ones
    again, _ = orc.training_samples(pts, tets, None, B, S, seed=9)
    other, _ = orc.training_samples(pts, tets, None, B, S, seed=10)
    assert np.array_equal(again, samples) and not np.array_equal(other, samples)


def test_cell_choice_is_uniform(orc):
    """Cells are chosen uniformly: counts over 8 cells of 200k draws stay within 5 sigma."""
    pts, tets = wl.jittered_tet_mesh(n=1, seed=0)   # 6 tets of one cube
    tets = np.vstack([tets, tets[:2]])              # 8 cells, two duplicated
    samples, _ = orc.training_samples(pts, tets, None, 1, 200000, seed=1)
    # attribute each point back to its generating cell by locating it in the cube's tets
    _, cell = orc.sample_tets(pts, tets[:6], np.zeros(pts.shape[0]), samples.reshape(-1, 3))
    counts = np.bincount(cell[cell >= 0], minlength=6)
    expect = np.array([2, 2, 1, 1, 1, 1]) * 200000 / 8.0
    assert np.all(np.abs(counts - expect) <= 5 * np.sqrt(expect))


def test_rejects_bad_mesh():
    from gpu_mesh_sampling import sample_training_batches
    pts, tets = wl.jittered_tet_mesh(n=2, seed=0)
    with pytest.raises(RuntimeError):
        sample_training_batches(pts, tets + pts.shape[0], np.zeros(pts.shape[0]), 1, 10)
    with pytest.raises(RuntimeError):
        sample_training_batches(pts, tets[:0], np.zeros(pts.shape[0]), 1, 10)
    with pytest.raises(RuntimeError):
        sample_training_batches(pts, tets, np.zeros(3), 1, 10)


def _hex_cells(n):
    """VTK hexahedra of the n^3 grid that jittered_tet_mesh(n) splits into tetrahedra."""
    N1 = n + 1
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()

    def vid(di, dj, dk):
        return (k + dk) * N1 * N1 + (j + dj) * N1 + (i + di)

    conn = np.stack([vid(0, 0, 0), vid(1, 0, 0), vid(1, 1, 0), vid(0, 1, 0),
                     vid(0, 0, 1), vid(1, 0, 1), vid(1, 1, 1), vid(0, 1, 1)], 1).reshape(-1)
    C = n ** 3
    return conn.astype(np.int64), np.full(C, 12, np.int64), np.arange(C, dtype=np.int64) * 8


@pytest.mark.gpu
@pytest.mark.parametrize("n,B,S,seed", [(16, 3, 10000, 7), (4, 1, 1, 0), (8, 5, 4097, 123456789012345),
                                        (12, 130, 257, 3)])
def test_gpu_batches_bit_exact(cuda, orc, n, B, S, seed):
    from gpu_mesh_sampling import sample_training_batches
    pts, tets = wl.jittered_tet_mesh(n=n, seed=5)
    vals = wl.blob_field(pts).astype(np.float64)
    samples, gt = sample_training_batches(pts, tets, vals, B, S, seed=seed)
    ref_s, ref_g = orc.training_samples(pts, tets, vals, B, S, seed=seed)
    np.testing.assert_array_equal(samples.cpu().numpy(), ref_s)
    np.testing.assert_array_equal(gt.cpu().numpy(), ref_g)


@pytest.mark.gpu
def test_gpu_batches_ground_truth_from_hexahedra(cuda, orc):
    """Points from the tetrahedra, ground truth from the untriangulated hexahedral mesh."""
    from gpu_mesh_sampling import sample_training_batches
    n = 8
    pts, tets = wl.jittered_tet_mesh(n=n, seed=6)
    vals = wl.blob_field(pts).astype(np.float64)
    cells = _hex_cells(n)
    samples, gt = sample_training_batches(pts, tets, vals, 2, 30000, seed=4, gt_cells=cells)
    ref_s, _ = orc.training_samples(pts, tets, None, 2, 30000, seed=4)
    np.testing.assert_array_equal(samples.cpu().numpy(), ref_s)
    ref_g, _ = orc.sample_cells(pts, cells[1], cells[2], cells[0], vals, ref_s.reshape(-1, 3))
    np.testing.assert_array_equal(gt.cpu().numpy().reshape(-1), ref_g.astype(np.float32))
    assert (gt != -1).float().mean().item() > 0.99


@pytest.mark.gpu
def test_gpu_batches_large(cuda, orc):
    """4 batches of 1M points on a 64^3 grid (1.57M tetrahedra)."""
    from gpu_mesh_sampling import sample_training_batches
    pts, tets = wl.jittered_tet_mesh(n=64, seed=8)
    vals = wl.blob_field(pts).astype(np.float64)
    samples, gt = sample_training_batches(pts, tets, vals, 4, 1 << 20, seed=11)
    ref_s, ref_g = orc.training_samples(pts, tets, vals, 4, 1 << 20, seed=11)
    np.testing.assert_array_equal(samples.cpu().numpy(), ref_s)
    np.testing.assert_array_equal(gt.cpu().numpy(), ref_g)
