"""The oracle's restatements of the reference's Python layers against fixtures produced by
running the reference's own functions (tests/golden/make_golden.py)."""
import os

import numpy as np
import torch

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_python.npz")


def test_morton21_render_order(orc):
    d = np.load(GOLDEN)
    np.testing.assert_array_equal(orc.morton21(d["morton_pts"], clamp=False), d["morton_render"])
    np.testing.assert_array_equal(orc.morton21(d["ply_xyz"], clamp=False), d["ply_morton"])


def test_morton21_sample_order(orc):
    d = np.load(GOLDEN)
    np.testing.assert_array_equal(orc.morton21(d["morton_pts"], clamp=True), d["morton_train"])


def test_activations_on_trained_mixture(orc):
    d = np.load(GOLDEN)
    args = [torch.tensor(d[k], dtype=torch.float32) for k in
            ("ply_xyz", "ply_raw_scale", "ply_raw_rot", "ply_raw_weight", "ply_raw_value")]
    _, s, q, w, v = orc.activations(*args, xp=torch)
    np.testing.assert_allclose(s.numpy(), d["ply_scale"], rtol=1e-6)
    np.testing.assert_allclose(q.numpy(), d["ply_rot"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(w.numpy(), d["ply_weight"], rtol=1e-6)
    np.testing.assert_allclose(v.numpy(), d["ply_value"], rtol=1e-6)
    # numpy FP64 restatement agrees too
    _, s64, q64, w64, v64 = orc.activations(*[a.double().numpy() for a in args])
    np.testing.assert_allclose(s64, d["ply_scale"], rtol=1e-5)


def test_trained_mixture_forward_is_finite(orc):
    """The shipped trained mixture through the oracle: finite outputs, valid samples."""
    d = np.load(GOLDEN)
    args = [torch.tensor(d[k], dtype=torch.float32) for k in
            ("ply_xyz", "ply_raw_scale", "ply_raw_rot", "ply_raw_weight", "ply_raw_value")]
    m, s, q, w, v = [a.numpy() for a in orc.activations(*args, xp=torch)]
    lo, hi = m.min(0), m.max(0)
    samples = (lo + np.random.default_rng(0).random((20000, 3)) * (hi - lo)).astype(np.float32)
    _, c64, bb = orc.preprocess(m, s, q, w.ravel())
    out, outw = orc.forward(m, v.ravel(), w.ravel(), c64, bb, samples)
    assert np.isfinite(out).all() and (out != -1).any()
