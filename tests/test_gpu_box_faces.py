"""Samples exactly on the Gaussians' AABB faces: the closed-box test of the evaluation
kernels at equality.

The FP32 forward compares (lo <= x <= hi); the tensor-core backward tests the sign bits of
x - lo and hi - x.  On a face one of those differences is exactly zero, and both tests
must keep the pair, as the oracle (forward.cu:224-230, backward.cu:252-256: closed box)
does.  The oracle is given the GPU's own conics and boxes, so any difference is a box or
window decision; the weights are high enough that the power on a face lies inside the
window, so a dropped face pair shows in W and in the gradients.
"""
import numpy as np
import pytest

import gvc_native
from test_gpu_candlog import modes, step
from test_gpu_rasterizer import assert_grads_close, compare_forward, gpu_preprocess

pytestmark = pytest.mark.gpu


def face_case(orc, seed=7, P=64):
    """P small isotropic Gaussians (scale 0.02, w = 0.005: their boxes' faces lie at about
    2.8 sigma, power -4, well inside the window) over one wide Gaussian that keeps every
    sample above the 0.01 cutoff; 48 samples exactly on each small Gaussian's faces, near
    the face centres."""
    rng = np.random.default_rng(seed)
    means = np.vstack([rng.uniform(0.2, 0.8, (P, 3)), [[0.5, 0.5, 0.5]]]).astype(np.float32)
    scales = np.vstack([np.full((P, 3), 0.02), [[0.3, 0.3, 0.3]]]).astype(np.float32)
    q = rng.normal(size=(P + 1, 4))
    rots = (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)
    values = rng.uniform(0.1, 0.9, (P + 1, 1)).astype(np.float32)
    weights = np.vstack([np.full((P, 1), 0.005), [[0.9]]]).astype(np.float32)
    return means, scales, rots, values, weights, rng


@pytest.mark.parametrize("path", ["plain", "tensor_core"])
def test_samples_on_box_faces(cuda, orc, path):
    means, scales, rots, values, weights, rng = face_case(orc)
    _, gb = gpu_preprocess(gvc_native.Context(), cuda, means, scales, rots, weights.ravel())
    pts = []
    for i in range(len(means) - 1):
        lo, hi = gb[i, :3].astype(np.float64), gb[i, 3:].astype(np.float64)
        mid, half = 0.5 * (lo + hi), 0.5 * (hi - lo)
        for _ in range(48):
            p = mid + 0.3 * half * (2 * rng.random(3) - 1)
            ax = int(rng.integers(0, 3))
            p[ax] = lo[ax] if rng.random() < 0.5 else hi[ax]  # exactly on a face (float32 value)
            pts.append(p)
    samples = np.asarray(pts, np.float32)
    case = (means, scales, rots, values.ravel(), weights.ravel(), samples)
    S = len(samples)
    gout = rng.normal(size=S).astype(np.float32)
    gw = rng.normal(size=S).astype(np.float32)
    with modes(path):
        got, out, outw, conics, _ = step(cuda, case, gout, gw)
    c64 = conics.astype(np.float64)
    m, v, w = means, values.ravel(), weights.ravel()
    ro, rw = orc.forward(m, v, w, c64, gb, samples)
    assert (rw > 0.01).all()
    # the face pairs matter: without them (boxes shrunk by one ulp) W moves by > 1e-4
    shrunk = gb.copy()
    shrunk[:, :3] = np.nextafter(gb[:, :3], np.float32(np.inf))
    shrunk[:, 3:] = np.nextafter(gb[:, 3:], np.float32(-np.inf))
    _, rw_in = orc.forward(m, v, w, c64, shrunk, samples)
    assert (np.abs(rw_in - rw) / rw > 1e-4).mean() > 0.5
    tol = 2e-5 if path == "plain" else 1e-4
    compare_forward(out, outw, ro, rw, tol, tol)
    g = orc.backward(m, v, w, c64, gb, samples, out, outw, gout, gw)
    ds, dq = orc.cov_backward(scales, rots, conics, g["dconics"])
    assert_grads_close(got, [g["dmeans"], ds, dq, g["dvalues"].reshape(-1, 1), g["dweights"].reshape(-1, 1)])
