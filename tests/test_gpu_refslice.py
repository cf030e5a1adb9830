"""The GPU kernels against the reference's OWN rasterizer code compiled for the host
(oracle/_ref/libgvc_ref.so, built from diff-gaussian-rasterization/cuda_rasterizer/
forward.cu and backward.cu by oracle/build_ref.py; skipped when it was not built).

All GPU calls go through the C ABI (the drop-in `_C` module).  Tolerances:
  * conics bit-exact (prep.cu rounds every operation as the reference's source is written);
    AABB corners within 4 ulps of their addends (m from double here, logf there);
  * forward, every evaluation path and both BVH modes: |d out| <= 2e-5 and |d outw| <=
    2e-5 outw against the reference's FP32 sums, with the -14 floor allowance of
    test_gpu_rasterizer;
  * backward, every mode, with the reference-compatible covariance adjoint: max |d grad|
    <= 1e-4 of max |grad| for means, values, weights; 5e-4 for scales and rotations.
"""
import numpy as np
import pytest

import refslice
from test_gpu_rasterizer import (assert_grads_close, compare_forward, gpu_preprocess, run_backward,
                                 run_forward)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refslice.available(), reason="oracle/_ref not built")]


@pytest.fixture(scope="module")
def case(cuda, orc):
    means, scales, rots, values, weights = orc.mixture_small(seed=0, P=4096)
    return means, scales, rots, values, weights, orc.grid_centres(64)


def test_preprocess_matches_reference_code(cuda, case):
    import gvc_native
    means, scales, rots, values, weights, _ = case
    rc, rb = refslice.preprocess(means, scales, rots, weights)
    gc, gb = gpu_preprocess(gvc_native.Context(), cuda, means, scales, rots, weights)
    np.testing.assert_array_equal(gc, rc)
    mm = np.concatenate([means, means], 1)
    mag = np.maximum(np.maximum(np.abs(rb), np.abs(mm)), np.abs(rb - mm)).astype(np.float32)
    assert np.all(np.abs(gb - rb) <= 4 * np.spacing(mag))


@pytest.mark.parametrize("path,use_gaussian_bvh", [("plain", False), ("plain", True), ("tensor_core", False),
                                                   ("plain_tile", False)])
def test_forward_matches_reference_code(cuda, case, path, use_gaussian_bvh):
    from bvh_diff_gaussian_rasterization import _C
    means, scales, rots, values, weights, samples = case
    _C.set_eval_path(path)
    try:
        out, outw, _ = run_forward(cuda, means, scales, rots, values, weights, samples, use_gaussian_bvh)
    finally:
        _C.set_eval_path("plain")
    rc, rb = refslice.preprocess(means, scales, rots, weights)
    ro, rw, _ = refslice.forward(means, values, weights, samples, rc, rb)
    compare_forward(out.cpu().numpy(), outw.cpu().numpy(), ro.astype(np.float64), rw.astype(np.float64),
                    2e-5, 2e-5)


@pytest.mark.parametrize("mode", ["deterministic", "atomic", "tensor_core"])
def test_backward_matches_reference_code(cuda, case, mode):
    means, scales, rots, values, weights, samples = case
    S = samples.shape[0]
    rng = np.random.default_rng(31)
    gout = rng.normal(size=S).astype(np.float32)
    gw = (0.1 * rng.normal(size=S)).astype(np.float32)
    got, out, outw, conics = run_backward(cuda, case, gout, gw, mode, False, cov="ref_compat")
    rc, rb = refslice.preprocess(means, scales, rots, weights)
    np.testing.assert_array_equal(conics, rc)
    # the reference's backward on the GPU forward's own outputs
    refslice.config(serial=True)
    try:
        g = refslice.backward(means, scales, rots, rc, values, weights, rb, samples, out, outw, gout, gw)
    finally:
        refslice.config(serial=False)
    ref = [g["dmeans"], g["dscales"], g["drots"], g["dvalues"].reshape(-1, 1), g["dweights"].reshape(-1, 1)]
    assert_grads_close(got, ref)
