"""Candidate log: the tensor-core backward reading the forward's candidates back.

With the tensor-core backward selected before the forward (GVC_OPT_BWD_MODE = 3), the
block-group forward records every block's candidate Gaussians and the backward reads
them instead of walking the Gaussian LBVH again (GVC_OPT_CAND_LOG, on by default).
Checks, with the tolerances of test_gpu_rasterizer:

* the logged backward against the oracle's FP64 adjoint (both forwards);
* at scale (200k clustered Gaussians x 1M samples) against the same backward walking the
  tree (log off): the same fields, gradients within the atomic-order tolerance;
* a block with more candidates than its log slots (4096) falls back to walking;
* a backward whose Gaussians are not the forward's (a different P) walks the tree;
* a log recorded by the forward's stackless traversal serves the backward the same way.
"""
import contextlib

import numpy as np
import pytest

from test_gpu_rasterizer import T, assert_grads_close, oracle_backward

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def modes(path="plain", log=True):
    from bvh_diff_gaussian_rasterization import _C
    _C.set_eval_path(path)
    _C.set_backward_mode("tensor_core")
    _C.set_candidate_log(log)
    try:
        yield _C
    finally:
        _C.set_eval_path("plain")
        _C.set_backward_mode("auto")
        _C.set_candidate_log(True)


def step(dev, case, gout, gw, count=False):
    """build_bvh, forward and backward with the modes already set (the forward logs)."""
    from bvh_diff_gaussian_rasterization import _C
    means, scales, rots, values, weights, samples = case
    _C.build_bvh(T(samples, dev), False, False)
    if count:
        _C.set_count_pairs(True)
    try:
        out, outw, conics = _C.rasterize_gaussians(T(means, dev), T(scales, dev), T(rots, dev), T(values, dev),
                                                   T(weights, dev), 1.0, 0, 0, 0, 1, 1, 1, -1.0, False, False)
        g = _C.rasterize_gaussians_backward(T(means, dev), T(scales, dev), T(rots, dev), conics, T(values, dev),
                                            T(weights, dev), out, outw, 1.0, 0, 0, 0, 1, 1, 1, -1.0, T(gout, dev),
                                            T(gw, dev), False, False)
        _C.check_status()
        st = _C.stats() if count else None
    finally:
        _C.set_count_pairs(False)
    return ([x.cpu().numpy() for x in g], out.cpu().numpy(), outw.cpu().numpy(),
            conics.cpu().numpy().reshape(-1, 6), st)


@pytest.fixture(scope="module")
def small_case(cuda, orc):
    means, scales, rots, values, weights = orc.mixture_small(seed=0, P=4096)
    return means, scales, rots, values, weights, orc.grid_centres(64)


@pytest.mark.parametrize("path", ["plain", "tensor_core"])
def test_logged_backward_matches_oracle(cuda, orc, small_case, path):
    S = small_case[-1].shape[0]
    rng = np.random.default_rng(51)
    gout = rng.normal(size=S).astype(np.float32)
    gw = rng.normal(size=S).astype(np.float32)
    with modes(path):
        got, out, outw, conics, st = step(cuda, small_case, gout, gw, count=True)
    assert st["bwd_node_visits"] == 0  # every block read its candidates from the log
    ref = oracle_backward(orc, small_case, out, outw, conics, gout, gw)
    assert_grads_close(got, ref)


def test_logged_equals_walked_at_scale(cuda, orc):
    """200k clustered Gaussians x 1M samples: the logged backward (its groups' candidates
    filtered from the enclosing forward groups' logs) against the backward walking the
    tree: the same evaluated rows and contributing pairs, gradients within tolerance."""
    case = orc.mixture_large(seed=4, P=200_000, S=1_000_000)
    S = case[-1].shape[0]
    rng = np.random.default_rng(52)
    gout = rng.normal(size=S).astype(np.float32)
    gw = np.zeros(S, np.float32)
    with modes(log=True):
        ga, oa, wa, _, sa = step(cuda, case, gout, gw, count=True)
    with modes(log=False):
        gb, ob, wb, _, sb = step(cuda, case, gout, gw, count=True)
    np.testing.assert_array_equal(oa, ob)  # same forward kernel and order
    np.testing.assert_array_equal(wa, wb)
    assert sa["bwd_node_visits"] == 0 and sb["bwd_node_visits"] > 0
    assert sa["bwd_contributing"] == sb["bwd_contributing"]
    assert sa["bwd_rows"] == sb["bwd_rows"]  # same groups, same candidates per group
    for k in range(5):
        assert np.abs(ga[k] - gb[k]).max() <= 5e-4 * np.abs(gb[k]).max(), k


def test_log_overflow_and_stale_log_walk(cuda, orc):
    """Every block of a mixture of 5000 large Gaussians has more candidates than its 4096
    log slots: the backward walks the tree for them.  A backward with a different number
    of Gaussians than the forward's does not use the log."""
    means, scales, rots, values, weights = orc.mixture_small(seed=6, P=5000)
    scales = (scales * 0 + 0.2).astype(np.float32)  # every box covers most of the cube
    samples = orc.grid_centres(16)
    case = (means, scales, rots, values, weights, samples)
    S = samples.shape[0]
    rng = np.random.default_rng(53)
    gout = rng.normal(size=S).astype(np.float32)
    gw = rng.normal(size=S).astype(np.float32)
    with modes():
        got, out, outw, conics, st = step(cuda, case, gout, gw, count=True)
    assert st["bwd_node_visits"] > 0
    assert_grads_close(got, oracle_backward(orc, case, out, outw, conics, gout, gw))


def test_backward_of_other_gaussians_walks(cuda, orc, small_case):
    """Forward on 4096 Gaussians (log written), backward on the first 4000 of them with
    the forward's outputs: the log does not belong to them, the backward walks."""
    from bvh_diff_gaussian_rasterization import _C
    means, scales, rots, values, weights, samples = small_case
    S = samples.shape[0]
    rng = np.random.default_rng(54)
    gout = rng.normal(size=S).astype(np.float32)
    gw = rng.normal(size=S).astype(np.float32)
    n = 4000
    sub = tuple(a[:n] for a in (means, scales, rots, values, weights)) + (samples,)
    with modes():
        _C.build_bvh(T(samples, cuda), False, False)
        _C.set_count_pairs(True)  # the forward clears the counters
        try:
            out, outw, conics = _C.rasterize_gaussians(T(means, cuda), T(scales, cuda), T(rots, cuda),
                                                       T(values, cuda), T(weights, cuda), 1.0, 0, 0, 0, 1, 1, 1,
                                                       -1.0, False, False)
            c6 = conics.reshape(-1, 6)[:n].contiguous().reshape(-1)
            g = _C.rasterize_gaussians_backward(T(sub[0], cuda), T(sub[1], cuda), T(sub[2], cuda), c6,
                                                T(sub[3], cuda), T(sub[4], cuda), out, outw, 1.0, 0, 0, 0, 1, 1, 1,
                                                -1.0, T(gout, cuda), T(gw, cuda), False, False)
            _C.check_status()
            st = _C.stats()
        finally:
            _C.set_count_pairs(False)
    assert st["bwd_node_visits"] > 0
    got = [x.cpu().numpy() for x in g]
    ref = oracle_backward(orc, sub, out.cpu().numpy(), outw.cpu().numpy(), c6.cpu().numpy().reshape(-1, 6), gout, gw)
    assert_grads_close(got, ref)


def test_logged_backward_with_stackless_forward(cuda, orc, small_case):
    """The stackless traversal hands the forward's producer the same candidates in another
    order; the log it records serves the backward just the same."""
    from bvh_diff_gaussian_rasterization import _C
    S = small_case[-1].shape[0]
    rng = np.random.default_rng(55)
    gout = rng.normal(size=S).astype(np.float32)
    gw = rng.normal(size=S).astype(np.float32)
    _C.set_traversal("stackless")
    try:
        with modes():
            got, out, outw, conics, st = step(cuda, small_case, gout, gw, count=True)
    finally:
        _C.set_traversal("stack")
    assert st["bwd_node_visits"] == 0
    assert_grads_close(got, oracle_backward(orc, small_case, out, outw, conics, gout, gw))
