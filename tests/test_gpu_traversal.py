"""Stackless LBVH traversal on the GPU (gvc_set_option(GVC_OPT_TRAVERSAL, 1)).

* The escape edges the builder stores in the nodes equal the CPU model's
  (test_traversal_model.escape_edges over the oracle's topology), for the tree sizes and
  key patterns of the LBVH bit-exactness test.
* The block-group forwards (FP32 and tensor-core exponent) and the tensor-core backward
  with the stackless traversal meet the same oracle tolerances as with the stack
  (test_gpu_rasterizer / test_gpu_tc).
* At scale (200k clustered Gaussians x 1M samples) both traversals hand over the same
  candidates: the pair counters agree exactly, and the fields agree within the FP32
  reordering tolerance.
"""
import contextlib

import numpy as np
import pytest
import torch

import gvc_native
from test_gpu_rasterizer import (assert_grads_close, compare_forward, gpu_lbvh, gpu_preprocess, oracle_backward,
                                 run_backward, run_forward, stream)
from test_traversal_model import escape_edges, make_boxes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(cuda):
    return gvc_native.Context()


@contextlib.contextmanager
def settings(traversal="stack", path="plain"):
    from bvh_diff_gaussian_rasterization import _C
    _C.set_traversal(traversal)
    _C.set_eval_path(path)
    try:
        yield _C
    finally:
        _C.set_traversal("stack")
        _C.set_eval_path("plain")


@pytest.mark.parametrize("n,kind", [(1, "rand"), (2, "rand"), (3, "rand"), (33, "rand"), (1000, "rand"),
                                    (4097, "dup"), (300000, "rand"), (300000, "cluster")])
def test_escape_edges_match_model(ctx, cuda, orc, n, kind):
    boxes = make_boxes(n, kind, n)
    gpu_lbvh(ctx, cuda, boxes)
    esc = torch.empty(max(n - 1, 1), dtype=torch.int32, device=cuda)
    ctx.call("gvc_debug_lbvh_escape", gvc_native.ptr(esc), stream())
    torch.cuda.synchronize()
    got = esc.cpu().numpy().view(np.uint32)
    if n == 1:
        assert got[0] == 0xFFFFFFFF
        return
    _, _, left, right, _ = orc.lbvh_build(boxes)
    np.testing.assert_array_equal(got, escape_edges(left, right).astype(np.uint32))


@pytest.fixture(scope="module")
def small_case(cuda, orc):
    means, scales, rots, values, weights = orc.mixture_small(seed=0, P=4096)
    return means, scales, rots, values, weights, orc.grid_centres(64)


@pytest.mark.parametrize("path,tol", [("plain", 2e-5), ("tensor_core", 1e-4)])
def test_stackless_forward_matches_oracle(ctx, cuda, orc, small_case, path, tol):
    means, scales, rots, values, weights, samples = small_case
    with settings("stackless", path):
        out, outw, conics = run_forward(cuda, *small_case)
    out, outw = out.cpu().numpy(), outw.cpu().numpy()
    gc = conics.cpu().numpy().reshape(-1, 6)
    _, gb = gpu_preprocess(ctx, cuda, means, scales, rots, weights)
    ro, rw = orc.forward(means, values, weights, gc.astype(np.float64), gb, samples)
    compare_forward(out, outw, ro, rw, tol, tol)
    assert (out != -1).mean() > 0.5


@pytest.mark.parametrize("gw_scale", [0.0, 1.0])
def test_stackless_tensor_core_backward_matches_oracle(cuda, orc, small_case, gw_scale):
    S = small_case[-1].shape[0]
    rng = np.random.default_rng(41)
    gout = rng.normal(size=S).astype(np.float32)
    gw = (gw_scale * rng.normal(size=S)).astype(np.float32)
    with settings("stackless"):
        got, out, outw, conics = run_backward(cuda, small_case, gout, gw, "tensor_core")
    ref = oracle_backward(orc, small_case, out, outw, conics, gout, gw)
    assert_grads_close(got, ref)


def test_stackless_edge_cases(cuda, orc):
    """One and two Gaussians (a single-leaf tree and a root with two leaves), a partial
    block, and samples outside every box."""
    means, scales, rots, values, weights = orc.mixture_small(seed=5, P=7)
    rng = np.random.default_rng(2)
    for P in (1, 2, 7):
        smp = (np.repeat(means[:1], 33, 0) + rng.normal(0, 0.01, (33, 3))).astype(np.float32)
        for path in ("plain", "tensor_core"):
            with settings("stackless", path):
                o, ow, c = run_forward(cuda, means[:P], scales[:P], rots[:P], values[:P], weights[:P], smp)
            ro, rw = orc.forward(means[:P], values[:P], weights[:P],
                                 c.cpu().numpy().reshape(-1, 6).astype(np.float64),
                                 orc.preprocess(means[:P], scales[:P], rots[:P], weights[:P])[2], smp)
            np.testing.assert_allclose(ow.cpu().numpy(), rw, rtol=1e-4, atol=1e-7)
    pts = rng.random((50, 3)).astype(np.float32) + 5.0
    with settings("stackless"):
        o, ow, _ = run_forward(cuda, means, scales, rots, values, weights, pts)
    assert bool((o == -1).all()) and bool((ow == 0).all())


def _step_counts(cuda, case, traversal, path):
    from test_gpu_rasterizer import run_backward as rb
    S = case[-1].shape[0]
    rng = np.random.default_rng(43)
    gout = rng.normal(size=S).astype(np.float32)
    gw = np.zeros(S, np.float32)
    with settings(traversal, path) as _C:
        _C.set_count_pairs(True)
        try:
            g, out, outw, _ = rb(cuda, case, gout, gw, "tensor_core")
            st = _C.stats()
        finally:
            _C.set_count_pairs(False)
    return g, out, outw, st


@pytest.mark.parametrize("path", ["plain", "tensor_core"])
def test_stackless_same_candidates_at_scale(cuda, orc, path):
    means, scales, rots, values, weights, samples = orc.mixture_large(seed=3, P=200_000, S=1_000_000)
    case = (means, scales, rots, values, weights, samples)
    ga, oa, wa, sa = _step_counts(cuda, case, "stack", path)
    gb, ob, wb, sb = _step_counts(cuda, case, "stackless", path)
    for key in ("fwd_leaf_hits", "fwd_candidates", "fwd_contributing", "bwd_leaf_hits", "bwd_contributing"):
        assert sa[key] == sb[key], (key, sa[key], sb[key])
    for key in ("fwd_node_visits", "bwd_node_visits", "fwd_lane_evals", "bwd_rows"):  # order-dependent
        print("%s: stack %d, stackless %d" % (key, sa[key], sb[key]))
    near = np.abs(wa - 0.01) <= 1e-6 + 4e-6
    ok = ~near
    assert np.array_equal(oa[ok] == -1, ob[ok] == -1)
    v = ok & (oa != -1)
    assert ((np.abs(wb[v] - wa[v]) - 4e-6) / wa[v]).max() <= 2e-5
    assert (np.abs(ob[v] - oa[v]) - 4e-6 / wa[v]).max() <= 2e-5
    # two runs of the atomic tensor-core backward, each within the oracle tolerance (1e-4 of
    # max; 5e-4 for the covariance adjoint: scales, rotations), differ by at most twice it
    for k in range(5):
        tol = 1e-3 if k in (1, 2) else 2e-4
        assert np.abs(gb[k] - ga[k]).max() <= tol * np.abs(ga[k]).max(), k
