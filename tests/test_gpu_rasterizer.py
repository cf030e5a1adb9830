"""GPU parity of the rasterizer path against the oracle (all calls go through the C ABI,
directly or through the drop-in Python API).

Tolerances (FP32 kernels vs the FP64 oracle):
  * preprocess conics: bit-exact; AABBs: bit-exact except <= 1 ulp where CUDA's and the
    host's double log differ (<= 0.1% of boxes);
  * LBVH keys / permutation / topology / node boxes, sample order: bit-exact;
  * forward given the same conics and boxes: |d out| <= 2e-5, |d outw| <= 2e-5 outw, plus
    an allowance for pairs at the -14 power floor (see FLOOR_PAIR);
  * forward vs the full FP64 pipeline: relative error <= 1e-4 (out and outw), same allowance;
  * backward given the same inputs: max |d grad| <= 1e-4 max |grad| per field (5e-4 for
    the covariance adjoint);
  * gradients vs FP64 central finite differences: |an - fd| <= 1e-3 max(|fd|, 1e-3).
Samples whose FP64 weight is within 1e-5 (relative) of the 0.01 cutoff are excluded
from value comparisons (the cutoff is a discontinuity).
"""
import ctypes

import numpy as np
import pytest
import torch

import gvc_native

pytestmark = pytest.mark.gpu


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.fixture(scope="module")
def ctx(cuda):
    return gvc_native.Context()


def gpu_preprocess(ctx, dev, means, scales, rots, weights, sm=1.0):
    P = means.shape[0]
    dm, ds, dq, dw = (T(means, dev), T(scales, dev), T(rots, dev), T(weights, dev))
    c = torch.empty(P * 6, device=dev)
    bb = torch.empty(P * 6, device=dev)
    ctx.call("gvc_debug_preprocess", P, gvc_native.ptr(dm), gvc_native.ptr(ds), gvc_native.ptr(dq),
             gvc_native.ptr(dw), sm, gvc_native.ptr(c), gvc_native.ptr(bb), stream())
    torch.cuda.synchronize()
    return c.cpu().numpy().reshape(P, 6), bb.cpu().numpy().reshape(P, 6)


def ulp_diff(a, b):
    return np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))


def test_preprocess_bit_exact(ctx, cuda, orc):
    means, scales, rots, values, weights = orc.mixture_small(seed=0, P=4096)
    scales[:64, 1] *= 0.01          # ill-conditioned: FP64 inverse
    weights[64:80] = 5e-4           # w < 1e-3: the box collapses to the mean
    c32, c64, bb = orc.preprocess(means, scales, rots, weights)
    gc, gb = gpu_preprocess(ctx, cuda, means, scales, rots, weights)
    np.testing.assert_array_equal(gc, c32)
    d = ulp_diff(gb, bb)
    assert d.max() <= 1 and (d > 0).mean() <= 1e-3
    np.testing.assert_array_equal(gb[64:80, :3], means[64:80])


def gpu_lbvh(ctx, dev, boxes):
    n = boxes.shape[0]
    b = T(boxes.astype(np.float32), dev)
    keys = torch.empty(n, dtype=torch.int32, device=dev)
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    left = torch.empty(max(n - 1, 1), dtype=torch.int32, device=dev)
    right = torch.empty(max(n - 1, 1), dtype=torch.int32, device=dev)
    nb = torch.empty(max(n - 1, 1) * 6, device=dev)
    ctx.call("gvc_debug_lbvh", n, gvc_native.ptr(b), gvc_native.ptr(keys), gvc_native.ptr(perm),
             gvc_native.ptr(left), gvc_native.ptr(right), gvc_native.ptr(nb), stream())
    torch.cuda.synchronize()
    return (keys.cpu().numpy().view(np.uint32), perm.cpu().numpy(), left.cpu().numpy()[:n - 1],
            right.cpu().numpy()[:n - 1], nb.cpu().numpy().reshape(-1, 6)[:n - 1])


# 4096 keys per radix-sort tile: 300k keys are one wave of tiles; 2.5M keys (611 tiles) are
# more than the 592 blocks resident at once, so later tiles look back over finished ones
@pytest.mark.parametrize("n,kind", [(1, "rand"), (2, "rand"), (3, "rand"), (33, "rand"), (1000, "rand"),
                                    (4097, "dup"), (20000, "same"), (300000, "rand"), (300000, "dup"),
                                    (2500000, "dup")])
def test_lbvh_bit_exact(ctx, cuda, orc, n, kind):
    rng = np.random.default_rng(n)
    c = rng.random((n, 3)).astype(np.float32)
    if kind == "dup":
        c = (np.round(c * 16) / 16).astype(np.float32)
    if kind == "same":
        c[:] = 0.25
    e = (rng.random((n, 3)) * 0.01).astype(np.float32)
    boxes = np.concatenate([c - e, c + e], 1).astype(np.float32)
    ref = orc.lbvh_build(boxes)
    got = gpu_lbvh(ctx, cuda, boxes)
    for name, a, b in zip(("keys", "perm", "left", "right", "node_boxes"), got, ref):
        np.testing.assert_array_equal(a, b, err_msg=name)


@pytest.mark.parametrize("S", [100003, 5000001])
def test_sample_order_bit_exact(cuda, orc, S):
    from bvh_diff_gaussian_rasterization import _C
    rng = np.random.default_rng(11)
    pts = rng.random((S, 3)).astype(np.float32)
    pts[:S // 100] = np.round(pts[:S // 100] * 4) / 4  # duplicate keys
    _C.build_bvh(T(pts, cuda), False, False)
    perm = torch.empty(S, dtype=torch.int32, device=cuda)
    keys = torch.empty(S, dtype=torch.int32, device=cuda)
    _C.context().call("gvc_debug_sample_order", gvc_native.ptr(perm), gvc_native.ptr(keys), stream())
    torch.cuda.synchronize()
    _, skeys, sperm = orc.morton30_points(pts)
    np.testing.assert_array_equal(keys.cpu().numpy().view(np.uint32), skeys)
    np.testing.assert_array_equal(perm.cpu().numpy(), sperm)


def run_forward(dev, means, scales, rots, values, weights, samples, use_gaussian_bvh=False):
    from bvh_diff_gaussian_rasterization import _C
    _C.build_bvh(T(samples, dev), False, use_gaussian_bvh)
    out, outw, conics = _C.rasterize_gaussians(T(means, dev), T(scales, dev), T(rots, dev), T(values, dev),
                                               T(weights, dev), 1.0, 0, 0, 0, 1, 1, 1, -1.0, use_gaussian_bvh,
                                               False)
    _C.check_status()
    return out, outw, conics


# A pair whose power lies within rounding of the -14 floor (forward.cu:235) may be kept by
# one side and dropped by the other; its contribution is w e^-14 <= 8.4e-7.  Every sample
# is allowed two such pairs: |dW| <= rtol W + 2e-6 and |d out| <= atol + 2e-6 / W.
FLOOR_PAIR = 2e-6


def compare_forward(out, outw, ref_out, ref_w, atol_out, rtol_w):
    near = np.abs(ref_w - 0.01) <= 1e-5 * 0.01 + FLOOR_PAIR
    ok = ~near
    vo, vr = out[ok] != -1, ref_out[ok] != -1
    assert np.array_equal(vo, vr)
    both = ok.copy()
    both[ok] = vo
    W = ref_w[both]
    err_o = (np.abs(out[both] - ref_out[both]) - FLOOR_PAIR / W).max(initial=0)
    err_w = ((np.abs(outw[both] - W) - FLOOR_PAIR) / W).max(initial=0)
    assert err_o <= atol_out, err_o
    assert err_w <= rtol_w, err_w
    return err_o, err_w


@pytest.fixture(scope="module")
def small_case(cuda, orc):
    means, scales, rots, values, weights = orc.mixture_small(seed=0, P=4096)
    samples = orc.grid_centres(64)
    return means, scales, rots, values, weights, samples


@pytest.mark.parametrize("use_gaussian_bvh", [False, True])
def test_forward_matches_oracle(ctx, cuda, orc, small_case, use_gaussian_bvh):
    means, scales, rots, values, weights, samples = small_case
    out, outw, conics = run_forward(cuda, means, scales, rots, values, weights, samples, use_gaussian_bvh)
    out, outw = out.cpu().numpy(), outw.cpu().numpy()
    gc = conics.cpu().numpy().reshape(-1, 6)
    _, gb = gpu_preprocess(ctx, cuda, means, scales, rots, weights)
    ref_o, ref_w = orc.forward(means, values, weights, gc.astype(np.float64), gb, samples)
    compare_forward(out, outw, ref_o, ref_w, 2e-5, 2e-5)
    # against the full FP64 pipeline (FP64 conics)
    _, c64, bb = orc.preprocess(means, scales, rots, weights)
    t_o, t_w = orc.forward(means, values, weights, c64, bb, samples)
    compare_forward(out, outw, t_o, t_w, 1e-4, 1e-4)
    assert (out != -1).mean() > 0.5


def test_forward_is_deterministic(cuda, orc, small_case):
    a = run_forward(cuda, *small_case)
    b = run_forward(cuda, *small_case)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def run_backward(dev, case, gout, gw, mode="auto", use_gaussian_bvh=False, cov="true"):
    from bvh_diff_gaussian_rasterization import _C
    means, scales, rots, values, weights, samples = case
    out, outw, conics = run_forward(dev, means, scales, rots, values, weights, samples, use_gaussian_bvh)
    _C.set_backward_mode(mode)
    _C.set_cov_grad_mode(cov)
    try:
        g = _C.rasterize_gaussians_backward(T(means, dev), T(scales, dev), T(rots, dev), conics, T(values, dev),
                                            T(weights, dev), out, outw, 1.0, 0, 0, 0, 1, 1, 1, -1.0,
                                            T(gout, dev), T(gw, dev), use_gaussian_bvh, False)
        _C.check_status()
    finally:
        _C.set_backward_mode("auto")
        _C.set_cov_grad_mode("true")
    return [x.cpu().numpy() for x in g], out.cpu().numpy(), outw.cpu().numpy(), conics.cpu().numpy().reshape(-1, 6)


def oracle_backward(orc, case, out, outw, conics, gout, gw, ref_compat=False):
    means, scales, rots, values, weights, samples = case
    _, bb, = orc.preprocess(means, scales, rots, weights)[::2]
    g = orc.backward(means, values, weights, conics.astype(np.float64), bb, samples, out, outw, gout, gw)
    ds, dq = orc.cov_backward(scales, rots, conics, g["dconics"], ref_compat=ref_compat)
    return [g["dmeans"], ds, dq, g["dvalues"].reshape(-1, 1), g["dweights"].reshape(-1, 1)]


def assert_grads_close(got, ref, tol=1e-4, cov_tol=5e-4):
    for k, name in enumerate(("means", "scales", "rots", "values", "weights")):
        scale = np.abs(ref[k]).max()
        t = cov_tol if name in ("scales", "rots") else tol
        err = np.abs(got[k] - ref[k]).max()
        assert err <= t * scale, (name, err, scale)


@pytest.mark.parametrize("mode,use_gaussian_bvh", [("auto", False), ("auto", True), ("deterministic", True),
                                                   ("atomic", False)])
def test_backward_matches_oracle(cuda, orc, small_case, mode, use_gaussian_bvh):
    S = small_case[-1].shape[0]
    rng = np.random.default_rng(21)
    gout = rng.normal(size=S).astype(np.float32)
    gw = rng.normal(size=S).astype(np.float32)
    got, out, outw, conics = run_backward(cuda, small_case, gout, gw, mode, use_gaussian_bvh)
    ref = oracle_backward(orc, small_case, out, outw, conics, gout, gw)
    assert_grads_close(got, ref)


def test_backward_ref_compat(cuda, orc, small_case):
    S = small_case[-1].shape[0]
    rng = np.random.default_rng(22)
    gout = rng.normal(size=S).astype(np.float32)
    gw = np.zeros(S, np.float32)
    got, out, outw, conics = run_backward(cuda, small_case, gout, gw, cov="ref_compat")
    ref = oracle_backward(orc, small_case, out, outw, conics, gout, gw, ref_compat=True)
    assert_grads_close(got, ref)


def test_deterministic_backward_is_bitwise_reproducible(cuda, small_case):
    S = small_case[-1].shape[0]
    gout = np.random.default_rng(3).normal(size=S).astype(np.float32)
    gw = np.zeros(S, np.float32)
    a, *_ = run_backward(cuda, small_case, gout, gw, "deterministic")
    b, *_ = run_backward(cuda, small_case, gout, gw, "deterministic")
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_backward_reuse_matches_rebuild(cuda, small_case):
    """A backward handed the very arrays of the last forward reuses that forward's AABBs,
    LBVH-ordered records and (FP32 forward) its (out, W) per sorted sample; handed copies,
    it rebuilds the first two and gathers the outputs from the caller's order.  Both
    routes give the same gradients bit for bit (deterministic backward, nonzero dL/dW)."""
    from bvh_diff_gaussian_rasterization import _C
    means, scales, rots, values, weights, samples = small_case
    S = samples.shape[0]
    rng = np.random.default_rng(11)
    gout = T(rng.normal(size=S).astype(np.float32), cuda)
    gw = T(rng.normal(size=S).astype(np.float32), cuda)
    params = [T(a, cuda) for a in (means, scales, rots, values, weights)]
    _C.build_bvh(T(samples, cuda), False, False)
    out, outw, conics = _C.rasterize_gaussians(*params, 1.0, 0, 0, 0, 1, 1, 1, -1.0, False, False)

    def bwd(p, cn, o, ow):
        m, s_, r, v, w = p
        return _C.rasterize_gaussians_backward(m, s_, r, cn, v, w, o, ow, 1.0, 0, 0, 0, 1, 1, 1, -1.0, gout, gw,
                                               False, False)

    for mode in ("deterministic", "tensor_core"):
        _C.set_backward_mode(mode)
        try:
            a = bwd(params, conics, out, outw)
            b = bwd([x.clone() for x in params], conics.clone(), out.clone(), outw.clone())
            c = bwd(params, conics, out, outw)  # after the rebuild: records of the copies, same values
            _C.check_status()
        finally:
            _C.set_backward_mode("auto")
        assert any(bool(x.abs().max() > 0) for x in a)
        for x, y, z in zip(a, b, c):
            if mode == "deterministic":
                assert torch.equal(x, y) and torch.equal(x, z)
            else:  # FP32 atomics in varying order
                tol = 1e-5 * float(x.abs().max())
                assert float((x - y).abs().max()) <= tol and float((x - z).abs().max()) <= tol


def _raw_params(kind):
    """Pre-activation parameters: 'small' (512 Gaussians on a 24^3 grid) or 'config1'
    (4096 Gaussians, means U[0,1]^3, log-scales N(log 0.02, 0.3), random quaternions,
    weights sigmoid(N(0,1)), values U[0,1] through the sigmoid getter, 64^3 cell centres,
    seed 0)."""
    rng = np.random.default_rng(0)
    if kind == "small":
        P, n = 512, 24
        xyz = rng.random((P, 3))
        raw_s = rng.normal(np.log(0.04), 0.3, (P, 3))
        raw_q = rng.normal(size=(P, 4))
        raw_w = rng.normal(size=(P, 1))
        raw_v = rng.normal(size=(P, 1))
    else:
        P, n = 4096, 64
        xyz = rng.random((P, 3))
        raw_s = rng.normal(np.log(0.02), 0.3, (P, 3))
        raw_q = rng.normal(size=(P, 4))
        raw_w = rng.normal(size=(P, 1))
        u = rng.uniform(0.01, 0.99, (P, 1))
        raw_v = np.log(u / (1 - u))
    return rng, n, (xyz, raw_s, raw_q, raw_w, raw_v)


@pytest.mark.parametrize("kind,bwd_mode", [("small", "auto"), ("small", "tensor_core"), ("config1", "auto"),
                                           ("config1", "tensor_core")])
def test_gradients_match_finite_differences(cuda, orc, kind, bwd_mode):
    """Full chain: pre-activation params -> activations (torch) -> GaussianRasterizer
    (GPU forward + adjoint, the deterministic FP32 backward or the tensor-core backward the
    benchmark times) -> masked L1; FD in FP64 over the frozen pair set (h = 1e-4, 64
    random parameters): |an - fd| <= 1e-3 max(|fd|, 1e-3)."""
    import bvh_diff_gaussian_rasterization as R
    from bvh_diff_gaussian_rasterization import _C
    rng, n, raw = _raw_params(kind)
    xyz, raw_s, raw_q, raw_w, raw_v = raw
    samples = orc.grid_centres(n)
    gt = orc.blob_target(samples)
    m32, s32, q32, w32, v32 = [np.asarray(a, np.float32) for a in orc.activations(xyz, raw_s, raw_q, raw_w, raw_v)]
    _, c64, bb = orc.preprocess(m32, s32, q32, w32)
    out64, outw64 = orc.forward(m32, v32, w32, c64, bb, samples)
    ps, pg = orc.pair_list(m32, c64, bb, samples, outw=outw64)
    mask = (out64 != -1)
    S = samples.shape[0]
    gsel = np.where(mask, np.sign(out64 - gt) / mask.sum(), 0.0)
    # GPU analytic gradient through the autograd Function
    settings = R.GaussianRasterizationSettings((0, 0, 0), (1, 1, 1), n, -1.0, 1.0, False, False)
    rast = R.GaussianRasterizer(settings)
    rast.build_bvh(T(samples, cuda))
    leaves = [torch.tensor(a, dtype=torch.float32, device=cuda, requires_grad=True) for a in raw]
    m, s, q, w, v = orc.activations(*leaves, xp=torch)
    _C.set_backward_mode(bwd_mode)
    try:
        cells, weights = rast(m, s, q, v, w)
        torch.autograd.backward(cells, torch.tensor(gsel, dtype=torch.float32, device=cuda))
        _C.check_status()
    finally:
        _C.set_backward_mode("auto")
    # FP64 FD over the frozen pairs
    ts = torch.tensor(samples, dtype=torch.float64)
    tmask = torch.tensor(mask)
    tg = torch.tensor(gsel)

    def loss(params):
        mm, ss, qq, ww, vv = orc.activations(*params, xp=torch)
        W, V = orc.torch_forward_pairs(ps, pg, ts, mm, ss, qq, vv, ww, S=S)
        o = V / torch.where(W > 0, W, torch.ones_like(W))
        return (torch.where(tmask, o, torch.zeros_like(o)) * tg).sum()

    base = [torch.tensor(a, dtype=torch.float64) for a in raw]
    live = np.unique(pg[mask[ps]])
    h = 1e-4
    for _ in range(64):
        t = int(rng.integers(0, 5))
        i = int(rng.choice(live))
        j = int(rng.integers(0, base[t].shape[1]))
        p1 = [b.clone() for b in base]
        p2 = [b.clone() for b in base]
        p1[t][i, j] += h
        p2[t][i, j] -= h
        fd = (loss(p1) - loss(p2)).item() / (2 * h)
        an = leaves[t].grad[i, j].item()
        assert abs(an - fd) <= 1e-3 * max(abs(fd), 1e-3), (t, i, j, an, fd)


def test_edge_cases(cuda, orc):
    from bvh_diff_gaussian_rasterization import _C
    means, scales, rots, values, weights = orc.mixture_small(seed=5, P=7)
    # S = 0
    _C.build_bvh(torch.zeros(0, 3, device=cuda), False, False)
    out, outw, con = _C.rasterize_gaussians(T(means, cuda), T(scales, cuda), T(rots, cuda), T(values, cuda),
                                            T(weights, cuda), 1.0, 0, 0, 0, 1, 1, 1, -1.0, False, False)
    assert out.numel() == 0 and con.numel() == 42
    g = _C.rasterize_gaussians_backward(T(means, cuda), T(scales, cuda), T(rots, cuda), con, T(values, cuda),
                                        T(weights, cuda), out, outw, 1.0, 0, 0, 0, 1, 1, 1, -1.0, out, outw,
                                        False, False)
    assert all(float(x.abs().sum()) == 0.0 for x in g)
    # P = 0: zeros (rasterize_points.cu:51)
    pts = np.random.default_rng(1).random((50, 3)).astype(np.float32)
    _C.build_bvh(T(pts, cuda), False, False)
    z = torch.zeros(0, 3, device=cuda)
    out, outw, con = _C.rasterize_gaussians(z, z, torch.zeros(0, 4, device=cuda), torch.zeros(0, device=cuda),
                                            torch.zeros(0, device=cuda), 1.0, 0, 0, 0, 1, 1, 1, -1.0, False, False)
    assert float(out.abs().sum()) == 0 and out.numel() == 50
    # P = 1, S = 1 and a partial tile (S = 33); samples exactly at the mean
    for S in (1, 33):
        m1 = means[:1]
        smp = np.repeat(m1, S, 0).astype(np.float32)
        smp[1:] += np.random.default_rng(S).normal(0, 0.01, (S - 1, 3)).astype(np.float32)
        o, ow, c = run_forward(cuda, m1, scales[:1], rots[:1], values[:1], weights[:1], smp)
        _, c64, bb = orc.preprocess(m1, scales[:1], rots[:1], weights[:1])
        ro, rw = orc.forward(m1, values[:1], weights[:1], c.cpu().numpy().reshape(-1, 6).astype(np.float64), bb, smp)
        np.testing.assert_allclose(ow.cpu().numpy(), rw, rtol=2e-5, atol=1e-7)
    # every sample outside every box
    o, ow, _ = run_forward(cuda, means, scales, rots, values, weights, pts + 5.0)
    assert bool((o == -1).all()) and bool((ow == 0).all())
    # debug mode synchronises, prints timings and checks the status word
    _C.build_bvh(T(pts, cuda), True, False)
    _C.rasterize_gaussians(T(means, cuda), T(scales, cuda), T(rots, cuda), T(values, cuda), T(weights, cuda),
                           1.0, 0, 0, 0, 1, 1, 1, -1.0, False, True)


def test_large_clustered_properties(cuda, orc):
    """A scaled config-4 workload (clustered means, half the samples near means): no
    traversal overflow, deterministic forward, subsets against the oracle, and the two
    backward modes agree."""
    from bvh_diff_gaussian_rasterization import _C
    means, scales, rots, values, weights, samples = orc.mixture_large(seed=1, P=200_000, S=2_000_000)
    case = (means, scales, rots, values, weights, samples)
    _C.set_count_pairs(True)
    try:
        out, outw, conics = run_forward(cuda, *case)
        st = _C.stats()
    finally:
        _C.set_count_pairs(False)
    assert st["max_stack_fwd"] < 1024 - 128 and st["fwd_contributing"] > 0
    out2, outw2, _ = run_forward(cuda, *case)
    assert torch.equal(out, out2) and torch.equal(outw, outw2)
    out, outw = out.cpu().numpy(), outw.cpu().numpy()
    gc = conics.cpu().numpy().reshape(-1, 6)
    _, gb = gpu_preprocess(gvc_native.Context(), cuda, means, scales, rots, weights)
    sub = np.random.default_rng(2).choice(samples.shape[0], 20000, replace=False)
    ro, rw = orc.forward(means, values, weights, gc.astype(np.float64), gb, samples[sub])
    compare_forward(out[sub], outw[sub], ro, rw, 2e-5, 2e-5)
    S = samples.shape[0]
    gout = np.random.default_rng(4).normal(size=S).astype(np.float32)
    gw = np.zeros(S, np.float32)
    a, *_ = run_backward(cuda, case, gout, gw, "deterministic")
    b, *_ = run_backward(cuda, case, gout, gw, "atomic")
    assert_grads_close(b, a, tol=1e-4, cov_tol=1e-3)


@pytest.mark.parametrize("path", ["plain", "tensor_core", "plain_tile"])
def test_power_window_at_minus_14(cuda, orc, path):
    """Pairs just inside (-13.98) and just outside (-14.02) the power floor of
    forward.cu:235, inside the pair's box: only the first adds w e^p to W."""
    from bvh_diff_gaussian_rasterization import _C
    from test_oracle import window_case, window_points
    case = window_case()
    means, scales, rots, values, weights = case
    x, powers, _, _ = window_points(orc, case)
    _C.set_eval_path(path)
    try:
        out, outw, conics = run_forward(cuda, means, scales, rots, values, weights, x)
    finally:
        _C.set_eval_path("plain")
    outw = outw.cpu().numpy().astype(np.float64)
    gc = conics.cpu().numpy().reshape(-1, 6).astype(np.float64)
    _, gb = gpu_preprocess(gvc_native.Context(), cuda, means, scales, rots, weights)
    _, w_wide = orc.forward(means[1:], values[1:], weights[1:], gc[1:], gb[1:], x)
    pair = outw - w_wide
    expect = np.where(powers >= -14.0, 0.9 * np.exp(powers), 0.0)
    assert np.all(outw > 0.01)
    np.testing.assert_allclose(pair, expect, rtol=1e-3, atol=1e-7)


@pytest.mark.parametrize("path", ["plain", "tensor_core", "plain_tile"])
def test_weight_cutoff_known_answer(cuda, orc, path):
    """One isotropic Gaussian sampled at its mean: W = w just above the 0.01 cutoff gives
    out = v, outw = w; just below gives out = -1, outw = 0 (config.h:9,
    forward.cu:250-256)."""
    from bvh_diff_gaussian_rasterization import _C
    m = np.array([[0.5, 0.5, 0.5]], np.float32)
    s = np.array([[0.05, 0.05, 0.05]], np.float32)
    q = np.array([[1, 0, 0, 0]], np.float32)
    v = np.array([0.3], np.float32)
    x = np.repeat(m, 33, 0)  # a partial tile of samples all at the mean
    _C.set_eval_path(path)
    try:
        for w, expect in ((0.0101, 0.3), (0.0099, -1.0)):
            out, outw, _ = run_forward(cuda, m, s, q, v, np.array([w], np.float32), x)
            out, outw = out.cpu().numpy(), outw.cpu().numpy()
            np.testing.assert_allclose(out, expect, rtol=1e-6)
            np.testing.assert_allclose(outw, w if expect > 0 else 0.0, rtol=1e-6)
    finally:
        _C.set_eval_path("plain")
