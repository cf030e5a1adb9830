"""CPU checks of the oracle: known answers, the reference's quirks, gradients (FP64
autograd and central finite differences) and the LBVH specification."""
import numpy as np
import pytest


def one_gaussian(mu=(0.5, 0.5, 0.5), s=(0.05, 0.05, 0.05), q=(1, 0, 0, 0), w=0.8, v=0.3):
    return (np.array([mu], np.float32), np.array([s], np.float32), np.array([q], np.float32),
            np.array([v], np.float32), np.array([w], np.float32))


def test_isotropic_known_answer(orc):
    m, s, q, v, w = one_gaussian()
    c32, c64, bb = orc.preprocess(m, s, q, w)
    # conic of an isotropic Gaussian: (1 + 1e-5)^-1 / s^2 on the diagonal
    np.testing.assert_allclose(c64[0], [1 / (0.0025 * (1 + 1e-5)), 0, 0, 1 / (0.0025 * (1 + 1e-5)), 0,
                                        1 / (0.0025 * (1 + 1e-5))], rtol=1e-6)
    # box half-extent m * s with m = sqrt(-2 ln(1e-3 / w))
    mh = np.sqrt(-2 * np.log(1e-3 / 0.8)) * 0.05
    np.testing.assert_allclose(bb[0], [0.5 - mh] * 3 + [0.5 + mh] * 3, rtol=1e-6)
    x = np.array([[0.5, 0.5, 0.5], [0.55, 0.5, 0.5], [0.5 + 1.01 * mh, 0.5, 0.5]], np.float32)
    out, outw = orc.forward(m, v, w, c64, bb, x)
    assert out[0] == pytest.approx(0.3, rel=1e-7) and outw[0] == pytest.approx(0.8, rel=1e-7)
    e = 0.8 * np.exp(-0.5 * 0.05 ** 2 * c64[0, 0])
    assert outw[1] == pytest.approx(e, rel=1e-6) and out[1] == pytest.approx(0.3, rel=1e-6)
    assert out[2] == -1.0 and outw[2] == 0.0  # outside the box: no contribution


def test_weight_cutoff(orc):
    for w, expect in [(0.0101, 0.3), (0.0099, -1.0)]:
        m, s, q, v, wt = one_gaussian(w=w)
        c32, c64, bb = orc.preprocess(m, s, q, wt)
        out, outw = orc.forward(m, v, wt, c64, bb, m.copy())
        assert out[0] == pytest.approx(expect, rel=1e-6)
        assert outw[0] == (pytest.approx(w, rel=1e-6) if expect > 0 else 0.0)


def test_tiny_weight_collapses_box(orc):
    m, s, q, v, w = one_gaussian(w=5e-4)
    _, _, bb = orc.preprocess(m, s, q, w)
    np.testing.assert_array_equal(bb[0], [0.5] * 6)  # NaN corners are ignored by fminf/fmaxf


def test_empty_inputs(orc):
    m = np.zeros((0, 3), np.float32)
    out, outw = orc.forward(m, np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros((0, 6)),
                            np.zeros((0, 6), np.float32), np.random.rand(5, 3).astype(np.float32))
    np.testing.assert_array_equal(out, 0.0)  # rasterize_points.cu:51: P == 0 returns zeros
    np.testing.assert_array_equal(outw, 0.0)
    mm, s, q, v, w = one_gaussian()
    _, c64, bb = orc.preprocess(mm, s, q, w)
    out, outw = orc.forward(mm, v, w, c64, bb, np.zeros((0, 3), np.float32))
    assert out.shape == (0,)


def test_box_uses_transposed_rotation(orc):
    rng = np.random.default_rng(3)
    q = rng.normal(size=(1, 4)).astype(np.float32)
    q /= np.linalg.norm(q)
    s = np.array([[0.05, 0.01, 0.02]], np.float32)
    m = np.array([[0.5, 0.5, 0.5]], np.float32)
    w = np.array([0.7], np.float32)
    _, _, bb = orc.preprocess(m, s, q, w)
    r, x, y, z = q[0].astype(np.float64)
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - r * z), 2 * (x * z + r * y)],
                  [2 * (x * y + r * z), 1 - 2 * (x * x + z * z), 2 * (y * z - r * x)],
                  [2 * (x * z - r * y), 2 * (y * z + r * x), 1 - 2 * (x * x + y * y)]])
    mh = np.sqrt(-2 * np.log(1e-3 / 0.7))
    half_rows = (np.abs(R) * (s[0] * mh)[:, None]).sum(0)   # corners along rows of R (quirk)
    half_cols = (np.abs(R) * (s[0] * mh)[None, :]).sum(1)   # corners along columns (principal axes)
    np.testing.assert_allclose(bb[0, 3:] - 0.5, half_rows, rtol=1e-5)
    assert not np.allclose(half_rows, half_cols, rtol=1e-3)


def test_conic_fp64_threshold(orc):
    # an elongated Gaussian (condition ~ 1e4) is inverted in FP64 and rounded once
    m, s, q, v, w = one_gaussian(s=(0.05, 0.0005, 0.02), q=(0.9, 0.1, 0.3, 0.2))
    q = q / np.linalg.norm(q)
    c32, c64, _ = orc.preprocess(m, s, q.astype(np.float32), w)
    np.testing.assert_array_equal(c32, c64.astype(np.float32))


def _frozen_chain(orc, P=256, n=20, seed=0):
    import torch
    torch.set_default_dtype(torch.float64)
    means, scales, rots, values, weights = orc.mixture_small(seed=seed, P=P)
    samples = orc.grid_centres(n)
    c32, c64, bb = orc.preprocess(means, scales, rots, weights)
    out, outw = orc.forward(means, values, weights, c64, bb, samples)
    ps, pg = orc.pair_list(means, c64, bb, samples, outw=outw)
    return means, scales, rots, values, weights, samples, c32, c64, bb, out, outw, ps, pg


def test_backward_matches_autograd(orc):
    """FP64: per-pair adjoint + true covariance adjoint == autograd of the frozen-pair forward."""
    import torch
    means, scales, rots, values, weights, samples, c32, c64, bb, out, outw, ps, pg = _frozen_chain(orc)
    S = samples.shape[0]
    rng = np.random.default_rng(5)
    gout = rng.normal(size=S).astype(np.float32)
    gw = rng.normal(size=S).astype(np.float32)
    T = lambda a: torch.tensor(np.asarray(a, np.float64), requires_grad=True)
    tm, ts, tq, tv, tw = T(means), T(scales), T(rots), T(values), T(weights)
    W, V = orc.torch_forward_pairs(ps, pg, torch.tensor(samples, dtype=torch.float64), tm, ts, tq, tv, tw, S=S)
    mask = W > 0.01
    o = torch.where(mask, V / torch.where(mask, W, torch.ones_like(W)), -torch.ones_like(W))
    ow = torch.where(mask, W, torch.zeros_like(W))
    L = (torch.tensor(gout, dtype=torch.float64) * o).sum() + (torch.tensor(gw, dtype=torch.float64) * ow).sum()
    L.backward()
    g = orc.backward(means, values, weights, c64, bb, samples, out.astype(np.float32), outw.astype(np.float32),
                     gout, gw)
    ds, dq = orc.cov_backward(scales, rots, c64.astype(np.float32), g["dconics"])
    for name, ours, ref in [("means", g["dmeans"], tm.grad), ("values", g["dvalues"], tv.grad),
                            ("weights", g["dweights"], tw.grad), ("scales", ds, ts.grad), ("rots", dq, tq.grad)]:
        ref = ref.numpy().reshape(ours.shape)
        scale = np.abs(ref).max()
        # out/outw enter the adjoint as float32 (as the saved forward outputs do)
        assert np.abs(ours - ref).max() <= 2e-5 * scale, name


def test_ref_compat_differs_only_in_covariance(orc):
    means, scales, rots, values, weights, samples, c32, c64, bb, out, outw, ps, pg = _frozen_chain(orc, P=512, n=20)
    g = orc.backward(means, values, weights, c64, bb, samples, out.astype(np.float32), outw.astype(np.float32),
                     np.ones(samples.shape[0], np.float32), np.zeros(samples.shape[0], np.float32))
    ds_t, dq_t = orc.cov_backward(scales, rots, c32, g["dconics"], ref_compat=False)
    ds_r, dq_r = orc.cov_backward(scales, rots, c32, g["dconics"], ref_compat=True)
    live = np.abs(g["dconics"]).sum(1) > 0
    assert live.sum() > 10
    # the reference's closed form is not the gradient of its forward (backward.cu:75-79, :105, :114-116)
    assert np.abs(ds_t[live] - ds_r[live]).max() > 1e-3 * np.abs(ds_t[live]).max()


def test_finite_differences_full_chain(orc):
    """Config-1 style: 64 random pre-activation parameters, FP64 central differences
    (h = 1e-4) of the masked L1 loss against the analytic chain (oracle adjoint +
    autograd through the activations)."""
    import torch
    torch.set_default_dtype(torch.float64)
    rng = np.random.default_rng(0)
    P, n = 512, 24
    xyz = rng.random((P, 3))
    raw_s = rng.normal(np.log(0.02 * 2.0), 0.3, (P, 3))
    raw_q = rng.normal(size=(P, 4))
    raw_w = rng.normal(size=(P, 1))
    raw_v = rng.normal(size=(P, 1))
    samples = orc.grid_centres(n)
    gt = orc.blob_target(samples)
    act = orc.activations(xyz, raw_s, raw_q, raw_w, raw_v)
    m32, s32, q32, w32, v32 = [np.asarray(a, np.float32) for a in act]
    _, c64, bb = orc.preprocess(m32, s32, q32, w32)
    out, outw = orc.forward(m32, v32, w32, c64, bb, samples)
    ps, pg = orc.pair_list(m32, c64, bb, samples, outw=outw)
    mask = torch.tensor((out != -1) & (gt != -1))
    S = samples.shape[0]
    ts = torch.tensor(samples, dtype=torch.float64)
    tgt = torch.tensor(gt)

    def loss(params):
        m, s, q, w, v = orc.activations(*params, xp=torch)
        W, V = orc.torch_forward_pairs(ps, pg, ts, m, s, q, v, w, S=S)
        o = V / torch.where(W > 0, W, torch.ones_like(W))
        return torch.abs(o - tgt)[mask].mean()

    base = [torch.tensor(a, dtype=torch.float64) for a in (xyz, raw_s, raw_q, raw_w, raw_v)]
    # analytic: oracle adjoint for the activated params, autograd for the activation chain
    leaves = [b.clone().requires_grad_(True) for b in base]
    m, s, q, w, v = orc.activations(*leaves, xp=torch)
    with torch.no_grad():
        o_sel = torch.tensor(out)
        gout = torch.where(mask, torch.sign(o_sel - tgt) / mask.sum(), torch.zeros_like(o_sel))
    g = orc.backward(m32, v32, w32, c64, bb, samples, out.astype(np.float32), outw.astype(np.float32),
                     gout.numpy().astype(np.float32), np.zeros(S, np.float32))
    ds, dq = orc.cov_backward(s32, q32, c64.astype(np.float32), g["dconics"])
    torch.autograd.backward([m, s, q, w, v], [torch.tensor(g["dmeans"]), torch.tensor(ds), torch.tensor(dq),
                                              torch.tensor(g["dweights"]).reshape(-1, 1),
                                              torch.tensor(g["dvalues"]).reshape(-1, 1)])
    # 64 random parameters among Gaussians that touch at least one masked sample
    live = np.unique(pg[np.isin(ps, np.nonzero(mask.numpy())[0])])
    picks = []
    for _ in range(64):
        t = int(rng.integers(0, 5))
        i = int(rng.choice(live))
        j = int(rng.integers(0, base[t].shape[1]))
        picks.append((t, i, j))
    h = 1e-4
    for t, i, j in picks:
        p1 = [b.clone() for b in base]
        p2 = [b.clone() for b in base]
        p1[t][i, j] += h
        p2[t][i, j] -= h
        fd = (loss(p1) - loss(p2)).item() / (2 * h)
        an = leaves[t].grad[i, j].item()
        assert abs(an - fd) <= 1e-3 * max(abs(fd), 1e-3), (t, i, j, an, fd)


# ------------------------------------------------------------------------------------
# LBVH specification
# ------------------------------------------------------------------------------------
def _random_boxes(n, seed, dup=False):
    rng = np.random.default_rng(seed)
    c = rng.random((n, 3)).astype(np.float32)
    if dup:
        c = np.round(c * 8) / 8
    e = rng.random((n, 3)).astype(np.float32) * 0.02
    return np.concatenate([c - e, c + e], 1).astype(np.float32)


@pytest.mark.parametrize("n,dup", [(2, False), (3, False), (17, False), (1000, False), (5000, True)])
def test_lbvh_is_a_valid_tree(orc, n, dup):
    boxes = _random_boxes(n, n, dup)
    keys, perm, left, right, nb = orc.lbvh_build(boxes)
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    assert sorted(perm.tolist()) == list(range(n))
    # stable: equal keys keep the input order
    eq = np.nonzero(np.diff(keys.astype(np.int64)) == 0)[0]
    assert np.all(perm[eq] < perm[eq + 1])
    leaf_seen = np.zeros(n, int)
    node_seen = np.zeros(n - 1, int)
    for ch in np.concatenate([left, right]).astype(np.int64):
        if ch < 0:
            leaf_seen[ch & 0x7fffffff] += 1
        else:
            node_seen[ch] += 1
    assert np.all(leaf_seen == 1)
    assert node_seen[0] == 0 and np.all(node_seen[1:] == 1)
    sb = boxes[perm]
    for k in range(n - 1):
        for ch in (left[k], right[k]):
            ch = int(ch)
            cb = sb[ch & 0x7fffffff] if ch < 0 else nb[ch]
            assert np.all(nb[k, :3] <= cb[:3]) and np.all(nb[k, 3:] >= cb[3:])


def test_morton_keys_known_answers(orc):
    # corners of the bounds: lo -> 0, hi -> all 30 bits set; x takes bit 0 of each triple
    pts = np.array([[0, 0, 0], [1, 1, 1], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    keys, skeys, perm = orc.morton30_points(pts)
    assert keys.tolist() == [0, (1 << 30) - 1, 0x09249249, 0x09249249 << 1, 0x09249249 << 2]


def window_case():
    """An elongated Gaussian turned 45 degrees about z, whose box (built from the rows of the
    rotation, forward.cu:91-112) reaches far past its ellipsoid, plus a wide isotropic one
    that keeps W above the 0.01 cutoff; points on the first one's minor axis at powers
    -13.98, -14.02 (either side of the -14 floor, forward.cu:235), -10 and -20."""
    c, s = np.cos(np.pi / 8), np.sin(np.pi / 8)
    means = np.array([[0.5, 0.5, 0.5], [0.5, 0.5, 0.5]], np.float32)
    scales = np.array([[0.2, 0.004, 0.004], [0.3, 0.3, 0.3]], np.float32)
    rots = np.array([[c, 0, 0, s], [1, 0, 0, 0]], np.float32)
    weights = np.array([0.9, 0.05], np.float32)
    values = np.array([0.2, 0.7], np.float32)
    return means, scales, rots, values, weights


def window_points(orc, case):
    means, scales, rots, values, weights = case
    _, c64, bb = orc.preprocess(means, scales, rots, weights)
    C = np.array([[c64[0, 0], c64[0, 1], c64[0, 2]], [c64[0, 1], c64[0, 3], c64[0, 4]],
                  [c64[0, 2], c64[0, 4], c64[0, 5]]])
    u = np.linalg.eigh(C)[1][:, -1]  # minor axis of the elongated Gaussian
    powers = np.array([-13.98, -14.02, -10.0, -20.0])
    t = np.sqrt(-2 * powers / (u @ C @ u))
    x = (means[0][None, :].astype(np.float64) + t[:, None] * u[None, :]).astype(np.float32)
    return x, powers, c64, bb


def test_power_window_bounds(orc):
    case = window_case()
    means, scales, rots, values, weights = case
    x, powers, c64, bb = window_points(orc, case)
    assert np.all((x >= bb[0, :3]) & (x <= bb[0, 3:]))  # every point inside the first box
    _, outw = orc.forward(means, values, weights, c64, bb, x)
    _, w_wide = orc.forward(means[1:], values[1:], weights[1:], c64[1:], bb[1:], x)
    pair = outw - w_wide
    d = x.astype(np.float64) - means[0]
    C = np.array([[c64[0, 0], c64[0, 1], c64[0, 2]], [c64[0, 1], c64[0, 3], c64[0, 4]],
                  [c64[0, 2], c64[0, 4], c64[0, 5]]])
    p = -0.5 * np.einsum("ni,ij,nj->n", d, C, d)
    expect = np.where(p >= -14.0, 0.9 * np.exp(p), 0.0)
    np.testing.assert_allclose(pair, expect, rtol=1e-6, atol=1e-11)
    assert pair[0] > 0 and pair[1] == 0 and pair[2] > 0 and pair[3] == 0
