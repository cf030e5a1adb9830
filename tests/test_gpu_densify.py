"""Densify / prune sequence through one module state (scene/gaussian_model.py:727-799,
train.py:551-592): the sample set and its BVH are built once, then the Gaussian count
grows (new Gaussians initialised with distCUDA2 as densify_in_empty does) and shrinks
(prune by weight).  Every stage's forward and backward must match the oracle, so the
context's Gaussian workspace is reused and regrown correctly between calls.
"""
import numpy as np
import pytest
import torch

import gvc_native
from test_gpu_rasterizer import gpu_preprocess

pytestmark = pytest.mark.gpu

FLOOR_PAIR = 2e-6  # two pairs at the -14 power floor may differ (w e^-14 each)


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def forward_backward(dev, params, gout, gw, eval_path, bwd_mode):
    from bvh_diff_gaussian_rasterization import _C
    means, scales, rots, values, weights = params
    _C.set_eval_path(eval_path)
    _C.set_backward_mode(bwd_mode)
    try:
        args = [T(a, dev) for a in (means, scales, rots, values, weights)]
        out, outw, conics = _C.rasterize_gaussians(*args, 1.0, 0, 0, 0, 1, 1, 1, -1.0, False, False)
        g = _C.rasterize_gaussians_backward(args[0], args[1], args[2], conics, args[3], args[4], out, outw, 1.0,
                                            0, 0, 0, 1, 1, 1, -1.0, T(gout, dev), T(gw, dev), False, False)
        _C.check_status()
    finally:
        _C.set_eval_path("plain")
        _C.set_backward_mode("auto")
    return out.cpu().numpy(), outw.cpu().numpy(), conics.cpu().numpy().reshape(-1, 6), [x.cpu().numpy() for x in g]


def check_stage(orc, params, samples, res, gout, gw, tol_fwd, tol_bwd):
    means, scales, rots, values, weights = params
    out, outw, conics, grads = res
    _, gb = gpu_preprocess(gvc_native.Context(), torch.device("cuda:0"), means, scales, rots, weights)
    ref_o, ref_w = orc.forward(means, values, weights, conics.astype(np.float64), gb, samples)
    ok = np.abs(ref_w - 0.01) > tol_fwd * 0.01 + FLOOR_PAIR
    assert np.array_equal(out[ok] != -1, ref_o[ok] != -1)
    both = ok & (ref_o != -1)
    W = ref_w[both]
    assert (np.abs(out[both] - ref_o[both]) - FLOOR_PAIR / W).max(initial=0) <= tol_fwd
    assert ((np.abs(outw[both] - W) - FLOOR_PAIR) / W).max(initial=0) <= tol_fwd
    _, _, bb = orc.preprocess(means, scales, rots, weights)
    g = orc.backward(means, values, weights, conics.astype(np.float64), bb, samples, out, outw, gout, gw)
    ds, dq = orc.cov_backward(scales, rots, conics, g["dconics"])
    ref = [g["dmeans"], ds, dq, g["dvalues"].reshape(-1, 1), g["dweights"].reshape(-1, 1)]
    for k, name in enumerate(("means", "scales", "rots", "values", "weights")):
        scale = np.abs(ref[k]).max()
        t = tol_bwd * (5 if name in ("scales", "rots") else 1)
        err = np.abs(grads[k].reshape(ref[k].shape) - ref[k]).max()
        assert err <= t * scale, (name, err, scale)


@pytest.mark.parametrize("eval_path,bwd_mode,tol_fwd,tol_bwd", [("plain", "auto", 2e-5, 1e-4),
                                                                ("plain", "tensor_core", 2e-5, 1e-4),
                                                                ("tensor_core", "auto", 1e-4, 1e-4)])
def test_densify_prune_sequence(cuda, orc, eval_path, bwd_mode, tol_fwd, tol_bwd):
    from bvh_diff_gaussian_rasterization import _C
    from simple_knn._C import distCUDA2
    rng = np.random.default_rng(5)
    means, scales, rots, values, weights = orc.mixture_small(seed=1, P=4096)
    samples = orc.grid_centres(48)
    S = samples.shape[0]
    gout = rng.normal(size=S).astype(np.float32)
    gw = rng.normal(size=S).astype(np.float32)
    _C.build_bvh(T(samples, cuda), False, False)

    stages = []
    params = [means, scales, rots, values, weights]
    stages.append([a.copy() for a in params])
    # densify_in_empty: 8192 new Gaussians at random points, isotropic scale
    # sqrt(max(0.1 * distCUDA2(all points), 1e-7)), identity rotation, weight 0.01
    new = rng.random((8192, 3), dtype=np.float32)
    allp = torch.cat([T(means, cuda), T(new, cuda)], 0)
    d2 = torch.clamp_min(distCUDA2(allp) * 0.1, 0.0000001)[means.shape[0]:]
    new_s = torch.sqrt(d2)[:, None].repeat(1, 3).cpu().numpy()
    new_q = np.tile(np.array([[1, 0, 0, 0]], np.float32), (8192, 1))
    params = [np.vstack([means, new]), np.vstack([scales, new_s]), np.vstack([rots, new_q]),
              np.concatenate([values, rng.random(8192, dtype=np.float32)]),
              np.concatenate([weights, np.full(8192, 0.01, np.float32)])]
    stages.append([a.copy() for a in params])
    # prune by weight (densify_and_prune: weight < min_weight)
    keep = params[4] >= 0.3
    stages.append([a[keep].copy() for a in params])
    # and grow once more past the first size
    stages.append([np.concatenate([a, a[:5000]]) for a in stages[1]])

    for p in stages:
        res = forward_backward(cuda, p, gout, gw, eval_path, bwd_mode)
        check_stage(orc, p, samples, res, gout, gw, tol_fwd, tol_bwd)
        assert (res[0] != -1).mean() > 0.3
