"""Tensor-core (tcgen05) path: the MMA building block through the C ABI, and the forward with
the tensor-core exponent (and the warp-per-tile FP32 kernel) against the oracle; the
default FP32 CTA forward is covered by test_gpu_rasterizer.py.

Tolerances: the GEMM hook is exact on small integers and within 1e-6 (relative to the
row norm) on random BF16 data; the plain CTA forward meets the plain tolerance (2e-5);
the tensor-core forward is checked at 1e-4 (the power is a dot product of ~100-sized
terms accumulated in FP32 on the tensor cores) with the same -14-floor allowance."""
import ctypes

import numpy as np
import pytest
import torch

import gvc_native
from test_gpu_rasterizer import T, compare_forward, gpu_preprocess, run_forward

pytestmark = pytest.mark.gpu


def bf16(a, dev):
    return torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(dev)


@pytest.mark.parametrize("N", [32, 64, 128, 256])
def test_tc_gemm_exact_on_integers(cuda, N):
    rng = np.random.default_rng(N)
    A = rng.integers(-4, 5, (128, 16)).astype(np.float32)
    B = rng.integers(-4, 5, (N, 16)).astype(np.float32)
    ctx = gvc_native.Context()
    dA, dB = bf16(A, cuda), bf16(B, cuda)
    D = torch.empty(128 * N, device=cuda)
    ctx.call("gvc_debug_tc_gemm", gvc_native.ptr(dA), gvc_native.ptr(dB), N, gvc_native.ptr(D),
             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    ctx.sync_status(torch.cuda.current_stream().cuda_stream)
    np.testing.assert_array_equal(D.cpu().numpy().reshape(128, N), A @ B.T)


def test_tc_gemm_random_bf16(cuda):
    rng = np.random.default_rng(5)
    A = rng.normal(size=(128, 16)).astype(np.float32)
    B = rng.normal(size=(64, 16)).astype(np.float32)
    dA, dB = bf16(A, cuda), bf16(B, cuda)
    A64 = dA.float().cpu().numpy().astype(np.float64)
    B64 = dB.float().cpu().numpy().astype(np.float64)
    ctx = gvc_native.Context()
    D = torch.empty(128 * 64, device=cuda)
    ctx.call("gvc_debug_tc_gemm", gvc_native.ptr(dA), gvc_native.ptr(dB), 64, gvc_native.ptr(D),
             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    ctx.sync_status(torch.cuda.current_stream().cuda_stream)
    ref = A64 @ B64.T
    scale = np.abs(A64).sum(1)[:, None] * np.abs(B64).max()
    assert (np.abs(D.cpu().numpy().reshape(128, 64) - ref) / scale).max() <= 1e-6


def run_path(dev, case, path):
    from bvh_diff_gaussian_rasterization import _C
    _C.set_eval_path(path)
    try:
        return run_forward(dev, *case)
    finally:
        _C.set_eval_path("plain")


@pytest.fixture(scope="module")
def case(cuda, orc):
    means, scales, rots, values, weights = orc.mixture_small(seed=0, P=4096)
    return means, scales, rots, values, weights, orc.grid_centres(64)


@pytest.mark.parametrize("path,tol", [("plain_tile", 2e-5), ("tensor_core", 1e-4)])
def test_cta_forward_matches_oracle(cuda, orc, case, path, tol):
    means, scales, rots, values, weights, samples = case
    out, outw, conics = run_path(cuda, case, path)
    out, outw = out.cpu().numpy(), outw.cpu().numpy()
    gc = conics.cpu().numpy().reshape(-1, 6)
    _, gb = gpu_preprocess(gvc_native.Context(), cuda, means, scales, rots, weights)
    ro, rw = orc.forward(means, values, weights, gc.astype(np.float64), gb, samples)
    e_same = compare_forward(out, outw, ro, rw, tol, tol)
    _, c64, bb = orc.preprocess(means, scales, rots, weights)
    to, tw = orc.forward(means, values, weights, c64, bb, samples)
    e64 = compare_forward(out, outw, to, tw, 1e-4, 1e-4)
    print("%s: error vs oracle (same conics) out %.2e outw %.2e; vs FP64 pipeline out %.2e outw %.2e"
          % (path, e_same[0], e_same[1], e64[0], e64[1]))


def test_tensor_core_forward_large_clustered(cuda, orc):
    """Scaled large-evaluation workload: the tensor-core field agrees with the plain one."""
    means, scales, rots, values, weights, samples = orc.mixture_large(seed=3, P=200_000, S=1_000_000)
    case = (means, scales, rots, values, weights, samples)
    a = [x.cpu().numpy() for x in run_path(cuda, case, "plain")[:2]]
    b = [x.cpu().numpy() for x in run_path(cuda, case, "tensor_core")[:2]]
    c = [x.cpu().numpy() for x in run_path(cuda, case, "plain_tile")[:2]]
    for other, tol in ((c, 2e-5), (b, 1e-4)):
        near = np.abs(a[1] - 0.01) <= 1e-6 + 4e-6
        ok = ~near
        assert np.array_equal(a[0][ok] == -1, other[0][ok] == -1)
        v = ok & (a[0] != -1)
        assert ((np.abs(other[1][v] - a[1][v]) - 4e-6) / a[1][v]).max() <= tol
        assert (np.abs(other[0][v] - a[0][v]) - 4e-6 / a[1][v]).max() <= tol


def run_backward_path(dev, case, gout, gw, path, mode="auto"):
    from bvh_diff_gaussian_rasterization import _C
    from test_gpu_rasterizer import run_backward
    _C.set_eval_path(path)
    try:
        return run_backward(dev, case, gout, gw, mode)
    finally:
        _C.set_eval_path("plain")


@pytest.mark.parametrize("gw_scale,path,mode", [(0.0, "tensor_core", "auto"), (1.0, "tensor_core", "auto"),
                                                (1.0, "plain", "tensor_core")])
def test_tensor_core_backward_matches_oracle(cuda, orc, case, gw_scale, path, mode):
    """The tensor-core backward (per-Gaussian reduction over samples as a split-BF16 GEMM
    in tensor memory) against the oracle's FP64 adjoint at the forward's own outputs, on
    the tensor-core path and selected explicitly after the FP32 forward."""
    from test_gpu_rasterizer import assert_grads_close, oracle_backward
    S = case[-1].shape[0]
    rng = np.random.default_rng(31)
    gout = rng.normal(size=S).astype(np.float32)
    gw = (gw_scale * rng.normal(size=S)).astype(np.float32)
    got, out, outw, conics = run_backward_path(cuda, case, gout, gw, path, mode)
    ref = oracle_backward(orc, case, out, outw, conics, gout, gw)
    for k, name in enumerate(("means", "scales", "rots", "values", "weights")):
        print("%s: max err / max |ref| = %.2e" % (name, np.abs(got[k] - ref[k]).max() / np.abs(ref[k]).max()))
    assert_grads_close(got, ref)


@pytest.mark.parametrize("path,mode", [("tensor_core", "auto"), ("plain", "tensor_core"),
                                       ("plain", "deterministic")])
def test_backward_large_clustered_vs_oracle(cuda, orc, path, mode):
    """Scaled large-evaluation workload (200k clustered Gaussians, 1M samples): the
    gradients of 20k random Gaussians against the oracle's FP64 adjoint over all samples
    of the step (with the GPU forward's own outputs), then the covariance adjoint."""
    means, scales, rots, values, weights, samples = orc.mixture_large(seed=4, P=200_000, S=1_000_000)
    case = (means, scales, rots, values, weights, samples)
    rng = np.random.default_rng(32)
    gout = rng.normal(size=samples.shape[0]).astype(np.float32)
    gw = np.zeros(samples.shape[0], np.float32)
    got, out, outw, conics = run_backward_path(cuda, case, gout, gw, path, mode)
    sel = np.sort(rng.choice(means.shape[0], 20000, replace=False))
    _, _, bb = orc.preprocess(means[sel], scales[sel], rots[sel], weights[sel])
    g = orc.backward(means[sel], values[sel], weights[sel], conics[sel].astype(np.float64), bb, samples, out, outw,
                     gout, gw)
    ds, dq = orc.cov_backward(scales[sel], rots[sel], conics[sel], g["dconics"])
    ref = [g["dmeans"], ds, dq, g["dvalues"].reshape(-1, 1), g["dweights"].reshape(-1, 1)]
    for k, name in enumerate(("means", "scales", "rots", "values", "weights")):
        a = got[k].reshape(means.shape[0], -1)[sel]
        err = np.abs(a - ref[k]).max() / np.abs(ref[k]).max()
        print("%s: max err / max |fp64| = %.2e" % (name, err))
        assert err <= (5e-4 if name in ("scales", "rots") else 1e-4), name
