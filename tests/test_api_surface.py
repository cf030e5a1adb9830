"""Host-side API of the drop-in packages: names, signatures and the reference's error
behaviour for bad arguments (no GPU needed: every case fails before any device work)."""
import inspect

import numpy as np
import pytest
import torch


def test_rasterizer_public_surface():
    import bvh_diff_gaussian_rasterization as m
    for name in ("rasterize_gaussians", "_RasterizeGaussians", "GaussianRasterizationSettings",
                 "GaussianRasterizer", "cpu_deep_copy_tuple"):
        assert hasattr(m, name)
    assert m.GaussianRasterizationSettings._fields == (
        "volume_mins", "volume_maxes", "cell_count", "bg", "scale_modifier", "use_gaussian_bvh", "debug")
    sig = inspect.signature(m.GaussianRasterizer.forward)
    assert list(sig.parameters) == ["self", "means3D", "scales", "rotations", "values", "weights", "debug"]
    sig = inspect.signature(m.GaussianRasterizer.build_bvh)
    assert list(sig.parameters) == ["self", "samples", "force_debug", "use_gaussian_bvh"]
    for op in ("build_bvh", "rasterize_gaussians", "rasterize_gaussians_backward"):
        assert hasattr(m._C, op)
    assert len(inspect.signature(m._C.rasterize_gaussians).parameters) == 15
    assert len(inspect.signature(m._C.rasterize_gaussians_backward).parameters) == 20


def _settings():
    import bvh_diff_gaussian_rasterization as m
    return m.GaussianRasterizationSettings((0, 0, 0), (1, 1, 1), 64, -1.0, 1.0, False, False)


def test_forward_requires_all_parameters():
    import bvh_diff_gaussian_rasterization as m
    r = m.GaussianRasterizer(_settings())
    x = torch.zeros(4, 3)
    with pytest.raises(Exception, match="scale/rotation"):
        r(x, scales=None, rotations=torch.zeros(4, 4), values=torch.zeros(4, 1), weights=torch.zeros(4, 1))
    with pytest.raises(Exception, match="scalar values"):
        r(x, scales=torch.zeros(4, 3), rotations=torch.zeros(4, 4), values=None, weights=torch.zeros(4, 1))
    with pytest.raises(Exception, match="scalar weights"):
        r(x, scales=torch.zeros(4, 3), rotations=torch.zeros(4, 4), values=torch.zeros(4, 1), weights=None)
    with pytest.raises(NameError):
        r.intersect(x, torch.zeros(4, 3), torch.zeros(4, 4))


def test_native_ops_reject_host_tensors():
    import bvh_diff_gaussian_rasterization as m
    with pytest.raises(RuntimeError, match="CUDA"):
        m._C.build_bvh(torch.zeros(8, 3), False, False)
    with pytest.raises(RuntimeError, match="means3D must have dimensions"):
        m._C.rasterize_gaussians(torch.zeros(4, 2), None, None, None, None, 1.0, 0, 0, 0, 1, 1, 1, -1.0,
                                 False, False)
    with pytest.raises(RuntimeError, match="expected scalar type Float"):
        m._C.build_bvh(torch.zeros(8, 3, dtype=torch.float64), False, False)


def test_mesh_sampler_argument_errors():
    from gpu_mesh_sampling import gpu_sample, gpu_sampleu
    dims = np.array([4, 4, 4])
    with pytest.raises(RuntimeError, match="does not match dims"):
        gpu_sample(dims, np.zeros(3), np.ones(3), np.zeros(10), np.zeros((2, 3)))
    with pytest.raises(RuntimeError, match="Unsupported values dtype"):
        gpu_sample(dims, np.zeros(3), np.ones(3), np.zeros(64, np.int32), np.zeros((2, 3)))
    pts = np.random.rand(8, 3).astype(np.float32)
    with pytest.raises(RuntimeError, match="Unsupported VTK cell type: 42"):
        gpu_sampleu(pts, np.arange(4), np.array([42]), np.array([0]), np.zeros(8), np.zeros((1, 3)))
    with pytest.raises(RuntimeError, match="does not match its VTK cell type"):
        gpu_sampleu(pts, np.arange(5), np.array([12]), np.array([0]), np.zeros(8), np.zeros((1, 3)))


def test_mesh_sampler_output_dtypes_without_samples():
    from gpu_mesh_sampling import gpu_sample
    for dt in (np.float64, np.float32, np.uint16, np.uint8):
        out = gpu_sample(np.array([2, 2, 2]), np.zeros(3), np.ones(3), np.zeros(8, dt), np.zeros((0, 3)))
        assert out.dtype == dt and out.shape == (0,)
