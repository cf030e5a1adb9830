"""The reference's own callers, unchanged, on the drop-in packages.

gaussian_renderer/__init__.py (init_rasterizer, build_bvh, render with its Morton argsort
and gathers, :1-97) and scene/gaussian_model.py (GaussianModel: create_from_pcd with
distCUDA2 initial scales, :139-205; training_setup and Adam, :207-247; densify_and_prune
with densify_in_empty and prune_points, :727-799) are imported from the reference tree as
they are; the packages they import (bvh_diff_gaussian_rasterization, simple_knn,
gpu_mesh_sampling) resolve to this repository's drop-ins, which come first on the import
path.  Only pyvista and plyfile, which these code paths import but never call, are
replaced by empty modules.  The loss is the reference's masked L1 (train.py:389-396,
utils/loss_utils.py l1_loss).

The reference tree is located by $GVC_REFERENCE_ROOT or where oracle/build_ref.py found
it; without it these tests skip.

Checks (tolerances as in test_gpu_rasterizer): render's cells against the oracle's
forward of the model's activated parameters; one step's gradients of the raw parameters
against FP64 central finite differences of the restated getters and forward (h = 1e-4,
|an - fd| <= 1e-3 max(|fd|, 1e-3)); a training sequence (Adam steps, densify and prune,
rebuilt LBVHs) stays finite and changes the mixture as the reference's methods say.
"""
import os
import sys
import types
from types import SimpleNamespace

import numpy as np
import pytest
import torch

import refslice

pytestmark = pytest.mark.gpu

ROOT = refslice.reference_root()
HAVE_REF = bool(ROOT) and os.path.isfile(os.path.join(ROOT, "gaussian_renderer", "__init__.py")) and \
    os.path.isfile(os.path.join(ROOT, "scene", "gaussian_model.py"))


@pytest.fixture(scope="module")
def ref(cuda):
    if not HAVE_REF:
        pytest.skip("the reference tree is not present")
    for name, attrs in (("pyvista", ("PolyData", "UnstructuredGrid", "read")), ("plyfile", ("PlyData", "PlyElement"))):
        if name not in sys.modules:
            m = types.ModuleType(name)
            for a in attrs:
                setattr(m, a, object)
            sys.modules[name] = m
    if ROOT not in sys.path:
        sys.path.append(ROOT)  # after the drop-in packages
    import gaussian_renderer
    import bvh_diff_gaussian_rasterization
    import simple_knn._C
    from scene.gaussian_model import GaussianModel
    from utils.graphics_utils import BasicPointCloud
    from utils.loss_utils import l1_loss
    pkg = os.path.dirname(os.path.abspath(bvh_diff_gaussian_rasterization.__file__))
    assert not pkg.startswith(os.path.abspath(ROOT)), "the drop-in must shadow the reference's extension"
    assert "gaussian-volume-compression_b200" in simple_knn._C.__file__
    return SimpleNamespace(GR=gaussian_renderer, GaussianModel=GaussianModel, BasicPointCloud=BasicPointCloud,
                           l1_loss=l1_loss)


OPT = SimpleNamespace(percent_dense=0.01, position_lr_init=0.00016, position_lr_final=0.0000016,
                      position_lr_delay_mult=0.01, position_lr_max_steps=30_000, weight_lr=0.025, scaling_lr=0.001,
                      rotation_lr=0.0001, values_lr=0.0025)  # arguments/__init__.py OptimizationParams defaults


def make_model(ref, volume, P, seed=0):
    import gvc_workloads as wl
    pts, vals = wl.lattice_init(volume, P, seed=seed)
    gm = ref.GaussianModel()
    mesh = SimpleNamespace(bounds=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0))
    # values as [N, 1], as scene/dataset_readers.py:51-53 passes them
    gm.create_from_pcd(ref.BasicPointCloud(points=pts.cpu().numpy(), values=vals.cpu().numpy().reshape(-1, 1)), mesh)
    return gm


def volume_targets(volume, samples):
    from gpu_mesh_sampling import gpu_sample
    n = volume.shape[0]
    return torch.from_numpy(gpu_sample(np.array([n, n, n]), np.zeros(3, np.float32),
                                       np.full(3, 1.0 / (n - 1), np.float32), volume.cpu().numpy().reshape(-1),
                                       samples.cpu().numpy())).to(samples.device)


def activated(gm):
    return [t.detach().cpu().numpy().astype(np.float32) for t in
            (gm.get_xyz, gm.get_scaling, gm.get_rotation, gm.get_values, gm.get_weight)]


def test_render_matches_oracle(ref, cuda, orc):
    import gvc_workloads as wl
    from test_gpu_rasterizer import compare_forward
    volume = wl.volume_blobs_sine(n=64, device=cuda)
    gm = make_model(ref, volume, 20000)
    ref.GR.init_rasterizer(gm, SimpleNamespace(debug=False))
    samples = torch.rand(300000, 3, device=cuda)
    ref.GR.build_bvh(samples)
    out = ref.GR.render(gm)
    cells, weights = out["cells"].detach().cpu().numpy(), out["weights"].detach().cpu().numpy()
    m, s, q, v, w = activated(gm)
    c32, _, bb = orc.preprocess(m, s, q, w.ravel())
    ro, rw = orc.forward(m, v.ravel(), w.ravel(), c32.astype(np.float64), bb, samples.cpu().numpy())
    compare_forward(cells, weights, ro, rw, 2e-5, 2e-5)
    assert (cells != -1).mean() > 0.5


def test_gradients_match_finite_differences(ref, cuda, orc):
    """One step of the reference's loss through its render on a small model: gradients of
    the raw parameters (_xyz, _scaling, _rotation, _weight, _values) against FP64 finite
    differences over the frozen pair set."""
    import gvc_workloads as wl
    volume = wl.volume_blobs_sine(n=24, device=cuda)
    gm = make_model(ref, volume, 400, seed=1)
    ref.GR.init_rasterizer(gm, SimpleNamespace(debug=False))
    samples = orc.grid_centres(24)
    gt = volume_targets(volume, torch.from_numpy(samples).to(cuda)).float()
    ref.GR.build_bvh(torch.from_numpy(samples).to(cuda))
    cells = ref.GR.render(gm)["cells"]
    mask = torch.logical_and(gt != -1, cells != -1)
    loss = ref.l1_loss(cells[mask], gt[mask])
    loss.backward()
    raw = [gm._xyz, gm._scaling, gm._rotation, gm._weight, gm._values]
    base = [t.detach().cpu().double() for t in raw]
    # FP64 forward over the frozen pairs, through the restated getters
    m, s, q, v, w = activated(gm)
    _, c64, bb = orc.preprocess(m, s, q, w.ravel())
    out64, outw64 = orc.forward(m, v.ravel(), w.ravel(), c64, bb, samples)
    ps, pg = orc.pair_list(m, c64, bb, samples, outw=outw64)
    valid = torch.tensor(mask.cpu().numpy())
    ts = torch.tensor(samples, dtype=torch.float64)
    tgt = gt.cpu().double()
    S = samples.shape[0]

    def lossf(params):
        xyz, ls, rq, rw, rv = params
        mm, ss, qq, ww, vv = orc.activations(xyz, ls, rq, rw, rv, xp=torch)
        W, V = orc.torch_forward_pairs(ps, pg, ts, mm, ss, qq, vv, ww, S=S)
        o = V / torch.where(W > 0, W, torch.ones_like(W))
        return torch.abs(o[valid] - tgt[valid]).mean()

    rng = np.random.default_rng(5)
    live = np.unique(pg)
    h = 1e-4
    checked = 0
    for _ in range(48):
        t = int(rng.integers(0, 5))
        i = int(rng.choice(live))
        j = int(rng.integers(0, base[t].shape[1]))
        p1 = [b.clone() for b in base]
        p2 = [b.clone() for b in base]
        p1[t][i, j] += h
        p2[t][i, j] -= h
        fd = (lossf(p1) - lossf(p2)).item() / (2 * h)
        an = raw[t].grad[i, j].item()
        assert abs(an - fd) <= 1e-3 * max(abs(fd), 1e-3), (t, i, j, an, fd)
        checked += 1
    assert checked == 48


def test_training_sequence_with_densify_and_prune(ref, cuda):
    """Adam steps, then densify_and_prune (new Gaussians in empty space with distCUDA2
    scales, low-weight Gaussians pruned), then more steps on the rebuilt mixture."""
    import gvc_workloads as wl
    from bvh_diff_gaussian_rasterization import _C
    volume = wl.volume_blobs_sine(n=64, device=cuda)
    gm = make_model(ref, volume, 20000, seed=2)
    gm.training_setup(OPT)
    ref.GR.init_rasterizer(gm, SimpleNamespace(debug=False))
    losses = []

    def step(it):
        samples = torch.rand(262144, 3, device=cuda)
        gt = volume_targets(volume, samples).float()
        ref.GR.build_bvh(samples)
        gm.update_learning_rate(it)
        cells = ref.GR.render(gm)["cells"]
        mask = torch.logical_and(gt != -1, cells != -1)
        loss = ref.l1_loss(cells[mask], gt[mask])
        loss.backward()
        gm.optimizer.step()
        gm.optimizer.zero_grad(set_to_none=True)
        losses.append(float(loss))

    xyz0 = gm.get_xyz.detach().clone()
    for it in range(1, 6):
        step(it)
    assert not torch.equal(gm.get_xyz.detach(), xyz0)  # Adam moved the means
    P0 = gm.get_xyz.shape[0]
    min_weight = 0.005  # the new Gaussians (weight 0.01, densify_in_empty) survive the prune
    expect = P0 + 2000 - int((gm.get_weight < min_weight).sum())
    empty = torch.rand(2000, 3, device=cuda)
    gm.densify_and_prune(0.0, min_weight, 0.01, empty,
                         volume_targets(volume, empty).float().clamp(0.01, 0.99).reshape(-1, 1))
    assert gm.get_xyz.shape[0] == expect
    for it in range(6, 11):
        step(it)
    _C.check_status()
    assert np.isfinite(losses).all()
    for t in (gm._xyz, gm._scaling, gm._rotation, gm._weight, gm._values):
        assert torch.isfinite(t).all()
