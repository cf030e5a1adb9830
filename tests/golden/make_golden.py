"""Generates tests/golden/reference_python.npz by RUNNING the reference's own Python code.

    python tests/golden/make_golden.py [reference_root]

The reference root is the argument, else $GVC_REFERENCE_ROOT.

The reference modules import packages that are absent here (plyfile, pyvista,
simple_knn, the CUDA extensions), so the functions on the hot path's Python side are
extracted from the reference sources with `ast` and executed as written:

  * morton3d_unit          gaussian_renderer/__init__.py:45-58  (Gaussian order in render())
  * part1by2_torch + clamp train.py:292-315                    (sample order in training)
  * GaussianModel._apply_cap scene/gaussian_model.py:71-77      (scale activation cap)

Inputs: seeded random points (with edge cases at 0, 1, above 1 and below 0) and a
1024-Gaussian subset of a trained mixture shipped with the reference
(finals/MITO1024WVEG/point_cloud/iteration_1000/point_cloud.ply, binary little-endian
float32: x y z value weight scale_0..2 rot_0..3, pre-activation).

Only this script reads the reference; the tests read the .npz.
"""
import ast
import os
import sys
import textwrap

import numpy as np
import torch

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GVC_REFERENCE_ROOT", "")
if not os.path.isdir(REF):
    sys.exit("usage: make_golden.py REFERENCE_ROOT (or set GVC_REFERENCE_ROOT)")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_python.npz")


def extract(path, name):
    """Source of the (possibly nested) function `name` in file `path`."""
    src = open(os.path.join(REF, path)).read()
    tree = ast.parse(src)
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name == name:
            return textwrap.dedent(ast.get_source_segment(src, node))
    raise KeyError(name)


def load_ply(path):
    raw = open(os.path.join(REF, path), "rb").read()
    end = raw.index(b"end_header\n") + len(b"end_header\n")
    header = raw[:end].decode()
    n = int([l for l in header.splitlines() if l.startswith("element vertex")][0].split()[-1])
    props = [l.split()[-1] for l in header.splitlines() if l.startswith("property float")]
    arr = np.frombuffer(raw[end:end + 4 * len(props) * n], dtype="<f4").reshape(n, len(props))
    return props, arr


def main():
    ns = {"torch": torch}
    exec(extract("gaussian_renderer/__init__.py", "morton3d_unit"), ns)
    exec(extract("train.py", "part1by2_torch"), ns)
    cap_src = extract("scene/gaussian_model.py", "_apply_cap")
    exec(cap_src, ns)

    class _Self:
        max_scale = 0.02  # scene/gaussian_model.py:68

    rng = np.random.default_rng(1234)
    pts = rng.random((509, 3), dtype=np.float32)
    edge = np.array([[0, 0, 0], [1, 1, 1], [0.5, 0.25, 0.125], [1.0000001, 0.3, 0.7], [1.5, 0.2, 0.9],
                     [-0.25, 0.5, 0.5], [0.999999, 0.999999, 0.999999]], dtype=np.float32)
    pts = np.concatenate([pts, edge]).astype(np.float32)
    t = torch.from_numpy(pts)
    m_render = ns["morton3d_unit"](t).numpy()

    # train.py:306-314: clamp to [0,1], scale by 2^21 - 1, interleave
    scale = (1 << 21) - 1
    q = (torch.clamp(t, 0.0, 1.0) * scale).to(torch.int64)
    p1 = ns["part1by2_torch"]
    m_train = (p1(q[:, 0]) | (p1(q[:, 1]) << 1) | (p1(q[:, 2]) << 2)).numpy()

    props, arr = load_ply("finals/MITO1024WVEG/point_cloud/iteration_1000/point_cloud.ply")
    sel = np.sort(np.random.default_rng(7).choice(arr.shape[0], 1024, replace=False))
    sub = arr[sel].copy()
    col = {p: i for i, p in enumerate(props)}
    xyz = sub[:, [col["x"], col["y"], col["z"]]]
    raw_scale = sub[:, [col["scale_0"], col["scale_1"], col["scale_2"]]]
    raw_rot = sub[:, [col["rot_0"], col["rot_1"], col["rot_2"], col["rot_3"]]]
    raw_w = sub[:, [col["weight"]]]
    raw_v = sub[:, [col["value"]]]
    s_act = ns["_apply_cap"](_Self(), torch.exp(torch.from_numpy(raw_scale))).numpy()   # get_scaling
    q_act = torch.nn.functional.normalize(torch.from_numpy(raw_rot)).numpy()            # get_rotation
    w_act = torch.sigmoid(torch.from_numpy(raw_w)).numpy()                              # get_weight
    v_act = torch.sigmoid(torch.from_numpy(raw_v)).numpy()                              # get_values
    m_ply = ns["morton3d_unit"](torch.from_numpy(xyz)).numpy()

    np.savez_compressed(
        OUT, morton_pts=pts, morton_render=m_render, morton_train=m_train,
        ply_xyz=xyz, ply_raw_scale=raw_scale, ply_raw_rot=raw_rot, ply_raw_weight=raw_w,
        ply_raw_value=raw_v, ply_scale=s_act, ply_rot=q_act, ply_weight=w_act, ply_value=v_act,
        ply_morton=m_ply)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
