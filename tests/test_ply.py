"""Gaussian PLY files without plyfile (scene/gaussian_model.py:257-383, :801-819).

Pinned by the golden fixture, which holds 1024 raw records that make_golden.py read from
a trained reference point cloud.  Where the reference tree is present, the reader
must also recover that selection from the file itself, and the writer must reproduce the
file byte for byte and its ASCII copy character for character.
"""
import os

import numpy as np
import pytest

import gvc_ply
import refslice

HERE = os.path.dirname(os.path.abspath(__file__))
# the trained point cloud inside the reference tree ($GVC_REFERENCE_ROOT, or where
# oracle/build_ref.py found the reference); tests that need it skip without it
_ROOT = refslice.reference_root()
REF_PLY = os.path.join(_ROOT, "finals", "MITO1024WVEG", "point_cloud", "iteration_1000",
                       "point_cloud.ply") if _ROOT else ""

HEADER = (b"ply\nformat binary_little_endian 1.0\nelement vertex 1024\n" +
          b"".join(b"property float %s\n" % p.encode() for p in
                   ["x", "y", "z", "value", "weight", "scale_0", "scale_1", "scale_2",
                    "rot_0", "rot_1", "rot_2", "rot_3"]) + b"end_header\n")


@pytest.fixture(scope="module")
def golden():
    d = np.load(os.path.join(HERE, "golden", "reference_python.npz"))
    return {"xyz": d["ply_xyz"], "values": d["ply_raw_value"], "weights": d["ply_raw_weight"],
            "scales": d["ply_raw_scale"], "rots": d["ply_raw_rot"]}


def test_write_read_round_trip(tmp_path, golden):
    p = str(tmp_path / "pc" / "point_cloud.ply")
    gvc_ply.write_gaussian_ply(p, golden["xyz"], golden["values"], golden["weights"], golden["scales"],
                               golden["rots"])
    raw = open(p, "rb").read()
    assert raw[:len(HEADER)] == HEADER
    assert len(raw) == len(HEADER) + 1024 * 12 * 4
    for path in (p, p.replace(".ply", "_ascii.ply")):
        back = gvc_ply.read_gaussian_ply(path)
        for k, v in golden.items():
            assert back[k].dtype == np.float32 and back[k].shape == v.shape
            np.testing.assert_array_equal(back[k], v)


def test_ascii_copy_layout(tmp_path, golden):
    p = str(tmp_path / "a.ply")
    gvc_ply.write_gaussian_ply(p, golden["xyz"][:3], golden["values"][:3], golden["weights"][:3],
                               golden["scales"][:3], golden["rots"][:3])
    lines = open(str(tmp_path / "a_ascii.ply")).read().splitlines()
    assert lines[:3] == ["ply", "format ascii 1.0", "element vertex 3"]
    assert lines[15] == "end_header" and len(lines) == 19
    row = np.concatenate([golden[k][0].reshape(-1) for k in ("xyz", "values", "weights", "scales", "rots")])
    assert lines[16] == " ".join(str(np.float32(v)) for v in row)


def test_generic_reader_types_and_orders(tmp_path):
    dt = [("a", "u1"), ("b", "i4"), ("c", "f8"), ("d", "u2")]
    rows = np.array([(1, -2, 0.5, 7), (255, 2 ** 31 - 1, -1e300, 65535)], dtype=dt)
    hdr = ("ply\nformat %s 1.0\ncomment made here\nelement thing 2\nproperty uchar a\nproperty int b\n"
           "property double c\nproperty ushort d\nelement empty 0\nproperty float x\nend_header\n")
    for fmt, order in (("binary_little_endian", "<"), ("binary_big_endian", ">")):
        p = tmp_path / (fmt + ".ply")
        body = rows.astype([(n, order + t) for n, t in dt]).tobytes()
        p.write_bytes((hdr % fmt).encode() + body)
        el = gvc_ply.read_ply(str(p))
        assert len(el["empty"]) == 0
        for n, _ in dt:
            np.testing.assert_array_equal(el["thing"][n], rows[n])
    p = tmp_path / "ascii.ply"
    p.write_text(hdr % "ascii" + "1 -2 0.5 7\n255 2147483647 -1e300 65535\n")
    el = gvc_ply.read_ply(str(p))
    for n, _ in dt:
        np.testing.assert_array_equal(el["thing"][n], rows[n])


def test_reader_errors(tmp_path):
    bad = tmp_path / "bad.ply"
    bad.write_bytes(b"not a ply\n")
    with pytest.raises(ValueError):
        gvc_ply.read_ply(str(bad))
    bad.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement face 1\n"
                    b"property list uchar int vertex_indices\nend_header\n")
    with pytest.raises(ValueError):
        gvc_ply.read_ply(str(bad))
    bad.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 4\nproperty float x\nend_header\n"
                    + b"\0" * 12)
    with pytest.raises(ValueError):
        gvc_ply.read_ply(str(bad))


@pytest.mark.skipif(not os.path.exists(REF_PLY), reason="the reference tree is not present")
def test_reference_file_bytes(tmp_path, golden):
    g = gvc_ply.read_gaussian_ply(REF_PLY)
    n = g["xyz"].shape[0]
    sel = np.sort(np.random.default_rng(7).choice(n, 1024, replace=False))  # make_golden.py's subset
    for k, v in golden.items():
        np.testing.assert_array_equal(g[k][sel], v)
    p = str(tmp_path / "point_cloud.ply")
    gvc_ply.write_gaussian_ply(p, g["xyz"], g["values"], g["weights"], g["scales"], g["rots"])
    assert open(p, "rb").read() == open(REF_PLY, "rb").read()
    assert open(p.replace(".ply", "_ascii.ply")).read() == open(REF_PLY.replace(".ply", "_ascii.ply")).read()
