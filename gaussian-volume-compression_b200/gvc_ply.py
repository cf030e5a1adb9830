"""Gaussian point-cloud PLY files without plyfile.

The reference stores its Gaussians with plyfile (scene/gaussian_model.py:257-283
save_ply, :285-301 save_ply_activated, :310-383 load_ply, :801-819
convert_ply_to_ascii): one element "vertex" with float32 properties
x y z value weight scale_0..2 rot_0..3, written binary little-endian, plus an ASCII copy
`<name>_ascii.ply`.  This module reads and writes the same files with numpy alone:

  * write_gaussian_ply(path, xyz, values, weights, scales, rots, ascii_copy=True)
  * read_gaussian_ply(path) -> dict(xyz, values, weights, scales, rots), float32, shapes as
    load_ply builds them (scale_* and rot_* columns ordered by their index suffix)
  * read_ply(path) -> {element name: numpy structured array} for any file with scalar
    properties (ascii, binary little- or big-endian)
  * ply_to_ascii(path) -> the ASCII copy's path (every property declared float, values
    printed as numpy prints them, like convert_ply_to_ascii)
"""
import os

import numpy as np

_TYPES = {
    "char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1",
    "short": "i2", "int16": "i2", "ushort": "u2", "uint16": "u2",
    "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
    "float": "f4", "float32": "f4", "double": "f8", "float64": "f8",
}


def construct_list_of_attributes(n_scale=3, n_rot=4):
    """Property order of scene/gaussian_model.py:257-263."""
    return (["x", "y", "z", "value", "weight"] + ["scale_%d" % i for i in range(n_scale)] +
            ["rot_%d" % i for i in range(n_rot)])


def _header(fmt, elements):
    lines = ["ply", "format %s 1.0" % fmt]
    for name, count, props in elements:
        lines.append("element %s %d" % (name, count))
        for pname, ptype in props:
            lines.append("property %s %s" % (ptype, pname))
    lines.append("end_header")
    return ("\n".join(lines) + "\n").encode("ascii")


def write_gaussian_ply(path, xyz, values, weights, scales, rots, ascii_copy=True):
    """save_ply (scene/gaussian_model.py:265-283): binary little-endian float32 records in
    the order x y z value weight scale_* rot_*; with ascii_copy also `<name>_ascii.ply`."""
    cols = [np.asarray(a, dtype=np.float32).reshape(len(np.asarray(xyz)), -1)
            for a in (xyz, values, weights, scales, rots)]
    n = cols[0].shape[0]
    if cols[0].shape[1] != 3 or cols[1].shape[1] != 1 or cols[2].shape[1] != 1:
        raise ValueError("xyz must be [N,3], values and weights [N] or [N,1]")
    names = construct_list_of_attributes(cols[3].shape[1], cols[4].shape[1])
    data = np.concatenate(cols, axis=1)
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "wb") as f:
        f.write(_header("binary_little_endian", [("vertex", n, [(p, "float") for p in names])]))
        f.write(np.ascontiguousarray(data, dtype="<f4").tobytes())
    if ascii_copy:
        ply_to_ascii(path)
    return path


def _parse_header(f):
    first = f.readline()
    if first.strip() != b"ply":
        raise ValueError("not a PLY file")
    fmt = None
    elements = []
    while True:
        line = f.readline()
        if not line:
            raise ValueError("PLY header has no end_header")
        tok = line.decode("ascii", "replace").split()
        if not tok:
            continue
        if tok[0] == "format":
            fmt = tok[1]
        elif tok[0] == "element":
            elements.append([tok[1], int(tok[2]), []])
        elif tok[0] == "property":
            if not elements:
                raise ValueError("property before any element")
            if tok[1] == "list":
                raise ValueError("list properties are not supported (element %s)" % elements[-1][0])
            if tok[1] not in _TYPES:
                raise ValueError("unknown property type " + tok[1])
            elements[-1][2].append((tok[2], tok[1]))
        elif tok[0] == "end_header":
            break
        elif tok[0] in ("comment", "obj_info"):
            continue
        else:
            raise ValueError("unexpected PLY header line: " + line.decode("ascii", "replace").strip())
    if fmt not in ("ascii", "binary_little_endian", "binary_big_endian"):
        raise ValueError("unsupported PLY format %r" % fmt)
    return fmt, elements


def read_ply(path):
    """{element name: structured array} of a PLY file with scalar properties."""
    out = {}
    with open(path, "rb") as f:
        fmt, elements = _parse_header(f)
        if fmt == "ascii":
            rest = f.read().decode("ascii").split("\n")
            pos = 0
            for name, count, props in elements:
                dt = np.dtype([(p, _TYPES[t]) for p, t in props])
                arr = np.empty(count, dtype=dt)
                for r in range(count):
                    while pos < len(rest) and not rest[pos].strip():
                        pos += 1
                    if pos >= len(rest):
                        raise ValueError("PLY body ends early in element " + name)
                    vals = rest[pos].split()
                    pos += 1
                    if len(vals) != len(props):
                        raise ValueError("row %d of element %s has %d values, expected %d"
                                         % (r, name, len(vals), len(props)))
                    arr[r] = tuple(np.array(v, dtype=_TYPES[t]) for v, (_, t) in zip(vals, props))
                out[name] = arr
        else:
            order = "<" if fmt == "binary_little_endian" else ">"
            for name, count, props in elements:
                dt = np.dtype([(p, order + _TYPES[t]) for p, t in props])
                raw = f.read(dt.itemsize * count)
                if len(raw) != dt.itemsize * count:
                    raise ValueError("PLY body ends early in element " + name)
                out[name] = np.frombuffer(raw, dtype=dt).astype(dt.newbyteorder("="))
    return out


def read_gaussian_ply(path):
    """load_ply (scene/gaussian_model.py:310-383) without the model: the raw (not
    activated) parameters as float32 arrays xyz [N,3], values [N,1], weights [N,1],
    scales [N,k], rots [N,m]."""
    el = read_ply(path)
    if "vertex" not in el:
        raise ValueError("PLY file has no vertex element")
    v = el["vertex"]
    names = v.dtype.names

    def cols(prefix):
        ps = sorted((p for p in names if p.startswith(prefix)), key=lambda x: int(x.split("_")[-1]))
        return np.stack([np.asarray(v[p], dtype=np.float32) for p in ps], axis=1) if ps else \
            np.zeros((len(v), 0), np.float32)

    return {
        "xyz": np.stack([np.asarray(v[a], dtype=np.float32) for a in ("x", "y", "z")], axis=1),
        "values": np.asarray(v["value"], dtype=np.float32)[:, None],
        "weights": np.asarray(v["weight"], dtype=np.float32)[:, None],
        "scales": cols("scale_"),
        "rots": cols("rot"),
    }


def ply_to_ascii(binary_ply_file_path):
    """convert_ply_to_ascii (scene/gaussian_model.py:801-819): `<name>_ascii.ply` with
    every property declared float and each row's values joined by spaces."""
    ascii_path = binary_ply_file_path.replace(".ply", "_ascii.ply")
    el = read_ply(binary_ply_file_path)
    with open(ascii_path, "w") as f:
        f.write("ply\nformat ascii 1.0\n")
        for name, arr in el.items():
            f.write("element %s %d\n" % (name, len(arr)))
            for p in arr.dtype.names:
                f.write("property float %s\n" % p)
        f.write("end_header\n")
        for name, arr in el.items():
            cols = [arr[p] for p in arr.dtype.names]
            for r in range(len(arr)):
                f.write(" ".join(str(c[r]) for c in cols) + "\n")
    return ascii_path
