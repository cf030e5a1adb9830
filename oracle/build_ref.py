"""Builds oracle/_ref/libgvc_ref.so: the reference's own rasterizer kernels compiled for
the host CPU.  TEST INFRASTRUCTURE ONLY (a checker and the timed CPU baseline; never part
of the product).

    python oracle/build_ref.py [reference_root]

The reference root comes from the argument, else $GVC_REFERENCE_ROOT, else
/root/reference.  Sources compiled, where they lie (nothing of them is committed here):

  diff-gaussian-rasterization/cuda_rasterizer/forward.cu   preprocessCUDA, sampleRenderCUDA,
                                                           FORWARD::preprocess / render
  diff-gaussian-rasterization/cuda_rasterizer/backward.cu  preprocessCUDA, sampleRenderCUDA,
                                                           BACKWARD::render

The one rewrite applied to the text is the CUDA launch syntax, which C++ cannot parse:
`kernel<<<grid, block>>>(args);` becomes `ref_launch(dim3(grid), dim3(block), kernel, args);`.
The rewritten translation units go to oracle/_ref/ (a build directory, git-ignored) with
#line directives pointing back at the original lines.  The absent third-party headers
(glm, cuBQL, cooperative groups, the CUDA runtime) are replaced by the stand-ins in
oracle/refshim/.  Two builds are made:

  libgvc_ref.so      -ffp-contract=off: every float operation rounded as written;
  libgvc_ref_fma.so  -ffp-contract=fast -mfma: the compiler may fuse multiply-adds, as
                     nvcc does by default when it builds the reference (the fused
                     positions differ between the two compilers, so this build shows
                     how large contraction effects are, not the reference binary's bits).

The recipe also records where it found the reference in oracle/_ref/REFERENCE_ROOT, so
that the CPU tests that read reference files can find them without a fixed path.
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "refshim")
DRIVER = os.path.join(HERE, "ref_driver.cpp")
LIB = os.path.join(OUT, "libgvc_ref.so")
LIB_FMA = os.path.join(OUT, "libgvc_ref_fma.so")
RASTER = os.path.join("diff-gaussian-rasterization", "cuda_rasterizer")
UNITS = ("forward.cu", "backward.cu")


def reference_root(arg=None):
    for cand in (arg, os.environ.get("GVC_REFERENCE_ROOT"), "/root/reference"):
        if cand and os.path.isfile(os.path.join(cand, RASTER, "forward.cu")):
            return cand
    return None


def _split_top(s):
    """Splits a launch configuration at its top-level commas."""
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return [p.strip() for p in parts]


LAUNCH = re.compile(r"(\w+)\s*<\s*<\s*<(.*?)>\s*>\s*>\s*\(", re.S)


def rewrite_launches(src):
    """Rewrites every `k<<<g, b>>>(args)` into `ref_launch(dim3(g), dim3(b), k, args)`."""
    out, pos, n = [], 0, 0
    while True:
        m = LAUNCH.search(src, pos)
        if not m:
            out.append(src[pos:])
            break
        cfg = _split_top(m.group(2))
        if len(cfg) != 2:
            raise ValueError("unexpected launch configuration: " + m.group(2))
        # the argument list ends at the parenthesis that closes the one the match ends on
        depth, i = 1, m.end()
        while depth:
            depth += {"(": 1, ")": -1}.get(src[i], 0)
            i += 1
        args = src[m.end():i - 1]
        out.append(src[pos:m.start()])
        # keep the line count of the original text (newlines inside the launch stay)
        out.append("ref_launch(dim3(%s), dim3(%s), %s, %s)" % (cfg[0], cfg[1], m.group(1), args))
        pos = i
        n += 1
    return "".join(out), n


def build(root=None, force=False, verbose=False):
    root = reference_root(root)
    if root is None:
        return None
    os.makedirs(OUT, exist_ok=True)
    srcs = [os.path.join(root, RASTER, u) for u in UNITS]
    deps = srcs + [DRIVER, __file__] + [os.path.join(d, f) for d, _, fs in os.walk(SHIM) for f in fs]
    if not force and all(os.path.exists(p) for p in (LIB, LIB_FMA)):
        t = min(os.path.getmtime(LIB), os.path.getmtime(LIB_FMA))
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    units = []
    for s in srcs:
        text, n = rewrite_launches(open(s).read())
        if n == 0:
            raise ValueError("no kernel launch found in " + s)
        dst = os.path.join(OUT, os.path.basename(s).replace(".cu", "_host.cpp"))
        with open(dst, "w") as f:
            f.write('#line 1 "%s"\n' % s)
            f.write(text)
        units.append(dst)
    with open(os.path.join(OUT, "REFERENCE_ROOT"), "w") as f:
        f.write(os.path.abspath(root) + "\n")
    base = ["g++", "-std=c++17", "-O2", "-fopenmp", "-fPIC", "-shared", "-fno-fast-math",
            "-include", os.path.join(SHIM, "refshim_prelude.h"), "-I", SHIM, "-I", os.path.join(root, RASTER),
            "-w", "-o"]
    for lib, fp in ((LIB, ["-ffp-contract=off"]), (LIB_FMA, ["-ffp-contract=fast", "-mfma"])):
        cmd = base + [lib] + units + [DRIVER] + fp
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode != 0:
            sys.stdout.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("reference host build failed")
    return LIB


if __name__ == "__main__":
    path = build(sys.argv[1] if len(sys.argv) > 1 else None, force=True, verbose="-v" in sys.argv)
    print(path or "reference sources not found; nothing built")
