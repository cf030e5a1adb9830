"""Builds libgvc.so (sm_100a) next to this file.

    python gaussian-volume-compression_b200/build.py [-v]

prep.cu and mesh.cu are compiled with --fmad=false so that their float/double
arithmetic rounds after every operation (bit-reproducible against the CPU oracle);
the evaluation kernels keep FMA contraction.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgvc.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
                 "-I", os.path.join(HERE, "..", "include")]
SOURCES = {
    "lbvh.cu": [],
    "render.cu": [],
    "capi.cu": [],
    "prep.cu": ["--fmad=false"],
    "mesh.cu": ["--fmad=false"],
    "noalloc.cu": [],
    "cta.cu": [],
    "fwd_tc.cu": [],
    "bwd_tc.cu": [],
    "knn.cu": [],
    "trainsamp.cu": [],
}


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose=False, ptxas_info=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "gvc.h"))
    nvcc = _nvcc()
    jobs = []
    objs = []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if not force and _newer(o, [s] + headers):
            continue
        cmd = [nvcc, "-c", s, "-o", o] + COMMON + extra
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or ptxas_info or r.returncode != 0:
                sys.stdout.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError("nvcc failed for " + cmd[2])
    if jobs or not os.path.exists(LIB) or not _newer(LIB, objs):
        cmd = [nvcc, "-shared", "-o", LIB] + ARCH + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode != 0:
            sys.stdout.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("link of libgvc.so failed")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv, force="-f" in sys.argv)
    print(LIB)
