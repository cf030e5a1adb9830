#!/usr/bin/env python
"""Benchmark of the Gaussian-mixture volume training step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config large|medium|small|slice|tiny] [--eval-path plain|tensor_core|plain_tile] [--mesh] [--knn]

Default configuration: FP32 forward (CTA pipeline) and the tensor-core backward reduction
(--bwd-mode tensor_core); tc_vs_plain times FP32 throughout (the library default) and
tensor cores throughout on the same step.

Metric: fwd+bwd ms per step at 2M Gaussians x 16M points (the "large evaluation"
configuration: clustered means, half the samples near Gaussian means).  One step is what
the reference's training loop does per iteration on this path: build the sample index
(build_bvh, train.py:366), forward (render, train.py:370), the masked L1 loss gradient
(train.py:389-396) and the backward (train.py:445), all on device-resident inputs.

N > 1 (torchrun): weak scaling -- every rank holds all Gaussians and its own 16M
samples; the per-Gaussian gradients are summed with one NCCL all-reduce per step.

--impl reference: the reference's own rasterizer kernels (forward.cu, backward.cu)
compiled for the host CPU (oracle/_ref; the reference's CUDA extension cannot be built on
the GPU -- its cuBQL/glm sources are not vendored), in its default sample-BVH mode, timed
on bounded samples of the points with all host threads and extrapolated to the full step;
rank 0 only.  Without oracle/_ref it falls back to the FP64 restatement (oracle/).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gaussian-volume-compression_b200")
sys.path.insert(0, PKG)

CONFIGS = {
    # name: (P, S, description)
    "large": (2_000_000, 16_000_000, "large evaluation: 2M clustered Gaussians x 16M points (8M uniform + 8M near means)"),
    "medium": (200_000, 4_000_000, "scaled large evaluation: 200k clustered Gaussians x 4M points"),
    "small": (200_000, 2_000_000, "profiling case: 200k clustered Gaussians x 2M points"),
    "slice": (2_000_000, 4_000_000, "profiling case with the large evaluation's Gaussians: 2M clustered Gaussians x 4M points"),
    "tiny": (4_096, 262_144, "CPU-runnable case: 4096 clustered Gaussians x 64^3 points"),
    "config1": (4_096, 262_144, "small mixture: 4096 Gaussians (means U[0,1]^3, log-scales N(log 0.02, 0.3)) "
                                "at the 64^3 cell centres"),
    "config2": (200_000, 4_000_000, "structured-volume fit step: 256^3 volume (64 anisotropic blobs + "
                                    "0.1 sin 8pi x sin 8pi y sin 8pi z), 200k Gaussians at random lattice points "
                                    "(isotropic 3-NN scales, q = (1,0,0,0), w = 0.1, v = the volume there), 4M uniform "
                                    "points, targets through gpu_sample"),
}
METRIC = "fwd+bwd ms/step (2M Gaussians×16M pts), TC vs plain FP32 at stated FP64 err"
# Algorithmic FP32 work per pair (FORWARD forward.cu:224-256, BACKWARD backward.cu:252-298):
F_CAND = 24            # d = x - mu, quadratic form, -0.5 (every candidate pair)
F_FWD_CONTRIB = 28     # + w e, two accumulations (contributing pair, plus one EX2)
F_BWD_CONTRIB = 64     # recompute + adjoint (contributing pair with W > 0.01, plus one EX2)
EX2_EQUIV = 8          # MUFU ex2 issue cost in FP32-lane units (16/clk/SM vs 128/clk/SM)
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the dominant
# kernels at the 2M x 16M workload, from one single-pass capture of
# `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum --clock-control none
#  -k regex:"k_backward_cta|k_forward_cta" -s 2 -c 2 python bench.py --profile --steps 1 --warmup 1`
# (and of k_backward_gauss with --bwd-mode deterministic); other workloads report null.
# Tensor-pipe activity (sm__pipe_tc_cycles_active, share of peak) of the tensor-core kernels
# in their committed --set full captures of the 2M x 4M profiling case (profiles/).
TENSOR_PIPE_ACTIVE = {"k_backward_cta": 0.358, "k_forward_tc": 0.189}
MEASURED_TRAFFIC = {("large", "k_backward_cta"): 1.291e9 + 0.142e9,
                    ("large", "k_backward_gauss"): 1.475e9 + 0.125e9,
                    ("large", "k_forward_cta"): 1.585e9 + 1.774e9}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="large", choices=list(CONFIGS))
    # default: the fastest configuration within tolerance of the FP64 oracle (FP32 forward,
    # tensor-core backward reduction); the library's own default backward is the
    # deterministic one ("auto"), timed beside it in tc_vs_plain
    p.add_argument("--bwd-mode", default="tensor_core", choices=["auto", "deterministic", "atomic", "tensor_core"])
    p.add_argument("--eval-path", default="plain", choices=["plain", "tensor_core", "plain_tile"])
    p.add_argument("--traversal", default="stack", choices=["stack", "stackless"],
                   help="Gaussian-LBVH traversal of the block-group kernels (both are timed in tc_vs_plain)")
    p.add_argument("--use-gaussian-bvh", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile", action="store_true", help="minimal run for ncu (no e2e, no CPU baseline)")
    p.add_argument("--knn", action="store_true",
                   help="also time distCUDA2 (3-NN mean squared distance) on the 2M clustered Gaussian means "
                        "and add a knn3 object")
    p.add_argument("--fit", type=int, default=0, metavar="ITERS",
                   help="also run the end-to-end fit of the 512^3 turbulent volume (configuration 5) for ITERS "
                        "iterations per evaluation path and add a fit object")
    p.add_argument("--mesh", action="store_true",
                   help="also time the mesh samplers (128^3 jittered hex grid split into 12.6M tetrahedra, "
                        "256^3 uniform grid, 8M points each) and add a mesh_sampler object")
    return p.parse_args()


TARGETS = {}  # config -> target values of the workload's samples (configurations that define them)


def config2_workload(P, S, seed=0):
    """Config 2 as stated: the GaussianModel.create_from_pcd initialisation
    (scene/gaussian_model.py:175-192: log-scale = log sqrt(max(distCUDA2, 1e-7)) on all
    three axes, q = (1, 0, 0, 0), w = 0.1, v = the volume's value) activated by the
    model's getters (:71-77, :114-132: exp + tanh soft cap at 0.02, normalise, identity for
    the already activated w and v), S uniform points per step and their targets sampled
    from the volume with gpu_sample (trilinear, as the training targets are made)."""
    import torch
    import gvc_workloads as wl
    from gpu_mesh_sampling import gpu_sample
    from simple_knn._C import distCUDA2
    dev = torch.device("cuda", torch.cuda.current_device())
    n = 256
    vol = wl.volume_blobs_sine(n=n, seed=seed, device=dev)
    pts, vals = wl.lattice_init(vol, P, seed=seed)
    s = torch.sqrt(torch.clamp_min(distCUDA2(pts), 1e-7))[:, None].repeat(1, 3)
    r = torch.linalg.norm(s, dim=1, keepdim=True) + 1e-8
    s = s * ((0.02 * torch.tanh(r / 0.02)) / r)
    rots = torch.zeros(P, 4, device=dev)
    rots[:, 0] = 1.0
    g = torch.Generator(device="cpu").manual_seed(seed + 7)
    samples = torch.rand(S, 3, generator=g).numpy()
    target = gpu_sample(np.array([n, n, n]), np.zeros(3, np.float32), np.full(3, 1.0 / (n - 1), np.float32),
                        vol.reshape(-1).cpu().numpy(), samples)
    f = lambda t: np.ascontiguousarray(t.detach().cpu().numpy().astype(np.float32))
    return (f(pts), f(s), f(rots), f(vals), np.full(P, 0.1, np.float32), samples.astype(np.float32),
            np.ascontiguousarray(target.astype(np.float32)))


def workload(cfg, rank):
    import gvc_workloads as wl
    P, S, desc = CONFIGS[cfg]
    if cfg == "config1":
        means, scales, rots, values, weights = wl.mixture_small(seed=0, P=P)
        return means, scales, rots, values, weights, wl.grid_centres(64), desc
    if cfg == "config2":
        means, scales, rots, values, weights, samples, target = config2_workload(P, S, seed=rank)
        TARGETS[cfg] = target
        return means, scales, rots, values, weights, samples, desc
    means, scales, rots, values, weights, _ = wl.mixture_large(seed=0, P=P, S=2)
    # per-rank sample set (weak scaling); rank 0 uses the config's own seed
    _, _, _, _, _, samples = wl.mixture_large(seed=0 if rank == 0 else 1000 + rank, P=P, S=S)
    return means, scales, rots, values, weights, samples, desc


def target_field(samples_t):
    """Synthetic target of the L1 loss (the large configuration names none)."""
    import torch
    x, y, z = samples_t[:, 0], samples_t[:, 1], samples_t[:, 2]
    return 0.5 + 0.4 * torch.sin(6 * x) * torch.sin(5 * y) * torch.sin(4 * z)


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained"), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


# ----------------------------------------------------------------------------------------
# CPU legs: the reference's own rasterizer kernels compiled for the host (oracle/_ref,
# "reference"), else the FP64 restatement (oracle/gvc_oracle.c, "port"), on bounded
# samples of the workload's points with all Gaussians, extrapolated linearly in S
# ----------------------------------------------------------------------------------------
def _oracle_path():
    p = os.path.join(ROOT, "oracle")
    if p not in sys.path:
        sys.path.insert(0, p)


def host_threads():
    """Host threads the CPU arms use: every core this process may run on.  Set explicitly
    because torch.distributed.run exports OMP_NUM_THREADS=1 to its ranks."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def cpu_kind():
    _oracle_path()
    import refslice
    return "reference" if refslice.available() else "port"


def cpu_step_time(kind, means, scales, rots, values, weights, samples, n_sub, seed=5, target=None):
    """One CPU step on n_sub of the points: preprocess, forward, masked-L1 gradient,
    backward (covariance adjoint included).  kind "reference": the reference's kernels in
    its default (sample-BVH) mode, FP32, all host threads; "port": the FP64 oracle."""
    _oracle_path()
    rng = np.random.default_rng(seed)
    pick = rng.choice(samples.shape[0], n_sub, replace=False)
    sub = samples[pick]
    if target is not None:
        gt = target[pick]
    else:
        gt = (0.5 + 0.4 * np.sin(6 * sub[:, 0]) * np.sin(5 * sub[:, 1]) * np.sin(4 * sub[:, 2])).astype(np.float32)
    nt = host_threads()
    t0 = time.perf_counter()
    if kind == "reference":
        import refslice
        refslice.config(nthreads=nt)
        rc, rb = refslice.preprocess(means, scales, rots, weights)
        out, outw, _ = refslice.forward(means, values, weights, sub, rc, rb, use_gaussian_bvh=False)
        mask = out != -1
        g = (np.where(mask, np.sign(out - gt), 0.0) / max(int(mask.sum()), 1)).astype(np.float32)
        refslice.backward(means, scales, rots, rc, values, weights, rb, sub, out, outw, g,
                          np.zeros(n_sub, np.float32), use_gaussian_bvh=False)
    else:
        import oracle
        c32, _, bb = oracle.preprocess(means, scales, rots, weights, nthreads=nt)
        out, outw = oracle.forward(means, values, weights, c32.astype(np.float64), bb, sub, nthreads=nt)
        mask = out != -1
        g = np.where(mask, np.sign(out - gt), 0.0) / max(int(mask.sum()), 1)
        r = oracle.backward(means, values, weights, c32.astype(np.float64), bb, sub, out.astype(np.float32),
                            outw.astype(np.float32), g.astype(np.float32), np.zeros(n_sub, np.float32), nthreads=nt)
        oracle.cov_backward(scales, rots, c32, r["dconics"], nthreads=nt)
    return time.perf_counter() - t0


CPU_DESC = {"reference": "the reference's own kernels (diff-gaussian-rasterization/cuda_rasterizer/forward.cu, "
                         "backward.cu) compiled for the host by oracle/build_ref.py, FP32, its default sample-BVH "
                         "mode (forward.cu:116-182, backward.cu:127-337), OpenMP over blocks; a uniform grid stands "
                         "in for the unvendored cuBQL BVH",
            "port": "the oracle's FP64 restatement (oracle/gvc_oracle.c, OpenMP)"}


def cpu_extrapolated(kind, means, scales, rots, values, weights, samples, n_a, n_b, reps_b=1, warmup=0):
    """Times n_a points once and n_b points reps_b times (median) after `warmup` untimed
    n_b runs; extrapolates t = fixed + slope * S to the full step."""
    threads = host_threads()
    S = samples.shape[0]
    tg = TARGETS.get("config2") if means.shape[0] == CONFIGS["config2"][0] and S == CONFIGS["config2"][1] else None
    t_a = cpu_step_time(kind, means, scales, rots, values, weights, samples, n_a, target=tg)
    for _ in range(warmup):
        cpu_step_time(kind, means, scales, rots, values, weights, samples, n_b, target=tg)
    tb = [cpu_step_time(kind, means, scales, rots, values, weights, samples, n_b, seed=10 + k, target=tg)
          for k in range(reps_b)]
    t_b = float(np.median(tb))
    slope = (t_b - t_a) / (n_b - n_a)
    fixed = max(t_a - slope * n_a, 0.0)
    full_ms = (fixed + slope * S) * 1e3
    return {"value": full_ms, "unit": "ms/step", "cores": threads, "kind": kind,
            "sample": "%s: fwd+bwd on %d (x1) and %d (x%d, median) of the %d points with all %d Gaussians "
                      "(%.2f s, %.2f s per sample step), linearly extrapolated to the full step"
                      % (CPU_DESC[kind], n_a, n_b, reps_b, S, means.shape[0], t_a, t_b),
            "extrapolated": True,
            "timed": {"points_a": int(n_a), "reps_a": 1, "seconds_a": t_a, "points_b": int(n_b),
                      "reps_b": int(reps_b), "seconds_b_median": t_b, "fixed_s": fixed, "per_point_us": slope * 1e6,
                      "full_step_equivalents": (n_a + reps_b * n_b) / S}}


def cpu_baseline(means, scales, rots, values, weights, samples):
    """Our line's cpu_baseline: the same measurement as the reference arm, one repetition."""
    kind = cpu_kind()
    S = samples.shape[0]
    if S <= 300_000:
        threads = host_threads()
        t = cpu_step_time(kind, means, scales, rots, values, weights, samples, S)
        return {"value": t * 1e3, "unit": "ms/step", "cores": threads, "kind": kind,
                "sample": "%s: the full step, all %d points and %d Gaussians" % (CPU_DESC[kind], S, means.shape[0]),
                "extrapolated": False}
    return cpu_extrapolated(kind, means, scales, rots, values, weights, samples, min(125_000, S // 8),
                            min(500_000, S // 2))


def fp64_errors(means, scales, rots, values, weights, samples, paths, n_sub=1_000_000, seed=7):
    """Checker, outside every timed region: each path's forward (cells = V/W and W) against
    the oracle's FP64 evaluation of the same conics at a random subset of points.  Reports
    the largest and the 99.99th-percentile relative error over points the reference marks
    valid, and the share of points above 1e-4.  Points whose W lies within 1e-6 of the 0.01
    validity threshold are left out (either answer is within rounding)."""
    _oracle_path()
    import oracle
    n_sub = min(n_sub, samples.shape[0])
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(samples.shape[0], n_sub, replace=False))
    sub = samples[idx]
    _, _, bb = oracle.preprocess(means, scales, rots, weights)
    res = {"points": int(n_sub), "reference": "oracle FP64 evaluation (C) of the path's own FP32 conics"}
    for name, d in paths.items():
        ro, rw = oracle.forward(means, values, weights, d["conics"].astype(np.float64), bb, sub)
        o, w = d["out"][idx].astype(np.float64), d["outw"][idx].astype(np.float64)
        ok = (ro != -1) & (np.abs(rw - 0.01) > 1e-6)
        e_out = np.abs(o[ok] - ro[ok]) / np.maximum(np.abs(ro[ok]), 1e-6)
        e_w = np.abs(w[ok] - rw[ok]) / rw[ok]
        mism = int(((o != -1) != (ro != -1))[np.abs(rw - 0.01) > 1e-6].sum())
        res[name] = {"cells_max_rel": float(e_out.max()) if e_out.size else 0.0,
                     "cells_p9999_rel": float(np.quantile(e_out, 0.9999)) if e_out.size else 0.0,
                     "weights_max_rel": float(e_w.max()) if e_w.size else 0.0,
                     "share_above_1e-4": float((np.maximum(e_out, e_w) > 1e-4).mean()) if e_out.size else 0.0,
                     "validity_mismatches": mism, "valid_points": int(ok.sum())}
    return res


GRAD_FIELDS = ("means", "scales", "rotations", "values", "weights")


def grad_errors(means, scales, rots, values, weights, samples, runs, n_gauss=10_000, seed=8):
    """Checker, outside every timed region: each backward's gradients of a random subset of
    n_gauss Gaussians against the oracle's FP64 adjoint (backward.cu:252-298 restated) over
    ALL samples of the step, with the same forward outputs and loss gradient the GPU used,
    then the covariance adjoint (true gradient).  Per field: max |gpu - fp64| / max |fp64|
    over the subset, and the 99.9th percentile of the per-Gaussian relative error."""
    _oracle_path()
    import oracle
    P = means.shape[0]
    rng = np.random.default_rng(seed)
    sel = np.sort(rng.choice(P, min(n_gauss, P), replace=False))
    res = {"gaussians": int(sel.size), "reference": "oracle FP64 adjoint over all samples of the step "
                                                     "(the path's own forward outputs and conics)"}
    for name, r in runs.items():
        conics = r["conics"][sel]
        _, _, bb = oracle.preprocess(means[sel], scales[sel], rots[sel], weights[sel])
        g = oracle.backward(means[sel], values[sel], weights[sel], conics.astype(np.float64), bb, samples,
                            r["out"], r["outw"], r["gout"], np.zeros(samples.shape[0], np.float32))
        ds, dq = oracle.cov_backward(scales[sel], rots[sel], conics, g["dconics"])
        ref = [g["dmeans"], ds, dq, g["dvalues"].reshape(-1, 1), g["dweights"].reshape(-1, 1)]
        out = {}
        for k, f in enumerate(GRAD_FIELDS):
            got = r["grads"][k].reshape(P, -1)[sel].astype(np.float64)
            rf = ref[k].reshape(sel.size, -1)
            scale = np.abs(rf).max()
            rel = np.abs(got - rf).max(1) / np.maximum(np.abs(rf).max(1), 1e-30)
            big = np.abs(rf).max(1) > 1e-3 * scale
            out[f] = {"max_abs_err_over_max": float(np.abs(got - rf).max() / scale) if scale > 0 else 0.0,
                      "p999_rel_err": float(np.quantile(rel[big], 0.999)) if big.any() else 0.0}
        res[name] = out
    return res


def config_dict(args, desc, P, S, world):
    """The config object of both arms' lines (identical for the same arguments)."""
    return {"workload": desc, "P": P, "S_per_gpu": S, "path": args.eval_path, "backward": args.bwd_mode,
            "traversal": args.traversal, "use_gaussian_bvh": bool(args.use_gaussian_bvh),
            "l2": "inputs larger than L2 (samples %d MB, Gaussian records %d MB)" % (S * 12 // 2**20, P * 80 // 2**20),
            "parallelism": "samples sharded per rank, NCCL all-reduce of gradients" if world > 1 else "single GPU"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    means, scales, rots, values, weights, samples, desc = workload(args.config, 0)
    kind = cpu_kind()
    S = samples.shape[0]
    if S <= 300_000:
        for _ in range(args.warmup):
            cpu_step_time(kind, means, scales, rots, values, weights, samples, S)
        t = [cpu_step_time(kind, means, scales, rots, values, weights, samples, S, seed=10 + k)
             for k in range(args.steps)]
        full_ms = float(np.median(t)) * 1e3
        cpu = {"value": full_ms, "unit": "ms/step", "cores": host_threads(), "kind": kind,
               "sample": "%s: the full step (all %d points, %d Gaussians), median of %d" %
                         (CPU_DESC[kind], S, means.shape[0], args.steps), "extrapolated": False}
        extra = {"extrapolated": False}
    else:
        # each sample step: all Gaussians and n_b of the points, sized so that the whole
        # run stays within a few minutes on the host cores
        n_a, n_b = min(62_500, S // 16), min(250_000, S // 4)
        cpu = cpu_extrapolated(kind, means, scales, rots, values, weights, samples, n_a, n_b, reps_b=args.steps,
                               warmup=max(args.warmup - 1, 0))
        full_ms = cpu["value"]
        extra = {"extrapolated": True,
                 "steps_note": "each of the %d steps is a bounded sample (%d of the %d points, all Gaussians); "
                               "value and ms_per_step are the linear extrapolation to the full step, and the "
                               "timed work equals %.3f full steps" % (args.steps, n_b, S,
                                                                       cpu["timed"]["full_step_equivalents"])}
    line = {"metric": METRIC, "value": full_ms, "unit": "ms/step", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": full_ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if kind == "reference" else "f64",
            "data": "synthetic", "config": config_dict(args, desc, means.shape[0], S, 1),
            "cpu_baseline": cpu,
            "e2e": {"value": full_ms, "unit": "ms/step", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's CUDA extension cannot be built on the GPU (its cuBQL and glm sources are not "
                    "vendored); this arm runs the reference's own kernel source compiled for the host CPU"
                    if kind == "reference" else
                    "the reference's sources were not available where oracle/_ref is built; this arm is the "
                    "oracle's FP64 restatement"}
    line.update(extra)
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------
# Mesh samplers (sample_meshu / sample_mesh): device-resident inputs, CUDA-event timing
# ----------------------------------------------------------------------------------------
def mesh_bench(dev, steps, warmup, with_cpu):
    import ctypes
    import torch
    import gvc_native
    import gvc_workloads as wl
    rng = np.random.default_rng(11)
    n_pts = 8_000_000
    res = {}
    ctx = gvc_native.Context()
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.sync_status(stream.cuda_stream)
        return e0.elapsed_time(e1) / steps

    # tetrahedra: 128^3 jittered hex grid, 6 tets per hex (12,582,912 cells), 8M points
    pts, tets = wl.jittered_tet_mesh(n=128, seed=7)
    vals = wl.blob_field(pts).astype(np.float64)
    q = rng.random((n_pts, 3), dtype=np.float32)
    d_pts, d_tets, d_vals, d_q = T(pts), T(tets.astype(np.int32)), T(vals), T(q)
    d_out = torch.empty(n_pts, dtype=torch.float64, device=dev)
    d_cell = torch.empty(n_pts, dtype=torch.int64, device=dev)
    ms = timed(lambda: ctx.call("gvc_sample_tets", pts.shape[0], gvc_native.ptr(d_pts), tets.shape[0],
                                gvc_native.ptr(d_tets), gvc_native.ptr(d_vals), n_pts, gvc_native.ptr(d_q),
                                gvc_native.ptr(d_out), gvc_native.ptr(d_cell), sp))
    tet = {"cells": int(tets.shape[0]), "points": n_pts, "ms_per_call": ms, "points_per_s": n_pts / (ms * 1e-3),
           "includes": "cell LBVH build (keys, sort, Karras, refit) + point sort + locate + interpolate",
           "found": float((d_cell >= 0).float().mean().item())}
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        sub = q[:1_000_000]
        t0 = time.perf_counter()
        r_out, r_cell = oracle.sample_tets(pts, tets, vals, sub, nthreads=host_threads())
        t = time.perf_counter() - t0
        tet["cpu_oracle"] = {"points_per_s": sub.shape[0] / t, "cores": host_threads(),
                             "sample": "oracle (C, OpenMP, uniform grid locator) on 1M of the points, "
                                       "locator build included (%.2f s)" % t}
        g_out = d_out[:sub.shape[0]].cpu().numpy()
        g_cell = d_cell[:sub.shape[0]].cpu().numpy()
        tet["bit_exact_vs_oracle"] = {"points": int(sub.shape[0]),
                                      "cell_ids": bool(np.array_equal(g_cell, r_cell)),
                                      "values": bool(np.array_equal(g_out, r_out)),
                                      "cell_id_mismatches": int((g_cell != r_cell).sum())}
    res["tets"] = tet
    # training batches (train.py:34-61, :273-315): 100 batches of 128^3 points in random
    # tetrahedra, per-batch Morton sort, float32 ground truth, all on the device
    B, S = 100, 128 ** 3
    d_bs = torch.empty((B, S, 3), dtype=torch.float32, device=dev)
    d_bg = torch.empty((B, S), dtype=torch.float32, device=dev)
    ms = timed(lambda: ctx.call("gvc_training_samples", pts.shape[0], gvc_native.ptr(d_pts), tets.shape[0],
                                gvc_native.ptr(d_tets), gvc_native.ptr(d_vals), B, S, ctypes.c_uint64(0),
                                gvc_native.ptr(d_bs), gvc_native.ptr(d_bg), sp))
    tb = {"batches": B, "batch_size": S, "cells": int(tets.shape[0]), "ms_per_call": ms,
          "points_per_s": B * S / (ms * 1e-3),
          "includes": "Philox points in random tets + 3-word radix sort (batch, 63-bit Morton) + gather "
                      "+ cell LBVH build + locate + interpolate + float32 conversion",
          "found": float((d_bg[:4] != -1).float().mean().item())}
    del d_bs, d_bg
    if with_cpu:
        t0 = time.perf_counter()
        oracle.training_samples(pts, tets, vals, 1, 2_000_000, seed=0, nthreads=host_threads())
        t = time.perf_counter() - t0
        tb["cpu_oracle"] = {"points_per_s": 2_000_000 / t, "cores": host_threads(),
                            "sample": "oracle (C Philox points, numpy stable Morton sort, C grid locator) on "
                                      "one batch of 2M points (%.2f s)" % t}
    res["training_batches"] = tb
    del d_pts, d_tets, d_vals
    # uniform grid: 256^3 float32 point values, trilinear, 8M points
    dims = np.array([256, 256, 256], np.int64)
    origin = np.zeros(3, np.float32)
    spacing = np.full(3, 1.0 / 255, np.float32)
    gvals = rng.random(int(dims.prod()), dtype=np.float32)
    d_g = T(gvals.view(np.uint8))
    d_o = torch.empty(n_pts * 4, dtype=torch.uint8, device=dev)
    ms = timed(lambda: ctx.call("gvc_sample_uniform", gvc_native.ptr(dims), gvc_native.ptr(origin),
                                gvc_native.ptr(spacing), gvc_native.ptr(d_g), gvc_native.DTYPE_CODES["float32"],
                                n_pts, gvc_native.ptr(d_q), gvc_native.ptr(d_o), sp))
    res["uniform"] = {"dims": [256, 256, 256], "dtype": "float32", "points": n_pts, "ms_per_call": ms,
                      "points_per_s": n_pts / (ms * 1e-3)}
    return res


# ----------------------------------------------------------------------------------------
# End-to-end fit (configuration 5): wall time to a volume PSNR, per evaluation path
# ----------------------------------------------------------------------------------------
FIT_PATHS = {"plain": ("plain", "auto"), "tensor_core": ("tensor_core", "auto"),
             "plain_fwd_tc_bwd": ("plain", "tensor_core")}
FIT_EVAL_AT = (0, 5, 10, 20, 30, 50, 75)  # then every 100 iterations


def fit_bench(dev, iters, paths=("plain", "tensor_core", "plain_fwd_tc_bwd"), n_vol=512, P0=500_000,
              cap=3_000_000, batch=8_000_000, seed=0):
    """A training run over the drop-in API that follows train.py's loop: per iteration a
    sample batch (uniform points with their targets, drawn from cached batches as
    train.py:286-345 does), build_bvh, the GaussianModel getters' activations
    (scene/gaussian_model.py:71-77, 114-132), the render's Morton argsort and gathers
    (gaussian_renderer/__init__.py:61-82), the masked L1 plus the false-negative term
    (train.py:389-429, encode_surface off), backward and Adam with the default learning
    rates (arguments/__init__.py:82-91, eps 1e-15).  Every 100 iterations: densify in the
    samples of largest error (train.py:551-586: k = min(500k, cap - P + dead + 1000) new
    Gaussians at the top-k samples with their target value, weight 0.01, scale from
    distCUDA2 x 0.1, gaussian_model.py:727-765) and prune weights below 0.005, and the
    volume PSNR on a fixed 1M-point set (volume_metrics.py:345-346: -10 log10(mse + 1e-8),
    empty samples counted with their -1).  Reports, per path, the wall time (host clock,
    synchronised, evaluations excluded) to 30, 35 and 40 dB and the PSNR history (evaluated
    at iterations 0, 5, 10, 20, 30, 50, 75 and every 100)."""
    import ctypes
    import torch
    import gvc_native
    import gvc_workloads as wl
    import bvh_diff_gaussian_rasterization as R
    from bvh_diff_gaussian_rasterization import _C
    from simple_knn._C import distCUDA2
    torch.manual_seed(seed)
    vol = wl.volume_turbulent(n=n_vol, seed=seed, device=dev)
    ctx = gvc_native.Context()
    sp = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    dims = np.array([n_vol] * 3, np.int64)
    origin = np.zeros(3, np.float32)
    spacing = np.full(3, 1.0 / (n_vol - 1), np.float32)
    vbytes = vol.reshape(-1).contiguous().view(torch.uint8)

    def targets(pts):
        out = torch.empty(pts.shape[0], dtype=torch.float32, device=dev)
        ctx.call("gvc_sample_uniform", gvc_native.ptr(dims), gvc_native.ptr(origin), gvc_native.ptr(spacing),
                 gvc_native.ptr(vbytes), gvc_native.DTYPE_CODES["float32"], pts.shape[0], gvc_native.ptr(pts),
                 gvc_native.ptr(out), sp)
        return out

    nb = 8
    batches = []
    for _ in range(nb):
        pts = torch.rand(batch, 3, device=dev)
        batches.append((pts, targets(pts)))
    eval_pts = torch.rand(1_000_000, 3, device=dev)
    eval_gt = targets(eval_pts)
    inv_sig = lambda x: torch.log(x / (1 - x))

    def morton(xyz):
        q = (xyz * ((1 << 21) - 1)).long()

        def part(n):
            n = n & 0x1fffff
            n = (n | (n << 32)) & 0x1f00000000ffff
            n = (n | (n << 16)) & 0x1f0000ff0000ff
            n = (n | (n << 8)) & 0x100f00f00f00f00f
            n = (n | (n << 4)) & 0x10c30c30c30c30c3
            n = (n | (n << 2)) & 0x1249249249249249
            return n
        return part(q[:, 0]) | (part(q[:, 1]) << 1) | (part(q[:, 2]) << 2)

    results = {}
    for path in paths:
        _C.set_eval_path(FIT_PATHS[path][0])
        _C.set_backward_mode(FIT_PATHS[path][1])
        pts, vals = wl.lattice_init(vol, P0, seed=seed)
        d2 = torch.clamp_min(distCUDA2(pts), 1e-7)
        params = {"xyz": pts.clone(), "scaling": torch.log(torch.sqrt(d2))[:, None].repeat(1, 3),
                  "rotation": torch.tensor([[1.0, 0, 0, 0]], device=dev).repeat(P0, 1),
                  "weight": inv_sig(torch.full((P0, 1), 0.1, device=dev)),
                  "value": inv_sig(vals.clamp(1e-3, 1 - 1e-3))[:, None]}
        lrs = {"xyz": 0.00016, "weight": 0.025, "scaling": 0.001, "rotation": 0.0001, "value": 0.0025}
        for k in params:
            params[k] = torch.nn.Parameter(params[k].contiguous())
        opt = torch.optim.Adam([{"params": [params[k]], "lr": lrs[k], "name": k} for k in params], lr=0.0, eps=1e-15)
        settings = R.GaussianRasterizationSettings((0, 0, 0), (1, 1, 1), 0, -1.0, 1.0, False, False)
        rast = R.GaussianRasterizer(settings)

        def activated():
            s = torch.exp(params["scaling"])
            r = torch.linalg.norm(s, dim=1, keepdim=True) + 1e-8
            s = s * ((0.02 * torch.tanh(r / 0.02)) / r)
            return (params["xyz"], s, torch.nn.functional.normalize(params["rotation"]),
                    torch.sigmoid(params["value"]), torch.sigmoid(params["weight"]))

        def render():
            m, sc, q, v, w = activated()
            order = torch.argsort(morton(m))
            return rast(m[order], sc[order], q[order], v[order], w[order])

        def replace(new):  # swap parameters, keeping (and extending or cutting) Adam's state
            for grp in opt.param_groups:
                old = grp["params"][0]
                k = grp["name"]
                st = opt.state.pop(old, None)
                p_new = torch.nn.Parameter(new[k]["tensor"].contiguous())
                if st is not None:
                    for key in ("exp_avg", "exp_avg_sq"):
                        st[key] = new[k]["state"](st[key])
                    opt.state[p_new] = st
                grp["params"][0] = p_new
                params[k] = p_new

        def densify_and_prune(samples, cells, gt):
            with torch.no_grad():
                P = params["xyz"].shape[0]
                dead = int((torch.sigmoid(params["weight"]) <= 0.005).sum())
                diff = torch.abs(cells - gt)
                k = int(min(500_000, cap - P + dead + 1000, diff.numel()))
                if k > 0:
                    idx = torch.topk(diff, k).indices
                    newp = samples[idx]
                    d2n = torch.clamp_min(distCUDA2(torch.cat([params["xyz"].detach(), newp])) * 0.1, 1e-7)[P:]
                    ext = {"xyz": newp, "scaling": torch.log(torch.sqrt(d2n))[:, None].repeat(1, 3),
                           "rotation": torch.tensor([[1.0, 0, 0, 0]], device=dev).repeat(k, 1),
                           "weight": inv_sig(torch.full((k, 1), 0.01, device=dev)),
                           "value": inv_sig(gt[idx].clamp(1e-3, 1 - 1e-3))[:, None]}
                    replace({n: {"tensor": torch.cat([params[n].detach(), ext[n]]),
                                 "state": (lambda t, e=ext[n]: torch.cat([t, torch.zeros_like(e)]))} for n in params})
                keep = (torch.sigmoid(params["weight"]) >= 0.005).squeeze(1)
                replace({n: {"tensor": params[n].detach()[keep], "state": (lambda t, kk=keep: t[kk])} for n in params})

        def psnr():
            with torch.no_grad():
                rast.build_bvh(eval_pts)
                cells, _ = render()
                mse = torch.mean((cells - eval_gt) ** 2)
                return float(-10 * torch.log10(mse + 1e-8))

        hist = []
        t_train = 0.0
        reached = {}

        def record(it):
            ps = psnr()
            hist.append({"iteration": it, "train_s": t_train, "psnr_db": ps, "gaussians": int(params["xyz"].shape[0])})
            for thr in (30.0, 35.0, 40.0):
                if ps >= thr and str(thr) not in reached:
                    reached[str(thr)] = {"train_s": t_train, "iteration": it}

        torch.cuda.synchronize()
        record(0)
        for it in range(1, iters + 1):
            t0 = time.perf_counter()
            smp, gt = batches[it % nb]
            rast.build_bvh(smp)
            cells, weights = render()
            valid = (gt != -1) & (cells != -1)
            l1 = torch.abs(cells[valid] - gt[valid]).mean()
            fn_mask = (gt != -1) & (weights > 0.0) & (weights < 0.011)
            fn_vals = torch.clamp(0.011 - weights[fn_mask], min=0)
            loss = l1 + 0.5 * fn_vals.sum() / ((fn_vals > 0).sum().float() + 1e-8)
            loss.backward()
            if it % 100 == 0 and params["xyz"].shape[0] < cap:
                densify_and_prune(smp, cells.detach(), gt)
            else:
                opt.step()
            opt.zero_grad(set_to_none=True)
            torch.cuda.synchronize()
            t_train += time.perf_counter() - t0
            if it % 100 == 0 or it == iters or it in FIT_EVAL_AT:
                record(it)
        _C.check_status()
        results[path] = {"seconds_to_psnr_db": reached, "final_psnr_db": hist[-1]["psnr_db"],
                         "train_s": t_train, "ms_per_iteration": 1e3 * t_train / iters, "history": hist}
    _C.set_eval_path("plain")
    _C.set_backward_mode("auto")
    return {"volume": "%d^3 turbulent spectral field (256 modes, |k|^-5/3)" % n_vol, "initial_gaussians": P0,
            "paths_desc": {k: "eval path %s, backward %s" % v for k, v in FIT_PATHS.items() if k in paths},
            "cap": cap, "points_per_iteration": batch, "iterations": iters, "paths": results,
            "note": "capped run of %d iterations (the configuration states 3000); densify/prune every 100" % iters}


# ----------------------------------------------------------------------------------------
# Three-nearest-neighbour distances (distCUDA2 drop-in): device-resident points
# ----------------------------------------------------------------------------------------
def knn_bench(dev, means, steps, warmup, with_cpu):
    import torch
    from simple_knn._C import distCUDA2
    pts = means.to(dev).contiguous()
    n = int(pts.shape[0])
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        distCUDA2(pts)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        out = distCUDA2(pts)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    res = {"points": n, "ms_per_call": ms, "points_per_s": n / (ms * 1e-3),
           "includes": "point LBVH build (keys, sort, Karras, refit) + exact 3-NN traversal",
           "points_desc": "Gaussian means of the headline workload (256 clusters)"}
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        host = pts.cpu().numpy()
        t0 = time.perf_counter()
        ref = oracle.knn3_mean_dist2(host, nthreads=host_threads())
        t = time.perf_counter() - t0
        res["bit_exact_vs_oracle"] = bool(np.array_equal(ref, out.cpu().numpy()))
        res["cpu_oracle"] = {"ms_per_call": t * 1e3, "cores": host_threads(),
                             "sample": "oracle (C, OpenMP, uniform grid) on all %d points" % n}
    return res


# ----------------------------------------------------------------------------------------
# Our arm
# ----------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    import gvc_dist
    import gvc_native
    from bvh_diff_gaussian_rasterization import _C
    import bvh_diff_gaussian_rasterization as R

    rank, world, local = gvc_dist.init_from_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    means, scales, rots, values, weights, samples, desc = workload(args.config, rank)
    P, S = means.shape[0], samples.shape[0]
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    d_means, d_scales, d_rots, d_values, d_weights, d_samples = map(T, (means, scales, rots, values, weights, samples))
    d_gt = T(TARGETS[args.config]) if args.config in TARGETS else target_field(d_samples)
    zeros_w = torch.zeros(S, device=dev)
    ugb = bool(args.use_gaussian_bvh)
    _C.set_backward_mode(args.bwd_mode)
    _C.set_eval_path(args.eval_path)
    _C.set_traversal(args.traversal)
    bounds = (0.0, 0.0, 0.0, 1.0, 1.0, 1.0)

    def step():
        _C.build_bvh(d_samples, False, ugb)
        out, outw, conics = _C.rasterize_gaussians(d_means, d_scales, d_rots, d_values, d_weights, 1.0,
                                                   *bounds, -1.0, ugb, False)
        # masked L1 (train.py:389-396): d|cells - gt|.mean() over the valid mask
        mask = (out != -1) & (d_gt != -1)
        g = torch.where(mask, torch.sign(out - d_gt), torch.zeros_like(out)) / mask.sum().clamp_min(1)
        grads = _C.rasterize_gaussians_backward(d_means, d_scales, d_rots, conics, d_values, d_weights, out, outw,
                                                1.0, *bounds, -1.0, g, zeros_w, ugb, False)
        return gvc_dist.allreduce_grads(list(grads))

    # pair counts of this workload (one untimed step)
    _C.set_count_pairs(True)
    step()
    counts = _C.stats()
    _C.set_count_pairs(False)
    _C.check_status()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    _C.set_time_kernels(True)
    launches0 = gvc_native.launch_count()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = gvc_native.launch_count() - launches0
    kt = _C.stats()
    _C.set_time_kernels(False)
    _C.check_status()
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop() if clocks else None
    ms = gvc_dist.max_over_ranks(ms, dev)

    # roofline of the dominant evaluation kernel
    n_cand, n_fc, n_bc = counts["fwd_candidates"], counts["fwd_contributing"], counts["bwd_contributing"]
    f_fwd = F_CAND * n_cand + (F_FWD_CONTRIB - F_CAND + EX2_EQUIV) * n_fc
    f_bwd = F_CAND * n_cand + (F_BWD_CONTRIB - F_CAND + EX2_EQUIV) * n_bc
    t_fwd = kt["fwd_kernel_ms"] / max(kt["fwd_kernel_calls"], 1)
    t_bwd = kt["bwd_kernel_ms"] / max(kt["bwd_kernel_calls"], 1)
    hbm, bf16, bf16s, src = measured_peaks()
    bwd_kernel = "k_backward_cta" if args.bwd_mode == "tensor_core" or (
        args.eval_path == "tensor_core" and args.bwd_mode == "auto") else (
        "k_backward_tiles" if args.bwd_mode == "atomic" or (args.bwd_mode == "auto" and ugb) else "k_backward_gauss")
    fwd_kernel = "k_forward" if args.eval_path == "plain_tile" else "k_forward_cta"
    if t_bwd >= t_fwd:
        name, flops, t_k = bwd_kernel, f_bwd, t_bwd
    else:
        name, flops, t_k = fwd_kernel, f_fwd, t_fwd
    traffic = MEASURED_TRAFFIC.get((args.config, name))
    achieved = flops / (t_k * 1e-3) / 1e12
    # the two kinds of work, each against its own peak: tensor FLOPs the kernel issues
    # (split products, padded shapes included) and the algorithmic FP32 pair work
    tensor = None
    if name == "k_backward_cta":
        # per (candidate, row) element of a 16-row chunk: 5 split products x 2 x N (32 features)
        tf = counts["bwd_rows"] * 5 * 2 * 32
        tensor = {"flops_per_launch": tf, "achieved_tflops": tf / (t_k * 1e-3) / 1e12,
                  "frac_of_bf16_peak": tf / (t_k * 1e-3) / 1e12 / bf16,
                  "pipe_active_ncu_2M_x_4M": TENSOR_PIPE_ACTIVE.get(name),
                  "per_element": "5 split-BF16 products x 2 x 32 features per (Gaussian, row) of each 16-row chunk"}
    roofline = {"bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
                "frac": achieved / bf16, "traffic": traffic, "kernel": name, "kernel_ms": t_k,
                "achieved_kind": "algorithmic FP32-equivalent pair work (pair counts x FLOPs per pair, ex2 as 8) "
                                 "divided by the bf16 tensor peak; the tensor-pipe and FP32-pipe figures are "
                                 "reported separately in tensor_pipe and fp32_simt",
                "tensor_pipe": tensor,
                "fp32_simt": {"achieved_tflops": achieved, "nominal_tflops": FP32_NOMINAL_TFLOPS,
                              "frac": achieved / FP32_NOMINAL_TFLOPS},
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one full-size launch"
                                  if traffic else None,
                "peak_source": ("measured bf16 dense burst (MEASURED_PEAKS.json)" if src == "measured" else
                                "fallback bf16 dense 1.59 PFLOP/s (MEASURED_PEAKS.json absent)"),
                "fp32_simt_nominal_tflops": FP32_NOMINAL_TFLOPS,
                "frac_of_fp32_simt_nominal": achieved / FP32_NOMINAL_TFLOPS,
                "fwd_kernel_ms": t_fwd, "bwd_kernel_ms": t_bwd,
                "pairs": {"candidates": n_cand, "fwd_contributing": n_fc, "bwd_contributing": n_bc,
                          "fwd_tile_gaussian_evals": counts["fwd_leaf_hits"],
                          "fwd_node_visits": counts["fwd_node_visits"],
                          "bwd_leaf_evals": counts["bwd_leaf_hits"],
                          "bwd_node_visits": counts["bwd_node_visits"],
                          "fwd_lane_evals": counts["fwd_lane_evals"], "bwd_rows": counts["bwd_rows"]},
                "flops_per_pair": {"candidate": F_CAND, "fwd_contributing": F_FWD_CONTRIB,
                                   "bwd_contributing": F_BWD_CONTRIB, "ex2_fp32_equiv": EX2_EQUIV}}

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e and not args.profile:
        h_samples = torch.from_numpy(samples).pin_memory()
        # the target values travel with their samples, as the training loop's sorted
        # (samples, ground truth) batches do (train.py:286-315)
        h_gt = (torch.from_numpy(TARGETS[args.config]) if args.config in TARGETS else
                target_field(torch.from_numpy(samples))).pin_memory()
        h_params = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
                    for a in (means, scales, rots, values.reshape(-1, 1), weights.reshape(-1, 1))]
        settings = R.GaussianRasterizationSettings((0, 0, 0), (1, 1, 1), 0, -1.0, 1.0, ugb, False)
        rast = R.GaussianRasterizer(settings)
        h2d = h_samples.numel() * 4 + h_gt.numel() * 4 + sum(p.numel() * 4 for p in h_params)

        # double-buffered uploads: the inputs of step k + 1 are copied on a second stream
        # while step k computes (every step's copy is inside the timed region)
        copy_stream = torch.cuda.Stream(dev)
        hosts = [h_samples, h_gt] + h_params
        bufs = [[torch.empty(h.shape, dtype=h.dtype, device=dev) for h in hosts] for _ in range(2)]
        ready = [torch.cuda.Event(), torch.cuda.Event()]
        # each step's loss lands in pinned memory; the host reads step k's value after step
        # k + 1 is queued, so the GPU is not idle while the host reads
        h_loss = [torch.zeros(1, dtype=torch.float32).pin_memory() for _ in range(2)]
        loss_done = [torch.cuda.Event(), torch.cuda.Event()]
        losses = []

        def issue_copy(b):
            copy_stream.wait_stream(stream)  # the buffer's previous step has finished with it
            with torch.cuda.stream(copy_stream):
                for d_, h in zip(bufs[b], hosts):
                    d_.copy_(h, non_blocking=True)
                ready[b].record(copy_stream)

        def e2e_step(k, n):
            b = k % 2
            stream.wait_event(ready[b])
            if k + 1 < n:
                issue_copy(1 - b)
            s_d, gt = bufs[b][0], bufs[b][1]
            leaves = [p.detach().requires_grad_(True) for p in bufs[b][2:]]
            rast.build_bvh(s_d)
            cells, cw = rast(leaves[0], leaves[1], leaves[2], leaves[3], leaves[4])
            # masked mean without boolean indexing (no device-to-host size query)
            mask = ((cells != -1) & (gt != -1)).float()
            loss = (torch.abs(cells - gt) * mask).sum() / mask.sum().clamp_min(1.0)
            loss.backward()
            if world > 1:
                gvc_dist.allreduce_grads([l.grad for l in leaves])
            h_loss[b].copy_(loss.detach().reshape(1), non_blocking=True)
            loss_done[b].record(stream)
            if k > 0:  # the previous step's result, read while this step runs
                loss_done[1 - b].synchronize()
                losses.append(float(h_loss[1 - b][0]))

        def e2e_run(n):
            issue_copy(0)
            for k in range(n):
                e2e_step(k, n)
            loss_done[(n - 1) % 2].synchronize()
            losses.append(float(h_loss[(n - 1) % 2][0]))

        e2e_run(max(1, args.warmup))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n_e2e = max(3, min(args.steps, 10))
        a0.record(stream)
        e2e_run(n_e2e)
        a1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = gvc_dist.max_over_ranks(a0.elapsed_time(a1) / n_e2e, dev)
        e2e = {"value": e2e_ms, "unit": "ms/step", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 4,
               "steps": n_e2e, "last_loss": losses[-1],
               "path": "GaussianRasterizer (autograd) + masked L1; every step uploads its pinned host inputs "
                       "(samples, their target values, parameters; double-buffered on a copy stream) and "
                       "reads its loss back to pinned host memory (checked on the host while the next step runs)"}

    # the two evaluation paths side by side: full step time, forward outputs and the
    # gradients of one step (kept on the host for the FP64 comparisons below)
    paths = {}
    grad_runs = {}
    paths_extra = {}
    if not args.profile:
        # (forward path, backward mode, traversal, candidate log): FP32 throughout, tensor cores
        # throughout, the FP32 forward with the tensor-core backward reduction, and (timed
        # only) that with the backward walking the tree again instead of reading the forward's
        # candidate log, and with the stackless Gaussian-LBVH traversal in both kernels
        for name, path, bmode, trav, clog in (("plain", "plain", "auto", "stack", True),
                                              ("tensor_core", "tensor_core", "auto", "stack", True),
                                              ("plain_fwd_tc_bwd", "plain", "tensor_core", "stack", True),
                                              ("walk", "plain", "tensor_core", "stack", False),
                                              ("stackless", "plain", "tensor_core", "stackless", False)):
            _C.set_eval_path(path)
            _C.set_backward_mode(bmode)
            _C.set_traversal(trav)
            _C.set_candidate_log(clog)
            for _ in range(2):
                step()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            b0.record(stream)
            for _ in range(args.steps):
                step()
            b1.record(stream)
            torch.cuda.synchronize()
            pm = gvc_dist.max_over_ranks(b0.elapsed_time(b1) / args.steps, dev)
            if name in ("walk", "stackless"):
                paths_extra["plain_fwd_tc_bwd_%s_ms_per_step" % name] = pm
                continue
            # one more step, outputs and gradients kept (untimed)
            _C.build_bvh(d_samples, False, ugb)
            o, ow, cn = _C.rasterize_gaussians(d_means, d_scales, d_rots, d_values, d_weights, 1.0, *bounds, -1.0,
                                               ugb, False)
            mask = (o != -1) & (d_gt != -1)
            gl = torch.where(mask, torch.sign(o - d_gt), torch.zeros_like(o)) / mask.sum().clamp_min(1)
            gr = _C.rasterize_gaussians_backward(d_means, d_scales, d_rots, cn, d_values, d_weights, o, ow, 1.0,
                                                 *bounds, -1.0, gl, zeros_w, ugb, False)
            _C.check_status()
            run = {"ms_per_step": pm, "out": o.cpu().numpy(), "outw": ow.cpu().numpy(),
                   "conics": cn.cpu().numpy().reshape(-1, 6), "gout": gl.cpu().numpy(),
                   "grads": [x.cpu().numpy() for x in gr]}
            grad_runs[name] = run
            if name == "plain_fwd_tc_bwd":
                paths_extra["plain_fwd_tc_bwd_ms_per_step"] = pm
                continue
            paths[name] = run
        _C.set_eval_path(args.eval_path)
        _C.set_backward_mode(args.bwd_mode)
        _C.set_traversal(args.traversal)
        _C.set_candidate_log(True)
        _C.check_status()

    cpu = None
    fp64 = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile:
        cpu = cpu_baseline(means, scales, rots, values, weights, samples)
        fp64 = fp64_errors(means, scales, rots, values, weights, samples, paths)
        fp64["gradients"] = grad_errors(means, scales, rots, values, weights, samples, grad_runs)
    tc_vs_plain = None
    if paths:
        tc_vs_plain = {"plain_ms_per_step": paths["plain"]["ms_per_step"],
                       "tensor_core_ms_per_step": paths["tensor_core"]["ms_per_step"],
                       "speedup_tc_over_plain": paths["plain"]["ms_per_step"] / paths["tensor_core"]["ms_per_step"],
                       "paths": {"plain": "FP32 CTA forward + FP32 deterministic Gaussian-owned backward",
                                 "tensor_core": "tcgen05 split-BF16 exponent forward + tcgen05 moment backward",
                                 "plain_fwd_tc_bwd": "FP32 CTA forward + tcgen05 moment backward",
                                 "plain_fwd_tc_bwd_walk": "the same with the backward walking the Gaussian "
                                                          "LBVH again instead of reading the forward's "
                                                          "candidate log",
                                 "plain_fwd_tc_bwd_stackless": "the same walking in both kernels by the "
                                                               "stackless traversal (escape edges)"},
                       "fp64_error": fp64}
        tc_vs_plain.update(paths_extra)

    if rank == 0:
        line = {"metric": METRIC, "value": ms, "unit": "ms/step", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_dict(args, desc, P, S, world),
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "e2e": e2e, "tc_vs_plain": tc_vs_plain,
                "gpu_launches": int(launches), "gpu_launches_per_step": launches / args.steps}
        if args.knn and world == 1:
            line["knn3"] = knn_bench(dev, d_means, 10, 3, not args.no_cpu_baseline)
        if args.mesh and world == 1:
            line["mesh_sampler"] = mesh_bench(dev, 5, 2, not args.no_cpu_baseline)
        if args.fit and world == 1:
            line["fit"] = fit_bench(dev, args.fit)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
