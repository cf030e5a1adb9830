"""bench.py's reference arm runs on the host cores (the reference's kernels compiled for
the host, or the oracle), so its JSON contract is checked here without a GPU: one line
with the metric, the CPU baseline description, a zero-copy e2e object and the same config
object as our arm; ranks other than 0 print nothing and exit 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "tiny",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [l for l in r.stdout.splitlines() if l.strip()]


def test_reference_arm_line():
    lines = _run({"RANK": "0"})
    assert len(lines) == 1
    line = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["unit"] == "ms/step" and line["steps"] == 1 and line["warmup"] == 3
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "ms/step", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert "workload" in line["config"]
    assert line["extrapolated"] is False and cb["extrapolated"] is False
    # the same config object as our arm prints for the same arguments
    sys.path.insert(0, ROOT)
    import bench
    ns = type("A", (), {"eval_path": "plain", "bwd_mode": "tensor_core", "use_gaussian_bvh": False,
                       "traversal": "stack"})()
    P, S, desc = bench.CONFIGS["tiny"]
    assert line["config"] == bench.config_dict(ns, desc, P, S, 1)


def test_reference_arm_other_ranks_are_silent():
    assert _run({"RANK": "1"}) == []
