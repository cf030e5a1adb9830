"""Multi-rank host logic on CPU (gloo, world size 2): samples sharded across ranks, each
rank computes the per-Gaussian adjoint of its shard (the oracle stands in for the GPU
kernels here), one all-reduce sums them; the result equals the single-process adjoint."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    sys.path[:0] = [os.path.join(ROOT, "gaussian-volume-compression_b200"), os.path.join(ROOT, "oracle")]
    import torch
    import torch.distributed as dist
    import gvc_dist
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    r, w, _ = gvc_dist.init_from_env(backend="gloo", timeout_s=60)
    means, scales, rots, values, weights = oracle.mixture_small(seed=2, P=256)
    samples = oracle.grid_centres(16)
    lo, hi = gvc_dist.shard_range(samples.shape[0], r, w)
    _, c64, bb = oracle.preprocess(means, scales, rots, weights)
    mine = samples[lo:hi]
    out, outw = oracle.forward(means, values, weights, c64, bb, mine, nthreads=1)
    gout = np.ones(mine.shape[0], np.float32)
    g = oracle.backward(means, values, weights, c64, bb, mine, out.astype(np.float32), outw.astype(np.float32),
                        gout, np.zeros(mine.shape[0], np.float32), nthreads=1)
    grads = [torch.tensor(g["dmeans"]), torch.tensor(g["dvalues"]), torch.tensor(g["dweights"])]
    red = gvc_dist.allreduce_grads(grads)
    t = gvc_dist.max_over_ranks(float(r))
    if r == 0:
        q.put(([x.numpy() for x in red], t, (lo, hi)))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_adjoint_allreduce_matches_single_process(orc):
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    red, tmax, rng0 = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert tmax == 1.0 and rng0 == (0, 2048)
    means, scales, rots, values, weights = orc.mixture_small(seed=2, P=256)
    samples = orc.grid_centres(16)
    _, c64, bb = orc.preprocess(means, scales, rots, weights)
    out, outw = orc.forward(means, values, weights, c64, bb, samples)
    g = orc.backward(means, values, weights, c64, bb, samples, out.astype(np.float32), outw.astype(np.float32),
                     np.ones(samples.shape[0], np.float32), np.zeros(samples.shape[0], np.float32))
    for a, b in zip(red, (g["dmeans"], g["dvalues"], g["dweights"])):
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-12)


def test_shard_ranges_cover_everything():
    sys.path.insert(0, os.path.join(ROOT, "gaussian-volume-compression_b200"))
    import gvc_dist
    for n in (0, 1, 7, 32, 1000):
        for w in (1, 2, 3, 8):
            r = [gvc_dist.shard_range(n, k, w) for k in range(w)]
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(r[k][1] == r[k + 1][0] for k in range(w - 1))
            assert max(b - a for a, b in r) - min(b - a for a, b in r) <= 1
