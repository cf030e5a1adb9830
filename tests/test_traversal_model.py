"""Stackless LBVH traversal (escape edges): a CPU model of the device algorithm.

The device code (warp_traverse_stackless in csrc/traverse.cuh, escape edges written by
k_pack_nodes in csrc/lbvh.cu) has no counterpart in the reference, whose queries go
through cuBQL's fixedBoxQuery (diff-gaussian-rasterization/cuda_rasterizer/forward.cu:150,
209).  These tests restate the algorithm step for step in Python over the oracle's LBVH
(the topology the GPU builder reproduces bit for bit) and check, for random query boxes
of every size, that it hands over each overlapping leaf exactly once and nothing else,
and that every lane's walk ends within the bound the kernel enforces.  The GPU tests
(test_gpu_traversal.py) check the device's escape edges against escape_edges() below
and the kernels' results against the oracle.
"""
import numpy as np
import pytest

LEAF = np.uint32(0x80000000)
END = 0xFFFFFFFF


def escape_edges(left, right):
    """Per internal node k: the edge after k's subtree in pre-order, 2p + 1 for the nearest
    ancestor-or-self of k that is the left child of p, END on the root's right spine."""
    n1 = len(left)
    lu, ru = left.view(np.uint32), right.view(np.uint32)
    parent = np.full(n1, -1, np.int64)
    for k in range(n1):
        for c in (lu[k], ru[k]):
            if not c & LEAF:
                parent[c] = k
    esc = np.empty(n1, np.uint64)
    for k in range(n1):
        x, p = k, parent[k]
        while p >= 0 and ru[p] == x:
            x, p = p, parent[p]
        esc[k] = END if p < 0 else 2 * p + 1
    return esc


class Tree:
    def __init__(self, boxes, orc):
        keys, perm, left, right, nb = orc.lbvh_build(boxes)
        self.left, self.right = left.view(np.uint32), right.view(np.uint32)
        self.leaf_boxes = boxes[perm]
        self.node_boxes = nb
        self.esc = escape_edges(left, right)
        self.n1 = len(left)

    def child_box(self, c):
        return self.leaf_boxes[c & ~LEAF] if c & LEAF else self.node_boxes[c]


def overlap(b, q):
    return bool(np.all(b[:3] <= q[3:]) and np.all(b[3:] >= q[:3]))


def stackless_query(t, q):
    """Returns (leaves handed over, in order; longest lane walk in edges; levels)."""
    out = []
    frontier = [0]
    walk = False
    levels = 0
    while frontier:
        levels += 1
        assert levels <= t.n1 + 1
        hits = []
        for k in frontier:  # lane order
            cl, cr = t.left[k], t.right[k]
            hits.append((cl, overlap(t.child_box(cl), q), cr, overlap(t.child_box(cr), q)))
        il = [cl for cl, hl, _, _ in hits if hl and not cl & LEAF]
        ir = [cr for _, _, cr, hr in hits if hr and not cr & LEAF]
        if len(il) + len(ir) > 32:
            walk = True
            break
        out += [int(cl & ~LEAF) for cl, hl, _, _ in hits if hl and cl & LEAF]
        out += [int(cr & ~LEAF) for _, _, cr, hr in hits if hr and cr & LEAF]
        frontier = [int(c) for c in il + ir]
    longest = 0
    if walk:
        assert len(frontier) <= 32
        for f in frontier:  # one lane each; the device runs them in lock step
            cur, stop, steps = 2 * f, int(t.esc[f]), 0
            while cur != stop:
                steps += 1
                assert steps <= 2 * t.n1
                k, s = cur >> 1, cur & 1
                child = t.right[k] if s else t.left[k]
                hit = overlap(t.child_box(child), q)
                if hit and not child & LEAF:
                    cur = 2 * int(child)
                else:
                    if hit:
                        out.append(int(child & ~LEAF))
                    cur = int(t.esc[k]) if s else cur | 1
            longest = max(longest, steps)
    return out, longest, levels


def brute(t, q):
    lb = t.leaf_boxes
    m = np.all(lb[:, :3] <= q[3:], 1) & np.all(lb[:, 3:] >= q[:3], 1)
    return set(np.nonzero(m)[0].tolist())


def make_boxes(n, kind, seed):
    rng = np.random.default_rng(seed)
    c = rng.random((n, 3)).astype(np.float32)
    if kind == "dup":
        c = (np.round(c * 8) / 8).astype(np.float32)
    if kind == "cluster":
        c = (0.5 + 0.05 * rng.normal(size=(n, 3))).astype(np.float32)
    e = (rng.random((n, 3)) * 0.02).astype(np.float32)
    return np.concatenate([c - e, c + e], 1).astype(np.float32)


@pytest.mark.parametrize("n,kind", [(2, "rand"), (3, "rand"), (33, "rand"), (1000, "rand"), (4097, "dup"),
                                    (6000, "cluster")])
def test_escape_edges_follow_preorder(orc, n, kind):
    """Walking edge to edge from (0, 0) by the rule visits every edge once, in pre-order."""
    t = Tree(make_boxes(n, kind, n), orc)
    order = []
    stack = [(0, 1), (0, 0)]
    while stack:
        k, s = stack.pop()
        order.append(2 * k + s)
        c = t.right[k] if s else t.left[k]
        if not c & LEAF:
            stack += [(int(c), 1), (int(c), 0)]
    walked, cur = [], 0
    while cur != END:
        walked.append(cur)
        k, s = cur >> 1, cur & 1
        c = t.right[k] if s else t.left[k]
        cur = 2 * int(c) if not c & LEAF else (int(t.esc[k]) if s else cur | 1)
        assert len(walked) <= 2 * t.n1
    assert walked == order


@pytest.mark.parametrize("n,kind", [(2, "rand"), (33, "rand"), (1000, "rand"), (4097, "dup"), (20000, "rand"),
                                    (20000, "cluster")])
def test_stackless_query_finds_each_overlapping_leaf_once(orc, n, kind):
    t = Tree(make_boxes(n, kind, 7 + n), orc)
    rng = np.random.default_rng(n)
    walked = 0
    for i in range(60):
        c = rng.random(3).astype(np.float32)
        h = np.float32(10.0 ** rng.uniform(-3, -0.3))  # from a few leaves to most of the tree
        q = np.concatenate([c - h, c + h]).astype(np.float32)
        got, longest, levels = stackless_query(t, q)
        assert len(got) == len(set(got))
        assert set(got) == brute(t, q)
        walked += longest > 0
    if n >= 1000:
        assert walked > 0  # the per-lane phase ran
