"""Seeded synthetic workloads of the benchmark configurations.

The reference measures on no public dataset (its trained meshes are not shipped), so
every configuration is a seeded synthetic stand-in with the shapes, sizes and value
distributions the configuration names.  Used by bench.py and by the tests.
"""
import numpy as np


def mixture_small(seed=0, P=4096):
    """Config 1: P anisotropic Gaussians, mu ~ U[0,1]^3, log-scales ~ N(log 0.02, 0.3),
    random unit quaternions, w = sigmoid(N(0,1)), v ~ U[0,1] (activated, float32)."""
    rng = np.random.default_rng(seed)
    means = rng.random((P, 3), dtype=np.float32)
    scales = np.exp(rng.normal(np.log(0.02), 0.3, (P, 3))).astype(np.float32)
    q = rng.normal(size=(P, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    weights = (1.0 / (1.0 + np.exp(-rng.normal(size=P)))).astype(np.float32)
    values = rng.random(P, dtype=np.float32)
    return means, scales, q.astype(np.float32), values, weights


def grid_centres(n=64):
    """The n^3 cell centres (i + 0.5) / n of [0,1]^3 (x fastest)."""
    c = (np.arange(n, dtype=np.float32) + 0.5) / n
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.float32)


def blob_target(samples, seed=0, nblobs=16):
    """Config 1 target: sum of isotropic blobs (centres U[0,1]^3, sigma U[0.05,0.15],
    amplitude U[0.5,1])."""
    rng = np.random.default_rng(seed + 1000)
    c = rng.random((nblobs, 3))
    sg = rng.uniform(0.05, 0.15, nblobs)
    a = rng.uniform(0.5, 1.0, nblobs)
    d2 = ((samples[:, None, :].astype(np.float64) - c[None]) ** 2).sum(-1)
    return (a[None] * np.exp(-0.5 * d2 / sg[None] ** 2)).sum(-1)


def mixture_large(seed=0, P=2_000_000, S=16_000_000):
    """Config 4: P Gaussians clustered around 256 centres (sigma 0.05, clamped to
    [0,1]), log-scales ~ N(log 0.004, 0.4), random quaternions, v ~ U[0,1],
    w = sigmoid(N(0,1)); S/2 uniform samples + S/2 samples at mu_j + N(0, s_j^2)."""
    rng = np.random.default_rng(seed)
    centres = rng.random((256, 3))
    lab = rng.integers(0, 256, P)
    means = np.clip(centres[lab] + rng.normal(0, 0.05, (P, 3)), 0, 1).astype(np.float32)
    scales = np.exp(rng.normal(np.log(0.004), 0.4, (P, 3))).astype(np.float32)
    q = rng.normal(size=(P, 4)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    values = rng.random(P, dtype=np.float32)
    weights = (1.0 / (1.0 + np.exp(-rng.normal(size=P)))).astype(np.float32)
    half = S // 2
    uni = rng.random((half, 3), dtype=np.float32)
    j = rng.integers(0, P, S - half)
    near = (means[j] + rng.normal(size=(S - half, 3)).astype(np.float32) * scales[j]).astype(np.float32)
    samples = np.concatenate([uni, near], axis=0)
    return means, scales, q, values, weights, samples


def volume_blobs_sine(n=256, seed=0, nblobs=64, device="cpu"):
    """Config 2 volume: an n^3 float32 point field on the lattice i / (n - 1) of [0,1]^3
    (x fastest), the sum of `nblobs` random anisotropic Gaussian blobs (centres U[0,1]^3,
    standard deviations U[0.03, 0.1] per axis, random rotation, amplitude U[0.5, 1]) plus
    0.1 sin(8 pi x) sin(8 pi y) sin(8 pi z), mapped linearly onto [0.01, 0.99] (the
    values initialise Gaussian values through the inverse sigmoid, so they must stay
    inside (0, 1)).  Computed with torch on `device` (a CUDA device makes 256^3 fast)."""
    import torch
    rng = np.random.default_rng(seed + 2000)
    c = torch.tensor(rng.random((nblobs, 3)), dtype=torch.float32, device=device)
    sd = rng.uniform(0.03, 0.1, (nblobs, 3))
    q = rng.normal(size=(nblobs, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    r, x, y, z = q.T
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - r * z), 2 * (x * z + r * y)], -1),
                  np.stack([2 * (x * y + r * z), 1 - 2 * (x * x + z * z), 2 * (y * z - r * x)], -1),
                  np.stack([2 * (x * z - r * y), 2 * (y * z + r * x), 1 - 2 * (x * x + y * y)], -1)], -2)
    prec = np.einsum("bij,bj,bkj->bik", R, 1.0 / sd ** 2, R)  # Sigma^-1 = R diag(1/s^2) R^T
    prec = torch.tensor(prec, dtype=torch.float32, device=device)
    amp = torch.tensor(rng.uniform(0.5, 1.0, nblobs), dtype=torch.float32, device=device)
    t = torch.arange(n, dtype=torch.float32, device=device) / (n - 1)
    out = torch.empty(n, n, n, dtype=torch.float32, device=device)  # [z][y][x]
    zz, yy, xx = torch.meshgrid(t, t, t, indexing="ij")
    pts = torch.stack([xx, yy, zz], -1).reshape(-1, 3)
    acc = torch.zeros(pts.shape[0], dtype=torch.float32, device=device)
    chunk = 1 << 21
    for a in range(0, pts.shape[0], chunk):
        p = pts[a:a + chunk]
        for b in range(nblobs):
            d = p - c[b]
            acc[a:a + chunk] += amp[b] * torch.exp(-0.5 * ((d @ prec[b]) * d).sum(-1))
    acc += 0.1 * torch.sin(8 * np.pi * pts[:, 0]) * torch.sin(8 * np.pi * pts[:, 1]) * torch.sin(8 * np.pi * pts[:, 2])
    lo, hi = acc.min(), acc.max()
    out = (0.01 + 0.98 * (acc - lo) / (hi - lo)).reshape(n, n, n)
    return out


def volume_turbulent(n=512, seed=0, modes=256, kmax=32, device="cpu"):
    """Config 5 volume: an n^3 float32 point field on the lattice i / (n - 1) of [0,1]^3
    (x fastest), a spectral sum of `modes` random Fourier modes
    sum_m |k_m|^(-5/3) cos(2 pi k_m . x + phi_m) with integer wave vectors k_m uniform in
    [-kmax, kmax]^3 other than 0 and phases U[0, 2 pi), normalised to [0, 1]."""
    import torch
    rng = np.random.default_rng(seed + 3000)
    k = rng.integers(-kmax, kmax + 1, (modes, 3))
    k[np.all(k == 0, axis=1)] = [1, 0, 0]
    amp = np.linalg.norm(k, axis=1) ** (-5.0 / 3.0)
    phi = rng.uniform(0, 2 * np.pi, modes)
    K = torch.tensor(2 * np.pi * k, dtype=torch.float32, device=device)
    A = torch.tensor(amp, dtype=torch.float32, device=device)
    Ph = torch.tensor(phi, dtype=torch.float32, device=device)
    t = torch.arange(n, dtype=torch.float32, device=device) / (n - 1)
    out = torch.empty(n ** 3, dtype=torch.float32, device=device)
    plane = n * n
    yy, xx = torch.meshgrid(t, t, indexing="ij")
    xy = torch.stack([xx.reshape(-1), yy.reshape(-1)], 1)
    for z in range(n):
        p = torch.cat([xy, torch.full((plane, 1), float(t[z]), device=device)], 1)
        out[z * plane:(z + 1) * plane] = torch.cos(p @ K.T + Ph) @ A
    lo, hi = out.min(), out.max()
    return ((out - lo) / (hi - lo)).reshape(n, n, n)


def lattice_init(volume, P, seed=0):
    """Config 2 initial mixture positions: P distinct random lattice points of the volume
    (its voxel centres on [0,1]^3) and the volume's values there; returns (points [P,3]
    float32, values [P] float32) on the volume's device."""
    import torch
    n = volume.shape[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    idx = torch.randperm(n ** 3, generator=g)[:P].to(volume.device)
    x, y, z = idx % n, (idx // n) % n, idx // (n * n)
    pts = torch.stack([x, y, z], 1).float() / (n - 1)
    return pts.contiguous(), volume.reshape(-1)[idx].contiguous()


def jittered_tet_mesh(n=16, seed=0, jitter=0.2):
    """Config 3 geometry: an n^3 hex grid on [0,1]^3, interior vertices jittered by
    U[-jitter, jitter]*h, each hex split into 6 tets along its main diagonal (Kuhn
    split: vertex 0 -> 7 of every tet, declared).  Returns (pts [V,3] f32, tets [C,4])."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    c = np.arange(n + 1) * h
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    pts = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    interior = np.all((pts > 0.5 * h) & (pts < 1 - 0.5 * h), axis=1)
    pts[interior] += rng.uniform(-jitter, jitter, (interior.sum(), 3)) * h
    pts = pts.astype(np.float32)
    N1 = n + 1
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()

    def vid(di, dj, dk):
        return (k + dk) * N1 * N1 + (j + dj) * N1 + (i + di)

    v = [vid(0, 0, 0), vid(1, 0, 0), vid(0, 1, 0), vid(1, 1, 0), vid(0, 0, 1), vid(1, 0, 1), vid(0, 1, 1), vid(1, 1, 1)]
    # the six monotone lattice paths from corner 0 to corner 7 (x=1, y=2, z=4 bit steps)
    paths = [(1, 2, 4), (1, 4, 2), (2, 1, 4), (2, 4, 1), (4, 1, 2), (4, 2, 1)]
    tets = []
    for a, b, _ in paths:
        tets.append(np.stack([v[0], v[a], v[a | b], v[7]], axis=1))
    tets = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int64)
    return pts, tets


def mixed_cell_mesh(n=6, seed=0, jitter=0.2, kinds=(12, 13, 14, 10), extras=True):
    """A conforming mixed explicit mesh in VTK layout over an n^3 hex grid on [0,1]^3.
    Each (i, j) column of hexes is one kind: 12 a hexahedron per grid cell, 13 two wedges
    split along the cell's (1, 3) diagonal, 14 six pyramids on the cell's faces with the
    cell centre as apex, 10 the six Kuhn tetrahedra.  Columns keep shared faces conforming
    (hex, wedge-side and pyramid-base faces are the same bilinear quads; triangles meet
    triangles).  Tetrahedra split quads into triangles, so with 10 among the kinds the grid
    is mapped by a random affine map instead of jittered (every quad stays planar).
    extras appends zero-volume cells (VTK 1, 3, 5, 9) that never contain a point.
    Returns (pts [V,3] f32, conn int64, types int64 [C], offsets int64 [C+1])."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    c = np.arange(n + 1) * h
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    grid = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    if 10 in kinds:
        A = np.eye(3) + rng.uniform(-0.25, 0.25, (3, 3))
        grid = grid @ A.T + rng.uniform(-1, 1, 3)
    else:
        interior = np.all((grid > 0.5 * h) & (grid < 1 - 0.5 * h), axis=1)
        grid[interior] += rng.uniform(-jitter, jitter, (interior.sum(), 3)) * h
    N1 = n + 1

    def vid(i, j, k):
        return (k * N1 + j) * N1 + i

    centres = []
    conn, types = [], []
    col_kind = rng.choice(np.asarray(kinds), size=(n, n))
    for k in range(n):
        for j in range(n):
            for i in range(n):
                hx = [vid(i, j, k), vid(i + 1, j, k), vid(i + 1, j + 1, k), vid(i, j + 1, k),
                      vid(i, j, k + 1), vid(i + 1, j, k + 1), vid(i + 1, j + 1, k + 1), vid(i, j + 1, k + 1)]
                kind = int(col_kind[j, i])
                if kind == 12:
                    conn.append(hx); types.append(12)
                elif kind == 13:
                    conn.append([hx[0], hx[1], hx[3], hx[4], hx[5], hx[7]]); types.append(13)
                    conn.append([hx[1], hx[2], hx[3], hx[5], hx[6], hx[7]]); types.append(13)
                elif kind == 14:
                    apex = grid.shape[0] + len(centres)
                    centres.append(grid[hx].mean(axis=0))
                    for f in ((0, 1, 2, 3), (4, 7, 6, 5), (0, 4, 5, 1), (3, 2, 6, 7), (0, 3, 7, 4), (1, 5, 6, 2)):
                        conn.append([hx[q] for q in f] + [apex]); types.append(14)
                else:
                    lat = [vid(i + (b & 1), j + ((b >> 1) & 1), k + ((b >> 2) & 1)) for b in range(8)]
                    for a, b in ((1, 2), (1, 4), (2, 1), (2, 4), (4, 1), (4, 2)):
                        conn.append([lat[0], lat[a], lat[a | b], lat[7]]); types.append(10)
    pts = np.concatenate([grid, np.asarray(centres).reshape(-1, 3)]) if centres else grid
    if extras:
        V = grid.shape[0]
        for t, m in ((1, 1), (3, 2), (5, 3), (9, 4)):
            at = int(rng.integers(0, len(conn) + 1))
            conn.insert(at, [int(q) for q in rng.integers(0, V, m)]); types.insert(at, t)
    offsets = np.zeros(len(conn) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum([len(q) for q in conn])
    flat = np.asarray([q for cc in conn for q in cc], dtype=np.int64)
    return pts.astype(np.float32), flat, np.asarray(types, dtype=np.int64), offsets


def blob_field(pts, seed=0, nblobs=32):
    rng = np.random.default_rng(seed + 7)
    c = rng.random((nblobs, 3))
    sg = rng.uniform(0.05, 0.2, nblobs)
    a = rng.uniform(0.2, 1.0, nblobs)
    d2 = ((pts[:, None, :].astype(np.float64) - c[None]) ** 2).sum(-1)
    return (a[None] * np.exp(-0.5 * d2 / sg[None] ** 2)).sum(-1).astype(np.float32)
