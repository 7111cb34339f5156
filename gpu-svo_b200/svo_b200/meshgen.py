"""Seeded synthetic meshes for the benchmark workloads.

No public dataset is involved; every mesh is generated from a fixed seed:

  icosphere_l5   icosahedron subdivided 5x (10,242 vertices, 20,480 triangles),
                 each vertex radius scaled by 1+U(-0.02, 0.02) (seed 0),
                 bbox-normalised to the unit cube; built at resolution 128.
  torus_slivers  1,000,000-triangle soup (seed 1): 900,000 triangles from a
                 900x500-quad torus (R=0.35, r=0.12, centred in the unit cube)
                 with Gaussian vertex jitter of sigma = 0.01*r, then 100,000
                 sliver triangles inside the unit cube (length U(0.005, 0.05),
                 aspect ratio U(50, 500), random orientation); resolution 512.
  heightfield    z = 0.5 + sum of 16 sinusoids (amplitude U(0, 0.03), wave
                 number U(1, 40), direction and phase uniform; seed 2) on a
                 1582x1582 vertex grid over [0,1]^2: 4,999,122 triangles;
                 resolution 2048.
  batch          256 meshes (seed 3): jittered icospheres (level 2-6) or
                 jittered tori, triangle counts log-uniform in [320, 80000],
                 resolution drawn from {64, 128, 256, 512}.
"""
from __future__ import annotations

import numpy as np

_PHI = (1.0 + 5.0 ** 0.5) / 2.0
_ICO_V = np.array(
    [[-1, _PHI, 0], [1, _PHI, 0], [-1, -_PHI, 0], [1, -_PHI, 0],
     [0, -1, _PHI], [0, 1, _PHI], [0, -1, -_PHI], [0, 1, -_PHI],
     [_PHI, 0, -1], [_PHI, 0, 1], [-_PHI, 0, -1], [-_PHI, 0, 1]], dtype=np.float64)
_ICO_F = np.array(
    [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
     [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
     [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
     [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)


def icosphere(level: int):
    """Unit icosphere by midpoint subdivision with re-projection."""
    v = _ICO_V / np.linalg.norm(_ICO_V, axis=1, keepdims=True)
    f = _ICO_F.copy()
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mid])
        nf = f.shape[0]
        m01, m12, m20 = (base + inv[:nf], base + inv[nf:2 * nf], base + inv[2 * nf:])
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f


def _normalise(v: np.ndarray) -> np.ndarray:
    lo, hi = v.min(0), v.max(0)
    return (v - lo) / (hi - lo).max()


def jittered_icosphere(level: int, rng: np.random.Generator, jitter: float = 0.02):
    v, f = icosphere(level)
    v = v * (1.0 + rng.uniform(-jitter, jitter, size=(v.shape[0], 1)))
    return _normalise(v).astype(np.float32), f.astype(np.int32)


def torus(nu: int, nv: int, R: float, r: float, rng: np.random.Generator, sigma: float,
          center=(0.5, 0.5, 0.5)):
    u = np.arange(nu) * (2 * np.pi / nu)
    w = np.arange(nv) * (2 * np.pi / nv)
    U, W = np.meshgrid(u, w, indexing="ij")
    x = (R + r * np.cos(W)) * np.cos(U)
    y = (R + r * np.cos(W)) * np.sin(U)
    z = r * np.sin(W)
    v = np.stack([x, y, z], -1).reshape(-1, 3) + np.asarray(center)
    v += rng.normal(0.0, sigma, size=v.shape)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    a = (i * nv + j)
    b = (((i + 1) % nu) * nv + j)
    c = (((i + 1) % nu) * nv + (j + 1) % nv)
    d = (i * nv + (j + 1) % nv)
    f = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)])
    return v.astype(np.float32), f.astype(np.int32)


def _unit(x: np.ndarray) -> np.ndarray:
    return x / np.linalg.norm(x, axis=-1, keepdims=True)


def slivers(n: int, rng: np.random.Generator) -> np.ndarray:
    """n sliver triangles as an (n, 3, 3) float32 array."""
    c = rng.uniform(0.05, 0.95, size=(n, 3))
    L = rng.uniform(0.005, 0.05, size=(n, 1))
    A = rng.uniform(50.0, 500.0, size=(n, 1))
    d = _unit(rng.normal(size=(n, 3)))
    e = rng.normal(size=(n, 3))
    e = _unit(e - (e * d).sum(1, keepdims=True) * d)
    p0 = c - d * L / 2
    p1 = c + d * L / 2
    p2 = c + e * (L / A) + d * L * rng.uniform(-0.5, 0.5, size=(n, 1))
    return np.stack([p0, p1, p2], 1).astype(np.float32)


def icosphere_l5():
    """Plain method, small: (points, tris, res)."""
    rng = np.random.default_rng(0)
    v, f = jittered_icosphere(5, rng)
    return v, f, 128


def torus_slivers(n_total: int = 1_000_000):
    """Plain method at scale: soup points (3 per triangle), tris=None, res."""
    rng = np.random.default_rng(1)
    n_torus = n_total * 9 // 10
    nu = 900
    nv = n_torus // (2 * nu)
    v, f = torus(nu, nv, 0.35, 0.12, rng, 0.01 * 0.12)
    soup_t = v[f]
    soup_s = slivers(n_total - soup_t.shape[0], rng)
    soup = np.concatenate([soup_t, soup_s]).reshape(-1, 3)
    return np.ascontiguousarray(soup, dtype=np.float32), None, 512


def heightfield(n: int = 1582):
    """Plain method, large: (points, tris, res)."""
    rng = np.random.default_rng(2)
    amp = rng.uniform(0.0, 0.03, 16)
    kmag = rng.uniform(1.0, 40.0, 16)
    ang = rng.uniform(0.0, 2 * np.pi, 16)
    ph = rng.uniform(0.0, 2 * np.pi, 16)
    g = np.linspace(0.0, 1.0, n)
    X, Y = np.meshgrid(g, g, indexing="ij")
    Z = np.full_like(X, 0.5)
    for k in range(16):
        Z += amp[k] * np.sin(kmag[k] * (np.cos(ang[k]) * X + np.sin(ang[k]) * Y) + ph[k])
    v = np.stack([X, Y, Z], -1).reshape(-1, 3).astype(np.float32)
    i = np.arange(n - 1)[:, None]
    j = np.arange(n - 1)[None, :]
    a = i * n + j
    b = (i + 1) * n + j
    c = (i + 1) * n + j + 1
    d = i * n + j + 1
    f = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)])
    return v, f.astype(np.int32), 2048


def batch_mesh(rng: np.random.Generator):
    """One mesh of the batched / served distribution: (points, tris)."""
    target = float(np.exp(rng.uniform(np.log(320.0), np.log(80000.0))))
    if rng.uniform() < 0.5:
        level = int(np.clip(np.rint(np.log(target / 20.0) / np.log(4.0)), 2, 6))
        return jittered_icosphere(level, rng)
    nu = max(8, int(np.sqrt(target / 2.0 * 2.5)))
    nv = max(4, int(target / 2.0 / nu))
    R = rng.uniform(0.25, 0.4)
    r = rng.uniform(0.05, 0.2) * R / 0.35
    v, f = torus(nu, nv, R, r, rng, 0.01 * r)
    return _normalise(v).astype(np.float32), f


def batch(n: int = 256, seed: int = 3):
    """Batched: list of (points, tris, res)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        v, f = batch_mesh(rng)
        res = int(rng.choice([64, 128, 256, 512]))
        out.append((v, f, res))
    return out


def write_obj(path: str, points: np.ndarray, tris) -> None:
    """Writes `v x y z` / `f a b c` lines (1-based), every line terminated."""
    pts = np.asarray(points, dtype=np.float32).reshape(-1, 3)
    if tris is None:
        tris = np.arange(pts.shape[0], dtype=np.int64).reshape(-1, 3)
    with open(path, "w") as fh:
        fh.write("".join(f"v {x!r} {y!r} {z!r}\n" for x, y, z in pts.tolist()))
        fh.write("".join(f"f {a + 1} {b + 1} {c + 1}\n" for a, b, c in np.asarray(tris).tolist()))
