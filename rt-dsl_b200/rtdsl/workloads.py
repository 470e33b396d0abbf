"""Seeded synthetic workloads standing in for the reference's datasets.

The reference benchmarks on 3DRoad / KITTI / 3DIono / Porto (README.md:19-33),
which are not available; these generators reproduce the shapes, sizes and
value distributions of the five workload definitions:

  plain_knn_small   100,000 U[0,1]^3 points (seed 0); 10,000 queries = points
                    drawn without replacement + N(0, 1e-3) jitter; k = 5.
  clustered_1p8m    1.8M points: 90% from 64 anisotropic Gaussians (centres
                    U[0,100]^3, per-axis sigma log-uniform in [0.05, 5]), 10%
                    uniform in [0,100]^3; 400,000 queries = sampled points +
                    N(0, 0.01) jitter (3DIono's size).
  sheet_10m         10M points on a 2-D-like sheet: x,y from 2,000 hotspots
                    with Zipf(1.2) weights and sigma log-uniform in
                    [1e-3, 1e-1] inside [0,10]^2, z ~ N(0, 1e-4); 1M queries
                    from the same distribution (Porto's shape).
  clouds_256        256 clouds, sizes log-uniform in [1e3, 2e5], alternately
                    U[0,1]^3 and an 8-Gaussian mixture in [0,1]^3; queries =
                    0.25 x size; per-cloud k from {1, 5, 16, 64}.
  plummer           Plummer sphere, scale radius 1, total mass 1, equal masses.
"""
from __future__ import annotations

import numpy as np


def plain_knn_small(n: int = 100_000, nq: int = 10_000, seed: int = 0):
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 3), dtype=np.float64).astype(np.float32)
    sel = rng.choice(n, size=nq, replace=False)
    q = (pts[sel].astype(np.float64) + rng.normal(0.0, 1e-3, size=(nq, 3))).astype(np.float32)
    return pts, q


def clustered(n: int = 1_800_000, nq: int = 400_000, seed: int = 1, n_clusters: int = 64,
              box: float = 100.0, bg_frac: float = 0.1):
    rng = np.random.default_rng(seed)
    n_bg = int(round(n * bg_frac))
    n_cl = n - n_bg
    centres = rng.uniform(0.0, box, size=(n_clusters, 3))
    sig = np.exp(rng.uniform(np.log(0.05), np.log(5.0), size=(n_clusters, 3)))
    lab = rng.integers(0, n_clusters, size=n_cl)
    cl = centres[lab] + rng.normal(size=(n_cl, 3)) * sig[lab]
    bg = rng.uniform(0.0, box, size=(n_bg, 3))
    pts = np.concatenate([cl, bg]).astype(np.float32)
    pts = pts[rng.permutation(n)]
    sel = rng.integers(0, n, size=nq)
    q = (pts[sel].astype(np.float64) + rng.normal(0.0, 0.01, size=(nq, 3))).astype(np.float32)
    return np.ascontiguousarray(pts), np.ascontiguousarray(q)


def _sheet_sample(rng, m, centres, sig, w):
    lab = rng.choice(len(w), size=m, p=w)
    xy = centres[lab] + rng.normal(size=(m, 2)) * sig[lab, None]
    xy = np.clip(xy, 0.0, 10.0)
    z = rng.normal(0.0, 1e-4, size=(m, 1))
    return np.concatenate([xy, z], axis=1).astype(np.float32)


def sheet(n: int = 10_000_000, nq: int = 1_000_000, seed: int = 2, n_hot: int = 2000):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 10.0, size=(n_hot, 2))
    sig = np.exp(rng.uniform(np.log(1e-3), np.log(1e-1), size=n_hot))
    w = 1.0 / np.arange(1, n_hot + 1) ** 1.2
    w /= w.sum()
    pts = _sheet_sample(rng, n, centres, sig, w)
    q = _sheet_sample(rng, nq, centres, sig, w)
    return pts, q


def clouds(n_clouds: int = 256, seed: int = 3, lo: float = 1e3, hi: float = 2e5,
           q_frac: float = 0.25, ks=(1, 5, 16, 64)):
    """Returns a list of dicts {points, queries, k} (float32 arrays)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_clouds)).astype(np.int64)
    out = []
    for c in range(n_clouds):
        n = int(sizes[c])
        if c % 2 == 0:
            pts = rng.random((n, 3))
        else:
            cen = rng.uniform(0.1, 0.9, size=(8, 3))
            sg = rng.uniform(0.01, 0.08, size=8)
            lab = rng.integers(0, 8, size=n)
            pts = np.clip(cen[lab] + rng.normal(size=(n, 3)) * sg[lab, None], 0.0, 1.0)
        pts = pts.astype(np.float32)
        nq = max(1, int(round(q_frac * n)))
        sel = rng.integers(0, n, size=nq)
        q = np.clip(pts[sel] + rng.normal(0.0, 1e-3, size=(nq, 3)), 0.0, 1.0).astype(np.float32)
        k = int(ks[rng.integers(0, len(ks))])
        out.append({"points": pts, "queries": q, "k": k})
    return out


def plummer(n: int = 1_000_000, seed: int = 7, a: float = 1.0, total_mass: float = 1.0,
            r_max: float | None = None):
    """Plummer sphere: r = a / sqrt(X^(-2/3) - 1), isotropic directions;
    equal masses total_mass / n.  r_max (in units of a) optionally rejects
    far outliers."""
    rng = np.random.default_rng(seed)
    pos = np.empty((n, 3))
    filled = 0
    while filled < n:
        m = n - filled
        x = rng.uniform(1e-10, 1.0, size=m)
        r = a / np.sqrt(x ** (-2.0 / 3.0) - 1.0)
        if r_max is not None:
            r = r[r <= r_max * a]
        m = len(r)
        cz = rng.uniform(-1.0, 1.0, size=m)
        ph = rng.uniform(0.0, 2 * np.pi, size=m)
        sz = np.sqrt(1.0 - cz * cz)
        pos[filled:filled + m] = np.stack([r * sz * np.cos(ph), r * sz * np.sin(ph), r * cz], 1)
        filled += m
    mass = np.full(n, total_mass / n)
    return pos.astype(np.float32), mass.astype(np.float32)
