"""Generates the golden fixtures under tests/golden/.

The reference ships no golden vectors.  Its own validators use scipy's
cKDTree as ground truth for k-NN (gprt-sandbox/validate_full.py:20-22,
validate_knn.py:13-16) and an FP64 numpy direct sum for Barnes-Hut
(gprt-sandbox/verify_physics.py:16-28); these fixtures record the outputs of
those same routes on small seeded inputs, plus Morton codes computed by an
independent bit-by-bit interleave, so the CPU oracle can be pinned to them.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os

import numpy as np
from scipy.spatial import cKDTree

HERE = os.path.dirname(os.path.abspath(__file__))


def morton_bitwise(x: int, y: int, z: int) -> int:
    """x<<2 | y<<1 | z interleave of 10-bit coordinates, bit by bit."""
    code = 0
    for b in range(10):
        code |= ((x >> b) & 1) << (3 * b + 2)
        code |= ((y >> b) & 1) << (3 * b + 1)
        code |= ((z >> b) & 1) << (3 * b)
    return code


def morton_codes_np(pts: np.ndarray) -> np.ndarray:
    """compute_morton_codes (gprt-core/src/morton.rs:19-48) in float32 numpy."""
    p = pts.astype(np.float32)
    mn = p.min(axis=0)
    mx = p.max(axis=0)
    ext = np.maximum(mx - mn, np.float32(1e-6)).astype(np.float32)
    t = ((p - mn) / ext * np.float32(1023.0)).astype(np.float32)
    q = np.clip(np.floor(np.maximum(t, 0)), 0, 1023).astype(np.int64)
    return np.array([morton_bitwise(*map(int, r)) for r in q], dtype=np.uint32)


def main() -> None:
    rng = np.random.default_rng(2024)

    # --- Morton known answers
    coords = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1023, 1023, 1023],
                       [5, 9, 17], [512, 3, 1000], [1023, 0, 0], [0, 1023, 0], [0, 0, 1023]],
                      dtype=np.int64)
    coords = np.concatenate([coords, rng.integers(0, 1024, size=(40, 3))])
    codes = np.array([morton_bitwise(*map(int, c)) for c in coords], dtype=np.uint32)
    mpts = rng.random((500, 3)).astype(np.float32) * np.float32(7.5) - np.float32(2.0)
    np.savez_compressed(os.path.join(HERE, "morton.npz"), coords=coords, codes=codes,
                        pts=mpts, pts_codes=morton_codes_np(mpts))

    # --- kNN: uniform cloud, cKDTree ground truth (validate_full.py route)
    pts = rng.random((3000, 3)).astype(np.float32)
    q = (pts[rng.choice(3000, 400, replace=False)] + rng.normal(0, 1e-3, (400, 3))).astype(np.float32)
    d, i = cKDTree(pts.astype(np.float64)).query(q.astype(np.float64), k=8)
    np.savez_compressed(os.path.join(HERE, "knn_uniform.npz"), pts=pts, q=q, k=8,
                        ids=i.astype(np.int64), dist=d)

    # --- kNN: clustered cloud with exact duplicates (ties)
    base = (rng.normal(size=(600, 3)) * 0.05 + 0.5).astype(np.float32)
    pts2 = np.concatenate([base, base[:200], base[:50]]).astype(np.float32)
    q2 = np.concatenate([base[:100], (rng.normal(size=(100, 3)) * 0.05 + 0.5)]).astype(np.float32)
    d2, i2 = cKDTree(pts2.astype(np.float64)).query(q2.astype(np.float64), k=6)
    np.savez_compressed(os.path.join(HERE, "knn_dups.npz"), pts=pts2, q=q2, k=6,
                        ids=i2.astype(np.int64), dist=d2)

    # --- range: clustered cloud, cKDTree query_ball_point
    pts3 = np.concatenate([(rng.normal(size=(1500, 3)) * 0.1 + c) for c in
                           ([0.2, 0.2, 0.2], [0.7, 0.6, 0.5])]).astype(np.float32)
    q3 = pts3[rng.choice(len(pts3), 300, replace=False)] + rng.normal(0, 0.01, (300, 3)).astype(np.float32)
    q3 = q3.astype(np.float32)
    r3 = 0.05
    lists = cKDTree(pts3.astype(np.float64)).query_ball_point(q3.astype(np.float64), r3)
    counts = np.array([len(l) for l in lists], dtype=np.int64)
    pairs = np.array([(qi, pi) for qi, l in enumerate(lists) for pi in sorted(l)],
                     dtype=np.int64).reshape(-1, 2)
    np.savez_compressed(os.path.join(HERE, "range_clustered.npz"), pts=pts3, q=q3, r=r3,
                        counts=counts, pairs=pairs)

    # --- Barnes-Hut physics check (verify_physics.py:5-45): N bodies in
    # U[-100,100]^3, masses U[0.5,1.5], FP64 direct sum with that script's
    # law G*mi*mj/(d^3 + 1e-12), d > 1e-6; the sum of force magnitudes.
    prng = np.random.RandomState(42)
    N = 2000
    mass = prng.uniform(0.5, 1.5, N)
    pos = prng.uniform(-100, 100, (N, 3))
    G = 6.674e-11
    forces = np.zeros((N, 3))
    for a in range(N):
        diff = pos - pos[a]
        dsq = np.sum(diff ** 2, axis=1)
        dd = np.sqrt(dsq)
        mask = dd > 1e-6
        fm = G * mass[a] * mass / (dsq * dd + 1e-12)
        forces[a] = np.sum(diff[mask] * fm[mask, None], axis=0)
    np.savez_compressed(os.path.join(HERE, "bh_physics.npz"), pos=pos.astype(np.float32),
                        mass=mass.astype(np.float32), forces=forces,
                        mag_sum=np.sum(np.linalg.norm(forces, axis=1)))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
