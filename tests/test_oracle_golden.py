"""Pins the CPU oracle to the golden fixtures (cKDTree / FP64 direct sum,
the reference's own validation routes) before it is trusted as the checker."""
import os

import numpy as np

from conftest import GOLDEN


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_morton_known_answers(orc):
    g = _load("morton.npz")
    for (x, y, z), c in zip(g["coords"], g["codes"]):
        assert orc.morton3(int(x), int(y), int(z)) == int(c)
    np.testing.assert_array_equal(orc.morton_codes(g["pts"]), g["pts_codes"])


def _check_knn_against_ckdtree(orc, g):
    pts, q, k = g["pts"], g["q"], int(g["k"])
    ids, d2 = orc.knn(pts, q, k)
    # distances of the oracle's picks, recomputed in FP64
    dd = np.linalg.norm(pts[ids.astype(np.int64)].astype(np.float64) - q[:, None, :].astype(np.float64), axis=2)
    # validate_knn_robust.py:21-43 route: sorted distances agree with cKDTree
    np.testing.assert_allclose(dd, g["dist"], rtol=0, atol=1e-6)
    # validate_full.py:46-56 route: exact ID match, or all picks within the
    # true k-th distance (+1e-5) where distances tie
    exact = np.all(ids.astype(np.int64) == g["ids"], axis=1)
    tie_ok = np.all(dd <= g["dist"][:, -1:] + 1e-5, axis=1)
    assert np.all(exact | tie_ok)
    return exact


def test_knn_uniform_vs_ckdtree(orc):
    exact = _check_knn_against_ckdtree(orc, _load("knn_uniform.npz"))
    assert exact.mean() > 0.99   # no distance ties in a continuous cloud


def test_knn_duplicates_vs_ckdtree(orc):
    g = _load("knn_dups.npz")
    _check_knn_against_ckdtree(orc, g)
    # ties resolve to the lower index
    ids, d2 = orc.knn(g["pts"], g["q"], int(g["k"]))
    for row_i, row_d in zip(ids, d2):
        for a in range(len(row_i) - 1):
            assert row_d[a] < row_d[a + 1] or (row_d[a] == row_d[a + 1] and row_i[a] < row_i[a + 1])


def test_range_vs_ckdtree(orc):
    g = _load("range_clustered.npz")
    pairs = orc.range_pairs(g["pts"], g["q"], float(g["r"]))
    counts, total = orc.range_count(g["pts"], g["q"], float(g["r"]))
    # FP32 key vs FP64 distance can differ only for points within rounding of r
    ref = {tuple(p) for p in g["pairs"]}
    got = {tuple(map(int, p)) for p in pairs}
    diff = ref ^ got
    r = float(g["r"])
    for qi, pi in diff:
        d = np.linalg.norm(g["pts"][pi].astype(np.float64) - g["q"][qi].astype(np.float64))
        assert abs(d - r) < 1e-6
    assert len(diff) <= 2
    assert total == len(pairs) == counts.sum()


def test_bh_physics_sum_within_2pct(orc):
    """verify_physics.py:42-45: the sum of force magnitudes of the reference BH
    (theta 0.5) within 2% of the FP64 direct sum."""
    g = _load("bh_physics.npz")
    nodes, order, root = orc.bh_build(g["pos"], g["mass"])
    f = orc.bh_ref_forces(g["pos"], g["mass"], nodes, order, 0.5)
    mag = np.sum(np.linalg.norm(f.astype(np.float64), axis=1))
    assert abs(mag - float(g["mag_sum"])) / float(g["mag_sum"]) < 0.02


def test_bh_tree_invariants(orc):
    g = _load("bh_physics.npz")
    pos, mass = g["pos"], g["mass"]
    nodes, order, root = orc.bh_build(pos, mass, bucket=16)
    n = len(pos)
    assert sorted(order.tolist()) == list(range(n))
    leaves = nodes[nodes["is_leaf"] == 1]
    assert leaves["num_particles"].sum() == n
    assert np.all(leaves["num_particles"] <= 16)
    # pre-order: next_idx = self + 1, autorope past the subtree
    idx = np.arange(len(nodes))
    assert np.all(nodes["next_idx"] == idx + 1)
    assert nodes["autorope"][0] == len(nodes)
    assert np.all(nodes["autorope"][nodes["is_leaf"] == 1] == idx[nodes["is_leaf"] == 1] + 1)
    # root mass is the total mass; COM is the mass-weighted mean
    assert abs(nodes["mass"][0] - mass.sum()) / mass.sum() < 1e-5
    com = (pos.astype(np.float64) * mass[:, None]).sum(0) / mass.sum()
    np.testing.assert_allclose(nodes["com"][0], com, atol=1e-3)


def test_bh_ref_walk_theta0_is_direct_sum(orc):
    """With theta = 0 no internal node is accepted (width < 1e-5 fails for
    cells wider than that), so the walk is an exact direct sum."""
    rng = np.random.default_rng(5)
    pos = rng.uniform(-1, 1, (700, 3)).astype(np.float32)
    mass = rng.uniform(0.5, 1.5, 700).astype(np.float32)
    nodes, order, _ = orc.bh_build(pos, mass, bucket=8)
    f = orc.bh_ref_forces(pos, mass, nodes, order, 0.0, 1.0)
    ref = orc.direct_ref_f64(pos, mass, np.arange(700), 1.0)
    np.testing.assert_allclose(f, ref, rtol=2e-4, atol=1e-4 * np.abs(ref).max())


def test_dbscan_matches_scikit_learn(orc):
    """The oracle's DBSCAN (FP32 range membership) labels points exactly as
    scikit-learn's DBSCAN does on data with no pair at distance ~ eps."""
    from sklearn.cluster import DBSCAN
    rng = np.random.default_rng(3)
    blobs = [rng.normal(c, s, size=(700, 3)) for c, s in ((0.2, 0.03), (0.6, 0.05), (0.8, 0.02))]
    pts = np.concatenate(blobs + [rng.random((900, 3))]).astype(np.float32)
    rng.shuffle(pts)
    d = np.sqrt(((pts[:, None, :].astype(np.float64) - pts[None, :, :]) ** 2).sum(-1))
    for eps0, mp in ((0.04, 8), (0.08, 5), (0.02, 3)):
        # nudge eps until no pair distance lies within FP32 rounding of it
        eps = next(e for e in (eps0 * (1 + 1e-4 * j) for j in range(100))
                   if np.abs(d - e).min() > 1e-6 * e)
        ref = DBSCAN(eps=eps, min_samples=mp).fit(pts.astype(np.float64)).labels_
        labels, nc = orc.dbscan(pts, eps, mp)
        np.testing.assert_array_equal(labels, ref)
        assert nc == ref.max() + 1
