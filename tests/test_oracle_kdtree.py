"""The oracle's exact k-d tree checker (orc_kd_*) against the oracle's brute
force: identical k-NN ids and FP32 keys, range counts and (query, id) pairs,
on clouds built to stress the pruning bound (duplicates, a flat sheet, all
points equal, NaN and infinite coordinates, k above the point count)."""
import numpy as np
import pytest


def clouds():
    rng = np.random.default_rng(1)
    out = []
    n = 2500
    out.append(("duplicates", (np.round(rng.random((n, 3)) * 4) / 4)))
    p = rng.random((n, 3))
    p[::7] = np.nan
    p[::11, 1] = np.inf
    out.append(("nan_inf", p))
    out.append(("all_equal", np.zeros((n, 3))))
    out.append(("sheet", rng.normal(size=(n, 3)) * np.array([1, 1, 1e-4])))
    out.append(("one_point", rng.random((1, 3))))
    return [(name, c.astype(np.float32)) for name, c in out]


@pytest.mark.parametrize("name,pts", clouds(), ids=[c[0] for c in clouds()])
def test_kdtree_knn_equals_brute_force(orc, name, pts):
    rng = np.random.default_rng(2)
    q = (rng.random((400, 3)) * 2 - 0.5).astype(np.float32)
    q[:5] = pts[np.arange(5) % len(pts)]
    q[7] = np.nan
    tree = orc.KdTree(pts)
    for k in (1, 5, 16, 64, 65, 300, len(pts) + 3):
        ti, td = tree.knn(q, k)
        bi, bd = orc.knn(pts, q, k)
        np.testing.assert_array_equal(ti, bi)
        np.testing.assert_array_equal(td.view(np.uint32), bd.view(np.uint32))


@pytest.mark.parametrize("name,pts", clouds(), ids=[c[0] for c in clouds()])
def test_kdtree_range_equals_brute_force(orc, name, pts):
    rng = np.random.default_rng(3)
    q = (rng.random((300, 3)) * 2 - 0.5).astype(np.float32)
    q[:5] = pts[np.arange(5) % len(pts)]
    tree = orc.KdTree(pts)
    for r in (0.0, 0.05, 0.3, 2.0):
        tc, tt = tree.range_count(q, r)
        bc, bt = orc.range_count(pts, q, r)
        np.testing.assert_array_equal(tc, bc)
        assert tt == bt
        np.testing.assert_array_equal(tree.range_pairs(q, r), orc.range_pairs(pts, q, r))


def test_kdtree_empty_cloud(orc):
    tree = orc.KdTree(np.zeros((0, 3), np.float32))
    ids, d2 = tree.knn(np.zeros((3, 3), np.float32), 4)
    assert np.all(ids == 0xFFFFFFFF) and np.all(np.isinf(d2))
    assert tree.range_count(np.zeros((3, 3), np.float32), 1.0)[1] == 0


def test_cpu_bvh_range_matches_membership(orc):
    """The reference CPU range search (timed baseline) finds exactly the
    oracle's members."""
    rng = np.random.default_rng(4)
    pts = rng.random((4000, 3)).astype(np.float32)
    q = rng.random((200, 3)).astype(np.float32)
    c1, t1 = orc.cpu_bvh_range(pts, q, 0.08)
    c2, t2 = orc.range_count(pts, q, 0.08)
    np.testing.assert_array_equal(c1, c2)
    assert t1 == t2


def test_targeted_reference_walk_and_direct_sum(orc):
    """The sampled-target forms equal the all-body forms bit for bit."""
    rng = np.random.default_rng(5)
    pos = rng.random((3000, 3)).astype(np.float32)
    m = (rng.random(3000) + 0.5).astype(np.float32)
    tg = np.array([0, 17, 2999])
    nodes, order, _ = orc.bh_build(pos, m, bucket=16)
    f = orc.bh_ref_forces(pos, m, nodes, order, 0.5)
    np.testing.assert_array_equal(orc.bh_ref_forces_at(pos, m, nodes, order, tg, 0.5), f[tg])
    _, phi, acc = orc.direct_plummer_f64(pos, m, 1e-3, 1.0)
    ph2, ac2 = orc.direct_plummer_at_f64(pos, m, tg, 1e-3, 1.0)
    np.testing.assert_array_equal(ph2, phi[tg])
    np.testing.assert_array_equal(ac2, acc[tg])
