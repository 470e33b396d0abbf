"""Range-query parity: counts and (query, id) pairs from the CUDA count/fill
passes against the oracle, bit-exact membership (FP32 key <= RN(r*r))."""
import numpy as np
import pytest
import torch

from rtdsl import workloads

pytestmark = pytest.mark.gpu


def gpu_range(rtd, pts, q, r, sort=True, **sched):
    s = rtd.default_schedule(**sched)
    ix = rtd.Index().build(torch.from_numpy(np.ascontiguousarray(pts)).cuda(), s)
    qt = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    counts, total = ix.range_count(qt, r, s)
    pairs = ix.range_fill(qt, r, total, sort_pairs=sort, schedule=s)
    torch.cuda.synchronize()
    return counts.cpu().numpy().view(np.uint32), total, pairs.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("leaf", [1, 4, 16, 64])
def test_range_clustered_sorted(rtd, orc, cuda, leaf):
    pts, q = workloads.clustered(n=30_000, nq=3_000, seed=21, n_clusters=10, box=10.0)
    r = 0.08
    counts, total, pairs = gpu_range(rtd, pts, q, r, leaf_size=leaf)
    oc, ot = orc.range_count(pts, q, r)
    np.testing.assert_array_equal(counts, oc)
    assert total == ot
    np.testing.assert_array_equal(pairs, orc.range_pairs(pts, q, r))


def test_range_unsorted_is_same_set(rtd, orc, cuda):
    pts, q = workloads.clustered(n=30_000, nq=2_000, seed=22, n_clusters=10, box=10.0)
    r = 0.2   # heavy output: exercises the staging-buffer overflow path
    counts, total, pairs = gpu_range(rtd, pts, q, r, sort=False)
    ref = orc.range_pairs(pts, q, r)
    assert total == len(ref) == len(pairs)
    key = lambda a: np.sort(a[:, 0].astype(np.uint64) << np.uint64(32) | a[:, 1].astype(np.uint64))
    np.testing.assert_array_equal(key(pairs), key(ref))


def test_range_radius_zero_and_duplicates(rtd, orc, cuda):
    rng = np.random.default_rng(4)
    base = rng.random((300, 3)).astype(np.float32)
    pts = np.concatenate([base, base[:100]])
    q = np.concatenate([base[:50], rng.random((50, 3)).astype(np.float32)])
    counts, total, pairs = gpu_range(rtd, pts, q, 0.0)
    np.testing.assert_array_equal(pairs, orc.range_pairs(pts, q, 0.0))
    assert np.all(counts[:50] == 2) and np.all(counts[50:] == 0)


def test_range_empty_inputs(rtd, cuda):
    counts, total, pairs = gpu_range(rtd, np.zeros((0, 3), np.float32),
                                     np.random.rand(20, 3).astype(np.float32), 1.0)
    assert total == 0 and np.all(counts == 0) and len(pairs) == 0


def test_range_overflow_reports_required_size(rtd, cuda):
    pts, q = workloads.clustered(n=5_000, nq=500, seed=23, n_clusters=4, box=2.0)
    s = rtd.default_schedule()
    ix = rtd.Index().build(torch.from_numpy(pts).cuda(), s)
    qt = torch.from_numpy(q).cuda()
    _, total = ix.range_count(qt, 0.3, s)
    assert total > 10
    with pytest.raises(rtd.RtdError) as e:
        ix.range_fill(qt, 0.3, total // 2, schedule=s)
    assert e.value.status == 4
    # the index stays usable afterwards
    pairs = ix.range_fill(qt, 0.3, total, sort_pairs=True, schedule=s)
    assert len(pairs) == total


def test_range_host_api(rtd, orc, cuda):
    pts, q = workloads.clustered(n=8_000, nq=400, seed=24, n_clusters=4, box=5.0)
    pairs = rtd.range_query(pts, q, 0.15)
    np.testing.assert_array_equal(pairs, orc.range_pairs(pts, q, 0.15))


@pytest.mark.slow
def test_range_large_property(rtd, orc, cuda):
    """400K queries on 1.8M points: the count pass and the fill agree
    (sum of counts = pairs written, per-query histogram of the pairs equals
    the counts), and every count and every pair equals the oracle's (exact
    k-d tree)."""
    from rtdsl.api import radius_for_mean_count
    pts, q = workloads.clustered()
    s = rtd.default_schedule()
    ix = rtd.Index().build(torch.from_numpy(pts).cuda(), s)
    r = radius_for_mean_count(ix, torch.from_numpy(q).cuda(), 50.0)
    counts, total, pairs = gpu_range(rtd, pts, q, r)
    assert 40 <= total / len(q) <= 60          # the workload's mean of 50 neighbours
    assert counts.max() > 1000                 # with a heavy tail in the dense clusters
    assert counts.sum() == total == len(pairs)
    np.testing.assert_array_equal(np.bincount(pairs[:, 0], minlength=len(q)), counts)
    assert np.all(np.diff(pairs[:, 0].astype(np.int64)) >= 0)
    tree = orc.KdTree(pts)
    oc, ot = tree.range_count(q, r)
    np.testing.assert_array_equal(counts, oc)
    # every (query, id) pair of every query equals the oracle's
    ref = tree.range_pairs(q, r)
    assert ot == len(ref) == len(pairs)
    key = lambda a: np.sort(a[:, 0].astype(np.uint64) << np.uint64(32) | a[:, 1].astype(np.uint64))
    np.testing.assert_array_equal(key(pairs), key(ref))


@pytest.mark.parametrize("r", [0.05, 0.3, 2.0])
@pytest.mark.parametrize("leaf", [1, 8])
def test_range_dense_clusters_contained_subtrees(rtd, orc, cuda, r, leaf):
    """Tight clusters and radii up to the whole cloud: most hits come from
    subtrees whose box lies inside the ball (counted and copied without a
    per-point test); counts and pairs must still equal the oracle's."""
    pts, q = workloads.clustered(n=20_000, nq=1_500, seed=31, n_clusters=6, box=1.0)
    counts, total, pairs = gpu_range(rtd, pts, q, r, leaf_size=leaf)
    oc, ot = orc.range_count(pts, q, r)
    np.testing.assert_array_equal(counts, oc)
    assert total == ot
    np.testing.assert_array_equal(pairs, orc.range_pairs(pts, q, r))
    counts_u, total_u, pairs_u = gpu_range(rtd, pts, q, r, sort=False, leaf_size=leaf)
    assert total_u == ot
    key = lambda a: np.sort(a[:, 0].astype(np.uint64) << np.uint64(32) | a[:, 1].astype(np.uint64))
    np.testing.assert_array_equal(key(pairs_u), key(pairs))


@pytest.mark.parametrize("r", [0.1, 10.0])
def test_range_non_finite(rtd, orc, cuda, r):
    """NaN / infinite points are never neighbours, also when their subtree
    would otherwise lie inside the ball; a NaN query has none."""
    rng = np.random.default_rng(12)
    pts = rng.random((4000, 3)).astype(np.float32)
    pts[10] = [np.nan, 0.5, 0.5]
    pts[11] = [0.5, 0.5, np.nan]
    pts[20] = [np.inf, 0.5, 0.5]
    pts[30] = [0.5, -np.inf, 0.5]
    q = rng.random((200, 3)).astype(np.float32)
    q[0] = [np.nan, 0.1, 0.1]
    q[1] = [np.inf, 0.1, 0.1]
    q[2] = [1e30, 1e30, 1e30]
    counts, total, pairs = gpu_range(rtd, pts, q, r)
    oc, ot = orc.range_count(pts, q, r)
    np.testing.assert_array_equal(counts, oc)
    assert total == ot and counts[0] == 0
    np.testing.assert_array_equal(pairs, orc.range_pairs(pts, q, r))


def _pair_keys(a):
    return np.sort(a[:, 0].astype(np.uint64) << np.uint64(32) | a[:, 1].astype(np.uint64))


def test_range_fill_after_count_is_grouped_by_query(rtd, orc, cuda):
    """A fill that follows the count of the same queries writes each query's
    pairs into its own segment: even unsorted, the pairs come out grouped
    by query in the caller's order, and the set equals the oracle's."""
    pts, q = workloads.clustered(n=30_000, nq=2_000, seed=41, n_clusters=10, box=10.0)
    r = 0.2
    counts, total, pairs = gpu_range(rtd, pts, q, r, sort=False)
    assert np.all(np.diff(pairs[:, 0].astype(np.int64)) >= 0)
    np.testing.assert_array_equal(np.bincount(pairs[:, 0], minlength=len(q)), counts)
    np.testing.assert_array_equal(_pair_keys(pairs), _pair_keys(orc.range_pairs(pts, q, r)))


def test_range_fill_without_matching_count(rtd, orc, cuda):
    """Fills that do not follow a count of the same queries at the same
    radius (no count at all, another radius, a k-NN search in between, other
    queries) push pairs through the warp-staged cursor and give the same
    set."""
    pts, q = workloads.clustered(n=30_000, nq=2_000, seed=42, n_clusters=10, box=10.0)
    s = rtd.default_schedule()
    ix = rtd.Index().build(torch.from_numpy(pts).cuda(), s)
    qt = torch.from_numpy(q).cuda()
    ref = _pair_keys(orc.range_pairs(pts, q, 0.15))
    n_ref = len(ref)
    # no count on this index yet
    np.testing.assert_array_equal(_pair_keys(ix.range_fill(qt, 0.15, n_ref, schedule=s).cpu().numpy().view(np.uint32)), ref)
    # the last count was at another radius
    ix.range_count(qt, 0.1, s)
    np.testing.assert_array_equal(_pair_keys(ix.range_fill(qt, 0.15, n_ref, schedule=s).cpu().numpy().view(np.uint32)), ref)
    # a k-NN search reordered queries after the count
    ix.range_count(qt, 0.15, s)
    ix.knn(qt, 5, s)
    np.testing.assert_array_equal(_pair_keys(ix.range_fill(qt, 0.15, n_ref, schedule=s).cpu().numpy().view(np.uint32)), ref)
    # the count was over another query buffer
    ix.range_count(qt[:1000].clone(), 0.15, s)
    np.testing.assert_array_equal(_pair_keys(ix.range_fill(qt, 0.15, n_ref, schedule=s).cpu().numpy().view(np.uint32)), ref)


def test_range_fill_detects_queries_changed_after_count(rtd, orc, cuda):
    """Queries overwritten in place between the count and the fill: the fill
    stays inside each query's segment, reports the mismatch, and the index
    keeps working."""
    pts, q = workloads.clustered(n=20_000, nq=1_000, seed=43, n_clusters=6, box=5.0)
    s = rtd.default_schedule()
    ix = rtd.Index().build(torch.from_numpy(pts).cuda(), s)
    qt = torch.from_numpy(q).cuda()
    _, total = ix.range_count(qt, 0.2, s)
    qt.copy_(torch.from_numpy(np.ascontiguousarray(q[::-1])).cuda())   # other hit counts per slot
    pairs = torch.zeros((total + 1024, 2), dtype=torch.int32, device="cuda")
    with pytest.raises(rtd.RtdError) as e:
        ix.range_fill(qt, 0.2, total, schedule=s, out_pairs=pairs)
    assert e.value.status == 1
    assert torch.all(pairs[total:] == 0)      # nothing written past the counted total
    _, total2 = ix.range_count(qt, 0.2, s)
    got = ix.range_fill(qt, 0.2, total2, sort_pairs=True, schedule=s).cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(got, orc.range_pairs(pts, q[::-1].copy(), 0.2))


def test_range_repeated_count_fill_scatters_the_counts_pairs(rtd, orc, cuda):
    """Once a count has sized the index's pair buffer, later counts also push
    their pairs there and a fill of the same queries only scatters them into
    the segments: the pairs stay grouped by query with the count's counts
    and equal the oracle's.  A count whose pairs overflow that buffer (a
    larger radius) falls back to the segment fill's own traversal."""
    pts, q = workloads.clustered(n=30_000, nq=3_000, seed=44, n_clusters=10, box=10.0)
    s = rtd.default_schedule()
    ix = rtd.Index().build(torch.from_numpy(pts).cuda(), s)
    qt = torch.from_numpy(q).cuda()
    tree = orc.KdTree(pts)
    for r in (0.15, 0.15, 0.1, 0.3, 0.3):       # 0.3: more pairs than the buffer first
        counts, total = ix.range_count(qt, r, s)
        pairs = ix.range_fill(qt, r, total, sort_pairs=False, schedule=s)
        c = counts.cpu().numpy().view(np.uint32)
        p = pairs.cpu().numpy().view(np.uint32)
        oc, ot = tree.range_count(q, r)
        np.testing.assert_array_equal(c, oc)
        assert total == ot == len(p)
        assert np.all(np.diff(p[:, 0].astype(np.int64)) >= 0)
        np.testing.assert_array_equal(_pair_keys(p), _pair_keys(tree.range_pairs(q, r)))
        sp = ix.range_fill(qt, r, total, sort_pairs=True, schedule=s)   # the same count, again
        np.testing.assert_array_equal(sp.cpu().numpy().view(np.uint32), tree.range_pairs(q, r))


def test_range_changed_queries_detected_after_a_pushing_count(rtd, orc, cuda):
    """The same change as above, after a count that kept its pairs: the
    fill notices the queries differ from the count's (fingerprint), runs the
    segment fill, and reports the mismatch."""
    pts, q = workloads.clustered(n=20_000, nq=1_000, seed=45, n_clusters=6, box=5.0)
    s = rtd.default_schedule()
    ix = rtd.Index().build(torch.from_numpy(pts).cuda(), s)
    qt = torch.from_numpy(q).cuda()
    _, total = ix.range_count(qt, 0.2, s)          # sizes the pair buffer
    _, total = ix.range_count(qt, 0.2, s)          # pushes its pairs
    qt.copy_(torch.from_numpy(np.ascontiguousarray(q[::-1])).cuda())
    pairs = torch.zeros((total + 1024, 2), dtype=torch.int32, device="cuda")
    with pytest.raises(rtd.RtdError) as e:
        ix.range_fill(qt, 0.2, total, schedule=s, out_pairs=pairs)
    assert e.value.status == 1
    assert torch.all(pairs[total:] == 0)
