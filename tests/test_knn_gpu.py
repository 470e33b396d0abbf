"""k-NN parity: the CUDA path (through the C ABI) against the CPU oracle.
Neighbour ids must match bit-exactly (FP32 key, ties to the lower id) and the
returned squared distances must equal the oracle's FP32 keys bit-for-bit."""
import numpy as np
import pytest
import torch

from rtdsl import workloads

pytestmark = pytest.mark.gpu


def gpu_knn(rtd, pts, q, k, **sched):
    s = rtd.default_schedule(**sched)
    ix = rtd.Index().build(torch.from_numpy(np.ascontiguousarray(pts)).cuda(), s)
    ids, d2 = ix.knn(torch.from_numpy(np.ascontiguousarray(q)).cuda(), k, s)
    torch.cuda.synchronize()
    info = ix.info()
    return ids.cpu().numpy().view(np.uint32), d2.cpu().numpy(), info


def assert_same(orc_ids, orc_d2, ids, d2):
    bad = np.nonzero(np.any(orc_ids != ids, axis=1))[0]
    assert len(bad) == 0, (f"{len(bad)} queries differ; first {bad[:5]}: "
                           f"oracle {orc_ids[bad[:2]]} gpu {ids[bad[:2]]}")
    np.testing.assert_array_equal(orc_d2.view(np.uint32), d2.view(np.uint32))


def clustered_small(n=30_000, nq=3_000, seed=11):
    return workloads.clustered(n=n, nq=nq, seed=seed, n_clusters=12, box=10.0)


def test_plain_knn_small_config(rtd, orc, cuda):
    """100,000 uniform points, 10,000 jittered queries, k = 5: the CPU-runnable
    workload, checked exhaustively."""
    pts, q = workloads.plain_knn_small()
    ids, d2, info = gpu_knn(rtd, pts, q, 5)
    oi, od = orc.knn(pts, q, 5)
    assert_same(oi, od, ids, d2)
    assert info["n_points"] == len(pts)
    assert orc.knn_fp64_ambiguity(pts, q[:2000], ids[:2000]) <= 2


@pytest.mark.parametrize("k", [1, 2, 5, 8, 16, 32])
@pytest.mark.parametrize("mode", ["thread", "warp"])
def test_knn_k_and_traversal(rtd, orc, cuda, k, mode):
    pts, q = clustered_small()
    kw = {"thread": dict(lanes_per_query=1), "warp": dict(lanes_per_query=32)}[mode]
    ids, d2, _ = gpu_knn(rtd, pts, q, k, **kw)
    oi, od = orc.knn(pts, q, k)
    assert_same(oi, od, ids, d2)


@pytest.mark.parametrize("lanes", [1, 32])
@pytest.mark.parametrize("block", [64, 128, 256])
def test_knn_block_sizes(rtd, orc, cuda, lanes, block):
    pts, q = clustered_small(n=15_000, nq=1_500, seed=19)
    ids, d2, _ = gpu_knn(rtd, pts, q, 5, lanes_per_query=lanes, block_size=block)
    oi, od = orc.knn(pts, q, 5)
    assert_same(oi, od, ids, d2)


@pytest.mark.parametrize("k", [33, 64, 100, 256])
def test_knn_large_k_warp_list(rtd, orc, cuda, k):
    pts, q = clustered_small(n=20_000, nq=1_000, seed=12)
    ids, d2, _ = gpu_knn(rtd, pts, q, k)
    oi, od = orc.knn(pts, q, k)
    assert_same(oi, od, ids, d2)


@pytest.mark.parametrize("leaf", [1, 2, 4, 8, 16, 32, 64])
@pytest.mark.parametrize("bits", [30, 36, 48, 63])
def test_knn_leaf_and_key_width(rtd, orc, cuda, leaf, bits):
    pts, q = clustered_small(n=25_000, nq=2_000, seed=13)
    ids, d2, info = gpu_knn(rtd, pts, q, 5, leaf_size=leaf, morton_bits=bits)
    oi, od = orc.knn(pts, q, 5)
    assert_same(oi, od, ids, d2)
    assert info["morton_bits"] == bits


@pytest.mark.parametrize("heur,param", [(0, 2 ** -4), (1, 0.10), (1, 0.02), (2, 1e-6),
                                        (2, 100.0), (3, 0.0), (4, 0.5)])
def test_knn_radius_heuristics_do_not_change_results(rtd, orc, cuda, heur, param):
    pts, q = clustered_small(n=20_000, nq=2_000, seed=14)
    ids, d2, _ = gpu_knn(rtd, pts, q, 8, radius_heuristic=heur, radius_param=param)
    oi, od = orc.knn(pts, q, 8)
    assert_same(oi, od, ids, d2)


@pytest.mark.parametrize("k", [1, 5, 16, 40])
@pytest.mark.parametrize("bits", [30, 42, 63])
def test_knn_morton_window_seed(rtd, orc, cuda, k, bits):
    """RTD_RADIUS_MORTON_WINDOW: lists seeded with each query's 4k Morton
    neighbours, then one unbounded round that skips them; ids and keys equal
    the oracle's for every key width, for duplicates, far queries and tiny
    clouds (k = 40 takes the warp path, where the heuristic is the sampled
    1-NN radius)."""
    pts, q = clustered_small(n=20_000, nq=2_000, seed=19)
    rng = np.random.default_rng(19)
    pts = np.concatenate([pts, pts[:500]])                        # exact duplicates
    q = np.concatenate([q, rng.uniform(-50.0, 60.0, size=(200, 3)).astype(np.float32)])
    ids, d2, _ = gpu_knn(rtd, pts, q, k, radius_heuristic=4, radius_param=0.5, morton_bits=bits,
                         leaf_size=8)
    oi, od = orc.knn(pts, q, k)
    assert_same(oi, od, ids, d2)
    for n in (1, 3, 2 * k + 1, 4 * k + 1):
        ids, d2, _ = gpu_knn(rtd, pts[:n], q[:50], k, radius_heuristic=4, morton_bits=bits)
        oi, od = orc.knn(pts[:n], q[:50], k)
        assert_same(oi, od, ids, d2)


@pytest.mark.parametrize("mult,rounds", [(2.0, 1), (2.0, 2), (1.05, 32), (3.0, 30), (64.0, 4)])
def test_knn_round_schedules(rtd, orc, cuda, mult, rounds):
    pts, q = clustered_small(n=20_000, nq=2_000, seed=15)
    ids, d2, _ = gpu_knn(rtd, pts, q, 5, radius_increment_mult=mult, max_rounds=rounds)
    oi, od = orc.knn(pts, q, 5)
    assert_same(oi, od, ids, d2)


def test_knn_unsorted_queries(rtd, orc, cuda):
    pts, q = clustered_small(n=20_000, nq=2_000, seed=16)
    ids, d2, _ = gpu_knn(rtd, pts, q, 5, use_morton_lbv=0)
    oi, od = orc.knn(pts, q, 5)
    assert_same(oi, od, ids, d2)


def test_knn_duplicates_and_ties(rtd, orc, cuda):
    rng = np.random.default_rng(3)
    base = rng.integers(0, 8, size=(500, 3)).astype(np.float32)   # integer lattice: many ties
    pts = np.concatenate([base, base, base[:100]])
    q = np.concatenate([base[:200], rng.integers(0, 8, size=(200, 3)).astype(np.float32) + 0.5])
    for k in (1, 5, 16, 40):
        for lanes in (1, 32):
            if lanes == 1 and k > 32:
                continue
            ids, d2, _ = gpu_knn(rtd, pts, q, k, lanes_per_query=lanes)
            oi, od = orc.knn(pts, q, k)
            assert_same(oi, od, ids, d2)


def test_knn_all_points_identical(rtd, orc, cuda):
    pts = np.full((5000, 3), 0.25, dtype=np.float32)
    q = np.array([[0.25, 0.25, 0.25], [1.0, 2.0, 3.0], [-5.0, 0.0, 0.0]], dtype=np.float32)
    ids, d2, _ = gpu_knn(rtd, pts, q, 7)
    oi, od = orc.knn(pts, q, 7)
    assert_same(oi, od, ids, d2)
    assert ids[0].tolist() == list(range(7))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7])
def test_knn_fewer_points_than_k(rtd, orc, cuda, n):
    rng = np.random.default_rng(n)
    pts = rng.random((n, 3)).astype(np.float32)
    q = rng.random((50, 3)).astype(np.float32)
    for lanes in (1, 32):
        ids, d2, _ = gpu_knn(rtd, pts, q, 8, lanes_per_query=lanes)
        oi, od = orc.knn(pts, q, 8)
        assert_same(oi, od, ids, d2)
        assert np.all(ids[:, n:] == 0xFFFFFFFF) and np.all(np.isinf(d2[:, n:]))


def test_knn_empty_inputs(rtd, cuda):
    s = rtd.default_schedule()
    ix = rtd.Index().build(torch.zeros((0, 3), device="cuda"), s)
    ids, d2 = ix.knn(torch.rand((10, 3), device="cuda"), 4, s)
    torch.cuda.synchronize()
    assert np.all(ids.cpu().numpy().view(np.uint32) == 0xFFFFFFFF)
    ix2 = rtd.Index().build(torch.rand((100, 3), device="cuda"), s)
    ids2, _ = ix2.knn(torch.zeros((0, 3), device="cuda"), 4, s)
    assert ids2.shape == (0, 4)


def test_knn_non_finite(rtd, orc, cuda):
    rng = np.random.default_rng(9)
    pts = rng.random((3000, 3)).astype(np.float32)
    pts[10] = [np.nan, 0.5, 0.5]
    pts[20] = [np.inf, 0.5, 0.5]
    pts[30] = [0.5, -np.inf, 0.5]
    q = rng.random((300, 3)).astype(np.float32)
    q[0] = [np.nan, 0.1, 0.1]
    q[1] = [np.inf, 0.1, 0.1]
    q[2] = [1e30, 1e30, 1e30]
    for lanes in (1, 32):
        ids, d2, _ = gpu_knn(rtd, pts, q, 6, lanes_per_query=lanes)
        oi, od = orc.knn(pts, q, 6)
        assert_same(oi, od, ids, d2)
        assert np.all(ids[0] == 0xFFFFFFFF)


def test_knn_far_queries_and_large_coordinates(rtd, orc, cuda):
    rng = np.random.default_rng(10)
    pts = (rng.random((4000, 3)) * 1e6).astype(np.float32)
    q = np.concatenate([(rng.random((200, 3)) * 1e6), rng.normal(0, 1e8, (50, 3))]).astype(np.float32)
    ids, d2, _ = gpu_knn(rtd, pts, q, 5)
    oi, od = orc.knn(pts, q, 5)
    assert_same(oi, od, ids, d2)


def test_knn_host_api_k_nn(rtd, orc, cuda):
    pts, q = clustered_small(n=10_000, nq=500, seed=17)
    out = rtd.k_nn(pts, q, 5)
    oi, _ = orc.knn(pts, q, 5)
    assert out == oi.astype(np.int64).tolist()
    few = rtd.k_nn(pts[:3], q[:4], 5)
    assert all(len(r) == 3 for r in few)


@pytest.mark.parametrize("order", [0, 1])
def test_knn_host_context_overlap(rtd, orc, cuda, order):
    """rtd_k_nn_host copies and orders the queries on a second stream while
    the index is built: ids and d2 equal the oracle's with and without query
    ordering, across repeated calls of different sizes on one context."""
    ctx = rtd.Context()
    s = rtd.default_schedule(use_morton_lbv=order, leaf_size=8, morton_bits=42)
    for n, nq, seed in [(30_000, 3_000, 51), (5_000, 7_000, 52), (30_000, 1, 53), (1, 300, 54)]:
        pts, q = clustered_small(n=n, nq=nq, seed=seed)
        if nq == 1:
            q = q[:1]
        ids, d2 = ctx.k_nn(pts, q, 5, s, with_d2=True)
        oi, od = orc.knn(pts, q, 5)
        assert_same(oi, od, ids, d2)


@pytest.mark.parametrize("sched", [dict(radius_heuristic=4, leaf_size=5, morton_bits=39),
                                   dict(use_morton_lbv=0), dict(lanes_per_query=32)])
def test_knn_host_chunked_results(rtd, orc, cuda, sched):
    """With 65,536 queries or more, rtd_k_nn_host searches the queries in
    eight chunks of the caller's order (ordered by chunk, then Morton code),
    each on its own stream, and copies each chunk's rows out while the later
    chunks search.  Rows land in the caller's order, equal to the oracle's,
    for uneven chunks, every launch mode, and repeated calls on one
    context."""
    ctx = rtd.Context()
    s = rtd.default_schedule(**sched)
    for n, nq, seed, k in [(30_000, 70_001, 81, 5), (12_000, 65_536, 82, 8), (30_000, 65_535, 83, 5)]:
        pts, q = clustered_small(n=n, nq=nq, seed=seed)
        ids, d2 = ctx.k_nn(pts, q, k, s, with_d2=True)
        sel = np.random.default_rng(seed).choice(nq, 4_000, replace=False)
        sel = np.concatenate([sel, np.arange(8) * nq // 8, np.arange(1, 9) * nq // 8 - 1])
        oi, od = orc.knn(pts, q[sel], k)
        assert_same(oi, od, ids[sel], d2[sel])
        assert np.all(ids < n) and np.all(np.diff(d2, axis=1) >= 0)


@pytest.mark.parametrize("sched", [dict(), dict(use_morton_lbv=0),
                                   dict(radius_heuristic=4, leaf_size=5, morton_bits=39),
                                   dict(lanes_per_query=32)])
def test_knn_device_k_nn_one_call(rtd, orc, cuda, sched):
    """rtd_k_nn builds and searches in one call, ordering the queries on a
    second stream during the build: same ids and keys as the oracle, on
    repeated calls over different clouds and query counts."""
    ix = rtd.Index()
    s = rtd.default_schedule(**sched)
    for n, nq, seed, k in [(30_000, 3_000, 61, 5), (8_000, 9_000, 62, 16), (20_000, 1, 63, 8),
                           (3, 100, 64, 5), (0, 10, 65, 5)]:
        pts, q = clustered_small(n=max(n, 1), nq=max(nq, 1), seed=seed)
        pts, q = pts[:n], q[:nq]
        ids, d2 = ix.k_nn(torch.from_numpy(np.ascontiguousarray(pts).reshape(-1, 3)).cuda(),
                          torch.from_numpy(np.ascontiguousarray(q)).cuda(), k, s)
        torch.cuda.synchronize()
        oi, od = orc.knn(pts.reshape(-1, 3), q, k)
        assert_same(oi, od, ids.cpu().numpy().view(np.uint32), d2.cpu().numpy())


@pytest.mark.parametrize("sched", [dict(radius_heuristic=4, leaf_size=5, morton_bits=39), dict(),
                                   dict(use_morton_lbv=0), dict(lanes_per_query=32)])
def test_knn_graph_replays_whole_pipeline(rtd, orc, cuda, sched):
    """rtd_knn_graph: k_nn! captured once over fixed tensors and replayed.
    Results equal the oracle's after create and after every launch, also
    when the points' and queries' contents change between launches (each
    launch rebuilds and searches, nothing is cached); a launch counts the
    graph's kernels."""
    s = rtd.default_schedule(**sched)
    k = 5 if sched.get("lanes_per_query", 1) == 1 else 40
    pts, q = clustered_small(n=30_000, nq=4_000, seed=91)
    P, Q = torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda()
    g = rtd.KnnGraph(P, Q, k, s)
    oi, od = orc.knn(pts, q, k)
    assert_same(oi, od, g.ids.cpu().numpy().view(np.uint32), g.d2.cpu().numpy())
    lib = rtd.load()
    for seed in (92, 93):
        pts2, q2 = clustered_small(n=30_000, nq=4_000, seed=seed)
        P.copy_(torch.from_numpy(pts2))
        Q.copy_(torch.from_numpy(q2))
        before = lib.rtd_launch_count()
        ids, d2 = g.launch()
        assert lib.rtd_launch_count() - before > 10
        g.check()
        oi, od = orc.knn(pts2, q2, k)
        assert_same(oi, od, ids.cpu().numpy().view(np.uint32), d2.cpu().numpy())
    g.close()


@pytest.mark.parametrize("n,nq,k", [(1, 7, 3), (4, 5, 8), (40, 1, 5), (3_000, 2, 16), (500, 0, 5)])
def test_knn_graph_small_and_empty(rtd, orc, cuda, n, nq, k):
    """Captured pipelines over clouds whose root is a leaf, k above the
    point count, one query, and no queries: launches equal the oracle."""
    s = rtd.default_schedule(radius_heuristic=4, leaf_size=5, morton_bits=39)
    rng = np.random.default_rng(n + nq + k)
    pts = rng.random((n, 3)).astype(np.float32)
    q = rng.random((nq, 3)).astype(np.float32)
    P = torch.from_numpy(pts).cuda()
    Q = torch.from_numpy(q).cuda() if nq else torch.zeros((0, 3), device="cuda")
    g = rtd.KnnGraph(P, Q, k, s)
    for _ in range(2):
        ids, d2 = g.launch()
        g.check()
        if nq:
            oi, od = orc.knn(pts, q, k)
            assert_same(oi, od, ids.cpu().numpy().view(np.uint32), d2.cpu().numpy())
    g.close()


def _pinned(a):
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


@pytest.mark.parametrize("nq,k", [(3_000, 5), (70_001, 5), (65_536, 8)])
def test_knn_host_graph(rtd, orc, cuda, nq, k):
    """The captured host-buffer pipeline (rtd_knn_graph_create_host) copies
    in, builds, searches and copies out on every launch -- in chunks from
    65,536 queries -- and its rows equal the oracle's after the points and
    queries change in place between launches."""
    s = rtd.default_schedule(radius_heuristic=4, leaf_size=5, morton_bits=39)
    pts, q = clustered_small(n=30_000, nq=nq, seed=95)
    tp, hp = _pinned(pts)
    tq, hq = _pinned(q)
    ti = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    td = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    g = rtd.KnnHostGraph(hp, hq, k, s, out_ids=ti.numpy().view(np.uint32), out_d2=td.numpy())
    for seed in (96, 97):
        pts, q = clustered_small(n=30_000, nq=nq, seed=seed)
        hp[:] = pts
        hq[:] = q
        ids, d2 = g.launch()
        sel = np.random.default_rng(seed).choice(nq, min(nq, 3_000), replace=False)
        sel = np.concatenate([sel, [0, nq - 1]])
        oi, od = orc.knn(pts, q[sel], k)
        assert_same(oi, od, ids[sel], d2[sel])
    g.close()


def test_knn_host_graph_needs_page_locked_buffers(rtd, cuda):
    pts = np.random.default_rng(0).random((100, 3)).astype(np.float32)
    with pytest.raises(rtd.RtdError):
        rtd.KnnHostGraph(pts, pts, 4)


def test_knn_graph_rejects_bad_arguments(rtd, cuda):
    P = torch.rand((100, 3), device="cuda")
    with pytest.raises(rtd.RtdError):
        rtd.KnnGraph(P, P, 0)
    with pytest.raises(rtd.RtdError):
        rtd.KnnGraph(P, P, 4, rtd.default_schedule(radius_increment_mult=1.0))


@pytest.mark.parametrize("k", [257, 300, 1000, 2048, 2049, 5000])
def test_knn_large_k_uniform(rtd, orc, cuda, k):
    """k above the register lists (the reference's slab takes any k): the
    warp's sorted list in shared memory up to 2,048 entries, in the index's
    device slab above that.  100,000 uniform points, the plain workload's
    jittered queries (a 1,500-query slice), against the oracle."""
    pts, q = workloads.plain_knn_small()
    q = q[:1500]
    ids, d2, _ = gpu_knn(rtd, pts, q, k)
    oi, od = orc.KdTree(pts).knn(q, k)
    assert_same(oi, od, ids, d2)


@pytest.mark.parametrize("k", [300, 1000, 3000])
def test_knn_large_k_clustered(rtd, orc, cuda, k):
    """Clustered points with duplicates and far queries, k above 256."""
    pts, q = clustered_small(n=20_000, nq=800, seed=61)
    pts[::9] = pts[::9][::-1]          # shuffled duplicates
    pts[1::50] = pts[0]
    q[-20:] = q[-20:] * 5.0            # queries far outside the cloud
    ids, d2, _ = gpu_knn(rtd, pts, q, k, max_rounds=6)
    oi, od = orc.KdTree(pts).knn(q, k)
    assert_same(oi, od, ids, d2)


def test_knn_large_k_above_point_count(rtd, orc, cuda):
    """k above the number of points: every point in order, then empty slots."""
    rng = np.random.default_rng(62)
    pts = rng.random((700, 3)).astype(np.float32)
    q = rng.random((300, 3)).astype(np.float32)
    for k in (700, 701, 4000):
        ids, d2, _ = gpu_knn(rtd, pts, q, k)
        oi, od = orc.knn(pts, q, k)
        assert_same(oi, od, ids, d2)
        assert np.all(ids[:, 700:] == 0xFFFFFFFF) and np.all(np.isinf(d2[:, 700:]))


def test_knn_large_k_graph(rtd, orc, cuda):
    """The captured pipeline with k = 600 (shared-memory list) and 2,500
    (device slab): both replays exact."""
    pts, q = clustered_small(n=30_000, nq=1_000, seed=63)
    P, Q = torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda()
    tree = orc.KdTree(pts)
    for k in (600, 2500):
        g = rtd.KnnGraph(P, Q, k)
        for _ in range(2):
            ids, d2 = g.launch()
            g.check()
            oi, od = tree.knn(q, k)
            assert_same(oi, od, ids.cpu().numpy().view(np.uint32), d2.cpu().numpy())
        g.close()


def test_knn_deterministic_and_reusable_index(rtd, cuda):
    pts, q = clustered_small(n=20_000, nq=2_000, seed=18)
    s = rtd.default_schedule()
    ix = rtd.Index().build(torch.from_numpy(pts).cuda(), s)
    qt = torch.from_numpy(q).cuda()
    a, _ = ix.knn(qt, 8, s)
    b, _ = ix.knn(qt, 8, s)
    c, _ = ix.knn(qt[:100], 8, s)
    torch.cuda.synchronize()
    assert torch.equal(a, b) and torch.equal(a[:100], c)


@pytest.mark.slow
def test_knn_clustered_1p8m_window_headline(rtd, orc, cuda):
    """The 1.8M-point / 400K-query workload with the headline schedule
    (Morton-window seed, leaf 5, 39-bit keys) through rtd_k_nn: every one
    of the 400K queries against the oracle (exact k-d tree), ids and FP32
    keys bit for bit."""
    pts, q = workloads.clustered()
    win = rtd.default_schedule(radius_heuristic=4, leaf_size=5, morton_bits=39)
    ids, d2 = rtd.Index().k_nn(torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda(), 5, win)
    torch.cuda.synchronize()
    ids = ids.cpu().numpy().view(np.uint32)
    d2 = d2.cpu().numpy()
    oi, od = orc.KdTree(pts).knn(q, 5)
    assert_same(oi, od, ids, d2)


@pytest.mark.slow
def test_knn_clustered_1p8m_graph_all_queries(rtd, orc, cuda):
    """The same workload through the captured pipeline (rtd_knn_graph), the
    bench's timed path, replayed twice: every query against the oracle."""
    pts, q = workloads.clustered()
    win = rtd.default_schedule(radius_heuristic=4, leaf_size=5, morton_bits=39)
    P, Q = torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda()
    g = rtd.KnnGraph(P, Q, 5, win)
    g.launch()
    ids, d2 = g.launch()
    g.check()
    oi, od = orc.KdTree(pts).knn(q, 5)
    assert_same(oi, od, ids.cpu().numpy().view(np.uint32), d2.cpu().numpy())
    g.close()


@pytest.mark.slow
def test_knn_clustered_1p8m_all_queries(rtd, orc, cuda):
    """The 1.8M-point / 400K-query workload with the default schedule
    (sampled radius, radius rounds): every query against the oracle."""
    pts, q = workloads.clustered()
    ids, d2, _ = gpu_knn(rtd, pts, q, 5)
    oi, od = orc.KdTree(pts).knn(q, 5)
    assert_same(oi, od, ids, d2)
