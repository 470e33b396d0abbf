"""Batched many-cloud k-NN: every cloud's result must equal the oracle's
exact k-NN of that cloud alone, bit for bit (cloud-local ids, FP32 keys),
whether the pass runs eagerly or as a replayed CUDA graph; the batched
backward must equal the analytic gradient of the returned distances."""
import numpy as np
import pytest
import torch

from rtdsl import workloads

pytestmark = pytest.mark.gpu


def packed(cl):
    pts = np.concatenate([c["points"] for c in cl]).astype(np.float32)
    q = np.concatenate([c["queries"] for c in cl]).astype(np.float32)
    sizes = [(len(c["points"]), len(c["queries"]), c["k"]) for c in cl]
    return pts, q, sizes


def check_against_oracle(orc, batch, cl, ids, d2):
    ids = ids.cpu().numpy().view(np.uint32)
    d2 = d2.cpu().numpy()
    for c, (ci, cd) in enumerate(zip(batch.split(ids), batch.split(d2))):
        oi, od = orc.knn(cl[c]["points"], cl[c]["queries"], cl[c]["k"])
        bad = np.nonzero(np.any(oi != ci, axis=1))[0]
        assert len(bad) == 0, f"cloud {c} (k={cl[c]['k']}): {len(bad)} queries differ"
        np.testing.assert_array_equal(od.view(np.uint32), cd.view(np.uint32))


def mixed_clouds(seed=5):
    """Clouds of 0 .. 20,000 points, k from 1 to 3,000 (every k class of the
    search, the memory list above 256 included), duplicates, k above the
    cloud size and a cloud without queries."""
    rng = np.random.default_rng(seed)
    cl = []
    for c, (n, k) in enumerate([(20_000, 5), (1, 1), (3, 8), (1500, 16), (0, 4), (700, 32),
                                (4000, 64), (900, 200), (12_000, 1), (50, 64), (2, 2),
                                (5000, 12), (6000, 40), (8, 16), (3000, 300), (8000, 1000),
                                (150, 400), (5000, 3000)]):
        if c % 3 == 0:
            p = rng.random((n, 3)) * (1 + c)
        elif c % 3 == 1:
            p = rng.normal(size=(n, 3)) * 0.01 + c
        else:
            base = rng.random((max(n // 4, 1), 3))
            p = base[rng.integers(0, len(base), size=n)] if n else np.zeros((0, 3))
        p = p.astype(np.float32)
        nq = 0 if c == 9 else max(1, n // 3 + 7)
        lo = p.min(0) if n else np.zeros(3)
        hi = p.max(0) if n else np.ones(3)
        q = (lo + (hi - lo) * rng.random((nq, 3)) * 1.1 - 0.05 * (hi - lo)).astype(np.float32)
        cl.append({"points": p.reshape(-1, 3), "queries": q, "k": k})
    return cl


@pytest.mark.parametrize("use_graph", [False, True])
def test_batched_mixed_clouds(rtd, orc, cuda, use_graph):
    cl = mixed_clouds()
    pts, q, sizes = packed(cl)
    b = rtd.Batch(sizes)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        P, Q = torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda()
        for _ in range(2 if use_graph else 1):   # capture, then replay
            ids, d2 = b.knn(P, Q, use_graph=use_graph, stream=st)
            st.synchronize()
            check_against_oracle(orc, b, cl, ids, d2)


@pytest.mark.parametrize("leaf", [1, 4, 16])
def test_batched_workload_clouds(rtd, orc, cuda, leaf):
    """64 clouds of the many-cloud workload (uniform and clustered, k in
    {1, 5, 16, 64}), scaled down."""
    cl = workloads.clouds(n_clouds=64, seed=7, lo=200, hi=20_000)
    pts, q, sizes = packed(cl)
    b = rtd.Batch(sizes, rtd.default_schedule(leaf_size=leaf))
    ids, d2 = b.knn(torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda())
    torch.cuda.synchronize()
    check_against_oracle(orc, b, cl, ids, d2)


@pytest.mark.slow
@pytest.mark.parametrize("tuned", [False, True])
def test_batched_full_256_clouds(rtd, orc, cuda, tuned):
    """The full many-cloud workload (256 clouds, 1,000-200,000 points each,
    k in {1, 5, 16, 64}) in one batched pass with the default and the tuned
    schedule: every query of every cloud against the oracle's exact k-NN of
    that cloud (k-d tree), ids and FP32 keys bit for bit."""
    from rtdsl import autotune
    cl = workloads.clouds()
    assert len(cl) == 256
    pts, q, sizes = packed(cl)
    s = autotune.schedule_for(autotune.batch_key(len(pts), len(q), len(cl)),
                              rtd.default_batch_schedule()) if tuned else None
    b = rtd.Batch(sizes, s)
    ids, d2 = b.knn(torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda(), use_graph=tuned)
    torch.cuda.synchronize()
    ids = ids.cpu().numpy().view(np.uint32)
    d2 = d2.cpu().numpy()
    for c, (ci, cd) in enumerate(zip(b.split(ids), b.split(d2))):
        oi, od = orc.KdTree(cl[c]["points"]).knn(cl[c]["queries"], cl[c]["k"])
        bad = np.nonzero(np.any(oi != ci, axis=1))[0]
        assert len(bad) == 0, f"cloud {c} (k={cl[c]['k']}): {len(bad)} queries differ"
        np.testing.assert_array_equal(od.view(np.uint32), cd.view(np.uint32))


def test_batched_fixed_radius_schedule(rtd, orc, cuda):
    """A fixed initial radius far too small still ends exact (radius expansion
    then the unbounded last round)."""
    cl = workloads.clouds(n_clouds=12, seed=9, lo=500, hi=5000)
    pts, q, sizes = packed(cl)
    s = rtd.default_schedule(radius_heuristic=rtd.RADIUS_FIXED, radius_param=1e-6, max_rounds=4)
    b = rtd.Batch(sizes, s)
    ids, d2 = b.knn(torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda())
    torch.cuda.synchronize()
    check_against_oracle(orc, b, cl, ids, d2)


def test_batched_graph_replay(rtd, orc, cuda):
    """The captured graph replays the whole pass: new data written into the
    same buffers gives that data's exact result."""
    cl_a = workloads.clouds(n_clouds=24, seed=21, lo=300, hi=8000)
    rng = np.random.default_rng(4)
    cl_b = [{"points": (c["points"] + rng.normal(size=c["points"].shape) * 0.02).astype(np.float32),
             "queries": c["queries"], "k": c["k"]} for c in cl_a]
    pa, qa, sizes = packed(cl_a)
    pb, _, _ = packed(cl_b)
    b = rtd.Batch(sizes)
    dp = torch.from_numpy(pa).cuda()
    dq = torch.from_numpy(qa).cuda()
    ids = torch.empty(b.n_out, dtype=torch.int32, device=cuda)
    d2 = torch.empty(b.n_out, dtype=torch.float32, device=cuda)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        b.knn(dp, dq, ids, d2, use_graph=True, stream=st)      # eager + capture
        st.synchronize()
        check_against_oracle(orc, b, cl_a, ids, d2)
        ids.fill_(-1)
        b.knn(dp, dq, ids, d2, use_graph=True, stream=st)      # replay
        st.synchronize()
        check_against_oracle(orc, b, cl_a, ids, d2)
        dp.copy_(torch.from_numpy(pb).cuda())
        b.knn(dp, dq, ids, d2, use_graph=True, stream=st)      # replay, new points
        st.synchronize()
        check_against_oracle(orc, b, cl_b, ids, d2)


def test_batched_backward(rtd, cuda):
    """grad_q = sum_j 2 g_j (q - p_j), grad_p[p_j] -= 2 g_j (q - p_j), against an
    FP64 restatement with the same ids."""
    cl = workloads.clouds(n_clouds=10, seed=13, lo=300, hi=3000)
    pts, q, sizes = packed(cl)
    b = rtd.Batch(sizes)
    dp = torch.from_numpy(pts).cuda()
    dq = torch.from_numpy(q).cuda()
    ids, d2 = b.knn(dp, dq)
    g = torch.randn(b.n_out, device=cuda)
    gq, gp = b.backward(dp, dq, ids, g)
    torch.cuda.synchronize()
    ids_h = ids.cpu().numpy().view(np.uint32)
    g_h = g.cpu().numpy().astype(np.float64)
    eq = np.zeros((len(q), 3))
    ep = np.zeros((len(pts), 3))
    for c, (npnt, nq, k) in enumerate(sizes):
        po, qo, oo = int(b.point_offset[c]), int(b.query_offset[c]), int(b.out_offset[c])
        cid = ids_h[oo:oo + nq * k].reshape(nq, k)
        cg = g_h[oo:oo + nq * k].reshape(nq, k)
        for j in range(k):
            ok = cid[:, j] != 0xFFFFFFFF
            pi = po + cid[ok, j].astype(np.int64)
            diff = q[qo:qo + nq][ok].astype(np.float64) - pts[pi].astype(np.float64)
            w = 2.0 * cg[ok, j][:, None]
            eq[qo:qo + nq][ok] += w * diff
            np.add.at(ep, pi, -w * diff)
    np.testing.assert_allclose(gq.cpu().numpy(), eq, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(gp.cpu().numpy(), ep, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("lanes,param,mult", [(32, 1.0, 2.0), (0, 0.25, 4.0), (0, 4.0, 2.0)])
def test_batched_schedules(rtd, orc, cuda, lanes, param, mult):
    """Warp-per-query search for every k <= 32 and other radius settings give
    the same exact result."""
    cl = mixed_clouds(seed=8)
    pts, q, sizes = packed(cl)
    s = rtd.default_batch_schedule(lanes_per_query=lanes, radius_param=param,
                                   radius_increment_mult=mult)
    b = rtd.Batch(sizes, s)
    ids, d2 = b.knn(torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda())
    torch.cuda.synchronize()
    check_against_oracle(orc, b, cl, ids, d2)


def test_batched_backward_central_differences(rtd, cuda):
    """The loss of the many-cloud workload, L = sum_q mean_j d2_qj with ids
    fixed, differentiated by the batched backward, against FP64 central
    differences (h = 1e-4) on 64 sampled query and point coordinates."""
    cl = workloads.clouds(n_clouds=16, seed=17, lo=200, hi=4000)
    pts, q, sizes = packed(cl)
    b = rtd.Batch(sizes)
    dp = torch.from_numpy(pts).cuda()
    dq = torch.from_numpy(q).cuda()
    ids, _ = b.knn(dp, dq)
    g = torch.empty(b.n_out, device=cuda)
    for c, (_, nq, k) in enumerate(sizes):
        o = int(b.out_offset[c])
        g[o:o + nq * k] = 1.0 / k
    gq, gp = b.backward(dp, dq, ids, g)
    torch.cuda.synchronize()
    ids_h = ids.cpu().numpy().view(np.uint32)
    # flat (query row, point row) index of every output slot
    qrow = np.empty(b.n_out, np.int64)
    prow = np.empty(b.n_out, np.int64)
    wt = np.empty(b.n_out)
    for c, (_, nq, k) in enumerate(sizes):
        o = int(b.out_offset[c])
        qrow[o:o + nq * k] = int(b.query_offset[c]) + np.repeat(np.arange(nq), k)
        loc = ids_h[o:o + nq * k].astype(np.int64)
        prow[o:o + nq * k] = int(b.point_offset[c]) + np.where(loc == 0xFFFFFFFF, 0, loc)
        wt[o:o + nq * k] = np.where(loc == 0xFFFFFFFF, 0.0, 1.0 / k)

    def loss(Q, P):
        d = Q[qrow] - P[prow]
        return float(np.sum(wt * np.sum(d * d, axis=1)))

    Q64 = q.astype(np.float64)
    P64 = pts.astype(np.float64)
    rng = np.random.default_rng(0)
    h = 1e-4
    for which, arr, grad in (("q", Q64, gq.cpu().numpy()), ("p", P64, gp.cpu().numpy())):
        used = np.unique(qrow if which == "q" else prow[wt > 0])
        for _ in range(32):
            r = int(rng.choice(used))
            a = int(rng.integers(0, 3))
            old = arr[r, a]
            arr[r, a] = old + h
            lp = loss(Q64, P64)
            arr[r, a] = old - h
            lm = loss(Q64, P64)
            arr[r, a] = old
            fd = (lp - lm) / (2 * h)
            assert abs(grad[r, a] - fd) <= 1e-4 * max(1.0, abs(fd)), (which, r, a, grad[r, a], fd)
