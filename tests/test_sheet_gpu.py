"""The dense-cluster stress workload at full size: 10M points on a thin
sheet (z ~ N(0, 1e-4)) drawn from 2,000 Zipf-weighted Gaussian hotspots
(sigma 1e-3 .. 1e-1 in [0,10]^2), 1M queries from the same distribution.
k in {5, 16, 64} (k = 64 runs the warp-striped list) and a range query
at the radius of 200 mean neighbours (a heavy-tailed, exactly sized
output).  Checked against the oracle (exact k-d tree) bit for bit: the
k-NN ids and FP32 keys and the range count of every query, and the range
pairs of a 20,000-query sample."""
import numpy as np
import pytest
import torch

from rtdsl import workloads

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


@pytest.fixture(scope="module")
def sheet(cuda):
    pts, q = workloads.sheet()
    return pts, q, torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda()


@pytest.fixture(scope="module")
def sheet_tree(orc, sheet):
    return orc.KdTree(sheet[0])


@pytest.fixture(scope="module")
def sheet_index(rtd, sheet):
    s = rtd.default_schedule()
    return rtd.Index().build(sheet[2], s), s


@pytest.mark.parametrize("k", [5, 16, 64])
def test_sheet_knn(rtd, orc, sheet, sheet_index, sheet_tree, k):
    pts, q, P, Q = sheet
    ix, s = sheet_index
    ids, d2 = ix.knn(Q, k, s)
    torch.cuda.synchronize()
    info = ix.info()
    assert info["morton_bits"] == 48
    ids = ids.cpu().numpy().view(np.uint32)
    d2 = d2.cpu().numpy()
    assert np.all(ids < len(pts))
    assert np.all(np.diff(d2, axis=1) >= 0)
    oi, od = sheet_tree.knn(q, k)
    bad = np.nonzero(np.any(ids != oi, axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} of {len(q)} queries differ, first {bad[:5]}"
    np.testing.assert_array_equal(d2.view(np.uint32), od.view(np.uint32))


def test_sheet_range_mean_200(rtd, orc, sheet, sheet_index, sheet_tree):
    from rtdsl.api import radius_for_mean_count
    pts, q, P, Q = sheet
    ix, s = sheet_index
    r = radius_for_mean_count(ix, Q, 200.0, schedule=s)
    counts, total = ix.range_count(Q, r, s)
    pairs = ix.range_fill(Q, r, total, sort_pairs=False, schedule=s)
    torch.cuda.synchronize()
    assert 180 <= total / len(q) <= 220
    c = counts.cpu().numpy().view(np.uint32)
    assert c.sum() == total == pairs.shape[0]
    assert c.max() > 10 * 200          # heavy tail in the dense hotspots
    per_q = torch.bincount(pairs[:, 0].long(), minlength=len(q)).cpu().numpy()
    np.testing.assert_array_equal(per_q, c)
    oc, ot = sheet_tree.range_count(q, r)
    np.testing.assert_array_equal(c, oc)
    # every pair of a 20,000-query sample equals the oracle's
    sel = np.sort(np.random.default_rng(1).choice(len(q), 20_000, replace=False))
    p = pairs.cpu().numpy().view(np.uint32)
    mine = p[np.isin(p[:, 0], sel)]
    ref = sheet_tree.range_pairs(q[sel], r)
    ref[:, 0] = sel[ref[:, 0]]
    key = lambda a: np.sort(a[:, 0].astype(np.uint64) << np.uint64(32) | a[:, 1].astype(np.uint64))
    np.testing.assert_array_equal(key(mine), key(ref))
