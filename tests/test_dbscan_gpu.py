"""DBSCAN and spatial join over the range query, against the oracle's
DBSCAN (same FP32 membership, labels of the sequential expansion in index
order; itself checked against scikit-learn) and the oracle's range pairs."""
import numpy as np
import pytest
import torch

from rtdsl import workloads

pytestmark = pytest.mark.gpu


def blobs(seed, n_noise=1500):
    rng = np.random.default_rng(seed)
    parts = [rng.normal(c, s, size=(m, 3)) for c, s, m in
             ((0.2, 0.02, 1500), (0.5, 0.04, 2500), (0.8, 0.01, 800), ((0.2, 0.8, 0.5), 0.03, 1200))]
    pts = np.concatenate(parts + [rng.random((n_noise, 3))]).astype(np.float32)
    rng.shuffle(pts)
    return pts


@pytest.mark.parametrize("eps,min_pts", [(0.02, 10), (0.05, 5), (0.01, 3), (0.03, 1), (0.0, 2)])
def test_dbscan_matches_oracle(rtd, orc, cuda, eps, min_pts):
    pts = blobs(7)
    labels, nc = rtd.dbscan(torch.from_numpy(pts).cuda(), eps, min_pts)
    ref, ref_nc = orc.dbscan(pts, eps, min_pts)
    np.testing.assert_array_equal(labels.cpu().numpy(), ref)
    assert nc == ref_nc


def test_dbscan_duplicates_and_clustered(rtd, orc, cuda):
    pts, _ = workloads.clustered(n=12_000, nq=10, seed=5, n_clusters=8, box=1.0)
    pts = np.concatenate([pts, pts[:2000]])   # exact duplicates
    for eps, mp in ((0.015, 6), (0.008, 8), (0.005, 8), (0.002, 4)):
        labels, nc = rtd.dbscan(torch.from_numpy(pts).cuda(), eps, mp)
        ref, ref_nc = orc.dbscan(pts, eps, mp)
        np.testing.assert_array_equal(labels.cpu().numpy(), ref)
        assert nc == ref_nc


def test_dbscan_empty_and_errors(rtd, cuda):
    labels, nc = rtd.dbscan(torch.zeros((0, 3), device="cuda"), 0.1, 3)
    assert labels.shape == (0,) and nc == 0
    pts = torch.rand((100, 3), device="cuda")
    with pytest.raises(rtd.RtdError):
        rtd.dbscan(pts, 0.1, 0)
    ix = rtd.Index().build(torch.rand((50, 3), device="cuda"))
    with pytest.raises(rtd.RtdError):   # index over other points
        rtd.dbscan(pts, 0.1, 3, index=ix)


def test_spatial_join(rtd, orc, cuda):
    rng = np.random.default_rng(2)
    a = rng.random((5000, 3)).astype(np.float32)
    b = rng.random((3000, 3)).astype(np.float32)
    pairs = rtd.spatial_join(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), 0.05)
    np.testing.assert_array_equal(pairs.cpu().numpy().view(np.uint32), orc.range_pairs(a, b, 0.05))
    self_pairs = rtd.spatial_join(torch.from_numpy(a).cuda(), torch.from_numpy(a).cuda(), 0.03,
                                  exclude_self=True).cpu().numpy().view(np.uint32)
    ref = orc.range_pairs(a, a, 0.03)
    np.testing.assert_array_equal(self_pairs, ref[ref[:, 0] != ref[:, 1]])


def test_dbscan_reuses_index_scratch(rtd, orc, cuda):
    """DBSCAN keeps its scratch on the index: calls on one index with more,
    then fewer neighbour pairs (larger, then smaller eps) and on rebuilt
    point sets of other sizes all match the oracle."""
    ix = rtd.Index()
    for n_noise, eps, mp in ((1500, 0.02, 10), (1500, 0.06, 5), (300, 0.01, 3), (4000, 0.03, 8)):
        pts = blobs(11, n_noise=n_noise)
        P = torch.from_numpy(pts).cuda()
        ix.build(P)
        labels, nc = rtd.dbscan(P, eps, mp, index=ix)
        ref, ref_nc = orc.dbscan(pts, eps, mp)
        np.testing.assert_array_equal(labels.cpu().numpy(), ref)
        assert nc == ref_nc
