"""The autotuner on small workloads with small grids: it times every
candidate through the funnel, checks that all candidates return the same
neighbours, and caches the winner under the workload's feature key, from
which schedule_for then returns it (written to a temporary cache file)."""
import numpy as np
import pytest
import torch

from rtdsl import workloads

pytestmark = pytest.mark.gpu


def test_tune_knn_small_grid(rtd, orc, cuda, tmp_path):
    from rtdsl import autotune
    path = str(tmp_path / "wisdom.json")
    pts, q = workloads.clustered(n=30_000, nq=20_000, seed=91, n_clusters=8, box=5.0)
    P, Q = torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda()
    grid = {"leaf_size": [4, 8], "morton_bits": [42, 48],
            "radius_heuristic": [rtd.RADIUS_SAMPLED_NN, rtd.RADIUS_MORTON_WINDOW],
            "mode": ["thread", "warp"]}
    best, table, key = autotune.tune_knn(P, Q, 5, grid=grid, reps=1,
                                         funnel=((2_000, 4), (8_000, 2), (20_000, 1)), path=path)
    assert key.dist == "clustered" and key.size_class == "k<=8"
    assert len(table) == 1
    got = autotune.schedule_for(key, path=path)
    assert got.as_dict() == best.as_dict()
    ix = rtd.Index().build(P, got)
    ids, d2 = ix.knn(Q, 5, got)
    oi, od = orc.KdTree(pts).knn(q, 5)
    np.testing.assert_array_equal(ids.cpu().numpy().view(np.uint32), oi)


def test_tune_range_batch_and_bh_small(rtd, cuda, tmp_path):
    from rtdsl import autotune
    from rtdsl.api import radius_for_mean_count
    path = str(tmp_path / "wisdom.json")
    pts, q = workloads.clustered(n=30_000, nq=6_000, seed=92, n_clusters=8, box=5.0)
    P, Q = torch.from_numpy(pts).cuda(), torch.from_numpy(q).cuda()
    s = rtd.default_schedule()
    r = radius_for_mean_count(rtd.Index().build(P, s), Q, 20.0, schedule=s)
    best, table, key = autotune.tune_range(P, Q, r, 20.0, grid={"leaf_size": [8, 16]}, reps=1,
                                           funnel=((2_000, 1), (6_000, 1)), path=path)
    assert key.kind == "range" and autotune.lookup(key, path)["radius"] == pytest.approx(r)

    cl = workloads.clouds(n_clouds=8, seed=93, lo=500, hi=5_000)
    bp = torch.from_numpy(np.concatenate([c["points"] for c in cl])).cuda()
    bq = torch.from_numpy(np.concatenate([c["queries"] for c in cl])).cuda()
    sizes = [(len(c["points"]), len(c["queries"]), c["k"]) for c in cl]
    best, table, key = autotune.tune_batch(bp, bq, sizes, grid={"leaf_size": [8, 32]}, reps=1,
                                           path=path)
    assert autotune.schedule_for(key, path=path).leaf_size == best.leaf_size

    pos, mass = workloads.plummer(20_000, seed=94)
    bucket, table, key = autotune.tune_bh_bucket(torch.from_numpy(pos).cuda(),
                                                 torch.from_numpy(mass).cuda(), buckets=(16, 32),
                                                 reps=1, path=path)
    assert autotune.bh_bucket_for(20_000, path=path) == bucket
