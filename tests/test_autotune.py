"""The autotuner's cache: keys from workload features (sizes, k class or
mean neighbour count, point distribution, GPU), nearest-size lookup, copies
of the default schedule, and the reference's own wisdom files read through
rtdsl.wisdom.  CPU only; the tuner itself runs in test_autotune_gpu.py."""
import glob
import os

import numpy as np
import pytest

from rtdsl import workloads

REFERENCE = "/root/reference"


def test_describe_tags_the_workloads():
    from rtdsl import autotune
    assert autotune.describe(workloads.clustered()[0]) == "clustered"
    assert autotune.describe(workloads.plain_knn_small()[0]) == "uniform"
    rng = np.random.default_rng(0)
    sheet = rng.random((50_000, 3)).astype(np.float32) * np.float32([10, 10, 1e-3])
    assert autotune.describe(sheet) == "sheet"
    assert autotune.describe(np.zeros((0, 3), np.float32)) == "uniform"


def test_keys_and_classes():
    from rtdsl import autotune
    assert [autotune.k_class(k) for k in (1, 5, 8, 9, 32, 64, 200, 257, 5000)] == \
        ["k=1", "k<=8", "k<=8", "k<=16", "k<=32", "k<=64", "k<=256", "k>256", "k>256"]
    k = autotune.knn_key(1_800_000, 400_000, 5, "clustered", "G")
    assert k.text() == "knn|n=2^21|q=2^19|k<=8|clustered|G"
    assert autotune.WorkloadKey.parse(k.text()) == k
    assert autotune.WorkloadKey.parse("clustered_1p8m_k5") is None
    r = autotune.range_key(1_800_000, 400_000, 50, "clustered", "G")
    assert r.size_class == "r~2^6"


def test_lookup_exact_nearest_and_miss(tmp_path, rtd):
    from rtdsl import autotune
    path = str(tmp_path / "wisdom.json")
    g = "GPU-X"
    s = rtd.default_schedule(leaf_size=7, morton_bits=45)
    autotune.save(autotune.knn_key(1 << 20, 1 << 18, 5, "clustered", g), s, {"n": 1 << 20},
                  path)
    s2 = rtd.default_schedule(leaf_size=3)
    autotune.save(autotune.knn_key(1 << 24, 1 << 22, 5, "clustered", g), s2, {}, path)
    # exact
    got = autotune.schedule_for(autotune.knn_key(1 << 20, 1 << 18, 5, "clustered", g), path=path)
    assert (got.leaf_size, got.morton_bits) == (7, 45)
    # nearest within a factor 4: 2^21 points -> the 2^20 entry; 2^23 -> the 2^24 one
    got = autotune.schedule_for(autotune.knn_key(3 << 20, 1 << 19, 8, "clustered", g), path=path)
    assert got.leaf_size == 7
    got = autotune.schedule_for(autotune.knn_key(1 << 23, 1 << 21, 6, "clustered", g), path=path)
    assert got.leaf_size == 3
    # another distribution, k class, GPU, or a size too far: defaults
    base = rtd.default_schedule()
    for key in (autotune.knn_key(1 << 20, 1 << 18, 5, "uniform", g),
                autotune.knn_key(1 << 20, 1 << 18, 64, "clustered", g),
                autotune.knn_key(1 << 20, 1 << 18, 5, "clustered", "GPU-Y"),
                autotune.knn_key(1 << 14, 1 << 12, 5, "clustered", g)):
        assert autotune.schedule_for(key, base, path=path).as_dict() == base.as_dict()
    assert autotune.bh_bucket_for(1 << 20, default=48, path=path) == 48


def test_shipped_cache_covers_the_bench_workloads(rtd):
    """wisdom.json holds tuned entries for the bench's workloads on B200."""
    from rtdsl import autotune
    g = "NVIDIA B200"
    pts, q = workloads.clustered()
    s = autotune.schedule_for(autotune.knn_key(len(pts), len(q), 5, "clustered", g))
    assert s.as_dict() != rtd.default_schedule().as_dict()
    assert autotune.lookup(autotune.range_key(len(pts), len(q), 50, "clustered", g))
    assert autotune.lookup(autotune.batch_key(8_961_867, 2_240_466, 256, g))
    assert autotune.lookup(autotune.bh_key(1_000_000, "plummer", g))["bucket"] in (16, 32, 64)


@pytest.mark.skipif(not os.path.isdir(REFERENCE), reason="reference checkout not present")
def test_reference_wisdom_files_load(rtd):
    """The reference's shipped wisdom files (*_wisdom.json at its top level,
    written by its profiler) read into rtd_schedule.  They hold
    radius_increment_mult, max_hits_per_query, use_morton_lbv,
    radius_heuristic and memory_strategy only (no build_strategy or
    geom_type); the fields without a counterpart are ignored."""
    import json
    from rtdsl import wisdom
    files = sorted(glob.glob(os.path.join(REFERENCE, "*_wisdom.json")))
    assert len(files) >= 4
    for f in files:
        d = json.load(open(f))
        s = wisdom.load(f)
        assert s.radius_increment_mult == pytest.approx(d["radius_increment_mult"])
        assert s.use_morton_lbv == int(bool(d["use_morton_lbv"]))
        h = d["radius_heuristic"]
        assert s.radius_heuristic == rtd.RADIUS_SAMPLED_PERCENTILE
        assert s.radius_param == pytest.approx(h["SampledPercentile"])
        # and written back in the reference's layout with its defaults filled in
        back = wisdom.wisdom_from_schedule(s)
        assert back["radius_heuristic"] == {"SampledPercentile": pytest.approx(h["SampledPercentile"])}
        assert set(back) >= set(d)
