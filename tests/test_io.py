"""The reference harness's formats: point files parsed as load_points_fast
does (gprt-sandbox/src/io.rs:8-30), knn_results.txt lines as the Rust
driver writes them and validate_full.py reads them back.  CPU only."""
import re

import numpy as np
import pytest

FLOAT = re.compile(r"^[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?$|^[+-]?(inf|infinity|nan)$", re.I)


def rust_like(text: str) -> np.ndarray:
    """Restatement of the loader's filter: lines split on '\\n', empty lines
    skipped, first three ','-fields trimmed and parsed, else the line is
    skipped."""
    out = []
    for line in text.split("\n"):
        if not line:
            continue
        f = line.split(",")
        if len(f) < 3:
            continue
        vals = [s.strip() for s in f[:3]]
        if all(FLOAT.match(v) for v in vals):
            out.append([np.float32(float(v)) for v in vals])
    return np.array(out, dtype=np.float32).reshape(-1, 3)


def test_point_file_edge_cases(tmp_path, rtd):
    from rtdsl.io import load_points_csv
    text = ("1,2,3\n"
            "\n"
            "  4.5 , -6e-3,\t7E2  \r\n"
            "1,2\n"                      # too few fields
            "a,b,c\n"                    # not numbers
            "8,9,10,extra,fields\n"
            "0x10,1,2\n"                 # hex is not a Rust f32
            "+1.,.5,-inf\n"
            "nan,INF,Infinity\n"
            "1 2,3,4\n"                  # inner space
            "11,12,13")                  # no final newline
    p = tmp_path / "pts.csv"
    p.write_text(text)
    got = load_points_csv(str(p))
    ref = rust_like(text)
    assert got.shape == (6, 3)
    np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_point_file_large_parallel(tmp_path, rtd):
    """Several MB: parsed in parallel chunks, line order kept."""
    from rtdsl.io import load_points_csv
    rng = np.random.default_rng(0)
    pts = (rng.random((150_000, 3)) * 100 - 50).astype(np.float32)
    lines = [f"{x!r},{y!r},{z!r}" for x, y, z in pts.tolist()]
    lines[1000] = "broken,line"
    p = tmp_path / "big.csv"
    p.write_text("\n".join(lines) + "\n")
    got = load_points_csv(str(p))
    want = np.delete(pts, 1000, axis=0)
    np.testing.assert_array_equal(got, want)


def test_knn_results_round_trip(tmp_path):
    from rtdsl.io import result_line, write_knn_results
    ids = np.array([[3, 1, 2], [5, 0xFFFFFFFF, 0xFFFFFFFF], [7, 8, 9]], dtype=np.uint32)
    path = tmp_path / "knn_results.txt"
    write_knn_results(str(path), ids)
    lines = path.read_text().splitlines()
    assert lines[0] == "Q0:[3, 1, 2]" and lines[1] == "Q1:[5]"
    for i, line in enumerate(lines):   # as gprt-sandbox/validate_full.py parses it
        neighbors = eval(line.strip().split(":")[1])
        assert neighbors == [int(v) for v in ids[i] if v != 0xFFFFFFFF]
    assert result_line("data.csv", 3, 3, 1.23456, 7) == "data.csv,3,3,1.235,7"


def test_reference_wisdom_round_trip(tmp_path, rtd):
    """gprt_wisdom.json (serde JSON of gprt_ir::Schedule) maps onto
    rtd_schedule and back."""
    from rtdsl import wisdom
    text = """{
  "radius_increment_mult": 2.5,
  "max_hits_per_query": 512,
  "use_morton_lbv": true,
  "radius_heuristic": {"SampledPercentile": 0.05},
  "memory_strategy": "GlobalMemory",
  "build_strategy": "PreferFastBuild",
  "geom_type": "Spheres"
}"""
    s = wisdom.schedule_from_wisdom(text)
    assert s.radius_increment_mult == 2.5 and s.use_morton_lbv == 1
    assert s.radius_heuristic == rtd.RADIUS_SAMPLED_PERCENTILE and abs(s.radius_param - 0.05) < 1e-7
    for h, (mode, param) in (("\"SampledMax\"", (rtd.RADIUS_SAMPLED_MAX, 1.0)),
                             ("{\"Fixed\": 0.25}", (rtd.RADIUS_FIXED, 0.25))):
        s2 = wisdom.schedule_from_wisdom('{"radius_heuristic": %s}' % h)
        assert (s2.radius_heuristic, s2.radius_param) == (mode, param)
    p = tmp_path / "gprt_wisdom.json"
    wisdom.save(str(p), s)
    back = wisdom.load(str(p))
    assert back.as_dict() == s.as_dict()
    import json
    d = json.loads(p.read_text())
    assert d["radius_heuristic"] == {"SampledPercentile": float(np.float32(0.05))}
    assert set(d) == set(wisdom.REFERENCE_DEFAULTS)
    with pytest.raises(ValueError):
        wisdom.schedule_from_wisdom('{"radius_heuristic": {"Bogus": 1}}')
