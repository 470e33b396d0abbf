"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/rtdsl.h declares, and rejects bad arguments before touching the
device."""
import ctypes as C
import os
import re

import pytest

from conftest import REPO


def _header_functions():
    hdrs = [os.path.join(REPO, "include", f) for f in os.listdir(os.path.join(REPO, "include"))
            if f.endswith(".h")]
    names = set()
    for h in hdrs:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(rtd_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_symbols_exported(rtd):
    lib = rtd.load()
    names = _header_functions()
    assert "rtd_knn" in names and "rtd_index_build" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_header(rtd):
    from rtdsl import _capi
    assert set(_header_functions()) <= set(_capi.declared_symbols())


def test_schedule_defaults(rtd):
    s = rtd.default_schedule()
    assert s.radius_increment_mult == 2.0
    assert s.radius_heuristic == rtd.RADIUS_SAMPLED_NN
    assert abs(s.radius_param - 2 ** -4) < 1e-12
    assert s.use_morton_lbv == 1 and s.leaf_size == 4 and s.max_rounds == 32


def test_cached_schedule_leaves_default_alone(rtd):
    from rtdsl import autotune
    base = rtd.default_schedule()
    before = base.as_dict()
    g = "NVIDIA B200"
    for key in (autotune.knn_key(1_800_000, 400_000, 5, "clustered", g),
                autotune.range_key(1_800_000, 400_000, 50, "clustered", g),
                autotune.batch_key(8_961_867, 2_240_466, 256, g),
                autotune.knn_key(10, 10, 5, "sheet", "no such GPU")):
        s = autotune.schedule_for(key, base)
        assert s is not base
    assert base.as_dict() == before


def test_status_strings(rtd):
    lib = rtd.load()
    assert lib.rtd_status_string(0) == b"RTD_OK"
    assert lib.rtd_status_string(4) == b"RTD_ERR_OVERFLOW"
    assert lib.rtd_version() == 100


def test_invalid_arguments_without_device(rtd):
    lib = rtd.load()
    s = rtd.default_schedule()
    # NULL index / NULL out pointers are rejected on the host
    assert lib.rtd_knn(None, None, 0, 5, C.byref(s), None, None, None) == 1
    assert lib.rtd_index_create(None) == 1
    assert b"NULL" in lib.rtd_last_error() or b"not built" in lib.rtd_last_error()
    h = C.c_void_p()
    assert lib.rtd_index_create(C.byref(h)) == 0
    # an index that was never built refuses searches
    assert lib.rtd_knn(h, None, 10, 5, C.byref(s), None, None, None) == 1
    assert lib.rtd_index_destroy(h) == 0


def test_sort_and_scan_diagnostics_reject_bad_arguments_without_device(rtd):
    """rtd_radix_sort_pairs / rtd_exclusive_scan check their arguments on
    the host before any device call; n = 0 is a no-op."""
    lib = rtd.load()
    p = C.c_void_p(16)   # never dereferenced: each call fails or returns first
    assert lib.rtd_radix_sort_pairs(p, 2, p, 4, 8, None) == 1          # key_bytes
    assert lib.rtd_radix_sort_pairs(p, 8, p, 4, 0, None) == 1          # end_bit 0
    assert lib.rtd_radix_sort_pairs(p, 4, p, 4, 33, None) == 1         # end_bit > 32
    assert lib.rtd_radix_sort_pairs(None, 8, p, 4, 39, None) == 1      # NULL keys
    assert lib.rtd_radix_sort_pairs(p, 8, None, 4, 39, None) == 1      # NULL values
    assert lib.rtd_radix_sort_pairs(None, 8, None, 0, 39, None) == 0   # nothing to sort
    assert lib.rtd_exclusive_scan(None, p, None, 5, None, None) == 1   # NULL input
    assert lib.rtd_exclusive_scan(p, None, None, 5, None, None) == 1   # NULL output


def test_python_api_rejects_bad_shapes(rtd):
    from rtdsl.api import _as_vec3
    with pytest.raises(ValueError):
        _as_vec3([[1.0, 2.0]], "data")
    assert _as_vec3([[1, 2, 3]], "q").dtype.name == "float32"
