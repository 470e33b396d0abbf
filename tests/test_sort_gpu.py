"""The two device primitives of the index build, through their diagnostic
entry points: the radix sort (rtd_radix_sort_pairs) against numpy's stable
argsort, and the exclusive scan with stream compaction (rtd_exclusive_scan)
against numpy's cumsum and nonzero.  64-bit keys of 33 to 48 bits take the
split sort the index build runs (one or two passes over the low bits, then
four over the top 32 bits as 32-bit keys); wider ones and 32-bit keys the
plain passes.  The sizes cross the tile (3,072 keys for the sort, 2,048
entries for the scan), group (32 tiles) and super-group (1,024 tiles)
boundaries."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SORT_TILE = 3072
SCAN_TILE = 2048
GROUP = 32


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _sort(lib, keys: np.ndarray, end_bit: int):
    kb = keys.dtype.itemsize
    tk = torch.from_numpy(keys.view(np.int64 if kb == 8 else np.int32).copy()).cuda()
    tv = torch.empty(len(keys), dtype=torch.int32, device="cuda")
    st = lib.rtd_radix_sort_pairs(C.c_void_p(tk.data_ptr()), kb, C.c_void_p(tv.data_ptr()),
                                  len(keys), end_bit, _stream())
    assert st == 0, lib.rtd_last_error()
    return (tk.cpu().numpy().view(keys.dtype), tv.cpu().numpy().view(np.uint32))


def _keys(rng, n, bits, kind, dtype):
    if kind == "uniform":
        k = rng.integers(0, 1 << bits, size=n, dtype=np.uint64)
    elif kind == "few":          # heavy duplicates: stability decides the order
        k = rng.integers(0, 7, size=n, dtype=np.uint64) << np.uint64(bits - 3)
    elif kind == "equal":
        k = np.full(n, (1 << bits) - 1, dtype=np.uint64)
    else:                        # clustered high digits, random low ones
        hi = rng.integers(0, 3, size=n, dtype=np.uint64) << np.uint64(bits - 2)
        k = hi | rng.integers(0, 1 << 12, size=n, dtype=np.uint64)
    return k.astype(dtype)


SIZES = [1, 2, 100, SORT_TILE - 1, SORT_TILE, SORT_TILE + 1, GROUP * SORT_TILE - 1,
         GROUP * SORT_TILE, GROUP * SORT_TILE + 1, (GROUP + 1) * SORT_TILE + 5]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dtype,bits", [(np.uint64, 39), (np.uint64, 33), (np.uint64, 41),
                                        (np.uint64, 56), (np.uint32, 30)])
def test_radix_sort_sizes(rtd, cuda, n, dtype, bits):
    rng = np.random.default_rng(n + bits)
    keys = _keys(rng, n, bits, "uniform", dtype)
    sk, sv = _sort(rtd.load(), keys, bits)
    ref = np.argsort(keys, kind="stable")
    assert np.array_equal(sv, ref.astype(np.uint32))
    assert np.array_equal(sk, keys[ref])


@pytest.mark.parametrize("kind", ["few", "equal", "clustered"])
@pytest.mark.parametrize("dtype,bits", [(np.uint64, 48), (np.uint64, 63), (np.uint32, 32)])
def test_radix_sort_duplicates_stable(rtd, cuda, kind, dtype, bits):
    n = 70 * SORT_TILE + 11
    keys = _keys(np.random.default_rng(5), n, bits, kind, dtype)
    sk, sv = _sort(rtd.load(), keys, bits)
    ref = np.argsort(keys, kind="stable")
    assert np.array_equal(sv, ref.astype(np.uint32))
    assert np.array_equal(sk, keys[ref])


@pytest.mark.parametrize("n", [1_800_000, 5_000_000])
def test_radix_sort_full_size_waves(rtd, cuda, n):
    """1.8M keys (586 tiles: every tile resident) and 5M keys (1,628 tiles,
    several waves), 39-bit keys as the headline index builds them."""
    keys = _keys(np.random.default_rng(n), n, 39, "uniform", np.uint64)
    sk, sv = _sort(rtd.load(), keys, 39)
    ref = np.argsort(keys, kind="stable")
    assert np.array_equal(sv, ref.astype(np.uint32))
    assert np.array_equal(sk, keys[ref])


def test_radix_sort_rejects_bad_arguments(rtd, cuda):
    lib = rtd.load()
    t = torch.zeros(4, dtype=torch.int64, device="cuda")
    v = torch.zeros(4, dtype=torch.int32, device="cuda")
    p, pv = C.c_void_p(t.data_ptr()), C.c_void_p(v.data_ptr())
    assert lib.rtd_radix_sort_pairs(p, 2, pv, 4, 8, _stream()) == 1
    assert lib.rtd_radix_sort_pairs(p, 8, pv, 4, 0, _stream()) == 1
    assert lib.rtd_radix_sort_pairs(p, 8, pv, 4, 65, _stream()) == 1
    assert lib.rtd_radix_sort_pairs(None, 8, pv, 4, 8, _stream()) == 1
    assert lib.rtd_radix_sort_pairs(None, 8, None, 0, 8, _stream()) == 0


def _scan(lib, x: np.ndarray, select: bool):
    n = len(x)
    ti = torch.from_numpy(x.view(np.int32).copy()).cuda()
    to = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    ts = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda") if select else None
    total = C.c_uint32(0xDEAD)
    st = lib.rtd_exclusive_scan(C.c_void_p(ti.data_ptr()), C.c_void_p(to.data_ptr()),
                                C.c_void_p(ts.data_ptr()) if select else None, n,
                                C.byref(total), _stream())
    assert st == 0, lib.rtd_last_error()
    out = to.cpu().numpy().view(np.uint32)[:n]
    sel = ts.cpu().numpy().view(np.uint32) if select else None
    return out, sel, total.value


SCAN_SIZES = [0, 1, 5, SCAN_TILE - 1, SCAN_TILE, SCAN_TILE + 1, GROUP * SCAN_TILE - 1,
              GROUP * SCAN_TILE, GROUP * SCAN_TILE + 1, 1_799_999, 4_000_000]


@pytest.mark.parametrize("n", SCAN_SIZES)
def test_scan_select_flags(rtd, cuda, n):
    rng = np.random.default_rng(n)
    flags = (rng.random(n) < 0.27).astype(np.uint32)
    out, sel, total = _scan(rtd.load(), flags, True)
    ref = np.cumsum(flags, dtype=np.uint64) - flags
    assert np.array_equal(out, ref.astype(np.uint32))
    assert total == int(flags.sum())
    nz = np.nonzero(flags)[0].astype(np.uint32)
    assert np.array_equal(sel[:len(nz)], nz)


@pytest.mark.parametrize("n", [GROUP * SCAN_TILE + 3, 3_000_000])
def test_scan_counts(rtd, cuda, n):
    counts = np.random.default_rng(n).integers(0, 300, size=n).astype(np.uint32)
    out, _, total = _scan(rtd.load(), counts, False)
    ref = np.cumsum(counts, dtype=np.uint64) - counts
    assert np.array_equal(out, ref.astype(np.uint32))
    assert total == int(counts.sum())
