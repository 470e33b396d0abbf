"""Failure statuses of the bounded device loops, provoked without a GPU
fault: every limit here makes a loop give up early and report its status
through the C ABI, and the context stays usable afterwards.

- RTD_ERR_TIMEOUT: the bounded wait helper (spin_more) run on a device flag
  that nothing sets (rtd_wait_selftest).  No product kernel waits on
  another block: the sort and scan passes are count + scatter kernels.
- RTD_ERR_NOT_CONVERGED: the reference's round cap (schedule.partial_results)
  with a radius too small to reach k hits in max_rounds.  The partial lists
  must equal the oracle's k smallest keys within the last radius.
- RTD_ERR_OVERFLOW from the Barnes-Hut walks' traversal stack: the per-warp
  stack limit lowered with rtd_limits_set; pushes past it are refused."""
import ctypes as C

import numpy as np
import pytest
import torch

from rtdsl import workloads

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_with_timeout(rtd, cuda):
    lib = rtd.load()
    st = torch.cuda.current_stream().cuda_stream
    assert lib.rtd_wait_selftest(10_000, 0, C.c_void_p(st)) == 6        # RTD_ERR_TIMEOUT
    assert b"iteration limit" in lib.rtd_last_error()
    assert lib.rtd_wait_selftest(10_000, 1, C.c_void_p(st)) == 0        # flag set: no wait
    # the context is still usable
    x = torch.arange(10, device="cuda").sum().item()
    assert x == 45


@pytest.mark.parametrize("lanes", [1, 32])
@pytest.mark.parametrize("k", [5, 40, 300])
def test_round_cap_partial_results_not_converged(rtd, orc, cuda, lanes, k):
    """Fixed radius 0.006 on 40,000 points in the unit box, M = 2, two rounds
    (about 0.3 points expected within the last radius): most queries end
    short of k hits.  The call's device flags report NOT_CONVERGED; every
    list holds exactly the oracle's smallest keys <= the second round's
    bound, RN(RN(r*r) * RN(M*M)), then empty slots."""
    if lanes == 1 and k > 16:
        pytest.skip("thread lists hold k <= 16")
    rng = np.random.default_rng(71)
    pts = rng.random((40_000, 3)).astype(np.float32)
    q = rng.random((2_000, 3)).astype(np.float32)
    r, m = np.float32(0.006), np.float32(2.0)
    s = rtd.default_schedule(radius_heuristic=rtd.RADIUS_FIXED, radius_param=float(r),
                             radius_increment_mult=float(m), max_rounds=2, partial_results=1,
                             lanes_per_query=lanes)
    ix = rtd.Index().build(torch.from_numpy(pts).cuda(), s)
    ids, d2 = ix.knn(torch.from_numpy(q).cuda(), k, s)
    torch.cuda.synchronize()
    with pytest.raises(rtd.RtdError) as e:
        ix.info()
    assert e.value.status == 5                                          # NOT_CONVERGED
    ids = ids.cpu().numpy().view(np.uint32)
    d2 = d2.cpu().numpy()
    bound = np.float32(np.float32(r * r) * np.float32(m * m))
    oi, od = orc.knn(pts, q, k)
    keep = od <= bound
    exp_i = np.where(keep, oi, np.uint32(0xFFFFFFFF))
    exp_d = np.where(keep, od, np.float32(np.inf)).astype(np.float32)
    assert (~keep).any(axis=1).mean() > 0.5                            # most queries short
    np.testing.assert_array_equal(ids, exp_i)
    np.testing.assert_array_equal(d2.view(np.uint32), exp_d.view(np.uint32))
    # the flags were cleared by the report; an exact search on the same index is clean
    ex = rtd.default_schedule(lanes_per_query=lanes)
    ids2, d22 = ix.knn(torch.from_numpy(q).cuda(), k, ex)
    ix.info()
    np.testing.assert_array_equal(ids2.cpu().numpy().view(np.uint32), oi)


def test_round_cap_converged_is_exact(rtd, orc, cuda):
    """With enough rounds the capped search reaches k everywhere: no flag,
    exact lists."""
    pts, q = workloads.plain_knn_small(n=20_000, nq=1_000, seed=72)
    s = rtd.default_schedule(partial_results=1, max_rounds=30)
    ix = rtd.Index().build(torch.from_numpy(pts).cuda(), s)
    ids, d2 = ix.knn(torch.from_numpy(q).cuda(), 5, s)
    ix.info()
    oi, od = orc.knn(pts, q, 5)
    np.testing.assert_array_equal(ids.cpu().numpy().view(np.uint32), oi)


def _plummer_tree(rtd, n=50_000, bucket=16):
    from rtdsl._capi import BH_LAW_PLUMMER, default_bh_params
    pos, mass = workloads.plummer(n, seed=73)
    p = default_bh_params(law=BH_LAW_PLUMMER, theta=0.5, eps=1e-3, G=1.0, bucket=bucket)
    bh = rtd.BarnesHut().build(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda(), p)
    return bh, p


def _set_stack_limit(lib, entries):
    from rtdsl._capi import Limits
    lim = Limits()
    lim.bh_stack_entries = entries
    assert lib.rtd_limits_set(C.byref(lim)) == 0
    got = Limits()
    lib.rtd_limits_get(C.byref(got))
    assert got.bh_stack_entries == (entries or 8192)


def test_bh_stack_limit_overflow_reported(rtd, cuda):
    """A walk whose traversal needs more stack than the per-warp limit
    refuses the push and reports RTD_ERR_OVERFLOW (forward, the allocation
    -free forward and the adjoint); at the default limit the same tree walks
    clean and records its deepest stack."""
    lib = rtd.load()
    bh, p = _plummer_tree(rtd)
    acc, phi = bh.forward(p)
    depth = bh.info()["max_stack"]
    assert 8 < depth <= 8192
    try:
        _set_stack_limit(lib, 8)
        bh.forward(p)
        with pytest.raises(rtd.RtdError) as e:
            bh.info()
        assert e.value.status == 4                                      # OVERFLOW
        st = torch.cuda.current_stream().cuda_stream
        a2 = torch.empty_like(acc)
        f2 = torch.empty_like(phi)
        assert lib.rtd_bh_forward_noalloc(bh._h, C.byref(p), C.c_void_p(a2.data_ptr()),
                                          C.c_void_p(f2.data_ptr()), C.c_void_p(st)) == 0
        with pytest.raises(rtd.RtdError) as e:
            bh.info()
        assert e.value.status == 4
        bh.backward(acc, torch.ones_like(phi), p)
        with pytest.raises(rtd.RtdError) as e:
            bh.info()
        assert e.value.status == 4
        from rtdsl._capi import Limits
        bad = Limits()
        bad.bh_stack_entries = 9000                                     # above the maximum
        assert lib.rtd_limits_set(C.byref(bad)) == 1                    # INVALID_ARGUMENT
    finally:
        _set_stack_limit(lib, 0)
    acc3, _ = bh.forward(p)
    bh.info()
    np.testing.assert_array_equal(acc3.cpu().numpy(), acc.cpu().numpy())


def test_bh_release_frees_device_memory(rtd, cuda):
    """rtd_bh_release gives back the tree, its walk structures and stacks;
    a new build walks again with the same results."""
    bh, p = _plummer_tree(rtd, n=400_000)
    acc, _ = bh.forward(p)
    bh.backward(acc, None, p)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    bh.release()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 - free0 > 40 << 20, f"release gave back {(free1 - free0) >> 20} MiB"
    with pytest.raises(rtd.RtdError):
        bh.forward(p)
    pos, mass = workloads.plummer(400_000, seed=73)
    bh.build(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda(), p)
    acc2, _ = bh.forward(p)
    np.testing.assert_array_equal(acc2.cpu().numpy(), acc.cpu().numpy())
