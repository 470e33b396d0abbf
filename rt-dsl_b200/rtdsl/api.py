"""Host-side mirror of the reference's search API over the C ABI.

``k_nn`` / ``range_query`` / ``barnes_hut`` keep the argument meaning of the
reference macros (gprt-macros/src/lib.rs:408 ``k_nn!(data, queries, k, out
[, schedule])``, README ``range_query!``, lib.rs:752 ``barnes_hut!(bodies,
theta, G, out)``): data and queries are Vec3 arrays (N x 3 float32), k_nn
returns one id list per query sorted by distance.  ``Index`` is the
device-tensor interface (torch CUDA tensors in, torch CUDA tensors out, on
the current stream).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import EMPTY_ID, RtdError, Schedule, check, default_schedule, load


def _as_vec3(a, name: str) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if arr.ndim != 2 or arr.shape[1] != 3:
        raise ValueError(f"{name} must be an (N, 3) array of Vec3, got shape {arr.shape}")
    return arr


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a.size else None


class Context:
    """rtd_context: device staging buffers + a stream for host-buffer calls."""

    def __init__(self):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.rtd_context_create(C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rtd_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def k_nn(self, data, queries, k: int, schedule: Schedule | None = None,
             with_d2: bool = False, out_ids: np.ndarray | None = None,
             out_d2: np.ndarray | None = None):
        data = _as_vec3(data, "data")
        queries = _as_vec3(queries, "queries")
        nq = queries.shape[0]
        ids = out_ids if out_ids is not None else np.empty((nq, k), dtype=np.uint32)
        d2 = out_d2 if out_d2 is not None else (np.empty((nq, k), dtype=np.float32) if with_d2 else None)
        s = schedule if schedule is not None else default_schedule()
        check(self._lib.rtd_k_nn_host(self._h, _ptr(data), data.shape[0], _ptr(queries), nq, k,
                                      C.byref(s), _ptr(ids), _ptr(d2) if d2 is not None else None))
        return (ids, d2) if with_d2 else ids

    def range_query(self, data, queries, radius: float, capacity: int | None = None) -> np.ndarray:
        data = _as_vec3(data, "data")
        queries = _as_vec3(queries, "queries")
        n_pairs = C.c_uint64(0)
        if capacity is None:
            # size by a first call with no room, as the count pass reports it
            st = self._lib.rtd_range_query_host(self._h, _ptr(data), data.shape[0], _ptr(queries),
                                                queries.shape[0], C.c_float(radius), None, 0,
                                                C.byref(n_pairs))
            if st not in (_capi.RTD_OK, _capi.RTD_ERR_OVERFLOW):
                check(st)
            capacity = n_pairs.value
        pairs = np.empty((max(capacity, 1), 2), dtype=np.uint32)
        check(self._lib.rtd_range_query_host(self._h, _ptr(data), data.shape[0], _ptr(queries),
                                             queries.shape[0], C.c_float(radius), _ptr(pairs),
                                             capacity, C.byref(n_pairs)))
        return pairs[: n_pairs.value]


_ctx: Context | None = None


def _context() -> Context:
    global _ctx
    if _ctx is None:
        _ctx = Context()
    return _ctx


def k_nn(data, queries, k: int, schedule: Schedule | None = None) -> list[list[int]]:
    """k_nn!(data, queries, k, out[, schedule]): per query, its k nearest
    point ids sorted by distance (ties to the lower id).  Slots past the
    number of points are dropped, as a Vec<Vec<u32>> would be shorter."""
    ids = _context().k_nn(data, queries, k, schedule)
    return [[int(v) for v in row if v != EMPTY_ID] for row in ids]


def k_nn_array(data, queries, k: int, schedule: Schedule | None = None, with_d2: bool = True):
    """Array form of k_nn: ids [Q, k] uint32 (EMPTY_ID padded), d2 [Q, k]."""
    return _context().k_nn(data, queries, k, schedule, with_d2=with_d2)


def range_query(data, queries, radius: float) -> np.ndarray:
    """range_query!(data, queries, r, out): (query, id) uint32 pairs of every
    point within r of every query, sorted by (query, id)."""
    return _context().range_query(data, queries, radius)


# --------------------------------------------------------------- devices
def _stream_handle(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _check_points_tensor(t, name: str):
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.float32 or t.dim() != 2 or t.shape[1] != 3 or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous float32 (N, 3) tensor")


class Index:
    """rtd_index over a CUDA tensor of points (N x 3 float32)."""

    def __init__(self):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.rtd_index_create(C.byref(h)))
        self._h = h
        self.points = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rtd_index_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self, points, schedule: Schedule | None = None, stream=None) -> "Index":
        _check_points_tensor(points, "points")
        s = schedule if schedule is not None else default_schedule()
        check(self._lib.rtd_index_build(self._h, C.c_void_p(points.data_ptr()), points.shape[0],
                                        C.byref(s), _stream_handle(stream)))
        self.points = points
        return self

    def profile(self, enable: bool = True) -> "Index":
        check(self._lib.rtd_index_profile_enable(self._h, int(enable)))
        return self

    def timings(self) -> dict:
        """Phase times (ms) of the last build and search, from CUDA events."""
        p = _capi.Profile()
        check(self._lib.rtd_index_profile_get(self._h, C.byref(p)))
        return p.as_dict()

    def info(self, stream=None) -> dict:
        inf = _capi.IndexInfo()
        check(self._lib.rtd_index_info_get(self._h, C.byref(inf), _stream_handle(stream)))
        return {"n_points": inf.n_points, "n_internal": inf.n_internal,
                "leaf_size": inf.leaf_size, "morton_bits": inf.morton_bits,
                "lo": list(inf.lo), "hi": list(inf.hi)}

    def knn(self, queries, k: int, schedule: Schedule | None = None, with_d2: bool = True,
            out_ids=None, out_d2=None, stream=None):
        import torch
        _check_points_tensor(queries, "queries")
        nq = queries.shape[0]
        dev = queries.device
        ids = out_ids if out_ids is not None else torch.empty((nq, k), dtype=torch.int32, device=dev)
        d2 = out_d2 if out_d2 is not None else (
            torch.empty((nq, k), dtype=torch.float32, device=dev) if with_d2 else None)
        s = schedule if schedule is not None else default_schedule()
        check(self._lib.rtd_knn(self._h, C.c_void_p(queries.data_ptr()), nq, k, C.byref(s),
                                C.c_void_p(ids.data_ptr()),
                                C.c_void_p(d2.data_ptr()) if d2 is not None else None,
                                _stream_handle(stream)))
        return ids, d2

    def k_nn(self, points, queries, k: int, schedule: Schedule | None = None,
             with_d2: bool = True, out_ids=None, out_d2=None, stream=None):
        """k_nn! on CUDA tensors: builds this index over `points` and
        searches `queries` in one call (the queries are ordered on a second
        stream while the index builds).  Returns (ids, d2) as knn does."""
        import torch
        _check_points_tensor(points, "points")
        _check_points_tensor(queries, "queries")
        nq = queries.shape[0]
        dev = queries.device
        ids = out_ids if out_ids is not None else torch.empty((nq, k), dtype=torch.int32, device=dev)
        d2 = out_d2 if out_d2 is not None else (
            torch.empty((nq, k), dtype=torch.float32, device=dev) if with_d2 else None)
        s = schedule if schedule is not None else default_schedule()
        check(self._lib.rtd_k_nn(self._h, C.c_void_p(points.data_ptr()), points.shape[0],
                                 C.c_void_p(queries.data_ptr()), nq, k, C.byref(s),
                                 C.c_void_p(ids.data_ptr()),
                                 C.c_void_p(d2.data_ptr()) if d2 is not None else None,
                                 _stream_handle(stream)))
        self.points = points
        return ids, d2

    def range_count(self, queries, radius: float, schedule: Schedule | None = None,
                    out_counts=None, stream=None):
        import torch
        _check_points_tensor(queries, "queries")
        nq = queries.shape[0]
        counts = out_counts if out_counts is not None else torch.empty(
            (nq,), dtype=torch.int32, device=queries.device)
        total = C.c_uint64(0)
        s = schedule if schedule is not None else default_schedule()
        check(self._lib.rtd_range_count(self._h, C.c_void_p(queries.data_ptr()), nq,
                                        C.c_float(radius), C.byref(s),
                                        C.c_void_p(counts.data_ptr()), C.byref(total),
                                        _stream_handle(stream)))
        return counts, total.value

    def range_fill(self, queries, radius: float, capacity: int, sort_pairs: bool = False,
                   schedule: Schedule | None = None, out_pairs=None, stream=None):
        import torch
        _check_points_tensor(queries, "queries")
        pairs = out_pairs if out_pairs is not None else torch.empty(
            (max(capacity, 1), 2), dtype=torch.int32, device=queries.device)
        written = C.c_uint64(0)
        s = schedule if schedule is not None else default_schedule()
        check(self._lib.rtd_range_fill(self._h, C.c_void_p(queries.data_ptr()), queries.shape[0],
                                       C.c_float(radius), C.byref(s),
                                       C.c_void_p(pairs.data_ptr()), capacity, int(sort_pairs),
                                       C.byref(written), _stream_handle(stream)))
        return pairs[: written.value]


class KnnGraph:
    """k_nn! over fixed CUDA tensors, captured once as a CUDA graph
    (rtd_knn_graph_create) and replayed by launch(): each launch rebuilds
    the index from the points' current contents and searches the queries'
    current contents into out_ids / out_d2, without per-kernel launch cost.
    The tensors must keep their storage until close()."""

    def __init__(self, points, queries, k: int, schedule: Schedule | None = None,
                 out_ids=None, out_d2=None, with_d2: bool = True, stream=None):
        import torch
        _check_points_tensor(points, "points")
        _check_points_tensor(queries, "queries")
        self._lib = load()
        nq = queries.shape[0]
        dev = queries.device
        self.ids = out_ids if out_ids is not None else torch.empty((nq, k), dtype=torch.int32, device=dev)
        self.d2 = out_d2 if out_d2 is not None else (
            torch.empty((nq, k), dtype=torch.float32, device=dev) if with_d2 else None)
        self.points, self.queries = points, queries   # keep the storage alive
        s = schedule if schedule is not None else default_schedule()
        h = C.c_void_p()
        check(self._lib.rtd_knn_graph_create(
            C.c_void_p(points.data_ptr()), points.shape[0], C.c_void_p(queries.data_ptr()), nq, k,
            C.byref(s), C.c_void_p(self.ids.data_ptr()),
            C.c_void_p(self.d2.data_ptr()) if self.d2 is not None else None,
            _stream_handle(stream), C.byref(h)))
        self._h = h

    def launch(self, stream=None):
        check(self._lib.rtd_knn_graph_launch(self._h, _stream_handle(stream)))
        return self.ids, self.d2

    def check(self, stream=None):
        """Device error flags of the last launch (synchronises)."""
        check(self._lib.rtd_knn_graph_errors(self._h, _stream_handle(stream)))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rtd_knn_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KnnHostGraph:
    """k_nn! with host buffers (as Context.k_nn), captured once as a CUDA
    graph over fixed page-locked numpy arrays (rtd_knn_graph_create_host):
    each launch() copies the points' and queries' current contents in,
    rebuilds, searches and copies the results out (ids, and d2 with
    with_d2), then synchronises.  The arrays must be page-locked, e.g.
    torch.empty(...).pin_memory().numpy(), and outlive close()."""

    def __init__(self, data: np.ndarray, queries: np.ndarray, k: int,
                 schedule: Schedule | None = None, out_ids: np.ndarray | None = None,
                 out_d2: np.ndarray | None = None, with_d2: bool = False):
        for a, name in ((data, "data"), (queries, "queries")):
            if a.dtype != np.float32 or a.ndim != 2 or a.shape[1] != 3 or not a.flags.c_contiguous:
                raise ValueError(f"{name} must be a contiguous float32 (N, 3) array")
        self._lib = load()
        nq = queries.shape[0]
        self.ids = out_ids if out_ids is not None else np.empty((nq, k), dtype=np.uint32)
        self.d2 = out_d2 if out_d2 is not None else (np.empty((nq, k), dtype=np.float32)
                                                    if with_d2 else None)
        self.data, self.queries = data, queries
        s = schedule if schedule is not None else default_schedule()
        h = C.c_void_p()
        check(self._lib.rtd_knn_graph_create_host(
            _ptr(data), data.shape[0], _ptr(queries), nq, k, C.byref(s), _ptr(self.ids),
            _ptr(self.d2) if self.d2 is not None else None, C.byref(h)))
        self._h = h

    def launch(self):
        check(self._lib.rtd_knn_graph_launch(self._h, None))
        check(self._lib.rtd_knn_graph_errors(self._h, None))   # synchronises
        return (self.ids, self.d2) if self.d2 is not None else self.ids

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rtd_knn_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def radius_for_mean_count(index: "Index", queries, target_mean: float, sample: int = 20000,
                          iters: int = 30, schedule: Schedule | None = None) -> float:
    """Radius whose mean neighbour count over a query sample is target_mean,
    found by bisection on the GPU count pass (log-scale)."""
    import torch
    qs = queries[:: max(1, queries.shape[0] // sample)].contiguous()
    lo, hi = 0.0, 1.0
    # grow hi until it is large enough
    for _ in range(60):
        _, tot = index.range_count(qs, hi, schedule)
        if tot / qs.shape[0] >= target_mean:
            break
        lo, hi = hi, hi * 2.0
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        _, tot = index.range_count(qs, mid, schedule)
        if tot / qs.shape[0] < target_mean:
            lo = mid
        else:
            hi = mid
    return float(hi)


def spatial_join(a, b, radius: float, schedule: Schedule | None = None, exclude_self: bool = False,
                 stream=None):
    """All (i, j) with |b_i - a_j| <= radius (FP32 key <= RN(r*r)), sorted by
    (i, j): the range query with b as queries over an index of a.  With
    exclude_self (a and b the same set) the pairs (i, i) are dropped."""
    _check_points_tensor(a, "a")
    _check_points_tensor(b, "b")
    s = schedule if schedule is not None else default_schedule()
    ix = Index().build(a, s, stream=stream)
    _, total = ix.range_count(b, radius, s, stream=stream)
    pairs = ix.range_fill(b, radius, total, sort_pairs=True, schedule=s, stream=stream)
    if exclude_self:
        pairs = pairs[pairs[:, 0] != pairs[:, 1]]
    return pairs


def dbscan(points, eps: float, min_pts: int, schedule: Schedule | None = None, index=None,
           stream=None):
    """(labels int32 CUDA tensor, n_clusters): DBSCAN over the range query;
    clusters numbered by their smallest core point, noise -1."""
    import torch
    _check_points_tensor(points, "points")
    lib = load()
    if index is None:
        index = Index().build(points, schedule if schedule is not None else default_schedule(),
                              stream=stream)
    labels = torch.empty((points.shape[0],), dtype=torch.int32, device=points.device)
    nc = C.c_uint64(0)
    check(lib.rtd_dbscan(index._h, C.c_void_p(points.data_ptr()), points.shape[0], C.c_float(eps),
                         int(min_pts), C.c_void_p(labels.data_ptr()), C.byref(nc),
                         _stream_handle(stream)))
    return labels, nc.value


def knn_backward(queries, points, ids, grad_d2, grad_q=None, grad_p=None, stream=None):
    """dL/dq (overwritten) and dL/dp (accumulated) for d2 = |q - p_id|^2."""
    import torch
    lib = load()
    nq, k = ids.shape
    if grad_q is None:
        grad_q = torch.empty_like(queries)
    if grad_p is None:
        grad_p = torch.zeros_like(points)
    check(lib.rtd_knn_backward(C.c_void_p(queries.data_ptr()), nq, C.c_void_p(points.data_ptr()),
                               points.shape[0], k, C.c_void_p(ids.data_ptr()),
                               C.c_void_p(grad_d2.contiguous().data_ptr()),
                               C.c_void_p(grad_q.data_ptr()), C.c_void_p(grad_p.data_ptr()),
                               _stream_handle(stream)))
    return grad_q, grad_p
