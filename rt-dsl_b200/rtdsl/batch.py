"""Batched exact k-NN over many independent point clouds (rtd_batch_*).

The reference searches one scene per ``k_nn!`` call (gprt-macros/src/lib.rs:
316-476); a workload of many small clouds there pays one BVH build and one
launch per cloud.  ``Batch`` plans the packed layout once, then each call
builds every cloud's LBVH as one forest and searches all queries in one
persistent launch per k class, optionally replayed as a CUDA graph.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import Cloud, Schedule, check, default_batch_schedule, load
from .api import _check_points_tensor, _stream_handle


class Batch:
    """A plan for clouds packed in order in one point and one query tensor.

    ``sizes`` is a sequence of (n_points, n_queries, k) per cloud; the k
    results of cloud c's query j start at ``out_offset[c] + j * k_c`` of the
    flat outputs (``split`` gives per-cloud (n_q, k) views).  Ids are
    cloud-local point indices.
    """

    def __init__(self, sizes, schedule: Schedule | None = None):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.rtd_batch_create(C.byref(h)))
        self._h = h
        sizes = [tuple(int(v) for v in s) for s in sizes]
        n = len(sizes)
        arr = (Cloud * max(n, 1))()
        po = qo = oo = 0
        self.point_offset = np.zeros(n, np.int64)
        self.query_offset = np.zeros(n, np.int64)
        self.out_offset = np.zeros(n, np.int64)
        for c, (npnt, nq, k) in enumerate(sizes):
            arr[c].point_offset, arr[c].query_offset, arr[c].out_offset = po, qo, oo
            arr[c].n_points, arr[c].n_queries, arr[c].k = npnt, nq, k
            self.point_offset[c], self.query_offset[c], self.out_offset[c] = po, qo, oo
            po += npnt
            qo += nq
            oo += nq * k
        self.sizes = sizes
        self.n_points, self.n_queries, self.n_out = po, qo, oo
        self.schedule = schedule if schedule is not None else default_batch_schedule()
        check(self._lib.rtd_batch_plan(self._h, arr, n, C.byref(self.schedule)))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rtd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def knn(self, points, queries, out_ids=None, out_d2=None, with_d2: bool = True,
            use_graph: bool = False, stream=None):
        """Flat (n_out,) int32 ids and float32 squared distances."""
        import torch
        _check_points_tensor(points, "points")
        _check_points_tensor(queries, "queries")
        if points.shape[0] != self.n_points or queries.shape[0] != self.n_queries:
            raise ValueError("points / queries do not match the plan")
        dev = queries.device
        ids = out_ids if out_ids is not None else torch.empty(
            (max(self.n_out, 1),), dtype=torch.int32, device=dev)
        d2 = out_d2 if out_d2 is not None else (
            torch.empty((max(self.n_out, 1),), dtype=torch.float32, device=dev) if with_d2 else None)
        check(self._lib.rtd_knn_batched(self._h, C.c_void_p(points.data_ptr()),
                                        C.c_void_p(queries.data_ptr()), C.c_void_p(ids.data_ptr()),
                                        C.c_void_p(d2.data_ptr()) if d2 is not None else None,
                                        int(use_graph), _stream_handle(stream)))
        return ids[: self.n_out], (d2[: self.n_out] if d2 is not None else None)

    def backward(self, points, queries, ids, grad_d2, grad_q=None, grad_p=None, stream=None):
        """dL/dq (overwritten) and dL/dp (accumulated) for the batched d2."""
        import torch
        if grad_q is None:
            grad_q = torch.empty_like(queries)
        if grad_p is None:
            grad_p = torch.zeros_like(points)
        check(self._lib.rtd_knn_batched_backward(
            self._h, C.c_void_p(points.data_ptr()), C.c_void_p(queries.data_ptr()),
            C.c_void_p(ids.data_ptr()), C.c_void_p(grad_d2.contiguous().data_ptr()),
            C.c_void_p(grad_q.data_ptr()), C.c_void_p(grad_p.data_ptr()), _stream_handle(stream)))
        return grad_q, grad_p

    def split(self, flat):
        """Per-cloud (n_q, k) views of a flat output."""
        out = []
        for c, (_, nq, k) in enumerate(self.sizes):
            o = int(self.out_offset[c])
            out.append(flat[o:o + nq * k].reshape(nq, k))
        return out
