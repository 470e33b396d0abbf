"""Barnes-Hut over the C ABI: device-tensor handle and the host-buffer
barnes_hut!(bodies, theta, G, out) mirror (gprt-macros/src/lib.rs:752-834)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import BH_LAW_PLUMMER, BH_LAW_REFERENCE, check, default_bh_params, load

FLAT_NODE_DTYPE = np.dtype([("com", np.float32, 3), ("mass", np.float32), ("width", np.float32),
                            ("is_leaf", np.uint32), ("next_idx", np.uint32),
                            ("autorope", np.uint32), ("bucket_start", np.uint32),
                            ("num_particles", np.uint32)])

BODY_DTYPE = np.dtype([("pos", np.float32, 3), ("mass", np.float32), ("velocity", np.float32, 3)])


def _stream(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class BarnesHut:
    """rtd_bh: octree over CUDA tensors pos (N x 3) and mass (N) float32."""

    def __init__(self):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.rtd_bh_create(C.byref(h)))
        self._h = h
        self.n = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rtd_bh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self, pos, mass, params: _capi.BhParams | None = None, stream=None) -> "BarnesHut":
        p = params if params is not None else default_bh_params()
        if pos.dtype.is_floating_point is False or pos.shape[-1] != 3:
            raise ValueError("pos must be (N, 3) float32")
        pos = pos.contiguous()
        mass = mass.contiguous()
        check(self._lib.rtd_bh_build(self._h, _ptr(pos), _ptr(mass), pos.shape[0], C.byref(p),
                                     _stream(stream)))
        self.n = pos.shape[0]
        self._keep = (pos, mass)
        return self

    def release(self):
        check(self._lib.rtd_bh_release(self._h))

    def forward(self, params: _capi.BhParams | None = None, out=None, phi=None, want_phi=True,
                stream=None):
        import torch
        p = params if params is not None else default_bh_params()
        dev = self._keep[0].device if self.n else torch.device("cuda")
        out = out if out is not None else torch.empty((self.n, 3), dtype=torch.float32, device=dev)
        if phi is None and want_phi and p.law == BH_LAW_PLUMMER:
            phi = torch.empty((self.n,), dtype=torch.float32, device=dev)
        check(self._lib.rtd_bh_forward(self._h, C.byref(p), _ptr(out), _ptr(phi), _stream(stream)))
        return out, phi

    def backward(self, g_acc, g_phi=None, params: _capi.BhParams | None = None, stream=None,
                 out_pos=None, out_mass=None):
        import torch
        p = params if params is not None else default_bh_params(law=BH_LAW_PLUMMER)
        g_acc = g_acc.contiguous()
        g_phi = g_phi.contiguous() if g_phi is not None else None
        g_pos = out_pos if out_pos is not None else torch.empty(
            (self.n, 3), dtype=torch.float32, device=g_acc.device)
        g_mass = out_mass if out_mass is not None else torch.empty(
            (self.n,), dtype=torch.float32, device=g_acc.device)
        check(self._lib.rtd_bh_backward(self._h, C.byref(p), _ptr(g_acc), _ptr(g_phi),
                                        _ptr(g_pos), _ptr(g_mass), _stream(stream)))
        return g_pos, g_mass

    def info(self, stream=None) -> dict:
        inf = _capi.BhInfo()
        check(self._lib.rtd_bh_info_get(self._h, C.byref(inf), _stream(stream)))
        return {"n_bodies": inf.n_bodies, "n_nodes": inf.n_nodes, "n_leaves": inf.n_leaves,
                "depth": inf.depth, "root_min": list(inf.root_min), "root_max": list(inf.root_max),
                "max_stack": inf.max_stack, "log_pages": inf.log_pages}

    def leapfrog(self, pos, vel, mass, dt: float, steps: int,
                 params: _capi.BhParams | None = None, acc=None, stream=None):
        """Advances pos / vel (CUDA tensors, in place) by `steps` leapfrog
        steps of the Plummer law; returns the acceleration at the final
        positions (pass it back as `acc` to continue without recomputing)."""
        import torch
        p = params if params is not None else default_bh_params(law=BH_LAW_PLUMMER)
        for t, name in ((pos, "pos"), (vel, "vel"), (mass, "mass")):
            if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
                raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
        valid = acc is not None
        if acc is None:
            acc = torch.empty_like(pos)
        check(self._lib.rtd_bh_leapfrog(self._h, C.byref(p), _ptr(pos), _ptr(vel), _ptr(mass),
                                        pos.shape[0], C.c_float(dt), int(steps), _ptr(acc),
                                        int(valid), _stream(stream)))
        self.n = pos.shape[0]
        self._keep = (pos, mass)
        return acc

    def interaction_counts(self, theta: float, stride: int = 64, stream=None) -> dict:
        """Mean accepted cells and leaf bodies per body of the Plummer walk
        (every stride-th body in tree order)."""
        cells, bodies, ns = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(self._lib.rtd_bh_interaction_counts(self._h, C.c_float(theta), int(stride),
                                                  C.byref(cells), C.byref(bodies), C.byref(ns),
                                                  _stream(stream)))
        n = max(ns.value, 1)
        return {"cells_per_body": cells.value / n, "bodies_per_body": bodies.value / n,
                "sampled": ns.value}

    def export(self, stream=None):
        """(FlatNode structured array, flat body order)."""
        info = self.info(stream)
        nodes = np.zeros(int(info["n_nodes"]), dtype=FLAT_NODE_DTYPE)
        order = np.zeros(self.n, dtype=np.uint32)
        check(self._lib.rtd_bh_export(self._h, C.c_void_p(nodes.ctypes.data) if nodes.size else None,
                                      C.c_void_p(order.ctypes.data) if order.size else None,
                                      _stream(stream)))
        return nodes, order


def barnes_hut(bodies, theta: float, G: float = 6.674e-11, context=None) -> np.ndarray:
    """barnes_hut!(bodies, theta, G, out): bodies as a BODY_DTYPE structured
    array (or an (N, 4) x,y,z,mass array); returns (N, 3) forces with the
    reference law."""
    from .api import _context
    b = np.asarray(bodies)
    if b.dtype != BODY_DTYPE:
        arr = np.ascontiguousarray(b, dtype=np.float32)
        if arr.ndim != 2 or arr.shape[1] < 4:
            raise ValueError("bodies must be Body records or an (N, 4) x,y,z,mass array")
        b = np.zeros(len(arr), dtype=BODY_DTYPE)
        b["pos"] = arr[:, :3]
        b["mass"] = arr[:, 3]
    b = np.ascontiguousarray(b)
    out = np.empty((len(b), 3), dtype=np.float32)
    ctx = context if context is not None else _context()
    check(load().rtd_barnes_hut_host(ctx._h, C.c_void_p(b.ctypes.data) if len(b) else None, len(b),
                                     C.c_float(theta), C.c_float(G),
                                     C.c_void_p(out.ctypes.data) if len(b) else None))
    return out
