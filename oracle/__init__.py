"""CPU oracle for rt-dsl's spatial-search path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm import
this package, and only as the checker or as the timed CPU port of the
reference's own CPU search.  The product (rt-dsl_b200/rtdsl) never imports
it.  See oracle.c for what each function restates and how it is pinned.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle.c")
LIB = os.path.join(HERE, "liboracle.so")
CFLAGS = ["-std=gnu11", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
          "-shared", "-Wall"]

EMPTY = 0xFFFFFFFF

_lock = threading.Lock()
_lib = None


class FlatNode(C.Structure):
    """FlatNode, gprt-core/src/lib.rs:299-308."""
    _fields_ = [("com", C.c_float * 3), ("mass", C.c_float), ("width", C.c_float),
                ("is_leaf", C.c_uint32), ("next_idx", C.c_uint32), ("autorope", C.c_uint32),
                ("bucket_start", C.c_uint32), ("num_particles", C.c_uint32)]


FLAT_NODE_DTYPE = np.dtype([("com", np.float32, 3), ("mass", np.float32), ("width", np.float32),
                            ("is_leaf", np.uint32), ("next_idx", np.uint32),
                            ("autorope", np.uint32), ("bucket_start", np.uint32),
                            ("num_particles", np.uint32)])


def build(force: bool = False) -> str:
    """Compile oracle.c with gcc (no FMA contraction, no fast-math)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    tmp = LIB + f".tmp{os.getpid()}"
    r = subprocess.run(["gcc", *CFLAGS, "-o", tmp, SRC, "-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


def lib() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(LIB)
            P = C.c_void_p
            I64 = C.c_int64
            F = C.c_float
            L.orc_num_threads.restype = C.c_int
            L.orc_set_num_threads.argtypes = [C.c_int]
            L.orc_morton3.restype = C.c_uint32
            L.orc_morton3.argtypes = [C.c_uint32] * 3
            L.orc_morton_codes.argtypes = [P, I64, P]
            L.orc_knn.argtypes = [P, I64, P, I64, C.c_int, P, P]
            L.orc_knn_fp64_ambiguity.argtypes = [P, I64, P, I64, C.c_int, P]
            L.orc_knn_fp64_ambiguity.restype = I64
            L.orc_range_count.argtypes = [P, I64, P, I64, F, P]
            L.orc_range_count.restype = I64
            L.orc_range_pairs.argtypes = [P, I64, P, I64, F, P, P]
            L.orc_dbscan.argtypes = [P, I64, F, C.c_uint32, P]
            L.orc_dbscan.restype = I64
            L.orc_radius_sampled_percentile.argtypes = [P, I64, P, I64, C.c_int, F]
            L.orc_radius_sampled_percentile.restype = F
            L.orc_radius_sampled_nn.argtypes = [P, I64, F]
            L.orc_radius_sampled_nn.restype = F
            L.orc_cpu_bvh_knn.argtypes = [P, I64, P, I64, C.c_int, F, F, C.c_int, P, P]
            L.orc_cpu_bvh_knn.restype = C.c_int
            L.orc_bh_build.argtypes = [P, P, I64, C.c_uint32, F, P, P, P]
            L.orc_bh_build.restype = I64
            L.orc_bh_ref_forces.argtypes = [P, P, I64, P, I64, P, F, F, P]
            L.orc_direct_ref_f64.argtypes = [P, P, I64, P, I64, C.c_double, P]
            L.orc_key_public.argtypes = [P, P]
            L.orc_key_public.restype = F
            L.orc_bh_plummer_eval.argtypes = [P, I64, P, P, P, I64, F, C.c_double, C.c_double,
                                              C.c_int, P, P]
            L.orc_bh_plummer_eval.restype = C.c_double
            L.orc_direct_plummer_f64.argtypes = [P, P, I64, C.c_double, C.c_double, P, P, P, P]
            L.orc_direct_plummer_f64.restype = C.c_double
            L.orc_kd_build.argtypes = [P, I64]
            L.orc_kd_build.restype = P
            L.orc_kd_free.argtypes = [P]
            L.orc_kd_size.argtypes = [P]
            L.orc_kd_size.restype = I64
            L.orc_kd_knn.argtypes = [P, P, I64, C.c_int, P, P]
            L.orc_kd_range_count.argtypes = [P, P, I64, F, P]
            L.orc_kd_range_count.restype = I64
            L.orc_kd_range_pairs.argtypes = [P, P, I64, F, P, P]
            L.orc_cpu_bvh_range.argtypes = [P, I64, P, I64, F, P]
            L.orc_cpu_bvh_range.restype = I64
            L.orc_direct_plummer_at_f64.argtypes = [P, P, I64, C.c_double, C.c_double, P, I64, P, P]
            L.orc_bh_ref_forces_at.argtypes = [P, P, I64, P, I64, P, F, F, P, I64, P]
            _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None and a.size else None


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def morton3(x: int, y: int, z: int) -> int:
    return int(lib().orc_morton3(x, y, z))


def morton_codes(xyz) -> np.ndarray:
    xyz = _f32(xyz)
    out = np.empty(len(xyz), dtype=np.uint32)
    lib().orc_morton_codes(_p(xyz), len(xyz), _p(out))
    return out


def key(q, p) -> float:
    q = _f32(q)
    p = _f32(p)
    return float(lib().orc_key_public(_p(q), _p(p)))


def knn(pts, q, k: int):
    """Exact kNN: (ids [Q,k] uint32, d2 [Q,k] float32), (key, id) ascending."""
    pts = _f32(pts)
    q = _f32(q)
    ids = np.empty((len(q), k), dtype=np.uint32)
    d2 = np.empty((len(q), k), dtype=np.float32)
    lib().orc_knn(_p(pts), len(pts), _p(q), len(q), k, _p(ids), _p(d2))
    return ids, d2


def knn_fp64_ambiguity(pts, q, ids) -> int:
    pts = _f32(pts)
    q = _f32(q)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    return int(lib().orc_knn_fp64_ambiguity(_p(pts), len(pts), _p(q), len(q), ids.shape[1], _p(ids)))


def range_count(pts, q, r: float):
    pts = _f32(pts)
    q = _f32(q)
    counts = np.empty(len(q), dtype=np.uint32)
    total = lib().orc_range_count(_p(pts), len(pts), _p(q), len(q), C.c_float(r), _p(counts))
    return counts, int(total)


def dbscan(pts, eps: float, min_pts: int):
    """(labels int32 [N], n_clusters): DBSCAN over the FP32 range membership,
    clusters numbered in the order of their smallest core point, border
    points in the first cluster that reaches them, noise -1."""
    pts = _f32(pts)
    labels = np.empty(len(pts), dtype=np.int32)
    nc = lib().orc_dbscan(_p(pts), len(pts), C.c_float(eps), int(min_pts), _p(labels))
    return labels, int(nc)


def range_pairs(pts, q, r: float) -> np.ndarray:
    """(query, id) pairs sorted by query then id."""
    pts = _f32(pts)
    q = _f32(q)
    counts, total = range_count(pts, q, r)
    off = np.zeros(len(q), dtype=np.uint64)
    if len(q) > 1:
        off[1:] = np.cumsum(counts[:-1].astype(np.uint64))
    pairs = np.empty((max(total, 1), 2), dtype=np.uint32)
    lib().orc_range_pairs(_p(pts), len(pts), _p(q), len(q), C.c_float(r), _p(off), _p(pairs))
    return pairs[:total]


def radius_sampled_percentile(pts, q, k: int, p: float) -> float:
    pts = _f32(pts)
    q = _f32(q)
    return float(lib().orc_radius_sampled_percentile(_p(pts), len(pts), _p(q), len(q), k,
                                                     C.c_float(p)))


def radius_sampled_nn(pts, mult: float) -> float:
    pts = _f32(pts)
    return float(lib().orc_radius_sampled_nn(_p(pts), len(pts), C.c_float(mult)))


def cpu_bvh_knn(pts, q, k: int, radius0: float, mult: float, use_morton: bool = True):
    """The reference's CPU search (gprt-core Scene::build/traverse inside the
    k_nn! round loop).  Returns (ids, d2, rounds)."""
    pts = _f32(pts)
    q = _f32(q)
    ids = np.empty((len(q), k), dtype=np.uint32)
    d2 = np.empty((len(q), k), dtype=np.float32)
    rounds = lib().orc_cpu_bvh_knn(_p(pts), len(pts), _p(q), len(q), k, C.c_float(radius0),
                                   C.c_float(mult), int(use_morton), _p(ids), _p(d2))
    return ids, d2, int(rounds)


def cpu_bvh_range(pts, q, r: float):
    """The reference's CPU range search (Scene::build + one Scene::traverse
    per query at radius r, hits pushed per query).  Returns (counts, total)."""
    pts = _f32(pts)
    q = _f32(q)
    counts = np.empty(len(q), dtype=np.uint32)
    total = lib().orc_cpu_bvh_range(_p(pts), len(pts), _p(q), len(q), C.c_float(r), _p(counts))
    return counts, int(total)


def bh_build(pos, mass, bucket: int = 128, min_width: float = 1e-5):
    """Reference Barnes-Hut tree: (nodes structured array, flat body order,
    root box [min xyz, max xyz, width])."""
    pos = _f32(pos)
    mass = _f32(mass)
    n = len(pos)
    nodes = np.zeros(2 * n + 1, dtype=FLAT_NODE_DTYPE)
    order = np.empty(n, dtype=np.uint32)
    root = np.empty(7, dtype=np.float32)
    nn = lib().orc_bh_build(_p(pos), _p(mass), n, bucket, C.c_float(min_width), _p(nodes),
                            _p(order), _p(root))
    return nodes[:nn].copy(), order, root


def bh_ref_forces(pos, mass, nodes, order, theta: float, G: float = 6.674e-11) -> np.ndarray:
    pos = _f32(pos)
    mass = _f32(mass)
    nodes = np.ascontiguousarray(nodes, dtype=FLAT_NODE_DTYPE)
    order = np.ascontiguousarray(order, dtype=np.uint32)
    out = np.empty((len(pos), 3), dtype=np.float32)
    lib().orc_bh_ref_forces(_p(pos), _p(mass), len(pos), _p(nodes), len(nodes), _p(order),
                            C.c_float(theta), C.c_float(G), _p(out))
    return out


def bh_ref_forces_at(pos, mass, nodes, order, targets, theta: float,
                     G: float = 6.674e-11) -> np.ndarray:
    """bh_ref_forces for the caller bodies listed in targets only."""
    pos = _f32(pos)
    mass = _f32(mass)
    nodes = np.ascontiguousarray(nodes, dtype=FLAT_NODE_DTYPE)
    order = np.ascontiguousarray(order, dtype=np.uint32)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    out = np.empty((len(t), 3), dtype=np.float32)
    lib().orc_bh_ref_forces_at(_p(pos), _p(mass), len(pos), _p(nodes), len(nodes), _p(order),
                               C.c_float(theta), C.c_float(G), _p(t), len(t), _p(out))
    return out


def direct_ref_f64(pos, mass, targets, G: float = 6.674e-11) -> np.ndarray:
    pos = _f32(pos)
    mass = _f32(mass)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    out = np.empty((len(t), 3), dtype=np.float64)
    lib().orc_direct_ref_f64(_p(pos), _p(mass), len(pos), _p(t), len(t), C.c_double(G), _p(out))
    return out


class PlummerFrozen:
    """Plummer-law BH with the decisions of one configuration frozen (the
    reference tree of `bucket`; per-body FP32 MAC decisions as the GPU makes
    them, from this configuration's tree and positions), evaluated in FP64
    for perturbed positions and masses."""

    def __init__(self, pos, mass, theta: float, bucket: int, min_width: float = 1e-5):
        pos = _f32(pos)
        mass = _f32(mass)
        self.nodes, self.order, _ = bh_build(pos, mass, bucket=bucket, min_width=min_width)
        self.n = len(pos)
        self.theta = theta
        self.fpos32 = np.ascontiguousarray(pos[self.order])

    def eval(self, pos, mass, eps: float, G: float, quad: bool = True):
        """(L, phi [N], acc [N,3]) in FP64, caller order."""
        p = np.ascontiguousarray(np.asarray(pos, dtype=np.float64)[self.order])
        m = np.ascontiguousarray(np.asarray(mass, dtype=np.float64)[self.order])
        phi = np.empty(self.n)
        acc = np.empty((self.n, 3))
        L = lib().orc_bh_plummer_eval(_p(self.nodes), len(self.nodes), _p(self.fpos32), _p(p),
                                      _p(m), self.n, C.c_float(self.theta), eps, G, int(quad),
                                      _p(phi), _p(acc))
        out_phi = np.empty(self.n)
        out_acc = np.empty((self.n, 3))
        out_phi[self.order] = phi
        out_acc[self.order] = acc
        return float(L), out_phi, out_acc


def direct_plummer_at_f64(pos, mass, targets, eps: float, G: float):
    """FP64 direct-sum (phi [T], acc [T,3]) at the listed bodies only."""
    pos = _f32(pos)
    mass = _f32(mass)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    phi = np.empty(len(t))
    acc = np.empty((len(t), 3))
    lib().orc_direct_plummer_at_f64(_p(pos), _p(mass), len(pos), eps, G, _p(t), len(t), _p(phi),
                                    _p(acc))
    return phi, acc


def direct_plummer_f64(pos, mass, eps: float, G: float, grad: bool = False):
    """FP64 direct sum: (L, phi, acc[, g_pos, g_mass]) for L = sum phi + 0.5 sum |a|^2."""
    p = np.ascontiguousarray(np.asarray(pos, dtype=np.float64))
    m = np.ascontiguousarray(np.asarray(mass, dtype=np.float64))
    n = len(p)
    phi = np.empty(n)
    acc = np.empty((n, 3))
    gp = np.empty((n, 3)) if grad else None
    gm = np.empty(n) if grad else None
    L = lib().orc_direct_plummer_f64(_p(p), _p(m), n, eps, G, _p(phi), _p(acc), _p(gp), _p(gm))
    return (float(L), phi, acc, gp, gm) if grad else (float(L), phi, acc)


class KdTree:
    """Exact k-NN / range checker for large clouds (orc_kd_*): the same
    results as knn() / range_count() / range_pairs(), in O(log n) per query.
    Subtrees are pruned only when the FP32 key of their box's nearest point
    is strictly above the k-th key (or RN(r*r)), a lower bound of every key
    inside, so no tolerance is involved."""

    def __init__(self, pts):
        self._pts = _f32(pts)
        self._L = lib()
        self._h = self._L.orc_kd_build(_p(self._pts), len(self._pts))

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._L.orc_kd_free(h)

    def __len__(self):
        return int(self._L.orc_kd_size(self._h))

    def knn(self, q, k: int):
        q = _f32(q).reshape(-1, 3)
        ids = np.empty((len(q), k), dtype=np.uint32)
        d2 = np.empty((len(q), k), dtype=np.float32)
        if len(q) and k > 0:
            self._L.orc_kd_knn(self._h, _p(q), len(q), k, _p(ids), _p(d2))
        return ids, d2

    def range_count(self, q, r: float):
        q = _f32(q).reshape(-1, 3)
        counts = np.empty(len(q), dtype=np.uint32)
        total = self._L.orc_kd_range_count(self._h, _p(q), len(q), C.c_float(r), _p(counts))
        return counts, int(total)

    def range_pairs(self, q, r: float) -> np.ndarray:
        """(query, id) pairs sorted by query then id; query = row of q."""
        q = _f32(q).reshape(-1, 3)
        counts, total = self.range_count(q, r)
        off = np.zeros(len(q), dtype=np.uint64)
        if len(q) > 1:
            off[1:] = np.cumsum(counts[:-1].astype(np.uint64))
        pairs = np.empty((max(total, 1), 2), dtype=np.uint32)
        self._L.orc_kd_range_pairs(self._h, _p(q), len(q), C.c_float(r), _p(off), _p(pairs))
        return pairs[:total]


def knn_exact(pts, q, k: int):
    """knn() through a k-d tree: for clouds too large for brute force."""
    return KdTree(pts).knn(q, k)
