"""Autotuner for the search and Barnes-Hut launch knobs, with a JSON "wisdom"
cache keyed by workload features.

The reference tunes its Schedule offline and stores one gprt_wisdom.json per
dataset (gprt-sandbox/src/main.rs:53-77; grid + subsample funnel in
gprt-profiler/src/main.rs:40-126; hill-climb in gprt-macros/src/lib.rs:
120-214).  Here the knobs are the LBVH leaf size and key width, the
initial-radius heuristic (sampled 1-NN radius with its multiplier and growth
factor, or the Morton-window seed), the block size and the traversal mode
(thread or warp per query) for the k-NN and range searches, the batched
schedule, and the Barnes-Hut leaf bucket.  Every candidate returns identical
results (exact search), so the tuner only times them; it still checks each
candidate's ids against the first candidate's and refuses one that differs.

Cache key (WorkloadKey): kind (knn / range / batch / bh), the point and query
counts as powers of two, the k class (1, <=8, <=16, <=32, <=64, <=256, >256)
or the mean neighbour count's power of two for range queries, the point
distribution (uniform / clustered / sheet, from describe()), and the GPU
name.  A lookup takes the exact key, else the entry of the same kind, k
class, distribution and GPU whose sizes are nearest (at most a factor 4 in
points and in queries), else the defaults.

Funnel (tune_knn / tune_range), after the profiler's: every candidate on a
5,000-query subsample, the best 20 on 25,000 queries, the best 5 on 100,000
(or all) queries, the fastest of those wins.  The points stay at full size
(the build is part of every step here).
"""
from __future__ import annotations

import ctypes
import itertools
import json
import math
import os
import time
from dataclasses import dataclass

from . import _capi

WISDOM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "wisdom.json")

DEFAULT_GRID = {
    "leaf_size": [2, 4, 5, 8],
    "morton_bits": [39, 42, 48],
    "radius_heuristic": [_capi.RADIUS_SAMPLED_NN, _capi.RADIUS_MORTON_WINDOW],
    "radius_param": [0.0625, 0.25, 0.5, 1.0],
    "radius_increment_mult": [2.0, 4.0],
    "block_size": [128, 256],
    "mode": ["thread", "warp"],
}

# the profiler's funnel: (queries, candidates kept for the next stage)
FUNNEL = ((5_000, 20), (25_000, 5), (100_000, 1))

_MODES = {"thread": dict(lanes_per_query=1), "warp": dict(lanes_per_query=32)}


def gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "unknown"


# ------------------------------------------------------------ workload key
def _log2(x: int) -> int:
    return int(round(math.log2(max(int(x), 1))))


def k_class(k: int) -> str:
    for lim in (1, 8, 16, 32, 64, 256):
        if k <= lim:
            return f"k<={lim}" if lim > 1 else "k=1"
    return "k>256"


def describe(points, sample: int = 2048, seed: int = 0) -> str:
    """Distribution tag of a point cloud (numpy or torch, [n, 3]):
    "sheet" when the smallest box extent is below 2 % of the largest;
    else "clustered" when the median nearest-neighbour distance within a
    stride sample is below half of what uniform points in the same box would
    give; else "uniform"."""
    import numpy as np
    p = points
    n = int(p.shape[0])
    if n == 0:
        return "uniform"
    step = max(1, n // sample)
    p = p[::step][:sample]
    if hasattr(p, "cpu"):
        p = p.detach().cpu().numpy()
    p = np.asarray(p, dtype=np.float64)
    p = p[np.isfinite(p).all(axis=1)]
    m = len(p)
    if m < 8:
        return "uniform"
    ext = p.max(axis=0) - p.min(axis=0)
    if ext.max() <= 0:
        return "clustered"
    if ext.min() < 0.02 * ext.max():
        return "sheet"
    d2 = ((p[:, None, :] - p[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d2, np.inf)
    nn = np.sqrt(d2.min(axis=1))
    # median 1-NN distance of m uniform points in this box (Poisson: 0.554 x spacing)
    uniform = 0.554 * (float(np.prod(ext)) / m) ** (1.0 / 3.0)
    return "clustered" if float(np.median(nn)) < 0.5 * uniform else "uniform"


@dataclass(frozen=True)
class WorkloadKey:
    kind: str            # knn / range / batch / bh
    n_log2: int          # points (bodies), as a power of two
    q_log2: int          # queries (0 for bh)
    size_class: str      # k class, "r~2^j" mean neighbours, or "clouds=2^j"
    dist: str            # uniform / clustered / sheet / plummer / mixed
    gpu: str

    def text(self) -> str:
        return (f"{self.kind}|n=2^{self.n_log2}|q=2^{self.q_log2}|{self.size_class}|{self.dist}|"
                f"{self.gpu}")

    @staticmethod
    def parse(text: str) -> "WorkloadKey | None":
        f = text.split("|")
        if len(f) != 6 or not f[1].startswith("n=2^") or not f[2].startswith("q=2^"):
            return None
        return WorkloadKey(f[0], int(f[1][4:]), int(f[2][4:]), f[3], f[4], f[5])


def knn_key(n: int, nq: int, k: int, dist: str, gpu: str | None = None) -> WorkloadKey:
    return WorkloadKey("knn", _log2(n), _log2(nq), k_class(k), dist, gpu or gpu_name())


def range_key(n: int, nq: int, mean_neighbours: float, dist: str,
              gpu: str | None = None) -> WorkloadKey:
    return WorkloadKey("range", _log2(n), _log2(nq), f"r~2^{_log2(mean_neighbours)}", dist,
                       gpu or gpu_name())


def batch_key(n: int, nq: int, clouds: int, gpu: str | None = None) -> WorkloadKey:
    return WorkloadKey("batch", _log2(n), _log2(nq), f"clouds=2^{_log2(clouds)}", "mixed",
                       gpu or gpu_name())


def bh_key(n: int, dist: str = "plummer", gpu: str | None = None) -> WorkloadKey:
    return WorkloadKey("bh", _log2(n), 0, "theta", dist, gpu or gpu_name())


# ------------------------------------------------------------------ cache
def _load(path: str | None = None) -> dict:
    path = path or WISDOM
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def _store(d: dict, path: str | None = None) -> None:
    path = path or WISDOM
    tmp = path + f".tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
        f.write("\n")
    os.replace(tmp, path)


def lookup(key: WorkloadKey, path: str | None = None) -> dict | None:
    """The cached entry for key: exact, else the nearest size of the same
    kind, class, distribution and GPU within a factor 4 in points and in
    queries, else None."""
    d = _load(path)
    e = d.get(key.text())
    if e is not None:
        return e
    best, best_dist = None, None
    for text, entry in d.items():
        k2 = WorkloadKey.parse(text)
        if k2 is None or (k2.kind, k2.size_class, k2.dist, k2.gpu) != (
                key.kind, key.size_class, key.dist, key.gpu):
            continue
        dn, dq = abs(k2.n_log2 - key.n_log2), abs(k2.q_log2 - key.q_log2)
        if dn > 2 or dq > 2:
            continue
        if best_dist is None or dn + dq < best_dist:
            best, best_dist = entry, dn + dq
    return best


def schedule_for(key: WorkloadKey, default: _capi.Schedule | None = None,
                 path: str | None = None) -> _capi.Schedule:
    """The cached schedule for the workload (a copy), else a copy of
    `default` (the single-cloud defaults when None)."""
    s = _capi.Schedule()
    base = default if default is not None else _capi.default_schedule()
    ctypes.memmove(ctypes.addressof(s), ctypes.addressof(base), ctypes.sizeof(s))
    entry = lookup(key, path)
    if entry and "schedule" in entry:
        for k, v in entry["schedule"].items():
            if hasattr(s, k):
                setattr(s, k, v)
    return s


def save(key: WorkloadKey, schedule: _capi.Schedule | None, meta: dict,
         path: str | None = None) -> None:
    d = _load(path)
    entry = dict(meta)
    if schedule is not None:
        entry["schedule"] = schedule.as_dict()
    entry["tuned_at"] = time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())
    d[key.text()] = entry
    _store(d, path)


# ------------------------------------------------------------------ tuners
def _candidates(grid: dict, k: int) -> list[dict]:
    keys = list(grid)
    cands, seen = [], set()
    for combo in itertools.product(*(grid[k_] for k_ in keys)):
        kw = dict(zip(keys, combo))
        mode = kw.pop("mode", "thread")
        if mode != "warp" and k > 16:
            continue
        if kw.get("radius_heuristic") == _capi.RADIUS_MORTON_WINDOW:
            if mode != "thread":
                continue   # the window seed runs in the thread-per-query kernel only
            # one unbounded round: the radius knobs do not apply
            kw["radius_param"] = grid.get("radius_param", [0.5])[0]
            kw["radius_increment_mult"] = grid.get("radius_increment_mult", [2.0])[0]
        kw.update(_MODES[mode])
        key = tuple(sorted(kw.items()))
        if key in seen:
            continue
        seen.add(key)
        cands.append(kw)
    return cands


def _funnel(cands: list[dict], nq: int, time_fn, funnel=FUNNEL, log=None):
    """Runs the funnel: time_fn(kw, n_queries) -> (ms, ids); returns the
    final stage's [(ms, kw)] sorted, fastest first."""
    import torch
    stage = [(None, kw) for kw in cands]
    ref = {}
    for target, keep in funnel:
        m = min(target, nq)
        timed = []
        for _, kw in stage:
            ms, ids = time_fn(kw, m)
            if m not in ref:
                ref[m] = ids.clone()
            elif not bool(torch.equal(ids, ref[m])):
                raise RuntimeError(f"autotune: candidate {kw} returned different neighbours")
            timed.append((ms, kw))
            if log:
                log(f"stage {m} queries: {ms:.4f} ms {kw}")
        timed.sort(key=lambda x: x[0])
        stage = timed[:keep] if keep else timed
        if m == nq:
            break
    return stage


def _time_knn(P, Q, k, s, reps: int):
    import torch
    from .api import Index
    ix = Index().profile(True)
    ids = torch.empty((Q.shape[0], k), dtype=torch.int32, device=Q.device)
    d2 = torch.empty((Q.shape[0], k), dtype=torch.float32, device=Q.device)
    ix.build(P, s)
    ix.knn(Q, k, s, out_ids=ids, out_d2=d2)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        ix.build(P, s)
        ix.knn(Q, k, s, out_ids=ids, out_d2=d2)
        t = ix.timings()
        best = min(best, sum(t.values()))
    return best, ids


def tune_knn(P, Q, k: int, grid: dict | None = None, reps: int = 3, funnel=FUNNEL,
             save_result: bool = True, path: str | None = None, dist: str | None = None,
             log=None):
    """Times build + search (index phase events) for every grid point
    through the funnel; caches the winner under the workload's key.
    Returns (schedule, final stage table, key)."""
    grid = grid or DEFAULT_GRID
    nq = int(Q.shape[0])
    # fixed query subsets: the first m queries of a seeded permutation
    import torch
    perm = torch.randperm(nq, generator=torch.Generator().manual_seed(0)).to(Q.device)

    def time_fn(kw, m):
        return _time_knn(P, Q[perm[:m]].contiguous(), k, _capi.default_schedule(**kw), reps)

    table = _funnel(_candidates(grid, k), nq, time_fn, funnel, log)
    best_ms, best_kw = table[0]
    best = _capi.default_schedule(**best_kw)
    key = knn_key(P.shape[0], nq, k, dist or describe(P))
    if save_result:
        save(key, best, {"n": int(P.shape[0]), "nq": nq, "k": k,
                         "build_plus_search_ms": best_ms}, path)
    return best, table, key


RANGE_GRID = {
    "leaf_size": [8, 12, 16],
    "morton_bits": [42, 48],
    "block_size": [128, 256],
}


def tune_range(P, Q, radius: float, mean_neighbours: float, grid: dict | None = None,
               reps: int = 3, funnel=FUNNEL, save_result: bool = True, path: str | None = None,
               dist: str | None = None, log=None):
    """Times build + count + fill for every grid point through the funnel
    (pairs compared as sorted (query, id) lists); caches the winner."""
    import torch
    from .api import Index
    grid = grid or RANGE_GRID
    nq = int(Q.shape[0])
    perm = torch.randperm(nq, generator=torch.Generator().manual_seed(0)).to(Q.device)

    def time_fn(kw, m):
        s = _capi.default_schedule(**kw)
        q = Q[perm[:m]].contiguous()
        ix = Index()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = float("inf")
        pairs = None
        for r in range(reps + 1):
            e0.record()
            ix.build(P, s)
            _, total = ix.range_count(q, radius, s)
            pairs = ix.range_fill(q, radius, total, sort_pairs=True, schedule=s)
            e1.record()
            e1.synchronize()
            if r:
                best = min(best, e0.elapsed_time(e1))
        return best, pairs

    cands = [dict(zip(grid, c)) for c in itertools.product(*grid.values())]
    table = _funnel(cands, nq, time_fn, funnel, log)
    best_ms, best_kw = table[0]
    best = _capi.default_schedule(**best_kw)
    key = range_key(P.shape[0], nq, mean_neighbours, dist or describe(P))
    if save_result:
        save(key, best, {"n": int(P.shape[0]), "nq": nq, "mean_neighbours": mean_neighbours,
                         "radius": radius, "count_plus_fill_ms": best_ms}, path)
    return best, table, key


BATCH_GRID = {
    "leaf_size": [8, 16, 32, 64],
    "radius_param": [0.5, 1.0, 2.0],
    "radius_increment_mult": [2.0, 4.0],
    "lanes_per_query": [0, 32],
    "morton_bits": [42, 48, 63],
}


def tune_batch(P, Q, sizes, grid: dict | None = None, reps: int = 3, save_result: bool = True,
               path: str | None = None, log=None):
    """Times the batched pass (forest build + persistent search) for every
    grid point; every candidate must return the first candidate's ids."""
    import torch
    from .batch import Batch
    grid = grid or BATCH_GRID
    keys = list(grid)
    table = []
    ref_ids = None
    for combo in itertools.product(*(grid[k_] for k_ in keys)):
        kw = dict(zip(keys, combo))
        s = _capi.default_batch_schedule(**kw)
        b = Batch(sizes, s)
        ids = torch.empty(max(b.n_out, 1), dtype=torch.int32, device=Q.device)
        b.knn(P, Q, out_ids=ids, with_d2=False)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        best = float("inf")
        for _ in range(reps):
            e0.record()
            b.knn(P, Q, out_ids=ids, with_d2=False)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        if ref_ids is None:
            ref_ids = ids.clone()
        elif not bool((ids == ref_ids).all()):
            raise RuntimeError(f"autotune: batch candidate {kw} returned different neighbours")
        table.append((best, kw))
        b.close()
        if log:
            log(f"batch {best:.4f} ms {kw}")
    table.sort(key=lambda x: x[0])
    best_ms, best_kw = table[0]
    best = _capi.default_batch_schedule(**best_kw)
    key = batch_key(P.shape[0], Q.shape[0], len(sizes))
    if save_result:
        save(key, best, {"n": int(P.shape[0]), "nq": int(Q.shape[0]), "clouds": len(sizes),
                         "batch_ms": best_ms}, path)
    return best, table, key


def tune_bh_bucket(pos, mass, buckets=(16, 32, 64), theta: float = 0.5, eps: float = 1e-3,
                   reps: int = 3, save_result: bool = True, path: str | None = None, log=None):
    """Leaf bucket of the Plummer-law tree minimising build + forward +
    adjoint time."""
    import torch
    from .bh import BarnesHut
    from ._capi import BH_LAW_PLUMMER, default_bh_params
    n = pos.shape[0]
    ones = torch.ones((n,), device=pos.device)
    table = []
    for bucket in buckets:
        p = default_bh_params(law=BH_LAW_PLUMMER, theta=theta, eps=eps, G=1.0, quadrupole=1,
                              bucket=bucket)
        bh = BarnesHut()
        best = float("inf")
        for r in range(reps + 1):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            bh.build(pos, mass, p)
            acc, _ = bh.forward(p)
            bh.backward(acc, ones, p)
            e1.record()
            e1.synchronize()
            if r:
                best = min(best, e0.elapsed_time(e1))
        bh.close()
        table.append((best, bucket))
        if log:
            log(f"bh bucket {bucket}: {best:.3f} ms")
    table.sort()
    key = bh_key(n)
    if save_result:
        save(key, None, {"bucket": table[0][1], "step_ms": table[0][0], "n": int(n),
                         "theta": theta}, path)
    return table[0][1], table, key


def bh_bucket_for(n: int, default: int = 32, path: str | None = None) -> int:
    e = lookup(bh_key(n), path)
    return int(e["bucket"]) if e and "bucket" in e else default


def main():
    """Tunes the bench workloads and writes wisdom.json:
    python -m rtdsl.autotune"""
    import numpy as np
    import torch
    from . import workloads
    from .api import Index, radius_for_mean_count
    log = lambda m: print(m, flush=True)   # noqa: E731
    pts, q = workloads.clustered()
    P = torch.from_numpy(pts).cuda()
    Q = torch.from_numpy(q).cuda()
    grid = {"leaf_size": [2, 3, 4, 5, 6, 8], "radius_param": [0.25, 0.5, 1.0],
            "radius_increment_mult": [2.0, 4.0], "block_size": [128, 256],
            "morton_bits": [39, 42, 48],
            "radius_heuristic": [_capi.RADIUS_SAMPLED_NN, _capi.RADIUS_MORTON_WINDOW],
            "mode": ["thread", "warp"]}
    best, table, key = tune_knn(P, Q, 5, grid=grid, log=log)
    log(f"{key.text()} best {table[0]}")
    s = _capi.default_schedule(leaf_size=12, morton_bits=42)
    r = radius_for_mean_count(Index().build(P, s), Q, 50.0, schedule=s)
    best, table, key = tune_range(P, Q, r, 50.0, log=log)
    log(f"{key.text()} best {table[0]}")
    cl = workloads.clouds()
    P = torch.from_numpy(np.concatenate([c["points"] for c in cl])).cuda()
    Q = torch.from_numpy(np.concatenate([c["queries"] for c in cl])).cuda()
    sizes = [(len(c["points"]), len(c["queries"]), c["k"]) for c in cl]
    best, table, key = tune_batch(P, Q, sizes, log=log)
    log(f"{key.text()} best {table[0]}")
    pos, mass = workloads.plummer(1_000_000, seed=7)
    bucket, table, key = tune_bh_bucket(torch.from_numpy(pos).cuda(),
                                        torch.from_numpy(mass).cuda(), log=log)
    log(f"{key.text()} best bucket {bucket}")


if __name__ == "__main__":
    main()
