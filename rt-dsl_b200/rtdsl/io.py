"""The reference harness's file formats, so its own validators run on this
library's output unchanged.

- point files: ``load_points_fast`` (gprt-sandbox/src/io.rs:8-30), "x,y,z"
  lines; parsed by ``rtd_load_points_csv`` in the native library;
- ``knn_results.txt``: one ``Q{i}:[a, b, ...]`` line per query
  (gprt-sandbox/src/main.rs:89-94, Rust's debug format of a Vec<u32>),
  which gprt-sandbox/validate_full.py reads;
- the result line the benchmark driver parses:
  ``{data_path},{n_queries},{k},{milliseconds:.3},{total_neighbours}``
  (gprt-sandbox/src/main.rs:96).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._capi import EMPTY_ID, check, load


def load_points_csv(path: str) -> np.ndarray:
    """(N, 3) float32 points of a reference point file."""
    lib = load()
    size = os.path.getsize(path)
    cap = size // 5 + 1            # a valid line holds at least "a,b,c"
    out = np.empty((cap, 3), dtype=np.float32)
    n = C.c_uint64(0)
    check(lib.rtd_load_points_csv(os.fsencode(path), C.c_void_p(out.ctypes.data), cap,
                                  C.byref(n)))
    return np.ascontiguousarray(out[: n.value])


def knn_lines(ids) -> list[str]:
    """``Q{i}:[a, b, ...]`` lines; empty slots (fewer than k points) are left
    out, as the reference's per-query vectors hold only found neighbours."""
    ids = np.asarray(ids).view(np.uint32) if np.asarray(ids).dtype == np.int32 else np.asarray(ids)
    out = []
    for i, row in enumerate(ids):
        row = row[row != EMPTY_ID]
        out.append(f"Q{i}:[" + ", ".join(str(int(v)) for v in row) + "]")
    return out


def write_knn_results(path: str, ids) -> None:
    """Writes ``knn_results.txt`` in the reference's format."""
    with open(path, "w") as f:
        for line in knn_lines(ids):
            f.write(line + "\n")


def result_line(data_path: str, n_queries: int, k: int, milliseconds: float,
                total_neighbours: int) -> str:
    return f"{data_path},{n_queries},{k},{milliseconds:.3f},{total_neighbours}"
