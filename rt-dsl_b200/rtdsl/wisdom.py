"""The reference's tuned-schedule files (``gprt_wisdom.json``, written and
read by gprt-sandbox/src/main.rs:53-77 as the serde JSON of
``gprt_ir::Schedule``, gprt-ir/src/lib.rs:58-89) mapped onto rtd_schedule.

serde writes the enums externally tagged: ``"SampledMax"`` or
``{"SampledPercentile": 0.1}`` or ``{"Fixed": 0.5}`` for the radius
heuristic.  The fields with a counterpart here are radius_increment_mult,
radius_heuristic and use_morton_lbv; max_hits_per_query, memory_strategy,
build_strategy and geom_type describe the reference's OptiX hit slab and
BVH builder and have none (a search here has no per-query hit cap and one
BVH builder), so reading ignores them and writing fills in the reference's
defaults.
"""
from __future__ import annotations

import json

from ._capi import (RADIUS_FIXED, RADIUS_SAMPLED_MAX, RADIUS_SAMPLED_PERCENTILE, Schedule,
                    default_schedule)

# gprt_ir::Schedule::default() (gprt-ir/src/lib.rs:76-88)
REFERENCE_DEFAULTS = {
    "radius_increment_mult": 3.0,
    "max_hits_per_query": 2000,
    "use_morton_lbv": False,
    "radius_heuristic": {"SampledPercentile": 0.10},
    "memory_strategy": "PayloadRegisterHeap",
    "build_strategy": "PreferFastTrace",
    "geom_type": "Spheres",
}


def schedule_from_wisdom(wisdom, base: Schedule | None = None) -> Schedule:
    """rtd_schedule from a reference wisdom (JSON text, path-free dict)."""
    d = json.loads(wisdom) if isinstance(wisdom, (str, bytes)) else dict(wisdom)
    s = base if base is not None else default_schedule()
    if "radius_increment_mult" in d:
        s.radius_increment_mult = float(d["radius_increment_mult"])
    if "use_morton_lbv" in d:
        s.use_morton_lbv = int(bool(d["use_morton_lbv"]))
    h = d.get("radius_heuristic")
    if h is not None:
        if h == "SampledMax":
            s.radius_heuristic, s.radius_param = RADIUS_SAMPLED_MAX, 1.0
        elif isinstance(h, dict) and "SampledPercentile" in h:
            s.radius_heuristic, s.radius_param = RADIUS_SAMPLED_PERCENTILE, float(h["SampledPercentile"])
        elif isinstance(h, dict) and "Fixed" in h:
            s.radius_heuristic, s.radius_param = RADIUS_FIXED, float(h["Fixed"])
        else:
            raise ValueError(f"unknown radius_heuristic {h!r}")
    return s


def wisdom_from_schedule(s: Schedule) -> dict:
    """The reference's wisdom JSON object for a schedule (fields without a
    counterpart take the reference's defaults)."""
    d = dict(REFERENCE_DEFAULTS)
    d["radius_increment_mult"] = float(s.radius_increment_mult)
    d["use_morton_lbv"] = bool(s.use_morton_lbv)
    if s.radius_heuristic == RADIUS_SAMPLED_MAX:
        d["radius_heuristic"] = "SampledMax"
    elif s.radius_heuristic == RADIUS_SAMPLED_PERCENTILE:
        d["radius_heuristic"] = {"SampledPercentile": float(s.radius_param)}
    elif s.radius_heuristic == RADIUS_FIXED:
        d["radius_heuristic"] = {"Fixed": float(s.radius_param)}
    else:
        raise ValueError("the sampled-NN and Morton-window seeds have no counterpart in the "
                         "reference's Schedule")
    return d


def load(path: str, base: Schedule | None = None) -> Schedule:
    with open(path) as f:
        return schedule_from_wisdom(f.read(), base)


def save(path: str, s: Schedule) -> None:
    """Writes the schedule as the reference writes gprt_wisdom.json (pretty)."""
    with open(path, "w") as f:
        json.dump(wisdom_from_schedule(s), f, indent=2)
