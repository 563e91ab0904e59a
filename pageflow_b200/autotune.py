"""The autotuner of the fused join + group-by: the first call of a shape
class times a few candidate launch configurations on the call's own inputs
with CUDA events (outside any caller's timed region), keeps the fastest, and
caches it per shape class in a JSON file, so later calls and later processes
start from it.

Knobs (pf_join_knobs plus the fan-out):

  B         first radix pass fan-out, a power of two; seeded by the build
            rows a partition should hold (pf_join_aggregate_pick_b) and tried
            at half and double that (the workload's 2^8-2^12 range at the
            150M-row build)
  table     the shared-memory join's table: 8-byte hash slots or 4-byte
            fingerprinted slots
  sub_rows  build rows a sub-partition aims at (1365 or 682)
  counted   1: both radix passes count their rows first, instead of
            scattering into regions sized from the expected counts (which a
            skewed input overflows, paying for a pass it then runs again)

The search is coordinate-wise in that order (B with the default table and
sub_rows, then the table at the best B, then sub_rows, then counted), each
candidate run
once to warm up and then timed over ``reps`` runs; ties keep the earlier
candidate, so the same timings always give the same choice.  A shape class
is the rounded-up log2 of the build rows, probe rows and groups, with the
device's name.  The cache file is $PAGEFLOW_TUNE_CACHE, else
~/.cache/pageflow_b200/autotune.json.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import Callable, Dict, List, Optional

DEFAULT_SUB_ROWS = 1365
SUB_ROWS = (1365, 682)
TABLES = (0, 1)
COUNTED = (0, 1)
B_MAX = 4096


@dataclass(frozen=True)
class Choice:
    B: int
    table: int = 0
    sub_rows: int = DEFAULT_SUB_ROWS
    counted: int = 0

    def label(self) -> str:
        s = f"B={self.B},table={self.table},sub_rows={self.sub_rows}"
        return s + ",counted=1" if self.counted else s


@dataclass
class Result:
    choice: Choice
    times_ms: Dict[str, float] = field(default_factory=dict)
    cached: bool = False


def cache_path() -> Path:
    p = os.environ.get("PAGEFLOW_TUNE_CACHE")
    if p:
        return Path(p)
    return Path.home() / ".cache" / "pageflow_b200" / "autotune.json"


def shape_class(device_name: str, n_build: int, n_probe: int, n_groups: int) -> str:
    def lg(x: int) -> int:
        return max(0, math.ceil(math.log2(max(1, int(x)))))
    return f"{device_name}|join_aggregate|b{lg(n_build)}|p{lg(n_probe)}|g{lg(n_groups)}"


def b_candidates(seed_b: int) -> List[int]:
    """The seed first, then half and double of it, within [1, B_MAX]."""
    out = [seed_b]
    for b in (seed_b // 2, seed_b * 2):
        if 1 <= b <= B_MAX and b not in out:
            out.append(b)
    return out


def search(seed_b: int, time_of: Callable[[Choice], float]) -> Result:
    """Coordinate-wise search from the seed: every timing goes through
    time_of (milliseconds); the first of equal times wins."""
    times: Dict[str, float] = {}

    def best_of(cands: List[Choice]) -> Choice:
        best, best_t = None, math.inf
        for c in cands:
            t = times.get(c.label())
            if t is None:
                t = float(time_of(c))
                times[c.label()] = t
            if t < best_t:
                best, best_t = c, t
        return best

    cur = best_of([Choice(b) for b in b_candidates(seed_b)])
    cur = best_of([Choice(cur.B, t, cur.sub_rows) for t in TABLES])
    cur = best_of([Choice(cur.B, cur.table, s) for s in SUB_ROWS])
    cur = best_of([Choice(cur.B, cur.table, cur.sub_rows, k) for k in COUNTED])
    return Result(cur, times)


def load_cache(path: Optional[Path] = None) -> dict:
    path = path or cache_path()
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def store(key: str, result: Result, path: Optional[Path] = None) -> None:
    """Adds one shape class's choice to the cache file (written whole, via a
    temporary file renamed over it)."""
    path = path or cache_path()
    data = load_cache(path)
    data[key] = {"choice": asdict(result.choice), "times_ms": result.times_ms}
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(path.suffix + f".{os.getpid()}.tmp")
    tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
    os.replace(tmp, path)


def lookup(key: str, path: Optional[Path] = None) -> Optional[Result]:
    entry = load_cache(path).get(key)
    if not entry:
        return None
    c = entry["choice"]
    return Result(Choice(int(c["B"]), int(c["table"]), int(c["sub_rows"]),
                         int(c.get("counted", 0))),
                  dict(entry.get("times_ms", {})), cached=True)


def tune(key: str, seed_b: int, time_of: Callable[[Choice], float],
         path: Optional[Path] = None) -> Result:
    """The cached choice of this shape class, else a search stored for the
    next call."""
    hit = lookup(key, path)
    if hit is not None:
        return hit
    res = search(seed_b, time_of)
    store(key, res, path)
    return res
