"""ORACLE — benchmark and test infrastructure only (the product never imports
it).  The reference's own GPU path for the join -> group-by, as its UVM
executor composes it (the "plain form" the speedup target is quoted
against):

  per side, per morsel (256 MiB of rows, uvm/morsel.py:16-29): the reference's
  compiled partition_sort kernel into B padded buckets (uvm/join.py:66-95);
  B from the reference's rule (operators/partitions.py:54-85 via
  hashjoin.join_partition_count, hashjoin.py:581-633);
  whole buckets packed into core calls of half the chunk budget
  (hashjoin.pack_core_calls, hashjoin.py:567-578);
  per call: the reference's compiled join_unique_hash kernel
  (join_core.py:97-113), then index_select of the carried columns
  (hashjoin._gather_join_result);
  per call's output (a morsel of the aggregation's input): KeyedAggregate.pass1
  (aggregate.py:1511-1563): the grouping hash (the group key's packed word
  times a coefficient), torch.unique with inverse, SUM by a float64 bincount
  rounded to int64 (operator_utils.py:389-398), COUNT by bincount;
  then pass 2, reduce_tick_slice over every partial (sorted_run_merge.py:54-83).

The kernels are the reference's own, compiled from its sources by
oracle/build_ref.sh into oracle/_ref/; everything between them is torch, as
in the reference.  Requires that module (GPU box: it travels with the tree).
"""
from __future__ import annotations

import sys
from math import gcd
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

CHUNK_B = 256 * 1024 ** 2       # the reference's default --chunk_size_mb
BUDGET_B = 512 * 1024 ** 2      # the reference's default --partition_budget_mb
COEFF = 9_999_991               # a grouping-hash coefficient (one packed word)

_mod = None


def available() -> bool:
    return any(REF_DIR.glob("tqpkernels*.so"))


def kernels():
    """The reference's compiled tqpkernels module."""
    global _mod
    if _mod is None:
        if not available():
            raise ImportError("oracle/_ref/tqpkernels*.so is missing: run oracle/build_ref.sh")
        sys.path.insert(0, str(REF_DIR))
        try:
            import tqpkernels as m  # noqa: PLC0415
        finally:
            sys.path.remove(str(REF_DIR))
        _mod = m
    return _mod


def _row_bytes(t):
    return t.element_size() * (t.shape[1] if t.dim() == 2 else 1)


def _padded_starts(counts, rb):
    unit = 512 // gcd(rb, 512)
    starts, at = [], 0
    for c in counts:
        starts.append(at)
        at += -(-c // unit) * unit
    return starts, at


def _partition_side(cols, B, host):
    """Per morsel, the reference kernel's partition of `cols` (key first):
    a list of (per-column bucket lists) per morsel, and the bucket counts."""
    tk = kernels()
    rows = cols[0].shape[0]
    rb = sum(_row_bytes(c) for c in cols) + 8
    step = max(1, min(1 << 30, CHUNK_B // rb))
    morsels, totals = [], [0] * B
    for a in range(0, rows, step):
        b = min(rows, a + step)
        outs = tk.partition_sort([c[a:b].contiguous() for c in cols], [0] * len(cols), 0, None,
                                 b - a, a, B, False, host)
        counts = host[:B].tolist()
        per_col = []
        for t in outs[:-1]:                      # the gidx is not needed here
            starts, _ = _padded_starts(counts, _row_bytes(t))
            per_col.append([t[s:s + c] for s, c in zip(starts, counts)])
        morsels.append(per_col)
        totals = [x + y for x, y in zip(totals, counts)]
    return morsels, totals


def _pack(points, limit):
    ends, i, last = [], 0, len(points) - 1
    while i < last:
        j = i + 1
        while j + 1 <= last and points[j + 1] - points[i] <= limit:
            j += 1
        ends.append(j)
        i = j
    return ends


def join_aggregate(bkey, bgrp, pfk, price, disc, scale, B=None):
    """(groups ascending, int64 sums, int64 counts) of SELECT group,
    SUM(price * (scale - disc)), COUNT(*) ... GROUP BY group, computed the
    reference's way on the GPU."""
    from pageflow_b200.partitions import JOIN_B_MAX, partition_count
    tk = kernels()
    dev = bkey.device
    nb, npr = bkey.numel(), pfk.numel()
    host = torch.empty(JOIN_B_MAX + 5, dtype=torch.int64, pin_memory=True)
    jhost = torch.empty(2, dtype=torch.int64, pin_memory=True)
    sides = [(nb, 8 + 4 + 8, nb), (npr, 8 + 8 + 8 + 8, min(npr, nb))]
    if B is None:
        B, _ = partition_count(sides, BUDGET_B, JOIN_B_MAX)
    lm, lrows = _partition_side([bkey, bgrp], B, host)
    rm, rrows = _partition_side([pfk, price, disc], B, host)
    pair_b = [lrows[b] * 20 + rrows[b] * 32 for b in range(B)]
    points = [0]
    for x in pair_b:
        points.append(points[-1] + x)
    bounds = [0] + _pack(points, CHUNK_B // 2)
    partial = []
    for lo, hi in zip(bounds[:-1], bounds[1:]):
        cols_l = [torch.cat([m[c][b] for b in range(lo, hi) for m in lm]) for c in range(2)]
        cols_r = [torch.cat([m[c][b] for b in range(lo, hi) for m in rm]) for c in range(3)]
        if cols_l[0].numel() == 0 or cols_r[0].numel() == 0:
            continue
        bi, pi = tk.join_unique_hash([cols_l[0]], [cols_r[0]], jhost)
        n = int(jhost[0])
        bi, pi = bi[:n], pi[:n]
        grp = cols_l[1].index_select(0, bi)
        value = cols_r[1].index_select(0, pi) * (scale - cols_r[2].index_select(0, pi))
        # pass 1 over this morsel of the aggregation's input
        h = grp.to(torch.int64) * COEFF
        uh, inv = torch.unique(h, return_inverse=True)
        rep = torch.zeros(uh.numel(), dtype=grp.dtype, device=dev)
        rep.scatter_(0, inv, grp)
        s = torch.round(torch.bincount(inv, weights=value.to(torch.float64),
                                       minlength=uh.numel())).to(torch.int64)
        c = torch.bincount(inv, minlength=uh.numel())
        partial.append((uh, rep, s, c))
    if not partial:
        e = torch.empty(0, dtype=torch.int64, device=dev)
        return e, e.clone(), e.clone()
    # pass 2: reduce_tick_slice over the concatenated partials
    hh = torch.cat([p[0] for p in partial])
    uh, inv = torch.unique(hh, return_inverse=True)
    vals = []
    for k, op in ((1, "amax"), (2, "sum"), (3, "sum")):
        v = torch.cat([p[k] for p in partial]).to(torch.int64)
        r = torch.zeros(uh.numel(), dtype=torch.int64, device=dev)
        r.scatter_reduce_(0, inv, v, reduce=op, include_self=False)
        vals.append(r)
    order = torch.argsort(vals[0])
    return vals[0][order], vals[1][order], vals[2][order]
