"""ORACLE — benchmark and test infrastructure only (the product never imports
it).  The reference's own GPU path for the join -> group-by, as its UVM
executor composes it (the "plain form" the speedup target is quoted
against).  The reference's Python does not travel to the GPU box, so its
steps are restated here in the same torch calls; its compiled kernels are
its own.

The join (uvm/join.py:98-225):
  per side, per morsel (the 256 MiB chunk budget over the side's bytes a
  row, uvm/morsel.py:16-29): the reference's compiled partition_sort kernel
  into B padded buckets (uvm/join.py:66-95), B from the reference's rule
  (operators/partitions.py:54-85 via hashjoin.join_partition_count,
  hashjoin.py:581-633; restated in pageflow_b200/partitions.py and pinned to
  the reference's values by tests/golden/partitions.json);
  whole buckets packed into core calls of half the chunk budget
  (hashjoin.pack_core_calls, hashjoin.py:567-578, tick_cutter.pack);
  per call: the reference's compiled join_unique_hash kernel
  (join_core.py:97-113), then index_select of the columns the aggregation
  reads (hashjoin._gather_join_result, hashjoin.py:359-377); the calls'
  outputs concatenated column by column.
The aggregation (uvm/aggregate.py:147-212), over the join's output:
  B from the partition budget (operators/aggregate.py:1644-1668 ->
  operators/partitions.agg_partitions; the hash route's run of 8 + 4 + 8 + 8
  bytes a row);
  pass 1 per morsel (KeyedAggregate.pass1, aggregate.py:1511-1563): the
  grouping hash of the int32 key's packed word times the coefficient
  _make_key_coeffs draws (aggregate.py:526-548: a generator on the device
  seeded with 2029, randint(2, 10_000_000)), torch.unique with inverse, the
  key's representative by scatter, SUM(price * (scale - disc)) by a float64
  bincount rounded to int64 (operator_utils.py:389-398), COUNT by bincount,
  each group's bucket (_bucket_ids, aggregate.py:95-116) and the partials
  sorted stably by it (uvm/aggregate.py:70-93);
  pass 2 per round of whole buckets packed to the partition budget
  (pass2_rounds, aggregate.py:169-184): reduce_tick_slice over the round's
  rows of every morsel (torch.unique, scatter_reduce amax / sum / sum;
  sorted_run_merge.py:54-83); the rounds' groups concatenated.

The kernels are the reference's own, compiled from its sources by
oracle/build_ref.sh into oracle/_ref/.  Requires that module (GPU box: it
travels with the tree).
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
COEFF_SEED = 2029               # the reference's _COEFF_BASE_SEED
MIX_M1 = 0xff51afd7ed558ccd - (1 << 64)
MIX_M2 = 0xc4ceb9fe1a85ec53 - (1 << 64)
LOW31 = (1 << 31) - 1

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


def _mix64(h):
    k = h ^ ((h >> 33) & LOW31)
    k = k * MIX_M1
    k = k ^ ((k >> 33) & LOW31)
    k = k * MIX_M2
    return k ^ ((k >> 33) & LOW31)


def _bucket_ids(h, B):
    if B == 1:
        return torch.zeros(h.shape[0], dtype=torch.int32, device=h.device)
    return ((_mix64(h) >> (64 - (B.bit_length() - 1))) & (B - 1)).to(torch.int32)


def _coeff(dev):
    g = torch.Generator(device=dev)
    g.manual_seed(COEFF_SEED)
    return torch.randint(2, 10_000_000, (1,), dtype=torch.int64, device=dev, generator=g)


def _pass1(grp, price, disc, scale, coeff, B):
    """One morsel's partials [hash, key, sum, count], in bucket order, and
    the rows of each bucket."""
    # the int32 key's packed word: its four bytes, zero-extended
    word = grp.to(torch.int64) & 0xFFFFFFFF
    h = word * coeff
    uh, inv = torch.unique(h, return_inverse=True)
    rep = torch.zeros(uh.numel(), dtype=grp.dtype, device=grp.device)
    rep.scatter_(0, inv, grp)
    value = price * (scale - disc)
    s = torch.round(torch.bincount(inv, weights=value.to(torch.float64),
                                   minlength=uh.numel())).to(torch.int64)
    c = torch.bincount(inv, minlength=uh.numel())
    outs = [uh, rep, s, c]
    if B == 1:
        return outs, [uh.numel()]
    bucket = _bucket_ids(uh, B)
    counts = torch.bincount(bucket, minlength=B).tolist()
    order = torch.sort(bucket, stable=True).indices
    return [t.index_select(0, order) for t in outs], counts


def _rounds(bucket_rows, row_b):
    points = [0]
    for x in bucket_rows:
        points.append(points[-1] + x)
    if points[-1] * row_b <= BUDGET_B:
        return [len(bucket_rows)]
    return _pack([p * row_b for p in points], BUDGET_B)


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
    # ---- the join
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
    joined = ([], [], [])
    for lo, hi in zip(bounds[:-1], bounds[1:]):
        cols_l = [torch.cat([m[c][b] for b in range(lo, hi) for m in lm]) for c in range(2)]
        cols_r = [torch.cat([m[c][b] for b in range(lo, hi) for m in rm]) for c in range(3)]
        if cols_l[0].numel() == 0 or cols_r[0].numel() == 0:
            continue
        bi, pi = tk.join_unique_hash([cols_l[0]], [cols_r[0]], jhost)
        n = int(jhost[0])
        bi, pi = bi[:n], pi[:n]
        joined[0].append(cols_l[1].index_select(0, bi))
        joined[1].append(cols_r[1].index_select(0, pi))
        joined[2].append(cols_r[2].index_select(0, pi))
        del cols_l, cols_r, bi, pi
    del lm, rm
    if not joined[0]:
        e = torch.empty(0, dtype=torch.int64, device=dev)
        return e, e.clone(), e.clone()
    grp, jprice, jdisc = (torch.cat(c) for c in joined)
    del joined
    return aggregate(grp, jprice, jdisc, scale)


def aggregate(grp, jprice, jdisc, scale):
    """The keyed aggregation over the join's output columns (any device):
    (groups ascending, int64 sums, int64 counts)."""
    from pageflow_b200.partitions import agg_partitions
    dev = grp.device
    rows = grp.numel()
    step = max(1, min(1 << 30, CHUNK_B // (4 + 8 + 8)))
    spans = [(a, min(rows, a + step)) for a in range(0, rows, step)]
    row_b = 8 + 4 + 8 + 8
    B2, _, _ = agg_partitions(rows, len(spans), None, row_b, None, BUDGET_B)
    coeff = _coeff(dev)
    parts = []
    for a, b in spans:
        outs, counts = _pass1(grp[a:b], jprice[a:b], jdisc[a:b], scale, coeff, B2)
        starts = [0]
        for c in counts[:-1]:
            starts.append(starts[-1] + c)
        parts.append((outs, counts, starts))
    bucket_rows = [sum(p[1][k] for p in parts) for k in range(B2)]
    ends = _rounds(bucket_rows, row_b)
    groups = []
    for lo, hi in zip([0] + ends[:-1], ends):
        cols = []
        for i in range(4):
            pieces = []
            for outs, counts, starts in parts:
                a = starts[lo]
                b = starts[hi - 1] + counts[hi - 1]
                pieces.append(outs[i][a:b])
            cols.append(torch.cat(pieces))
        if cols[0].numel() == 0:
            continue
        uh, inv = torch.unique(cols[0], return_inverse=True)
        merged = []
        for v, op in ((cols[1], "amax"), (cols[2], "sum"), (cols[3], "sum")):
            r = torch.zeros(uh.numel(), dtype=v.dtype, device=dev)
            r.scatter_reduce_(0, inv, v, reduce=op, include_self=False)
            merged.append(r)
        groups.append(merged)
    key = torch.cat([g[0] for g in groups]).to(torch.int64)
    s = torch.cat([g[1] for g in groups])
    c = torch.cat([g[2] for g in groups])
    order = torch.argsort(key)
    return key[order], s[order], c[order]
