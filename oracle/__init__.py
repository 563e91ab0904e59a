"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke() and
bench.py's CPU baseline import it; the product never does).

A numpy front end over ``liboracle.so``, the plain-C restatement of
PageFlow's semantics for the relational hot path (``oracle.c`` lists the
reference lines each function follows).  Inputs and outputs are numpy arrays.
Pinned by ``tests/golden`` (vectors produced by the reference's own Python
code) in ``tests/test_oracle.py``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_c_i64 = ctypes.c_int64
_lib = None


def build() -> Path:
    """Compiles liboracle.so when oracle.c or synth.h is newer."""
    deps = [HERE / "oracle.c", HERE.parent / "pageflow_b200" / "csrc" / "synth.h"]
    if not LIB.exists() or any(d.stat().st_mtime > LIB.stat().st_mtime for d in deps):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        L.or_mix64.argtypes = [_i64p, _u64p, _c_i64]
        L.or_bucket.argtypes = [_i64p, _c_i64, ctypes.c_int, _i32p]
        L.or_partition_order.argtypes = [_i64p, _c_i64, ctypes.c_int, _i64p, _i64p]
        L.or_partition_order.restype = ctypes.c_int
        L.or_join_unique.argtypes = [_i64p, _i64p, _c_i64, _i64p, _i64p, _c_i64,
                                     ctypes.c_int, _i64p, _i64p]
        L.or_join_unique.restype = _c_i64
        L.or_semi_anti.argtypes = [_i64p, ctypes.c_void_p, _c_i64, _i64p,
                                   ctypes.c_void_p, _c_i64, ctypes.c_int,
                                   ctypes.c_int, _i64p]
        L.or_semi_anti.restype = _c_i64
        L.or_join_aggregate.argtypes = [_i64p, _i32p, _c_i64, _i64p, _i64p,
                                        ctypes.c_void_p, _c_i64, _c_i64, _c_i64,
                                        _c_i64, ctypes.c_int, ctypes.c_int, _i64p,
                                        _i64p, ctypes.POINTER(ctypes.c_uint64)]
        L.or_join_aggregate.restype = _c_i64
        L.or_gen_build.argtypes = [ctypes.c_uint64, _c_i64, _c_i64, _c_i64, _c_i64,
                                   _i64p, _i32p]
        L.or_gen_probe.argtypes = [ctypes.c_int, ctypes.c_uint64, _c_i64, _c_i64,
                                   _c_i64, _i64p, _i64p, _i64p]
        L.or_expected_groups.argtypes = [ctypes.c_int, ctypes.c_uint64, _c_i64,
                                         _c_i64, _c_i64, _c_i64, _c_i64,
                                         ctypes.c_int, _i64p, _i64p]
        L.or_expected_groups.restype = _c_i64
        L.or_gen_batch_probe.argtypes = [ctypes.c_uint64, _c_i64, _c_i64, _c_i64, ctypes.c_int,
                                         _i64p, _u64p, _i64p, _i64p]
        _u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
        L.or_page_decode.argtypes = [_u8p, _c_i64, _i64p, _c_i64]
        L.or_page_decode.restype = _c_i64
        L.or_gen_paged.argtypes = [ctypes.c_uint64, _c_i64, ctypes.c_int, _i64p, _u64p,
                                   _c_i64, _c_i64] + [_i64p] * 6
        L.or_gen_serve_dim.argtypes = [ctypes.c_uint64, _c_i64, ctypes.c_uint64, _c_i64, _c_i64,
                                       _c_i64, _i64p, _i32p]
        L.or_gen_serve_fact.argtypes = [ctypes.c_uint64, _c_i64, ctypes.c_int, _i64p, _u64p,
                                        _c_i64, _c_i64, _i64p, _i32p, _i64p]
        _lib = L
    return _lib


def _a(x, dtype=np.int64):
    return np.ascontiguousarray(x, dtype=dtype)


def threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


# ---- hash and partition ----------------------------------------------------

def mix64(keys) -> np.ndarray:
    """Murmur3 fmix64 of int64 keys, as uint64."""
    k = _a(keys)
    out = np.empty(k.shape[0], np.uint64)
    lib().or_mix64(k, out, k.shape[0])
    return out


def bucket(keys, B: int) -> np.ndarray:
    """Each key's radix bucket among B: the top log2(B) bits of mix64."""
    k = _a(keys)
    out = np.empty(k.shape[0], np.int32)
    lib().or_bucket(k, k.shape[0], B, out)
    return out


def rows_per_unit(row_bytes: int) -> int:
    return 512 // int(np.gcd(int(row_bytes), 512))


def partition(cols, key_pos: int, mask, goff: int, B: int):
    """The reference test's partition: mask -> mix64 bucket -> stable sort
    by bucket -> per-bucket split.  ``cols`` are raw (pre-mask) numpy
    columns.  Returns (counts, outputs): one list of per-bucket arrays per
    column, then the gidx's."""
    n_pre = cols[key_pos].shape[0] if mask is None else mask.shape[0]
    gidx = np.arange(goff, goff + n_pre, dtype=np.int64)
    if mask is not None:
        keep = np.asarray(mask).astype(bool)
        cols = [c[keep] for c in cols]
        gidx = gidx[keep]
    key = _a(cols[key_pos])
    counts = np.zeros(B, np.int64)
    order = np.empty(key.shape[0], np.int64)
    rc = lib().or_partition_order(key, key.shape[0], B, counts, order)
    if rc:
        raise ValueError(f"or_partition_order failed ({rc})")
    bounds = np.cumsum(counts)[:-1]
    outs = [np.split(c[order], bounds) for c in list(cols) + [gidx]]
    return counts, outs


def padded_layout(counts, row_b: int):
    """Each bucket's first row and the total rows of the padded layout: a
    non-empty bucket takes whole units of rows_per_unit(row_b) rows."""
    unit = rows_per_unit(row_b)
    starts, at = [], 0
    for c in counts:
        starts.append(at)
        at += -(-int(c) // unit) * unit
    return starts, at


# ---- joins --------------------------------------------------------------------

def join_unique(build_keys, probe_keys):
    """(build rows, probe rows) of a unique-build inner join, probe order."""
    nk = len(build_keys)
    b0 = _a(build_keys[0])
    b1 = _a(build_keys[1]) if nk == 2 else b0
    p0 = _a(probe_keys[0])
    p1 = _a(probe_keys[1]) if nk == 2 else p0
    bi = np.empty(p0.shape[0], np.int64)
    pi = np.empty(p0.shape[0], np.int64)
    m = lib().or_join_unique(b0, b1, b0.shape[0], p0, p1, p0.shape[0], nk, bi, pi)
    if m < 0:
        raise MemoryError("or_join_unique")
    return bi[:m], pi[:m]


OPS = {None: 0, "<>": 1, "<": 2, "<=": 3, ">": 4, ">=": 5}


def semi_anti(bk, pk, anti: bool, bv=None, pv=None, op=None):
    """Probe rows, ascending, with (semi) or without (anti) a build row of
    their key passing build.v OP probe.v."""
    bk, pk = _a(bk), _a(pk)
    bv_a = _a(bv) if bv is not None else None
    pv_a = _a(pv) if pv is not None else None
    out = np.empty(pk.shape[0], np.int64)
    m = lib().or_semi_anti(
        bk, bv_a.ctypes.data if bv_a is not None else None, bk.shape[0], pk,
        pv_a.ctypes.data if pv_a is not None else None, pk.shape[0], OPS[op],
        int(anti), out)
    if m < 0:
        raise MemoryError("or_semi_anti")
    return out[:m]


def expand(sorted_ids, start, length):
    """The sort/search pairs: probe row i's run sorted_ids[start[i] :
    start[i] + length[i]], in probe-row order."""
    sorted_ids, start, length = _a(sorted_ids), _a(start), _a(length)
    cr = np.repeat(np.arange(length.shape[0], dtype=np.int64), length)
    first = np.repeat(start, length)
    run0 = np.repeat(np.cumsum(length) - length, length)
    within = np.arange(cr.shape[0], dtype=np.int64) - run0
    return sorted_ids[first + within], cr


def join_aggregate(bkey, bgrp, pfk, pprice, pdisc, scale: int, group_min: int,
                   n_groups: int, B: int = 64, n_threads: int | None = None):
    """Dense (sum, count) over [group_min, group_min + n_groups) of
    SUM(price * (scale - disc)), COUNT(*) per build group of the
    unique-build join; returns (sum, count, matched, max |sum|)."""
    bkey, pfk, pprice = _a(bkey), _a(pfk), _a(pprice)
    bgrp = _a(bgrp, np.int32)
    pdisc_a = _a(pdisc) if pdisc is not None else None
    s = np.empty(n_groups, np.int64)
    c = np.empty(n_groups, np.int64)
    mx = ctypes.c_uint64(0)
    m = lib().or_join_aggregate(
        bkey, bgrp, bkey.shape[0], pfk, pprice,
        pdisc_a.ctypes.data if pdisc_a is not None else None, scale,
        pfk.shape[0], group_min, n_groups, B, n_threads or threads(), s, c,
        ctypes.byref(mx))
    if m < 0:
        raise MemoryError("or_join_aggregate")
    return s, c, int(m), int(mx.value)


# ---- workload generator ------------------------------------------------------

def gen_build(seed: int, n_build: int, n_groups: int, lo: int = 0, rows=None):
    rows = n_build - lo if rows is None else rows
    key = np.empty(rows, np.int64)
    grp = np.empty(rows, np.int32)
    lib().or_gen_build(seed, n_build, n_groups, lo, rows, key, grp)
    return key, grp


def gen_probe(config: int, seed: int, n_build: int, lo: int, rows: int):
    fk = np.empty(rows, np.int64)
    price = np.empty(rows, np.int64)
    disc = np.empty(rows, np.int64)
    lib().or_gen_probe(config, seed, n_build, lo, rows, fk, price, disc)
    return fk, price, disc


def gen_batch_probe(seed: int, n_build: int, lo: int, rows: int, edges, thr):
    """One batching instance's probe rows (fk, value) from its Zipf table."""
    fk = np.empty(rows, np.int64)
    val = np.empty(rows, np.int64)
    e = _a(edges)
    t = np.ascontiguousarray(thr, dtype=np.uint64)
    lib().or_gen_batch_probe(seed, n_build, lo, rows, t.shape[0], e, t, fk, val)
    return fk, val


def expected_groups(config: int, seed: int, n_build: int, n_groups: int,
                    lo: int, rows: int, scale: int = 100, n_threads=None):
    """Exact per-group (sum, count) of the workload's probe rows [lo, lo +
    rows), from the generator alone; and the matched rows."""
    s = np.empty(n_groups, np.int64)
    c = np.empty(n_groups, np.int64)
    m = lib().or_expected_groups(config, seed, n_build, n_groups, scale, lo,
                                 rows, n_threads or threads(), s, c)
    if m < 0:
        raise MemoryError("or_expected_groups")
    return s, c, int(m)


# ---- compressed pages ------------------------------------------------------

def page_decode(page) -> np.ndarray:
    """The values of one PFC1 page (int64; int32 columns sign-extended).
    Raises ValueError for a malformed page."""
    if isinstance(page, np.ndarray):
        b = np.ascontiguousarray(page, dtype=np.uint8)
    else:
        b = np.frombuffer(bytes(page), np.uint8)
    n = int(b[8:12].view(np.uint32)[0]) if b.shape[0] >= 12 else 0
    out = np.empty(max(n, 1), np.int64)
    got = lib().or_page_decode(b, b.shape[0], out, out.shape[0])
    if got < 0:
        raise ValueError(f"malformed page (status {got})")
    return out[:got]


PAGED_COLUMNS = ("fk", "date", "price", "quantity", "flag", "status")


def gen_paged(seed: int, n_build: int, lo: int, rows: int, edges, thr):
    """Rows [lo, lo + rows) of the paged workload's 6 columns (int64 each)."""
    cols = [np.empty(rows, np.int64) for _ in PAGED_COLUMNS]
    e = _a(edges)
    t = np.ascontiguousarray(thr, dtype=np.uint64)
    lib().or_gen_paged(seed, n_build, t.shape[0], e, t, lo, rows, *cols)
    return dict(zip(PAGED_COLUMNS, cols))


def paged_scan(cols: dict, n_rows: int, rows_per_page: int, groups_per_batch: int,
               filter_col: str, lo: int, hi: int, key_col: str, B: int):
    """The decode -> range filter -> radix partition of a paged table, per
    batch of groups_per_batch row groups: for each batch, the per-bucket row
    counts and each kept column's rows in bucket order (stable within a
    bucket; the product's order within a bucket is unspecified).  Follows
    IO/transfer/pre_comp_stage.py:54-73 (mask compaction), operators/
    filter.py:10-16 (the range mask) and the partition of
    tests/operators/test_partition_sort.py:106-118."""
    rows_b = rows_per_page * groups_per_batch
    out = []
    for r0 in range(0, n_rows, rows_b):
        r1 = min(n_rows, r0 + rows_b)
        f = cols[filter_col][r0:r1]
        keep = (f >= lo) & (f < hi)
        keys = cols[key_col][r0:r1][keep]
        bk = bucket(keys, B)
        order = np.argsort(bk, kind="stable")
        counts = np.bincount(bk, minlength=B).astype(np.int64)
        batch = {"counts": counts}
        for name, v in cols.items():
            if name != filter_col:
                batch[name] = v[r0:r1][keep][order]
        out.append(batch)
    return out


# ---- serving workload -----------------------------------------------------

def gen_serve_dim(seed: int, n_ranks: int, group_seed: int, n_groups: int, lo: int, rows: int):
    """Dimension rows [lo, lo + rows): (keys int64, groups int32)."""
    k = np.empty(rows, np.int64)
    g = np.empty(rows, np.int32)
    lib().or_gen_serve_dim(seed, n_ranks, group_seed, n_groups, lo, rows, k, g)
    return k, g


def gen_serve_fact(seed: int, n_ranks: int, lo: int, rows: int, edges, thr):
    """Fact rows [lo, lo + rows): (fk int64, date int32, value int64)."""
    fk = np.empty(rows, np.int64)
    d = np.empty(rows, np.int32)
    v = np.empty(rows, np.int64)
    e = _a(edges)
    t = np.ascontiguousarray(thr, dtype=np.uint64)
    lib().or_gen_serve_fact(seed, n_ranks, t.shape[0], e, t, lo, rows, fk, d, v)
    return fk, d, v


def serve_request(dim_keys, dim_groups, n_groups: int, fk, date, value, date_lo: int,
                  date_hi: int):
    """One serving request: SELECT group, SUM(value), COUNT(*) FROM fact JOIN
    dim ON fact.fk = dim.key WHERE date_lo <= date < date_hi GROUP BY
    dim.group, as (groups ascending, sums, counts) of the occupied groups:
    the filter (operators/filter.py:10-16), mask compaction
    (utility/tensor_utils.py:12-39), then or_join_aggregate."""
    keep = (np.asarray(date) >= date_lo) & (np.asarray(date) < date_hi)
    s, c, _, _ = join_aggregate(dim_keys, dim_groups, np.asarray(fk)[keep],
                                np.asarray(value)[keep], None, 1, 0, n_groups, B=16)
    occ = np.nonzero(c)[0]
    return occ.astype(np.int64), s[occ], c[occ]


# ---- join semantics ------------------------------------------------------------

def join_rows(left_key, right_key, join_type: str, keep=None):
    """The output rows of PageFlow's join core call (operators/hashjoin.py:
    293-356, 444-494) as (left row or -64, right row) pairs, sorted: inner =
    every (l, r) with equal keys that `keep(l, r)` passes; right-semi = the
    right rows with such a pair (left -64 dropped: left rows are empty);
    right-anti = the right rows with none; right-outer = the inner pairs
    plus every right row with none, its left side -64."""
    lk = np.asarray(left_key)
    rk = np.asarray(right_key)
    order = np.argsort(lk, kind="stable")
    sk = lk[order]
    lo = np.searchsorted(sk, rk, "left")
    hi = np.searchsorted(sk, rk, "right")
    pairs = []
    matched = np.zeros(rk.shape[0], bool)
    for r in range(rk.shape[0]):
        for j in range(lo[r], hi[r]):
            l = int(order[j])
            if keep is None or keep(l, r):
                pairs.append((l, r))
                matched[r] = True
    if join_type == "inner":
        out = pairs
    elif join_type == "right-semi":
        out = [(-64, r) for r in np.nonzero(matched)[0].tolist()]
    elif join_type == "right-anti":
        out = [(-64, r) for r in np.nonzero(~matched)[0].tolist()]
    elif join_type == "right-outer":
        out = pairs + [(-64, r) for r in np.nonzero(~matched)[0].tolist()]
    else:
        raise ValueError(join_type)
    return sorted(out)
