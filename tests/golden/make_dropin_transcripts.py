"""Records how the reference's own operator wrappers call its native module,
for the drop-in replay test (tests/test_dropin_replay_gpu.py).

The reference's ``operators/partition_sort.py`` and ``operators/join_core.py``
are imported unchanged from a checkout, with ``TQPlib.tqpkernels`` bound to a
recording stand-in.  The stand-in answers each call in the native module's
contract (worst-case-sized outputs, counts and flags in ``host_out``), with
the results computed by this repository's oracle; the wrapper then narrows
and checks them as it does in the engine.  Written per call: the exact
arguments the wrapper passed, and what the wrapper returned.  The replay test
makes the same calls into ``pageflow_b200.tqpkernels`` on a GPU and checks
that the outputs, read back through ``host_out`` the way the wrapper reads
them, equal what the wrapper returned.  Run where the reference is present:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_dropin_transcripts.py /path/to/PageFlow

Cases follow the reference's tests/operators/test_partition_sort.py (tick
sizes, six columns of four widths, masks under both prologues and both
raw-column modes, mixed columns, one crowded bucket, a global offset near
6e9, B = 1 and 512) and tests/operators/test_join_core.py (semi / anti with
and without a residual summary, expand with empty runs).  The wrappers take
their own mask prologue by their own thresholds; nothing is forced.
"""
from __future__ import annotations

import json
import os
import sys
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

import oracle  # noqa: E402
from tests.golden.make_golden import import_reference  # noqa: E402

OUT = HERE / "dropin_transcripts.npz"
WIDTH_CLASSES = 4


def _np(t):
    return None if t is None else t.detach().cpu().numpy()


def _row_bytes(a: np.ndarray) -> int:
    return a.dtype.itemsize * (a.shape[1] if a.ndim == 2 else 1)


class Recorder:
    """The stand-in for TQPlib.tqpkernels: records each call's arguments and
    answers it in the native module's contract from the oracle."""

    def __init__(self):
        self.calls = []

    def partition_sort(self, cols, comp, key_idx, mask, n_valid, goff, B, select_first,
                       host_out):
        np_cols = [_np(c) for c in cols]
        np_mask = _np(mask)
        # the oracle takes every column raw (the mask's rows): restore the
        # compacted ones to full length around the kept rows
        full = []
        for a, c in zip(np_cols, comp):
            if c:
                f = np.zeros((np_mask.shape[0],) + a.shape[1:], dtype=a.dtype)
                f[np_mask.astype(bool)] = a
                a = f
            full.append(a)
        counts, bucket_rows = oracle.partition(full, key_idx, np_mask, goff, B)
        widths = []
        for a in np_cols:
            if _row_bytes(a) not in widths:
                widths.append(_row_bytes(a))
        if 8 not in widths:
            widths.append(8)
        outs, totals = [], {}
        kinds = [(a.dtype, a.shape[1:]) for a in np_cols] + [(np.dtype(np.int64), ())]
        for (dt, tail), rows in zip(kinds, bucket_rows):
            rb = dt.itemsize * (tail[0] if tail else 1)
            starts, total = oracle.padded_layout(counts, rb)
            cap = n_valid + B * (oracle.rows_per_unit(rb) - 1)
            o = np.zeros((cap,) + tuple(tail), dtype=dt)
            for s, r in zip(starts, rows):
                o[s:s + len(r)] = r
            outs.append(torch.from_numpy(o))
            totals[rb] = total
        host_out[:B] = torch.from_numpy(counts.astype(np.int64))
        for k, w in enumerate(widths):
            host_out[B + k] = totals[w]
        host_out[B + WIDTH_CLASSES] = int(counts.sum()) if mask is not None else -1
        self.calls.append(dict(fn="partition_sort", cols=np_cols, comp=list(comp),
                               key_idx=key_idx, mask=np_mask, n_valid=int(n_valid),
                               goff=int(goff), B=int(B), select_first=bool(select_first)))
        return outs

    def join_semi_anti(self, build_key, probe_key, build_val, probe_val, op, anti, host_out):
        bk, pk, bv, pv = _np(build_key), _np(probe_key), _np(build_val), _np(probe_val)
        name = {0: None, 1: '<>', 2: '<', 3: '<=', 4: '>', 5: '>='}[op]
        rows = oracle.semi_anti(bk, pk, anti, bv if op else None, pv if op else None, name)
        out = np.zeros(pk.shape[0], dtype=np.int64)
        out[:len(rows)] = rows
        host_out[0] = len(rows)
        host_out[1] = int((bk == np.iinfo(np.int64).min).any())
        self.calls.append(dict(fn="join_semi_anti", build_key=bk, probe_key=pk, build_val=bv,
                               probe_val=pv, op=int(op), anti=bool(anti)))
        return torch.from_numpy(out)

    def join_expand(self, sorted_ids, start, length, host_out):
        cs, cr = oracle.expand(_np(sorted_ids), _np(start), _np(length))
        host_out[0] = len(cs)
        self.calls.append(dict(fn="join_expand", sorted_ids=_np(sorted_ids), start=_np(start),
                               length=_np(length)))
        return [torch.from_numpy(cs), torch.from_numpy(cr)]


def _gen(seed):
    return torch.Generator(device="cpu").manual_seed(seed)


def _column(n, kind, seed):
    g = _gen(seed)
    if kind == "i64":
        return torch.randint(-(1 << 62), 1 << 62, (n,), dtype=torch.int64, generator=g)
    if kind == "i32":
        return torch.randint(-(1 << 30), 1 << 30, (n,), dtype=torch.int32, generator=g)
    if kind == "i16":
        return torch.randint(-(1 << 14), 1 << 14, (n,), dtype=torch.int16, generator=g)
    if kind == "i8":
        return torch.randint(-128, 128, (n,), dtype=torch.int8, generator=g)
    if kind == "s25":
        return torch.randint(0, 256, (n, 25), dtype=torch.uint8, generator=g)
    raise ValueError(kind)


def _table(n, kinds, seed, key_pos=0, skew=False):
    cols = [_column(n, k, seed + 1 + c) for c, k in enumerate(kinds)]
    key = (torch.full((n,), 7, dtype=torch.int64) if skew else
           torch.randint(-(1 << 40), 1 << 40, (n,), dtype=torch.int64, generator=_gen(seed)))
    cols.insert(key_pos, key)
    return cols


def _mask(n, keep, seed):
    return torch.rand(n, generator=_gen(seed)) < keep


def partition_cases():
    """(name, cols, key_pos, mask, goff, B, n_valid) in the spirit of the
    reference's partition tests."""
    yield "plain 4097 rows", _table(4097, ["i64"], 1), 0, None, 0, 32, None
    yield "six columns, four widths", _table(3001, ["i64", "i32", "i8", "s25", "i64"], 3, 2), \
        2, None, 0, 64, None
    yield "one crowded bucket", _table(2500, ["i64", "s25"], 5, skew=True), 0, None, 0, 64, None
    yield "offset near 6e9", _table(4096, ["i64"], 6), 0, None, 6_000_000_000 - 4096, 512, None
    yield "B = 1", _table(1000, ["i32"], 7), 0, None, 11, 1, None
    for keep, seed in ((0.3, 21), (0.63, 22)):
        cols = _table(3000, ["i64", "s25"], seed)
        m = _mask(3000, keep, seed + 100)
        yield f"compacted, keep {keep}", [c[m] for c in cols], 0, m, 777, 32, None
    for keep, seed in ((0.1, 31), (0.6, 32)):
        cols = _table(3000, ["i64", "s25", "i16"], seed)
        m = _mask(3000, keep, seed + 100)
        yield f"raw with the count, keep {keep}", cols, 0, m, 99, 64, int(m.sum())
    cols = _table(2500, ["i64", "s25", "i32"], 41)
    m = _mask(2500, 0.4, 42)
    mixed = [c[m] if k else c for c, k in zip(cols, [False, True, False, True])]
    yield "raw and compacted mixed", mixed, 0, m, 5, 64, int(m.sum())


def main(root: str):
    import_reference(root)
    rec = Recorder()
    mod = types.ModuleType("TQPlib.tqpkernels")
    for name in ("partition_sort", "join_semi_anti", "join_expand"):
        setattr(mod, name, getattr(rec, name))
    sys.modules["TQPlib.tqpkernels"] = mod
    pkg = sys.modules.setdefault("TQPlib", types.ModuleType("TQPlib"))
    pkg.tqpkernels = mod
    from operators import join_core, partition_sort  # the reference's, unchanged
    # each wrapper's host_out is a pinned buffer it makes on first use; this
    # machine has no driver to pin with, so the buffer it would make is handed
    # in as plain host memory (the wrappers' code runs as it is)
    partition_sort._host = torch.empty(partition_sort._B_MAX + partition_sort._MAX_WIDTHS + 1,
                                       dtype=torch.int64)
    join_core._host = torch.empty(2, dtype=torch.int64)

    arrays, meta = {}, []

    def put(key, a):
        if a is not None:
            arrays[key] = np.ascontiguousarray(a)

    for name, cols, key_pos, mask, goff, B, n_valid in partition_cases():
        before = len(rec.calls)
        got = partition_sort.partition(cols, key_pos, mask, goff, B, n_valid=n_valid)
        assert len(rec.calls) == before + 1
        i = len(meta)
        call = rec.calls[-1]
        for j, a in enumerate(call["cols"]):
            put(f"c{i}_in{j}", a)
        put(f"c{i}_mask", call["mask"])
        for j, pt in enumerate(got):
            put(f"c{i}_out{j}", _np(pt.tensor))
        meta.append(dict(case=name, fn="partition_sort", ncols=len(call["cols"]),
                         comp=call["comp"], key_idx=call["key_idx"],
                         has_mask=call["mask"] is not None, n_valid=call["n_valid"],
                         goff=call["goff"], B=call["B"], select_first=call["select_first"],
                         counts=got[0].partition_row_counts, nout=len(got)))

    g = _gen(51)
    bk = torch.randint(-50, 700, (2000,), dtype=torch.int64, generator=g)
    pk = torch.randint(-60, 1400, (1500,), dtype=torch.int64, generator=g)
    bv = torch.randint(0, 4, (2000,), dtype=torch.int64, generator=g)
    pv = torch.randint(0, 4, (1500,), dtype=torch.int64, generator=g)
    for anti in (False, True):
        for summary in (None, (bv, pv, '<'), (bv, pv, '<>'), (bv, pv, '>=')):
            got = join_core.semi_anti(bk, pk, anti, summary)
            i = len(meta)
            call = rec.calls[-1]
            put(f"c{i}_build_key", call["build_key"])
            put(f"c{i}_probe_key", call["probe_key"])
            put(f"c{i}_build_val", call["build_val"])
            put(f"c{i}_probe_val", call["probe_val"])
            put(f"c{i}_out0", _np(got))
            meta.append(dict(case=f"{'anti' if anti else 'semi'} {summary and summary[2]}",
                             fn="join_semi_anti", op=call["op"], anti=call["anti"],
                             has_vals=call["build_val"] is not None, nout=1))

    for lengths, seed in (([1, 0, 2, 0, 0, 3, 0], 61), (None, 62)):
        gg = _gen(seed)
        if lengths is None:
            length = torch.randint(0, 7, (3000,), dtype=torch.int64, generator=gg)
            length[torch.randint(0, 10, (3000,), generator=gg) < 4] = 0
        else:
            length = torch.tensor(lengths, dtype=torch.int64)
        n_build = 8000
        sorted_ids = torch.randperm(n_build, generator=gg)
        start = torch.minimum(torch.randint(0, n_build, (length.numel(),), generator=gg),
                              n_build - length)
        got = join_core.expand(sorted_ids, start, length)
        i = len(meta)
        call = rec.calls[-1]
        put(f"c{i}_sorted_ids", call["sorted_ids"])
        put(f"c{i}_start", call["start"])
        put(f"c{i}_length", call["length"])
        put(f"c{i}_out0", _np(got[0]))
        put(f"c{i}_out1", _np(got[1]))
        meta.append(dict(case=f"expand {seed}", fn="join_expand", nout=2))

    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"{len(meta)} recorded calls written to {OUT}")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PAGEFLOW_REFERENCE")
    if not ref:
        sys.exit("usage: make_dropin_transcripts.py <reference checkout> "
                 "(or set PAGEFLOW_REFERENCE)")
    main(ref)
