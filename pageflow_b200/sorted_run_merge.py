"""The sorted-run merge of the two-pass aggregation's pass 2, on the sm_100a
kernels: the mirror of PageFlow's ``operators/sorted_run_merge.py`` (same
functions, arguments and results).

- ``reduce_tick_slice(keys, vals, ops)``: the slice's unique keys ascending
  and each value column reduced per key (pf_unique_reduce: a radix sort of
  the keys, the segment heads, warp-combined atomics per segment);
- ``merge_sorted_unique_runs_inplace(key_buf, val_bufs, run_len, tick_keys,
  tick_vals, ops)``: the tick run merged into the running run held in the
  fixed buffers, returning the merged length (pf_merge_sorted_runs: binary
  searches place every key, matched keys combine; the merge is computed out
  of place into a temporary of the merged size and copied back, where the
  reference shifts in place in chunks: the same result, a larger peak).
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence, Tuple

import torch

from . import _native
from ._native import arr, check, lib, ptr, stream_of

MERGEABLE_OPS = ('sum', 'amax', 'amin')
_OP = {'sum': 0, 'amax': 1, 'amin': 2}
_KIND = {torch.int64: (0, 8), torch.int32: (0, 4), torch.float64: (1, 8), torch.float32: (1, 4)}
_PLACE_CHUNK = 1 << 26  # accepted for the reference's interface; the merge is one pass


def _describe(vals: Sequence[torch.Tensor], ops: Sequence[str], what: str):
    if len(vals) != len(ops):
        raise ValueError(f"{what}: {len(vals)} value columns, {len(ops)} ops")
    if len(vals) > 16:
        raise ValueError(f"{what}: at most 16 value columns")
    kinds, sizes, widths, opc = [], [], [], []
    for v, op in zip(vals, ops):
        if op not in _OP:
            raise ValueError(f"{what}: op {op!r} is not one of {MERGEABLE_OPS}")
        if v.dtype not in _KIND:
            raise TypeError(f"{what}: values of {v.dtype} (int32, int64, float32, float64 "
                            f"supported)")
        k, e = _KIND[v.dtype]
        w = 1
        for d in v.shape[1:]:
            w *= d
        kinds.append(k)
        sizes.append(e)
        widths.append(max(1, w))
        opc.append(_OP[op])
    return (arr(ctypes.c_int, kinds), arr(ctypes.c_int, sizes), arr(ctypes.c_int, widths),
            arr(ctypes.c_int, opc))


def reduce_tick_slice(keys: torch.Tensor, vals: Sequence[torch.Tensor],
                      ops: Sequence[str]) -> Tuple[torch.Tensor, List[torch.Tensor]]:
    """(unique ascending keys, each value column reduced per key) of one
    tick slice (sorted_run_merge.py:62-92)."""
    _native.require_cuda(keys, "keys")
    if keys.dtype != torch.int64 or keys.dim() != 1:
        raise TypeError("reduce_tick_slice: keys must be 1-D int64")
    keys = keys.contiguous()
    vals = [v.contiguous() for v in vals]
    n = keys.numel()
    for v in vals:
        if v.shape[0] != n:
            raise ValueError("reduce_tick_slice: value rows differ from the keys")
    kinds, sizes, widths, opc = _describe(vals, ops, "reduce_tick_slice")
    dev = keys.device
    out_k = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    outs = [torch.empty((max(n, 1),) + tuple(v.shape[1:]), dtype=v.dtype, device=dev)
            for v in vals]
    ws = _native.workspace(lib().pf_unique_reduce_workspace(n), dev)
    nu = ctypes.c_int64()
    vin = (ctypes.c_void_p * max(1, len(vals)))(*[ptr(v) for v in vals])
    vout = (ctypes.c_void_p * max(1, len(vals)))(*[ptr(o) for o in outs])
    check(lib().pf_unique_reduce(ptr(keys), n, len(vals), vin, vout, kinds, sizes, widths, opc,
                                 ptr(out_k), ctypes.byref(nu), ptr(ws), ws.numel(),
                                 stream_of(dev)), "reduce_tick_slice")
    u = nu.value
    return out_k[:u], [o[:u] for o in outs]


def merge_sorted_unique_runs_inplace(key_buf: torch.Tensor, val_bufs: Sequence[torch.Tensor],
                                     run_len: int, tick_keys: torch.Tensor,
                                     tick_vals: Sequence[torch.Tensor], ops: Sequence[str],
                                     place_chunk_rows: int = None) -> int:
    """Merge the ascending unique tick run into the running run held in
    ``key_buf[:run_len]`` / ``val_bufs[i][:run_len]``; the merged run lands in
    the same buffers at ``[:M]``; returns M (sorted_run_merge.py:94-174)."""
    T = tick_keys.numel()
    if T == 0:
        return run_len
    if run_len == 0:
        key_buf[:T] = tick_keys
        for vb, tv in zip(val_bufs, tick_vals):
            vb[:T] = tv
        return T
    R = run_len
    dev = key_buf.device
    kinds, sizes, widths, opc = _describe(list(tick_vals), ops, "merge_sorted_unique_runs")
    tick_keys = tick_keys.contiguous()
    tick_vals = [t.contiguous() for t in tick_vals]
    run_vals = [vb[:R].contiguous() for vb in val_bufs]
    cap = R + T
    out_k = torch.empty(cap, dtype=torch.int64, device=dev)
    outs = [torch.empty((cap,) + tuple(vb.shape[1:]), dtype=vb.dtype, device=dev)
            for vb in val_bufs]
    ws = _native.workspace(lib().pf_merge_sorted_runs_workspace(T), dev)
    m = ctypes.c_int64()
    nc = max(1, len(val_bufs))
    a = (ctypes.c_void_p * nc)(*[ptr(v) for v in run_vals])
    b = (ctypes.c_void_p * nc)(*[ptr(v) for v in tick_vals])
    o = (ctypes.c_void_p * nc)(*[ptr(v) for v in outs])
    run_keys = key_buf[:R].contiguous()
    check(lib().pf_merge_sorted_runs(ptr(run_keys), a, R, ptr(tick_keys), b, T,
                                     len(val_bufs), kinds, sizes, widths, opc, ptr(out_k), o,
                                     ctypes.byref(m), ptr(ws), ws.numel(), stream_of(dev)),
          "merge_sorted_unique_runs")
    M = m.value
    assert M <= key_buf.shape[0], (
        f"merge capacity exhausted: M={M} > buf={key_buf.shape[0]} — the buffers must be "
        f"sized to the pass2 total input rows")
    key_buf[:M] = out_k[:M]
    for vb, ov in zip(val_bufs, outs):
        vb[:M] = ov[:M]
    return M


def sort_pairs(keys: torch.Tensor, vals: torch.Tensor | None = None):
    """(keys ascending, their values or row numbers), a stable radix sort."""
    _native.require_cuda(keys, "keys")
    keys = keys.contiguous()
    n = keys.numel()
    dev = keys.device
    ko = torch.empty(n, dtype=torch.int64, device=dev)
    vo = torch.empty(n, dtype=torch.int64, device=dev)
    ws = _native.workspace(lib().pf_sort_pairs_workspace(n), dev)
    vals = vals.contiguous() if vals is not None else None
    check(lib().pf_sort_pairs(ptr(keys), ptr(vals), n,
                              ptr(ko), ptr(vo), ptr(ws), ws.numel(), stream_of(dev)),
          "sort_pairs")
    return ko, vo
