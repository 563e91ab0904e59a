"""The hash route of the keyed (GROUP BY) aggregation's pass 1 on the sm_100a
kernels: the mirror of PageFlow's ``KeyedAggregate.pass1`` (operators/
aggregate.py:1511-1563) for aggregates over plain columns.

One chunk's rows are reduced to one row per group:

  hash      each row's grouping hash, the linear hash of its key columns'
            packed words with the deterministic coefficients of
            ``_make_key_coeffs`` (:529-548; pf_group_hash)
  groups    the unique hashes ascending, one representative of every key
            column per group, and each aggregate's partial (pf_unique_reduce:
            radix sort of the hashes, segment reduction; a key column travels
            as its packed words)
  buckets   with B > 1, each group's bucket (``_bucket_ids``) and the groups
            per bucket, on the host and on the device (pf_hash_buckets)

Aggregates: ``('sum', col)``, ``('count', None)`` (every row) or
``('count', col)`` (the rows whose value is not the null -64), ``('min',
col)``, ``('max', col)`` (folded from 0, as the reference's partial is) and
``('avg', col)`` (its state: [sum of every row, count of the non-null
ones]), each as the reference's pass 1 computes it.  SUM of an
integer column is exact in int64 (the reference sums through a float64
bincount, :395-398, which equals it while every partial stays below 2^53).
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Sequence, Tuple

import torch

from . import _native
from ._native import check, lib, ptr, stream_of
from .sorted_run_merge import reduce_tick_slice

NULL = -64   # the reference's null value (constants.null)
COEFF_BASE_SEED = int(os.environ.get('TQP_HASH_SEED', '2029')) & 0x7FFF_FFFF_FFFF_FFFF


def packed_width(col: torch.Tensor) -> int:
    """int64 words of a (N, W) tensor's rows (_packed_width, :477-479)."""
    return (col.shape[1] * col.element_size() + 7) // 8


def make_key_coeffs(key_tensors: Sequence[torch.Tensor], device) -> List[torch.Tensor]:
    """The reference's coefficients: a local generator on the device seeded
    with the base seed, one randint(2, 10_000_000) vector per packed key
    column (_make_key_coeffs, :529-548)."""
    g = torch.Generator(device=device)
    g.manual_seed(COEFF_BASE_SEED)
    return [torch.randint(2, 10_000_000, (packed_width(c),), dtype=torch.int64, device=device,
                          generator=g) for c in key_tensors]


def _as_2d(col: torch.Tensor) -> torch.Tensor:
    return col.unsqueeze(1) if col.dim() < 2 else col


def group_hash(key_tensors: Sequence[torch.Tensor], coeffs: Sequence[torch.Tensor]) -> torch.Tensor:
    """Each row's grouping hash (_hash_key_columns, :551-564), one launch."""
    keys = [_as_2d(k).contiguous() for k in key_tensors]
    n = keys[0].shape[0]
    dev = keys[0].device
    out = torch.empty(n, dtype=torch.int64, device=dev)
    coeffs = [c.contiguous() for c in coeffs]
    cols = (ctypes.c_void_p * len(keys))(*[ptr(k) for k in keys])
    rb = (ctypes.c_int * len(keys))(*[k.shape[1] * k.element_size() for k in keys])
    cf = (ctypes.c_void_p * len(keys))(*[ptr(c) for c in coeffs])
    check(lib().pf_group_hash(cols, rb, cf, len(keys), n, ptr(out), stream_of(dev)), "group_hash")
    return out


def hash_buckets(hashes: torch.Tensor, B: int):
    """(bucket int32, counts on the host, counts on the device)."""
    n = hashes.numel()
    dev = hashes.device
    bucket = torch.empty(n, dtype=torch.int32, device=dev)
    counts = torch.empty(B, dtype=torch.int64, device=dev)
    check(lib().pf_hash_buckets(ptr(hashes), n, B, ptr(bucket), ptr(counts), stream_of(dev)),
          "hash_buckets")
    return bucket, counts.tolist(), counts


def _pack_words(col: torch.Tensor) -> torch.Tensor:
    """A (N, W) tensor's rows as int64 words, zero-padded (_pack_as_int64)."""
    n, w = col.shape
    rb = w * col.element_size()
    raw = col.contiguous().view(torch.uint8).reshape(n, rb)
    tb = (rb + 7) // 8 * 8
    if tb == rb:
        return raw.view(torch.int64)
    buf = torch.zeros(n, tb, dtype=torch.uint8, device=col.device)
    buf[:, :rb] = raw
    return buf.view(torch.int64)


def _unpack_words(words: torch.Tensor, like: torch.Tensor) -> torch.Tensor:
    n = words.shape[0]
    rb = like.shape[1] * like.element_size()
    raw = words.contiguous().view(torch.uint8).reshape(n, -1)[:, :rb].contiguous()
    return raw.view(like.dtype).reshape(n, like.shape[1])


class KeyedPass1:
    """Pass 1 of a keyed aggregation over plain columns: ``key_ids`` group
    the rows (``emitted_ids``, default all of them, are carried out as key
    representatives); ``aggs`` is a list of (op, column id or None)."""

    def __init__(self, key_ids: Sequence[int], aggs: Sequence[Tuple[str, int]],
                 emitted_ids: Sequence[int] | None = None):
        self.key_ids = list(key_ids)
        self.emitted = list(self.key_ids if emitted_ids is None else emitted_ids)
        self.aggs = list(aggs)
        for op, _ in self.aggs:
            if op not in ('sum', 'count', 'min', 'max', 'avg'):
                raise NotImplementedError(f"KeyedPass1: aggregate {op!r}")
        self._coeffs = None

    def pass1(self, columns: Dict[int, torch.Tensor], B: int = 1):
        """``[hash] + keys + values`` of one chunk (hash ascending, unique),
        and the buckets (None at B = 1 or with no group, else (bucket,
        counts, counts_t)), as KeyedAggregate.pass1 returns them."""
        keys = [_as_2d(columns[k]) for k in self.key_ids]
        if self._coeffs is None:
            self._coeffs = make_key_coeffs(keys, keys[0].device)
        h = group_hash(keys, self._coeffs)
        vals, ops, post = [], [], []
        emitted = [_as_2d(columns[k]) for k in self.emitted]
        for e in emitted:
            vals.append(_pack_words(e))
            ops.append('amax')   # every row of a group holds the same key
        n = h.numel()
        for op, cid in self.aggs:
            if op == 'count':
                # COUNT(x) counts the rows whose x is not the null value
                # (operator_utils.py:384-385); COUNT(*) every row
                if cid is None:
                    vals.append(torch.ones(n, dtype=torch.int64, device=h.device))
                else:
                    vals.append((columns[cid] != NULL).to(torch.int64))
                ops.append('sum')
                post.append(('count', len(vals) - 1))
            elif op == 'avg':
                # the state [SUM(x), COUNT(x)] (aggregate.py:249-250, 323-336):
                # the sum over every row, the count over the non-null ones
                v = columns[cid]
                vals.append(v if v.dtype in (torch.float32, torch.float64) else v.to(torch.int64))
                ops.append('sum')
                vals.append((v != NULL).to(torch.int64))
                ops.append('sum')
                post.append(('avg', len(vals) - 2))
            else:
                v = columns[cid]
                if v.dtype in (torch.float32, torch.float64):
                    pass
                elif op == 'sum' or v.dtype not in (torch.int64, torch.int32):
                    v = v.to(torch.int64)   # integer sums in int64, as the reference's result
                vals.append(v)
                ops.append({'sum': 'sum', 'min': 'amin', 'max': 'amax'}[op])
                post.append((op, len(vals) - 1))
        u, red = reduce_tick_slice(h, vals, ops)
        key_reps = []
        for i, e in enumerate(emitted):
            rep = _unpack_words(red[i], e)
            key_reps.append(rep.squeeze(1) if rep.shape[1] == 1 else rep)
        agg_vals = []
        for op, j in post:
            if op == 'avg':
                agg_vals.append(torch.stack([red[j].to(torch.float64),
                                             red[j + 1].to(torch.float64)], dim=1))
            elif op == 'max':
                # MAX folds into a zeroed partial (a scatter_reduce into zeros
                # that includes them, operator_utils.py:365-369), so a group
                # whose values are all negative has the partial 0
                agg_vals.append(torch.clamp_min(red[j], 0))
            else:
                agg_vals.append(red[j])
        buckets = None
        if B > 1 and u.numel() > 0:
            buckets = hash_buckets(u, B)
        return [u] + key_reps + agg_vals, buckets
