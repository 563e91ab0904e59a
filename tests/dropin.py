"""Test helpers that call the drop-in module (``pageflow_b200.tqpkernels``,
the stand-in for the reference's ``TQPlib.tqpkernels``) the way a caller
does, and read each call's outputs back through its ``host_out`` contract:

- ``partition``: one ``partition_sort`` call; each output narrowed to its
  row-width class's padded total, the bucket counts and the kept rows the
  kernel found returned beside it;
- ``unique_pairs`` / ``semi_anti_rows`` / ``expand_pairs``: the join cores,
  narrowed to ``host_out[0]`` rows.

The caller picks the mask prologue (``select_first``) itself, so a test can
force either one; no selectivity rule lives here.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import torch

from pageflow_b200 import tqpkernels

WIDTH_CLASSES = tqpkernels.MAXCLS


def _host(n: int) -> torch.Tensor:
    return torch.empty(n, dtype=torch.int64, pin_memory=True)


def row_bytes(t: torch.Tensor) -> int:
    return t.element_size() * (t.shape[1] if t.dim() == 2 else 1)


def padded_starts(counts, rb: int):
    """First row of each bucket and the total rows of the padded layout:
    every non-empty bucket rounded up to whole units of lcm(rb, 512) bytes."""
    unit = 512 // __import__("math").gcd(rb, 512)
    starts, rows = [], 0
    for c in counts:
        starts.append(rows)
        rows += -(-c // unit) * unit
    return starts, rows


@dataclass
class Partitioned:
    tensor: torch.Tensor
    counts: List[int]

    def buckets(self):
        starts, _ = padded_starts(self.counts, row_bytes(self.tensor))
        return [self.tensor[s:s + c] for s, c in zip(starts, self.counts)]


@dataclass
class PartitionCall:
    outputs: List[Partitioned]
    counts: List[int]
    totals: List[int]
    found: int          # kept rows a mask prologue counted, -1 without one


def partition(cols: List[torch.Tensor], key_pos: int, mask: Optional[torch.Tensor],
              goff: int, B: int, n_valid: Optional[int] = None,
              select_first: bool = False) -> PartitionCall:
    """One drop-in ``partition_sort`` call.  Without a mask every column is
    raw; with one, a column of the mask's length is raw and a shorter one is
    compacted (``n_valid`` is then its length unless given)."""
    n_pre = mask.shape[0] if mask is not None else cols[key_pos].shape[0]
    comp = [0] * len(cols) if mask is None else [int(t.shape[0] != n_pre) for t in cols]
    if n_valid is None:
        short = [t.shape[0] for t, c in zip(cols, comp) if c]
        n_valid = short[0] if short else n_pre
    widths: List[int] = []
    for t in cols:
        if row_bytes(t) not in widths:
            widths.append(row_bytes(t))
    if 8 not in widths:
        widths.append(8)
    host = _host(B + WIDTH_CLASSES + 1)
    outs = tqpkernels.partition_sort([t.contiguous() for t in cols], comp, key_pos,
                                     None if mask is None else mask.contiguous(), n_valid,
                                     goff, B, select_first, host)
    counts = host[:B].tolist()
    totals = host[B:B + len(widths)].tolist()
    narrowed = [Partitioned(t[:totals[widths.index(row_bytes(t))]], counts) for t in outs]
    return PartitionCall(narrowed, counts, totals, int(host[B + WIDTH_CLASSES]))


def unique_pairs(build_keys, probe_keys):
    host = _host(2)
    bi, pi = tqpkernels.join_unique_hash(list(build_keys), list(probe_keys), host)
    n = int(host[0])
    return bi[:n], pi[:n]


def semi_anti_rows(build_key, probe_key, anti: bool, build_val=None, probe_val=None, op=0):
    """The kept probe rows, or None when a build key is the empty-slot value."""
    host = _host(2)
    out = tqpkernels.join_semi_anti(build_key, probe_key, build_val, probe_val, op, anti, host)
    n, bad = host.tolist()
    return None if bad else out[:n]


def expand_pairs(sorted_ids, start, length):
    return tuple(tqpkernels.join_expand(sorted_ids, start, length, _host(2)))
