"""The join sort pipe's hash partition on the sm_100a kernel: the mirror of
PageFlow's ``operators/partition_sort.py`` (same function, thresholds,
limits, results and errors), calling ``pageflow_b200.tqpkernels``.

One call puts a tick's transfer set into the padded per-bucket layout
(each non-empty bucket starts on a whole ``lcm(row bytes, 512)``-byte unit):
a row's bucket is the top log2(B) bits of mix64(key), rows keep their source
order inside a bucket, and the global index (``goff`` + the row's pre-mask
position) is computed in the kernel.  Padding rows are left unwritten.
"""
from __future__ import annotations

from math import gcd
from typing import List, Optional

import torch

from . import tqpkernels
from .partitions import JOIN_B_MAX as _B_MAX

# Kept rows per mask row below which a masked tick collects its kept rows'
# ids first (select-first) rather than walking the pre-mask rows; the same
# crossover points as the reference (operators/partition_sort.py:39-46).
SELECT_FIRST_BELOW = 0.5
SELECT_FIRST_RAW_BELOW = 0.3

_MAX_COLS = 6
_MAX_WIDTHS = 4          # row widths, the gidx's 8 B included
_MAX_ROWS = (1 << 31) - 1
COMPRESSION_ALIGNMENT = 512

_host: Optional[torch.Tensor] = None


def _host_buffer() -> torch.Tensor:
    global _host
    if _host is None:
        _host = torch.empty(_B_MAX + _MAX_WIDTHS + 1, dtype=torch.int64, pin_memory=True)
    return _host


def row_bytes(t: torch.Tensor) -> int:
    """Bytes of one row: element size times width (1 for a 1-D tensor)."""
    return t.element_size() * (t.shape[1] if t.dim() == 2 else 1)


def aligned_partition_layout(partition_row_counts, row_b: int, align_unit_b: int):
    """(padded counts, byte starts, total rows) of the padded layout: each
    non-empty bucket rounded up to whole ``align_unit_b`` units (the layout
    of the reference's IO/codec/batched_compress.py:27-59)."""
    assert align_unit_b % row_b == 0
    unit = align_unit_b // row_b
    padded, starts, rows = [], [], 0
    for c in partition_row_counts:
        starts.append(rows * row_b)
        p = 0 if c == 0 else -(-c // unit) * unit
        padded.append(p)
        rows += p
    return padded, starts, rows


class PartitionedTensor:
    """One tensor holding B buckets, ``partition_row_counts[b]`` rows each, in
    bucket order, in the padded layout (the reference's
    IO/pipeline/common.py:22-45)."""
    __slots__ = ("tensor", "partition_row_counts")

    def __init__(self, tensor, partition_row_counts):
        self.tensor = tensor
        self.partition_row_counts = list(partition_row_counts)

    def bucket_starts(self):
        rb = row_bytes(self.tensor)
        _, starts, _ = aligned_partition_layout(
            self.partition_row_counts, rb,
            rb * COMPRESSION_ALIGNMENT // gcd(rb, COMPRESSION_ALIGNMENT))
        return [s // rb for s in starts]

    def buckets(self):
        """Each bucket's rows (views)."""
        starts = self.bucket_starts()
        return [self.tensor[s:s + c] for s, c in zip(starts, self.partition_row_counts)]


def partition(cols: List[torch.Tensor], key_pos: int, mask: Optional[torch.Tensor],
              goff: int, B: int, n_valid: Optional[int] = None) -> List[PartitionedTensor]:
    """``cols``: the tick's columns in output order, the int64 join key at
    ``key_pos``; with ``mask`` (the pre-mask mask), each column compacted or
    raw, and ``n_valid`` the mask's kept rows (needed when a column is raw);
    ``goff`` the tick's first global row.  Returns one PartitionedTensor per
    column, then the gidx's.  Raises ValueError for a tick outside the
    kernel's limits and RuntimeError for a count the mask contradicts."""
    key = cols[key_pos]
    n_pre = mask.shape[0] if mask is not None else key.shape[0]
    widths = []
    for t in cols:
        rb = row_bytes(t)
        if rb not in widths:
            widths.append(rb)
    if 8 not in widths:
        widths.append(8)
    if (not 1 <= B <= _B_MAX or B & (B - 1) or len(cols) > _MAX_COLS
            or len(widths) > _MAX_WIDTHS or key.dtype != torch.int64
            or key.dim() != 1 or n_pre > _MAX_ROWS
            or any(t.dim() not in (1, 2) for t in cols)
            or (mask is not None and (mask.dim() != 1 or mask.element_size() != 1))):
        raise ValueError(
            f"partition_sort: the tick is outside the kernel's limits (B={B}, "
            f"{len(cols)} columns of widths {widths}, a {key.dtype} key, "
            f"{n_pre} rows; at most B={_B_MAX}, {_MAX_COLS} columns, "
            f"{_MAX_WIDTHS} widths with the gidx's 8 B, a 1-D int64 key, "
            f"{_MAX_ROWS} rows, 1-D or 2-D columns, a 1-D 1-byte mask)")
    select_first = False
    if mask is None:
        comp = [0] * len(cols)
        n_valid = n_pre
    else:
        comp = [int(t.shape[0] != n_pre) for t in cols]
        lengths = {t.shape[0] for t, c in zip(cols, comp) if c}
        if len(lengths) > 1:
            raise ValueError(f"partition_sort: compacted columns of {sorted(lengths)} rows")
        if lengths:
            rows = lengths.pop()
            if n_valid is not None and n_valid != rows:
                raise RuntimeError(f"partition_sort: compacted columns hold {rows} rows, "
                                   f"the mask keeps {n_valid}")
            n_valid = rows
        elif n_valid is None:
            raise ValueError("partition_sort: raw columns under a mask need the mask's "
                             "kept rows")
        mask = mask.contiguous()
        below = SELECT_FIRST_BELOW if all(comp) else SELECT_FIRST_RAW_BELOW
        select_first = n_valid < below * n_pre
    host = _host_buffer()
    outs = tqpkernels.partition_sort([t.contiguous() for t in cols], comp, key_pos, mask,
                                     n_valid, goff, B, select_first, host)
    counts = host[:B].tolist()
    totals = host[B:B + len(widths)].tolist()
    kept = sum(counts)
    found = int(host[B + _MAX_WIDTHS])
    if found < 0:
        found = kept
    if found != n_valid or kept != n_valid:
        raise RuntimeError(f"partition_sort: the mask keeps {found} rows and {kept} were "
                           f"partitioned; the caller gave {n_valid}")
    return [PartitionedTensor(t[:totals[widths.index(row_bytes(t))]], counts) for t in outs]
