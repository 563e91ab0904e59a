"""Late materialization: the rows of several columns at one index array in
one launch (pf_gather), the replacement of the reference's per-column
``torch.index_select`` and ``conversion.index_with_null`` (conversion.py:
39-50) in the join tail (operators/hashjoin.py:355-377)."""
from __future__ import annotations

import ctypes
from typing import List, Sequence

import torch

from . import _native
from ._native import arr, check, lib, ptr, stream_of

NULL = -64   # the reference's constants.null
MAX_COLUMNS = 16


def null_bits(dtype: torch.dtype) -> int:
    """The bit pattern of the null value (-64) as one element of dtype
    (what ``masked_fill(mask, constants.null)`` writes)."""
    one = torch.full((1,), NULL, dtype=dtype)
    return int.from_bytes(bytes(one.view(torch.uint8).tolist()), "little")


def _gather(cols: Sequence[torch.Tensor], idx: torch.Tensor, allow_null: bool,
            check_range: bool = False) -> List[torch.Tensor]:
    """The kernel never reads outside a column: an index outside [0, rows)
    yields a null row and is counted; with check_range the call waits for
    the count and raises IndexError as torch.index_select would."""
    if not cols:
        return []
    if len(cols) > MAX_COLUMNS:
        return (_gather(cols[:MAX_COLUMNS], idx, allow_null, check_range)
                + _gather(cols[MAX_COLUMNS:], idx, allow_null, check_range))
    _native.require_cuda(idx, "gather index")
    if idx.dtype != torch.int64 or idx.dim() != 1:
        raise RuntimeError("gather index must be 1-D int64")
    idx = idx.contiguous()
    n = idx.numel()
    n_src = cols[0].shape[0]
    outs, rb, eb, nb = [], [], [], []
    srcs, dsts = [], []
    for c in cols:
        _native.require_cuda(c, "gather column")
        if c.shape[0] != n_src:
            raise RuntimeError("gather columns have different row counts")
        out = torch.empty((n,) + tuple(c.shape[1:]), dtype=c.dtype, device=c.device)
        outs.append(out)
        width = 1
        for d in c.shape[1:]:
            width *= d
        if width == 0:
            continue  # rows of no bytes: nothing to copy
        c = c.contiguous()
        srcs.append(c)
        dsts.append(out)
        rb.append(width * c.element_size())
        eb.append(c.element_size())
        nb.append(null_bits(c.dtype))
    if n == 0 or not srcs:
        return outs
    if n_src == 0 and not allow_null:
        raise RuntimeError("index out of range: gather from an empty column")
    bad = torch.zeros(1, dtype=torch.int64, device=idx.device)
    ins = (ctypes.c_void_p * len(srcs))(*[ptr(c) if c.numel() else None for c in srcs])
    ous = (ctypes.c_void_p * len(dsts))(*[ptr(o) for o in dsts])
    check(lib().pf_gather(ins, ous, arr(ctypes.c_int, rb), arr(ctypes.c_int, eb),
                          arr(ctypes.c_uint64, nb), len(srcs), ptr(idx), n, n_src,
                          1 if allow_null else 0, NULL, ptr(bad), stream_of(idx.device)),
          "gather")
    if check_range and int(bad.item()):
        raise IndexError(f"gather: {int(bad.item())} indexes outside [0, {n_src})")
    return outs


def index_select_many(cols: Sequence[torch.Tensor], idx: torch.Tensor,
                      check_range: bool = False) -> List[torch.Tensor]:
    """``[torch.index_select(c, 0, idx) for c in cols]`` in one launch."""
    return _gather(cols, idx, False, check_range)


def index_with_null_many(cols: Sequence[torch.Tensor], idx: torch.Tensor) -> List[torch.Tensor]:
    """``[conversion.index_with_null(c, idx) for c in cols]`` in one launch:
    a row of nulls (-64 as the column's dtype) where ``idx`` is -64."""
    return _gather(cols, idx, True)


def index_select(x: torch.Tensor, idx: torch.Tensor) -> torch.Tensor:
    return _gather([x], idx, False)[0]


def index_with_null(x: torch.Tensor, idx: torch.Tensor) -> torch.Tensor:
    return _gather([x], idx, True)[0]
