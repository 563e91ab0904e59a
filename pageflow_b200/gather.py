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


def gather_from_host(segments: Sequence[Sequence[torch.Tensor]], seg_rows: Sequence[int],
                     idx: torch.Tensor, allow_null: bool = True, base: int = 0,
                     sorted_reads: bool = True) -> tuple:
    """Zero-copy late materialization (pf_gather_segments): ``segments[c][s]``
    is column c's segment s in pinned host memory, holding rows
    ``[seg_rows[s], seg_rows[s + 1])``; returns each column's rows
    ``idx + base`` on idx's device, read in place over the host link, a null
    row (-64 as the dtype) where idx is -64, and the count of indexes outside
    the segments (their rows are null too).  With ``sorted_reads`` the rows
    are fetched in ascending index order, so neighbouring threads read
    neighbouring host rows (the reference's zero_copy_rearrange argsorts its
    indexes for the same reason, IO/zero_copy_reader.cu:84-90)."""
    _native.require_cuda(idx, "gather index")
    if idx.dtype != torch.int64 or idx.dim() != 1:
        raise RuntimeError("gather index must be 1-D int64")
    ncols, nseg = len(segments), len(seg_rows) - 1
    if ncols < 1 or ncols > MAX_COLUMNS or nseg < 1:
        raise RuntimeError("gather_from_host: 1-16 columns of at least one segment")
    idx = idx.contiguous()
    n = idx.numel()
    dev = idx.device
    outs, rb, eb, nb, ptrs = [], [], [], [], []
    for col in segments:
        if len(col) != nseg:
            raise RuntimeError("gather_from_host: every column has one tensor a segment")
        like = col[0]
        for s, t in enumerate(col):
            if t.device.type != "cpu" or not t.is_contiguous() or (t.numel() and
                                                                  not t.is_pinned()):
                raise RuntimeError("gather_from_host: segments must be contiguous pinned "
                                   "host tensors")
            if t.shape[0] != seg_rows[s + 1] - seg_rows[s] or t.dtype != like.dtype \
                    or t.shape[1:] != like.shape[1:]:
                raise RuntimeError("gather_from_host: a segment's rows or type disagree")
        width = 1
        for d in like.shape[1:]:
            width *= d
        outs.append(torch.empty((n,) + tuple(like.shape[1:]), dtype=like.dtype, device=dev))
        rb.append(max(1, width) * like.element_size())
        eb.append(like.element_size())
        nb.append(null_bits(like.dtype))
        ptrs.extend(t.data_ptr() if t.numel() else None for t in col)
    bad = torch.zeros(1, dtype=torch.int64, device=dev)
    if n == 0:
        return outs, 0
    order = torch.argsort(idx) if sorted_reads else None
    L = lib()
    ws_bytes = L.pf_gather_segments_workspace(ncols, nseg)
    ws = _native.workspace(ws_bytes, dev)
    check(L.pf_gather_segments(arr(ctypes.c_void_p, ptrs), arr(ctypes.c_int64, list(seg_rows)),
                               nseg, base, ncols, arr(ctypes.c_int, rb), arr(ctypes.c_int, eb),
                               arr(ctypes.c_uint64, nb), ptr(idx),
                               ptr(order) if order is not None else None, n,
                               1 if allow_null else 0, NULL, arr(ctypes.c_void_p,
                                                                 [ptr(o) for o in outs]),
                               ptr(bad), ws.data_ptr(), ws_bytes, stream_of(dev)),
          "gather_segments")
    return outs, int(bad.item())
