"""The dense slab group-by on sm_100a kernels: ``DenseAggregationSlab`` with
the interface of PageFlow's ``operators/aggregation_slab.py:170-246`` (one
allocation; an occupancy byte and one reduction-identity value segment per
aggregate over a direct-addressed key range; ``add`` folds a tick in,
``finish`` gives the occupied keys ascending with their states), with add and
finish done by pf_slab_add / pf_slab_finish.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import torch

from . import _native as N

ValueSpec = Tuple[torch.dtype, Tuple[int, ...]]

_DT = {torch.int64: 0, torch.float64: 1, torch.int32: 2}
_OP = {"sum": 0, "amax": 1, "amin": 2}


def _align_up(v: int, a: int) -> int:
    return (v + a - 1) // a * a


def _identity(dtype: torch.dtype, op: str):
    if op == "sum":
        return 0
    if dtype.is_floating_point:
        return -torch.inf if op == "amax" else torch.inf
    info = torch.iinfo(dtype)
    return info.min if op == "amax" else info.max


def _layout(capacity: int, specs: Sequence[ValueSpec]):
    cursor, segs = 0, []
    for dtype, trailing in specs:
        es = torch.empty((), dtype=dtype).element_size()
        cursor = _align_up(cursor, max(es, 1))
        width = 1
        for e in trailing:
            width *= int(e)
        size = capacity * width * es
        segs.append((cursor, size, dtype, tuple(trailing)))
        cursor += size
    return segs, _align_up(cursor, 8)


class DenseAggregationSlab:
    """One direct-addressed aggregation workspace over ``key_min..key_max``."""

    def __init__(self, key_min: int, key_max: int, key_dtype: torch.dtype,
                 value_specs: Sequence[ValueSpec], ops: Sequence[str], device):
        if key_max < key_min:
            raise ValueError(f"invalid key range [{key_min}, {key_max}]")
        if len(value_specs) != len(ops):
            raise ValueError("value_specs and ops must have the same length")
        for dtype, _ in value_specs:
            if dtype not in _DT:
                raise ValueError(f"unsupported slab value dtype {dtype}")
        for op in ops:
            if op not in _OP:
                raise ValueError(f"unsupported slab reduction {op!r}")
        self.key_min, self.key_max = int(key_min), int(key_max)
        self.key_dtype = key_dtype
        self.capacity = self.key_max - self.key_min + 1
        self.ops = tuple(ops)
        specs = [(torch.bool, ())] + list(value_specs)
        segs, total = _layout(self.capacity, specs)
        self.storage = torch.empty(total, dtype=torch.uint8, device=device)
        cols = [self.storage[o:o + s].view(dt).view((self.capacity,) + tr)
                for o, s, dt, tr in segs]
        self.occupied = cols[0]
        self.occupied.fill_(False)
        self.values = cols[1:]
        for v, op in zip(self.values, self.ops):
            v.fill_(_identity(v.dtype, op))
        self._err = torch.zeros(1, dtype=torch.int64, device=device)

    @staticmethod
    def required_bytes(capacity: int, value_specs: Sequence[ValueSpec]) -> int:
        return _layout(capacity, [(torch.bool, ())] + list(value_specs))[1]

    @property
    def nbytes(self) -> int:
        return self.storage.numel()

    def add(self, keys: torch.Tensor, values: Sequence[torch.Tensor]) -> None:
        """Fold one tick's rows in (every key must lie in the slab's range)."""
        if keys.dim() != 1:
            raise ValueError(f"slab keys must be 1-D, got {tuple(keys.shape)}")
        if len(values) != len(self.values):
            raise ValueError("tick value count does not match slab value count")
        if keys.numel() == 0:
            return
        if keys.dtype not in (torch.int64, torch.int32):
            keys = keys.to(torch.int64)
        keys = keys.contiguous()
        srcs = []
        for dst, src in zip(self.values, values):
            if src.shape[0] != keys.numel() or src.shape[1:] != dst.shape[1:]:
                raise ValueError(f"tick value shape {tuple(src.shape)} does not match slab "
                                 f"row shape {tuple(dst.shape[1:])}")
            srcs.append(src.to(dst.dtype).contiguous())
        L = N.lib()
        widths = [max(1, v[0].numel()) if v.dim() > 1 else 1 for v in self.values]
        with torch.cuda.device(keys.device):
            rc = L.pf_slab_add(
                keys.data_ptr(), 0 if keys.dtype == torch.int64 else 2, keys.numel(),
                self.key_min, self.capacity, self.occupied.data_ptr(), len(self.values),
                N.arr(N._vp, [v.data_ptr() for v in self.values]),
                N.arr(N._vp, [s.data_ptr() for s in srcs]),
                N.arr(N._int, [_DT[v.dtype] for v in self.values]),
                N.arr(N._int, [_OP[o] for o in self.ops]),
                N.arr(N._int, widths), self._err.data_ptr(), N.stream_of(keys.device))
        N.check(rc, "slab add")

    def out_of_range(self) -> int:
        """Rows ``add`` skipped because their key was outside the range."""
        return int(self._err.item())

    def finish(self):
        """(ascending populated keys, their aggregate states)."""
        dev = self.storage.device
        keys = torch.empty(self.capacity, dtype=torch.int64, device=dev)
        outs = [torch.empty_like(v) for v in self.values]
        host = torch.empty(2, dtype=torch.int64, pin_memory=True)
        widths = [max(1, v[0].numel()) if v.dim() > 1 else 1 for v in self.values]
        L = N.lib()
        with torch.cuda.device(dev):
            ws_bytes = L.pf_slab_finish_workspace(self.capacity)
            ws = N.workspace(ws_bytes, dev)
            rc = L.pf_slab_finish(
                self.occupied.data_ptr(), self.key_min, self.capacity, len(self.values),
                N.arr(N._vp, [v.data_ptr() for v in self.values]),
                N.arr(N._int, [_DT[v.dtype] for v in self.values]),
                N.arr(N._int, widths), keys.data_ptr(),
                N.arr(N._vp, [o.data_ptr() for o in outs]), host.data_ptr(),
                ws.data_ptr(), ws_bytes, N.stream_of(dev))
        N.check(rc, "slab finish")
        n = int(host[0])
        return keys[:n].to(self.key_dtype), [o[:n] for o in outs]
