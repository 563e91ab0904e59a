"""The join core pipe's kernels on sm_100a: the mirror of PageFlow's
``operators/join_core.py`` (same functions, limits and results), calling
``pageflow_b200.tqpkernels``.

- ``unique_hash_pairs``: inner join on a build tuple (1-2 int64 keys) proven
  unique, one partner per probe row, pairs in probe-row order;
- ``semi_anti``: semi or anti join on a hash set of the build keys, with an
  optional per-key min/max summary answering one residual comparison;
- ``expand``: the pairs of the sort/search probe.
"""
from __future__ import annotations

from typing import Optional, Sequence, Tuple

import torch

from . import tqpkernels

MAX_ROWS = (1 << 31) - (1 << 16)
SUMMARY_OPS = {'<>': 1, '<': 2, '<=': 3, '>': 4, '>=': 5}

_host: Optional[torch.Tensor] = None


def _host_buffer() -> torch.Tensor:
    global _host
    if _host is None:
        _host = torch.empty(2, dtype=torch.int64, pin_memory=True)
    return _host


def _empty(device) -> torch.Tensor:
    return torch.empty(0, dtype=torch.int64, device=device)


def expand(sorted_ids: torch.Tensor, start: torch.Tensor,
           length: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    """(build rows, probe rows) of every probe row's run ``sorted_ids[start[i]
    : start[i] + length[i]]``, in probe-row order."""
    return tuple(tqpkernels.join_expand(sorted_ids, start, length, _host_buffer()))


def unique_hash_peak_bytes(n_build: int, n_probe: int) -> int:
    """Scratch of a ``unique_hash_pairs`` call, the figure the join's dispatch
    compares with its limit (reference operators/join_core.py:64-68): the
    table (two 4-byte slots a build row), the 4-byte partner and the two
    8-byte outputs of every probe row.  The library's workspace adds a few
    bytes per 4096 probe rows for block counts."""
    return 2 * n_build * 4 + n_probe * (4 + 8 + 8)


def _validate_keys(build_keys: Sequence[torch.Tensor], probe_keys: Sequence[torch.Tensor]):
    if len(build_keys) not in (1, 2) or len(build_keys) != len(probe_keys):
        raise ValueError("unique_hash_pairs expects one or two aligned build/probe keys")
    device = build_keys[0].device
    for side, keys in (("build", build_keys), ("probe", probe_keys)):
        rows = keys[0].numel()
        for key in keys:
            if not key.is_cuda or key.dtype != torch.int64 or key.dim() != 1:
                raise ValueError(f"{side} keys must be 1-D CUDA int64 tensors; got "
                                 f"device={key.device}, dtype={key.dtype}, "
                                 f"shape={tuple(key.shape)}")
            if not key.is_contiguous():
                raise ValueError(f"{side} keys must be contiguous")
            if key.numel() != rows:
                raise ValueError(f"{side} key lengths disagree")
            if key.device != device:
                raise ValueError("all build/probe keys must be on one CUDA device")
        if rows > MAX_ROWS:
            raise ValueError(f"unique hash core takes at most {MAX_ROWS} rows a side")


def unique_hash_pairs(build_keys: Sequence[torch.Tensor],
                      probe_keys: Sequence[torch.Tensor]) -> Tuple[torch.Tensor, torch.Tensor]:
    """(build rows, probe rows) of an inner join whose build tuple is unique,
    in probe-row order."""
    _validate_keys(build_keys, probe_keys)
    device = build_keys[0].device
    if build_keys[0].numel() == 0 or probe_keys[0].numel() == 0:
        return _empty(device), _empty(device)
    host = _host_buffer()
    build_idx, probe_idx = tqpkernels.join_unique_hash(list(build_keys), list(probe_keys), host)
    n = int(host[0])
    return build_idx[:n], probe_idx[:n]


def semi_anti(build_key: torch.Tensor, probe_key: torch.Tensor, anti: bool,
              summary: Optional[Tuple[torch.Tensor, torch.Tensor, str]] = None
              ) -> Optional[torch.Tensor]:
    """The probe rows, ascending, that have a matching build key (semi) or
    none (anti); with ``summary = (build column, probe column, op)`` a match
    must also pass ``build column op probe column``.  None when a build key
    equals int64 min (the table's empty-slot value)."""
    device = build_key.device
    n_build, n_probe = build_key.numel(), probe_key.numel()
    if n_probe == 0:
        return _empty(device)
    if n_build == 0:
        return torch.arange(n_probe, dtype=torch.int64, device=device) if anti else _empty(device)
    build_val = probe_val = None
    op = 0
    if summary is not None:
        build_val, probe_val, op_name = summary
        op = SUMMARY_OPS[op_name]
    host = _host_buffer()
    out = tqpkernels.join_semi_anti(build_key, probe_key, build_val, probe_val, op, anti, host)
    n, bad = host.tolist()
    if bad:
        return None
    return out[:n]
