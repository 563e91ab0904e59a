"""Drop-in for PageFlow's native module ``TQPlib.tqpkernels``: the four
functions of ``operators/kernels/tqpkernels.cu:8-46`` with the same names,
arguments, outputs and errors, backed by the sm_100a kernels of
libpageflow_b200.so through its C ABI.

As in the reference, outputs are allocated by torch on the key's device and
the current stream (so whatever allocator torch has, e.g. a pooled arena,
backs them), sized for the worst case, and narrowed by the caller from
``host_out``, a caller-owned pinned int64 buffer; argument violations raise
RuntimeError; each call waits for the GPU once.  Install it under the
reference's module name with ``pageflow_b200.install_as_tqplib()``.
"""
from __future__ import annotations

from typing import List, Optional

import torch

from . import _native as N

MAXC = 6
MAXCLS = 4
BMAX = 512


def _check_host(host_out: torch.Tensor, need: int, what: str) -> None:
    if not (isinstance(host_out, torch.Tensor) and host_out.device.type == "cpu"
            and host_out.is_pinned() and host_out.dtype == torch.int64
            and host_out.is_contiguous() and host_out.numel() >= need):
        raise RuntimeError(f"{what}: host_out must be pinned int64 with {need} elements")


def _row_bytes(t: torch.Tensor) -> int:
    return t.element_size() * (t.shape[1] if t.dim() == 2 else 1)


def partition_sort(cols: List[torch.Tensor], comp: List[int], key_idx: int,
                   mask: Optional[torch.Tensor], n_valid: int, goff: int, B: int,
                   select_first: bool, host_out: torch.Tensor) -> List[torch.Tensor]:
    """Stable hash partition of a tick into the padded bucket layout
    (reference operators/kernels/partition_sort.cu:601-768).  Returns each
    column's output, then the int64 gidx, each sized n_valid +
    B*(rows_per_unit - 1) rows; host_out[:B] receives the bucket counts,
    host_out[B:B+4] each row-width class's padded total, host_out[B+4] the
    kept rows a mask prologue found (or -1)."""
    ncols = len(cols)
    if not 1 <= ncols <= MAXC:
        raise RuntimeError(f"partition_sort: 1-{MAXC} columns, got {ncols}")
    if len(comp) != ncols:
        raise RuntimeError("partition_sort: one comp flag per column")
    if not (1 <= B <= BMAX and B & (B - 1) == 0):
        raise RuntimeError(f"partition_sort: B must be a power of two in [1, {BMAX}], got {B}")
    if not 0 <= key_idx < ncols:
        raise RuntimeError("partition_sort: key index out of range")
    key = cols[key_idx]
    if key.dtype != torch.int64 or key.dim() != 1:
        raise RuntimeError("partition_sort: int64 1-D key")
    _check_host(host_out, B + MAXCLS + 1, "partition_sort")
    N.require_cuda(key, "partition_sort: the key")
    has_mask = mask is not None
    n_dom = mask.shape[0] if has_mask else key.shape[0]
    if has_mask:
        if not (mask.is_cuda and mask.dim() == 1 and mask.is_contiguous()
                and mask.element_size() == 1):
            raise RuntimeError("partition_sort: 1-D contiguous 1-byte mask")
    if not 0 <= n_valid <= n_dom:
        raise RuntimeError(f"partition_sort: n_valid {n_valid} outside [0, {n_dom}]")
    if n_dom >= 1 << 31:
        raise RuntimeError("partition_sort: a tick must hold fewer than 2^31 rows")
    widths: List[int] = []
    outs = []
    for c, t in enumerate(cols):
        if not (t.is_cuda and t.device == key.device and t.is_contiguous()
                and t.dim() in (1, 2)):
            raise RuntimeError(f"partition_sort: column {c} must be a contiguous 1-D or "
                               f"2-D tensor on the key's device")
        if comp[c] and not has_mask:
            raise RuntimeError("partition_sort: a compacted column needs the mask")
        want = n_valid if comp[c] else n_dom
        if t.shape[0] != want:
            raise RuntimeError(f"partition_sort: column {c} has {t.shape[0]} rows, "
                               f"expected {want}")
        rb = _row_bytes(t)
        if rb < 1:
            raise RuntimeError("partition_sort: empty rows")
        if rb not in widths:
            widths.append(rb)
        shape = list(t.shape)
        shape[0] = n_valid + B * (N.lib().pf_rows_per_unit(rb) - 1)
        outs.append(torch.empty(shape, dtype=t.dtype, device=t.device))
    if 8 not in widths:
        widths.append(8)
    if len(widths) > MAXCLS:
        raise RuntimeError(f"partition_sort: more than {MAXCLS} row widths")
    gout = torch.empty(n_valid + B * (N.lib().pf_rows_per_unit(8) - 1),
                       dtype=torch.int64, device=key.device)
    L = N.lib()
    with torch.cuda.device(key.device):
        ws_bytes = L.pf_partition_sort_workspace(n_dom, n_valid, B, int(has_mask),
                                                 int(bool(select_first)))
        ws = N.workspace(ws_bytes, key.device)
        rc = L.pf_partition_sort(
            N.arr(N._vp, [t.data_ptr() for t in cols]),
            N.arr(N._vp, [o.data_ptr() for o in outs]),
            N.arr(N._int, [_row_bytes(t) for t in cols]),
            N.arr(N._int, [int(bool(x)) for x in comp]),
            ncols, key_idx, N.ptr(mask), n_dom, n_valid, goff, B,
            int(bool(select_first)), gout.data_ptr(), host_out.data_ptr(),
            ws.data_ptr(), ws_bytes, N.stream_of(key.device))
    N.check(rc, "partition_sort")
    return outs + [gout]


def _check_keys(keys, what, like):
    for t in keys:
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.device == like.device
                and t.dtype == torch.int64 and t.dim() == 1 and t.is_contiguous()):
            raise RuntimeError(f"join_core: {what} must be a contiguous 1-D int64 tensor "
                               f"on the key's device")


def join_unique_hash(build_keys: List[torch.Tensor], probe_keys: List[torch.Tensor],
                     host_out: torch.Tensor) -> List[torch.Tensor]:
    """Inner join on a unique build tuple (reference
    operators/kernels/join_core.cu:297-351): (build rows, probe rows) sized
    for every probe row; the first host_out[0] are the matches, in probe-row
    order."""
    if len(build_keys) not in (1, 2) or len(build_keys) != len(probe_keys):
        raise RuntimeError("join_core: one or two aligned build/probe keys")
    key = build_keys[0]
    _check_keys(build_keys, "a build key", key)
    _check_keys(probe_keys, "a probe key", key)
    nb, np_ = key.numel(), probe_keys[0].numel()
    if any(t.numel() != nb for t in build_keys):
        raise RuntimeError("join_core: build keys differ in length")
    if any(t.numel() != np_ for t in probe_keys):
        raise RuntimeError("join_core: probe keys differ in length")
    _check_host(host_out, 2, "join_core")
    if nb == 0 or np_ == 0:
        raise RuntimeError("join_core: unique hash needs rows on both sides")
    two = len(build_keys) == 2
    build_idx = torch.empty(np_, dtype=torch.int64, device=key.device)
    probe_idx = torch.empty(np_, dtype=torch.int64, device=key.device)
    L = N.lib()
    with torch.cuda.device(key.device):
        ws_bytes = L.pf_join_unique_hash_workspace(nb, np_)
        ws = N.workspace(ws_bytes, key.device)
        rc = L.pf_join_unique_hash(
            build_keys[0].data_ptr(), build_keys[1].data_ptr() if two else None, nb,
            probe_keys[0].data_ptr(), probe_keys[1].data_ptr() if two else None, np_,
            2 if two else 1, build_idx.data_ptr(), probe_idx.data_ptr(),
            host_out.data_ptr(), ws.data_ptr(), ws_bytes, N.stream_of(key.device))
    N.check(rc, "join_unique_hash")
    return [build_idx, probe_idx]


def join_semi_anti(build_key: torch.Tensor, probe_key: torch.Tensor,
                   build_val: Optional[torch.Tensor], probe_val: Optional[torch.Tensor],
                   op: int, anti: bool, host_out: torch.Tensor) -> torch.Tensor:
    """Semi / anti join on a hash set of the build keys with an optional
    min/max summary for one residual comparison (reference
    operators/kernels/join_core.cu:353-400): the kept probe rows, the first
    host_out[0], ascending; host_out[1] = 1 when a build key equals INT64_MIN."""
    _check_keys([build_key], "the build key", build_key)
    _check_keys([probe_key], "the probe key", build_key)
    _check_host(host_out, 2, "join_core")
    nb, np_ = build_key.numel(), probe_key.numel()
    if nb == 0 or np_ == 0:
        raise RuntimeError("join_core: semi/anti needs rows on both sides")
    if not 0 <= op <= 5:
        raise RuntimeError(f"join_core: unknown residual operator {op}")
    if op != 0:
        if build_val is None or probe_val is None:
            raise RuntimeError("join_core: a residual needs both value columns")
        _check_keys([build_val], "the build value", build_key)
        _check_keys([probe_val], "the probe value", build_key)
        if build_val.numel() != nb or probe_val.numel() != np_:
            raise RuntimeError("join_core: a value column differs in length from its key")
    out = torch.empty(np_, dtype=torch.int64, device=build_key.device)
    L = N.lib()
    with torch.cuda.device(build_key.device):
        ws_bytes = L.pf_join_semi_anti_workspace(nb, np_, op)
        ws = N.workspace(ws_bytes, build_key.device)
        rc = L.pf_join_semi_anti(
            build_key.data_ptr(), nb, probe_key.data_ptr(), np_,
            N.ptr(build_val) if op else None, N.ptr(probe_val) if op else None, op,
            int(bool(anti)), out.data_ptr(), host_out.data_ptr(), ws.data_ptr(),
            ws_bytes, N.stream_of(build_key.device))
    N.check(rc, "join_semi_anti")
    return out


def join_expand(sorted_ids: torch.Tensor, start: torch.Tensor, len: torch.Tensor,
                host_out: torch.Tensor) -> List[torch.Tensor]:
    """The sort/search probe's pairs (reference
    operators/kernels/join_core.cu:259-295): waits for the pair count
    (host_out[0]), then returns (build rows, probe rows) of every pair in
    probe-row order and run order."""
    length = len  # the reference's argument name
    _check_keys([sorted_ids], "sorted_ids", sorted_ids)
    _check_keys([start], "start", sorted_ids)
    _check_keys([length], "len", sorted_ids)
    _check_host(host_out, 2, "join_core")
    if start.numel() != length.numel():
        raise RuntimeError("join_core: start and len differ in length")
    m = length.numel()
    dev = sorted_ids.device
    if m == 0:
        e = torch.empty(0, dtype=torch.int64, device=dev)
        return [e, e.clone()]
    L = N.lib()
    with torch.cuda.device(dev):
        ws_bytes = L.pf_join_expand_workspace(m)
        ws = N.workspace(ws_bytes, dev)
        st = N.stream_of(dev)
        N.check(L.pf_join_expand_prepare(length.data_ptr(), m, host_out.data_ptr(),
                                         ws.data_ptr(), ws_bytes, st), "join_expand")
        n_pairs = int(host_out[0])
        cs = torch.empty(n_pairs, dtype=torch.int64, device=dev)
        cr = torch.empty(n_pairs, dtype=torch.int64, device=dev)
        if n_pairs > 0:
            N.check(L.pf_join_expand(sorted_ids.data_ptr(), start.data_ptr(),
                                     length.data_ptr(), m, n_pairs, cs.data_ptr(),
                                     cr.data_ptr(), ws.data_ptr(), ws_bytes, st),
                    "join_expand")
    return [cs, cr]
