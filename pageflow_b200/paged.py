"""Compressed column pages decoded on arrival, fused with a range filter and
the first radix-partition pass.

The reference stages compressed records per tick: one H2D pack of the
selected records (IO/transfer/in_stage.py:406), one nvCOMP CASCADED
decompress per codec group (IO/transfer/tick_layout.py:141-190,
compression/nvcomp_manager.cu:679), the filter mask (operators/filter.py:
10-16), mask compaction (IO/transfer/pre_comp_stage.py:54-73,
utility/tensor_utils.py:12-39) and then partition_sort, each an HBM round
trip.  Here the pages travel compressed over the link into a three-deep
staging ring and one pipeline per batch of row groups decodes them in
registers, filters and scatters the surviving rows by radix bucket
(pf_paged_scan in include/pageflow_b200.h).

Pages use the PFC1 format of pageflow_b200/csrc/codec.h (FOR / DELTA / RLE /
RAW over 1024-value mini-blocks), written by pf_page_encode.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from ._native import arr, check, lib, ptr, stream_of

PAGED_COLUMNS = ("fk", "date", "price", "quantity", "flag", "status")
PAGED_ESIZES = (8, 4, 8, 8, 4, 4)


@dataclass(frozen=True)
class PagedSpec:
    """The paged workload: n_rows probe rows of PAGED_COLUMNS, fk Zipf(s)
    over n_build keys, row groups of rows_per_page rows (1 MiB pages of the
    int64 columns at 131072 rows), kept rows lo <= date < hi."""
    seed: int
    n_rows: int
    n_build: int
    zipf_s: float
    rows_per_page: int
    date_lo: int
    date_hi: int


# 2.4B rows; dates span [8035, 10591]: [9000, 9384) keeps 384 of 2557 days (15.0%)
PAGED = PagedSpec(2, 2_400_000_000, 200_000_000, 0.8, 131072, 9000, 9384)


def scaled(spec: PagedSpec, factor: float) -> PagedSpec:
    return PagedSpec(spec.seed, max(1, int(spec.n_rows / factor)),
                     max(1, int(spec.n_build / factor)), spec.zipf_s, spec.rows_per_page,
                     spec.date_lo, spec.date_hi)


def encode_page(values: np.ndarray) -> np.ndarray:
    """One PFC1 page of an int32 or int64 column (uint8 array)."""
    v = np.ascontiguousarray(values)
    if v.dtype not in (np.int32, np.int64):
        raise TypeError("encode_page: int32 or int64 values")
    cap = 64 + 16 * 4 + v.shape[0] * 8 + (v.shape[0] // 1024 + 2) * 64 + 64
    out = np.empty(cap, np.uint8)
    n = lib().pf_page_encode(v.ctypes.data, v.dtype.itemsize, v.shape[0], out.ctypes.data, cap)
    if n < 0:
        check(int(n), "encode_page")
    return out[:n]


def page_capacity(rows: int, esize: int) -> int:
    """Bytes a PFC1 page of `rows` values takes at most (RAW, or a stream of
    64-bit fields, whichever the encoder picks is never larger than both)."""
    blocks = (rows + 1023) // 1024
    return 64 + 16 + 32 * blocks + 8 * rows + 16 + 64


def encode_pages_device(values: torch.Tensor, page_rows) -> tuple:
    """Output-side encoding on the GPU (pf_encode_pages): ``values`` (a 1-D
    int32 / int64 CUDA tensor) cut at ``page_rows`` (ascending, from 0 to
    its length) into PFC1 pages, the same bytes pf_page_encode writes.
    Returns (the pages, a uint8 CUDA tensor, and each page's byte offset
    with the total)."""
    _native.require_cuda(values, "encode_pages values")
    if values.dtype not in (torch.int32, torch.int64) or values.dim() != 1:
        raise TypeError("encode_pages: a 1-D int32 or int64 tensor")
    values = values.contiguous()
    rows = [int(r) for r in page_rows]
    npages = len(rows) - 1
    if npages < 1 or rows[0] != 0 or rows[-1] != values.numel():
        raise ValueError("encode_pages: page rows run from 0 to the column's length")
    es = values.element_size()
    cap = sum(page_capacity(b - a, es) for a, b in zip(rows[:-1], rows[1:]))
    out = torch.empty(cap, dtype=torch.uint8, device=values.device)
    offs = (ctypes.c_int64 * (npages + 1))()
    L = lib()
    ws_bytes = L.pf_encode_pages_workspace(npages)
    ws = _native.workspace(ws_bytes, values.device)
    check(L.pf_encode_pages(ptr(values), es, arr(ctypes.c_int64, rows), npages, ptr(out), cap,
                            offs, ptr(ws), ws_bytes, stream_of(values.device)), "encode_pages")
    offsets = list(offs)
    return out[:offsets[-1]], offsets


class PagedTable:
    """A table as PFC1 pages in pinned host memory: row group g holds every
    column's page of rows [g * rows_per_page, (g + 1) * rows_per_page), in
    column order; directory[g * ncols + c] is that page's byte offset."""

    def __init__(self, pages: torch.Tensor, directory: np.ndarray, n_rows: int,
                 rows_per_page: int, names, esizes):
        self.pages = pages
        self.directory = np.ascontiguousarray(directory, dtype=np.int64)
        self.n_rows = int(n_rows)
        self.rows_per_page = int(rows_per_page)
        self.names = tuple(names)
        self.esizes = tuple(int(e) for e in esizes)
        self.n_groups = (self.n_rows + self.rows_per_page - 1) // self.rows_per_page
        if self.directory.shape[0] != self.n_groups * len(self.names):
            raise ValueError("PagedTable: directory does not match the row groups")

    @property
    def total_bytes(self) -> int:
        return int(self.pages.numel())

    @property
    def raw_bytes(self) -> int:
        """The table's uncompressed bytes."""
        return self.n_rows * sum(self.esizes)

    @classmethod
    def from_columns(cls, columns: dict, rows_per_page: int, pin: bool = True) -> "PagedTable":
        """Encodes numpy int32 / int64 columns page by page."""
        names = list(columns)
        cols = [np.ascontiguousarray(columns[n]) for n in names]
        n_rows = cols[0].shape[0]
        if any(c.shape[0] != n_rows for c in cols):
            raise ValueError("from_columns: columns of different lengths")
        blobs, directory, off = [], [], 0
        for r0 in range(0, max(n_rows, 1), rows_per_page):
            for c in cols:
                p = encode_page(c[r0:r0 + rows_per_page])
                directory.append(off)
                blobs.append(p)
                off += p.shape[0]
        flat = np.concatenate(blobs) if blobs else np.zeros(0, np.uint8)
        pages = torch.from_numpy(flat)
        if pin:
            pages = pages.pin_memory()
        return cls(pages, np.array(directory, np.int64), n_rows, rows_per_page, names,
                   [c.dtype.itemsize for c in cols])

    @classmethod
    def generate(cls, spec: PagedSpec, threads: int | None = None,
                 pin: bool = True) -> "PagedTable":
        """The paged workload's table, generated and encoded on host threads
        into (pinned) pages."""
        from .datagen import zipf_table
        edges, thr = zipf_table(spec.n_build, spec.zipf_s)
        edges = np.ascontiguousarray(edges, np.int64)
        thr = np.ascontiguousarray(thr, np.uint64)
        threads = threads or max(1, len(os.sched_getaffinity(0)))
        handle = ctypes.c_void_p()
        total = ctypes.c_int64()
        check(lib().pf_paged_generate(spec.seed, spec.n_rows, spec.rows_per_page, spec.n_build,
                                      edges.ctypes.data, thr.ctypes.data, thr.shape[0], threads,
                                      ctypes.byref(handle), ctypes.byref(total)),
              "paged_generate")
        n_groups = (spec.n_rows + spec.rows_per_page - 1) // spec.rows_per_page
        pages = torch.empty(max(total.value, 1), dtype=torch.uint8, pin_memory=pin)[:total.value]
        directory = np.empty(n_groups * len(PAGED_COLUMNS), np.int64)
        ng = ctypes.c_int64()
        check(lib().pf_paged_fetch(handle, pages.data_ptr(), directory.ctypes.data,
                                   ctypes.byref(ng)), "paged_fetch")
        t = cls(pages, directory, spec.n_rows, spec.rows_per_page, PAGED_COLUMNS, PAGED_ESIZES)
        t.zipf = (edges, thr)
        return t


@dataclass
class PagedPartitions:
    """The scan's output: the kept rows of every non-filter column (dict name
    -> device tensor of capacity rows, rows [0, rows) written), grouped per
    batch and, inside a batch, per bucket: bucket_offsets[k, b] is bucket b's
    first row in batch k (-1: batch skipped, no room), bucket_offsets[k, B]
    the batch's rows."""
    columns: dict
    bucket_offsets: torch.Tensor
    stats: torch.Tensor
    B: int
    groups_per_batch: int

    def read_stats(self) -> dict:
        s = self.stats.cpu().tolist()
        return {"rows": s[0], "batches_skipped": s[1], "bad_pages": s[2]}


class PagedScan:
    """A reusable scan plan over one PagedTable: the workspace (staging ring
    of three batches, per-CTA histograms) and the outputs are allocated once;
    run() queues one decode -> filter -> partition pass over the whole table
    on the current stream."""

    def __init__(self, table: PagedTable, filter_col: str, lo: int, hi: int, key_col: str,
                 B: int = 256, groups_per_batch: int = 64, capacity_rows: int | None = None,
                 keep=None, device=None):
        self.table = table
        dev = torch.device("cuda") if device is None else torch.device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        names = table.names
        self.fc = names.index(filter_col)
        self.kc = names.index(key_col)
        self.lo, self.hi = int(lo), int(hi)
        self.B = int(B)
        self.gpb = int(max(1, min(groups_per_batch, table.n_groups)))
        self.n_batches = (table.n_groups + self.gpb - 1) // self.gpb
        self.capacity = int(table.n_rows if capacity_rows is None else capacity_rows)
        keep = set(n for n in names if n != filter_col) if keep is None else set(keep) | {key_col}
        self.columns = {}
        for c, n in enumerate(names):
            if n in keep and c != self.fc:
                dt = torch.int64 if table.esizes[c] == 8 else torch.int32
                self.columns[n] = torch.empty(max(self.capacity, 1), dtype=dt, device=self.device)
        self.bucket_offsets = torch.empty((self.n_batches, self.B + 1), dtype=torch.int64,
                                          device=self.device)
        self.stats = torch.zeros(4, dtype=torch.int64, device=self.device)
        ws = lib().pf_paged_scan_workspace(table.directory.ctypes.data, table.n_groups,
                                           len(names), table.total_bytes, self.gpb, self.B)
        self.ws = _native.workspace(ws, self.device)
        self._outs = (ctypes.c_void_p * len(names))(
            *[ptr(self.columns[n]) if n in self.columns else None for n in names])
        self._es = arr(ctypes.c_int, table.esizes)

    def run(self) -> PagedPartitions:
        t = self.table
        with torch.cuda.device(self.device):
            check(lib().pf_paged_scan(
                t.pages.data_ptr(), t.directory.ctypes.data, t.n_groups, len(t.names),
                ctypes.addressof(self._es), t.total_bytes, t.n_rows, t.rows_per_page, self.fc,
                self.lo, self.hi, self.kc, self.B, self.gpb, ctypes.addressof(self._outs),
                self.capacity, ptr(self.bucket_offsets), ptr(self.stats), ptr(self.ws),
                self.ws.numel(), stream_of(self.device)), "paged_scan")
        return PagedPartitions(self.columns, self.bucket_offsets, self.stats, self.B, self.gpb)


def paged_scan(table: PagedTable, filter_col: str, lo: int, hi: int, key_col: str,
               B: int = 256, groups_per_batch: int = 64, capacity_rows: int | None = None,
               device=None) -> PagedPartitions:
    """One decode -> filter -> partition pass (allocates a PagedScan)."""
    return PagedScan(table, filter_col, lo, hi, key_col, B, groups_per_batch, capacity_rows,
                     device=device).run()
