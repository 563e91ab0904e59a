"""pf_paged_scan on the GPU against the oracle: decode of every PFC1 scheme,
the range filter, the per-batch radix partition (bucket counts bit-exact,
each bucket's rows the same multiset), capacity skips and bad pages."""
import numpy as np
import pytest
import torch

import oracle
from pageflow_b200 import paged

pytestmark = pytest.mark.gpu


def _rows(cols, names, lo, hi):
    """The rows [lo, hi) of the named columns, sorted (a multiset)."""
    m = np.stack([cols[n][lo:hi].astype(np.int64) for n in names])
    if m.shape[1] == 0:
        return m
    return m[:, np.lexsort(m[::-1])]


def _check(parts: paged.PagedPartitions, want, names):
    offs = parts.bucket_offsets.cpu().numpy()
    got = {n: parts.columns[n].cpu().numpy() for n in names}
    B = parts.B
    assert offs.shape[0] == len(want)
    base = 0
    for k, w in enumerate(want):
        counts = w["counts"]
        assert offs[k, B] == counts.sum(), k
        starts = base + np.concatenate([[0], np.cumsum(counts)[:-1]])
        assert np.array_equal(offs[k, :B], starts), k
        wstart = np.concatenate([[0], np.cumsum(counts)])
        for b in np.nonzero(counts)[0]:
            g = _rows(got, names, offs[k, b], offs[k, b] + counts[b])
            e = _rows(w, names, wstart[b], wstart[b + 1])
            assert np.array_equal(g, e), (k, b)
        base += int(counts.sum())
    s = parts.read_stats()
    assert s["rows"] == base and s["batches_skipped"] == 0 and s["bad_pages"] == 0


@pytest.mark.parametrize("B,gpb,lo,hi", [(256, 2, 9000, 9384), (16, 3, 8035, 10592),
                                        (4096, 1, 8500, 8501), (1, 4, 8035, 9000)])
def test_generated_table_scan(B, gpb, lo, hi):
    spec = paged.PagedSpec(2, 150_000, 40_000, 0.8, 16384, lo, hi)
    t = paged.PagedTable.generate(spec, threads=4)
    edges, thr = t.zipf
    cols = oracle.gen_paged(spec.seed, spec.n_build, 0, spec.n_rows, edges, thr)
    want = oracle.paged_scan(cols, spec.n_rows, spec.rows_per_page, gpb, "date", lo, hi, "fk", B)
    parts = paged.paged_scan(t, "date", lo, hi, "fk", B=B, groups_per_batch=gpb)
    torch.cuda.synchronize()
    _check(parts, want, ["fk", "price", "quantity", "flag", "status"])


def _edge_columns(n, seed=5):
    rng = np.random.default_rng(seed)
    I64, I32 = np.iinfo(np.int64), np.iinfo(np.int32)
    return {
        "key": rng.integers(I64.min, I64.max, n, dtype=np.int64),                  # RAW
        "filter": np.repeat(np.arange(n // 700 + 1), 700)[:n].astype(np.int32),   # RLE
        "sorted": np.cumsum(rng.integers(0, 1 << 20, n)).astype(np.int64),         # DELTA
        "small": rng.integers(-3, 3, n).astype(np.int32),                          # FOR
        "extremes": np.tile(np.array([I64.min, I64.max], np.int64), n // 2 + 1)[:n],
        "runs64": np.repeat(rng.integers(I64.min, I64.max, n // 37 + 1, dtype=np.int64),
                            37)[:n],
        "i32wide": rng.integers(I32.min, I32.max, n).astype(np.int32),
    }


@pytest.mark.parametrize("n", [16384 * 3 + 1000, 16384, 5])
def test_every_scheme_decodes(n):
    cols = _edge_columns(n)
    t = paged.PagedTable.from_columns(cols, rows_per_page=16384)
    parts = paged.paged_scan(t, "filter", -(1 << 62), 1 << 62, "key", B=64, groups_per_batch=2)
    torch.cuda.synchronize()
    names = [k for k in cols if k != "filter"]
    want = oracle.paged_scan(cols, n, 16384, 2, "filter", -(1 << 62), 1 << 62, "key", 64)
    _check(parts, want, names)


def test_empty_filter_and_capacity_skip():
    spec = paged.PagedSpec(2, 100_000, 10_000, 0.8, 16384, 0, 0)
    t = paged.PagedTable.generate(spec, threads=2)
    parts = paged.paged_scan(t, "date", 9000, 9000, "fk", B=32, groups_per_batch=2)
    torch.cuda.synchronize()
    assert parts.read_stats()["rows"] == 0
    assert np.all(parts.bucket_offsets.cpu().numpy()[:, 32] == 0)
    # every date passes; room for two batches of 2 x 16384 rows, not three
    parts = paged.paged_scan(t, "date", 0, 1 << 20, "fk", B=32, groups_per_batch=2,
                             capacity_rows=2 * 32768 + 10)
    torch.cuda.synchronize()
    s = parts.read_stats()
    offs = parts.bucket_offsets.cpu().numpy()
    assert s["batches_skipped"] == 2 and s["rows"] == 2 * 32768
    assert np.all(offs[2:, :32] == -1) and np.all(offs[:2, :32] >= 0)
    assert np.array_equal(offs[:, 32], [32768, 32768, 32768, 100_000 - 3 * 32768])


def test_bad_page_is_counted_and_dropped():
    cols = _edge_columns(16384 * 3)
    t = paged.PagedTable.from_columns(cols, rows_per_page=16384)
    pages = t.pages.clone().pin_memory()
    pages[int(t.directory[len(cols) * 1 + 2])] ^= 0xFF     # group 1, column 2: magic
    bad = paged.PagedTable(pages, t.directory, t.n_rows, t.rows_per_page, t.names, t.esizes)
    parts = paged.paged_scan(bad, "filter", -(1 << 62), 1 << 62, "key", B=8, groups_per_batch=1)
    torch.cuda.synchronize()
    s = parts.read_stats()
    assert s["bad_pages"] == 4                              # the group's 4 CTAs
    assert s["rows"] == 2 * 16384
    assert parts.bucket_offsets.cpu().numpy()[1, 8] == 0
