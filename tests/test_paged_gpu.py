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


# ---- output-side encoding on the device --------------------------------------------

def _host_pages(values: np.ndarray, rows):
    return [paged.encode_page(values[a:b]) for a, b in zip(rows[:-1], rows[1:])]


def _encode_and_compare(kind):
    """Every page the device encoder writes is byte for byte the host
    encoder's page of the same values (so the same scheme is chosen), and
    the oracle's decoder gives the values back; returns the schemes seen."""
    rng = np.random.default_rng(sum(map(ord, kind)))
    n = 300_000
    if kind == "sorted_runs":        # DELTA / FOR: dates sorted within runs
        v = (8035 + (np.arange(n) % 70_000) * 2557 // 70_000).astype(np.int32)
    elif kind == "random_small":     # FOR
        v = rng.integers(1, 50, n).astype(np.int64)
    elif kind == "random_wide":      # RAW
        v = rng.integers(-(1 << 62), 1 << 62, n).astype(np.int64)
    elif kind == "constant":         # RLE, one run a page
        v = np.full(n, 12345, np.int64)
    elif kind == "few_runs":         # RLE with thousands of runs, and one page over its limit
        v = np.repeat(rng.integers(0, 1 << 40, 6000), 50).astype(np.int64)
    elif kind == "int32_negative":
        v = rng.integers(-(1 << 31), 1 << 31, n).astype(np.int32) // 3
    elif kind == "extremes":
        v = rng.choice(np.array([np.iinfo(np.int64).min, np.iinfo(np.int64).max, 0, -1]),
                       n).astype(np.int64)
    else:
        v = rng.integers(0, 1000, 5001).astype(np.int64)
    n = v.shape[0]
    cuts = sorted({0, n, *rng.integers(0, n, 5).tolist(), min(n, 1024), min(n, 1)})
    if kind == "few_runs":
        cuts = [0, 50 * 4000, n]         # 4000 runs, then 2000
    if kind == "ragged":
        cuts = [0, 0, 1, 1025, 1025, 2048, n]   # empty and one-value pages
    got, offs = paged.encode_pages_device(torch.from_numpy(v).cuda(), cuts)
    got = got.cpu().numpy()
    want = _host_pages(v, cuts)
    schemes = set()
    for p, w in enumerate(want):
        page = got[offs[p]:offs[p + 1]]
        assert page.shape == w.shape and np.array_equal(page, w), f"page {p}"
        schemes.add(int(page[4]))
        dec = oracle.page_decode(page)
        assert np.array_equal(dec.astype(v.dtype), v[cuts[p]:cuts[p + 1]])
    assert offs[-1] == sum(w.shape[0] for w in want)
    return schemes


@pytest.mark.parametrize("kind", ["sorted_runs", "random_small", "random_wide", "constant",
                                  "few_runs", "int32_negative", "extremes", "ragged"])
def test_device_encoder_writes_the_host_encoders_bytes(kind):
    _encode_and_compare(kind)


def test_device_encoder_takes_every_scheme():
    seen = set()
    for kind in ("sorted_runs", "random_small", "random_wide", "constant"):
        seen |= _encode_and_compare(kind)
    assert seen == {0, 1, 2, 3}


def test_partitioned_output_encoded_bucket_by_bucket():
    """A partitioned column (the drop-in partition's padded layout) encoded
    a bucket a page: each bucket's page decodes to its rows."""
    from pageflow_b200 import tqpkernels
    from tests.dropin import padded_starts
    rng = np.random.default_rng(3)
    n, B = 200_000, 16
    key = torch.from_numpy(rng.integers(-(1 << 40), 1 << 40, n)).cuda()
    qty = torch.from_numpy(rng.integers(1, 51, n).astype(np.int64)).cuda()
    host = torch.empty(B + 5, dtype=torch.int64, pin_memory=True)
    outs = tqpkernels.partition_sort([key, qty], [0, 0], 0, None, n, 0, B, False, host)
    counts = host[:B].tolist()
    starts, _ = padded_starts(counts, 8)
    rows = []
    for s0, c in zip(starts, counts):
        rows += [s0, s0 + c]
    # pages over the buckets' rows only (the padding between them is a page
    # of its own, skipped)
    cuts = sorted(set([0] + rows + [outs[1].numel()]))
    pages, offs = paged.encode_pages_device(outs[1], cuts)
    pages = pages.cpu().numpy()
    col = outs[1].cpu().numpy()
    for s0, c in zip(starts, counts):
        p = cuts.index(s0)
        assert cuts[p + 1] == s0 + c
        assert np.array_equal(oracle.page_decode(pages[offs[p]:offs[p + 1]]), col[s0:s0 + c])
