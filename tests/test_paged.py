"""PFC1 pages on the CPU: the product's encoder (pf_page_encode, the paged
workload's page builder) against the oracle's independent decoder and
generator twin.  No GPU."""
import numpy as np
import pytest

import oracle
from pageflow_b200 import paged

I64 = np.iinfo(np.int64)
I32 = np.iinfo(np.int32)


def _cases():
    rng = np.random.default_rng(7)
    return {
        "empty": np.zeros(0, np.int64),
        "one": np.array([5], np.int64),
        "one_block_edge": np.arange(1024, dtype=np.int64) * 3,
        "block_plus_one": np.arange(1025, dtype=np.int64) - 512,
        "constant": np.full(5000, -7, np.int64),
        "runs": np.repeat(rng.integers(-100, 100, 300), rng.integers(1, 50, 300)).astype(np.int64),
        "sorted": np.sort(rng.integers(0, 1 << 40, 10000)).astype(np.int64),
        "full_range": rng.integers(I64.min, I64.max, 3000, dtype=np.int64),
        "extremes": np.array([I64.min, I64.max] * 1500, np.int64),
        "int32_negative": rng.integers(I32.min, I32.max, 4097).astype(np.int32),
        "int32_small": rng.integers(0, 3, 2049).astype(np.int32),
        "int32_extremes": np.array([I32.min, I32.max, 0, -1] * 700, np.int32),
        "too_many_runs": np.repeat(np.arange(5000), 2).astype(np.int64),
        "max_runs": np.repeat(np.arange(4096), 3).astype(np.int64),
    }


@pytest.mark.parametrize("name", list(_cases()))
def test_encode_round_trip(name):
    v = _cases()[name]
    page = paged.encode_page(v)
    assert page.shape[0] % 16 == 0
    assert np.array_equal(oracle.page_decode(page), v.astype(np.int64))


def test_encoder_picks_each_scheme():
    c = _cases()
    scheme = {k: int(paged.encode_page(v)[4]) for k, v in c.items() if v.shape[0] > 1}
    assert scheme["runs"] == 3 and scheme["constant"] == 3 and scheme["max_runs"] == 3
    assert scheme["too_many_runs"] != 3          # more than 4096 runs: no RLE
    assert scheme["int32_small"] == 1            # FOR: 2 bits a value
    assert scheme["sorted"] == 2                 # DELTA
    assert scheme["full_range"] == 0             # RAW


def test_encode_rejects_bad_input():
    with pytest.raises(TypeError):
        paged.encode_page(np.zeros(4, np.float64))


def test_oracle_decoder_rejects_malformed_pages():
    page = paged.encode_page(np.arange(3000, dtype=np.int64) * 7).copy()
    bad = page.copy()
    bad[0] ^= 0xFF                                # magic
    with pytest.raises(ValueError):
        oracle.page_decode(bad)
    with pytest.raises(ValueError):
        oracle.page_decode(page[:page.shape[0] // 2])  # truncated
    bad = page.copy()
    bad[5] = 3                                    # element size
    with pytest.raises(ValueError):
        oracle.page_decode(bad)


def _small_spec(n_rows=70_000, rpp=16384):
    return paged.PagedSpec(2, n_rows, 20_000, 0.8, rpp, 9000, 9384)


def test_generated_pages_match_the_generator_twin():
    spec = _small_spec()
    t = paged.PagedTable.generate(spec, threads=3, pin=False)
    assert t.n_groups == 5 and t.directory.shape[0] == 5 * 6
    assert np.all(np.diff(t.directory) > 0)
    edges, thr = t.zipf
    want = oracle.gen_paged(spec.seed, spec.n_build, 0, spec.n_rows, edges, thr)
    pages = t.pages.numpy()
    ends = list(t.directory[1:]) + [t.total_bytes]
    for g in range(t.n_groups):
        r0, r1 = g * spec.rows_per_page, min(spec.n_rows, (g + 1) * spec.rows_per_page)
        for c, name in enumerate(paged.PAGED_COLUMNS):
            k = g * 6 + c
            got = oracle.page_decode(pages[t.directory[k]:ends[k]])
            assert np.array_equal(got, want[name][r0:r1]), (g, name)
    # the workload's shape: dates sorted in 2^20-row runs over [8035, 10591]
    assert want["date"].min() == 8035 and np.all(np.diff(want["date"]) >= 0)
    assert want["fk"].min() >= 1 and want["fk"].max() <= spec.n_build
    assert set(np.unique(want["flag"])) <= {0, 1, 2}
    assert t.total_bytes < t.raw_bytes / 2        # compresses


def test_generated_columns_use_the_cascade():
    spec = _small_spec(n_rows=16384 * 2)
    t = paged.PagedTable.generate(spec, threads=2, pin=False)
    pages = t.pages.numpy()
    schemes = [int(pages[t.directory[c] + 4]) for c in range(6)]
    assert schemes[1] == 3                        # date: RLE
    assert schemes[4] == 1 and schemes[5] == 1    # flag, status: FOR (bit packing)


def test_oracle_scan_counts():
    spec = _small_spec()
    edges, thr = paged.PagedTable.generate(spec, threads=2, pin=False).zipf
    cols = oracle.gen_paged(spec.seed, spec.n_build, 0, spec.n_rows, edges, thr)
    out = oracle.paged_scan(cols, spec.n_rows, spec.rows_per_page, 2, "date", 8100, 8200, "fk", 16)
    assert len(out) == 3
    kept = (cols["date"] >= 8100) & (cols["date"] < 8200)
    assert sum(int(b["counts"].sum()) for b in out) == int(kept.sum())
    for b in out:
        assert np.all(np.diff(oracle.bucket(b["fk"], 16)) >= 0)
