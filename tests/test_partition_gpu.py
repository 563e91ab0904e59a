"""The drop-in partition kernel (``tqpkernels.partition_sort``, called as the
reference's operators/partition_sort.py calls it) against the oracle's stable
partition, on the cases of the reference's
tests/operators/test_partition_sort.py: tick sizes around the sub-tile, every
bucket count, six columns of four widths, every row width, all rows in one
bucket, a global offset near 6e9, masks from none to all kept in both
prologues and both raw-column modes, mixed raw and compacted columns, offset
views, counts the mask contradicts (flagged through host_out, the GPU still
usable), a tick past a thousand sub-tiles.  Every output's bucket rows and
counts must equal the oracle's bit for bit; padding rows are not compared."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from tests.dropin import padded_starts, partition, row_bytes

pytestmark = pytest.mark.gpu


def _gen(seed):
    return torch.Generator(device="cpu").manual_seed(seed)


def _keys(n, seed, skew=False):
    if skew:
        return torch.full((n,), 7, dtype=torch.int64, device="cuda")
    return torch.randint(-(1 << 40), 1 << 40, (n,), dtype=torch.int64, generator=_gen(seed)).cuda()


def _column(n, kind, seed):
    g = _gen(seed)
    if kind == "i64":
        return torch.randint(-(1 << 62), 1 << 62, (n,), dtype=torch.int64, generator=g).cuda()
    if kind == "i32":
        return torch.randint(-(1 << 30), 1 << 30, (n,), dtype=torch.int32, generator=g).cuda()
    if kind == "i16":
        return torch.randint(-(1 << 14), 1 << 14, (n,), dtype=torch.int16, generator=g).cuda()
    if kind == "i8":
        return torch.randint(-128, 128, (n,), dtype=torch.int8, generator=g).cuda()
    if kind == "s25":
        return torch.randint(0, 256, (n, 25), dtype=torch.uint8, generator=g).cuda()
    if kind.startswith("u8x"):
        return torch.randint(0, 256, (n, int(kind[3:])), dtype=torch.uint8, generator=g).cuda()
    if kind == "i64x2":
        return torch.randint(-(1 << 62), 1 << 62, (n, 2), dtype=torch.int64, generator=g).cuda()
    if kind == "i64x5":
        return torch.randint(-(1 << 62), 1 << 62, (n, 5), dtype=torch.int64, generator=g).cuda()
    raise ValueError(kind)


def _table(n, kinds, seed, skew=False, key_pos=0):
    cols = [_column(n, k, seed + 1 + c) for c, k in enumerate(kinds)]
    cols.insert(key_pos, _keys(n, seed, skew))
    return cols


def _mask(n, keep, seed):
    if keep <= 0:
        return torch.zeros(n, dtype=torch.bool, device="cuda")
    if keep >= 1:
        return torch.ones(n, dtype=torch.bool, device="cuda")
    return (torch.rand(n, generator=_gen(seed)) < keep).cuda()


def _check(cols, key_pos, mask, goff, B, compact=None, count=False, select_first=False):
    """The kernel on ``cols`` (raw, or compacted by ``mask`` where
    ``compact`` says so; every column when None), with the mask's kept rows
    when ``count``, in the prologue ``select_first`` picks, against the
    oracle."""
    if mask is None:
        given = list(cols)
    else:
        compact = compact if compact is not None else [True] * len(cols)
        given = [c[mask] if k else c for c, k in zip(cols, compact)]
    n_valid = int(mask.sum()) if mask is not None else None
    call = partition(given, key_pos, mask, goff, B, n_valid=n_valid, select_first=select_first)
    got = call.outputs
    np_cols = [c.cpu().numpy() for c in cols]
    np_mask = mask.cpu().numpy() if mask is not None else None
    counts, outs = oracle.partition(np_cols, key_pos, np_mask, goff, B)
    kept = int(counts.sum())
    assert sum(call.counts) == kept
    assert call.found in (-1, kept)
    assert len(got) == len(outs)
    for g, want in zip(got, outs):
        assert g.counts == counts.tolist()
        t = g.tensor
        starts, total = oracle.padded_layout(counts, row_bytes(t))
        assert padded_starts(g.counts, row_bytes(t)) == (starts, total)
        assert t.shape[0] == total
        host = t.cpu().numpy()
        for b, (s, c) in enumerate(zip(starts, counts)):
            assert np.array_equal(host[s:s + c], want[b]), f"bucket {b} differs"
    return got


def _contradicted(call, n_valid):
    """host_out shows a count the mask contradicts: the rows a prologue found
    or the rows partitioned differ from the caller's count."""
    found = call.found if call.found >= 0 else sum(call.counts)
    return found != n_valid or sum(call.counts) != n_valid


@pytest.mark.parametrize("n", [0, 1, 25, 4095, 4096, 4097, 300_000])
def test_unmasked_tick_sizes(n):
    _check(_table(n, ["i64"], seed=n), 0, None, 0, 32)


@pytest.mark.parametrize("B", [1, 2, 8, 16, 32, 64, 128, 256, 512])
def test_every_bucket_count(B):
    _check(_table(100_000, ["i64"], seed=B), 0, None, 12345, B)


@pytest.mark.parametrize("B", [64, 512])
def test_six_columns_of_four_widths_with_the_key_inside(B):
    cols = _table(70_001, ["i64", "i32", "i8", "s25", "i64"], seed=3, key_pos=2)
    _check(cols, 2, None, 0, B)


@pytest.mark.parametrize("kind", ["i32", "i16", "i8", "s25", "u8x2", "u8x3", "u8x4", "u8x8",
                                  "i64x2", "i64x5"])
def test_each_row_width(kind):
    _check(_table(50_000, [kind], seed=11), 0, None, 0, 16)


def test_one_bucket_holds_every_row():
    _check(_table(40_000, ["i64", "s25"], seed=5, skew=True), 0, None, 0, 64)


def test_global_offset_near_six_billion():
    n = 1 << 18
    _check(_table(n, ["i64"], seed=6), 0, None, 6_000_000_000 - n, 64)


@pytest.mark.parametrize("keep", [0.0, 0.01, 0.095, 0.3, 0.63, 1.0])
@pytest.mark.parametrize("select_first", [False, True])
def test_compacted_columns_under_a_mask(keep, select_first):
    n = 200_003
    cols = _table(n, ["i64", "s25"], seed=int(keep * 1000) + 1)
    _check(cols, 0, _mask(n, keep, seed=21), 777, 32, count=True, select_first=select_first)


@pytest.mark.parametrize("keep", [0.0, 0.01, 0.095, 0.3, 0.63, 1.0])
@pytest.mark.parametrize("select_first", [False, True])
def test_raw_columns_with_the_mask_count(keep, select_first):
    n = 150_001
    cols = _table(n, ["i64", "s25", "i16"], seed=int(keep * 1000) + 3)
    _check(cols, 0, _mask(n, keep, seed=33), 99, 64, compact=[False] * 4, count=True,
           select_first=select_first)


@pytest.mark.parametrize("select_first", [False, True])
def test_raw_and_compacted_columns_mixed(select_first):
    n = 90_000
    cols = _table(n, ["i64", "s25", "i32"], seed=41)
    mask = _mask(n, 0.4, seed=42)
    for compact in ([False, True, False, True], [True, False, True, False]):
        _check(cols, 0, mask, 5, 64, compact=compact, count=True, select_first=select_first)


@pytest.mark.parametrize("offset", [3, 5])
def test_offset_mask_views(offset):
    n = 64_000
    cols = [c[offset:] for c in _table(n, ["i64", "s25"], seed=51)]
    mask = _mask(n, 0.2, seed=52)[offset:]
    for sf in (False, True):
        _check(cols, 0, mask, 0, 32, select_first=sf)
        _check(cols, 0, mask, 0, 32, compact=[False, False, False], count=True, select_first=sf)


def test_small_masked_ticks():
    for n in (1, 25, 4097):
        cols = _table(n, ["i64"], seed=n)
        for sf in (False, True):
            _check(cols, 0, _mask(n, 0.5, seed=n), 0, 8, select_first=sf)
            _check(cols, 0, _mask(n, 0.0, seed=n), 0, 8, select_first=sf)


def test_repeated_calls_reuse_the_count_buffer():
    for i, B in enumerate((64, 8, 512, 1, 128, 256, 16)):
        _check(_table(30_000 + i, ["i32"], seed=60 + i), 0, None, i, B)


@pytest.mark.parametrize("select_first", [False, True])
@pytest.mark.parametrize("off", [-37, 41])
def test_a_count_the_mask_contradicts_is_flagged(select_first, off):
    """Raw columns with a wrong count are flagged in both prologues without
    touching memory past what the count sized: the GPU is still usable after."""
    n = 100_003
    cols = _table(n, ["i64", "s25"], seed=91)
    mask = _mask(n, 0.1, seed=92)
    wrong = int(mask.sum()) + off
    call = partition(list(cols), 0, mask, 0, 32, n_valid=wrong, select_first=select_first)
    torch.cuda.synchronize()
    assert _contradicted(call, wrong)
    _check(cols, 0, mask, 0, 32, compact=[False] * 3, count=True, select_first=select_first)


@pytest.mark.parametrize("select_first", [False, True])
def test_compacted_columns_of_another_mask_are_flagged(select_first):
    n = 100_003
    cols = _table(n, ["i64", "s25"], seed=93)
    kept = _mask(n, 0.3, seed=94)
    packed = [c[kept] for c in cols]
    for other in (0.2, 0.4):
        call = partition(list(packed), 0, _mask(n, other, seed=95), 0, 16,
                         select_first=select_first)
        assert _contradicted(call, packed[0].shape[0])
    torch.cuda.synchronize()
    _check(cols, 0, kept, 0, 16, select_first=select_first)


@pytest.mark.parametrize("B", [16, 512])
@pytest.mark.parametrize("mode", ["plain", "compacted-input", "select-first", "fold",
                                  "raw-select-first"])
def test_a_tick_past_a_thousand_subtiles(mode, B):
    n = 5_000_011
    cols = _table(n, ["i32"], seed=96)
    if mode == "plain":
        _check(cols, 0, None, 7, B)
        return
    raw = mode in ("fold", "raw-select-first")
    _check(cols, 0, _mask(n, 0.45, seed=97), 7, B, compact=[not raw] * 2, count=raw,
           select_first=mode in ("select-first", "raw-select-first"))


@pytest.mark.parametrize("B", [1, 128, 256, 512])
@pytest.mark.parametrize("select_first", [False, True])
def test_masked_ticks_at_one_to_512_buckets(select_first, B):
    n = 80_000
    cols = _table(n, ["i64", "s25"], seed=98)
    mask = _mask(n, 0.37, seed=99)
    _check(cols, 0, mask, 0, B, select_first=select_first)
    _check(cols, 0, mask, 0, B, compact=[False] * 3, count=True, select_first=select_first)


def test_uint8_mask_and_bool_mask_agree():
    n = 20_000
    cols = _table(n, ["i64"], seed=7)
    mask = _mask(n, 0.5, seed=8)
    a = partition([c[mask] for c in cols], 0, mask, 0, 32).outputs
    b = partition([c[mask] for c in cols], 0, mask.to(torch.uint8), 0, 32).outputs
    for x, y in zip(a, b):
        assert x.counts == y.counts
        for bx, by in zip(x.buckets(), y.buckets()):
            assert torch.equal(bx, by)
