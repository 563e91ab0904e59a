"""The one-launch gather (pageflow_b200.gather, pf_gather) against torch's
index_select and the reference's null rule (a row of -64 where the index is
the null sentinel; conversion.py:39-50): every dtype, rows of one to several
words with nulls and a ragged tail, and out-of-range indexes counted without
a read outside the column."""
from __future__ import annotations

import pytest
import torch

from pageflow_b200 import gather

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [torch.int8, torch.int16, torch.int32, torch.int64,
                                   torch.float16, torch.float32, torch.float64, torch.bool,
                                   torch.uint8])
def test_gather_matches_index_with_null(dtype):
    g = torch.Generator().manual_seed(13)
    src = (torch.randint(0, 100, (777, 3), generator=g) % 2 == 0) if dtype == torch.bool else \
        torch.randint(-100, 100, (777, 3), generator=g).to(dtype)
    idx = torch.randint(0, 777, (5000,), generator=g, dtype=torch.int64)
    idx[::7] = -64
    out = gather.index_with_null(src.cuda(), idx.cuda()).cpu()
    mask = idx == -64
    want = src[idx.masked_fill(mask, 0)]
    want[mask] = torch.full((1,), -64, dtype=dtype) if dtype != torch.bool else True
    assert torch.equal(out, want)
    sel = gather.index_select_many([src.cuda(), src[:, 0].contiguous().cuda()],
                                   idx.clamp(min=0).cuda())
    assert torch.equal(sel[0].cpu(), src[idx.clamp(min=0)])
    assert torch.equal(sel[1].cpu(), src[idx.clamp(min=0), 0])


@pytest.mark.parametrize("ncols", [1, 2, 3, 4])
def test_gather_one_word_rows_with_nulls_and_a_ragged_tail(ncols):
    """Columns whose rows are one 1-16 byte word take the batched kernel:
    nulls, an out-of-range index and a row count that is not a multiple of
    the rows a block takes."""
    g = torch.Generator().manual_seed(17 + ncols)
    n_src, n = 1000, 3 * 1024 + 37
    pool = [torch.randint(-(1 << 40), 1 << 40, (n_src,), generator=g),
            torch.randint(-(1 << 30), 1 << 30, (n_src,), generator=g, dtype=torch.int32),
            torch.randint(-100, 100, (n_src,), generator=g).to(torch.int16),
            torch.randint(-100, 100, (n_src,), generator=g).to(torch.int8),
            torch.randint(-(1 << 40), 1 << 40, (n_src, 2), generator=g),
            torch.randn(n_src, generator=g, dtype=torch.float64)]
    cols = [pool[(ncols + k) % len(pool)] for k in range(ncols)]
    idx = torch.randint(0, n_src, (n,), generator=g)
    idx[::5] = -64
    idx[7] = n_src
    out = gather.index_with_null_many([c.cuda() for c in cols], idx.cuda())
    bad = (idx == n_src) | (idx == -64)
    for o, c in zip(out, cols):
        want = c[idx.clamp(0, n_src - 1)]
        want[bad] = torch.full((1,), -64, dtype=c.dtype)
        assert torch.equal(o.cpu(), want)
    sel = gather.index_select_many([c.cuda() for c in cols], idx.clamp(0, n_src - 1).cuda())
    for o, c in zip(sel, cols):
        assert torch.equal(o.cpu(), c[idx.clamp(0, n_src - 1)])


def test_gather_counts_out_of_range_and_reads_nothing_outside():
    src = torch.arange(100, dtype=torch.int64, device="cuda")
    idx = torch.tensor([0, 99, 100, -1, 5, 1 << 40], dtype=torch.int64, device="cuda")
    with pytest.raises(IndexError):
        gather.index_select_many([src], idx, check_range=True)
    out = gather.index_select_many([src], idx)[0].cpu().tolist()
    assert out[0] == 0 and out[1] == 99 and out[4] == 5
    assert out[2] == out[3] == out[5] == -64
    # a slice (unaligned base) and an empty gather
    sl = src[1:]
    assert gather.index_select(sl, torch.tensor([0, 98], device="cuda")).cpu().tolist() == [1, 99]
    assert gather.index_select(src, torch.empty(0, dtype=torch.int64, device="cuda")).numel() == 0


@pytest.mark.parametrize("sorted_reads", [False, True])
def test_gather_from_pinned_host_segments(sorted_reads):
    """Rows read in place from pinned host memory (three segments of uneven
    size, one empty), per dtype and row width: equal to indexing the
    concatenated column, null rows for the null index and for indexes
    outside the segments (counted, never read)."""
    g = torch.Generator().manual_seed(31)
    sizes = [700, 0, 1301, 55]
    rows = [0]
    for s in sizes:
        rows.append(rows[-1] + s)
    base = 1000
    full = [torch.randint(-(1 << 40), 1 << 40, (rows[-1],), generator=g),
            torch.randint(-100, 100, (rows[-1], 3), generator=g).to(torch.int16),
            torch.randn(rows[-1], generator=g, dtype=torch.float64),
            torch.randint(0, 255, (rows[-1], 25), generator=g).to(torch.uint8)]
    segs = [[c[a:b].contiguous().pin_memory() for a, b in zip(rows[:-1], rows[1:])]
            for c in full]
    seg_rows = [r + base for r in rows]
    n = 5000
    idx = torch.randint(0, rows[-1], (n,), generator=g)
    idx[::9] = -64
    idx[5] = rows[-1] + 3          # past the last segment
    idx[6] = -5                    # before the first
    outs, bad = gather.gather_from_host(segs, seg_rows, idx.cuda(), base=base,
                                        sorted_reads=sorted_reads)
    assert bad == 2
    nul = (idx == -64) | (idx < 0) | (idx >= rows[-1])
    for o, c in zip(outs, full):
        want = c[idx.clamp(0, rows[-1] - 1)]
        want[nul] = torch.full((1,), -64, dtype=c.dtype)
        assert torch.equal(o.cpu(), want)
