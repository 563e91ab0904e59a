"""The drop-in kernels against the reference's own CUDA kernels, run side by
side on the GPU: PageFlow's operators/kernels/*.cu compiled unmodified for
sm_100a by oracle/build_ref.sh (oracle/_ref/tqpkernels*.so).  Every output
must be identical: partition counts, padded totals and every bucket's rows of
every column and the gidx (padding excluded); unique-hash pairs; semi/anti
rows; expand pairs.  The reference's whole GPU path for the join -> group-by
(oracle/plain_form.py) must give the fused path's groups, sums and counts."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import plain_form
from pageflow_b200 import datagen, tqpkernels
from pageflow_b200.join_aggregate import JoinAggregate

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not plain_form.available(),
                                 reason="the reference's kernels are not built (oracle/build_ref.sh)")]


def _host(n):
    return torch.zeros(n, dtype=torch.int64, pin_memory=True)


def _gen(seed):
    return torch.Generator().manual_seed(seed)


def _cols(n, seed):
    g = _gen(seed)
    key = torch.randint(-(1 << 40), 1 << 40, (n,), dtype=torch.int64, generator=g)
    c1 = torch.randint(-(1 << 30), 1 << 30, (n,), dtype=torch.int32, generator=g)
    c2 = torch.randint(0, 256, (n, 25), dtype=torch.uint8, generator=g)
    c3 = torch.randint(-128, 128, (n,), dtype=torch.int8, generator=g)
    return [t.cuda() for t in (key, c1, c2, c3)]


def _bucket_rows(t, counts):
    rb = t.element_size() * (t.shape[1] if t.dim() == 2 else 1)
    unit = 512 // np.gcd(rb, 512)
    out, at = [], 0
    for c in counts:
        out.append(t[at:at + c])
        at += -(-c // unit) * unit
    return out


def _same_partition(cols, comp, mask, n_valid, goff, B, select_first):
    ref = plain_form.kernels()
    h1, h2 = _host(512 + 5), _host(512 + 5)
    a = ref.partition_sort(cols, comp, 0, mask, n_valid, goff, B, select_first, h1)
    b = tqpkernels.partition_sort(cols, comp, 0, mask, n_valid, goff, B, select_first, h2)
    assert h1[:B + 4].tolist() == h2[:B + 4].tolist()   # counts and padded totals
    assert int(h1[B + 4]) == int(h2[B + 4])             # prologue's kept rows
    counts = h1[:B].tolist()
    assert len(a) == len(b)
    for x, y in zip(a, b):
        for bx, by in zip(_bucket_rows(x, counts), _bucket_rows(y, counts)):
            assert torch.equal(bx, by)


@pytest.mark.parametrize("B", [1, 16, 128, 512])
@pytest.mark.parametrize("n", [1, 4097, 250_001])
def test_partition_sort_is_the_references(B, n):
    _same_partition(_cols(n, B + n), [0, 0, 0, 0], None, n, 1234, B, False)


@pytest.mark.parametrize("select_first", [False, True])
@pytest.mark.parametrize("keep", [0.05, 0.6])
def test_masked_partition_sort_is_the_references(select_first, keep):
    n = 300_003
    cols = _cols(n, 7)
    mask = (torch.rand(n, generator=_gen(8)) < keep).cuda()
    kept = int(mask.sum())
    # raw columns folded or gathered, and every column compacted
    _same_partition(cols, [0, 0, 0, 0], mask, kept, 5, 64, select_first)
    packed = [c[mask] for c in cols]
    _same_partition(packed, [1, 1, 1, 1], mask, kept, 5, 64, select_first)


def test_unique_hash_is_the_references():
    ref = plain_form.kernels()
    nb, np_ = 400_000, 1_500_000
    bk = (torch.randperm(4 * nb, generator=_gen(3))[:nb].to(torch.int64) * 7919).cuda()
    pk = bk[torch.randint(0, nb, (np_,), generator=_gen(4)).cuda()]
    pk[::7] += 1
    h1, h2 = _host(2), _host(2)
    a = ref.join_unique_hash([bk], [pk], h1)
    b = tqpkernels.join_unique_hash([bk], [pk], h2)
    n = int(h1[0])
    assert n == int(h2[0])
    assert torch.equal(a[0][:n], b[0][:n]) and torch.equal(a[1][:n], b[1][:n])


@pytest.mark.parametrize("op", [0, 1, 2, 5])
@pytest.mark.parametrize("anti", [False, True])
def test_semi_anti_is_the_references(op, anti):
    ref = plain_form.kernels()
    g = _gen(op * 2 + anti)
    bk = torch.randint(-50, 30_000, (100_000,), generator=g).cuda()
    pk = torch.randint(-60, 60_000, (200_000,), generator=g).cuda()
    bv = torch.randint(0, 4, (100_000,), generator=g).cuda()
    pv = torch.randint(0, 4, (200_000,), generator=g).cuda()
    h1, h2 = _host(2), _host(2)
    a = ref.join_semi_anti(bk, pk, bv if op else None, pv if op else None, op, anti, h1)
    b = tqpkernels.join_semi_anti(bk, pk, bv if op else None, pv if op else None, op, anti, h2)
    n = int(h1[0])
    assert h1.tolist() == h2.tolist()
    assert torch.equal(a[:n], b[:n])


def test_expand_is_the_references():
    ref = plain_form.kernels()
    g = _gen(11)
    length = torch.randint(0, 6, (500_000,), generator=g).cuda()
    start = torch.randint(0, 1_000_000, (500_000,), generator=g).cuda()
    sorted_ids = torch.randperm(1_000_006, generator=g).cuda()
    a = ref.join_expand(sorted_ids, start, length, _host(2))
    b = tqpkernels.join_expand(sorted_ids, start, length, _host(2))
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


def test_the_references_gpu_path_gives_the_fused_result():
    w = datagen.scaled(datagen.SCALE, 1 / 200)   # 750K x 3M, 7500 groups
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    keys, sums, counts = plain_form.join_aggregate(bkey, bgrp, fk, price, disc, w.scale)
    plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda")
    k2, s2, c2 = plan.run(bkey, bgrp, fk, price, disc)
    assert torch.equal(keys, k2) and torch.equal(sums, s2) and torch.equal(counts, c2)
