"""The oracle pinned against the golden vectors that PageFlow's own Python
code produced (tests/golden/make_golden.py): mix64 and the radix buckets, the
padded partition layout, the unique-build join pairs, and the small workload's
join + group-by end to end.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from tests.golden import load

pytestmark = pytest.mark.usefixtures("oracle_lib")


def test_mix64_is_the_references_finalizer():
    import oracle
    g = load("mix64.npz")
    got = oracle.mix64(g["keys"])
    assert np.array_equal(got.view(np.int64), g["mix"])


@pytest.mark.parametrize("B", [1, 2, 8, 64, 256, 512, 1024, 4096])
def test_bucket_is_the_references_top_bits(B):
    import oracle
    g = load("buckets.npz")
    assert np.array_equal(oracle.bucket(g["keys"], B), g[f"B{B}"])


@pytest.mark.parametrize("case", range(4))
def test_padded_layout_is_the_references(case):
    """The oracle's stable partition, laid out padded, gives the bucket rows,
    bucket starts and totals of the reference's _partition_outputs."""
    import oracle
    g = load("partition_layout.npz")
    B = int(g[f"c{case}_B"][0])
    bucket = g[f"c{case}_bucket"]
    counts = np.bincount(bucket, minlength=B)
    assert np.array_equal(counts, g[f"c{case}_counts"])
    order = np.argsort(bucket, kind="stable")
    for j in range(3):
        t = g[f"c{case}_in{j}"]
        rb = t.dtype.itemsize * (t.shape[1] if t.ndim == 2 else 1)
        starts, total = oracle.padded_layout(counts, rb)
        ref_total, ref_rows = g[f"c{case}_total{j}"]
        assert total == ref_total == ref_rows
        assert list(starts) == list(g[f"c{case}_starts{j}"])
        assert np.array_equal(t[order], g[f"c{case}_rows{j}"])


def test_oracle_partition_orders_rows_like_a_stable_sort():
    import oracle
    rng = np.random.default_rng(5)
    keys = rng.integers(-(1 << 40), 1 << 40, 20_000)
    for B in (1, 16, 512):
        counts, outs = oracle.partition([keys], 0, None, 77, B)
        b = oracle.bucket(keys, B)
        order = np.argsort(b, kind="stable")
        assert np.array_equal(np.concatenate(outs[0]), keys[order])
        assert np.array_equal(np.concatenate(outs[1]), 77 + order)
        assert np.array_equal(counts, np.bincount(b, minlength=B))


@pytest.mark.parametrize("tag", ["one", "two"])
def test_unique_join_pairs_are_the_references(tag):
    import oracle
    g = load("join_small.npz")
    if tag == "one":
        bi, pi = oracle.join_unique([g["one_b0"]], [g["one_p0"]])
    else:
        bi, pi = oracle.join_unique([g["two_b0"], g["two_b1"]], [g["two_p0"], g["two_p1"]])
    assert np.array_equal(bi, g[f"{tag}_build_idx"])
    assert np.array_equal(pi, g[f"{tag}_probe_idx"])


def test_small_workload_inputs_are_the_fixtures():
    import oracle
    g = load("config0.npz")
    bkey, bgrp = oracle.gen_build(0, 250_000, 25)
    fk, price, disc = oracle.gen_probe(0, 0, 250_000, 0, 1_000_000)
    want = g["input_checksum"]
    got = [int(np.bitwise_xor.reduce(bkey.view(np.uint64))),
           int(np.bitwise_xor.reduce(fk.view(np.uint64))), int(price.sum()), int(disc.sum()),
           int(bgrp.sum())]
    assert [int(x) for x in want] == got
    assert np.array_equal(np.sort(bkey), np.arange(1, 250_001))


def test_small_workload_join_aggregate_is_the_references():
    """The oracle's join + group-by equals the reference's
    _sort_search_pairs -> KeyedAggregate.pass1 -> reduce_tick_slice."""
    import oracle
    g = load("config0.npz")
    bkey, bgrp = oracle.gen_build(0, 250_000, 25)
    fk, price, disc = oracle.gen_probe(0, 0, 250_000, 0, 1_000_000)
    s, c, matched, max_abs = oracle.join_aggregate(bkey, bgrp, fk, price, disc, 100, 0, 25)
    present = np.nonzero(c)[0]
    assert np.array_equal(present, g["groups"])
    assert np.array_equal(s[present], g["sums"])
    assert np.array_equal(c[present], g["counts"])
    assert matched == int(g["matched"][0])
    assert max_abs < 1 << 53  # the reference's float64 SUM is exact here


def test_expected_groups_agree_with_the_join():
    import oracle
    bkey, bgrp = oracle.gen_build(1, 20_000, 300)
    fk, price, disc = oracle.gen_probe(1, 1, 20_000, 0, 80_000)
    s, c, m, _ = oracle.join_aggregate(bkey, bgrp, fk, price, disc, 100, 0, 300, B=8)
    s2, c2, m2 = oracle.expected_groups(1, 1, 20_000, 300, 0, 80_000)
    assert m == m2 and np.array_equal(s, s2) and np.array_equal(c, c2)
    # one in ten probe rows misses the build keys
    assert 0.88 < m / 80_000 < 0.92


def test_semi_anti_oracle_matches_brute_force():
    import oracle
    rng = np.random.default_rng(3)
    bk = rng.integers(-50, 700, 2000)
    pk = rng.integers(-60, 1400, 1500)
    bv = rng.integers(0, 4, 2000)
    pv = rng.integers(0, 4, 1500)
    ops = {None: None, "<>": np.not_equal, "<": np.less, "<=": np.less_equal,
           ">": np.greater, ">=": np.greater_equal}
    for op, fn in ops.items():
        hit = bk[:, None] == pk[None, :]
        if fn is not None:
            hit &= fn(bv[:, None], pv[None, :])
        keep = hit.any(axis=0)
        for anti in (False, True):
            want = np.nonzero(~keep if anti else keep)[0]
            got = oracle.semi_anti(bk, pk, anti, bv if op else None, pv if op else None, op)
            assert np.array_equal(got, want), (op, anti)


def test_expand_oracle():
    import oracle
    sorted_ids = np.arange(100, 120)
    start = np.array([0, 5, 5, 10, 0])
    length = np.array([2, 0, 3, 1, 0])
    cs, cr = oracle.expand(sorted_ids, start, length)
    assert cs.tolist() == [100, 101, 105, 106, 107, 110]
    assert cr.tolist() == [0, 0, 2, 2, 2, 3]


def test_plain_forms_aggregation_is_the_references():
    """The GPU plain form's aggregation steps (oracle/plain_form.aggregate:
    KeyedAggregate.pass1 per morsel, buckets, reduce_tick_slice per round),
    run on the CPU over the small workload's joined rows, give the
    reference's own result (config0.npz, made by its _sort_search_pairs,
    KeyedAggregate.pass1 and reduce_tick_slice)."""
    import torch

    import oracle
    from oracle import plain_form
    g = load("config0.npz")
    bkey, bgrp = oracle.gen_build(0, 250_000, 25)
    fk, price, disc = oracle.gen_probe(0, 0, 250_000, 0, 1_000_000)
    bi, pi = oracle.join_unique([bkey], [fk])
    keys, sums, counts = plain_form.aggregate(torch.from_numpy(bgrp[bi]),
                                              torch.from_numpy(price[pi]),
                                              torch.from_numpy(disc[pi]), 100)
    assert np.array_equal(keys.numpy(), g["groups"])
    assert np.array_equal(sums.numpy(), g["sums"])
    assert np.array_equal(counts.numpy(), g["counts"])
