"""The slab group-by and the fused join -> group-by on the GPU:

* DenseAggregationSlab (pf_slab_add / pf_slab_finish) against the vectors the
  reference's own DenseAggregationSlab produced (tests/golden/slab.json), and
  its feed-chunking invariance and identities (the reference's
  tests/aggregate_merge/test_aggregation_slab.py cases);
* the fused join + group-by (pf_join_aggregate) against the small workload's
  golden result from the reference's operators, against the oracle on random
  inputs (every fan-out, slices of a partition over the table budget, empty
  and ragged inputs, groups out of range, negative and extreme keys), and the
  device generator against the CPU one.  Every fused test runs on both join
  paths (PF_JOIN_PATH=rounds: L2 tables in rounds; smem: a second radix pass
  and shared-memory tables).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from pageflow_b200 import datagen
from pageflow_b200.aggregation_slab import DenseAggregationSlab
from pageflow_b200.join_aggregate import JoinAggregate, join_group_aggregate
from tests.golden import load

pytestmark = pytest.mark.gpu


# ---- slab -------------------------------------------------------------------------

@pytest.mark.parametrize("case", range(4))
def test_slab_matches_the_references_vectors(case):
    g = load("slab.json")[case]
    specs = [(torch.int64, ()), (torch.int64, ()), (torch.int64, ()), (torch.float64, (2,))]
    s = DenseAggregationSlab(g["lo"], g["hi"], torch.int64, specs, g["ops"], "cuda")
    for k, v1, v2, v3, v4 in g["ticks"]:
        s.add(torch.tensor(k, device="cuda"),
              [torch.tensor(v1, device="cuda"), torch.tensor(v2, device="cuda"),
               torch.tensor(v3, device="cuda"),
               torch.tensor(v4, dtype=torch.float64, device="cuda")])
    keys, vals = s.finish()
    assert keys.tolist() == g["keys"]
    for got, want in zip(vals, g["vals"]):
        # integer values bit-exact; the float sums hold small integers, exact too
        assert got.tolist() == want


def test_feed_chunking_does_not_change_slab_result():
    keys = torch.tensor([4, 2, 4, 7, 2, 4, 7, 3], device="cuda")
    states = torch.tensor([[1.0, 1.0], [2.0, 1.0], [3.0, 1.0], [4.0, 1.0], [5.0, 1.0],
                           [6.0, 1.0], [7.0, 1.0], [8.0, 1.0]], dtype=torch.float64,
                          device="cuda")
    one = DenseAggregationSlab(2, 7, torch.int64, [(torch.float64, (2,))], ["sum"], "cuda")
    one.add(keys, [states])
    many = DenseAggregationSlab(2, 7, torch.int64, [(torch.float64, (2,))], ["sum"], "cuda")
    for lo, hi in ((0, 1), (1, 5), (5, 6), (6, 8)):
        many.add(keys[lo:hi], [states[lo:hi]])
    ka, va = one.finish()
    kb, vb = many.finish()
    assert torch.equal(ka, kb) and torch.equal(va[0], vb[0])
    assert ka.tolist() == [2, 3, 4, 7]
    assert va[0].tolist() == [[7.0, 2.0], [8.0, 1.0], [10.0, 3.0], [11.0, 2.0]]


def test_amax_and_amin_identities_do_not_poison_first_value():
    s = DenseAggregationSlab(10, 12, torch.int64, [(torch.int64, ()), (torch.int64, ())],
                             ["amax", "amin"], "cuda")
    s.add(torch.tensor([10, 10, 12], device="cuda"),
          [torch.tensor([-8, -3, -11], device="cuda"), torch.tensor([8, 3, 11], device="cuda")])
    keys, values = s.finish()
    assert keys.tolist() == [10, 12]
    assert values[0].tolist() == [-3, -11] and values[1].tolist() == [3, 11]


def test_slab_large_sum_is_exact_int64():
    n, G = 5_000_000, 100_003
    g = torch.Generator().manual_seed(9)
    keys = torch.randint(0, G, (n,), generator=g)
    vals = torch.randint(-(1 << 40), 1 << 40, (n,), generator=g)
    s = DenseAggregationSlab(0, G - 1, torch.int64, [(torch.int64, ())], ["sum"], "cuda")
    s.add(keys.cuda(), [vals.cuda()])
    k, (v,) = s.finish()
    want = np.zeros(G, np.int64)
    np.add.at(want, keys.numpy(), vals.numpy())
    present = np.unique(keys.numpy())
    assert np.array_equal(k.cpu().numpy(), present)
    assert np.array_equal(v.cpu().numpy(), want[present])


# ---- the fused join -> group-by ---------------------------------------------------

@pytest.fixture(params=["rounds", "smem", "smem-counted"])
def join_path(request, monkeypatch):
    """The round path, the shared-memory path (regions sized from the
    expected rows, counted again on an overflow) and the shared-memory path
    with both radix passes counted first."""
    monkeypatch.setenv("PF_JOIN_PATH", request.param.split("-")[0])
    if request.param.endswith("counted"):
        monkeypatch.setenv("PF_COUNTED", "1")
    else:
        monkeypatch.delenv("PF_COUNTED", raising=False)
    return request.param


def _counted_passes():
    from pageflow_b200 import _native
    return _native.lib().pf_join_aggregate_counted_passes()


def _oracle_groups(bkey, bgrp, fk, price, disc, group_min, n_groups, scale=100):
    s, c, matched, _ = oracle.join_aggregate(
        bkey.cpu().numpy(), bgrp.cpu().numpy(), fk.cpu().numpy(), price.cpu().numpy(),
        disc.cpu().numpy() if disc is not None else None, scale, group_min, n_groups, B=16)
    present = np.nonzero(c)[0]
    return group_min + present, s[present], c[present], matched


def _assert_groups(got, want):
    keys, sums, counts = got
    assert np.array_equal(keys.cpu().numpy(), want[0])
    assert np.array_equal(sums.cpu().numpy(), want[1])
    assert np.array_equal(counts.cpu().numpy(), want[2])


def test_small_workload_is_the_references_result(join_path):
    """250K x 1M, seed 0: the groups, sums and counts of the reference's
    join + KeyedAggregate.pass1 + reduce_tick_slice."""
    g = load("config0.npz")
    w = datagen.SMALL
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda")
    keys, sums, counts = plan.run(bkey, bgrp, fk, price, disc)
    assert np.array_equal(keys.cpu().numpy(), g["groups"])
    assert np.array_equal(sums.cpu().numpy(), g["sums"])
    assert np.array_equal(counts.cpu().numpy(), g["counts"])
    st = plan.read_stats()
    assert st.matched == int(g["matched"][0]) and st.overflow == 0 and st.bad_groups == 0
    assert st.device_error == 0


def test_device_generator_is_the_cpu_generator():
    w = datagen.scaled(datagen.SCALE, 1 / 1000)
    bkey, bgrp = datagen.gen_build(w, "cuda", lo=17, rows=50_000)
    fk, price, disc = datagen.gen_probe(w, "cuda", lo=123_456, rows=200_000)
    obk, obg = oracle.gen_build(w.seed, w.n_build, w.n_groups, 17, 50_000)
    ofk, opr, odi = oracle.gen_probe(w.config, w.seed, w.n_build, 123_456, 200_000)
    assert np.array_equal(bkey.cpu().numpy(), obk) and np.array_equal(bgrp.cpu().numpy(), obg)
    assert np.array_equal(fk.cpu().numpy(), ofk)
    assert np.array_equal(price.cpu().numpy(), opr)
    assert np.array_equal(disc.cpu().numpy(), odi)


@pytest.mark.parametrize("B", [1, 2, 16, 64, 256, 512, 1024, 4096])
def test_every_fan_out_matches_the_oracle(B, join_path):
    w = datagen.scaled(datagen.SCALE, 1 / 500)   # 300K x 1.2M, 3000 groups
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 0, w.n_groups)
    plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda", B=B)
    _assert_groups(plan.run(bkey, bgrp, fk, price, disc), want)
    st = plan.read_stats()
    assert st.matched == want[3] and st.overflow == 0 and st.device_error == 0


def test_partitions_over_the_table_budget_take_slices(monkeypatch, join_path):
    """B = 1 and 2 over 3M build rows: partitions over the 768K-row table
    budget, joined in slices, each probe row meeting every slice."""
    w = datagen.scaled(datagen.SCALE, 1 / 50)   # 3M x 12M
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 0, w.n_groups)
    for B in (1, 2):
        plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda", B=B)
        _assert_groups(plan.run(bkey, bgrp, fk, price, disc), want)
        assert plan.read_stats().matched == want[3]


def _random_case(nb, np_, G, seed, gmin=0):
    g = torch.Generator().manual_seed(seed)
    bkey = (torch.randperm(max(4 * nb, 1), generator=g)[:nb].to(torch.int64) * 104729
            - (1 << 50))
    bgrp = torch.randint(gmin, gmin + G, (nb,), generator=g, dtype=torch.int32)
    if nb:
        fk = bkey[torch.randint(0, nb, (np_,), generator=g)]
        fk = torch.where(torch.rand(np_, generator=g) < 0.2, fk + 1, fk)
    else:
        fk = torch.randint(-100, 100, (np_,), generator=g)
    price = torch.randint(-(1 << 30), 1 << 30, (np_,), generator=g)
    disc = torch.randint(0, 11, (np_,), generator=g)
    return [t.cuda() for t in (bkey, bgrp, fk, price, disc)]


@pytest.mark.parametrize("nb,np_,G", [(0, 10, 5), (10, 0, 5), (1, 1, 1), (3, 4097, 2),
                                      (4097, 3, 7), (50_000, 200_003, 1),
                                      (123_457, 654_321, 50_000)])
def test_ragged_and_empty_inputs(nb, np_, G, join_path):
    bkey, bgrp, fk, price, disc = _random_case(nb, np_, G, nb + np_, gmin=-3)
    want = _oracle_groups(bkey, bgrp, fk, price, disc, -3, G)
    got = join_group_aggregate(bkey, bgrp, fk, price, disc, group_min=-3, n_groups=G, B=32)
    _assert_groups(got, want)


def test_no_discount_column_and_another_scale(join_path):
    bkey, bgrp, fk, price, disc = _random_case(20_000, 90_000, 100, 5)
    want = _oracle_groups(bkey, bgrp, fk, price, None, 0, 100)
    _assert_groups(join_group_aggregate(bkey, bgrp, fk, price, None, group_min=0, n_groups=100),
                   want)
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 0, 100, scale=7)
    _assert_groups(join_group_aggregate(bkey, bgrp, fk, price, disc, scale=7, group_min=0,
                                        n_groups=100), want)


def test_groups_outside_the_range_are_counted_not_aggregated(join_path):
    bkey, bgrp, fk, price, disc = _random_case(10_000, 40_000, 50, 6)
    plan = JoinAggregate(10_000, 40_000, 10, 20, "cuda", B=8)   # groups [10, 30) only
    keys, sums, counts = plan.run(bkey, bgrp, fk, price, disc)
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 10, 20)
    _assert_groups((keys, sums, counts), want)
    st = plan.read_stats()
    assert st.bad_groups == int(((bgrp < 10) | (bgrp >= 30)).sum())


def test_repeated_runs_of_one_plan_are_identical(join_path):
    w = datagen.scaled(datagen.SCALE, 1 / 1000)
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda")
    first = [t.clone() for t in plan.run(bkey, bgrp, fk, price, disc)]
    for _ in range(3):
        for a, b in zip(first, plan.run(bkey, bgrp, fk, price, disc)):
            assert torch.equal(a, b)


def test_scale_workload_tenth_matches_the_generator_expectation(join_path):
    """A tenth of the 150M x 600M workload (15M x 60M, 150K groups) against
    the exact expectation from the generator (every group's sum and count)."""
    w = datagen.scaled(datagen.SCALE, 1 / 10)
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda")
    plan.aggregate(bkey, bgrp, fk, price, disc)
    s, c, m = oracle.expected_groups(w.config, w.seed, w.n_build, w.n_groups, 0, w.n_probe)
    assert np.array_equal(plan.sum.cpu().numpy(), s)
    assert np.array_equal(plan.count.cpu().numpy(), c)
    assert plan.read_stats().matched == m


def test_sub_partition_over_the_shared_table_is_joined_in_chunks(join_path):
    """Build keys chosen so that the top 3 bits of their mix64 agree: at
    B = 1 the second pass cannot split them below one sub-partition of ~10K
    build rows, over the shared-memory table's capacity, so it is joined in
    table-sized chunks of build rows, each against every probe row."""
    g = torch.Generator().manual_seed(11)
    cand = torch.randint(-(1 << 62), 1 << 62, (80_000,), generator=g).numpy()
    top = oracle.mix64(cand) >> np.uint64(61)
    bkey = torch.from_numpy(np.unique(cand[top == 0])).cuda()
    nb = bkey.numel()
    assert nb > 8_000
    bgrp = torch.randint(0, 300, (nb,), generator=g, dtype=torch.int32).cuda()
    pick = torch.randint(0, nb, (200_000,), generator=g).cuda()
    fk = torch.where(torch.rand(200_000, generator=g).cuda() < 0.1, bkey[pick] + 1, bkey[pick])
    price = torch.randint(-(1 << 30), 1 << 30, (200_000,), generator=g).cuda()
    disc = torch.randint(0, 11, (200_000,), generator=g).cuda()
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 0, 300)
    plan = JoinAggregate(nb, 200_000, 0, 300, "cuda", B=1)
    _assert_groups(plan.run(bkey, bgrp, fk, price, disc), want)
    assert plan.read_stats().matched == want[3]


def _unmix64(h: int) -> int:
    """The key whose mix64 is h (each step of the finalizer inverted)."""
    M = (1 << 64) - 1
    h ^= h >> 33
    h = (h * pow(0xc4ceb9fe1a85ec53, -1, 1 << 64)) & M
    h ^= h >> 33
    h = (h * pow(0xff51afd7ed558ccd, -1, 1 << 64)) & M
    h ^= h >> 33
    return h - (1 << 64) if h >> 63 else h


def test_extreme_keys_join(join_path):
    """INT64_MIN and INT64_MAX as keys on both sides, and the key whose mix64
    is 2^63 (the shared-memory table's free mark among hashes), beside
    ordinary keys."""
    I = np.iinfo(np.int64)
    ks = _unmix64(1 << 63)
    assert int(oracle.mix64(np.array([ks], np.int64))[0]) == 1 << 63
    bkey = torch.tensor([I.min, I.max, 0, -1, 5, I.min + 1, ks], dtype=torch.int64).cuda()
    bgrp = torch.tensor([0, 1, 2, 3, 4, 5, 6], dtype=torch.int32).cuda()
    fk = torch.tensor([I.min, I.min, I.max, 7, -1, I.min + 1, 0, I.min, ks, ks, ks + 1],
                      dtype=torch.int64).cuda()
    price = torch.arange(1, 12, dtype=torch.int64).cuda() * 1000
    disc = torch.zeros(11, dtype=torch.int64).cuda()
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 0, 7)
    for B in (1, 4):
        plan = JoinAggregate(7, 11, 0, 7, "cuda", B=B)
        _assert_groups(plan.run(bkey, bgrp, fk, price, disc), want)
        assert plan.read_stats().matched == want[3] == 9


@pytest.mark.parametrize("B", [1, 64])
def test_skewed_probe_keys(B, join_path):
    """Zipf-like probe keys: a few build keys take most probe rows, so their
    sub-partitions hold far more probe rows than the rest and their table
    cells (or L2 slots) take most of the adds."""
    g = torch.Generator().manual_seed(21)
    nb, np_ = 200_000, 2_000_000
    bkey = torch.randperm(4 * nb, generator=g)[:nb].to(torch.int64) * 104729 - (1 << 40)
    bgrp = torch.randint(0, 5_000, (nb,), generator=g, dtype=torch.int32)
    ranks = torch.rand(np_, generator=g).pow(6).mul(nb).to(torch.int64).clamp_(max=nb - 1)
    fk = bkey[ranks]
    fk[::13] += 1                                     # some rows match nothing
    price = torch.randint(-(1 << 28), 1 << 28, (np_,), generator=g)
    disc = torch.randint(0, 11, (np_,), generator=g)
    args = [t.cuda() for t in (bkey, bgrp, fk, price, disc)]
    want = _oracle_groups(*args, 0, 5_000)
    plan = JoinAggregate(nb, np_, 0, 5_000, "cuda", B=B)
    _assert_groups(plan.run(*args), want)
    assert plan.read_stats().matched == want[3]
    top = torch.bincount(ranks, minlength=nb).max().item()
    assert top > np_ // 50                            # the hottest key takes > 2% of the rows
    if join_path == "smem":
        # the hot keys crowd their (sub-)buckets past the regions: the pass
        # that overflowed ran again, counted
        assert _counted_passes() & (1 if B > 1 else 2)


def _unmix64_array(h):
    """The keys whose mix64 hashes are h (numpy uint64), like _unmix64."""
    k = h.copy()
    with np.errstate(over="ignore"):
        k ^= k >> np.uint64(33)
        k *= np.uint64(pow(0xc4ceb9fe1a85ec53, -1, 1 << 64))
        k ^= k >> np.uint64(33)
        k *= np.uint64(pow(0xff51afd7ed558ccd, -1, 1 << 64))
        k ^= k >> np.uint64(33)
    return k.view(np.int64)


def test_second_pass_overflow_alone_is_run_again_counted(monkeypatch):
    """Build keys spread exactly evenly over 64 buckets and their 4
    sub-buckets (keys made from chosen hashes), ten probe rows a key, and one
    key repeated 3000 times more: its bucket stays inside its first-pass
    region (31250 + 3000 of 34832 rows) while its sub-bucket passes its
    second-pass region (7812 + 3000 of 10588), so only the second pass runs
    again, counted from the first pass's cursors."""
    monkeypatch.delenv("PF_JOIN_PATH", raising=False)
    monkeypatch.delenv("PF_COUNTED", raising=False)
    rng = np.random.default_rng(5)
    nb, B, G = 200_000, 64, 5_000
    cell = np.arange(nb, dtype=np.uint64) % np.uint64(B * 4)      # (bucket, sub-bucket)
    low = rng.integers(0, 1 << 56, nb, dtype=np.uint64)
    h = (cell << np.uint64(56)) | low
    h = np.unique(h)
    assert len(h) == nb
    bkey_np = _unmix64_array(h)
    assert np.array_equal(oracle.mix64(bkey_np).view(np.uint64), h)
    bkey_np = bkey_np[rng.permutation(nb)]
    bgrp_np = rng.integers(0, G, nb, dtype=np.int32)
    fk_np = np.concatenate([np.repeat(bkey_np, 10), np.full(3000, bkey_np[7])])
    fk_np = fk_np[rng.permutation(len(fk_np))]
    np_ = len(fk_np)
    price_np = rng.integers(0, 1 << 30, np_, dtype=np.int64)
    disc_np = rng.integers(0, 11, np_, dtype=np.int64)
    args = [torch.from_numpy(x).cuda() for x in (bkey_np, bgrp_np, fk_np, price_np, disc_np)]
    want = _oracle_groups(*args, 0, G)
    plan = JoinAggregate(nb, np_, 0, G, "cuda", B=B)
    _assert_groups(plan.run(*args), want)
    assert plan.read_stats().matched == want[3] == np_
    assert _counted_passes() == 2


def test_host_batches_streamed_equal_one_call_each():
    """run_stream over pinned host batches (each crossing the link while the
    one before it joins, into alternating device buffers) gives every batch
    the groups that one call on its device copy gives."""
    w = datagen.scaled(datagen.SCALE, 1 / 500)
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda", B=64)
    batches, want = [], []
    for shift in (0, 7, 1000):
        cols = (bkey, bgrp, fk, price + shift, (disc + shift) % 11 if shift else None)
        keys, sums, counts = plan.run(*cols)
        want.append((keys.cpu(), sums.cpu(), counts.cpu()))
        batches.append(tuple(None if c is None else c.cpu().pin_memory() for c in cols))
    got = list(plan.run_stream(batches + batches[:1]))
    assert len(got) == 4
    for g, wnt in zip(got, want + want[:1]):
        for a, b in zip(g, wnt):
            assert torch.equal(a, b)
    assert not torch.equal(got[0][1], got[1][1])


def test_uniform_keys_fill_the_regions_without_counting(join_path):
    w = datagen.scaled(datagen.SCALE, 1 / 300)   # 500K x 2M, 5000 groups
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 0, w.n_groups)
    plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda", B=64)
    _assert_groups(plan.run(bkey, bgrp, fk, price, disc), want)
    assert {"rounds": 1, "smem": 0, "smem-counted": 3}[join_path] == _counted_passes()


@pytest.mark.parametrize("knobs", [dict(path=0, table=1, sub_rows=0, counted=0),
                                   dict(path=0, table=1, sub_rows=682, counted=0),
                                   dict(path=0, table=0, sub_rows=300, counted=0),
                                   dict(path=0, table=1, sub_rows=0, counted=1),
                                   dict(path=1, table=0, sub_rows=0, counted=0)])
def test_every_knob_setting_gives_the_oracles_groups(knobs):
    """pf_join_aggregate_ex with the autotuner's knobs set by hand: the join's
    table, the sub-partition size, counted passes and the round path all
    give the same groups."""
    w = datagen.scaled(datagen.SCALE, 1 / 400)   # 375K x 1.5M, 3750 groups
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 0, w.n_groups)
    for B in (16, 128):
        plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda", B=B, knobs=knobs)
        _assert_groups(plan.run(bkey, bgrp, fk, price, disc), want)
        assert plan.read_stats().matched == want[3]


def test_fingerprint_table_with_extreme_and_skewed_keys():
    """The fingerprinted table reserves no hash as a free mark: the key whose
    mix64 is 2^63 and INT64_MIN / INT64_MAX join like any other; skewed
    probe keys take the counted passes."""
    knobs = dict(path=0, table=1, sub_rows=0, counted=0)
    I = np.iinfo(np.int64)
    ks = _unmix64(1 << 63)
    bkey = torch.tensor([I.min, I.max, 0, -1, 5, I.min + 1, ks], dtype=torch.int64).cuda()
    bgrp = torch.tensor([0, 1, 2, 3, 4, 5, 6], dtype=torch.int32).cuda()
    fk = torch.tensor([I.min, I.min, I.max, 7, -1, I.min + 1, 0, I.min, ks, ks, ks + 1],
                      dtype=torch.int64).cuda()
    price = torch.arange(1, 12, dtype=torch.int64).cuda() * 1000
    disc = torch.zeros(11, dtype=torch.int64).cuda()
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 0, 7)
    for B in (1, 4):
        plan = JoinAggregate(7, 11, 0, 7, "cuda", B=B, knobs=knobs)
        _assert_groups(plan.run(bkey, bgrp, fk, price, disc), want)
    g = torch.Generator().manual_seed(22)
    nb, np_ = 100_000, 1_000_000
    bkey = torch.randperm(4 * nb, generator=g)[:nb].to(torch.int64) * 7919 - (1 << 41)
    bgrp = torch.randint(0, 2_000, (nb,), generator=g, dtype=torch.int32)
    ranks = torch.rand(np_, generator=g).pow(8).mul(nb).to(torch.int64).clamp_(max=nb - 1)
    args = [t.cuda() for t in (bkey, bgrp, bkey[ranks], torch.randint(0, 1 << 30, (np_,),
                                                                   generator=g),
                               torch.randint(0, 11, (np_,), generator=g))]
    want = _oracle_groups(*args, 0, 2_000)
    plan = JoinAggregate(nb, np_, 0, 2_000, "cuda", B=32, knobs=knobs)
    _assert_groups(plan.run(*args), want)


def test_autotuned_plan_matches_the_oracle_and_caches_its_choice(tmp_path, monkeypatch):
    monkeypatch.setenv("PAGEFLOW_TUNE_CACHE", str(tmp_path / "tune.json"))
    for v in ("PF_JOIN_PATH", "PF_SJ_FP", "PF_SJ_TARGET", "PF_COUNTED"):
        monkeypatch.delenv(v, raising=False)
    w = datagen.scaled(datagen.SCALE, 1 / 200)   # 750K x 3M, 7500 groups
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    want = _oracle_groups(bkey, bgrp, fk, price, disc, 0, w.n_groups)
    plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda")
    assert plan.autotune
    _assert_groups(plan.run(bkey, bgrp, fk, price, disc), want)
    t = plan.tuning
    assert t is not None and not t.cached and len(t.times_ms) >= 5
    assert plan.B == t.choice.B and all(v > 0 for v in t.times_ms.values())
    again = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda")
    _assert_groups(again.run(bkey, bgrp, fk, price, disc), want)
    assert again.tuning.cached and again.tuning.choice == t.choice
