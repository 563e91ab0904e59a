"""Generates the golden vectors under tests/golden from PageFlow's own Python
code, imported read-only from a checkout of the reference (its compiled
TQPlib modules are replaced by empty stand-ins: only pure-torch code runs).
Run where the reference is present:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py /path/to/PageFlow

Writes (all small):
  mix64.npz            operators/aggregate.py:_mix64 on extremes and random int64
  buckets.npz          operators/aggregate.py:_bucket_ids for B in 1..4096
  partition_layout.npz operators/aggregate.py:_partition_outputs (the padded
                       bucket layout, bucket rows only) and
                       IO/codec/batched_compress.py:aligned_partition_layout
  partitions.json      operators/partitions.py: max_load, partition_count,
                       agg_partitions over a grid of inputs
  slab.json            operators/aggregation_slab.py:DenseAggregationSlab vectors
  sorted_run.npz       operators/sorted_run_merge.py: reduce_tick_slice and
                       merge_sorted_unique_runs_inplace on random runs
  join_small.npz       operators/hashjoin.py:_sort_search_pairs pairs for unique
                       builds (one and two keys), the expand step restated from
                       tests/operators/test_join_core.py:55-61
  config0.npz          the small workload (250K x 1M, seed 0) end to end:
                       the join by _sort_search_pairs, then KeyedAggregate.pass1
                       + reduce_tick_slice (SUM(price*(100-disc)), COUNT by group)
Inputs of config0 come from this repository's oracle generator; the fixture
keeps a checksum of them so a generator change is caught.
"""
from __future__ import annotations

import json
import sys
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def import_reference(root: str):
    sys.dont_write_bytecode = True
    sys.path.insert(0, root)
    for name in ["TQPlib.tqpkernels.tqpkernels", "TQPlib.tqpcompress.tqpcompress",
                 "TQPlib.tqpmemory.tqpmemory", "TQPlib.tqpcache.tqpcache",
                 "TQPlib.zero_copy_reader.zero_copy_reader", "TQPlib.tqpkernels",
                 "TQPlib.tqpcompress", "TQPlib.tqpmemory", "TQPlib.tqpcache",
                 "TQPlib.zero_copy_reader"]:
        sys.modules[name] = types.ModuleType(name)
    sys.modules["TQPlib.tqpcache.tqpcache"].split_at_granules = None
    sys.modules["TQPlib.tqpcache"].split_at_granules = None


def expand_cpu(sorted_ids, start, length):
    """The pairs of each probe row's run (the repeat_interleave form of the
    reference test's expand reference)."""
    rows = torch.arange(length.numel())
    cr = torch.repeat_interleave(rows, length)
    first = torch.repeat_interleave(start, length)
    run0 = torch.repeat_interleave(torch.cumsum(length, 0) - length, length)
    within = torch.arange(cr.numel()) - run0
    return sorted_ids[first + within], cr


def main(root: str) -> None:
    import_reference(root)
    from IO.codec.batched_compress import aligned_partition_layout
    from operators import aggregate, hashjoin, join_core, partitions
    from operators.aggregation_slab import DenseAggregationSlab
    from operators.sorted_run_merge import (merge_sorted_unique_runs_inplace,
                                            reduce_tick_slice)
    from uvm.column import UColumn

    sys.path.insert(0, str(REPO))
    import oracle

    rng = np.random.default_rng(2029)
    i64 = np.iinfo(np.int64)

    # -- mix64 / buckets
    h = rng.integers(i64.min, i64.max, 4096, dtype=np.int64)
    h[:8] = [0, 1, -1, i64.min, i64.max, 1 << 33, -(1 << 33), 42]
    mixed = aggregate._mix64(torch.from_numpy(h)).numpy()
    np.savez_compressed(HERE / "mix64.npz", keys=h, mix=mixed)
    bk = {}
    for B in (1, 2, 8, 64, 256, 512, 1024, 4096):
        bk[f"B{B}"] = aggregate._bucket_ids(torch.from_numpy(h), B).numpy()
    np.savez_compressed(HERE / "buckets.npz", keys=h, **bk)

    # -- the padded partition layout (pass 1's _partition_outputs)
    lay = {}
    for case, (B, n) in enumerate([(2, 1), (8, 63), (64, 1000), (256, 7001)]):
        g = torch.Generator().manual_seed(B * 7919 + n)
        used = torch.randperm(B, generator=g)[:max(1, B * 3 // 4)]
        bucket = used[torch.randint(0, len(used), (n,), generator=g)].to(torch.int32)
        outs = [torch.randint(-2 ** 62, 2 ** 62, (n,), dtype=torch.int64, generator=g),
                torch.randint(-128, 127, (n,), dtype=torch.int8, generator=g),
                torch.randint(-128, 127, (n, 25), dtype=torch.int8, generator=g)]
        counts_t = torch.bincount(bucket, minlength=B)
        counts = counts_t.tolist()
        got = aggregate._partition_outputs(outs, bucket, counts, counts_t)
        lay[f"c{case}_B"] = np.array([B])
        lay[f"c{case}_bucket"] = bucket.numpy()
        lay[f"c{case}_counts"] = counts_t.numpy()
        for j, (t, pt) in enumerate(zip(outs, got)):
            rb = t.element_size() * (t.shape[1] if t.dim() == 2 else 1)
            unit = rb * 512 // np.gcd(rb, 512)
            padded, starts, total = aligned_partition_layout(counts, rb, unit)
            lay[f"c{case}_in{j}"] = t.numpy()
            lay[f"c{case}_total{j}"] = np.array([total, pt.tensor.shape[0]])
            lay[f"c{case}_starts{j}"] = np.array(pt.bucket_starts())
            rows = [pt.tensor[s // rb: s // rb + c] for s, c in zip(starts, counts)]
            lay[f"c{case}_rows{j}"] = torch.cat(rows).numpy()
    np.savez_compressed(HERE / "partition_layout.npz", **lay)

    # -- the partition-count rule
    rule = {"max_load": [], "partition_count": [], "agg_partitions": []}
    for m in (0, 1, 5, 31, 100, 1000, 4096, 10 ** 6, 1.5e8):
        for n in (1, 2, 16, 64, 512, 4096):
            rule["max_load"].append([m, n, partitions.max_load(m, n)])
    for parts, budget, bmax in [
            ([(150_000_000, 12), (600_000_000, 16)], 512 << 20, 512),
            ([(250_000, 12), (1_000_000, 16)], 512 << 20, 512),
            ([(1000, 8, 10)], 100, 512), ([(10 ** 9, 24, 3)], 1 << 20, 512),
            ([(5_000_000, 24)], 256 << 10, 256), ([], 1, 512)]:
        rule["partition_count"].append(
            [parts, budget, bmax, list(partitions.partition_count(parts, budget, bmax))])
    for args in [(10 ** 8, 100, 1_500_000, 24, None, 512 << 20),
                 (10 ** 6, 4, 25, 24, 25, 512 << 20),
                 (10 ** 9, 1000, None, 40, None, 256 << 20),
                 (5_000_000, 10, 4_000_000, 16, 8_000_000, 1 << 20)]:
        rule["agg_partitions"].append([list(args), list(partitions.agg_partitions(*args))])
    rule["JOIN_B_MAX"] = partitions.JOIN_B_MAX
    rule["AGG_B_MAX"] = partitions.AGG_B_MAX
    (HERE / "partitions.json").write_text(json.dumps(rule, indent=0))

    # -- slab vectors
    slab = []
    for seed in range(4):
        g = torch.Generator().manual_seed(100 + seed)
        lo, hi = -5 + seed, 40 + 3 * seed
        specs = [(torch.int64, ()), (torch.int64, ()), (torch.int64, ()), (torch.float64, (2,))]
        ops = ["sum", "amax", "amin", "sum"]
        s = DenseAggregationSlab(lo, hi, torch.int64, specs, ops, "cpu")
        ticks = []
        for t in range(3):
            n = 50 + 17 * t
            k = torch.randint(lo, hi + 1, (n,), generator=g)
            v1 = torch.randint(-1000, 1000, (n,), generator=g)
            v2 = torch.randint(-1000, 1000, (n,), generator=g)
            v3 = torch.randint(-1000, 1000, (n,), generator=g)
            v4 = torch.randint(0, 64, (n, 2), generator=g).to(torch.float64)
            s.add(k, [v1, v2, v3, v4])
            ticks.append([k.tolist(), v1.tolist(), v2.tolist(), v3.tolist(), v4.tolist()])
        keys, vals = s.finish()
        slab.append({"lo": lo, "hi": hi, "ops": ops, "ticks": ticks, "keys": keys.tolist(),
                     "vals": [v.tolist() for v in vals]})
    (HERE / "slab.json").write_text(json.dumps(slab))

    # -- sorted-run merge
    sr = {}
    for case in range(3):
        g = torch.Generator().manual_seed(7 + case)
        keys = torch.randint(-50, 50 + 100 * case, (300 + 50 * case,), generator=g)
        v = torch.randint(-10 ** 6, 10 ** 6, (keys.numel(),), generator=g)
        w = torch.randint(-10 ** 6, 10 ** 6, (keys.numel(),), generator=g)
        u, (rs, rm) = reduce_tick_slice(keys, [v, w], ["sum", "amax"])
        sr[f"c{case}_keys"], sr[f"c{case}_v"], sr[f"c{case}_w"] = keys.numpy(), v.numpy(), w.numpy()
        sr[f"c{case}_u"], sr[f"c{case}_sum"], sr[f"c{case}_max"] = u.numpy(), rs.numpy(), rm.numpy()
        half = keys.numel() // 2
        ua, (sa,) = reduce_tick_slice(keys[:half], [v[:half]], ["sum"])
        ub, (sb,) = reduce_tick_slice(keys[half:], [v[half:]], ["sum"])
        kb = torch.empty(ua.numel() + ub.numel(), dtype=torch.int64)
        vb = torch.empty_like(kb)
        kb[:ua.numel()], vb[:ua.numel()] = ua, sa
        m = merge_sorted_unique_runs_inplace(kb, [vb], ua.numel(), ub, [sb], ["sum"],
                                             place_chunk_rows=7)
        sr[f"c{case}_merged_keys"], sr[f"c{case}_merged_sum"] = kb[:m].numpy(), vb[:m].numpy()
    np.savez_compressed(HERE / "sorted_run.npz", **sr)

    # -- unique-build joins through _sort_search_pairs
    join_core.expand = expand_cpu
    hashjoin.join_core.expand = expand_cpu
    js = {}
    g = torch.Generator().manual_seed(11)
    for two in (False, True):
        nb, npr = 3000, 5000
        k0 = torch.randperm(nb * 4, generator=g)[:nb].to(torch.int64)
        picks = torch.randint(0, nb, (npr,), generator=g)
        miss = torch.randint(0, 4, (npr,), generator=g) == 0
        p0 = torch.where(miss, k0[picks] + nb * 8, k0[picks])
        if two:
            bl, pl = [k0 // 3, k0 % 3], [p0 // 3, p0 % 3]
            # the sort/search core joins on the first key; the second filters
            li, ri = hashjoin._sort_search_pairs({}, {}, bl[0], pl[0], [], None,
                                                 torch.device("cpu"))
            keep = bl[1][li] == pl[1][ri]
            li, ri = li[keep], ri[keep]
        else:
            bl, pl = [k0], [p0]
            li, ri = hashjoin._sort_search_pairs({}, {}, k0, p0, [], None, torch.device("cpu"))
        order = torch.argsort(ri, stable=True)
        tag = "two" if two else "one"
        js[f"{tag}_b0"], js[f"{tag}_p0"] = bl[0].numpy(), pl[0].numpy()
        if two:
            js[f"{tag}_b1"], js[f"{tag}_p1"] = bl[1].numpy(), pl[1].numpy()
        js[f"{tag}_build_idx"], js[f"{tag}_probe_idx"] = li[order].numpy(), ri[order].numpy()
    np.savez_compressed(HERE / "join_small.npz", **js)

    # -- the small workload end to end through the reference's operators
    bkey, bgrp = oracle.gen_build(0, 250_000, 25)
    fk, price, disc = oracle.gen_probe(0, 0, 250_000, 0, 1_000_000)
    tb, tg = torch.from_numpy(bkey), torch.from_numpy(bgrp)
    tf, tp, td = torch.from_numpy(fk), torch.from_numpy(price), torch.from_numpy(disc)
    li, ri = hashjoin._sort_search_pairs({}, {}, tb, tf, [], None, torch.device("cpu"))
    grp = tg[li]
    pr = tp[ri]
    dc = td[ri]
    results = [["grp#1"],
               [[[['sum', [['price#2', '*', ['100', '-', 'disc#3']]]], '#', '9001'], 'AS', 'out#200']],
               [[[['count', ['1']], '#', '9001'], 'AS', 'out#201']]]
    args = {'name': 'Aggregate', 'keys': ['grp#1'], 'input ids': [1, 2, 3],
            'results': results, 'out key ids': [1], 'out agg ids': [200, 201],
            'agg ops': ['sum', 'count'], 'output ids': [1, 200, 201]}
    tgroup = {1: UColumn(grp, 'int'), 2: UColumn(pr, 'int'), 3: UColumn(dc, 'int')}
    spec = aggregate.KeyedAggregate(args, tgroup, [1, 2, 3], [torch.int32, torch.int64, torch.int64])
    # two morsels, as the UVM executor would feed pass 1, merged by pass 2
    half = grp.numel() // 2
    parts = []
    for a, b in ((0, half), (half, grp.numel())):
        outs, _ = spec.pass1('cpu', {1: grp[a:b], 2: pr[a:b], 3: dc[a:b]}, 1)
        parts.append(outs)
    cat = [torch.cat([p[i] for p in parts]) for i in range(4)]
    _, merged = reduce_tick_slice(cat[0], cat[1:], ['amax'] + spec.merge_ops)
    order = torch.argsort(merged[0])
    np.savez_compressed(
        HERE / "config0.npz", groups=merged[0][order].numpy().astype(np.int64),
        sums=merged[1][order].numpy(), counts=merged[2][order].numpy(),
        matched=np.array([li.numel()]),
        input_checksum=np.array([int(np.bitwise_xor.reduce(bkey.view(np.uint64))),
                                 int(np.bitwise_xor.reduce(fk.view(np.uint64))),
                                 int(price.sum()), int(disc.sum()), int(bgrp.sum())],
                                dtype=np.uint64))
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    import os
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PAGEFLOW_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout> (or set PAGEFLOW_REFERENCE)")
    main(ref)
