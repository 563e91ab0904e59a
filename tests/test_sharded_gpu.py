"""The sharded join's two rank-local phases on the GPU (pf_join_partition,
pf_join_aggregate_buckets), with W ranks emulated one after another on one
device: each emulated rank partitions its slice, the buckets are moved to
their owners by the exchange plan (device copies in place of the
point-to-point messages), each owner joins its buckets, and the owners'
slabs are added.  The result must equal the oracle's join + group-by of the
whole input.  No kernel waits on another rank's."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from pageflow_b200 import datagen
from pageflow_b200.sharded import CudaPhases, dense_groups, exchange_plan, owned_buckets

pytestmark = pytest.mark.gpu


def _emulate(world, B, inputs, G, knobs=None):
    bkey, bgrp, fk, price, disc = inputs
    nb, npr = bkey.numel(), fk.numel()
    bcut = [nb * r // world for r in range(world + 1)]
    pcut = [npr * r // world + (r % 2) * 7 * (0 < r < world) for r in range(world + 1)]
    ph = CudaPhases("cuda", knobs)
    parts = []
    for r in range(world):
        sb, sp = slice(bcut[r], bcut[r + 1]), slice(pcut[r], pcut[r + 1])
        parts.append(ph.partition(bkey[sb], bgrp[sb], fk[sp], price[sp], disc[sp], 100, B))
    allc = [p[3].tolist() for p in parts]
    total_s = torch.zeros(G, dtype=torch.int64, device="cuda")
    total_c = torch.zeros(G, dtype=torch.int64, device="cuda")
    for r in range(world):
        plan = exchange_plan(allc, r, world, B)
        n = [sum(plan.counts[0]), sum(plan.counts[1])]
        rh = torch.empty(n[0], dtype=torch.int64, device="cuda")
        rg = torch.empty(n[0], dtype=torch.int32, device="cuda")
        rp = torch.empty((n[1], 2), dtype=torch.int64, device="cuda")
        for side, dst, k in ((0, rh, 0), (0, rg, 1), (1, rp, 2)):
            for s in range(world):
                starts = exchange_plan(allc, s, world, B).starts
                for q in owned_buckets(r, world, B):
                    c = allc[s][side][q]
                    if c:
                        o = plan.recv_off[side][(q, s)]
                        dst[o:o + c].copy_(parts[s][k][starts[side][q]:starts[side][q] + c])
        if len(plan.mine):
            s_, c_ = ph.join_buckets(rh, rg, rp, torch.tensor(plan.counts), B.bit_length() - 1,
                                     0, G)
            total_s += s_
            total_c += c_
    return dense_groups(total_s, total_c, 0)


@pytest.mark.parametrize("world,B", [(2, 64), (3, 256), (8, 256), (4, 1024)])
def test_emulated_ranks_match_the_oracle(world, B):
    w = datagen.scaled(datagen.SCALE, 1 / 300)    # 500K x 2M, 5000 groups
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    s, c, _, _ = oracle.join_aggregate(bkey.cpu().numpy(), bgrp.cpu().numpy(),
                                       fk.cpu().numpy(), price.cpu().numpy(),
                                       disc.cpu().numpy(), 100, 0, w.n_groups, B=16)
    present = np.nonzero(c)[0]
    for knobs in (None, dict(path=0, table=1, sub_rows=0, counted=1)):
        keys, sums, counts = _emulate(world, B, (bkey, bgrp, fk, price, disc), w.n_groups,
                                      knobs)
        assert np.array_equal(keys.cpu().numpy(), present)
        assert np.array_equal(sums.cpu().numpy(), s[present])
        assert np.array_equal(counts.cpu().numpy(), c[present])


def test_partition_phase_is_the_oracles_bucket_layout():
    w = datagen.scaled(datagen.SCALE, 1 / 3000)   # 50K x 200K
    bkey, bgrp = datagen.gen_build(w, "cuda")
    fk, price, disc = datagen.gen_probe(w, "cuda")
    B = 128
    bh, bg, pr, counts = CudaPhases("cuda").partition(bkey, bgrp, fk, price, disc, 100, B)
    bk = bkey.cpu().numpy()
    assert counts[0].tolist() == np.bincount(oracle.bucket(bk, B), minlength=B).tolist()
    assert counts[1].tolist() == np.bincount(oracle.bucket(fk.cpu().numpy(), B),
                                             minlength=B).tolist()
    h = bh.cpu().numpy()
    assert np.array_equal(np.sort(h), np.sort(oracle.mix64(bk).view(np.int64)))
    # every bucket's rows carry that bucket's top bits, and each row its group
    top = (h.view(np.uint64) >> np.uint64(57)).astype(np.int64)
    assert np.array_equal(top, np.repeat(np.arange(B), counts[0].tolist()))
    by_hash = dict(zip(oracle.mix64(bk).view(np.int64).tolist(), bgrp.cpu().numpy().tolist()))
    assert all(by_hash[x] == y for x, y in zip(h[:2000].tolist(), bg.cpu().numpy()[:2000]))
    val = (price * (100 - disc)).cpu().numpy()
    ph = pr[:, 0].cpu().numpy()
    assert np.array_equal(np.sort(ph), np.sort(oracle.mix64(fk.cpu().numpy()).view(np.int64)))
    assert np.array_equal(np.sort(pr[:, 1].cpu().numpy()), np.sort(val))
