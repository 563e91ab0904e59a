"""The sharded join + group-by's exchange over world_size 2 and 3 gloo ranks
on CPU (no GPU): each rank holds a slice of both sides; the rank-local phases
are the oracle's (hash, stable radix partition by the top bits of mix64,
join by hash), the exchange, ownership and reduction are the product's
(pageflow_b200.sharded).  Every rank's result must equal the oracle's join +
group-by of the whole input."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle


class OraclePhases:
    """The two rank-local phases restated on the CPU from the oracle."""

    device = torch.device("cpu")

    def partition(self, bkey, bgrp, fk, price, disc, scale, B):
        bk, fkn = bkey.numpy(), fk.numpy()
        bb = oracle.bucket(bk, B).astype(np.int64)
        pb = oracle.bucket(fkn, B).astype(np.int64)
        ob = np.argsort(bb, kind="stable")
        op = np.argsort(pb, kind="stable")
        bh = oracle.mix64(bk).view(np.int64)[ob]
        val = price.numpy() * (scale - disc.numpy()) if disc is not None else price.numpy()
        pr = np.stack([oracle.mix64(fkn).view(np.int64)[op], val[op]], axis=1)
        counts = np.stack([np.bincount(bb, minlength=B), np.bincount(pb, minlength=B)])
        return (torch.from_numpy(bh.copy()), torch.from_numpy(bgrp.numpy()[ob].copy()),
                torch.from_numpy(np.ascontiguousarray(pr)), torch.from_numpy(counts))

    def join_buckets(self, bh, bg, pr, counts, logB, group_min, n_groups):
        h, g = bh.numpy(), bg.numpy().astype(np.int64)
        order = np.argsort(h, kind="stable")
        hs = h[order]
        ph, pv = pr[:, 0].numpy(), pr[:, 1].numpy()
        pos = np.searchsorted(hs, ph)
        pos_c = np.minimum(pos, max(len(hs) - 1, 0))
        hit = (pos < len(hs)) & (hs[pos_c] == ph) if len(hs) else np.zeros(len(ph), bool)
        grp = g[order][pos_c[hit]] - group_min
        ok = (grp >= 0) & (grp < n_groups)
        sums = np.zeros(n_groups, np.int64)
        cnts = np.zeros(n_groups, np.int64)
        np.add.at(sums, grp[ok], pv[hit][ok])
        np.add.at(cnts, grp[ok], 1)
        # every bucket's rows share their top logB hash bits
        return torch.from_numpy(sums), torch.from_numpy(cnts)


def _data(seed, nb, npr, G):
    g = torch.Generator().manual_seed(seed)
    bkey = torch.randperm(4 * nb, generator=g)[:nb].to(torch.int64) * 104729 - (1 << 45)
    bgrp = torch.randint(0, G, (nb,), generator=g, dtype=torch.int32)
    fk = bkey[torch.randint(0, nb, (npr,), generator=g)]
    fk = torch.where(torch.rand(npr, generator=g) < 0.15, fk + 1, fk)
    price = torch.randint(90_000, 10_500_000, (npr,), generator=g)
    disc = torch.randint(0, 11, (npr,), generator=g)
    return bkey, bgrp, fk, price, disc


def _rank_main(rank, world, port, B, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pageflow_b200.sharded import ShardedJoinAggregate, dense_groups
        nb, npr, G = 20_000, 90_000, 300
        bkey, bgrp, fk, price, disc = _data(7, nb, npr, G)
        # each rank holds an uneven slice of both sides
        bs = [0, nb // 3, nb] if world == 2 else [0, nb // 5, nb // 2, nb]
        ps = [0, npr // 2 + 17, npr] if world == 2 else [0, npr // 4, npr // 2 + 5, npr]
        sl = slice(bs[rank], bs[rank + 1])
        pl = slice(ps[rank], ps[rank + 1])
        job = ShardedJoinAggregate(0, G, B, scale=100, phases=OraclePhases())
        sums, cnts = job.run(bkey[sl], bgrp[sl], fk[pl], price[pl], disc[pl])
        keys, s, c = dense_groups(sums, cnts, 0)
        out_q.put((rank, keys.numpy(), s.numpy(), c.numpy(), job.last))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,B", [(2, 2), (2, 16), (3, 8), (3, 64)])
def test_sharded_exchange_matches_the_oracle(world, B):
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, B, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    results = [q.get() for _ in range(world)]
    bkey, bgrp, fk, price, disc = _data(7, 20_000, 90_000, 300)
    s, c, matched, _ = oracle.join_aggregate(bkey.numpy(), bgrp.numpy(), fk.numpy(),
                                              price.numpy(), disc.numpy(), 100, 0, 300, B=8)
    present = np.nonzero(c)[0]
    received = [0, 0]
    for rank, keys, sums, cnts, last in results:
        assert np.array_equal(keys, present)
        assert np.array_equal(sums, s[present]) and np.array_equal(cnts, c[present])
        received[0] += last["received_rows"][0]
        received[1] += last["received_rows"][1]
    # every row went to exactly one owner
    assert received == [20_000, 90_000]
    assert int(c.sum()) == matched


def test_ownership_covers_every_bucket_once():
    from pageflow_b200.sharded import owned_buckets
    for world in (1, 2, 3, 5, 8):
        for B in (8, 64, 256):
            if B < world:
                continue
            seen = [b for r in range(world) for b in owned_buckets(r, world, B)]
            assert seen == list(range(B))
