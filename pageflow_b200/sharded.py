"""The fused join + group-by sharded over ranks, one process a GPU.

Each rank holds a slice of both sides.  A join key's owner is the rank that
owns its first-pass bucket (the top log2(B) bits of mix64(key); rank r owns
buckets [r*B/W, (r+1)*B/W)), so the exchange moves whole buckets:

  1. partition: each rank hashes and radix-partitions its own rows into B
     contiguous buckets (pf_join_partition: build rows as (hash, group),
     probe rows as {hash, value} records) and learns every rank's bucket
     rows (one all-gather of 2B counts a rank);
  2. exchange: every bucket goes to its owner, one point-to-point message a
     (bucket, side column, peer), batched into one group of sends and
     receives; a rank receives each bucket's pieces from every rank one
     after another, so each of its buckets arrives contiguous;
  3. join: each rank runs the second radix pass and the shared-memory join
     over the buckets it owns (pf_join_aggregate_buckets) into a dense slab
     of every group;
  4. the ranks' slabs are added (one int64 all-reduce of sums and counts;
     int64 sums wrap modulo 2^64 as the single-GPU join's do).

The rank-local phases run behind a backend: CudaPhases (the library's
kernels) is the product's; the exchange and the reduction take the process
group's backend (NCCL on GPUs).  Point-to-point messages carry no bulk copy
from a peer's memory and no multicast.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional

import torch
import torch.distributed as dist

from . import _native as N


def owned_buckets(rank: int, world: int, B: int) -> range:
    """The buckets rank ``rank`` of ``world`` owns: a contiguous run."""
    return range(rank * B // world, (rank + 1) * B // world)


class ExchangePlan:
    """Where rank r's buckets lie before the exchange and where its own
    buckets land after it: ``starts[side][b]`` the first row of bucket b in
    r's partitioned side; ``recv_off[side][(q, s)]`` the first row of the
    piece of bucket q from rank s in r's receive buffer (r's buckets in
    order, each one's pieces by source rank, so each bucket is contiguous);
    ``counts[side][i]`` the rows of r's i-th bucket."""

    def __init__(self, mine, starts, recv_off, counts):
        self.mine, self.starts, self.recv_off, self.counts = mine, starts, recv_off, counts


def exchange_plan(allc: List[List[List[int]]], r: int, W: int, B: int) -> ExchangePlan:
    """The plan of rank r from every rank's bucket rows, allc[s][side][b]."""
    mine = owned_buckets(r, W, B)
    starts = []
    for side in range(2):
        run, st = 0, []
        for b in range(B):
            st.append(run)
            run += allc[r][side][b]
        starts.append(st)
    counts = [[sum(allc[s][side][q] for s in range(W)) for q in mine] for side in range(2)]
    recv_off = []
    for side in range(2):
        offs, run = {}, 0
        for q in mine:
            for s in range(W):
                offs[(q, s)] = run
                run += allc[s][side][q]
        recv_off.append(offs)
    return ExchangePlan(mine, starts, recv_off, counts)


class CudaPhases:
    """The rank-local phases on this GPU (libpageflow_b200.so)."""

    def __init__(self, device, knobs: Optional[dict] = None):
        self.device = torch.device(device)
        self.knobs = None if knobs is None else N.JoinKnobs(**knobs)

    def partition(self, bkey, bgrp, fk, price, disc, scale: int, B: int):
        """(build hash, build group, probe records [n, 2], counts int64 [2, B]
        on the host): both sides in B contiguous buckets."""
        nb, npr = bkey.numel(), fk.numel()
        L = N.lib()
        bh = torch.empty(nb, dtype=torch.int64, device=self.device)
        bg = torch.empty(nb, dtype=torch.int32, device=self.device)
        pr = torch.empty((npr, 2), dtype=torch.int64, device=self.device)
        counts = torch.zeros((2, B), dtype=torch.int64, pin_memory=True)
        with torch.cuda.device(self.device):
            ws_bytes = L.pf_join_partition_workspace(nb, npr, B)
            ws = N.workspace(ws_bytes, self.device)
            N.check(L.pf_join_partition(bkey.data_ptr(), bgrp.data_ptr(), nb, fk.data_ptr(),
                                        price.data_ptr(), N.ptr(disc), scale, npr, B,
                                        bh.data_ptr(), bg.data_ptr(), pr.data_ptr(),
                                        counts.data_ptr(), ws.data_ptr(), ws_bytes,
                                        N.stream_of(self.device)), "join_partition")
        return bh, bg, pr, counts.clone()

    def join_buckets(self, bh, bg, pr, counts, logB: int, group_min: int, n_groups: int):
        """(sums, counts) [n_groups] of the buckets this rank holds."""
        L = N.lib()
        c = counts.to(torch.int64).contiguous()
        nbk = c.shape[1]
        sums = torch.empty(n_groups, dtype=torch.int64, device=self.device)
        cnts = torch.empty(n_groups, dtype=torch.int64, device=self.device)
        stats = torch.zeros(4, dtype=torch.int64, device=self.device)
        kn = None if self.knobs is None else ctypes.byref(self.knobs)
        with torch.cuda.device(self.device):
            ws_bytes = L.pf_join_aggregate_buckets_workspace(c.data_ptr(), nbk, n_groups, kn)
            ws = N.workspace(ws_bytes, self.device)
            N.check(L.pf_join_aggregate_buckets(
                bh.data_ptr(), bg.data_ptr(), pr.data_ptr(), c.data_ptr(), nbk, logB, group_min,
                n_groups, sums.data_ptr(), cnts.data_ptr(), stats.data_ptr(), kn,
                ws.data_ptr(), ws_bytes, N.stream_of(self.device)), "join_aggregate_buckets")
        return sums, cnts


class ShardedJoinAggregate:
    """SELECT group, SUM(price * (scale - disc)), COUNT(*) over the ranks'
    rows of a unique-build FK join: every rank gets the dense (sums,
    counts) of [group_min, group_min + n_groups)."""

    def __init__(self, group_min: int, n_groups: int, B: int, scale: int = 100,
                 phases=None, group=None):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        if B < self.world or B & (B - 1) or B > 4096:
            raise ValueError(f"B={B}: a power of two in [world size {self.world}, 4096]")
        self.B = B
        self.logB = B.bit_length() - 1
        self.group_min, self.n_groups, self.scale = int(group_min), int(n_groups), int(scale)
        self.phases = phases
        self.last = {}

    def _device(self):
        return self.phases.device

    def run(self, bkey, bgrp, fk, price, disc=None):
        W, r, B = self.world, self.rank, self.B
        dev = self._device()
        bh, bg, pr, counts = self.phases.partition(bkey, bgrp, fk, price, disc, self.scale, B)
        # every rank's bucket rows
        c = counts.to(dev)
        every = [torch.empty_like(c) for _ in range(W)]
        dist.all_gather(every, c, group=self.group)
        allc = torch.stack(every).cpu().tolist()          # [W][2][B]
        plan = exchange_plan(allc, r, W, B)
        mine, starts, recv_off, recv_counts = plan.mine, plan.starts, plan.recv_off, plan.counts
        nrows = [sum(recv_counts[0]), sum(recv_counts[1])]
        rh = torch.empty(nrows[0], dtype=torch.int64, device=dev)
        rg = torch.empty(nrows[0], dtype=torch.int32, device=dev)
        rp = torch.empty((nrows[1], 2), dtype=torch.int64, device=dev)
        cols = [(0, bh, rh), (0, bg, rg), (1, pr, rp)]
        ops = []
        for side, src, dst in cols:
            # sends: each peer's buckets, bucket by bucket
            for d in range(W):
                for q in owned_buckets(d, W, B):
                    n = allc[r][side][q]
                    if n == 0:
                        continue
                    piece = src[starts[side][q]:starts[side][q] + n]
                    if d == r:
                        o = recv_off[side][(q, r)]
                        dst[o:o + n].copy_(piece)
                    else:
                        ops.append(dist.P2POp(dist.isend, piece, d, self.group))
            # receives: every peer's pieces of my buckets, in the same order
            for s in range(W):
                if s == r:
                    continue
                for q in mine:
                    n = allc[s][side][q]
                    if n == 0:
                        continue
                    o = recv_off[side][(q, s)]
                    ops.append(dist.P2POp(dist.irecv, dst[o:o + n], s, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        del bh, bg, pr
        bucket_counts = torch.tensor(recv_counts, dtype=torch.int64)
        if len(mine):
            sums, cnts = self.phases.join_buckets(rh, rg, rp, bucket_counts, self.logB,
                                                  self.group_min, self.n_groups)
        else:
            sums = torch.zeros(self.n_groups, dtype=torch.int64, device=dev)
            cnts = torch.zeros(self.n_groups, dtype=torch.int64, device=dev)
        self.last = {"received_rows": nrows,
                     "kept_rows": [sum(allc[r][side][q] for q in mine) for side in range(2)]}
        dist.all_reduce(sums, group=self.group)
        dist.all_reduce(cnts, group=self.group)
        return sums, cnts


def dense_groups(sums: torch.Tensor, counts: torch.Tensor, group_min: int):
    """(keys, sums, counts) of the groups present (count > 0), ascending."""
    keep = counts > 0
    keys = torch.nonzero(keep).view(-1) + group_min
    return keys, sums[keep], counts[keep]

