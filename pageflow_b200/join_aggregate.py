"""The fused join -> group-by on sm_100a (pf_join_aggregate_ex): two radix
passes of both sides into sub-partitions, a shared-memory hash table per
sub-partition, probe rows aggregated into their build row's cell and each
build row flushed once into a dense group slab, then the occupied groups
compacted.  The fan-out and the join's table are picked by the autotuner
(pageflow_b200.autotune) unless given.

    keys, sums, counts = join_group_aggregate(build_key, build_group,
                                              probe_fk, price, disc)

computes ``SELECT group, SUM(price * (scale - disc)), COUNT(*) FROM build
JOIN probe ON build.key = probe.fk GROUP BY group`` for a unique build key:
the result the reference produces by partition_sort -> join_unique_hash ->
index_select -> KeyedAggregate.pass1 -> reduce_tick_slice (uvm/join.py,
uvm/aggregate.py), with exact int64 sums.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Optional

import torch

from . import _native as N


# Environment overrides of the knobs (for sweeps and tests); while one is set
# the autotuner stays off.
_OVERRIDES = ("PF_JOIN_PATH", "PF_SJ_FP", "PF_SJ_TARGET", "PF_COUNTED")


@dataclass
class JoinAggregateStats:
    matched: int          # probe rows that found their build row
    bad_groups: int       # build rows whose group lay outside the range
    overflow: int         # build rows no table slot took (0 unless broken)
    device_error: int     # nonzero: a kernel gave up a bounded wait (results invalid)


class JoinAggregate:
    """A reusable plan for one input shape: its workspace and output slabs
    are allocated once, so repeated ``run`` calls allocate nothing (and the
    queued work can be timed or captured as is)."""

    def __init__(self, n_build: int, n_probe: int, group_min: int, n_groups: int,
                 device, B: Optional[int] = None, scale: int = 100,
                 knobs: Optional[dict] = None, autotune: Optional[bool] = None):
        """``B`` and ``knobs`` (pf_join_knobs fields: path, table, sub_rows,
        counted) fix the launch configuration; with neither given (and no
        PF_* override in the environment) the first ``aggregate`` call picks
        B, table and sub_rows by timing candidates on its inputs (a cached
        choice of the shape class is used as is); with autotune=False, B
        comes from pf_join_aggregate_pick_b."""
        self.n_build, self.n_probe = int(n_build), int(n_probe)
        self.group_min, self.n_groups = int(group_min), int(n_groups)
        self.scale = int(scale)
        self.device = torch.device(device)
        L = N.lib()
        self.knobs = None if knobs is None else N.JoinKnobs(**knobs)
        if autotune is None:
            # the environment's overrides (sweeps, tests) fix the configuration
            autotune = B is None and knobs is None and not any(
                os.environ.get(v) for v in _OVERRIDES)
        self.autotune = bool(autotune)
        self.tuning = None          # the autotuner's Result once it has run
        self.B = int(B) if B else int(L.pf_join_aggregate_pick_b(self.n_build, self.n_probe))
        self.ws = None
        self.ws_bytes = 0
        if not self.autotune:
            self._reserve()
        self.sum = torch.empty(self.n_groups, dtype=torch.int64, device=self.device)
        self.count = torch.empty(self.n_groups, dtype=torch.int64, device=self.device)
        self.stats = torch.zeros(4, dtype=torch.int64, device=self.device)
        self.keys_out = torch.empty(self.n_groups, dtype=torch.int64, device=self.device)
        self.sums_out = torch.empty(self.n_groups, dtype=torch.int64, device=self.device)
        self.counts_out = torch.empty(self.n_groups, dtype=torch.int64, device=self.device)
        self.fin_bytes = int(L.pf_groups_finish_workspace(self.n_groups))
        self.fin_ws = N.workspace(self.fin_bytes, self.device)
        self.host = torch.zeros(2, dtype=torch.int64, pin_memory=True)

    def _ws_for(self, B, knobs) -> int:
        return int(N.lib().pf_join_aggregate_workspace_ex(
            self.n_build, self.n_probe, B, self.n_groups,
            None if knobs is None else ctypes.byref(knobs)))

    def _reserve(self, need: Optional[int] = None) -> None:
        need = self._ws_for(self.B, self.knobs) if need is None else need
        if self.ws is None or self.ws_bytes < need:
            self.ws = None
            self.ws = N.workspace(need, self.device)
            self.ws_bytes = need

    def _launch(self, B, knobs, args) -> None:
        build_key, build_group, probe_fk, probe_price, probe_disc = args
        L = N.lib()
        with torch.cuda.device(self.device):
            rc = L.pf_join_aggregate_ex(
                build_key.data_ptr(), build_group.data_ptr(), self.n_build,
                probe_fk.data_ptr(), probe_price.data_ptr(), N.ptr(probe_disc), self.scale,
                self.n_probe, B, self.group_min, self.n_groups, self.sum.data_ptr(),
                self.count.data_ptr(), self.stats.data_ptr(),
                None if knobs is None else ctypes.byref(knobs), self.ws.data_ptr(),
                self.ws_bytes, N.stream_of(self.device))
        N.check(rc, "join_aggregate")

    def _tune(self, args) -> None:
        from . import autotune as T
        key = T.shape_class(torch.cuda.get_device_name(self.device), self.n_build,
                            self.n_probe, self.n_groups)

        def knobs_of(c):
            return N.JoinKnobs(path=0, table=c.table, sub_rows=c.sub_rows, counted=c.counted)

        def time_of(c):
            kn = knobs_of(c)
            self._reserve(self._ws_for(c.B, kn))
            stream = torch.cuda.current_stream(self.device)
            self._launch(c.B, kn, args)           # warm-up
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            reps = 2
            e0.record(stream)
            for _ in range(reps):
                self._launch(c.B, kn, args)
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1) / reps

        self.tuning = T.tune(key, self.B, time_of)
        c = self.tuning.choice
        self.B = c.B
        self.knobs = knobs_of(c)
        self._reserve()
        self.autotune = False

    def aggregate(self, build_key, build_group, probe_fk, probe_price, probe_disc=None):
        """Queues the join + dense aggregation into ``self.sum`` /
        ``self.count`` (waits once, at the end, for the radix passes'
        overflow words; again only after an overflow)."""
        for t, n, dt, name in ((build_key, self.n_build, torch.int64, "build_key"),
                               (build_group, self.n_build, torch.int32, "build_group"),
                               (probe_fk, self.n_probe, torch.int64, "probe_fk"),
                               (probe_price, self.n_probe, torch.int64, "probe_price")):
            if not (t.is_cuda and t.dtype == dt and t.dim() == 1 and t.numel() == n
                    and t.is_contiguous()):
                raise ValueError(f"{name} must be a contiguous 1-D {dt} CUDA tensor of {n} rows")
        if probe_disc is not None and not (probe_disc.is_cuda and probe_disc.dtype == torch.int64
                                           and probe_disc.numel() == self.n_probe
                                           and probe_disc.is_contiguous()):
            raise ValueError("probe_disc must match probe_fk")
        args = (build_key, build_group, probe_fk, probe_price, probe_disc)
        if self.autotune:
            self._tune(args)
        self._launch(self.B, self.knobs, args)

    def finish(self):
        """The occupied groups, ascending: (keys, sums, counts)."""
        L = N.lib()
        with torch.cuda.device(self.device):
            rc = L.pf_groups_finish(self.sum.data_ptr(), self.count.data_ptr(), self.group_min,
                                    self.n_groups, self.keys_out.data_ptr(),
                                    self.sums_out.data_ptr(), self.counts_out.data_ptr(),
                                    self.host.data_ptr(), self.fin_ws.data_ptr(),
                                    self.fin_bytes, N.stream_of(self.device))
        N.check(rc, "groups_finish")
        n = int(self.host[0])
        return self.keys_out[:n], self.sums_out[:n], self.counts_out[:n]

    def run(self, build_key, build_group, probe_fk, probe_price, probe_disc=None):
        self.aggregate(build_key, build_group, probe_fk, probe_price, probe_disc)
        return self.finish()

    def run_stream(self, batches):
        """Joins a sequence of host-resident batches of this plan's shape,
        each a tuple (build_key, build_group, probe_fk, probe_price,
        probe_disc or None) of pinned host tensors, and yields each batch's
        occupied groups as host tensors (keys, sums, counts).  A batch's
        columns cross to the device on a copy stream while the batch before
        it is joined, into one of two sets of device buffers (a set is
        refilled only after the join that read it), so the host link and
        the GPU work overlap; every batch still crosses the link whole."""
        dev = self.device
        compute = torch.cuda.current_stream(dev)
        copy = torch.cuda.Stream(dev)
        copy.wait_stream(compute)
        sets, ready, free = [None, None], [None, None], [None, None]

        def stage(slot, batch):
            if sets[slot] is None:
                sets[slot] = [None] * len(batch)
            for i, h in enumerate(batch):
                if h is not None and sets[slot][i] is None:
                    sets[slot][i] = torch.empty(h.shape, dtype=h.dtype, device=dev)
            with torch.cuda.stream(copy):
                if free[slot] is not None:
                    copy.wait_event(free[slot])
                for d, h in zip(sets[slot], batch):
                    if h is not None:
                        d.copy_(h, non_blocking=True)
                        d.record_stream(copy)   # not reused while the copy may run
                ready[slot] = torch.cuda.Event()
                ready[slot].record(copy)

        it = iter(batches)
        nxt = next(it, None)
        if nxt is None:
            return
        slot = 0
        stage(slot, nxt)
        while nxt is not None:
            cur, nxt = nxt, next(it, None)
            if nxt is not None:
                stage(slot ^ 1, nxt)        # crosses the link while this one joins
            compute.wait_event(ready[slot])
            dev_in = [d if h is not None else None for d, h in zip(sets[slot], cur)]
            keys, sums, counts = self.run(*dev_in)
            out = tuple(torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
                        for t in (keys, sums, counts))
            for h, d in zip(out, (keys, sums, counts)):
                h.copy_(d, non_blocking=True)
            free[slot] = torch.cuda.Event()
            free[slot].record(compute)
            free[slot].synchronize()
            yield out
            slot ^= 1

    def read_stats(self) -> JoinAggregateStats:
        s = self.stats.tolist()
        return JoinAggregateStats(matched=s[0], bad_groups=s[2], overflow=s[3],
                                  device_error=s[1])


def join_group_aggregate(build_key, build_group, probe_fk, probe_price, probe_disc=None,
                         scale: int = 100, group_min: Optional[int] = None,
                         n_groups: Optional[int] = None, B: Optional[int] = None):
    """One-shot form: (group keys ascending, int64 sums, int64 counts).  The
    group range defaults to the build groups' [min, max] (one host read)."""
    if group_min is None or n_groups is None:
        if build_group.numel() == 0:
            e = torch.empty(0, dtype=torch.int64, device=build_key.device)
            return e, e.clone(), e.clone()
        lo, hi = torch.aminmax(build_group)
        group_min, n_groups = int(lo), int(hi) - int(lo) + 1
    plan = JoinAggregate(build_key.numel(), probe_fk.numel(), group_min, n_groups,
                         build_key.device, B=B, scale=scale)
    return plan.run(build_key, build_group, probe_fk, probe_price, probe_disc)
