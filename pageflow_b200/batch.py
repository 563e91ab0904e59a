"""Batched join -> group-by: thousands of independent instances of uneven
size in one persistent launch fed by a device work queue (pf_batch_*), with
the run capturable in a CUDA graph.

    b = BatchJoinAggregate(instances, device)   # prepare once (one wait)
    b.run()                                     # queue one run (no host sync)
    g = b.graph()                               # or capture the run ...
    g.replay()                                  # ... and replay it
    sums, counts = b.result(i)                  # instance i's dense groups

Each instance is (build_key int64, build_group int32, probe_fk int64,
probe_value int64, group_min, n_groups): SELECT group, SUM(value), COUNT(*)
FROM build JOIN probe ON key = fk GROUP BY group, with a unique build key.
The reference runs such joins one at a time (per-instance launches of its
torch path); here one launch serves them all.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence

import torch

from . import _native as N


@dataclass
class Instance:
    build_key: torch.Tensor
    build_group: torch.Tensor
    probe_fk: torch.Tensor
    probe_value: torch.Tensor
    group_min: int
    n_groups: int


class BatchJoinAggregate:
    def __init__(self, instances: Sequence[Instance], device):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.instances: List[Instance] = list(instances)
        n = len(self.instances)
        if n == 0:
            raise ValueError("a batch needs at least one instance")
        arr = (N.BatchInstance * n)()
        for i, x in enumerate(self.instances):
            for t, dt, name in ((x.build_key, torch.int64, "build_key"),
                                (x.build_group, torch.int32, "build_group"),
                                (x.probe_fk, torch.int64, "probe_fk"),
                                (x.probe_value, torch.int64, "probe_value")):
                if t.numel() and not (t.is_cuda and t.dtype == dt and t.dim() == 1
                                      and t.is_contiguous() and t.device == self.device):
                    raise ValueError(f"instance {i}: {name} must be a contiguous 1-D {dt} "
                                     f"tensor on {self.device}")
            if x.build_key.numel() != x.build_group.numel():
                raise ValueError(f"instance {i}: build key and group differ in length")
            if x.probe_fk.numel() != x.probe_value.numel():
                raise ValueError(f"instance {i}: probe fk and value differ in length")
            arr[i] = N.BatchInstance(N.ptr(x.build_key) or None, N.ptr(x.build_group) or None,
                                     x.build_key.numel(), N.ptr(x.probe_fk) or None,
                                     N.ptr(x.probe_value) or None, x.probe_fk.numel(),
                                     int(x.group_min), int(x.n_groups))
        self._desc = arr
        L = N.lib()
        self.ws_bytes = int(L.pf_batch_workspace(ctypes.addressof(arr), n))
        self.ws = N.workspace(self.ws_bytes, self.device)
        self.stats = torch.zeros(4, dtype=torch.int64, device=self.device)
        with torch.cuda.device(self.device):
            N.check(L.pf_batch_prepare(ctypes.addressof(arr), n, self.ws.data_ptr(), self.ws_bytes,
                                       N.stream_of(self.device)), "batch prepare")
        self.rows = sum(x.build_key.numel() + x.probe_fk.numel() for x in self.instances)

    def run(self) -> None:
        """Queues one run over every instance (device work only)."""
        with torch.cuda.device(self.device):
            N.check(N.lib().pf_batch_run(self.ws.data_ptr(), self.stats.data_ptr(),
                                         N.stream_of(self.device)), "batch run")

    def graph(self) -> "torch.cuda.CUDAGraph":
        """A CUDA graph of one run (reset + the persistent launch)."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.run()                     # warm the launch path outside capture
        torch.cuda.current_stream(self.device).wait_stream(s)
        with torch.cuda.graph(g, stream=s):
            self.run()
        return g

    def slab(self, i: int) -> torch.Tensor:
        """Instance i's dense slab: [n_groups, 2] int64 (sum, count)."""
        ng = int(self.instances[i].n_groups)
        p = N.lib().pf_batch_slab(self.ws.data_ptr(), i)
        if not p:
            raise RuntimeError("batch slab: unknown instance")
        off = p - self.ws.data_ptr()
        return self.ws[off:off + 16 * ng].view(torch.int64).view(ng, 2)

    def result(self, i: int):
        """Instance i's (dense sums, dense counts) over its group range."""
        s = self.slab(i)
        return s[:, 0], s[:, 1]

    def read_stats(self):
        s = self.stats.tolist()
        return {"matched": s[0], "device_error": s[1], "bad_groups": s[2], "overflow": s[3]}
