"""Serving: join -> date filter -> group-by requests against device-resident
dimension tables, folded into persistent launches.

Each request is SELECT dim.group, SUM(fact.value), COUNT(*) FROM fact JOIN
dim_d ON fact.fk = dim_d.key WHERE lo <= fact.date < hi GROUP BY dim.group,
over a slice of the resident fact rows.  The dimension tables' hash tables
are built once (pf_dim_build) and persist across requests.  The server:

  admission   FIFO; a request is admitted when its device memory (its
              (sum, count) slab and result columns) fits the HBM budget left
              after the resident tables, and its result fits the pinned
              result pool
  launches    iteration-level batching: each launch (pf_serve_run) takes the
              admitted requests with rows left, smallest remainder first, up
              to iter_rows probe rows in all; a request whose last rows are in
              the launch is finished in it (groups compacted, done word set)
  completion  the host polls each finishing request's pinned done word and
              copies its groups back on a copy stream while the launch goes
              on; latency = result on the host - arrival

The reference has no serving layer (its executors run one query at a time);
the per-request plain form it would run is the filter (operators/filter.py:
10-16), mask compaction (utility/tensor_utils.py:12-39) and the unique-build
join + group-by (uvm/join.py:98-225, uvm/aggregate.py:147-212).
"""
from __future__ import annotations

import bisect
import ctypes
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native
from ._native import check, lib, ptr

DATE_LO = 8035
DATE_DAYS = 2557


def _logspace_int(a: float, b: float, n: int):
    return tuple(int(round(a * (b / a) ** (i / (n - 1)))) for i in range(n))


@dataclass(frozen=True)
class ServeSpec:
    """The serving workload: 8 dimensions of log-spaced key counts (the most
    referenced ranks of n_ranks), a resident fact pool, request probe sizes
    log-uniform in [probe_min, probe_max], filter selectivity uniform in
    [sel_min, sel_max], an HBM budget for admission."""
    seed: int
    n_ranks: int
    dim_keys: tuple
    dim_groups: tuple
    fact_rows: int
    zipf_s: float
    probe_min: int
    probe_max: int
    sel_min: float
    sel_max: float
    budget_bytes: int


SERVE = ServeSpec(4, 200_000_000, _logspace_int(1e5, 2e8, 8),
                  (16, 100, 1000, 5000, 25_000, 100_000, 500_000, 1_500_000),
                  1_000_000_000, 0.8, 100_000, 1_000_000_000, 0.01, 0.50, 150 * 10 ** 9)


def scaled(spec: ServeSpec, factor: float) -> ServeSpec:
    """The same workload with every row count divided by `factor`."""
    keys = tuple(max(100, int(k / factor)) for k in spec.dim_keys)
    groups = tuple(max(1, min(g, k)) for g, k in zip(spec.dim_groups, keys))
    return ServeSpec(spec.seed, max(keys[-1], int(spec.n_ranks / factor)), keys, groups,
                     max(1000, int(spec.fact_rows / factor)), spec.zipf_s,
                     max(10, int(spec.probe_min / factor)),
                     max(100, int(spec.probe_max / factor)), spec.sel_min, spec.sel_max,
                     max(1 << 26, int(spec.budget_bytes / factor)))


@dataclass
class Request:
    id: int
    dim: int
    row0: int
    n_rows: int
    date_lo: int
    date_hi: int
    arrival: float = 0.0
    # filled in by the server
    t_admit: float = math.nan
    t_done: float = math.nan
    result: tuple | None = None
    n_groups_out: int = -1

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


def make_requests(spec: ServeSpec, n: int, seed: int | None = None) -> list[Request]:
    """n requests (seeded): dimension uniform, probe rows log-uniform, a
    contiguous slice of the fact pool, a date range of uniform selectivity."""
    rng = np.random.default_rng(spec.seed if seed is None else seed)
    out = []
    lo_l, hi_l = math.log(spec.probe_min), math.log(min(spec.probe_max, spec.fact_rows))
    for i in range(n):
        rows = int(round(math.exp(rng.uniform(lo_l, hi_l))))
        rows = max(1, min(rows, spec.fact_rows))
        dim = int(rng.integers(0, len(spec.dim_keys)))
        row0 = int(rng.integers(0, spec.fact_rows - rows + 1))
        sel = float(rng.uniform(spec.sel_min, spec.sel_max))
        width = max(1, min(DATE_DAYS, int(round(sel * DATE_DAYS))))
        d0 = DATE_LO + int(rng.integers(0, DATE_DAYS - width + 1))
        out.append(Request(i, dim, row0, rows, d0, d0 + width))
    return out


def poisson_arrivals(n: int, rate: float, seed: int = 4) -> np.ndarray:
    """Arrival times (seconds from 0) of a Poisson process of `rate` per
    second; the same seed gives the same unit gaps at every rate."""
    gaps = np.random.default_rng(seed).exponential(1.0, n)
    return np.cumsum(gaps) / rate


# ---- resident tables -----------------------------------------------------------

class Dimensions:
    """The dimension tables: keys, groups and the persistent hash tables."""

    def __init__(self, spec: ServeSpec, device):
        self.spec = spec
        self.device = device
        self.keys, self.groups, self.tables = [], [], []
        L = lib()
        st = _native.stream_of(device)
        stats = torch.zeros(2, dtype=torch.int64, device=device)
        for d, (nk, ng) in enumerate(zip(spec.dim_keys, spec.dim_groups)):
            k = torch.empty(nk, dtype=torch.int64, device=device)
            g = torch.empty(nk, dtype=torch.int32, device=device)
            check(L.pf_gen_serve_dim(spec.seed, spec.n_ranks, self.group_seed(d), nk, ng, 0, nk,
                                     ptr(k), ptr(g), st), "gen_serve_dim")
            tb = L.pf_dim_table_bytes(nk)
            t = torch.empty(tb, dtype=torch.uint8, device=device)
            check(L.pf_dim_build(ptr(k), ptr(g), nk, ng, ptr(t), tb, ptr(stats), st), "dim_build")
            s = stats.cpu().tolist()
            if s != [0, 0]:
                raise RuntimeError(f"dimension {d}: {s[0]} groups out of range, {s[1]} overflows")
            self.keys.append(k)
            self.groups.append(g)
            self.tables.append(t)

    def group_seed(self, d: int) -> int:
        return self.spec.seed * 1_000_003 + 17 * (d + 1)

    @property
    def nbytes(self) -> int:
        return sum(k.numel() * 12 + t.numel() for k, t in zip(self.keys, self.tables))


class FactPool:
    """The resident fact rows: fk int64, date int32, value int64."""

    def __init__(self, spec: ServeSpec, device, chunk: int = 1 << 27):
        from .datagen import zipf_table
        edges, thr = zipf_table(spec.n_ranks, spec.zipf_s)
        self.edges = np.ascontiguousarray(edges, np.int64)
        self.thr = np.ascontiguousarray(thr, np.uint64)
        n = spec.fact_rows
        self.fk = torch.empty(n, dtype=torch.int64, device=device)
        self.date = torch.empty(n, dtype=torch.int32, device=device)
        self.value = torch.empty(n, dtype=torch.int64, device=device)
        e = torch.from_numpy(self.edges).to(device)
        t = torch.from_numpy(self.thr.view(np.int64)).to(device)
        st = _native.stream_of(device)
        for lo in range(0, n, chunk):
            rows = min(chunk, n - lo)
            check(lib().pf_gen_serve_fact(spec.seed, spec.n_ranks, self.thr.shape[0], ptr(e),
                                          ptr(t), lo, rows, ptr(self.fk[lo:]),
                                          ptr(self.date[lo:]), ptr(self.value[lo:]), st),
                  "gen_serve_fact")
        self.n_rows = n

    @property
    def nbytes(self) -> int:
        return self.n_rows * 20


# ---- host-side allocation ------------------------------------------------------------

class Arena:
    """First-fit allocator of [0, capacity) in `align`-byte units (the
    admission budget's bookkeeping; offsets into one device or pinned
    buffer)."""

    def __init__(self, capacity: int, align: int = 256):
        self.align = align
        self.capacity = capacity // align * align
        self.free = [(0, self.capacity)]      # sorted (offset, size)
        self.used = {}

    def alloc(self, nbytes: int):
        n = max(self.align, (nbytes + self.align - 1) // self.align * self.align)
        for i, (off, size) in enumerate(self.free):
            if size >= n:
                if size == n:
                    self.free.pop(i)
                else:
                    self.free[i] = (off + n, size - n)
                self.used[off] = n
                return off
        return None

    def release(self, off: int) -> None:
        n = self.used.pop(off)
        i = bisect.bisect_left(self.free, (off, 0))
        self.free.insert(i, (off, n))
        # merge with the neighbours
        if i + 1 < len(self.free) and off + n == self.free[i + 1][0]:
            self.free[i] = (off, n + self.free[i + 1][1])
            self.free.pop(i + 1)
        if i > 0 and self.free[i - 1][0] + self.free[i - 1][1] == self.free[i][0]:
            self.free[i - 1] = (self.free[i - 1][0], self.free[i - 1][1] + self.free[i][1])
            self.free.pop(i)

    @property
    def in_use(self) -> int:
        return sum(self.used.values())


def plan_launch(active, quota: int):
    """The next launch's shares: active requests (objects with `left` rows
    and `cursor`), smallest remainder first, until `quota` probe rows are
    handed out; a request whose remaining rows all fit finishes.  Returns
    [(request, begin, end, finish)].  A request with no rows left (finish
    pending) costs nothing and always goes in."""
    out = []
    left = quota
    for r in sorted(active, key=lambda r: (r.left, r.id)):
        if r.left == 0:
            out.append((r, r.cursor, r.cursor, True))
            continue
        if left <= 0:
            break
        take = min(r.left, left)
        out.append((r, r.cursor, r.cursor + take, take == r.left))
        left -= take
    return out


def lindley(arrivals: np.ndarray, service: np.ndarray) -> np.ndarray:
    """Completion - arrival of a single FIFO server (one request at a time)
    with the given service times."""
    t = 0.0
    out = np.empty(len(arrivals))
    for i, (a, s) in enumerate(zip(arrivals, service)):
        t = max(t, a) + s
        out[i] = t - a
    return out


@dataclass
class _Live:
    req: Request
    cursor: int
    left: int
    dev_off: int
    pin_off: int
    done_slot: int
    n_groups: int
    launched_finish: bool = False
    d2h: object = None
    id: int = 0


@dataclass
class ServeRun:
    requests: list
    wall_s: float
    launches: int
    rows: int
    max_admitted: int
    stats: dict = field(default_factory=dict)

    def latencies(self) -> np.ndarray:
        return np.array([r.latency for r in self.requests])


class Server:
    """The serving loop over resident dimensions and fact rows (one device,
    one host thread)."""

    def __init__(self, dims: Dimensions, fact: FactPool, budget_bytes: int, device,
                 iter_rows: int = 1 << 27, max_batch: int = 2048, pinned_bytes: int = 1 << 30,
                 max_live: int = 1 << 14):
        self.dims, self.fact, self.device = dims, fact, device
        self.iter_rows = int(iter_rows)
        self.max_batch = int(max_batch)
        resident = dims.nbytes + fact.nbytes
        cap = int(budget_bytes) - resident
        if cap < (1 << 20):
            raise ValueError(f"budget of {budget_bytes} bytes leaves no room beside the "
                             f"{resident} resident bytes")
        self.arena = Arena(cap)
        self.dev_pool = torch.empty(self.arena.capacity, dtype=torch.uint8, device=device)
        self.pin_arena = Arena(pinned_bytes)
        self.pin_pool = torch.empty(self.pin_arena.capacity, dtype=torch.uint8, pin_memory=True)
        self.done = torch.zeros(max_live, dtype=torch.int64, pin_memory=True)
        self.done_np = self.done.numpy()
        self.free_slots = list(range(max_live - 1, -1, -1))
        self.ws = _native.workspace(lib().pf_serve_workspace(self.max_batch), device)
        self.stats = torch.zeros(4, dtype=torch.int64, device=device)
        self.stream = torch.cuda.Stream(device)
        self.copy_stream = torch.cuda.Stream(device)

    @staticmethod
    def device_bytes(n_groups: int) -> int:
        return 16 * n_groups + 24 * n_groups + 256 * 5

    def _dev(self, off: int, elems: int, dtype=torch.int64) -> torch.Tensor:
        nb = elems * torch.tensor([], dtype=dtype).element_size()
        return self.dev_pool[off:off + nb].view(dtype)

    def _layout(self, lv: _Live):
        """(slab, keys, sums, counts, out_n) tensors of a live request."""
        g = lv.n_groups
        a = lv.dev_off
        slab = self._dev(a, 2 * g)
        a += (16 * g + 255) // 256 * 256
        keys = self._dev(a, g)
        a += (8 * g + 255) // 256 * 256
        sums = self._dev(a, g)
        a += (8 * g + 255) // 256 * 256
        counts = self._dev(a, g)
        a += (8 * g + 255) // 256 * 256
        out_n = self._dev(a, 1)
        return slab, keys, sums, counts, out_n

    def run(self, requests: list[Request], keep_results: bool = True,
            timeout_s: float = 600.0) -> ServeRun:
        """Serves the requests at their arrival times (seconds after the
        call starts); returns when every request is complete."""
        L = lib()
        spec_keys = self.dims.spec.dim_keys
        spec_groups = self.dims.spec.dim_groups
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.id)))
        waiting: deque = deque()
        active: list[_Live] = []
        finishing: list[_Live] = []
        inflight: deque = deque()
        done = 0
        launches = rows = max_admitted = 0
        st_ptr = self.stream.cuda_stream
        self.stats.zero_()
        t0 = time.perf_counter()
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            while done < len(requests):
                now = time.perf_counter() - t0
                if now > timeout_s:
                    raise TimeoutError(f"serving: {len(requests) - done} requests left after "
                                       f"{timeout_s} s")
                while pending and pending[0].arrival <= now:
                    waiting.append(pending.popleft())
                # admission, FIFO, by the device budget and the pinned result pool
                while waiting and self.free_slots:
                    r = waiting[0]
                    g = spec_groups[r.dim]
                    off = self.arena.alloc(self.device_bytes(g))
                    if off is None:
                        break
                    poff = self.pin_arena.alloc(24 * g)
                    if poff is None:
                        self.arena.release(off)
                        break
                    waiting.popleft()
                    slot = self.free_slots.pop()
                    self.done_np[slot] = 0
                    lv = _Live(r, r.row0, r.n_rows, off, poff, slot, g, id=r.id)
                    r.t_admit = now
                    slab = self._layout(lv)[0]
                    slab.zero_()
                    active.append(lv)
                max_admitted = max(max_admitted, len(active) + len(finishing))
                # launch while fewer than two are in flight
                while inflight and inflight[0].query():
                    inflight.popleft()
                if active and len(inflight) < 2:
                    plan = plan_launch(active, self.iter_rows)[:self.max_batch]
                    arr = (_native.ServeRequest * len(plan))()
                    for j, (lv, b, e, fin) in enumerate(plan):
                        r = lv.req
                        slab, keys, sums, counts, out_n = self._layout(lv)
                        x = arr[j]
                        x.table = ptr(self.dims.tables[r.dim])
                        x.n_keys = spec_keys[r.dim]
                        x.n_groups = lv.n_groups
                        x.fk = ptr(self.fact.fk)
                        x.date = ptr(self.fact.date)
                        x.value = ptr(self.fact.value)
                        x.row_begin, x.row_end = b, e
                        x.date_lo, x.date_hi = r.date_lo, r.date_hi
                        x.finish = 1 if fin else 0
                        x.slab = ptr(slab)
                        x.out_keys, x.out_sums, x.out_counts = ptr(keys), ptr(sums), ptr(counts)
                        x.out_n = ptr(out_n)
                        x.done = self.done.data_ptr() + 8 * lv.done_slot if fin else None
                        lv.cursor = e
                        lv.left -= e - b
                        rows += e - b
                    check(L.pf_serve_run(arr, len(plan), ptr(self.ws), self.ws.numel(),
                                         ptr(self.stats), st_ptr), "serve_run")
                    ev = torch.cuda.Event()
                    ev.record(self.stream)
                    inflight.append(ev)
                    launches += 1
                    for lv, b, e, fin in plan:
                        if fin:
                            active.remove(lv)
                            finishing.append(lv)
                # completions: done word set -> copy the groups back
                still = []
                for lv in finishing:
                    if lv.d2h is None:
                        w = int(self.done_np[lv.done_slot])
                        if w < 0:
                            raise RuntimeError(f"serving: request {lv.req.id}: a device wait "
                                               f"gave up")
                        if w > 0:
                            n = w - 1
                            lv.req.n_groups_out = n
                            _, keys, sums, counts, _ = self._layout(lv)
                            host = self.pin_pool[lv.pin_off:lv.pin_off + 24 * max(n, 1)]
                            hk = host[:8 * n].view(torch.int64)
                            hs = host[8 * n:16 * n].view(torch.int64)
                            hc = host[16 * n:24 * n].view(torch.int64)
                            with torch.cuda.stream(self.copy_stream):
                                hk.copy_(keys[:n], non_blocking=True)
                                hs.copy_(sums[:n], non_blocking=True)
                                hc.copy_(counts[:n], non_blocking=True)
                                ev = torch.cuda.Event()
                                ev.record(self.copy_stream)
                            lv.d2h = (ev, hk, hs, hc)
                        still.append(lv)
                    elif lv.d2h[0].query():
                        lv.req.t_done = time.perf_counter() - t0
                        if keep_results:
                            _, hk, hs, hc = lv.d2h
                            lv.req.result = (hk.numpy().copy(), hs.numpy().copy(),
                                             hc.numpy().copy())
                        self.arena.release(lv.dev_off)
                        self.pin_arena.release(lv.pin_off)
                        self.free_slots.append(lv.done_slot)
                        done += 1
                    else:
                        still.append(lv)
                finishing = still
                if not finishing and not active and not waiting and pending:
                    wait = pending[0].arrival - (time.perf_counter() - t0)
                    if wait > 0.0005:
                        time.sleep(min(wait, 0.001))
            self.stream.synchronize()
        wall = time.perf_counter() - t0
        s = self.stats.cpu().tolist()
        if s[1]:
            raise RuntimeError("serving: a device wait gave up (error word set)")
        return ServeRun(list(requests), wall, launches, rows, max_admitted,
                        {"matched": s[0], "kept": s[2]})
