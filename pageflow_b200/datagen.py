"""Seeded synthetic inputs of the join + group-by workload, generated on the
device (pf_gen_build / pf_gen_probe; the CPU twin lives in the oracle and
produces the same columns from the same seed).

Workloads (rows and seeds of the benchmark configurations):
  small  build 250,000 keys (a permutation of 1..250,000), groups U[0,25);
         probe 1,000,000 FKs U[1,250,000], price U[90,000, 10,500,000] cents,
         discount U[0,10] hundredths; seed 0
  scale  build 150M keys permuted over 1..150M, groups U[0,1.5M); probe 600M
         FKs, 90% U over the build keys and 10% outside them; price and
         discount as above; seed 1
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N


@dataclass(frozen=True)
class Workload:
    name: str
    config: int        # generator config id (miss rate)
    seed: int
    n_build: int
    n_probe: int
    n_groups: int
    scale: int = 100   # value = price * (scale - discount)


SMALL = Workload("small", 0, 0, 250_000, 1_000_000, 25)
SCALE = Workload("scale", 1, 1, 150_000_000, 600_000_000, 1_500_000)


def scaled(w: Workload, factor: float, name: str | None = None) -> Workload:
    """The same workload with every row count scaled (groups scaled too,
    at least one)."""
    return Workload(name or f"{w.name}/{factor:g}", w.config, w.seed,
                    max(1, int(w.n_build * factor)), max(1, int(w.n_probe * factor)),
                    max(1, int(w.n_groups * factor)), w.scale)


def gen_build(w: Workload, device, lo: int = 0, rows: int | None = None):
    rows = w.n_build - lo if rows is None else rows
    key = torch.empty(rows, dtype=torch.int64, device=device)
    grp = torch.empty(rows, dtype=torch.int32, device=device)
    with torch.cuda.device(device):
        N.check(N.lib().pf_gen_build(w.config, w.seed, w.n_build, w.n_groups, lo, rows,
                                     key.data_ptr(), grp.data_ptr(), N.stream_of(device)),
                "gen_build")
    return key, grp


@dataclass(frozen=True)
class BatchSpec:
    """One instance of the batching workload (sizes drawn on the host from
    the workload seed, so the CPU oracle and the GPU draw the same rows)."""
    index: int
    seed: int           # the instance's own generator seed
    n_build: int        # unique keys, a permutation of 1..n_build
    n_probe: int
    skew: float         # Zipf exponent of the probe FKs over the build keys
    n_groups: int
    edges: np.ndarray   # Zipf table: bin b holds ranks [edges[b], edges[b+1])
    thr: np.ndarray     # cumulative bin probabilities scaled to 2^64 (uint64)


def zipf_table(n: int, s: float, bins: int = 256):
    """Geometric rank bins over [0, n) and their cumulative Zipf(s) masses
    (the integral of x^-s over each bin's ranks 1-based), as uint64
    thresholds; one bin for s = 0."""
    if s == 0.0 or n <= 1:
        return np.array([0, n], np.int64), np.array([np.iinfo(np.uint64).max], np.uint64)
    e = np.unique(np.floor(np.geomspace(1, n + 1, bins + 1)).astype(np.int64))
    e[0], e[-1] = 1, n + 1
    e = np.unique(e)
    lo, hi = e[:-1].astype(np.float64), e[1:].astype(np.float64)
    if abs(s - 1.0) < 1e-12:
        mass = np.log(hi) - np.log(lo)
    else:
        mass = (hi ** (1 - s) - lo ** (1 - s)) / (1 - s)
    cdf = np.cumsum(mass) / mass.sum()
    # the largest double below 2^64 is 2^64 - 2048; the last bin takes the rest
    thr = np.minimum(np.floor(cdf * 2.0 ** 64), 2.0 ** 64 - 2048.0)
    thr_u = np.array([int(x) for x in thr], dtype=np.uint64)
    thr_u = np.maximum.accumulate(thr_u)
    thr_u[-1] = np.iinfo(np.uint64).max
    return (e - 1).astype(np.int64), thr_u


def batch_workload(n_inst: int = 4096, seed: int = 3, build_range=(1_000, 4_000_000),
                   group_range=(4, 1_000_000), ratio_range=(4, 16), skews=(0.0, 0.8, 1.2)):
    """The batching workload: build sizes log-uniform in build_range, probe
    sizes 4-16x build, FK skew per instance from Zipf s in skews, group
    cardinality log-uniform in group_range, values in int64 cents."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_inst):
        nb = int(round(float(np.exp(rng.uniform(np.log(build_range[0]), np.log(build_range[1]))))))
        ratio = int(rng.integers(ratio_range[0], ratio_range[1] + 1))
        s = float(skews[int(rng.integers(0, len(skews)))])
        ng = int(round(float(np.exp(rng.uniform(np.log(group_range[0]), np.log(group_range[1]))))))
        edges, thr = zipf_table(nb, s)
        out.append(BatchSpec(i, seed * 1_000_003 + i, nb, nb * ratio, s, ng, edges, thr))
    return out


def gen_batch_instance(spec: BatchSpec, device):
    """(build_key, build_group, probe_fk, probe_value) of one instance on the
    device."""
    key = torch.empty(spec.n_build, dtype=torch.int64, device=device)
    grp = torch.empty(spec.n_build, dtype=torch.int32, device=device)
    fk = torch.empty(spec.n_probe, dtype=torch.int64, device=device)
    val = torch.empty(spec.n_probe, dtype=torch.int64, device=device)
    edges = torch.from_numpy(spec.edges).to(device)
    thr = torch.from_numpy(spec.thr.view(np.int64)).to(device)
    L = N.lib()
    with torch.cuda.device(device):
        st = N.stream_of(device)
        N.check(L.pf_gen_build(1, spec.seed, spec.n_build, spec.n_groups, 0, spec.n_build,
                               key.data_ptr(), grp.data_ptr(), st), "gen_build")
        N.check(L.pf_gen_batch_probe(spec.seed, spec.n_build, 0, spec.n_probe, thr.numel(),
                                     edges.data_ptr(), thr.data_ptr(), fk.data_ptr(),
                                     val.data_ptr(), st), "gen_batch_probe")
    torch.cuda.current_stream(device).synchronize()
    return key, grp, fk, val


def gen_probe(w: Workload, device, lo: int = 0, rows: int | None = None):
    rows = w.n_probe - lo if rows is None else rows
    fk = torch.empty(rows, dtype=torch.int64, device=device)
    price = torch.empty(rows, dtype=torch.int64, device=device)
    disc = torch.empty(rows, dtype=torch.int64, device=device)
    with torch.cuda.device(device):
        N.check(N.lib().pf_gen_probe(w.config, w.seed, w.n_build, lo, rows, fk.data_ptr(),
                                     price.data_ptr(), disc.data_ptr(), N.stream_of(device)),
                "gen_probe")
    return fk, price, disc
