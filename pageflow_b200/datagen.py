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
