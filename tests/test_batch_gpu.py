"""The batched join -> group-by (pageflow_b200.batch, one persistent launch
over many instances) against the oracle, instance by instance: uneven sizes,
uniform and Zipf-skewed FKs (hot keys combine per warp), groups from a
handful to tens of thousands, empty instances; a CUDA-graph replay must give
the same results as the first run (the epoch-tagged tables are never
cleared), and the device generator must be the CPU one."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from pageflow_b200 import datagen
from pageflow_b200.batch import BatchJoinAggregate, Instance

pytestmark = pytest.mark.gpu


def _specs(n, seed):
    return datagen.batch_workload(n, seed=seed, build_range=(1, 60_000), group_range=(1, 20_000))


def _instances(specs):
    out = []
    for sp in specs:
        key, grp, fk, val = datagen.gen_batch_instance(sp, "cuda")
        out.append(Instance(key, grp, fk, val, 0, sp.n_groups))
    return out


def _check(b, specs, insts):
    total = 0
    for i, (sp, x) in enumerate(zip(specs, insts)):
        s, c, m, _ = oracle.join_aggregate(x.build_key.cpu().numpy(), x.build_group.cpu().numpy(),
                                           x.probe_fk.cpu().numpy(), x.probe_value.cpu().numpy(),
                                           None, 0, 0, sp.n_groups, B=4)
        gs, gc = b.result(i)
        assert np.array_equal(gs.cpu().numpy(), s), f"instance {i} sums"
        assert np.array_equal(gc.cpu().numpy(), c), f"instance {i} counts"
        total += m
    st = b.read_stats()
    assert st["matched"] == total and st["device_error"] == 0 and st["overflow"] == 0


def test_batch_matches_the_oracle_instance_by_instance():
    specs = _specs(60, seed=31)
    assert {sp.skew for sp in specs} == {0.0, 0.8, 1.2}
    insts = _instances(specs)
    b = BatchJoinAggregate(insts, "cuda")
    b.run()
    _check(b, specs, insts)


def test_graph_replays_repeat_the_result():
    specs = _specs(24, seed=32)
    insts = _instances(specs)
    b = BatchJoinAggregate(insts, "cuda")
    g = b.graph()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    _check(b, specs, insts)


def test_device_generator_is_the_cpu_generator():
    sp = [s for s in _specs(16, seed=33) if s.skew > 0][0]
    key, grp, fk, val = datagen.gen_batch_instance(sp, "cuda")
    okey, ogrp = oracle.gen_build(sp.seed, sp.n_build, sp.n_groups)
    ofk, oval = oracle.gen_batch_probe(sp.seed, sp.n_build, 0, sp.n_probe, sp.edges, sp.thr)
    assert np.array_equal(key.cpu().numpy(), okey) and np.array_equal(grp.cpu().numpy(), ogrp)
    assert np.array_equal(fk.cpu().numpy(), ofk) and np.array_equal(val.cpu().numpy(), oval)


def test_a_hot_key_is_exact():
    """One instance whose every probe row hits the same build row: one group
    takes every atomic, combined per warp."""
    key = torch.arange(1, 1001, dtype=torch.int64, device="cuda")
    grp = (torch.arange(1000, dtype=torch.int32, device="cuda") % 7)
    fk = torch.full((3_000_001,), 500, dtype=torch.int64, device="cuda")
    val = torch.randint(-(1 << 40), 1 << 40, (3_000_001,), device="cuda")
    b = BatchJoinAggregate([Instance(key, grp, fk, val, 0, 7)], "cuda")
    b.run()
    s, c = b.result(0)
    g = int(grp[499])
    assert int(c[g]) == 3_000_001 and int(c.sum()) == 3_000_001
    assert int(s[g]) == int(val.cpu().numpy().astype(np.int64).sum())


def test_empty_instances_and_groups_out_of_range():
    e64 = torch.empty(0, dtype=torch.int64, device="cuda")
    e32 = torch.empty(0, dtype=torch.int32, device="cuda")
    key = torch.arange(10, dtype=torch.int64, device="cuda")
    grp = torch.arange(10, dtype=torch.int32, device="cuda")
    fk = torch.arange(-5, 15, dtype=torch.int64, device="cuda")
    val = torch.ones(20, dtype=torch.int64, device="cuda")
    insts = [Instance(e64, e32, fk, val, 0, 3), Instance(key, grp, e64, e64, 0, 10),
             Instance(key, grp, fk, val, 2, 5)]
    b = BatchJoinAggregate(insts, "cuda")
    b.run()
    assert b.result(0)[1].sum().item() == 0
    assert b.result(1)[1].sum().item() == 0
    s, c = b.result(2)
    assert c.tolist() == [1, 1, 1, 1, 1] and s.tolist() == [1, 1, 1, 1, 1]
    st = b.read_stats()
    assert st["matched"] == 10 and st["bad_groups"] == 5
