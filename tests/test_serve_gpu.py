"""The serving path on the GPU: resident dimension tables and fact rows
against the generator's CPU twin, every request's groups equal to the
oracle's, the same result alone and in the mix, admission under a tight HBM
budget, requests spread over many launches, and Poisson arrivals."""
import numpy as np
import pytest
import torch

import oracle
from pageflow_b200 import serve

pytestmark = pytest.mark.gpu

SPEC = serve.scaled(serve.SERVE, 2000)


@pytest.fixture(scope="module")
def world():
    dev = torch.device("cuda", 0)
    dims = serve.Dimensions(SPEC, dev)
    fact = serve.FactPool(SPEC, dev)
    torch.cuda.synchronize()
    cpu_dims = [oracle.gen_serve_dim(SPEC.seed, SPEC.n_ranks, dims.group_seed(d),
                                     SPEC.dim_groups[d], 0, SPEC.dim_keys[d])
                for d in range(len(SPEC.dim_keys))]
    cpu_fact = oracle.gen_serve_fact(SPEC.seed, SPEC.n_ranks, 0, SPEC.fact_rows, fact.edges,
                                     fact.thr)
    return dev, dims, fact, cpu_dims, cpu_fact


def _expected(world, r):
    _, _, _, cpu_dims, (fk, date, value) = world
    k, g = cpu_dims[r.dim]
    s = slice(r.row0, r.row0 + r.n_rows)
    return oracle.serve_request(k, g, SPEC.dim_groups[r.dim], fk[s], date[s], value[s],
                                r.date_lo, r.date_hi)


def _same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


def test_resident_tables_match_the_generator(world):
    dev, dims, fact, cpu_dims, (fk, date, value) = world
    for d, (k, g) in enumerate(cpu_dims):
        assert np.array_equal(dims.keys[d].cpu().numpy(), k)
        assert np.array_equal(dims.groups[d].cpu().numpy(), g)
    assert np.array_equal(fact.fk.cpu().numpy(), fk)
    assert np.array_equal(fact.date.cpu().numpy(), date)
    assert np.array_equal(fact.value.cpu().numpy(), value)


def test_burst_of_requests_matches_the_oracle(world):
    dev, dims, fact, _, _ = world
    reqs = serve.make_requests(SPEC, 48, seed=11)
    srv = serve.Server(dims, fact, SPEC.budget_bytes, dev, iter_rows=1 << 16,
                       pinned_bytes=1 << 24)
    run = srv.run(reqs)
    assert run.launches > 1 and run.rows == sum(r.n_rows for r in reqs)
    for r in reqs:
        assert _same(r.result, _expected(world, r)), r
        assert r.n_groups_out == r.result[0].shape[0]
        assert r.latency > 0
    kept = sum(int(((world[4][1][r.row0:r.row0 + r.n_rows] >= r.date_lo) &
                    (world[4][1][r.row0:r.row0 + r.n_rows] < r.date_hi)).sum()) for r in reqs)
    assert run.stats["kept"] == kept


def test_each_result_is_the_same_alone_and_in_the_mix(world):
    dev, dims, fact, _, _ = world
    reqs = serve.make_requests(SPEC, 24, seed=12)
    srv = serve.Server(dims, fact, SPEC.budget_bytes, dev, iter_rows=1 << 17,
                       pinned_bytes=1 << 24)
    mixed = srv.run(reqs)
    for r in reqs:
        alone = serve.Request(r.id, r.dim, r.row0, r.n_rows, r.date_lo, r.date_hi)
        srv.run([alone])
        assert _same(alone.result, r.result), r.id
    assert mixed.max_admitted > 1


def test_tight_budget_admits_few_and_stays_exact(world):
    dev, dims, fact, _, _ = world
    reqs = serve.make_requests(SPEC, 30, seed=13)
    biggest = max(SPEC.dim_groups[r.dim] for r in reqs)
    budget = dims.nbytes + fact.nbytes + 2 * serve.Server.device_bytes(biggest) + (1 << 20)
    srv = serve.Server(dims, fact, budget, dev, iter_rows=1 << 18, pinned_bytes=1 << 24)
    run = srv.run(reqs)
    assert run.max_admitted < len(reqs)
    for r in reqs:
        assert _same(r.result, _expected(world, r)), r
    with pytest.raises(ValueError):
        serve.Server(dims, fact, dims.nbytes + fact.nbytes, dev)


def test_poisson_arrivals_complete_in_order_of_need(world):
    dev, dims, fact, _, _ = world
    reqs = serve.make_requests(SPEC, 60, seed=14)
    for r, t in zip(reqs, serve.poisson_arrivals(len(reqs), 400.0, seed=14)):
        r.arrival = float(t)
    srv = serve.Server(dims, fact, SPEC.budget_bytes, dev, pinned_bytes=1 << 24)
    run = srv.run(reqs, keep_results=False)
    lat = run.latencies()
    assert np.all(np.isfinite(lat)) and np.all(lat > 0)
    assert all(r.t_done >= r.arrival and r.t_admit >= r.arrival for r in reqs)
    assert run.wall_s >= reqs[-1].arrival
