"""The serving layer's host logic on the CPU: the admission allocator, the
launch planner, the FIFO queue model of the plain form, the request and
arrival generators, and the oracle's request result against a direct
restatement.  No GPU."""
import numpy as np
import pytest

import oracle
from pageflow_b200 import serve


def test_arena_first_fit_and_merge():
    a = serve.Arena(4096, align=256)
    x = a.alloc(100)
    y = a.alloc(600)
    z = a.alloc(256)
    assert (x, y, z) == (0, 256, 1024)
    assert a.in_use == 256 + 768 + 256
    assert a.alloc(4096) is None
    a.release(y)
    assert a.alloc(512) == 256          # first fit inside the hole
    a.release(x)
    a.release(z)
    a.release(256)
    assert a.free == [(0, 4096)] and a.in_use == 0
    assert a.alloc(4096) == 0


def test_arena_random_sequences_never_overlap():
    rng = np.random.default_rng(3)
    a = serve.Arena(1 << 20, align=256)
    live = {}
    for _ in range(2000):
        if live and rng.random() < 0.45:
            off = list(live)[int(rng.integers(0, len(live)))]
            a.release(off)
            del live[off]
        else:
            n = int(rng.integers(1, 40000))
            off = a.alloc(n)
            if off is not None:
                live[off] = n
        spans = sorted((o, o + a.used[o]) for o in live)
        assert all(s[1] <= t[0] for s, t in zip(spans, spans[1:]))
        assert all(e <= a.capacity for _, e in spans)
        assert a.in_use + sum(s for _, s in a.free) == a.capacity


class _R:
    def __init__(self, id, left, cursor=0):
        self.id, self.left, self.cursor = id, left, cursor


def test_plan_launch_smallest_first_with_quota():
    rs = [_R(0, 500), _R(1, 50), _R(2, 5000), _R(3, 0, cursor=70)]
    plan = serve.plan_launch(rs, 1000)
    got = [(r.id, b, e, f) for r, b, e, f in plan]
    assert got == [(3, 70, 70, True), (1, 0, 50, True), (0, 0, 500, True), (2, 0, 450, False)]
    # quota exhausted: the rest wait; a finish with no rows left still goes in
    plan = serve.plan_launch([_R(5, 10), _R(6, 0)], 0)
    assert [(r.id, f) for r, _, _, f in plan] == [(6, True)]


def test_lindley_fifo_queue():
    arr = np.array([0.0, 0.1, 0.2, 5.0])
    svc = np.array([1.0, 1.0, 0.5, 0.1])
    lat = serve.lindley(arr, svc)
    assert np.allclose(lat, [1.0, 1.9, 2.3, 0.1])


def test_requests_and_arrivals_follow_the_workload():
    spec = serve.SERVE
    reqs = serve.make_requests(spec, 4000)
    rows = np.array([r.n_rows for r in reqs])
    assert rows.min() >= spec.probe_min and rows.max() <= spec.probe_max
    # log-uniform: the median is near the geometric mean of the range
    assert abs(np.log(np.median(rows)) - 0.5 * np.log(spec.probe_min * spec.probe_max)) < 0.3
    sel = np.array([(r.date_hi - r.date_lo) / serve.DATE_DAYS for r in reqs])
    assert sel.min() >= 0.009 and sel.max() <= 0.501
    assert all(0 <= r.row0 and r.row0 + r.n_rows <= spec.fact_rows for r in reqs)
    assert set(r.dim for r in reqs) == set(range(8))
    a = serve.poisson_arrivals(20000, 500.0)
    assert np.all(np.diff(a) > 0)
    assert abs(20000 / a[-1] - 500.0) < 25.0
    b = serve.poisson_arrivals(20000, 1000.0)
    assert np.allclose(a / 2, b)
    assert serve.make_requests(spec, 5)[3] == serve.make_requests(spec, 5)[3]


def test_scaled_spec_keeps_its_shape():
    s = serve.scaled(serve.SERVE, 2000)
    assert s.dim_keys[0] == 100 and s.dim_keys[-1] == 100_000
    assert all(g <= k for g, k in zip(s.dim_groups, s.dim_keys))
    assert s.fact_rows == 500_000 and s.probe_max == 500_000
    assert s.n_ranks >= s.dim_keys[-1]


def test_oracle_request_matches_a_direct_restatement():
    spec = serve.scaled(serve.SERVE, 20000)
    from pageflow_b200.datagen import zipf_table
    edges, thr = zipf_table(spec.n_ranks, spec.zipf_s)
    d = 5
    keys, groups = oracle.gen_serve_dim(spec.seed, spec.n_ranks, 99, spec.dim_groups[d], 0,
                                        spec.dim_keys[d])
    assert len(np.unique(keys)) == keys.shape[0]
    fk, date, value = oracle.gen_serve_fact(spec.seed, spec.n_ranks, 100, 20000, edges, thr)
    got = oracle.serve_request(keys, groups, spec.dim_groups[d], fk, date, value, 8500, 9500)
    # direct: a dict join
    grp = dict(zip(keys.tolist(), groups.tolist()))
    acc = {}
    for f, dt, v in zip(fk.tolist(), date.tolist(), value.tolist()):
        if 8500 <= dt < 9500 and f in grp:
            s, c = acc.get(grp[f], (0, 0))
            acc[grp[f]] = (s + v, c + 1)
    ks = sorted(acc)
    assert np.array_equal(got[0], ks)
    assert np.array_equal(got[1], [acc[k][0] for k in ks])
    assert np.array_equal(got[2], [acc[k][1] for k in ks])
    # smaller dimensions hold the hotter ranks: they match a larger share
    small = set(oracle.gen_serve_dim(spec.seed, spec.n_ranks, 1, 1, 0, spec.dim_keys[0])[0])
    share = np.mean([f in small for f in fk.tolist()])
    assert share > spec.dim_keys[0] / spec.n_ranks * 3
