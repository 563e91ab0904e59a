"""The sorted-run primitives on the GPU (pageflow_b200.sorted_run_merge, the
mirror of operators/sorted_run_merge.py): the radix sort against a stable
numpy sort (full int64 range, negatives, duplicates, one key, empty), and
reduce_tick_slice / merge_sorted_unique_runs_inplace against the golden
vectors the reference's own functions produced (tests/golden/sorted_run.npz)
and against numpy for every op, integer and float columns, 2-D values and
runs that share no, some or all keys."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from pageflow_b200 import sorted_run_merge as srm
from tests.golden import load

pytestmark = pytest.mark.gpu

I64 = np.iinfo(np.int64)


@pytest.mark.parametrize("case", ["full", "small", "dups", "one_value", "single", "empty",
                                  "negative", "large", "tiny_full"])
def test_radix_sort_is_a_stable_sort(case):
    rng = np.random.default_rng(sum(map(ord, case)))
    n = {"single": 1, "empty": 0, "large": 3_000_000, "tiny_full": 1000}.get(case, 50_000)
    if case in ("full", "tiny_full"):
        k = rng.integers(I64.min, I64.max, n, dtype=np.int64)
    elif case in ("small", "large"):
        k = rng.integers(-300, 300, n).astype(np.int64)
    elif case == "dups":
        k = rng.integers(0, 5, n).astype(np.int64) * (1 << 40)
    elif case == "one_value":
        k = np.full(n, -7, np.int64)
    elif case == "negative":
        k = -rng.integers(1, 1 << 50, n).astype(np.int64)
    else:
        k = rng.integers(-10, 10, n).astype(np.int64)
    ko, vo = srm.sort_pairs(torch.from_numpy(k).cuda())
    order = np.argsort(k, kind="stable")
    assert np.array_equal(ko.cpu().numpy(), k[order])
    assert np.array_equal(vo.cpu().numpy(), order)
    payload = torch.from_numpy(rng.integers(0, 1 << 60, n).astype(np.int64))
    ko2, vo2 = srm.sort_pairs(torch.from_numpy(k).cuda(), payload.cuda())
    assert np.array_equal(vo2.cpu().numpy(), payload.numpy()[order])


@pytest.mark.parametrize("case", [0, 1, 2])
def test_golden_reduce_and_merge(case):
    g = load("sorted_run.npz")
    keys = torch.from_numpy(g[f"c{case}_keys"]).cuda()
    v = torch.from_numpy(g[f"c{case}_v"]).cuda()
    w = torch.from_numpy(g[f"c{case}_w"]).cuda()
    u, (rs, rm) = srm.reduce_tick_slice(keys, [v, w], ["sum", "amax"])
    assert np.array_equal(u.cpu().numpy(), g[f"c{case}_u"])
    assert np.array_equal(rs.cpu().numpy(), g[f"c{case}_sum"])
    assert np.array_equal(rm.cpu().numpy(), g[f"c{case}_max"])
    half = keys.numel() // 2
    ua, (sa,) = srm.reduce_tick_slice(keys[:half], [v[:half]], ["sum"])
    ub, (sb,) = srm.reduce_tick_slice(keys[half:], [v[half:]], ["sum"])
    kb = torch.empty(ua.numel() + ub.numel(), dtype=torch.int64, device="cuda")
    vb = torch.empty_like(kb)
    kb[:ua.numel()], vb[:ua.numel()] = ua, sa
    m = srm.merge_sorted_unique_runs_inplace(kb, [vb], ua.numel(), ub, [sb], ["sum"],
                                             place_chunk_rows=7)
    assert np.array_equal(kb[:m].cpu().numpy(), g[f"c{case}_merged_keys"])
    assert np.array_equal(vb[:m].cpu().numpy(), g[f"c{case}_merged_sum"])


def _np_reduce(keys, vals, ops):
    u, inv = np.unique(keys, return_inverse=True)
    out = []
    for v, op in zip(vals, ops):
        res = np.zeros((u.shape[0],) + v.shape[1:], dtype=v.dtype)
        f = {"sum": np.add, "amax": np.maximum, "amin": np.minimum}[op]
        first = np.ones(u.shape[0], bool)
        for i in range(keys.shape[0]):
            j = inv[i]
            res[j] = v[i] if first[j] else f(res[j], v[i])
            first[j] = False
        out.append(res)
    return u, out


@pytest.mark.parametrize("dtype", [np.int64, np.int32])
def test_reduce_every_op_and_width(dtype):
    rng = np.random.default_rng(3)
    n = 20_000
    keys = rng.integers(-2000, 2000, n).astype(np.int64)
    vals = [rng.integers(-10**6, 10**6, n).astype(dtype) for _ in range(3)]
    vals.append(rng.integers(-50, 50, (n, 3)).astype(dtype))
    ops = ["sum", "amax", "amin", "amax"]
    u, outs = srm.reduce_tick_slice(torch.from_numpy(keys).cuda(),
                                    [torch.from_numpy(v).cuda() for v in vals], ops)
    eu, eouts = _np_reduce(keys, vals, ops)
    assert np.array_equal(u.cpu().numpy(), eu)
    for o, e in zip(outs, eouts):
        assert o.dtype == torch.from_numpy(e).dtype
        assert np.array_equal(o.cpu().numpy(), e)


def test_reduce_float_columns_within_tolerance():
    rng = np.random.default_rng(4)
    n = 30_000
    keys = rng.integers(0, 500, n).astype(np.int64)
    f64 = rng.standard_normal(n)
    f32 = rng.standard_normal((n, 2)).astype(np.float32)
    u, (s64, mx32, mn64) = srm.reduce_tick_slice(
        torch.from_numpy(keys).cuda(),
        [torch.from_numpy(f64).cuda(), torch.from_numpy(f32).cuda(),
         torch.from_numpy(f64).cuda()], ["sum", "amax", "amin"])
    eu, (es, emx, emn) = _np_reduce(keys, [f64, f32, f64], ["sum", "amax", "amin"])
    assert np.array_equal(u.cpu().numpy(), eu)
    assert np.allclose(s64.cpu().numpy(), es, rtol=1e-12, atol=1e-9)  # order of float adds
    assert np.array_equal(mx32.cpu().numpy(), emx) and np.array_equal(mn64.cpu().numpy(), emn)


@pytest.mark.parametrize("overlap", ["none", "some", "all", "tick_below", "tick_above"])
def test_merge_runs(overlap):
    rng = np.random.default_rng(5)
    a = np.unique(rng.integers(0, 100_000, 30_000)).astype(np.int64)
    if overlap == "none":
        b = np.setdiff1d(np.unique(rng.integers(0, 100_000, 20_000)), a).astype(np.int64)
    elif overlap == "all":
        b = a[::3].copy()
    elif overlap == "tick_below":
        b = np.arange(-5000, -10, dtype=np.int64)
    elif overlap == "tick_above":
        b = np.arange(200_000, 205_000, dtype=np.int64)
    else:
        b = np.unique(rng.integers(0, 100_000, 20_000)).astype(np.int64)
    av = [rng.integers(-10**6, 10**6, a.shape[0]), rng.integers(-9, 9, (a.shape[0], 2))]
    bv = [rng.integers(-10**6, 10**6, b.shape[0]), rng.integers(-9, 9, (b.shape[0], 2))]
    cap = a.shape[0] + b.shape[0] + 7
    kb = torch.zeros(cap, dtype=torch.int64, device="cuda")
    vb0 = torch.zeros(cap, dtype=torch.int64, device="cuda")
    vb1 = torch.zeros((cap, 2), dtype=torch.int64, device="cuda")
    kb[:a.shape[0]] = torch.from_numpy(a)
    vb0[:a.shape[0]] = torch.from_numpy(av[0])
    vb1[:a.shape[0]] = torch.from_numpy(av[1])
    m = srm.merge_sorted_unique_runs_inplace(kb, [vb0, vb1], a.shape[0], torch.from_numpy(b).cuda(),
                                             [torch.from_numpy(x).cuda() for x in bv],
                                             ["sum", "amin"])
    keys = np.concatenate([a, b])
    eu, (e0, e1) = _np_reduce(keys, [np.concatenate([av[0], bv[0]]),
                                     np.concatenate([av[1], bv[1]])], ["sum", "amin"])
    assert m == eu.shape[0]
    assert np.array_equal(kb[:m].cpu().numpy(), eu)
    assert np.array_equal(vb0[:m].cpu().numpy(), e0)
    assert np.array_equal(vb1[:m].cpu().numpy(), e1)


def test_merge_edges_and_errors():
    kb = torch.zeros(10, dtype=torch.int64, device="cuda")
    vb = torch.zeros(10, dtype=torch.int64, device="cuda")
    t = torch.tensor([3, 5], dtype=torch.int64, device="cuda")
    assert srm.merge_sorted_unique_runs_inplace(kb, [vb], 0, t, [t * 10], ["sum"]) == 2
    assert kb[:2].tolist() == [3, 5] and vb[:2].tolist() == [30, 50]
    e = torch.empty(0, dtype=torch.int64, device="cuda")
    assert srm.merge_sorted_unique_runs_inplace(kb, [vb], 2, e, [e], ["sum"]) == 2
    with pytest.raises(ValueError):
        srm.reduce_tick_slice(t, [t], ["mean"])
    with pytest.raises(TypeError):
        srm.reduce_tick_slice(t, [t.to(torch.int16)], ["sum"])
    u, outs = srm.reduce_tick_slice(e, [e], ["sum"])
    assert u.numel() == 0 and outs[0].numel() == 0
