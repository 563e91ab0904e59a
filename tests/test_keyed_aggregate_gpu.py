"""The keyed aggregation's hash route (pageflow_b200.keyed_aggregate, the
mirror of KeyedAggregate.pass1) against a numpy restatement of the
reference's pass 1 with the same coefficients: the linear hash of packed key
words, the unique hashes ascending, one key representative per group, the
partials, and the buckets (checked against the oracle's mix64 buckets)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from pageflow_b200 import keyed_aggregate as ka

pytestmark = pytest.mark.gpu


def _words(col: np.ndarray) -> np.ndarray:
    n = col.shape[0]
    raw = np.ascontiguousarray(col).view(np.uint8).reshape(n, -1)
    rb = raw.shape[1]
    tb = (rb + 7) // 8 * 8
    buf = np.zeros((n, tb), np.uint8)
    buf[:, :rb] = raw
    return buf.view(np.int64)


def _np_hash(keys, coeffs):
    h = np.zeros(keys[0].shape[0], np.uint64)
    for k, c in zip(keys, coeffs):
        w = _words(k if k.ndim == 2 else k[:, None]).astype(np.uint64)
        h += (w * c.astype(np.uint64)).sum(axis=1, dtype=np.uint64)
    return h.view(np.int64)


@pytest.mark.parametrize("case", ["int64", "int32_int64", "int16_wide", "float64", "bool_int8"])
def test_pass1_matches_the_restatement(case):
    rng = np.random.default_rng(sum(map(ord, case)))
    n = 40_000
    if case == "int64":
        keys = [rng.integers(-500, 500, n).astype(np.int64)]
    elif case == "int32_int64":
        keys = [rng.integers(0, 30, n).astype(np.int32), rng.integers(-3, 3, n).astype(np.int64)]
    elif case == "int16_wide":
        keys = [rng.integers(-4, 4, (n, 3)).astype(np.int16)]
    elif case == "float64":
        keys = [rng.integers(0, 200, n).astype(np.float64) / 8]
    else:
        keys = [rng.integers(0, 2, n).astype(bool), rng.integers(-2, 3, n).astype(np.int8)]
    v = rng.integers(-10**6, 10**6, n).astype(np.int64)
    w = rng.integers(-100, 100, n).astype(np.int32)
    f = rng.standard_normal(n)
    cols = {i + 1: torch.from_numpy(k).cuda() for i, k in enumerate(keys)}
    cols.update({10: torch.from_numpy(v).cuda(), 11: torch.from_numpy(w).cuda(),
                 12: torch.from_numpy(f).cuda()})
    p1 = ka.KeyedPass1(list(range(1, len(keys) + 1)),
                       [('sum', 10), ('count', None), ('min', 11), ('max', 11), ('sum', 11),
                        ('avg', 12)])
    out, buckets = p1.pass1(cols, B=64)
    coeffs = [c.cpu().numpy() for c in p1._coeffs]
    assert all(2 <= c.min() and c.max() < 10_000_000 for c in coeffs)
    h = _np_hash(keys, coeffs)
    u, inv = np.unique(h, return_inverse=True)
    assert np.array_equal(out[0].cpu().numpy(), u)
    nk = len(keys)
    for i, k in enumerate(keys):
        rep = np.zeros((u.shape[0],) + k.shape[1:], k.dtype)
        rep[inv] = k
        assert np.array_equal(out[1 + i].cpu().numpy(), rep), f"key {i}"
    agg = out[1 + nk:]
    sums = np.zeros(u.shape[0], np.int64)
    np.add.at(sums, inv, v)
    cnt = np.bincount(inv, minlength=u.shape[0])
    mn = np.full(u.shape[0], np.iinfo(np.int32).max, np.int32)
    mx = np.full(u.shape[0], np.iinfo(np.int32).min, np.int32)
    np.minimum.at(mn, inv, w)
    np.maximum.at(mx, inv, w)
    s11 = np.zeros(u.shape[0], np.int64)
    np.add.at(s11, inv, w.astype(np.int64))
    fs = np.zeros(u.shape[0])
    np.add.at(fs, inv, f)
    assert np.array_equal(agg[0].cpu().numpy(), sums)
    assert np.array_equal(agg[1].cpu().numpy(), cnt)
    assert np.array_equal(agg[2].cpu().numpy(), mn) and np.array_equal(agg[3].cpu().numpy(), mx)
    assert agg[4].dtype == torch.int64 and np.array_equal(agg[4].cpu().numpy(), s11)
    avg = agg[5].cpu().numpy()
    assert np.allclose(avg[:, 0], fs, rtol=1e-12, atol=1e-9) and np.array_equal(avg[:, 1], cnt)
    bucket, counts, counts_t = buckets
    eb = oracle.bucket(u, 64)
    assert np.array_equal(bucket.cpu().numpy(), eb)
    assert counts == np.bincount(eb, minlength=64).tolist()
    assert counts_t.tolist() == counts


def test_pass1_one_bucket_and_coefficients_are_deterministic():
    k = torch.arange(1000, dtype=torch.int64, device="cuda") % 7
    a = ka.KeyedPass1([1], [('count', None)])
    b = ka.KeyedPass1([1], [('count', None)])
    oa, ba = a.pass1({1: k}, B=1)
    ob, _ = b.pass1({1: k}, B=1)
    assert ba is None
    assert all(torch.equal(x, y) for x, y in zip(oa, ob))
    assert torch.equal(a._coeffs[0], b._coeffs[0])
    assert oa[2].tolist() == [143] * 6 + [142] or sorted(oa[2].tolist()) == [142] + [143] * 6
