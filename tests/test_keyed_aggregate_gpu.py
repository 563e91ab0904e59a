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
from tests.golden import load

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
    mx = np.maximum(mx, 0)           # the reference's MAX partial folds from 0
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


# ---- against the reference's own KeyedAggregate.pass1 ------------------------------

KEYED = load("keyed_pass1.npz")
KEYED_CASES = ["one", "two", "three", "wide"]


def _keyed_columns(case):
    nk = int(KEYED[f"{case}_nkeys"][0])
    cols = {i + 1: torch.from_numpy(KEYED[f"{case}_key{i}"]).cuda() for i in range(nk)}
    cols.update({10: torch.from_numpy(KEYED[f"{case}_v"]).cuda(),
                 11: torch.from_numpy(KEYED[f"{case}_w"]).cuda(),
                 12: torch.from_numpy(KEYED[f"{case}_f"]).cuda()})
    return nk, cols


@pytest.mark.parametrize("case", KEYED_CASES)
def test_pass1_is_the_references(case):
    """The chunk's groups bit for bit as the reference's KeyedAggregate.pass1
    returned them (tests/golden/make_keyed_golden.py): the grouping hashes
    ascending, every key column's representatives, SUM / COUNT / MIN / MAX and
    AVG's (sum, count) state, each group's bucket and the groups per bucket.
    The coefficients are the ones the reference drew on the CPU; that the
    module draws the same ones is pinned on the CPU
    (tests/test_keyed_coeffs.py)."""
    nk, cols = _keyed_columns(case)
    p1 = ka.KeyedPass1(list(range(1, nk + 1)),
                       [('sum', 10), ('count', None), ('min', 11), ('max', 11), ('avg', 12)])
    p1._coeffs = [torch.from_numpy(KEYED[f"{case}_coeff{i}"]).cuda() for i in range(nk)]
    out, buckets = p1.pass1(cols, B=64)
    assert len(out) == int(KEYED[f"{case}_nout"][0])
    for j, t in enumerate(out):
        want = KEYED[f"{case}_out{j}"]
        got = t.cpu().numpy()
        assert got.dtype == want.dtype and got.shape == want.shape, f"output {j}"
        assert np.array_equal(got, want), f"output {j}"   # AVG's sums are dyadic: exact
    bucket, counts, counts_t = buckets
    assert np.array_equal(bucket.cpu().numpy(), KEYED[f"{case}_bucket"])
    assert counts == KEYED[f"{case}_bucket_counts"].tolist() == counts_t.tolist()


@pytest.mark.parametrize("case", KEYED_CASES)
def test_pass1_outputs_partition_into_the_padded_layout(case):
    """Pass 1's outputs partitioned by their grouping hash through the
    drop-in partition kernel, as the reference's _partition_outputs lays
    them out (operators/aggregate.py:119-152): the groups per bucket are
    the reference's, every bucket holds its groups in ascending-hash order,
    each output column starts its buckets on whole lcm(row bytes, 512)-byte
    units."""
    from pageflow_b200 import tqpkernels
    from tests.dropin import padded_starts, row_bytes
    nout = int(KEYED[f"{case}_nout"][0])
    outs = [torch.from_numpy(KEYED[f"{case}_out{j}"]).cuda() for j in range(nout)]
    counts_want = KEYED[f"{case}_bucket_counts"]
    bucket = KEYED[f"{case}_bucket"]
    order = np.argsort(bucket, kind="stable")
    B = 64
    n = outs[0].shape[0]
    # the kernel takes six columns a call: the hash with up to five outputs
    # more (each call's widths within its four classes)
    got, srcs = [], []
    for k in range(1, nout, 3):
        cols = [outs[0]] + outs[k:k + 3]
        host = torch.empty(B + tqpkernels.MAXCLS + 1, dtype=torch.int64, pin_memory=True)
        res = tqpkernels.partition_sort(cols, [0] * len(cols), 0, None, n, 0, B, False, host)
        assert host[:B].tolist() == counts_want.tolist()
        got += res[:len(cols)]
        srcs += cols
    for t, src in zip(got, srcs):
        starts, _ = padded_starts(counts_want.tolist(), row_bytes(t))
        want_rows = src.cpu().numpy()[order]
        have = t.cpu().numpy()
        at = 0
        for s, c in zip(starts, counts_want):
            assert np.array_equal(have[s:s + c], want_rows[at:at + c])
            at += c


def _keys_for_buckets(bucket, B, seed):
    """Keys whose mix64 has the given top log2(B) bits (mix64 inverted on
    uint64 words), so the drop-in's hash buckets are exactly `bucket`."""
    logb = int(B).bit_length() - 1
    rng = np.random.default_rng(seed)
    low = rng.integers(0, 1 << 62, bucket.shape[0], dtype=np.int64).astype(np.uint64)
    if logb:
        h = (bucket.astype(np.uint64) << np.uint64(64 - logb)) | (low >> np.uint64(logb))
    else:
        h = low
    with np.errstate(over="ignore"):
        h ^= h >> np.uint64(33)
        h *= np.uint64(pow(0xc4ceb9fe1a85ec53, -1, 1 << 64))
        h ^= h >> np.uint64(33)
        h *= np.uint64(pow(0xff51afd7ed558ccd, -1, 1 << 64))
        h ^= h >> np.uint64(33)
    return h.view(np.int64)


@pytest.mark.parametrize("case", range(4))
def test_drop_in_layout_is_the_references_partition_outputs(case):
    """The reference's _partition_outputs vectors (tests/golden/
    partition_layout.npz: its bucket ids, three outputs of 8, 1 and 25-byte
    rows) through the drop-in kernel, keyed so that each row's hash bucket is
    its given bucket: the same padded totals, bucket starts and bucket rows."""
    from pageflow_b200 import tqpkernels
    from tests.dropin import row_bytes
    g = load("partition_layout.npz")
    B = int(g[f"c{case}_B"][0])
    bucket = g[f"c{case}_bucket"]
    key = _keys_for_buckets(bucket, B, case)
    assert np.array_equal(oracle.bucket(key, B), bucket)
    cols = [torch.from_numpy(key).cuda()] + [torch.from_numpy(g[f"c{case}_in{j}"]).cuda()
                                              for j in range(3)]
    host = torch.empty(B + tqpkernels.MAXCLS + 1, dtype=torch.int64, pin_memory=True)
    n = bucket.shape[0]
    outs = tqpkernels.partition_sort(cols, [0] * 4, 0, None, n, 0, B, False, host)
    counts = host[:B].tolist()
    assert counts == g[f"c{case}_counts"].tolist()
    widths = []
    for t in cols:
        if row_bytes(t) not in widths:
            widths.append(row_bytes(t))
    for j in range(3):
        t = outs[1 + j]
        total = int(host[B + widths.index(row_bytes(t))])
        ref_total = int(g[f"c{case}_total{j}"][0])
        assert total == ref_total
        starts = g[f"c{case}_starts{j}"]   # rows (PartitionedTensor.bucket_starts)
        have = t[:total].cpu().numpy()
        rows = np.concatenate([have[s:s + c]
                               for s, c in zip(starts.tolist(), counts)])
        assert np.array_equal(rows, g[f"c{case}_rows{j}"])
