"""The drop-in join cores (``tqpkernels.join_unique_hash``, ``join_semi_anti``
and ``join_expand``, narrowed by host_out as the reference's
operators/join_core.py does) against the oracle and brute force, on the cases of the reference's
tests/operators/test_join_core.py: expand with empty runs and random runs,
semi/anti with each residual operator over duplicate-heavy keys, the
all-true/all-false summaries, extreme keys and the empty-slot key, keys of one
radix bucket, unique-hash tuples of one and two keys; plus the golden pairs
the reference's _sort_search_pairs produced."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from tests.dropin import expand_pairs, semi_anti_rows, unique_pairs
from tests.golden import load

pytestmark = pytest.mark.gpu

_I64_MIN = -(1 << 63)
_I64_MAX = (1 << 63) - 1
NULL = -64
# residual operators, oriented build value OP probe value (the kernel's codes)
OPS = {'<>': 1, '<': 2, '<=': 3, '>': 4, '>=': 5}


def semi_anti(bk, pk, anti, summary=None):
    if summary is None:
        return semi_anti_rows(bk, pk, anti)
    bv, pv, op = summary
    return semi_anti_rows(bk, pk, anti, bv, pv, OPS[op])


def _cuda(values):
    return torch.tensor(values, dtype=torch.int64, device="cuda")


def _rand(n, lo, hi, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.randint(lo, hi, (n,), generator=g, dtype=torch.int64).cuda()


@pytest.mark.parametrize("lengths", [[], [0], [0, 0, 0], [1], [3], [1, 0, 2, 0, 0, 3, 0],
                                     [0, 0, 5], [5, 0, 0], [2, 2, 2, 2]])
def test_expand_matches_oracle_with_empty_runs(lengths):
    length = _cuda(lengths)
    n_build = max(8, sum(lengths) + 3)
    sorted_ids = torch.randperm(n_build, device="cuda")
    start = _cuda([(3 * i) % (n_build - n) if n_build > n else 0 for i, n in enumerate(lengths)])
    cs, cr = expand_pairs(sorted_ids, start, length)
    ref_cs, ref_cr = oracle.expand(sorted_ids.cpu().numpy(), start.cpu().numpy(),
                                   length.cpu().numpy())
    assert np.array_equal(cs.cpu().numpy(), ref_cs) and np.array_equal(cr.cpu().numpy(), ref_cr)


def test_expand_random_runs():
    n_probe, n_build = 60_000, 200_000
    length = _rand(n_probe, 0, 7, 1)
    length[_rand(n_probe, 0, 10, 2) < 4] = 0
    start = torch.minimum(_rand(n_probe, 0, n_build, 3), n_build - length)
    sorted_ids = torch.randperm(n_build, device="cuda")
    cs, cr = expand_pairs(sorted_ids, start, length)
    ref_cs, ref_cr = oracle.expand(sorted_ids.cpu().numpy(), start.cpu().numpy(),
                                   length.cpu().numpy())
    assert np.array_equal(cs.cpu().numpy(), ref_cs) and np.array_equal(cr.cpu().numpy(), ref_cr)


def test_expand_long_runs_and_many_rows():
    n = 3_000_000
    length = _rand(n, 0, 3, 4)
    length[::100_000] = 5000
    start = torch.zeros(n, dtype=torch.int64, device="cuda")
    sorted_ids = torch.arange(6000, dtype=torch.int64, device="cuda")
    cs, cr = expand_pairs(sorted_ids, start, length)
    ref_cs, ref_cr = oracle.expand(sorted_ids.cpu().numpy(), start.cpu().numpy(),
                                   length.cpu().numpy())
    assert np.array_equal(cs.cpu().numpy(), ref_cs) and np.array_equal(cr.cpu().numpy(), ref_cr)


@pytest.mark.parametrize("anti", [False, True])
@pytest.mark.parametrize("op", [None, '<>', '<', '<=', '>', '>='])
@pytest.mark.parametrize("n_build,n_probe", [(1, 1), (7, 300), (2000, 1500),
                                             (40_000, 3000), (300_000, 1_000_000)])
def test_semi_anti_matches_oracle(anti, op, n_build, n_probe):
    seed = n_build * 7 + n_probe
    bk = _rand(n_build, -50, max(n_build // 3, 1), seed)
    pk = _rand(n_probe, -60, 2 * max(n_build // 3, 1), seed + 1)
    bv = _rand(n_build, 0, 4, seed + 2)
    pv = _rand(n_probe, 0, 4, seed + 3)
    summary = (bv, pv, op) if op is not None else None
    got = semi_anti(bk, pk, anti, summary)
    want = oracle.semi_anti(bk.cpu().numpy(), pk.cpu().numpy(), anti,
                            bv.cpu().numpy() if op else None, pv.cpu().numpy() if op else None,
                            op)
    assert np.array_equal(got.cpu().numpy(), want)


@pytest.mark.parametrize("anti", [False, True])
def test_summary_all_true_and_all_false(anti):
    bk = _cuda([1, 1, 1, 2, 2, 3])
    pk = _cuda([1, 2, 3, 4, 1])
    same = _cuda([9] * 6)
    got = semi_anti(bk, pk, anti, (same, _cuda([9] * 5), '<>'))
    assert got.tolist() == ([0, 1, 2, 3, 4] if anti else [])
    got = semi_anti(bk, pk, anti, (same, _cuda([5] * 5), '<>'))
    assert got.tolist() == ([3] if anti else [0, 1, 2, 4])


def test_semi_anti_extreme_keys_and_null_sentinel():
    keys = [_I64_MIN + 1, -1, 0, NULL, _I64_MAX, 42]
    bk = _cuda(keys[:4])
    pk = _cuda(keys + [_I64_MIN])
    assert semi_anti(bk, pk, False).tolist() == [0, 1, 2, 3]
    assert semi_anti(bk, pk, True).tolist() == [4, 5, 6]


def test_semi_anti_refuses_the_empty_slot_key():
    assert semi_anti(_cuda([3, _I64_MIN]), _cuda([3]), False) is None


def _one_bucket_keys(n, B=128, bucket=5, seed=0):
    cand = torch.randperm(n * B * 2, generator=torch.Generator().manual_seed(seed))
    b = oracle.bucket(cand.numpy().astype(np.int64), B)
    cand = cand[torch.from_numpy(b == bucket)][:n]
    assert cand.numel() == n
    return cand.cuda()


def test_tables_with_keys_of_one_radix_bucket():
    keys = _one_bucket_keys(20_000)
    probe = torch.cat((keys[::3], keys[1::7] + (1 << 40)))
    got = semi_anti(keys, probe, False)
    want = oracle.semi_anti(keys.cpu().numpy(), probe.cpu().numpy(), False)
    assert np.array_equal(got.cpu().numpy(), want)
    build_idx, probe_idx = unique_pairs([keys], [probe])
    assert torch.equal(probe[probe_idx], keys[build_idx])
    assert probe_idx.tolist() == list(range(keys[::3].numel()))


@pytest.mark.parametrize("two", [False, True])
def test_unique_hash_random_tuples(two):
    n_build, n_probe = 30_000, 50_000
    k0 = torch.randperm(n_build * 4, device="cuda")[:n_build]
    build = [k0 // 3, k0 % 3] if two else [k0]
    picks = _rand(n_probe, 0, n_build, 11)
    miss = _rand(n_probe, 0, 4, 12) == 0
    p0 = torch.where(miss, k0[picks] + n_build * 8, k0[picks])
    probe = [p0 // 3, p0 % 3] if two else [p0]
    build_idx, probe_idx = unique_pairs(build, probe)
    assert torch.equal(probe_idx, torch.nonzero(~miss).view(-1))
    assert torch.equal(build_idx, picks[probe_idx])


@pytest.mark.parametrize("tag", ["one", "two"])
def test_unique_hash_pairs_are_the_references(tag):
    g = load("join_small.npz")
    if tag == "one":
        b, p = [torch.from_numpy(g["one_b0"]).cuda()], [torch.from_numpy(g["one_p0"]).cuda()]
    else:
        b = [torch.from_numpy(g["two_b0"]).cuda(), torch.from_numpy(g["two_b1"]).cuda()]
        p = [torch.from_numpy(g["two_p0"]).cuda(), torch.from_numpy(g["two_p1"]).cuda()]
    bi, pi = unique_pairs(b, p)
    assert np.array_equal(bi.cpu().numpy(), g[f"{tag}_build_idx"])
    assert np.array_equal(pi.cpu().numpy(), g[f"{tag}_probe_idx"])


def test_unique_hash_extreme_keys():
    bk = _cuda([_I64_MIN, _I64_MAX, 0, -1, NULL])
    pk = _cuda([-1, 5, _I64_MIN, NULL, _I64_MAX, _I64_MAX])
    bi, pi = unique_pairs([bk], [pk])
    assert pi.tolist() == [0, 2, 3, 4, 5]
    assert bi.tolist() == [3, 0, 4, 1, 1]


def test_unique_hash_large_vs_oracle():
    nb, np_ = 2_000_000, 8_000_000
    bk = torch.randperm(4 * nb, device="cuda")[:nb].to(torch.int64) * 7919 - (1 << 35)
    pk = bk[_rand(np_, 0, nb, 21)]
    pk[_rand(np_, 0, 10, 22) == 0] += 1
    bi, pi = unique_pairs([bk], [pk])
    obi, opi = oracle.join_unique([bk.cpu().numpy()], [pk.cpu().numpy()])
    assert np.array_equal(pi.cpu().numpy(), opi) and np.array_equal(bi.cpu().numpy(), obi)


def test_unique_hash_chains_of_one_fingerprint():
    """Build keys whose hashes differ only in bits 30-35: one home slot and one
    fingerprint for all of them (the table keeps the hash's low bits beside
    the row), so a probe walks a chain of fingerprint matches and checks each
    candidate's key; probe keys made the same way but absent walk it to the
    end and miss."""
    from tests.test_aggregate_gpu import _unmix64
    h0 = 0x5DEECE66D1234567
    chain = [_unmix64((h0 + (j << 30)) & ((1 << 64) - 1)) for j in range(80)]
    rest = (torch.randperm(1 << 20, generator=torch.Generator().manual_seed(5))[:1000] + 7).tolist()
    bk = _cuda(chain[:64] + [k for k in rest if k not in set(chain)])
    probe = chain[::-1] + rest[::3] + chain[60:70] + [k + (1 << 40) for k in rest[:50]]
    pk = _cuda(probe)
    bi, pi = unique_pairs([bk], [pk])
    obi, opi = oracle.join_unique([bk.cpu().numpy()], [pk.cpu().numpy()])
    assert np.array_equal(pi.cpu().numpy(), opi) and np.array_equal(bi.cpu().numpy(), obi)
    assert torch.equal(pk[pi], bk[bi]) and pi.numel() == 64 + len(rest[::3]) + 4


def test_empty_sides_are_refused_by_the_kernel_entry():
    """A side without rows is the caller's to short-circuit (the reference's
    wrappers return before the kernel); the entry points refuse it."""
    e = torch.empty(0, dtype=torch.int64, device="cuda")
    k = _cuda([1, 2])
    with pytest.raises(RuntimeError, match="both sides"):
        unique_pairs([e], [k])
    with pytest.raises(RuntimeError, match="both sides"):
        semi_anti(e, k, True)
    with pytest.raises(RuntimeError, match="both sides"):
        semi_anti(k, e, False)
    cs, cr = expand_pairs(k, _cuda([]), _cuda([]))
    assert cs.numel() == 0 and cr.numel() == 0
