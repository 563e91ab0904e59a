"""The join core dispatch (pageflow_b200.hashjoin.join_kernel_new, the mirror
of operators/hashjoin.py) and the one-launch gather (pageflow_b200.gather)
against the oracle's join semantics: every join type, the unique-hash core
with one and two keys and residuals, the hash semi / anti set with its
summary residual and its INT64_MIN refusal, the sort/search core with
bucket counts, each guard's fallback, right-outer nulls per dtype, and the
gather's null and range handling."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from pageflow_b200 import gather, hashjoin

pytestmark = pytest.mark.gpu

L_KEY, L_V, L_F, L_K2 = 1, 2, 3, 4
R_KEY, R_V, R_X, R_K2 = 11, 12, 13, 14


def _tables(n_left, n_right, unique_left, seed, key_range=None):
    g = torch.Generator().manual_seed(seed)
    kr = key_range or max(4, n_left * 2)
    if unique_left:
        lk = torch.randperm(kr, generator=g)[:n_left].to(torch.int64)
    else:
        lk = torch.randint(0, max(2, n_left // 3), (n_left,), generator=g, dtype=torch.int64)
    rk = torch.randint(0, kr, (n_right,), generator=g, dtype=torch.int64)
    left = {L_KEY: lk, L_V: torch.randint(-50, 50, (n_left,), generator=g, dtype=torch.int64),
            L_F: torch.randn(n_left, generator=g, dtype=torch.float32),
            L_K2: torch.randint(0, 3, (n_left,), generator=g, dtype=torch.int64)}
    right = {R_KEY: rk, R_V: torch.randint(-50, 50, (n_right,), generator=g, dtype=torch.int64),
             R_X: torch.randint(0, 100, (n_right, 2), generator=g, dtype=torch.int32),
             R_K2: torch.randint(0, 3, (n_right,), generator=g, dtype=torch.int64)}
    cpu = ({k: v.clone() for k, v in left.items()}, {k: v.clone() for k, v in right.items()})
    return ({k: v.cuda() for k, v in left.items()}, {k: v.cuda() for k, v in right.items()},
            cpu)


def _rows(out, n_out_cols):
    """The output rows as sorted tuples (global indexes last)."""
    cols = [c.cpu() for c in out]
    n = cols[0].shape[0] if cols else 0
    rows = []
    for i in range(n):
        row = []
        for c in cols:
            v = c[i]
            row.extend(v.reshape(-1).tolist())
        rows.append(tuple(row))
    return sorted(rows)


def _expected(cpu, pairs, keys):
    left, right = cpu
    rows = []
    for l, r in pairs:
        row = []
        for k in keys:
            if k in left:
                v = left[k][l] if l != -64 else torch.full_like(left[k][0], -64)
            else:
                v = right[k][r]
            row.extend(v.reshape(-1).tolist())
        row.extend([l if l != -64 else -64, r])  # global indexes: the identity here
        rows.append(tuple(row))
    return sorted(rows)


def _run(left, right, jt, conds=None, eq=None, uniq=None, keys=(L_KEY, L_V, L_F, R_V, R_X),
         buckets=None, limit=None):
    lg = torch.arange(left[L_KEY].numel(), dtype=torch.int64, device="cuda")
    rg = torch.arange(right[R_KEY].numel(), dtype=torch.int64, device="cuda")
    out = hashjoin.join_kernel_new(left, right, L_KEY, R_KEY, conds or [], list(keys), True, jt,
                                   lg, rg, bucket_counts=buckets, equality_keys=eq,
                                   unique_key_sets=uniq, hash_scratch_limit_bytes=limit)
    return out


KEYS = (L_KEY, L_V, L_F, R_V, R_X)


@pytest.mark.parametrize("jt", ["inner", "right-semi", "right-anti", "right-outer"])
@pytest.mark.parametrize("unique", [True, False])
def test_join_types_match_the_oracle(jt, unique):
    left, right, cpu = _tables(3000, 9000, unique, seed=1 + unique)
    eq = ([L_KEY], [R_KEY])
    uniq = ([[L_KEY]], []) if unique else ([], [])
    before = sum(hashjoin.fallback_reasons.values())
    out = _run(left, right, jt, eq=eq, uniq=uniq)
    pairs = oracle.join_rows(cpu[0][L_KEY].numpy(), cpu[1][R_KEY].numpy(), jt)
    if jt in ("right-semi", "right-anti"):
        # no left rows in the output: left columns come back empty
        assert all(o.shape[0] == 0 for o in out[:3])
        got = sorted(zip(out[-1].cpu().tolist()))
        assert got == sorted((r,) for _, r in pairs)
        return
    assert _rows(out, len(KEYS)) == _expected(cpu, pairs, KEYS)
    if jt == "inner" and unique:
        assert sum(hashjoin.fallback_reasons.values()) == before  # the unique-hash core ran


def test_right_outer_nulls_per_dtype():
    left, right, cpu = _tables(500, 3000, True, seed=5, key_range=5000)
    out = _run(left, right, "right-outer", eq=([L_KEY], [R_KEY]), uniq=([[L_KEY]], []))
    lv, lf = out[1].cpu(), out[2].cpu()
    lgi = out[-2].cpu()
    nul = lgi == -64
    assert int(nul.sum()) > 0
    assert bool((lv[nul] == -64).all()) and bool((lf[nul] == -64.0).all())


@pytest.mark.parametrize("unique", [True, False])
def test_residual_condition_on_pairs(unique):
    left, right, cpu = _tables(2000, 6000, unique, seed=7, key_range=3000)
    conds = [['v#2', '<', 'w#12']]
    out = _run(left, right, "inner", conds=conds, eq=([L_KEY], [R_KEY]),
               uniq=([[L_KEY]], []) if unique else ([], []))
    lv, rv = cpu[0][L_V].numpy(), cpu[1][R_V].numpy()
    pairs = oracle.join_rows(cpu[0][L_KEY].numpy(), cpu[1][R_KEY].numpy(), "inner",
                             keep=lambda l, r: lv[l] < rv[r])
    assert _rows(out, len(KEYS)) == _expected(cpu, pairs, KEYS)


def test_two_key_hash_with_the_second_equality_dropped():
    left, right, cpu = _tables(2000, 6000, True, seed=8, key_range=3000)
    eq = ([L_KEY, L_K2], [R_KEY, R_K2])
    conds = [['a#4', '=', 'b#14'], [['NOT', ['v#2', '=', 'w#12']]]]
    out = _run(left, right, "inner", conds=conds, eq=eq, uniq=([[L_KEY, L_K2]], []))
    l2, r2 = cpu[0][L_K2].numpy(), cpu[1][R_K2].numpy()
    lv, rv = cpu[0][L_V].numpy(), cpu[1][R_V].numpy()
    pairs = oracle.join_rows(cpu[0][L_KEY].numpy(), cpu[1][R_KEY].numpy(), "inner",
                             keep=lambda l, r: l2[l] == r2[r] and lv[l] != rv[r])
    assert _rows(out, len(KEYS)) == _expected(cpu, pairs, KEYS)


@pytest.mark.parametrize("anti", [False, True])
def test_semi_anti_with_a_summary_residual(anti):
    left, right, cpu = _tables(3000, 8000, False, seed=9)
    conds = [['NOT', ['v#2', '>=', 'w#12']]]  # left.v < right.v
    jt = "right-anti" if anti else "right-semi"
    out = _run(left, right, jt, conds=conds)
    lv, rv = cpu[0][L_V].numpy(), cpu[1][R_V].numpy()
    pairs = oracle.join_rows(cpu[0][L_KEY].numpy(), cpu[1][R_KEY].numpy(), jt,
                             keep=lambda l, r: lv[l] < rv[r])
    assert sorted(out[-1].cpu().tolist()) == sorted(r for _, r in pairs)


def test_semi_falls_back_when_a_key_is_int64_min():
    left, right, cpu = _tables(1000, 4000, False, seed=10)
    left[L_KEY][3] = torch.iinfo(torch.int64).min
    cpu[0][L_KEY][3] = torch.iinfo(torch.int64).min
    out = _run(left, right, "right-semi")
    pairs = oracle.join_rows(cpu[0][L_KEY].numpy(), cpu[1][R_KEY].numpy(), "right-semi")
    assert sorted(out[-1].cpu().tolist()) == sorted(r for _, r in pairs)


def test_sort_search_with_bucket_counts():
    # both sides partitioned into 3 buckets by key range: runs never cross buckets
    g = torch.Generator().manual_seed(11)
    lk = torch.sort(torch.randint(0, 300, (1500,), generator=g)).values.to(torch.int64)
    rk = torch.sort(torch.randint(0, 300, (4000,), generator=g)).values.to(torch.int64)
    lb = [int((lk < 100).sum()), int(((lk >= 100) & (lk < 200)).sum()), int((lk >= 200).sum())]
    rb = [int((rk < 100).sum()), int(((rk >= 100) & (rk < 200)).sum()), int((rk >= 200).sum())]
    left = {L_KEY: lk.cuda(), L_V: torch.arange(1500, dtype=torch.int64).cuda()}
    right = {R_KEY: rk.cuda(), R_V: torch.arange(4000, dtype=torch.int64).cuda()}
    lg = torch.arange(1500, dtype=torch.int64, device="cuda")
    rg = torch.arange(4000, dtype=torch.int64, device="cuda")
    out = hashjoin.join_kernel_new(left, right, L_KEY, R_KEY, [], [L_V, R_V], False, "inner",
                                   lg, rg, bucket_counts=(lb, rb))
    pairs = oracle.join_rows(lk.numpy(), rk.numpy(), "inner")
    assert sorted(zip(out[0].cpu().tolist(), out[1].cpu().tolist())) == pairs


@pytest.mark.parametrize("guard", ["ratio", "scratch", "legacy", "no_proof"])
def test_guards_fall_back_to_sort_search(guard):
    n_left, n_right = (20000, 1000) if guard == "ratio" else (3000, 9000)
    left, right, cpu = _tables(n_left, n_right, True, seed=12)
    hashjoin.fallback_reasons.clear()
    reason = {"ratio": "build_probe_ratio_guard", "scratch": "scratch_guard",
              "legacy": "gate_legacy", "no_proof": "selected_keys_not_proven_unique"}[guard]
    uniq = ([], []) if guard == "no_proof" else ([[L_KEY]], [])
    try:
        if guard == "legacy":
            hashjoin.set_join_core_mode("legacy")
        out = _run(left, right, "inner", eq=([L_KEY], [R_KEY]), uniq=uniq,
                   limit=1000 if guard == "scratch" else None)
    finally:
        hashjoin.set_join_core_mode("unique_hash")
    assert hashjoin.fallback_reasons[reason] == 1
    pairs = oracle.join_rows(cpu[0][L_KEY].numpy(), cpu[1][R_KEY].numpy(), "inner")
    assert _rows(out, len(KEYS)) == _expected(cpu, pairs, KEYS)


@pytest.mark.parametrize("dtype", [torch.int8, torch.int16, torch.int32, torch.int64,
                                   torch.float16, torch.float32, torch.float64, torch.bool,
                                   torch.uint8])
def test_gather_matches_index_with_null(dtype):
    g = torch.Generator().manual_seed(13)
    src = (torch.randint(0, 100, (777, 3), generator=g) % 2 == 0) if dtype == torch.bool else \
        torch.randint(-100, 100, (777, 3), generator=g).to(dtype)
    idx = torch.randint(0, 777, (5000,), generator=g, dtype=torch.int64)
    idx[::7] = -64
    out = gather.index_with_null(src.cuda(), idx.cuda()).cpu()
    mask = idx == -64
    want = src[idx.masked_fill(mask, 0)]
    want[mask] = torch.full((1,), -64, dtype=dtype) if dtype != torch.bool else True
    assert torch.equal(out, want)
    sel = gather.index_select_many([src.cuda(), src[:, 0].contiguous().cuda()],
                                   idx.clamp(min=0).cuda())
    assert torch.equal(sel[0].cpu(), src[idx.clamp(min=0)])
    assert torch.equal(sel[1].cpu(), src[idx.clamp(min=0), 0])


@pytest.mark.parametrize("ncols", [1, 2, 3, 4])
def test_gather_one_word_rows_with_nulls_and_a_ragged_tail(ncols):
    """Columns whose rows are one 1-16 byte word take the batched kernel:
    nulls, an out-of-range index and a row count that is not a multiple of
    the rows a block takes."""
    g = torch.Generator().manual_seed(17 + ncols)
    n_src, n = 1000, 3 * 1024 + 37
    pool = [torch.randint(-(1 << 40), 1 << 40, (n_src,), generator=g),
            torch.randint(-(1 << 30), 1 << 30, (n_src,), generator=g, dtype=torch.int32),
            torch.randint(-100, 100, (n_src,), generator=g).to(torch.int16),
            torch.randint(-100, 100, (n_src,), generator=g).to(torch.int8),
            torch.randint(-(1 << 40), 1 << 40, (n_src, 2), generator=g),
            torch.randn(n_src, generator=g, dtype=torch.float64)]
    cols = [pool[(ncols + k) % len(pool)] for k in range(ncols)]
    idx = torch.randint(0, n_src, (n,), generator=g)
    idx[::5] = -64
    idx[7] = n_src
    out = gather.index_with_null_many([c.cuda() for c in cols], idx.cuda())
    bad = (idx == n_src) | (idx == -64)
    for o, c in zip(out, cols):
        want = c[idx.clamp(0, n_src - 1)]
        want[bad] = torch.full((1,), -64, dtype=c.dtype)
        assert torch.equal(o.cpu(), want)
    sel = gather.index_select_many([c.cuda() for c in cols], idx.clamp(0, n_src - 1).cuda())
    for o, c in zip(sel, cols):
        assert torch.equal(o.cpu(), c[idx.clamp(0, n_src - 1)])


def test_gather_counts_out_of_range_and_reads_nothing_outside():
    src = torch.arange(100, dtype=torch.int64, device="cuda")
    idx = torch.tensor([0, 99, 100, -1, 5, 1 << 40], dtype=torch.int64, device="cuda")
    with pytest.raises(IndexError):
        gather.index_select_many([src], idx, check_range=True)
    out = gather.index_select_many([src], idx)[0].cpu().tolist()
    assert out[0] == 0 and out[1] == 99 and out[4] == 5
    assert out[2] == out[3] == out[5] == -64
    # a slice (unaligned base) and an empty gather
    sl = src[1:]
    assert gather.index_select(sl, torch.tensor([0, 98], device="cuda")).cpu().tolist() == [1, 99]
    assert gather.index_select(src, torch.empty(0, dtype=torch.int64, device="cuda")).numel() == 0
