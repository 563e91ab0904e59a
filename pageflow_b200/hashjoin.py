"""The join core dispatch of PageFlow's ``operators/hashjoin.py`` on the
sm_100a kernels: ``join_kernel_new`` and its helpers, with the same guards,
fallbacks, join-type tails and outputs (operators/hashjoin.py:56-494).

  unique-hash core   pf_join_unique_hash when the equality keys hold a proven
                     unique tuple of one side (``_try_unique_hash_pairs``,
                     :87-163): the smaller proven side builds, the build side
                     is at most 8x the probe side, the scratch at most 2 GiB
  semi / anti        pf_join_semi_anti with the per-key summary answering one
                     residual comparison (``_try_hash_semi_anti``, :223-244)
  sort / search      per bucket sort + searchsorted, pairs by pf_join_expand,
                     residuals on the pairs (``_sort_search_pairs``, :380-441)
  tail               inner / right-semi / right-anti / right-outer output
                     rows (``_finish_join_result``, :293-356), then every
                     output column gathered in one pf_gather launch, nulls
                     (-64) for right-outer's unmatched rows (:359-377)

Residual conditions are expression trees as the plan writes them
(``[lhs, op, rhs]``, ``['NOT', x]``, column tokens ``name#id``, int and float
literals, single-item list wrappers); this module evaluates comparisons, the
four arithmetic operators and AND / OR / NOT on the GPU, the subset join
residuals use.
"""
from __future__ import annotations

import re
from collections import Counter
from typing import Literal

import torch

from . import join_core
from .gather import NULL, index_select_many, index_with_null_many

UNIQUE_HASH_MAX_BUILD_PROBE_RATIO = 8            # hashjoin.py:49
UNIQUE_HASH_SCRATCH_LIMIT_BYTES = 2 * 1024 ** 3  # hashjoin.py:55
INT_ROWS_MAX = (1 << 31) - 1

_JOIN_CORE_MODES = {"legacy", "unique_hash"}
_join_core_mode = "unique_hash"
# Why the unique-hash core was refused, by guard name (for telemetry).
fallback_reasons: Counter = Counter()


def set_join_core_mode(mode: str) -> None:
    global _join_core_mode
    if mode not in _JOIN_CORE_MODES:
        raise ValueError(
            f"join core mode must be one of {sorted(_JOIN_CORE_MODES)}, got {mode!r}")
    _join_core_mode = mode


def _fallback(reason: str):
    fallback_reasons[reason] += 1
    return None


def _proof_is_covered(unique_key_sets, selected_ids) -> bool:
    selected = set(selected_ids)
    return any(set(u) <= selected for u in (unique_key_sets or []))


def _valid_hash_key(t: torch.Tensor) -> bool:
    return t.is_cuda and t.dtype == torch.int64 and t.dim() == 1 and t.is_contiguous()


# ---- expressions --------------------------------------------------------------

_COLUMN_REF = re.compile(r'#(\d+)L?$')


def column_ref(token):
    """The column id of a ``name#id`` token (``#idL`` too), else None; the
    ``Brand#NN`` literal family is no reference (parsing/expressions.py:17-33)."""
    if not isinstance(token, str) or token.startswith('Brand#'):
        return None
    head = token.split(' as', 1)[0] if ' as' in token else token
    m = _COLUMN_REF.search(head)
    return int(m.group(1)) if m else None


def normalize_expr_tree(tree):
    while isinstance(tree, list) and len(tree) == 1:
        tree = tree[0]
    return tree


_CMP = {'=': torch.eq, '==': torch.eq, '<>': torch.ne, '!=': torch.ne, '<': torch.lt,
        '<=': torch.le, '>': torch.gt, '>=': torch.ge}
_ARITH = {'+': torch.add, '-': torch.sub, '*': torch.mul, '/': torch.true_divide}


def _literal(token):
    try:
        return int(token)
    except (TypeError, ValueError):
        pass
    try:
        return float(token)
    except (TypeError, ValueError):
        raise NotImplementedError(f"join residual: unsupported token {token!r}")


def evaluate_join(tensors_left, tensors_right, tree, left_idx, right_idx):
    """The residual condition at every pair (left_idx[i], right_idx[i]): a
    bool tensor (hashjoin.py:246-253; a column the left side holds is read
    from the left side)."""
    cache = {}

    def leaf(cid):
        if cid not in cache:
            if cid in tensors_left:
                cache[cid] = index_select_many([tensors_left[cid]], left_idx)[0]
            elif cid in tensors_right:
                cache[cid] = index_select_many([tensors_right[cid]], right_idx)[0]
            else:
                raise KeyError(f"join residual: column #{cid} on neither side")
        return cache[cid]

    def ev(t):
        t = normalize_expr_tree(t)
        if isinstance(t, str):
            cid = column_ref(t)
            return leaf(cid) if cid is not None else _literal(t)
        if isinstance(t, (int, float)):
            return t
        if isinstance(t, list) and len(t) == 2 and t[0] == 'NOT':
            return torch.logical_not(ev(t[1]))
        if isinstance(t, list) and len(t) == 3 and isinstance(t[1], str):
            op = t[1]
            if op in ('AND', 'OR'):
                f = torch.logical_and if op == 'AND' else torch.logical_or
                return f(ev(t[0]), ev(t[2]))
            a, b = ev(t[0]), ev(t[2])
            if op in _CMP:
                if not torch.is_tensor(a):
                    a = torch.full_like(b, a) if torch.is_tensor(b) else torch.tensor(a)
                return _CMP[op](a, b)
            if op in _ARITH:
                return _ARITH[op](a, b)
        raise NotImplementedError(f"join residual: unsupported expression {t!r}")

    out = ev(tree)
    if not torch.is_tensor(out):
        out = torch.full((left_idx.numel(),), bool(out), dtype=torch.bool, device=left_idx.device)
    return out.to(torch.bool).reshape(-1)


# ---- cores --------------------------------------------------------------------

def try_unique_hash_pairs(tensors_left, tensors_right, left_key, right_key, join_type,
                          equality_keys, unique_key_sets, scratch_limit_bytes):
    """``(left_idx, right_idx, hashed_pairs)`` from the unique-build hash
    core, or None for the sort/search core (hashjoin.py:87-163)."""
    if _join_core_mode == "legacy":
        return _fallback("gate_legacy")
    if join_type != "inner":
        return _fallback("join_type")
    if equality_keys is None or unique_key_sets is None:
        return _fallback("missing_proof_metadata")
    left_eq, right_eq = equality_keys
    if len(left_eq) != len(right_eq) or not left_eq:
        return _fallback("unaligned_equality_keys")
    selected = []
    for lid, rid in zip(left_eq, right_eq):
        if lid not in tensors_left or rid not in tensors_right:
            continue
        if _valid_hash_key(tensors_left[lid]) and _valid_hash_key(tensors_right[rid]):
            selected.append((lid, rid))
    if (left_key, right_key) not in selected:
        return _fallback("primary_key_layout_or_dtype")
    if len(selected) not in (1, 2):
        return _fallback("unsupported_key_count")
    left_ids = [p[0] for p in selected]
    right_ids = [p[1] for p in selected]
    left_unique, right_unique = unique_key_sets
    can_left = _proof_is_covered(left_unique, left_ids)
    can_right = _proof_is_covered(right_unique, right_ids)
    if not can_left and not can_right:
        return _fallback("selected_keys_not_proven_unique")
    left_rows = tensors_left[left_ids[0]].numel()
    right_rows = tensors_right[right_ids[0]].numel()
    build_left = can_left and (not can_right or left_rows <= right_rows)
    if build_left:
        build_ids, probe_ids, bt, pt = left_ids, right_ids, tensors_left, tensors_right
    else:
        build_ids, probe_ids, bt, pt = right_ids, left_ids, tensors_right, tensors_left
    n_build, n_probe = bt[build_ids[0]].numel(), pt[probe_ids[0]].numel()
    if n_probe > 0 and n_build > UNIQUE_HASH_MAX_BUILD_PROBE_RATIO * n_probe:
        return _fallback("build_probe_ratio_guard")
    if (scratch_limit_bytes is not None
            and join_core.unique_hash_peak_bytes(n_build, n_probe) > scratch_limit_bytes):
        return _fallback("scratch_guard")
    build_idx, probe_idx = join_core.unique_hash_pairs([bt[k] for k in build_ids],
                                                       [pt[k] for k in probe_ids])
    hashed = frozenset(selected)
    if build_left:
        return build_idx, probe_idx, hashed
    return probe_idx, build_idx, hashed


_NEGATED_OP = {'=': '<>', '<': '>=', '<=': '>', '>': '<=', '>=': '<'}
_FLIPPED_OP = {'<>': '<>', '<': '>', '<=': '>=', '>': '<', '>=': '<='}


def _summary_column(token):
    token = normalize_expr_tree(token)
    if not isinstance(token, str) or ' ' in token:
        return None
    return column_ref(token)


def residual_summary(condition, tensors_left, tensors_right):
    """``(build column, probe column, op)`` when the condition compares one
    left column with one right column, both int64, by an operator the
    per-key summary answers (hashjoin.py:183-220); else None."""
    tree = normalize_expr_tree(condition)
    negated = False
    while isinstance(tree, list) and len(tree) == 2 and tree[0] == 'NOT':
        negated = not negated
        tree = normalize_expr_tree(tree[1])
    if not (isinstance(tree, list) and len(tree) == 3 and isinstance(tree[1], str)):
        return None
    first, op, second = _summary_column(tree[0]), tree[1], _summary_column(tree[2])
    if negated:
        op = _NEGATED_OP.get(op)
    if any(c in tensors_left and c in tensors_right for c in (first, second)):
        return None
    if first in tensors_left and second in tensors_right:
        build_id, probe_id = first, second
    elif first in tensors_right and second in tensors_left:
        build_id, probe_id, op = second, first, _FLIPPED_OP.get(op)
    else:
        return None
    if op not in join_core.SUMMARY_OPS:
        return None
    build, probe = tensors_left[build_id], tensors_right[probe_id]
    if not (_valid_hash_key(build) and _valid_hash_key(probe)):
        return None
    return build, probe, op


def try_hash_semi_anti(tensors_left, tensors_right, left_key, right_key, condition_list, anti):
    """The kept right rows of a semi or anti join on a hash set of the left
    keys, or None for the sort/search path (hashjoin.py:223-244)."""
    build, probe = tensors_left[left_key], tensors_right[right_key]
    if not (_valid_hash_key(build) and _valid_hash_key(probe)):
        return None
    summary = None
    if condition_list:
        if len(condition_list) != 1:
            return None
        summary = residual_summary(condition_list[0], tensors_left, tensors_right)
        if summary is None:
            return None
    return join_core.semi_anti(build, probe, anti, summary)


def _condition_col_id(token):
    if not isinstance(token, str) or '#' not in token:
        return None
    try:
        return int(token.rsplit('#', 1)[1])
    except ValueError:
        return None


def _is_hashed_equality_condition(condition, hashed_pairs) -> bool:
    if not isinstance(condition, (list, tuple)) or len(condition) != 3 or condition[1] != '=':
        return False
    a, b = _condition_col_id(condition[0]), _condition_col_id(condition[2])
    return (a, b) in hashed_pairs or (b, a) in hashed_pairs


def apply_fast_path_conditions(tensors_left, tensors_right, condition_list, left_matched,
                               right_matched, device, hashed_pairs):
    """The residual conditions on the unique-hash pairs, except an equality
    the hashed tuple already holds (hashjoin.py:267-290)."""
    residual = [c for c in (condition_list or [])
                if not _is_hashed_equality_condition(c, hashed_pairs)]
    if not residual or left_matched.numel() == 0:
        return left_matched, right_matched
    mask = torch.ones(left_matched.numel(), dtype=torch.bool, device=device)
    for cond in residual:
        mask &= evaluate_join(tensors_left, tensors_right, cond, left_matched, right_matched)
    pos = torch.nonzero(mask, as_tuple=False).view(-1)
    if pos.numel() == 0:
        e = torch.empty(0, dtype=torch.int64, device=device)
        return e, e.clone()
    return index_select_many([left_matched, right_matched], pos)


def sort_search_pairs(tensors_left, tensors_right, left, right, condition_list, bucket_counts,
                      device, name="join"):
    """The sort/search core's (left rows, right rows), in right-row order
    (hashjoin.py:380-441); pairs by pf_join_expand."""
    nL, nR = left.size(0), right.size(0)
    lc, rc = bucket_counts if bucket_counts is not None else ([nL], [nR])
    assert len(lc) == len(rc), f"bucket_counts sides disagree: {len(lc)} vs {len(rc)} buckets"
    assert sum(lc) == nL and sum(rc) == nR, (
        f"bucket_counts misaligned with tick tensors: left {sum(lc)} != {nL} or right "
        f"{sum(rc)} != {nR}")
    sorted_ids = torch.empty(nL, dtype=torch.int64, device=device)
    start = torch.zeros(nR, dtype=torch.int64, device=device)
    length = torch.zeros(nR, dtype=torch.int64, device=device)
    ls = rs = 0
    for lcnt, rcnt in zip(lc, rc):
        le, re_ = ls + lcnt, rs + rcnt
        if lcnt > 0:
            sk, perm = torch.sort(left[ls:le])
            sorted_ids[ls:le] = perm.add_(ls)
            if rcnt > 0:
                rk = right[rs:re_]
                lo = torch.searchsorted(sk, rk)
                length[rs:re_] = torch.searchsorted(sk, rk, right=True) - lo
                start[rs:re_] = lo.add_(ls)
        ls, rs = le, re_
    if condition_list:
        n_pairs = int(length.sum().item())
        if n_pairs > INT_ROWS_MAX:
            raise RuntimeError(f"{name}: a core call of {nL} left and {nR} right rows makes "
                               f"{n_pairs} pairs, over the {INT_ROWS_MAX} its residual "
                               f"conditions take")
    left_matched, right_matched = join_core.expand(sorted_ids, start, length)
    if condition_list and left_matched.numel() > 0:
        mask = torch.ones(left_matched.numel(), dtype=torch.bool, device=device)
        for cond in condition_list:
            mask &= evaluate_join(tensors_left, tensors_right, cond, left_matched, right_matched)
        kept = torch.nonzero(mask, as_tuple=False).view(-1)
        left_matched, right_matched = index_select_many([left_matched, right_matched], kept)
    return left_matched, right_matched


# ---- tail -----------------------------------------------------------------------

def gather_join_result(tensors_left, tensors_right, join_output_keys, return_global_index,
                       left_out, right_out, left_global_idx, right_global_idx, with_null=False):
    """The output columns at the output rows of each side, then the two
    global indexes (hashjoin.py:359-377), the left side's and the right
    side's columns each in one gather launch."""
    lcols = [k for k in join_output_keys if k in tensors_left]
    rcols = [k for k in join_output_keys if k not in tensors_left]
    lsrc = [tensors_left[k] for k in lcols]
    rsrc = [tensors_right[k] for k in rcols]
    if return_global_index:
        lsrc.append(left_global_idx)
        rsrc.append(right_global_idx)
    lgather = index_with_null_many if with_null else index_select_many
    lout = lgather(lsrc, left_out) if lsrc else []
    rout = index_select_many(rsrc, right_out) if rsrc else []
    lmap = dict(zip(lcols, lout))
    rmap = dict(zip(rcols, rout))
    result = [lmap[k] if k in lmap else rmap[k] for k in join_output_keys]
    if return_global_index:
        result.extend([lout[-1], rout[-1]])
    return result


def finish_join_result(tensors_left, tensors_right, join_output_keys, return_global_index,
                       join_type, left_matched, right_matched, left_global_idx,
                       right_global_idx, n_right, device):
    """The join-type tail, then the gathers (hashjoin.py:293-356)."""
    e = torch.empty(0, dtype=torch.int64, device=device)
    with_null = False
    if join_type == 'inner':
        left_out, right_out = left_matched, right_matched
    elif join_type == 'right-semi':
        if right_matched.numel() > 0:
            m = torch.zeros(n_right, dtype=torch.bool, device=device)
            m.index_fill_(0, right_matched, True)
            right_out = torch.nonzero(m, as_tuple=False).view(-1)
        else:
            right_out = e
        left_out = e
    elif join_type == 'right-anti':
        m = torch.ones(n_right, dtype=torch.bool, device=device)
        if right_matched.numel() > 0:
            m.index_fill_(0, right_matched, False)
        right_out = torch.nonzero(m, as_tuple=False).view(-1)
        left_out = e
    elif join_type == 'right-outer':
        m = torch.ones(n_right, dtype=torch.bool, device=device)
        if right_matched.numel() > 0:
            m.index_fill_(0, right_matched, False)
        unmatched = torch.nonzero(m, as_tuple=False).view(-1)
        left_out, right_out = left_matched, right_matched
        nulls = unmatched.numel()
        if nulls > 0:
            right_out = torch.cat([right_out, unmatched])
            left_out = torch.cat([left_out, torch.full((nulls,), NULL, dtype=torch.int64,
                                                       device=device)])
            with_null = True
    else:
        raise NotImplementedError("unhandled join type")
    return gather_join_result(tensors_left, tensors_right, join_output_keys,
                              return_global_index, left_out, right_out, left_global_idx,
                              right_global_idx, with_null)


def join_kernel_new(tensors_left, tensors_right, left_key, right_key, condition_list,
                    join_output_keys, return_global_index,
                    type: Literal['inner', 'right-semi', 'right-anti', 'right-outer'],
                    left_global_idx, right_global_idx, bucket_counts=None, equality_keys=None,
                    unique_key_sets=None, hash_scratch_limit_bytes=None, name="join"):
    """One join core call (hashjoin.py:444-494): the unique-hash core when
    its guards pass, the hash semi / anti set for semi and anti joins, else
    the sort/search core; then the join-type tail and the gathered outputs."""
    assert type in {'inner', 'right-semi', 'right-anti', 'right-outer'}, "Invalid Join type."
    left = tensors_left[left_key]
    right = tensors_right[right_key]
    device = right.device
    nR = right.size(0)
    fast = try_unique_hash_pairs(
        tensors_left, tensors_right, left_key, right_key, type, equality_keys, unique_key_sets,
        UNIQUE_HASH_SCRATCH_LIMIT_BYTES if hash_scratch_limit_bytes is None
        else hash_scratch_limit_bytes)
    if fast is not None:
        lm, rm, hashed = fast
        lm, rm = apply_fast_path_conditions(tensors_left, tensors_right, condition_list, lm, rm,
                                            device, hashed)
        return finish_join_result(tensors_left, tensors_right, join_output_keys,
                                  return_global_index, type, lm, rm, left_global_idx,
                                  right_global_idx, nR, device)
    if type in ('right-semi', 'right-anti'):
        kept = try_hash_semi_anti(tensors_left, tensors_right, left_key, right_key,
                                  condition_list, anti=type == 'right-anti')
        if kept is not None:
            return gather_join_result(tensors_left, tensors_right, join_output_keys,
                                      return_global_index,
                                      torch.empty(0, dtype=torch.int64, device=device), kept,
                                      left_global_idx, right_global_idx)
    lm, rm = sort_search_pairs(tensors_left, tensors_right, left, right, condition_list,
                               bucket_counts, device, name)
    return finish_join_result(tensors_left, tensors_right, join_output_keys,
                              return_global_index, type, lm, rm, left_global_idx,
                              right_global_idx, nR, device)
