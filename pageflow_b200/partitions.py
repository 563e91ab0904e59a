"""The hash-partition count B of a join or a keyed aggregation, from a
partition budget: the same rule as PageFlow's ``operators/partitions.py``
(the smallest power of two B whose largest unit is predicted to fit the
budget), so the fan-out the kernels get for a given input is the reference's.
Host logic only (stdlib), tested on the CPU.

The prediction spreads an input's rows over its estimated distinct keys, all
of a key's rows in one bucket, with the fullest bucket's keys at about its
90th percentile (``max_load``).
"""
from __future__ import annotations

import math
from typing import Optional, Sequence

B_MIN = 1
JOIN_B_MAX = 512   # the partition kernel's bucket limit (PF_PART_B_MAX)
AGG_B_MAX = 256


def max_load(m: float, n: int) -> float:
    """The fullest of ``n`` bins' load, at about its 90th percentile, after
    ``m`` equal balls.  With m/n >= 32 the Raab-Steger bound m/n +
    sqrt(2 (m/n) ln n); below it the largest k that a tenth of a bin is
    expected to reach under Binomial(m, 1/n) (union bound)."""
    if m <= 0:
        return 0.0
    if n <= 1:
        return float(m)
    mean = m / n
    if mean >= 32:
        return mean + math.sqrt(2.0 * mean * math.log(n))
    m = int(math.ceil(m))
    p = 1.0 / n
    pmf = (1.0 - p) ** m      # P(X = k - 1)
    below = 0.0               # P(X <= k - 2)
    for k in range(1, m + 1):
        below += pmf          # now P(X <= k - 1)
        if n * (1.0 - below) < 0.1:
            return float(k - 1)
        pmf *= (m - k + 1) / k * p / (1.0 - p)
    return float(m)


def partition_count(parts: Sequence[tuple], budget_b: int, b_max: int) -> tuple[int, float]:
    """The smallest power of two B in [B_MIN, ``b_max``] whose largest unit
    (the sum over ``parts`` of each part's predicted largest bucket, in
    bytes) fits ``budget_b``, and that unit's bytes; when none fits, the
    smallest B with the least predicted unit.  ``parts``: one ``(rows,
    row_bytes[, keys])`` per input a unit holds a bucket of."""
    assert b_max >= B_MIN and b_max & (b_max - 1) == 0, b_max
    best_b, best = B_MIN, math.inf
    b = B_MIN
    while b <= b_max:
        largest = 0.0
        for part in parts:
            rows, rb = part[0], part[1]
            keys = min(part[2], rows) if len(part) > 2 else rows
            if rows > 0 and keys > 0:
                largest += rows / keys * max_load(keys, b) * rb
        if largest <= budget_b:
            return b, largest
        if largest < best:
            best_b, best = b, largest
        b <<= 1
    return best_b, best


def agg_partitions(rows: int, ticks: int, groups: Optional[int], row_b: int,
                   cap_rows: Optional[int], budget_b: int) -> tuple[int, float, str]:
    """A keyed aggregation's B, its largest pass-2 round's predicted bytes
    and why: ``fits`` (B = 1), ``budget`` (the smallest B whose largest
    bucket fits) or ``at cap`` (none up to AGG_B_MAX fits)."""
    g = rows if groups is None else min(groups, rows)
    r1 = min(rows, ticks * g)
    held = r1 if cap_rows is None else min(r1, cap_rows)
    if held * row_b <= budget_b:
        return 1, float(held * row_b), "fits"
    b, pred = partition_count([(r1, row_b, g)], budget_b, AGG_B_MAX)
    return b, pred, "budget" if pred <= budget_b else "at cap"
