"""Generates tests/golden/keyed_pass1.npz from PageFlow's own
``KeyedAggregate.pass1`` (operators/aggregate.py:1511-1563), imported
read-only from a checkout of the reference with its compiled TQPlib modules
replaced by empty stand-ins (pass 1 is pure torch).  Run where the reference
is present:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_keyed_golden.py /path/to/PageFlow

Per case (keys of one, two and three columns, one of them 2-D; B = 64), on
CPU tensors: the chunk's columns, the coefficients ``_make_key_coeffs``
draws for them on the CPU, and everything pass 1 returns: the unique
grouping hashes ascending, one representative of every key column, the
partials of SUM(v), COUNT(*), MIN(w), MAX(w) and AVG(f) (its state: float64
sum and count), and each group's bucket with the groups per bucket.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from tests.golden.make_golden import import_reference  # noqa: E402

OUT = HERE / "keyed_pass1.npz"
B = 64


def cases(g):
    n = 4000
    yield "one", [torch.randint(-500, 500, (n,), generator=g)]
    yield "two", [torch.randint(0, 30, (n,), generator=g, dtype=torch.int32),
                  torch.randint(-3, 3, (n,), generator=g)]
    yield "three", [torch.randint(0, 12, (n,), generator=g, dtype=torch.int32),
                    torch.randint(-3, 3, (n,), generator=g),
                    torch.randint(-2, 2, (n,), generator=g, dtype=torch.int16)]
    yield "wide", [torch.randint(-4, 4, (n, 3), generator=g, dtype=torch.int16),
                   torch.randint(0, 5, (n,), generator=g, dtype=torch.int8)]


def main(root: str) -> None:
    import_reference(root)
    from operators import aggregate
    from uvm.column import UColumn

    g = torch.Generator().manual_seed(2029)
    out = {}
    for name, keys in cases(g):
        n = keys[0].shape[0]
        v = torch.randint(-10 ** 6, 10 ** 6, (n,), generator=g)
        w = torch.randint(-100, 100, (n,), generator=g, dtype=torch.int32)
        f = torch.randint(-1000, 1000, (n,), generator=g).to(torch.float64) / 8
        ids = list(range(1, len(keys) + 1))
        kref = [f"k{i}#{i}" for i in ids]
        results = [[r] for r in kref] + [
            [[[['sum', ['v#10']], '#', '9001'], 'AS', 'out#200']],
            [[[['count', ['1']], '#', '9001'], 'AS', 'out#201']],
            [[[['min', ['w#11']], '#', '9001'], 'AS', 'out#202']],
            [[[['max', ['w#11']], '#', '9001'], 'AS', 'out#203']],
            [[[['avg', ['f#12']], '#', '9001'], 'AS', 'out#204']]]
        args = {'name': 'Aggregate', 'keys': kref, 'input ids': ids + [10, 11, 12],
                'results': results, 'out key ids': ids,
                'out agg ids': [200, 201, 202, 203, 204],
                'agg ops': ['sum', 'count', 'min', 'max', 'avg'],
                'output ids': ids + [200, 201, 202, 203, 204]}
        cols = {i: k for i, k in zip(ids, keys)}
        cols.update({10: v, 11: w, 12: f})
        tgroup = {i: UColumn(t, 'float' if t.is_floating_point() else 'int')
                  for i, t in cols.items()}
        spec = aggregate.KeyedAggregate(args, tgroup, ids + [10, 11, 12],
                                        [t.dtype for t in cols.values()])
        outs, buckets = spec.pass1('cpu', cols, B)
        out[f"{name}_nkeys"] = np.array([len(keys)])
        for i, k in enumerate(keys):
            out[f"{name}_key{i}"] = k.numpy()
            out[f"{name}_coeff{i}"] = spec._coeffs[i].numpy()
        out[f"{name}_v"], out[f"{name}_w"], out[f"{name}_f"] = v.numpy(), w.numpy(), f.numpy()
        for j, t in enumerate(outs):
            out[f"{name}_out{j}"] = t.numpy()
        out[f"{name}_nout"] = np.array([len(outs)])
        out[f"{name}_bucket"] = buckets[0].numpy()
        out[f"{name}_bucket_counts"] = np.array(buckets[1])
    np.savez_compressed(OUT, **out)
    print("written", OUT)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PAGEFLOW_REFERENCE")
    if not ref:
        sys.exit("usage: make_keyed_golden.py <reference checkout> (or set PAGEFLOW_REFERENCE)")
    main(ref)
