"""The keyed aggregation's grouping coefficients (CPU): the module draws,
for the same key columns, exactly the vectors the reference's
_make_key_coeffs (operators/aggregate.py:526-548: a local generator seeded
with 2029 on the columns' device, one randint(2, 10_000_000) vector of each
column's packed int64 width) drew when tests/golden/make_keyed_golden.py ran
it on the CPU.  The same sequence of generator calls on the GPU gives the
reference's GPU coefficients; the GPU pass-1 tests then run on these."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from pageflow_b200 import keyed_aggregate as ka
from tests.golden import load

KEYED = load("keyed_pass1.npz")


@pytest.mark.parametrize("case", ["one", "two", "three", "wide"])
def test_coefficients_are_the_references(case):
    nk = int(KEYED[f"{case}_nkeys"][0])
    keys = [torch.from_numpy(KEYED[f"{case}_key{i}"]) for i in range(nk)]
    keys = [k.unsqueeze(1) if k.dim() == 1 else k for k in keys]
    got = ka.make_key_coeffs(keys, "cpu")
    assert len(got) == nk
    for i, c in enumerate(got):
        assert np.array_equal(c.numpy(), KEYED[f"{case}_coeff{i}"])


def test_hash_of_the_references_coefficients_on_the_host():
    """The linear hash over packed words (_hash_key_columns, :551-564) of the
    golden keys with the golden coefficients gives the reference's unique
    grouping hashes."""
    for case in ("one", "two", "three", "wide"):
        nk = int(KEYED[f"{case}_nkeys"][0])
        h = np.zeros(KEYED[f"{case}_key0"].shape[0], np.uint64)
        for i in range(nk):
            k = KEYED[f"{case}_key{i}"]
            k = k[:, None] if k.ndim == 1 else k
            raw = np.ascontiguousarray(k).view(np.uint8).reshape(k.shape[0], -1)
            tb = (raw.shape[1] + 7) // 8 * 8
            buf = np.zeros((k.shape[0], tb), np.uint8)
            buf[:, :raw.shape[1]] = raw
            w = buf.view(np.uint64)
            with np.errstate(over="ignore"):
                h += (w * KEYED[f"{case}_coeff{i}"].astype(np.uint64)).sum(axis=1,
                                                                         dtype=np.uint64)
        assert np.array_equal(np.unique(h.view(np.int64)), KEYED[f"{case}_out0"])
