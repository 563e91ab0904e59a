"""The reference's own operator wrappers over the drop-in module.

``tests/golden/dropin_transcripts.npz`` holds calls that the reference's
unchanged ``operators/partition_sort.partition``, ``operators/join_core.semi_anti``
and ``join_core.expand`` made into their native module (every argument as
passed, the mask prologue their thresholds chose included) and what each
wrapper returned after narrowing the outputs by ``host_out`` and checking its
counts (make_dropin_transcripts.py).  Here the same calls go into
``pageflow_b200.tqpkernels`` on the GPU: the ``host_out`` words a wrapper
reads must pass its checks, and the outputs narrowed by them must equal what
the wrapper returned (padding rows aside, which the layout leaves unwritten).
"""
from __future__ import annotations

import json

import numpy as np
import pytest
import torch

from pageflow_b200 import tqpkernels
from tests.dropin import padded_starts, row_bytes
from tests.golden import load

pytestmark = pytest.mark.gpu

T = load("dropin_transcripts.npz")
META = json.loads(bytes(T["meta"]))


def _cuda(name):
    return torch.from_numpy(T[name]).cuda()


def _pinned(n):
    return torch.empty(n, dtype=torch.int64, pin_memory=True)


@pytest.mark.parametrize("i", [i for i, m in enumerate(META) if m["fn"] == "partition_sort"],
                         ids=lambda i: META[i]["case"])
def test_partition_sort_calls_of_the_references_wrapper(i):
    m = META[i]
    cols = [_cuda(f"c{i}_in{j}") for j in range(m["ncols"])]
    mask = _cuda(f"c{i}_mask") if m["has_mask"] else None
    B = m["B"]
    host = _pinned(B + tqpkernels.MAXCLS + 1)
    outs = tqpkernels.partition_sort(cols, m["comp"], m["key_idx"], mask, m["n_valid"],
                                     m["goff"], B, m["select_first"], host)
    # what the wrapper reads back: counts, each width class's padded total,
    # the rows a mask prologue found (operators/partition_sort.py:125-143)
    counts = host[:B].tolist()
    assert counts == m["counts"]
    kept = sum(counts)
    found = int(host[B + tqpkernels.MAXCLS])
    assert (found if found >= 0 else kept) == m["n_valid"] == kept
    widths = []
    for t in cols:
        if row_bytes(t) not in widths:
            widths.append(row_bytes(t))
    if 8 not in widths:
        widths.append(8)
    assert len(outs) == m["nout"]
    for j, t in enumerate(outs):
        want = T[f"c{i}_out{j}"]
        total = int(host[B + widths.index(row_bytes(t))])
        assert total == want.shape[0]
        got = t[:total].cpu().numpy()
        starts, rows = padded_starts(counts, row_bytes(t))
        assert rows == total
        for s, c in zip(starts, counts):
            assert np.array_equal(got[s:s + c], want[s:s + c]), f"output {j} differs"


@pytest.mark.parametrize("i", [i for i, m in enumerate(META) if m["fn"] == "join_semi_anti"],
                         ids=lambda i: META[i]["case"])
def test_semi_anti_calls_of_the_references_wrapper(i):
    m = META[i]
    bv = _cuda(f"c{i}_build_val") if m["has_vals"] else None
    pv = _cuda(f"c{i}_probe_val") if m["has_vals"] else None
    host = _pinned(2)
    out = tqpkernels.join_semi_anti(_cuda(f"c{i}_build_key"), _cuda(f"c{i}_probe_key"), bv, pv,
                                    m["op"], m["anti"], host)
    n, bad = host.tolist()
    assert bad == 0
    assert np.array_equal(out[:n].cpu().numpy(), T[f"c{i}_out0"])


@pytest.mark.parametrize("i", [i for i, m in enumerate(META) if m["fn"] == "join_expand"],
                         ids=lambda i: META[i]["case"])
def test_expand_calls_of_the_references_wrapper(i):
    host = _pinned(2)
    cs, cr = tqpkernels.join_expand(_cuda(f"c{i}_sorted_ids"), _cuda(f"c{i}_start"),
                                    _cuda(f"c{i}_length"), host)
    assert np.array_equal(cs.cpu().numpy(), T[f"c{i}_out0"])
    assert np.array_equal(cr.cpu().numpy(), T[f"c{i}_out1"])
