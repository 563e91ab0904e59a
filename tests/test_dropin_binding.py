"""The drop-in as the reference's operators see it (CPU; needs a checkout of
the reference, named by $PAGEFLOW_REFERENCE or found as a `reference`
directory beside this repository, and skips without one).

After ``pageflow_b200.install_as_tqplib()``, the reference's unchanged
``operators/partition_sort.py``, ``operators/join_core.py`` and
``operators/hashjoin.py`` import and bind this package's functions as their
``TQPlib.tqpkernels``; a call through a wrapper reaches the drop-in (whose
argument checks answer here, without a GPU, with the RuntimeError the
reference's TORCH_CHECK raises).  The GPU side of the same boundary is
tests/test_dropin_replay_gpu.py."""
from __future__ import annotations

import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
REF = Path(os.environ.get("PAGEFLOW_REFERENCE", str(REPO.parent / "reference")))

pytestmark = pytest.mark.skipif(not (REF / "operators" / "partition_sort.py").exists(),
                                reason="no reference checkout")


def test_reference_wrappers_bind_the_drop_in():
    # a fresh interpreter: the reference's modules must not leak into others
    code = textwrap.dedent(f"""
        import sys, types
        sys.dont_write_bytecode = True
        sys.path.insert(0, {str(REPO)!r})
        sys.path.insert(1, {str(REF)!r})
        import torch
        import pageflow_b200
        from pageflow_b200 import tqpkernels as ours
        pageflow_b200.install_as_tqplib()
        # the reference's other native modules are not part of this boundary
        for name in ["TQPlib.tqpcompress", "TQPlib.tqpcompress.tqpcompress",
                     "TQPlib.tqpmemory", "TQPlib.tqpmemory.tqpmemory",
                     "TQPlib.tqpcache", "TQPlib.tqpcache.tqpcache",
                     "TQPlib.zero_copy_reader", "TQPlib.zero_copy_reader.zero_copy_reader"]:
            sys.modules.setdefault(name, types.ModuleType(name))
        sys.modules["TQPlib.tqpcache"].split_at_granules = None
        sys.modules["TQPlib.tqpcache.tqpcache"].split_at_granules = None
        from operators import partition_sort, join_core, hashjoin
        for mod in (partition_sort, join_core):
            for fn in ("partition_sort", "join_unique_hash", "join_semi_anti", "join_expand"):
                assert getattr(mod.tqpkernels, fn) is getattr(ours, fn), (mod.__name__, fn)
        assert hashjoin.join_core is join_core
        # a call through the reference's wrapper reaches the drop-in's checks
        partition_sort._host = torch.empty(600, dtype=torch.int64)
        key = torch.arange(100, dtype=torch.int64)
        try:
            partition_sort.partition([key], 0, None, 0, 16)
        except RuntimeError as e:
            assert "host_out must be pinned" in str(e), e
        else:
            raise AssertionError("the drop-in accepted a pageable host_out")
        print("bound")
    """)
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=300, cwd=str(REPO))
    assert res.returncode == 0, res.stderr[-3000:]
    assert "bound" in res.stdout
