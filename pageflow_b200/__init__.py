"""pageflow_b200: PageFlow's relational hot path (radix partition -> hash
join -> slab group-by) as hand-written sm_100a CUDA behind a C ABI
(include/pageflow_b200.h, libpageflow_b200.so):

  tqpkernels        drop-in for TQPlib.tqpkernels (partition_sort,
                    join_unique_hash, join_semi_anti, join_expand); the
                    reference's own operators/partition_sort.py,
                    join_core.py and hashjoin.py run unchanged over it once
                    install_as_tqplib() has registered it
  gather            late materialization: every output column of a join in
                    one launch, null rows for outer joins
  partitions        the fan-out rule (operators/partitions.py)
  aggregation_slab  operators/aggregation_slab.DenseAggregationSlab
  join_aggregate    the fused partition -> join -> group-by
  datagen           seeded synthetic workloads on the device
"""
from __future__ import annotations

import sys
import types

from . import _native

__version__ = "0.1.0"


def native_library():
    """The loaded C-ABI library (raises when it is not built)."""
    return _native.lib()


def install_as_tqplib() -> None:
    """Registers this package's kernels under the reference's module names
    (``TQPlib.tqpkernels`` and ``TQPlib.tqpkernels.tqpkernels``), so that
    PageFlow's unchanged operators/partition_sort.py, operators/join_core.py
    and, through them, operators/hashjoin.py import them."""
    from . import tqpkernels as tk
    pkg = sys.modules.get("TQPlib") or types.ModuleType("TQPlib")
    pkg.__path__ = getattr(pkg, "__path__", [])
    sub = types.ModuleType("TQPlib.tqpkernels")
    inner = types.ModuleType("TQPlib.tqpkernels.tqpkernels")
    for name in ("partition_sort", "join_unique_hash", "join_semi_anti", "join_expand"):
        setattr(sub, name, getattr(tk, name))
        setattr(inner, name, getattr(tk, name))
    sub.tqpkernels = inner
    pkg.tqpkernels = sub
    sys.modules["TQPlib"] = pkg
    sys.modules["TQPlib.tqpkernels"] = sub
    sys.modules["TQPlib.tqpkernels.tqpkernels"] = inner
