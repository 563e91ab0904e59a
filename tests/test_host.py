"""CPU tests of the host side: the C-ABI library loads and exports every
function include/pageflow_b200.h declares (no GPU work is started), the
argument checks that run before any kernel, the partition-count rule against
the reference's own values, and the drop-in module's validation."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest
import torch

from tests.golden import load

REPO = Path(__file__).resolve().parents[1]


def header_functions():
    text = (REPO / "include" / "pageflow_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pf_\w+)\s*\(", text)))


def test_library_exports_every_declared_function():
    from pageflow_b200 import _native
    L = _native.lib()
    declared = header_functions()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    # and the Python binding covers each of them
    assert sorted(_native.exported_symbols()) == declared


def test_library_is_the_in_tree_build():
    from pageflow_b200 import _native
    assert _native.LIB_PATH.parent == REPO / "pageflow_b200"
    assert _native.lib().pf_version().decode() == "0.1.0"


def test_rows_per_unit_is_lcm_over_row_bytes():
    from pageflow_b200 import _native
    L = _native.lib()
    for rb in (1, 2, 3, 4, 8, 16, 25, 24, 512, 1000):
        import math
        assert L.pf_rows_per_unit(rb) == math.lcm(rb, 512) // rb


def test_workspace_sizes_are_host_arithmetic():
    from pageflow_b200 import _native
    L = _native.lib()
    a = L.pf_partition_sort_workspace(1 << 20, 1 << 20, 64, 0, 0)
    b = L.pf_partition_sort_workspace(1 << 24, 1 << 24, 512, 1, 1)
    assert 0 < a < b
    # a table of 2 x n_build 4-byte slots and a 4-byte partner a probe row
    assert L.pf_join_unique_hash_workspace(1000, 2000) >= 2 * 1000 * 4 + 2000 * 4
    assert L.pf_join_aggregate_workspace(1000, 4000, 1, 25) >= 1000 * 12 + 4000 * 16
    assert L.pf_join_aggregate_pick_b(250_000, 1_000_000) == 1
    assert 256 <= L.pf_join_aggregate_pick_b(150_000_000, 600_000_000) <= 4096


def test_invalid_arguments_fail_before_any_kernel():
    """Argument checks return PF_EINVAL with a message and touch no GPU."""
    from pageflow_b200 import _native
    L = _native.lib()
    rc = L.pf_partition_sort(None, None, None, None, 0, 0, None, 10, 10, 0, 32, 0, None, None,
                             None, 0, None)
    assert rc == _native.PF_EINVAL
    assert "columns" in L.pf_last_error().decode()
    ptrs = (ctypes.c_void_p * 1)(1)
    rb = (ctypes.c_int * 1)(8)
    comp = (ctypes.c_int * 1)(0)
    rc = L.pf_partition_sort(ptrs, ptrs, rb, comp, 1, 0, None, 10, 10, 0, 24, 0, 1, 1, None,
                             0, None)
    assert rc == _native.PF_EINVAL and "power of two" in L.pf_last_error().decode()
    rc = L.pf_join_unique_hash(1, None, 0, 1, None, 5, 1, 1, 1, 1, None, 0, None)
    assert rc == _native.PF_EINVAL and "both sides" in L.pf_last_error().decode()
    rc = L.pf_join_aggregate(1, 1, 10, 1, 1, None, 100, 10, 24, 0, 5, 1, 1, 1, None, 0, None)
    assert rc == _native.PF_EINVAL and "power of two" in L.pf_last_error().decode()


def test_workspace_off_a_256_byte_boundary_is_refused_before_any_kernel():
    """A workspace must start on a 256-byte boundary (the kernels' 16-byte
    vector accesses and bulk copies rely on it): one that does not is refused
    with PF_ENOSPACE before any device work, however large it is."""
    from pageflow_b200 import _native
    L = _native.lib()
    need = L.pf_join_aggregate_workspace(10, 10, 4, 5)
    for base in ((1 << 20) + 8, (1 << 20) + 128):
        rc = L.pf_join_aggregate(1, 1, 10, 1, 1, None, 100, 10, 4, 0, 5, 1, 1, 1, base,
                                 need + 4096, None)
        assert rc == _native.PF_ENOSPACE, rc
        assert "workspace" in L.pf_last_error().decode()
    need = L.pf_join_unique_hash_workspace(10, 10)
    rc = L.pf_join_unique_hash(1, None, 10, 1, None, 10, 1, 1, 1, 1, (1 << 20) + 16, need + 4096,
                               None)
    assert rc == _native.PF_ENOSPACE


def test_partition_count_rule_is_the_references():
    from pageflow_b200 import partitions
    g = load("partitions.json")
    assert partitions.JOIN_B_MAX == g["JOIN_B_MAX"]
    assert partitions.AGG_B_MAX == g["AGG_B_MAX"]
    for m, n, want in g["max_load"]:
        assert partitions.max_load(m, n) == pytest.approx(want, rel=1e-12, abs=0)
    for parts, budget, bmax, want in g["partition_count"]:
        got = partitions.partition_count([tuple(p) for p in parts], budget, bmax)
        assert got[0] == want[0]
        assert got[1] == pytest.approx(want[1], rel=1e-12)
    for args, want in g["agg_partitions"]:
        got = partitions.agg_partitions(*args)
        assert got[0] == want[0] and got[2] == want[2]
        assert got[1] == pytest.approx(want[1], rel=1e-12)


def test_bucket_limit_is_the_join_cap():
    from pageflow_b200 import partitions, tqpkernels
    assert partitions.JOIN_B_MAX == tqpkernels.BMAX
    h = (REPO / "include" / "pageflow_b200.h").read_text()
    assert re.search(r"#define PF_PART_B_MAX (\d+)", h).group(1) == str(partitions.JOIN_B_MAX)


@pytest.mark.parametrize("case", ["five widths", "seven columns", "int32 key", "B=1024",
                                  "B=24", "B=0", "host_out too short", "pageable host_out"])
def test_drop_in_partition_refuses_bad_arguments_before_any_kernel(case):
    """The drop-in's argument checks raise RuntimeError, as the reference's
    TORCH_CHECKs do, before touching a device (CPU tensors suffice)."""
    from pageflow_b200 import tqpkernels
    n = 1000
    key = torch.arange(n, dtype=torch.int64)
    host = torch.empty(512 + 5, dtype=torch.int64, pin_memory=torch.cuda.is_available())
    cols, B = {
        "five widths": ([key, key.to(torch.int32), key.to(torch.int16), key.to(torch.int8),
                         torch.zeros(n, 25, dtype=torch.uint8)], 32),
        "seven columns": ([key] * 7, 32),
        "int32 key": ([key.to(torch.int32)], 32),
        "B=1024": ([key], 1024),
        "B=24": ([key], 24),
        "B=0": ([key], 0),
        "host_out too short": ([key], 32),
        "pageable host_out": ([key], 32),
    }[case]
    if case == "host_out too short":
        host = host[:10]
    if case == "pageable host_out":
        host = torch.empty(512 + 5, dtype=torch.int64)
    with pytest.raises(RuntimeError):
        tqpkernels.partition_sort(cols, [0] * len(cols), 0, None, n, 0, B, False, host)


def test_drop_in_join_cores_refuse_bad_arguments_before_any_kernel():
    from pageflow_b200 import tqpkernels
    k = torch.arange(4, dtype=torch.int64)
    host = torch.empty(2, dtype=torch.int64)
    with pytest.raises(RuntimeError, match="one or two"):
        tqpkernels.join_unique_hash([k, k, k], [k, k, k], host)
    with pytest.raises(RuntimeError):
        tqpkernels.join_unique_hash([k], [k], host)
    with pytest.raises(RuntimeError):
        tqpkernels.join_semi_anti(k, k, None, None, 0, False, host)
    with pytest.raises(RuntimeError):
        tqpkernels.join_expand(k, k, k, host)


def test_slab_rejects_bad_specs_on_the_host():
    from pageflow_b200.aggregation_slab import DenseAggregationSlab
    with pytest.raises(ValueError, match="invalid key range"):
        DenseAggregationSlab(5, 4, torch.int64, [], [], "cpu")
    with pytest.raises(ValueError, match="unsupported slab reduction"):
        DenseAggregationSlab(0, 4, torch.int64, [(torch.int64, ())], ["mean"], "cpu")


def test_static_scratch_join_refuses_sizes_before_any_device_work():
    # the size check runs on the host before the scratch is looked up, so it
    # answers without a GPU; the pointers are never dereferenced
    from pageflow_b200 import _native
    L = _native.lib()
    fake = ctypes.c_void_p(256)
    for nb, npr in [(540000, 1048576), (1100000, 10), (10, 4 * 1048576)]:
        rc = L.pf_join_unique_hash_static(fake, None, nb, fake, None, npr, 1, fake, fake, fake,
                                          None)
        assert rc == _native.PF_EINVAL
        assert b"static scratch" in L.pf_last_error()
    rc = L.pf_join_unique_hash_static(fake, None, 10, fake, None, 10, 3, fake, fake, fake, None)
    assert rc == _native.PF_EINVAL


def test_bench_functions_name_only_defined_names():
    # every name a bench.py function loads is a local, a module-level name or
    # a builtin: the GPU-only paths cannot fail on a misspelt name at run time
    import ast
    import builtins
    tree = ast.parse((REPO / "bench.py").read_text())
    top = set()
    for n in tree.body:
        if isinstance(n, (ast.FunctionDef, ast.ClassDef)):
            top.add(n.name)
        elif isinstance(n, ast.Assign):
            top |= {t.id for t in n.targets if isinstance(t, ast.Name)}
        elif isinstance(n, (ast.Import, ast.ImportFrom)):
            top |= {a.asname or a.name.split(".")[0] for a in n.names}
    missing = []
    for fn in (n for n in tree.body if isinstance(n, ast.FunctionDef)):
        local = {a.arg for a in fn.args.args + fn.args.kwonlyargs}
        for node in ast.walk(fn):
            if isinstance(node, ast.Name) and isinstance(node.ctx, ast.Store):
                local.add(node.id)
            elif isinstance(node, (ast.Import, ast.ImportFrom)):
                local |= {a.asname or a.name.split(".")[0] for a in node.names}
            elif isinstance(node, (ast.FunctionDef, ast.Lambda)) and node is not fn:
                local |= {a.arg for a in node.args.args}
                if isinstance(node, ast.FunctionDef):
                    local.add(node.name)
            elif isinstance(node, ast.ExceptHandler) and node.name:
                local.add(node.name)
        for node in ast.walk(fn):
            if (isinstance(node, ast.Name) and isinstance(node.ctx, ast.Load)
                    and node.id not in local and node.id not in top
                    and not hasattr(builtins, node.id)):
                missing.append(f"{fn.name}:{node.lineno}:{node.id}")
    assert missing == []


def test_unique_hash_workspace_fits_the_references_scratch_figure():
    # the reference's dispatch compares 2 * n_build * 4 + n_probe * 20 bytes
    # (operators/join_core.py:64-68) with its limit; the library's own
    # workspace for the table and the partners fits in that figure's share of
    # them plus the per-block counts
    from pageflow_b200 import _native
    nb, npr = 10**6, 4 * 10**6
    ws = _native.lib().pf_join_unique_hash_workspace(nb, npr)
    assert 2 * nb * 4 + npr * 4 <= ws <= 2 * nb * 4 + npr * 4 + 64 * 1024
