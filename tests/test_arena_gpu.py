"""The library's device buffers come from whatever allocator torch has.

PageFlow installs its pooled device arena as torch's allocator
(main.py:1389-1395, the C ABI of memory/cuda_memory_allocator.cc:1234-1241).
Here a counting allocator (tests/arena/counting_alloc.cpp, built on the fly)
is installed the same way, in a fresh process before any CUDA tensor exists;
then the drop-in partition and join cores, the fused join + group-by and the
gather run, and every workspace and output they used must lie in a block the
allocator served, while the device's free memory drops by no more than the
allocator's live bytes (the library allocates nothing beside them)."""
from __future__ import annotations

import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parents[1]


def _build(tmp: Path) -> Path:
    so = tmp / "libcounting_alloc.so"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.run([nvcc, "-O2", "-shared", "-Xcompiler", "-fPIC", "-x", "cu",
                    str(REPO / "tests" / "arena" / "counting_alloc.cpp"), "-o", str(so),
                    "-lcudart"], check=True)
    return so


def test_every_device_buffer_comes_from_the_installed_allocator(tmp_path):
    so = _build(tmp_path)
    code = textwrap.dedent(f"""
        import ctypes, sys
        sys.path.insert(0, {str(REPO)!r})
        import torch
        so = {str(so)!r}
        alloc = torch.cuda.memory.CUDAPluggableAllocator(so, "pf_test_alloc", "pf_test_free")
        torch.cuda.memory.change_current_allocator(alloc)
        A = ctypes.CDLL(so)
        A.pf_test_owns.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        A.pf_test_live_bytes.restype = ctypes.c_size_t
        A.pf_test_served_blocks.restype = ctypes.c_size_t
        from pageflow_b200 import tqpkernels, gather
        from pageflow_b200.join_aggregate import JoinAggregate
        from pageflow_b200 import datagen

        def owned(t):
            return t.numel() == 0 or A.pf_test_owns(t.data_ptr(), t.numel() * t.element_size())

        def run():
            w = datagen.scaled(datagen.SCALE, 1 / 1000)
            bkey, bgrp = datagen.gen_build(w, "cuda")
            fk, price, disc = datagen.gen_probe(w, "cuda")
            host = torch.empty(64 + 5, dtype=torch.int64, pin_memory=True)
            parts = tqpkernels.partition_sort([bkey, bgrp], [0, 0], 0, None, w.n_build, 0, 64,
                                              False, host)
            jh = torch.empty(2, dtype=torch.int64, pin_memory=True)
            pairs = tqpkernels.join_unique_hash([bkey], [fk], jh)
            plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, "cuda", B=64)
            keys, sums, counts = plan.run(bkey, bgrp, fk, price, disc)
            g = gather.index_select_many([price, disc], pairs[1][:int(jh[0])])
            torch.cuda.synchronize()
            held = parts + pairs + [plan.ws, plan.sum, plan.count, plan.fin_ws, keys, sums,
                                    counts] + g
            assert all(owned(t) for t in held), [owned(t) for t in held]
            return held

        first = run()                      # loads the library's kernels
        del first
        torch.cuda.synchronize()
        live0 = A.pf_test_live_bytes()
        free0 = torch.cuda.mem_get_info()[0]
        held = run()
        live1 = A.pf_test_live_bytes()
        free1 = torch.cuda.mem_get_info()[0]
        assert A.pf_test_served_blocks() > 10
        # the device's drop is the allocator's growth, to its 2 MiB pages
        drop = free0 - free1
        assert drop <= (live1 - live0) + 64 * (2 << 20), (drop, live1 - live0)
        print("arena ok", A.pf_test_served_blocks(), live1)
    """)
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=600, cwd=str(REPO))
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    assert "arena ok" in res.stdout
