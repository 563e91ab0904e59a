"""Builds the native library in-tree: every CUDA source of pageflow_b200/csrc
compiled for sm_100a with nvcc and linked into pageflow_b200/libpageflow_b200.so
(a plain C-ABI shared library; no torch headers).

    python -m pageflow_b200.build            # build when a source is newer
    python -m pageflow_b200.build --force    # always rebuild
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
OBJ = PKG / "_obj"
LIB = PKG / "libpageflow_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-Wall", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"),
                 "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build "
                       "pageflow_b200")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def headers() -> list[Path]:
    return (sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h"))
            + sorted(INCLUDE.glob("*.h")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, extra: list[str]) -> Path:
    OBJ.mkdir(exist_ok=True)
    obj = OBJ / (src.stem + ".o")
    if _stale(obj, [src] + headers()):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-I", str(INCLUDE), "-c",
               str(src), "-o", str(obj)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}"
                               f"{res.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False,
          extra: list[str] | None = None) -> Path:
    """Compiles every source (in parallel) and links the library; returns
    its path."""
    if force and OBJ.exists():
        shutil.rmtree(OBJ)
    srcs = sources()
    extra = list(extra or [])
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs),
               "-o", str(LIB), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}{res.stderr}")
    if verbose:
        print(LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true",
                    help="print registers / spills / shared memory per kernel")
    args = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if args.ptxas_info else []
    if args.ptxas_info:
        for src in sources():
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-I", str(INCLUDE),
                   "-c", str(src), "-o", os.devnull]
            res = subprocess.run(cmd, capture_output=True, text=True)
            sys.stdout.write(res.stdout + res.stderr)
        return 0
    build(force=args.force, verbose=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
