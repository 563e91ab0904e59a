#!/bin/bash
# Builds the reference's own CUDA operator kernels (PageFlow
# operators/kernels/{tqpkernels,partition_sort,join_core}.cu, compiled where
# they lie, unmodified) for sm_100a into oracle/_ref/tqpkernels.so: the
# Python extension module `tqpkernels` that TQPlib/tqpkernels re-exports.
# Test infrastructure only (GPU parity of the drop-in against the reference's
# kernels, and the GPU baseline of the reference's path); the product never
# loads it.  Usage: oracle/build_ref.sh /path/to/PageFlow (or PAGEFLOW_REFERENCE)
set -euo pipefail
REF=${1:-${PAGEFLOW_REFERENCE:?give the reference checkout as the first argument or in PAGEFLOW_REFERENCE}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
SRC="$REF/operators/kernels"
[ -d "$SRC" ] || { echo "no reference sources at $SRC" >&2; exit 1; }
mkdir -p "$OUT"
PY=${PYTHON:-python}
read -r TORCH_INC TORCH_INC2 TORCH_LIB PYB_INC PY_INC EXT <<<"$($PY - <<'EOF'
import sysconfig, torch.utils.cpp_extension as c, pybind11
inc = c.include_paths()
print(inc[0], inc[1], c.library_paths()[0], pybind11.get_include(),
      sysconfig.get_paths()["include"], sysconfig.get_config_var("EXT_SUFFIX"))
EOF
)"
ABI=$($PY -c "import torch; print(int(torch._C._GLIBCXX_USE_CXX11_ABI))")
FLAGS=(-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -lineinfo
       -Xcompiler -fPIC -D_GLIBCXX_USE_CXX11_ABI=$ABI -DTORCH_EXTENSION_NAME=tqpkernels
       -DTORCH_API_INCLUDE_EXTENSION_H --expt-relaxed-constexpr
       -I "$TORCH_INC" -I "$TORCH_INC2" -I "$PYB_INC" -I "$PY_INC" -I "$SRC")
for f in tqpkernels partition_sort join_core; do
  nvcc "${FLAGS[@]}" -c "$SRC/$f.cu" -o "$OUT/$f.o" &
done
wait
nvcc -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fPIC \
  "$OUT/tqpkernels.o" "$OUT/partition_sort.o" "$OUT/join_core.o" \
  -L "$TORCH_LIB" -lc10 -lc10_cuda -ltorch -ltorch_cpu -ltorch_cuda -ltorch_python \
  -Xlinker -rpath -Xlinker "$TORCH_LIB" -o "$OUT/tqpkernels$EXT"
rm -f "$OUT"/*.o
echo "$OUT/tqpkernels$EXT"
