#!/bin/sh
# Compiles the reference Tagore module from its own four .cu files, read in
# place, for sm_100a into oracle/_ref/ (git-ignored). The module generates
# golden fixtures (tests/golden/make_golden.py) and runs the interop tests on a
# GPU host; oracle/_ref/merge_ref runs the reference's largeIndex merger on the
# CPU (tests/test_large_ref_cpu.py).
# The reference includes <boost/dynamic_bitset.hpp> for dead CPU code only
# (src/common.cu:65-148); a small stand-in header is written instead.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
# The reference sources: TAGORE_REF, else a `reference` folder beside the repository.
REF=${TAGORE_REF:-$HERE/../../reference}
[ -d "$REF/src" ] || { echo "reference sources not found at $REF (set TAGORE_REF)"; exit 1; }
OUT="$HERE/_ref"
mkdir -p "$OUT/include/boost"
cat > "$OUT/include/boost/dynamic_bitset.hpp" <<'HDR'
#pragma once
#include <cstddef>
#include <vector>
namespace boost {
template <class Block = unsigned long>
struct dynamic_bitset : std::vector<bool> {
  dynamic_bitset(std::size_t n, unsigned long v) : std::vector<bool>(n, v != 0) {}
};
}
HDR
PYINC=$(python3 -c 'import sysconfig; print(sysconfig.get_paths()["include"])')
PBINC=$(python3 -c 'import pybind11; print(pybind11.get_include())')
SUFFIX=$(python3 -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')
/usr/local/cuda/bin/nvcc -ccbin /usr/bin/g++ -gencode arch=compute_100a,code=sm_100a -rdc=true -O3 \
  -std=c++17 -Xcompiler -fPIC,-fopenmp -w \
  -I"$REF/include" -I"$OUT/include" -I"$PBINC" -I"$PYINC" -shared \
  "$REF/pybind.cu" "$REF/src/common.cu" "$REF/src/Tagore_src.cu" "$REF/src/large_index.cu" \
  -o "$OUT/Tagore$SUFFIX" -lgomp
echo "built $OUT/Tagore$SUFFIX"
# The reference's largeIndex host half (order_merge_main + order_merge_new) on
# given local graphs, for tests/test_large_ref_cpu.py.
/usr/local/cuda/bin/nvcc -ccbin /usr/bin/g++ -gencode arch=compute_100a,code=sm_100a -rdc=true -O2 \
  -std=c++17 -Xcompiler -fopenmp -w -I"$REF/include" -I"$OUT/include" \
  "$HERE/merge_ref_main.cu" "$REF/src/common.cu" "$REF/src/Tagore_src.cu" "$REF/src/large_index.cu" \
  -o "$OUT/merge_ref" -lgomp
echo "built $OUT/merge_ref"
