#!/usr/bin/env bash
# Builds the reference DREAM delay-and-sum CPU implementation, unmodified, from
# its own sources into oracle/_ref/ as the pybind11 modules `das` (FP64) and
# `das_f` (FP32), and the reference's rectangular-transducer SIR kernel
# (opencl/dreamrect.cl, OpenCL C that compiles as plain C through
# oracle/cl_shim.h) as libref_dreamrect.so, and the reference's array helpers
# (src/arr_functions.cc: focusing, steering and apodisation of array elements)
# with oracle/ref_arr_driver.cc as libref_arr.so, and the reference's CPU conv(),
# dreamrect and dream_arr_rect as libref_cpu.so (FFTW replaced by the stub in
# oracle/fftw_stub/, see below). These are test infrastructure: they pin the
# oracles and serve as CPU baselines. Nothing on the product path loads them.
#
# Sources compiled (paths inside the reference tree):
#   python/src/py_das.cc  extra_src/das.cc  src/affinity.cc  src/dream_error.cc
#   opencl/dreamrect.cl  src/arr_functions.cc
#   extra_src/conv.cc  src/dreamrect.cc  src/dream_arr_rect.cc  src/attenuation.cc
# Flags: -O3 -ffp-contract=off, no -march=native, so the x86-64 baseline ISA
# (no FMA) computes every product and sum exactly as written.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
#   default: $DREAM_REFERENCE_SRC, else the directory "reference" beside this repository
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${DREAM_REFERENCE_SRC:-$(cd "$HERE/../.." && pwd)/reference}}"
OUT="$HERE/_ref"
if [ ! -f "$REF/extra_src/das.cc" ]; then
  echo "build_ref: reference sources not found under $REF" >&2
  exit 1
fi
PY="${PYTHON:-python3}"
PYINC="$($PY -c 'import sysconfig; print(sysconfig.get_paths()["include"])')"
PBINC="$($PY -c 'import pybind11; print(pybind11.get_include())')"
EXT="$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')"
mkdir -p "$OUT"
SRCS=("$REF/python/src/py_das.cc" "$REF/extra_src/das.cc" "$REF/src/affinity.cc" "$REF/src/dream_error.cc")
FLAGS=(-O3 -ffp-contract=off -std=c++14 -shared -fPIC -DDREAM_PYTHON
       -I "$REF/include" -I "$REF/python/include" -I "$PYINC" -I "$PBINC" -lpthread)
g++ "${FLAGS[@]}" "${SRCS[@]}" -o "$OUT/das$EXT"
g++ "${FLAGS[@]}" -DUSE_FLOAT "${SRCS[@]}" -o "$OUT/das_f$EXT"
gcc -O2 -ffp-contract=off -std=gnu99 -shared -fPIC -include "$HERE/cl_shim.h" -x c "$REF/opencl/dreamrect.cl" \
    -x none "$HERE/cl_dreamrect_driver.c" -o "$OUT/libref_dreamrect.so" -lm
g++ -O2 -ffp-contract=off -std=c++14 -shared -fPIC -DDREAM_PYTHON -I "$REF/include" -I "$PYINC" -I "$PBINC" \
    "$REF/src/arr_functions.cc" "$HERE/ref_arr_driver.cc" -o "$OUT/libref_arr.so" -lm
# The reference's CPU conv() (extra_src/conv.cc), dreamrect (src/dreamrect.cc) and dream_arr_rect
# (src/dream_arr_rect.cc) in its Python module's configuration (DREAM_PYTHON, HAVE_FFTW), with
# oracle/fftw_stub/fftw3.h standing in for FFTW: planning succeeds, a transform aborts. Without
# attenuation (alpha = 0) the reference plans but never transforms.
gcc -O2 -std=gnu99 -fPIC -c "$HERE/fftw_stub.c" -I "$HERE" -o "$OUT/fftw_stub.o"
g++ -O2 -ffp-contract=off -std=c++17 -shared -fPIC -DDREAM_PYTHON -DHAVE_FFTW -I "$HERE/fftw_stub" -I "$HERE" \
    -I "$REF/include" -I "$PYINC" -I "$PBINC" "$REF/extra_src/conv.cc" "$REF/src/dreamrect.cc" \
    "$REF/src/dream_arr_rect.cc" "$REF/src/arr_functions.cc" "$REF/src/attenuation.cc" "$REF/src/affinity.cc" \
    "$REF/src/dream_error.cc" "$HERE/ref_cpu_driver.cc" "$OUT/fftw_stub.o" -o "$OUT/libref_cpu.so" -lpthread -lm
rm -f "$OUT/fftw_stub.o"
echo "build_ref: built $OUT/das$EXT, $OUT/das_f$EXT, $OUT/libref_dreamrect.so, $OUT/libref_arr.so and $OUT/libref_cpu.so"
