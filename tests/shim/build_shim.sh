#!/bin/sh
# build_shim.sh -- TEST RECIPE.
#
# Compiles the eigensolve_lanczos drop-in (nemo3d_b200/shim/
# eigensolve_lanczos_tbgpu.c) against a NEMO-3D tree's own declaration and
# nml headers -- the compiler checks the definition against the reference's
# prototype (eigen/include/lanczos.h:365-391) -- and links it with the test
# allocation stubs (tests/shim/nml_stub.c) and libtbgpu.so into
# tests/shim/_build/libtbgpu_shim.so, which the GPU tests load.
#
# Usage: tests/shim/build_shim.sh <path to the NEMO_3D directory of the reference>
#        (or set NEMO3D_SRC to it)
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/../.." && pwd)
R=${1:-${NEMO3D_SRC:-}}
if [ -z "$R" ] || [ ! -f "$R/eigen/include/lanczos.h" ]; then
  echo "build_shim.sh: reference headers not found (give the NEMO_3D directory); skipped" >&2
  exit 0
fi
OUT="$HERE/_build"
mkdir -p "$OUT"
INC="-I$R/eigen/include -I$R/nml/include -I$R/nemo3d/src/base -I$R/nemo3d/src/io \
 -I$R/nemo3d/src/util -I$ROOT/include"
FLAGS="-O2 -fPIC -Wall -Werror=implicit-function-declaration -Wno-unused-function -Wno-unused-variable -DFAKE_MPI -DLINUX"
gcc $FLAGS $INC -c "$ROOT/nemo3d_b200/shim/eigensolve_lanczos_tbgpu.c" -o "$OUT/shim.o"
gcc $FLAGS $INC -c "$HERE/nml_stub.c" -o "$OUT/nml_stub.o"
gcc -shared -o "$OUT/libtbgpu_shim.so" "$OUT/shim.o" "$OUT/nml_stub.o" \
  -L"$ROOT/nemo3d_b200" -ltbgpu -Wl,-rpath,"$ROOT/nemo3d_b200" -Wl,--no-undefined
echo "$OUT/libtbgpu_shim.so"
