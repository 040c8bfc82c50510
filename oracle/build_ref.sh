#!/bin/sh
# build_ref.sh -- TEST INFRASTRUCTURE ONLY.
#
# Compiles the reference's Slater-Koster routines
# (nemo3d/src/ham/mb_ham_spds_micro.c) and its zincblende cell
# (nemo3d/src/base/Cell.c) from the NEMO-3D source tree, where they lie,
# together with oracle/ref_sk_driver.cc into oracle/_ref/ref_sk.  The tests
# use it to check the oracle's restatement of the bond blocks, the strain
# diagonal correction, the on-site/spin-orbit block, the sp3s* parameter
# conversion and the dangling-bond passivation.  Outputs go to oracle/_ref/
# only.
#
# Usage: oracle/build_ref.sh <path to the NEMO_3D directory of the reference>
#        (or set NEMO3D_SRC to it)
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
R=${1:-${NEMO3D_SRC:-}}
OUT="$HERE/_ref"
if [ -z "$R" ]; then
  echo "build_ref.sh: give the reference's NEMO_3D directory (argument or NEMO3D_SRC); skipped" >&2
  exit 0
fi
if [ ! -f "$R/nemo3d/src/ham/mb_ham_spds_micro.c" ]; then
  # machines without the reference tree use the prebuilt binary, if any
  echo "build_ref.sh: reference sources not found under $R; skipped" >&2
  exit 0
fi
mkdir -p "$OUT"
INC="-I$R/nemo3d/src/base -I$R/nemo3d/src/ham -I$R/nemo3d/src/math -I$R/nemo3d/src/io \
 -I$R/nemo3d/src/util -I$R/nemo3d/src/top -I$R/eigen/include -I$R/nml/include \
 -I$R/XMLtoC/apps/ioNemo3D/src -I$R/XMLtoC/src -I$R/xerces-c-src2_1_0/include \
 -I$R/xerces-c-src2_1_0/src -I$R/xerces-c-src2_1_0/src/xercesc"
# the reference's own macro set (mb_ham_spds_micro.h:74-80) plus the serial build
DEFS="-DFAKE_MPI -DLINUX"
FLAGS="-O2 -ffp-contract=off -fpermissive -w -ffunction-sections -fdata-sections"
g++ -x c++ $FLAGS $DEFS $INC -c "$R/nemo3d/src/ham/mb_ham_spds_micro.c" -o "$OUT/mb_ham_spds_micro.o"
# the zincblende cell (neighbour map, positions) for the passivation check
g++ -x c++ $FLAGS $DEFS $INC -c "$R/nemo3d/src/base/Cell.c" -o "$OUT/Cell.o"
g++ $FLAGS $DEFS $INC -c "$HERE/ref_sk_driver.cc" -o "$OUT/ref_sk_driver.o"
# routines the driver never reaches (geometry, dense eigensolvers) are
# dropped by --gc-sections together with their unresolved references
g++ -Wl,--gc-sections -o "$OUT/ref_sk" "$OUT/ref_sk_driver.o" "$OUT/mb_ham_spds_micro.o" \
  "$OUT/Cell.o" -lm
# the reference's Lanczos drivers (eigen/src/lanczos.c, lanczos_blk.c) and
# its serial MPI layer, with nml routines, dstebz forwarded to scipy's bundled OpenBLAS
# and the oracle's H*x as its matmul: oracle/_ref/libref_lanczos.so
BLAS=$(python3 -c "import glob, os, scipy; print(sorted(glob.glob(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), 'scipy.libs', 'libscipy_openblas-*.so')))[0])" 2>/dev/null || true)
if [ -n "$BLAS" ] && [ -f "$HERE/liboracle.so" ]; then
  FPIC="-fPIC"
  g++ -x c++ $FLAGS $FPIC $DEFS $INC -c "$R/eigen/src/lanczos.c" -o "$OUT/lanczos.o"
  g++ -x c++ $FLAGS $FPIC $DEFS $INC -c "$R/eigen/src/mpi_fake.c" -o "$OUT/mpi_fake.o"
  # the block Lanczos (LAPACK names with one trailing underscore; the
  # function form of the serial Allreduce_MPI_sp, which the driver defines
  # with MPI's meaning, for the double and complex pointers the source passes;
  # ref_blk_compat.h also supplies the memset header the source omits)
  g++ -x c++ $FLAGS $FPIC $DEFS -DFORTRAN_UNDERSCORE -DNoGnuStatementExpre $INC \
    -include "$HERE/ref_blk_compat.h" \
    -c "$R/eigen/src/lanczos_blk.c" -o "$OUT/lanczos_blk.o"
  g++ $FLAGS $FPIC $DEFS -DNoGnuStatementExpre $INC -I"$HERE" -c "$HERE/ref_lanczos_driver.cc" \
    -o "$OUT/ref_lanczos_driver.o"
  g++ -shared -o "$OUT/libref_lanczos.so" "$OUT/ref_lanczos_driver.o" "$OUT/lanczos.o" \
    "$OUT/lanczos_blk.o" "$OUT/mpi_fake.o" "$HERE/liboracle.so" "$BLAS" -Wl,-rpath,"$HERE" \
    -Wl,-rpath,"$(dirname "$BLAS")" -Wl,--no-undefined -lm
  echo "$OUT/libref_lanczos.so"
fi
echo "$OUT/ref_sk"
