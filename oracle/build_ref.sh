#!/usr/bin/env bash
# build_ref.sh -- TEST INFRASTRUCTURE ONLY: compile the reference solver
# (tobjec/parallel-critical-collapse) from its own sources into oracle/_ref/.
#
# The reference's CMake build cannot configure here (no pkg-config fftw3 or
# lapacke), so this recipe calls g++ directly on src/*.cpp with:
#   * oracle/shims/fftw3.h + fftw_shim.cpp  -- the FFTW3 subset it uses,
#   * oracle/shims/lapacke.h                 -- LAPACKE_dgesv/dgels declarations,
#     linked against the LP64 OpenBLAS 0.3.15 of the opencv-python-headless wheel,
#   * nlohmann/json 3.11.3 from the cudnn_frontend include tree of the venv.
# The sources are copied into oracle/_ref/src (git-ignored, never committed)
# and exactly one line is changed there: src/NewtonSolver.cpp:456 passes
# &config to ShootingSolver::shoot, without which the OpenMP build dereferences
# a null config at ShootingSolver.cpp:85 on its first Jacobian column.
#
# OpenMP objects are compiled with -fopenmp and linked against libgomp
# directly (this image has no libgomp.spec for the -fopenmp link step).
#
# Outputs (all under oracle/_ref/): libpcc_ref.so (reference objects + the
# ref_harness.cpp C-ABI, OpenMP build), cc_openmp and cc_serial executables,
# and the copied sources and headers (src/, include/) that PCC_REF_NATIVE=1
# rebuilds from on the timing host (native/libpcc_ref.so).
# Runs only where the reference tree exists; the GPU box uses the prebuilt files.
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# The reference checkout: $PCC_REFERENCE_ROOT, else /root/reference.
REF="${PCC_REFERENCE_ROOT:-/root/reference}"
OUT="$HERE/_ref"
SITE="$(python3 -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])')"
JSON_INC="$SITE/include/cudnn_frontend/thirdparty"
BLAS_DIR="$SITE/opencv_python_headless.libs"
BLAS_LIB="$(ls "$BLAS_DIR"/libopenblasp-r0-*.so | head -1)"

CXX=${PCC_ORACLE_CXX:-g++}  # not $CXX: it may name a toolchain without libgomp
LINK="-L$BLAS_DIR -l:$(basename "$BLAS_LIB") -Wl,--disable-new-dtags,-rpath,$BLAS_DIR -Wl,-rpath-link,$BLAS_DIR -lm"

# PCC_REF_NATIVE=1: rebuild only the shared library, -march=native as the
# reference's own CMake build does, from the sources and headers an earlier
# run copied (and patched) into oracle/_ref, into oracle/_ref/native/.  This
# runs on the machine that times the reference (which has no reference tree).
if [ "${PCC_REF_NATIVE:-0}" = "1" ]; then
    [ -d "$OUT/src" ] && [ -d "$OUT/include" ] || { echo "build_ref.sh: no copied sources in $OUT" >&2; exit 1; }
    NAT="$OUT/native"
    mkdir -p "$NAT/obj"
    NFLAGS="-std=c++17 -O3 -DNDEBUG -march=native -fPIC -w -I$HERE/shims -I$OUT/include -I$JSON_INC"
    $CXX $NFLAGS -c "$HERE/shims/fftw_shim.cpp" -o "$NAT/fftw_shim.o"
    for f in "$OUT"/src/*.cpp; do
        b="$(basename "$f" .cpp)"
        [ "$b" = "main" ] && continue
        $CXX $NFLAGS -fopenmp -DUSE_OPENMP -c "$f" -o "$NAT/obj/$b.o" &
    done
    $CXX $NFLAGS -fopenmp -DUSE_OPENMP -c "$HERE/ref_harness.cpp" -o "$NAT/ref_harness.o" &
    wait
    $CXX -shared -o "$NAT/libpcc_ref.so" "$NAT"/obj/*.o "$NAT/ref_harness.o" "$NAT/fftw_shim.o" $LINK -lgomp -lpthread
    echo "built $NAT/libpcc_ref.so (-march=native)"
    exit 0
fi

if [ ! -d "$REF/src" ]; then
    echo "build_ref.sh: reference tree not found at $REF; keeping prebuilt oracle/_ref" >&2
    exit 0
fi

mkdir -p "$OUT/src" "$OUT/include" "$OUT/obj_omp" "$OUT/obj_ser"
cp "$REF"/src/*.cpp "$OUT/src/"
cp "$REF"/include/*.hpp "$OUT/include/"
sed -i '456s/mismatchOut_local);/mismatchOut_local, \&config);/' "$OUT/src/NewtonSolver.cpp"
grep -q 'mismatchOut_local, &config);' "$OUT/src/NewtonSolver.cpp" || { echo "patch at :456 failed" >&2; exit 1; }

# x86-64-v3 (AVX2+FMA) instead of the reference's -march=native so that the
# binaries also run on the GPU host's CPU (which rebuilds the library
# -march=native with PCC_REF_NATIVE=1 before timing it).
FLAGS="-std=c++17 -O3 -DNDEBUG -march=x86-64-v3 -fPIC -w -I$HERE/shims -I$REF/include -I$JSON_INC"

$CXX $FLAGS -c "$HERE/shims/fftw_shim.cpp" -o "$OUT/fftw_shim.o"
for f in "$OUT"/src/*.cpp; do
    b="$(basename "$f" .cpp)"
    $CXX $FLAGS -fopenmp -DUSE_OPENMP -c "$f" -o "$OUT/obj_omp/$b.o" &
    $CXX $FLAGS -c "$f" -o "$OUT/obj_ser/$b.o" &
done
wait
$CXX $FLAGS -fopenmp -DUSE_OPENMP -c "$HERE/ref_harness.cpp" -o "$OUT/ref_harness.o"

OMP_OBJS="$(ls "$OUT"/obj_omp/*.o | grep -v /main.o)"
$CXX -shared -o "$OUT/libpcc_ref.so" $OMP_OBJS "$OUT/ref_harness.o" "$OUT/fftw_shim.o" $LINK -lgomp -lpthread
$CXX -o "$OUT/cc_openmp" "$OUT"/obj_omp/*.o "$OUT/fftw_shim.o" $LINK -lgomp -lpthread
$CXX -o "$OUT/cc_serial" "$OUT"/obj_ser/*.o "$OUT/fftw_shim.o" $LINK
echo "built $OUT/libpcc_ref.so cc_openmp cc_serial"
