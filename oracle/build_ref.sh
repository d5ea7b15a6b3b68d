#!/bin/bash
# Build the reference's own B-spline cost function (Plastimatch, CPU flavours)
# into oracle/_ref/libplmref.so, for use as a TEST ORACLE and as the timed
# CPU baseline.  Nothing in the product links it.
#
# The reference sources are compiled where they lie under the reference tree
# (read-only); no source is copied.  ITK is not installed, so
# oracle/ref/prelude.h is force-included to stand in for the few ITK-facing
# headers on the path, and oracle/ref/ holds stand-ins for the two
# cmake-generated headers (plm_config.h, plm_version.h).
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT   (or PLM_REFERENCE in the
# environment)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${PLM_REFERENCE:-}}"
if [ -z "$REF" ]; then
    echo "build_ref: give the reference tree as an argument or PLM_REFERENCE" >&2
    exit 1
fi
SRC="$REF/src"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
if [ ! -d "$SRC/register" ]; then
    echo "build_ref: reference tree not found at $REF" >&2
    exit 1
fi
mkdir -p "$OBJ"
# The system gcc carries libgomp; a CXX/CC exported by the environment may
# point at a toolchain without it, so they are not consulted.
CXX="${REF_CXX:-$(command -v /usr/bin/g++ || command -v g++)}"
CC="${REF_CC:-$(command -v /usr/bin/gcc || command -v gcc)}"
# -O3 -fopenmp as the CPU baseline is quoted; x86-64-v3 (AVX2) rather than
# -march=native because the library is built here and run on the GPU host.
# -ffp-contract=off keeps the reference's float arithmetic free of FMA
# contraction, so the restated oracle (oracle/bspline_oracle.c) can match it
# bit for bit.
OPT="${REF_OPT:--O3 -march=x86-64-v3 -ffp-contract=off}"
CXXFLAGS="-std=c++11 $OPT -fopenmp -fPIC -w -include $HERE/ref/prelude.h \
  -I$HERE/ref -I$SRC/sys -I$SRC/base -I$SRC/util -I$SRC/register \
  -I$REF/libs/liblbfgs-1.9/include"

UNITS="
base/volume base/direction_cosines base/direction_matrices base/interpolate
base/bspline_interpolate base/bspline_warp base/bspline_xform base/bspline_header base/volume_grad
base/volume_header base/volume_resample base/mha_io base/xpm base/pointset
util/bspline_correspond
register/bspline register/bspline_mse register/bspline_score
register/bspline_state register/bspline_parms register/bspline_mi
register/joint_histogram register/histogram register/bspline_regularize
register/bspline_regularize_analytic register/bspline_regularize_numeric
register/bspline_regularize_semi_analytic register/metric_state
register/bspline_landmarks register/bspline_gm register/similarity_metric_type
register/bspline_optimize register/bspline_optimize_liblbfgs
register/bspline_optimize_steepest
sys/logfile sys/print_and_exit sys/plm_timer sys/string_util sys/file_util
sys/path_util sys/plm_endian sys/plm_fwrite
"
OBJS=()
pids=()
for u in $UNITS; do
    o="$OBJ/$(echo "$u" | tr / _).o"
    OBJS+=("$o")
    $CXX $CXXFLAGS -c "$SRC/$u.cxx" -o "$o" &
    pids+=($!)
done
$CC $OPT -fPIC -w -I"$REF/libs/liblbfgs-1.9/include" \
    -c "$REF/libs/liblbfgs-1.9/lib/lbfgs.c" -o "$OBJ/lbfgs.o" &
pids+=($!)
$CXX $CXXFLAGS -c "$HERE/ref/ref_driver.cxx" -o "$OBJ/ref_driver.o" &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
$CXX -shared -fopenmp -Wl,--no-undefined -o "$OUT/libplmref.so" \
    "${OBJS[@]}" "$OBJ/lbfgs.o" "$OBJ/ref_driver.o" -lm
echo "build_ref: wrote $OUT/libplmref.so"

# The reference-side drop-in (oracle/ref/b200_adapter.cxx): the adapter a
# maintainer would add, compiled against the reference headers and linked
# with both libraries, for the tests that drive the product through it.
B200="$HERE/../plastimatch_b200"
if [ -f "$B200/libplastimatch_b200.so" ]; then
    $CXX $CXXFLAGS -c "$HERE/ref/b200_adapter.cxx" -o "$OBJ/b200_adapter.o"
    $CXX -shared -fopenmp -o "$OUT/libb200adapter.so" "$OBJ/b200_adapter.o" \
        -L"$OUT" -lplmref -L"$B200" -lplastimatch_b200 \
        -Wl,-rpath,'$ORIGIN' -Wl,-rpath,'$ORIGIN/../../plastimatch_b200'
    echo "build_ref: wrote $OUT/libb200adapter.so"
fi
