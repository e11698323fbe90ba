#!/usr/bin/env bash
# TEST INFRASTRUCTURE (oracle).  Builds the reference's own NSPT code as an
# oracle binary, from the sources where they lie (nothing is copied into the
# repository; every output goes under oracle/_ref/, which git ignores).
#
#   oracle/build_ref.sh N BC GF NTX NTY NTZ [ACTION]
#     N    perturbative order: allocORD = PTORD = N  (choices.h:30)
#     BC   pbc | tw          periodic, or twisted in y and z (choices.h:42-49)
#     GF   local | fa        local stochastic gauge fixing (nspt.cc:660-862)
#                            or Fourier accelerated (nspt.cc:866-948)
#     NTX NTY NTZ            OpenMP block grid (choices.h:124-128); 1 1 1 for
#                            parity runs, larger only for CPU timing
#     ACTION                 wil (default) | tlsym | iwa | dbw2: GAUGE_ACTION
#                            (choices.h:110, periodic builds only)
#     UPDATE                 jacobi (default): UPDATE_ONTHEFLY off, the parity
#                            builds; otf: the reference's default on-the-fly
#                            (Gauss-Seidel) update, for statistical comparisons
#
# The build uses the reference's flags (Makefile:2: -DUSE_RAND55
# -D__PARALLEL_OMP__ -O3 -fopenmp -std=c++0x) plus
#   * a choices.h generated from the reference's copy with sed: allocORD = N,
#     UPDATE_ONTHEFLY off (the reference's Jacobi option, nspt.cc:428-430 and
#     nspt.cc:992), the boundary conditions and the thread grid, and
#     __WILLOOP_2x2__ on (choices.h:77, periodic builds; WL2x2 only adds a
#     measurement that the harness runs on request);
#   * -DPBC for periodic builds, which the FA path needs for p2hat[0]
#     (lattice.h:1144-1149) and the zero-momentum cut (nspt.cc:881-883);
#   * -D__FA_GAUGE_FIXING__ for GF=fa (nspt.cc:1019-1023);
#   * oracle/fftw_shim in place of FFTW3, which is not installed here;
#   * oracle/ref_harness.cc in place of Quenched.cc's main.
# `-I-` makes the generated choices.h win over the one beside the reference's
# sources for every `#include "choices.h"`.
set -euo pipefail
REF=${REF:-$(cd "$(dirname "$0")/../.." && pwd)/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
N=${1:?N}; BC=${2:?BC}; GF=${3:?GF}; NTX=${4:-1}; NTY=${5:-1}; NTZ=${6:-1}; ACT=${7:-wil}
UPD=${8:-jacobi}
NAME=ref_N${N}_${BC}_${GF}_t${NTX}${NTY}${NTZ}
if [ "$ACT" != wil ]; then NAME=${NAME}_${ACT}; fi
if [ "$UPD" = otf ]; then NAME=${NAME}_otf; elif [ "$UPD" != jacobi ]; then
  echo "build_ref: unknown update $UPD" >&2; exit 2
fi
OUT=$HERE/_ref/$NAME
if [ ! -f "$REF/nspt.cc" ]; then
  echo "build_ref: reference sources not found at $REF" >&2
  exit 3
fi
mkdir -p "$OUT/cfg" "$OUT/obj"
SED=(-e "s/^#define allocORD 6\$/#define allocORD $N/"
     -e "s/^#define ntx  1\$/#define ntx  $NTX/"
     -e "s/^#define nty  1\$/#define nty  $NTY/"
     -e "s/^#define ntz  1\$/#define ntz  $NTZ/"
     -e "s/^\/\/#define __WILLOOP_2x2__\$/#define __WILLOOP_2x2__/")
if [ "$UPD" = jacobi ]; then
  SED+=(-e "s/^#define UPDATE_ONTHEFLY\$/\/* UPDATE_ONTHEFLY off: Jacobi update *\//")
fi
DEFS=(-DDSFMT_MEXP=19937 -DUSE_RAND55 -D__PARALLEL_OMP__)
if [ "$BC" = tw ]; then
  SED+=(-e "s/^#define PERIODIC_BC\$/\/* PERIODIC_BC off *\//"
        -e "s/^\/\/#define TWISTED_BC\$/#define TWISTED_BC/")
else
  DEFS+=(-DPBC)
fi
if [ "$GF" = fa ]; then DEFS+=(-D__FA_GAUGE_FIXING__); fi
case "$ACT" in
  wil) ;;
  tlsym|iwa|dbw2)
    UP=$(echo "$ACT" | tr a-z A-Z)
    SED+=(-e "s/^#define GAUGE_ACTION WIL \/\/Alternatives/#define GAUGE_ACTION $UP \/\/Alternatives/") ;;
  *) echo "build_ref: unknown action $ACT" >&2; exit 2 ;;
esac
sed "${SED[@]}" "$REF/choices.h" > "$OUT/cfg/choices.h.new"
if ! cmp -s "$OUT/cfg/choices.h.new" "$OUT/cfg/choices.h" 2>/dev/null; then
  mv "$OUT/cfg/choices.h.new" "$OUT/cfg/choices.h"
else
  rm -f "$OUT/cfg/choices.h.new"
fi
grep -q "^#define allocORD $N\$" "$OUT/cfg/choices.h"
grep -q "^#define __WILLOOP_2x2__" "$OUT/cfg/choices.h"  # inside #ifdef PERIODIC_BC
CXX=${ORACLE_CXX:-/usr/bin/g++}
FLAGS=(-O3 -fopenmp -std=c++11 -w "${DEFS[@]}" -I"$OUT/cfg" -I- -I"$REF"
       -I"$REF/ranlxd" -I"$HERE/fftw_shim")
STAMP="$OUT/obj/.stamp"
if [ ! -x "$OUT/ref_harness" ] || [ "$HERE/ref_harness.cc" -nt "$OUT/ref_harness" ] \
   || [ "$OUT/cfg/choices.h" -nt "$OUT/ref_harness" ]; then
  for src in nspt.cc QCDpt.cc MyMath.cc MyRand.cc MyQCD.cc; do
    $CXX "${FLAGS[@]}" -c "$REF/$src" -o "$OUT/obj/${src%.cc}.o" 2>&1 \
      | grep -v "obsolete option" >&2 || true
  done
  $CXX "${FLAGS[@]}" -c "$REF/ranlxd/ranlxd.cc" -o "$OUT/obj/ranlxd.o" 2>&1 \
    | grep -v "obsolete option" >&2 || true
  $CXX "${FLAGS[@]}" -c "$HERE/ref_harness.cc" -o "$OUT/obj/ref_harness.o" 2>&1 \
    | grep -v "obsolete option" >&2 || true
  /usr/bin/gcc -O2 -std=c99 -D_DEFAULT_SOURCE -I"$HERE/fftw_shim" -c "$HERE/fftw_shim/fftw_shim.c" -o "$OUT/obj/fftw_shim.o"
  /usr/bin/gcc -O2 -std=c99 -D_DEFAULT_SOURCE -I"$HERE/fftw_shim" -c "$HERE/fftw_shim/oracle_dft.c" -o "$OUT/obj/oracle_dft.o"
  $CXX -O3 -fopenmp -o "$OUT/ref_harness" "$OUT"/obj/*.o -lm
  touch "$STAMP"
fi
echo "$OUT/ref_harness"
