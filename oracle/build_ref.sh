#!/usr/bin/env bash
# Builds the reference's own serial Monte Carlo functions into oracle/_ref/.
#
# Test infrastructure only.  The reference (MCnptColloid.c) is compiled from
# where it lies; it is never copied into this repository.  It does not compile
# as shipped, so six one-line fixes are applied on the fly (sed -> gcc stdin):
#   366, 3765  missing comma after `int block_offset[3]` in a prototype/definition
#   5027       copy_cell: undeclared `dst` (the parameter is `dest`)
#   5185       `neighbor_idx` used outside the loop that declares it
#   4913       reset_cell(&c) passes Cell** (an error from gcc 14 on)
#   main       renamed to ref_main (-Dmain=ref_main) so a driver can call functions
# None of them touches the Monte Carlo path.  mpistub/ supplies no-op MPI symbols
# (there is no MPI here).  Outputs:
#   oracle/_ref/libmcref_serial.so  -O2 -ffp-contract=off, no OpenMP: the
#                                   arithmetic of the README's plain build, used
#                                   for bit-exact golden vectors
#   oracle/_ref/libmcref_omp.so     -O3 -fopenmp: the reference's OpenMP
#                                   pragmas enabled, used as the timed CPU baseline
#
# Usage: build_ref.sh <reference directory>   (or LCMC_REFERENCE_DIR set)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REFDIR="${1:-${LCMC_REFERENCE_DIR:-}}"
if [ -z "$REFDIR" ]; then
    echo "build_ref.sh: give the reference directory (argument or LCMC_REFERENCE_DIR); oracle/_ref not rebuilt" >&2
    exit 0
fi
REF="$REFDIR/MCnptColloid.c"
OUT="$HERE/_ref"
if [ ! -f "$REF" ]; then
    echo "build_ref.sh: $REF not found; oracle/_ref not rebuilt" >&2
    exit 0
fi
mkdir -p "$OUT"
patch_ref() {
    sed -e '366s/int block_offset\[3\] *$/int block_offset[3],/' \
        -e '3765s/int block_offset\[3\] *$/int block_offset[3],/' \
        -e '5027s/unpack_cell(dst, buf);/unpack_cell(dest, buf);/' \
        -e '5185s/^\( *\)neighbor_idx = 0;/\1int neighbor_idx = 0;/' \
        -e '4913s/reset_cell(&c);/reset_cell(c);/' \
        "$REF"
}
build() {  # $1 = output name, rest = flags
    local name="$1"; shift
    patch_ref | gcc -x c -std=gnu11 -fPIC -w "$@" -I"$HERE/mpistub" -Dmain=ref_main -c - -o "$OUT/$name.ref.o"
    gcc -std=gnu11 -fPIC -O2 "$@" -c "$HERE/ref_driver.c" -o "$OUT/$name.drv.o"
    gcc -std=gnu11 -fPIC -O2 -c "$HERE/mpistub/mpistub.c" -o "$OUT/$name.mpi.o"
    gcc -shared "$@" -o "$OUT/$name.so" "$OUT/$name.ref.o" "$OUT/$name.drv.o" "$OUT/$name.mpi.o" -lm
    rm -f "$OUT/$name.ref.o" "$OUT/$name.drv.o" "$OUT/$name.mpi.o"
}
build libmcref_serial -O2 -ffp-contract=off
build libmcref_omp -O3 -march=x86-64-v3 -fopenmp
echo "built $OUT/libmcref_serial.so $OUT/libmcref_omp.so"
