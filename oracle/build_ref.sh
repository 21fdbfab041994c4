#!/usr/bin/env bash
# Builds the test oracle oracle/_ref/libmidapack_ref.so from the reference's
# own, unmodified C sources (read in place, never copied) plus the
# project-written shims in oracle/shim/ that stand in for MPI, FFTW3, LAPACKE
# and CFITSIO, none of which exist in this image.  Test infrastructure only.
#
# Usage: oracle/build_ref.sh [--if-present] [REFERENCE_ROOT]
#   REFERENCE_ROOT defaults to $MIDAPACK_REFERENCE, else /root/reference.
#   --if-present: exit 0 without building when the sources are not there
#   (a machine that only has the prebuilt oracle/_ref).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
IF_PRESENT=0
if [ "${1:-}" = "--if-present" ]; then IF_PRESENT=1; shift; fi
REF="${1:-${MIDAPACK_REFERENCE:-/root/reference}}"
OUT="$HERE/_ref"
if [ ! -d "$REF/algebra" ]; then
  if [ "$IF_PRESENT" = 1 ]; then exit 0; fi
  echo "build_ref.sh: reference sources not found at $REF" >&2
  exit 2
fi
mkdir -p "$OUT/obj"

CFLAGS=(-O2 -g -fPIC -std=gnu11 -DW_MPI -w -rdynamic
  -I"$HERE/shim"
  -I"$REF/algebra/include" -I"$REF/algebra/include/mapmat" -I"$REF/algebra/include/toeplitz"
  -I"$REF/algebra/include/templates"
  -I"$REF/mappraiser/include" -I"$REF/mappraiser/include/mappraiser")

# the reference ships two libraries (libmidapack: algebra/, libmappraiser:
# mappraiser/) that define a few symbols twice (defineBlocks_avg, transpose_nn);
# they are kept as two shared objects, each bound to its own definitions.
ALG_SRCS=(
  algebra/src/mapmat/mapmat.c algebra/src/mapmat/csort.c algebra/src/mapmat/cindex.c
  algebra/src/mapmat/als.c algebra/src/mapmat/alm.c algebra/src/mapmat/bitop.c
  algebra/src/mapmat/ring.c algebra/src/mapmat/butterfly.c
  algebra/src/toeplitz/toeplitz.c algebra/src/toeplitz/toeplitz_block.c
  algebra/src/toeplitz/toeplitz_params.c algebra/src/toeplitz/toeplitz_rshp.c
  algebra/src/toeplitz/toeplitz_nofft.c algebra/src/toeplitz/toeplitz_wizard.c
  algebra/src/toeplitz/toeplitz_seq.c algebra/src/toeplitz/toeplitz_utils.c
  algebra/src/toeplitz/toeplitz_gappy.c
  algebra/src/templates/templates.c
)
MAP_SRCS=(
  mappraiser/src/pcg_true.c mappraiser/src/precond.c mappraiser/src/create_toeplitz.c
  mappraiser/src/mappraiser.c
)

compile() { gcc "${CFLAGS[@]}" -c "$1" -o "$2"; }
SHIM_OBJS=()
for s in shim_mpi.c shim_fftw.c shim_lapacke.c shim_fits.c; do
  compile "$HERE/shim/$s" "$OUT/obj/$s.o"; SHIM_OBJS+=("$OUT/obj/$s.o")
done
gcc -shared -Wl,-Bsymbolic -o "$OUT/libmidapack_ref_shims.so" "${SHIM_OBJS[@]}" -lm -lpthread
ALG_OBJS=()
for s in "${ALG_SRCS[@]}"; do
  o="$OUT/obj/$(echo "$s" | tr '/' '_').o"; compile "$REF/$s" "$o"; ALG_OBJS+=("$o")
done
gcc -shared -Wl,-Bsymbolic -o "$OUT/libmidapack_ref_algebra.so" "${ALG_OBJS[@]}" \
  -L"$OUT" -lmidapack_ref_shims -Wl,-rpath,'$ORIGIN' -lm
MAP_OBJS=()
for s in "${MAP_SRCS[@]}"; do
  o="$OUT/obj/$(echo "$s" | tr '/' '_').o"; compile "$REF/$s" "$o"; MAP_OBJS+=("$o")
done
compile "$HERE/ref_driver.c" "$OUT/obj/ref_driver.o"; MAP_OBJS+=("$OUT/obj/ref_driver.o")
gcc -shared -Wl,-Bsymbolic -o "$OUT/libmidapack_ref.so" "${MAP_OBJS[@]}" \
  -L"$OUT" -lmidapack_ref_algebra -lmidapack_ref_shims -Wl,-rpath,'$ORIGIN' -lm -lpthread
echo "built $OUT/libmidapack_ref.so"
