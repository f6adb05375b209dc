#!/usr/bin/env bash
# Build the CPU oracles (test infrastructure only).
#
#  oracle/libhop_oracle.so            own restatement (oracle/hop_oracle.c)
#  oracle/_ref/libplqcd_ref_patched.so the reference's plain-C hopping pair
#                                     (lib/dirac.c, lib/start.c, lib/utils.c),
#                                     compiled from the read-only reference
#                                     with the two one-line fixes applied at
#                                     compile time
#  oracle/_ref/libplqcd_ref_shipped.so the same sources exactly as shipped
#
# The reference is compiled where it lies: no reference source is copied.
# lib/dirac.c is fed to gcc through a pipe, with sed changing line 643's
# forward link u[4*i] to u[4*(i+V/2)] for the patched build; the su3.h macro
# fix comes from the forced-include prelude oracle/ref_fix_su3.h. MPI is the
# single-rank stub in oracle/mpi_stub. -DASSYMBLY without -DSSE2/-DSSE3
# selects the plain-C macros (the inline-asm ones miscompile with gcc 13).
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
#        oracle/build_ref.sh --root      (print the reference root and exit)
# The root is the argument, else $PLQCD_REFERENCE_ROOT, else /root/reference.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
if [ "${1:-}" = "--root" ]; then
    echo "${PLQCD_REFERENCE_ROOT:-/root/reference}"
    exit 0
fi
REF="${1:-${PLQCD_REFERENCE_ROOT:-/root/reference}}"
CC="${CC:-gcc}"
# -B points the driver at a gcc install dir that holds libgomp.spec (the
# wrapper compiler in this image lacks it; harmless elsewhere).
GCCDIR="$(dirname "$("$CC" -print-libgcc-file-name)")"
if [ ! -f "$GCCDIR/libgomp.spec" ]; then
    for d in /usr/lib/gcc/x86_64-linux-gnu/*/; do
        if [ -f "$d/libgomp.spec" ]; then GCCDIR="${d%/}"; fi
    done
fi
CFLAGS="-std=gnu99 -fcommon -fopenmp -O2 -fPIC -w -B$GCCDIR/"

"$CC" $CFLAGS -shared -o "$HERE/libhop_oracle.so" "$HERE/hop_oracle.c" -lm

if [ ! -f "$REF/lib/dirac.c" ]; then
    echo "build_ref.sh: reference sources not found under $REF; skipping oracle/_ref" >&2
    exit 0
fi
OUT="$HERE/_ref"
mkdir -p "$OUT"
INC="-I$HERE/mpi_stub -I$REF/include"
LINE643="$(sed -n 643p "$REF/lib/dirac.c")"
case "$LINE643" in
    *"ub0 = &u[4*i];"*) ;;
    *) echo "build_ref.sh: unexpected lib/dirac.c:643: $LINE643" >&2; exit 1 ;;
esac

build() {  # $1 = variant name, $2 = extra flags, $3 = sed expression for dirac.c
    local name="$1" extra="$2" sedexpr="$3" tmpd
    tmpd="$(mktemp -d)"
    sed -e "$sedexpr" "$REF/lib/dirac.c" | "$CC" $CFLAGS -DASSYMBLY $INC $extra -x c -c - -o "$tmpd/dirac.o"
    "$CC" $CFLAGS -DASSYMBLY $INC $extra -c "$REF/lib/start.c" -o "$tmpd/start.o"
    "$CC" $CFLAGS -DASSYMBLY $INC $extra -c "$REF/lib/utils.c" -o "$tmpd/utils.o"
    "$CC" $CFLAGS -DASSYMBLY $INC $extra -c "$HERE/ref_shim.c" -o "$tmpd/shim.o"
    "$CC" -shared -fopenmp -B"$GCCDIR/" -Wl,-Bsymbolic -o "$OUT/libplqcd_ref_$name.so" \
        "$tmpd/dirac.o" "$tmpd/start.o" "$tmpd/utils.o" "$tmpd/shim.o" -lm
    rm -f "$tmpd"/*.o
    rmdir "$tmpd"
}
build patched "-include $HERE/ref_fix_su3.h" '643s/ub0 = &u\[4\*i\];/ub0 = \&u[4*(i+V\/2)];/'
build shipped "" ''
echo "built $OUT/libplqcd_ref_patched.so $OUT/libplqcd_ref_shipped.so"
