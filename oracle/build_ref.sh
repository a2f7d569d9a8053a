#!/usr/bin/env bash
# Builds the reference's own step implementation into oracle/_ref/ (test
# infrastructure).  Compiles src/unit_1.cu and src/kernel.cu unmodified, where
# they lie under the reference checkout, with NO_TREE (the shipped .conf files
# run with the tree off), plus oracle/ref_shim.c for the host globals the
# reference's src/main.c would otherwise provide.  Outputs go only to
# oracle/_ref/, which git ignores; the .so travels to the GPU machine.
#
#   VX_REFERENCE_DIR=<reference checkout> oracle/build_ref.sh
# (default: the checkout this repository was built beside, /root/reference).
# Exits 3 when the reference sources are not there.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${VX_REFERENCE_DIR:-${REF:-/root/reference}}"
OUT="$HERE/_ref"
NVCC="${NVCC:-nvcc}"
if [ ! -f "$REF/src/unit_1.cu" ] || [ ! -f "$REF/src/kernel.cu" ]; then
    echo "build_ref: reference sources not found under $REF" >&2
    exit 3
fi
mkdir -p "$OUT"
ARCH="-gencode arch=compute_100a,code=sm_100a"
FLAGS="-O2 -DNO_TREE -I$REF/include -w -rdc=true -Xcompiler -fPIC $ARCH"
"$NVCC" $FLAGS -c "$REF/src/unit_1.cu" -o "$OUT/unit_1.o"
"$NVCC" $FLAGS -c "$REF/src/kernel.cu" -o "$OUT/kernel.o"
gcc -O2 -fPIC -std=gnu99 -DNO_TREE -I"$REF/include" -I/usr/local/cuda/include \
    -c "$HERE/ref_shim.c" -o "$OUT/ref_shim.o"
"$NVCC" -shared -rdc=true $ARCH -Xcompiler -fPIC -o "$OUT/libvortex_ref.so" \
    "$OUT/unit_1.o" "$OUT/kernel.o" "$OUT/ref_shim.o" -lcudart_static -lm
# The reference's whole program (its own src/main.c driver), for end-to-end
# comparisons, and the same main.c linked against this repository's library
# in place of src/unit_1.cu + src/kernel.cu (the link-swap drop-in).
gcc -O2 -std=gnu99 -DNO_TREE -Wno-unused-result -I"$REF/include" -I/usr/local/cuda/include \
    -c "$REF/src/main.c" -o "$OUT/main.o"
"$NVCC" $FLAGS -c "$REF/src/unit_1.cu" -o "$OUT/unit_1.o"
"$NVCC" $FLAGS -c "$REF/src/kernel.cu" -o "$OUT/kernel.o"
"$NVCC" -rdc=true $ARCH -o "$OUT/vortex_ref" "$OUT/main.o" "$OUT/unit_1.o" "$OUT/kernel.o" -lm
LIBDIR="$(cd "$HERE/../vortex_b200" && pwd)"
if [ -f "$LIBDIR/libvortex_b200.so" ]; then
    gcc -o "$OUT/vortex_linkswap" "$OUT/main.o" -L"$LIBDIR" -lvortex_b200 \
        -Wl,-rpath,'$ORIGIN/../../vortex_b200' -L/usr/local/cuda/lib64 -lcudart -lm
fi
rm -f "$OUT"/*.o
echo "built $OUT/libvortex_ref.so $OUT/vortex_ref $OUT/vortex_linkswap"
