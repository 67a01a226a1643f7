#!/usr/bin/env bash
# Builds the reference renderer's CPU path into oracle/_ref/ (TEST
# INFRASTRUCTURE: the checker and the timed CPU baseline, never the product).
#
# The reference (HardCoreCodin/SlimTracinCpp) is MSVC/Win32-only as shipped.
# Its sources are read where they lie, copied to a temporary directory and
# given three portability patches there; nothing of them enters this
# repository and the temporary copy is deleted after the build:
#   1. core/base.h: `u32`/`i32` are `unsigned/signed long int`, 8 bytes on
#      LP64, which breaks every binary layout -> `unsigned/signed int`.
#   2. math/mat3.h: GCC rejects vec3 members in mat3's anonymous union of
#      {X,Y,Z} and {right,up,forward} -> plain `vec3 X, Y, Z;`, and the
#      only users of the aliases (scene/camera.h) renamed to X/Y/Z.
#   3. unqualified abs/sqrt/pow on floats: force-included ref/ref_shim.h
#      (no source edit).
#   (a fourth, for the bmp2texture tool only, is described where it is built)
# Flags: -mfma so the reference's fast_mul_add is fmaf (FP_FAST_FMAF), and
# -ffp-contract=off so nothing else is fused -- the floating-point policy the
# CUDA kernels follow (-fmad=false with explicit fmaf at the same sites).
# -ftrivial-auto-var-init=zero makes the reference's reads of never-written
# locals deterministic (hitsDefaultTetrahedron copies a local RayHit whose
# scaling_factor/id it never sets, core/ray.h:223,304-306): they read 0, the
# value every other never-written tracer member has in the reference app.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_SRC="${SLIM_REFERENCE_SRC:-/root/reference/src}"
OUT="$HERE/_ref"
if [ ! -d "$REF_SRC/slim" ]; then
    echo "build_ref.sh: reference sources not found at $REF_SRC" >&2
    exit 2
fi
mkdir -p "$OUT"
# Where the sources were read, for checks that read the reference's shipped
# assets (examples/*.mesh, *.texture) in place.
printf '%s\n' "$REF_SRC" > "$OUT/reference_src.txt"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
cp -r "$REF_SRC/slim" "$TMP/slim"
sed -i -e 's/typedef unsigned long int  u32;/typedef unsigned int u32;/' \
       -e 's/typedef signed   long int  i32;/typedef signed int i32;/' "$TMP/slim/core/base.h"
grep -q 'typedef unsigned int u32;' "$TMP/slim/core/base.h"
grep -q 'typedef signed int i32;' "$TMP/slim/core/base.h"
python3 - "$TMP/slim/math/mat3.h" <<'EOF'
import sys, re
p = sys.argv[1]
s = open(p).read()
pat = re.compile(r"union\s*\{\s*struct\s*\{\s*vec3 X, Y, Z;\s*\};\s*struct\s*\{\s*vec3 right, up, forward;\s*\};\s*\};")
s2, n = pat.subn("vec3 X, Y, Z;", s)
assert n == 1, "mat3 union not found"
open(p, "w").write(s2)
EOF
sed -i -e 's/orientation\.right/orientation.X/g' -e 's/orientation\.up/orientation.Y/g' \
       -e 's/orientation\.forward/orientation.Z/g' "$TMP/slim/scene/camera.h"

CXXFLAGS=(-std=c++17 -O3 -march=x86-64-v3 -mfma -ffp-contract=off -fno-fast-math -DNDEBUG
          -ftrivial-auto-var-init=zero
          -fPIC -pthread -w -include "$HERE/ref/ref_shim.h" -I "$TMP")
g++ "${CXXFLAGS[@]}" -shared -o "$OUT/libslimref.so.tmp" "$HERE/ref/ref_driver.cpp"
mv "$OUT/libslimref.so.tmp" "$OUT/libslimref.so"
echo "built $OUT/libslimref.so"

# The reference's texture converter (src/bmp2texture.cpp), unmodified, with
# a Windows.h of the few Win32 calls it uses (ref/win32/Windows.h: stdio and
# calloc underneath): oracle/_ref/bmp2texture, the checker of this library's
# host and GPU texture bakers.
cp "$REF_SRC/bmp2texture.cpp" "$TMP/bmp2texture.cpp"
# 4. bmp2texture.cpp keeps its 2D mip loaders in a local `mips` and never
#    sets `loader_mips`, which the final 8-bit pass then dereferences (null)
#    for every texture that is not a cube map: as shipped the converter
#    only bakes cube maps.  The one change the author evidently meant: the
#    2D loaders are also `loader_mips`.
sed -i 's/auto \*mips = new TextureMipLoader\[texture.mip_count\];/auto *mips = loader_mips = new TextureMipLoader[texture.mip_count];/' \
    "$TMP/bmp2texture.cpp"
grep -q 'auto \*mips = loader_mips = new TextureMipLoader' "$TMP/bmp2texture.cpp"
g++ -std=c++17 -O2 -DNDEBUG -march=x86-64-v3 -mfma -ffp-contract=off -fno-fast-math -w \
    -include "$HERE/ref/ref_shim.h" -I "$HERE/ref/win32" -I "$TMP" \
    -o "$OUT/bmp2texture.tmp" "$TMP/bmp2texture.cpp"
mv "$OUT/bmp2texture.tmp" "$OUT/bmp2texture"
echo "built $OUT/bmp2texture"

# The timed CPU baseline: the same sources with plain release flags
# (-O3 -DNDEBUG, the compiler's default contraction, no parity flags).  The
# GPU host that times it may be another CPU than this build machine, so
# instead of -march=native there is one build per ISA level and the timing
# code loads the one the host supports: x86-64-v4 (AVX-512) and x86-64-v3
# (AVX2 + FMA).
for LEVEL in v3 v4; do
    g++ -std=c++17 -O3 -DNDEBUG -march=x86-64-$LEVEL -fPIC -pthread -w -include "$HERE/ref/ref_shim.h" -I "$TMP" \
        -shared -o "$OUT/libslimref_timed_$LEVEL.so.tmp" "$HERE/ref/ref_driver.cpp"
    mv "$OUT/libslimref_timed_$LEVEL.so.tmp" "$OUT/libslimref_timed_$LEVEL.so"
    echo "built $OUT/libslimref_timed_$LEVEL.so"
done
