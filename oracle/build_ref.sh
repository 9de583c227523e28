#!/usr/bin/env bash
# Compile the reference's target-specific QBX module (pytential/qbx/target_specific:
# impl.pyx + helmholtz_utils.c) from its sources into oracle/_ref/, as a CPU checker
# for the 3D QBX near field.  Sources are read in place and never copied into the
# repository; outputs go only to oracle/_ref/ (git-ignored).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
# the reference checkout: $PYTENTIAL_REFERENCE, else a "reference" directory beside
# this repository
REF=${PYTENTIAL_REFERENCE:-"$(cd "$HERE/../.." && pwd)/reference"}
SRC="$REF/pytential/qbx/target_specific"
OUT="$HERE/_ref"
if [ ! -f "$SRC/impl.pyx" ]; then
  echo "reference sources not found at $SRC: oracle/_ref not built (set PYTENTIAL_REFERENCE)" >&2
  exit 0
fi
mkdir -p "$OUT/build"
PY=${PYTHON:-python3}
EXT=$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')
INC=$($PY -c 'import sysconfig; print(sysconfig.get_paths()["include"])')
cython -3 "$SRC/impl.pyx" -o "$OUT/build/impl.c"
/usr/bin/gcc -O2 -fopenmp -fPIC -shared -w -I"$INC" -I"$SRC" \
  "$OUT/build/impl.c" "$SRC/helmholtz_utils.c" -o "$OUT/impl$EXT" -lm
touch "$OUT/__init__.py"
echo "built $OUT/impl$EXT"
