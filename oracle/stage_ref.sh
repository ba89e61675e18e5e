#!/usr/bin/env bash
# Stage the reference's shipped kgwas, kgwas_2d and build_index binaries into oracle/_ref/ so that it can
# be RUN as a black box (CPU baseline and golden-vector generation).  The
# reference cannot be rebuilt from source here: src/kgwas.cpp includes
# <Eigen/Dense> and links OpenBLAS, neither of which is installed.  The binary
# is only executed, never inspected.  oracle/_ref/ is git-ignored.
#
# Its OpenBLAS dependency is satisfied with the OpenBLAS build that ships in
# the Python environment's opencv wheel (symlinked as libopenblas.so.0).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:?usage: stage_ref.sh REFERENCE_DIR (the reference checkout holding bin/kgwas)}"
OUT="$HERE/_ref"
if [[ ! -x "$REF/bin/kgwas" ]]; then
  echo "reference binary not found at $REF/bin/kgwas" >&2
  exit 1
fi
mkdir -p "$OUT"
cp -f "$REF/bin/kgwas" "$OUT/kgwas"
# the 2-D pair test and the index builder that produces its input
for b in kgwas_2d build_index; do
  [[ -x "$REF/bin/$b" ]] && cp -f "$REF/bin/$b" "$OUT/$b"
done
PY="$(command -v python3)"
LIBS="$("$PY" -c 'import os,glob,sys; d=[p for p in sys.path if p.endswith("site-packages")]; g=[x for s in d for x in glob.glob(os.path.join(s,"opencv_python_headless.libs"))]; print(g[0] if g else "")')"
if [[ -n "$LIBS" ]]; then
  BLAS="$(ls "$LIBS"/libopenblas*.so 2>/dev/null | head -1 || true)"
  [[ -n "$BLAS" ]] && ln -sf "$BLAS" "$OUT/libopenblas.so.0"
  echo "$LIBS" > "$OUT/libdirs.txt"
fi
echo "staged $OUT/kgwas"
