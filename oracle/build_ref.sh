#!/usr/bin/env bash
# Build the reference's own simulated-annealing, steepest-descent and SQA
# (rotor and path-integral) extensions from their sources, for use as test
# oracles and as the timed CPU baseline.  Test infrastructure only.
#
# Sources (read in place, never copied into the repository):
#   <ref>/dwave/samplers/sa/simulated_annealing.pyx   (Cython binding)
#   <ref>/dwave/samplers/sa/src/cpu_sa.cpp, cpu_sa.h   (C++ core)
# Flags follow the reference's meson.build:4-12,22 (C++17, -O3, release
# => -DNDEBUG, -g1; no -march, no fast-math).
#
# Output: oracle/_ref/simulated_annealing<EXT_SUFFIX> (git-ignored; it travels
# with the working tree to machines that do not have the reference sources).
set -euo pipefail

# The reference checkout: the first argument, else $B200SA_REFERENCE_DIR,
# else the checkout mounted beside the repository on the build machine.
REF="${1:-${B200SA_REFERENCE_DIR:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
SA="$REF/dwave/samplers/sa"

if [ ! -f "$SA/simulated_annealing.pyx" ]; then
    echo "reference sources not found under $REF; skipping" >&2
    exit 0
fi

mkdir -p "$OUT"
PY="${PYTHON:-python}"
EXT_SUFFIX="$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')"
PYINC="$($PY -c 'import sysconfig; print(sysconfig.get_paths()["include"])')"
NPINC="$($PY -c 'import numpy; print(numpy.get_include())')"

# Cython writes the generated C++ next to the requested output path.
$PY -m cython --cplus -3 -Xfreethreading_compatible=True \
    -o "$OUT/simulated_annealing.cpp" "$SA/simulated_annealing.pyx"

g++ -O3 -std=c++17 -g1 -DNDEBUG -fPIC -shared -Wall -Wno-unused-function \
    -I"$SA/src" -I"$PYINC" -I"$NPINC" \
    "$OUT/simulated_annealing.cpp" "$SA/src/cpu_sa.cpp" \
    -o "$OUT/simulated_annealing$EXT_SUFFIX"

rm -f "$OUT/simulated_annealing.cpp"
echo "built $OUT/simulated_annealing$EXT_SUFFIX"

# The reference's steepest-descent extension (the step after annealing):
#   <ref>/dwave/samplers/greedy/descent.pyx, decl.pxd   (Cython binding)
#   <ref>/dwave/samplers/greedy/src/descent.cpp, descent.h (C++ core)
GR="$REF/dwave/samplers/greedy"
if [ -f "$GR/descent.pyx" ]; then
    $PY -m cython --cplus -3 -Xfreethreading_compatible=True -I "$REF" \
        -o "$OUT/descent.cpp" "$GR/descent.pyx"
    g++ -O3 -std=c++17 -g1 -DNDEBUG -fPIC -shared -Wall -Wno-unused-function \
        -I"$GR/src" -I"$PYINC" -I"$NPINC" \
        "$OUT/descent.cpp" "$GR/src/descent.cpp" \
        -o "$OUT/descent$EXT_SUFFIX"
    rm -f "$OUT/descent.cpp"
    echo "built $OUT/descent$EXT_SUFFIX"
fi

# The reference's rotor-model annealing extension (SQA):
#   <ref>/dwave/samplers/sqa/rotormc_annealing.pyx, src/cpu_rotormc.cpp, .h
SQ="$REF/dwave/samplers/sqa"
if [ -f "$SQ/rotormc_annealing.pyx" ]; then
    $PY -m cython --cplus -3 -Xfreethreading_compatible=True -I "$REF" \
        -o "$OUT/rotormc_annealing.cpp" "$SQ/rotormc_annealing.pyx"
    g++ -O3 -std=c++17 -g1 -DNDEBUG -fPIC -shared -Wall -Wno-unused-function \
        -I"$SQ/src" -I"$PYINC" -I"$NPINC" \
        "$OUT/rotormc_annealing.cpp" "$SQ/src/cpu_rotormc.cpp" \
        -o "$OUT/rotormc_annealing$EXT_SUFFIX"
    rm -f "$OUT/rotormc_annealing.cpp"
    echo "built $OUT/rotormc_annealing$EXT_SUFFIX"
fi

# The reference's path-integral Monte Carlo extension (SQA):
#   <ref>/dwave/samplers/sqa/pimc_annealing.pyx, src/localPIMC.cpp, .h
if [ -f "$SQ/pimc_annealing.pyx" ]; then
    $PY -m cython --cplus -3 -Xfreethreading_compatible=True -I "$REF" \
        -o "$OUT/pimc_annealing.cpp" "$SQ/pimc_annealing.pyx"
    g++ -O3 -std=c++17 -g1 -DNDEBUG -fPIC -shared -Wall -Wno-unused-function \
        -Wno-sign-compare -I"$SQ/src" -I"$PYINC" -I"$NPINC" \
        "$OUT/pimc_annealing.cpp" "$SQ/src/localPIMC.cpp" \
        -o "$OUT/pimc_annealing$EXT_SUFFIX"
    rm -f "$OUT/pimc_annealing.cpp"
    echo "built $OUT/pimc_annealing$EXT_SUFFIX"
fi
