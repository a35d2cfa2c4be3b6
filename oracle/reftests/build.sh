#!/bin/bash
# Compiles the reference's own unit-test sources, read in place from the
# reference checkout given as $1, against shim/refapi.h (the reference's API
# restated over the CPU oracle), one binary per suite into
# oracle/_ref/reftests/.  With "planted" as $2 the oracle is first rebuilt
# with ORC_PLANTED_MISTAKE (a deliberate error in the linear transfer kernel
# and in trilinear sampling) and the suites go to oracle/_ref/reftests_planted/,
# to show that the replay catches an error.  Test infrastructure only.
# Usage: oracle/reftests/build.sh <reference root> [planted]
set -euo pipefail
REF=${1:?usage: build.sh <reference root> [planted]}
MODE=${2:-}
HERE=$(cd "$(dirname "$0")" && pwd)
ORACLE=$(cd "$HERE/.." && pwd)
CXX=${CXX:-g++}
GOMP=""
[ -f /usr/lib/gcc/x86_64-linux-gnu/13/libgomp.spec ] && GOMP="-B/usr/lib/gcc/x86_64-linux-gnu/13/"
if [ "$MODE" = planted ]; then
  LIBDIR="$ORACLE/_ref/planted"
  OUT="$ORACLE/_ref/reftests_planted"
  mkdir -p "$LIBDIR"
  "$CXX" -O2 -std=c++17 -fPIC -fopenmp -ffp-contract=off -w $GOMP -DORC_PLANTED_MISTAKE -shared \
      -o "$LIBDIR/libhfg_oracle.so" "$ORACLE/hfg_oracle.cpp"
else
  LIBDIR="$ORACLE/_build"
  OUT="$ORACLE/_ref/reftests"
  make -s -C "$ORACLE"
fi
mkdir -p "$OUT"
# suite name -> test source under TestCase/MPhysics
declare -A SUITES=(
  [ParticlesAdvection]="Euler/UnitTest-ParticlesAdvection/UnitTest-ParticlesAdvection.cu"
  [SemiLagrangian]="Euler/UnitTest-SemiLagrangian/UnitTest-SemiLagrangian.cu"
  [BoundarySDF]="Euler/UnitTest-BoundarySDF/UnitTest-BoundarySDF.cu"
  [ExternalForces]="Euler/UnitTest-ExternalForces/UnitTest-ExternalForces.cu"
  [Extrapolation]="Euler/UnitTest-Extrapolation/UnitTest-Extrapolation.cu"
  [PressureSolver]="Euler/UnitTest-PressureSolver/UnitTest-PressureSolver.cu"
  [HybridHelper]="Hybrid/UnitTest-HybridHelper/UnitTest-HybridHelper.cu"
  [GridFluidSolver]="Euler/IntegrationTest-GridFluidSolver/IntegrationTest-GridFluidSolver.cpp"
  [CellCenteredScalarField]="DataStructure/UnitTest-ScalarGrid/UnitTest-CellCenteredScalarField.cu"
  [CellCenteredVectorField]="DataStructure/UnitTest-CellCenteredVectorGrid/UnitTest-CellCenteredVectorField.cu"
  [FaceCenteredVectorField]="DataStructure/UnitTest-FaceCenteredVectorGrid/UnitTest-FaceCenteredVectorField.cu"
)
# main.cpp once, then each suite; the suites build in parallel
(cd "$HERE" && "$CXX" -std=c++17 -O1 -w -c main.cpp -o "$OUT/main.o")
pids=()
for s in "${!SUITES[@]}"; do
  src="$REF/TestCase/MPhysics/${SUITES[$s]}"
  # The source is read from stdin so that its own directory (with the
  # reference's pch.h) is not searched before shim/ for quoted includes.
  (cd "$HERE/shim" && "$CXX" -std=c++17 -O1 -w $GOMP -x c++ -I. - -x none "$OUT/main.o" \
      -L"$LIBDIR" -Wl,-rpath,"$LIBDIR" -lhfg_oracle -fopenmp -o "$OUT/$s" < "$src") &
  pids+=($!)
done
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
[ $rc -eq 0 ] || { echo "build failed" >&2; exit 1; }
echo "built ${#SUITES[@]} suites into $OUT"
