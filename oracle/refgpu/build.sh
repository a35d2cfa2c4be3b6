#!/bin/bash
# Builds the reference's own grid step for sm_100a: its MPhysics CUDA/C++
# sources compiled unmodified where they lie in the reference checkout given
# as $1 (host .cpp files as CUDA, relocatable device code), against the
# stand-in headers of shim/ for the Windows, boost, assimp and D3D11 headers
# they name, plus stubs.cpp for the two mesh/CLD entry points that
# GridFluidSolver.cpp links against and driver.cu (the C ABI the tests and
# the bench's reference arm load).  Output: oracle/_ref/refgpu/libhfg_refgpu.so,
# or with "fp64" as $2 the reference's FP64 build (its own -DDOUBLE_REAL
# switch) as oracle/_ref/refgpu/libhfg_refgpu64.so.
# Test infrastructure only; nothing is copied out of the reference.
# Usage: oracle/refgpu/build.sh <reference root> [fp64]
set -euo pipefail
REF=${1:?usage: build.sh <reference root> [fp64]}
VARIANT=${2:-}
SRC="$REF/MPhysics"
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/../_ref/refgpu"
NVCC=${NVCC:-nvcc}
FLAGS=(-x cu -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -rdc=true -Xcompiler -fPIC -w
       -I"$HERE/shim" -I"$SRC")
if [ "$VARIANT" = fp64 ]; then
  OBJ="$OUT/obj64"
  LIB="$OUT/libhfg_refgpu64.so"
  FLAGS+=(-DDOUBLE_REAL)
else
  OBJ="$OUT/obj"
  LIB="$OUT/libhfg_refgpu.so"
fi
mkdir -p "$OBJ"
# the grid step and everything it links (GridFluidSolver.cpp names the four
# HybridSimulator / CLD kernels files at the end of the list)
UNITS=(EulerSolverTool.cu FieldMathTool.cu EulerParticlesTool.cu EulerMathTool.cu BoundaryTool.cu ThrustWapper.cu
       CudaContextManager.cpp CuDenseVector.cpp CuMatrixFreePCG.cpp SimulationConfigManager.cpp
       Grid.cpp Field.cpp ScalarGrid.cpp VectorGrid.cpp CellCenteredScalarGrid.cpp CellCenteredVectorGrid.cpp
       FaceCenteredVectorGrid.cpp ScalarField.cpp VectorField.cpp CellCenteredScalarField.cpp
       CellCenteredVectorField.cpp FaceCenteredVectorField.cpp
       EulerParticles.cpp AdvectionSolver.cpp SemiLagrangian.cpp ParticleInCell.cpp FluidImplicitParticle.cpp
       MixPICAndFLIP.cpp ExternalForcesSolver.cpp Boundary.cpp PressureSolver.cpp GridFluidSolver.cpp
       HybridSimulatorMixFieldWithDensity.cu HybridSimulatorSamplingSDFFromCLDGrid.cu HybridSimulatorBuildSDF.cu
       CLDGridInterpolate.cu)
JOBS=${JOBS:-$(nproc)}
compile() {  # source object
  local src=$1 obj=$2
  if [ ! -f "$obj" ] || [ "$src" -nt "$obj" ] || [ "$HERE/shim/windows.h" -nt "$obj" ]; then
    "$NVCC" "${FLAGS[@]}" -c "$src" -o "$obj"
  fi
}
export -f compile
export NVCC HERE
FLAGS_STR="${FLAGS[*]}"
export FLAGS_STR
{
  for u in "${UNITS[@]}"; do printf '%s\n%s\n' "$SRC/$u" "$OBJ/${u%.*}.o"; done
  printf '%s\n%s\n' "$HERE/stubs.cpp" "$OBJ/stubs.o" "$HERE/driver.cu" "$OBJ/driver.o"
} | xargs -d '\n' -n 2 -P "$JOBS" bash -c 'read -ra FLAGS <<< "$FLAGS_STR"; compile "$0" "$1"' \
  || { echo "reference build failed" >&2; exit 1; }
OBJS=()
for u in "${UNITS[@]}"; do OBJS+=("$OBJ/${u%.*}.o"); done
OBJS+=("$OBJ/stubs.o" "$OBJ/driver.o")
"$NVCC" -gencode arch=compute_100a,code=sm_100a -dlink -Xcompiler -fPIC "${OBJS[@]}" -o "$OBJ/dlink.o"
g++ -shared -o "$LIB" "${OBJS[@]}" "$OBJ/dlink.o" -L"${CUDA_HOME:-/usr/local/cuda}/lib64" \
    -lcudart -lcublas -lcusparse -Wl,--no-undefined
echo "built $LIB"
