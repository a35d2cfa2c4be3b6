// stubs.cpp -- definitions the reference's GridFluidSolver.cpp links against
// for mesh boundaries (generateSDF, BoundaryHelper.cpp) and cubic Lagrange
// discrete grids (CubicLagrangeDiscreteGrid.cpp).  Both need libraries that
// are not built here (assimp, D3D11), and the grid step with analytic SDF
// solids never calls them; each throws if it is reached.
#include "Common.h"
#include "BoundaryHelper.h"
#include "CubicLagrangeDiscreteGrid.h"

void generateSDF(string, CCellCenteredScalarField&, bool) {
  throw std::runtime_error("generateSDF: mesh voxelisation is not built (needs assimp and D3D11)");
}

thrust::device_vector<Real>& CCubicLagrangeDiscreteGrid::getField(UInt) {
  throw std::runtime_error("CCubicLagrangeDiscreteGrid is not built");
}

thrust::device_vector<UInt>& CCubicLagrangeDiscreteGrid::getCell() {
  throw std::runtime_error("CCubicLagrangeDiscreteGrid is not built");
}

SCLDGridInfo CCubicLagrangeDiscreteGrid::getCLDGridInfo() const {
  throw std::runtime_error("CCubicLagrangeDiscreteGrid is not built");
}
