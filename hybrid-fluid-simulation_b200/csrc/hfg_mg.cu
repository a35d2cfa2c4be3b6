// hfg_mg.cu -- geometric multigrid preconditioner for the pressure CG.
#include "hfg_solver.h"

namespace hfg {

struct Multigrid {
  int dummy;
};

Multigrid* mgCreate(const Dim3i&, int, int, bool) {
  throw CudaError("multigrid preconditioner not available in this build", HFG_ERR_UNSUPPORTED);
}
void mgDestroy(Multigrid* m) { delete m; }
void mgSetup(Multigrid*, const Code*, float, float, float, cudaStream_t, long long&) {}
void mgRunCg(Multigrid*, const Dim3i&, float, float, float, const Code*, float*, float*, double*, CgState*,
             CgState*, cudaStream_t, long long&) {
  throw CudaError("multigrid preconditioner not available in this build", HFG_ERR_UNSUPPORTED);
}

}  // namespace hfg
