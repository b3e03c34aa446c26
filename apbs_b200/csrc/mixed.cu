// Mixed-precision PMG (placeholder until the FP32 hierarchy lands).
#include "mixed.cuh"
#include "solver_internal.cuh"

namespace pmgb {
struct MixedState {
  int unused;
};
int mixed_solve(pmgb_solver* s, double errtol) {
  (void)s;
  (void)errtol;
  set_error("mixed precision path not built yet");
  return 0;
}
void mixed_destroy(MixedState* m) { delete m; }
}  // namespace pmgb
