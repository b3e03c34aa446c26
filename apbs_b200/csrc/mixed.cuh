// Mixed-precision PMG: FP32 V-cycles inside an FP64 refinement loop.
#pragma once

struct pmgb_solver;

namespace pmgb {
struct MixedState;
// Solve the problem held by s (LPBE or NPBE) in mixed precision.  Leaves the
// FP64 solution in s->lev[0].x (Dirichlet values not yet restored).
int mixed_solve(pmgb_solver* s, double errtol);
void mixed_destroy(MixedState* m);
}  // namespace pmgb
