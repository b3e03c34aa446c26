// Mixed-precision PMG: FP32 V-cycles inside an FP64 refinement loop.
#pragma once

struct pmgb_solver;

namespace pmgb {
struct MixedState;
// Solve the problem held by s (LPBE or NPBE) in mixed precision.  Leaves the
// FP64 solution in s->lev[0].x (Dirichlet values not yet restored).
int mixed_solve(pmgb_solver* s, double errtol, int itmax);
void mixed_destroy(MixedState* m);
void mixed_mark_stale(MixedState* m);
// Inner linear solve of one Newton step in mixed precision.
int mixed_newton_inner(pmgb_solver* s, double errtol_s);
// Damped inexact Newton driver (solver.cu); mixed selects the inner solver.
int newton_driver(pmgb_solver* s, double errtol, int itmax, int mixed);
void set_error(const char* fmt, ...);
int mixed_time_gs7(pmgb_solver* s, int parity, double* bytes);
int mixed_prepare_sweep(pmgb_solver* s);
int mixed_time_gs7_sweep(pmgb_solver* s, double* bytes);
int mixed_time_tail(pmgb_solver* s, double* bytes);
// FP64 path, LPBE: exact-to-round-off solve of the FP64 coarsest level
// (FP64 refinement over FP32 V-cycles of extra Galerkin levels).
int coarse_exact_prepare(pmgb_solver* s);
// operator build of solver.cu (Galerkin hierarchy, coarsest factor)
int solver_build(pmgb_solver* s);
int launch_coarse_exact(pmgb_solver* s, cudaStream_t st, const double* cc, const double* b,
                        double* x);
}  // namespace pmgb
