/*
 * pmg_oracle.h -- CPU restatement of the APBS PMG solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  Written for this project from the reference's
 * algorithm (file:line citations in pmg_oracle.c); pinned against the
 * reference sources compiled unchanged (oracle/_ref) by the test suite.
 * Only tests/, the smoke check and the CPU-baseline leg of the benchmark
 * load it; the CUDA library never does.
 */
#ifndef PMG_ORACLE_H
#define PMG_ORACLE_H

#include "pmgb_params.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Same contract as ref_pmg_run in oracle/ref_driver.c:
 *   u (N), maps (5N: charge, epsx, epsy, epsz, kappa),
 *   faces (2*(ny*nz + nx*nz + nx*ny)), out[16], reslog[reslog_cap].
 * out: [0] energy kT [1] progress messages [2] reslog entries [3..6] phase
 *      seconds (ctor, fillco, solve, energy) [7] qf [8] diel [9] qm
 *      [10] outer V-cycles (LPBE) or Newton iterations (NPBE)
 *      [11] total V-cycles.
 * Returns 1 on success, 0 on failure. */
int oracle_pmg_run(const pmgb_params *p, int natoms, const double *xyz,
                   const double *q, const double *r, double *u, double *maps,
                   double *faces, double *out, double *reslog, int reslog_cap,
                   int verbose);

/* Two-level focusing chain, as initMG builds it for an ELEC block with
 * bcfl focus after a solved one (routines.c:1458-1475): the coarse
 * calculation pc (bcfl zero/sdh) is solved, the fine one pf (bcfl focus)
 * takes its faces from the coarse potential (focusFillBound) and the energy
 * outside its domain from the coarse solution (extEnergy), then is solved.
 * u, faces: the fine calculation's; out as above for the fine calculation
 * (energies include the external terms) plus [12..14] extQf, extDiel,
 * extQm and [15] the coarse energy; [1], [2] and reslog cover both solves. */
int oracle_pmg_focus(const pmgb_params *pc, const pmgb_params *pf, int natoms,
                     const double *xyz, const double *q, const double *r,
                     double *u, double *faces, double *out, double *reslog,
                     int reslog_cap, int verbose);

/* Coefficient fill only (Vpmg_fillco): maps and faces as above. */
int oracle_pmg_fill(const pmgb_params *p, int natoms, const double *xyz,
                    const double *q, const double *r, double *maps,
                    double *faces);

#ifdef __cplusplus
}
#endif

#endif /* PMG_ORACLE_H */
