/*
 * apbs_b200.h -- C ABI of the B200-native PMG Poisson-Boltzmann solver.
 *
 * Plain C: opaque handles, plain pointers and sizes, no C++ or torch types.
 * Each entry point replaces one step of the reference's Vpmg C API for an
 * mg-manual calculation (APBS 3.4.1, src/mg/vpmg.h):
 *
 *   pmgb_create         <- Vpmg_ctor / Vpmg_ctor2   (vpmg.h:226, 242;
 *                                                  vpmg.c:141-399)
 *   pmgb_fillco         <- Vpmg_fillco             (vpmg.h:281; vpmg.c:5250)
 *   pmgb_set_coefficients  the arrays Vpmg_fillco leaves in struct sVpmg
 *                          (charge, epsx/y/z, kappa, gxcf/gycf/gzcf,
 *                          vpmg.h:116-193) for callers that fill on the host
 *   pmgb_solve          <- Vpmg_solve              (vpmg.h:306; vpmg.c:401)
 *   pmgb_energy         <- Vpmg_energy             (vpmg.h:334; vpmg.c:1248)
 *   pmgb_get_potential  <- reading thee->u after Vpmg_solve
 *   pmgb_destroy        <- Vpmg_dtor               (vpmg.h:260)
 *
 * Return convention follows Vpmg: 1 = success, 0 = failure; on failure
 * pmgb_last_error() describes the cause.  The library never aborts the
 * process and never falls back to a CPU path: without a usable CUDA device
 * every entry point fails.
 *
 * Grid arrays are x-fastest, index (k*ny + j)*nx + i (IJK, vpmg.h:1383).
 * Boundary faces use the reference layout: gxcf[s][k][j], gycf[s][k][i],
 * gzcf[s][j][i], s = 0 (low face) or 1 (high face) (IJKx/IJKy/IJKz,
 * vpmg.h:1384-1386).
 */
#ifndef APBS_B200_H
#define APBS_B200_H

#include <stddef.h>

#include "pmgb_params.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PMGB_FP64 0   /* plain FP64 PMG, drop-in for Vpmg_solve */
#define PMGB_MIXED 1  /* FP32 V-cycles inside FP64 iterative refinement */

typedef struct pmgb_solver pmgb_solver;

typedef struct pmgb_stats {
    int vcycles;          /* V-cycles executed (all Newton steps included) */
    int newton_iters;     /* Newton iterations (NPBE), 0 for LPBE */
    int refinements;      /* outer refinement steps (PMGB_MIXED) */
    int coarse_method;    /* coarsest solve: 0 conjugate gradients, 1 band Cholesky,
                             2 dense inverse (mixed), 3 exact refinement (FP64, large) */
    double rel_residual;  /* final relative residual of the stopping test */
    double t_fill_ms;     /* coefficient fill, device time */
    double t_setup_ms;    /* operator build + Galerkin + coarse factor */
    double t_solve_ms;    /* iterations */
    double t_energy_ms;
    double energy_kT;     /* last pmgb_energy result */
    double qf, diel, qm;  /* energy components (kT) */
    int sas_points;       /* accessible surface points used by the fill */
    int status;           /* 0 ok, nonzero: last device-side status code */
    double ext_qf, ext_diel, ext_qm; /* energies outside the domain (focusing) */
    int converged;        /* 1 if the last solve met its tolerance; 0 if it stopped at
                             itmax (pmgb_params.itmax), which -- as Vpmg_solve --
                             still returns success */
} pmgb_stats;

/* Vpmg_ctor: allocate device state for one calculation on the current CUDA
 * device.  precision: PMGB_FP64 or PMGB_MIXED. */
int pmgb_create(const pmgb_params *params, int precision, pmgb_solver **out);

/* Run all device work of this calculation on the given CUDA stream
 * (a cudaStream_t passed as void*; NULL restores the solver's own stream).
 * The caller keeps ownership of the stream. */
int pmgb_set_stream(pmgb_solver *s, void *cuda_stream);

/* Vpmg_fillco: spl2 charge, molecular (mol/smol) dielectric, ion
 * accessibility and sdh/zero boundary values, computed on the device from
 * host atom arrays: xyz[3*natoms] (Angstrom), charge[natoms] (e),
 * radius[natoms] (Angstrom). */
int pmgb_fillco(pmgb_solver *s, int natoms, const double *xyz, const double *charge,
                const double *radius);

/* Same, with the atom arrays already in device memory. */
int pmgb_fillco_device(pmgb_solver *s, int natoms, const double *d_xyz,
                       const double *d_charge, const double *d_radius);

/* Focusing: Vpmg_ctor with focusFlag = 1 and pmgOLD = coarse (vpmg.h:226;
 * vpmg.c:225-262).  Fills the Dirichlet faces of `fine` by trilinear
 * interpolation of the solved coarse potential (focusFillBound,
 * vpmg.c:1914-2414) and, when calc_energy is nonzero (energyFlag != PCE_NO),
 * the energy of the coarse solution outside the fine domain, kept for the
 * fine pmgb_energy (extEnergy, vpmg.c:2416-2545).  `fine` must have been
 * created with bcfl PMGB_BCFL_FOCUS and be filled afterwards with
 * pmgb_fillco (which then leaves the faces alone, vpmg.c:5404-5409); the
 * fine domain must lie inside the coarse one (the reference asserts).  Both
 * solvers must be on the current device.  The coarse solver is not
 * destroyed (the reference's Vpmg_ctor2 destroys pmgOLD; call
 * pmgb_destroy when done).  Work is ordered after the coarse solver's
 * stream and issued on the fine solver's stream. */
int pmgb_focus(pmgb_solver *fine, pmgb_solver *coarse, int calc_energy);

/* Load coefficient maps produced elsewhere (host arrays of N = nx*ny*nz
 * doubles; faces as in the header comment).  The atom list is needed only
 * for the sdh boundary, which is given here, so this replaces the fill. */
int pmgb_set_coefficients(pmgb_solver *s, const double *charge, const double *epsx,
                          const double *epsy, const double *epsz, const double *kappa,
                          const double *gxcf, const double *gycf, const double *gzcf);

/* Vpmg_solve: build the operators and solve (LPBE: linear PMG; NPBE:
 * damped inexact Newton).  The potential stays on the device.  As in the
 * reference, reaching the iteration limit (pmgb_params.itmax) without
 * meeting the tolerance is not a failure: the call returns 1 with the last
 * iterate and pmgb_stats.converged = 0.  A non-finite residual, a device
 * error or a device wait that ran out returns 0. */
int pmgb_solve(pmgb_solver *s);

/* Vpmg_energy(extFlag = 1) of a non-focused calculation, in kT. */
int pmgb_energy(pmgb_solver *s, double *energy_kT);

/* Forces on every atom of the last fill, from the last solve, in kT/A
 * (arrays of 3 doubles per atom; any may be NULL):
 *   qf  charge-field force, Vpmg_qfForce (src/mg/vpmg.c:5862-6154), for
 *       chgm spl2 or spl0;
 *   db  dielectric boundary force, Vpmg_dbForce (vpmg.c:5605-5860);
 *   ib  ionic boundary force, Vpmg_ibForce (vpmg.c:5440-5603);
 * db and ib need srfm spl2 (the reference's rule: forces need spline-based
 * surfaces).  Atoms outside the domain get zero, as in the reference; an
 * atom whose dielectric-boundary window crosses the grid edge fails the call
 * (the reference's Vpmg_dbForce returns 0 for it).  One call replaces the
 * per-atom Vpmg_force loop of forceMG (src/routines.c). */
int pmgb_forces(pmgb_solver *s, double *qf, double *db, double *ib);

/* Testing hook for the failure path of the plane-parallel GS27 wavefront:
 * shifts the step counter of one plane of one level, so that the next solve
 * has its neighbours' bounded waits run out (no device fault).  That solve
 * fails with an error naming the waits and restarts the counters; the one
 * after it runs normally.  No reference counterpart. */
int pmgb_debug_shift_wave_counter(pmgb_solver *s, int level, int plane, int delta);

/* OpenDX output, byte for byte the file writedataMG writes through
 * Vgrid_writeDX (src/routines.c:2620-2920, src/mg/vgrid.c:1206-1420):
 * pmgb_write_dx writes one map of a calculation with its partition weights
 * (which = PMGB_DX_*; title NULL = the reference's title for that map;
 * package NULL = "APBS 3.4.1" for the "# Data from" line);
 * pmgb_write_dx_host writes a caller's host array (pvec NULL = every
 * point).  The values are formatted by several host threads. */
#define PMGB_DX_POT 0     /* u (kT/e) */
#define PMGB_DX_CHARGE 1  /* charge / zmagic (e) */
#define PMGB_DX_KAPPA 2
#define PMGB_DX_DIELX 3
#define PMGB_DX_DIELY 4
#define PMGB_DX_DIELZ 5
int pmgb_write_dx(pmgb_solver *s, int which, const char *path, const char *title,
                  const char *package);
int pmgb_write_dx_host(const char *path, int nx, int ny, int nz, double hx, double hy,
                       double hz, double xmin, double ymin, double zmin, const double *data,
                       const double *pvec, const char *title, const char *package);

/* OpenDX reader (Vgrid_readDX, src/mg/vgrid.c:586-790): counts, spacings
 * and origin of the file's grid, and with data non-NULL its values in the
 * x-fastest IJK layout (nx*ny*nz doubles). */
int pmgb_read_dx_host(const char *path, int *dims, double *h, double *origin, double *data);

/* Maps given on their own grids, as the deck's "usemap" (Vpmg_fillco's
 * dielXMap..chargeMap arguments, src/mg/vpmg.c:5250-5316): from the next
 * pmgb_fillco the dielectric and kappa maps replace the surface
 * (fillcoCoefMap, vpmg.c:4098-4221; all three dielectric maps are needed,
 * and the kappa map when there are ions), the charge map replaces the atom
 * charges (fillcoChargeMap, 4938-4984, and the energy then integrates the
 * charge map as Vpmg_qfEnergyVolume does).  Values are interpolated as
 * Vgrid_value does.  data (host, IJK) is copied; NULL stops using the map. */
#define PMGB_MAP_DIELX 0
#define PMGB_MAP_DIELY 1
#define PMGB_MAP_DIELZ 2
#define PMGB_MAP_KAPPA 3
#define PMGB_MAP_CHARGE 4
#define PMGB_MAP_POT 5    /* boundary values of bcfl map (bcfl_map + focusFillBound,
                             vpmg.c:3953-3993, 1914-2414) */
#define PMGB_MAP_COUNT 6
int pmgb_set_map(pmgb_solver *s, int which, int nx, int ny, int nz, double hx, double hy,
                 double hz, double xmin, double ymin, double zmin, const double *data);

/* Copy the potential (thee->u, Dirichlet values restored) to host memory. */
int pmgb_get_potential(pmgb_solver *s, double *u);

/* Copy the coefficient maps and faces to host memory (any pointer may be
 * NULL): maps = charge, epsx, epsy, epsz, kappa (5*N doubles). */
int pmgb_get_maps(pmgb_solver *s, double *maps, double *faces);

int pmgb_get_stats(pmgb_solver *s, pmgb_stats *stats);

/* Relative-residual history of the last solve (one entry per stopping
 * test, as the reference's Vprtstp reports it).  Returns the count. */
int pmgb_get_residual_history(pmgb_solver *s, double *buf, int cap);

void pmgb_destroy(pmgb_solver *s);

/* One call from host buffers to energy: create + fillco + solve + energy
 * (+ optional potential copy) + destroy. */
int pmgb_solve_molecule(const pmgb_params *params, int precision, int natoms,
                        const double *xyz, const double *charge, const double *radius,
                        double *energy_kT, double *u_or_null, pmgb_stats *stats_or_null);

/* Kernels that pmgb_time_kernel can time in isolation. */
#define PMGB_K_GS7_FP64 0    /* fine-level 7-point GS, one colour (half-sweep) */
#define PMGB_K_GS27_WAVE 1   /* level-2 ordered 27-point GS, 2 sweeps + residual */
#define PMGB_K_RESID_FP64 2  /* fine-level 7-point residual */
#define PMGB_K_GS7_FP32 3    /* fine-level FP32 7-point GS half-sweep (mixed) */
#define PMGB_K_CG_COARSE 4   /* coarsest-level CG (NPBE), up to 100 iterations */
/* 5 and 6 are not used */
#define PMGB_K_VCYCLE_TAIL 7    /* mixed: coarse-level V-cycle tail (one cluster kernel) */
#define PMGB_K_GS7_SWEEP_FP64 8 /* fine-level 7-point GS, one full sweep in one pass, FP64 */
#define PMGB_K_GS7_SWEEP_FP32 9 /* the same, FP32 (mixed) */

/* Launch-shape tunables.  pmgb_set_tuning sets the process-wide defaults a
 * calculation copies when it is created; pmgb_solver_set_tuning changes one
 * calculation (its captured V-cycle graphs are rebuilt on the next solve).
 * The autotuner (apbs_b200/autotune.py) times whole solves per grid shape
 * and keeps the best values in a table.  No key changes a result beyond
 * round-off; the FP64 smoother and wavefront keys change none at all. */
#define PMGB_TUNE_MIXED_CHEBYSHEV 0   /* mixed: smoothing of the 27-point FP32 levels, 0 = the
                                          8-colour Gauss-Seidel (PMGB_TUNE_MIXED_COARSE_SWEEPS
                                          sweeps), K > 0 = Jacobi-preconditioned Chebyshev of
                                          degree K (rounded up to even) */
#define PMGB_TUNE_GS27_LAG 1          /* plane-parallel GS27: wavefronts between successive
                                          half-sweeps (>= 4, default 6); a larger lag lets a
                                          plane run ahead of the plane above it */
/* key 3 is not used */
#define PMGB_TUNE_GS27_CLUSTER 2       /* CTAs per cluster of the ordered GS27 on levels with
                                          >= 60 interior points per axis (0 = device max) */
#define PMGB_TUNE_BAND_ALWAYS 4        /* 1: FP64 LPBE coarsest level always by the banded
                                          Cholesky of the reference, 0: exact refinement
                                          above 512 unknowns */
#define PMGB_TUNE_GS7_COLOUR_PASSES 5  /* fine smoother: 0 = default (FP64 single-pass sweep
                                          kernel, FP32 one launch per colour), 1 = one launch
                                          per colour, 2 = single-pass sweeps in FP32 too */
#define PMGB_TUNE_GS7_SWEEP_KCHUNK 6   /* planes per CTA of the single-pass sweep; 0 (default)
                                          = as many chunks as fill the resident CTA slots */
#define PMGB_TUNE_GS27_CLUSTER_MID 7   /* the same as key 2 for levels with 28-59 interior
                                          points per axis (0 = 8) */
#define PMGB_TUNE_TAIL_MAX_POINTS 8    /* mixed: largest level (interior points) run inside
                                          the one-cluster V-cycle tail (default 70000) */
#define PMGB_TUNE_MC_COOPERATIVE 9    /* mixed: 8-colour GS on levels above 200000 interior
                                          points as one cooperative launch per smoothing call
                                          (1) instead of one launch per colour (0) */
#define PMGB_TUNE_MIXED_COARSE_SWEEPS 10 /* mixed: 8-colour GS sweeps before and after each
                                            coarse correction on 27-point levels (default 2) */
#define PMGB_TUNE_MIXED_FINE_SWEEPS 11 /* mixed: red-black sweeps on the fine level (default 2) */
#define PMGB_TUNE_GS7_SWEEP_SHAPE 12 /* single-pass sweep launch shape: bits 0-3 threads per
                                          CTA (0 = 256, 1 = 512, 2 = 1024), bits 4-7 pair
                                          slots per thread (1-4, 0 = 2); a CTA owns a flat range
                                          of 2 x (slots - nx - 3) points of each plane;
                                          default 0x12: 1024 threads, 1 slot */
#define PMGB_TUNE_GS27_PLANES 13      /* ordered GS27: 0 (default) = one CTA per plane
                                          holding its plane and both neighbours in shared
                                          memory, updates passed through a mailbox, on
                                          levels where three planes fit (else as 2);
                                          2 = one CTA per plane synchronised with its
                                          neighbour planes by step counters on every level
                                          whose planes fit on the device; 1 = one cluster
                                          with a barrier per wavefront everywhere */
#define PMGB_TUNE_CG_CLUSTER 14       /* coarsest-level CG of the FP64 NPBE path: CTAs per
                                          cluster of the slab kernel (0 = smallest that fits;
                                          4, 8 or 16); 1 = the strided cluster kernel that
                                          levels too large for slabs use */
#define PMGB_TUNE_GS27_PLANES_POLL 15 /* plane-parallel GS27: 0 = one thread of a CTA waits
                                          for the neighbour planes, then a block barrier;
                                          1 = every thread waits itself */
#define PMGB_TUNE_NKEYS 16
int pmgb_set_tuning(int key, int value);
int pmgb_get_tuning(int key);
int pmgb_solver_set_tuning(pmgb_solver *s, int key, int value);
int pmgb_solver_get_tuning(pmgb_solver *s, int key);

/* Launch one kernel `reps` times back to back on the solver's stream (after
 * a solve, on its state) and report the mean device time per launch (CUDA
 * events) and the algorithmic bytes one launch must move. */
int pmgb_time_kernel(pmgb_solver *s, int which, int reps, double *ms_per_launch,
                     double *bytes_per_launch);

/* Largest grid dimension pmgb_energy_noalloc accepts (points per axis). */
#define PMGB_NOALLOC_MAX_DIM 1025

/* Energy of a solved potential (as pmgb_energy) computed from device arrays
 * the caller already holds, without allocating any device memory.  It has
 * no counterpart in the reference; it serves callers that cannot allocate
 * at this point -- code inside another framework's memory pool, whose
 * device memory belongs to that pool and where cudaMalloc would synchronise
 * the device, and fixed-footprint embedded callers.  d_u is the potential
 * with its boundary values, the maps are those of the fill (N = nx*ny*nz
 * doubles; the dielectric and kappa maps may be NULL for LPBE).  Grids up
 * to PMGB_NOALLOC_MAX_DIM points per axis and 0..PMGB_MAXION ion species;
 * anything else is rejected before any device work.  The scratch is one
 * fixed 64 KiB device array per device, shared by every call: the first
 * call on a device looks its address up (make that call before any stream
 * capture on that device), and calls that overlap on the GPU race on it.
 * cuda_stream may be NULL (default stream); the call copies the partition
 * weights from host memory and waits for its result on that stream. */
int pmgb_energy_noalloc(const pmgb_params *params, const double *d_u, const double *d_charge,
                        const double *d_epsx, const double *d_epsy, const double *d_epsz,
                        const double *d_kappa, void *cuda_stream, double *energy_kT);

/* Solve many filled mixed-precision LPBE calculations (each from
 * pmgb_create(..., PMGB_MIXED) + pmgb_fillco) in one persistent kernel:
 * one thread-block cluster per calculation runs its whole refinement loop on
 * the device, so calculations of uneven grid sizes share one launch.  Each
 * calculation's level 1 must fit the one-cluster tail (fine grids up to 65^3
 * with the default tail limit).  Afterwards each calculation is solved as by
 * pmgb_solve (pmgb_energy, pmgb_get_potential, pmgb_get_stats).  Work runs on
 * cuda_stream (NULL: the first calculation's stream).  No counterpart in the
 * reference, which solves its calculations one after another. */
int pmgb_batch_solve(pmgb_solver *const *solvers, int n, void *cuda_stream);

/* Reuse a calculation for another one on the same grid (nx, ny, nz, nlev):
 * new centre, spacing, physics and boundary kind; the device arrays stay
 * allocated.  It has no counterpart in the reference (which builds a new
 * Vpmg per ELEC block); it lets a serving loop keep grids resident. */
int pmgb_reconfigure(pmgb_solver *s, const pmgb_params *params);

/* Device bytes a calculation of this shape holds once filled and solved
 * with natoms atoms (used for admission by HBM footprint). */
size_t pmgb_footprint(const pmgb_params *params, int precision, int natoms);

/* ------------------------------------------------------------------------
 * Serving loop: many independent calculations on one GPU.
 *
 * A native request loop with no counterpart in the reference (whose main
 * loop runs ELEC blocks one after another, src/main.c:529).  Requests are
 * queued in arrival order; `max_inflight` worker threads, each with its own
 * CUDA stream, take the head of the queue as soon as a worker is free and
 * the request's device footprint fits the budget next to the calculations
 * already resident, so requests that arrive while others run are admitted
 * as slots and memory free up and their work overlaps on the device.
 * Finished calculations stay resident in a pool keyed by grid shape and are
 * reused (pmgb_reconfigure) by later requests of that shape; idle ones are
 * released, oldest first, when a new request needs their memory.
 * ------------------------------------------------------------------------ */
typedef struct pmgb_server pmgb_server;

typedef struct pmgb_server_config {
    int precision;            /* PMGB_FP64 or PMGB_MIXED */
    int max_inflight;         /* worker slots (concurrent calculations), >= 1 */
    size_t hbm_budget_bytes;  /* admission limit; 0 = 80% of the device's free memory */
    int pool_per_shape;       /* idle calculations kept per grid shape:
                                 0 = max(2, max_inflight) * max_batch, < 0 = none */
    int max_batch;            /* mixed LPBE requests up to 65^3 admitted together and
                                 solved in one persistent kernel (pmgb_batch_solve):
                                 0 = 16, 1 = no batching */
} pmgb_server_config;

typedef struct pmgb_result {
    int status;               /* 1 done, 0 queued or running, -1 failed */
    double energy_kT;         /* Vpmg_energy of the calculation */
    double latency_ms;        /* submit -> done */
    double queue_ms;          /* submit -> start */
    double service_ms;        /* start -> done */
    long long admit_order;    /* 1-based position in the order of admission */
    pmgb_stats stats;
    char error[256];
} pmgb_result;

typedef struct pmgb_server_stats {
    long long submitted, done, failed;
    double p50_ms, p99_ms, mean_ms;   /* latency (submit -> done) of finished requests */
    double mean_service_ms;
    size_t bytes_in_use, bytes_peak, budget;
    long long created, reused, evicted; /* calculations built, pooled ones reused, released */
    int inflight_peak;
    long long batches, batched;       /* persistent-kernel launches and the requests in them */
    int batch_peak;
} pmgb_server_stats;

int pmgb_server_create(const pmgb_server_config *config, pmgb_server **out);

/* The device side of the loop as plain callbacks.  pmgb_server_create uses
 * the CUDA calculation (pmgb_create, pmgb_fillco, pmgb_solve, pmgb_energy);
 * pmgb_server_create_ex takes a replacement, so the queueing, admission
 * and pooling logic can be exercised without a GPU. */
typedef struct pmgb_server_backend {
    void *ctx;
    size_t (*footprint)(void *ctx, const pmgb_params *params, int precision, int natoms);
    void *(*create)(void *ctx, const pmgb_params *params, int precision);
    int (*reconfigure)(void *ctx, void *calc, const pmgb_params *params);
    /* fill + solve + energy; returns 1 on success */
    int (*run)(void *ctx, void *calc, int natoms, const double *xyz, const double *charge,
               const double *radius, double *energy_kT);
    void (*destroy)(void *ctx, void *calc);
} pmgb_server_backend;

int pmgb_server_create_ex(const pmgb_server_config *config, const pmgb_server_backend *backend,
                          pmgb_server **out);
/* Queue one calculation (fill from the host atom arrays, solve, energy).
 * The arrays are copied; u_out, when not NULL, receives the potential
 * (nx*ny*nz doubles) and must stay valid until the request is done.
 * Returns the request id (> 0), or 0 when the request can never fit. */
long long pmgb_server_submit(pmgb_server *srv, const pmgb_params *params, int natoms,
                             const double *xyz, const double *charge, const double *radius,
                             double *u_out);
/* Status of a request without waiting (the return value is result->status). */
int pmgb_server_poll(pmgb_server *srv, long long id, pmgb_result *result);
/* Launch-shape tunable (PMGB_TUNE_*) for every calculation of this grid
 * shape (nx, ny, nz, nlev of params) the loop builds from now on. */
int pmgb_server_set_shape_tuning(pmgb_server *srv, const pmgb_params *shape, int key, int value);
/* Wait for a request to finish. */
int pmgb_server_wait(pmgb_server *srv, long long id, pmgb_result *result);
/* Wait until every submitted request has finished. */
int pmgb_server_drain(pmgb_server *srv);
int pmgb_server_get_stats(pmgb_server *srv, pmgb_server_stats *stats);
/* Drain, stop the workers and release every calculation. */
void pmgb_server_destroy(pmgb_server *srv);

const char *pmgb_last_error(void);

/* Number of kernel launches issued by the calling thread since the last
 * reset (instrumentation for the benchmark). */
long long pmgb_launch_count(int reset);

#ifdef __cplusplus
}
#endif

#endif /* APBS_B200_H */
