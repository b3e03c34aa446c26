// Kernel declarations of the FP64 multigrid path (mg_kernels.cu).
#pragma once
#include "common.cuh"

namespace pmgb {

// ---- operators ------------------------------------------------------------
void launch_build_fine(cudaStream_t s, Grid g, const double* xf, const double* yf,
                       const double* zf, const double* a1, const double* a2,
                       const double* a3, const double* ccf, const double* fcf,
                       const double* gx, const double* gy, const double* gz,
                       double* oC, double* oE, double* oN, double* uC, double* cc,
                       double* fc);
void launch_galerkin(cudaStream_t s, Grid gf, Op fine, Grid gc, double* const* coarse);

// ---- grid transfer ---------------------------------------------------------
void launch_restrict(cudaStream_t s, Grid gf, const double* xin, Grid gc, double* xout);
// x_f += (num/den) * P x_c   (num, den: device scalars)
void launch_interp_axpy(cudaStream_t s, Grid gc, const double* xc, Grid gf, double* xf,
                        const double* num, const double* den);

// ---- stencils ----------------------------------------------------------------
void launch_gs7_colour(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                       double* x, int parity);
// one full red-black sweep in one pass, xin -> xout (boundaries of both
// zero; diag from launch_diag; shape: PMGB_TUNE_GS7_SWEEP_SHAPE)
int launch_gs7_sweep64(cudaStream_t s, Grid g, Op op, const double* diag, const double* fc,
                       const double* xin, double* xout, int first_parity, int kchunk,
                       int shape);
// the single-pass sweep handles this grid (odd nx and ny, 32-bit offsets)
int gs7_sweep_supported(Grid g);
// D = oC + cc inside, 1 on the boundary
void launch_diag(cudaStream_t s, Grid g, const double* oC, const double* cc, double* D);
extern int g_tune[16];
void launch_resid(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                  const double* x, double* r);
void launch_matvec(cudaStream_t s, Grid g, Op op, const double* cc, const double* x, double* y);
// *num = <x, w0>, *den = <x, (A + cc) x> over the interior in one launch
// (part: 2 * reduce_parts(interior) doubles; *done: a zero word the launch
// leaves zero)
void launch_xdamp_sums(cudaStream_t s, Grid g, Op op, const double* cc, const double* x,
                       const double* w0, double* part, unsigned* done, double* num,
                       double* den);

// Ordered 27-point Gauss-Seidel: nsweep red-black sweeps (2*nsweep
// half-sweeps) pipelined along wavefronts t = j + 2k, optionally followed by
// the residual r = f - (A + cc) x.  first_parity: colour of the first
// half-sweep ((i+j+k)%2, 0-based).
struct Gs27Plan {
  int cluster;   // CTAs per cluster (1 = single CTA)
  int threads;   // threads per CTA
};
// Sets kernel attributes; returns the largest usable GS27 cluster size.
int mg_init();
// One CTA per interior plane, neighbour planes synchronised by step counters
// (kWavePlanesMax counters per level, never reset between launches; *err
// counts waits that ran out).  wave_planes_fit: the level has few enough
// planes for one resident CTA each.
constexpr int kWavePlanesMax = 1024;
constexpr int kWaveCounterBase = 16;  // words before level 0's counters
constexpr int kWaveDampTicket = 8;    // the word launch_xdamp_sums counts blocks in
constexpr int kWaveMixedDampTicket = 9;  // the same for the mixed path's damping sums
constexpr size_t kWaveWords = kWaveCounterBase + 16 * (size_t)kWavePlanesMax;
int wave_planes_fit(Grid g);
// wlag: wavefronts between successive half-sweeps (>= 4)
int launch_gs27_planes(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                       double* x, double* r, int nsweep, int first_parity, unsigned* counters,
                       int* err, int poll_all, int wlag);
int launch_gs27_wave(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                     double* x, double* r, int nsweep, int first_parity, Gs27Plan plan);
// The same schedule with each CTA's plane and its neighbours in shared
// memory and updates passed through a self-validating mailbox (mail_words(g)
// 64-bit words per level, zeroed whenever the level's counters restart);
// wave_mail_fit: three planes fit in one CTA's shared memory and the level's
// planes on the device.  Returns 0 (nothing launched) where it does not fit.
size_t mail_words(Grid g);
int wave_mail_fit(Grid g);
int launch_gs27_mail(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                     double* x, double* r, int nsweep, int first_parity, unsigned* counters,
                     int* err, int wlag, unsigned long long* mail);

// ---- BLAS-1 on interior points -------------------------------------------
void launch_zero(cudaStream_t s, double* x, size_t n);
void launch_copy_interior(cudaStream_t s, Grid g, const double* x, double* y);
void launch_axpy_interior(cudaStream_t s, Grid g, const double* a_dev, double a_host,
                          const double* x, double* y);
// Reductions write one double to out_dev (deterministic two-pass sum).
void launch_nrm1(cudaStream_t s, Grid g, const double* x, double* part, double* out_dev);
void launch_dot(cudaStream_t s, Grid g, const double* x, const double* y, double* part,
                double* out_dev);
size_t reduce_parts(size_t n);

// ---- coarsest solves -------------------------------------------------------
// Band storage of the coarsest operator exactly as Vbuildband1_27 writes it.
void launch_band_build(cudaStream_t s, Grid g, Op op, double* abd, int m, int lda);
void launch_band_factor(cudaStream_t s, double* abd, int n, int m, int lda, int* info);
void launch_band_solve(cudaStream_t s, Grid g, const double* abd, int n, int m, int lda,
                       const double* rhs, double* x);
// CG on the coarsest level (Vcghs), all iterations in one cluster launch.
int launch_cg_coarse(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                     double* x, double* r, double* p, double* ap, int itmax, double errtol,
                     int* iters_dev, int want_cluster = 0);

// ---- nonlinear (Newton) -----------------------------------------------------
struct IonTable {
  int nion;
  double q[8];
  double sconc[8];  // concentration scaled by 0.5/I
};
// r = f + (off-diagonal stencil) x - oC x - c(x) on the fine level
void launch_nresid(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                   const double* x, double* r, IonTable ions);
// k_nresid and the 1-norm of r into out_dev (bitwise the launch_nrm1 value),
// and c'(x) into cp on the interior when cp is not null
void launch_nresid_nrm1(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                        const double* x, double* r, IonTable ions, double* part,
                        double* out_dev, double* cp);
// out = x + a y on interior points
void launch_xpay_interior(cudaStream_t s, Grid g, const double* x, double a, const double* y,
                          double* out);
// cp = c'(x) on every point
void launch_dcvec(cudaStream_t s, Grid g, const double* cc, const double* x, double* cp,
                  IonTable ions);

// ---- boundary restore and energies -------------------------------------------
void launch_fbound(cudaStream_t s, Grid g, double* x, const double* gx, const double* gy,
                   const double* gz);
struct EnergyArgs {
  Grid g;
  const double* u;
  const double* charge;
  const double* epsx;
  const double* epsy;
  const double* epsz;
  const double* kappa;
  const double* wx;
  const double* wy;
  const double* wz;
  double hx, hy, hz;
  int nonlin;          // also sum the dielectric and mobile-ion terms
  IonTable ions;       // raw concentrations in sconc for the qm term
  double zks2;
  int linear_qm = 0;   // mobile-ion term in the LPBE form pvec zkappa2 kappa u^2
  double zkappa2 = 0.0;
  int complement = 0;  // weights flipped as extEnergy flips the coarse pvec
};
// out_dev[0] = sum pvec u charge, [1] = dielectric sum, [2] = mobile-ion sum,
// [3] = number of clamped exponentials
void launch_energy_sums(cudaStream_t s, const EnergyArgs& a, double* part, double* out_dev);

}  // namespace pmgb
