// Energy of a solved potential without any device allocation.
//
// For callers that cannot allocate device memory at the point where they
// need the energy: code running inside another framework's memory pool,
// whose device memory belongs to that pool and where a cudaMalloc would
// synchronise the device, and embedded or real-time callers whose device
// footprint is fixed up front.  They already hold the potential and the
// coefficient maps in device memory; this entry point only reads them.
// The call copies the partition weights in from host memory and waits for
// its own result on the stream before it returns.
//
// The per-block partial sums and the partition weights live in one
// file-scope device array of fixed size.  Its device address is looked up
// once per device (cudaGetSymbolAddress, with that device current) on the
// first call made there, so make that first call before any stream capture
// on that device.
// Every call on a device uses the same array: calls that overlap on the GPU
// (different streams, or host threads calling concurrently) race on it and
// must be serialised by the caller.  Nothing in the array needs to start at
// zero: each call writes every slot it reads.
#include <math.h>
#include <string.h>

#include "apbs_b200.h"
#include "mg_kernels.cuh"

namespace pmgb {
void set_error(const char* fmt, ...);
}
using namespace pmgb;

namespace {

// Layout of the scratch array (doubles):
//   [0, 4736)       per-block partial sums, 4 per block, at most 1184 blocks
//   [4736, 4740)    the four global sums
//   [4744, 4744 + nx + ny + nz)  partition weights wx | wy | wz
constexpr int kPartOff = 0;
constexpr int kSumOff = 4736;
constexpr int kWeightOff = 4744;
constexpr int kScratchDoubles = 8192;  // 64 KiB per device

static __device__ __align__(256) double g_energy_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// Per-axis partition weights of Vpmg_setPart (src/mg/vpmg.c:627-870) for a
// partition equal to the mg-manual domain.
void axis_weights(int n, double h, double cent, double* w) {
  const double small = 1.0e-12;
  const double lo = cent - 0.5 * ((n - 1) * h), hi = cent + 0.5 * ((n - 1) * h);
  const double xmin = cent - 0.5 * h * (n - 1);
  for (int i = 0; i < n; i++) {
    const double x = i * h + xmin;
    double ok;
    if ((x < (hi - h / 2)) && (x > (lo + h / 2))) ok = 1.0;
    else if (fabs(x - lo) < small) ok = 1.0;
    else if (fabs(x - hi) < small) ok = 1.0;
    else if ((x > (hi + h / 2)) || (x < (lo - h / 2))) ok = 0.0;
    else if ((x < (hi + h / 2)) || (x > (lo - h / 2))) {
      const double x0 = (x - h / 2 >= lo) ? x - h / 2 : lo;
      const double x1 = (x + h / 2 <= hi) ? x + h / 2 : hi;
      ok = fabs(x1 - x0) / h;
      if (ok < 0.0 && fabs(ok) < small) ok = 0.0;
      if (ok > 1.0 && fabs(ok - 1.0) < small) ok = 1.0;
    } else ok = 0.0;
    w[i] = ok;
  }
}

}  // namespace

extern "C" int pmgb_energy_noalloc(const pmgb_params* p, const double* d_u,
                                   const double* d_charge, const double* d_epsx,
                                   const double* d_epsy, const double* d_epsz,
                                   const double* d_kappa, void* cuda_stream,
                                   double* energy_kT) {
  if (!p || !d_u || !d_charge || !energy_kT) {
    set_error("pmgb_energy_noalloc: null argument");
    return 0;
  }
  if (p->nx < 3 || p->ny < 3 || p->nz < 3 || p->nx > PMGB_NOALLOC_MAX_DIM ||
      p->ny > PMGB_NOALLOC_MAX_DIM || p->nz > PMGB_NOALLOC_MAX_DIM) {
    set_error("pmgb_energy_noalloc: grid %dx%dx%d outside 3..%d points per axis", p->nx, p->ny,
              p->nz, PMGB_NOALLOC_MAX_DIM);
    return 0;
  }
  if (p->nion < 0 || p->nion > PMGB_MAXION) {
    set_error("pmgb_energy_noalloc: %d ion species outside 0..%d", p->nion, PMGB_MAXION);
    return 0;
  }
  if (p->chgm != PMGB_CHGM_SPL2) {
    set_error("pmgb_energy_noalloc: the charge-map energy needs chgm spl2");
    return 0;
  }
  if (p->nonlin && (!d_epsx || !d_epsy || !d_epsz || !d_kappa)) {
    set_error("pmgb_energy_noalloc: NPBE needs the dielectric and kappa maps");
    return 0;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error("pmgb_energy_noalloc: no usable CUDA device");
    return 0;
  }
  if (!g_scratch_ptr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_energy_scratch);
    if (e != cudaSuccess || !ptr) {
      set_error("pmgb_energy_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return 0;
    }
    g_scratch_ptr[dev] = (double*)ptr;
  }
  double* scratch = g_scratch_ptr[dev];
  cudaStream_t st = (cudaStream_t)cuda_stream;

  // physical scalars (Vpbe_ctor2, src/generic/vpbe.c:380-411)
  const double N_A = 6.022045000e+23, e_c = 4.803242384e-10, k_B = 1.380662000e-16;
  const double pi = 4. * atan(1.);
  double ionstr = 0.0;
  for (int i = 0; i < p->nion; i++) ionstr += (0.5 * p->ion_conc[i] * (p->ion_q[i] * p->ion_q[i]));
  double zkappa2 = 0.0;
  if (ionstr != 0.) {
    const double xk = sqrt(ionstr * 1.0e-16 *
                           ((8.0 * pi * N_A * e_c * e_c) / (1000.0 * p->sdie * k_B * p->temp)));
    zkappa2 = p->sdie * (xk * xk);
  }
  const double zmagic = ((4.0 * pi * e_c * e_c) / (k_B * p->temp)) * 1.0e+8;

  // partition weights into the scratch array (a copy, not an allocation)
  double w[3 * PMGB_NOALLOC_MAX_DIM];
  axis_weights(p->nx, p->hx, p->center[0], w);
  axis_weights(p->ny, p->hy, p->center[1], w + p->nx);
  axis_weights(p->nz, p->hz, p->center[2], w + p->nx + p->ny);
  cudaError_t e = cudaMemcpyAsync(scratch + kWeightOff, w,
                                  sizeof(double) * (p->nx + p->ny + p->nz),
                                  cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    set_error("pmgb_energy_noalloc: weight copy: %s", cudaGetErrorString(e));
    return 0;
  }
  EnergyArgs a;
  a.g = Grid{p->nx, p->ny, p->nz};
  a.u = d_u;
  a.charge = d_charge;
  a.epsx = d_epsx;
  a.epsy = d_epsy;
  a.epsz = d_epsz;
  a.kappa = d_kappa;
  a.wx = scratch + kWeightOff;
  a.wy = scratch + kWeightOff + p->nx;
  a.wz = scratch + kWeightOff + p->nx + p->ny;
  a.hx = p->hx;
  a.hy = p->hy;
  a.hz = p->hz;
  a.nonlin = (p->nonlin && ionstr > 0.) ? 1 : 0;
  a.ions.nion = p->nion;
  for (int i = 0; i < p->nion; i++) {
    a.ions.q[i] = p->ion_q[i];
    a.ions.sconc[i] = p->ion_conc[i];
  }
  a.zks2 = (ionstr > 0.0) ? 0.5 * zkappa2 / ionstr : 0.0;
  launch_energy_sums(st, a, scratch + kPartOff, scratch + kSumOff);
  double sums[4];
  e = cudaMemcpyAsync(sums, scratch + kSumOff, sizeof(sums), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_error("pmgb_energy_noalloc: %s", cudaGetErrorString(e));
    return 0;
  }
  // Vpmg_energy (src/mg/vpmg.c:1248-1277), extFlag without external terms
  const double qf = sums[0] * p->hx * p->hy * p->hz / zmagic;
  double en;
  if (a.nonlin) {
    double diel = 0.5 * sums[1] * p->hx * p->hy * p->hz;
    diel = diel / zmagic;
    double qm = 0.0;
    if (!(zkappa2 < 1.0e-9)) {
      if (sums[3] > 0.0) {
        set_error("pmgb_energy_noalloc: clamped exponentials in the mobile-ion energy");
        return 0;
      }
      qm = sums[2] * p->hx * p->hy * p->hz;
      qm = qm / zmagic;
    }
    en = qf - diel - qm;
  } else {
    en = 0.5 * qf;
  }
  *energy_kT = en;
  return 1;
}
