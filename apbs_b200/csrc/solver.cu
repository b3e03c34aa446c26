// Host orchestration of the B200 PMG solver and the C ABI (apbs_b200.h).
//
// The control flow restates the reference drivers: Vpmg_fillco
// (src/mg/vpmg.c:5250-5414), Vpmg_solve (401-558), Vmgdriv2
// (src/pmgc/mgdrvd.c:190-558), Vmvcs (src/pmgc/mgcsd.c:57-565), Vnewdriv2 /
// Vnewton (src/pmgc/newdrvd.c:169-350, newtond.c:162-598) and Vpmg_energy
// (vpmg.c:1248-1891).  All arithmetic runs in CUDA kernels; the host keeps
// only the decisions the reference takes on scalar norms (stopping tests,
// Newton damping), reading one scalar per decision.
#include <math.h>

#include <cmath>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "apbs_b200.h"
#include "fill_kernels.cuh"
#include "mg_kernels.cuh"
#include "mixed.cuh"
#include "solver_internal.cuh"

namespace pmgb {

static thread_local char g_err[512] = "";
static thread_local long long g_launches = 0;

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
void note_launches(long long n) { g_launches += n; }

// Per-axis partition weights of Vpmg_setPart (src/mg/vpmg.c:763-863) for the
// partition [lo, hi] with no neighbouring processors (bflags all 0).
void part_weights(int n, double h, double cent, double lo, double hi, double* w) {
  const double small = 1.0e-12;
  double xmin = cent - 0.5 * h * (n - 1);
  for (int i = 0; i < n; i++) {
    double x = i * h + xmin, ok;
    if ((x < (hi - h / 2)) && (x > (lo + h / 2))) ok = 1.0;
    else if (fabs(x - lo) < small) ok = 1.0;
    else if (fabs(x - hi) < small) ok = 1.0;
    else if ((x > (hi + h / 2)) || (x < (lo - h / 2))) ok = 0.0;
    else if ((x < (hi + h / 2)) || (x > (lo - h / 2))) {
      double x0 = (x - h / 2 >= lo) ? x - h / 2 : lo;
      double x1 = (x + h / 2 <= hi) ? x + h / 2 : hi;
      ok = fabs(x1 - x0) / h;
      if (ok < 0.0 && fabs(ok) < small) ok = 0.0;
      if (ok > 1.0 && fabs(ok - 1.0) < small) ok = 1.0;
    } else ok = 0.0;
    w[i] = ok;
  }
}

}  // namespace pmgb

using namespace pmgb;

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e__ = (call);                                                          \
    if (e__ != cudaSuccess) {                                                          \
      set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e__));  \
      return 0;                                                                        \
    }                                                                                  \
  } while (0)

namespace {

int dalloc(double** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(double));
  if (e != cudaSuccess) {
    set_error("cudaMalloc(%zu doubles): %s", n, cudaGetErrorString(e));
    *p = nullptr;
    return 0;
  }
  cudaMemset(*p, 0, n * sizeof(double));
  return 1;
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

// Stream-ordered (re)allocation with geometric growth: a calculation reused
// for a larger molecule neither synchronises the device (as cudaFree does)
// nor reallocates for every small increase.
template <typename T>
int grow(T** p, size_t* cap, size_t need, cudaStream_t st) {
  if (*p && need <= *cap) return 1;
  const size_t n = std::max(need, *cap + *cap / 2);
  if (*p) cudaFreeAsync(*p, st);
  *p = nullptr;
  *cap = 0;
  const cudaError_t e = cudaMallocAsync((void**)p, std::max<size_t>(n, 1) * sizeof(T), st);
  if (e != cudaSuccess) {
    *p = nullptr;
    set_error("cudaMallocAsync(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    return 0;
  }
  *cap = n;
  return 1;
}

// Vpbe_ctor2 scalars (src/generic/vpbe.c:264-411) and the ion tables of
// Vpmg_ctor2 (src/mg/vpmg.c:340-377).
void phys_setup(pmgb_solver* s, int natoms, const double* xyz, const double* r) {
  const pmgb_params& p = s->p;
  const double N_A = 6.022045000e+23, e_c = 4.803242384e-10, k_B = 1.380662000e-16;
  const double pi = 4. * atan(1.);
  double mn[3], mx[3], radius = 0.0;
  for (int i = 0; i < 3; i++) mn[i] = mx[i] = xyz[i];
  for (int a = 0; a < natoms; a++)
    for (int i = 0; i < 3; i++) {
      double v = xyz[3 * a + i];
      if (v < mn[i]) mn[i] = v;
      if (v > mx[i]) mx[i] = v;
    }
  for (int i = 0; i < 3; i++) s->soluteCenter[i] = 0.5 * (mx[i] + mn[i]);
  for (int a = 0; a < natoms; a++) {
    double d0 = xyz[3 * a] - s->soluteCenter[0];
    double d1 = xyz[3 * a + 1] - s->soluteCenter[1];
    double d2 = xyz[3 * a + 2] - s->soluteCenter[2];
    double dist = (d0 * d0) + (d1 * d1) + (d2 * d2);
    dist = sqrt(dist) + r[a];
    if (dist > radius) radius = dist;
  }
  s->soluteRadius = radius;
  s->ionstr = 0.0;
  s->maxIonRadius = 0.0;
  for (int i = 0; i < p.nion; i++) {
    if (p.ion_radius[i] > s->maxIonRadius) s->maxIonRadius = p.ion_radius[i];
    s->ionstr += (0.5 * p.ion_conc[i] * (p.ion_q[i] * p.ion_q[i]));
  }
  if (s->ionstr == 0.) {
    s->xkappa = 0.;
    s->zkappa2 = 0.;
  } else {
    s->xkappa = sqrt(s->ionstr * 1.0e-16 *
                     ((8.0 * pi * N_A * e_c * e_c) / (1000.0 * p.sdie * k_B * p.temp)));
    s->zkappa2 = p.sdie * (s->xkappa * s->xkappa);
  }
  s->zmagic = ((4.0 * pi * e_c * e_c) / (k_B * p.temp)) * 1.0e+8;
  const double zks2 = (s->ionstr > 0.0) ? 0.5 / s->ionstr : 0.0;
  s->ions.nion = p.nion;
  s->ions_e.nion = p.nion;
  for (int i = 0; i < p.nion && i < 8; i++) {
    s->ions.q[i] = p.ion_q[i];
    s->ions.sconc[i] = zks2 * p.ion_conc[i];
    s->ions_e.q[i] = p.ion_q[i];
    s->ions_e.sconc[i] = p.ion_conc[i];
  }
}

// Reference sphere of VaccSurf_refSphere (src/generic/vacc.c:924-978), built
// with the host libm exactly as the reference builds it.
int ref_sphere(int npts, std::vector<double>& pts) {
  const double pi = 3.14159265358979323846;
  const double frac = ((double)npts) / 4.0;
  const int ntheta = (int)floor(sqrt(pi * frac) + 0.5);
  const double dtheta = pi / ((double)ntheta);
  const int nphimax = 2 * ntheta;
  pts.clear();
  for (int it = 0; it < ntheta; it++) {
    const double theta = dtheta * ((double)it);
    const double st = sin(theta), ct = cos(theta);
    const int nphi = (int)floor(st * nphimax + 0.5);
    if (nphi != 0) {
      const double dphi = 2 * pi / ((double)nphi);
      for (int ip = 0; ip < nphi; ip++) {
        const double phi = dphi * ((double)ip);
        pts.push_back(cos(phi) * st);
        pts.push_back(sin(phi) * st);
        pts.push_back(ct);
      }
    }
  }
  return (int)(pts.size() / 3);
}

float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

int read_scalar(pmgb_solver* s, int slot, double* v) {
  CK(cudaMemcpyAsync(v, s->scal + slot, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  // a plane-wavefront wait that ran out leaves the iterates undefined: stop
  // at the next read instead of iterating on them (pmgb_solve reports it)
  int nerr = 0;
  if (s->wave_used)
    CK(cudaMemcpyAsync(&nerr, s->d_wave, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (nerr) {
    set_error("%d bounded device waits ran out (gs27 plane wavefront)", nerr);
    return 0;
  }
  return 1;
}

// GS27 launch shape per level (cluster of CTAs for the wavefront).
int max_cluster() {
  static const int mc = mg_init();  // probed once, thread-safely
  return mc;
}

Gs27Plan plan_for(Grid g, const int* tune) {
  const int ni = std::max(g.nx, std::max(g.ny, g.nz)) - 2;
  Gs27Plan p;
  const int mc = max_cluster();
  auto pick = [&](int want, int dflt) {
    int c = want > 0 ? want : dflt;
    c = std::min(c, mc);
    int p2 = 1;  // a power of two
    while (p2 * 2 <= c) p2 *= 2;
    return p2;
  };
  if (ni >= 60) p.cluster = pick(tune[2], mc);
  else if (ni >= 28) p.cluster = pick(tune[7], 8);
  else if (ni >= 12) p.cluster = 2;
  else p.cluster = 1;
  p.threads = (p.cluster >= 8) ? 512 : 256;
  return p;
}

}  // namespace

// ===========================================================================
// construction
// ===========================================================================
static int set_geometry(pmgb_solver* s);

// Restarts the wavefront step counters of every level and zeroes the
// mailboxes with them (a mailbox tag is a counter value plus one, so old
// slots must not outlive the counters they were tagged from).
static void wave_reset(pmgb_solver* s, cudaStream_t st) {
  if (s->d_wave) cudaMemsetAsync(s->d_wave, 0, kWaveWords * sizeof(unsigned), st);
  if (s->d_mail) cudaMemsetAsync(s->d_mail, 0, s->mail_total * sizeof(unsigned long long), st);
}

extern "C" int pmgb_create(const pmgb_params* params, int precision, pmgb_solver** out) {
  *out = nullptr;
  if (!params) {
    set_error("pmgb_create: params is NULL");
    return 0;
  }
  const pmgb_params& p = *params;
  if (p.nx < 5 || p.ny < 5 || p.nz < 5 || p.nlev < 2 || p.nlev > 11) {
    set_error("pmgb_create: unsupported grid %dx%dx%d nlev %d", p.nx, p.ny, p.nz, p.nlev);
    return 0;
  }
  if (p.chgm != PMGB_CHGM_SPL2 && p.chgm != PMGB_CHGM_TRIL && p.chgm != PMGB_CHGM_SPL4) {
    set_error("pmgb_create: chgm %d not implemented (spl0, spl2 and spl4 are)", p.chgm);
    return 0;
  }
  if (p.srfm != PMGB_SRFM_MOL && p.srfm != PMGB_SRFM_SMOL && p.srfm != PMGB_SRFM_SPL2 &&
      p.srfm != PMGB_SRFM_SPL3 && p.srfm != PMGB_SRFM_SPL4) {
    set_error("pmgb_create: srfm %d not implemented (mol, smol, spl2, spl3 and spl4 are)",
              p.srfm);
    return 0;
  }
  if (p.nion > 8) {
    set_error("pmgb_create: at most 8 ion species");
    return 0;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    set_error("pmgb_create: no CUDA device available");
    return 0;
  }
  // every level must coarsen exactly (Vcorsr, src/pmgc/mgsubd.c:426-444)
  {
    int nx = p.nx, ny = p.ny, nz = p.nz;
    for (int l = 1; l < p.nlev; l++) {
      if ((nx - 1) % 2 || (ny - 1) % 2 || (nz - 1) % 2) {
        set_error("pmgb_create: dime %d %d %d does not coarsen %d times", p.nx, p.ny, p.nz,
                  p.nlev - 1);
        return 0;
      }
      nx = (nx - 1) / 2 + 1;
      ny = (ny - 1) / 2 + 1;
      nz = (nz - 1) / 2 + 1;
      if (nx < 3 || ny < 3 || nz < 3) {
        set_error("pmgb_create: too many levels for dime %d %d %d", p.nx, p.ny, p.nz);
        return 0;
      }
    }
  }
  pmgb_solver* s = new pmgb_solver();
  memset(&s->st, 0, sizeof(s->st));
  s->p = p;
  s->precision = precision;
  s->device = dev;
  s->g = Grid{p.nx, p.ny, p.nz};
  s->n = s->g.n();
  s->mixed = nullptr;
  if (cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("pmgb_create: stream creation failed");
    delete s;
    return 0;
  }
  s->stream = s->own_stream;
  if (cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("pmgb_create: stream creation failed");
    cudaStreamDestroy(s->own_stream);
    delete s;
    return 0;
  }
  for (int i = 0; i < 16; i++) s->tune[i] = g_tune[i];
  for (int i = 0; i < 8; i++) cudaEventCreate(&s->ev[i]);
  cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming);
  const size_t n = s->n;
  int ok = 1;
  ok &= dalloc(&s->charge, n) && dalloc(&s->epsx, n) && dalloc(&s->epsy, n) &&
        dalloc(&s->epsz, n) && dalloc(&s->kappa, n) && dalloc(&s->ccf, n);
  ok &= dalloc(&s->gx, 2 * (size_t)p.ny * p.nz) && dalloc(&s->gy, 2 * (size_t)p.nx * p.nz) &&
        dalloc(&s->gz, 2 * (size_t)p.nx * p.ny);
  ok &= dalloc(&s->xf, p.nx) && dalloc(&s->yf, p.ny) && dalloc(&s->zf, p.nz) &&
        dalloc(&s->wx, p.nx) && dalloc(&s->wy, p.ny) && dalloc(&s->wz, p.nz) &&
        dalloc(&s->mom, 16);
  // the dielectric byte maps (DielMask), 3 bytes per point
  if (ok && cudaMalloc(&s->dmask, 3 * n) != cudaSuccess) {
    set_error("cudaMalloc(%zu bytes) failed", 3 * n);
    s->dmask = nullptr;
    ok = 0;
  }
  // hierarchy (Vbuildstr, src/pmgc/mgsubd.c:261-343)
  s->nlev = p.nlev;
  for (int l = 0; ok && l < s->nlev; l++) {
    Level& L = s->lev[l];
    if (l == 0) L.g = s->g;
    else
      L.g = Grid{(s->lev[l - 1].g.nx - 1) / 2 + 1, (s->lev[l - 1].g.ny - 1) / 2 + 1,
                 (s->lev[l - 1].g.nz - 1) / 2 + 1};
    L.nop = (l == 0) ? 4 : 14;
    const size_t nl = L.g.n();
    for (int c = 0; c < 14; c++) L.op[c] = nullptr;
    for (int c = 0; c < L.nop; c++) ok &= dalloc(&L.op[c], nl);
    ok &= dalloc(&L.cc, nl) && dalloc(&L.fc, nl) && dalloc(&L.x, nl) && dalloc(&L.w0, nl);
    ok &= dalloc(&L.cp, nl) && dalloc(&L.rhs, nl) && dalloc(&L.xt, nl);
    s->plan[l] = plan_for(L.g, s->tune);
  }
  ok &= dalloc(&s->w1, n) && dalloc(&s->w2, n) && dalloc(&s->w3, n) && dalloc(&s->xs, n);
  ok &= dalloc(&s->dg[0], n) && dalloc(&s->dg[1], n);
  ok &= dalloc(&s->nw_r0, n) && dalloc(&s->nw_ws, n) && dalloc(&s->nw_keepx, n) &&
        dalloc(&s->nw_keepr, n);
  ok &= dalloc(&s->part, 4 * 1184 + 64) && dalloc(&s->scal, S_COUNT);
  if (ok) ok &= (cudaMalloc(&s->d_iters, 16 * sizeof(int)) == cudaSuccess);
  if (ok) ok &= (cudaMalloc(&s->d_info, 16 * sizeof(int)) == cudaSuccess);
  if (ok) ok &= (cudaMalloc(&s->d_npts, sizeof(int)) == cudaSuccess);
  if (ok) ok &= (cudaMalloc(&s->d_wave, kWaveWords * sizeof(unsigned)) == cudaSuccess);
  if (ok) ok &= (cudaMemset(s->d_wave, 0, kWaveWords * sizeof(unsigned)) == cudaSuccess);
  // mailboxes for the levels the ordered GS27 smooths (all but the
  // coarsest) where the shared-memory plane wavefront fits
  s->mail_total = 0;
  for (int l = 0; l < 12; l++) {
    s->mail_off[l] = -1;
    if (l >= 1 && l < s->nlev - 1 && wave_mail_fit(s->lev[l].g)) {
      s->mail_off[l] = (long long)s->mail_total;
      s->mail_total += mail_words(s->lev[l].g);
    }
  }
  if (ok && s->mail_total) {
    ok &= (cudaMalloc(&s->d_mail, s->mail_total * sizeof(unsigned long long)) == cudaSuccess);
    if (ok)
      ok &= (cudaMemset(s->d_mail, 0, s->mail_total * sizeof(unsigned long long)) ==
             cudaSuccess);
  }
  if (ok) ok &= (cudaMalloc(&s->d_opptrs, sizeof(double*) * 14 * 16) == cudaSuccess);
  if (ok) {
    // the operator arrays never move, so the pointer table is written once
    double* tab[14 * 16] = {nullptr};
    for (int l = 0; l < s->nlev; l++)
      for (int c = 0; c < 14; c++) tab[14 * l + c] = s->lev[l].op[c];
    ok &= (cudaMemcpy(s->d_opptrs, tab, sizeof(tab), cudaMemcpyHostToDevice) == cudaSuccess);
  }
  if (!ok) {
    pmgb_destroy(s);
    return 0;
  }
  if (!set_geometry(s)) {
    pmgb_destroy(s);
    return 0;
  }
  s->vc_exec[0] = s->vc_exec[1] = nullptr;
  s->vc_kernels[0] = s->vc_kernels[1] = 0;
  // the allocations above zero-fill on the legacy stream
  if (cudaStreamSynchronize(0) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    set_error("pmgb_create: device error during setup");
    pmgb_destroy(s);
    return 0;
  }
  *out = s;
  return 1;
}

// Geometry (Vpmg_fillco, vpmg.c:5332-5366), the coordinate arrays and the
// partition weights of the calculation's domain, from s->p.
static int set_geometry(pmgb_solver* s) {
  const pmgb_params& p = s->p;
  {
    const double xlen = (p.nx - 1) * p.hx, ylen = (p.ny - 1) * p.hy, zlen = (p.nz - 1) * p.hz;
    s->G.g = s->g;
    s->G.h[0] = p.hx; s->G.h[1] = p.hy; s->G.h[2] = p.hz;
    s->G.xmin[0] = p.center[0] - (xlen / 2.0);
    s->G.xmin[1] = p.center[1] - (ylen / 2.0);
    s->G.xmin[2] = p.center[2] - (zlen / 2.0);
    s->G.xmax[0] = p.center[0] + (xlen / 2.0);
    s->G.xmax[1] = p.center[1] + (ylen / 2.0);
    s->G.xmax[2] = p.center[2] + (zlen / 2.0);
    std::vector<double> xf(p.nx), yf(p.ny), zf(p.nz), wx(p.nx), wy(p.ny), wz(p.nz);
    for (int i = 0; i < p.nx; i++) xf[i] = s->G.xmin[0] + i * p.hx;
    for (int i = 0; i < p.ny; i++) yf[i] = s->G.xmin[1] + i * p.hy;
    for (int i = 0; i < p.nz; i++) zf[i] = s->G.xmin[2] + i * p.hz;
    part_weights(p.nx, p.hx, p.center[0], p.center[0] - 0.5 * ((p.nx - 1) * p.hx),
                 p.center[0] + 0.5 * ((p.nx - 1) * p.hx), wx.data());
    part_weights(p.ny, p.hy, p.center[1], p.center[1] - 0.5 * ((p.ny - 1) * p.hy),
                 p.center[1] + 0.5 * ((p.ny - 1) * p.hy), wy.data());
    part_weights(p.nz, p.hz, p.center[2], p.center[2] - 0.5 * ((p.nz - 1) * p.hz),
                 p.center[2] + 0.5 * ((p.nz - 1) * p.hz), wz.data());
    cudaMemcpy(s->xf, xf.data(), sizeof(double) * p.nx, cudaMemcpyHostToDevice);
    cudaMemcpy(s->yf, yf.data(), sizeof(double) * p.ny, cudaMemcpyHostToDevice);
    cudaMemcpy(s->zf, zf.data(), sizeof(double) * p.nz, cudaMemcpyHostToDevice);
    cudaMemcpy(s->wx, wx.data(), sizeof(double) * p.nx, cudaMemcpyHostToDevice);
    cudaMemcpy(s->wy, wy.data(), sizeof(double) * p.ny, cudaMemcpyHostToDevice);
    cudaStream_t st = s->stream;
    // plane counts per level change with the grid: restart the wavefront
    // step counters so every level's counters start equal
    wave_reset(s, st);
    CK(cudaMemcpyAsync(s->xf, xf.data(), sizeof(double) * p.nx, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->yf, yf.data(), sizeof(double) * p.ny, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->zf, zf.data(), sizeof(double) * p.nz, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->wx, wx.data(), sizeof(double) * p.nx, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->wy, wy.data(), sizeof(double) * p.ny, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->wz, wz.data(), sizeof(double) * p.nz, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
  }
  return 1;
}

extern "C" int pmgb_reconfigure(pmgb_solver* s, const pmgb_params* params) {
  if (!s || !params) {
    set_error("pmgb_reconfigure: null argument");
    return 0;
  }
  const pmgb_params& p = *params;
  if (p.nx != s->p.nx || p.ny != s->p.ny || p.nz != s->p.nz || p.nlev != s->p.nlev) {
    set_error("pmgb_reconfigure: grid %dx%dx%d/%d differs from the calculation's %dx%dx%d/%d",
              p.nx, p.ny, p.nz, p.nlev, s->p.nx, s->p.ny, s->p.nz, s->p.nlev);
    return 0;
  }
  if (p.nion < 0 || p.nion > PMGB_MAXION) {
    set_error("pmgb_reconfigure: nion %d outside 0..%d", p.nion, PMGB_MAXION);
    return 0;
  }
  CK(cudaStreamSynchronize(s->stream));
  s->p = p;
  if (!set_geometry(s)) return 0;
  s->filled = s->solved = s->built = 0;
  s->focused = 0;
  s->ext_qf = s->ext_di = s->ext_qm = 0.0;
  memset(&s->st, 0, sizeof(s->st));
  return 1;
}

extern "C" int pmgb_set_stream(pmgb_solver* s, void* stream) {
  if (!s) return 0;
  const cudaError_t e = cudaStreamSynchronize(s->stream);
  // switch even after an error, so no stale stream handle is kept; captured
  // V-cycle graphs hold no stream and stay valid
  s->stream = stream ? (cudaStream_t)stream : s->own_stream;
  if (e != cudaSuccess) {
    set_error("pmgb_set_stream: %s", cudaGetErrorString(e));
    return 0;
  }
  return 1;
}

// Device bytes one calculation holds once filled and solved: the maps,
// the level hierarchy with its work vectors, the FP32 hierarchy (mixed
// precision, or the FP64 path's exact coarsest solve), the banded factor
// of a small FP64 coarsest level, and per-atom fill work (accessible-
// surface flags dominate: ~4 pi (r_max + srad)^2 sdens reference points per
// atom, with r_max taken as 3 A).
extern "C" size_t pmgb_footprint(const pmgb_params* params, int precision, int natoms) {
  if (!params) return 0;
  const pmgb_params& p = *params;
  size_t nl[16];
  int gx[16], gy[16], gz[16];
  int nlev = p.nlev < 1 ? 1 : (p.nlev > 12 ? 12 : p.nlev);
  gx[0] = p.nx; gy[0] = p.ny; gz[0] = p.nz;
  for (int l = 1; l < nlev; l++) {
    gx[l] = (gx[l - 1] - 1) / 2 + 1;
    gy[l] = (gy[l - 1] - 1) / 2 + 1;
    gz[l] = (gz[l - 1] - 1) / 2 + 1;
  }
  for (int l = 0; l < nlev; l++) nl[l] = (size_t)gx[l] * gy[l] * gz[l];
  const size_t n = nl[0];
  size_t d = 0;  // doubles
  d += 6 * n + 3 * n + 4 * n;  // maps, w1-3, Newton vectors
  d += 2 * ((size_t)p.ny * p.nz + (size_t)p.nx * p.nz + (size_t)p.nx * p.ny);
  d += 2 * (size_t)(p.nx + p.ny + p.nz) + 16 + 4 * 1184 + 64 + S_COUNT;
  for (int l = 0; l < nlev; l++) d += (size_t)((l == 0 ? 4 : 14) + 7) * nl[l];
  size_t bytes = d * sizeof(double);
  bytes += 3 * n;  // the dielectric byte maps
  // mailboxes of the shared-memory GS27 wavefront (levels whose three planes
  // fit in a CTA's shared memory; an upper bound where the device says no)
  for (int l = 1; l < nlev - 1; l++)
    if ((size_t)3 * gx[l] * gy[l] * sizeof(double) + 1024 <= 232448)
      bytes += 2 * sizeof(unsigned long long) * (size_t)(gz[l] - 2) * 4 * (gy[l] - 2) *
               ((gx[l] - 1) / 2);
  // FP32 hierarchy from level lo, plus Galerkin levels down to <= 512 unknowns
  const int lo = (precision == PMGB_MIXED) ? 0 : nlev - 1;
  const size_t nc_int = (size_t)(gx[nlev - 1] - 2) * (gy[nlev - 1] - 2) * (gz[nlev - 1] - 2);
  const bool fp32 = (precision == PMGB_MIXED) || (!p.nonlin && nc_int > 512);
  if (fp32) {
    for (int l = lo; l < nlev; l++)
      bytes += (size_t)((l == 0 ? 4 : 14) + 3) * nl[l] * sizeof(float);
    if (precision != PMGB_MIXED) bytes += 15 * nl[lo] * sizeof(double);
    int cx = gx[nlev - 1], cy = gy[nlev - 1], cz = gz[nlev - 1];
    size_t nint = nc_int;
    while (nint > 512 && (cx - 1) % 2 == 0 && (cy - 1) % 2 == 0 && (cz - 1) % 2 == 0 && cx > 3) {
      cx = (cx - 1) / 2 + 1;
      cy = (cy - 1) / 2 + 1;
      cz = (cz - 1) / 2 + 1;
      const size_t nc = (size_t)cx * cy * cz;
      bytes += 15 * nc * sizeof(double) + 17 * nc * sizeof(float);
      nint = (size_t)(cx - 2) * (cy - 2) * (cz - 2);
    }
    bytes += 2 * nl[lo] * sizeof(float) + nint * nint * sizeof(double);
  } else if (!p.nonlin) {
    const size_t ex = gx[nlev - 1] - 2, exy = ex * (gy[nlev - 1] - 2);
    bytes += ((exy + ex + 2) * nc_int + nc_int) * sizeof(double);
  }
  const double pi = 3.14159265358979323846;
  const double nref = 4.0 * pi * (3.0 + p.srad) * (3.0 + p.srad) * (p.sdens > 0 ? p.sdens : 10.0);
  bytes += (size_t)natoms * ((size_t)nref * sizeof(unsigned) + 64 + 18 * sizeof(double) +
                            2 * sizeof(int) + 513 * sizeof(int));
  return bytes;
}

extern "C" void pmgb_destroy(pmgb_solver* s) {
  if (!s) return;
  cudaStreamSynchronize(s->stream);
  for (int m = 0; m < 2; m++)
    if (s->vc_exec[m]) cudaGraphExecDestroy(s->vc_exec[m]);
  if (s->mixed) mixed_destroy(s->mixed);
  dfree(s->charge); dfree(s->epsx); dfree(s->epsy); dfree(s->epsz); dfree(s->kappa);
  dfree(s->ccf); dfree(s->gx); dfree(s->gy); dfree(s->gz); dfree(s->xf); dfree(s->yf);
  dfree(s->zf); dfree(s->wx); dfree(s->wy); dfree(s->wz); dfree(s->mom);
  if (s->dmask) cudaFree(s->dmask);
  for (int l = 0; l < s->nlev; l++) {
    Level& L = s->lev[l];
    for (int c = 0; c < 14; c++) dfree(L.op[c]);
    dfree(L.cc); dfree(L.fc); dfree(L.x); dfree(L.w0); dfree(L.cp); dfree(L.rhs); dfree(L.xt);
  }
  dfree(s->w1); dfree(s->w2); dfree(s->w3); dfree(s->xs);
  dfree(s->dg[0]); dfree(s->dg[1]);
  dfree(s->nw_r0); dfree(s->nw_ws); dfree(s->nw_keepx); dfree(s->nw_keepr);
  dfree(s->part); dfree(s->scal); dfree(s->d_iters); dfree(s->d_info); dfree(s->d_npts); dfree(s->d_wave); dfree(s->d_forces);
  if (s->d_mail) cudaFree(s->d_mail);
  dfree(s->d_opptrs);
  dfree(s->band);
  dfree(s->focus_w);
  dfree(s->cell_count); dfree(s->cell_start); dfree(s->cell_fillpos); dfree(s->cell_of);
  dfree(s->cell_sorted); dfree(s->sas_list); dfree(s->sas_nbr); dfree(s->d_ref); dfree(s->atom_terms);
  dfree(s->ch_count); dfree(s->ch_start); dfree(s->ch_fill); dfree(s->ch_atoms);
  dfree(s->d_spl3);
  dfree(s->a_xyz); dfree(s->a_q); dfree(s->a_r);
  free_maps(s);
  for (int i = 0; i < 8; i++) cudaEventDestroy(s->ev[i]);
  cudaEventDestroy(s->fork_ev);
  cudaEventDestroy(s->join_ev);
  cudaStreamDestroy(s->side);
  cudaStreamDestroy(s->own_stream);
  delete s;
}

// ===========================================================================
// fill (Vpmg_fillco)
// ===========================================================================
// Statistics of a fill issued without waiting (time, surface points).
static int settle_fill(pmgb_solver* s) {
  if (!s->fill_pending) return 1;
  CK(cudaEventSynchronize(s->ev[1]));
  s->st.t_fill_ms = elapsed_ms(s->ev[0], s->ev[1]);
  int npts = 0;
  CK(cudaMemcpy(&npts, s->d_npts, sizeof(int), cudaMemcpyDeviceToHost));
  s->st.sas_points = npts;
  s->fill_pending = 0;
  return 1;
}

// sdh / mdh boundary values (bcCalc, vpmg.c:3369-3645 and 3289-3367) on
// stream `sd`; the atom term buffer is already sized.
static int side_boundary(pmgb_solver* s, cudaStream_t sd) {
  const pmgb_params& p = s->p;
  const int natoms = s->natoms;
  const double pi = 3.14159265358979323846;
  CK(cudaMemsetAsync(s->gx, 0, sizeof(double) * 2 * p.ny * p.nz, sd));
  CK(cudaMemsetAsync(s->gy, 0, sizeof(double) * 2 * p.nx * p.nz, sd));
  CK(cudaMemsetAsync(s->gz, 0, sizeof(double) * 2 * p.nx * p.ny, sd));
  if (p.bcfl == PMGB_BCFL_SDH) {
    SdhArgs A;
    A.g = s->g;
    for (int d = 0; d < 3; d++) A.center[d] = s->soluteCenter[d];
    A.size = s->soluteRadius;
    A.xkappa = s->xkappa;
    A.eps_p = p.pdie;
    A.eps_w = p.sdie;
    A.pre = (1.6021773e-19 * 1.6021773e-19) /
            (4 * pi * 8.8541878e-12 * 1.3806581e-23 * p.temp);
    A.pre = A.pre * (1.0e10);
    launch_sdh(sd, A, natoms, s->d_xyz, s->d_q, s->atom_terms, s->mom, s->xf, s->yf, s->zf,
               s->gx, s->gy, s->gz);
    note_launches(3);
  } else {
    // bcflnew (vpmg.c:3289-3367)
    MdhArgs A;
    A.g = s->g;
    A.xf = s->xf;
    A.yf = s->yf;
    A.zf = s->zf;
    A.gx = s->gx;
    A.gy = s->gy;
    A.gz = s->gz;
    A.pre1 = ((1.6021773e-19) / (4 * pi * 8.8541878e-12 * p.sdie * 1.3806581e-23 * p.temp)) *
             (1.0e10);
    A.xkappa = s->xkappa;
    launch_mdh(sd, A, natoms, s->d_xyz, s->d_q, s->d_r);
    note_launches(1);
  }
  CK(cudaGetLastError());
  return 1;
}

static int do_fill(pmgb_solver* s, const double* h_xyz, const double* h_r, int wait) {
  const pmgb_params& p = s->p;
  cudaStream_t st = s->stream;
  const size_t n = s->n;
  const int natoms = s->natoms;
  phys_setup(s, natoms, h_xyz, h_r);
  const int side_bc = (p.bcfl == PMGB_BCFL_SDH || p.bcfl == PMGB_BCFL_MDH);
  if (p.bcfl == PMGB_BCFL_SDH &&
      !grow(&s->atom_terms, &s->terms_alloc, 13 * (size_t)natoms, st))
    return 0;
  if (!uses_charge_map(s)) {
    const size_t nt = charge_tile_count(s->g) + 1;
    size_t a1 = s->ch_tiles_alloc, a2 = s->ch_tiles_alloc, a3 = s->ch_tiles_alloc;
    if (!grow(&s->ch_count, &a1, nt, st) || !grow(&s->ch_start, &a2, nt, st) ||
        !grow(&s->ch_fill, &a3, nt, st) ||
        !grow(&s->ch_atoms, &s->ch_atoms_alloc, (size_t)std::max(natoms, 1), st))
      return 0;
    s->ch_tiles_alloc = std::min(a1, std::min(a2, a3));
  }
  CK(cudaEventRecord(s->ev[0], st));
  CK(cudaMemsetAsync(s->d_npts, 0, sizeof(int), st));
  // The charge map and the sdh/mdh boundary values depend on the atoms only:
  // they run on the side stream while this stream builds the dielectric and
  // ion maps, and every return from here on joins the two.
  CK(cudaEventRecord(s->fork_ev, st));
  CK(cudaStreamWaitEvent(s->side, s->fork_ev, 0));
  struct SideJoin {
    pmgb_solver* s;
    int joined = 0;
    cudaError_t join() {
      if (joined) return cudaSuccess;
      joined = 1;
      cudaError_t e = cudaEventRecord(s->join_ev, s->side);
      return e == cudaSuccess ? cudaStreamWaitEvent(s->stream, s->join_ev, 0) : e;
    }
    ~SideJoin() { join(); }
  } side_join{s};
  cudaStream_t sd = s->side;
  // charge (fillcoChargeSpline2)
  if (uses_charge_map(s)) {
    // the charge map is read below (fillcoChargeMap)
    CK(cudaMemsetAsync(s->charge, 0, n * sizeof(double), st));
  } else {
    launch_charge(sd, p.chgm == PMGB_CHGM_TRIL ? 1 : (p.chgm == PMGB_CHGM_SPL4 ? 4 : 2), s->G,
                  natoms, s->d_xyz, s->d_q,
                  s->zmagic, s->ch_count, s->ch_start, s->ch_fill, s->ch_atoms, s->charge);
    note_launches(4);
  }
  if (side_bc && !side_boundary(s, sd)) return 0;
  // with coefficient maps the operator is never a plain Laplacian
  // (Vpmg_fillco, vpmg.c:5354-5361)
  const int coef_maps = uses_coef_maps(s);
  const int islap = !coef_maps && (s->ionstr < 1.0e-12) && (fabs(p.pdie - p.sdie) < 1.0e-12);
  if (coef_maps) {
    // the maps are read below (fillcoCoefMap)
  } else if (!islap && (p.srfm == PMGB_SRFM_SPL2 || p.srfm == PMGB_SRFM_SPL3 ||
                         p.srfm == PMGB_SRFM_SPL4)) {
    // spline surface: kappa and the dielectric maps together
    // (fillcoCoefSpline, fillcoCoefSpline4)
    const double ionmask = (s->ionstr > 1.0e-12) ? 1.0 : 0.0;
    const double win = (p.swin > 0.0) ? p.swin : 0.3;
    const double* coef3 = nullptr;
    if (p.srfm == PMGB_SRFM_SPL3) {
      // the 5th-order window polynomials per atom, made on the host with the
      // reference's pow() (spline3_table)
      std::vector<double> tab;
      spline3_table(natoms, h_r, s->maxIonRadius, win, tab);
      if (!grow(&s->d_spl3, &s->spl3_alloc, tab.size(), st)) return 0;
      CK(cudaMemcpyAsync(s->d_spl3, tab.data(), sizeof(double) * tab.size(),
                         cudaMemcpyHostToDevice, st));
      coef3 = s->d_spl3;
    }
    launch_spline_fill(st, p.srfm, s->G, natoms, s->d_xyz, s->d_r, s->maxIonRadius, win,
                       ionmask, p.pdie, p.sdie, coef3, s->kappa, s->epsx, s->epsy, s->epsz);
    note_launches(1);
  } else if (!islap) {
    // dielectric (fillcoCoefMolDielNoSmooth) as byte maps, then the maps
    // from them, smoothed (fillcoCoefMolDielSmooth) or not
    const int smol = p.srfm == PMGB_SRFM_SMOL;
    DielMask M;
    for (int d = 0; d < 3; d++) M.m[d] = s->dmask + d * n;
    CK(cudaMemsetAsync(s->dmask, 0, 3 * n, st));
    launch_mark_atoms_diel(st, s->G, natoms, s->d_xyz, s->d_r, p.srad, M);
    note_launches(1);
    if (p.srad > 1.0e-9) {
      // Vacc_storeParms sphere density with the Vclist probe radius
      const double clist_rad =
          ((s->maxIonRadius > p.srad) ? s->maxIonRadius : p.srad) + 0.5;
      double maxrad = 0.0, lo[3], hi[3];
      for (int a = 0; a < natoms; a++) maxrad = std::max(maxrad, h_r[a]);
      const double rad_total = maxrad + clist_rad;
      const double maxarea = 4.0 * 3.14159265358979323846 * rad_total * rad_total;
      const int nsphere = (int)ceil(maxarea * p.sdens);
      std::vector<double> ref;
      const int nref = ref_sphere(nsphere, ref);
      if (!grow(&s->d_ref, &s->ref_alloc, 3 * (size_t)nref, st)) return 0;
      s->nref = nref;
      CK(cudaMemcpyAsync(s->d_ref, ref.data(), sizeof(double) * 3 * nref,
                         cudaMemcpyHostToDevice, st));
      // atom cell grid
      for (int d = 0; d < 3; d++) { lo[d] = 1e300; hi[d] = -1e300; }
      for (int a = 0; a < natoms; a++)
        for (int d = 0; d < 3; d++) {
          lo[d] = std::min(lo[d], h_xyz[3 * a + d]);
          hi[d] = std::max(hi[d], h_xyz[3 * a + d]);
        }
      CellGrid C;
      C.cs = maxrad + p.srad + 1.0e-6;
      int ncell = 1;
      for (int d = 0; d < 3; d++) {
        C.lo[d] = lo[d] - C.cs;
        C.n[d] = (int)ceil((hi[d] - C.lo[d]) / C.cs) + 2;
        ncell *= C.n[d];
      }
      {
        size_t c1 = s->ncell_alloc, c2 = s->ncell_alloc, c3 = s->ncell_alloc;
        if (!grow(&s->cell_count, &c1, (size_t)ncell + 1, st) ||
            !grow(&s->cell_start, &c2, (size_t)ncell + 1, st) ||
            !grow(&s->cell_fillpos, &c3, (size_t)ncell + 1, st))
          return 0;
        s->ncell_alloc = std::min(c1, std::min(c2, c3));
        size_t a1 = s->cellof_alloc, a2 = s->cellof_alloc;
        if (!grow(&s->cell_of, &a1, (size_t)natoms, st) ||
            !grow(&s->cell_sorted, &a2, (size_t)natoms, st))
          return 0;
        s->cellof_alloc = std::min(a1, a2);
      }
      launch_cell_build(st, C, natoms, s->d_xyz, s->cell_count, s->cell_start,
                        s->cell_fillpos, s->cell_of, s->cell_sorted);
      note_launches(3);
      const size_t npairs = (size_t)natoms * nref;
      if (npairs >= 0x7fffffffu) {
        set_error("fillco: %d atoms x %d surface points exceed the 2^31 point list", natoms,
                  nref);
        return 0;
      }
      if (!grow(&s->sas_list, &s->sas_list_alloc, npairs, st)) return 0;
      if (!grow(&s->sas_nbr, &s->sas_nbr_alloc, sas_nbr_ints(natoms), st)) return 0;
      launch_sas_test(st, C, natoms, s->d_xyz, s->d_r, s->d_ref, nref, p.srad, s->cell_start,
                      s->cell_sorted, s->sas_nbr, s->sas_list, s->d_npts);
      note_launches(2);
      launch_sas_mark(st, s->G, natoms, s->d_xyz, s->d_r, s->d_ref, nref, p.srad,
                      s->sas_list, s->d_npts, M);
      note_launches(1);
    }
    launch_diel_maps(st, s->g, M, smol, p.pdie, p.sdie, s->epsx, s->epsy, s->epsz);
    note_launches(1);
    // ion accessibility (fillcoCoefMolIon)
    const double ionmask = (s->ionstr > 1.0e-12) ? 1.0 : 0.0;
    launch_fill_value(st, s->kappa, n, ionmask);
    note_launches(1);
    if (!(s->ionstr < 1.0e-12)) {
      launch_mark_atoms_kappa(st, s->G, natoms, s->d_xyz, s->d_r, s->maxIonRadius, s->kappa);
      note_launches(1);
    }
  } else {
    launch_fill_value(st, s->kappa, n, 0.0);
    launch_fill_value(st, s->epsx, n, p.pdie);
    launch_fill_value(st, s->epsy, n, p.pdie);
    launch_fill_value(st, s->epsz, n, p.pdie);
    note_launches(4);
  }
  if (!fill_from_maps(s)) return 0;
  // boundary values (bcCalc), except when focusing (vpmg.c:5404-5409): the
  // faces were set from the coarse solution by pmgb_focus
  if (p.bcfl == PMGB_BCFL_MAP) {
    if (!map_faces(s)) return 0;
  } else if (p.bcfl == PMGB_BCFL_FOCUS) {
    if (!s->focused) {
      set_error("pmgb_fillco: bcfl focus needs pmgb_focus with a solved coarse calculation first");
      return 0;
    }
  } else if (!side_bc) {
    if (p.bcfl != PMGB_BCFL_ZERO) {
      set_error("pmgb_fillco: bcfl %d not implemented (zero, sdh, mdh, focus and map are)",
                p.bcfl);
      return 0;
    }
    CK(cudaMemsetAsync(s->gx, 0, sizeof(double) * 2 * p.ny * p.nz, st));
    CK(cudaMemsetAsync(s->gy, 0, sizeof(double) * 2 * p.nx * p.nz, st));
    CK(cudaMemsetAsync(s->gz, 0, sizeof(double) * 2 * p.nx * p.ny, st));
  }
  CK(side_join.join());
  CK(cudaEventRecord(s->ev[1], st));
  CK(cudaGetLastError());
  s->filled = 1;
  s->built = 0;
  s->solved = 0;
  s->fill_pending = 1;
  if (wait) {
    CK(cudaStreamSynchronize(st));
    return settle_fill(s);
  }
  return 1;
}

// Atom data must be finite: a NaN or infinite coordinate, charge or radius
// would pass every on-mesh test of the fill and poison the maps.  The
// calculation is left unfilled, so a following solve fails too.
static int check_atoms(pmgb_solver* s, const char* who, int natoms, const double* xyz,
                       const double* charge, const double* radius) {
  for (int a = 0; a < natoms; a++) {
    const double v[5] = {xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2], charge[a], radius[a]};
    for (int c = 0; c < 5; c++)
      if (!std::isfinite(v[c])) {
        static const char* what[5] = {"x", "y", "z", "charge", "radius"};
        set_error("%s: atom %d has a non-finite %s", who, a, what[c]);
        s->filled = 0;
        s->solved = 0;
        return 0;
      }
  }
  return 1;
}

static int fillco_host(pmgb_solver* s, int natoms, const double* xyz, const double* charge,
                       const double* radius, int wait) {
  if (!s || natoms <= 0 || !xyz || !charge || !radius) {
    set_error("pmgb_fillco: bad arguments");
    return 0;
  }
  if (!check_atoms(s, "pmgb_fillco", natoms, xyz, charge, radius)) return 0;
  {
    size_t c1 = 3 * s->atoms_cap, c2 = s->atoms_cap, c3 = s->atoms_cap;
    if (!grow(&s->a_xyz, &c1, 3 * (size_t)natoms, s->stream) ||
        !grow(&s->a_q, &c2, (size_t)natoms, s->stream) ||
        !grow(&s->a_r, &c3, (size_t)natoms, s->stream))
      return 0;
    s->atoms_cap = std::min(c1 / 3, std::min(c2, c3));
  }
  s->d_xyz = s->a_xyz;
  s->d_q = s->a_q;
  s->d_r = s->a_r;
  s->natoms = natoms;
  CK(cudaMemcpyAsync(s->d_xyz, xyz, sizeof(double) * 3 * natoms, cudaMemcpyHostToDevice,
                     s->stream));
  CK(cudaMemcpyAsync(s->d_q, charge, sizeof(double) * natoms, cudaMemcpyHostToDevice,
                     s->stream));
  CK(cudaMemcpyAsync(s->d_r, radius, sizeof(double) * natoms, cudaMemcpyHostToDevice,
                     s->stream));
  return do_fill(s, xyz, radius, wait);
}

extern "C" int pmgb_fillco(pmgb_solver* s, int natoms, const double* xyz, const double* charge,
                           const double* radius) {
  return fillco_host(s, natoms, xyz, charge, radius, 1);
}

int pmgb::fillco_issue(pmgb_solver* s, int natoms, const double* xyz, const double* charge,
                       const double* radius) {
  return fillco_host(s, natoms, xyz, charge, radius, 0);
}

extern "C" int pmgb_fillco_device(pmgb_solver* s, int natoms, const double* d_xyz,
                                  const double* d_charge, const double* d_radius) {
  if (!s || natoms <= 0) {
    set_error("pmgb_fillco_device: bad arguments");
    return 0;
  }
  // host copies of positions and radii for the scalar setup (bounding box,
  // solute radius, sphere density)
  std::vector<double> xyz(3 * (size_t)natoms), q(natoms), r(natoms);
  CK(cudaMemcpy(xyz.data(), d_xyz, sizeof(double) * 3 * natoms, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(q.data(), d_charge, sizeof(double) * natoms, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(r.data(), d_radius, sizeof(double) * natoms, cudaMemcpyDeviceToHost));
  if (!check_atoms(s, "pmgb_fillco_device", natoms, xyz.data(), q.data(), r.data())) return 0;
  s->d_xyz = const_cast<double*>(d_xyz);
  s->d_q = const_cast<double*>(d_charge);
  s->d_r = const_cast<double*>(d_radius);
  s->natoms = natoms;
  return do_fill(s, xyz.data(), r.data(), 1);
}

extern "C" int pmgb_set_coefficients(pmgb_solver* s, const double* charge, const double* epsx,
                                     const double* epsy, const double* epsz,
                                     const double* kappa, const double* gxcf,
                                     const double* gycf, const double* gzcf) {
  if (!s) return 0;
  const size_t n = s->n;
  const pmgb_params& p = s->p;
  CK(cudaMemcpy(s->charge, charge, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->epsx, epsx, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->epsy, epsy, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->epsz, epsz, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->kappa, kappa, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->gx, gxcf, 2 * (size_t)p.ny * p.nz * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->gy, gycf, 2 * (size_t)p.nx * p.nz * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->gz, gzcf, 2 * (size_t)p.nx * p.ny * sizeof(double), cudaMemcpyHostToDevice));
  // scalar physics without atoms: ionic strength and Debye parameters
  double dummy_xyz[3] = {p.center[0], p.center[1], p.center[2]}, dummy_r = 0.0;
  phys_setup(s, 1, dummy_xyz, &dummy_r);
  s->natoms = 0;  // no atom list: the point-charge (spl0) energy is unavailable
  s->filled = 1;
  s->built = 0;
  s->solved = 0;
  return 1;
}

// ===========================================================================
// operator build (Vbuildops ido=0,1: src/pmgc/mgsubd.c:61-259)
// ===========================================================================
static int build_ops(pmgb_solver* s) {
  cudaStream_t st = s->stream;
  const size_t n = s->n;
  // ccf = zkappa2 * kappa, or 0 (Vpmg_solve, vpmg.c:436-448)
  if (s->zkappa2 > 1.0e-12) launch_ccf(st, n, s->kappa, s->zkappa2, s->ccf);
  else CK(cudaMemsetAsync(s->ccf, 0, n * sizeof(double), st));
  Level& F = s->lev[0];
  launch_build_fine(st, F.g, s->xf, s->yf, s->zf, s->epsx, s->epsy, s->epsz, s->ccf,
                    s->charge, s->gx, s->gy, s->gz, F.op[OC], F.op[OE], F.op[ON], F.op[UC],
                    F.cc, F.fc);
  // the FP64 smoother's divisor oC + cc, summed once per operator
  if (s->precision == PMGB_FP64) {
    launch_diag(st, F.g, F.op[OC], F.cc, s->dg[0]);
    note_launches(1);
  }
  note_launches(2);
  for (int l = 1; l < s->nlev; l++) {
    Level& C = s->lev[l];
    Level& P = s->lev[l - 1];
    launch_galerkin(st, P.g, P.ops(), C.g, s->d_opptrs + 14 * l);
    launch_restrict(st, P.g, P.cc, C.g, C.cc);
    launch_restrict(st, P.g, P.fc, C.g, C.fc);
    note_launches(3);
  }
  // the mixed-precision path re-derives its FP32 hierarchy from these
  if (s->mixed) mixed_mark_stale(s->mixed);
  // coarsest direct solve for the linear problem (Vbuildband, buildBd.c:57-117);
  // the mixed-precision path solves its own, coarser, level densely instead
  s->mgsolv = (s->p.nonlin || s->precision == PMGB_MIXED) ? 0 : 1;
  if (s->mgsolv == 1) {
    // a coarsest level above 512 unknowns is solved by exact refinement
    // instead: the banded factor and its substitutions are sequential
    const Grid gc = s->lev[s->nlev - 1].g;
    if ((size_t)(gc.nx - 2) * (gc.ny - 2) * (gc.nz - 2) > 512 && s->tune[4] == 0 &&
        coarse_exact_prepare(s))
      s->mgsolv = 2;
  }
  if (s->mgsolv == 1) {
    Level& C = s->lev[s->nlev - 1];
    const int ex = C.g.nx - 2, exy = (C.g.nx - 2) * (C.g.ny - 2);
    const int nb = (C.g.nx - 2) * (C.g.ny - 2) * (C.g.nz - 2);
    const int m = exy + ex + 1, lda = m + 1;
    if (nb != s->bn || m != s->bm) {
      dfree(s->band);
      s->band = nullptr;
      if (!dalloc(&s->band, (size_t)lda * nb + nb)) return 0;
    }
    s->bn = nb;
    s->bm = m;
    s->blda = lda;
    launch_band_build(st, C.g, C.ops(), s->band, m, lda);
    launch_band_factor(st, s->band, nb, m, lda, s->d_info);
    note_launches(2);
    int info = 0;
    CK(cudaMemcpyAsync(&info, s->d_info, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (info != 0) s->mgsolv = 0;  // "Changing your mgsolv to iterative" (mgsubd.c:248-254)
  }
  CK(cudaGetLastError());
  s->built = 1;
  return 1;
}

int pmgb::solver_build(pmgb_solver* s) { return build_ops(s); }

// ===========================================================================
// one V-cycle (body of the do-loop of Vmvcs, src/pmgc/mgcsd.c:312-562)
// ===========================================================================
// ordered 27-point smoothing of level l (two sweeps, optional residual):
// the plane-parallel wavefront on every level that fits it, else the
// one-cluster wavefront (PMGB_TUNE_GS27_PLANES = 1: always the latter)
static int gs27_smooth(pmgb_solver* s, cudaStream_t st, int l, const double* cc,
                       const double* fc, double* x, double* r, int first_parity) {
  const Level& L = s->lev[l];
  if (s->tune[PMGB_TUNE_GS27_PLANES] == 0 && s->mail_off[l] >= 0 &&
      launch_gs27_mail(st, L.g, L.ops(), cc, fc, x, r, 2, first_parity,
                       s->d_wave + kWaveCounterBase + (size_t)l * kWavePlanesMax,
                       reinterpret_cast<int*>(s->d_wave), s->tune[PMGB_TUNE_GS27_LAG],
                       s->d_mail + s->mail_off[l])) {
    s->wave_used = 1;
    return 1;
  }
  (void)cudaGetLastError();  // a refused launch above leaves no error behind
  if (s->tune[PMGB_TUNE_GS27_PLANES] != 1 && wave_planes_fit(L.g)) {
    s->wave_used = 1;
    return launch_gs27_planes(st, L.g, L.ops(), cc, fc, x, r, 2, first_parity,
                              s->d_wave + kWaveCounterBase + (size_t)l * kWavePlanesMax,
                              reinterpret_cast<int*>(s->d_wave),
                              s->tune[PMGB_TUNE_GS27_PLANES_POLL], s->tune[PMGB_TUNE_GS27_LAG]);
  }
  return launch_gs27_wave(st, L.g, L.ops(), cc, fc, x, r, 2, first_parity, s->plan[l]);
}

static int vcycle_body(pmgb_solver* s, int newton) {
  cudaStream_t st = s->stream;
  const int nlev = s->nlev;
  Level& F = s->lev[0];
  auto CC = [&](int l) -> double* { return newton ? s->lev[l].cp : s->lev[l].cc; };
  auto X = [&](int l) -> double* { return newton ? s->lev[l].xt : s->lev[l].x; };
  double* FC0 = newton ? F.rhs : F.fc;
  const double* DG = s->dg[newton ? 1 : 0];
  const int colour_passes = s->tune[5] == 1 || !gs7_sweep_supported(F.g);
  long long k = 0;
  // nu1 = 2 pre-smoothings on the fine level, then the residual
  if (colour_passes) {
    for (int sw = 0; sw < 2; sw++) {
      launch_gs7_colour(st, F.g, F.ops(), CC(0), FC0, X(0), 1);
      launch_gs7_colour(st, F.g, F.ops(), CC(0), FC0, X(0), 0);
      k += 2;
    }
    launch_resid(st, F.g, F.ops(), CC(0), FC0, X(0), s->w1);
    k += 1;
  } else {
    // two single-pass sweeps, x -> xs -> x
    if (!launch_gs7_sweep64(st, F.g, F.ops(), DG, FC0, X(0), s->xs, 1, s->tune[6], s->tune[12]) ||
        !launch_gs7_sweep64(st, F.g, F.ops(), DG, FC0, s->xs, X(0), 1, s->tune[6], s->tune[12])) {
      set_error("gs7 sweep launch failed");
      return 0;
    }
    launch_resid(st, F.g, F.ops(), CC(0), FC0, X(0), s->w1);
    k += 3;
  }
  launch_copy_interior(st, F.g, s->w1, F.w0);
  k += 1;
  // down
  for (int l = 1; l < nlev; l++) {
    Level& C = s->lev[l];
    Level& P = s->lev[l - 1];
    launch_restrict(st, P.g, s->w1, C.g, C.w0);
    k++;
    if (l != nlev - 1) {
      launch_zero(st, X(l), C.g.n());
      if (!gs27_smooth(s, st, l, CC(l), C.w0, X(l), s->w1, 1)) {
        set_error("gs27 launch failed at level %d", l);
        return 0;
      }
      k += 2;
    }
  }
  // coarsest
  {
    Level& C = s->lev[nlev - 1];
    if (s->mgsolv == 1) {
      launch_band_solve(st, C.g, s->band, s->bn, s->bm, s->blda, C.w0, X(nlev - 1));
      k++;
    } else if (s->mgsolv == 2) {
      if (!launch_coarse_exact(s, st, CC(nlev - 1), C.w0, X(nlev - 1))) return 0;
      k++;
    } else {
      launch_zero(st, X(nlev - 1), C.g.n());
      if (!launch_cg_coarse(st, C.g, C.ops(), CC(nlev - 1), C.w0, X(nlev - 1), s->w1, s->w2,
                            s->w3, 100, 2.220446049250313e-16, s->d_iters,
                            s->tune[PMGB_TUNE_CG_CLUSTER])) {
        set_error("coarse CG launch failed");
        return 0;
      }
      k += 2;
    }
  }
  // up
  for (int l = nlev - 2; l >= 0; l--) {
    Level& C = s->lev[l + 1];
    Level& P = s->lev[l];
    launch_xdamp_sums(st, C.g, C.ops(), CC(l + 1), X(l + 1), C.w0, s->part,
                      s->d_wave + kWaveDampTicket, s->scal + S_XNUM_L + l,
                      s->scal + S_XDEN_L + l);
    launch_interp_axpy(st, C.g, X(l + 1), P.g, X(l), s->scal + S_XNUM_L + l,
                       s->scal + S_XDEN_L + l);
    k += 2;
    if (l == 0) {
      if (colour_passes) {
        for (int sw = 0; sw < 2; sw++) {
          launch_gs7_colour(st, F.g, F.ops(), CC(0), FC0, X(0), 0);
          launch_gs7_colour(st, F.g, F.ops(), CC(0), FC0, X(0), 1);
          k += 2;
        }
      } else {
        if (!launch_gs7_sweep64(st, F.g, F.ops(), DG, FC0, X(0), s->xs, 0, s->tune[6], s->tune[12]) ||
            !launch_gs7_sweep64(st, F.g, F.ops(), DG, FC0, s->xs, X(0), 0, s->tune[6], s->tune[12])) {
          set_error("gs7 sweep launch failed");
          return 0;
        }
        k += 2;
      }
    } else {
      if (!gs27_smooth(s, st, l, CC(l), P.w0, X(l), nullptr, 0)) {
        set_error("gs27 launch failed at level %d", l);
        return 0;
      }
      k++;
    }
  }
  // stopping test residual
  launch_resid(st, F.g, F.ops(), CC(0), FC0, X(0), s->w1);
  launch_nrm1(st, F.g, s->w1, s->part, s->scal + S_RSNRM);
  k += 3;
  s->vc_kernels[newton] = k;
  return 1;
}

static int ensure_graph(pmgb_solver* s, int newton) {
  if (s->vc_exec[newton] && s->vc_mgsolv[newton] != s->mgsolv) {
    cudaGraphExecDestroy(s->vc_exec[newton]);
    s->vc_exec[newton] = nullptr;
  }
  if (s->vc_exec[newton]) return 1;
  s->vc_mgsolv[newton] = s->mgsolv;
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  int ok = vcycle_body(s, newton);
  cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
  if (!ok) return 0;
  if (e != cudaSuccess) {
    set_error("graph capture failed: %s", cudaGetErrorString(e));
    return 0;
  }
  CK(cudaGraphInstantiate(&s->vc_exec[newton], graph, 0));
  cudaGraphDestroy(graph);
  return 1;
}

// V-cycles until the stopping test holds (Vmvcs).  istop0: rsden = 1
// (istop = 0, the Newton inner solve) instead of ||f||_1.
static int vcycles(pmgb_solver* s, int newton, double errtol, int itmax, int istop0,
                   int* iters_out) {
  Level& F = s->lev[0];
  double* FC0 = newton ? F.rhs : F.fc;
  double rsden = 1.0, rsnrm;
  if (!istop0) {
    launch_nrm1(s->stream, F.g, FC0, s->part, s->scal + S_RSDEN);
    note_launches(2);
    if (!read_scalar(s, S_RSDEN, &rsden)) return 0;
  }
  if (rsden == 0.0) rsden = 1.0;
  rsnrm = rsden;
  s->reslog.push_back(rsnrm / rsden);
  if (!ensure_graph(s, newton)) return 0;
  int iters = 0;
  do {
    CK(cudaGraphLaunch(s->vc_exec[newton], s->stream));
    note_launches(s->vc_kernels[newton]);
    if (!read_scalar(s, S_RSNRM, &rsnrm)) return 0;
    iters++;
    s->st.vcycles++;
    s->reslog.push_back(rsnrm / rsden);
    if (!(rsnrm == rsnrm)) {
      set_error("non-finite residual in V-cycle %d", iters);
      return 0;
    }
  } while (iters < itmax && (rsnrm / rsden) > errtol);
  s->st.rel_residual = rsnrm / rsden;
  *iters_out = iters;
  return 1;
}

// ||N(x)||_1 with r = N(x); with cp not null also c'(x) (one pass)
static int nresid_norm(pmgb_solver* s, const double* x, double* r, double* out,
                       double* cp = nullptr) {
  Level& F = s->lev[0];
  launch_nresid_nrm1(s->stream, F.g, F.ops(), F.cc, F.fc, x, r, s->ions, s->part,
                     s->scal + S_NRM, cp);
  note_launches(2);
  return read_scalar(s, S_NRM, out);
}


// Damped inexact Newton (Vnewton, src/pmgc/newtond.c:162-548).  The inner
// linear solve of each step is the FP64 V-cycle iteration (Vmvcs with
// istop = 0), or FP32 V-cycles with FP64 refinement when mixed != 0.
int pmgb::newton_driver(pmgb_solver* s, double errtol, int itmax, int mixed) {
  cudaStream_t st = s->stream;
  Level& F = s->lev[0];
  const size_t n = s->n;
  double rsden, rsnrm, xnorm_old, xnorm_new, xnorm_med = 0.0;
  // rsden = ||N(0)||_1
  CK(cudaMemsetAsync(s->nw_ws, 0, n * sizeof(double), st));
  if (!nresid_norm(s, s->nw_ws, s->nw_keepx, &rsden)) return 0;
  if (rsden == 0.0) rsden = 1.0;
  rsnrm = rsden;
  s->reslog.push_back(rsnrm / rsden);
  // the residual of the current iterate is the next Jacobian system's
  // right-hand side: it is written there directly where no damping trial
  // can replace it, else copied from the kept trial
  if (!nresid_norm(s, F.x, F.rhs, &xnorm_old)) return 0;
  int rhs_ready = 1;
  int iters = 0, idamp = 1;
  // work vectors of the damping loop: trial iterate and residual, and the
  // best ones kept; "keep" is a swap of the two pairs (no copies)
  double *ws = s->nw_ws, *r0 = s->nw_r0, *keepx = s->nw_keepx, *keepr = s->nw_keepr;
  int cp_ready = 0;  // F.cp already holds c'(F.x) (computed with the last residual)
  for (;;) {
    iters++;
    // Vgetjac (newtond.c:550-598).  Only the fine right-hand side is used:
    // every coarse level's right-hand side is the restricted residual of
    // the V-cycle itself.
    if (!rhs_ready) {
      launch_copy_interior(st, F.g, r0, F.rhs);
      note_launches(1);
    }
    rhs_ready = 0;
    if (!cp_ready) {
      launch_dcvec(st, F.g, F.cc, F.x, F.cp, s->ions);
      note_launches(1);
    }
    if (!mixed) {
      launch_diag(st, F.g, F.op[OC], F.cp, s->dg[1]);
      note_launches(1);
    }
    for (int l = 1; l < s->nlev; l++) {
      launch_restrict(st, s->lev[l - 1].g, s->lev[l - 1].cp, s->lev[l].g, s->lev[l].cp);
      note_launches(1);
    }
    const double errtol_s =
        (0.9 * xnorm_old <= 1.0 * pow(xnorm_old, 2.0)) ? 0.9 * xnorm_old : 1.0 * pow(xnorm_old, 2.0);
    CK(cudaMemsetAsync(F.xt, 0, n * sizeof(double), st));
    int it_s = 0;
    if (mixed) {
      if (!mixed_newton_inner(s, errtol_s)) return 0;
    } else {
      if (!vcycles(s, 1, errtol_s, 1000, 1, &it_s)) return 0;
    }
    cp_ready = 0;
    if (idamp == 1) {
      double damp = 1.0;
      int iter_d = 0, mode = 0;
      // ws = x + damp xt (the reference's copy then axpy, newtond.c:430-445)
      launch_xpay_interior(st, F.g, F.x, damp, F.xt, ws);
      note_launches(1);
      if (!nresid_norm(s, ws, r0, &xnorm_new)) return 0;
      while (iter_d < 10) {
        if (mode == 0) {
          if (xnorm_new < xnorm_old) mode = 1;
        } else if (xnorm_new > xnorm_med) {
          break;
        }
        // keep this trial: its iterate and residual become the kept pair
        std::swap(ws, keepx);
        std::swap(r0, keepr);
        xnorm_med = xnorm_new;
        damp = damp / 2.0;
        launch_xpay_interior(st, F.g, F.x, damp, F.xt, ws);
        note_launches(1);
        if (!nresid_norm(s, ws, r0, &xnorm_new)) return 0;
        iter_d++;
      }
      launch_copy_interior(st, F.g, keepx, F.x);
      note_launches(1);
      std::swap(keepr, r0);
      xnorm_new = xnorm_med;
      xnorm_old = xnorm_new;
      if ((iter_d - 1) == 0) idamp = 0;
    } else {
      launch_axpy_interior(st, F.g, nullptr, 1.0, F.xt, F.x);
      note_launches(1);
      // the residual pass also gives c'(x) for the next Jacobian
      if (!nresid_norm(s, F.x, F.rhs, &xnorm_new, F.cp)) return 0;
      cp_ready = 1;
      rhs_ready = 1;
      xnorm_old = xnorm_new;
    }
    rsnrm = xnorm_new;
    s->reslog.push_back(rsnrm / rsden);
    if ((rsnrm / rsden) <= errtol) break;
    if (iters >= itmax) break;
  }
  s->nw_ws = ws;
  s->nw_r0 = r0;
  s->nw_keepx = keepx;
  s->nw_keepr = keepr;
  s->st.rel_residual = rsnrm / rsden;
  s->st.newton_iters = iters;
  return 1;
}

// Reads (and clears) the count of plane-wavefront waits that ran out; a
// nonzero count fails the solve (the iterates are not the ordered sweep's).
static int wave_check(pmgb_solver* s) {
  // wave_used stays set: graphs captured with the plane kernel replay it in
  // every later solve without passing through gs27_smooth again
  if (!s->wave_used) return 1;
  int nerr = 0;
  CK(cudaMemcpyAsync(&nerr, s->d_wave, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (nerr) {
    // the counters of the levels may now disagree: restart them all
    wave_reset(s, s->stream);
    CK(cudaStreamSynchronize(s->stream));
    set_error("%d bounded device waits ran out (gs27 plane wavefront)", nerr);
    return 0;
  }
  return 1;
}

// Testing hook: shift one plane's step counter so that its neighbours'
// waits run out on the next solve (a failure made without a device fault).
extern "C" int pmgb_debug_shift_wave_counter(pmgb_solver* s, int level, int plane, int delta) {
  if (!s || level < 0 || level >= s->nlev || plane < 0 || plane >= kWavePlanesMax) {
    set_error("pmgb_debug_shift_wave_counter: bad arguments");
    return 0;
  }
  unsigned* c = s->d_wave + kWaveCounterBase + (size_t)level * kWavePlanesMax + plane;
  unsigned v = 0;
  CK(cudaMemcpy(&v, c, sizeof(v), cudaMemcpyDeviceToHost));
  v += (unsigned)delta;
  CK(cudaMemcpy(c, &v, sizeof(v), cudaMemcpyHostToDevice));
  return 1;
}

extern "C" int pmgb_solve(pmgb_solver* s) {
  if (!s) return 0;
  if (!s->filled) {
    set_error("pmgb_solve: call pmgb_fillco first (Vpmg_solve requires filled maps)");
    return 0;
  }
  cudaStream_t st = s->stream;
  s->reslog.clear();
  s->st.vcycles = 0;
  s->st.newton_iters = 0;
  s->st.refinements = 0;
  CK(cudaEventRecord(s->ev[2], st));
  if (!s->built && !build_ops(s)) return 0;
  CK(cudaEventRecord(s->ev[3], st));
  s->st.coarse_method = (s->precision == PMGB_MIXED) ? 2 : (s->mgsolv == 2 ? 3 : s->mgsolv);
  const double errtol = (s->p.etol > 0.0) ? s->p.etol : 1.0e-6;
  // Vpmgp itmax (vpmgp.c:131): V-cycles (LPBE) or Newton steps (NPBE)
  const int itmax = (s->p.itmax > 0) ? s->p.itmax : 200;
  s->st.converged = 0;
  int ok;
  if (s->precision == PMGB_MIXED) {
    ok = mixed_solve(s, errtol, itmax);
  } else {
    // u = 0 (Vazeros + VfboundPMG00, mgdrvd.c:462-483 / newdrvd.c:300)
    CK(cudaMemsetAsync(s->lev[0].x, 0, s->n * sizeof(double), st));
    if (!s->p.nonlin) {
      int iters = 0;
      ok = vcycles(s, 0, errtol, itmax, 0, &iters);
    } else {
      ok = newton_driver(s, errtol, itmax, 0);
    }
  }
  if (!ok) {
    // a wavefront wait that ran out is the cause to report (and its
    // counters are restarted)
    wave_check(s);
    return 0;
  }
  // restore Dirichlet values (VfboundPMG, mgdrvd.c:557)
  launch_fbound(st, s->g, s->lev[0].x, s->gx, s->gy, s->gz);
  note_launches(1);
  CK(cudaEventRecord(s->ev[4], st));
  if (!wave_check(s)) return 0;
  CK(cudaStreamSynchronize(st));
  CK(cudaGetLastError());
  s->st.t_setup_ms = elapsed_ms(s->ev[2], s->ev[3]);
  s->st.t_solve_ms = elapsed_ms(s->ev[3], s->ev[4]);
  // like Vpmg_solve, a solve that stops at itmax still succeeds (the
  // reference only sets ierror, mgcsd.c:564); the stats say so
  s->st.converged = (s->st.rel_residual <= errtol) ? 1 : 0;
  s->solved = 1;
  return 1;
}

// Vpmg_energy (src/mg/vpmg.c:1248-1277) with extFlag = 1: the external
// terms are those pmgb_focus left (zero for a non-focused calculation)
extern "C" int pmgb_energy(pmgb_solver* s, double* energy_kT) {
  if (!s || !s->solved) {
    set_error("pmgb_energy: no solution");
    return 0;
  }
  cudaStream_t st = s->stream;
  EnergyArgs a;
  a.g = s->g;
  a.u = s->lev[0].x;
  a.charge = s->charge;
  a.epsx = s->epsx;
  a.epsy = s->epsy;
  a.epsz = s->epsz;
  a.kappa = s->kappa;
  a.wx = s->wx;
  a.wy = s->wy;
  a.wz = s->wz;
  a.hx = s->p.hx;
  a.hy = s->p.hy;
  a.hz = s->p.hz;
  a.nonlin = (s->p.nonlin && s->ionstr > 0.) ? 1 : 0;
  a.ions = s->ions_e;
  a.zks2 = (s->ionstr > 0.0) ? 0.5 * s->zkappa2 / s->ionstr : 0.0;
  CK(cudaEventRecord(s->ev[5], st));
  launch_energy_sums(st, a, s->part, s->scal + S_E0);
  note_launches(2);
  double sums[4];
  CK(cudaMemcpyAsync(sums, s->scal + S_E0, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaEventRecord(s->ev[6], st));
  CK(cudaStreamSynchronize(st));
  const pmgb_params& p = s->p;
  double qf = sums[0] * p.hx * p.hy * p.hz / s->zmagic;
  if (p.chgm != PMGB_CHGM_SPL2 && !uses_charge_map(s)) {
    // Vpmg_qfEnergyPoint (vpmg.c:1704-1789): charges at the atoms (every
    // discretisation but spl2 without a charge map, Vpmg_qfEnergy 1692-1699)
    if (s->natoms <= 0 || !s->d_xyz) {
      set_error("pmgb_energy: chgm spl0/spl4 needs the atom list (pmgb_fillco)");
      return 0;
    }
    launch_qf_point(st, s->G, s->natoms, s->d_xyz, s->d_q, s->lev[0].x, s->part,
                    s->scal + S_TMP);
    note_launches(2);
    CK(cudaMemcpyAsync(&qf, s->scal + S_TMP, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  qf += s->ext_qf;
  double diel = 0.0, qm = 0.0, e;
  if (a.nonlin) {
    diel = 0.5 * sums[1] * p.hx * p.hy * p.hz;
    diel = diel / s->zmagic;
    diel += s->ext_di;
    if (!(s->zkappa2 < 1.0e-9)) {
      if (sums[3] > 0.0) {
        set_error("pmgb_energy: clamped exponentials in the mobile-ion energy");
        return 0;
      }
      qm = sums[2] * p.hx * p.hy * p.hz;
      qm = qm / s->zmagic;
      qm += s->ext_qm;
    }
    e = qf - diel - qm;
  } else {
    e = 0.5 * qf;
  }
  s->st.qf = qf;
  s->st.diel = diel;
  s->st.qm = qm;
  s->st.energy_kT = e;
  s->st.t_energy_ms = elapsed_ms(s->ev[5], s->ev[6]);
  *energy_kT = e;
  return 1;
}

extern "C" int pmgb_get_potential(pmgb_solver* s, double* u) {
  if (!s || !s->solved || !u) {
    set_error("pmgb_get_potential: no solution");
    return 0;
  }
  CK(cudaMemcpyAsync(u, s->lev[0].x, s->n * sizeof(double), cudaMemcpyDeviceToHost,
                     s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 1;
}

extern "C" int pmgb_get_maps(pmgb_solver* s, double* maps, double* faces) {
  if (!s || !s->filled) {
    set_error("pmgb_get_maps: not filled");
    return 0;
  }
  const size_t n = s->n;
  const pmgb_params& p = s->p;
  CK(cudaStreamSynchronize(s->stream));
  if (maps) {
    CK(cudaMemcpy(maps, s->charge, n * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(maps + n, s->epsx, n * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(maps + 2 * n, s->epsy, n * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(maps + 3 * n, s->epsz, n * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(maps + 4 * n, s->kappa, n * sizeof(double), cudaMemcpyDeviceToHost));
  }
  if (faces) {
    const size_t fx = 2 * (size_t)p.ny * p.nz, fy = 2 * (size_t)p.nx * p.nz;
    const size_t fz = 2 * (size_t)p.nx * p.ny;
    CK(cudaMemcpy(faces, s->gx, fx * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(faces + fx, s->gy, fy * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(faces + fx + fy, s->gz, fz * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return 1;
}

extern "C" int pmgb_get_stats(pmgb_solver* s, pmgb_stats* out) {
  if (!s || !out) return 0;
  if (!settle_fill(s)) return 0;
  *out = s->st;
  return 1;
}

extern "C" int pmgb_get_residual_history(pmgb_solver* s, double* buf, int cap) {
  if (!s) return 0;
  const int n = (int)s->reslog.size();
  for (int i = 0; i < n && i < cap; i++) buf[i] = s->reslog[i];
  return n;
}

extern "C" int pmgb_solve_molecule(const pmgb_params* params, int precision, int natoms,
                                   const double* xyz, const double* charge,
                                   const double* radius, double* energy_kT, double* u,
                                   pmgb_stats* stats) {
  pmgb_solver* s = nullptr;
  if (!pmgb_create(params, precision, &s)) return 0;
  int ok = pmgb_fillco(s, natoms, xyz, charge, radius) && pmgb_solve(s) &&
           pmgb_energy(s, energy_kT);
  if (ok && u) ok = pmgb_get_potential(s, u);
  if (ok && stats) pmgb_get_stats(s, stats);
  pmgb_destroy(s);
  return ok;
}

extern "C" int pmgb_time_kernel(pmgb_solver* s, int which, int reps, double* ms,
                                double* bytes) {
  if (!s || !s->built || reps < 1) {
    set_error("pmgb_time_kernel: solve first");
    return 0;
  }
  if ((which == PMGB_K_GS7_FP32 || which == PMGB_K_VCYCLE_TAIL ||
       which == PMGB_K_GS7_SWEEP_FP32) &&
      s->precision != PMGB_MIXED) {
    set_error("pmgb_time_kernel: kernel %d belongs to the mixed-precision path", which);
    return 0;
  }
  cudaStream_t st = s->stream;
  Level& F = s->lev[0];
  const double fint = (double)(F.g.nx - 2) * (F.g.ny - 2) * (F.g.nz - 2);
  double b = 0.0;
  if (which == PMGB_K_GS7_SWEEP_FP32 && !mixed_prepare_sweep(s)) return 0;
  CK(cudaStreamSynchronize(st));
  CK(cudaEventRecord(s->ev[6], st));
  for (int r = 0; r < reps; r++) {
    switch (which) {
      case PMGB_K_GS7_FP64:
        // reads oE oN uC oC cc fc and x, writes x: 56 B per point per sweep
        launch_gs7_colour(st, F.g, F.ops(), F.cc, F.fc, F.x, r & 1);
        b = 28.0 * fint;
        break;
      case PMGB_K_GS27_WAVE: {
        if (s->nlev < 3) { set_error("pmgb_time_kernel: needs >= 3 levels"); return 0; }
        Level& C = s->lev[1];
        const double cint = (double)(C.g.nx - 2) * (C.g.ny - 2) * (C.g.nz - 2);
        if (!gs27_smooth(s, st, 1, C.cc, C.w0, C.x, s->w1, 1))
          return 0;
        // 14 coefficients + cc + f read, x read and written: 144 B per point
        // per sweep; the residual pass reads the same and writes r
        b = (2.0 * 144.0 + 144.0) * cint;
        break;
      }
      case PMGB_K_RESID_FP64:
        launch_resid(st, F.g, F.ops(), F.cc, F.fc, F.x, s->w1);
        b = 56.0 * fint;
        break;
      case PMGB_K_CG_COARSE: {
        Level& C = s->lev[s->nlev - 1];
        const double cint = (double)(C.g.nx - 2) * (C.g.ny - 2) * (C.g.nz - 2);
        if (!launch_cg_coarse(st, C.g, C.ops(), C.cc, C.w0, C.x, s->w1, s->w2, s->w3, 100,
                              2.220446049250313e-16, s->d_iters, s->tune[PMGB_TUNE_CG_CLUSTER]))
          return 0;
        b = 100.0 * (16.0 + 2.0 + 6.0) * 8.0 * cint;
        break;
      }
      case PMGB_K_GS7_FP32:
        if (!mixed_time_gs7(s, r & 1, &b)) return 0;
        break;
      case PMGB_K_VCYCLE_TAIL:
        if (!mixed_time_tail(s, &b)) return 0;
        break;
      case PMGB_K_GS7_SWEEP_FP64:
        // one full sweep: oE oN uC D=oC+cc fc and x read, x written: 56 B per point
        if (r == 0 && s->precision != PMGB_FP64) launch_diag(st, F.g, F.op[OC], F.cc, s->dg[0]);
        if (!launch_gs7_sweep64(st, F.g, F.ops(), s->dg[0], F.fc, (r & 1) ? s->xs : F.x,
                                (r & 1) ? F.x : s->xs, 1, s->tune[6], s->tune[12])) {
          set_error("gs7 sweep launch failed");
          return 0;
        }
        b = 56.0 * fint;
        break;
      case PMGB_K_GS7_SWEEP_FP32:
        if (!mixed_time_gs7_sweep(s, &b)) return 0;
        break;
      default:
        set_error("pmgb_time_kernel: unknown kernel %d", which);
        return 0;
    }
  }
  CK(cudaEventRecord(s->ev[7], st));
  CK(cudaEventSynchronize(s->ev[7]));
  CK(cudaGetLastError());
  *ms = elapsed_ms(s->ev[6], s->ev[7]) / reps;
  *bytes = b;
  note_launches(reps);
  return 1;
}

extern "C" int pmgb_set_tuning(int key, int value) {
  if (key < 0 || key >= PMGB_TUNE_NKEYS) {
    set_error("pmgb_set_tuning: bad key %d", key);
    return 0;
  }
  if ((key == PMGB_TUNE_MIXED_COARSE_SWEEPS || key == PMGB_TUNE_MIXED_FINE_SWEEPS) &&
      (value < 1 || value > 4)) {
    set_error("pmgb_set_tuning: sweeps must be 1..4");
    return 0;
  }
  if (key == PMGB_TUNE_GS27_LAG && (value < 4 || value > 64)) {
    set_error("pmgb_set_tuning: the wavefront lag must be 4..64");
    return 0;
  }
  g_tune[key] = value;
  return 1;
}

extern "C" int pmgb_get_tuning(int key) {
  if (key < 0 || key >= PMGB_TUNE_NKEYS) return -1;
  return g_tune[key];
}

extern "C" int pmgb_solver_set_tuning(pmgb_solver* s, int key, int value) {
  if (!s || key < 0 || key >= PMGB_TUNE_NKEYS) {
    set_error("pmgb_solver_set_tuning: bad solver or key %d", key);
    return 0;
  }
  if ((key == PMGB_TUNE_MIXED_COARSE_SWEEPS || key == PMGB_TUNE_MIXED_FINE_SWEEPS) &&
      (value < 1 || value > 4)) {
    set_error("pmgb_solver_set_tuning: sweeps must be 1..4");
    return 0;
  }
  if (key == PMGB_TUNE_CG_CLUSTER && value != 0 && value != 1 && value != 4 && value != 8 &&
      value != 16) {
    set_error("pmgb_solver_set_tuning: CG cluster must be 0, 1, 4, 8 or 16");
    return 0;
  }
  if (key == PMGB_TUNE_GS27_LAG && (value < 4 || value > 64)) {
    set_error("pmgb_solver_set_tuning: the wavefront lag must be 4..64");
    return 0;
  }
  if (s->tune[key] == value) return 1;
  CK(cudaStreamSynchronize(s->stream));
  s->tune[key] = value;
  // launch shapes are baked into the captured V-cycle graphs
  for (int m = 0; m < 2; m++)
    if (s->vc_exec[m]) {
      cudaGraphExecDestroy(s->vc_exec[m]);
      s->vc_exec[m] = nullptr;
    }
  for (int l = 0; l < s->nlev; l++) s->plan[l] = plan_for(s->lev[l].g, s->tune);
  if (s->mixed) {
    // the FP32 hierarchy and its graphs are rebuilt with the new shapes
    mixed_destroy(s->mixed);
    s->mixed = nullptr;
    s->built = 0;
    s->solved = 0;
  }
  return 1;
}

extern "C" int pmgb_solver_get_tuning(pmgb_solver* s, int key) {
  if (!s || key < 0 || key >= PMGB_TUNE_NKEYS) return -1;
  return s->tune[key];
}

extern "C" const char* pmgb_last_error(void) { return g_err; }

extern "C" long long pmgb_launch_count(int reset) {
  long long v = g_launches;
  if (reset) g_launches = 0;
  return v;
}
