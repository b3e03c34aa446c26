// Spline-based molecular surfaces (srfm spl2, spl3, spl4) and the forces on the atoms.
//
// Surface: fillcoCoefSpline (src/mg/vpmg.c:4631-4854); fillcoCoefSpline3
// (7525-7840) and fillcoCoefSpline4 (7052-7366) are the same with a 5th- and a
// 7th-order polynomial on the window.  kappa, epsx, epsy
// and epsz start at 1 everywhere; for every on-mesh atom with a positive
// radius, in atom order, each grid point inside the atom's search box has
// its values multiplied by the cubic spline accessibility of the point (0
// well inside the atom, 1 outside the window, 0.75 s^2/w^2 - 0.25 s^3/w^3
// between), each map only while it is above VPMGSMALL; kappa uses the
// radius inflated by the largest ion radius, the eps maps are evaluated at
// the staggered points (i+1/2, j, k), (i, j+1/2, k), (i, j, k+1/2).  Then
// kappa *= ionmask and eps = (epsw - epsp) eps + epsp.
//
// The reference scatters atom by atom; here a CTA owns a block of grid
// points, scans the atoms in index order and keeps those whose search box
// (the reference's own imin..kmax) meets the block, in order, in shared
// memory.  Each thread applies them to its points in that order with the
// reference's expressions, so each point sees the same factors in the same
// order and the maps are bitwise equal.
//
// Forces: Vpmg_qfForce (vpmg.c:5862-5904 with qfForceSpline1 5906-6041,
// qfForceSpline2 6043-6154 and qfForceSpline4 6156-6272), Vpmg_dbForce (5605-5860) and Vpmg_ibForce
// (5440-5603) with Vacc_splineAccGradAtomNorm (src/generic/vacc.c:314-373).
// One thread per atom walks the reference's loops in their order, so each
// sum is taken in the reference's order.
#include <algorithm>
#include <vector>

#include "apbs_b200.h"
#include "fill_kernels.cuh"
#include "solver_internal.cuh"

namespace pmgb {

namespace {

constexpr double kPmgSmall = 1e-12;  // VPMGSMALL (src/generic/vhal.h)
constexpr double kVSmall = 1e-9;     // VSMALL (maloc)
constexpr double kExpMax = 85.0;     // EXPMAX / -EXPMIN (src/generic/vcap.h)

// ---------------------------------------------------------------------------
// srfm spl2 fill
// ---------------------------------------------------------------------------
struct SplineArgs {
  FillGeom G;
  int natoms;
  const double* xyz;
  const double* r;
  double irad;      // largest ion radius
  double win;       // spline window
  double ionmask;   // 1 if the ionic strength is positive
  double epsp, epsw;
  const double* c3;  // spl3: spline3_table's 18 coefficients per atom
  double *kappa, *epsx, *epsy, *epsz;
};

struct SplAtom {
  double pos[3];  // position relative to the grid origin
  double arad;
  int box[6];     // imin, imax, jmin, jmax, kmin, kmax
  int idx;        // atom index
};

constexpr int kBX = 8, kBY = 8, kBZ = 8;        // grid points per CTA block
constexpr int kSplThreads = 256;                 // two points per thread
constexpr int kSplCap = 512;                     // candidate atoms held at once

// the search box of atom a (fillcoCoefSpline), or false if the atom is
// skipped (off the mesh or of zero radius)
__device__ __forceinline__ bool spline_atom(const SplineArgs& A, int a, SplAtom& s) {
  const FillGeom& G = A.G;
  const double* apos = A.xyz + 3 * a;
  const double arad = A.r[a];
  if ((apos[0] <= G.xmin[0]) || (apos[0] >= G.xmax[0]) || (apos[1] <= G.xmin[1]) ||
      (apos[1] >= G.xmax[1]) || (apos[2] <= G.xmin[2]) || (apos[2] >= G.xmax[2]))
    return false;
  if (!(arad > kPmgSmall)) return false;
  for (int d = 0; d < 3; d++) s.pos[d] = apos[d] - G.xmin[d];
  s.arad = arad;
  s.idx = a;
  const double itot = A.irad + arad + A.win;
  const double stot = arad + A.win;
  const double rtot = (itot > stot) ? itot : stot;
  const int n[3] = {G.g.nx, G.g.ny, G.g.nz};
  for (int d = 0; d < 3; d++) {
    const double dd = rtot + 0.5 * G.h[d];
    s.box[2 * d] = max(0, (int)floor((s.pos[d] - dd) / G.h[d]));
    s.box[2 * d + 1] = min(n[d] - 1, (int)ceil((s.pos[d] + dd) / G.h[d]));
  }
  return true;
}

__device__ __forceinline__ double spline_value(double dist, double rad, double win, double w2i,
                                               double w3i) {
  const double sm = dist - rad + win;
  const double sm2 = sm * sm;
  return 0.75 * sm2 * w2i - 0.25 * sm * sm2 * w3i;
}

// Coefficients of the 7th-order accessibility polynomial on the window
// [rad - win, rad + win] (fillcoCoefSpline4, vpmg.c:7119-7175, and
// Vacc_splineAccGradAtomNorm4, vacc.c:1004-1095): 0 and 1 with three
// vanishing derivatives at the ends.
__device__ __forceinline__ void spline7_coef(double rad, double win, double* c) {
  const double b = rad - win, e = rad + win;
  const double e2 = e * e, e3 = e2 * e, e4 = e3 * e, e5 = e4 * e, e6 = e5 * e, e7 = e6 * e;
  const double b2 = b * b, b3 = b2 * b, b4 = b3 * b, b5 = b4 * b, b6 = b5 * b, b7 = b6 * b;
  const double denom = e7 - 7.0 * b * e6 + 21.0 * b2 * e5 - 35.0 * e4 * b3 + 35.0 * e3 * b4 -
                       21.0 * b5 * e2 + 7.0 * e * b6 - b7;
  c[0] = b4 * (35.0 * e3 - 21.0 * b * e2 + 7 * e * b2 - b3) / denom;
  c[1] = -140.0 * b3 * e3 / denom;
  c[2] = 210.0 * e2 * b2 * (e + b) / denom;
  c[3] = -140.0 * e * b * (e2 + 3.0 * b * e + b2) / denom;
  c[4] = 35.0 * (e3 + 9.0 * b * e2 + 9.0 * e * b2 + b3) / denom;
  c[5] = -84.0 * (e2 + 3.0 * b * e + b2) / denom;
  c[6] = 70.0 * (e + b) / denom;
  c[7] = -20.0 / denom;
}

// the 7th-order accessibility at distance sm (sm2 as the reference forms it
// for that map), clamped to [0, 1]
__device__ __forceinline__ double spline7_value(const double* c, double sm, double sm2) {
  const double sm3 = sm2 * sm, sm4 = sm3 * sm, sm5 = sm4 * sm, sm6 = sm5 * sm, sm7 = sm6 * sm;
  double value = c[0] + c[1] * sm + c[2] * sm2 + c[3] * sm3 + c[4] * sm4 + c[5] * sm5 +
                 c[6] * sm6 + c[7] * sm7;
  if (value > 1.0) value = 1.0;
  else if (value < 0.0) value = 0.0;
  return value;
}

// the 5th-order accessibility of fillcoCoefSpline3 at distance sm (sm2 as the
// reference forms it for that map), clamped to [0, 1]
__device__ __forceinline__ double spline5_value(const double* c, double sm, double sm2) {
  const double sm3 = sm2 * sm, sm4 = sm3 * sm, sm5 = sm4 * sm;
  double value = c[0] + c[1] * sm + c[2] * sm2 + c[3] * sm3 + c[4] * sm4 + c[5] * sm5;
  if (value > 1.0) value = 1.0;
  else if (value < 0.0) value = 0.0;
  return value;
}

// ORDER 2: cubic window (srfm spl2, fillcoCoefSpline); ORDER 3: 5th-order
// polynomial (srfm spl3, fillcoCoefSpline3, vpmg.c:7525-7840) with the
// per-atom coefficients of spline3_table; ORDER 4: 7th-order polynomial
// (srfm spl4, fillcoCoefSpline4, vpmg.c:7052-7366)
template <int ORDER>
__global__ void __launch_bounds__(kSplThreads) k_spline_fill(SplineArgs A) {
  __shared__ SplAtom cand[kSplCap];
  __shared__ int wcount[kSplThreads / 32];
  __shared__ int ncand;
  const FillGeom& G = A.G;
  const int nx = G.g.nx, ny = G.g.ny, nz = G.g.nz;
  const double hx = G.h[0], hy = G.h[1], hz = G.h[2];
  const int bi = blockIdx.x * kBX, bj = blockIdx.y * kBY, bk = blockIdx.z * kBZ;
  const int tx = threadIdx.x % kBX, ty = (threadIdx.x / kBX) % kBY, tz = threadIdx.x / (kBX * kBY);
  const int i = bi + tx, j = bj + ty;
  const int kk[2] = {bk + tz, bk + tz + kBZ / 2};
  const bool on[2] = {i < nx && j < ny && kk[0] < nz, i < nx && j < ny && kk[1] < nz};
  double kap[2] = {1.0, 1.0}, ex[2] = {1.0, 1.0}, ey[2] = {1.0, 1.0}, ez[2] = {1.0, 1.0};
  const double win = A.win;
  const double w2i = 1.0 / (win * win);
  const double w3i = 1.0 / (win * win * win);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) ncand = 0;
  __syncthreads();

  auto apply = [&](int count) {
    for (int c = 0; c < count; c++) {
      const SplAtom& s = cand[c];
      if (i < s.box[0] || i > s.box[1] || j < s.box[2] || j > s.box[3]) continue;
      const double arad = s.arad;
      const double itot = A.irad + arad + win, itot2 = itot * itot;
      const double ictot = fmax(0.0, (A.irad + arad - win)), ictot2 = ictot * ictot;
      const double stot = arad + win, stot2 = stot * stot;
      const double sctot = fmax(0.0, (arad - win)), sctot2 = sctot * sctot;
      const double dx2 = (s.pos[0] - hx * i) * (s.pos[0] - hx * i);
      const double dy2 = (s.pos[1] - hy * j) * (s.pos[1] - hy * j);
      for (int p = 0; p < 2; p++) {
        const int k = kk[p];
        if (!on[p] || k < s.box[4] || k > s.box[5]) continue;
        const double dz2 = (s.pos[2] - k * hz) * (s.pos[2] - k * hz);
        if (kap[p] > kPmgSmall) {
          const double dist2 = dz2 + dy2 + dx2;
          if (dist2 <= ictot2) kap[p] = 0.0;
          if ((dist2 < itot2) && (dist2 > ictot2)) {
            const double dist = sqrt(dist2);
            if (ORDER == 2) {
              kap[p] *= spline_value(dist, arad + A.irad, win, w2i, w3i);
            } else if (ORDER == 3) {
              kap[p] *= spline5_value(A.c3 + 18 * (size_t)s.idx + 6, dist, dist2);
            } else {
              double c[8];
              spline7_coef(A.irad + arad, win, c);
              kap[p] *= spline7_value(c, dist, dist2);
            }
          }
        }
        if (ex[p] > kPmgSmall) {
          const double t = s.pos[0] - (i + 0.5) * hx;
          const double dist2 = dz2 + dy2 + t * t;
          if (dist2 <= sctot2) ex[p] = 0.0;
          if ((dist2 > sctot2) && (dist2 < stot2)) {
            const double dist = sqrt(dist2);
            if (ORDER == 2) {
              ex[p] *= spline_value(dist, arad, win, w2i, w3i);
            } else if (ORDER == 3) {
              ex[p] *= spline5_value(A.c3 + 18 * (size_t)s.idx, dist, dist * dist);
            } else {
              double c[8];
              spline7_coef(arad, win, c);
              ex[p] *= spline7_value(c, dist, dist * dist);
            }
          }
        }
        if (ey[p] > kPmgSmall) {
          const double t = s.pos[1] - (j + 0.5) * hy;
          const double dist2 = dz2 + dx2 + t * t;
          if (dist2 <= sctot2) ey[p] = 0.0;
          if ((dist2 > sctot2) && (dist2 < stot2)) {
            const double dist = sqrt(dist2);
            if (ORDER == 2) {
              ey[p] *= spline_value(dist, arad, win, w2i, w3i);
            } else if (ORDER == 3) {
              ey[p] *= spline5_value(A.c3 + 18 * (size_t)s.idx, dist, dist * dist);
            } else {
              double c[8];
              spline7_coef(arad, win, c);
              ey[p] *= spline7_value(c, dist, dist * dist);
            }
          }
        }
        if (ez[p] > kPmgSmall) {
          const double t = s.pos[2] - (k + 0.5) * hz;
          const double dist2 = dy2 + dx2 + t * t;
          if (dist2 <= sctot2) ez[p] = 0.0;
          if ((dist2 > sctot2) && (dist2 < stot2)) {
            const double dist = sqrt(dist2);
            if (ORDER == 2) {
              ez[p] *= spline_value(dist, arad, win, w2i, w3i);
            } else if (ORDER == 3) {
              ez[p] *= spline5_value(A.c3 + 18 * (size_t)s.idx, dist, dist2);
            } else {
              double c[8];
              spline7_coef(arad, win, c);
              ez[p] *= spline7_value(c, dist, dist2);
            }
          }
        }
      }
    }
  };

  const int ilast = min(bi + kBX, nx) - 1, jlast = min(bj + kBY, ny) - 1,
            klast = min(bk + kBZ, nz) - 1;
  for (int base = 0; base < A.natoms; base += kSplThreads) {
    // the atoms base .. base+255 whose search box meets this block, appended
    // in atom order
    const int a = base + threadIdx.x;
    SplAtom s;
    bool keep = false;
    if (a < A.natoms && spline_atom(A, a, s))
      keep = !(s.box[1] < bi || s.box[0] > ilast || s.box[3] < bj || s.box[2] > jlast ||
               s.box[5] < bk || s.box[4] > klast);
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) wcount[wid] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < kSplThreads / 32; w++) {
      if (w < wid) before += wcount[w];
      total += wcount[w];
    }
    const int start = ncand;
    if (start + total > kSplCap) {
      // no room: apply what is held, then start a new list
      apply(start);
      __syncthreads();
      if (keep) cand[before + __popc(m & ((1u << lane) - 1u))] = s;
      __syncthreads();
      if (threadIdx.x == 0) ncand = total;
    } else {
      if (keep) cand[start + before + __popc(m & ((1u << lane) - 1u))] = s;
      __syncthreads();
      if (threadIdx.x == 0) ncand = start + total;
    }
    __syncthreads();
  }
  apply(ncand);
  for (int p = 0; p < 2; p++) {
    if (!on[p]) continue;
    const size_t id = G.g.idx(i, j, kk[p]);
    A.kappa[id] = A.ionmask * kap[p];
    A.epsx[id] = (A.epsw - A.epsp) * ex[p] + A.epsp;
    A.epsy[id] = (A.epsw - A.epsp) * ey[p] + A.epsp;
    A.epsz[id] = (A.epsw - A.epsp) * ez[p] + A.epsp;
  }
}

// ---------------------------------------------------------------------------
// forces
// ---------------------------------------------------------------------------
struct ForceArgs {
  FillGeom G;
  int natoms;
  const double *xyz, *q, *r;
  const double* u;
  const double *epsx, *epsy, *epsz, *kappa;
  int chgm;         // PMGB_CHGM_*
  int boundary;     // compute the dielectric and ionic boundary forces
  int order;        // surface: 2 = spl2, 3 = spl3, 4 = spl4 (Vpmg_splineSelect)
  const double* c3; // spl3: spline3_table's coefficients
  int nonlin;
  double win, irad, srad, epsp, epsw, zkappa2, izmagic, ionstr;
  int nion;
  double ion_q[8], ion_conc[8];
  double* out;      // 9 per atom: qf, db, ib
  int* status;      // per atom: 1, or 0 if the dielectric boundary force failed
};

__device__ __forceinline__ double bspline2d(double x) {
  double m2m, m2, m3;
  if ((x >= 0.0) && (x <= 2.0)) m2m = 1.0 - fabs(x - 1.0);
  else m2m = 0.0;
  if ((x >= 1.0) && (x <= 3.0)) m2 = 1.0 - fabs(x - 2.0);
  else m2 = 0.0;
  if ((x >= 0.0) && (x <= 3.0)) m3 = 0.5 * x * m2m + 0.5 * (3.0 - x) * m2;
  else m3 = 0.0;
  return m3;
}
// derivative of the quadratic B-spline (dbspline2, vpmg.c:5107-5120)
__device__ __forceinline__ double dbspline2d(double x) {
  double m2m, m2;
  if ((x >= 0.0) && (x <= 2.0)) m2m = 1.0 - fabs(x - 1.0);
  else m2m = 0.0;
  if ((x >= 1.0) && (x <= 3.0)) m2 = 1.0 - fabs(x - 2.0);
  else m2 = 0.0;
  return m2m - m2;
}

// gradient of the log of one atom's spline accessibility at a point
// (Vacc_splineAccGradAtomNorm, vacc.c:314-373)
__device__ __forceinline__ void spline_grad(const double* center, double win, double infrad,
                                            const double* apos, double radius, double* grad) {
  const double w2i = 1.0 / (win * win);
  const double w3i = 1.0 / (win * win * win);
  grad[0] = grad[1] = grad[2] = 0.0;
  if (!(radius > 0.0)) return;
  const double arad = radius + infrad;
  const double d0 = apos[0] - center[0], d1 = apos[1] - center[1], d2 = apos[2] - center[2];
  const double dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  double mychi, mygrad;
  if (dist < (arad - win)) return;
  else if (dist > (arad + win)) return;
  else if ((fabs(dist - (arad - win)) < kVSmall) || (fabs(dist - (arad + win)) < kVSmall)) return;
  else {
    const double sm = dist - arad + win;
    const double sm2 = sm * sm;
    mychi = 0.75 * sm2 * w2i - 0.25 * sm * sm2 * w3i;
    mygrad = 1.5 * sm * w2i - 0.75 * sm2 * w3i;
  }
  for (int d = 0; d < 3; d++) grad[d] = -(mygrad / mychi) * ((center[d] - apos[d]) / dist);
}

// the same for the 7th-order polynomial (Vacc_splineAccGradAtomNorm4,
// vacc.c:1004-1095)
__device__ __forceinline__ void spline_grad4(const double* center, double win, double infrad,
                                             const double* apos, double radius, double* grad) {
  grad[0] = grad[1] = grad[2] = 0.0;
  if (!(radius > 0.0)) return;
  const double arad = radius + infrad;
  double c[8];
  spline7_coef(arad, win, c);
  const double d0 = apos[0] - center[0], d1 = apos[1] - center[1], d2 = apos[2] - center[2];
  const double dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  double mychi, mygrad;
  if (dist < (arad - win)) return;
  else if (dist > (arad + win)) return;
  else if ((fabs(dist - (arad - win)) < kVSmall) || (fabs(dist - (arad + win)) < kVSmall)) return;
  else {
    const double sm = dist, sm2 = sm * sm, sm3 = sm2 * sm, sm4 = sm3 * sm, sm5 = sm4 * sm,
                 sm6 = sm5 * sm, sm7 = sm6 * sm;
    mychi = c[0] + c[1] * sm + c[2] * sm2 + c[3] * sm3 + c[4] * sm4 + c[5] * sm5 + c[6] * sm6 +
            c[7] * sm7;
    mygrad = c[1] + 2.0 * c[2] * sm + 3.0 * c[3] * sm2 + 4.0 * c[4] * sm3 + 5.0 * c[5] * sm4 +
             6.0 * c[6] * sm5 + 7.0 * c[7] * sm6;
    if (mychi <= 0.0) return;
    else if (mychi > 1.0) mychi = 1.0;
  }
  for (int d = 0; d < 3; d++) grad[d] = -(mygrad / mychi) * ((center[d] - apos[d]) / dist);
}

// the same for the 5th-order polynomial (Vacc_splineAccGradAtomNorm3,
// vacc.c:1097-1180); c: the atom's coefficients for this inflation
__device__ __forceinline__ void spline_grad3(const double* center, double win, double infrad,
                                             const double* apos, double radius, const double* c,
                                             double* grad) {
  grad[0] = grad[1] = grad[2] = 0.0;
  if (!(radius > 0.0)) return;
  const double arad = radius + infrad;
  const double d0 = apos[0] - center[0], d1 = apos[1] - center[1], d2 = apos[2] - center[2];
  const double dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  double mychi, mygrad;
  if (dist < (arad - win)) return;
  else if (dist > (arad + win)) return;
  else if ((fabs(dist - (arad - win)) < kVSmall) || (fabs(dist - (arad + win)) < kVSmall)) return;
  else {
    const double sm = dist, sm2 = sm * sm, sm3 = sm2 * sm, sm4 = sm3 * sm, sm5 = sm4 * sm;
    mychi = c[0] + c[1] * sm + c[2] * sm2 + c[3] * sm3 + c[4] * sm4 + c[5] * sm5;
    mygrad = c[1] + 2.0 * c[2] * sm + 3.0 * c[3] * sm2 + 4.0 * c[4] * sm3 + 5.0 * c[5] * sm4;
    if (mychi <= 0.0) return;
    else if (mychi > 1.0) mychi = 1.0;
  }
  for (int d = 0; d < 3; d++) grad[d] = -(mygrad / mychi) * ((center[d] - apos[d]) / dist);
}

// Vcap_exp (src/generic/vcap.c:59-73)
__device__ __forceinline__ double cap_exp(double x) {
  if (x > kExpMax) return exp(kExpMax);
  if (x < -kExpMax) return exp(-kExpMax);
  return exp(x);
}

// infrad is 0 (dielectric) or the largest ion radius (ion accessibility),
// which picks the spl3 coefficient set of atom a
__device__ __forceinline__ void surf_grad(const ForceArgs& A, int a, const double* center,
                                          double infrad, const double* apos, double radius,
                                          double* grad) {
  if (A.order == 4) spline_grad4(center, A.win, infrad, apos, radius, grad);
  else if (A.order == 3)
    spline_grad3(center, A.win, infrad, apos, radius,
                 A.c3 + 18 * (size_t)a + (infrad == 0.0 ? 0 : 12), grad);
  else spline_grad(center, A.win, infrad, apos, radius, grad);
}

__global__ void k_forces(ForceArgs A) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= A.natoms) return;
  const FillGeom& G = A.G;
  const int nx = G.g.nx, ny = G.g.ny, nz = G.g.nz;
  const double hx = G.h[0], hy = G.h[1], hzed = G.h[2];
  const double xmin = G.xmin[0], ymin = G.xmin[1], zmin = G.xmin[2];
  const double xmax = G.xmax[0], ymax = G.xmax[1], zmax = G.xmax[2];
  const double* apos = A.xyz + 3 * a;
  const double charge = A.q[a], radius = A.r[a];
  const double* u = A.u;
  auto IJK = [&](int i, int j, int k) { return ((size_t)k * ny + j) * nx + i; };
  double* out = A.out + 9 * (size_t)a;
  for (int d = 0; d < 9; d++) out[d] = 0.0;
  int status = 1;

  // partition flag of Vpmg_setPart (vpmg.c:673-720) for the domain box
  double part_id = 1.0;
  for (int d = 0; d < 3; d++) {
    const double lo = G.xmin[d], hi = G.xmax[d];
    double ok;
    if ((apos[d] < hi) && (apos[d] > lo)) ok = 1;
    else if (fabs(apos[d] - lo) < kPmgSmall) ok = 1;
    else if (fabs(apos[d] - hi) < kPmgSmall) ok = 1;
    else ok = 0;
    part_id = (d == 0) ? ok : part_id * ok;
  }

  // ---- charge-field force
  if (part_id != 0.0) {
    double* f = out;
    if (A.chgm == PMGB_CHGM_SPL2) {
      if (!((apos[0] <= (xmin + hx)) || (apos[0] >= (xmax - hx)) || (apos[1] <= (ymin + hy)) ||
            (apos[1] >= (ymax - hy)) || (apos[2] <= (zmin + hzed)) ||
            (apos[2] >= (zmax - hzed)))) {
        const double ifloat = (apos[0] - xmin) / hx;
        const double jfloat = (apos[1] - ymin) / hy;
        const double kfloat = (apos[2] - zmin) / hzed;
        const int ip2 = min((int)ceil(ifloat) + 1, nx - 1);
        const int im2 = max((int)floor(ifloat) - 1, 0);
        const int jp2 = min((int)ceil(jfloat) + 1, ny - 1);
        const int jm2 = max((int)floor(jfloat) - 1, 0);
        const int kp2 = min((int)ceil(kfloat) + 1, nz - 1);
        const int km2 = max((int)floor(kfloat) - 1, 0);
        for (int ii = im2; ii <= ip2; ii++) {
          const double mx = bspline2d(1.5 + ((double)ii - ifloat));
          const double dmx = dbspline2d(1.5 + ((double)ii - ifloat));
          for (int jj = jm2; jj <= jp2; jj++) {
            const double my = bspline2d(1.5 + ((double)jj - jfloat));
            const double dmy = dbspline2d(1.5 + ((double)jj - jfloat));
            for (int kk = km2; kk <= kp2; kk++) {
              const double mz = bspline2d(1.5 + ((double)kk - kfloat));
              const double dmz = dbspline2d(1.5 + ((double)kk - kfloat));
              const double uv = u[IJK(ii, jj, kk)];
              f[0] += (charge * dmx * my * mz * uv) / hx;
              f[1] += (charge * mx * dmy * mz * uv) / hy;
              f[2] += (charge * mx * my * dmz * uv) / hzed;
            }
          }
        }
      }
    } else if (A.chgm == PMGB_CHGM_SPL4) {
      // handled below: qfForceSpline4 has no partition test
    } else if (!((apos[0] <= xmin) || (apos[0] >= xmax) || (apos[1] <= ymin) ||
                 (apos[1] >= ymax) || (apos[2] <= zmin) || (apos[2] >= zmax))) {
      // trilinear charges (qfForceSpline1)
      const double ifloat = (apos[0] - xmin) / hx;
      const double jfloat = (apos[1] - ymin) / hy;
      const double kfloat = (apos[2] - zmin) / hzed;
      const int ihi = (int)ceil(ifloat), ilo = (int)floor(ifloat);
      const int jhi = (int)ceil(jfloat), jlo = (int)floor(jfloat);
      const int khi = (int)ceil(kfloat), klo = (int)floor(kfloat);
      const double dx = ifloat - (double)(ilo);
      const double dy = jfloat - (double)(jlo);
      const double dz = kfloat - (double)(klo);
      if ((dx > kPmgSmall) && (fabs(1.0 - dx) > kPmgSmall)) {
        f[0] = -charge *
               (dy * dz * u[IJK(ihi, jhi, khi)] + dy * (1 - dz) * u[IJK(ihi, jhi, klo)] +
                (1 - dy) * dz * u[IJK(ihi, jlo, khi)] +
                (1 - dy) * (1 - dz) * u[IJK(ihi, jlo, klo)] - dy * dz * u[IJK(ilo, jhi, khi)] -
                dy * (1 - dz) * u[IJK(ilo, jhi, klo)] - (1 - dy) * dz * u[IJK(ilo, jlo, khi)] -
                (1 - dy) * (1 - dz) * u[IJK(ilo, jlo, klo)]) /
               hx;
      }
      if ((dy > kPmgSmall) && (fabs(1.0 - dy) > kPmgSmall)) {
        f[1] = -charge *
               (dx * dz * u[IJK(ihi, jhi, khi)] + dx * (1 - dz) * u[IJK(ihi, jhi, klo)] -
                dx * dz * u[IJK(ihi, jlo, khi)] - dx * (1 - dz) * u[IJK(ihi, jlo, klo)] +
                (1 - dx) * dz * u[IJK(ilo, jhi, khi)] +
                (1 - dx) * (1 - dz) * u[IJK(ilo, jhi, klo)] -
                (1 - dx) * dz * u[IJK(ilo, jlo, khi)] -
                (1 - dx) * (1 - dz) * u[IJK(ilo, jlo, klo)]) /
               hy;
      }
      if ((dz > kPmgSmall) && (fabs(1.0 - dz) > kPmgSmall)) {
        f[2] = -charge *
               (dy * dx * u[IJK(ihi, jhi, khi)] - dy * dx * u[IJK(ihi, jhi, klo)] +
                (1 - dy) * dx * u[IJK(ihi, jlo, khi)] - (1 - dy) * dx * u[IJK(ihi, jlo, klo)] +
                dy * (1 - dx) * u[IJK(ilo, jhi, khi)] - dy * (1 - dx) * u[IJK(ilo, jhi, klo)] +
                (1 - dy) * (1 - dx) * u[IJK(ilo, jlo, khi)] -
                (1 - dy) * (1 - dx) * u[IJK(ilo, jlo, klo)]) /
               hzed;
      }
    }
  }
  if (A.chgm == PMGB_CHGM_SPL4 &&
      !((apos[0] <= (xmin + 2 * hx)) || (apos[0] >= (xmax - 2 * hx)) ||
        (apos[1] <= (ymin + 2 * hy)) || (apos[1] >= (ymax - 2 * hy)) ||
        (apos[2] <= (zmin + 2 * hzed)) || (apos[2] >= (zmax - 2 * hzed)))) {
    // qfForceSpline4 (vpmg.c:6156-6272): the field of the 5th-order B-spline
    // charge at the atom, times its charge
    const double ifloat = (apos[0] - xmin) / hx;
    const double jfloat = (apos[1] - ymin) / hy;
    const double kfloat = (apos[2] - zmin) / hzed;
    const int ip2 = min((int)ceil(ifloat) + 2, nx - 1), im2 = max((int)floor(ifloat) - 2, 0);
    const int jp2 = min((int)ceil(jfloat) + 2, ny - 1), jm2 = max((int)floor(jfloat) - 2, 0);
    const int kp2 = min((int)ceil(kfloat) + 2, nz - 1), km2 = max((int)floor(kfloat) - 2, 0);
    double e[3] = {0.0, 0.0, 0.0};
    for (int ii = im2; ii <= ip2; ii++) {
      const double mi = (2.5 + ((double)(ii) - (ifloat)));
      const double mx = bspline4(mi), dmx = dbspline4(mi);
      for (int jj = jm2; jj <= jp2; jj++) {
        const double mj = (2.5 + ((double)(jj) - (jfloat)));
        const double my = bspline4(mj), dmy = dbspline4(mj);
        for (int kk = km2; kk <= kp2; kk++) {
          const double mk = (2.5 + ((double)(kk) - (kfloat)));
          const double mz = bspline4(mk), dmz = dbspline4(mk);
          const double f = u[IJK(ii, jj, kk)];
          e[0] += f * dmx * my * mz / hx;
          e[1] += f * mx * dmy * mz / hy;
          e[2] += f * mx * my * dmz / hzed;
        }
      }
    }
    for (int d = 0; d < 3; d++) out[d] = e[d] * charge;
  }
  if (!A.boundary || part_id == 0.0) {
    A.status[a] = status;
    return;
  }

  // ---- dielectric boundary force
  if (!(fabs(A.epsp - A.epsw) < kPmgSmall)) {
    const double deps = (A.epsw - A.epsp);
    const double depsi = 1.0 / deps;
    const double rtot = (radius + A.win + A.srad);
    if (!((apos[0] <= xmin + rtot) || (apos[0] >= xmax - rtot) || (apos[1] <= ymin + rtot) ||
          (apos[1] >= ymax - rtot) || (apos[2] <= zmin + rtot) || (apos[2] >= zmax - rtot))) {
      const double position[3] = {apos[0] - xmin, apos[1] - ymin, apos[2] - zmin};
      const int imin = (int)floor((position[0] - rtot) / hx);
      const int imax = (int)ceil((position[0] + rtot) / hx);
      const int jmin = (int)floor((position[1] - rtot) / hy);
      const int jmax = (int)ceil((position[1] + rtot) / hy);
      const int kmin = (int)floor((position[2] - rtot) / hzed);
      const int kmax = (int)ceil((position[2] + rtot) / hzed);
      if (imin < 1 || imax > nx - 2 || jmin < 1 || jmax > ny - 2 || kmin < 1 || kmax > nz - 2) {
        status = 0;  // "Atom off grid": the reference returns 0 here
      } else {
        double dbF[3] = {0.0, 0.0, 0.0};
        for (int i = imin; i <= imax; i++) {
          for (int j = jmin; j <= jmax; j++) {
            for (int k = kmin; k <= kmax; k++) {
              double gpos[3], dHx[3], dHy[3], dHz[3], dHxm[3], dHym[3], dHzm[3];
              gpos[0] = (i + 0.5) * hx + xmin; gpos[1] = j * hy + ymin; gpos[2] = k * hzed + zmin;
              const double Hxijk = (A.epsx[IJK(i, j, k)] - A.epsp) * depsi;
              surf_grad(A, a, gpos, 0., apos, radius, dHx);
              for (int l = 0; l < 3; l++) dHx[l] *= Hxijk;
              gpos[0] = i * hx + xmin; gpos[1] = (j + 0.5) * hy + ymin; gpos[2] = k * hzed + zmin;
              const double Hyijk = (A.epsy[IJK(i, j, k)] - A.epsp) * depsi;
              surf_grad(A, a, gpos, 0., apos, radius, dHy);
              for (int l = 0; l < 3; l++) dHy[l] *= Hyijk;
              gpos[0] = i * hx + xmin; gpos[1] = j * hy + ymin; gpos[2] = (k + 0.5) * hzed + zmin;
              const double Hzijk = (A.epsz[IJK(i, j, k)] - A.epsp) * depsi;
              surf_grad(A, a, gpos, 0., apos, radius, dHz);
              for (int l = 0; l < 3; l++) dHz[l] *= Hzijk;
              gpos[0] = (i - 0.5) * hx + xmin; gpos[1] = j * hy + ymin; gpos[2] = k * hzed + zmin;
              const double Hxim1jk = (A.epsx[IJK(i - 1, j, k)] - A.epsp) * depsi;
              surf_grad(A, a, gpos, 0., apos, radius, dHxm);
              for (int l = 0; l < 3; l++) dHxm[l] *= Hxim1jk;
              gpos[0] = i * hx + xmin; gpos[1] = (j - 0.5) * hy + ymin; gpos[2] = k * hzed + zmin;
              const double Hyijm1k = (A.epsy[IJK(i, j - 1, k)] - A.epsp) * depsi;
              surf_grad(A, a, gpos, 0., apos, radius, dHym);
              for (int l = 0; l < 3; l++) dHym[l] *= Hyijm1k;
              gpos[0] = i * hx + xmin; gpos[1] = j * hy + ymin; gpos[2] = (k - 0.5) * hzed + zmin;
              const double Hzijkm1 = (A.epsz[IJK(i, j, k - 1)] - A.epsp) * depsi;
              surf_grad(A, a, gpos, 0., apos, radius, dHzm);
              for (int l = 0; l < 3; l++) dHzm[l] *= Hzijkm1;
              const double u0 = u[IJK(i, j, k)];
              const double dbFmag = u0;
              const double uxp = u[IJK(i + 1, j, k)], uxm = u[IJK(i - 1, j, k)];
              const double uyp = u[IJK(i, j + 1, k)], uym = u[IJK(i, j - 1, k)];
              const double uzp = u[IJK(i, j, k + 1)], uzm = u[IJK(i, j, k - 1)];
              for (int l = 0; l < 3; l++) {
                const double tg = (dHx[l] * (uxp - u0) + dHxm[l] * (uxm - u0)) / (hx * hx) +
                                  (dHy[l] * (uyp - u0) + dHym[l] * (uym - u0)) / (hy * hy) +
                                  (dHz[l] * (uzp - u0) + dHzm[l] * (uzm - u0)) / (hzed * hzed);
                dbF[l] += (dbFmag * tg);
              }
            }
          }
        }
        for (int l = 0; l < 3; l++)
          out[3 + l] = -dbF[l] * hx * hy * hzed * deps * 0.5 * A.izmagic;
      }
    }
  }

  // ---- ionic boundary force
  if (!(A.zkappa2 < kPmgSmall) &&
      !((apos[0] <= xmin) || (apos[0] >= xmax) || (apos[1] <= ymin) || (apos[1] >= ymax) ||
        (apos[2] <= zmin) || (apos[2] >= zmax))) {
    const double position[3] = {apos[0] - xmin, apos[1] - ymin, apos[2] - zmin};
    const double rtot = (A.irad + radius + A.win);
    const double rtot2 = rtot * rtot;
    double ibF[3] = {0.0, 0.0, 0.0};
    const double ddx = rtot + 0.5 * hx;
    const int imin = max(0, (int)ceil((position[0] - ddx) / hx));
    const int imax = min(nx - 1, (int)floor((position[0] + ddx) / hx));
    for (int i = imin; i <= imax; i++) {
      const double dx2 = (position[0] - hx * i) * (position[0] - hx * i);
      double dy;
      if (rtot2 > dx2) dy = sqrt(rtot2 - dx2) + 0.5 * hy;
      else dy = 0.5 * hy;
      const int jmin = max(0, (int)ceil((position[1] - dy) / hy));
      const int jmax = min(ny - 1, (int)floor((position[1] + dy) / hy));
      for (int j = jmin; j <= jmax; j++) {
        const double dy2 = (position[1] - hy * j) * (position[1] - hy * j);
        double dz;
        if (rtot2 > (dx2 + dy2)) dz = sqrt(rtot2 - dx2 - dy2) + 0.5 * hzed;
        else dz = 0.5 * hzed;
        const int kmin = max(0, (int)ceil((position[2] - dz) / hzed));
        const int kmax = min(nz - 1, (int)floor((position[2] + dz) / hzed));
        for (int k = kmin; k <= kmax; k++) {
          const double dz2 = (k * hzed - position[2]) * (k * hzed - position[2]);
          if ((dz2 + dy2 + dx2) <= rtot2) {
            double gpos[3], tgrad[3];
            gpos[0] = i * hx + xmin;
            gpos[1] = j * hy + ymin;
            gpos[2] = k * hzed + zmin;
            surf_grad(A, a, gpos, A.irad, apos, radius, tgrad);
            const double uv = u[IJK(i, j, k)], kv = A.kappa[IJK(i, j, k)];
            double fmag;
            if (A.nonlin) {
              fmag = 0.0;
              for (int m = 0; m < A.nion; m++)
                fmag += kv * A.ion_conc[m] * (cap_exp(-A.ion_q[m] * uv) - 1.0) / A.ionstr;
            } else {
              fmag = (uv * uv) * kv;
            }
            for (int l = 0; l < 3; l++) ibF[l] += (A.zkappa2 * fmag * tgrad[l]);
          }
        }
      }
    }
    for (int l = 0; l < 3; l++) out[6 + l] = ibF[l] * 0.5 * hx * hy * hzed * A.izmagic;
  }
  A.status[a] = status;
}

}  // namespace

void launch_spline_fill(cudaStream_t st, int order, const FillGeom& G, int natoms,
                        const double* xyz, const double* r, double irad, double win,
                        double ionmask, double epsp, double epsw, const double* coef3,
                        double* kappa, double* epsx, double* epsy, double* epsz) {
  SplineArgs A;
  A.G = G;
  A.natoms = natoms;
  A.xyz = xyz;
  A.r = r;
  A.irad = irad;
  A.win = win;
  A.ionmask = ionmask;
  A.epsp = epsp;
  A.epsw = epsw;
  A.c3 = coef3;
  A.kappa = kappa;
  A.epsx = epsx;
  A.epsy = epsy;
  A.epsz = epsz;
  dim3 grid((G.g.nx + kBX - 1) / kBX, (G.g.ny + kBY - 1) / kBY, (G.g.nz + kBZ - 1) / kBZ);
  if (order == 4) k_spline_fill<4><<<grid, kSplThreads, 0, st>>>(A);
  else if (order == 3) k_spline_fill<3><<<grid, kSplThreads, 0, st>>>(A);
  else k_spline_fill<2><<<grid, kSplThreads, 0, st>>>(A);
}

// The window polynomials of fillcoCoefSpline3 (vpmg.c:7590-7641) and
// Vacc_splineAccGradAtomNorm3 (vacc.c:1118-1143) for window [b, e]:
// c_k / (e - b)^5 with the reference's expressions and its pow().
static void spline3_poly(double b, double e, double* c) {
  const double e2 = e * e;
  const double b2 = b * b, b3 = b2 * b, b4 = b3 * b, b5 = b4 * b;
  const double denom = pow((e - b), 5.0);
  c[0] = (-10.0 * e2 * b3 + 5.0 * e * b4 - b5) / denom;
  c[1] = (30.0 * e2 * b2) / denom;
  c[2] = (-30.0 * (e2 * b + e * b2)) / denom;
  c[3] = (10.0 * (e2 + 4.0 * e * b + b2)) / denom;
  c[4] = (-15.0 * (e + b)) / denom;
  c[5] = 6.0 / denom;
}

// Per atom, 18 coefficients: [0, 6) the dielectric window (radius +- win),
// used by the eps maps and by the dielectric-boundary gradient; [6, 12) what
// fillcoCoefSpline3 multiplies kappa by: the dielectric coefficients divided
// once more by the ion window's (e - b)^5 (vpmg.c:7630-7641 assign
// ic0 = c0/denom ... after c0..c5 were divided already, so the ion window's
// own polynomial is never used there); [12, 18) the ion window's own
// polynomial (radius + irad +- win), used by the ionic-boundary gradient.
void spline3_table(int natoms, const double* r, double irad, double win,
                   std::vector<double>& tab) {
  tab.assign(18 * (size_t)natoms, 0.0);
  for (int a = 0; a < natoms; a++) {
    double* t = tab.data() + 18 * (size_t)a;
    const double arad = r[a];
    spline3_poly(arad - win, arad + win, t);
    const double bi = irad + arad - win, ei = irad + arad + win;
    const double idenom = pow((ei - bi), 5.0);
    for (int k = 0; k < 6; k++) t[6 + k] = t[k] / idenom;
    const double ar = arad + irad;
    spline3_poly(ar - win, ar + win, t + 12);
  }
}

}  // namespace pmgb

using namespace pmgb;

// Per-atom forces of the last solve (Vpmg_qfForce, Vpmg_dbForce, Vpmg_ibForce).
extern "C" int pmgb_forces(pmgb_solver* s, double* qf, double* db, double* ib) {
  if (!s || !s->solved) {
    set_error("pmgb_forces: no solution (call pmgb_solve first)");
    return 0;
  }
  const pmgb_params& p = s->p;
  const int natoms = s->natoms;
  const int boundary = (db || ib) ? 1 : 0;
  if (boundary && p.srfm != PMGB_SRFM_SPL2 && p.srfm != PMGB_SRFM_SPL3 &&
      p.srfm != PMGB_SRFM_SPL4) {
    set_error("pmgb_forces: the boundary forces need srfm spl2, spl3 or spl4 (spline-based "
              "surfaces)");
    return 0;
  }
  if (p.chgm != PMGB_CHGM_SPL2 && p.chgm != PMGB_CHGM_TRIL && p.chgm != PMGB_CHGM_SPL4) {
    set_error("pmgb_forces: chgm %d has no charge-field force", p.chgm);
    return 0;
  }
  if (natoms <= 0) return 1;
  cudaStream_t st = s->stream;
  const size_t need = (size_t)natoms * 10;  // 9 doubles and a status word per atom
  if (!s->d_forces || s->forces_alloc < need) {
    if (s->d_forces) cudaFreeAsync(s->d_forces, st);
    s->d_forces = nullptr;
    s->forces_alloc = 0;
    PMGB_CUDA_OK(cudaMallocAsync((void**)&s->d_forces, need * sizeof(double), st));
    s->forces_alloc = need;
  }
  ForceArgs A;
  A.G = s->G;
  A.natoms = natoms;
  A.xyz = s->d_xyz;
  A.q = s->d_q;
  A.r = s->d_r;
  A.u = s->lev[0].x;
  A.epsx = s->epsx;
  A.epsy = s->epsy;
  A.epsz = s->epsz;
  A.kappa = s->kappa;
  A.chgm = p.chgm;
  A.boundary = boundary;
  A.order = (p.srfm == PMGB_SRFM_SPL4) ? 4 : (p.srfm == PMGB_SRFM_SPL3 ? 3 : 2);
  A.c3 = s->d_spl3;
  A.nonlin = p.nonlin;
  A.win = (p.swin > 0.0) ? p.swin : 0.3;
  A.irad = s->maxIonRadius;
  A.srad = p.srad;
  A.epsp = p.pdie;
  A.epsw = p.sdie;
  A.zkappa2 = s->zkappa2;
  A.izmagic = 1.0 / s->zmagic;
  A.ionstr = s->ionstr;
  A.nion = p.nion;
  for (int i = 0; i < 8; i++) {
    A.ion_q[i] = (i < p.nion) ? p.ion_q[i] : 0.0;
    A.ion_conc[i] = (i < p.nion) ? p.ion_conc[i] : 0.0;
  }
  A.out = s->d_forces;
  A.status = reinterpret_cast<int*>(s->d_forces + 9 * (size_t)natoms);
  k_forces<<<(natoms + 127) / 128, 128, 0, st>>>(A);
  note_launches(1);
  std::vector<double> h(9 * (size_t)natoms);
  std::vector<int> stat(natoms);
  PMGB_CUDA_OK(cudaMemcpyAsync(h.data(), A.out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
  PMGB_CUDA_OK(cudaMemcpyAsync(stat.data(), A.status, sizeof(int) * natoms, cudaMemcpyDeviceToHost, st));
  PMGB_CUDA_OK(cudaStreamSynchronize(st));
  PMGB_CUDA_OK(cudaGetLastError());
  for (int a = 0; a < natoms; a++)
    for (int d = 0; d < 3; d++) {
      if (qf) qf[3 * a + d] = h[9 * (size_t)a + d];
      if (db) db[3 * a + d] = h[9 * (size_t)a + 3 + d];
      if (ib) ib[3 * a + d] = h[9 * (size_t)a + 6 + d];
    }
  if (boundary)
    for (int a = 0; a < natoms; a++)
      if (!stat[a]) {
        set_error("pmgb_forces: atom %d too close to the grid edge for the dielectric "
                  "boundary force (Vpmg_dbForce off grid)", a);
        return 0;
      }
  return 1;
}
