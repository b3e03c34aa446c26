// Coefficient-map fill of the B200 PMG solver (Vpmg_fillco,
// src/mg/vpmg.c:5250-5414) and the sdh Dirichlet boundary values.
//
// Compiled with -fmad=false and written with the reference's expression
// trees: the integer index bounds (ceil/floor of FP64 expressions) and the
// FP64 comparisons that decide which grid points a sphere marks are then
// identical to the reference's, so the maps are bitwise equal.
#include <algorithm>

#include "fill_kernels.cuh"

namespace pmgb {

// ---------------------------------------------------------------------------
// Charge: fillcoChargeSpline2 + bspline2 (vpmg.c:5091-5248), the trilinear
// fillcoChargeSpline1 (vpmg.c:4986-5121) and the 5th-order B-spline of
// fillcoPermanentMultipole with atomic charges (vpmg.c:6835-7000), gathered per tile of grid
// points (k_charge_gather below) so that every point adds its atoms'
// contributions in atom order, as the reference's atom loop does: the map is
// the reference's bit for bit and the same on every run.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double bspline2(double x) {
  double m2m, m2, m3;
  if ((x >= 0.0) && (x <= 2.0)) m2m = 1.0 - fabs(x - 1.0);
  else m2m = 0.0;
  if ((x >= 1.0) && (x <= 3.0)) m2 = 1.0 - fabs(x - 2.0);
  else m2 = 0.0;
  if ((x >= 0.0) && (x <= 3.0)) m3 = 0.5 * x * m2m + 0.5 * (3.0 - x) * m2;
  else m3 = 0.0;
  return m3;
}

// Products and sums rounded one by one, as the reference's C evaluates
// them: the geometry tests below never fuse a multiply-add.
__device__ __forceinline__ double sq_rn(double v) { return __dmul_rn(v, v); }
// (pos - h f)^2 of markSphere
__device__ __forceinline__ double off2_rn(double pos, double h, double f) {
  return sq_rn(__dsub_rn(pos, __dmul_rn(h, f)));
}

// ---------------------------------------------------------------------------
// markSphere (vpmg.c:6444-6491) for one sphere on one (possibly staggered)
// grid, executed by the calling thread group.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void mark_sphere_group(double rtot, double cx, double cy, double cz,
                                                  Grid g, double hx, double hy, double hz,
                                                  double xmin, double ymin, double zmin,
                                                  T* array, T markVal, int lane, int nlanes) {
  const double posx = cx - xmin, posy = cy - ymin, posz = cz - zmin;
  const double rtot2 = __dmul_rn(rtot, rtot);
  const double xr = rtot + 0.5 * hx, yr = rtot + 0.5 * hy, zr = rtot + 0.5 * hz;
  const int imin = max(0, (int)ceil((posx - xr) / hx));
  const int jmin = max(0, (int)ceil((posy - yr) / hy));
  const int kmin = max(0, (int)ceil((posz - zr) / hz));
  const int imax = min(g.nx - 1, (int)floor((posx + xr) / hx));
  const int jmax = min(g.ny - 1, (int)floor((posy + yr) / hy));
  const int kmax = min(g.nz - 1, (int)floor((posz + zr) / hz));
  if (imax < imin || jmax < jmin || kmax < kmin) return;
  const int ni = imax - imin + 1, nj = jmax - jmin + 1;
  // lanes take (i, j) columns, consecutive lanes consecutive i so a warp's
  // stores to one plane fall on a few contiguous runs; the column test of the
  // reference prunes whole columns before the k loop.  Every store writes the
  // same value, so the order of the stores does not matter.
  for (int t = lane; t < ni * nj; t += nlanes) {
    const int ii = imin + t % ni, jj = jmin + t / ni;
    const double fi = (double)ii, fj = (double)jj;
    const double dx2 = off2_rn(posx, hx, fi);
    const double dy2 = off2_rn(posy, hy, fj);
    if (__dadd_rn(dx2, dy2) > rtot2) continue;
    T* col = array + g.idx(ii, jj, 0);
    const size_t sz = (size_t)g.nx * g.ny;
    for (int kk = kmin; kk <= kmax; kk++) {
      const double dz2 = off2_rn(posz, hz, (double)kk);
      if (__dadd_rn(__dadd_rn(dz2, dy2), dx2) <= rtot2) col[kk * sz] = markVal;
    }
  }
}

// The same marking by one warp with the squared z offsets of the sphere's
// planes computed once (lane kk - kmin computes plane kk's into the warp's
// dz2 buffer of 32 doubles) instead of once per column: the inner loop is
// then the reference's two additions and its comparison.  Spheres more than
// 32 planes thick use mark_sphere_group.
template <typename T>
__device__ __forceinline__ void mark_sphere_warp(double rtot, double cx, double cy, double cz,
                                                 Grid g, double hx, double hy, double hz,
                                                 double xmin, double ymin, double zmin,
                                                 T* array, T markVal, int lane, double* dz2b) {
  const double posx = cx - xmin, posy = cy - ymin, posz = cz - zmin;
  const double rtot2 = __dmul_rn(rtot, rtot);
  const double xr = rtot + 0.5 * hx, yr = rtot + 0.5 * hy, zr = rtot + 0.5 * hz;
  const int imin = max(0, (int)ceil((posx - xr) / hx));
  const int jmin = max(0, (int)ceil((posy - yr) / hy));
  const int kmin = max(0, (int)ceil((posz - zr) / hz));
  const int imax = min(g.nx - 1, (int)floor((posx + xr) / hx));
  const int jmax = min(g.ny - 1, (int)floor((posy + yr) / hy));
  const int kmax = min(g.nz - 1, (int)floor((posz + zr) / hz));
  if (imax < imin || jmax < jmin || kmax < kmin) return;
  const int nk = kmax - kmin + 1;
  if (nk > 32) {
    mark_sphere_group(rtot, cx, cy, cz, g, hx, hy, hz, xmin, ymin, zmin, array, markVal, lane,
                      32);
    return;
  }
  __syncwarp();  // the previous sphere's buffer is read by every lane
  if (lane < nk) dz2b[lane] = off2_rn(posz, hz, (double)(kmin + lane));
  __syncwarp();
  const int ni = imax - imin + 1, nj = jmax - jmin + 1;
  const size_t sz = (size_t)g.nx * g.ny;
  for (int t = lane; t < ni * nj; t += 32) {
    const int ii = imin + t % ni, jj = jmin + t / ni;
    const double dx2 = off2_rn(posx, hx, (double)ii);
    const double dy2 = off2_rn(posy, hy, (double)jj);
    if (__dadd_rn(dx2, dy2) > rtot2) continue;
    T* col = array + g.idx(ii, jj, 0);
    for (int q = 0; q < nk; q++)
      if (__dadd_rn(__dadd_rn(dz2b[q], dy2), dx2) <= rtot2) col[(kmin + q) * sz] = markVal;
  }
}

__global__ void k_fill_value(double* a, size_t n, double v) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x)
    a[q] = v;
}

// The dielectric maps of fillcoCoefMolDielNoSmooth (vpmg.c:4390-4496) take only
// two values, epsw and epsp, so they are built as one byte per point per
// staggered grid (0 = epsw, 1 = epsp) in the reference's order -- all epsw,
// the inflated atom spheres set to epsp, the probe spheres at accessible
// surface points back to epsw -- and written as doubles once, smoothed or
// not (k_diel_maps, k_smooth): an eighth of the bytes for the fill, the
// scattered marking and the smoothing's reads, the same maps bit for bit.
//
// Atom spheres (vpmg.c:4390-4446): one block per atom, the three staggered
// grids marked 1.
__global__ void k_mark_atoms_diel(FillGeom G, int natoms, const double* __restrict__ xyz,
                                  const double* __restrict__ r, double srad, DielMask M) {
  const int a = blockIdx.x;
  if (a >= natoms) return;
  const double ax = xyz[3 * a], ay = xyz[3 * a + 1], az = xyz[3 * a + 2], arad = r[a];
  if ((ax <= G.xmin[0]) || (ax >= G.xmax[0]) || (ay <= G.xmin[1]) || (ay >= G.xmax[1]) ||
      (az <= G.xmin[2]) || (az >= G.xmax[2]))
    return;
  if (!(arad > 1.0e-9)) return;
  const double hx = G.h[0], hy = G.h[1], hz = G.h[2];
  const unsigned char one = 1;
  mark_sphere_group(arad + srad, ax, ay, az, G.g, hx, hy, hz, (G.xmin[0] + 0.5 * hx),
                    G.xmin[1], G.xmin[2], M.m[0], one, threadIdx.x, blockDim.x);
  mark_sphere_group(arad + srad, ax, ay, az, G.g, hx, hy, hz, G.xmin[0],
                    (G.xmin[1] + 0.5 * hy), G.xmin[2], M.m[1], one, threadIdx.x, blockDim.x);
  mark_sphere_group(arad + srad, ax, ay, az, G.g, hx, hy, hz, G.xmin[0], G.xmin[1],
                    (G.xmin[2] + 0.5 * hz), M.m[2], one, threadIdx.x, blockDim.x);
}

// Ion accessibility of fillcoCoefMolIon (vpmg.c:4237-4333).
__global__ void k_mark_atoms_kappa(FillGeom G, int natoms, const double* __restrict__ xyz,
                                   const double* __restrict__ r, double irad, double* kappa) {
  const int a = blockIdx.x;
  if (a >= natoms) return;
  const double ax = xyz[3 * a], ay = xyz[3 * a + 1], az = xyz[3 * a + 2], arad = r[a];
  if (!(arad > 1.0e-9)) return;
  if ((ax < (G.xmin[0] - irad - arad)) || (ax > (G.xmax[0] + irad + arad)) ||
      (ay < (G.xmin[1] - irad - arad)) || (ay > (G.xmax[1] + irad + arad)) ||
      (az < (G.xmin[2] - irad - arad)) || (az > (G.xmax[2] + irad + arad)))
    return;
  mark_sphere_group((irad + arad), ax, ay, az, G.g, G.h[0], G.h[1], G.h[2], G.xmin[0],
                    G.xmin[1], G.xmin[2], kappa, 0.0, threadIdx.x, blockDim.x);
}

// ---------------------------------------------------------------------------
// Solvent-accessible surface points (Vacc_atomSurf, src/generic/vacc.c:866-922)
// and their exclusion test (ivdwAccExclus, vacc.c:78-128).  The candidate
// blockers of a point come from a uniform cell grid whose cells are at least
// (max radius + probe) wide, so the 27 cells around the point hold every atom
// that can exclude it -- the same atoms the reference's Vclist cell holds
// (vclist.c:231-342); the decision is an exact FP64 comparison either way.
// ---------------------------------------------------------------------------
__global__ void k_cell_count(CellGrid C, int natoms, const double* __restrict__ xyz,
                             int* count, int* cell_of) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  int c[3];
  for (int d = 0; d < 3; d++) {
    int v = (int)floor((xyz[3 * a + d] - C.lo[d]) / C.cs);
    c[d] = min(max(v, 0), C.n[d] - 1);
  }
  const int cell = (c[2] * C.n[1] + c[1]) * C.n[0] + c[0];
  cell_of[a] = cell;
  atomicAdd(count + cell, 1);
}

__global__ void k_scan_single(const int* count, int n, int* start) {
  // one block: thread t sums a chunk of counts, the chunk sums are scanned
  // with warp shuffles, then each thread writes its chunk's prefixes
  __shared__ int wsum[32];
  const int t = threadIdx.x, nt = blockDim.x, lane = t & 31, w = t >> 5;
  const int chunk = (n + nt - 1) / nt;
  const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
  int s = 0;
  for (int i = lo; i < hi; i++) s += count[i];
  int v = s;  // inclusive scan within the warp
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) wsum[w] = v;
  __syncthreads();
  if (w == 0) {
    int u = (lane < nt / 32) ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, u, o);
      if (lane >= o) u += y;
    }
    wsum[lane] = u;
  }
  __syncthreads();
  int acc = v - s + (w > 0 ? wsum[w - 1] : 0);
  for (int i = lo; i < hi; i++) {
    start[i] = acc;
    acc += count[i];
  }
  if (t == nt - 1) start[n] = acc;
}

__global__ void k_cell_fill(int natoms, const int* __restrict__ cell_of, int* fillpos,
                            int* atoms_sorted) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  const int p = atomicAdd(fillpos + cell_of[a], 1);
  atoms_sorted[p] = a;
}

// Surface point t of atom a: (r_a + srad) ref_t + x_a (Vacc_atomSurf,
// vacc.c:889-891), rounded as the reference computes it.
__device__ __forceinline__ void sas_point(const double* __restrict__ xyz,
                                          const double* __restrict__ r,
                                          const double* __restrict__ ref, int a, int t,
                                          double srad, double& px, double& py, double& pz) {
  const double rad = r[a] + srad;
  px = __dadd_rn(__dmul_rn(rad, ref[3 * t + 0]), xyz[3 * a + 0]);
  py = __dadd_rn(__dmul_rn(rad, ref[3 * t + 1]), xyz[3 * a + 1]);
  pz = __dadd_rn(__dmul_rn(rad, ref[3 * t + 2]), xyz[3 * a + 2]);
}
// ivdwAccExclus's squared distance (vacc.c:118-119)
__device__ __forceinline__ double dist2_rn(double d0, double d1, double d2) {
  return __dadd_rn(__dadd_rn(sq_rn(d0), sq_rn(d1)), sq_rn(d2));
}

// The atoms that can exclude a surface point of atom a: a point lies at
// r_a + srad from a, and b excludes it only within r_b + srad, so b is
// within r_a + r_b + 2 srad of a.  One warp per atom collects them from the
// cells within two cell edges (the cell edge is max r + srad) into a list of
// up to kNbrCap entries; a longer list is only counted, and its atom's
// points fall back to the cell search.  Any superset of the possible
// excluders, in any order, gives the same exclusion decisions; the cells are
// visited centre-out (kCellRing) so that the nearest atoms, which exclude
// most buried points, come first in the list.
constexpr int kNbrCap = 512;

// the 125 cell offsets (dx, dy, dz) in -2..2, coded 25 (dz+2) + 5 (dy+2) + (dx+2),
// sorted by dx^2 + dy^2 + dz^2
struct CellRing {
  int v[125];
  constexpr CellRing() : v() {
    int n = 0;
    for (int d2 = 0; d2 <= 12; d2++)
      for (int code = 0; code < 125; code++) {
        const int dx = code % 5 - 2, dy = (code / 5) % 5 - 2, dz = code / 25 - 2;
        if (dx * dx + dy * dy + dz * dz == d2) v[n++] = code;
      }
  }
};
__constant__ CellRing kCellRingTab = CellRing();
#define kCellRing (kCellRingTab.v)

__global__ void k_sas_nbr(CellGrid C, int natoms, const double* __restrict__ xyz,
                          const double* __restrict__ r, double srad,
                          const int* __restrict__ start, const int* __restrict__ atoms_sorted,
                          int* nbr, int* ncount) {
  const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (a >= natoms) return;
  const double ax = xyz[3 * a], ay = xyz[3 * a + 1], az = xyz[3 * a + 2];
  int c[3];
  const double pp[3] = {ax, ay, az};
  for (int d = 0; d < 3; d++) c[d] = (int)floor((pp[d] - C.lo[d]) / C.cs);
  int count = 0;
  for (int o = 0; o < 125; o++) {
        const int code = kCellRing[o];
        const int cx = c[0] + (code % 5) - 2, cy = c[1] + (code / 5) % 5 - 2,
                  cz = c[2] + code / 25 - 2;
        if (cx < 0 || cy < 0 || cz < 0 || cx >= C.n[0] || cy >= C.n[1] || cz >= C.n[2])
          continue;
        const int cell = (cz * C.n[1] + cy) * C.n[0] + cx;
        const int s0 = start[cell], s1 = start[cell + 1];
        for (int base = s0; base < s1; base += 32) {
          const int s = base + lane;
          bool keep = false;
          int b = -1;
          if (s < s1) {
            b = atoms_sorted[s];
            if (b != a) {
              const double d0 = ax - xyz[3 * b], d1 = ay - xyz[3 * b + 1], d2 = az - xyz[3 * b + 2];
              const double cut = r[a] + r[b] + 2.0 * srad + 1.0e-6;
              keep = (d0 * d0 + d1 * d1 + d2 * d2) < cut * cut;
            }
          }
          const unsigned m = __ballot_sync(0xffffffffu, keep);
          const int slot = count + __popc(m & ((1u << lane) - 1u));
          if (keep && slot < kNbrCap) nbr[(size_t)a * kNbrCap + slot] = b;
          count += __popc(m);
        }
  }
  if (lane == 0) ncount[a] = count;
}

// One thread per (atom, reference point); the accessible points are appended
// to a list (warp-aggregated), so the marking pass runs over them only.
// Block row y takes atoms y, y + gridDim.y, ...: an atom's excluder list (coordinates and (r_b + srad)^2)
// is staged in shared memory once for the row's points.  The test is the
// reference's FP64 comparison, dist^2 < (r_b + srad)^2 (Vacc_atomSASPoints
// via ivdwAccExclus, src/generic/vacc.c).
__global__ void __launch_bounds__(256) k_sas_test(
    CellGrid C, int natoms, const double* __restrict__ xyz, const double* __restrict__ r,
    const double* __restrict__ ref, int nref, double srad, const int* __restrict__ start,
    const int* __restrict__ atoms_sorted, const int* __restrict__ nbr,
    const int* __restrict__ ncount, unsigned* list, int* npts) {
  __shared__ double4 ex[kNbrCap];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  for (int a = blockIdx.y; a < natoms; a += gridDim.y) {
    const double arad = r[a];
    if (arad < 1.0e-9) continue;  // the whole block: no points on this atom
    const int cnt = ncount[a];
    const bool staged = cnt <= kNbrCap;
    if (staged) {
      const int* lst = nbr + (size_t)a * kNbrCap;
      for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
        const int b = lst[q];
        const double rr = r[b] + srad;
        ex[q] = make_double4(xyz[3 * b], xyz[3 * b + 1], xyz[3 * b + 2], sq_rn(rr));
      }
      __syncthreads();
    }
    bool acc = false;
    if (t < nref) {
      double px, py, pz;
      sas_point(xyz, r, ref, a, t, srad, px, py, pz);
      acc = true;
      if (staged) {
        for (int q = 0; q < cnt; q++) {
          const double4 e = ex[q];
          if (dist2_rn(px - e.x, py - e.y, pz - e.z) < e.w) {
            acc = false;
            break;
          }
        }
      } else {
        auto excludes = [&](int b) {
          const double rr = r[b] + srad;
          return dist2_rn(px - xyz[3 * b], py - xyz[3 * b + 1], pz - xyz[3 * b + 2]) < sq_rn(rr);
        };
        int c[3];
        const double pp[3] = {px, py, pz};
        for (int d = 0; d < 3; d++) c[d] = (int)floor((pp[d] - C.lo[d]) / C.cs);
        for (int dz = -1; dz <= 1 && acc; dz++)
          for (int dy = -1; dy <= 1 && acc; dy++)
            for (int dx = -1; dx <= 1 && acc; dx++) {
              const int cx = c[0] + dx, cy = c[1] + dy, cz = c[2] + dz;
              if (cx < 0 || cy < 0 || cz < 0 || cx >= C.n[0] || cy >= C.n[1] || cz >= C.n[2])
                continue;
              const int cell = (cz * C.n[1] + cy) * C.n[0] + cx;
              for (int s = start[cell]; s < start[cell + 1]; s++) {
                const int b = atoms_sorted[s];
                if (b == a) continue;
                if (excludes(b)) {
                  acc = false;
                  break;
                }
              }
            }
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, acc);
    if (m) {
      const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(npts, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (acc) list[base + __popc(m & ((1u << lane) - 1u))] = (unsigned)a * (unsigned)nref + t;
    }
    __syncthreads();  // the next atom restages ex
  }
}

// Probe spheres around accessible SAS points reset the three dielectric
// grids to epsw, byte 0 (vpmg.c:4456-4496).  One warp per listed surface point; the
// grid is sized for the device and strides over the list, whose length the
// test pass left in *npts.
__global__ void k_sas_mark(FillGeom G, const double* __restrict__ xyz,
                           const double* __restrict__ r, const double* __restrict__ ref,
                           int nref, double srad, const unsigned* __restrict__ list,
                           const int* __restrict__ npts, DielMask M) {
  __shared__ double dz2s[8][32];  // one buffer per warp of the 256-thread block
  double* dz2b = dz2s[threadIdx.x >> 5];
  const int n = *npts;
  const int lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const double hx = G.h[0], hy = G.h[1], hz = G.h[2];
  for (long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; w < n;
       w += nwarps) {
    const unsigned tid = list[w];
    double px, py, pz;
    sas_point(xyz, r, ref, (int)(tid / (unsigned)nref), (int)(tid % (unsigned)nref), srad, px,
              py, pz);
    const unsigned char zero = 0;
    mark_sphere_warp(srad, px, py, pz, G.g, hx, hy, hz, (G.xmin[0] + 0.5 * hx), G.xmin[1],
                     G.xmin[2], M.m[0], zero, lane, dz2b);
    mark_sphere_warp(srad, px, py, pz, G.g, hx, hy, hz, G.xmin[0], (G.xmin[1] + 0.5 * hy),
                     G.xmin[2], M.m[1], zero, lane, dz2b);
    mark_sphere_warp(srad, px, py, pz, G.g, hx, hy, hz, G.xmin[0], G.xmin[1],
                     (G.xmin[2] + 0.5 * hz), M.m[2], zero, lane, dz2b);
  }
}

// 9-point harmonic-mean smoothing, fillcoCoefMolDielSmooth (vpmg.c:4500-4628),
// of the maps the byte maps describe: 1 / a is 1/epsp or 1/epsw (the correctly
// rounded quotients, as 1.0 / a gives them).
struct InvPair {
  const unsigned char* m0;
  const unsigned char* m1;
  const unsigned char* m2;
  double rp, rw;
  __device__ __forceinline__ double operator()(const unsigned char* m, size_t q) const {
    return __ldg(m + q) ? rp : rw;
  }
};

__global__ void k_smooth(Grid g, InvPair inv, double* epsx, double* epsy, double* epsz) {
  const unsigned char* a1 = inv.m0;
  const unsigned char* a2 = inv.m1;
  const unsigned char* a3 = inv.m2;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t n = g.n();
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    split3(q, nx, ny, i, j, k);
    double frac;
    int np;
    frac = inv(a1, q);
    frac += inv(a2, q);
    frac += inv(a3, q);
    np = 3;
    if (j > 0) { frac += inv(a2, g.idx(i, j - 1, k)); np += 1; }
    if (k > 0) { frac += inv(a3, g.idx(i, j, k - 1)); np += 1; }
    if (i < (nx - 1)) {
      frac += inv(a2, g.idx(i + 1, j, k));
      frac += inv(a3, g.idx(i + 1, j, k));
      np += 2;
      if (j > 0) { frac += inv(a2, g.idx(i + 1, j - 1, k)); np += 1; }
      if (k > 0) { frac += inv(a3, g.idx(i + 1, j, k - 1)); np += 1; }
    }
    epsx[q] = np / frac;

    frac = inv(a2, q);
    frac += inv(a1, q);
    frac += inv(a3, q);
    np = 3;
    if (i > 0) { frac += inv(a1, g.idx(i - 1, j, k)); np += 1; }
    if (k > 0) { frac += inv(a3, g.idx(i, j, k - 1)); np += 1; }
    if (j < (ny - 1)) {
      frac += inv(a1, g.idx(i, j + 1, k));
      frac += inv(a3, g.idx(i, j + 1, k));
      np += 2;
      if (i > 0) { frac += inv(a1, g.idx(i - 1, j + 1, k)); np += 1; }
      if (k > 0) { frac += inv(a3, g.idx(i, j + 1, k - 1)); np += 1; }
    }
    epsy[q] = np / frac;

    frac = inv(a3, q);
    frac += inv(a1, q);
    frac += inv(a2, q);
    np = 3;
    if (i > 0) { frac += inv(a1, g.idx(i - 1, j, k)); np += 1; }
    if (j > 0) { frac += inv(a2, g.idx(i, j - 1, k)); np += 1; }
    if (k < (nz - 1)) {
      frac += inv(a1, g.idx(i, j, k + 1));
      frac += inv(a2, g.idx(i, j, k + 1));
      np += 2;
      if (i > 0) { frac += inv(a1, g.idx(i - 1, j, k + 1)); np += 1; }
      if (j > 0) { frac += inv(a2, g.idx(i, j - 1, k + 1)); np += 1; }
    }
    epsz[q] = np / frac;
  }
}

// The unsmoothed maps (srfm mol) from the byte maps.
__global__ void k_diel_maps(size_t n, DielMask M, double epsp, double epsw, double* epsx,
                            double* epsy, double* epsz) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    epsx[q] = M.m[0][q] ? epsp : epsw;
    epsy[q] = M.m[1][q] ? epsp : epsw;
    epsz[q] = M.m[2][q] ? epsp : epsw;
  }
}

// ---------------------------------------------------------------------------
// sdh boundary (bcfl_sdh + multipolebc, vpmg.c:3369-3645).  The 13 moment
// sums run one per thread in atom order, as the reference accumulates them.
// ---------------------------------------------------------------------------
// Per-atom moment terms in parallel, then one thread per moment sums them in
// atom order (the reference's accumulation order, so the sums are bitwise
// those of the reference).
__global__ void k_sdh_terms(int natoms, const double* __restrict__ xyz,
                            const double* __restrict__ q, double cx, double cy, double cz,
                            double* terms) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  const double xr = xyz[3 * a] - cx, yr = xyz[3 * a + 1] - cy, zr = xyz[3 * a + 2] - cz;
  const double c = q[a];
  double tr[9];
  tr[0] = xr * xr * c; tr[1] = xr * yr * c; tr[2] = xr * zr * c;
  tr[3] = yr * xr * c; tr[4] = yr * yr * c; tr[5] = yr * zr * c;
  tr[6] = zr * xr * c; tr[7] = zr * yr * c; tr[8] = zr * zr * c;
  const double qave = (tr[0] + tr[4] + tr[8]) / 3.0;
  terms[0 * (size_t)natoms + a] = c;
  terms[1 * (size_t)natoms + a] = xr * c;
  terms[2 * (size_t)natoms + a] = yr * c;
  terms[3 * (size_t)natoms + a] = zr * c;
  for (int e = 0; e < 9; e++) {
    const double v = (e == 0 || e == 4 || e == 8) ? (tr[e] - qave) : (tr[e]);
    terms[(4 + e) * (size_t)natoms + a] = 1.5 * v;
  }
}

__global__ void k_sdh_moments(int natoms, const double* __restrict__ terms, double* mom) {
  // chunks of the 13 term rows are staged in shared memory by the whole
  // block; thread m then adds its row in atom order
  constexpr int CH = 384;
  __shared__ double buf[13][CH];
  double acc = 0.0;
  const int m = threadIdx.x;
  for (int a0 = 0; a0 < natoms; a0 += CH) {
    const int len = min(CH, natoms - a0);
    for (int t = threadIdx.x; t < 13 * CH; t += blockDim.x) {
      const int r = t / CH, c = t % CH;
      if (c < len) buf[r][c] = terms[(size_t)r * natoms + a0 + c];
    }
    __syncthreads();
    if (m < 13)
      for (int c = 0; c < len; c++) acc += buf[m][c];
    __syncthreads();
  }
  if (m < 13) mom[m] = acc;
}

__device__ void multipolebc(double r, double kappa, double eps_p, double eps_w, double rad,
                            double tsr[3]) {
  const double eps_r = eps_w / eps_p;
  const double r2 = r * r, r3 = r2 * r, r5 = r3 * r2;
  tsr[0] = (1.0 / eps_w) / r;
  tsr[1] = (1.0 / eps_w) * (-1.0) / r3;
  tsr[2] = (1.0 / eps_w) * (3.0) / r5;
  if (kappa < 1.0e-9) {
    tsr[1] = (3.0 * eps_r) / (1.0 + 2.0 * eps_r) * tsr[1];
    tsr[2] = (5.0 * eps_r) / (2.0 + 3.0 * eps_r) * tsr[2];
  } else {
    const double ka = kappa * rad, ka2 = ka * ka, ka3 = ka2 * ka;
    const double kr = kappa * r, kr2 = kr * kr;
    tsr[0] = exp(ka - kr) / (1.0 + ka) * tsr[0];
    tsr[1] = 3.0 * eps_r * exp(ka - kr) * (1.0 + kr) * tsr[1];
    tsr[1] = tsr[1] / (1.0 + ka + eps_r * (2.0 + 2.0 * ka + ka2));
    tsr[2] = 5.0 * eps_r * exp(ka - kr) * (3.0 + 3.0 * kr + kr2) * tsr[2];
    tsr[2] = tsr[2] / (6.0 + 6.0 * ka + 2.0 * ka2 + eps_r * (9.0 + 9.0 * ka + 4.0 * ka2 + ka3));
  }
}

// One thread per face point of the three face pairs; a grid point on an edge
// is evaluated once per face it belongs to (identical value).
__global__ void k_sdh_faces(SdhArgs A, const double* __restrict__ mom,
                            const double* __restrict__ xf, const double* __restrict__ yf,
                            const double* __restrict__ zf, double* gx, double* gy, double* gz) {
  const Grid g = A.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t fx = (size_t)ny * nz, fy = (size_t)nx * nz, fz = (size_t)nx * ny;
  const size_t tot = 2 * (fx + fy + fz);
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < tot;
       t += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    double* out;
    if (t < 2 * fx) {
      const int s = (int)(t / fx);
      const size_t rem = t % fx;
      k = (int)(rem / ny); j = (int)(rem % ny); i = s ? nx - 1 : 0;
      out = gx + t;
    } else if (t < 2 * fx + 2 * fy) {
      const size_t u = t - 2 * fx;
      const int s = (int)(u / fy);
      const size_t rem = u % fy;
      k = (int)(rem / nx); i = (int)(rem % nx); j = s ? ny - 1 : 0;
      out = gy + u;
    } else {
      const size_t u = t - 2 * fx - 2 * fy;
      const int s = (int)(u / fz);
      const size_t rem = u % fz;
      j = (int)(rem / nx); i = (int)(rem % nx); k = s ? nz - 1 : 0;
      out = gz + u;
    }
    const double xr = xf[i] - A.center[0], yr = yf[j] - A.center[1], zr = zf[k] - A.center[2];
    const double dist = sqrt((xr * xr) + (yr * yr) + (zr * zr));
    double t3[3];
    multipolebc(dist, A.xkappa, A.eps_p, A.eps_w, A.size, t3);
    const double pre = A.pre;
    const double sq = mom[0], ux = mom[1], uy = mom[2], uz = mom[3];
    const double qxx = mom[4] / 3.0, qxy = mom[5] / 3.0, qxz = mom[6] / 3.0;
    const double qyy = mom[8] / 3.0, qyz = mom[9] / 3.0, qzz = mom[12] / 3.0;
    double val = pre * sq * t3[0];
    val -= pre * ux * xr * t3[1];
    val -= pre * uy * yr * t3[1];
    val -= pre * uz * zr * t3[1];
    val += pre * qxx * xr * xr * t3[2];
    val += pre * qyy * yr * yr * t3[2];
    val += pre * qzz * zr * zr * t3[2];
    val += pre * 2.0 * qxy * xr * yr * t3[2];
    val += pre * 2.0 * qxz * xr * zr * t3[2];
    val += pre * 2.0 * qyz * yr * zr * t3[2];
    *out = val;
  }
}

// ccf = zkappa2 * kappa (Vpmg_solve, vpmg.c:436-448)
__global__ void k_ccf(size_t n, const double* __restrict__ kappa, double zkappa2, double* ccf) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x)
    ccf[q] = zkappa2 * kappa[q];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_fill_value(cudaStream_t s, double* a, size_t n, double v) {
  k_fill_value<<<blocks_for(n), kThreads, 0, s>>>(a, n, v);
}
// ---------------------------------------------------------------------------
// chgm spl0: fillcoChargeSpline1 (src/mg/vpmg.c:4986-5089), the charge of each
// on-mesh atom split trilinearly over its 8 nearest points (FP64 atomics:
// grid points shared by several atoms sum in a different order than the
// reference's atom loop).
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// bcfl mdh: bcflnew (src/mg/vpmg.c:3289-3367, packUnpack 3220-3287).  One
// thread per stored face value sums, over all atoms in atom order, the
// Debye-Hueckel potential of each charge at that boundary point (a point on
// several faces gets the same value on each); atoms are staged through
// shared memory in chunks.
// ---------------------------------------------------------------------------
constexpr int kMdhChunk = 256;

__global__ void __launch_bounds__(256) k_mdh_faces(MdhArgs A, int natoms,
                                                  const double* __restrict__ xyz,
                                                  const double* __restrict__ q,
                                                  const double* __restrict__ r) {
  __shared__ double sx[kMdhChunk], sy_[kMdhChunk], sz_[kMdhChunk], sq[kMdhChunk], sr[kMdhChunk];
  const int nx = A.g.nx, ny = A.g.ny, nz = A.g.nz;
  const long long nfx = 2LL * ny * nz, nfy = 2LL * nx * nz, nfz = 2LL * nx * ny;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool valid = t < nfx + nfy + nfz;
  double gxp = 0.0, gyp = 0.0, gzp = 0.0;
  double* dst = nullptr;
  if (valid) {
    if (t < nfx) {
      const int j = (int)(t % ny), k = (int)((t / ny) % nz), slot = (int)(t / ((long long)ny * nz));
      gxp = A.xf[slot ? nx - 1 : 0]; gyp = A.yf[j]; gzp = A.zf[k];
      dst = A.gx + t;
    } else if (t < nfx + nfy) {
      const long long u = t - nfx;
      const int i = (int)(u % nx), k = (int)((u / nx) % nz), slot = (int)(u / ((long long)nx * nz));
      gxp = A.xf[i]; gyp = A.yf[slot ? ny - 1 : 0]; gzp = A.zf[k];
      dst = A.gy + u;
    } else {
      const long long u = t - nfx - nfy;
      const int i = (int)(u % nx), j = (int)((u / nx) % ny), slot = (int)(u / ((long long)nx * ny));
      gxp = A.xf[i]; gyp = A.yf[j]; gzp = A.zf[slot ? nz - 1 : 0];
      dst = A.gz + u;
    }
  }
  const double ec = 1.6021773e-19;
  double val = 0.0;
  for (int a0 = 0; a0 < natoms; a0 += kMdhChunk) {
    const int na = min(kMdhChunk, natoms - a0);
    __syncthreads();
    for (int c = threadIdx.x; c < na; c += blockDim.x) {
      sx[c] = xyz[3 * (a0 + c)];
      sy_[c] = xyz[3 * (a0 + c) + 1];
      sz_[c] = xyz[3 * (a0 + c) + 2];
      sq[c] = ec * q[a0 + c];
      sr[c] = r[a0 + c];
    }
    __syncthreads();
    if (valid) {
      for (int c = 0; c < na; c++) {
        const double dx = gxp - sx[c], dy = gyp - sy_[c], dz = gzp - sz_[c];
        const double dist = sqrt((dx * dx) + (dy * dy) + (dz * dz));
        if (A.xkappa > 1.0e-9)
          val += A.pre1 * (sq[c] / dist) * exp(-A.xkappa * (dist - sr[c])) /
                 (1 + A.xkappa * sr[c]);
        else
          val += A.pre1 * (sq[c] / dist);
      }
    }
  }
  if (valid) *dst = 0.0 + val;
}

void launch_mdh(cudaStream_t s, const MdhArgs& A, int natoms, const double* xyz, const double* q,
                const double* r) {
  const long long total = 2LL * ((long long)A.g.ny * A.g.nz + (long long)A.g.nx * A.g.nz +
                                 (long long)A.g.nx * A.g.ny);
  k_mdh_faces<<<(int)((total + 255) / 256), 256, 0, s>>>(A, natoms, xyz, q, r);
}

// ---------------------------------------------------------------------------
// Vpmg_qfEnergyPoint (src/mg/vpmg.c:1704-1789) for chgm spl0: the potential
// interpolated trilinearly at each atom times its charge and its partition
// weight (Vpmg_setPart's atom rule for the domain box, vpmg.c:673-720);
// per-block partial sums, then one block adds them.
// ---------------------------------------------------------------------------
struct QfBox {
  int complement;   // weight 1 - membership of [lo, hi] instead of membership of the domain
  double lo[3], hi[3];
};

__global__ void __launch_bounds__(256) k_qf_point(FillGeom G, int natoms,
                                                 const double* __restrict__ xyz,
                                                 const double* __restrict__ q,
                                                 const double* __restrict__ u, double* part,
                                                 QfBox box) {
  __shared__ double sh[32];
  const int nx = G.g.nx, ny = G.g.ny, nz = G.g.nz;
  double acc = 0.0;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < natoms; a += gridDim.x * blockDim.x) {
    const double* pos = xyz + 3 * a;
    // Vpmg_setPart's atom weight (vpmg.c:680-723, no disjoint sides)
    double part_id = 1.0;
    for (int d = 0; d < 3; d++) {
      const double lo = box.complement ? box.lo[d] : G.xmin[d];
      const double hi = box.complement ? box.hi[d] : G.xmax[d];
      double ok;
      if ((pos[d] < hi) && (pos[d] > lo)) ok = 1;
      else if (fabs(pos[d] - lo) < 1.0e-12) ok = 1;
      else if (fabs(pos[d] - hi) < 1.0e-12) ok = 1;
      else ok = 0;
      part_id = (d == 0) ? ok : part_id * ok;
    }
    if (box.complement) {
      // extEnergy's flip (vpmg.c:2533-2534)
      if (part_id > 1.0e-9) part_id = 1.0;
      part_id = (1 - part_id) * (1.0 * 1.0 * 1.0);
    }
    const double fi = (pos[0] - G.xmin[0]) / G.h[0];
    const double fj = (pos[1] - G.xmin[1]) / G.h[1];
    const double fk = (pos[2] - G.xmin[2]) / G.h[2];
    const int ihi = (int)ceil(fi), ilo = (int)floor(fi);
    const int jhi = (int)ceil(fj), jlo = (int)floor(fj);
    const int khi = (int)ceil(fk), klo = (int)floor(fk);
    if (!(part_id > 0)) continue;
    if (!((ihi < nx) && (jhi < ny) && (khi < nz) && (ilo >= 0) && (jlo >= 0) && (klo >= 0)))
      continue;
    const double dx = fi - (double)(ilo), dy = fj - (double)(jlo), dz = fk - (double)(klo);
    auto U = [&](int i, int j, int k) { return u[((size_t)k * ny + j) * nx + i]; };
    const double uval =
        dx * dy * dz * U(ihi, jhi, khi) + dx * (1.0 - dy) * dz * U(ihi, jlo, khi) +
        dx * dy * (1.0 - dz) * U(ihi, jhi, klo) + dx * (1.0 - dy) * (1.0 - dz) * U(ihi, jlo, klo) +
        (1.0 - dx) * dy * dz * U(ilo, jhi, khi) + (1.0 - dx) * (1.0 - dy) * dz * U(ilo, jlo, khi) +
        (1.0 - dx) * dy * (1.0 - dz) * U(ilo, jhi, klo) +
        (1.0 - dx) * (1.0 - dy) * (1.0 - dz) * U(ilo, jlo, klo);
    acc += (uval * q[a] * part_id);
  }
  const double t = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_qf_point_final(const double* __restrict__ part, int nparts, double* out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[i];
  const double t = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) out[0] = t;
}

void launch_qf_point(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                     const double* q, const double* u, double* part, double* out,
                     const double* box) {
  const int nb = std::max(1, std::min(1184, (natoms + 255) / 256));
  QfBox b;
  b.complement = box ? 1 : 0;
  for (int d = 0; d < 3; d++) {
    b.lo[d] = box ? box[d] : 0.0;
    b.hi[d] = box ? box[3 + d] : 0.0;
  }
  k_qf_point<<<nb, 256, 0, s>>>(G, natoms, xyz, q, u, part, b);
  k_qf_point_final<<<1, 256, 0, s>>>(part, nb, out);
}

// ---------------------------------------------------------------------------
// Deterministic charge spreading.  Atoms inside the method's acceptance band
// are binned by the 8^3 tile of grid points that holds floor(position / h);
// an atom's stencil (floor - 1 .. ceil + 1 per axis) reaches at most the
// neighbouring tiles (the 5th-order B-spline's floor - 2 .. ceil + 2 too).
// One CTA per tile gathers the atoms of the 27 bins
// around it, sorts them by atom index and adds their contributions point by
// point in that order, each term the reference's expression.  A tile with
// more than kChCap candidates (far denser than any molecule) runs in passes
// over windows of kChCap consecutive atom indices, which keeps the order.
// ---------------------------------------------------------------------------
constexpr int kChTile = 8;
constexpr int kChCap = 512;
constexpr int kChThreads = 128;

// KIND 2: bspline2 (fillcoChargeSpline2), KIND 1: trilinear, KIND 4: 5th-order
// B-spline (fillcoPermanentMultipole)
template <int KIND>
__device__ __forceinline__ bool charge_in_band(const FillGeom& G, double ax, double ay,
                                               double az) {
  if (KIND == 4)
    return !((ax <= (G.xmin[0] - 2 * G.h[0])) || (ax >= (G.xmax[0] + 2 * G.h[0])) ||
             (ay <= (G.xmin[1] - 2 * G.h[1])) || (ay >= (G.xmax[1] + 2 * G.h[1])) ||
             (az <= (G.xmin[2] - 2 * G.h[2])) || (az >= (G.xmax[2] + 2 * G.h[2])));
  if (KIND == 2)
    return !((ax <= (G.xmin[0] - G.h[0])) || (ax >= (G.xmax[0] + G.h[0])) ||
             (ay <= (G.xmin[1] - G.h[1])) || (ay >= (G.xmax[1] + G.h[1])) ||
             (az <= (G.xmin[2] - G.h[2])) || (az >= (G.xmax[2] + G.h[2])));
  return !((ax <= G.xmin[0]) || (ax >= G.xmax[0]) || (ay <= G.xmin[1]) ||
           (ay >= G.xmax[1]) || (az <= G.xmin[2]) || (az >= G.xmax[2]));
}

__device__ __forceinline__ int charge_tile_axis(double f, int ntile) {
  const int fl = (int)floor(f);
  const int t = fl >= 0 ? fl / kChTile : -1;
  return min(max(t, 0), ntile - 1);
}

template <int KIND>
__device__ __forceinline__ int charge_tile(const FillGeom& G, const int* nt, const double* xyz,
                                           int a) {
  const double fi = (xyz[3 * a] - G.xmin[0]) / G.h[0];
  const double fj = (xyz[3 * a + 1] - G.xmin[1]) / G.h[1];
  const double fk = (xyz[3 * a + 2] - G.xmin[2]) / G.h[2];
  return (charge_tile_axis(fk, nt[2]) * nt[1] + charge_tile_axis(fj, nt[1])) * nt[0] +
         charge_tile_axis(fi, nt[0]);
}

struct ChargeTiles {
  int n[3];
};

template <int KIND>
__global__ void k_chtile_count(FillGeom G, ChargeTiles T, int natoms,
                               const double* __restrict__ xyz, int* count) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  if (!charge_in_band<KIND>(G, xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2])) return;
  atomicAdd(count + charge_tile<KIND>(G, T.n, xyz, a), 1);
}

template <int KIND>
__global__ void k_chtile_fill(FillGeom G, ChargeTiles T, int natoms,
                              const double* __restrict__ xyz, int* fillpos, int* atoms) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  if (!charge_in_band<KIND>(G, xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2])) return;
  atoms[atomicAdd(fillpos + charge_tile<KIND>(G, T.n, xyz, a), 1)] = a;
}

template <int KIND>
__global__ void __launch_bounds__(kChThreads) k_charge_gather(
    FillGeom G, ChargeTiles T, int natoms, const double* __restrict__ xyz,
    const double* __restrict__ q, double zmagic, const int* __restrict__ start,
    const int* __restrict__ atoms, double* charge) {
  // thread t owns the points (i, j) = (t % 8, (t / 8) % 8) of planes
  // t / 64 + 2 r of the tile, r = 0..3
  constexpr int PPT = kChTile * kChTile * kChTile / kChThreads;
  __shared__ int cand[kChCap], sorted[kChCap];
  __shared__ double cf[3][kChCap];  // fi, fj, fk
  __shared__ double cq[kChCap];     // q zmagic / (hx hy hz)
  __shared__ int cb[6][kChCap];     // stencil bounds per axis (lo, hi)
  __shared__ int ncand, total;
  const int tx = blockIdx.x % T.n[0], ty = (blockIdx.x / T.n[0]) % T.n[1];
  const int tz = blockIdx.x / (T.n[0] * T.n[1]);
  const int nx = G.g.nx, ny = G.g.ny, nz = G.g.nz;
  const double hx = G.h[0], hy = G.h[1], hz = G.h[2];
  const int i = tx * kChTile + threadIdx.x % kChTile;
  const int j = ty * kChTile + (threadIdx.x / kChTile) % kChTile;
  const int kb = tz * kChTile + threadIdx.x / (kChTile * kChTile);
  if (threadIdx.x == 0) total = 0;
  __syncthreads();
  // threads 0..26 own one neighbour bin each
  int b0 = 0, b1 = 0;
  if (threadIdx.x < 27) {
    const int bx = tx + threadIdx.x % 3 - 1, by = ty + (threadIdx.x / 3) % 3 - 1,
              bz = tz + threadIdx.x / 9 - 1;
    if (bx >= 0 && by >= 0 && bz >= 0 && bx < T.n[0] && by < T.n[1] && bz < T.n[2]) {
      const int b = (bz * T.n[1] + by) * T.n[0] + bx;
      b0 = start[b];
      b1 = start[b + 1];
      if (b1 > b0) atomicAdd(&total, b1 - b0);
    }
  }
  __syncthreads();
  const int tot = total;
  double acc[PPT];
#pragma unroll
  for (int r = 0; r < PPT; r++) acc[r] = 0.0;
  const int npass = tot <= kChCap ? (tot > 0 ? 1 : 0) : (natoms + kChCap - 1) / kChCap;
  for (int pass = 0; pass < npass; pass++) {
    const int wlo = npass == 1 ? 0 : pass * kChCap;
    const int whi = npass == 1 ? natoms : min(natoms, wlo + kChCap);
    if (threadIdx.x == 0) ncand = 0;
    __syncthreads();
    for (int e = b0; e < b1; e++) {
      const int a = atoms[e];
      if (a >= wlo && a < whi) cand[atomicAdd(&ncand, 1)] = a;
    }
    __syncthreads();
    const int nc = ncand;
    // rank sort by atom index (the indices are distinct)
    for (int e = threadIdx.x; e < nc; e += kChThreads) {
      const int key = cand[e];
      int rank = 0;
      for (int f = 0; f < nc; f++) rank += cand[f] < key;
      sorted[rank] = key;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nc; e += kChThreads) {
      const int a = sorted[e];
      const double px = xyz[3 * a] - G.xmin[0], py = xyz[3 * a + 1] - G.xmin[1],
                   pz = xyz[3 * a + 2] - G.xmin[2];
      const double fi = px / hx, fj = py / hy, fk = pz / hz;
      // fillcoPermanentMultipole scales by f = zmagic / (hx hy hzed) first
      cq[e] = KIND == 4 ? q[a] * (zmagic / (hx * hy * hz)) : q[a] * zmagic / (hx * hy * hz);
      cf[0][e] = fi;
      cf[1][e] = fj;
      cf[2][e] = fk;
      if (KIND == 4) {
        // the loop bounds of fillcoPermanentMultipole (vpmg.c:6937-6965)
        cb[0][e] = max((int)floor(fi) - 2, 0);
        cb[1][e] = min((int)ceil(fi) + 2, nx - 1);
        cb[2][e] = max((int)floor(fj) - 2, 0);
        cb[3][e] = min((int)ceil(fj) + 2, ny - 1);
        cb[4][e] = max((int)floor(fk) - 2, 0);
        cb[5][e] = min((int)ceil(fk) + 2, nz - 1);
      } else if (KIND == 2) {
        // the loop bounds of fillcoChargeSpline2 (vpmg.c:5207-5224)
        cb[0][e] = max((int)floor(fi) - 1, 0);
        cb[1][e] = min((int)ceil(fi) + 1, nx - 1);
        cb[2][e] = max((int)floor(fj) - 1, 0);
        cb[3][e] = min((int)ceil(fj) + 1, ny - 1);
        cb[4][e] = max((int)floor(fk) - 1, 0);
        cb[5][e] = min((int)ceil(fk) + 1, nz - 1);
      } else {
        cb[0][e] = (int)floor(fi);
        cb[1][e] = (int)ceil(fi);
        cb[2][e] = (int)floor(fj);
        cb[3][e] = (int)ceil(fj);
        cb[4][e] = (int)floor(fk);
        cb[5][e] = (int)ceil(fk);
      }
    }
    __syncthreads();
    if (i < nx && j < ny) {
      for (int e = 0; e < nc; e++) {
        if (KIND == 4) {
          if (i < cb[0][e] || i > cb[1][e] || j < cb[2][e] || j > cb[3][e]) continue;
          const double c = cq[e], fk = cf[2][e];
          const double mi = (2.5 + ((double)(i) - (cf[0][e])));
          const double mj = (2.5 + ((double)(j) - (cf[1][e])));
          const double mx = bspline4(mi), dmx = dbspline4(mi), d2mx = d2bspline4(mi);
          const double my = bspline4(mj), dmy = dbspline4(mj), d2my = d2bspline4(mj);
          // the dipole and quadrupole terms of the reference's expression,
          // with the zero moments of plain atomic charges
          const double ux = 0.0, uy = 0.0, uz = 0.0, qxx = 0.0, qyx = 0.0, qyy = 0.0,
                       qzx = 0.0, qzy = 0.0, qzz = 0.0;
#pragma unroll
          for (int r = 0; r < PPT; r++) {
            const int k = kb + 2 * r;
            if (k < cb[4][e] || k > cb[5][e]) continue;
            const double mk = (2.5 + ((double)(k) - (fk)));
            const double mz = bspline4(mk), dmz = dbspline4(mk), d2mz = d2bspline4(mk);
            acc[r] += mx * my * mz * c - dmx * my * mz * ux - mx * dmy * mz * uy -
                      mx * my * dmz * uz + d2mx * my * mz * qxx + dmx * dmy * mz * qyx +
                      mx * d2my * mz * qyy + dmx * my * dmz * qzx + mx * dmy * dmz * qzy +
                      mx * my * d2mz * qzz;
          }
        } else if (KIND == 2) {
          if (i < cb[0][e] || i > cb[1][e] || j < cb[2][e] || j > cb[3][e]) continue;
          const double c = cq[e], fk = cf[2][e];
          const double mx = bspline2(1.5 + ((double)i - cf[0][e]));
          const double my = bspline2(1.5 + ((double)j - cf[1][e]));
#pragma unroll
          for (int r = 0; r < PPT; r++) {
            const int k = kb + 2 * r;
            if (k < cb[4][e] || k > cb[5][e]) continue;
            const double mz = bspline2(1.5 + ((double)k - fk));
            acc[r] += (c * mx * my * mz);
          }
        } else {
          const int ilo = cb[0][e], ihi = cb[1][e], jlo = cb[2][e], jhi = cb[3][e];
          const int klo = cb[4][e], khi = cb[5][e];
          if ((i != ihi && i != ilo) || (j != jhi && j != jlo)) continue;
          const double c = cq[e];
          const double dx = cf[0][e] - (double)(ilo), dy = cf[1][e] - (double)(jlo),
                       dz = cf[2][e] - (double)(klo);
#pragma unroll
          for (int r = 0; r < PPT; r++) {
            const int k = kb + 2 * r;
            if (k != khi && k != klo) continue;
            double v = acc[r];
            // the eight corner terms in the reference's statement order
            if (i == ihi && j == jhi && k == khi) v += (dx * dy * dz * c);
            if (i == ihi && j == jlo && k == khi) v += (dx * (1.0 - dy) * dz * c);
            if (i == ihi && j == jhi && k == klo) v += (dx * dy * (1.0 - dz) * c);
            if (i == ihi && j == jlo && k == klo) v += (dx * (1.0 - dy) * (1.0 - dz) * c);
            if (i == ilo && j == jhi && k == khi) v += ((1.0 - dx) * dy * dz * c);
            if (i == ilo && j == jlo && k == khi) v += ((1.0 - dx) * (1.0 - dy) * dz * c);
            if (i == ilo && j == jhi && k == klo) v += ((1.0 - dx) * dy * (1.0 - dz) * c);
            if (i == ilo && j == jlo && k == klo)
              v += ((1.0 - dx) * (1.0 - dy) * (1.0 - dz) * c);
            acc[r] = v;
          }
        }
      }
    }
    __syncthreads();  // the next pass refills the candidate arrays
  }
  if (i < nx && j < ny)
#pragma unroll
    for (int r = 0; r < PPT; r++) {
      const int k = kb + 2 * r;
      if (k < nz) charge[G.g.idx(i, j, k)] = acc[r];
    }
}

size_t charge_tile_count(const Grid& g) {
  return (size_t)((g.nx + kChTile - 1) / kChTile) * ((g.ny + kChTile - 1) / kChTile) *
         ((g.nz + kChTile - 1) / kChTile);
}

// kind 2: bspline2, 1: trilinear, 4: 5th-order B-spline.  count, start, fillpos: charge_tile_count + 1
// ints; atoms: natoms ints.  Every point of the map is written.
void launch_charge(cudaStream_t s, int kind, const FillGeom& G, int natoms, const double* xyz,
                   const double* q, double zmagic, int* count, int* start, int* fillpos,
                   int* atoms, double* charge) {
  ChargeTiles T;
  T.n[0] = (G.g.nx + kChTile - 1) / kChTile;
  T.n[1] = (G.g.ny + kChTile - 1) / kChTile;
  T.n[2] = (G.g.nz + kChTile - 1) / kChTile;
  const int nt = T.n[0] * T.n[1] * T.n[2];
  const int nb = std::max(1, (natoms + 255) / 256);
  cudaMemsetAsync(count, 0, sizeof(int) * nt, s);
  if (natoms > 0) {
    if (kind == 4) k_chtile_count<4><<<nb, 256, 0, s>>>(G, T, natoms, xyz, count);
    else if (kind == 2) k_chtile_count<2><<<nb, 256, 0, s>>>(G, T, natoms, xyz, count);
    else k_chtile_count<1><<<nb, 256, 0, s>>>(G, T, natoms, xyz, count);
  }
  k_scan_single<<<1, 1024, 0, s>>>(count, nt, start);
  cudaMemcpyAsync(fillpos, start, sizeof(int) * nt, cudaMemcpyDeviceToDevice, s);
  if (natoms > 0) {
    if (kind == 4) k_chtile_fill<4><<<nb, 256, 0, s>>>(G, T, natoms, xyz, fillpos, atoms);
    else if (kind == 2) k_chtile_fill<2><<<nb, 256, 0, s>>>(G, T, natoms, xyz, fillpos, atoms);
    else k_chtile_fill<1><<<nb, 256, 0, s>>>(G, T, natoms, xyz, fillpos, atoms);
  }
  if (kind == 4)
    k_charge_gather<4><<<nt, kChThreads, 0, s>>>(G, T, natoms, xyz, q, zmagic, start, atoms,
                                                 charge);
  else if (kind == 2)
    k_charge_gather<2><<<nt, kChThreads, 0, s>>>(G, T, natoms, xyz, q, zmagic, start, atoms,
                                                 charge);
  else
    k_charge_gather<1><<<nt, kChThreads, 0, s>>>(G, T, natoms, xyz, q, zmagic, start, atoms,
                                                 charge);
}

void launch_mark_atoms_diel(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                            const double* r, double srad, const DielMask& M) {
  if (natoms <= 0) return;
  k_mark_atoms_diel<<<natoms, 256, 0, s>>>(G, natoms, xyz, r, srad, M);
}
void launch_mark_atoms_kappa(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                             const double* r, double irad, double* kappa) {
  if (natoms <= 0) return;
  k_mark_atoms_kappa<<<natoms, 256, 0, s>>>(G, natoms, xyz, r, irad, kappa);
}
void launch_cell_build(cudaStream_t s, const CellGrid& C, int natoms, const double* xyz,
                       int* count, int* start, int* fillpos, int* cell_of, int* sorted) {
  const int ncell = C.n[0] * C.n[1] * C.n[2];
  cudaMemsetAsync(count, 0, sizeof(int) * ncell, s);
  k_cell_count<<<(natoms + 255) / 256, 256, 0, s>>>(C, natoms, xyz, count, cell_of);
  k_scan_single<<<1, 1024, 0, s>>>(count, ncell, start);
  cudaMemcpyAsync(fillpos, start, sizeof(int) * ncell, cudaMemcpyDeviceToDevice, s);
  k_cell_fill<<<(natoms + 255) / 256, 256, 0, s>>>(natoms, cell_of, fillpos, sorted);
}
size_t sas_nbr_ints(int natoms) { return (size_t)natoms * (kNbrCap + 1); }

void launch_sas_test(cudaStream_t s, const CellGrid& C, int natoms, const double* xyz,
                     const double* r, const double* ref, int nref, double srad,
                     const int* start, const int* sorted, int* nbr, unsigned* list, int* npts) {
  const long long tot = (long long)natoms * nref;
  if (tot <= 0) return;
  cudaMemsetAsync(npts, 0, sizeof(int), s);
  int* ncount = nbr + (size_t)natoms * kNbrCap;
  k_sas_nbr<<<(natoms + 7) / 8, 256, 0, s>>>(C, natoms, xyz, r, srad, start, sorted, nbr, ncount);
  k_sas_test<<<dim3((nref + 255) / 256, std::min(natoms, 65535)), 256, 0, s>>>(
      C, natoms, xyz, r, ref, nref, srad, start, sorted, nbr, ncount, list, npts);
}

void launch_sas_mark(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                     const double* r, const double* ref, int nref, double srad,
                     const unsigned* list, const int* npts, const DielMask& M) {
  const long long tot = (long long)natoms * nref;
  if (tot <= 0) return;
  static const int nblocks = [] {
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sas_mark, 256, 0) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    return sms * per_sm;
  }();
  const long long want = (tot + 7) / 8;  // 8 warps per block
  const unsigned nb = (unsigned)std::min<long long>(nblocks, want);
  k_sas_mark<<<nb, 256, 0, s>>>(G, xyz, r, ref, nref, srad, list, npts, M);
}
void launch_diel_maps(cudaStream_t s, Grid g, const DielMask& M, int smooth, double epsp,
                      double epsw, double* epsx, double* epsy, double* epsz) {
  if (smooth) {
    InvPair inv{M.m[0], M.m[1], M.m[2], 1.0 / epsp, 1.0 / epsw};
    k_smooth<<<blocks_for(g.n()), kThreads, 0, s>>>(g, inv, epsx, epsy, epsz);
  } else {
    k_diel_maps<<<blocks_for(g.n()), kThreads, 0, s>>>(g.n(), M, epsp, epsw, epsx, epsy, epsz);
  }
}
void launch_sdh(cudaStream_t s, const SdhArgs& A, int natoms, const double* xyz,
                const double* q, double* terms, double* mom, const double* xf,
                const double* yf, const double* zf, double* gx, double* gy, double* gz) {
  k_sdh_terms<<<(natoms + 127) / 128, 128, 0, s>>>(natoms, xyz, q, A.center[0], A.center[1],
                                                   A.center[2], terms);
  k_sdh_moments<<<1, 256, 0, s>>>(natoms, terms, mom);
  const size_t tot = 2 * ((size_t)A.g.ny * A.g.nz + (size_t)A.g.nx * A.g.nz +
                          (size_t)A.g.nx * A.g.ny);
  k_sdh_faces<<<blocks_for(tot), kThreads, 0, s>>>(A, mom, xf, yf, zf, gx, gy, gz);
}
void launch_ccf(cudaStream_t s, size_t n, const double* kappa, double zkappa2, double* ccf) {
  k_ccf<<<blocks_for(n), kThreads, 0, s>>>(n, kappa, zkappa2, ccf);
}

}  // namespace pmgb
