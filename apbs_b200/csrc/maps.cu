// Coefficient and charge maps given on their own grids ("usemap diel",
// "usemap kappa", "usemap charge"): fillcoCoefMap (src/mg/vpmg.c:4098-4221)
// and fillcoChargeMap (4938-4984), each grid value taken from the map by
// Vgrid_value (src/mg/vgrid.c:179-270), and the OpenDX reader of the
// files those maps come in (Vgrid_readDX, vgrid.c:586-790).
//
// Vgrid_value interpolates trilinearly between the map points around the
// position; a position within 1e-4 (Vcompare) of a map edge snaps to it,
// and a position off the map is an error.  The kappa map is first scanned
// for its maximum (an error if negative anywhere) and divided by it when
// the maximum exceeds 1; values below VPMGSMALL become 0.  The dielectric
// maps are read at the staggered positions (x + h/2, y, z) etc.  Every
// point is independent, so one thread per grid point evaluates exactly the
// reference's expressions: the maps are bitwise those of the reference.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "apbs_b200.h"
#include "solver_internal.cuh"

namespace pmgb {
namespace {

constexpr double kPmgSmall = 1e-12;  // VPMGSMALL
constexpr double kVcompare = 1e-4;   // Vcompare = 10^-(VGRID_DIGITS-2)

struct DevMap {
  int nx, ny, nz;
  double hx, hy, hz, xmin, ymin, zmin, xmax, ymax, zmax;
  const double* data;
};

// Vgrid_value: 1 and the interpolated value on the map, 0 off it
__device__ __forceinline__ int map_value(const DevMap& m, double px, double py, double pz,
                                         double* value) {
  const double ifloat = (px - m.xmin) / m.hx;
  const double jfloat = (py - m.ymin) / m.hy;
  const double kfloat = (pz - m.zmin) / m.hz;
  long long ihi = (int)ceil(ifloat), jhi = (int)ceil(jfloat), khi = (int)ceil(kfloat);
  long long ilo = (int)floor(ifloat), jlo = (int)floor(jfloat), klo = (int)floor(kfloat);
  if (fabs(px - m.xmin) < kVcompare) ilo = 0;
  if (fabs(py - m.ymin) < kVcompare) jlo = 0;
  if (fabs(pz - m.zmin) < kVcompare) klo = 0;
  if (fabs(px - m.xmax) < kVcompare) ihi = m.nx - 1;
  if (fabs(py - m.ymax) < kVcompare) jhi = m.ny - 1;
  if (fabs(pz - m.zmax) < kVcompare) khi = m.nz - 1;
  // the reference keeps these indices unsigned: a negative one is off the map
  if (ihi < 0 || jhi < 0 || khi < 0 || ihi >= m.nx || jhi >= m.ny || khi >= m.nz) return 0;
  if (ilo < 0 || jlo < 0 || klo < 0) return 0;
  const double dx = ifloat - (double)(ilo);
  const double dy = jfloat - (double)(jlo);
  const double dz = kfloat - (double)(klo);
  auto D = [&](long long i, long long j, long long k) {
    return m.data[((size_t)k * m.ny + (size_t)j) * m.nx + (size_t)i];
  };
  const double u = dx * dy * dz * (D(ihi, jhi, khi)) + dx * (1.0 - dy) * dz * (D(ihi, jlo, khi)) +
                   dx * dy * (1.0 - dz) * (D(ihi, jhi, klo)) +
                   dx * (1.0 - dy) * (1.0 - dz) * (D(ihi, jlo, klo)) +
                   (1.0 - dx) * dy * dz * (D(ilo, jhi, khi)) +
                   (1.0 - dx) * (1.0 - dy) * dz * (D(ilo, jlo, khi)) +
                   (1.0 - dx) * dy * (1.0 - dz) * (D(ilo, jhi, klo)) +
                   (1.0 - dx) * (1.0 - dy) * (1.0 - dz) * (D(ilo, jlo, klo));
  *value = u;
  return 1;
}

struct MapFillArgs {
  Grid g;
  const double *xf, *yf, *zf;
  double hx, hy, hz;
  DevMap diel[3], kappa, charge;
  int use_coef, use_kappa, use_charge;
  double zmagic;
  double* kmax;      // [0] maximum of the kappa map over the grid points
  int* err;          // [0] off-map reads, [1] negative kappa
  double *epsx, *epsy, *epsz, *kap, *chg;
};

// atomicMax on a double known to be >= -1
__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
  unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
  unsigned long long old = *a;
  while (__longlong_as_double((long long)old) < v) {
    const unsigned long long prev =
        atomicCAS(a, old, (unsigned long long)__double_as_longlong(v));
    if (prev == old) break;
    old = prev;
  }
}

__global__ void k_map_kappa_max(MapFillArgs A) {
  const size_t n = A.g.n();
  double best = -1.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % A.g.nx), j = (int)((q / A.g.nx) % A.g.ny),
              k = (int)(q / ((size_t)A.g.nx * A.g.ny));
    double t;
    if (!map_value(A.kappa, A.xf[i], A.yf[j], A.zf[k], &t)) {
      atomicAdd(&A.err[0], 1);
      continue;
    }
    if (t > best) best = t;
    if (t < 0.0) atomicAdd(&A.err[1], 1);
  }
  for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_down_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomic_max_pos(A.kmax, best);
}

__global__ void k_map_fill(MapFillArgs A) {
  const size_t n = A.g.n();
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % A.g.nx), j = (int)((q / A.g.nx) % A.g.ny),
              k = (int)(q / ((size_t)A.g.nx * A.g.ny));
    const double x = A.xf[i], y = A.yf[j], z = A.zf[k];
    double v;
    if (A.use_charge) {
      if (map_value(A.charge, x, y, z, &v)) A.chg[q] = v * A.zmagic;
      else atomicAdd(&A.err[0], 1);
    }
    if (!A.use_coef) continue;
    if (A.use_kappa) {
      double kmax = A.kmax[0];
      if (!(kmax > 1.0)) kmax = 1.0;
      if (map_value(A.kappa, x, y, z, &v)) {
        if (v < kPmgSmall) v = 0.0;
        A.kap[q] = (v / kmax);
      } else {
        atomicAdd(&A.err[0], 1);
      }
    }
    if (map_value(A.diel[0], x + 0.5 * A.hx, y, z, &v)) A.epsx[q] = v;
    else atomicAdd(&A.err[0], 1);
    if (map_value(A.diel[1], x, y + 0.5 * A.hy, z, &v)) A.epsy[q] = v;
    else atomicAdd(&A.err[0], 1);
    if (map_value(A.diel[2], x, y, z + 0.5 * A.hz, &v)) A.epsz[q] = v;
    else atomicAdd(&A.err[0], 1);
  }
}

DevMap dev_map(const pmgb_solver* s, int which) {
  const UserMap& u = s->maps[which];
  DevMap m;
  m.nx = u.n[0]; m.ny = u.n[1]; m.nz = u.n[2];
  m.hx = u.h[0]; m.hy = u.h[1]; m.hz = u.h[2];
  m.xmin = u.origin[0]; m.ymin = u.origin[1]; m.zmin = u.origin[2];
  // Vgrid_ctor (vgrid.c:116-121)
  m.xmax = m.xmin + (m.nx - 1) * m.hx;
  m.ymax = m.ymin + (m.ny - 1) * m.hy;
  m.zmax = m.zmin + (m.nz - 1) * m.hz;
  m.data = u.data;
  return m;
}

}  // namespace

int uses_coef_maps(const pmgb_solver* s) {
  return s->maps[PMGB_MAP_DIELX].data || s->maps[PMGB_MAP_DIELY].data ||
         s->maps[PMGB_MAP_DIELZ].data || s->maps[PMGB_MAP_KAPPA].data;
}
int uses_charge_map(const pmgb_solver* s) { return s->maps[PMGB_MAP_CHARGE].data != nullptr; }

// The map part of pmgb_fillco; issued on the calculation's stream and
// checked before returning (off-map reads and negative kappa are errors).
int fill_from_maps(pmgb_solver* s) {
  const int coef = uses_coef_maps(s), chg = uses_charge_map(s);
  if (!coef && !chg) return 1;
  const int use_kappa = s->ionstr > kPmgSmall;
  if (coef && (!s->maps[PMGB_MAP_DIELX].data || !s->maps[PMGB_MAP_DIELY].data ||
               !s->maps[PMGB_MAP_DIELZ].data ||
               (use_kappa && !s->maps[PMGB_MAP_KAPPA].data))) {
    set_error("pmgb_fillco: coefficient maps need all three dielectric maps and, with "
              "ions, the kappa map (fillcoCoefMap)");
    return 0;
  }
  cudaStream_t st = s->stream;
  MapFillArgs A;
  A.g = s->g;
  A.xf = s->xf; A.yf = s->yf; A.zf = s->zf;
  A.hx = s->p.hx; A.hy = s->p.hy; A.hz = s->p.hz;
  for (int d = 0; d < 3; d++) A.diel[d] = dev_map(s, PMGB_MAP_DIELX + d);
  A.kappa = dev_map(s, PMGB_MAP_KAPPA);
  A.charge = dev_map(s, PMGB_MAP_CHARGE);
  A.use_coef = coef;
  A.use_kappa = coef && use_kappa;
  A.use_charge = chg;
  A.zmagic = s->zmagic;
  A.kmax = s->map_scratch;
  A.err = reinterpret_cast<int*>(s->map_scratch + 1);
  A.epsx = s->epsx; A.epsy = s->epsy; A.epsz = s->epsz; A.kap = s->kappa; A.chg = s->charge;
  const double minus_one = -1.0;
  PMGB_CUDA_OK(cudaMemcpyAsync(s->map_scratch, &minus_one, sizeof(double),
                               cudaMemcpyHostToDevice, st));
  PMGB_CUDA_OK(cudaMemsetAsync(s->map_scratch + 1, 0, 2 * sizeof(int), st));
  if (coef && !use_kappa) PMGB_CUDA_OK(cudaMemsetAsync(s->kappa, 0, s->n * sizeof(double), st));
  const int blocks = (int)std::min<size_t>((s->n + 255) / 256, 148 * 8);
  if (A.use_kappa) k_map_kappa_max<<<blocks, 256, 0, st>>>(A);
  k_map_fill<<<blocks, 256, 0, st>>>(A);
  note_launches(A.use_kappa ? 2 : 1);
  int err[2] = {0, 0};
  PMGB_CUDA_OK(cudaMemcpyAsync(err, A.err, sizeof(err), cudaMemcpyDeviceToHost, st));
  PMGB_CUDA_OK(cudaStreamSynchronize(st));
  if (err[0]) {
    set_error("pmgb_fillco: %d grid positions fall off a map (Vgrid_value)", err[0]);
    return 0;
  }
  if (err[1]) {
    set_error("pmgb_fillco: kappa map less than 0 at %d points", err[1]);
    return 0;
  }
  return 1;
}

void free_maps(pmgb_solver* s) {
  for (int w = 0; w < PMGB_MAP_COUNT; w++) {
    if (s->maps[w].data) cudaFree(s->maps[w].data);
    s->maps[w].data = nullptr;
  }
  if (s->map_scratch) cudaFree(s->map_scratch);
  s->map_scratch = nullptr;
}

}  // namespace pmgb

using namespace pmgb;

extern "C" int pmgb_set_map(pmgb_solver* s, int which, int nx, int ny, int nz, double hx,
                            double hy, double hz, double xmin, double ymin, double zmin,
                            const double* data) {
  if (!s || which < 0 || which >= PMGB_MAP_COUNT) {
    set_error("pmgb_set_map: bad calculation or map %d", which);
    return 0;
  }
  UserMap& m = s->maps[which];
  if (m.data) cudaFree(m.data);
  m.data = nullptr;
  if (!data) return 1;  // the map is no longer used
  if (nx < 2 || ny < 2 || nz < 2 || !(hx > 0) || !(hy > 0) || !(hz > 0)) {
    set_error("pmgb_set_map: bad map grid %dx%dx%d", nx, ny, nz);
    return 0;
  }
  const size_t n = (size_t)nx * ny * nz;
  PMGB_CUDA_OK(cudaMalloc((void**)&m.data, n * sizeof(double)));
  PMGB_CUDA_OK(cudaMemcpy(m.data, data, n * sizeof(double), cudaMemcpyHostToDevice));
  if (!s->map_scratch) PMGB_CUDA_OK(cudaMalloc((void**)&s->map_scratch, 4 * sizeof(double)));
  m.n[0] = nx; m.n[1] = ny; m.n[2] = nz;
  m.h[0] = hx; m.h[1] = hy; m.h[2] = hz;
  m.origin[0] = xmin; m.origin[1] = ymin; m.origin[2] = zmin;
  return 1;
}

// OpenDX reader (Vgrid_readDX, src/mg/vgrid.c:586-790): the grid positions
// (counts, origin, three deltas) and the "object 3" values, which the file
// stores x-major (z fastest); they are returned in the x-fastest IJK layout.
// With data NULL only the counts, spacings and origin are returned.
extern "C" int pmgb_read_dx_host(const char* path, int* dims, double* h, double* origin,
                                 double* data) {
  FILE* fp = path ? std::fopen(path, "r") : nullptr;
  if (!fp) {
    set_error("pmgb_read_dx_host: cannot open %s", path ? path : "(null)");
    return 0;
  }
  std::string text;
  {
    char buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), fp)) > 0) text.append(buf, got);
    std::fclose(fp);
  }
  // tokens, skipping '#' comments to the end of the line
  std::vector<std::pair<size_t, size_t>> tok;
  {
    size_t i = 0, n = text.size();
    while (i < n) {
      const char c = text[i];
      if (c == '#') {
        while (i < n && text[i] != '\n') i++;
      } else if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == ',') {
        i++;
      } else {
        const size_t a = i;
        while (i < n && !std::strchr(" \t\n\r,#", text[i])) i++;
        tok.emplace_back(a, i - a);
      }
    }
  }
  auto T = [&](size_t k) { return text.substr(tok[k].first, tok[k].second); };
  auto num = [&](size_t k) { return std::strtod(text.c_str() + tok[k].first, nullptr); };
  int n3[3] = {0, 0, 0};
  double o[3] = {0, 0, 0}, hh[3] = {0, 0, 0};
  size_t k = 0, ndelta = 0, items = 0, start = 0;
  bool got_counts = false, got_data = false;
  while (k < tok.size() && !got_data) {
    const std::string w = T(k);
    if (w == "counts" && !got_counts && k + 3 < tok.size()) {
      for (int d = 0; d < 3; d++) n3[d] = std::atoi(T(k + 1 + d).c_str());
      got_counts = true;
      k += 4;
    } else if (w == "origin" && k + 3 < tok.size()) {
      for (int d = 0; d < 3; d++) o[d] = num(k + 1 + d);
      k += 4;
    } else if (w == "delta" && k + 3 < tok.size() && ndelta < 3) {
      hh[ndelta] = num(k + 1 + ndelta);  // the diagonal entry of this delta
      ndelta++;
      k += 4;
    } else if (w == "items" && k + 1 < tok.size()) {
      items = (size_t)std::strtoull(T(k + 1).c_str(), nullptr, 10);
      k += 2;
      while (k < tok.size() && T(k) != "follows") k++;
      start = k + 1;
      got_data = true;
    } else {
      k++;
    }
  }
  if (!got_counts || !got_data || ndelta != 3 || n3[0] < 1 || n3[1] < 1 || n3[2] < 1 ||
      items != (size_t)n3[0] * n3[1] * n3[2] || start + items > tok.size()) {
    set_error("pmgb_read_dx_host: %s is not a regular-grid OpenDX file", path);
    return 0;
  }
  for (int d = 0; d < 3; d++) {
    if (dims) dims[d] = n3[d];
    if (h) h[d] = hh[d];
    if (origin) origin[d] = o[d];
  }
  if (data) {
    const int nx = n3[0], ny = n3[1], nz = n3[2];
    size_t t = start;
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny; j++)
        for (int kk = 0; kk < nz; kk++)
          data[((size_t)kk * ny + j) * nx + i] = num(t++);
  }
  return 1;
}
