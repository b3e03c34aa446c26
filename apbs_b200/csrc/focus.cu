// Focusing: boundary values of a fine calculation from a solved coarse one,
// and the coarse solution's energy outside the fine domain.
//
// focusFillBound (src/mg/vpmg.c:1914-2414) evaluates, for every point of the
// six faces of the fine grid, the trilinear interpolant of the coarse
// potential; extEnergy (vpmg.c:2416-2545) sums the coarse energies over the
// coarse points that the fine domain does not cover.  Both run here on the
// device against the coarse solver's resident potential and maps, so a
// focusing chain never copies a grid to the host.  The face values use the
// reference's expression for each point (this translation unit is compiled
// without fused multiply-add), so they equal the reference's bit for bit
// given the same coarse potential.
#include <math.h>

#include "solver_internal.cuh"

namespace pmgb {
void set_error(const char* fmt, ...);
void part_weights(int n, double h, double cent, double lo, double hi, double* w);
}  // namespace pmgb

namespace {

struct FocusArgs {
  const double* uc;  // coarse potential, boundary included
  int ncx, ncy, ncz;
  double hcx, hcy, hcz;
  double mnO[3], mxO[3];  // coarse domain corners
  int nfx, nfy, nfz;
  double hfx, hfy, hfz;
  double mnN[3], mxN[3];  // fine domain corners (snapped to the coarse ones)
  double* gx;  // fine faces, slots 0/1: gx[(slot*nz + k)*ny + j]
  double* gy;  //                        gy[(slot*nz + k)*nx + i]
  double* gz;  //                        gz[(slot*ny + j)*nx + i]
  int* status; // set to 1 when a face point lies off the coarse mesh
};

// One fine face point: the body of each face loop of focusFillBound
// (vpmg.c:2100-2129 and the five copies after it).
__device__ __forceinline__ double focus_point(const FocusArgs& a, double x, double y, double z) {
  const double small = 1.0e-9;  // VSMALL
  if (!((x >= (a.mnO[0] - small)) && (y >= (a.mnO[1] - small)) && (z >= (a.mnO[2] - small)) &&
        (x <= (a.mxO[0] + small)) && (y <= (a.mxO[1] + small)) && (z <= (a.mxO[2] + small)))) {
    atomicExch(a.status, 1);
    return 0.0;
  }
  const double ifl = (x - a.mnO[0]) / a.hcx;
  const double jfl = (y - a.mnO[1]) / a.hcy;
  const double kfl = (z - a.mnO[2]) / a.hcz;
  int ihi = (int)ceil(ifl);
  if (ihi > (a.ncx - 1)) ihi = a.ncx - 1;
  int ilo = (int)floor(ifl);
  if (ilo < 0) ilo = 0;
  int jhi = (int)ceil(jfl);
  if (jhi > (a.ncy - 1)) jhi = a.ncy - 1;
  int jlo = (int)floor(jfl);
  if (jlo < 0) jlo = 0;
  int khi = (int)ceil(kfl);
  if (khi > (a.ncz - 1)) khi = a.ncz - 1;
  int klo = (int)floor(kfl);
  if (klo < 0) klo = 0;
  const double dx = ifl - (double)(ilo);
  const double dy = jfl - (double)(jlo);
  const double dz = kfl - (double)(klo);
  const size_t sx = a.ncx, sxy = (size_t)a.ncx * a.ncy;
  const double* d = a.uc;
#define UC(i, j, k) d[(size_t)(k) * sxy + (size_t)(j) * sx + (i)]
  return dx * dy * dz * (UC(ihi, jhi, khi)) + dx * (1.0 - dy) * dz * (UC(ihi, jlo, khi)) +
         dx * dy * (1.0 - dz) * (UC(ihi, jhi, klo)) +
         dx * (1.0 - dy) * (1.0 - dz) * (UC(ihi, jlo, klo)) +
         (1.0 - dx) * dy * dz * (UC(ilo, jhi, khi)) +
         (1.0 - dx) * (1.0 - dy) * dz * (UC(ilo, jlo, khi)) +
         (1.0 - dx) * dy * (1.0 - dz) * (UC(ilo, jhi, klo)) +
         (1.0 - dx) * (1.0 - dy) * (1.0 - dz) * (UC(ilo, jlo, klo));
#undef UC
}

// One thread per stored face value: the x faces, then y, then z, each in
// its storage order, so consecutive threads write consecutive addresses.
__global__ void __launch_bounds__(256) k_focus_faces(FocusArgs a) {
  const long long nfx2 = 2LL * a.nfy * a.nfz, nfy2 = 2LL * a.nfx * a.nfz,
                  nfz2 = 2LL * a.nfx * a.nfy;
  const long long total = nfx2 + nfy2 + nfz2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    if (t < nfx2) {
      const int j = (int)(t % a.nfy);
      const long long r = t / a.nfy;
      const int k = (int)(r % a.nfz), slot = (int)(r / a.nfz);
      const double x = slot ? a.mxN[0] : a.mnN[0];
      const double y = a.mnN[1] + j * a.hfy;
      const double z = a.mnN[2] + k * a.hfz;
      a.gx[t] = focus_point(a, x, y, z);
    } else if (t < nfx2 + nfy2) {
      const long long u = t - nfx2;
      const int i = (int)(u % a.nfx);
      const long long r = u / a.nfx;
      const int k = (int)(r % a.nfz), slot = (int)(r / a.nfz);
      const double x = a.mnN[0] + i * a.hfx;
      const double y = slot ? a.mxN[1] : a.mnN[1];
      const double z = a.mnN[2] + k * a.hfz;
      a.gy[u] = focus_point(a, x, y, z);
    } else {
      const long long u = t - nfx2 - nfy2;
      const int i = (int)(u % a.nfx);
      const long long r = u / a.nfx;
      const int j = (int)(r % a.nfy), slot = (int)(r / a.nfy);
      const double x = a.mnN[0] + i * a.hfx;
      const double y = a.mnN[1] + j * a.hfy;
      const double z = slot ? a.mxN[2] : a.mnN[2];
      a.gz[u] = focus_point(a, x, y, z);
    }
  }
}

#define FCK(call)                                                                     \
  do {                                                                                \
    cudaError_t e__ = (call);                                                         \
    if (e__ != cudaSuccess) {                                                         \
      set_error("pmgb_focus: %s: %s", #call, cudaGetErrorString(e__));               \
      return 0;                                                                       \
    }                                                                                 \
  } while (0)

void domain(const pmgb_params& p, double mn[3], double mx[3]) {
  const int n[3] = {p.nx, p.ny, p.nz};
  const double h[3] = {p.hx, p.hy, p.hz};
  for (int d = 0; d < 3; d++) {
    mn[d] = p.center[d] - ((double)(n[d] - 1) * h[d]) / 2.0;
    mx[d] = p.center[d] + ((double)(n[d] - 1) * h[d]) / 2.0;
  }
}

}  // namespace

extern "C" int pmgb_focus(pmgb_solver* fine, pmgb_solver* coarse, int calc_energy) {
  if (!fine || !coarse || fine == coarse) {
    set_error("pmgb_focus: need two distinct solvers");
    return 0;
  }
  if (fine->p.bcfl != PMGB_BCFL_FOCUS) {
    set_error("pmgb_focus: the fine calculation must be created with bcfl focus");
    return 0;
  }
  // the coarse charge energy outside the fine box: a volume sum of the
  // charge map (spl2, or a charge map) or a point sum at the atoms (spl0, spl4)
  const int coarse_point_qf = coarse->p.chgm != PMGB_CHGM_SPL2 && !uses_charge_map(coarse);
  if (calc_energy && coarse_point_qf && (coarse->natoms <= 0 || !coarse->d_xyz)) {
    set_error("pmgb_focus: chgm spl0/spl4 needs the coarse calculation's atom list "
              "(pmgb_fillco)");
    return 0;
  }
  if (!coarse->solved) {
    set_error("pmgb_focus: the coarse calculation has not been solved");
    return 0;
  }
  int dev = -1;
  FCK(cudaGetDevice(&dev));
  if (fine->device != dev || coarse->device != dev) {
    set_error("pmgb_focus: both calculations must be on the current device");
    return 0;
  }
  const pmgb_params& pc = coarse->p;
  const pmgb_params& pf = fine->p;
  FocusArgs a;
  domain(pc, a.mnO, a.mxO);
  domain(pf, a.mnN, a.mxN);
  // "Check for rounding error" (vpmg.c:2054-2059)
  for (int d = 0; d < 3; d++) {
    if (fabs(a.mnO[d] - a.mnN[d]) < 1.0e-9) a.mnN[d] = a.mnO[d];
    if (fabs(a.mxO[d] - a.mxN[d]) < 1.0e-9) a.mxN[d] = a.mxO[d];
  }
  for (int d = 0; d < 3; d++)
    if (a.mxN[d] > a.mxO[d] || a.mnO[d] > a.mnN[d]) {
      set_error("pmgb_focus: fine mesh [%g, %g] on axis %d not contained in the coarse [%g, %g]",
                a.mnN[d], a.mxN[d], d, a.mnO[d], a.mxO[d]);
      return 0;
    }
  a.uc = coarse->lev[0].x;
  a.ncx = pc.nx;
  a.ncy = pc.ny;
  a.ncz = pc.nz;
  a.hcx = pc.hx;
  a.hcy = pc.hy;
  a.hcz = pc.hz;
  a.nfx = pf.nx;
  a.nfy = pf.ny;
  a.nfz = pf.nz;
  a.hfx = pf.hx;
  a.hfy = pf.hy;
  a.hfz = pf.hz;
  a.gx = fine->gx;
  a.gy = fine->gy;
  a.gz = fine->gz;
  a.status = fine->d_info + 8;  // slot 0 holds the band factor's info

  cudaStream_t st = fine->stream;
  cudaEvent_t coarse_done;
  FCK(cudaEventCreateWithFlags(&coarse_done, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(coarse_done, coarse->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, coarse_done, 0);
  cudaEventDestroy(coarse_done);
  if (e != cudaSuccess) {
    set_error("pmgb_focus: ordering after the coarse stream: %s", cudaGetErrorString(e));
    return 0;
  }
  FCK(cudaMemsetAsync(a.status, 0, sizeof(int), st));
  const long long total = 2LL * (pf.ny * (long long)pf.nz + pf.nx * (long long)pf.nz +
                                 pf.nx * (long long)pf.ny);
  const int blocks = (int)((total + 255) / 256 < 4 * 148 ? (total + 255) / 256 : 4 * 148);
  k_focus_faces<<<blocks, 256, 0, st>>>(a);
  note_launches(1);
  FCK(cudaGetLastError());

  double ext[3] = {0.0, 0.0, 0.0};
  double sums[4] = {0.0, 0.0, 0.0, 0.0};
  double qf_point = 0.0;
  if (calc_energy) {
    // extEnergy: coarse weights of the fine box, flipped (vpmg.c:2462-2509)
    const int nw = pc.nx + pc.ny + pc.nz;
    if (nw > fine->focus_w_alloc) {
      if (fine->focus_w) cudaFree(fine->focus_w);
      fine->focus_w = nullptr;
      fine->focus_w_alloc = 0;
      FCK(cudaMalloc(&fine->focus_w, sizeof(double) * nw));
      fine->focus_w_alloc = nw;
    }
    std::vector<double> w(nw);
    // the partition is the fine block's own (center -/+ glen/2)
    double lo[3], hi[3];
    domain(pf, lo, hi);
    part_weights(pc.nx, pc.hx, pc.center[0], lo[0], hi[0], w.data());
    part_weights(pc.ny, pc.hy, pc.center[1], lo[1], hi[1], w.data() + pc.nx);
    part_weights(pc.nz, pc.hz, pc.center[2], lo[2], hi[2], w.data() + pc.nx + pc.ny);
    FCK(cudaMemcpyAsync(fine->focus_w, w.data(), sizeof(double) * nw, cudaMemcpyHostToDevice,
                        st));
    EnergyArgs ea;
    ea.g = coarse->g;
    ea.u = coarse->lev[0].x;
    ea.charge = coarse->charge;
    ea.epsx = coarse->epsx;
    ea.epsy = coarse->epsy;
    ea.epsz = coarse->epsz;
    ea.kappa = coarse->kappa;
    ea.wx = fine->focus_w;
    ea.wy = fine->focus_w + pc.nx;
    ea.wz = fine->focus_w + pc.nx + pc.ny;
    ea.hx = pc.hx;
    ea.hy = pc.hy;
    ea.hz = pc.hz;
    ea.nonlin = 1;  // all three terms (Vpmg_qmEnergy, Vpmg_qfEnergy, Vpmg_dielEnergy)
    ea.ions = coarse->ions_e;
    ea.zks2 = (coarse->ionstr > 0.0) ? 0.5 * coarse->zkappa2 / coarse->ionstr : 0.0;
    ea.linear_qm = pc.nonlin ? 0 : 1;
    ea.zkappa2 = coarse->zkappa2;
    ea.complement = 1;
    // the coarse solver's reduction scratch, ordered on this stream after it
    launch_energy_sums(st, ea, coarse->part, coarse->scal + S_E0);
    note_launches(2);
    FCK(cudaMemcpyAsync(sums, coarse->scal + S_E0, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                        st));
    if (coarse_point_qf) {
      // Vpmg_qfEnergyPoint of the coarse calculation with the atoms' flipped
      // partition weights (vpmg.c:2518-2539)
      const double box[6] = {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]};
      launch_qf_point(st, coarse->G, coarse->natoms, coarse->d_xyz, coarse->d_q,
                      coarse->lev[0].x, coarse->part, coarse->scal + S_TMP, box);
      note_launches(2);
      FCK(cudaMemcpyAsync(&qf_point, coarse->scal + S_TMP, sizeof(double),
                          cudaMemcpyDeviceToHost, st));
    }
  }
  int status = 0;
  FCK(cudaMemcpyAsync(&status, a.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  FCK(cudaStreamSynchronize(st));
  if (status) {
    set_error("pmgb_focus: a fine face point lies off the coarse mesh");
    return 0;
  }
  if (calc_energy) {
    const double h3x = pc.hx, h3y = pc.hy, h3z = pc.hz;
    // Vpmg_qmEnergyNONLIN (vpmg.c:1437-1485)
    double qm = 0.0;
    if (!(coarse->zkappa2 < 1.0e-9)) {
      if (pc.nonlin) {
        if (sums[3] > 0.0) {
          set_error("pmgb_focus: clamped exponentials in the external mobile-ion energy");
          return 0;
        }
        qm = sums[2];
      } else {
        qm = 0.5 * sums[2];
      }
      qm = qm * h3x * h3y * h3z;
      qm = qm / coarse->zmagic;
      qm += coarse->ext_qm;
    }
    // Vpmg_qfEnergyVolume (vpmg.c:1883-1888) or Vpmg_qfEnergyPoint
    double qf = coarse_point_qf ? qf_point : sums[0] * h3x * h3y * h3z / coarse->zmagic;
    qf += coarse->ext_qf;
    // Vpmg_dielEnergy (vpmg.c:1333-1337)
    double di = 0.5 * sums[1] * h3x * h3y * h3z;
    di = di / coarse->zmagic;
    di += coarse->ext_di;
    ext[0] = qf;
    ext[1] = di;
    ext[2] = qm;
  }
  fine->ext_qf = ext[0];
  fine->ext_di = ext[1];
  fine->ext_qm = ext[2];
  fine->st.ext_qf = ext[0];
  fine->st.ext_diel = ext[1];
  fine->st.ext_qm = ext[2];
  fine->focused = 1;
  fine->built = 0;  // the fine right-hand side folds in the new faces
  fine->solved = 0;
  return 1;
}

// bcfl map (bcCalc, vpmg.c:4086-4089): the faces from a potential map, by
// the same interpolation focusFillBound applies to a coarse solution (it is
// called with the map standing in for the coarse grid, vpmg.c:2010-2025).
int pmgb::map_faces(pmgb_solver* s) {
  const UserMap& m = s->maps[PMGB_MAP_POT];
  if (!m.data) {
    set_error("pmgb_fillco: bcfl map needs a potential map (pmgb_set_map PMGB_MAP_POT)");
    return 0;
  }
  const pmgb_params& pf = s->p;
  FocusArgs a;
  for (int d = 0; d < 3; d++) {
    a.mnO[d] = m.origin[d];
    a.mxO[d] = m.origin[d] + (m.n[d] - 1) * m.h[d];  // Vgrid_ctor's xmax
  }
  domain(pf, a.mnN, a.mxN);
  for (int d = 0; d < 3; d++) {
    if (fabs(a.mnO[d] - a.mnN[d]) < 1.0e-9) a.mnN[d] = a.mnO[d];
    if (fabs(a.mxO[d] - a.mxN[d]) < 1.0e-9) a.mxN[d] = a.mxO[d];
  }
  for (int d = 0; d < 3; d++)
    if (a.mxN[d] > a.mxO[d] || a.mnO[d] > a.mnN[d]) {
      set_error("pmgb_fillco: grid [%g, %g] on axis %d not contained in the potential map "
                "[%g, %g]", a.mnN[d], a.mxN[d], d, a.mnO[d], a.mxO[d]);
      return 0;
    }
  a.uc = m.data;
  a.ncx = m.n[0]; a.ncy = m.n[1]; a.ncz = m.n[2];
  a.hcx = m.h[0]; a.hcy = m.h[1]; a.hcz = m.h[2];
  a.nfx = pf.nx; a.nfy = pf.ny; a.nfz = pf.nz;
  a.hfx = pf.hx; a.hfy = pf.hy; a.hfz = pf.hz;
  a.gx = s->gx; a.gy = s->gy; a.gz = s->gz;
  a.status = s->d_info + 8;
  cudaStream_t st = s->stream;
  FCK(cudaMemsetAsync(a.status, 0, sizeof(int), st));
  const long long total = 2LL * (pf.ny * (long long)pf.nz + pf.nx * (long long)pf.nz +
                                 pf.nx * (long long)pf.ny);
  const int blocks = (int)((total + 255) / 256 < 4 * 148 ? (total + 255) / 256 : 4 * 148);
  k_focus_faces<<<blocks, 256, 0, st>>>(a);
  note_launches(1);
  FCK(cudaGetLastError());
  int bad = 0;
  FCK(cudaMemcpyAsync(&bad, a.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  FCK(cudaStreamSynchronize(st));
  if (bad) {
    set_error("pmgb_fillco: a boundary point lies off the potential map");
    return 0;
  }
  return 1;
}
