// Kernel declarations of the coefficient-map fill (fill.cu).
#pragma once
#include <vector>

#include "common.cuh"

namespace pmgb {

// the 5th-order B-spline and its first two derivatives (bspline4,
// dbspline4, d2bspline4, vpmg.c:6731-6822)
__device__ __forceinline__ double bspline4(double x) {
  const double one6 = 1.0 / 6.0, one8 = 1.0 / 8.0, one24 = 1.0 / 24.0;
  const double thirteen24 = 13.0 / 24.0, fourtyseven24 = 47.0 / 24.0,
               seventeen24 = 17.0 / 24.0;
  double m, m2;
  if ((x > 0.0) && (x <= 1.0)) {
    m = x * x;
    return one24 * m * m;
  } else if ((x > 1.0) && (x <= 2.0)) {
    m = x - 1.0;
    m2 = m * m;
    return -one8 + one6 * x + m2 * (0.25 + one6 * m - one6 * m2);
  } else if ((x > 2.0) && (x <= 3.0)) {
    m = x - 2.0;
    m2 = m * m;
    return -thirteen24 + 0.5 * x + m2 * (-0.25 - 0.5 * m + 0.25 * m2);
  } else if ((x > 3.0) && (x <= 4.0)) {
    m = x - 3.0;
    m2 = m * m;
    return fourtyseven24 - 0.5 * x + m2 * (-0.25 + 0.5 * m - one6 * m2);
  } else if ((x > 4.0) && (x <= 5.0)) {
    m = x - 4.0;
    m2 = m * m;
    return seventeen24 - one6 * x + m2 * (0.25 - one6 * m + one24 * m2);
  }
  return 0.0;
}
__device__ __forceinline__ double dbspline4(double x) {
  const double one6 = 1.0 / 6.0, one3 = 1.0 / 3.0, two3 = 2.0 / 3.0, thirteen6 = 13.0 / 6.0;
  double m, m2;
  if ((x > 0.0) && (x <= 1.0)) {
    m2 = x * x;
    return one6 * x * m2;
  } else if ((x > 1.0) && (x <= 2.0)) {
    m = x - 1.0;
    m2 = m * m;
    return -one3 + 0.5 * x + m2 * (0.5 - two3 * m);
  } else if ((x > 2.0) && (x <= 3.0)) {
    m = x - 2.0;
    m2 = m * m;
    return 1.5 - 0.5 * x + m2 * (-1.5 + m);
  } else if ((x > 3.0) && (x <= 4.0)) {
    m = x - 3.0;
    m2 = m * m;
    return 1.0 - 0.5 * x + m2 * (1.5 - two3 * m);
  } else if ((x > 4.0) && (x <= 5.0)) {
    m = x - 4.0;
    m2 = m * m;
    return -thirteen6 + 0.5 * x + m2 * (-0.5 + one6 * m);
  }
  return 0.0;
}
__device__ __forceinline__ double d2bspline4(double x) {
  double m, m2;
  if ((x > 0.0) && (x <= 1.0)) {
    return 0.5 * x * x;
  } else if ((x > 1.0) && (x <= 2.0)) {
    m = x - 1.0;
    m2 = m * m;
    return -0.5 + x - 2.0 * m2;
  } else if ((x > 2.0) && (x <= 3.0)) {
    m = x - 2.0;
    m2 = m * m;
    return 5.5 - 3.0 * x + 3.0 * m2;
  } else if ((x > 3.0) && (x <= 4.0)) {
    m = x - 3.0;
    m2 = m * m;
    return -9.5 + 3.0 * x - 2.0 * m2;
  } else if ((x > 4.0) && (x <= 5.0)) {
    m = x - 4.0;
    m2 = m * m;
    return 4.5 - x + 0.5 * m2;
  }
  return 0.0;
}

struct FillGeom {
  Grid g;
  double h[3];
  double xmin[3];
  double xmax[3];
};

// Uniform atom cell grid used for the SAS exclusion test.
struct CellGrid {
  double lo[3];
  double cs;   // cell edge >= max atom radius + probe radius
  int n[3];
};

struct SdhArgs {
  Grid g;
  double center[3];  // solute centre
  double size;       // solute radius
  double xkappa;
  double eps_p, eps_w;
  double pre;        // e^2 / (4 pi eps0 kB T) * 1e10
};

void launch_fill_value(cudaStream_t s, double* a, size_t n, double v);
struct MdhArgs {
  Grid g;
  const double* xf;
  const double* yf;
  const double* zf;
  double* gx;
  double* gy;
  double* gz;
  double pre1;    // e_c / (4 pi eps0 eps_w k_B T) * 1e10
  double xkappa;  // 1/A
};
// charge map by fillcoChargeSpline2 (kind 2), fillcoChargeSpline1 (kind 1)
// or fillcoPermanentMultipole's charges (kind 4), every point written, each point's terms added in atom order.  count,
// start and fillpos hold charge_tile_count(g) + 1 ints, atoms natoms ints.
size_t charge_tile_count(const Grid& g);
void launch_charge(cudaStream_t s, int kind, const FillGeom& G, int natoms, const double* xyz,
                   const double* q, double zmagic, int* count, int* start, int* fillpos,
                   int* atoms, double* charge);
void launch_mdh(cudaStream_t s, const MdhArgs& A, int natoms, const double* xyz, const double* q,
                const double* r);
// sum over atoms of the trilinearly interpolated potential x charge (part:
// up to 1184 doubles of scratch; out: one double)
// Vpmg_qfEnergyPoint (vpmg.c:1704-1789): sum of q u(atom) over the atoms on
// the mesh, each weighted by its partition weight.  With box == NULL the
// weight is the atom's membership of the calculation's own domain
// (Vpmg_setPart with the mg-manual partition); with box = {lo[3], hi[3]} it
// is 1 minus the membership of that box, the flipped weight extEnergy gives
// the coarse calculation of a focusing step (vpmg.c:2525-2535).
void launch_qf_point(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                     const double* q, const double* u, double* part, double* out,
                     const double* box = nullptr);
// The three staggered dielectric grids as one byte per point: 1 = epsp,
// 0 = epsw (the maps of fillcoCoefMolDielNoSmooth take no other value).
struct DielMask {
  unsigned char* m[3];
};
// inflated atom spheres set 1
void launch_mark_atoms_diel(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                            const double* r, double srad, const DielMask& M);
void launch_mark_atoms_kappa(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                             const double* r, double irad, double* kappa);
void launch_cell_build(cudaStream_t s, const CellGrid& C, int natoms, const double* xyz,
                       int* count, int* start, int* fillpos, int* cell_of, int* sorted);
// ints of the per-atom excluder lists launch_sas needs (nbr)
size_t sas_nbr_ints(int natoms);
// accessible SAS points into list (atom * nref + point), their count into *npts
void launch_sas_test(cudaStream_t s, const CellGrid& C, int natoms, const double* xyz,
                     const double* r, const double* ref, int nref, double srad,
                     const int* start, const int* sorted, int* nbr, unsigned* list, int* npts);
// probe spheres of the *npts accessible points of list set 0 (epsw)
void launch_sas_mark(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                     const double* r, const double* ref, int nref, double srad,
                     const unsigned* list, const int* npts, const DielMask& M);
// the dielectric maps from the byte maps: 9-point harmonic smoothing
// (smooth) or the unsmoothed values
void launch_diel_maps(cudaStream_t s, Grid g, const DielMask& M, int smooth, double epsp,
                      double epsw, double* epsx, double* epsy, double* epsz);
void launch_sdh(cudaStream_t s, const SdhArgs& A, int natoms, const double* xyz,
                const double* q, double* terms, double* mom, const double* xf, const double* yf,
                const double* zf, double* gx, double* gy, double* gz);
void launch_ccf(cudaStream_t s, size_t n, const double* kappa, double zkappa2, double* ccf);
// srfm spl2/spl4 kappa and dielectric maps (fillcoCoefSpline, fillcoCoefSpline4), spline.cu
void launch_spline_fill(cudaStream_t st, int order, const FillGeom& G, int natoms,
                        const double* xyz, const double* r, double irad, double win,
                        double ionmask, double epsp, double epsw, const double* coef3,
                        double* kappa, double* epsx, double* epsy, double* epsz);
// srfm spl3: 18 window-polynomial coefficients per atom (spline.cu)
void spline3_table(int natoms, const double* r, double irad, double win,
                   std::vector<double>& tab);

}  // namespace pmgb
