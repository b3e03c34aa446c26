// Kernel declarations of the coefficient-map fill (fill.cu).
#pragma once
#include "common.cuh"

namespace pmgb {

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
// charge map by fillcoChargeSpline2 (kind 2) or fillcoChargeSpline1 (kind
// 1), every point written, each point's terms added in atom order.  count,
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
void launch_mark_atoms_diel(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                            const double* r, double srad, double epsp, double* epsx,
                            double* epsy, double* epsz);
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
// probe spheres of the *npts accessible points of list reset the dielectric
// maps to epsw
void launch_sas_mark(cudaStream_t s, const FillGeom& G, int natoms, const double* xyz,
                     const double* r, const double* ref, int nref, double srad, double epsw,
                     const unsigned* list, const int* npts, double* epsx, double* epsy,
                     double* epsz);
// the 9-point harmonic smoothing of maps a1..a3 whose values are mostly v0 or v1
void launch_smooth(cudaStream_t s, Grid g, const double* a1, const double* a2,
                   const double* a3, double v0, double v1, double* epsx, double* epsy,
                   double* epsz);
void launch_sdh(cudaStream_t s, const SdhArgs& A, int natoms, const double* xyz,
                const double* q, double* terms, double* mom, const double* xf, const double* yf,
                const double* zf, double* gx, double* gy, double* gz);
void launch_ccf(cudaStream_t s, size_t n, const double* kappa, double zkappa2, double* ccf);
// srfm spl2/spl4 kappa and dielectric maps (fillcoCoefSpline, fillcoCoefSpline4), spline.cu
void launch_spline_fill(cudaStream_t st, int order, const FillGeom& G, int natoms,
                        const double* xyz, const double* r, double irad, double win,
                        double ionmask, double epsp, double epsw, double* kappa, double* epsx,
                        double* epsy, double* epsz);

}  // namespace pmgb
