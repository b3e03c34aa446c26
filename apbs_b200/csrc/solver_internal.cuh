// Internal state of one PMG calculation (shared by solver.cu and mixed.cu).
#pragma once
#include <vector>

#include "apbs_b200.h"
#include "fill_kernels.cuh"
#include "mg_kernels.cuh"

namespace pmgb {
struct MixedState;
void note_launches(long long n);
}  // namespace pmgb

struct pmgb_solver;
namespace pmgb {
// pmgb_fillco without waiting for the device: the fill is queued on the
// calculation's stream and its statistics are read when first asked for.
int fillco_issue(pmgb_solver* s, int natoms, const double* xyz, const double* charge,
                 const double* radius);
// usemap (maps.cu): whether coefficient / charge maps replace the atom
// fill, the map fill itself (synchronous, checks off-map reads), cleanup
int uses_coef_maps(const pmgb_solver* s);
int uses_charge_map(const pmgb_solver* s);
int fill_from_maps(pmgb_solver* s);
void free_maps(pmgb_solver* s);
// bcfl map: the faces from the potential map (focus.cu)
int map_faces(pmgb_solver* s);
}  // namespace pmgb

namespace pmgb {

struct Level {
  Grid g;
  int nop;
  double* op[14];
  double* cc;
  double* fc;
  double* x;
  double* w0;
  double* cp;   // Newton: c'(u)
  double* rhs;  // Newton: rhs
  double* xt;   // Newton: correction
  Op ops() const {
    Op o;
    for (int c = 0; c < 14; c++) o.c[c] = (c < nop) ? op[c] : nullptr;
    o.nop = nop;
    return o;
  }
};

// Scalar slots in device memory.
enum Scal { S_RSDEN = 0, S_RSNRM, S_XNUM, S_XDEN, S_NRM, S_E0, S_E1, S_E2, S_E3, S_TMP,
            S_XNUM_L = 16, S_XDEN_L = 32, S_COUNT = 64 };

}  // namespace pmgb

using namespace pmgb;

// A coefficient or charge map on its own grid (pmgb_set_map), on the device.
struct UserMap {
  int n[3];
  double h[3], origin[3];
  double* data;  // IJK, NULL when the map is not used
};

struct pmgb_solver {
  // (types from namespace pmgb)
  pmgb_params p;
  int precision;
  int device;
  cudaStream_t stream;      // stream all work is issued on
  cudaStream_t own_stream;  // created with the solver
  // second stream of the fill: the charge map and the boundary values run on
  // it beside the dielectric and ion maps (forked from and joined to `stream`)
  cudaStream_t side;
  cudaEvent_t fork_ev, join_ev;
  size_t n;
  Grid g;
  // physics scalars (Vpbe_ctor2, src/generic/vpbe.c:264-450)
  double zmagic, xkappa, zkappa2, ionstr, maxIonRadius;
  double soluteCenter[3], soluteRadius;
  IonTable ions;    // scaled concentrations for c(u)
  IonTable ions_e;  // raw concentrations for the energy
  FillGeom G;
  // maps
  double *charge, *epsx, *epsy, *epsz, *kappa, *ccf;
  double *gx, *gy, *gz, *xf, *yf, *zf, *wx, *wy, *wz, *mom;
  unsigned char* dmask;  // the dielectric byte maps (DielMask), 3N bytes
  // atoms (d_* point at the owned buffers a_* or at the caller's arrays)
  int natoms;
  double *d_xyz, *d_q, *d_r;
  double *a_xyz, *a_q, *a_r;
  size_t atoms_cap;
  // hierarchy
  int nlev;
  Level lev[12];
  double *w1, *w2, *w3;
  double* xs;  // second fine iterate for the out-of-place sweep kernel (zero boundary)
  double* dg[2];  // fine-level oC + cc (dg[0]) and oC + c'(u) of the Newton system
                  // (dg[1]), 1 on the boundary: the single-pass sweep's divisor
  double *nw_r0, *nw_ws, *nw_keepx, *nw_keepr;  // Newton work vectors
  double* part;
  double* scal;
  double** d_opptrs;  // device table of operator pointers, 14 per level (16 levels)
  int* d_iters;
  int* d_info;
  // coarsest direct solve
  int mgsolv;
  double* band;
  int bn, bm, blda;
  // fill work
  // fill work, grown stream-ordered and geometrically (never shrinks)
  int *cell_count, *cell_start, *cell_fillpos, *cell_of, *cell_sorted;
  size_t ncell_alloc, cellof_alloc;
  unsigned* sas_list;  // accessible SAS points, (atom * nref + point)
  int* sas_nbr;        // per-atom lists of possible excluders, then their counts
  size_t sas_nbr_alloc;
  size_t sas_list_alloc;
  // srfm spl3: the per-atom window polynomials (spline3_table)
  double* d_spl3;
  size_t spl3_alloc;
  // atoms binned by tile of grid points for the charge gather
  int *ch_count, *ch_start, *ch_fill, *ch_atoms;
  size_t ch_tiles_alloc, ch_atoms_alloc;
  double* d_ref;
  int nref;
  size_t ref_alloc;
  int* d_npts;
  // step counters of the plane-parallel GS27 wavefront: word 0 counts waits
  // that ran out, level l's counters start at kWaveCounterBase + l *
  // kWavePlanesMax
  UserMap maps[PMGB_MAP_COUNT];  // usemap diel/kappa/charge
  double* map_scratch;      // kappa-map maximum and error counts
  double* d_forces;         // pmgb_forces: 9 doubles and a status word per atom
  size_t forces_alloc;
  unsigned* d_wave;
  int wave_used;  // the plane kernel has been launched or captured (stays set)
  // mailboxes of the shared-memory plane wavefront: level l's starts at word
  // mail_off[l] (levels it does not fit have none: mail_off[l] = -1); zeroed
  // with the step counters
  unsigned long long* d_mail;
  long long mail_off[12];
  size_t mail_total;
  double* atom_terms;  // 13 x natoms sdh moment terms
  size_t terms_alloc;
  // focusing: faces set from a coarse solution, energies outside the domain
  int focused;
  double ext_qf, ext_di, ext_qm;
  double* focus_w;  // coarse-grid partition weights for the external energy
  int focus_w_alloc;
  int tune[16];  // launch-shape tunables (PMGB_TUNE_*), copied from the defaults at creation
  // state
  int filled, solved, built;
  int fill_pending;  // fill issued without waiting; its statistics not yet read
  std::vector<double> reslog;
  pmgb_stats st;
  Gs27Plan plan[12];
  cudaEvent_t ev[8];
  // graphs of one V-cycle (linear / Newton system)
  cudaGraphExec_t vc_exec[2];
  long long vc_kernels[2];
  int vc_mgsolv[2];  // coarsest-solve kind each graph was captured with
  pmgb::MixedState* mixed;
};

