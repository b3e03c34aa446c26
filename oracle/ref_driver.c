/*
 * ref_driver.c -- runs the REFERENCE APBS PMG path (compiled unchanged from
 * the reference sources by oracle/Makefile) on one mg-manual calculation.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and CPU baseline).  Built into
 * oracle/_ref/libapbsref.so; never linked into the product library.
 *
 * The call sequence mirrors initMG / solveMG / setPartMG / energyMG of the
 * reference (src/routines.c:1314-1606, 1635-1674, 1676-1724, 1726-1801) for
 * a single non-focused mg-manual ELEC block (ref_pmg_run) or a coarse block
 * followed by a bcfl-focus block (ref_pmg_focus), starting from an in-memory atom
 * list instead of a PQR file (Valist_readPQR, src/generic/valist.c:606, is
 * replaced by filling the Valist directly and calling Valist_getStatistics).
 */
#include <stdio.h>
#include <time.h>
#include "apbscfg.h"
#include "maloc/maloc.h"
#include "generic/vhal.h"
#include "generic/valist.h"
#include "generic/vatom.h"
#include "generic/vpbe.h"
#include "generic/mgparm.h"
#include "generic/pbeparm.h"
#include "mg/vgrid.h"
#include "mg/vpmgp.h"
#include "mg/vpmg.h"
#include "pmgb_params.h"

void oracle_shim_set_log(double *buf, int cap);
int oracle_shim_log_count(void);
int oracle_shim_iter_count(void);
void oracle_shim_set_verbose(int v);

/* spline window passed to Vpmg_fillco (the deck's swin, default 0.3) */
#define SWIN(p) (((p)->swin > 0.0) ? (p)->swin : 0.3)

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static Valist *make_alist(int natoms, const double *xyz, const double *q,
                          const double *r) {
    int i;
    Valist *alist = Valist_ctor();
    alist->atoms = (Vatom *)Vmem_malloc(alist->vmem, (size_t)natoms,
                                        sizeof(Vatom));
    alist->number = natoms;
    for (i = 0; i < natoms; i++) {
        Vatom *a = &(alist->atoms[i]);
        a->position[0] = xyz[3 * i + 0];
        a->position[1] = xyz[3 * i + 1];
        a->position[2] = xyz[3 * i + 2];
        a->charge = q[i];
        a->radius = r[i];
        a->partID = 1.0;
        a->epsilon = 0.0;
        a->id = i;
    }
    Valist_getStatistics(alist);
    return alist;
}

/* MGparm for an mg-manual block (fields read by Vpmgp_ctor2, vpmgp.c:93-170,
 * and Vpmg_ctor2, vpmg.c:153-399). */
static MGparm *make_mgparm(const pmgb_params *p) {
    int i;
    MGparm *mg = MGparm_ctor(MCT_MANUAL);
    mg->dime[0] = p->nx; mg->dime[1] = p->ny; mg->dime[2] = p->nz;
    mg->setdime = 1;
    mg->nlev = p->nlev; mg->setnlev = 1;
    mg->grid[0] = p->hx; mg->grid[1] = p->hy; mg->grid[2] = p->hz;
    mg->setgrid = 1;
    mg->glen[0] = (p->nx - 1) * p->hx;
    mg->glen[1] = (p->ny - 1) * p->hy;
    mg->glen[2] = (p->nz - 1) * p->hz;
    mg->setglen = 1;
    for (i = 0; i < 3; i++) mg->center[i] = p->center[i];
    mg->cmeth = MCM_POINT;
    mg->setgcent = 1;
    mg->chgm = (Vchrg_Meth)p->chgm; mg->setchgm = 1;
    mg->chgs = VCM_CHARGE;
    if (p->etol > 0.0) { mg->etol = p->etol; mg->setetol = 1; }
    mg->useAqua = 0;
    for (i = 0; i < 6; i++) mg->partDisjOwnSide[i] = 0;
    if (p->nonlin) {
        mg->nonlintype = NONLIN_NPBE;
        mg->method = VSOL_Newton;
    } else {
        mg->nonlintype = NONLIN_LPBE;
        mg->method = VSOL_MG;
    }
    return mg;
}

/*
 * Run ctor + fillco + solve + setPart + energy.
 *   u      (out, optional) potential, nx*ny*nz doubles, IJK = k*nx*ny+j*nx+i
 *   maps   (out, optional) 5*N doubles: charge, epsx, epsy, epsz, kappa
 *   faces  (out, optional) 2*(ny*nz + nx*nz + nx*ny) doubles: gxcf slots 0,1
 *          then gycf slots 0,1 then gzcf slots 0,1 (vpmg.h:1384-1386 layout)
 *   out    (out) [0] energy (kT) [1] V-cycle/Newton progress messages
 *          [2] residual-log entries [3] t_ctor [4] t_fillco [5] t_solve
 *          [6] t_energy (seconds) [7] qf [8] diel [9] qm (kT, NPBE only)
 *   reslog (out, optional) relative residual of every progress message
 *   forces (out, optional) 9 doubles per atom: Vpmg_qfForce, Vpmg_dbForce,
 *          Vpmg_ibForce (kT/A), the last two for the spline surfaces only
 *   fstatus (out, optional) per atom, 1 if both boundary forces succeeded
 * Returns 1 on success (Vpmg convention), 0 on failure.
 */
static int run_impl(const pmgb_params *p, int natoms, const double *xyz,
                    const double *q, const double *r, double *u, double *maps,
                    double *faces, double *out, double *reslog, int reslog_cap,
                    int verbose, double *forces, int *fstatus, Vgrid **umap);

int ref_pmg_run(const pmgb_params *p, int natoms, const double *xyz,
                const double *q, const double *r, double *u, double *maps,
                double *faces, double *out, double *reslog, int reslog_cap,
                int verbose, double *forces, int *fstatus) {
    return run_impl(p, natoms, xyz, q, r, u, maps, faces, out, reslog, reslog_cap, verbose,
                    forces, fstatus, NULL);
}

/* ref_pmg_run with "usemap" maps given to Vpmg_fillco (vpmg.c:5250-5316):
 * map m (0..5 = dielx, diely, dielz, kappa, charge, pot) is used when
 * data[m] is non-NULL, on the grid dims[3m..3m+2], spacing geom[6m..6m+2]
 * and origin geom[6m+3..6m+5] (the Vgrid a map file would give). */
int ref_pmg_run_maps(const pmgb_params *p, int natoms, const double *xyz, const double *q,
                     const double *r, const int *dims, const double *geom, double **data,
                     double *u, double *maps, double *out) {
    Vgrid *g[6];
    int m, rc;
    for (m = 0; m < 6; m++) {
        g[m] = VNULL;
        if (data[m])
            g[m] = Vgrid_ctor(dims[3 * m], dims[3 * m + 1], dims[3 * m + 2], geom[6 * m],
                              geom[6 * m + 1], geom[6 * m + 2], geom[6 * m + 3],
                              geom[6 * m + 4], geom[6 * m + 5], data[m]);
    }
    rc = run_impl(p, natoms, xyz, q, r, u, maps, NULL, out, NULL, 0, 0, NULL, NULL, g);
    for (m = 0; m < 6; m++)
        if (g[m]) Vgrid_dtor(&g[m]);
    return rc;
}

static int run_impl(const pmgb_params *p, int natoms, const double *xyz,
                    const double *q, const double *r, double *u, double *maps,
                    double *faces, double *out, double *reslog, int reslog_cap,
                    int verbose, double *forces, int *fstatus, Vgrid **umap) {
    int i, n, rc;
    double t0, t1, t2, t3, t4;
    double ionc[PMGB_MAXION], ionr[PMGB_MAXION], ionq[PMGB_MAXION];
    double partMin[3], partMax[3];
    Valist *alist;
    MGparm *mg;
    Vpbe *pbe;
    Vpmgp *pmgp;
    Vpmg *pmg;

    oracle_shim_set_verbose(verbose);
    oracle_shim_set_log(reslog, reslog_cap);
    for (i = 0; i < p->nion && i < PMGB_MAXION; i++) {
        ionc[i] = p->ion_conc[i];
        ionr[i] = p->ion_radius[i];
        ionq[i] = p->ion_q[i];
    }
    t0 = now_s();
    alist = make_alist(natoms, xyz, q, r);
    mg = make_mgparm(p);
    pbe = Vpbe_ctor(alist, p->nion, ionc, ionr, ionq, p->temp, p->pdie,
                    p->sdie, p->srad, 0, p->sdens, 0.0, 0.0, 0.0, 0.0);
    if (pbe == VNULL) return 0;
    pmgp = Vpmgp_ctor(mg);
    if (p->itmax > 0) pmgp->itmax = p->itmax;
    pmgp->bcfl = (Vbcfl)p->bcfl;
    pmgp->xcent = p->center[0];
    pmgp->ycent = p->center[1];
    pmgp->zcent = p->center[2];
    pmg = Vpmg_ctor(pmgp, pbe, 0, VNULL, mg, PCE_NO);
    t1 = now_s();
    if (umap)
        rc = Vpmg_fillco(pmg, (Vsurf_Meth)p->srfm, SWIN(p), (Vchrg_Meth)p->chgm,
                         umap[0] != VNULL, umap[0], umap[1] != VNULL, umap[1],
                         umap[2] != VNULL, umap[2], umap[3] != VNULL, umap[3],
                         umap[5] != VNULL, umap[5], umap[4] != VNULL, umap[4]);
    else
        rc = Vpmg_fillco(pmg, (Vsurf_Meth)p->srfm, SWIN(p), (Vchrg_Meth)p->chgm,
                         0, VNULL, 0, VNULL, 0, VNULL, 0, VNULL, 0, VNULL, 0,
                         VNULL);
    t2 = now_s();
    if (rc != 1) return 0;
    n = p->nx * p->ny * p->nz;
    if (maps) {
        memcpy(maps + 0 * (size_t)n, pmg->charge, sizeof(double) * n);
        memcpy(maps + 1 * (size_t)n, pmg->epsx, sizeof(double) * n);
        memcpy(maps + 2 * (size_t)n, pmg->epsy, sizeof(double) * n);
        memcpy(maps + 3 * (size_t)n, pmg->epsz, sizeof(double) * n);
        memcpy(maps + 4 * (size_t)n, pmg->kappa, sizeof(double) * n);
    }
    if (faces) {
        size_t fx = (size_t)p->ny * p->nz, fy = (size_t)p->nx * p->nz,
               fz = (size_t)p->nx * p->ny;
        memcpy(faces, pmg->gxcf, sizeof(double) * 2 * fx);
        memcpy(faces + 2 * fx, pmg->gycf, sizeof(double) * 2 * fy);
        memcpy(faces + 2 * fx + 2 * fy, pmg->gzcf, sizeof(double) * 2 * fz);
    }
    rc = Vpmg_solve(pmg);
    t3 = now_s();
    if (rc != 1) return 0;
    if (u) memcpy(u, pmg->u, sizeof(double) * n);
    for (i = 0; i < 3; i++) {
        partMin[i] = mg->center[i] - 0.5 * mg->glen[i];
        partMax[i] = mg->center[i] + 0.5 * mg->glen[i];
    }
    Vpmg_setPart(pmg, partMin, partMax, mg->partDisjOwnSide);
    if (forces) {
        /* per atom: charge-field, dielectric-boundary and ionic-boundary
         * forces as Vpmg_force assembles them (vpmg.c:5418-5438); the two
         * boundary forces only for spline surfaces (their status, 1/0, in
         * fstatus) */
        for (i = 0; i < natoms; i++) {
            int rcf = 1;
            Vpmg_qfForce(pmg, forces + 9 * (size_t)i, i, (Vchrg_Meth)p->chgm);
            if (p->srfm == PMGB_SRFM_SPL2 || p->srfm == PMGB_SRFM_SPL3 ||
                p->srfm == PMGB_SRFM_SPL4) {
                rcf &= Vpmg_dbForce(pmg, forces + 9 * (size_t)i + 3, i, (Vsurf_Meth)p->srfm);
                rcf &= Vpmg_ibForce(pmg, forces + 9 * (size_t)i + 6, i, (Vsurf_Meth)p->srfm);
            } else {
                int d;
                for (d = 3; d < 9; d++) forces[9 * (size_t)i + d] = 0.0;
            }
            if (fstatus) fstatus[i] = rcf;
        }
    }
    out[0] = Vpmg_energy(pmg, 1);
    t4 = now_s();
    out[1] = (double)oracle_shim_iter_count();
    out[2] = (double)oracle_shim_log_count();
    out[3] = t1 - t0;
    out[4] = t2 - t1;
    out[5] = t3 - t2;
    out[6] = t4 - t3;
    out[7] = Vpmg_qfEnergy(pmg, 1);
    out[8] = (p->nonlin) ? Vpmg_dielEnergy(pmg, 1) : 0.0;
    out[9] = (p->nonlin) ? Vpmg_qmEnergy(pmg, 1) : 0.0;
    oracle_shim_set_log(VNULL, 0);

    Vpmg_dtor(&pmg);
    Vpmgp_dtor(&pmgp);
    Vpbe_dtor(&pbe);
    MGparm_dtor(&mg);
    Valist_dtor(&alist);
    return 1;
}

/* Focusing chain of two mg-manual ELEC blocks on one molecule, as main.c
 * runs them (src/main.c:529-620 via initMG/solveMG/setPartMG/energyMG): the
 * coarse block pc is built, filled, solved and its energy taken; the fine
 * block pf (bcfl focus) is constructed with focusFlag=1 and pmgOLD = the
 * coarse Vpmg (routines.c:1458-1469), which fills its faces from the coarse
 * potential, computes the external energies and destroys the coarse Vpmg
 * (vpmg.c:225-262, 396).  Outputs as ref_pmg_run for the fine block, plus
 * out[12..14] = extQf, extDiel, extQm and out[15] = the coarse energy; the
 * residual log and message count cover both solves. */
int ref_pmg_focus(const pmgb_params *pc, const pmgb_params *pf, int natoms,
                  const double *xyz, const double *q, const double *r,
                  double *u, double *faces, double *out, double *reslog,
                  int reslog_cap, int verbose) {
    int i, n, rc;
    double t0, t1, t2, t3, t4;
    double ionc[PMGB_MAXION], ionr[PMGB_MAXION], ionq[PMGB_MAXION];
    double partMin[3], partMax[3];
    Valist *alist;
    MGparm *mgc, *mgf;
    Vpbe *pbec, *pbef;
    Vpmgp *pmgpc, *pmgpf;
    Vpmg *pmgc, *pmgf;

    if (pf->bcfl != PMGB_BCFL_FOCUS || pc->bcfl == PMGB_BCFL_FOCUS) return 0;
    oracle_shim_set_verbose(verbose);
    oracle_shim_set_log(reslog, reslog_cap);
    for (i = 0; i < pc->nion && i < PMGB_MAXION; i++) {
        ionc[i] = pc->ion_conc[i];
        ionr[i] = pc->ion_radius[i];
        ionq[i] = pc->ion_q[i];
    }
    alist = make_alist(natoms, xyz, q, r);

    /* coarse block */
    mgc = make_mgparm(pc);
    pbec = Vpbe_ctor(alist, pc->nion, ionc, ionr, ionq, pc->temp, pc->pdie,
                     pc->sdie, pc->srad, 0, pc->sdens, 0.0, 0.0, 0.0, 0.0);
    if (pbec == VNULL) return 0;
    pmgpc = Vpmgp_ctor(mgc);
    pmgpc->bcfl = (Vbcfl)pc->bcfl;
    pmgpc->xcent = pc->center[0];
    pmgpc->ycent = pc->center[1];
    pmgpc->zcent = pc->center[2];
    pmgc = Vpmg_ctor(pmgpc, pbec, 0, VNULL, mgc, PCE_NO);
    rc = Vpmg_fillco(pmgc, (Vsurf_Meth)pc->srfm, SWIN(pc), (Vchrg_Meth)pc->chgm,
                     0, VNULL, 0, VNULL, 0, VNULL, 0, VNULL, 0, VNULL, 0,
                     VNULL);
    if (rc != 1) return 0;
    if (Vpmg_solve(pmgc) != 1) return 0;
    for (i = 0; i < 3; i++) {
        partMin[i] = mgc->center[i] - 0.5 * mgc->glen[i];
        partMax[i] = mgc->center[i] + 0.5 * mgc->glen[i];
    }
    Vpmg_setPart(pmgc, partMin, partMax, mgc->partDisjOwnSide);
    out[15] = Vpmg_energy(pmgc, 1);

    /* fine block: Vpmg_ctor with focusing destroys the coarse Vpmg */
    t0 = now_s();
    mgf = make_mgparm(pf);
    pbef = Vpbe_ctor(alist, pf->nion, ionc, ionr, ionq, pf->temp, pf->pdie,
                     pf->sdie, pf->srad, 1, pf->sdens, 0.0, 0.0, 0.0, 0.0);
    if (pbef == VNULL) return 0;
    pmgpf = Vpmgp_ctor(mgf);
    pmgpf->bcfl = (Vbcfl)pf->bcfl;
    pmgpf->xcent = pf->center[0];
    pmgpf->ycent = pf->center[1];
    pmgpf->zcent = pf->center[2];
    pmgf = Vpmg_ctor(pmgpf, pbef, 1, pmgc, mgf, PCE_TOTAL);
    out[12] = pmgf->extQfEnergy;
    out[13] = pmgf->extDiEnergy;
    out[14] = pmgf->extQmEnergy;
    Vpmgp_dtor(&pmgpc);
    Vpbe_dtor(&pbec);
    MGparm_dtor(&mgc);
    t1 = now_s();
    rc = Vpmg_fillco(pmgf, (Vsurf_Meth)pf->srfm, SWIN(pf), (Vchrg_Meth)pf->chgm,
                     0, VNULL, 0, VNULL, 0, VNULL, 0, VNULL, 0, VNULL, 0,
                     VNULL);
    t2 = now_s();
    if (rc != 1) return 0;
    n = pf->nx * pf->ny * pf->nz;
    if (faces) {
        size_t fx = (size_t)pf->ny * pf->nz, fy = (size_t)pf->nx * pf->nz,
               fz = (size_t)pf->nx * pf->ny;
        memcpy(faces, pmgf->gxcf, sizeof(double) * 2 * fx);
        memcpy(faces + 2 * fx, pmgf->gycf, sizeof(double) * 2 * fy);
        memcpy(faces + 2 * fx + 2 * fy, pmgf->gzcf, sizeof(double) * 2 * fz);
    }
    rc = Vpmg_solve(pmgf);
    t3 = now_s();
    if (rc != 1) return 0;
    if (u) memcpy(u, pmgf->u, sizeof(double) * n);
    for (i = 0; i < 3; i++) {
        partMin[i] = mgf->center[i] - 0.5 * mgf->glen[i];
        partMax[i] = mgf->center[i] + 0.5 * mgf->glen[i];
    }
    Vpmg_setPart(pmgf, partMin, partMax, mgf->partDisjOwnSide);
    out[0] = Vpmg_energy(pmgf, 1);
    t4 = now_s();
    out[1] = (double)oracle_shim_iter_count();
    out[2] = (double)oracle_shim_log_count();
    out[3] = t1 - t0;
    out[4] = t2 - t1;
    out[5] = t3 - t2;
    out[6] = t4 - t3;
    out[7] = Vpmg_qfEnergy(pmgf, 1);
    out[8] = (pf->nonlin) ? Vpmg_dielEnergy(pmgf, 1) : 0.0;
    out[9] = (pf->nonlin) ? Vpmg_qmEnergy(pmgf, 1) : 0.0;
    oracle_shim_set_log(VNULL, 0);

    Vpmg_dtor(&pmgf);
    Vpmgp_dtor(&pmgpf);
    Vpbe_dtor(&pbef);
    MGparm_dtor(&mgf);
    Valist_dtor(&alist);
    return 1;
}

/* Vgrid_writeDX (src/mg/vgrid.c:1206-1420) on a caller array: the OpenDX
 * file writedataMG writes for a map (routines.c:2620-2800), with pvec the
 * partition weights (NULL: every point).  Returns 1. */
int ref_write_dx(int nx, int ny, int nz, double hx, double hy, double hz, double xmin,
                 double ymin, double zmin, double *data, double *pvec, const char *path,
                 const char *title) {
    char t[256];
    Vgrid *grid = Vgrid_ctor(nx, ny, nz, hx, hy, hz, xmin, ymin, zmin, data);
    if (grid == VNULL) return 0;
    snprintf(t, sizeof(t), "%s", title);
    Vgrid_writeDX(grid, "FILE", "ASC", VNULL, path, t, pvec);
    Vgrid_dtor(&grid);
    return 1;
}

/* An mg-auto chain of nlevel mg-manual blocks on one molecule as main.c
 * runs the calculations NOsh_setupCalcMGAUTO makes of it
 * (src/generic/nosh.c:1828-2101): level 0 with its own boundary condition,
 * every later level focused on the one before (Vpmg_ctor with focusFlag = 1
 * and pmgOLD = the previous Vpmg, which it destroys), each filled, solved,
 * partitioned on its own box and its total energy taken (energyMG with
 * calcenergy total, src/routines.c:1726-1801).  energies[l] = Vpmg_energy of
 * level l in kT; u (optional) = the finest potential.  Returns 1 or 0. */
int ref_pmg_chain(const pmgb_params *levels, int nlevel, int natoms, const double *xyz,
                  const double *q, const double *r, double *energies, double *u) {
    int i, l, rc;
    double ionc[PMGB_MAXION], ionr[PMGB_MAXION], ionq[PMGB_MAXION];
    double partMin[3], partMax[3];
    Valist *alist;
    MGparm *mg = VNULL;
    Vpbe *pbe = VNULL;
    Vpmgp *pmgp = VNULL;
    Vpmg *pmg = VNULL;

    if (nlevel < 1) return 0;
    oracle_shim_set_verbose(0);
    oracle_shim_set_log(VNULL, 0);
    alist = make_alist(natoms, xyz, q, r);
    for (l = 0; l < nlevel; l++) {
        const pmgb_params *p = &levels[l];
        MGparm *mg_l;
        Vpbe *pbe_l;
        Vpmgp *pmgp_l;
        Vpmg *pmg_l;
        if ((l == 0) == (p->bcfl == PMGB_BCFL_FOCUS)) return 0;
        for (i = 0; i < p->nion && i < PMGB_MAXION; i++) {
            ionc[i] = p->ion_conc[i];
            ionr[i] = p->ion_radius[i];
            ionq[i] = p->ion_q[i];
        }
        mg_l = make_mgparm(p);
        pbe_l = Vpbe_ctor(alist, p->nion, ionc, ionr, ionq, p->temp, p->pdie, p->sdie,
                          p->srad, l > 0, p->sdens, 0.0, 0.0, 0.0, 0.0);
        if (pbe_l == VNULL) return 0;
        pmgp_l = Vpmgp_ctor(mg_l);
        if (p->itmax > 0) pmgp_l->itmax = p->itmax;
        pmgp_l->bcfl = (Vbcfl)p->bcfl;
        pmgp_l->xcent = p->center[0];
        pmgp_l->ycent = p->center[1];
        pmgp_l->zcent = p->center[2];
        /* the focused constructor destroys the previous Vpmg */
        pmg_l = Vpmg_ctor(pmgp_l, pbe_l, l > 0, pmg, mg_l, PCE_TOTAL);
        if (pmgp != VNULL) Vpmgp_dtor(&pmgp);
        if (pbe != VNULL) Vpbe_dtor(&pbe);
        if (mg != VNULL) MGparm_dtor(&mg);
        pmg = pmg_l;
        pmgp = pmgp_l;
        pbe = pbe_l;
        mg = mg_l;
        rc = Vpmg_fillco(pmg, (Vsurf_Meth)p->srfm, SWIN(p), (Vchrg_Meth)p->chgm, 0, VNULL, 0,
                         VNULL, 0, VNULL, 0, VNULL, 0, VNULL, 0, VNULL);
        if (rc != 1) return 0;
        if (Vpmg_solve(pmg) != 1) return 0;
        for (i = 0; i < 3; i++) {
            partMin[i] = mg->center[i] - 0.5 * mg->glen[i];
            partMax[i] = mg->center[i] + 0.5 * mg->glen[i];
        }
        Vpmg_setPart(pmg, partMin, partMax, mg->partDisjOwnSide);
        energies[l] = Vpmg_energy(pmg, 1);
    }
    if (u) memcpy(u, pmg->u, sizeof(double) * levels[nlevel - 1].nx * levels[nlevel - 1].ny *
                                 levels[nlevel - 1].nz);
    Vpmg_dtor(&pmg);
    Vpmgp_dtor(&pmgp);
    Vpbe_dtor(&pbe);
    MGparm_dtor(&mg);
    Valist_dtor(&alist);
    return 1;
}
