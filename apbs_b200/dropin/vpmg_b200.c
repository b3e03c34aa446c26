/*
 * vpmg_b200.c -- the Vpmg C API of APBS with Vpmg_solve on a B200.
 *
 * This file is compiled into APBS itself, next to the reference's own
 * src/mg/vpmg.c, and links against libapbs_b200.so (include/apbs_b200.h).
 * It defines three of the Vpmg entry points with their exact signatures
 * (src/mg/vpmg.h:226, 260, 306):
 *
 *   Vpmg_solve  builds a pmgb_params block from the Vpmg's own Vpmgp, Vpbe
 *               and fill settings, hands the host maps that Vpmg_fillco left
 *               in struct sVpmg (charge, epsx/y/z, kappa, gxcf/gycf/gzcf) to
 *               the device solver, solves there, and writes the potential
 *               back into thee->u, so every later Vpmg_* call (energies,
 *               forces, setPart, writedataMG) reads the same host state as
 *               after the reference's Vpmg_solve (vpmg.c:401-558);
 *   Vpmg_ctor   the reference's constructor, after releasing the device side
 *               of pmgOLD when focusing (Vpmg_ctor2 destroys pmgOLD itself,
 *               vpmg.c:396, through an internal call this file cannot see);
 *   Vpmg_dtor   releases the device side, then the reference's destructor.
 *
 * vpmg.c keeps its own definitions of these three under other names: it is
 * compiled with
 *   -DVpmg_solve=Vpmg_solve_host -DVpmg_ctor=Vpmg_ctor_host
 *   -DVpmg_dtor=Vpmg_dtor_host
 * so no line of APBS changes.  Vpmg_solve_host is never called: there is no
 * CPU fallback.  A calculation the device solver does not implement (other
 * solver methods or multigrid settings than the ones APBS's mg-manual and
 * mg-auto blocks use) and any device error make Vpmg_solve return 0 with a
 * message, which is the reference's own failure convention (vpmg.c:416-418).
 *
 * The device calculation of a Vpmg lives in a side table keyed by the Vpmg
 * pointer and is reused while the grid shape stays the same.
 * APBS_B200_PRECISION=mixed in the environment selects the FP32 V-cycles
 * inside FP64 refinement; the default is the FP64 solve that reproduces the
 * reference's potential to round-off.
 */
#include <stdlib.h>
#include <string.h>

#include "apbscfg.h"
#include "maloc/maloc.h"
#include "generic/vhal.h"
#include "generic/vpbe.h"
#include "generic/vacc.h"
#include "mg/vpmgp.h"
#include "mg/vpmg.h"

#include "apbs_b200.h"

/* the reference's definitions, renamed at compile time of vpmg.c */
Vpmg *Vpmg_ctor_host(Vpmgp *parms, Vpbe *pbe, int focusFlag, Vpmg *pmgOLD, MGparm *mgparm,
                     PBEparm_calcEnergy energyFlag);
void Vpmg_dtor_host(Vpmg **thee);

typedef struct B200Entry {
    const Vpmg *key;
    pmgb_solver *solver;
    int precision;
    struct B200Entry *next;
} B200Entry;

static B200Entry *b200_table = VNULL;

static B200Entry *b200_find(const Vpmg *key) {
    B200Entry *e;
    for (e = b200_table; e != VNULL; e = e->next)
        if (e->key == key) return e;
    return VNULL;
}

static void b200_release(const Vpmg *key) {
    B200Entry **pe = &b200_table;
    while (*pe != VNULL) {
        if ((*pe)->key == key) {
            B200Entry *e = *pe;
            *pe = e->next;
            if (e->solver) pmgb_destroy(e->solver);
            free(e);
            return;
        }
        pe = &((*pe)->next);
    }
}

static int b200_precision(void) {
    const char *v = getenv("APBS_B200_PRECISION");
    if (v != VNULL && (strcmp(v, "mixed") == 0 || strcmp(v, "MIXED") == 0)) return PMGB_MIXED;
    return PMGB_FP64;
}

/* The calculation as the device solver describes it: grid and multigrid
 * levels (Vpmgp), physics (Vpbe), fill settings (Vpmg_fillco's arguments
 * kept in the Vpmg).  Returns 0 for settings the device path does not
 * implement. */
static int b200_params(const Vpmg *thee, pmgb_params *p) {
    const Vpmgp *g = thee->pmgp;
    const Vpbe *pbe = thee->pbe;
    int i;

    if (!((g->meth == VSOL_MG && g->nonlin == NONLIN_LPBE) ||
          (g->meth == VSOL_Newton && g->nonlin == NONLIN_NPBE))) {
        Vnm_print(2, "Vpmg_solve (B200): solver method %d with nonlinearity %d is not "
                     "implemented on the device (lpbe and npbe are)\n", g->meth, g->nonlin);
        return 0;
    }
    /* the multigrid settings every mg-manual / mg-auto block gets from
     * Vpmgp_ctor2 (vpmgp.c:127-168) */
    if (g->mgcoar != 2 || g->mgkey != 0 || g->nu1 != 2 || g->nu2 != 2 || g->mgprol != 0 ||
        g->mgdisc != 0 || g->mgsmoo != 1 || g->istop != 1) {
        Vnm_print(2, "Vpmg_solve (B200): multigrid settings other than Vpmgp_ctor2's "
                     "defaults are not implemented on the device\n");
        return 0;
    }
    if (pbe->numIon > PMGB_MAXION) {
        Vnm_print(2, "Vpmg_solve (B200): %d ion species, at most %d\n", pbe->numIon,
                  PMGB_MAXION);
        return 0;
    }
    memset(p, 0, sizeof(*p));
    p->nx = g->nx;
    p->ny = g->ny;
    p->nz = g->nz;
    p->nlev = g->nlev;
    p->hx = g->hx;
    p->hy = g->hy;
    p->hz = g->hzed;
    p->center[0] = g->xcent;
    p->center[1] = g->ycent;
    p->center[2] = g->zcent;
    p->nonlin = (g->nonlin == NONLIN_NPBE) ? 1 : 0;
    p->srfm = (int)thee->surfMeth;
    p->chgm = (int)thee->chargeMeth;
    p->bcfl = (int)g->bcfl;
    p->pdie = pbe->soluteDiel;
    p->sdie = pbe->solventDiel;
    p->srad = pbe->solventRadius;
    p->sdens = (pbe->acc != VNULL) ? pbe->acc->surf_density : 0.0;
    p->temp = pbe->T;
    p->etol = g->errtol;
    p->itmax = g->itmax;
    p->nion = pbe->numIon;
    for (i = 0; i < pbe->numIon; i++) {
        p->ion_q[i] = pbe->ionQ[i];
        p->ion_conc[i] = pbe->ionConc[i];
        p->ion_radius[i] = pbe->ionRadii[i];
    }
    p->swin = thee->splineWin;
    return 1;
}

VPUBLIC Vpmg *Vpmg_ctor(Vpmgp *parms, Vpbe *pbe, int focusFlag, Vpmg *pmgOLD, MGparm *mgparm,
                        PBEparm_calcEnergy energyFlag) {
    /* Vpmg_ctor2 reads pmgOLD's host potential and then destroys it */
    if (focusFlag && pmgOLD != VNULL) b200_release(pmgOLD);
    return Vpmg_ctor_host(parms, pbe, focusFlag, pmgOLD, mgparm, energyFlag);
}

VPUBLIC void Vpmg_dtor(Vpmg **thee) {
    if (thee != VNULL && *thee != VNULL) b200_release(*thee);
    Vpmg_dtor_host(thee);
}

VPUBLIC int Vpmg_solve(Vpmg *thee) {
    pmgb_params p;
    B200Entry *e;
    int i, n, prec;
    double zkappa2;

    if (!(thee->filled)) {
        Vnm_print(2, "Vpmg_solve:  Need to call Vpmg_fillco()!\n");
        return 0;
    }
    if (!b200_params(thee, &p)) return 0;
    n = p.nx * p.ny * p.nz;

    /* the host arrays Vpmg_solve leaves behind (vpmg.c:421-451): some
     * callers read them after the solve */
    zkappa2 = Vpbe_getZkappa2(thee->pbe);
    for (i = 0; i < n; i++) {
        thee->tcf[i] = 0.0;
        thee->fcf[i] = thee->charge[i];
        thee->a1cf[i] = thee->epsx[i];
        thee->a2cf[i] = thee->epsy[i];
        thee->a3cf[i] = thee->epsz[i];
        thee->ccf[i] = (zkappa2 > VPMGSMALL) ? zkappa2 * thee->kappa[i] : 0.0;
    }

    prec = b200_precision();
    e = b200_find(thee);
    if (e != VNULL && e->precision == prec) {
        /* keep the device arrays when the grid is the same (a refused
         * reconfiguration means another grid: build anew) */
        if (!pmgb_reconfigure(e->solver, &p)) {
            b200_release(thee);
            e = VNULL;
        }
    } else if (e != VNULL) {
        b200_release(thee);
        e = VNULL;
    }
    if (e == VNULL) {
        e = (B200Entry *)calloc(1, sizeof(B200Entry));
        if (e == VNULL) {
            Vnm_print(2, "Vpmg_solve (B200): out of host memory\n");
            return 0;
        }
        if (!pmgb_create(&p, prec, &e->solver)) {
            Vnm_print(2, "Vpmg_solve (B200): %s\n", pmgb_last_error());
            free(e);
            return 0;
        }
        e->key = thee;
        e->precision = prec;
        e->next = b200_table;
        b200_table = e;
    }
    /* faces: slots 0 and 1 (low, high) lead each of gxcf/gycf/gzcf
     * (IJKx/IJKy/IJKz, vpmg.h:1384-1386) */
    if (!pmgb_set_coefficients(e->solver, thee->charge, thee->epsx, thee->epsy, thee->epsz,
                               thee->kappa, thee->gxcf, thee->gycf, thee->gzcf) ||
        !pmgb_solve(e->solver) || !pmgb_get_potential(e->solver, thee->u)) {
        Vnm_print(2, "Vpmg_solve (B200): %s\n", pmgb_last_error());
        b200_release(thee);
        return 0;
    }
    return 1;
}
