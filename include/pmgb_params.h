/*
 * pmgb_params.h -- plain-C description of one PMG calculation.
 *
 * One struct of scalars that carries what APBS spreads over MGparm,
 * PBEparm, Vpmgp and Vpbe for a single mg-manual ELEC block:
 *   dime/grid/gcent/nlev  (src/generic/mgparm.h:114-203, keyword parser
 *                          src/generic/mgparm.c:916-969)
 *   lpbe|npbe, bcfl, pdie, sdie, srfm, srad, sdens, swin, temp, ion, chgm
 *                         (src/generic/pbeparm.c:1215-1285)
 * It is shared by the CUDA library's C ABI (apbs_b200.h) and by the CPU
 * oracle, so both sides of every parity test are driven by identical input.
 */
#ifndef PMGB_PARAMS_H
#define PMGB_PARAMS_H

#define PMGB_MAXION 8

/* Surface method codes (values of Vsurf_Meth, src/generic/vhal.h:103-107). */
#define PMGB_SRFM_MOL 0
#define PMGB_SRFM_SMOL 1
#define PMGB_SRFM_SPL2 2   /* cubic-spline surface (fillcoCoefSpline) */
#define PMGB_SRFM_SPL3 3   /* 5th-order polynomial surface (fillcoCoefSpline3) */
#define PMGB_SRFM_SPL4 4   /* 7th-order polynomial surface (fillcoCoefSpline4) */
/* Charge method codes (Vchrg_Meth, src/generic/vhal.h:231-234). */
#define PMGB_CHGM_TRIL 0   /* chgm spl0: trilinear to the 8 nearest points */
#define PMGB_CHGM_SPL2 1
#define PMGB_CHGM_SPL4 2   /* chgm spl4: 5th-order B-spline to 6^3 points
                              (fillcoPermanentMultipole with atomic charges) */
/* Boundary condition codes (Vbcfl, src/generic/vhal.h:208-216). */
#define PMGB_BCFL_ZERO 0
#define PMGB_BCFL_SDH 1
#define PMGB_BCFL_MDH 2
#define PMGB_BCFL_FOCUS 4
#define PMGB_BCFL_MAP 6     /* faces from a potential map (pmgb_set_map PMGB_MAP_POT) */

typedef struct pmgb_params {
    int nx, ny, nz;         /* grid points per axis ("dime") */
    int nlev;               /* multigrid levels (MGparm_check rule if <= 0) */
    double hx, hy, hz;      /* grid spacing in Angstrom ("grid") */
    double center[3];       /* grid centre in Angstrom ("gcent") */
    int nonlin;             /* 0 = lpbe, 1 = npbe */
    int srfm;               /* PMGB_SRFM_* */
    int chgm;               /* PMGB_CHGM_TRIL (spl0), _SPL2 or _SPL4 */
    int bcfl;               /* PMGB_BCFL_* */
    double pdie;            /* solute dielectric */
    double sdie;            /* solvent dielectric */
    double srad;            /* solvent probe radius (Angstrom) */
    double sdens;           /* SAS sphere point density (1/Angstrom^2) */
    double temp;            /* temperature (K) */
    double etol;            /* relative residual tolerance; <= 0 -> 1e-6 */
    int nion;               /* mobile ion species */
    double ion_q[PMGB_MAXION];      /* valence (e) */
    double ion_conc[PMGB_MAXION];   /* bulk concentration (M) */
    double ion_radius[PMGB_MAXION]; /* radius (Angstrom) */
    double swin;            /* spline window of srfm spl2 and of the boundary
                               forces ("swin"); <= 0 -> 0.3 */
    int itmax;              /* iteration limit of the solve (Vpmgp itmax: V-cycles of
                               the LPBE solve, Newton steps of the NPBE solve);
                               <= 0 -> 200, the reference's default (vpmgp.c:131) */
} pmgb_params;

#endif /* PMGB_PARAMS_H */
