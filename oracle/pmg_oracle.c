/*
 * pmg_oracle.c -- CPU restatement of the APBS finite-difference PMG solve
 * path (Vpmg_fillco + Vpmg_solve + Vpmg_energy for one mg-manual block).
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA library is compared
 * against, and it is itself pinned against the reference sources compiled
 * unchanged in oracle/_ref (tests/test_oracle_pin.py).  Every routine names
 * the reference lines whose arithmetic it restates.  Where bitwise agreement
 * with the reference matters (integer index logic, comparisons deciding
 * which grid points are marked) the expression trees are the reference's;
 * floating-point sums are evaluated in the reference's order so that the
 * restatement agrees to the last few ulps.
 *
 * Indexing is 0-based; IJK(i,j,k) = (k*ny + j)*nx + i (src/mg/vpmg.h:1383).
 * Interior points are 1..n-2 on every axis.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "pmg_oracle.h"

#define VSMALL 1.0e-9
#define VPMGSMALL 1.0e-12
#define MAX_SPLINE_WINDOW 0.5
#define EXPCLAMP 85.0
#define ZSMALL 1.0e-20
#define ZLARGE 1.0e20

typedef struct {
    int nx, ny, nz;
    size_t n;
    int nop;            /* 4 (7-point) or 14 (27-point) stored coefficients */
    double *op[14];     /* oC oE oN uC oNE oNW uE uW uN uS uNE uNW uSE uSW */
    double *cc, *fc;    /* Helmholtz diagonal and right-hand side */
    double *x, *w0;     /* iterate and restricted residual */
    double *cp, *rhs;   /* Newton: c'(u) and Newton rhs, all levels */
    double *xt;         /* Newton: correction iterate, all levels */
} Level;

typedef struct {
    int nlev;
    Level lev[12];
    double *w1, *w2, *w3;          /* fine-sized scratch */
    double *band;                  /* factored coarsest band matrix */
    int bn, bm, blda;
    int mgsolv;                    /* 1 band Cholesky, 0 CG */
    double *reslog;
    int reslog_cap, reslog_n, progress;
    int total_cycles;
} Solver;

#define IJK(i, j, k) (((size_t)(k) * ny + (j)) * nx + (i))

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void logres(Solver *s, double relres) {
    if (s->reslog && s->reslog_n < s->reslog_cap) s->reslog[s->reslog_n] = relres;
    s->reslog_n++;
    s->progress++;
}

/* ===================================================================== */
/* Physical constants (src/generic/vpbe.c:264-411, src/generic/vunit.h)   */
/* ===================================================================== */
typedef struct {
    double zmagic, xkappa, zkappa2, ionstr, maxIonRadius;
    double soluteCenter[3], soluteRadius;
    double sconc[PMGB_MAXION];     /* ionConc * 0.5/I (vpmg.c:340-377) */
} Phys;

static void phys_setup(const pmgb_params *p, int natoms, const double *xyz,
                       const double *r, Phys *ph) {
    const double N_A = 6.022045000e+23, e_c = 4.803242384e-10,
                 k_B = 1.380662000e-16;
    const double pi = 4. * atan(1.);
    double mn[3], mx[3], radius = 0.0;
    int i, a;
    /* Valist_getStatistics (src/generic/valist.c): bounding-box centre */
    for (i = 0; i < 3; i++) mn[i] = mx[i] = xyz[i];
    for (a = 0; a < natoms; a++)
        for (i = 0; i < 3; i++) {
            double v = xyz[3 * a + i];
            if (v < mn[i]) mn[i] = v;
            if (v > mx[i]) mx[i] = v;
        }
    for (i = 0; i < 3; i++) ph->soluteCenter[i] = 0.5 * (mx[i] + mn[i]);
    /* solute radius (vpbe.c:312-338) */
    for (a = 0; a < natoms; a++) {
        double d0 = xyz[3 * a] - ph->soluteCenter[0];
        double d1 = xyz[3 * a + 1] - ph->soluteCenter[1];
        double d2 = xyz[3 * a + 2] - ph->soluteCenter[2];
        double dist = (d0 * d0) + (d1 * d1) + (d2 * d2);
        dist = sqrt(dist) + r[a];
        if (dist > radius) radius = dist;
    }
    ph->soluteRadius = radius;
    ph->ionstr = 0.0;
    ph->maxIonRadius = 0.0;
    for (i = 0; i < p->nion; i++) {
        if (p->ion_radius[i] > ph->maxIonRadius) ph->maxIonRadius = p->ion_radius[i];
        ph->ionstr += (0.5 * p->ion_conc[i] * (p->ion_q[i] * p->ion_q[i]));
    }
    if (ph->ionstr == 0.) {
        ph->xkappa = 0.;
        ph->zkappa2 = 0.;
    } else {
        ph->xkappa = sqrt(ph->ionstr * 1.0e-16 *
                          ((8.0 * pi * N_A * e_c * e_c) /
                           (1000.0 * p->sdie * k_B * p->temp)));
        ph->zkappa2 = p->sdie * (ph->xkappa * ph->xkappa);
    }
    ph->zmagic = ((4.0 * pi * e_c * e_c) / (k_B * p->temp)) * 1.0e+8;
    for (i = 0; i < p->nion; i++) {
        double zks2 = (ph->ionstr > 0.0) ? 0.5 / ph->ionstr : 0.0;
        ph->sconc[i] = zks2 * p->ion_conc[i];
    }
}

/* ===================================================================== */
/* Coefficient fill (src/mg/vpmg.c:5250-5414)                             */
/* ===================================================================== */

/* bspline2, vpmg.c:5091-5105 */
static double bspline2(double x) {
    double m2m, m2, m3;
    if ((x >= 0.0) && (x <= 2.0)) m2m = 1.0 - fabs(x - 1.0);
    else m2m = 0.0;
    if ((x >= 1.0) && (x <= 3.0)) m2 = 1.0 - fabs(x - 2.0);
    else m2 = 0.0;
    if ((x >= 0.0) && (x <= 3.0)) m3 = 0.5 * x * m2m + 0.5 * (3.0 - x) * m2;
    else m3 = 0.0;
    return m3;
}

/* fillcoChargeSpline2, vpmg.c:5123-5248 */
static void fill_charge_spl2(const pmgb_params *p, const Phys *ph, int natoms,
                             const double *xyz, const double *q,
                             const double *xmn, const double *xmx,
                             double *charge) {
    int nx = p->nx, ny = p->ny, nz = p->nz, a;
    double hx = p->hx, hy = p->hy, hz = p->hz;
    memset(charge, 0, sizeof(double) * (size_t)nx * ny * nz);
    for (a = 0; a < natoms; a++) {
        const double *ap = xyz + 3 * a;
        if ((ap[0] <= (xmn[0] - hx)) || (ap[0] >= (xmx[0] + hx)) ||
            (ap[1] <= (xmn[1] - hy)) || (ap[1] >= (xmx[1] + hy)) ||
            (ap[2] <= (xmn[2] - hz)) || (ap[2] >= (xmx[2] + hz)))
            continue;
        double px = ap[0] - xmn[0], py = ap[1] - xmn[1], pz = ap[2] - xmn[2];
        double c = q[a] * ph->zmagic / (hx * hy * hz);
        double fi = px / hx, fj = py / hy, fk = pz / hz;
        int ip1 = (int)ceil(fi), im1 = (int)floor(fi);
        int jp1 = (int)ceil(fj), jm1 = (int)floor(fj);
        int kp1 = (int)ceil(fk), km1 = (int)floor(fk);
        int ip2 = ip1 + 1, im2 = im1 - 1, jp2 = jp1 + 1, jm2 = jm1 - 1;
        int kp2 = kp1 + 1, km2 = km1 - 1;
        int ii, jj, kk;
        if (ip2 > nx - 1) ip2 = nx - 1;
        if (ip1 > nx - 1) ip1 = nx - 1;
        if (im1 < 0) im1 = 0;
        if (im2 < 0) im2 = 0;
        if (jp2 > ny - 1) jp2 = ny - 1;
        if (jp1 > ny - 1) jp1 = ny - 1;
        if (jm1 < 0) jm1 = 0;
        if (jm2 < 0) jm2 = 0;
        if (kp2 > nz - 1) kp2 = nz - 1;
        if (kp1 > nz - 1) kp1 = nz - 1;
        if (km1 < 0) km1 = 0;
        if (km2 < 0) km2 = 0;
        (void)jp1; (void)kp1; (void)ip1; (void)jm1; (void)km1;
        for (ii = im2; ii <= ip2; ii++) {
            double mx_ = bspline2(1.5 + ((double)ii - fi));
            for (jj = jm2; jj <= jp2; jj++) {
                double my_ = bspline2(1.5 + ((double)jj - fj));
                for (kk = km2; kk <= kp2; kk++) {
                    double mz_ = bspline2(1.5 + ((double)kk - fk));
                    charge[IJK(ii, jj, kk)] += (c * mx_ * my_ * mz_);
                }
            }
        }
    }
}

/* fillcoChargeSpline1 (chgm spl0), vpmg.c:4986-5089 */
static void fill_charge_tril(const pmgb_params *p, const Phys *ph, int natoms,
                             const double *xyz, const double *q,
                             const double *xmn, const double *xmx,
                             double *charge) {
    int nx = p->nx, ny = p->ny, nz = p->nz, a;
    double hx = p->hx, hy = p->hy, hz = p->hz;
    memset(charge, 0, sizeof(double) * (size_t)nx * ny * nz);
    for (a = 0; a < natoms; a++) {
        const double *ap = xyz + 3 * a;
        double px, py, pz, c, fi, fj, fk, dx, dy, dz;
        int ihi, ilo, jhi, jlo, khi, klo;
        if ((ap[0] <= xmn[0]) || (ap[0] >= xmx[0]) || (ap[1] <= xmn[1]) ||
            (ap[1] >= xmx[1]) || (ap[2] <= xmn[2]) || (ap[2] >= xmx[2]))
            continue;
        px = ap[0] - xmn[0];
        py = ap[1] - xmn[1];
        pz = ap[2] - xmn[2];
        c = q[a] * ph->zmagic / (hx * hy * hz);
        fi = px / hx;
        fj = py / hy;
        fk = pz / hz;
        ihi = (int)ceil(fi);
        ilo = (int)floor(fi);
        jhi = (int)ceil(fj);
        jlo = (int)floor(fj);
        khi = (int)ceil(fk);
        klo = (int)floor(fk);
        dx = fi - (double)ilo;
        dy = fj - (double)jlo;
        dz = fk - (double)klo;
        charge[IJK(ihi, jhi, khi)] += (dx * dy * dz * c);
        charge[IJK(ihi, jlo, khi)] += (dx * (1.0 - dy) * dz * c);
        charge[IJK(ihi, jhi, klo)] += (dx * dy * (1.0 - dz) * c);
        charge[IJK(ihi, jlo, klo)] += (dx * (1.0 - dy) * (1.0 - dz) * c);
        charge[IJK(ilo, jhi, khi)] += ((1.0 - dx) * dy * dz * c);
        charge[IJK(ilo, jlo, khi)] += ((1.0 - dx) * (1.0 - dy) * dz * c);
        charge[IJK(ilo, jhi, klo)] += ((1.0 - dx) * dy * (1.0 - dz) * c);
        charge[IJK(ilo, jlo, klo)] += ((1.0 - dx) * (1.0 - dy) * (1.0 - dz) * c);
    }
}

/* markSphere, vpmg.c:6444-6491 */
static void mark_sphere(double rtot, const double *tpos, int nx, int ny, int nz,
                        double hx, double hy, double hz, double xmin,
                        double ymin, double zmin, double *array,
                        double markVal) {
    int i, j, k, imin, imax, jmin, jmax, kmin, kmax;
    double fi, fj, fk, dx2, dy2, dz2;
    double posx = tpos[0] - xmin, posy = tpos[1] - ymin, posz = tpos[2] - zmin;
    double rtot2 = rtot * rtot;
    double xr = rtot + 0.5 * hx, yr = rtot + 0.5 * hy, zr = rtot + 0.5 * hz;
    imin = (int)ceil((posx - xr) / hx); if (imin < 0) imin = 0;
    jmin = (int)ceil((posy - yr) / hy); if (jmin < 0) jmin = 0;
    kmin = (int)ceil((posz - zr) / hz); if (kmin < 0) kmin = 0;
    imax = (int)floor((posx + xr) / hx); if (imax > nx - 1) imax = nx - 1;
    jmax = (int)floor((posy + yr) / hy); if (jmax > ny - 1) jmax = ny - 1;
    kmax = (int)floor((posz + zr) / hz); if (kmax > nz - 1) kmax = nz - 1;
    for (i = imin, fi = imin; i <= imax; i++, fi += 1.) {
        dx2 = (posx - hx * fi) * (posx - hx * fi);
        for (j = jmin, fj = jmin; j <= jmax; j++, fj += 1.) {
            dy2 = (posy - hy * fj) * (posy - hy * fj);
            if ((dx2 + dy2) > rtot2) continue;
            for (k = kmin, fk = kmin; k <= kmax; k++, fk += 1.) {
                dz2 = (posz - hz * fk) * (posz - hz * fk);
                if ((dz2 + dy2 + dx2) <= rtot2) array[IJK(i, j, k)] = markVal;
            }
        }
    }
}

/* Reference sphere points, VaccSurf_refSphere (src/generic/vacc.c:924-978).
 * Returns the point count; xyz[3*count] allocated by the caller (upper bound
 * 4*npts + 16). */
static int ref_sphere(int npts, double *pts) {
    double frac = ((double)npts) / 4.0;
    const double pi = 3.14159265358979323846;
    int ntheta = (int)floor(sqrt(pi * frac) + 0.5);
    double dtheta = pi / ((double)ntheta);
    int nphimax = 2 * ntheta, it, ip, n = 0;
    for (it = 0; it < ntheta; it++) {
        double theta = dtheta * ((double)it);
        double st = sin(theta), ct = cos(theta);
        int nphi = (int)floor(st * nphimax + 0.5);
        if (nphi != 0) {
            double dphi = 2 * pi / ((double)nphi);
            for (ip = 0; ip < nphi; ip++) {
                double phi = dphi * ((double)ip);
                pts[3 * n + 0] = cos(phi) * st;
                pts[3 * n + 1] = sin(phi) * st;
                pts[3 * n + 2] = ct;
                n++;
            }
        }
    }
    return n;
}

static int ref_sphere_count(int npts) {
    double frac = ((double)npts) / 4.0;
    const double pi = 3.14159265358979323846;
    int ntheta = (int)floor(sqrt(pi * frac) + 0.5), it, n = 0;
    double dtheta = pi / ((double)ntheta);
    for (it = 0; it < ntheta; it++) {
        double st = sin(dtheta * ((double)it));
        n += (int)floor(st * (2 * ntheta) + 0.5);
    }
    return n;
}

/* fillcoCoefMolDielNoSmooth (vpmg.c:4346-4498) with the SAS point sets of
 * Vacc_atomSurf (vacc.c:866-922) and the exclusion test ivdwAccExclus
 * (vacc.c:78-128).  The exclusion test here scans every atom: the reference
 * scans the atoms of the point's Vclist cell, which holds every atom whose
 * inflated sphere can reach the point (vclist.c:231-342), so both decide
 * the same. */
static void fill_diel(const pmgb_params *p, const Phys *ph, int natoms,
                      const double *xyz, const double *r, const double *xmn,
                      const double *xmx, double *epsx, double *epsy,
                      double *epsz) {
    int nx = p->nx, ny = p->ny, nz = p->nz, a, b, t;
    double hx = p->hx, hy = p->hy, hz = p->hz;
    double srad = p->srad, epsw = p->sdie, epsp = p->pdie;
    size_t n = (size_t)nx * ny * nz, i;
    for (i = 0; i < n; i++) { epsx[i] = epsw; epsy[i] = epsw; epsz[i] = epsw; }
    for (a = 0; a < natoms; a++) {
        const double *ap = xyz + 3 * a;
        double arad = r[a];
        if ((ap[0] <= xmn[0]) || (ap[0] >= xmx[0]) || (ap[1] <= xmn[1]) ||
            (ap[1] >= xmx[1]) || (ap[2] <= xmn[2]) || (ap[2] >= xmx[2]))
            continue;
        if (arad > VSMALL) {
            mark_sphere(arad + srad, ap, nx, ny, nz, hx, hy, hz,
                        (xmn[0] + 0.5 * hx), xmn[1], xmn[2], epsx, epsp);
            mark_sphere(arad + srad, ap, nx, ny, nz, hx, hy, hz, xmn[0],
                        (xmn[1] + 0.5 * hy), xmn[2], epsy, epsp);
            mark_sphere(arad + srad, ap, nx, ny, nz, hx, hy, hz, xmn[0],
                        xmn[1], (xmn[2] + 0.5 * hz), epsz, epsp);
        }
    }
    if (!(srad > VSMALL)) return;
    {
        /* Vacc_storeParms (vacc.c:146-189) with the Vclist probe radius of
         * Vpbe_ctor2 (vpbe.c:419-421) */
        double clist_rad = (ph->maxIonRadius > srad ? ph->maxIonRadius : srad) +
                           MAX_SPLINE_WINDOW;
        double maxrad = 0.0, maxarea;
        int nsphere, nref;
        double *ref;
        for (a = 0; a < natoms; a++) if (r[a] > maxrad) maxrad = r[a];
        maxrad = maxrad + clist_rad;
        maxarea = 4.0 * 3.14159265358979323846 * maxrad * maxrad;
        nsphere = (int)ceil(maxarea * p->sdens);
        nref = ref_sphere_count(nsphere);
        ref = (double *)malloc(sizeof(double) * 3 * (size_t)(nref + 1));
        nref = ref_sphere(nsphere, ref);
        for (a = 0; a < natoms; a++) {
            double arad = r[a];
            const double *ap = xyz + 3 * a;
            double rad;
            if (arad < VSMALL) continue;
            rad = arad + srad;
            for (t = 0; t < nref; t++) {
                double pos[3];
                int acc = 1;
                pos[0] = rad * (ref[3 * t + 0]) + ap[0];
                pos[1] = rad * (ref[3 * t + 1]) + ap[1];
                pos[2] = rad * (ref[3 * t + 2]) + ap[2];
                for (b = 0; b < natoms; b++) {
                    double d0, d1, d2, dist2, rr;
                    if (b == a) continue;
                    d0 = pos[0] - xyz[3 * b];
                    d1 = pos[1] - xyz[3 * b + 1];
                    d2 = pos[2] - xyz[3 * b + 2];
                    dist2 = d0 * d0 + d1 * d1 + d2 * d2;
                    rr = r[b] + srad;
                    if (dist2 < rr * rr) { acc = 0; break; }
                }
                if (!acc) continue;
                mark_sphere(srad, pos, nx, ny, nz, hx, hy, hz,
                            (xmn[0] + 0.5 * hx), xmn[1], xmn[2], epsx, epsw);
                mark_sphere(srad, pos, nx, ny, nz, hx, hy, hz, xmn[0],
                            (xmn[1] + 0.5 * hy), xmn[2], epsy, epsw);
                mark_sphere(srad, pos, nx, ny, nz, hx, hy, hz, xmn[0], xmn[1],
                            (xmn[2] + 0.5 * hz), epsz, epsw);
            }
        }
        free(ref);
    }
}

/* fillcoCoefMolDielSmooth, vpmg.c:4500-4628 */
static void smooth_diel(const pmgb_params *p, double *epsx, double *epsy,
                        double *epsz) {
    int nx = p->nx, ny = p->ny, nz = p->nz, i, j, k, np;
    size_t n = (size_t)nx * ny * nz;
    double *a1 = (double *)malloc(sizeof(double) * n * 3), *a2 = a1 + n,
           *a3 = a2 + n, frac;
    memcpy(a1, epsx, sizeof(double) * n);
    memcpy(a2, epsy, sizeof(double) * n);
    memcpy(a3, epsz, sizeof(double) * n);
    for (i = 0; i < nx; i++)
        for (j = 0; j < ny; j++)
            for (k = 0; k < nz; k++) {
                frac = 1.0 / a1[IJK(i, j, k)];
                frac += 1.0 / a2[IJK(i, j, k)];
                frac += 1.0 / a3[IJK(i, j, k)];
                np = 3;
                if (j > 0) { frac += 1.0 / a2[IJK(i, j - 1, k)]; np += 1; }
                if (k > 0) { frac += 1.0 / a3[IJK(i, j, k - 1)]; np += 1; }
                if (i < (nx - 1)) {
                    frac += 1.0 / a2[IJK(i + 1, j, k)];
                    frac += 1.0 / a3[IJK(i + 1, j, k)];
                    np += 2;
                    if (j > 0) { frac += 1.0 / a2[IJK(i + 1, j - 1, k)]; np += 1; }
                    if (k > 0) { frac += 1.0 / a3[IJK(i + 1, j, k - 1)]; np += 1; }
                }
                epsx[IJK(i, j, k)] = np / frac;

                frac = 1.0 / a2[IJK(i, j, k)];
                frac += 1.0 / a1[IJK(i, j, k)];
                frac += 1.0 / a3[IJK(i, j, k)];
                np = 3;
                if (i > 0) { frac += 1.0 / a1[IJK(i - 1, j, k)]; np += 1; }
                if (k > 0) { frac += 1.0 / a3[IJK(i, j, k - 1)]; np += 1; }
                if (j < (ny - 1)) {
                    frac += 1.0 / a1[IJK(i, j + 1, k)];
                    frac += 1.0 / a3[IJK(i, j + 1, k)];
                    np += 2;
                    if (i > 0) { frac += 1.0 / a1[IJK(i - 1, j + 1, k)]; np += 1; }
                    if (k > 0) { frac += 1.0 / a3[IJK(i, j + 1, k - 1)]; np += 1; }
                }
                epsy[IJK(i, j, k)] = np / frac;

                frac = 1.0 / a3[IJK(i, j, k)];
                frac += 1.0 / a1[IJK(i, j, k)];
                frac += 1.0 / a2[IJK(i, j, k)];
                np = 3;
                if (i > 0) { frac += 1.0 / a1[IJK(i - 1, j, k)]; np += 1; }
                if (j > 0) { frac += 1.0 / a2[IJK(i, j - 1, k)]; np += 1; }
                if (k < (nz - 1)) {
                    frac += 1.0 / a1[IJK(i, j, k + 1)];
                    frac += 1.0 / a2[IJK(i, j, k + 1)];
                    np += 2;
                    if (i > 0) { frac += 1.0 / a1[IJK(i - 1, j, k + 1)]; np += 1; }
                    if (j > 0) { frac += 1.0 / a2[IJK(i, j - 1, k + 1)]; np += 1; }
                }
                epsz[IJK(i, j, k)] = np / frac;
            }
    free(a1);
}

/* fillcoCoefMolIon, vpmg.c:4237-4333 */
static void fill_kappa(const pmgb_params *p, const Phys *ph, int natoms,
                       const double *xyz, const double *r, const double *xmn,
                       const double *xmx, double *kappa) {
    int nx = p->nx, ny = p->ny, nz = p->nz, a;
    size_t n = (size_t)nx * ny * nz, i;
    double irad = ph->maxIonRadius;
    double ionmask = (ph->ionstr > VPMGSMALL) ? 1.0 : 0.0;
    for (i = 0; i < n; i++) kappa[i] = ionmask;
    if (ph->ionstr < VPMGSMALL) return;
    for (a = 0; a < natoms; a++) {
        const double *ap = xyz + 3 * a;
        double arad = r[a];
        if (!(arad > VSMALL)) continue;
        if ((ap[0] < (xmn[0] - irad - arad)) || (ap[0] > (xmx[0] + irad + arad)) ||
            (ap[1] < (xmn[1] - irad - arad)) || (ap[1] > (xmx[1] + irad + arad)) ||
            (ap[2] < (xmn[2] - irad - arad)) || (ap[2] > (xmx[2] + irad + arad)))
            continue;
        mark_sphere((irad + arad), ap, nx, ny, nz, p->hx, p->hy, p->hz, xmn[0],
                    xmn[1], xmn[2], kappa, 0.0);
    }
}

/* multipolebc, vpmg.c:3369-3477 */
static void multipolebc(double r, double kappa, double eps_p, double eps_w,
                        double rad, double tsr[3]) {
    double r2, r3, r5, eps_r, ka, ka2, ka3, kr, kr2;
    eps_r = eps_w / eps_p;
    r2 = r * r;
    r3 = r2 * r;
    r5 = r3 * r2;
    tsr[0] = (1.0 / eps_w) / r;
    tsr[1] = (1.0 / eps_w) * (-1.0) / r3;
    tsr[2] = (1.0 / eps_w) * (3.0) / r5;
    if (kappa < VSMALL) {
        tsr[1] = (3.0 * eps_r) / (1.0 + 2.0 * eps_r) * tsr[1];
        tsr[2] = (5.0 * eps_r) / (2.0 + 3.0 * eps_r) * tsr[2];
    } else {
        ka = kappa * rad;
        ka2 = ka * ka;
        ka3 = ka2 * ka;
        kr = kappa * r;
        kr2 = kr * kr;
        tsr[0] = exp(ka - kr) / (1.0 + ka) * tsr[0];
        tsr[1] = 3.0 * eps_r * exp(ka - kr) * (1.0 + kr) * tsr[1];
        tsr[1] = tsr[1] / (1.0 + ka + eps_r * (2.0 + 2.0 * ka + ka2));
        tsr[2] = 5.0 * eps_r * exp(ka - kr) * (3.0 + 3.0 * kr + kr2) * tsr[2];
        tsr[2] = tsr[2] / (6.0 + 6.0 * ka + 2.0 * ka2 +
                           eps_r * (9.0 + 9.0 * ka + 4.0 * ka2 + ka3));
    }
}

/* bcfl_sdh, vpmg.c:3479-3645.  Faces: gx[2][nz][ny], gy[2][nz][nx],
 * gz[2][ny][nx] (IJKx/IJKy/IJKz, vpmg.h:1384-1386). */
static void bc_sdh(const pmgb_params *p, const Phys *ph, int natoms,
                   const double *xyz, const double *q, const double *xf,
                   const double *yf, const double *zf, double *gx, double *gy,
                   double *gz) {
    int nx = p->nx, ny = p->ny, nz = p->nz, i, j, k, a;
    const double pi = 3.14159265358979323846;
    double eps_w = p->sdie, eps_p = p->pdie;
    double pre = (1.6021773e-19 * 1.6021773e-19) /
                 (4 * pi * 8.8541878e-12 * 1.3806581e-23 * p->temp);
    double sq = 0.0, dip[3] = {0, 0, 0}, quad[9] = {0}, tr[9];
    double ux, uy, uz, qxx, qxy, qxz, qyy, qyz, qzz;
    const double *pos = ph->soluteCenter;
    pre = pre * (1.0e10);
    for (a = 0; a < natoms; a++) {
        double xr = xyz[3 * a] - pos[0], yr = xyz[3 * a + 1] - pos[1],
               zr = xyz[3 * a + 2] - pos[2], c = q[a], qave;
        sq += c;
        dip[0] += xr * c;
        dip[1] += yr * c;
        dip[2] += zr * c;
        tr[0] = xr * xr * c; tr[1] = xr * yr * c; tr[2] = xr * zr * c;
        tr[3] = yr * xr * c; tr[4] = yr * yr * c; tr[5] = yr * zr * c;
        tr[6] = zr * xr * c; tr[7] = zr * yr * c; tr[8] = zr * zr * c;
        qave = (tr[0] + tr[4] + tr[8]) / 3.0;
        quad[0] += 1.5 * (tr[0] - qave);
        quad[1] += 1.5 * (tr[1]);
        quad[2] += 1.5 * (tr[2]);
        quad[3] += 1.5 * (tr[3]);
        quad[4] += 1.5 * (tr[4] - qave);
        quad[5] += 1.5 * (tr[5]);
        quad[6] += 1.5 * (tr[6]);
        quad[7] += 1.5 * (tr[7]);
        quad[8] += 1.5 * (tr[8] - qave);
    }
    ux = dip[0]; uy = dip[1]; uz = dip[2];
    qxx = quad[0] / 3.0; qxy = quad[1] / 3.0; qxz = quad[2] / 3.0;
    qyy = quad[4] / 3.0; qyz = quad[5] / 3.0; qzz = quad[8] / 3.0;
    memset(gx, 0, sizeof(double) * 2 * ny * nz);
    memset(gy, 0, sizeof(double) * 2 * nx * nz);
    memset(gz, 0, sizeof(double) * 2 * nx * ny);
    for (k = 0; k < nz; k++)
        for (j = 0; j < ny; j++)
            for (i = 0; i < nx; i++) {
                double xr, yr, zr, dist, t[3], val;
                if (!((k == 0) || (k == nz - 1) || (j == 0) || (j == ny - 1) ||
                      (i == 0) || (i == nx - 1)))
                    continue;
                xr = xf[i] - pos[0];
                yr = yf[j] - pos[1];
                zr = zf[k] - pos[2];
                dist = sqrt((xr * xr) + (yr * yr) + (zr * zr));
                multipolebc(dist, ph->xkappa, eps_p, eps_w, ph->soluteRadius, t);
                val = pre * sq * t[0];
                val -= pre * ux * xr * t[1];
                val -= pre * uy * yr * t[1];
                val -= pre * uz * zr * t[1];
                val += pre * qxx * xr * xr * t[2];
                val += pre * qyy * yr * yr * t[2];
                val += pre * qzz * zr * zr * t[2];
                val += pre * 2.0 * qxy * xr * yr * t[2];
                val += pre * 2.0 * qxz * xr * zr * t[2];
                val += pre * 2.0 * qyz * yr * zr * t[2];
                if (i == 0) gx[((size_t)0 * nz + k) * ny + j] = val;
                if (i == nx - 1) gx[((size_t)1 * nz + k) * ny + j] = val;
                if (j == 0) gy[((size_t)0 * nz + k) * nx + i] = val;
                if (j == ny - 1) gy[((size_t)1 * nz + k) * nx + i] = val;
                if (k == 0) gz[((size_t)0 * ny + j) * nx + i] = val;
                if (k == nz - 1) gz[((size_t)1 * ny + j) * nx + i] = val;
            }
}

typedef struct {
    double *charge, *epsx, *epsy, *epsz, *kappa;
    double *gx, *gy, *gz;
    double *xf, *yf, *zf;
    double xmn[3], xmx[3];
} Fill;

/* bcflnew (bcfl mdh), vpmg.c:3289-3367 with packAtoms/packUnpack
 * (3195-3287): every boundary point gets the sum over all atoms, in atom
 * order, of the Debye-Hueckel potential of each charge; a point on several
 * faces gets the same value on each. */
static double mdh_value(const Phys *ph, double pre1, int natoms, const double *xyz,
                        const double *q, const double *r, double gx, double gy,
                        double gz) {
    const double ec = 1.6021773e-19;
    double val = 0.0;
    int a;
    for (a = 0; a < natoms; a++) {
        double dx = gx - xyz[3 * a], dy = gy - xyz[3 * a + 1], dz = gz - xyz[3 * a + 2];
        double dist = sqrt((dx * dx) + (dy * dy) + (dz * dz));
        double charge = ec * q[a];
        if (ph->xkappa > VSMALL)
            val += pre1 * (charge / dist) * exp(-ph->xkappa * (dist - r[a])) /
                   (1 + ph->xkappa * r[a]);
        else
            val += pre1 * (charge / dist);
    }
    return val;
}

static void bc_mdh(const pmgb_params *p, const Phys *ph, int natoms, const double *xyz,
                   const double *q, const double *r, const Fill *f) {
    const double ec = 1.6021773e-19, eps0 = 8.8541878e-12, kb = 1.3806581e-23;
    const double pi = 3.14159265358979323846;
    const double pre1 = ((ec) / (4 * pi * eps0 * p->sdie * kb * p->temp)) * (1.0e10);
    int nx = p->nx, ny = p->ny, nz = p->nz, i, j, k;
    for (k = 0; k < nz; k++)
        for (j = 0; j < ny; j++) {
            f->gx[((size_t)0 * nz + k) * ny + j] =
                0.0 + mdh_value(ph, pre1, natoms, xyz, q, r, f->xf[0], f->yf[j], f->zf[k]);
            f->gx[((size_t)1 * nz + k) * ny + j] =
                0.0 + mdh_value(ph, pre1, natoms, xyz, q, r, f->xf[nx - 1], f->yf[j], f->zf[k]);
        }
    for (k = 0; k < nz; k++)
        for (i = 0; i < nx; i++) {
            f->gy[((size_t)0 * nz + k) * nx + i] =
                0.0 + mdh_value(ph, pre1, natoms, xyz, q, r, f->xf[i], f->yf[0], f->zf[k]);
            f->gy[((size_t)1 * nz + k) * nx + i] =
                0.0 + mdh_value(ph, pre1, natoms, xyz, q, r, f->xf[i], f->yf[ny - 1], f->zf[k]);
        }
    for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
            f->gz[((size_t)0 * ny + j) * nx + i] =
                0.0 + mdh_value(ph, pre1, natoms, xyz, q, r, f->xf[i], f->yf[j], f->zf[0]);
            f->gz[((size_t)1 * ny + j) * nx + i] =
                0.0 + mdh_value(ph, pre1, natoms, xyz, q, r, f->xf[i], f->yf[j], f->zf[nz - 1]);
        }
}

static void do_fill(const pmgb_params *p, const Phys *ph, int natoms,
                    const double *xyz, const double *q, const double *r,
                    Fill *f) {
    int nx = p->nx, ny = p->ny, nz = p->nz, i;
    double xlen = (nx - 1) * p->hx, ylen = (ny - 1) * p->hy,
           zlen = (nz - 1) * p->hz;
    int islap;
    /* vpmg.c:5332-5366 */
    f->xmn[0] = p->center[0] - (xlen / 2.0);
    f->xmn[1] = p->center[1] - (ylen / 2.0);
    f->xmn[2] = p->center[2] - (zlen / 2.0);
    f->xmx[0] = p->center[0] + (xlen / 2.0);
    f->xmx[1] = p->center[1] + (ylen / 2.0);
    f->xmx[2] = p->center[2] + (zlen / 2.0);
    for (i = 0; i < nx; i++) f->xf[i] = f->xmn[0] + i * p->hx;
    for (i = 0; i < ny; i++) f->yf[i] = f->xmn[1] + i * p->hy;
    for (i = 0; i < nz; i++) f->zf[i] = f->xmn[2] + i * p->hz;
    islap = (ph->ionstr < VPMGSMALL) && (fabs(p->pdie - p->sdie) < VPMGSMALL);
    if (p->chgm == PMGB_CHGM_TRIL)
        fill_charge_tril(p, ph, natoms, xyz, q, f->xmn, f->xmx, f->charge);
    else
        fill_charge_spl2(p, ph, natoms, xyz, q, f->xmn, f->xmx, f->charge);
    if (!islap) {
        fill_diel(p, ph, natoms, xyz, r, f->xmn, f->xmx, f->epsx, f->epsy, f->epsz);
        if (p->srfm == PMGB_SRFM_SMOL) smooth_diel(p, f->epsx, f->epsy, f->epsz);
        fill_kappa(p, ph, natoms, xyz, r, f->xmn, f->xmx, f->kappa);
    } else {
        size_t n = (size_t)nx * ny * nz, t;
        for (t = 0; t < n; t++) {
            f->kappa[t] = 0.0;
            f->epsx[t] = f->epsy[t] = f->epsz[t] = p->pdie;
        }
    }
    if (p->bcfl == PMGB_BCFL_FOCUS) {
        /* Vpmg_fillco leaves the faces alone when focusing (vpmg.c:5404-5409):
         * they were set from the coarse solution by focus_fill_bound. */
    } else if (p->bcfl == PMGB_BCFL_SDH) {
        bc_sdh(p, ph, natoms, xyz, q, f->xf, f->yf, f->zf, f->gx, f->gy, f->gz);
    } else if (p->bcfl == PMGB_BCFL_MDH) {
        bc_mdh(p, ph, natoms, xyz, q, r, f);
    } else {
        memset(f->gx, 0, sizeof(double) * 2 * ny * nz);
        memset(f->gy, 0, sizeof(double) * 2 * nx * nz);
        memset(f->gz, 0, sizeof(double) * 2 * nx * ny);
    }
}

/* ===================================================================== */
/* Operators                                                              */
/* ===================================================================== */
enum { OC, OE, ON, UC, ONE, ONW, UE, UW, UN, US, UNE, UNW, USE, USW };

/* VbuildA_fv, src/pmgc/buildAd.c:105-283 */
static void build_fine(const pmgb_params *p, const Fill *f, const double *ccf,
                       Level *L) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k;
    const double *xf = f->xf, *yf = f->yf, *zf = f->zf;
    const double *a1 = f->epsx, *a2 = f->epsy, *a3 = f->epsz;
    const double *fcf = f->charge;
    double *oC = L->op[OC], *oE = L->op[OE], *oN = L->op[ON], *uC = L->op[UC];
    (void)p;
    for (k = 1; k <= nz - 2; k++) {
        double hzm1 = zf[k] - zf[k - 1], hz = zf[k + 1] - zf[k];
        for (j = 1; j <= ny - 2; j++) {
            double hym1 = yf[j] - yf[j - 1], hy = yf[j + 1] - yf[j];
            for (i = 1; i <= nx - 2; i++) {
                double hxm1 = xf[i] - xf[i - 1], hx = xf[i + 1] - xf[i];
                double cE = 1.0 * (hym1 + hy) * (hzm1 + hz) / (4.0 * hx);
                double cEm = 1.0 * (hym1 + hy) * (hzm1 + hz) / (4.0 * hxm1);
                double cN = 1.0 * (hxm1 + hx) * (hzm1 + hz) / (4.0 * hy);
                double cNm = 1.0 * (hxm1 + hx) * (hzm1 + hz) / (4.0 * hym1);
                double cU = 1.0 * (hxm1 + hx) * (hym1 + hy) / (4.0 * hz);
                double cUm = 1.0 * (hxm1 + hx) * (hym1 + hy) / (4.0 * hzm1);
                double cF = 1.0 * (hxm1 + hx) * (hym1 + hy) * (hzm1 + hz) / 8.0;
                size_t id = IJK(i, j, k);
                int ike, jke, kke;
                double fc = cF * fcf[id];
                L->cc[id] = cF * ccf[id];
                oC[id] = cE * a1[id] + cEm * a1[IJK(i - 1, j, k)] + cN * a2[id] +
                         cNm * a2[IJK(i, j - 1, k)] + cU * a3[id] +
                         cUm * a3[IJK(i, j, k - 1)];
                ike = (i == nx - 2) ? 0 : 1;
                oE[id] = ike * cE * a1[id];
                fc += (1 - ike) * cE * a1[id] * f->gx[((size_t)1 * nz + k) * ny + j];
                jke = (j == ny - 2) ? 0 : 1;
                oN[id] = jke * cN * a2[id];
                fc += (1 - jke) * cN * a2[id] * f->gy[((size_t)1 * nz + k) * nx + i];
                kke = (k == nz - 2) ? 0 : 1;
                uC[id] = kke * cU * a3[id];
                fc += (1 - kke) * cU * a3[id] * f->gz[((size_t)1 * ny + j) * nx + i];
                ike = (i == 1) ? 0 : 1;
                fc += (1 - ike) * cEm * a1[IJK(i - 1, j, k)] *
                      f->gx[((size_t)0 * nz + k) * ny + j];
                jke = (j == 1) ? 0 : 1;
                fc += (1 - jke) * cNm * a2[IJK(i, j - 1, k)] *
                      f->gy[((size_t)0 * nz + k) * nx + i];
                kke = (k == 1) ? 0 : 1;
                fc += (1 - kke) * cUm * a3[IJK(i, j, k - 1)] *
                      f->gz[((size_t)0 * ny + j) * nx + i];
                L->fc[id] = fc;
            }
        }
    }
}

/* Matrix entry A(a, a+d) of a level operator for |d|_inf <= 1 (27 offsets),
 * excluding the Helmholtz diagonal: diag = oC, off-diagonal = -coefficient,
 * lower-half couplings read from the neighbour by symmetry (the stencil of
 * Vmatvec27_1s, src/pmgc/matvecd.c:153-228). */
static double op_entry(const Level *L, int i, int j, int k, int dx, int dy,
                       int dz) {
    int nx = L->nx, ny = L->ny;
    int code, si = i, sj = j, sk = k;
    /* canonical stored direction: dz>0, or dz==0&&dy>0, or dz==dy==0&&dx>0 */
    if (dx == 0 && dy == 0 && dz == 0) return L->op[OC][IJK(i, j, k)];
    if (dz < 0 || (dz == 0 && dy < 0) || (dz == 0 && dy == 0 && dx < 0)) {
        si = i + dx; sj = j + dy; sk = k + dz;
        dx = -dx; dy = -dy; dz = -dz;
    }
    if (dz == 0) {
        if (dy == 0) code = OE;
        else if (dx == 0) code = ON;
        else code = (dx > 0) ? ONE : ONW;
    } else {
        if (dx == 0 && dy == 0) code = UC;
        else if (dy == 0) code = (dx > 0) ? UE : UW;
        else if (dx == 0) code = (dy > 0) ? UN : US;
        else if (dy > 0) code = (dx > 0) ? UNE : UNW;
        else code = (dx > 0) ? USE : USW;
    }
    if (code >= L->nop) return 0.0;
    return -L->op[code][IJK(si, sj, sk)];
}

/* Galerkin coarse operator A_c = P^T A_f P with the trilinear prolongation
 * of VbuildPb_trilin (src/pmgc/buildPd.c:114-204: weights 1, 1/2, 1/4, 1/8
 * at interior coarse points, zero at coarse boundary points).  This is the
 * product that VbuildG_7 / VbuildG_27 (src/pmgc/buildGd.c:450-3115) expand
 * term by term; the result is stored as the 14 coefficients of the
 * symmetric 27-point stencil (Vbuildgaler0, src/pmgc/mgsubd.c:345-378). */
static void build_galerkin(const Level *F, Level *C) {
    int nx = C->nx, ny = C->ny, nz = C->nz;
    int I, J, K;
    for (K = 1; K <= nz - 2; K++)
        for (J = 1; J <= ny - 2; J++)
            for (I = 1; I <= nx - 2; I++) {
                double acc[27];
                int a0, a1, a2;
                memset(acc, 0, sizeof(acc));
                for (a2 = -1; a2 <= 1; a2++)
                    for (a1 = -1; a1 <= 1; a1++)
                        for (a0 = -1; a0 <= 1; a0++) {
                            int fi = 2 * I + a0, fj = 2 * J + a1, fk = 2 * K + a2;
                            double wa = 1.0 / (double)(1 << (abs(a0) + abs(a1) + abs(a2)));
                            int b0, b1, b2;
                            if (fi < 1 || fj < 1 || fk < 1 || fi > F->nx - 2 ||
                                fj > F->ny - 2 || fk > F->nz - 2)
                                continue;
                            for (b2 = -1; b2 <= 1; b2++)
                                for (b1 = -1; b1 <= 1; b1++)
                                    for (b0 = -1; b0 <= 1; b0++) {
                                        int gi = fi + b0, gj = fj + b1, gk = fk + b2;
                                        double aab;
                                        int c0, c1, c2;
                                        if (gi < 1 || gj < 1 || gk < 1 ||
                                            gi > F->nx - 2 || gj > F->ny - 2 ||
                                            gk > F->nz - 2)
                                            continue;
                                        aab = op_entry(F, fi, fj, fk, b0, b1, b2);
                                        if (aab == 0.0) continue;
                                        /* coarse points whose basis covers g */
                                        for (c2 = (gk - 1) / 2; c2 <= (gk + 1) / 2; c2++)
                                            for (c1 = (gj - 1) / 2; c1 <= (gj + 1) / 2; c1++)
                                                for (c0 = (gi - 1) / 2; c0 <= (gi + 1) / 2; c0++) {
                                                    int e0 = gi - 2 * c0, e1 = gj - 2 * c1,
                                                        e2 = gk - 2 * c2;
                                                    double wb;
                                                    if (abs(e0) > 1 || abs(e1) > 1 || abs(e2) > 1)
                                                        continue;
                                                    if (c0 < 1 || c1 < 1 || c2 < 1 ||
                                                        c0 > nx - 2 || c1 > ny - 2 || c2 > nz - 2)
                                                        continue;
                                                    if (abs(c0 - I) > 1 || abs(c1 - J) > 1 ||
                                                        abs(c2 - K) > 1)
                                                        continue;
                                                    wb = 1.0 / (double)(1 << (abs(e0) + abs(e1) + abs(e2)));
                                                    acc[((c2 - K + 1) * 3 + (c1 - J + 1)) * 3 +
                                                        (c0 - I + 1)] += wa * aab * wb;
                                                }
                                    }
                        }
                {
                    size_t id = IJK(I, J, K);
#define ACC(dx, dy, dz) acc[(((dz) + 1) * 3 + ((dy) + 1)) * 3 + ((dx) + 1)]
                    C->op[OC][id] = ACC(0, 0, 0);
                    C->op[OE][id] = -ACC(1, 0, 0);
                    C->op[ON][id] = -ACC(0, 1, 0);
                    C->op[UC][id] = -ACC(0, 0, 1);
                    C->op[ONE][id] = -ACC(1, 1, 0);
                    C->op[ONW][id] = -ACC(-1, 1, 0);
                    C->op[UE][id] = -ACC(1, 0, 1);
                    C->op[UW][id] = -ACC(-1, 0, 1);
                    C->op[UN][id] = -ACC(0, 1, 1);
                    C->op[US][id] = -ACC(0, -1, 1);
                    C->op[UNE][id] = -ACC(1, 1, 1);
                    C->op[UNW][id] = -ACC(-1, 1, 1);
                    C->op[USE][id] = -ACC(1, -1, 1);
                    C->op[USW][id] = -ACC(-1, -1, 1);
#undef ACC
                }
            }
}

/* Vrestrc2, src/pmgc/matvecd.c:801-911 (full weighting, interior coarse
 * points; output boundary zero) */
static void restrict_fw(const Level *F, const Level *C, const double *xin,
                        double *xout) {
    int nx = F->nx, ny = F->ny;
    int cx = C->nx, cy = C->ny, cz = C->nz, i, j, k;
    const double h = 0.5, qq = 0.25, e = 0.125;
    memset(xout, 0, sizeof(double) * C->n);
#define XI(a, b, c) xin[IJK(a, b, c)]
    for (k = 1; k <= cz - 2; k++) {
        int kk = 2 * k;
        for (j = 1; j <= cy - 2; j++) {
            int jj = 2 * j;
            for (i = 1; i <= cx - 2; i++) {
                int ii = 2 * i;
                double tO = +1.0 * XI(ii, jj, kk) + h * XI(ii, jj + 1, kk) +
                            h * XI(ii, jj - 1, kk) + h * XI(ii + 1, jj, kk) +
                            h * XI(ii - 1, jj, kk) + qq * XI(ii + 1, jj + 1, kk) +
                            qq * XI(ii - 1, jj + 1, kk) + qq * XI(ii + 1, jj - 1, kk) +
                            qq * XI(ii - 1, jj - 1, kk);
                double tU = +h * XI(ii, jj, kk + 1) + qq * XI(ii, jj + 1, kk + 1) +
                            qq * XI(ii, jj - 1, kk + 1) + qq * XI(ii + 1, jj, kk + 1) +
                            qq * XI(ii - 1, jj, kk + 1) + e * XI(ii + 1, jj + 1, kk + 1) +
                            e * XI(ii - 1, jj + 1, kk + 1) + e * XI(ii + 1, jj - 1, kk + 1) +
                            e * XI(ii - 1, jj - 1, kk + 1);
                double tD = +h * XI(ii, jj, kk - 1) + qq * XI(ii, jj + 1, kk - 1) +
                            qq * XI(ii, jj - 1, kk - 1) + qq * XI(ii + 1, jj, kk - 1) +
                            qq * XI(ii - 1, jj, kk - 1) + e * XI(ii + 1, jj + 1, kk - 1) +
                            e * XI(ii - 1, jj + 1, kk - 1) + e * XI(ii + 1, jj - 1, kk - 1) +
                            e * XI(ii - 1, jj - 1, kk - 1);
                xout[(size_t)(k * cy + j) * cx + i] = tO + tU + tD;
            }
        }
    }
#undef XI
}

/* VinterpPMG2, src/pmgc/matvecd.c:935-1074 (trilinear; coarse boundary
 * values are zero so the zero weights stored there drop out) */
static void interp_tl(const Level *C, const Level *F, const double *xc,
                      double *xf) {
    int cx = C->nx, cy = C->ny;
    int nx = F->nx, ny = F->ny, nz = F->nz, i, j, k;
    const double h = 0.5, qq = 0.25, e = 0.125;
#define XC(a, b, c) xc[(size_t)((c) * cy + (b)) * cx + (a)]
#define XF(a, b, c) xf[IJK(a, b, c)]
    for (k = 0; k <= nz - 3; k += 2) {
        int kk = k / 2;
        for (j = 0; j <= ny - 3; j += 2) {
            int jj = j / 2;
            for (i = 0; i <= nx - 3; i += 2) {
                int ii = i / 2;
                XF(i, j, k) = XC(ii, jj, kk);
                XF(i + 1, j, k) = h * XC(ii, jj, kk) + h * XC(ii + 1, jj, kk);
                XF(i, j + 1, k) = h * XC(ii, jj, kk) + h * XC(ii, jj + 1, kk);
                XF(i, j, k + 1) = h * XC(ii, jj, kk) + h * XC(ii, jj, kk + 1);
                XF(i + 1, j + 1, k) = qq * XC(ii, jj, kk) + qq * XC(ii + 1, jj, kk) +
                                      qq * XC(ii, jj + 1, kk) + qq * XC(ii + 1, jj + 1, kk);
                XF(i + 1, j, k + 1) = qq * XC(ii, jj, kk) + qq * XC(ii + 1, jj, kk) +
                                      qq * XC(ii, jj, kk + 1) + qq * XC(ii + 1, jj, kk + 1);
                XF(i, j + 1, k + 1) = qq * XC(ii, jj, kk) + qq * XC(ii, jj + 1, kk) +
                                      qq * XC(ii, jj, kk + 1) + qq * XC(ii, jj + 1, kk + 1);
                XF(i + 1, j + 1, k + 1) =
                    +e * XC(ii, jj, kk) + e * XC(ii + 1, jj, kk) + e * XC(ii, jj + 1, kk) +
                    e * XC(ii + 1, jj + 1, kk) + e * XC(ii, jj, kk + 1) +
                    e * XC(ii + 1, jj, kk + 1) + e * XC(ii, jj + 1, kk + 1) +
                    e * XC(ii + 1, jj + 1, kk + 1);
            }
        }
    }
    /* VfboundPMG00 on the output */
    for (k = 0; k < nz; k++)
        for (j = 0; j < ny; j++)
            for (i = 0; i < nx; i++)
                if (i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1)
                    XF(i, j, k) = 0.0;
#undef XC
#undef XF
}

/* Neighbour-coefficient products of the 27-point stencil in the order of
 * Vgsrb27x / Vmresid27_1s (src/pmgc/gsd.c:249-282, matvecd.c:563-594). */
#define STENCIL27(L, x, i, j, k, tO, tU, tD)                                       \
    do {                                                                           \
        double **o = (L)->op;                                                      \
        tO = +o[ON][IJK(i, j, k)] * x[IJK(i, j + 1, k)] +                          \
             o[ON][IJK(i, j - 1, k)] * x[IJK(i, j - 1, k)] +                       \
             o[OE][IJK(i, j, k)] * x[IJK(i + 1, j, k)] +                           \
             o[OE][IJK(i - 1, j, k)] * x[IJK(i - 1, j, k)] +                       \
             o[ONE][IJK(i, j, k)] * x[IJK(i + 1, j + 1, k)] +                      \
             o[ONW][IJK(i, j, k)] * x[IJK(i - 1, j + 1, k)] +                      \
             o[ONW][IJK(i + 1, j - 1, k)] * x[IJK(i + 1, j - 1, k)] +              \
             o[ONE][IJK(i - 1, j - 1, k)] * x[IJK(i - 1, j - 1, k)];               \
        tU = +o[UC][IJK(i, j, k)] * x[IJK(i, j, k + 1)] +                          \
             o[UN][IJK(i, j, k)] * x[IJK(i, j + 1, k + 1)] +                       \
             o[US][IJK(i, j, k)] * x[IJK(i, j - 1, k + 1)] +                       \
             o[UE][IJK(i, j, k)] * x[IJK(i + 1, j, k + 1)] +                       \
             o[UW][IJK(i, j, k)] * x[IJK(i - 1, j, k + 1)] +                       \
             o[UNE][IJK(i, j, k)] * x[IJK(i + 1, j + 1, k + 1)] +                  \
             o[UNW][IJK(i, j, k)] * x[IJK(i - 1, j + 1, k + 1)] +                  \
             o[USE][IJK(i, j, k)] * x[IJK(i + 1, j - 1, k + 1)] +                  \
             o[USW][IJK(i, j, k)] * x[IJK(i - 1, j - 1, k + 1)];                   \
        tD = +o[UC][IJK(i, j, k - 1)] * x[IJK(i, j, k - 1)] +                      \
             o[US][IJK(i, j + 1, k - 1)] * x[IJK(i, j + 1, k - 1)] +               \
             o[UN][IJK(i, j - 1, k - 1)] * x[IJK(i, j - 1, k - 1)] +               \
             o[UW][IJK(i + 1, j, k - 1)] * x[IJK(i + 1, j, k - 1)] +               \
             o[UE][IJK(i - 1, j, k - 1)] * x[IJK(i - 1, j, k - 1)] +               \
             o[USW][IJK(i + 1, j + 1, k - 1)] * x[IJK(i + 1, j + 1, k - 1)] +      \
             o[USE][IJK(i - 1, j + 1, k - 1)] * x[IJK(i - 1, j + 1, k - 1)] +      \
             o[UNW][IJK(i + 1, j - 1, k - 1)] * x[IJK(i + 1, j - 1, k - 1)] +      \
             o[UNE][IJK(i - 1, j - 1, k - 1)] * x[IJK(i - 1, j - 1, k - 1)];       \
    } while (0)

#define STENCIL7(L, x, i, j, k)                                                    \
    ((L)->op[ON][IJK(i, j, k)] * x[IJK(i, j + 1, k)] +                             \
     (L)->op[ON][IJK(i, j - 1, k)] * x[IJK(i, j - 1, k)] +                         \
     (L)->op[OE][IJK(i, j, k)] * x[IJK(i + 1, j, k)] +                             \
     (L)->op[OE][IJK(i - 1, j, k)] * x[IJK(i - 1, j, k)] +                         \
     (L)->op[UC][IJK(i, j, k - 1)] * x[IJK(i, j, k - 1)] +                         \
     (L)->op[UC][IJK(i, j, k)] * x[IJK(i, j, k + 1)])

/* Red-black Gauss-Seidel, Vgsrb7x / Vgsrb27x (src/pmgc/gsd.c:95-340).
 * The 27-point sweep visits one colour in lexicographic order, so
 * same-colour edge neighbours already updated in this sweep are read. */
static void smooth_gs(const Level *L, const double *cc, const double *fc,
                      double *x, int nsweep, int adjoint) {
    int nx = L->nx, ny = L->ny, nz = L->nz, it, colour, i, j, k;
    for (it = 0; it < nsweep; it++)
        for (colour = 0; colour < 2; colour++)
            for (k = 1; k <= nz - 2; k++)
                for (j = 1; j <= ny - 2; j++) {
                    /* (j+k+2)%2 in 1-based indices == (j+k)%2 here */
                    int par = (j + k) % 2;
                    int ioff = (colour == 0) ? (adjoint ? 1 - par : par)
                                             : (adjoint ? par : 1 - par);
                    for (i = 1 + ioff; i <= nx - 2; i += 2) {
                        size_t id = IJK(i, j, k);
                        if (L->nop == 4) {
                            x[id] = (fc[id] + L->op[ON][id] * x[IJK(i, j + 1, k)] +
                                     L->op[ON][IJK(i, j - 1, k)] * x[IJK(i, j - 1, k)] +
                                     L->op[OE][id] * x[IJK(i + 1, j, k)] +
                                     L->op[OE][IJK(i - 1, j, k)] * x[IJK(i - 1, j, k)] +
                                     L->op[UC][IJK(i, j, k - 1)] * x[IJK(i, j, k - 1)] +
                                     L->op[UC][id] * x[IJK(i, j, k + 1)]) /
                                    (L->op[OC][id] + cc[id]);
                        } else {
                            double tO, tU, tD;
                            STENCIL27(L, x, i, j, k, tO, tU, tD);
                            x[id] = (fc[id] + (tO + tU + tD)) / (L->op[OC][id] + cc[id]);
                        }
                    }
                }
}

/* r = f - (A + diag cc) x, Vmresid7_1s / Vmresid27_1s (matvecd.c:461-594) */
static void resid(const Level *L, const double *cc, const double *fc,
                  const double *x, double *r) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k;
    for (k = 1; k <= nz - 2; k++)
        for (j = 1; j <= ny - 2; j++)
            for (i = 1; i <= nx - 2; i++) {
                size_t id = IJK(i, j, k);
                if (L->nop == 4) {
                    r[id] = fc[id] + L->op[ON][id] * x[IJK(i, j + 1, k)] +
                            L->op[ON][IJK(i, j - 1, k)] * x[IJK(i, j - 1, k)] +
                            L->op[OE][id] * x[IJK(i + 1, j, k)] +
                            L->op[OE][IJK(i - 1, j, k)] * x[IJK(i - 1, j, k)] +
                            L->op[UC][IJK(i, j, k - 1)] * x[IJK(i, j, k - 1)] +
                            L->op[UC][id] * x[IJK(i, j, k + 1)] -
                            (L->op[OC][id] + cc[id]) * x[id];
                } else {
                    double tO, tU, tD;
                    STENCIL27(L, x, i, j, k, tO, tU, tD);
                    r[id] = fc[id] + tO + tU + tD - (L->op[OC][id] + cc[id]) * x[id];
                }
            }
}

/* y = (A + diag cc) x, Vmatvec7_1s / Vmatvec27_1s (matvecd.c:98-228) */
static void matvec(const Level *L, const double *cc, const double *x, double *y) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k;
    for (k = 1; k <= nz - 2; k++)
        for (j = 1; j <= ny - 2; j++)
            for (i = 1; i <= nx - 2; i++) {
                size_t id = IJK(i, j, k);
                if (L->nop == 4) {
                    y[id] = -L->op[ON][id] * x[IJK(i, j + 1, k)] -
                            L->op[ON][IJK(i, j - 1, k)] * x[IJK(i, j - 1, k)] -
                            L->op[OE][id] * x[IJK(i + 1, j, k)] -
                            L->op[OE][IJK(i - 1, j, k)] * x[IJK(i - 1, j, k)] -
                            L->op[UC][IJK(i, j, k - 1)] * x[IJK(i, j, k - 1)] -
                            L->op[UC][id] * x[IJK(i, j, k + 1)] +
                            (L->op[OC][id] + cc[id]) * x[id];
                } else {
                    double tO, tU, tD;
                    STENCIL27(L, x, i, j, k, tO, tU, tD);
                    y[id] = -tO - tU - tD + (L->op[OC][id] + cc[id]) * x[id];
                }
            }
}

/* Interior-point BLAS-1 (src/pmgc/mikpckd.c:57-328) */
static double nrm1(const Level *L, const double *x) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k;
    double s = 0.0;
    for (k = 1; k <= nz - 2; k++)
        for (j = 1; j <= ny - 2; j++)
            for (i = 1; i <= nx - 2; i++) s += fabs(x[IJK(i, j, k)]);
    return s;
}
static double dot(const Level *L, const double *x, const double *y) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k;
    double s = 0.0;
    for (k = 1; k <= nz - 2; k++)
        for (j = 1; j <= ny - 2; j++)
            for (i = 1; i <= nx - 2; i++) s += x[IJK(i, j, k)] * y[IJK(i, j, k)];
    return s;
}
static void axpy(const Level *L, double a, const double *x, double *y) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k;
    for (k = 1; k <= nz - 2; k++)
        for (j = 1; j <= ny - 2; j++)
            for (i = 1; i <= nx - 2; i++) y[IJK(i, j, k)] += a * x[IJK(i, j, k)];
}
static void copy_int(const Level *L, const double *x, double *y) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k;
    for (k = 1; k <= nz - 2; k++)
        for (j = 1; j <= ny - 2; j++)
            for (i = 1; i <= nx - 2; i++) y[IJK(i, j, k)] = x[IJK(i, j, k)];
}
static void scal(const Level *L, double a, double *x) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k;
    for (k = 1; k <= nz - 2; k++)
        for (j = 1; j <= ny - 2; j++)
            for (i = 1; i <= nx - 2; i++) x[IJK(i, j, k)] *= a;
}

/* Nonlinear ion term c(u) and c'(u), Vc_vecpmg / Vdc_vecpmg
 * (src/pmgc/mypdec.c:145-223, 366-433), over every grid point. */
static void c_vec(const pmgb_params *p, const Phys *ph, size_t n,
                  const double *coef, const double *u, double *out, int deriv) {
    size_t i;
    int s;
    for (i = 0; i < n; i++) out[i] = 0;
    for (s = 0; s < p->nion; s++) {
        double zcf2 = deriv ? ph->sconc[s] * p->ion_q[s] * p->ion_q[s]
                            : -1.0 * ph->sconc[s] * p->ion_q[s];
        double zu2 = -1.0 * p->ion_q[s];
        for (i = 0; i < n; i++) {
            double t = fabs(zcf2 * coef[i]);
            double am_zero = (ZSMALL <= t ? ZSMALL : t) * ZLARGE;
            double v = zu2 * u[i];
            double am_neg = (v <= 0.0 ? v : 0.0);
            double am_pos = (v >= 0.0 ? v : 0.0);
            if (!(am_neg >= -EXPCLAMP)) am_neg = -EXPCLAMP;
            if (!(am_pos <= EXPCLAMP)) am_pos = EXPCLAMP;
            out[i] = out[i] + zcf2 * coef[i] * exp(am_zero * (am_neg + am_pos));
        }
    }
}

/* Nonlinear residual r = f - A x - c(x) (Vnmresid7_1s, matvecd.c:633-691) */
static void nresid(const pmgb_params *p, const Phys *ph, const Level *L,
                   const double *cc, const double *fc, const double *x,
                   double *r, double *w) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k;
    c_vec(p, ph, L->n, cc, x, w, 0);
    for (k = 1; k <= nz - 2; k++)
        for (j = 1; j <= ny - 2; j++)
            for (i = 1; i <= nx - 2; i++) {
                size_t id = IJK(i, j, k);
                r[id] = fc[id] + STENCIL7(L, x, i, j, k) - L->op[OC][id] * x[id] - w[id];
            }
}

/* ===================================================================== */
/* Coarsest solves                                                        */
/* ===================================================================== */

/* Vbuildband1_27 (src/pmgc/buildBd.c:183-306): LINPACK upper band storage
 * of the coarsest operator WITHOUT the Helmholtz term (the reference stores
 * oC alone on the diagonal), with the couplings written exactly as the
 * reference does; then factor (Vdpbfa, src/pmgc/mlinpckd.c:194-233). */
static int build_band(Solver *s, const Level *L) {
    int nx = L->nx, ny = L->ny, nz = L->nz, i, j, k, jj = 0;
    int ex = nx - 2, exy = (nx - 2) * (ny - 2);
    int n = (nx - 2) * (ny - 2) * (nz - 2);
    int m = exy + ex + 1, lda = m + 1, col;
    double *abd = (double *)calloc((size_t)lda * n, sizeof(double));
#define AB(row, c) abd[(size_t)((c) - 1) * lda + ((row) - 1)]
#define PUT(off, val) AB((jj + (off)) - jj + m + 1, jj) = (val)
    for (k = 1; k <= nz - 2; k++)
        for (j = 1; j <= ny - 2; j++)
            for (i = 1; i <= nx - 2; i++) {
                jj++;
                PUT(0, L->op[OC][IJK(i, j, k)]);
                PUT(-1, -L->op[OE][IJK(i - 1, j, k)]);
                PUT(-ex, -L->op[ON][IJK(i, j - 1, k)]);
                PUT(-ex + 1, -L->op[ONE][IJK(i, j - 1, k)]);
                PUT(-ex - 1, -L->op[ONW][IJK(i, j - 1, k)]);
                PUT(-exy, -L->op[UC][IJK(i, j, k - 1)]);
                PUT(-exy + 1, -L->op[UE][IJK(i, j, k - 1)]);
                PUT(-exy - 1, -L->op[UW][IJK(i, j, k - 1)]);
                PUT(-exy + ex, -L->op[UN][IJK(i, j, k - 1)]);
                PUT(-exy - ex, -L->op[US][IJK(i, j, k - 1)]);
                PUT(-exy + ex + 1, -L->op[UNE][IJK(i, j, k - 1)]);
                PUT(-exy + ex - 1, -L->op[UNW][IJK(i, j, k - 1)]);
                PUT(-exy - ex + 1, -L->op[USE][IJK(i, j, k - 1)]);
                PUT(-exy - ex - 1, -L->op[USW][IJK(i, j, k - 1)]);
            }
#undef PUT
    /* Cholesky R^T R of the band (dpbfa) */
    for (col = 1; col <= n; col++) {
        double sacc = 0.0;
        int ik = m + 1, jk = (col - m > 1) ? col - m : 1;
        int mu = (m + 2 - col > 1) ? m + 2 - col : 1, kk;
        for (kk = mu; kk <= m; kk++) {
            double t, d = 0.0;
            int l;
            for (l = 0; l < kk - mu; l++) d += AB(ik + l, jk) * AB(mu + l, col);
            t = AB(kk, col) - d;
            t /= AB(m + 1, jk);
            AB(kk, col) = t;
            sacc += t * t;
            ik--;
            jk++;
        }
        sacc = AB(m + 1, col) - sacc;
        if (sacc <= 0.0) { free(abd); return 0; }
        AB(m + 1, col) = sqrt(sacc);
    }
#undef AB
    s->band = abd;
    s->bn = n;
    s->bm = m;
    s->blda = lda;
    return 1;
}

/* Vdpbsl (src/pmgc/mlinpckd.c:57-83): solve R^T R b' = b in place */
static void band_solve(const Solver *s, double *b) {
    int n = s->bn, m = s->bm, lda = s->blda, k, l;
    const double *abd = s->band;
#define AB(row, c) abd[(size_t)((c) - 1) * lda + ((row) - 1)]
    for (k = 1; k <= n; k++) {
        int lm = (k - 1 < m) ? k - 1 : m, la = m + 1 - lm, lb = k - lm;
        double t = 0.0;
        for (l = 0; l < lm; l++) t += AB(la + l, k) * b[lb - 1 + l];
        b[k - 1] = (b[k - 1] - t) / AB(m + 1, k);
    }
    for (k = n; k >= 1; k--) {
        int lm = (k - 1 < m) ? k - 1 : m, la = m + 1 - lm, lb = k - lm;
        double t;
        b[k - 1] /= AB(m + 1, k);
        t = -b[k - 1];
        for (l = 0; l < lm; l++) b[lb - 1 + l] += t * AB(la + l, k);
    }
#undef AB
}

/* Vcghs (src/pmgc/cgd.c:57-123): CG on the coarsest level, <= itmax
 * iterations, stop when ||r||_2 / ||f||_2 <= errtol */
static void cg_coarse(const Level *L, const double *cc, const double *fc,
                      double *x, double *pv, double *ap, double *r, int itmax,
                      double errtol) {
    double denom, rhok1 = 0.0, rhok2, alpha, beta;
    int iters = 0;
    resid(L, cc, fc, x, r);
    denom = sqrt(dot(L, r, r));
    if (denom == 0.0) return;
    for (;;) {
        rhok2 = dot(L, r, r);
        if (sqrt(rhok2) / denom <= errtol) break;
        if (iters >= itmax) break;
        if (iters == 0) {
            copy_int(L, r, pv);
        } else {
            beta = rhok2 / rhok1;
            axpy(L, 1.0 / beta, r, pv);
            scal(L, beta, pv);
        }
        matvec(L, cc, pv, ap);
        alpha = rhok2 / dot(L, pv, ap);
        rhok1 = rhok2;
        axpy(L, alpha, pv, x);
        axpy(L, -alpha, ap, r);
        iters++;
    }
}

/* ===================================================================== */
/* V-cycle driver, Vmvcs (src/pmgc/mgcsd.c:57-565)                        */
/* ===================================================================== */
/* cc_of(l) / fc_of(l): the Helmholtz term and the fine rhs the cycle uses:
 * the linear problem's arrays, or the Newton system's c'(u) and rhs. */
static void vcycles(Solver *s, int newton, double errtol, int itmax,
                    int istop0, int *iters_out) {
    int nlev = s->nlev, l, iters = 0;
    Level *F = &s->lev[0];
    double rsden, rsnrm;
#define CC(l) (newton ? s->lev[l].cp : s->lev[l].cc)
#define FC0 (newton ? F->rhs : F->fc)
#define X(l) (newton ? s->lev[l].xt : s->lev[l].x)
    if (istop0) rsden = 1.0;
    else rsden = nrm1(F, FC0);
    if (rsden == 0.0) rsden = 1.0;
    rsnrm = rsden;
    logres(s, rsnrm / rsden);
    do {
        /* pre-smooth on the fine level, residual to w1, copy to w0 */
        smooth_gs(F, CC(0), FC0, X(0), 2, 0);
        resid(F, CC(0), FC0, X(0), s->w1);
        copy_int(F, s->w1, F->w0);
        for (l = 1; l < nlev; l++) {
            Level *C = &s->lev[l], *P = &s->lev[l - 1];
            restrict_fw(P, C, (l == 1) ? s->w1 : s->w1, C->w0);
            if (l != nlev - 1) {
                memset(X(l), 0, sizeof(double) * C->n);
                smooth_gs(C, CC(l), C->w0, X(l), 2, 0);
                resid(C, CC(l), C->w0, X(l), s->w1);
            }
        }
        /* coarsest level */
        {
            Level *C = &s->lev[nlev - 1];
            if (s->mgsolv == 1) {
                int cx = C->nx, cy = C->ny, cz = C->nz, i, j, k, t = 0;
                int nx = cx, ny = cy;
                double *b = s->w2;
                for (k = 1; k <= cz - 2; k++)
                    for (j = 1; j <= cy - 2; j++)
                        for (i = 1; i <= cx - 2; i++) b[t++] = C->w0[IJK(i, j, k)];
                band_solve(s, b);
                memset(X(nlev - 1), 0, sizeof(double) * C->n);
                t = 0;
                for (k = 1; k <= cz - 2; k++)
                    for (j = 1; j <= cy - 2; j++)
                        for (i = 1; i <= cx - 2; i++) X(nlev - 1)[IJK(i, j, k)] = b[t++];
            } else {
                memset(X(nlev - 1), 0, sizeof(double) * C->n);
                cg_coarse(C, CC(nlev - 1), C->w0, X(nlev - 1), s->w1, s->w2, s->w3,
                          100, 2.220446049250313e-16);
            }
        }
        /* up */
        for (l = nlev - 2; l >= 0; l--) {
            Level *C = &s->lev[l + 1], *P = &s->lev[l];
            double xnum, xden, xdamp;
            interp_tl(C, P, X(l + 1), s->w1);
            matvec(C, CC(l + 1), X(l + 1), s->w2);
            xnum = dot(C, X(l + 1), C->w0);
            xden = dot(C, X(l + 1), s->w2);
            xdamp = xnum / xden;
            axpy(P, xdamp, s->w1, X(l));
            smooth_gs(P, CC(l), (l == 0) ? FC0 : P->w0, X(l), 2, 1);
        }
        iters++;
        s->total_cycles++;
        resid(F, CC(0), FC0, X(0), s->w1);
        rsnrm = nrm1(F, s->w1);
        logres(s, rsnrm / rsden);
    } while (iters < itmax && (rsnrm / rsden) > errtol);
    *iters_out = iters;
#undef CC
#undef FC0
#undef X
}

/* Damped inexact Newton, Vnewton (src/pmgc/newtond.c:162-548) */
static int newton(Solver *s, const pmgb_params *p, const Phys *ph,
                  double errtol, int itmax) {
    Level *F = &s->lev[0];
    int nlev = s->nlev, l, iters = 0, idamp = 1;
    size_t n = F->n;
    double rsden, rsnrm, xnorm_old, xnorm_new, xnorm_med = 0.0, xnorm_den;
    double *x = F->x;
    double *r0 = (double *)calloc(n, sizeof(double));   /* Newton w0 */
    double *ws = (double *)calloc(n, sizeof(double));   /* Newton w1 */
    double *keepx = (double *)calloc(n, sizeof(double));/* Newton w2 */
    double *keepr = (double *)calloc(n, sizeof(double));/* Newton w3 */
    double *tmpw = (double *)calloc(n, sizeof(double));
    /* rsden = ||N(0)||_1 */
    memset(ws, 0, sizeof(double) * n);
    nresid(p, ph, F, F->cc, F->fc, ws, keepx, tmpw);
    rsden = nrm1(F, keepx);
    if (rsden == 0.0) rsden = 1.0;
    rsnrm = rsden;
    logres(s, rsnrm / rsden);
    nresid(p, ph, F, F->cc, F->fc, x, r0, tmpw);
    xnorm_old = nrm1(F, r0);
    xnorm_den = rsden;
    (void)xnorm_den;
    for (;;) {
        double errtol_s;
        int it_s;
        iters++;
        /* Vgetjac (newtond.c:550-598) */
        copy_int(F, r0, F->rhs);
        c_vec(p, ph, n, F->cc, x, F->cp, 1);
        for (l = 1; l < nlev; l++) {
            restrict_fw(&s->lev[l - 1], &s->lev[l], s->lev[l - 1].rhs, s->lev[l].rhs);
            restrict_fw(&s->lev[l - 1], &s->lev[l], s->lev[l - 1].cp, s->lev[l].cp);
        }
        errtol_s = (0.9 * xnorm_old <= 1.0 * pow(xnorm_old, 2.0)) ? 0.9 * xnorm_old
                                                                 : 1.0 * pow(xnorm_old, 2.0);
        memset(F->xt, 0, sizeof(double) * n);
        vcycles(s, 1, errtol_s, 1000, 1, &it_s);
        if (idamp == 1) {
            double damp = 1.0;
            int iter_d = 0, mode = 0;
            copy_int(F, x, ws);
            axpy(F, damp, F->xt, ws);
            nresid(p, ph, F, F->cc, F->fc, ws, r0, tmpw);
            xnorm_new = nrm1(F, r0);
            while (iter_d < 10) {
                if (mode == 0) {
                    if (xnorm_new < xnorm_old) mode = 1;
                } else if (xnorm_new > xnorm_med) {
                    break;
                }
                copy_int(F, ws, keepx);
                copy_int(F, r0, keepr);
                xnorm_med = xnorm_new;
                copy_int(F, x, ws);
                damp = damp / 2.0;
                axpy(F, damp, F->xt, ws);
                nresid(p, ph, F, F->cc, F->fc, ws, r0, tmpw);
                xnorm_new = nrm1(F, r0);
                iter_d++;
            }
            copy_int(F, keepx, x);
            copy_int(F, keepr, r0);
            xnorm_new = xnorm_med;
            xnorm_old = xnorm_new;
            if ((iter_d - 1) == 0) idamp = 0;
        } else {
            axpy(F, 1.0, F->xt, x);
            nresid(p, ph, F, F->cc, F->fc, x, r0, tmpw);
            xnorm_new = nrm1(F, r0);
            xnorm_old = xnorm_new;
        }
        rsnrm = xnorm_new;
        logres(s, rsnrm / rsden);
        if ((rsnrm / rsden) <= errtol) break;
        if (iters >= itmax) break;
    }
    free(r0); free(ws); free(keepx); free(keepr); free(tmpw);
    return iters;
}

/* ===================================================================== */
/* Energies (src/mg/vpmg.c:1248-1891) and partition weights (627-870)     */
/* ===================================================================== */
static void part_weights(int n, double h, double cent, double lo, double hi,
                         double *w) {
    /* Vpmg_setPart per-axis weight (vpmg.c:763-863) for the partition
     * [lo, hi] with no neighbouring processors (bflags all 0) */
    int i;
    double xmin = cent - 0.5 * h * (n - 1);
    for (i = 0; i < n; i++) {
        double x = i * h + xmin, ok;
        if ((x < (hi - h / 2)) && (x > (lo + h / 2))) ok = 1.0;
        else if (fabs(x - lo) < VPMGSMALL) ok = 1.0;
        else if (fabs(x - hi) < VPMGSMALL) ok = 1.0;
        else if ((x > (hi + h / 2)) || (x < (lo - h / 2))) ok = 0.0;
        else if ((x < (hi + h / 2)) || (x > (lo - h / 2))) {
            double x0 = (x - h / 2 >= lo) ? x - h / 2 : lo;
            double x1 = (x + h / 2 <= hi) ? x + h / 2 : hi;
            ok = fabs(x1 - x0) / h;
            if (ok < 0.0 && fabs(ok) < VPMGSMALL) ok = 0.0;
            if (ok > 1.0 && fabs(ok - 1.0) < VPMGSMALL) ok = 1.0;
        } else ok = 0.0;
        w[i] = ok;
    }
}

/* Energy sums of one solved calculation with partition weights pvec:
 *   pvec = setPart(lo, hi) weights (vpmg.c:863-866), or, with complement,
 *   the flipped weights extEnergy gives the coarse grid (vpmg.c:2508-2509):
 *   1 - pvec where pvec <= VSMALL, else 0.
 * comps: 0 qf only; 1 qf, diel and qm in the form the calculation's own
 * nonlinearity selects (Vpmg_qmEnergyNONLIN linear/nonlinear branches).
 * sums[0] qf, [1] diel, [2] qm, all in kT (vpmg.c:1279-1488, 1861-1891). */
static void energy_terms(const pmgb_params *p, const Phys *ph, const Fill *f,
                         const double *u, const double lo[3],
                         const double hi[3], int complement, int comps,
                         double sums[3]) {
    int nx = p->nx, ny = p->ny, nz = p->nz, i, j, k, s;
    size_t n = (size_t)nx * ny * nz, t;
    double *wx = (double *)malloc(sizeof(double) * (nx + ny + nz));
    double *wy = wx + nx, *wz = wy + ny, *pvec;
    double qf = 0.0, diel = 0.0, qm = 0.0;
    part_weights(nx, p->hx, p->center[0], lo[0], hi[0], wx);
    part_weights(ny, p->hy, p->center[1], lo[1], hi[1], wy);
    part_weights(nz, p->hz, p->center[2], lo[2], hi[2], wz);
    pvec = (double *)malloc(sizeof(double) * n);
    for (k = 0; k < nz; k++)
        for (j = 0; j < ny; j++)
            for (i = 0; i < nx; i++) {
                double v = wx[i] * wy[j] * wz[k];
                v = (fabs(v) < VPMGSMALL) ? 0.0 : v;
                if (complement) {
                    if (v > VSMALL) v = 1.0;
                    v = (1 - v) * 1.0;
                }
                pvec[IJK(i, j, k)] = v;
            }
    /* Vpmg_qfEnergyVolume (vpmg.c:1861-1891) */
    for (t = 0; t < n; t++) qf += (pvec[t] * u[t] * f->charge[t]);
    qf = qf * p->hx * p->hy * p->hz / ph->zmagic;
    if (comps) {
        /* Vpmg_dielEnergy (vpmg.c:1279-1340) */
        for (k = 0; k < nz - 1; k++)
            for (j = 0; j < ny - 1; j++)
                for (i = 0; i < nx - 1; i++) {
                    double px = 0.5 * (pvec[IJK(i, j, k)] + pvec[IJK(i + 1, j, k)]);
                    double py = 0.5 * (pvec[IJK(i, j, k)] + pvec[IJK(i, j + 1, k)]);
                    double pz = 0.5 * (pvec[IJK(i, j, k)] + pvec[IJK(i, j, k + 1)]);
                    double gx = (u[IJK(i, j, k)] - u[IJK(i + 1, j, k)]) / p->hx;
                    double gy = (u[IJK(i, j, k)] - u[IJK(i, j + 1, k)]) / p->hy;
                    double gz = (u[IJK(i, j, k)] - u[IJK(i, j, k + 1)]) / p->hz;
                    double ex = f->epsx[IJK(i, j, k)] * px * (gx * gx);
                    double ey = f->epsy[IJK(i, j, k)] * py * (gy * gy);
                    double ez = f->epsz[IJK(i, j, k)] * pz * (gz * gz);
                    diel += (ex + ey + ez);
                }
        diel = 0.5 * diel * p->hx * p->hy * p->hz;
        diel = diel / ph->zmagic;
        /* Vpmg_qmEnergyNONLIN (vpmg.c:1401-1488) with Vcap_exp (vcap.c:59) */
        if (!(ph->zkappa2 < VSMALL)) {
            double zks2 = 0.5 * ph->zkappa2 / ph->ionstr;
            if (p->nonlin) {
                for (t = 0; t < n; t++) {
                    if (pvec[t] * f->kappa[t] > VSMALL) {
                        for (s = 0; s < p->nion; s++) {
                            double a = -p->ion_q[s] * u[t], e;
                            if (a > EXPCLAMP) e = exp(EXPCLAMP);
                            else if (a < -EXPCLAMP) e = exp(-EXPCLAMP);
                            else e = exp(a);
                            qm += (pvec[t] * f->kappa[t] * zks2 * p->ion_conc[s] * (e - 1.0));
                        }
                    }
                }
            } else {
                for (t = 0; t < n; t++)
                    if (pvec[t] * f->kappa[t] > VSMALL)
                        qm += (pvec[t] * ph->zkappa2 * f->kappa[t] * (u[t] * u[t]));
                qm = 0.5 * qm;
            }
            qm = qm * p->hx * p->hy * p->hz;
            qm = qm / ph->zmagic;
        }
    }
    sums[0] = qf;
    sums[1] = diel;
    sums[2] = qm;
    free(pvec);
    free(wx);
}

static void domain_box(const pmgb_params *p, double lo[3], double hi[3]) {
    /* setPartMG partition for mg-manual: center -/+ glen/2 (routines.c:1712-1718) */
    lo[0] = p->center[0] - 0.5 * ((p->nx - 1) * p->hx);
    hi[0] = p->center[0] + 0.5 * ((p->nx - 1) * p->hx);
    lo[1] = p->center[1] - 0.5 * ((p->ny - 1) * p->hy);
    hi[1] = p->center[1] + 0.5 * ((p->ny - 1) * p->hy);
    lo[2] = p->center[2] - 0.5 * ((p->nz - 1) * p->hz);
    hi[2] = p->center[2] + 0.5 * ((p->nz - 1) * p->hz);
}

/* Vpmg_energy (vpmg.c:1248-1277) with extFlag = 1: ext[] holds the
 * energies a focusing parent left outside this domain (zero otherwise). */
/* Vpmg_qfEnergyPoint (chgm spl0), vpmg.c:1704-1789: the potential
 * interpolated trilinearly at each atom, times its charge and its partition
 * weight (Vpmg_setPart's atom rule, vpmg.c:673-720, for the domain box). */
static double qf_point(const pmgb_params *p, const Fill *f, const double *u, int natoms,
                       const double *xyz, const double *q) {
    int nx = p->nx, ny = p->ny, nz = p->nz, a, d;
    double lo[3], hi[3], energy = 0.0;
    domain_box(p, lo, hi);
    for (a = 0; a < natoms; a++) {
        const double *pos = xyz + 3 * a;
        double ok[3], part, fi, fj, fk, dx, dy, dz, uval;
        int ihi, ilo, jhi, jlo, khi, klo;
        for (d = 0; d < 3; d++) {
            if ((pos[d] < hi[d]) && (pos[d] > lo[d])) ok[d] = 1;
            else if (fabs(pos[d] - lo[d]) < VPMGSMALL) ok[d] = 1;
            else if (fabs(pos[d] - hi[d]) < VPMGSMALL) ok[d] = 1;
            else ok[d] = 0;
        }
        part = ok[0] * ok[1] * ok[2];
        fi = (pos[0] - f->xmn[0]) / p->hx;
        fj = (pos[1] - f->xmn[1]) / p->hy;
        fk = (pos[2] - f->xmn[2]) / p->hz;
        ihi = (int)ceil(fi);
        ilo = (int)floor(fi);
        jhi = (int)ceil(fj);
        jlo = (int)floor(fj);
        khi = (int)ceil(fk);
        klo = (int)floor(fk);
        if (!(part > 0)) continue;
        if (!((ihi < nx) && (jhi < ny) && (khi < nz) && (ilo >= 0) && (jlo >= 0) && (klo >= 0)))
            continue;
        dx = fi - (double)ilo;
        dy = fj - (double)jlo;
        dz = fk - (double)klo;
        uval = dx * dy * dz * u[IJK(ihi, jhi, khi)] + dx * (1.0 - dy) * dz * u[IJK(ihi, jlo, khi)] +
               dx * dy * (1.0 - dz) * u[IJK(ihi, jhi, klo)] +
               dx * (1.0 - dy) * (1.0 - dz) * u[IJK(ihi, jlo, klo)] +
               (1.0 - dx) * dy * dz * u[IJK(ilo, jhi, khi)] +
               (1.0 - dx) * (1.0 - dy) * dz * u[IJK(ilo, jlo, khi)] +
               (1.0 - dx) * dy * (1.0 - dz) * u[IJK(ilo, jhi, klo)] +
               (1.0 - dx) * (1.0 - dy) * (1.0 - dz) * u[IJK(ilo, jlo, klo)];
        energy += (uval * q[a] * part);
    }
    return energy;
}

static void energies(const pmgb_params *p, const Phys *ph, const Fill *f,
                     const double *u, const double ext[3], int natoms, const double *xyz,
                     const double *q, double *out) {
    double lo[3], hi[3], t[3];
    int full = (p->nonlin && ph->ionstr > 0.);
    domain_box(p, lo, hi);
    energy_terms(p, ph, f, u, lo, hi, 0, full, t);
    if (p->chgm == PMGB_CHGM_TRIL) t[0] = qf_point(p, f, u, natoms, xyz, q);
    t[0] += ext[0];
    if (full) {
        t[1] += ext[1];
        /* Vpmg_qmEnergyNONLIN returns before adding extQmEnergy when the
         * ionic strength term vanishes (vpmg.c:1438-1445) */
        if (!(ph->zkappa2 < VSMALL)) t[2] += ext[2];
        out[0] = t[0] - t[1] - t[2];
    } else {
        out[0] = 0.5 * t[0];
        t[1] = t[2] = 0.0;
    }
    out[7] = t[0];
    out[8] = t[1];
    out[9] = t[2];
}

/* ===================================================================== */
/* Focusing (src/mg/vpmg.c:1914-2545)                                     */
/* ===================================================================== */

/* Trilinear value of the coarse potential at (x,y,z), focusFillBound's
 * per-point body (vpmg.c:2100-2129).  Returns 0 off the coarse mesh. */
static int focus_value(const pmgb_params *pc, const double *data,
                       const double mnO[3], const double mxO[3], double x,
                       double y, double z, double *uval) {
    int nx = pc->nx, ny = pc->ny, nz = pc->nz;
    double ifl, jfl, kfl, dx, dy, dz;
    int ihi, ilo, jhi, jlo, khi, klo;
    if (!((x >= (mnO[0] - VSMALL)) && (y >= (mnO[1] - VSMALL)) &&
          (z >= (mnO[2] - VSMALL)) && (x <= (mxO[0] + VSMALL)) &&
          (y <= (mxO[1] + VSMALL)) && (z <= (mxO[2] + VSMALL))))
        return 0;
    ifl = (x - mnO[0]) / pc->hx;
    jfl = (y - mnO[1]) / pc->hy;
    kfl = (z - mnO[2]) / pc->hz;
    ihi = (int)ceil(ifl);
    if (ihi > (nx - 1)) ihi = nx - 1;
    ilo = (int)floor(ifl);
    if (ilo < 0) ilo = 0;
    jhi = (int)ceil(jfl);
    if (jhi > (ny - 1)) jhi = ny - 1;
    jlo = (int)floor(jfl);
    if (jlo < 0) jlo = 0;
    khi = (int)ceil(kfl);
    if (khi > (nz - 1)) khi = nz - 1;
    klo = (int)floor(kfl);
    if (klo < 0) klo = 0;
    dx = ifl - (double)ilo;
    dy = jfl - (double)jlo;
    dz = kfl - (double)klo;
    *uval = dx * dy * dz * data[IJK(ihi, jhi, khi)] +
            dx * (1.0 - dy) * dz * data[IJK(ihi, jlo, khi)] +
            dx * dy * (1.0 - dz) * data[IJK(ihi, jhi, klo)] +
            dx * (1.0 - dy) * (1.0 - dz) * data[IJK(ihi, jlo, klo)] +
            (1.0 - dx) * dy * dz * data[IJK(ilo, jhi, khi)] +
            (1.0 - dx) * (1.0 - dy) * dz * data[IJK(ilo, jlo, khi)] +
            (1.0 - dx) * dy * (1.0 - dz) * data[IJK(ilo, jhi, klo)] +
            (1.0 - dx) * (1.0 - dy) * (1.0 - dz) * data[IJK(ilo, jlo, klo)];
    return 1;
}

/* focusFillBound (vpmg.c:1914-2414): Dirichlet slots 0/1 of the six fine
 * faces from the coarse solution; the Neumann slots are not stored. */
static int focus_fill_bound(const pmgb_params *pc, const double *uc,
                            const pmgb_params *pf, double *gx, double *gy,
                            double *gz) {
    double mnO[3], mxO[3], mnN[3], mxN[3];
    const double hO[3] = {pc->hx, pc->hy, pc->hz}, hN[3] = {pf->hx, pf->hy, pf->hz};
    const int nO[3] = {pc->nx, pc->ny, pc->nz}, nN[3] = {pf->nx, pf->ny, pf->nz};
    int d, i, j, k, nx = pf->nx, ny = pf->ny, nz = pf->nz;
    for (d = 0; d < 3; d++) {
        mnN[d] = pf->center[d] - ((double)(nN[d] - 1) * hN[d]) / 2.0;
        mxN[d] = pf->center[d] + ((double)(nN[d] - 1) * hN[d]) / 2.0;
        mnO[d] = pc->center[d] - ((double)(nO[d] - 1) * hO[d]) / 2.0;
        mxO[d] = pc->center[d] + ((double)(nO[d] - 1) * hO[d]) / 2.0;
    }
    for (d = 0; d < 3; d++) {
        if (fabs(mnO[d] - mnN[d]) < VSMALL) mnN[d] = mnO[d];
        if (fabs(mxO[d] - mxN[d]) < VSMALL) mxN[d] = mxO[d];
    }
    for (d = 0; d < 3; d++)
        if (mxN[d] > mxO[d] || mnO[d] > mnN[d]) return 0;
    for (k = 0; k < nz; k++)
        for (j = 0; j < ny; j++) {
            double y = mnN[1] + j * hN[1], z = mnN[2] + k * hN[2];
            if (!focus_value(pc, uc, mnO, mxO, mnN[0], y, z, &gx[((size_t)0 * nz + k) * ny + j]))
                return 0;
            if (!focus_value(pc, uc, mnO, mxO, mxN[0], y, z, &gx[((size_t)1 * nz + k) * ny + j]))
                return 0;
        }
    for (k = 0; k < nz; k++)
        for (i = 0; i < nx; i++) {
            double x = mnN[0] + i * hN[0], z = mnN[2] + k * hN[2];
            if (!focus_value(pc, uc, mnO, mxO, x, mnN[1], z, &gy[((size_t)0 * nz + k) * nx + i]))
                return 0;
            if (!focus_value(pc, uc, mnO, mxO, x, mxN[1], z, &gy[((size_t)1 * nz + k) * nx + i]))
                return 0;
        }
    for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
            double x = mnN[0] + i * hN[0], y = mnN[1] + j * hN[1];
            if (!focus_value(pc, uc, mnO, mxO, x, y, mnN[2], &gz[((size_t)0 * ny + j) * nx + i]))
                return 0;
            if (!focus_value(pc, uc, mnO, mxO, x, y, mxN[2], &gz[((size_t)1 * ny + j) * nx + i]))
                return 0;
        }
    return 1;
}

/* ===================================================================== */
/* Entry points                                                           */
/* ===================================================================== */
static void fill_alloc(const pmgb_params *p, Fill *f) {
    size_t n = (size_t)p->nx * p->ny * p->nz;
    f->charge = (double *)calloc(5 * n, sizeof(double));
    f->epsx = f->charge + n;
    f->epsy = f->epsx + n;
    f->epsz = f->epsy + n;
    f->kappa = f->epsz + n;
    f->gx = (double *)calloc(2 * ((size_t)p->ny * p->nz + (size_t)p->nx * p->nz +
                                  (size_t)p->nx * p->ny), sizeof(double));
    f->gy = f->gx + 2 * (size_t)p->ny * p->nz;
    f->gz = f->gy + 2 * (size_t)p->nx * p->nz;
    f->xf = (double *)calloc((size_t)(p->nx + p->ny + p->nz), sizeof(double));
    f->yf = f->xf + p->nx;
    f->zf = f->yf + p->ny;
}

static void fill_free(Fill *f) {
    free(f->charge);
    free(f->gx);
    free(f->xf);
}

int oracle_pmg_fill(const pmgb_params *p, int natoms, const double *xyz,
                    const double *q, const double *r, double *maps,
                    double *faces) {
    Phys ph;
    Fill f;
    size_t n = (size_t)p->nx * p->ny * p->nz;
    phys_setup(p, natoms, xyz, r, &ph);
    fill_alloc(p, &f);
    do_fill(p, &ph, natoms, xyz, q, r, &f);
    if (maps) memcpy(maps, f.charge, sizeof(double) * 5 * n);
    if (faces)
        memcpy(faces, f.gx, sizeof(double) * 2 * ((size_t)p->ny * p->nz +
                                                  (size_t)p->nx * p->nz +
                                                  (size_t)p->nx * p->ny));
    fill_free(&f);
    return 1;
}

/* What a solved calculation hands to a focused child: its maps, potential
 * and physical scalars (the reference keeps them in pmgOLD). */
typedef struct {
    Phys ph;
    Fill f;
    double *u;
    double ext[3];
} Kept;

static int run_calc(const pmgb_params *p, int natoms, const double *xyz,
                    const double *q, const double *r, const double *faces_in,
                    const double ext[3], double *u, double *maps, double *faces,
                    double *out, double *reslog, int reslog_cap, Kept *keep) {
    Phys ph;
    Fill f;
    Solver s;
    int l, nx = p->nx, ny = p->ny, nz = p->nz, i, j, k, iters = 0;
    size_t n = (size_t)nx * ny * nz, t;
    double t0, t1, t2, t3, t4, errtol = (p->etol > 0.0) ? p->etol : 1.0e-6;
    double *ccf;
    memset(&s, 0, sizeof(s));
    s.reslog = reslog;
    s.reslog_cap = reslog_cap;
    t0 = now_s();
    phys_setup(p, natoms, xyz, r, &ph);
    fill_alloc(p, &f);
    t1 = now_s();
    if (p->bcfl == PMGB_BCFL_FOCUS) {
        if (!faces_in) return 0;
        memcpy(f.gx, faces_in, sizeof(double) * 2 * ((size_t)ny * nz + (size_t)nx * nz +
                                                     (size_t)nx * ny));
    }
    do_fill(p, &ph, natoms, xyz, q, r, &f);
    t2 = now_s();
    if (maps) memcpy(maps, f.charge, sizeof(double) * 5 * n);
    if (faces)
        memcpy(faces, f.gx, sizeof(double) * 2 * ((size_t)ny * nz + (size_t)nx * nz +
                                                  (size_t)nx * ny));
    /* Vpmg_solve array preparation (vpmg.c:420-448) */
    ccf = (double *)calloc(n, sizeof(double));
    if (ph.zkappa2 > VPMGSMALL)
        for (t = 0; t < n; t++) ccf[t] = ph.zkappa2 * f.kappa[t];
    /* level hierarchy (Vbuildstr, mgsubd.c:261-343) */
    s.nlev = p->nlev;
    for (l = 0; l < s.nlev; l++) {
        Level *L = &s.lev[l];
        int d;
        L->nx = (l == 0) ? nx : (s.lev[l - 1].nx - 1) / 2 + 1;
        L->ny = (l == 0) ? ny : (s.lev[l - 1].ny - 1) / 2 + 1;
        L->nz = (l == 0) ? nz : (s.lev[l - 1].nz - 1) / 2 + 1;
        L->n = (size_t)L->nx * L->ny * L->nz;
        L->nop = (l == 0) ? 4 : 14;
        for (d = 0; d < L->nop; d++) L->op[d] = (double *)calloc(L->n, sizeof(double));
        L->cc = (double *)calloc(L->n, sizeof(double));
        L->fc = (double *)calloc(L->n, sizeof(double));
        L->x = (double *)calloc(L->n, sizeof(double));
        L->w0 = (double *)calloc(L->n, sizeof(double));
        L->cp = (double *)calloc(L->n, sizeof(double));
        L->rhs = (double *)calloc(L->n, sizeof(double));
        L->xt = (double *)calloc(L->n, sizeof(double));
    }
    s.w1 = (double *)calloc(n, sizeof(double));
    s.w2 = (double *)calloc(n, sizeof(double));
    s.w3 = (double *)calloc(n, sizeof(double));
    build_fine(p, &f, ccf, &s.lev[0]);
    for (l = 1; l < s.nlev; l++) {
        build_galerkin(&s.lev[l - 1], &s.lev[l]);
        restrict_fw(&s.lev[l - 1], &s.lev[l], s.lev[l - 1].cc, s.lev[l].cc);
        restrict_fw(&s.lev[l - 1], &s.lev[l], s.lev[l - 1].fc, s.lev[l].fc);
    }
    s.mgsolv = p->nonlin ? 0 : 1;
    if (s.mgsolv == 1 && !build_band(&s, &s.lev[s.nlev - 1])) s.mgsolv = 0;
    /* solve: u = 0, then restore Dirichlet values (mgdrvd.c:462-557) */
    /* Vpmgp itmax (vpmgp.c:131), 200 unless the parameters say otherwise */
    if (!p->nonlin) {
        vcycles(&s, 0, errtol, p->itmax > 0 ? p->itmax : 200, 0, &iters);
    } else {
        iters = newton(&s, p, &ph, errtol, p->itmax > 0 ? p->itmax : 200);
    }
    t3 = now_s();
    {
        double *x = s.lev[0].x;
        /* VfboundPMG (mikpckd.c:209-256): x faces, then y, then z */
        for (k = 0; k < nz; k++)
            for (j = 0; j < ny; j++) {
                x[IJK(0, j, k)] = f.gx[((size_t)0 * nz + k) * ny + j];
                x[IJK(nx - 1, j, k)] = f.gx[((size_t)1 * nz + k) * ny + j];
            }
        for (k = 0; k < nz; k++)
            for (i = 0; i < nx; i++) {
                x[IJK(i, 0, k)] = f.gy[((size_t)0 * nz + k) * nx + i];
                x[IJK(i, ny - 1, k)] = f.gy[((size_t)1 * nz + k) * nx + i];
            }
        for (j = 0; j < ny; j++)
            for (i = 0; i < nx; i++) {
                x[IJK(i, j, 0)] = f.gz[((size_t)0 * ny + j) * nx + i];
                x[IJK(i, j, nz - 1)] = f.gz[((size_t)1 * ny + j) * nx + i];
            }
        if (u) memcpy(u, x, sizeof(double) * n);
        energies(p, &ph, &f, x, ext, natoms, xyz, q, out);
        if (keep) {
            keep->ph = ph;
            keep->f = f;
            keep->u = (double *)malloc(sizeof(double) * n);
            memcpy(keep->u, x, sizeof(double) * n);
            keep->ext[0] = ext[0];
            keep->ext[1] = ext[1];
            keep->ext[2] = ext[2];
        }
    }
    t4 = now_s();
    out[1] = (double)s.progress;
    out[2] = (double)s.reslog_n;
    out[3] = t1 - t0;
    out[4] = t2 - t1;
    out[5] = t3 - t2;
    out[6] = t4 - t3;
    out[10] = (double)iters;
    out[11] = (double)s.total_cycles;
    for (l = 0; l < s.nlev; l++) {
        Level *L = &s.lev[l];
        int d;
        for (d = 0; d < L->nop; d++) free(L->op[d]);
        free(L->cc); free(L->fc); free(L->x); free(L->w0);
        free(L->cp); free(L->rhs); free(L->xt);
    }
    free(s.w1); free(s.w2); free(s.w3); free(s.band); free(ccf);
    if (!keep) fill_free(&f);
    return 1;
}

int oracle_pmg_run(const pmgb_params *p, int natoms, const double *xyz,
                   const double *q, const double *r, double *u, double *maps,
                   double *faces, double *out, double *reslog, int reslog_cap,
                   int verbose) {
    const double zero[3] = {0.0, 0.0, 0.0};
    (void)verbose;
    if (p->bcfl == PMGB_BCFL_FOCUS) return 0; /* needs a parent: oracle_pmg_focus */
    return run_calc(p, natoms, xyz, q, r, NULL, zero, u, maps, faces, out, reslog,
                    reslog_cap, NULL);
}

/* extEnergy (vpmg.c:2416-2545) for a non-parallel chain: the coarse
 * calculation's qf/diel/qm over the complement of the fine domain, each with
 * the coarse calculation's own external terms added (extFlag = 1). */
static void ext_energy(const pmgb_params *pc, const Kept *kc,
                       const pmgb_params *pf, double ext[3]) {
    double lo[3], hi[3], t[3];
    domain_box(pf, lo, hi);
    energy_terms(pc, &kc->ph, &kc->f, kc->u, lo, hi, 1, 1, t);
    ext[0] = t[0] + kc->ext[0];
    ext[1] = t[1] + kc->ext[1];
    ext[2] = (kc->ph.zkappa2 < VSMALL) ? 0.0 : t[2] + kc->ext[2];
}

int oracle_pmg_focus(const pmgb_params *pc, const pmgb_params *pf, int natoms,
                     const double *xyz, const double *q, const double *r,
                     double *u, double *faces, double *out, double *reslog,
                     int reslog_cap, int verbose) {
    const double zero[3] = {0.0, 0.0, 0.0};
    double outc[16], ext[3], *fin;
    size_t nfaces = 2 * ((size_t)pf->ny * pf->nz + (size_t)pf->nx * pf->nz +
                         (size_t)pf->nx * pf->ny);
    Kept kc;
    int rc, nlog;
    (void)verbose;
    if (pc->bcfl == PMGB_BCFL_FOCUS || pf->bcfl != PMGB_BCFL_FOCUS) return 0;
    if (pc->chgm != PMGB_CHGM_SPL2 || pf->chgm != PMGB_CHGM_SPL2) return 0;
    memset(outc, 0, sizeof(outc));
    if (!run_calc(pc, natoms, xyz, q, r, NULL, zero, NULL, NULL, NULL, outc, reslog,
                  reslog_cap, &kc))
        return 0;
    fin = (double *)calloc(nfaces, sizeof(double));
    rc = focus_fill_bound(pc, kc.u, pf, fin, fin + 2 * (size_t)pf->ny * pf->nz,
                          fin + 2 * ((size_t)pf->ny * pf->nz + (size_t)pf->nx * pf->nz));
    if (rc) {
        ext_energy(pc, &kc, pf, ext);
        nlog = (int)outc[2];
        rc = run_calc(pf, natoms, xyz, q, r, fin, ext, u, NULL, faces, out,
                      reslog ? reslog + (nlog < reslog_cap ? nlog : reslog_cap) : NULL,
                      reslog_cap - (nlog < reslog_cap ? nlog : reslog_cap), NULL);
        out[1] += outc[1];
        out[2] += outc[2];
        out[12] = ext[0];
        out[13] = ext[1];
        out[14] = ext[2];
        out[15] = outc[0];
    }
    free(fin);
    free(kc.u);
    fill_free(&kc.f);
    return rc;
}
