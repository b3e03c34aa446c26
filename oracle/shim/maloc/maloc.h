/*
 * Project-written stand-in for the FETK "maloc" utility header.
 *
 * TEST INFRASTRUCTURE ONLY.  This header exists so that the reference
 * APBS C sources of the PMG solve path (src/pmgc/*.c, src/mg/vpmg.c, ...)
 * compile unchanged with gcc into oracle/_ref, where they serve as the
 * parity checker for the CUDA implementation.  It is never linked into the
 * product library.
 *
 * maloc itself (FETK, not vendored in the reference tree; fetched at
 * configure time by cmake/ImportFETK.cmake) is absent.  The reference's hot
 * path only uses a small, arithmetic-free part of it: memory management
 * (Vmem_*), printing/timers (Vnm_*), the Vio stream type (input parsing
 * only, not reached by the solve path), assertion macros and a set of
 * math/limit macros.  Those are restated here.  The numeric constants follow
 * maloc's published definitions: VSMALL 1e-9, VLARGE 1e9, VPI to 20 digits,
 * VRINT(x) = floor(x + 0.5).  Vmem_malloc zero-fills (calloc), which the PMG
 * code relies on (e.g. prolongation weights at coarse boundary points are
 * read but never written).
 */
#ifndef ORACLE_MALOC_SHIM_H
#define ORACLE_MALOC_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <stdarg.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <time.h>

#ifdef __cplusplus
#  define VEXTERNC extern "C"
#else
#  define VEXTERNC extern
#endif
#define VPUBLIC
#define VPRIVATE static
#define VNULL NULL
#define VINLINE

#define VMAX_ARGNUM 50
#define VMAX_ARGLEN 1024
#define VMAX_BUFSIZE 8192

#define VSMALL 1.0e-9
#define VLARGE 1.0e9
#define VPI 3.14159265358979323846

#define VABS(x)    ((x) >= 0 ? (x) : -(x))
#define VMIN2(x, y) ((x) <= (y) ? (x) : (y))
#define VMAX2(x, y) ((x) >= (y) ? (x) : (y))
#define VSQR(x)    ((x) * (x))
#define VSQRT(x)   (sqrt(x))
#define VEXP(x)    (exp(x))
#ifndef VLOG
#define VLOG(x)    (log(x))
#endif
#define VPOW(x, y) (pow(x, y))
#define VSIN(x)    (sin(x))
#define VCOS(x)    (cos(x))
#define VTAN(x)    (tan(x))
#define VSINH(x)   (sinh(x))
#define VCOSH(x)   (cosh(x))
#define VATAN(x)   (atan(x))
#define VATAN2(y, x) (atan2(y, x))
#define VFLOOR(x)  (floor(x))
#define VCEIL(x)   (ceil(x))
#define VRINT(x)   ((int)(floor((x) + 0.5)))
#define VEVEN(x)   (((x) & 1) == 0)
#define VODD(x)    (((x) & 1) == 1)
#define VRAND      (rand())
#define VRANDMAX   (RAND_MAX)

#define VASSERT(expr) do { if (!(expr)) { \
    fprintf(stderr, "VASSERT: %s:%d: (%s) failed\n", __FILE__, __LINE__, #expr); \
    abort(); } } while (0)
#define VWARN(expr) do { if (!(expr)) { \
    fprintf(stderr, "VWARN: %s:%d: (%s)\n", __FILE__, __LINE__, #expr); } } while (0)
#define VJMPERR1(expr) do { if (!(expr)) goto VERROR1; } while (0)
#define VJMPERR2(expr) do { if (!(expr)) goto VERROR2; } while (0)

/* ---- Vmem: calloc-backed memory accounting --------------------------- */
typedef struct sVmem {
    char name[VMAX_ARGLEN];
    size_t bytes;
    size_t highwater;
} Vmem;

VEXTERNC Vmem *Vmem_ctor(char *name);
VEXTERNC void Vmem_dtor(Vmem **thee);
VEXTERNC void *Vmem_malloc(Vmem *thee, size_t num, size_t size);
VEXTERNC void Vmem_free(Vmem *thee, size_t num, size_t size, void **ram);
VEXTERNC void *Vmem_realloc(Vmem *thee, size_t num, size_t size, void **ram,
                            size_t newNum);
VEXTERNC size_t Vmem_bytes(Vmem *thee);
VEXTERNC size_t Vmem_highWater(Vmem *thee);
VEXTERNC size_t Vmem_bytesTotal(void);
VEXTERNC size_t Vmem_mallocBytesTotal(void);
VEXTERNC size_t Vmem_highWaterTotal(void);
VEXTERNC void Vmem_print(Vmem *thee);
VEXTERNC void Vmem_printTotal(void);

/* ---- Vnm: printing, timers, machine epsilon -------------------------- */
VEXTERNC int Vnm_print(int unit, const char *format, ...);
VEXTERNC int Vnm_tprint(int unit, const char *format, ...);
VEXTERNC void Vnm_tstart(int timer, const char *name);
VEXTERNC void Vnm_tstop(int timer, const char *name);
VEXTERNC double Vnm_epsmac(void);
VEXTERNC void Vnm_redirect(int flag);
VEXTERNC int Vnm_system(char *cmd);

/* ---- Vio: byte streams.  Only "FILE" sockets opened for writing do
 * anything (the OpenDX writer, Vgrid_writeDX); the rest are inert. */
typedef struct sVio {
    void *fp;   /* FILE* of a "FILE" socket opened with "w", else NULL */
} Vio;

VEXTERNC Vio *Vio_ctor(const char *socktype, const char *datafrmt,
                       const char *hostname, const char *filename,
                       const char *rwkey);
VEXTERNC void Vio_dtor(Vio **thee);
VEXTERNC int Vio_scanf(Vio *thee, char *parms, ...);
VEXTERNC int Vio_printf(Vio *thee, char *parms, ...);
VEXTERNC void Vio_setWhiteChars(Vio *thee, char *whiteChars);
VEXTERNC void Vio_setCommChars(Vio *thee, char *commChars);
VEXTERNC int Vio_accept(Vio *thee, int nonblock);
VEXTERNC void Vio_acceptFree(Vio *thee);
VEXTERNC int Vio_connect(Vio *thee, int nonblock);
VEXTERNC void Vio_connectFree(Vio *thee);
VEXTERNC Vio *Vio_socketOpen(char *key, const char *iodev,
                             const char *iofmt, const char *iohost,
                             const char *iofile);
VEXTERNC void Vio_socketClose(Vio **sock);
VEXTERNC int Vio_read(Vio *thee, char *buf, int bufsize);
VEXTERNC int Vio_write(Vio *thee, char *buf, int bufsize);

/* ---- Vset: container type embedded (unused) in the Vacc struct ------- */
typedef struct sVset {
    void *data;
    int size;
} Vset;

/* ---- Vcom: single-rank communicator ---------------------------------- */
typedef struct sVcom {
    int mypid;
    int nproc;
} Vcom;

#endif /* ORACLE_MALOC_SHIM_H */
