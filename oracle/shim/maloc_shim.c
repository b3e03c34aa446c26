/*
 * Project-written implementation of the maloc subset declared in
 * shim/maloc/maloc.h.  TEST INFRASTRUCTURE ONLY: linked into
 * oracle/_ref/libapbsref.so together with the reference APBS sources so the
 * reference PMG path can run here as the parity checker.
 *
 * Besides memory and printing, Vnm_print records the multigrid progress
 * messages that the reference's Vprtstp (src/pmgc/mgsubd.c:507-556) emits
 * ("iteration = N", "relative residual = R") so the checker can compare
 * V-cycle counts and residual histories with the CUDA solver.
 */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "maloc/maloc.h"

/* ---------------------------------------------------------------------- */
/* Memory                                                                  */
/* ---------------------------------------------------------------------- */
static size_t g_bytes_total = 0;
static size_t g_highwater_total = 0;

Vmem *Vmem_ctor(char *name) {
    Vmem *m = (Vmem *)calloc(1, sizeof(Vmem));
    if (m && name) {
        strncpy(m->name, name, VMAX_ARGLEN - 1);
    }
    return m;
}

void Vmem_dtor(Vmem **thee) {
    if (thee && *thee) {
        free(*thee);
        *thee = NULL;
    }
}

void *Vmem_malloc(Vmem *thee, size_t num, size_t size) {
    void *p;
    if (num == 0 || size == 0) {
        return NULL;
    }
    p = calloc(num, size);
    if (p == NULL) {
        fprintf(stderr, "Vmem_malloc: out of memory (%zu x %zu)\n", num, size);
        abort();
    }
    g_bytes_total += num * size;
    if (g_bytes_total > g_highwater_total) {
        g_highwater_total = g_bytes_total;
    }
    if (thee) {
        thee->bytes += num * size;
        if (thee->bytes > thee->highwater) {
            thee->highwater = thee->bytes;
        }
    }
    return p;
}

void Vmem_free(Vmem *thee, size_t num, size_t size, void **ram) {
    if (ram == NULL || *ram == NULL) {
        return;
    }
    free(*ram);
    *ram = NULL;
    if (g_bytes_total >= num * size) {
        g_bytes_total -= num * size;
    }
    if (thee && thee->bytes >= num * size) {
        thee->bytes -= num * size;
    }
}

void *Vmem_realloc(Vmem *thee, size_t num, size_t size, void **ram,
                   size_t newNum) {
    void *p = Vmem_malloc(thee, newNum, size);
    if (ram && *ram) {
        memcpy(p, *ram, (num < newNum ? num : newNum) * size);
        Vmem_free(thee, num, size, ram);
    }
    return p;
}

size_t Vmem_bytes(Vmem *thee) { return thee ? thee->bytes : 0; }
size_t Vmem_highWater(Vmem *thee) { return thee ? thee->highwater : 0; }
size_t Vmem_bytesTotal(void) { return g_bytes_total; }
size_t Vmem_mallocBytesTotal(void) { return g_bytes_total; }
size_t Vmem_highWaterTotal(void) { return g_highwater_total; }
void Vmem_print(Vmem *thee) { (void)thee; }
void Vmem_printTotal(void) {}

/* ---------------------------------------------------------------------- */
/* Printing, progress capture, timers                                      */
/* ---------------------------------------------------------------------- */
static int g_verbose = 0;
static double *g_log = NULL;   /* relative residual of each Vprtstp call */
static int g_log_cap = 0;
static int g_log_n = 0;
static int g_iter_msgs = 0;    /* number of "iteration = N" messages */

void oracle_shim_set_log(double *buf, int cap) {
    g_log = buf;
    g_log_cap = cap;
    g_log_n = 0;
    g_iter_msgs = 0;
}

int oracle_shim_log_count(void) { return g_log_n; }
int oracle_shim_iter_count(void) { return g_iter_msgs; }
void oracle_shim_set_verbose(int v) { g_verbose = v; }

static void capture(const char *text) {
    const char *p;
    p = strstr(text, "iteration = ");
    if (p) {
        g_iter_msgs++;
    }
    p = strstr(text, "relative residual = ");
    if (p) {
        double v = atof(p + strlen("relative residual = "));
        if (g_log && g_log_n < g_log_cap) {
            g_log[g_log_n] = v;
        }
        g_log_n++;
    }
}

int Vnm_print(int unit, const char *format, ...) {
    char buf[4096];
    va_list ap;
    va_start(ap, format);
    vsnprintf(buf, sizeof(buf), format, ap);
    va_end(ap);
    capture(buf);
    if (g_verbose || unit == 2) {
        if (g_verbose > 1 || unit == 2) {
            fputs(buf, stderr);
        }
    }
    return 0;
}

int Vnm_tprint(int unit, const char *format, ...) {
    char buf[4096];
    va_list ap;
    va_start(ap, format);
    vsnprintf(buf, sizeof(buf), format, ap);
    va_end(ap);
    capture(buf);
    if (g_verbose > 1) {
        fputs(buf, stderr);
    }
    (void)unit;
    return 0;
}

void Vnm_tstart(int timer, const char *name) { (void)timer; (void)name; }
void Vnm_tstop(int timer, const char *name) { (void)timer; (void)name; }
double Vnm_epsmac(void) { return DBL_EPSILON; }
void Vnm_redirect(int flag) { (void)flag; }
int Vnm_system(char *cmd) { (void)cmd; return -1; }

/* ---------------------------------------------------------------------- */
/* Vio: "FILE" sockets opened for writing go to a stdio stream (used by    */
/* the OpenDX writer); everything else is inert                            */
/* ---------------------------------------------------------------------- */
Vio *Vio_ctor(const char *socktype, const char *datafrmt, const char *hostname,
              const char *filename, const char *rwkey) {
    Vio *v;
    FILE *fp;
    (void)datafrmt; (void)hostname;
    if (!socktype || !filename || !rwkey || strcmp(socktype, "FILE") != 0 ||
        strcmp(rwkey, "w") != 0)
        return NULL;
    fp = fopen(filename, "w");
    if (!fp) return NULL;
    v = (Vio *)calloc(1, sizeof(Vio));
    if (!v) { fclose(fp); return NULL; }
    v->fp = fp;
    return v;
}
void Vio_dtor(Vio **thee) {
    if (thee && *thee) {
        if ((*thee)->fp) fclose((FILE *)(*thee)->fp);
        free(*thee);
    }
    if (thee) *thee = NULL;
}
int Vio_scanf(Vio *thee, char *parms, ...) { (void)thee; (void)parms; return 0; }
int Vio_printf(Vio *thee, char *parms, ...) {
    va_list ap;
    int n;
    if (!thee || !thee->fp) return 0;
    va_start(ap, parms);
    n = vfprintf((FILE *)thee->fp, parms, ap);
    va_end(ap);
    return n;
}
void Vio_setWhiteChars(Vio *thee, char *w) { (void)thee; (void)w; }
void Vio_setCommChars(Vio *thee, char *c) { (void)thee; (void)c; }
int Vio_accept(Vio *thee, int nonblock) { (void)thee; (void)nonblock; return -1; }
void Vio_acceptFree(Vio *thee) { (void)thee; }
int Vio_connect(Vio *thee, int nonblock) { (void)nonblock; return (thee && thee->fp) ? 0 : -1; }
void Vio_connectFree(Vio *thee) { (void)thee; }
Vio *Vio_socketOpen(char *key, const char *iodev, const char *iofmt,
                    const char *iohost, const char *iofile) {
    (void)key; (void)iodev; (void)iofmt; (void)iohost; (void)iofile;
    return NULL;
}
void Vio_socketClose(Vio **sock) { if (sock) *sock = NULL; }
int Vio_read(Vio *thee, char *buf, int bufsize) { (void)thee; (void)buf; (void)bufsize; return -1; }
int Vio_write(Vio *thee, char *buf, int bufsize) { (void)thee; (void)buf; (void)bufsize; return -1; }
