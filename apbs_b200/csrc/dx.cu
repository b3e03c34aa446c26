// OpenDX output of grid data, as writedataMG (src/routines.c:2620-2800)
// writes it through Vgrid_writeDX (src/mg/vgrid.c:1206-1420).
//
// The file is byte for byte the reference's: four comment lines, the grid
// positions (origin and deltas in "%12.6e %12.6e %12.6e"), the connections,
// then the values in x-major order (i outer, k inner), each "%12.6e " with a
// newline after every third value, and the field trailer.  With partition
// weights, only points of positive weight are written and the origin and
// counts are those of that sub-box, as Vgrid_writeDX does with pvec.
//
// The values are formatted by several host threads at once with
// std::to_chars in scientific notation with six digits after the point,
// which rounds exactly like printf's "%12.6e", each thread on a slab of
// i, then written in order.
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "apbs_b200.h"
#include "solver_internal.cuh"

namespace {

// "%12.6e " of one value
inline char* put_value(char* p, double v) {
  char tmp[40];
  auto res = std::to_chars(tmp, tmp + sizeof(tmp), v, std::chars_format::scientific, 6);
  const int len = (int)(res.ptr - tmp);
  for (int pad = len; pad < 12; pad++) *p++ = ' ';
  std::memcpy(p, tmp, len);
  p += len;
  *p++ = ' ';
  return p;
}

}  // namespace

extern "C" int pmgb_write_dx_host(const char* path, int nx, int ny, int nz, double hx, double hy,
                                  double hz, double xmin, double ymin, double zmin,
                                  const double* data, const double* pvec, const char* title,
                                  const char* package) {
  if (!path || !data || nx < 1 || ny < 1 || nz < 1) {
    pmgb::set_error("pmgb_write_dx_host: bad arguments");
    return 0;
  }
  const size_t nxy = (size_t)nx * ny;
  auto IJK = [&](int i, int j, int k) { return (size_t)k * nxy + (size_t)j * nx + i; };
  // the points written: pvec > 0 (every point without pvec), counted per i slab
  std::vector<size_t> slab(nx + 1, 0);
  int nxP = nx, nyP = ny, nzP = nz;
  double x0 = xmin, y0 = ymin, z0 = zmin;
  if (pvec) {
    const double big = 1.0e9;  // VLARGE
    x0 = y0 = z0 = big;
    std::vector<char> anyi(nx, 0), anyj(ny, 0), anyk(nz, 0);
    for (int k = 0; k < nz; k++) {
      const double z = k * hz + zmin;
      for (int j = 0; j < ny; j++) {
        const double y = j * hy + ymin;
        for (int i = 0; i < nx; i++) {
          if (pvec[IJK(i, j, k)] > 0.0) {
            const double x = i * hx + xmin;
            if (x < x0) x0 = x;
            if (y < y0) y0 = y;
            if (z < z0) z0 = z;
            anyi[i] = anyj[j] = anyk[k] = 1;
            slab[i + 1]++;
          }
        }
      }
    }
    nxP = nyP = nzP = 0;
    for (int i = 0; i < nx; i++) nxP += anyi[i];
    for (int j = 0; j < ny; j++) nyP += anyj[j];
    for (int k = 0; k < nz; k++) nzP += anyk[k];
  } else {
    for (int i = 0; i < nx; i++) slab[i + 1] = (size_t)ny * nz;
  }
  for (int i = 0; i < nx; i++) slab[i + 1] += slab[i];
  const size_t total = slab[nx];

  FILE* fp = std::fopen(path, "w");
  if (!fp) {
    pmgb::set_error("pmgb_write_dx_host: cannot open %s", path);
    return 0;
  }
  char line[512];
  std::fprintf(fp, "# Data from %s\n", package ? package : "APBS 3.4.1");
  std::fprintf(fp, "# \n");
  std::fprintf(fp, "# %s\n", title ? title : "");
  std::fprintf(fp, "# \n");
  std::fprintf(fp, "object 1 class gridpositions counts %d %d %d\n", nxP, nyP, nzP);
  std::snprintf(line, sizeof(line), "%12.6e %12.6e %12.6e", x0, y0, z0);
  std::fprintf(fp, "origin %s\n", line);
  std::snprintf(line, sizeof(line), "%12.6e %12.6e %12.6e", hx, 0.0, 0.0);
  std::fprintf(fp, "delta %s\n", line);
  std::snprintf(line, sizeof(line), "%12.6e %12.6e %12.6e", 0.0, hy, 0.0);
  std::fprintf(fp, "delta %s\n", line);
  std::snprintf(line, sizeof(line), "%12.6e %12.6e %12.6e", 0.0, 0.0, hz);
  std::fprintf(fp, "delta %s\n", line);
  std::fprintf(fp, "object 2 class gridconnections counts %d %d %d\n", nxP, nyP, nzP);
  std::fprintf(fp, "object 3 class array type double rank 0 items %lu         data follows\n",
               (unsigned long)((long)nxP * nyP * nzP));

  // values: threads format slabs of i into their own buffers
  unsigned nthr = std::thread::hardware_concurrency();
  if (nthr < 1) nthr = 1;
  if (nthr > 32) nthr = 32;
  if ((size_t)nthr > (size_t)nx) nthr = (unsigned)nx;
  std::vector<std::string> out(nthr);
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nthr; t++) {
    pool.emplace_back([&, t]() {
      const int ia = (int)((size_t)nx * t / nthr), ib = (int)((size_t)nx * (t + 1) / nthr);
      const size_t count = slab[ib] - slab[ia];
      std::string& buf = out[t];
      buf.resize(count * 16 + count / 3 + 16);
      char* p = &buf[0];
      size_t g = slab[ia];  // index of the next value in the whole file
      for (int i = ia; i < ib; i++)
        for (int j = 0; j < ny; j++)
          for (int k = 0; k < nz; k++) {
            const size_t u = IJK(i, j, k);
            if (pvec && !(pvec[u] > 0.0)) continue;
            p = put_value(p, data[u]);
            if (++g % 3 == 0) *p++ = '\n';
          }
      buf.resize(p - &buf[0]);
    });
  }
  for (auto& th : pool) th.join();
  for (const auto& b : out) std::fwrite(b.data(), 1, b.size(), fp);
  if (total % 3 != 0) std::fputc('\n', fp);
  std::fprintf(fp, "attribute \"dep\" string \"positions\"\n");
  std::fprintf(fp, "object \"regular positions regular connections\"         class field\n");
  std::fprintf(fp, "component \"positions\" value 1\n");
  std::fprintf(fp, "component \"connections\" value 2\n");
  std::fprintf(fp, "component \"data\" value 3\n");
  const int bad = std::ferror(fp);
  if (std::fclose(fp) != 0 || bad) {
    pmgb::set_error("pmgb_write_dx_host: write to %s failed", path);
    return 0;
  }
  return 1;
}

using namespace pmgb;

// writedataMG for the maps a calculation holds: PMGB_DX_POT (u, kT/e),
// PMGB_DX_CHARGE (charge / zmagic, e), PMGB_DX_KAPPA, PMGB_DX_DIELX/Y/Z
// (Vpmg_fillArray, src/mg/vpmg.c:926-955), with the partition weights of
// the calculation.
extern "C" int pmgb_write_dx(pmgb_solver* s, int which, const char* path, const char* title,
                             const char* package) {
  if (!s || !s->filled) {
    set_error("pmgb_write_dx: no filled calculation");
    return 0;
  }
  if (which == PMGB_DX_POT && !s->solved) {
    set_error("pmgb_write_dx: the potential needs pmgb_solve first");
    return 0;
  }
  const pmgb_params& p = s->p;
  const size_t n = s->n;
  const double* src = nullptr;
  const char* deftitle = "";
  switch (which) {
    case PMGB_DX_POT: src = s->lev[0].x; deftitle = "POTENTIAL (kT/e)"; break;
    case PMGB_DX_CHARGE: src = s->charge; deftitle = "CHARGE DISTRIBUTION (e)"; break;
    case PMGB_DX_KAPPA: src = s->kappa; deftitle = "KAPPA MAP"; break;
    case PMGB_DX_DIELX: src = s->epsx; deftitle = "X-SHIFTED DIELECTRIC MAP"; break;
    case PMGB_DX_DIELY: src = s->epsy; deftitle = "Y-SHIFTED DIELECTRIC MAP"; break;
    case PMGB_DX_DIELZ: src = s->epsz; deftitle = "Z-SHIFTED DIELECTRIC MAP"; break;
    default: set_error("pmgb_write_dx: unknown map %d", which); return 0;
  }
  double* h = nullptr;
  PMGB_CUDA_OK(cudaMallocHost((void**)&h, sizeof(double) * 2 * n));
  std::vector<double> wx(p.nx), wy(p.ny), wz(p.nz);
  cudaError_t e = cudaMemcpyAsync(h, src, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(wx.data(), s->wx, sizeof(double) * p.nx, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(wy.data(), s->wy, sizeof(double) * p.ny, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(wz.data(), s->wz, sizeof(double) * p.nz, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) {
    cudaFreeHost(h);
    set_error("pmgb_write_dx: %s", cudaGetErrorString(e));
    return 0;
  }
  if (which == PMGB_DX_CHARGE)
    for (size_t q = 0; q < n; q++) h[q] = h[q] / s->zmagic;
  // pvec of Vpmg_setPart: the product of the per-axis weights
  double* pvec = h + n;
  for (int k = 0; k < p.nz; k++)
    for (int j = 0; j < p.ny; j++)
      for (int i = 0; i < p.nx; i++)
      {
        const double v = wx[i] * wy[j] * wz[k];
        pvec[((size_t)k * p.ny + j) * p.nx + i] = (fabs(v) < 1.0e-12) ? 0.0 : v;
      }
  const int ok = pmgb_write_dx_host(path, p.nx, p.ny, p.nz, p.hx, p.hy, p.hz, s->G.xmin[0],
                                    s->G.xmin[1], s->G.xmin[2], h, pvec,
                                    title ? title : deftitle, package);
  cudaFreeHost(h);
  return ok;
}
