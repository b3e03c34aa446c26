// FP64 multigrid kernels of the B200 PMG solver.
//
// Every kernel restates one loop nest of the reference PMG numerics
// (src/pmgc/*.c, cited per kernel).  This translation unit is compiled with
// -fmad=false and the arithmetic is written in the reference's evaluation
// order, so stencil updates round exactly as the reference's C does; only
// global sums (norms, dot products) are reassociated (tree reductions).
#include <cooperative_groups.h>

#include "gs7_rb.cuh"
#include "mg_kernels.cuh"

namespace cg = cooperative_groups;

namespace pmgb {

// ===========================================================================
// Fine-grid operator: VbuildA_fv (src/pmgc/buildAd.c:105-283)
// ===========================================================================
__global__ void k_build_fine(Grid g, const double* __restrict__ xf,
                             const double* __restrict__ yf, const double* __restrict__ zf,
                             const double* __restrict__ a1, const double* __restrict__ a2,
                             const double* __restrict__ a3, const double* __restrict__ ccf,
                             const double* __restrict__ fcf, const double* __restrict__ gx,
                             const double* __restrict__ gy, const double* __restrict__ gz,
                             double* oC, double* oE, double* oN, double* uC, double* cc,
                             double* fc) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const double hzm1 = zf[k] - zf[k - 1], hz = zf[k + 1] - zf[k];
    const double hym1 = yf[j] - yf[j - 1], hy = yf[j + 1] - yf[j];
    const double hxm1 = xf[i] - xf[i - 1], hx = xf[i + 1] - xf[i];
    const double cE = 1.0 * (hym1 + hy) * (hzm1 + hz) / (4.0 * hx);
    const double cEm = 1.0 * (hym1 + hy) * (hzm1 + hz) / (4.0 * hxm1);
    const double cN = 1.0 * (hxm1 + hx) * (hzm1 + hz) / (4.0 * hy);
    const double cNm = 1.0 * (hxm1 + hx) * (hzm1 + hz) / (4.0 * hym1);
    const double cU = 1.0 * (hxm1 + hx) * (hym1 + hy) / (4.0 * hz);
    const double cUm = 1.0 * (hxm1 + hx) * (hym1 + hy) / (4.0 * hzm1);
    const double cF = 1.0 * (hxm1 + hx) * (hym1 + hy) * (hzm1 + hz) / 8.0;
    const size_t id = g.idx(i, j, k);
    const double a1w = a1[g.idx(i - 1, j, k)], a2s = a2[g.idx(i, j - 1, k)],
                 a3d = a3[g.idx(i, j, k - 1)];
    double f = cF * fcf[id];
    cc[id] = cF * ccf[id];
    oC[id] = cE * a1[id] + cEm * a1w + cN * a2[id] + cNm * a2s + cU * a3[id] + cUm * a3d;
    int ike = (i == nx - 2) ? 0 : 1;
    oE[id] = ike * cE * a1[id];
    f += (1 - ike) * cE * a1[id] * gx[((size_t)1 * nz + k) * ny + j];
    int jke = (j == ny - 2) ? 0 : 1;
    oN[id] = jke * cN * a2[id];
    f += (1 - jke) * cN * a2[id] * gy[((size_t)1 * nz + k) * nx + i];
    int kke = (k == nz - 2) ? 0 : 1;
    uC[id] = kke * cU * a3[id];
    f += (1 - kke) * cU * a3[id] * gz[((size_t)1 * ny + j) * nx + i];
    ike = (i == 1) ? 0 : 1;
    f += (1 - ike) * cEm * a1w * gx[((size_t)0 * nz + k) * ny + j];
    jke = (j == 1) ? 0 : 1;
    f += (1 - jke) * cNm * a2s * gy[((size_t)0 * nz + k) * nx + i];
    kke = (k == 1) ? 0 : 1;
    f += (1 - kke) * cUm * a3d * gz[((size_t)0 * ny + j) * nx + i];
    fc[id] = f;
  }
}

void launch_build_fine(cudaStream_t s, Grid g, const double* xf, const double* yf,
                       const double* zf, const double* a1, const double* a2,
                       const double* a3, const double* ccf, const double* fcf,
                       const double* gx, const double* gy, const double* gz, double* oC,
                       double* oE, double* oN, double* uC, double* cc, double* fc) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  k_build_fine<<<blocks_for(nint), kThreads, 0, s>>>(g, xf, yf, zf, a1, a2, a3, ccf, fcf,
                                                      gx, gy, gz, oC, oE, oN, uC, cc, fc);
}

// ===========================================================================
// Galerkin coarse operator A_c = P^T A_f P (VbuildG_7 / VbuildG_27,
// src/pmgc/buildGd.c:450-3115) with the trilinear prolongation of
// VbuildPb_trilin (src/pmgc/buildPd.c:114-204): weight 2^-(|d|_1) at interior
// coarse points, zero at coarse boundary points.
// ===========================================================================
__device__ inline double op_entry(const Op& op, Grid g, int i, int j, int k, int dx, int dy,
                                  int dz) {
  if (dx == 0 && dy == 0 && dz == 0) return op.c[OC][g.idx(i, j, k)];
  int si = i, sj = j, sk = k;
  if (dz < 0 || (dz == 0 && dy < 0) || (dz == 0 && dy == 0 && dx < 0)) {
    si = i + dx; sj = j + dy; sk = k + dz;
    dx = -dx; dy = -dy; dz = -dz;
  }
  int code;
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
  if (code >= op.nop) return 0.0;
  return -op.c[code][g.idx(si, sj, sk)];
}

// Register-only form: with alpha = a - 2I (the fine point's offset in the
// support of coarse point I) and d the stencil offset of A, the product
// wa(alpha) A(a, a+d) reaches coarse target I + e with the trilinear weight
// W(v, e) = prod_axis w(v - 2e), v = alpha + d in [-2, 2]^3 (w(0) = 1,
// w(+-1) = 1/2, else 0).  Products are first summed per v (125 bins), then
// each bin is spread to its <= 8 targets.  Every index is a compile-time
// constant after unrolling, so the 27 accumulators stay in registers.
__device__ __forceinline__ double wtl(int v) { return v == 0 ? 1.0 : ((v == 1 || v == -1) ? 0.5 : 0.0); }

template <int NOP>
__device__ __forceinline__ double op_entry_static(const Op& op, Grid g, int i, int j, int k,
                                                  int dx, int dy, int dz) {
  // same lookup as op_entry with (dx, dy, dz) known at compile time
  if (dx == 0 && dy == 0 && dz == 0) return op.c[OC][g.idx(i, j, k)];
  int si = i, sj = j, sk = k;
  if (dz < 0 || (dz == 0 && dy < 0) || (dz == 0 && dy == 0 && dx < 0)) {
    si = i + dx; sj = j + dy; sk = k + dz;
    dx = -dx; dy = -dy; dz = -dz;
  }
  int code;
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
  if (code >= NOP) return 0.0;
  return -op.c[code][g.idx(si, sj, sk)];
}

template <int NOP>
__global__ void __launch_bounds__(128) k_galerkin(Grid gf, Op fine, Grid gc,
                                                  double* const* __restrict__ coarse_ptrs) {
  const int nx = gc.nx, ny = gc.ny, nz = gc.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int I, J, K;
    interior_ijk(q, nx, ny, I, J, K);
    // couplings to coarse boundary points are zero (P vanishes there)
    const bool okx[3] = {I - 1 >= 1, true, I + 1 <= nx - 2};
    const bool oky[3] = {J - 1 >= 1, true, J + 1 <= ny - 2};
    const bool okz[3] = {K - 1 >= 1, true, K + 1 <= nz - 2};
    double acc[27];
#pragma unroll
    for (int t = 0; t < 27; t++) acc[t] = 0.0;
#pragma unroll
    for (int vz = -2; vz <= 2; vz++)
#pragma unroll
      for (int vy = -2; vy <= 2; vy++)
#pragma unroll
        for (int vx = -2; vx <= 2; vx++) {
          double bin = 0.0;
#pragma unroll
          for (int az = -1; az <= 1; az++)
#pragma unroll
            for (int ay = -1; ay <= 1; ay++)
#pragma unroll
              for (int ax = -1; ax <= 1; ax++) {
                const int dx = vx - ax, dy = vy - ay, dz = vz - az;
                if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) continue;
                if (NOP == 4 && (abs(dx) + abs(dy) + abs(dz)) > 1) continue;
                const int fi = 2 * I + ax, fj = 2 * J + ay, fk = 2 * K + az;
                const double wa = wtl(ax) * wtl(ay) * wtl(az);
                bin += wa * op_entry_static<NOP>(fine, gf, fi, fj, fk, dx, dy, dz);
              }
#pragma unroll
          for (int ez = -1; ez <= 1; ez++)
#pragma unroll
            for (int ey = -1; ey <= 1; ey++)
#pragma unroll
              for (int ex = -1; ex <= 1; ex++) {
                const double w = wtl(vx - 2 * ex) * wtl(vy - 2 * ey) * wtl(vz - 2 * ez);
                if (w == 0.0) continue;
                if (okx[ex + 1] && oky[ey + 1] && okz[ez + 1])
                  acc[((ez + 1) * 3 + (ey + 1)) * 3 + (ex + 1)] += w * bin;
              }
        }
    double* coarse[14];
#pragma unroll
    for (int c = 0; c < 14; c++) coarse[c] = coarse_ptrs[c];
    const size_t id = gc.idx(I, J, K);
#define ACC(dx, dy, dz) acc[(((dz) + 1) * 3 + ((dy) + 1)) * 3 + ((dx) + 1)]
    coarse[OC][id] = ACC(0, 0, 0);
    coarse[OE][id] = -ACC(1, 0, 0);
    coarse[ON][id] = -ACC(0, 1, 0);
    coarse[UC][id] = -ACC(0, 0, 1);
    coarse[ONE][id] = -ACC(1, 1, 0);
    coarse[ONW][id] = -ACC(-1, 1, 0);
    coarse[UE][id] = -ACC(1, 0, 1);
    coarse[UW][id] = -ACC(-1, 0, 1);
    coarse[UN][id] = -ACC(0, 1, 1);
    coarse[US][id] = -ACC(0, -1, 1);
    coarse[UNE][id] = -ACC(1, 1, 1);
    coarse[UNW][id] = -ACC(-1, 1, 1);
    coarse[USE][id] = -ACC(1, -1, 1);
    coarse[USW][id] = -ACC(-1, -1, 1);
#undef ACC
  }
}

void launch_galerkin(cudaStream_t s, Grid gf, Op fine, Grid gc, double* const* coarse_dev) {
  size_t nint = (size_t)(gc.nx - 2) * (gc.ny - 2) * (gc.nz - 2);
  if (fine.nop == 4)
    k_galerkin<4><<<blocks_for(nint, 128), 128, 0, s>>>(gf, fine, gc, coarse_dev);
  else
    k_galerkin<14><<<blocks_for(nint, 128), 128, 0, s>>>(gf, fine, gc, coarse_dev);
}

// ===========================================================================
// Restriction, Vrestrc2 (src/pmgc/matvecd.c:801-911): interior coarse points
// only; the output boundary is zero.
// ===========================================================================
__global__ void k_restrict(Grid gf, const double* __restrict__ xin, Grid gc, double* xout) {
  const int cx = gc.nx, cy = gc.ny, cz = gc.nz;
  const size_t n = gc.n();
  const double h = 0.5, qq = 0.25, e = 0.125;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    split3(q, cx, cy, i, j, k);
    if (i == 0 || j == 0 || k == 0 || i == cx - 1 || j == cy - 1 || k == cz - 1) {
      xout[q] = 0.0;
      continue;
    }
    const int ii = 2 * i, jj = 2 * j, kk = 2 * k;
#define XI(a, b, c) xin[gf.idx(a, b, c)]
    const double tO = +1.0 * XI(ii, jj, kk) + h * XI(ii, jj + 1, kk) + h * XI(ii, jj - 1, kk) +
                      h * XI(ii + 1, jj, kk) + h * XI(ii - 1, jj, kk) +
                      qq * XI(ii + 1, jj + 1, kk) + qq * XI(ii - 1, jj + 1, kk) +
                      qq * XI(ii + 1, jj - 1, kk) + qq * XI(ii - 1, jj - 1, kk);
    const double tU = +h * XI(ii, jj, kk + 1) + qq * XI(ii, jj + 1, kk + 1) +
                      qq * XI(ii, jj - 1, kk + 1) + qq * XI(ii + 1, jj, kk + 1) +
                      qq * XI(ii - 1, jj, kk + 1) + e * XI(ii + 1, jj + 1, kk + 1) +
                      e * XI(ii - 1, jj + 1, kk + 1) + e * XI(ii + 1, jj - 1, kk + 1) +
                      e * XI(ii - 1, jj - 1, kk + 1);
    const double tD = +h * XI(ii, jj, kk - 1) + qq * XI(ii, jj + 1, kk - 1) +
                      qq * XI(ii, jj - 1, kk - 1) + qq * XI(ii + 1, jj, kk - 1) +
                      qq * XI(ii - 1, jj, kk - 1) + e * XI(ii + 1, jj + 1, kk - 1) +
                      e * XI(ii - 1, jj + 1, kk - 1) + e * XI(ii + 1, jj - 1, kk - 1) +
                      e * XI(ii - 1, jj - 1, kk - 1);
#undef XI
    xout[q] = tO + tU + tD;
  }
}

void launch_restrict(cudaStream_t s, Grid gf, const double* xin, Grid gc, double* xout) {
  k_restrict<<<blocks_for(gc.n()), kThreads, 0, s>>>(gf, xin, gc, xout);
}

// ===========================================================================
// Interpolation + damped coarse-grid correction:
//   w = VinterpPMG2(x_c) (src/pmgc/matvecd.c:935-1074), x_f += xdamp * w
// with xdamp = <x_c, w0_c> / <x_c, A_c x_c> (src/pmgc/mgcsd.c:465-485).
// Interior fine points only (Vxaxpy touches interior points).
// ===========================================================================
// One thread per coarse cell (ii..ii+1, jj..jj+1, kk..kk+1): its eight corner
// values, read once, give the up to eight fine interior points 2ii+oi,
// 2jj+oj, 2kk+ok of the cell, each with the reference's expression for its
// parity case -- bitwise the per-point evaluation with an eighth of its loads
// and index arithmetic.
__global__ void k_interp_axpy(Grid gc, const double* __restrict__ xc, Grid gf, double* xf,
                              const double* num, const double* den) {
  const double xdamp = num[0] / den[0];
  const double h = 0.5, qq = 0.25, e = 0.125;
  const int cx = gc.nx - 1, cy = gc.ny - 1, cz = gc.nz - 1;
  const size_t ncell = (size_t)cx * cy * cz;
  const size_t sy = gc.nx, sz = (size_t)gc.nx * gc.ny;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < ncell;
       q += (size_t)gridDim.x * blockDim.x) {
    int ii, jj, kk;
    split3(q, cx, cy, ii, jj, kk);
    const size_t c0 = gc.idx(ii, jj, kk);
    const double x000 = xc[c0], x100 = xc[c0 + 1], x010 = xc[c0 + sy], x110 = xc[c0 + sy + 1];
    const double x001 = xc[c0 + sz], x101 = xc[c0 + sz + 1], x011 = xc[c0 + sz + sy];
    const double x111 = xc[c0 + sz + sy + 1];
#pragma unroll
    for (int ok = 0; ok < 2; ok++) {
      const int k = 2 * kk + ok;
      if (k < 1 || k > gf.nz - 2) continue;
#pragma unroll
      for (int oj = 0; oj < 2; oj++) {
        const int j = 2 * jj + oj;
        if (j < 1 || j > gf.ny - 2) continue;
#pragma unroll
        for (int oi = 0; oi < 2; oi++) {
          const int i = 2 * ii + oi;
          if (i < 1 || i > gf.nx - 2) continue;
          double w;
          if (!oi && !oj && !ok) {
            w = x000;
          } else if (oi && !oj && !ok) {
            w = h * x000 + h * x100;
          } else if (!oi && oj && !ok) {
            w = h * x000 + h * x010;
          } else if (!oi && !oj && ok) {
            w = h * x000 + h * x001;
          } else if (oi && oj && !ok) {
            w = qq * x000 + qq * x100 + qq * x010 + qq * x110;
          } else if (oi && !oj && ok) {
            w = qq * x000 + qq * x100 + qq * x001 + qq * x101;
          } else if (!oi && oj && ok) {
            w = qq * x000 + qq * x010 + qq * x001 + qq * x011;
          } else {
            w = +e * x000 + e * x100 + e * x010 + e * x110 + e * x001 + e * x101 + e * x011 +
                e * x111;
          }
          const size_t id = gf.idx(i, j, k);
          xf[id] += xdamp * w;
        }
      }
    }
  }
}

void launch_interp_axpy(cudaStream_t s, Grid gc, const double* xc, Grid gf, double* xf,
                        const double* num, const double* den) {
  const size_t ncell = (size_t)(gc.nx - 1) * (gc.ny - 1) * (gc.nz - 1);
  k_interp_axpy<<<blocks_for(ncell), kThreads, 0, s>>>(gc, xc, gf, xf, num, den);
}

// ===========================================================================
// Stencil bodies in the reference's evaluation order
// ===========================================================================
// 7-point neighbour sum of Vgsrb7x / Vmresid7_1s (gsd.c:127-135,
// matvecd.c:480-488), starting from f.
__device__ __forceinline__ double sum7(const Op& op, Grid g, const double* x, size_t id,
                                       double f) {
  const size_t sx = 1, sy = g.nx, sz = (size_t)g.nx * g.ny;
  return f + op.c[ON][id] * x[id + sy] + op.c[ON][id - sy] * x[id - sy] +
         op.c[OE][id] * x[id + sx] + op.c[OE][id - sx] * x[id - sx] +
         op.c[UC][id - sz] * x[id - sz] + op.c[UC][id] * x[id + sz];
}

// tmpO + tmpU + tmpD of Vgsrb27x / Vmresid27_1s (gsd.c:249-282).
template <bool CG>
__device__ __forceinline__ void sum27(const Op& op, Grid g, const double* x, size_t id,
                                      double& tO, double& tU, double& tD) {
  const size_t sy = g.nx, sz = (size_t)g.nx * g.ny;
  auto X = [&](size_t p) -> double { return CG ? __ldcg(x + p) : x[p]; };
  const double* const* c = op.c;
  tO = +c[ON][id] * X(id + sy) + c[ON][id - sy] * X(id - sy) + c[OE][id] * X(id + 1) +
       c[OE][id - 1] * X(id - 1) + c[ONE][id] * X(id + sy + 1) +
       c[ONW][id] * X(id + sy - 1) + c[ONW][id - sy + 1] * X(id - sy + 1) +
       c[ONE][id - sy - 1] * X(id - sy - 1);
  tU = +c[UC][id] * X(id + sz) + c[UN][id] * X(id + sz + sy) + c[US][id] * X(id + sz - sy) +
       c[UE][id] * X(id + sz + 1) + c[UW][id] * X(id + sz - 1) +
       c[UNE][id] * X(id + sz + sy + 1) + c[UNW][id] * X(id + sz + sy - 1) +
       c[USE][id] * X(id + sz - sy + 1) + c[USW][id] * X(id + sz - sy - 1);
  tD = +c[UC][id - sz] * X(id - sz) + c[US][id - sz + sy] * X(id - sz + sy) +
       c[UN][id - sz - sy] * X(id - sz - sy) + c[UW][id - sz + 1] * X(id - sz + 1) +
       c[UE][id - sz - 1] * X(id - sz - 1) + c[USW][id - sz + sy + 1] * X(id - sz + sy + 1) +
       c[USE][id - sz + sy - 1] * X(id - sz + sy - 1) +
       c[UNW][id - sz - sy + 1] * X(id - sz - sy + 1) +
       c[UNE][id - sz - sy - 1] * X(id - sz - sy - 1);
}

// ===========================================================================
// 7-point red-black half-sweep, Vgsrb7x (src/pmgc/gsd.c:95-164).  All points
// of one colour are independent (7-point neighbours have the other colour).
// parity = (i+j+k)%2 of the colour updated (0-based indices).
// ===========================================================================
__global__ void k_gs7_colour(Grid g, Op op, const double* __restrict__ cc,
                             const double* __restrict__ fc, double* x, int parity) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int hr = (nx - 1) / 2;  // colour slots per row
  const size_t nslots = (size_t)hr * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nslots;
       q += (size_t)gridDim.x * blockDim.x) {
    int m, j, k;
    split3(q, hr, ny - 2, m, j, k);
    j += 1;
    k += 1;
    const int i = 1 + (((1 + j + k) & 1) != parity) + 2 * m;
    if (i > nx - 2) continue;
    const size_t id = g.idx(i, j, k);
    x[id] = sum7(op, g, x, id, fc[id]) / (op.c[OC][id] + cc[id]);
  }
}

int g_tune[16] = {2, 6, 0, 0, 0, 0, 0, 0, 70000, 0, 2, 2, 0x12, 0, 0, 0};

int launch_gs7_sweep64(cudaStream_t s, Grid g, Op op, const double* diag, const double* fc,
                       const double* xin, double* xout, int first_parity, int kchunk,
                       int shape) {
  Gs7Rb<double> a;
  a.oE = op.c[OE]; a.oN = op.c[ON]; a.uC = op.c[UC];
  a.D = diag; a.f = fc; a.xin = xin; a.xout = xout;
  a.nx = g.nx; a.S = g.nx * g.ny; a.nz = g.nz;
  a.kchunk = kchunk;  // 0: sized to the resident CTA slots
  return launch_gs7_rb<double>(s, a, first_parity, shape) == cudaSuccess;
}

int gs7_sweep_supported(Grid g) {
  return (g.nx & 1) && (g.ny & 1) && (double)g.n() * sizeof(double) < 2147483647.0;
}

// D = oC + cc on interior points (the FP64 sum the smoother divides by),
// 1 on boundary points (the single-pass sweep's boundary update is then 0/1)
__global__ void k_diag(Grid g, const double* __restrict__ oC, const double* __restrict__ cc,
                       double* D) {
  const size_t n = g.n();
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    split3(q, g.nx, g.ny, i, j, k);
    const bool inner = i > 0 && i < g.nx - 1 && j > 0 && j < g.ny - 1 && k > 0 && k < g.nz - 1;
    D[q] = inner ? oC[q] + cc[q] : 1.0;
  }
}

void launch_diag(cudaStream_t s, Grid g, const double* oC, const double* cc, double* D) {
  k_diag<<<blocks_for(g.n()), kThreads, 0, s>>>(g, oC, cc, D);
}

void launch_gs7_colour(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                       double* x, int parity) {
  size_t nslots = (size_t)((g.nx - 1) / 2) * (g.ny - 2) * (g.nz - 2);
  k_gs7_colour<<<blocks_for(nslots), kThreads, 0, s>>>(g, op, cc, fc, x, parity);
}

// ===========================================================================
// Residual and matrix-vector product (src/pmgc/matvecd.c:98-228, 461-594)
// ===========================================================================
__global__ void k_resid(Grid g, Op op, const double* __restrict__ cc,
                        const double* __restrict__ fc, const double* __restrict__ x, double* r) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const size_t id = g.idx(i, j, k);
    if (op.nop == 4) {
      r[id] = sum7(op, g, x, id, fc[id]) - (op.c[OC][id] + cc[id]) * x[id];
    } else {
      double tO, tU, tD;
      sum27<false>(op, g, x, id, tO, tU, tD);
      r[id] = fc[id] + tO + tU + tD - (op.c[OC][id] + cc[id]) * x[id];
    }
  }
}

void launch_resid(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                  const double* x, double* r) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  k_resid<<<blocks_for(nint), kThreads, 0, s>>>(g, op, cc, fc, x, r);
}

__global__ void k_matvec(Grid g, Op op, const double* __restrict__ cc,
                         const double* __restrict__ x, double* y) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  const size_t sx = 1, sy = nx, sz = (size_t)nx * ny;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const size_t id = g.idx(i, j, k);
    if (op.nop == 4) {
      y[id] = -op.c[ON][id] * x[id + sy] - op.c[ON][id - sy] * x[id - sy] -
              op.c[OE][id] * x[id + sx] - op.c[OE][id - sx] * x[id - sx] -
              op.c[UC][id - sz] * x[id - sz] - op.c[UC][id] * x[id + sz] +
              (op.c[OC][id] + cc[id]) * x[id];
    } else {
      // Vmatvec27_1s accumulates -a*x terms; (-a)*x == -(a*x) exactly.
      double tO, tU, tD;
      sum27<false>(op, g, x, id, tO, tU, tD);
      y[id] = -tO - tU - tD + (op.c[OC][id] + cc[id]) * x[id];
    }
  }
}

void launch_matvec(cudaStream_t s, Grid g, Op op, const double* cc, const double* x, double* y) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  k_matvec<<<blocks_for(nint), kThreads, 0, s>>>(g, op, cc, x, y);
}

// The two sums of the coarse-correction damping, <x, w0> and <x, (A + cc) x>
// (Vmatvec and the two Vxdot of mgcsd.c:465-485), in one pass with A x formed
// on the fly and never stored.  Each block writes its two partial sums; the
// block that finishes last (a ticket on *done, reset by that block) adds
// them in block order and writes num and den, so the result does not depend
// on which block is last.
constexpr int kDampThreads = 256;
__global__ void __launch_bounds__(kDampThreads)
    k_xdamp_sums(Grid g, Op op, const double* __restrict__ cc, const double* __restrict__ x,
                 const double* __restrict__ w0, double* part, unsigned* done, double* num,
                 double* den) {
  __shared__ double sh[32];
  __shared__ bool last;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  double a0 = 0.0, a1 = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const size_t id = g.idx(i, j, k);
    double ax;
    if (op.nop == 4) {
      const size_t sy = nx, sz = (size_t)nx * ny;
      ax = -op.c[ON][id] * x[id + sy] - op.c[ON][id - sy] * x[id - sy] -
           op.c[OE][id] * x[id + 1] - op.c[OE][id - 1] * x[id - 1] -
           op.c[UC][id - sz] * x[id - sz] - op.c[UC][id] * x[id + sz] +
           (op.c[OC][id] + cc[id]) * x[id];
    } else {
      double tO, tU, tD;
      sum27<false>(op, g, x, id, tO, tU, tD);
      ax = -tO - tU - tD + (op.c[OC][id] + cc[id]) * x[id];
    }
    a0 += x[id] * w0[id];
    a1 += x[id] * ax;
  }
  const double s0 = block_sum<kDampThreads>(a0, sh);
  const double s1 = block_sum<kDampThreads>(a1, sh);
  const int nb = gridDim.x;
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s0;
    part[nb + blockIdx.x] = s1;
    __threadfence();
    last = atomicAdd(done, 1u) == (unsigned)nb - 1u;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double b0 = 0.0, b1 = 0.0;
  for (int t = threadIdx.x; t < nb; t += blockDim.x) {
    b0 += __ldcg(part + t);
    b1 += __ldcg(part + nb + t);
  }
  const double n0 = block_sum<kDampThreads>(b0, sh);
  const double d0 = block_sum<kDampThreads>(b1, sh);
  if (threadIdx.x == 0) {
    num[0] = n0;
    den[0] = d0;
    *done = 0u;
  }
}

void launch_xdamp_sums(cudaStream_t s, Grid g, Op op, const double* cc, const double* x,
                       const double* w0, double* part, unsigned* done, double* num,
                       double* den) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  const int nb = (int)reduce_parts(nint);
  k_xdamp_sums<<<nb, kDampThreads, 0, s>>>(g, op, cc, x, w0, part, done, num, den);
}

// ===========================================================================
// Ordered 27-point Gauss-Seidel, Vgsrb27x (src/pmgc/gsd.c:167-340).
//
// The reference visits each colour lexicographically (k, then j, then i)
// and the 12 same-colour edge neighbours make later points read updated
// values.  Rows (j,k) with equal t = j + 2k have no dependence on each other
// and every earlier neighbour lies on a smaller t, so each half-sweep is a
// sequence of wavefronts.  Successive half-sweeps are pipelined with a lag
// of 4 wavefronts (an opposite-colour neighbour lies at most 3 wavefronts
// ahead), and the optional residual follows 4 wavefronts behind the last
// half-sweep.  One CTA cluster runs all steps; a cluster barrier separates
// steps, so every value a step reads was written in an earlier step.
// ===========================================================================
constexpr int kWaveLag = 4;

struct WavePhase {
  int t;          // wavefront of this phase at the current step
  int parity;     // colour (i+j+k)%2; -1 = residual (all points)
};

template <int CLUSTER>
__global__ void k_gs27_wave(Grid g, Op op, const double* __restrict__ cc,
                            const double* __restrict__ fc, double* x, double* r, int nhalf,
                            int first_parity, int do_resid) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tmin = 1 + 2 * 1, tmax = (ny - 2) + 2 * (nz - 2);
  const int nphase = nhalf + (do_resid ? 1 : 0);
  const int resid_lag = kWaveLag * (nhalf - 1) + 4;
  const int last_start = do_resid ? resid_lag : kWaveLag * (nhalf - 1);
  const int nsteps = (tmax - tmin + 1) + last_start;
  const int hr = (nx - 1) / 2;
  unsigned rank = 0;
  if (CLUSTER > 1) rank = cg::this_cluster().block_rank();
  const int gtid = rank * blockDim.x + threadIdx.x;
  const int nthr = CLUSTER * blockDim.x;
  for (int s = 0; s < nsteps; s++) {
    // enumerate (phase, row, slot) work items of this step
    int count[5], klo[5], tph[5];
    int total = 0;
    for (int ph = 0; ph < nphase; ph++) {
      const int lag = (ph < nhalf) ? kWaveLag * ph : resid_lag;
      const int t = tmin + s - lag;
      tph[ph] = t;
      count[ph] = 0;
      klo[ph] = 0;
      if (t < tmin || t > tmax) continue;
      // j = t - 2k in [1, ny-2], k in [1, nz-2]
      int kl = (t - (ny - 2) + 1) / 2;
      if (t - (ny - 2) > 0 && ((t - (ny - 2)) & 1)) kl = (t - (ny - 2) + 1) / 2;
      if (kl < 1) kl = 1;
      while (t - 2 * kl > ny - 2) kl++;
      int kh = (t - 1) / 2;
      if (kh > nz - 2) kh = nz - 2;
      if (kh < kl) continue;
      const int slots = (ph < nhalf) ? hr : (nx - 2);
      klo[ph] = kl;
      count[ph] = (kh - kl + 1) * slots;
      total += count[ph];
    }
    for (int item = gtid; item < total; item += nthr) {
      int ph = 0, rem = item;
      while (rem >= count[ph]) {
        rem -= count[ph];
        ph++;
      }
      const int slots = (ph < nhalf) ? hr : (nx - 2);
      const int k = klo[ph] + rem / slots;
      const int j = tph[ph] - 2 * k;
      const int m = rem % slots;
      if (ph < nhalf) {
        const int parity = (first_parity + ph) & 1;
        const int i = 1 + (((1 + j + k) & 1) != parity) + 2 * m;
        if (i > nx - 2) continue;
        const size_t id = g.idx(i, j, k);
        double tO, tU, tD;
        sum27<true>(op, g, x, id, tO, tU, tD);
        __stcg(x + id, (fc[id] + (tO + tU + tD)) / (op.c[OC][id] + cc[id]));
      } else {
        const int i = 1 + m;
        const size_t id = g.idx(i, j, k);
        double tO, tU, tD;
        sum27<true>(op, g, x, id, tO, tU, tD);
        r[id] = fc[id] + tO + tU + tD - (op.c[OC][id] + cc[id]) * __ldcg(x + id);
      }
    }
    if (CLUSTER > 1) {
      cg::this_cluster().sync();
    } else {
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// The same wavefront schedule with one CTA per interior plane k, synchronised
// point to point instead of by a barrier over all CTAs.
//
// A step's items on plane k read values of planes k-1, k and k+1 only; each
// CTA publishes the number of steps it has finished in a counter.  Successive
// half-sweeps run wlag wavefronts apart (wlag >= 4; the residual wlag after
// the last).  A point of half-sweep p reads, on the lower plane, values of
// half-sweep p written one wavefront earlier, and on the upper plane values
// of half-sweep p-1 written up to wlag-3 wavefronts earlier; so a CTA may
// start step s once the lower neighbour has finished step s-1 and the upper
// one step s-wlag+3.  Every value a step reads was written in an earlier
// step, and no value is overwritten before the step that reads it (a
// neighbour that would overwrite it waits for this plane first): the
// iterates are bitwise those of k_gs27_wave whatever the lag, and with wlag
// above 4 a plane may run ahead of the plane above it, so the planes
// pipeline instead of moving in lockstep.  tests/test_gs27_wave_deps.py
// checks both claims on adversarial interleavings.  Spreading the planes
// over up to all SMs (one CTA each, a cooperative launch so that all are
// resident together) divides the per-step work that bounds the one-cluster
// kernel by the number of planes.
//
// The counters of a level are never reset between launches: every CTA of a
// launch finishes all steps (after a wait that ran out it records the
// failure in *err and stops waiting), so at the start of a launch all
// counters of the level are equal and each CTA takes its own as the base.
// Differences are taken modulo 2^32.
// ---------------------------------------------------------------------------
constexpr long long kWaveWaitNs = 200LL * 1000 * 1000;  // 200 ms per wait

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Coefficients of one point's 27-point update in the order sum27 reads them.
struct Coef27 {
  double o[8], u[9], d[9], f, oc, cc;
};
__device__ __forceinline__ void load_coef27(const Op& op, const double* __restrict__ cc,
                                            const double* __restrict__ fc, size_t id, size_t sy,
                                            size_t sz, Coef27& C) {
  const double* const* c = op.c;
  C.o[0] = c[ON][id]; C.o[1] = c[ON][id - sy]; C.o[2] = c[OE][id]; C.o[3] = c[OE][id - 1];
  C.o[4] = c[ONE][id]; C.o[5] = c[ONW][id]; C.o[6] = c[ONW][id - sy + 1];
  C.o[7] = c[ONE][id - sy - 1];
  C.u[0] = c[UC][id]; C.u[1] = c[UN][id]; C.u[2] = c[US][id]; C.u[3] = c[UE][id];
  C.u[4] = c[UW][id]; C.u[5] = c[UNE][id]; C.u[6] = c[UNW][id]; C.u[7] = c[USE][id];
  C.u[8] = c[USW][id];
  C.d[0] = c[UC][id - sz]; C.d[1] = c[US][id - sz + sy]; C.d[2] = c[UN][id - sz - sy];
  C.d[3] = c[UW][id - sz + 1]; C.d[4] = c[UE][id - sz - 1]; C.d[5] = c[USW][id - sz + sy + 1];
  C.d[6] = c[USE][id - sz + sy - 1]; C.d[7] = c[UNW][id - sz - sy + 1];
  C.d[8] = c[UNE][id - sz - sy - 1];
  C.f = fc[id]; C.oc = c[OC][id]; C.cc = cc[id];
}
// tmpO, tmpU, tmpD of sum27<true> from prefetched coefficients: the same
// products added in the same order.
__device__ __forceinline__ void sum27_pre(const Coef27& C, const double* x, size_t id,
                                          size_t sy, size_t sz, double& tO, double& tU,
                                          double& tD) {
  auto X = [&](size_t p) -> double { return __ldcg(x + p); };
  tO = +C.o[0] * X(id + sy) + C.o[1] * X(id - sy) + C.o[2] * X(id + 1) +
       C.o[3] * X(id - 1) + C.o[4] * X(id + sy + 1) + C.o[5] * X(id + sy - 1) +
       C.o[6] * X(id - sy + 1) + C.o[7] * X(id - sy - 1);
  tU = +C.u[0] * X(id + sz) + C.u[1] * X(id + sz + sy) + C.u[2] * X(id + sz - sy) +
       C.u[3] * X(id + sz + 1) + C.u[4] * X(id + sz - 1) + C.u[5] * X(id + sz + sy + 1) +
       C.u[6] * X(id + sz + sy - 1) + C.u[7] * X(id + sz - sy + 1) +
       C.u[8] * X(id + sz - sy - 1);
  tD = +C.d[0] * X(id - sz) + C.d[1] * X(id - sz + sy) + C.d[2] * X(id - sz - sy) +
       C.d[3] * X(id - sz + 1) + C.d[4] * X(id - sz - 1) + C.d[5] * X(id - sz + sy + 1) +
       C.d[6] * X(id - sz + sy - 1) + C.d[7] * X(id - sz - sy + 1) +
       C.d[8] * X(id - sz - sy - 1);
}

constexpr int kPlanesThreads = 384;  // a step's items never exceed the CTA

template <bool POLL_ALL>
__global__ void __launch_bounds__(kPlanesThreads, 1)
    k_gs27_planes(Grid g, Op op, const double* __restrict__ cc, const double* __restrict__ fc,
                  double* x, double* r, int nhalf, int first_parity, int do_resid,
                  unsigned* counters, int* err, int wlag) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t sy = nx, sz = (size_t)nx * ny;
  const int tmin = 1 + 2 * 1, tmax = (ny - 2) + 2 * (nz - 2);
  const int nphase = nhalf + (do_resid ? 1 : 0);
  const int resid_lag = wlag * nhalf;
  const int last_start = do_resid ? resid_lag : wlag * (nhalf - 1);
  const int nsteps = (tmax - tmin + 1) + last_start;
  const int hr = (nx - 1) / 2;
  const int c = blockIdx.x, k = 1 + c;  // this CTA's plane
  const int ncta = gridDim.x;
  __shared__ unsigned base_sh;
  __shared__ volatile int failed_sh;
  if (threadIdx.x == 0) {
    base_sh = counters[c];
    failed_sh = 0;
  }
  __syncthreads();
  const unsigned base = base_sh;
  // this thread's item of step s: the point id, 0 = none, 1 = GS update,
  // 2 = residual (every item of a step is one thread's: blockDim covers them)
  auto item_of = [&](int s, size_t& id) -> int {
    int m = threadIdx.x;
    for (int ph = 0; ph < nphase; ph++) {
      const int lag = (ph < nhalf) ? wlag * ph : resid_lag;
      const int t = tmin + s - lag;
      const int j = t - 2 * k;
      if (t < tmin || t > tmax || j < 1 || j > ny - 2) continue;
      const int cnt = (ph < nhalf) ? hr : (nx - 2);
      if (m >= cnt) {
        m -= cnt;
        continue;
      }
      if (ph < nhalf) {
        const int parity = (first_parity + ph) & 1;
        const int i = 1 + (((1 + j + k) & 1) != parity) + 2 * m;
        if (i > nx - 2) return 0;
        id = g.idx(i, j, k);
        return 1;
      }
      id = g.idx(1 + m, j, k);
      return 2;
    }
    return 0;
  };
  size_t id = 0;
  int kind = (nsteps > 0) ? item_of(0, id) : 0;
  Coef27 C;
  if (kind) load_coef27(op, cc, fc, id, sy, sz, C);
  volatile int* verr = err;
  // waits for the lower neighbour plane to finish step s-1 and the upper
  // one step s-wlag+3 (every thread or only thread 0); the last counter
  // value seen of each is kept, so a neighbour known to be far enough ahead
  // costs no read; once any CTA has given up, nobody waits any more
  unsigned seen[2] = {base, base};
  auto wait_neighbours = [&](int s) {
    const unsigned long long t0 = global_ns();
    for (int side = 0; side < 2; side++) {
      const int nb = side == 0 ? c - 1 : c + 1;
      if (nb < 0 || nb >= ncta) continue;
      const unsigned need = base + (unsigned)(side == 0 ? s : s - wlag + 4);
      if ((int)(seen[side] - need) >= 0) continue;
      const unsigned* f = counters + nb;
      for (;;) {
        seen[side] = ld_acquire(f);
        if ((int)(seen[side] - need) >= 0) break;
        if (failed_sh || *verr) {
          failed_sh = 1;
          return;
        }
        if ((long long)(global_ns() - t0) > kWaveWaitNs) {
          failed_sh = 1;
          atomicAdd(err, 1);
          return;
        }
      }
    }
  };
  for (int s = 0; s < nsteps; s++) {
    if (s > 0) {
      if (POLL_ALL) {
        if (!failed_sh) wait_neighbours(s);
      } else {
        if (threadIdx.x == 0 && !failed_sh) wait_neighbours(s);
        __syncthreads();
      }
    }
    if (kind) {
      double tO, tU, tD;
      sum27_pre(C, x, id, sy, sz, tO, tU, tD);
      if (kind == 1) {
        __stcg(x + id, (C.f + (tO + tU + tD)) / (C.oc + C.cc));
      } else {
        r[id] = C.f + tO + tU + tD - (C.oc + C.cc) * __ldcg(x + id);
      }
    }
    // the next step's coefficients do not depend on this step: fetch them
    // while the neighbour planes finish.  Thread 0 publishes the step, and a
    // release waits for the thread's own loads, so it fetches after that.
    size_t nid = 0;
    const int nkind = (s + 1 < nsteps) ? item_of(s + 1, nid) : 0;
    if (nkind && threadIdx.x != 0) load_coef27(op, cc, fc, nid, sy, sz, C);
    __syncthreads();
    if (threadIdx.x == 0) {
      st_release(counters + c, base + (unsigned)(s + 1));
      if (nkind) load_coef27(op, cc, fc, nid, sy, sz, C);
    }
    kind = nkind;
    id = nid;
  }
}

int wave_planes_fit(Grid g) {
  static const int capacity = [] {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs27_planes<false>, kPlanesThreads,
                                                      0) != cudaSuccess)
      per_sm = 0;
    return sms * per_sm;
  }();
  const int planes = g.nz - 2;
  const int items = 4 * ((g.nx - 1) / 2) + (g.nx - 2);  // two sweeps + residual
  return planes >= 2 && planes <= kWavePlanesMax && planes <= capacity &&
         items <= kPlanesThreads;
}

int launch_gs27_planes(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                       double* x, double* r, int nsweep, int first_parity, unsigned* counters,
                       int* err, int poll_all, int wlag) {
  int nhalf = 2 * nsweep;
  int do_resid = (r != nullptr) ? 1 : 0;
  const int hr = (g.nx - 1) / 2;
  const int items = nhalf * hr + (do_resid ? g.nx - 2 : 0);
  if (items > kPlanesThreads) return 0;
  const int threads = std::max(64, (items + 31) / 32 * 32);
  if (wlag < 4) wlag = 4;
  void* args[] = {&g, &op, &cc, &fc, &x, &r,   &nhalf, &first_parity,
                  &do_resid, &counters, &err, &wlag};
  void* fn = poll_all ? (void*)k_gs27_planes<true> : (void*)k_gs27_planes<false>;
  return cudaLaunchCooperativeKernel(fn, dim3(g.nz - 2), dim3(threads), args, 0, s) ==
         cudaSuccess;
}

// ---------------------------------------------------------------------------
// The same schedule, one CTA per interior plane, with the CTA's plane and its
// two neighbour planes held in shared memory and every update passed to the
// neighbour planes through a mailbox in global memory instead of by step
// counters.
//
// The GS update of point (i, j, k) in half-sweep q goes into the CTA's own
// copy and into mailbox slot (k, q, j, m) as two 64-bit words, each holding
// one 32-bit half of the value beside the launch's tag.  A reader polls the
// slot until both tags are the launch's: the value validates itself, so no
// fence and no counter lies between one plane's update and the neighbour's
// use of it.  Every slot is written once per launch, so nothing is
// overwritten before it is read, and the tags of earlier launches never
// match.
//
// A CTA copies a neighbour's updates into its copy of that plane at the step
// that first needs them: half-sweep q at row j takes row j+1 of the lower
// plane's half-sweep q (finished one wavefront earlier) and row j+1 of the
// upper plane's half-sweep q-1 (finished wlag-3 wavefronts earlier), and at
// j = 1 row 1 of both too.  The rows a step reads then hold exactly the
// values the sequential order reads (the lower plane swept by this
// half-sweep, the upper one by the earlier ones), and the rows a step
// changes lie at least two rows from those any other half-sweep reads in
// that step or the one before, so one block barrier per step orders
// everything.  The iterates are bitwise those of k_gs27_wave whatever the
// order in which the planes run; tests/test_gs27_wave_deps.py runs this rule
// on adversarial interleavings.
//
// The counters hold the launch count of each plane (the tag is that plus
// one); a CTA writes its plane back to x at the end, after both neighbours
// have read theirs (with two or more half-sweeps a CTA waits on both
// neighbours' updates before it finishes).  A wait that runs out is counted
// in *err like the counter kernel's.
// ---------------------------------------------------------------------------
constexpr int kMailThreads = 384;
constexpr int kMailPoll = 2;     // mailbox slots one thread polls per step, at most
constexpr int kMailHalfMax = 4;  // half-sweeps per launch the mailbox holds

__device__ __forceinline__ void mail_put(unsigned long long* p, double v, unsigned tag) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  const unsigned long long hi = (unsigned long long)tag << 32;
  asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p),
               "l"((b & 0xffffffffull) | hi), "l"((b >> 32) | hi)
               : "memory");
}
__device__ __forceinline__ void mail_load(const unsigned long long* p, unsigned long long& w0,
                                          unsigned long long& w1) {
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(w0), "=l"(w1) : "l"(p));
}

size_t mail_words(Grid g) {
  const size_t hr = (g.nx - 1) / 2;
  return 2 * (size_t)(g.nz - 2) * kMailHalfMax * (g.ny - 2) * hr;
}
// shared memory of k_gs27_mail: three planes, each row split by the parity
// of i into two runs of (nx + 1) / 2 values
static size_t mail_smem(Grid g) {
  return 3 * (size_t)2 * ((g.nx + 1) / 2) * g.ny * sizeof(double);
}

__global__ void __launch_bounds__(kMailThreads, 1)
    k_gs27_mail(Grid g, Op op, const double* __restrict__ cc, const double* __restrict__ fc,
                double* x, double* r, int nhalf, int first_parity, int do_resid,
                unsigned* counters, int* err, int wlag, unsigned long long* mail) {
  // planes k-1, k, k+1 of x; each row as its even-i values then its odd-i
  // values, so the points one warp updates (one colour of a row) and each of
  // their stencil neighbours lie contiguously: two shared-memory wavefronts
  // per warp load instead of four
  extern __shared__ double pl[];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int pn = nx * ny;
  const int H = (nx + 1) / 2;
  const int ps = 2 * H * ny;  // doubles per plane in shared memory
  auto sidx = [&](int i, int j) -> int { return (2 * j + (i & 1)) * H + (i >> 1); };
  const size_t sy = nx, sz = (size_t)pn;
  const int tmin = 1 + 2 * 1, tmax = (ny - 2) + 2 * (nz - 2);
  const int nphase = nhalf + (do_resid ? 1 : 0);
  const int resid_lag = wlag * nhalf;
  const int last_start = do_resid ? resid_lag : wlag * (nhalf - 1);
  const int nsteps = (tmax - tmin + 1) + last_start;
  const int hr = (nx - 1) / 2;
  const int c = blockIdx.x, k = 1 + c;
  const int ncta = gridDim.x;
  double* P0 = pl;
  double* P1 = pl + ps;
  double* P2 = pl + 2 * ps;
  __shared__ unsigned tag_sh;
  __shared__ volatile int failed_sh;
  if (threadIdx.x == 0) {
    tag_sh = counters[c] + 1u;
    failed_sh = 0;
  }
  {
    // the three planes are contiguous in x; asynchronous 8-byte copies keep
    // all of them in flight at once
    const double* src = x + (size_t)(k - 1) * pn;
    for (int e = threadIdx.x; e < 3 * pn; e += blockDim.x) {
      const int p3 = e / pn, e2 = e - p3 * pn;
      const int jj = e2 / nx, ii = e2 - jj * nx;
      const unsigned dst = (unsigned)__cvta_generic_to_shared(pl + p3 * ps + sidx(ii, jj));
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src + e)
                   : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  }
  __syncthreads();
  const unsigned tag = tag_sh;
  auto slot = [&](int plane_c, int q, int j, int m) -> unsigned long long* {
    return mail + 2 * ((((size_t)plane_c * nhalf + q) * (ny - 2) + (j - 1)) * hr + m);
  };
  auto colour_i = [&](int j, int kk, int q, int m) -> int {
    const int parity = (first_parity + q) & 1;
    return 1 + (((1 + j + kk) & 1) != parity) + 2 * m;
  };
  // this thread's item: a fixed half-sweep (or the residual) and slot --
  // threads [q hr, (q+1) hr) sweep half-sweep q, slot tid - q hr, threads
  // from nhalf hr on the residual, point tid - nhalf hr -- at the row the
  // step reaches: 0 = none, 1 = GS update, 2 = residual; j, i and, for a GS
  // update, the slot m
  const int iq = (int)threadIdx.x < nhalf * hr ? (int)threadIdx.x / hr : nhalf;
  const int im = (int)threadIdx.x - iq * hr;
  const bool iworker = iq < nhalf || (do_resid && im < nx - 2);
  const int ilag = (iq < nhalf) ? wlag * iq : resid_lag;
  auto item_of = [&](int s, int& j, int& i, int& q, int& m) -> int {
    if (!iworker) return 0;
    const int t = tmin + s - ilag;
    const int jj = t - 2 * k;
    if (t < tmin || t > tmax || jj < 1 || jj > ny - 2) return 0;
    j = jj;
    q = iq;
    m = im;
    if (iq < nhalf) {
      i = colour_i(jj, k, iq, im);
      return (i > nx - 2) ? 0 : 1;
    }
    i = 1 + im;
    return 2;
  };
  // the mailbox slots this thread polls: thread group G = tid / hr takes the
  // lower plane's half-sweep G (G < nhalf) or the upper plane's half-sweep
  // G - nhalf, slot tid % hr, of row j+1 and, at j = 1, of row 1 too
  const int grp = threadIdx.x / hr, gm = threadIdx.x - grp * hr;
  const int pside = grp < nhalf ? 0 : 1;
  const int pq = grp - pside * nhalf;
  const int pph = pside == 0 ? pq : pq + 1;
  const int pnb = pside == 0 ? c - 1 : c + 1;
  const bool poller = grp < 2 * nhalf && pnb >= 0 && pnb < ncta && pph < nphase;
  const int plag = (pph < nhalf) ? wlag * pph : resid_lag;
  const unsigned long long* pp[kMailPoll];
  double* dp[kMailPoll];
  auto polls_of = [&](int s) -> unsigned {
    unsigned pend = 0;
    pp[0] = pp[1] = nullptr;
    dp[0] = dp[1] = nullptr;
    if (!poller) return 0;
    const int t = tmin + s - plag;
    const int j = t - 2 * k;
    if (t < tmin || t > tmax || j < 1 || j > ny - 2) return 0;
#pragma unroll
    for (int pass = 0; pass < kMailPoll; pass++) {
      const int jj = pass == 0 ? j + 1 : 1;
      if (pass == 0 ? (jj > ny - 2) : (j != 1)) continue;
      const int i = colour_i(jj, k - 1 + 2 * pside, pq, gm);
      if (i > nx - 2) continue;
      pp[pass] = slot(pnb, pq, jj, gm);
      dp[pass] = (pside == 0 ? P0 : P2) + sidx(i, jj);
      pend |= 1u << pass;
    }
    return pend;
  };
  volatile int* verr = err;
  unsigned long long w[kMailPoll][2];
  auto issue = [&](unsigned pend) {
#pragma unroll
    for (int n = 0; n < kMailPoll; n++)
      if (pend & (1u << n)) mail_load(pp[n], w[n][0], w[n][1]);
  };
  int j = 0, i = 0, q = 0, m = 0;
  int kind = (nsteps > 0) ? item_of(0, j, i, q, m) : 0;
  Coef27 C;
  if (kind) load_coef27(op, cc, fc, g.idx(i, j, k), sy, sz, C);
  // A step's polls are issued one step early, right after the previous
  // step's barrier, so that their round trip overlaps that step's update:
  // a slot that is already written then costs no wait at all.  (A plane's
  // own loop -- poll round trip plus update -- sets the period of the plane
  // below every other, and so of the whole wavefront.)
  unsigned pend = (nsteps > 0) ? polls_of(0) : 0u;
  issue(pend);
  for (int s = 0; s < nsteps; s++) {
    if (pend) {
      const unsigned long long t0 = global_ns();
      int spins = 0;
      for (;;) {
#pragma unroll
        for (int n = 0; n < kMailPoll; n++) {
          if ((pend & (1u << n)) && (unsigned)(w[n][0] >> 32) == tag &&
              (unsigned)(w[n][1] >> 32) == tag) {
            *dp[n] =
                __longlong_as_double((long long)((w[n][1] << 32) | (w[n][0] & 0xffffffffull)));
            pend &= ~(1u << n);
          }
        }
        if (!pend) break;
        if ((++spins & 15) == 0) {
          if (failed_sh || *verr) {
            failed_sh = 1;
            break;
          }
          if ((long long)(global_ns() - t0) > kWaveWaitNs) {
            failed_sh = 1;
            atomicAdd(err, 1);
            break;
          }
        }
        issue(pend);
      }
    }
    __syncthreads();
    // the next step's polls go out now (the slots they fill are rows no
    // update of this step reads, and they are copied in only after it)
    pend = (s + 1 < nsteps) ? polls_of(s + 1) : 0u;
    issue(pend);
    if (kind) {
      // the nine in-plane positions of the stencil (C: centre, N/S: j+-1,
      // E/W: i+-1)
      // (i +- 1 has the other parity: its run starts H further or H back,
      // and its index in the run is i >> 1 or one less, plus the parity of i)
      const int p = i & 1;
      const int oC = sidx(i, j), oN = oC + 2 * H, oS = oC - 2 * H;
      const int oE = oC + (1 - 2 * p) * H + p, oW = oE - 1;
      const int oNE = oE + 2 * H, oNW = oW + 2 * H;
      const int oSE = oE - 2 * H, oSW = oW - 2 * H;
      const double tO = +C.o[0] * P1[oN] + C.o[1] * P1[oS] + C.o[2] * P1[oE] +
                        C.o[3] * P1[oW] + C.o[4] * P1[oNE] + C.o[5] * P1[oNW] +
                        C.o[6] * P1[oSE] + C.o[7] * P1[oSW];
      const double tU = +C.u[0] * P2[oC] + C.u[1] * P2[oN] + C.u[2] * P2[oS] +
                        C.u[3] * P2[oE] + C.u[4] * P2[oW] + C.u[5] * P2[oNE] +
                        C.u[6] * P2[oNW] + C.u[7] * P2[oSE] + C.u[8] * P2[oSW];
      const double tD = +C.d[0] * P0[oC] + C.d[1] * P0[oN] + C.d[2] * P0[oS] +
                        C.d[3] * P0[oE] + C.d[4] * P0[oW] + C.d[5] * P0[oNE] +
                        C.d[6] * P0[oNW] + C.d[7] * P0[oSE] + C.d[8] * P0[oSW];
      if (kind == 1) {
        const double v = (C.f + (tO + tU + tD)) / (C.oc + C.cc);
        P1[oC] = v;
        mail_put(slot(c, q, j, m), v, tag);
      } else {
        r[g.idx(i, j, k)] = C.f + tO + tU + tD - (C.oc + C.cc) * P1[oC];
      }
    }
    // the next step's coefficients do not depend on this step: fetch them
    // while the neighbour planes finish
    const int nkind = (s + 1 < nsteps) ? item_of(s + 1, j, i, q, m) : 0;
    if (nkind) load_coef27(op, cc, fc, g.idx(i, j, k), sy, sz, C);
    kind = nkind;
  }
  __syncthreads();
  double* dst = x + (size_t)k * pn;
  for (int e = threadIdx.x; e < pn; e += blockDim.x) {
    const int jj = e / nx, ii = e - jj * nx;
    if (jj >= 1 && jj <= ny - 2 && ii >= 1 && ii <= nx - 2) __stcg(dst + e, P1[sidx(ii, jj)]);
  }
  if (threadIdx.x == 0) counters[c] = tag;
}

int wave_mail_fit(Grid g) {
  static int dev_smem = -1, sms = 0;
  if (dev_smem < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const int planes = g.nz - 2;
  const int hr = (g.nx - 1) / 2;
  const int items = kMailHalfMax * hr + (g.nx - 2);
  const int pollers = 2 * kMailHalfMax * hr;
  const size_t smem = mail_smem(g);
  return planes >= 2 && planes <= kWavePlanesMax && planes <= sms && items <= kMailThreads &&
         pollers <= kMailThreads && smem + 1024 <= (size_t)dev_smem;
}

int launch_gs27_mail(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                     double* x, double* r, int nsweep, int first_parity, unsigned* counters,
                     int* err, int wlag, unsigned long long* mail) {
  int nhalf = 2 * nsweep;
  int do_resid = (r != nullptr) ? 1 : 0;
  if (!mail || nhalf < 2 || nhalf > kMailHalfMax || !wave_mail_fit(g)) return 0;
  const int hr = (g.nx - 1) / 2;
  const int items = nhalf * hr + (do_resid ? g.nx - 2 : 0);
  int threads = std::max(items, 2 * nhalf * hr);
  threads = std::max(64, (threads + 31) / 32 * 32);
  if (threads > kMailThreads) return 0;
  const size_t smem = mail_smem(g);
  static size_t smem_set = 0;
  if (smem > smem_set) {
    if (cudaFuncSetAttribute(k_gs27_mail, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return 0;
    smem_set = smem;
  }
  int per_sm = 0, sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs27_mail, threads, smem) !=
          cudaSuccess ||
      per_sm * sms < g.nz - 2)
    return 0;
  if (wlag < 4) wlag = 4;
  void* args[] = {&g, &op, &cc, &fc, &x, &r, &nhalf, &first_parity, &do_resid,
                  &counters, &err, &wlag, &mail};
  return cudaLaunchCooperativeKernel((void*)k_gs27_mail, dim3(g.nz - 2), dim3(threads), args,
                                     smem, s) == cudaSuccess;
}

int mg_init() {
  cudaError_t e = cudaFuncSetAttribute(k_gs27_wave<16>,
                                       cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return 8;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(16, 1, 1);
  cfg.blockDim = dim3(512, 1, 1);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 16;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int nclusters = 0;
  e = cudaOccupancyMaxActiveClusters(&nclusters, k_gs27_wave<16>, &cfg);
  if (e != cudaSuccess || nclusters < 1) {
    cudaGetLastError();
    return 8;
  }
  return 16;
}

int launch_gs27_wave(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                     double* x, double* r, int nsweep, int first_parity, Gs27Plan plan) {
  const int nhalf = 2 * nsweep;
  const int do_resid = (r != nullptr) ? 1 : 0;
  if (plan.cluster <= 1) {
    k_gs27_wave<1><<<1, plan.threads, 0, s>>>(g, op, cc, fc, x, r, nhalf, first_parity,
                                               do_resid);
    return cudaGetLastError() == cudaSuccess;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(plan.cluster, 1, 1);
  cfg.blockDim = dim3(plan.threads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = plan.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e;
  switch (plan.cluster) {
    case 2:
      e = cudaLaunchKernelEx(&cfg, k_gs27_wave<2>, g, op, cc, fc, x, r, nhalf, first_parity,
                             do_resid);
      break;
    case 4:
      e = cudaLaunchKernelEx(&cfg, k_gs27_wave<4>, g, op, cc, fc, x, r, nhalf, first_parity,
                             do_resid);
      break;
    case 8:
      e = cudaLaunchKernelEx(&cfg, k_gs27_wave<8>, g, op, cc, fc, x, r, nhalf, first_parity,
                             do_resid);
      break;
    case 16:
      e = cudaLaunchKernelEx(&cfg, k_gs27_wave<16>, g, op, cc, fc, x, r, nhalf, first_parity,
                             do_resid);
      break;
    default:
      return 0;
  }
  return e == cudaSuccess;
}

// ===========================================================================
// BLAS-1 (src/pmgc/mikpckd.c:57-328) on interior points
// ===========================================================================
__global__ void k_zero(double* x, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x)
    x[q] = 0.0;
}
void launch_zero(cudaStream_t s, double* x, size_t n) {
  k_zero<<<blocks_for(n), kThreads, 0, s>>>(x, n);
}

__global__ void k_copy_interior(Grid g, const double* __restrict__ x, double* y) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const size_t id = g.idx(i, j, k);
    y[id] = x[id];
  }
}
void launch_copy_interior(cudaStream_t s, Grid g, const double* x, double* y) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  k_copy_interior<<<blocks_for(nint), kThreads, 0, s>>>(g, x, y);
}

__global__ void k_axpy_interior(Grid g, const double* a_dev, double a_host,
                                const double* __restrict__ x, double* y) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  const double a = a_dev ? a_dev[0] : a_host;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const size_t id = g.idx(i, j, k);
    y[id] += a * x[id];
  }
}
void launch_axpy_interior(cudaStream_t s, Grid g, const double* a_dev, double a_host,
                          const double* x, double* y) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  k_axpy_interior<<<blocks_for(nint), kThreads, 0, s>>>(g, a_dev, a_host, x, y);
}

// Two-pass deterministic reductions over interior points.
constexpr int kRedThreads = 256;
size_t reduce_parts(size_t n) {
  size_t b = (n + kRedThreads * 4 - 1) / (kRedThreads * 4);
  if (b > 1184) b = 1184;
  if (b < 1) b = 1;
  return b;
}

template <int MODE>  // 0: sum |x|, 1: sum x*y
__global__ void k_reduce_partial(Grid g, const double* __restrict__ x,
                                 const double* __restrict__ y, double* part) {
  __shared__ double sh[32];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  double acc = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const size_t id = g.idx(i, j, k);
    acc += (MODE == 0) ? fabs(x[id]) : x[id] * y[id];
  }
  double t = block_sum<kRedThreads>(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_reduce_final(const double* __restrict__ part, int nparts, double* out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[i];
  double t = block_sum<kRedThreads>(acc, sh);
  if (threadIdx.x == 0) out[0] = t;
}

void launch_nrm1(cudaStream_t s, Grid g, const double* x, double* part, double* out_dev) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  int nb = (int)reduce_parts(nint);
  k_reduce_partial<0><<<nb, kRedThreads, 0, s>>>(g, x, nullptr, part);
  k_reduce_final<<<1, kRedThreads, 0, s>>>(part, nb, out_dev);
}

void launch_dot(cudaStream_t s, Grid g, const double* x, const double* y, double* part,
                double* out_dev) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  int nb = (int)reduce_parts(nint);
  k_reduce_partial<1><<<nb, kRedThreads, 0, s>>>(g, x, y, part);
  k_reduce_final<<<1, kRedThreads, 0, s>>>(part, nb, out_dev);
}

// ===========================================================================
// Coarsest direct solve (LPBE): band storage of Vbuildband1_27
// (src/pmgc/buildBd.c:183-306), Cholesky factor R^T R of the band (the
// factorisation of Vdpbfa, src/pmgc/mlinpckd.c:194-233, computed
// right-looking) and the two triangular solves of Vdpbsl (mlinpckd.c:57-83).
// The band holds oC without the Helmholtz term and the diagonal couplings
// exactly as the reference writes them.
// ===========================================================================
__global__ void k_band_build(Grid g, Op op, double* abd, int m, int lda) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int ex = nx - 2, exy = (nx - 2) * (ny - 2);
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    double* col = abd + q * (size_t)lda;  // column jj = q+1
    // abd(kk, jj) with kk = off + m + 1 (1-based) -> col[off + m]
    auto put = [&](int off, double v) { col[off + m] = v; };
    const double* const* c = op.c;
    put(0, c[OC][g.idx(i, j, k)]);
    put(-1, -c[OE][g.idx(i - 1, j, k)]);
    put(-ex, -c[ON][g.idx(i, j - 1, k)]);
    put(-ex + 1, -c[ONE][g.idx(i, j - 1, k)]);
    put(-ex - 1, -c[ONW][g.idx(i, j - 1, k)]);
    put(-exy, -c[UC][g.idx(i, j, k - 1)]);
    put(-exy + 1, -c[UE][g.idx(i, j, k - 1)]);
    put(-exy - 1, -c[UW][g.idx(i, j, k - 1)]);
    put(-exy + ex, -c[UN][g.idx(i, j, k - 1)]);
    put(-exy - ex, -c[US][g.idx(i, j, k - 1)]);
    put(-exy + ex + 1, -c[UNE][g.idx(i, j, k - 1)]);
    put(-exy + ex - 1, -c[UNW][g.idx(i, j, k - 1)]);
    put(-exy - ex + 1, -c[USE][g.idx(i, j, k - 1)]);
    put(-exy - ex - 1, -c[USW][g.idx(i, j, k - 1)]);
  }
}

void launch_band_build(cudaStream_t s, Grid g, Op op, double* abd, int m, int lda) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  cudaMemsetAsync(abd, 0, sizeof(double) * (size_t)lda * nint, s);
  k_band_build<<<blocks_for(nint), kThreads, 0, s>>>(g, op, abd, m, lda);
}

// A(i,l) for 1-based i <= l, l - i <= m lives at abd[(l-1)*lda + (m + i - l)].
__global__ void __launch_bounds__(1024) k_band_factor(double* abd, int n, int m, int lda,
                                                      int* info) {
  __shared__ double rjj;
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int j = 1; j <= n; j++) {
    if (threadIdx.x == 0) {
      double d = abd[(size_t)(j - 1) * lda + m];
      if (!(d > 0.0)) {
        bad = j;
      } else {
        rjj = sqrt(d);
        abd[(size_t)(j - 1) * lda + m] = rjj;
      }
    }
    __syncthreads();
    if (bad) break;
    const int lend = (j + m < n) ? j + m : n;
    // R(j,l) = A(j,l) / R(j,j)
    for (int l = j + 1 + threadIdx.x; l <= lend; l += blockDim.x)
      abd[(size_t)(l - 1) * lda + (m + j - l)] /= rjj;
    __syncthreads();
    // A(i,l) -= R(j,i) R(j,l), j < i <= l <= j+m
    const int w = lend - j;
    const int tri = w * (w + 1) / 2;
    for (int t = threadIdx.x; t < tri; t += blockDim.x) {
      // map t -> (a, b) with 0 <= a <= b < w
      int b = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
      while ((b + 1) * (b + 2) / 2 <= t) b++;
      while (b * (b + 1) / 2 > t) b--;
      const int a = t - b * (b + 1) / 2;
      const int i = j + 1 + a, l = j + 1 + b;
      const double rji = abd[(size_t)(i - 1) * lda + (m + j - i)];
      const double rjl = abd[(size_t)(l - 1) * lda + (m + j - l)];
      abd[(size_t)(l - 1) * lda + (m + i - l)] -= rji * rjl;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) info[0] = bad;
}

void launch_band_factor(cudaStream_t s, double* abd, int n, int m, int lda, int* info) {
  k_band_factor<<<1, 1024, 0, s>>>(abd, n, m, lda, info);
}

// Forward and backward substitution with one warp; y in shared memory when
// it fits, else in the output vector.
__global__ void k_band_solve(Grid g, const double* __restrict__ abd, int n, int m, int lda,
                             const double* __restrict__ rhs, double* x, double* work) {
  // gather interior of rhs (Vxcopy_small) into work
  const int nx = g.nx, ny = g.ny;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const int i = 1 + q % (nx - 2);
    const int j = 1 + (q / (nx - 2)) % (ny - 2);
    const int k = 1 + q / ((nx - 2) * (ny - 2));
    work[q] = rhs[g.idx(i, j, k)];
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    // R^T y = b
    for (int k = 1; k <= n; k++) {
      const int lm = (k - 1 < m) ? k - 1 : m;
      const double* colk = abd + (size_t)(k - 1) * lda;
      double t = 0.0;
      for (int l = lane; l < lm; l += 32) t += colk[m - lm + l] * work[k - 1 - lm + l];
      t = warp_sum(t);
      if (lane == 0) work[k - 1] = (work[k - 1] - t) / colk[m];
      __syncwarp();
    }
    // R x = y
    for (int k = n; k >= 1; k--) {
      const int lm = (k - 1 < m) ? k - 1 : m;
      const double* colk = abd + (size_t)(k - 1) * lda;
      double bk = 0.0;
      if (lane == 0) {
        bk = work[k - 1] / colk[m];
        work[k - 1] = bk;
      }
      bk = __shfl_sync(0xffffffffu, bk, 0);
      const double tneg = -bk;
      for (int l = lane; l < lm; l += 32) work[k - 1 - lm + l] += tneg * colk[m - lm + l];
      __syncwarp();
    }
  }
  __syncthreads();
  // scatter (Vxcopy_large); boundary stays zero
  for (size_t q = threadIdx.x; q < g.n(); q += blockDim.x) x[q] = 0.0;
  __syncthreads();
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const int i = 1 + q % (nx - 2);
    const int j = 1 + (q / (nx - 2)) % (ny - 2);
    const int k = 1 + q / ((nx - 2) * (ny - 2));
    x[g.idx(i, j, k)] = work[q];
  }
}

void launch_band_solve(cudaStream_t s, Grid g, const double* abd, int n, int m, int lda,
                       const double* rhs, double* x) {
  // work vector: n doubles after the band storage is the caller's job; use
  // the tail of x's level as scratch is not safe, so the solver passes a
  // dedicated buffer via the band pointer layout (see solver.cu).
  double* work = const_cast<double*>(abd) + (size_t)lda * n;
  k_band_solve<<<1, 256, 0, s>>>(g, abd, n, m, lda, rhs, x, work);
}

// ===========================================================================
// Coarsest CG (NPBE), Vcghs (src/pmgc/cgd.c:57-123): r = f - A x (x = 0),
// then at most itmax Hestenes-Stiefel iterations stopping when
// ||r||_2 / ||f||_2 <= errtol; the direction update is p = beta (p + r/beta)
// as the reference writes it (Vxaxpy then Vxscal).  One cluster runs every
// iteration; cluster-wide sums go through distributed shared memory in rank
// order so all CTAs see identical scalars.
// ===========================================================================
template <int CLUSTER>
__device__ double cluster_sum(double v, double* sh, double* slots, int phase) {
  // block sum
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) b += sh[w];
    slots[phase] = b;
  }
  if (CLUSTER > 1) {
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    double tot = 0.0;
    for (int rnk = 0; rnk < CLUSTER; rnk++) {
      double* remote = cl.map_shared_rank(slots, rnk);
      tot += remote[phase];
    }
    return tot;
  } else {
    __syncthreads();
    return slots[phase];
  }
}

template <int CLUSTER>
__global__ void k_cg_coarse(Grid g, Op op, const double* __restrict__ cc,
                            const double* __restrict__ fc, double* x, double* r, double* p,
                            double* ap, int itmax, double errtol, int* iters_out) {
  __shared__ double sh[32];
  __shared__ double slots[8];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int nint = (nx - 2) * (ny - 2) * (nz - 2);
  unsigned rank = 0;
  if (CLUSTER > 1) rank = cg::this_cluster().block_rank();
  const int gtid = rank * blockDim.x + threadIdx.x;
  const int nthr = CLUSTER * blockDim.x;
  auto pid = [&](int q) {
    const int i = 1 + q % (nx - 2);
    const int j = 1 + (q / (nx - 2)) % (ny - 2);
    const int k = 1 + q / ((nx - 2) * (ny - 2));
    return g.idx(i, j, k);
  };
  auto csync = [&]() {
    if (CLUSTER > 1) cg::this_cluster().sync();
    else __syncthreads();
  };
  int phase = 0;
  // r = f - (A + cc) x   (x = 0 on entry)
  double acc = 0.0;
  for (int q = gtid; q < nint; q += nthr) {
    const size_t id = pid(q);
    double tO, tU, tD;
    sum27<true>(op, g, x, id, tO, tU, tD);
    const double rv = fc[id] + tO + tU + tD - (op.c[OC][id] + cc[id]) * __ldcg(x + id);
    __stcg(r + id, rv);
    acc += rv * rv;
  }
  const double denom = sqrt(cluster_sum<CLUSTER>(acc, sh, slots, phase));
  phase ^= 1;
  int iters = 0;
  if (denom != 0.0) {
    double rhok1 = 0.0;
    for (;;) {
      acc = 0.0;
      for (int q = gtid; q < nint; q += nthr) {
        const double rv = __ldcg(r + pid(q));
        acc += rv * rv;
      }
      const double rhok2 = cluster_sum<CLUSTER>(acc, sh, slots, phase);
      phase ^= 1;
      if (sqrt(rhok2) / denom <= errtol) break;
      if (iters >= itmax) break;
      if (iters == 0) {
        for (int q = gtid; q < nint; q += nthr) {
          const size_t id = pid(q);
          __stcg(p + id, __ldcg(r + id));
        }
      } else {
        const double beta = rhok2 / rhok1;
        const double alpha = 1.0 / beta;
        for (int q = gtid; q < nint; q += nthr) {
          const size_t id = pid(q);
          double pv = __ldcg(p + id);
          pv += alpha * __ldcg(r + id);
          pv *= beta;
          __stcg(p + id, pv);
        }
      }
      csync();
      acc = 0.0;
      for (int q = gtid; q < nint; q += nthr) {
        const size_t id = pid(q);
        double tO, tU, tD;
        sum27<true>(op, g, p, id, tO, tU, tD);
        const double pv = __ldcg(p + id);
        const double av = -tO - tU - tD + (op.c[OC][id] + cc[id]) * pv;
        __stcg(ap + id, av);
        acc += pv * av;
      }
      const double pAp = cluster_sum<CLUSTER>(acc, sh, slots, phase);
      phase ^= 1;
      const double alpha = rhok2 / pAp;
      rhok1 = rhok2;
      for (int q = gtid; q < nint; q += nthr) {
        const size_t id = pid(q);
        __stcg(x + id, __ldcg(x + id) + alpha * __ldcg(p + id));
        __stcg(r + id, __ldcg(r + id) + (-alpha) * __ldcg(ap + id));
      }
      iters++;
      csync();
    }
  }
  if (gtid == 0 && iters_out) iters_out[0] = iters;
  // no CTA may exit while another can still read its shared memory
  csync();
}

// The same iteration for a coarsest level that one CTA holds: the direction
// p lives in shared memory over the whole grid (zero boundary), x, r and A p
// of a thread's points stay in registers, and each sum is one barrier (every
// thread adds the warp partials itself).  Points are assigned to threads and
// partial sums are added in the same order as k_cg_coarse<1> with 512
// threads, so both kernels produce bitwise equal iterates; this one only
// saves the global-memory round trips and barriers between the vector passes.
constexpr int kCgThreads = 512, kCgPPT = 2;
constexpr size_t kCgSmemMax = 200 * 1024;

__global__ void __launch_bounds__(kCgThreads)
    k_cg_coarse_onchip(Grid g, Op op, const double* __restrict__ cc,
                       const double* __restrict__ fc, double* x, double* r, int itmax,
                       double errtol, int* iters_out) {
  extern __shared__ double ps[];
  __shared__ double sh[2][32];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int nint = (nx - 2) * (ny - 2) * (nz - 2);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (size_t q = threadIdx.x; q < g.n(); q += blockDim.x) ps[q] = 0.0;
  size_t id[kCgPPT];
  bool own[kCgPPT];
  double rl[kCgPPT], xl[kCgPPT], dg[kCgPPT], al[kCgPPT];
  double acc = 0.0;
  // r = f - (A + cc) x   (x = 0 on entry)
#pragma unroll
  for (int m = 0; m < kCgPPT; m++) {
    const int q = threadIdx.x + m * blockDim.x;
    own[m] = q < nint;
    id[m] = 0;
    rl[m] = xl[m] = dg[m] = al[m] = 0.0;
    if (!own[m]) continue;
    const int i = 1 + q % (nx - 2);
    const int j = 1 + (q / (nx - 2)) % (ny - 2);
    const int k = 1 + q / ((nx - 2) * (ny - 2));
    id[m] = g.idx(i, j, k);
    double tO, tU, tD;
    sum27<true>(op, g, x, id[m], tO, tU, tD);
    xl[m] = __ldcg(x + id[m]);
    dg[m] = op.c[OC][id[m]] + cc[id[m]];
    const double rv = fc[id[m]] + tO + tU + tD - (op.c[OC][id[m]] + cc[id[m]]) * xl[m];
    rl[m] = rv;
    acc += rv * rv;
  }
  int phase = 0;
  auto bsum = [&](double v) {
    v = warp_sum(v);
    if (lane == 0) sh[phase][wid] = v;
    __syncthreads();
    double b = 0.0;
    for (int w = 0; w < nw; w++) b += sh[phase][w];
    phase ^= 1;
    return b;
  };
  const double denom = sqrt(bsum(acc));
  int iters = 0;
  if (denom != 0.0) {
    double rhok1 = 0.0;
    for (;;) {
      acc = 0.0;
#pragma unroll
      for (int m = 0; m < kCgPPT; m++)
        if (own[m]) acc += rl[m] * rl[m];
      const double rhok2 = bsum(acc);
      if (sqrt(rhok2) / denom <= errtol) break;
      if (iters >= itmax) break;
      if (iters == 0) {
#pragma unroll
        for (int m = 0; m < kCgPPT; m++)
          if (own[m]) ps[id[m]] = rl[m];
      } else {
        const double beta = rhok2 / rhok1;
        const double alpha = 1.0 / beta;
#pragma unroll
        for (int m = 0; m < kCgPPT; m++) {
          if (!own[m]) continue;
          double pv = ps[id[m]];
          pv += alpha * rl[m];
          pv *= beta;
          ps[id[m]] = pv;
        }
      }
      __syncthreads();
      acc = 0.0;
#pragma unroll
      for (int m = 0; m < kCgPPT; m++) {
        if (!own[m]) continue;
        double tO, tU, tD;
        sum27<false>(op, g, ps, id[m], tO, tU, tD);
        const double pv = ps[id[m]];
        const double av = -tO - tU - tD + dg[m] * pv;
        al[m] = av;
        acc += pv * av;
      }
      const double pAp = bsum(acc);
      const double alpha = rhok2 / pAp;
      rhok1 = rhok2;
#pragma unroll
      for (int m = 0; m < kCgPPT; m++) {
        if (!own[m]) continue;
        xl[m] = xl[m] + alpha * ps[id[m]];
        rl[m] = rl[m] + (-alpha) * al[m];
      }
      iters++;
      // the next direction update writes only this thread's points of p; the
      // two barriers of the sums order it after every read of the matvec
    }
  }
#pragma unroll
  for (int m = 0; m < kCgPPT; m++) {
    if (!own[m]) continue;
    x[id[m]] = xl[m];
    r[id[m]] = rl[m];
  }
  if (threadIdx.x == 0 && iters_out) iters_out[0] = iters;
}

// The same iteration on a larger coarsest level, one cluster of CL CTAs:
// CTA `rank` owns the slab of planes k0 .. k1-1 and keeps p over its slab and
// one halo plane on either side in shared memory (zero boundary).  A
// direction update writes the slab's first and last planes into the
// neighbours' halo planes as well (stores to distributed shared memory ahead
// of the cluster barrier), and each CTA writes its block partial of a sum
// into every CTA's slot for it, so after the barrier every CTA adds the same
// partials in rank order from its own shared memory.  x, r and A p of the
// CTA's points stay in registers; where shared memory allows, the 26
// off-diagonal coefficients of its points are loaded once into it.
constexpr int kSlabThreads = 512, kSlabPPT = 2;
constexpr size_t kSlabSmemMax = 220 * 1024;

// tmpO + tmpU + tmpD of sum27 with x read from xs at the offset of xid - id
__device__ __forceinline__ void sum27_at(const Op& op, Grid g, const double* xs,
                                         ptrdiff_t off, size_t id, double& tO, double& tU,
                                         double& tD) {
  const size_t sy = g.nx, sz = (size_t)g.nx * g.ny;
  auto X = [&](size_t p) -> double { return xs[(ptrdiff_t)p + off]; };
  const double* const* c = op.c;
  tO = +c[ON][id] * X(id + sy) + c[ON][id - sy] * X(id - sy) + c[OE][id] * X(id + 1) +
       c[OE][id - 1] * X(id - 1) + c[ONE][id] * X(id + sy + 1) +
       c[ONW][id] * X(id + sy - 1) + c[ONW][id - sy + 1] * X(id - sy + 1) +
       c[ONE][id - sy - 1] * X(id - sy - 1);
  tU = +c[UC][id] * X(id + sz) + c[UN][id] * X(id + sz + sy) + c[US][id] * X(id + sz - sy) +
       c[UE][id] * X(id + sz + 1) + c[UW][id] * X(id + sz - 1) +
       c[UNE][id] * X(id + sz + sy + 1) + c[UNW][id] * X(id + sz + sy - 1) +
       c[USE][id] * X(id + sz - sy + 1) + c[USW][id] * X(id + sz - sy - 1);
  tD = +c[UC][id - sz] * X(id - sz) + c[US][id - sz + sy] * X(id - sz + sy) +
       c[UN][id - sz - sy] * X(id - sz - sy) + c[UW][id - sz + 1] * X(id - sz + 1) +
       c[UE][id - sz - 1] * X(id - sz - 1) + c[USW][id - sz + sy + 1] * X(id - sz + sy + 1) +
       c[USE][id - sz + sy - 1] * X(id - sz + sy - 1) +
       c[UNW][id - sz - sy + 1] * X(id - sz - sy + 1) +
       c[UNE][id - sz - sy - 1] * X(id - sz - sy - 1);
}

template <int CL>
__global__ void __launch_bounds__(kSlabThreads)
    k_cg_coarse_slab(Grid g, Op op, const double* __restrict__ cc,
                     const double* __restrict__ fc, double* x, double* r, int itmax,
                     double errtol, int* iters_out, int cache_coef) {
  extern __shared__ double ps[];  // planes k0-1 .. k1 of p, then the coefficients
  __shared__ double sh[32];
  __shared__ double slots[2][CL];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t sy = nx, pl = (size_t)nx * ny;
  const int per = (nz - 2 + CL - 1) / CL;
  const int k0 = 1 + rank * per;
  const int k1 = min(k0 + per, nz - 1);
  const int nown = (k1 > k0) ? (k1 - k0) * (nx - 2) * (ny - 2) : 0;
  const int ncap = per * (nx - 2) * (ny - 2);             // coefficient slots
  double* cf = ps + (size_t)(per + 2) * pl;              // [26][ncap]
  const ptrdiff_t off = -(ptrdiff_t)((size_t)(k0 - 1) * pl);  // global id -> ps index
  double* below = (rank > 0) ? cl.map_shared_rank(ps, rank - 1) + (size_t)(per + 1) * pl
                             : nullptr;                  // rank-1's upper halo plane
  double* above = (rank < CL - 1 && k1 < nz - 1) ? cl.map_shared_rank(ps, rank + 1) : nullptr;
  for (size_t q = threadIdx.x; q < (size_t)(per + 2) * pl; q += blockDim.x) ps[q] = 0.0;
  size_t id[kSlabPPT];
  int kk[kSlabPPT];
  bool own[kSlabPPT];
  double rl[kSlabPPT], xl[kSlabPPT], dg[kSlabPPT], al[kSlabPPT];
  double acc = 0.0;
#pragma unroll
  for (int m = 0; m < kSlabPPT; m++) {
    const int q = threadIdx.x + m * blockDim.x;
    own[m] = q < nown;
    id[m] = 0;
    kk[m] = 0;
    rl[m] = xl[m] = dg[m] = al[m] = 0.0;
    if (!own[m]) continue;
    const int i = 1 + q % (nx - 2);
    const int j = 1 + (q / (nx - 2)) % (ny - 2);
    const int k = k0 + q / ((nx - 2) * (ny - 2));
    kk[m] = k;
    id[m] = g.idx(i, j, k);
    double tO, tU, tD;
    sum27<true>(op, g, x, id[m], tO, tU, tD);
    xl[m] = __ldcg(x + id[m]);
    dg[m] = op.c[OC][id[m]] + cc[id[m]];
    const double rv = fc[id[m]] + tO + tU + tD - (op.c[OC][id[m]] + cc[id[m]]) * xl[m];
    rl[m] = rv;
    acc += rv * rv;
    if (cache_coef) {
      Coef27 C;
      load_coef27(op, cc, fc, id[m], sy, pl, C);
#pragma unroll
      for (int t = 0; t < 8; t++) cf[(size_t)t * ncap + q] = C.o[t];
#pragma unroll
      for (int t = 0; t < 9; t++) cf[(size_t)(8 + t) * ncap + q] = C.u[t];
#pragma unroll
      for (int t = 0; t < 9; t++) cf[(size_t)(17 + t) * ncap + q] = C.d[t];
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int phase = 0;
  auto csum = [&](double v) {
    v = warp_sum(v);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (threadIdx.x < CL) {
      double b = 0.0;
      for (int w = 0; w < nw; w++) b += sh[w];
      cl.map_shared_rank(&slots[0][0], (int)threadIdx.x)[phase * CL + rank] = b;
    }
    cl.sync();
    double tot = 0.0;
    for (int q = 0; q < CL; q++) tot += slots[phase][q];
    phase ^= 1;
    return tot;
  };
  const double denom = sqrt(csum(acc));
  int iters = 0;
  if (denom != 0.0) {
    double rhok1 = 0.0;
    for (;;) {
      acc = 0.0;
#pragma unroll
      for (int m = 0; m < kSlabPPT; m++)
        if (own[m]) acc += rl[m] * rl[m];
      const double rhok2 = csum(acc);
      if (sqrt(rhok2) / denom <= errtol) break;
      if (iters >= itmax) break;
      const double beta = (iters == 0) ? 0.0 : rhok2 / rhok1;
      const double alpha = (iters == 0) ? 0.0 : 1.0 / beta;
#pragma unroll
      for (int m = 0; m < kSlabPPT; m++) {
        if (!own[m]) continue;
        double pv;
        if (iters == 0) {
          pv = rl[m];
        } else {
          pv = ps[(ptrdiff_t)id[m] + off];
          pv += alpha * rl[m];
          pv *= beta;
        }
        ps[(ptrdiff_t)id[m] + off] = pv;
        const size_t inplane = id[m] % pl;
        if (kk[m] == k0 && below) below[inplane] = pv;
        if (kk[m] == k1 - 1 && above) above[inplane] = pv;
      }
      cl.sync();
      acc = 0.0;
#pragma unroll
      for (int m = 0; m < kSlabPPT; m++) {
        if (!own[m]) continue;
        double tO, tU, tD;
        if (cache_coef) {
          const int q = threadIdx.x + m * blockDim.x;
          const double* ps0 = ps + ((ptrdiff_t)id[m] + off);
          auto X = [&](ptrdiff_t d) -> double { return ps0[d]; };
          auto A = [&](int t) -> double { return cf[(size_t)t * ncap + q]; };
          const ptrdiff_t Y = (ptrdiff_t)sy, Z = (ptrdiff_t)pl;
          tO = +A(0) * X(Y) + A(1) * X(-Y) + A(2) * X(1) + A(3) * X(-1) + A(4) * X(Y + 1) +
               A(5) * X(Y - 1) + A(6) * X(-Y + 1) + A(7) * X(-Y - 1);
          tU = +A(8) * X(Z) + A(9) * X(Z + Y) + A(10) * X(Z - Y) + A(11) * X(Z + 1) +
               A(12) * X(Z - 1) + A(13) * X(Z + Y + 1) + A(14) * X(Z + Y - 1) +
               A(15) * X(Z - Y + 1) + A(16) * X(Z - Y - 1);
          tD = +A(17) * X(-Z) + A(18) * X(-Z + Y) + A(19) * X(-Z - Y) + A(20) * X(-Z + 1) +
               A(21) * X(-Z - 1) + A(22) * X(-Z + Y + 1) + A(23) * X(-Z + Y - 1) +
               A(24) * X(-Z - Y + 1) + A(25) * X(-Z - Y - 1);
        } else {
          sum27_at(op, g, ps, off, id[m], tO, tU, tD);
        }
        const double pv = ps[(ptrdiff_t)id[m] + off];
        const double av = -tO - tU - tD + dg[m] * pv;
        al[m] = av;
        acc += pv * av;
      }
      const double pAp = csum(acc);
      const double alpha2 = rhok2 / pAp;
      rhok1 = rhok2;
#pragma unroll
      for (int m = 0; m < kSlabPPT; m++) {
        if (!own[m]) continue;
        xl[m] = xl[m] + alpha2 * ps[(ptrdiff_t)id[m] + off];
        rl[m] = rl[m] + (-alpha2) * al[m];
      }
      iters++;
      // a neighbour reads this slab's halo copy in its matvec, before the
      // next sum's cluster barrier; this CTA writes it again only after that
    }
  }
#pragma unroll
  for (int m = 0; m < kSlabPPT; m++) {
    if (!own[m]) continue;
    x[id[m]] = xl[m];
    r[id[m]] = rl[m];
  }
  if (rank == 0 && threadIdx.x == 0 && iters_out) iters_out[0] = iters;
  cl.sync();  // no CTA may exit while a neighbour can still write its shared memory
}

template <int CL>
static int launch_cg_slab(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                          double* x, double* r, int itmax, double errtol, int* iters_dev,
                          size_t smem, int cache_coef) {
  static const cudaError_t attr_ok = [] {
    cudaError_t e = cudaFuncSetAttribute(k_cg_coarse_slab<CL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kSlabSmemMax);
    if (e == cudaSuccess && CL > 8)
      e = cudaFuncSetAttribute(k_cg_coarse_slab<CL>,
                               cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return e;
  }();
  if (attr_ok != cudaSuccess) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CL, 1, 1);
  cfg.blockDim = dim3(kSlabThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_cg_coarse_slab<CL>, g, op, cc, fc, x, r, itmax, errtol,
                            iters_dev, cache_coef) == cudaSuccess;
}

int launch_cg_coarse(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                     double* x, double* r, double* p, double* ap, int itmax, double errtol,
                     int* iters_dev, int want_cluster) {
  const int nint = (g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  const size_t smem = g.n() * sizeof(double);
  if (nint <= kCgThreads * kCgPPT && smem <= kCgSmemMax) {
    static const cudaError_t attr_ok = cudaFuncSetAttribute(
        k_cg_coarse_onchip, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCgSmemMax);
    if (attr_ok != cudaSuccess) return 0;
    k_cg_coarse_onchip<<<1, kCgThreads, smem, s>>>(g, op, cc, fc, x, r, itmax, errtol,
                                                   iters_dev);
    return cudaGetLastError() == cudaSuccess;
  }
  // slab clusters: the smallest size whose slabs give each thread at most two
  // points, else at most kSlabPPT, within one CTA's shared memory (or the
  // size asked for, if its slabs fit)
  for (int pass = 0; pass < 2; pass++) {
    static const int max_cl = [] {
      int dev = 0, ok = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&ok, cudaDevAttrClusterLaunch, dev);
      return ok ? 16 : 1;
    }();
    const int plane_pts = (g.nx - 2) * (g.ny - 2);
    const int limit = kSlabThreads * (pass == 0 ? 2 : kSlabPPT);
    for (int cl = 4; cl <= max_cl; cl *= 2) {
      if (want_cluster > 0 && cl != want_cluster) continue;
      const int per = (g.nz - 2 + cl - 1) / cl;
      size_t sm = (size_t)(per + 2) * g.nx * g.ny * sizeof(double);
      if (per * plane_pts > limit || sm > kSlabSmemMax) continue;
      const size_t sm_coef = sm + (size_t)26 * per * plane_pts * sizeof(double);
      const int cache = sm_coef <= kSlabSmemMax;
      if (cache) sm = sm_coef;
      switch (cl) {
        case 4:
          return launch_cg_slab<4>(s, g, op, cc, fc, x, r, itmax, errtol, iters_dev, sm, cache);
        case 8:
          return launch_cg_slab<8>(s, g, op, cc, fc, x, r, itmax, errtol, iters_dev, sm, cache);
        case 16:
          if (launch_cg_slab<16>(s, g, op, cc, fc, x, r, itmax, errtol, iters_dev, sm, cache))
            return 1;
          cudaGetLastError();  // no 16-CTA clusters here: the strided kernel below
          break;
      }
    }
  }
  int cluster = 1;
  if (nint > 4096) cluster = 8;
  else if (nint > 1024) cluster = 4;
  const int threads = kCgThreads;
  if (cluster == 1) {
    k_cg_coarse<1><<<1, threads, 0, s>>>(g, op, cc, fc, x, r, p, ap, itmax, errtol, iters_dev);
    return cudaGetLastError() == cudaSuccess;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = (cluster == 8)
                      ? cudaLaunchKernelEx(&cfg, k_cg_coarse<8>, g, op, cc, fc, x, r, p, ap,
                                           itmax, errtol, iters_dev)
                      : cudaLaunchKernelEx(&cfg, k_cg_coarse<4>, g, op, cc, fc, x, r, p, ap,
                                           itmax, errtol, iters_dev);
  return e == cudaSuccess;
}

// ===========================================================================
// Nonlinear ion term, Vc_vecpmg / Vdc_vecpmg (src/pmgc/mypdec.c:145-223,
// 366-433) and the nonlinear residual Vnmresid7_1s (matvecd.c:633-691)
// ===========================================================================
__device__ __forceinline__ double cvec_point(const IonTable& ions, double coef, double u,
                                             bool deriv) {
  double out = 0.0;
  for (int s = 0; s < ions.nion; s++) {
    const double zcf2 = deriv ? ions.sconc[s] * ions.q[s] * ions.q[s]
                              : -1.0 * ions.sconc[s] * ions.q[s];
    const double zu2 = -1.0 * ions.q[s];
    const double t = fabs(zcf2 * coef);
    const double am_zero = (1.0e-20 <= t ? 1.0e-20 : t) * 1.0e20;
    const double v = zu2 * u;
    double am_neg = (v <= 0.0 ? v : 0.0);
    double am_pos = (v >= 0.0 ? v : 0.0);
    if (!(am_neg >= -85.0)) am_neg = -85.0;
    if (!(am_pos <= 85.0)) am_pos = 85.0;
    out = out + zcf2 * coef * exp(am_zero * (am_neg + am_pos));
  }
  return out;
}

// cvec_point(..., false) and, where d is given, cvec_point(..., true) of the
// same point: the two share the exponential wherever their arguments agree
// (everywhere but where |zcf2 coef| is below 1e-20 for one of them), so the
// values are those of two separate calls.
__device__ __forceinline__ void cvec_pair(const IonTable& ions, double coef, double u,
                                          double* c, double* d) {
  double out = 0.0, dout = 0.0;
  for (int s = 0; s < ions.nion; s++) {
    const double zcf2 = -1.0 * ions.sconc[s] * ions.q[s];
    const double zcf2d = ions.sconc[s] * ions.q[s] * ions.q[s];
    const double zu2 = -1.0 * ions.q[s];
    const double t = fabs(zcf2 * coef);
    const double am_zero = (1.0e-20 <= t ? 1.0e-20 : t) * 1.0e20;
    const double v = zu2 * u;
    double am_neg = (v <= 0.0 ? v : 0.0);
    double am_pos = (v >= 0.0 ? v : 0.0);
    if (!(am_neg >= -85.0)) am_neg = -85.0;
    if (!(am_pos <= 85.0)) am_pos = 85.0;
    const double arg = am_zero * (am_neg + am_pos);
    const double e = exp(arg);
    out = out + zcf2 * coef * e;
    if (d) {
      const double td = fabs(zcf2d * coef);
      const double am_zero_d = (1.0e-20 <= td ? 1.0e-20 : td) * 1.0e20;
      const double argd = am_zero_d * (am_neg + am_pos);
      dout = dout + zcf2d * coef * (argd == arg ? e : exp(argd));
    }
  }
  *c = out;
  if (d) *d = dout;
}

__global__ void k_nresid(Grid g, Op op, const double* __restrict__ cc,
                         const double* __restrict__ fc, const double* __restrict__ x, double* r,
                         IonTable ions) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const size_t id = g.idx(i, j, k);
    const double w = cvec_point(ions, cc[id], x[id], false);
    r[id] = sum7(op, g, x, id, fc[id]) - op.c[OC][id] * x[id] - w;
  }
}

void launch_nresid(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                   const double* x, double* r, IonTable ions) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  k_nresid<<<blocks_for(nint), kThreads, 0, s>>>(g, op, cc, fc, x, r, ions);
}

// k_nresid fused with the 1-norm of r (the partial sums of k_reduce_partial
// with the same grid and traversal, so the norm is the same bits) and, when
// cp is not null, c'(x) on the interior (the update of k_dcvec)
// at most 48 registers: five 256-thread CTAs per SM keep enough loads in
// flight around the exponentials (76 registers allowed three)
__global__ void __launch_bounds__(256, 5) k_nresid_nrm(Grid g, Op op, const double* __restrict__ cc,
                             const double* __restrict__ fc, const double* __restrict__ x,
                             double* r, IonTable ions, double* part, double* cp) {
  __shared__ double sh[32];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  double acc = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const size_t id = g.idx(i, j, k);
    const double c = cc[id], xv = x[id];
    double w, dw;
    cvec_pair(ions, c, xv, &w, cp ? &dw : nullptr);
    const double rv = sum7(op, g, x, id, fc[id]) - op.c[OC][id] * xv - w;
    r[id] = rv;
    acc += fabs(rv);
    if (cp) cp[id] = dw;
  }
  const double t = block_sum<kRedThreads>(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

void launch_nresid_nrm1(cudaStream_t s, Grid g, Op op, const double* cc, const double* fc,
                        const double* x, double* r, IonTable ions, double* part,
                        double* out_dev, double* cp) {
  // about two points per thread (up to four times the usual partial count,
  // which the scratch holds): enough warps in flight to cover the loads
  // around the exponentials
  const size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  const int nb = (int)std::max<size_t>(1, std::min<size_t>(4 * 1184, (nint + 511) / 512));
  k_nresid_nrm<<<nb, kRedThreads, 0, s>>>(g, op, cc, fc, x, r, ions, part, cp);
  k_reduce_final<<<1, kRedThreads, 0, s>>>(part, nb, out_dev);
}

// out = x + a y on interior points (the reference's copy then axpy, one pass)
__global__ void k_xpay_interior(Grid g, const double* __restrict__ x, double a,
                                const double* __restrict__ y, double* out) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_ijk(q, nx, ny, i, j, k);
    const size_t id = g.idx(i, j, k);
    out[id] = x[id] + a * y[id];
  }
}

void launch_xpay_interior(cudaStream_t s, Grid g, const double* x, double a, const double* y,
                          double* out) {
  size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  k_xpay_interior<<<blocks_for(nint), kThreads, 0, s>>>(g, x, a, y, out);
}

__global__ void k_dcvec(size_t n, const double* __restrict__ cc, const double* __restrict__ x,
                        double* cp, IonTable ions) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x)
    cp[q] = cvec_point(ions, cc[q], x[q], true);
}

void launch_dcvec(cudaStream_t s, Grid g, const double* cc, const double* x, double* cp,
                  IonTable ions) {
  k_dcvec<<<blocks_for(g.n()), kThreads, 0, s>>>(g.n(), cc, x, cp, ions);
}

// ===========================================================================
// Dirichlet restore VfboundPMG (src/pmgc/mikpckd.c:209-256): x faces first,
// then y faces, then z faces, so edges take the later face's value.
// ===========================================================================
__global__ void k_fbound(Grid g, double* x, const double* __restrict__ gx,
                         const double* __restrict__ gy, const double* __restrict__ gz) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t n = g.n();
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    split3(q, nx, ny, i, j, k);
    if (k == 0) x[q] = gz[(size_t)j * nx + i];
    else if (k == nz - 1) x[q] = gz[((size_t)ny + j) * nx + i];
    else if (j == 0) x[q] = gy[(size_t)k * nx + i];
    else if (j == ny - 1) x[q] = gy[((size_t)nz + k) * nx + i];
    else if (i == 0) x[q] = gx[(size_t)k * ny + j];
    else if (i == nx - 1) x[q] = gx[((size_t)nz + k) * ny + j];
  }
}

void launch_fbound(cudaStream_t s, Grid g, double* x, const double* gx, const double* gy,
                   const double* gz) {
  k_fbound<<<blocks_for(g.n()), kThreads, 0, s>>>(g, x, gx, gy, gz);
}

// ===========================================================================
// Energy sums: Vpmg_qfEnergyVolume (src/mg/vpmg.c:1861-1891),
// Vpmg_dielEnergy (1279-1340), Vpmg_qmEnergyNONLIN (1401-1488) with the
// clamped exponential of Vcap_exp (src/generic/vcap.c:59-73).
// pvec(i,j,k) = wx[i] wy[j] wz[k] (Vpmg_setPart, vpmg.c:627-870).
// ===========================================================================
// With complement, the weight extEnergy gives the coarse grid of a focusing
// chain (vpmg.c:2508-2509): 1 - pvec where pvec <= VSMALL, else 0.
__device__ __forceinline__ double pvec_at(const EnergyArgs& a, int i, int j, int k) {
  double v = a.wx[i] * a.wy[j] * a.wz[k];
  v = (fabs(v) < 1.0e-12) ? 0.0 : v;
  if (a.complement) {
    if (v > 1.0e-9) v = 1.0;
    v = (1 - v) * 1.0;
  }
  return v;
}

__global__ void __launch_bounds__(256, 5) k_energy_partial(EnergyArgs a, double* part) {
  __shared__ double sh[32];
  const Grid g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t n = g.n();
  double qf = 0.0, diel = 0.0, qm = 0.0, nchop = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    split3(q, nx, ny, i, j, k);
    const double pv = pvec_at(a, i, j, k);
    const double u = a.u[q];
    qf += (pv * u * a.charge[q]);
    if (a.nonlin) {
      if (i < nx - 1 && j < ny - 1 && k < nz - 1) {
        const double px = 0.5 * (pv + pvec_at(a, i + 1, j, k));
        const double py = 0.5 * (pv + pvec_at(a, i, j + 1, k));
        const double pz = 0.5 * (pv + pvec_at(a, i, j, k + 1));
        const double gxv = (u - a.u[q + 1]) / a.hx;
        const double gyv = (u - a.u[q + nx]) / a.hy;
        const double gzv = (u - a.u[q + (size_t)nx * ny]) / a.hz;
        const double ex = a.epsx[q] * px * (gxv * gxv);
        const double ey = a.epsy[q] * py * (gyv * gyv);
        const double ez = a.epsz[q] * pz * (gzv * gzv);
        diel += (ex + ey + ez);
      }
      if (pv * a.kappa[q] > 1.0e-9 && a.linear_qm) {
        // Vpmg_qmEnergyNONLIN, LPBE branch (vpmg.c:1474-1479)
        qm += (pv * a.zkappa2 * a.kappa[q] * (u * u));
      } else if (pv * a.kappa[q] > 1.0e-9) {
        for (int s = 0; s < a.ions.nion; s++) {
          const double arg = -a.ions.q[s] * u;
          double e;
          if (arg > 85.0) { e = exp(85.0); nchop += 1.0; }
          else if (arg < -85.0) { e = exp(-85.0); nchop += 1.0; }
          else e = exp(arg);
          qm += (pv * a.kappa[q] * a.zks2 * a.ions.sconc[s] * (e - 1.0));
        }
      }
    }
  }
  double t0 = block_sum<kRedThreads>(qf, sh);
  double t1 = block_sum<kRedThreads>(diel, sh);
  double t2 = block_sum<kRedThreads>(qm, sh);
  double t3 = block_sum<kRedThreads>(nchop, sh);
  if (threadIdx.x == 0) {
    part[4 * blockIdx.x + 0] = t0;
    part[4 * blockIdx.x + 1] = t1;
    part[4 * blockIdx.x + 2] = t2;
    part[4 * blockIdx.x + 3] = t3;
  }
}

__global__ void k_energy_final(const double* __restrict__ part, int nparts, double* out) {
  __shared__ double sh[32];
  for (int c = 0; c < 4; c++) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[4 * i + c];
    double t = block_sum<kRedThreads>(acc, sh);
    if (threadIdx.x == 0) out[c] = t;
  }
}

void launch_energy_sums(cudaStream_t s, const EnergyArgs& a, double* part, double* out_dev) {
  int nb = (int)reduce_parts(a.g.n());
  k_energy_partial<<<nb, kRedThreads, 0, s>>>(a, part);
  k_energy_final<<<1, kRedThreads, 0, s>>>(part, nb, out_dev);
}

}  // namespace pmgb
