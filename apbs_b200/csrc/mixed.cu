// Mixed-precision PMG: FP32 V-cycles inside an FP64 refinement loop.
//
// The outer loop is the reference's own stopping rule in FP64: the fine
// residual r = f - (A + cc) x, its 1-norm against ||f||_1 (Vmvcs,
// src/pmgc/mgcsd.c:140, 540-562), and the FP64 correction x += e.  Each
// correction e solves A e = r approximately with one V-cycle run entirely in
// FP32 on an FP32 copy of the operator hierarchy.  Differences from the FP64
// V-cycle (they change rounding, not the fixed point of the outer loop):
//   * 27-point levels are smoothed by 8-colour Gauss-Seidel (colours
//     (i&1, j&1, k&1) have no 27-point neighbours in common), fully parallel,
//     instead of the lexicographic red-black order the FP64 path reproduces;
//   * the hierarchy is coarsened (Galerkin, trilinear P) below the
//     reference's coarsest level until at most 512 unknowns remain, and that
//     level is solved exactly with a dense FP64 Cholesky factorisation of
//     (A_c + diag cc_c).
// For NPBE the Newton iteration (newtond.c:162-548) is unchanged and in FP64;
// only its inner linear solves use FP32 V-cycles.
#include <cooperative_groups.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "mixed.cuh"
#include "solver_internal.cuh"

namespace cg = cooperative_groups;

namespace pmgb {

namespace {

struct MLevel {
  Grid g;
  int nop;
  float* op[14];
  double* op64[14];  // FP64 operator (owned only on levels below the FP64 hierarchy)
  int own64;
  double* cc64;      // FP64 Helmholtz term of this level (owned on extra levels)
  float* cc;
  float* w0;
  float* x;
  Op ops64() const {
    Op o;
    for (int c = 0; c < 14; c++) o.c[c] = (c < nop) ? op64[c] : nullptr;
    o.nop = nop;
    return o;
  }
};

struct OpF {
  const float* c[14];
  int nop;
};

}  // namespace

struct MixedState {
  int nlev;
  MLevel lev[16];
  float* r;      // fine-sized FP32 scratch
  float* w2;     // fine-sized FP32 scratch
  double* dense;  // coarsest dense factor (n x n)
  double* dvec;   // coarsest rhs / solution in FP64
  int nd;
  int* dinfo;
  cudaGraphExec_t exec[2];
  long long kernels[2];
  int cc_ready;
};

namespace {

#define CKM(call)                                                                      \
  do {                                                                                 \
    cudaError_t e__ = (call);                                                          \
    if (e__ != cudaSuccess) {                                                          \
      set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e__));  \
      return 0;                                                                        \
    }                                                                                  \
  } while (0)

OpF opf(const MLevel& L) {
  OpF o;
  for (int c = 0; c < 14; c++) o.c[c] = (c < L.nop) ? L.op[c] : nullptr;
  o.nop = L.nop;
  return o;
}

// ---------------------------------------------------------------------------
// conversions
// ---------------------------------------------------------------------------
__global__ void k_to_f32(const double* __restrict__ a, float* b, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x)
    b[q] = (float)a[q];
}

void to_f32(cudaStream_t s, const double* a, float* b, size_t n) {
  k_to_f32<<<blocks_for(n), kThreads, 0, s>>>(a, b, n);
}

// ---------------------------------------------------------------------------
// FP32 stencils
// ---------------------------------------------------------------------------
__device__ __forceinline__ float nb27(const OpF& o, Grid g, const float* x, size_t id) {
  const size_t sy = g.nx, sz = (size_t)g.nx * g.ny;
  const float* const* c = o.c;
  float t = c[ON][id] * x[id + sy] + c[ON][id - sy] * x[id - sy] + c[OE][id] * x[id + 1] +
            c[OE][id - 1] * x[id - 1];
  t += c[ONE][id] * x[id + sy + 1] + c[ONW][id] * x[id + sy - 1] +
       c[ONW][id - sy + 1] * x[id - sy + 1] + c[ONE][id - sy - 1] * x[id - sy - 1];
  t += c[UC][id] * x[id + sz] + c[UN][id] * x[id + sz + sy] + c[US][id] * x[id + sz - sy] +
       c[UE][id] * x[id + sz + 1] + c[UW][id] * x[id + sz - 1];
  t += c[UNE][id] * x[id + sz + sy + 1] + c[UNW][id] * x[id + sz + sy - 1] +
       c[USE][id] * x[id + sz - sy + 1] + c[USW][id] * x[id + sz - sy - 1];
  t += c[UC][id - sz] * x[id - sz] + c[US][id - sz + sy] * x[id - sz + sy] +
       c[UN][id - sz - sy] * x[id - sz - sy] + c[UW][id - sz + 1] * x[id - sz + 1] +
       c[UE][id - sz - 1] * x[id - sz - 1];
  t += c[USW][id - sz + sy + 1] * x[id - sz + sy + 1] +
       c[USE][id - sz + sy - 1] * x[id - sz + sy - 1] +
       c[UNW][id - sz - sy + 1] * x[id - sz - sy + 1] +
       c[UNE][id - sz - sy - 1] * x[id - sz - sy - 1];
  return t;
}

__device__ __forceinline__ float nb7(const OpF& o, Grid g, const float* x, size_t id) {
  const size_t sy = g.nx, sz = (size_t)g.nx * g.ny;
  return o.c[ON][id] * x[id + sy] + o.c[ON][id - sy] * x[id - sy] + o.c[OE][id] * x[id + 1] +
         o.c[OE][id - 1] * x[id - 1] + o.c[UC][id - sz] * x[id - sz] + o.c[UC][id] * x[id + sz];
}

__global__ void k_gs7_f32(Grid g, OpF o, const float* __restrict__ cc,
                          const float* __restrict__ fc, float* x, int parity) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int hr = (nx - 1) / 2;
  const size_t nslots = (size_t)hr * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nslots;
       q += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(q % hr);
    const int j = 1 + (int)((q / hr) % (ny - 2));
    const int k = 1 + (int)(q / ((size_t)hr * (ny - 2)));
    const int i = 1 + (((1 + j + k) & 1) != parity) + 2 * m;
    if (i > nx - 2) continue;
    const size_t id = g.idx(i, j, k);
    x[id] = (fc[id] + nb7(o, g, x, id)) / (o.c[OC][id] + cc[id]);
  }
}

// r = f - (A + cc) x on interior points (7- or 27-point)
__global__ void k_resid_f32(Grid g, OpF o, const float* __restrict__ cc,
                            const float* __restrict__ fc, const float* __restrict__ x, float* r) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(q % (nx - 2));
    const int j = 1 + (int)((q / (nx - 2)) % (ny - 2));
    const int k = 1 + (int)(q / ((size_t)(nx - 2) * (ny - 2)));
    const size_t id = g.idx(i, j, k);
    const float nb = (o.nop == 4) ? nb7(o, g, x, id) : nb27(o, g, x, id);
    r[id] = fc[id] + nb - (o.c[OC][id] + cc[id]) * x[id];
  }
}

__global__ void k_matvec_f32(Grid g, OpF o, const float* __restrict__ cc,
                             const float* __restrict__ x, float* y) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(q % (nx - 2));
    const int j = 1 + (int)((q / (nx - 2)) % (ny - 2));
    const int k = 1 + (int)(q / ((size_t)(nx - 2) * (ny - 2)));
    const size_t id = g.idx(i, j, k);
    const float nb = (o.nop == 4) ? nb7(o, g, x, id) : nb27(o, g, x, id);
    y[id] = (o.c[OC][id] + cc[id]) * x[id] - nb;
  }
}

// 8-colour Gauss-Seidel on a 27-point level: colour c = (i&1)|(j&1)<<1|(k&1)<<2.
// One cluster runs nsweep sweeps (colour order ascending, or descending when
// reverse) with a cluster barrier between colours.
template <int CLUSTER>
__global__ void k_gs27_mc_cluster(Grid g, OpF o, const float* __restrict__ cc,
                                  const float* __restrict__ fc, float* x, int nsweep,
                                  int reverse) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  unsigned rank = 0;
  if (CLUSTER > 1) rank = cg::this_cluster().block_rank();
  const int gtid = rank * blockDim.x + threadIdx.x;
  const int nthr = CLUSTER * blockDim.x;
  const int hx = (nx - 1) / 2, hy = (ny - 1) / 2, hz = (nz - 1) / 2;  // slots per axis
  for (int sw = 0; sw < nsweep; sw++) {
    for (int cc8 = 0; cc8 < 8; cc8++) {
      const int c = reverse ? 7 - cc8 : cc8;
      const int pi = c & 1, pj = (c >> 1) & 1, pk = (c >> 2) & 1;
      const int tot = hx * hy * hz;
      for (int t = gtid; t < tot; t += nthr) {
        const int mi = t % hx, mj = (t / hx) % hy, mk = t / (hx * hy);
        // interior index with parity: i = 1 + ((1 + p) & 1) ... first interior
        // index of parity p is 1 if p == 1 else 2
        const int i = (pi ? 1 : 2) + 2 * mi;
        const int j = (pj ? 1 : 2) + 2 * mj;
        const int k = (pk ? 1 : 2) + 2 * mk;
        if (i > nx - 2 || j > ny - 2 || k > nz - 2) continue;
        const size_t id = g.idx(i, j, k);
        x[id] = (fc[id] + nb27(o, g, x, id)) / (o.c[OC][id] + cc[id]);
      }
      if (CLUSTER > 1) cg::this_cluster().sync();
      else __syncthreads();
    }
  }
}

// one colour over the whole grid (large levels)
__global__ void k_gs27_mc_colour(Grid g, OpF o, const float* __restrict__ cc,
                                 const float* __restrict__ fc, float* x, int c) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int hx = (nx - 1) / 2, hy = (ny - 1) / 2, hz = (nz - 1) / 2;
  const int pi = c & 1, pj = (c >> 1) & 1, pk = (c >> 2) & 1;
  const size_t tot = (size_t)hx * hy * hz;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < tot;
       t += (size_t)gridDim.x * blockDim.x) {
    const int mi = (int)(t % hx), mj = (int)((t / hx) % hy), mk = (int)(t / ((size_t)hx * hy));
    const int i = (pi ? 1 : 2) + 2 * mi;
    const int j = (pj ? 1 : 2) + 2 * mj;
    const int k = (pk ? 1 : 2) + 2 * mk;
    if (i > nx - 2 || j > ny - 2 || k > nz - 2) continue;
    const size_t id = g.idx(i, j, k);
    x[id] = (fc[id] + nb27(o, g, x, id)) / (o.c[OC][id] + cc[id]);
  }
}

__global__ void k_restrict_f32(Grid gf, const float* __restrict__ xin, Grid gc, float* xout) {
  const int cx = gc.nx, cy = gc.ny, cz = gc.nz;
  const size_t n = gc.n();
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % cx), j = (int)((q / cx) % cy), k = (int)(q / ((size_t)cx * cy));
    if (i == 0 || j == 0 || k == 0 || i == cx - 1 || j == cy - 1 || k == cz - 1) {
      xout[q] = 0.f;
      continue;
    }
    const int ii = 2 * i, jj = 2 * j, kk = 2 * k;
    float acc = 0.f;
#pragma unroll
    for (int dz = -1; dz <= 1; dz++)
#pragma unroll
      for (int dy = -1; dy <= 1; dy++)
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
          const float w = 1.f / (float)(1 << (abs(dx) + abs(dy) + abs(dz)));
          acc += w * xin[gf.idx(ii + dx, jj + dy, kk + dz)];
        }
    xout[q] = acc;
  }
}

__global__ void k_interp_axpy_f32(Grid gc, const float* __restrict__ xc, Grid gf, float* xf,
                                  const double* num, const double* den) {
  const int nx = gf.nx, ny = gf.ny, nz = gf.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  const float xdamp = (float)(num[0] / den[0]);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(q % (nx - 2));
    const int j = 1 + (int)((q / (nx - 2)) % (ny - 2));
    const int k = 1 + (int)(q / ((size_t)(nx - 2) * (ny - 2)));
    const int ii = i >> 1, jj = j >> 1, kk = k >> 1;
    const int oi = i & 1, oj = j & 1, ok = k & 1;
    float w = 0.f;
    for (int c = 0; c <= ok; c++)
      for (int b = 0; b <= oj; b++)
        for (int a = 0; a <= oi; a++) w += xc[gc.idx(ii + a, jj + b, kk + c)];
    w *= 1.f / (float)(1 << (oi + oj + ok));
    xf[gf.idx(i, j, k)] += xdamp * w;
  }
}

// dot product of FP32 vectors on interior points, FP64 accumulation
__global__ void k_dot_f32(Grid g, const float* __restrict__ x, const float* __restrict__ y,
                          double* part) {
  __shared__ double sh[32];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  double acc = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(q % (nx - 2));
    const int j = 1 + (int)((q / (nx - 2)) % (ny - 2));
    const int k = 1 + (int)(q / ((size_t)(nx - 2) * (ny - 2)));
    const size_t id = g.idx(i, j, k);
    acc += (double)x[id] * (double)y[id];
  }
  const double t = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_sum_parts(const double* __restrict__ part, int n, double* out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += part[i];
  const double t = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) out[0] = t;
}

void dot_f32(cudaStream_t s, Grid g, const float* x, const float* y, double* part,
             double* out) {
  const size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  const int nb = (int)reduce_parts(nint);
  k_dot_f32<<<nb, 256, 0, s>>>(g, x, y, part);
  k_sum_parts<<<1, 256, 0, s>>>(part, nb, out);
}

// FP64 fine residual r = f - (A + cc) x written as the FP32 V-cycle rhs,
// with its FP64 1-norm (partials per block)
__global__ void k_resid64_to32(Grid g, Op op, const double* __restrict__ cc,
                               const double* __restrict__ fc, const double* __restrict__ x,
                               float* r32, double* part) {
  __shared__ double sh[32];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  const size_t sy = nx, sz = (size_t)nx * ny;
  double acc = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(q % (nx - 2));
    const int j = 1 + (int)((q / (nx - 2)) % (ny - 2));
    const int k = 1 + (int)(q / ((size_t)(nx - 2) * (ny - 2)));
    const size_t id = g.idx(i, j, k);
    const double r = fc[id] + op.c[ON][id] * x[id + sy] + op.c[ON][id - sy] * x[id - sy] +
                     op.c[OE][id] * x[id + 1] + op.c[OE][id - 1] * x[id - 1] +
                     op.c[UC][id - sz] * x[id - sz] + op.c[UC][id] * x[id + sz] -
                     (op.c[OC][id] + cc[id]) * x[id];
    r32[id] = (float)r;
    acc += fabs(r);
  }
  const double t = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// x += e on interior points (FP64 accumulation of the FP32 correction)
__global__ void k_add_corr(Grid g, const float* __restrict__ e, double* x) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t nint = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nint;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(q % (nx - 2));
    const int j = 1 + (int)((q / (nx - 2)) % (ny - 2));
    const int k = 1 + (int)(q / ((size_t)(nx - 2) * (ny - 2)));
    const size_t id = g.idx(i, j, k);
    x[id] += (double)e[id];
  }
}

// ---------------------------------------------------------------------------
// coarsest level: dense FP64 Cholesky of (A_c + diag cc) over interior points
// ---------------------------------------------------------------------------
__global__ void k_dense_build(Grid g, Op op, const double* __restrict__ cc, double* M, int n) {
  const int nx = g.nx, ny = g.ny;
  const int ex = nx - 2, ey = ny - 2;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n * n; t += gridDim.x * blockDim.x) {
    const int r = t / n, c = t % n;
    const int ri = 1 + r % ex, rj = 1 + (r / ex) % ey, rk = 1 + r / (ex * ey);
    const int ci = 1 + c % ex, cj = 1 + (c / ex) % ey, ck = 1 + c / (ex * ey);
    const int dx = ci - ri, dy = cj - rj, dz = ck - rk;
    double v = 0.0;
    if (abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1) {
      if (dx == 0 && dy == 0 && dz == 0) {
        v = op.c[OC][g.idx(ri, rj, rk)] + cc[g.idx(ri, rj, rk)];
      } else {
        int si = ri, sj = rj, sk = rk, ax = dx, ay = dy, az = dz;
        if (az < 0 || (az == 0 && ay < 0) || (az == 0 && ay == 0 && ax < 0)) {
          si = ci; sj = cj; sk = ck; ax = -ax; ay = -ay; az = -az;
        }
        int code;
        if (az == 0) code = (ay == 0) ? OE : (ax == 0) ? ON : (ax > 0 ? ONE : ONW);
        else if (ax == 0 && ay == 0) code = UC;
        else if (ay == 0) code = (ax > 0) ? UE : UW;
        else if (ax == 0) code = (ay > 0) ? UN : US;
        else if (ay > 0) code = (ax > 0) ? UNE : UNW;
        else code = (ax > 0) ? USE : USW;
        v = (code < op.nop) ? -op.c[code][g.idx(si, sj, sk)] : 0.0;
      }
    }
    M[t] = v;
  }
}

// In-place Cholesky (lower) by one CTA, right-looking.
__global__ void k_dense_chol(double* M, int n, int* info) {
  __shared__ double piv;
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int j = 0; j < n; j++) {
    if (threadIdx.x == 0) {
      const double d = M[j * n + j];
      if (!(d > 0.0)) bad = j + 1;
      else {
        piv = sqrt(d);
        M[j * n + j] = piv;
      }
    }
    __syncthreads();
    if (bad) break;
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) M[i * n + j] /= piv;
    __syncthreads();
    const int w = n - j - 1;
    for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
      const int a = t / w, b = t % w;
      if (b > a) continue;
      const int i = j + 1 + a, l = j + 1 + b;
      M[i * n + l] -= M[i * n + j] * M[l * n + j];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) info[0] = bad;
}

// x = M^{-1} b on the coarsest level: gather FP32 rhs, two triangular
// solves in FP64 (one warp), scatter to FP32 x (boundary zero).
__global__ void k_dense_solve(Grid g, const double* __restrict__ L, int n,
                              const float* __restrict__ rhs, float* x, double* v) {
  const int nx = g.nx, ny = g.ny;
  const int ex = nx - 2, ey = ny - 2;
  for (int q = threadIdx.x; q < n; q += blockDim.x)
    v[q] = (double)rhs[g.idx(1 + q % ex, 1 + (q / ex) % ey, 1 + q / (ex * ey))];
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    for (int i = 0; i < n; i++) {  // L y = b
      double t = 0.0;
      for (int c = lane; c < i; c += 32) t += L[i * n + c] * v[c];
      t = warp_sum(t);
      if (lane == 0) v[i] = (v[i] - t) / L[i * n + i];
      __syncwarp();
    }
    for (int i = n - 1; i >= 0; i--) {  // L^T x = y
      double t = 0.0;
      for (int c = i + 1 + lane; c < n; c += 32) t += L[c * n + i] * v[c];
      t = warp_sum(t);
      if (lane == 0) v[i] = (v[i] - t) / L[i * n + i];
      __syncwarp();
    }
  }
  __syncthreads();
  for (size_t q = threadIdx.x; q < g.n(); q += blockDim.x) x[q] = 0.f;
  __syncthreads();
  for (int q = threadIdx.x; q < n; q += blockDim.x)
    x[g.idx(1 + q % ex, 1 + (q / ex) % ey, 1 + q / (ex * ey))] = (float)v[q];
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
int mc_cluster_size(Grid g) {
  const size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  if (nint > 200000) return 0;  // grid-wide colour launches
  if (nint > 20000) return 8;
  if (nint > 2000) return 2;
  return 1;
}

int gs27_mc(cudaStream_t s, const MLevel& L, float* x, int nsweep, int reverse, long long& k) {
  const int cl = mc_cluster_size(L.g);
  const OpF o = opf(L);
  if (cl == 0) {
    const size_t tot = (size_t)((L.g.nx - 1) / 2) * ((L.g.ny - 1) / 2) * ((L.g.nz - 1) / 2);
    for (int sw = 0; sw < nsweep; sw++)
      for (int c8 = 0; c8 < 8; c8++) {
        k_gs27_mc_colour<<<blocks_for(tot), kThreads, 0, s>>>(L.g, o, L.cc, L.w0, x,
                                                               reverse ? 7 - c8 : c8);
        k++;
      }
    return 1;
  }
  if (cl == 1) {
    k_gs27_mc_cluster<1><<<1, 512, 0, s>>>(L.g, o, L.cc, L.w0, x, nsweep, reverse);
    k++;
    return 1;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl, 1, 1);
  cfg.blockDim = dim3(1024, 1, 1);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = (cl == 8) ? cudaLaunchKernelEx(&cfg, k_gs27_mc_cluster<8>, L.g, o,
                                                 (const float*)L.cc, (const float*)L.w0, x,
                                                 nsweep, reverse)
                            : cudaLaunchKernelEx(&cfg, k_gs27_mc_cluster<2>, L.g, o,
                                                 (const float*)L.cc, (const float*)L.w0, x,
                                                 nsweep, reverse);
  k++;
  if (e != cudaSuccess) {
    set_error("gs27 multicolour launch: %s", cudaGetErrorString(e));
    return 0;
  }
  return 1;
}

int falloc(float** p, size_t n) {
  if (n == 0) n = 1;
  if (cudaMalloc((void**)p, n * sizeof(float)) != cudaSuccess) {
    set_error("cudaMalloc(%zu floats) failed", n);
    *p = nullptr;
    return 0;
  }
  cudaMemset(*p, 0, n * sizeof(float));
  return 1;
}

int dalloc64(double** p, size_t n) {
  if (n == 0) n = 1;
  if (cudaMalloc((void**)p, n * sizeof(double)) != cudaSuccess) {
    set_error("cudaMalloc(%zu doubles) failed", n);
    *p = nullptr;
    return 0;
  }
  cudaMemset(*p, 0, n * sizeof(double));
  return 1;
}

}  // namespace

void mixed_destroy(MixedState* m) {
  if (!m) return;
  for (int e = 0; e < 2; e++)
    if (m->exec[e]) cudaGraphExecDestroy(m->exec[e]);
  for (int l = 0; l < m->nlev; l++) {
    MLevel& L = m->lev[l];
    for (int c = 0; c < 14; c++) {
      if (L.op[c]) cudaFree(L.op[c]);
      if (L.own64 && L.op64[c]) cudaFree(L.op64[c]);
    }
    if (L.own64 && L.cc64) cudaFree(L.cc64);
    if (L.cc) cudaFree(L.cc);
    if (L.w0) cudaFree(L.w0);
    if (L.x) cudaFree(L.x);
  }
  if (m->r) cudaFree(m->r);
  if (m->w2) cudaFree(m->w2);
  if (m->dense) cudaFree(m->dense);
  if (m->dvec) cudaFree(m->dvec);
  if (m->dinfo) cudaFree(m->dinfo);
  delete m;
}

namespace {

// Build the FP32 hierarchy from the FP64 one (plus extra Galerkin levels).
int mixed_setup(pmgb_solver* s) {
  if (s->mixed) return 1;
  MixedState* m = new MixedState();
  memset(m, 0, sizeof(*m));
  s->mixed = m;
  cudaStream_t st = s->stream;
  // levels shared with the FP64 hierarchy
  int nl = 0;
  for (int l = 0; l < s->nlev; l++, nl++) {
    MLevel& L = m->lev[l];
    L.g = s->lev[l].g;
    L.nop = s->lev[l].nop;
    for (int c = 0; c < L.nop; c++) L.op64[c] = s->lev[l].op[c];
    L.own64 = 0;
    L.cc64 = nullptr;
  }
  // extra coarse levels until <= 512 interior unknowns or the grid cannot
  // be coarsened exactly
  while (nl < 16) {
    const Grid g = m->lev[nl - 1].g;
    const size_t nint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
    if (nint <= 512) break;
    if ((g.nx - 1) % 2 || (g.ny - 1) % 2 || (g.nz - 1) % 2) break;
    const Grid c{(g.nx - 1) / 2 + 1, (g.ny - 1) / 2 + 1, (g.nz - 1) / 2 + 1};
    if (c.nx < 3 || c.ny < 3 || c.nz < 3) break;
    MLevel& L = m->lev[nl];
    L.g = c;
    L.nop = 14;
    L.own64 = 1;
    for (int q = 0; q < 14; q++)
      if (!dalloc64(&L.op64[q], c.n())) return 0;
    if (!dalloc64(&L.cc64, c.n())) return 0;
    nl++;
  }
  m->nlev = nl;
  // Galerkin operators of the extra levels
  double** dptrs = nullptr;
  CKM(cudaMalloc(&dptrs, sizeof(double*) * 14 * 16));
  for (int l = s->nlev; l < nl; l++) {
    CKM(cudaMemcpyAsync(dptrs + 14 * l, m->lev[l].op64, sizeof(double*) * 14,
                        cudaMemcpyHostToDevice, st));
    launch_galerkin(st, m->lev[l - 1].g, m->lev[l - 1].ops64(), m->lev[l].g, dptrs + 14 * l);
    note_launches(1);
  }
  CKM(cudaStreamSynchronize(st));
  cudaFree(dptrs);
  // FP32 storage and conversion
  for (int l = 0; l < nl; l++) {
    MLevel& L = m->lev[l];
    const size_t n = L.g.n();
    for (int c = 0; c < L.nop; c++) {
      if (!falloc(&L.op[c], n)) return 0;
      to_f32(st, L.op64[c], L.op[c], n);
      note_launches(1);
    }
    if (!falloc(&L.cc, n) || !falloc(&L.w0, n) || !falloc(&L.x, n)) return 0;
  }
  if (!falloc(&m->r, s->n) || !falloc(&m->w2, s->n)) return 0;
  const Grid gc = m->lev[nl - 1].g;
  m->nd = (gc.nx - 2) * (gc.ny - 2) * (gc.nz - 2);
  if (m->nd > 4096) {
    set_error("mixed: coarsest level too large (%d unknowns)", m->nd);
    return 0;
  }
  if (!dalloc64(&m->dense, (size_t)m->nd * m->nd) || !dalloc64(&m->dvec, m->nd)) return 0;
  CKM(cudaMalloc(&m->dinfo, sizeof(int) * 4));
  CKM(cudaStreamSynchronize(st));
  return 1;
}

// Helmholtz term on every mixed level from the fine FP64 term cc0:
// restrict through the FP64 levels (where not already present) and convert.
int mixed_set_cc(pmgb_solver* s, int newton) {
  MixedState* m = s->mixed;
  cudaStream_t st = s->stream;
  for (int l = 0; l < m->nlev; l++) {
    MLevel& L = m->lev[l];
    const double* src;
    if (l < s->nlev) {
      src = newton ? s->lev[l].cp : s->lev[l].cc;
    } else {
      const double* prev = (l - 1 < s->nlev) ? (newton ? s->lev[l - 1].cp : s->lev[l - 1].cc)
                                             : m->lev[l - 1].cc64;
      launch_restrict(st, m->lev[l - 1].g, prev, L.g, L.cc64);
      note_launches(1);
      src = L.cc64;
    }
    to_f32(st, src, L.cc, L.g.n());
    note_launches(1);
    if (l == m->nlev - 1) {
      // dense factor of (A_c + cc) on the coarsest level
      const int nd = m->nd;
      k_dense_build<<<blocks_for((size_t)nd * nd), kThreads, 0, st>>>(L.g, L.ops64(), src,
                                                                       m->dense, nd);
      k_dense_chol<<<1, 1024, 0, st>>>(m->dense, nd, m->dinfo);
      note_launches(2);
    }
  }
  int info = 0;
  CKM(cudaMemcpyAsync(&info, m->dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKM(cudaStreamSynchronize(st));
  if (info != 0) {
    set_error("mixed: coarsest operator not positive definite (pivot %d)", info);
    return 0;
  }
  m->cc_ready = 1;
  return 1;
}

// One FP32 V-cycle on A e = w0 (fine rhs already in lev[0].w0), e -> lev[0].x,
// then x64 += e, the FP64 residual of (fc64, cc64, x64) into lev[0].w0 and its
// 1-norm into scal[S_RSNRM].
int mixed_cycle_body(pmgb_solver* s, const double* cc64, const double* fc64, double* x64,
                     long long& k) {
  MixedState* m = s->mixed;
  cudaStream_t st = s->stream;
  const int nl = m->nlev;
  MLevel& F = m->lev[0];
  const OpF fo = opf(F);
  const size_t nslots = (size_t)((F.g.nx - 1) / 2) * (F.g.ny - 2) * (F.g.nz - 2);
  const size_t fint = (size_t)(F.g.nx - 2) * (F.g.ny - 2) * (F.g.nz - 2);
  CKM(cudaMemsetAsync(F.x, 0, F.g.n() * sizeof(float), st));
  for (int sw = 0; sw < 2; sw++) {
    k_gs7_f32<<<blocks_for(nslots), kThreads, 0, st>>>(F.g, fo, F.cc, F.w0, F.x, 1);
    k_gs7_f32<<<blocks_for(nslots), kThreads, 0, st>>>(F.g, fo, F.cc, F.w0, F.x, 0);
    k += 2;
  }
  k_resid_f32<<<blocks_for(fint), kThreads, 0, st>>>(F.g, fo, F.cc, F.w0, F.x, m->r);
  k++;
  for (int l = 1; l < nl; l++) {
    MLevel& C = m->lev[l];
    k_restrict_f32<<<blocks_for(C.g.n()), kThreads, 0, st>>>(m->lev[l - 1].g, m->r, C.g,
                                                             C.w0);
    k++;
    if (l != nl - 1) {
      CKM(cudaMemsetAsync(C.x, 0, C.g.n() * sizeof(float), st));
      if (!gs27_mc(st, C, C.x, 2, 0, k)) return 0;
      const size_t cint = (size_t)(C.g.nx - 2) * (C.g.ny - 2) * (C.g.nz - 2);
      k_resid_f32<<<blocks_for(cint), kThreads, 0, st>>>(C.g, opf(C), C.cc, C.w0, C.x, m->r);
      k++;
    }
  }
  {
    MLevel& C = m->lev[nl - 1];
    k_dense_solve<<<1, 256, 0, st>>>(C.g, m->dense, m->nd, C.w0, C.x, m->dvec);
    k++;
  }
  for (int l = nl - 2; l >= 0; l--) {
    MLevel& C = m->lev[l + 1];
    MLevel& P = m->lev[l];
    const size_t cint = (size_t)(C.g.nx - 2) * (C.g.ny - 2) * (C.g.nz - 2);
    k_matvec_f32<<<blocks_for(cint), kThreads, 0, st>>>(C.g, opf(C), C.cc, C.x, m->w2);
    dot_f32(st, C.g, C.x, C.w0, s->part, s->scal + S_XNUM_L + (l & 15));
    dot_f32(st, C.g, C.x, m->w2, s->part + 2368, s->scal + S_XDEN_L + (l & 15));
    const size_t pint = (size_t)(P.g.nx - 2) * (P.g.ny - 2) * (P.g.nz - 2);
    k_interp_axpy_f32<<<blocks_for(pint), kThreads, 0, st>>>(
        C.g, C.x, P.g, P.x, s->scal + S_XNUM_L + (l & 15), s->scal + S_XDEN_L + (l & 15));
    k += 6;
    if (l == 0) {
      for (int sw = 0; sw < 2; sw++) {
        k_gs7_f32<<<blocks_for(nslots), kThreads, 0, st>>>(F.g, fo, F.cc, F.w0, F.x, 0);
        k_gs7_f32<<<blocks_for(nslots), kThreads, 0, st>>>(F.g, fo, F.cc, F.w0, F.x, 1);
        k += 2;
      }
    } else {
      if (!gs27_mc(st, P, P.x, 2, 1, k)) return 0;
    }
  }
  // x64 += e ; r = f - (A + cc) x64 (FP64) -> FP32 rhs ; ||r||_1
  k_add_corr<<<blocks_for(fint), kThreads, 0, st>>>(F.g, F.x, x64);
  const int nb = (int)reduce_parts(fint);
  k_resid64_to32<<<nb, 256, 0, st>>>(F.g, s->lev[0].ops(), cc64, fc64, x64, F.w0, s->part);
  k_sum_parts<<<1, 256, 0, st>>>(s->part, nb, s->scal + S_RSNRM);
  k += 3;
  return 1;
}

int read_scal(pmgb_solver* s, int slot, double* v) {
  CKM(cudaMemcpyAsync(v, s->scal + slot, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CKM(cudaStreamSynchronize(s->stream));
  return 1;
}

// Refinement loop on (A + cc) x = f, all FP64 vectors on the fine level:
// stop when ||f - (A+cc)x||_1 / rsden <= errtol (rsden = ||f||_1, or 1 for
// the Newton inner solve).
int refine(pmgb_solver* s, int newton, const double* cc64, const double* fc64, double* x64,
           double errtol, int itmax, int istop0, int* iters_out) {
  MixedState* m = s->mixed;
  cudaStream_t st = s->stream;
  const Grid g = s->g;
  const size_t fint = (size_t)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  const int nb = (int)reduce_parts(fint);
  // initial residual (x64 as given) -> FP32 rhs and its norm
  k_resid64_to32<<<nb, 256, 0, st>>>(g, s->lev[0].ops(), cc64, fc64, x64, m->lev[0].w0,
                                     s->part);
  k_sum_parts<<<1, 256, 0, st>>>(s->part, nb, s->scal + S_RSNRM);
  note_launches(2);
  double rsden = 1.0, rsnrm;
  if (!istop0) {
    launch_nrm1(st, g, fc64, s->part + 2368, s->scal + S_RSDEN);
    note_launches(2);
    if (!read_scal(s, S_RSDEN, &rsden)) return 0;
    if (rsden == 0.0) rsden = 1.0;
  }
  if (!read_scal(s, S_RSNRM, &rsnrm)) return 0;
  s->reslog.push_back(istop0 ? 1.0 : rsnrm / rsden);
  if (!m->exec[newton]) {
    cudaGraph_t graph;
    long long k = 0;
    CKM(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int ok = mixed_cycle_body(s, cc64, fc64, x64, k);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (!ok) return 0;
    if (e != cudaSuccess) {
      set_error("mixed graph capture: %s", cudaGetErrorString(e));
      return 0;
    }
    CKM(cudaGraphInstantiate(&m->exec[newton], graph, 0));
    cudaGraphDestroy(graph);
    m->kernels[newton] = k;
  }
  int iters = 0;
  do {
    CKM(cudaGraphLaunch(m->exec[newton], st));
    note_launches(m->kernels[newton]);
    if (!read_scal(s, S_RSNRM, &rsnrm)) return 0;
    iters++;
    s->st.vcycles++;
    s->reslog.push_back(rsnrm / rsden);
    if (!(rsnrm == rsnrm)) {
      set_error("mixed: non-finite residual");
      return 0;
    }
  } while (iters < itmax && (rsnrm / rsden) > errtol);
  s->st.refinements += iters;
  s->st.rel_residual = rsnrm / rsden;
  *iters_out = iters;
  return 1;
}

}  // namespace

// Inner solve of one Newton step (called by the Newton driver in solver.cu
// with s->lev[*].cp and .rhs in place): xt = 0 and refine until
// ||rhs - J xt||_1 <= errtol_s.
int mixed_newton_inner(pmgb_solver* s, double errtol_s) {
  if (!mixed_setup(s)) return 0;
  if (!mixed_set_cc(s, 1)) return 0;
  Level& F = s->lev[0];
  CKM(cudaMemsetAsync(F.xt, 0, s->n * sizeof(double), s->stream));
  int it = 0;
  return refine(s, 1, F.cp, F.rhs, F.xt, errtol_s, 1000, 1, &it);
}

// One FP32 fine-level half-sweep for kernel timing; 6 FP32 arrays read and
// x read/written: 14 B per point per half-sweep.
int mixed_time_gs7(pmgb_solver* s, int parity, double* bytes) {
  if (!mixed_setup(s)) return 0;
  MixedState* m = s->mixed;
  MLevel& F = m->lev[0];
  const size_t nslots = (size_t)((F.g.nx - 1) / 2) * (F.g.ny - 2) * (F.g.nz - 2);
  k_gs7_f32<<<blocks_for(nslots), kThreads, 0, s->stream>>>(F.g, opf(F), F.cc, F.w0, F.x,
                                                            parity);
  *bytes = 14.0 * (double)(F.g.nx - 2) * (F.g.ny - 2) * (F.g.nz - 2);
  return 1;
}

int mixed_solve(pmgb_solver* s, double errtol) {
  if (!mixed_setup(s)) return 0;
  CKM(cudaMemsetAsync(s->lev[0].x, 0, s->n * sizeof(double), s->stream));
  if (!s->p.nonlin) {
    if (!s->mixed->cc_ready && !mixed_set_cc(s, 0)) return 0;
    int it = 0;
    Level& F = s->lev[0];
    return refine(s, 0, F.cc, F.fc, F.x, errtol, 200, 0, &it);
  }
  return newton_driver(s, errtol, 200, 1);
}

}  // namespace pmgb
