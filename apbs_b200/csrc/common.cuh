// Shared device helpers for the B200 PMG kernels.
#pragma once

#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <stdint.h>
#include <stdio.h>

namespace pmgb {

// Stored coefficients of one level operator, in the order of the reference's
// operator array (columns of MAT2(ac, n, 14) in src/pmgc/gsd.c:76-86).
enum Coef { OC = 0, OE, ON, UC, ONE, ONW, UE, UW, UN, US, UNE, UNW, USE, USW };

struct Grid {
  int nx, ny, nz;
  __host__ __device__ size_t n() const { return (size_t)nx * ny * nz; }
  __host__ __device__ size_t idx(int i, int j, int k) const {
    return ((size_t)k * ny + j) * nx + i;
  }
};

// Pointers of one level operator (4 coefficients on the finest level, 14 on
// Galerkin levels).
struct Op {
  const double* c[14];
  int nop;
};

constexpr int kThreads = 256;

inline int blocks_for(size_t n, int threads = kThreads) {
  size_t b = (n + threads - 1) / threads;
  if (b > 148u * 32u) b = 148u * 32u;
  if (b < 1) b = 1;
  return (int)b;
}

// Warp + block sum in a fixed order (deterministic for a fixed launch).
__device__ inline double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// q -> (q % a, (q / a) % b, q / (a b)), with 32-bit divisions while q fits
// (64-bit divisions are long instruction sequences in a grid-stride loop).
__device__ __forceinline__ void split3(size_t q, int a, int b, int& x, int& y, int& z) {
  if (q <= 0xffffffffull) {
    const unsigned u = (unsigned)q, t = u / (unsigned)a, zz = t / (unsigned)b;
    x = (int)(u - t * (unsigned)a);
    y = (int)(t - zz * (unsigned)b);
    z = (int)zz;
  } else {
    const size_t t = q / (size_t)a, zz = t / (size_t)b;
    x = (int)(q - t * (size_t)a);
    y = (int)(t - zz * (size_t)b);
    z = (int)zz;
  }
}

// Interior point q (i fastest) -> (i, j, k), 1-based interior indices, with
// 32-bit divisions where the interior count allows (it does up to 1025^3).
__device__ __forceinline__ void interior_ijk(size_t q, int nx, int ny, int& i, int& j, int& k) {
  const unsigned ex = (unsigned)(nx - 2), ey = (unsigned)(ny - 2);
  if (q <= 0xffffffffull) {
    const unsigned u = (unsigned)q, t = u / ex, kk = t / ey;
    i = 1 + (int)(u - t * ex);
    j = 1 + (int)(t - kk * ey);
    k = 1 + (int)kk;
  } else {
    const size_t t = q / ex, kk = t / ey;
    i = 1 + (int)(q - t * ex);
    j = 1 + (int)(t - kk * ey);
    k = 1 + (int)kk;
  }
}

template <int NT>
__device__ inline double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = (lane < NT / 32) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

}  // namespace pmgb

#define PMGB_CUDA_OK(call)                                                   \
  do {                                                                       \
    cudaError_t e__ = (call);                                                \
    if (e__ != cudaSuccess) {                                                \
      pmgb::set_error("%s:%d CUDA error %s", __FILE__, __LINE__,            \
                      cudaGetErrorString(e__));                              \
      return 0;                                                              \
    }                                                                        \
  } while (0)

namespace pmgb {
void set_error(const char* fmt, ...);
}
