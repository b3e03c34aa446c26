// One full red-black Gauss-Seidel sweep of the 7-point operator in a single
// pass over memory, out of place.
//
// Restates one iteration of Vgsrb7x (src/pmgc/gsd.c:95-164): first every
// point of colour c1 = (i+j+k)&1 is updated from the old values of its six
// neighbours (all of the other colour or on the boundary), then every point
// of colour c2 from the new c1 values, each with the reference's expression.
// Red-black GS on a 7-point stencil has no same-colour coupling, so the order
// inside a colour does not matter and the result equals the colour-pass
// result bit for bit.
//
// Each CTA owns a TX x TY tile of (i, j) columns over a chunk of planes and
// marches up k.  At plane k+1 it computes the new c1 values of the tile and a
// one-point ring around it (the ring is recomputed redundantly by the
// neighbouring tiles) into a three-plane shared-memory ring buffer, then the
// new c2 values of plane k from it.  Old values are
// read only from xin and results are written only to xout, so no CTA
// depends on another and a sweep needs one launch: every array is read from HBM once per sweep (the colour passes
// read each twice), plus the halo re-reads that neighbouring tiles serve
// from L2.  The boundary of xout is never written: it must hold the same
// (zero) boundary as xin.
#pragma once

#include <cuda_pipeline.h>

#include "common.cuh"

namespace pmgb {

template <typename T>
struct Gs7Sweep {
  Grid g;
  const T* oC;
  const T* oE;
  const T* oN;
  const T* uC;
  const T* cc;
  const T* fc;
  const T* xin;
  T* xout;
  int c1;      // colour updated first: (i + j + k) & 1 == c1
  int kchunk;  // planes per CTA
  int* err = nullptr;  // staged sweeps: count of bounded waits that ran out
};

template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX* TY) k_gs7_sweep(Gs7Sweep<T> a) {
  constexpr int RX = TX + 2, RY = TY + 2, RN = RX * RY;
  __shared__ T R[3][RN];  // colour-c1 values (new) and boundary values, tile + ring
  const Grid g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t sy = nx, sz = (size_t)nx * ny;
  const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
  const int k0 = 1 + blockIdx.z * a.kchunk;
  const int k1 = min(k0 + a.kchunk, nz - 1);  // planes k0 .. k1-1
  const int c1 = a.c1;
  const T* __restrict__ x = a.xin;

  // new colour-c1 values (and boundary values) of plane k on tile + ring
  auto first_colour = [&](int k) {
    T* Rk = R[k % 3];
    for (int t = threadIdx.x; t < RN; t += TX * TY) {
      const int i = i0 - 1 + t % RX, j = j0 - 1 + t / RX;
      if (i > nx - 1 || j > ny - 1) continue;
      const size_t id = (size_t)k * sz + (size_t)j * sy + i;
      if (i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1) {
        Rk[t] = x[id];
      } else if (((i + j + k) & 1) == c1) {
        Rk[t] = (a.fc[id] + a.oN[id] * x[id + sy] + a.oN[id - sy] * x[id - sy] +
                 a.oE[id] * x[id + 1] + a.oE[id - 1] * x[id - 1] + a.uC[id - sz] * x[id - sz] +
                 a.uC[id] * x[id + sz]) /
                (a.oC[id] + a.cc[id]);
      }
    }
  };

  first_colour(k0 - 1);
  first_colour(k0);
  const int ti = threadIdx.x % TX, tj = threadIdx.x / TX;
  const int i = i0 + ti, j = j0 + tj;
  const bool mine = (i <= nx - 2) && (j <= ny - 2);
  const int t = (tj + 1) * RX + (ti + 1);
  for (int k = k0; k < k1; k++) {
    first_colour(k + 1);
    __syncthreads();
    if (mine) {
      const size_t id = (size_t)k * sz + (size_t)j * sy + i;
      const T* Rm = R[(k + 2) % 3];  // plane k-1
      const T* R0 = R[k % 3];
      const T* Rp = R[(k + 1) % 3];
      T v;
      if (((i + j + k) & 1) == c1) {
        v = R0[t];
      } else {
        v = (a.fc[id] + a.oN[id] * R0[t + RX] + a.oN[id - sy] * R0[t - RX] +
             a.oE[id] * R0[t + 1] + a.oE[id - 1] * R0[t - 1] + a.uC[id - sz] * Rm[t] +
             a.uC[id] * Rp[t]) /
            (a.oC[id] + a.cc[id]);
      }
      a.xout[id] = v;
    }
    __syncthreads();  // plane k-1's buffer is refilled next
  }
}

// ---------------------------------------------------------------------------
// The same sweep with the plane tiles staged through shared memory by
// asynchronous copies (cp.async through the CUDA pipeline primitives).  Each
// CTA keeps five planes of the seven arrays (x, fc, oC, cc, oE, oN, uC) over
// its tile plus a two-point halo in a ring of shared-memory stages and
// issues the copies of plane k+3 before computing with planes k-1 .. k+2, so
// three planes of loads are in flight while it computes; the arithmetic reads
// the same values in the same order as k_gs7_sweep.
// ---------------------------------------------------------------------------
template <typename T, int TX, int TY>
struct SweepStage {
  static constexpr int WX = TX + 4, WY = TY + 4, WN = WX * WY;  // staged region
  static constexpr int RX = TX + 2, RN = RX * (TY + 2);         // tile + ring
  static constexpr int NA = 7, NS = 5;                          // arrays, stages
  static constexpr size_t bytes = (size_t)(NS * NA * WN + 3 * RN) * sizeof(T);
};

template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX* TY) k_gs7_sweep_async(Gs7Sweep<T> a) {
  using S = SweepStage<T, TX, TY>;
  constexpr int WX = S::WX, WN = S::WN, RX = S::RX, RN = S::RN, NA = S::NA, NS = S::NS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* stage = reinterpret_cast<T*>(smem_raw);  // [NS][NA][WN]
  T* R = stage + NS * NA * WN;                // [3][RN]
  const Grid g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t sy = nx, sz = (size_t)nx * ny;
  const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
  const int k0 = 1 + blockIdx.z * a.kchunk;
  const int k1 = min(k0 + a.kchunk, nz - 1);
  const int c1 = a.c1;
  const T* src[NA] = {a.xin, a.fc, a.oC, a.cc, a.oE, a.oN, a.uC};
  enum { AX = 0, AF, AO, AC, AE, AN, AU };
  auto arr = [&](int p, int ai) { return stage + ((p % NS + NS) % NS) * NA * WN + ai * WN; };

  // copies of plane p (region i0-2 .. i0+TX+1, j0-2 .. j0+TY+1), one group
  auto issue = [&](int p) {
    if (p >= 0 && p <= nz - 1) {
      for (int e = threadIdx.x; e < NA * WN; e += TX * TY) {
        const int ai = e / WN, q = e - ai * WN;
        const int i = i0 - 2 + q % WX, j = j0 - 2 + q / WX;
        if (i < 0 || j < 0 || i > nx - 1 || j > ny - 1) continue;
        __pipeline_memcpy_async(arr(p, ai) + q, src[ai] + (size_t)p * sz + (size_t)j * sy + i,
                                sizeof(T));
      }
    }
    __pipeline_commit();
  };
  // new colour-c1 values (and boundary values) of plane p on tile + ring
  auto first_colour = [&](int p) {
    T* Rp = R + (p % 3) * RN;
    const T* X0 = arr(p, AX);
    for (int t = threadIdx.x; t < RN; t += TX * TY) {
      const int i = i0 - 1 + t % RX, j = j0 - 1 + t / RX;
      if (i > nx - 1 || j > ny - 1) continue;
      const int q = (t / RX + 1) * WX + (t % RX + 1);
      if (i == 0 || j == 0 || p == 0 || i == nx - 1 || j == ny - 1 || p == nz - 1) {
        Rp[t] = X0[q];
      } else if (((i + j + p) & 1) == c1) {
        const T* Xm = arr(p - 1, AX);
        const T* Xp = arr(p + 1, AX);
        const T* ON_ = arr(p, AN);
        const T* OE_ = arr(p, AE);
        Rp[t] = (arr(p, AF)[q] + ON_[q] * X0[q + WX] + ON_[q - WX] * X0[q - WX] +
                 OE_[q] * X0[q + 1] + OE_[q - 1] * X0[q - 1] + arr(p - 1, AU)[q] * Xm[q] +
                 arr(p, AU)[q] * Xp[q]) /
                (arr(p, AO)[q] + arr(p, AC)[q]);
      }
    }
  };

  for (int p = k0 - 2; p <= k0 + 2; p++) issue(p);
  __pipeline_wait_prior(1);  // planes k0-2 .. k0+1
  __syncthreads();
  first_colour(k0 - 1);
  first_colour(k0);
  __syncthreads();
  const int ti = threadIdx.x % TX, tj = threadIdx.x / TX;
  const int i = i0 + ti, j = j0 + tj;
  const bool mine = (i <= nx - 2) && (j <= ny - 2);
  const int t = (tj + 1) * RX + (ti + 1);
  const int q = (tj + 2) * WX + (ti + 2);
  for (int k = k0; k < k1; k++) {
    issue(k + 3);             // into the stage plane k-2 used
    __pipeline_wait_prior(1);  // planes up to k+2
    __syncthreads();
    first_colour(k + 1);
    __syncthreads();
    if (mine) {
      const size_t id = (size_t)k * sz + (size_t)j * sy + i;
      const T* Rm = R + ((k + 2) % 3) * RN;  // plane k-1
      const T* R0 = R + (k % 3) * RN;
      const T* Rp = R + ((k + 1) % 3) * RN;
      T v;
      if (((i + j + k) & 1) == c1) {
        v = R0[t];
      } else {
        const T* ON_ = arr(k, AN);
        const T* OE_ = arr(k, AE);
        v = (arr(k, AF)[q] + ON_[q] * R0[t + RX] + ON_[q - WX] * R0[t - RX] +
             OE_[q] * R0[t + 1] + OE_[q - 1] * R0[t - 1] + arr(k - 1, AU)[q] * Rm[t] +
             arr(k, AU)[q] * Rp[t]) /
            (arr(k, AO)[q] + arr(k, AC)[q]);
      }
      a.xout[id] = v;
    }
    __syncthreads();  // stage k-1 and R of plane k-1 are refilled next
  }
  __pipeline_wait_prior(0);
}

template <typename T, int TX, int TY>
inline cudaError_t launch_gs7_sweep_async(cudaStream_t s, const Gs7Sweep<T>& a0) {
  using S = SweepStage<T, TX, TY>;
  static const cudaError_t attr = cudaFuncSetAttribute(
      k_gs7_sweep_async<T, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
  if (attr != cudaSuccess) return attr;
  Gs7Sweep<T> a = a0;
  const Grid g = a.g;
  if (a.kchunk < 1) a.kchunk = 16;
  dim3 grid((g.nx - 2 + TX - 1) / TX, (g.ny - 2 + TY - 1) / TY,
            (g.nz - 2 + a.kchunk - 1) / a.kchunk);
  k_gs7_sweep_async<T, TX, TY><<<grid, TX * TY, S::bytes, s>>>(a);
  return cudaGetLastError();
}

// TX x TY tile per CTA, a.kchunk planes per CTA (16 gives a few thousand
// CTAs on the fine grids; each chunk recomputes one plane of the first
// colour below it).
template <typename T, int TX, int TY>
inline cudaError_t launch_gs7_sweep(cudaStream_t s, const Gs7Sweep<T>& a0) {
  Gs7Sweep<T> a = a0;
  const Grid g = a.g;
  if (a.kchunk < 1) a.kchunk = 16;
  dim3 grid((g.nx - 2 + TX - 1) / TX, (g.ny - 2 + TY - 1) / TY,
            (g.nz - 2 + a.kchunk - 1) / a.kchunk);
  k_gs7_sweep<T, TX, TY><<<grid, TX * TY, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace pmgb
