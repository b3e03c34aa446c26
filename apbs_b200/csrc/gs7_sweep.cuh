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
