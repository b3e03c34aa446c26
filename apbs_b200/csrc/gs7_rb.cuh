// One full red-black Gauss-Seidel sweep of the fine-level 7-point operator in
// a single pass over memory, out of place (xin -> xout).
//
// Restates one iteration of Vgsrb7x (src/pmgc/gsd.c:95-164): every point of
// the first colour C1 is updated from the old values of its six neighbours,
// then every point of the other colour from the new C1 values, each with
// the reference's expression
//   x = (f + oN[p] x[p+nx] + oN[p-nx] x[p-nx] + oE[p] x[p+1] + oE[p-1] x[p-1]
//          + uC[p-S] x[p-S] + uC[p] x[p+S]) / (oC[p] + cc[p]),
// with the diagonal oC + cc read from one array D that holds that sum
// (the same FP64 addition, made once per operator).  The FP32 instance used
// by the mixed-precision inner cycles sums the six products first, as the
// FP32 colour passes do (f + (oN x + ... + uC x)).  There is no
// same-colour coupling, so the order inside a colour does not matter and
// the sweep equals the two colour passes bit for bit.
//
// The grid is handled as a flat array.  PMG grids have odd nx and ny, so
// the flat index p = (k ny + j) nx + i has the parity of i + j + k: the
// colour of a point is the parity of its flat index, and every 16-byte pair
// (2m, 2m+1) holds one point of each colour.  A thread owns pair slots; in
// each colour phase it updates the one element of the colour, so no lane
// idles on a colour test.
//
// Boundary points need no test either.  The operator's couplings of a
// boundary point and towards it are zero (VbuildA_fv folds the Dirichlet
// values into f, buildAd.c:241-274), f is zero there and D holds 1 there,
// so the same expression gives the boundary value 0.  The caller keeps the
// zero boundary of the fine-level iterate, as the reference does until the
// Dirichlet restore at the end of the solve (mgdrvd.c:557).
//
// A CTA owns a flat range of `core` points of every plane of a chunk of
// planes and marches up k.  Iteration k computes the new C1 values of plane
// k+1 over the core range widened by nx + 1 points on each side (the C1
// neighbours at p +- 1 and p +- nx of the core) into a three-plane ring in
// shared memory, then the new second-colour values of plane k's core from
// that ring, and writes both colours of plane k.  Reads of the old iterate
// come only from xin and results go only to xout, so no CTA depends on
// another.  All offsets are 32-bit (the host keeps grids below 2^31 bytes).
#pragma once

#include <algorithm>

#include "common.cuh"

namespace pmgb {

template <typename T>
struct Gs7Rb {
  const T* oE;
  const T* oN;
  const T* uC;
  const T* D;   // oC + cc, and 1 on boundary points
  const T* f;
  const T* xin;
  T* xout;
  int nx, S, nz;  // row length, plane size nx*ny, planes
  int core;       // core points of a CTA per plane (even)
  int E;          // pair slots of the widened range (shared-memory ring width)
  int kchunk;     // planes per CTA (0: as many chunks as fill the resident CTA slots)
};

// pair slot e of plane k covers flat indices 2 (base(k) + e) and 2 (base(k) + e) + 1
__device__ __forceinline__ int rb_base(int k, int S, int c0, int nx) {
  return (k * S + c0 - nx - 1) >> 1;  // floor, also for the negative first value
}

// the point update: FP64 in the reference's order (gsd.c:127-135), FP32 as
// the mixed path's colour passes
template <typename T>
__device__ __forceinline__ T rb_update(T f, T n1, T xn, T n0, T xs, T e1, T xe, T e0, T xw,
                                       T d0, T xd, T u1, T xu, T dg) {
  if constexpr (sizeof(T) == 8)
    return (f + n1 * xn + n0 * xs + e1 * xe + e0 * xw + d0 * xd + u1 * xu) / dg;
  else
    return (f + (n1 * xn + n0 * xs + e1 * xe + e0 * xw + d0 * xd + u1 * xu)) / dg;
}

// Q pair slots per thread (E = NT Q): the slot loops are unrolled so the
// loads of all of a thread's slots are in flight together.
template <typename T, int C1, int NT, int Q>
__global__ void __launch_bounds__(NT) k_gs7_rb(Gs7Rb<T> a) {
  constexpr int C2 = 1 - C1;
  extern __shared__ __align__(16) unsigned char rb_smem[];
  T* R = reinterpret_cast<T*>(rb_smem);  // [3][E]: new C1 values by pair slot
  const int nx = a.nx, S = a.S, E = a.E;
  const int c0 = blockIdx.x * a.core;
  const int c1e = min(c0 + a.core, S);
  const int k0 = 1 + blockIdx.y * a.kchunk;
  const int k1 = min(k0 + a.kchunk, a.nz - 1);
  const T* __restrict__ oE = a.oE;
  const T* __restrict__ oN = a.oN;
  const T* __restrict__ uC = a.uC;
  const T* __restrict__ D = a.D;
  const T* __restrict__ f = a.f;
  const T* __restrict__ x = a.xin;

  // new C1 values of plane k on the widened range -> ring slot k % 3
  auto phase_a = [&](int k) {
    T* Rk = R + (k % 3) * E;
    const int m0 = rb_base(k, S, c0, nx);
    const int lo = k * S, hi = lo + S;
    const bool boundary_plane = (k == 0) || (k == a.nz - 1);
#pragma unroll
    for (int r = 0; r < Q; r++) {
      const int e = threadIdx.x + r * NT;
      const int p = 2 * (m0 + e) + C1;
      T v = T(0);
      if (!boundary_plane && p >= lo && p < hi) {
        v = rb_update<T>(f[p], oN[p], x[p + nx], oN[p - nx], x[p - nx], oE[p], x[p + 1],
                         oE[p - 1], x[p - 1], uC[p - S], x[p - S], uC[p], x[p + S], D[p]);
      }
      Rk[e] = v;
    }
  };

  phase_a(k0 - 1);
  phase_a(k0);
  // slot offsets of the C1 neighbours of a second-colour point of pair m:
  // the neighbour at p + d (d odd) is the C1 element of pair m + (d + C2 - C1)/2
  constexpr int dW = (C2 - C1 - 1) / 2, dE = (C2 - C1 + 1) / 2;
  const int dS = (C2 - C1 - nx) / 2, dN = (C2 - C1 + nx) / 2;
  for (int k = k0; k < k1; k++) {
    phase_a(k + 1);
    __syncthreads();
    const T* Rm = R + ((k + 2) % 3) * E;  // plane k-1
    const T* R0 = R + (k % 3) * E;
    const T* Rp = R + ((k + 1) % 3) * E;
    const int m0 = rb_base(k, S, c0, nx);
    // slot of the same in-plane position on planes k-1 and k+1
    const int dD = m0 + (C2 - C1 - S) / 2 - rb_base(k - 1, S, c0, nx);
    const int dU = m0 + (C2 - C1 + S) / 2 - rb_base(k + 1, S, c0, nx);
    const int lo = k * S + c0, hi = k * S + c1e;
    T* __restrict__ xo = a.xout;
#pragma unroll
    for (int r = 0; r < Q; r++) {
      const int e = threadIdx.x + r * NT;
      const int m = m0 + e;
      const int p2 = 2 * m + C2;
      const int p1 = 2 * m + C1;
      const bool in2 = (p2 >= lo) && (p2 < hi);
      const bool in1 = (p1 >= lo) && (p1 < hi);
      if (!in1 && !in2) continue;
      const T v1 = R0[e];
      T v2 = T(0);
      if (in2) {
        v2 = rb_update<T>(f[p2], oN[p2], R0[e + dN], oN[p2 - nx], R0[e + dS], oE[p2],
                          R0[e + dE], oE[p2 - 1], R0[e + dW], uC[p2 - S], Rm[e + dD], uC[p2],
                          Rp[e + dU], D[p2]);
      }
      if (in1 && in2) {
        if constexpr (sizeof(T) == 8) {
          double2 w;
          w.x = C1 == 0 ? (double)v1 : (double)v2;
          w.y = C1 == 0 ? (double)v2 : (double)v1;
          *reinterpret_cast<double2*>(xo + 2 * m) = w;
        } else {
          float2 w;
          w.x = C1 == 0 ? (float)v1 : (float)v2;
          w.y = C1 == 0 ? (float)v2 : (float)v1;
          *reinterpret_cast<float2*>(xo + 2 * m) = w;
        }
      } else if (in1) {
        xo[p1] = v1;
      } else {
        xo[p2] = v2;
      }
    }
    __syncthreads();  // plane k-1's slot is refilled next
  }
}

// Pair slots and core length for NT threads with Q slots each: the widened
// range must hold core/2 + nx + 2 pairs.
inline int gs7_rb_core(int nx, int S, int slots) {
  int core = 2 * (slots - nx - 3);
  if (core < 2) return 0;
  return core > S ? ((S + 1) & ~1) : core;
}

// CTAs of one instance resident on the device at once (SMs x CTAs per SM)
template <typename T, int C1, int NT, int Q>
inline int gs7_rb_slots(size_t smem) {
  static const int slots = [smem] {
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_gs7_rb<T, C1, NT, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         96 * 1024);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs7_rb<T, C1, NT, Q>, NT,
                                                      smem) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    return sms * per_sm;
  }();
  return slots;
}

template <typename T, int NT, int Q>
inline cudaError_t launch_gs7_rb_q(cudaStream_t st, Gs7Rb<T> a, int c1) {
  a.E = NT * Q;
  a.core = gs7_rb_core(a.nx, a.S, a.E);
  if (a.core == 0) return cudaErrorInvalidValue;
  const size_t smem = (size_t)3 * a.E * sizeof(T);
  if (a.kchunk <= 0) {
    // one wave: as many plane chunks per flat range as the resident CTA
    // slots allow (the last wave of an uneven split leaves SMs idle)
    const int nranges = (a.S + a.core - 1) / a.core;
    const int slots = gs7_rb_slots<T, 0, NT, Q>(smem);
    const int nchunks = std::max(1, slots / nranges);
    a.kchunk = std::max(1, (a.nz - 2 + nchunks - 1) / nchunks);
  }
  const dim3 grid((a.S + a.core - 1) / a.core, (a.nz - 2 + a.kchunk - 1) / a.kchunk);
  if (c1) {
    static const cudaError_t attr = cudaFuncSetAttribute(
        k_gs7_rb<T, 1, NT, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    if (attr != cudaSuccess) return attr;
    k_gs7_rb<T, 1, NT, Q><<<grid, NT, smem, st>>>(a);
  } else {
    static const cudaError_t attr = cudaFuncSetAttribute(
        k_gs7_rb<T, 0, NT, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    if (attr != cudaSuccess) return attr;
    k_gs7_rb<T, 0, NT, Q><<<grid, NT, smem, st>>>(a);
  }
  return cudaGetLastError();
}

template <typename T, int NT>
inline cudaError_t launch_gs7_rb_nt(cudaStream_t st, const Gs7Rb<T>& a, int c1, int q) {
  switch (q) {
    case 1: return launch_gs7_rb_q<T, NT, 1>(st, a, c1);
    case 2: return launch_gs7_rb_q<T, NT, 2>(st, a, c1);
    case 3: return launch_gs7_rb_q<T, NT, 3>(st, a, c1);
    case 4: return launch_gs7_rb_q<T, NT, 4>(st, a, c1);
    default: return cudaErrorInvalidValue;
  }
}

// shape: bits 0-3 threads per CTA (0: 256, 1: 512, 2: 1024), bits 4-7 pair
// slots per thread (1-4, 0: 2); a CTA's widened range is threads x slots pairs
template <typename T>
inline cudaError_t launch_gs7_rb(cudaStream_t st, const Gs7Rb<T>& a, int c1, int shape) {
  const int nt = shape & 15, q = ((shape >> 4) & 15) ? ((shape >> 4) & 15) : 2;
  if (a.kchunk < 0 || (a.nx & 1) == 0 || (a.S & 1) == 0 ||
      (double)a.S * a.nz * sizeof(T) >= 2147483647.0)
    return cudaErrorInvalidValue;
  switch (nt) {
    case 1: return launch_gs7_rb_nt<T, 512>(st, a, c1, q);
    case 2: return launch_gs7_rb_nt<T, 1024>(st, a, c1, q);
    default: return launch_gs7_rb_nt<T, 256>(st, a, c1, q);
  }
}

}  // namespace pmgb
