// One full red-black Gauss-Seidel sweep of the 7-point operator in a single
// pass over memory, out of place, with one thread per (i, j) column.
//
// Restates one iteration of Vgsrb7x (src/pmgc/gsd.c:95-164) like
// k_gs7_sweep: every point of colour c1 = (i+j+k)&1 is updated from the old
// values of its six neighbours, then every point of colour c2 from the new c1
// values, each with the reference's expression and operand order, so the
// result equals the colour passes bit for bit.
//
// A CTA owns a TX x TY tile of columns and a chunk of planes.  Its threads
// cover the tile plus a two-point ring of columns; each thread owns one
// column and marches up k.  At step q a thread
//   * publishes its column's old x, oE and oN of plane q in shared memory,
//   * (tile and inner ring) computes the new c1 value of its column at plane
//     q (boundary columns and planes keep x), from old x of the in-plane
//     neighbours (shared memory) and of planes q-1, q+1 (its own registers),
//   * (tile) computes the new c2 value at plane q-1 from the new c1 values of
//     its in-plane neighbours (shared memory) and of planes q-2, q (its own
//     registers), and writes the plane q-1 result.
// The outer ring only supplies old x, oE and oN to the inner ring.  A
// thread's own column arrays are loaded into registers three (coefficients)
// and four (x) planes ahead of use, in a window that rotates by renaming
// (the march is unrolled by six), and the shared-memory values rotate
// through three slots, so one block barrier per plane suffices.  Threads are
// grouped by the parity of i+j, so the lanes of a warp take the same colour
// branch at every plane.  The boundary of xout is never written: it must
// hold the same boundary as xin.
#pragma once

#include "common.cuh"
#include "gs7_sweep.cuh"
#include "gs7_pairs.cuh"
#include "gs7_bulk.cuh"

namespace pmgb {

template <int TX, int TY>
struct MarchShape {
  static constexpr int RX = TX + 4, RY = TY + 4, RN = RX * RY;  // tile + 2-point ring
  static constexpr int HX = RX / 2;                             // columns per parity per row
  static constexpr int NG = (RN / 2 + 31) / 32 * 32;           // threads per parity group
  static constexpr int NT = 2 * NG;
  static_assert(TX % 2 == 0 && TY % 2 == 0, "tile sides must be even");
};

template <typename T>
struct ColCoef {
  T fc, oc, cc, oe, on, uc;
};

template <typename T, int TX, int TY>
__global__ void __launch_bounds__(MarchShape<TX, TY>::NT, 1) k_gs7_march(Gs7Sweep<T> a) {
  using S = MarchShape<TX, TY>;
  constexpr int RX = S::RX, RY = S::RY, RN = S::RN, HX = S::HX, NG = S::NG;
  extern __shared__ __align__(16) unsigned char march_smem[];
  T* X1 = reinterpret_cast<T*>(march_smem);  // [3][RN] old x of a plane
  T* EE = X1 + 3 * RN;                        // [3][RN] oE
  T* NN = EE + 3 * RN;                        // [3][RN] oN
  T* C1 = NN + 3 * RN;                        // [3][RN] new c1 values (boundary: x)
  const Grid g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t sz = (size_t)nx * ny;
  const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
  const int k0 = 1 + blockIdx.z * a.kchunk;
  const int k1 = min(k0 + a.kchunk, nz - 1);  // output planes k0 .. k1-1
  const int c1 = a.c1;

  // this thread's column: parity group, then row-major among that parity
  const int par = threadIdx.x / NG, m = threadIdx.x - par * NG;
  const int rj = m / HX;
  const int ri = 2 * (m - rj * HX) + ((rj & 1) ^ par);
  const int i = i0 - 2 + ri, j = j0 - 2 + rj;  // (i + j) & 1 == par
  const bool valid = m < RN / 2 && i >= 0 && j >= 0 && i <= nx - 1 && j <= ny - 1;
  const bool inner = ri >= 1 && ri <= RX - 2 && rj >= 1 && rj <= RY - 2;
  const bool bcol = i == 0 || j == 0 || i == nx - 1 || j == ny - 1;
  const bool upd = valid && inner;                 // computes c1 values
  const bool full = upd && !bcol;                  // loads every array
  const bool tile = valid && ri >= 2 && ri <= TX + 1 && rj >= 2 && rj <= TY + 1 &&
                    i <= nx - 2 && j <= ny - 2;    // computes c2 values and writes
  const int t = rj * RX + ri;
  const size_t col = (size_t)j * nx + i;

  auto load_x = [&](int p) -> T {
    return (valid && p >= 0 && p <= nz - 1) ? __ldg(a.xin + (size_t)p * sz + col) : T(0);
  };
  auto load_c = [&](int p, ColCoef<T>& c) {
    c.fc = c.oc = c.cc = c.oe = c.on = c.uc = T(0);
    if (!valid || p < 0 || p > nz - 1) return;
    const size_t id = (size_t)p * sz + col;
    c.oe = __ldg(a.oE + id);
    c.on = __ldg(a.oN + id);
    if (full) {
      c.uc = __ldg(a.uC + id);
      c.fc = __ldg(a.fc + id);
      c.oc = __ldg(a.oC + id);
      c.cc = __ldg(a.cc + id);
    }
  };

  const int qa = k0 - 1, qb = k1;  // c1 planes computed: qa .. qb
  // Register window, unrolled by six so that it rotates by renaming: at step
  // u (plane q), cs[u%3] holds the coefficients of plane q and cs[(u+1)%3],
  // cs[(u+2)%3] those of planes q+1, q+2 (in flight); xs[(u+d)%6] holds old x
  // of plane q-1+d.  After the step, plane q+3's coefficients go to cs[u%3]
  // and plane q+5's x to xs[u%6].
  ColCoef<T> cs[3];
  T xs[6];
  T fm1 = 0, om1 = 0, cm1 = 0, um1 = 0;  // fc, oC, cc, uC of plane q-1
  T um2 = 0;                             // uC of plane q-2
  {
    ColCoef<T> cprev;
    load_c(qa - 1, cprev);
    fm1 = cprev.fc; om1 = cprev.oc; cm1 = cprev.cc; um1 = cprev.uc;
  }
#pragma unroll
  for (int d = 0; d < 3; d++) load_c(qa + d, cs[d]);
#pragma unroll
  for (int d = 0; d < 6; d++) xs[d] = load_x(qa - 1 + d);
  T n1m2 = 0, n1m1 = 0, n1q = 0;  // new c1 values of planes q-2, q-1, q
  int s = 0, sm1 = 2;             // slots of planes q and q-1
  for (int q0 = qa; q0 <= qb; q0 += 6) {
#pragma unroll
    for (int u = 0; u < 6; u++) {
      const int q = q0 + u;
      if (q > qb) break;
      ColCoef<T>& c0 = cs[u % 3];
      const T xm1 = xs[u % 6], x0 = xs[(u + 1) % 6], xp1 = xs[(u + 2) % 6];
      if (valid) {
        X1[s * RN + t] = x0;
        EE[s * RN + t] = c0.oe;
        NN[s * RN + t] = c0.on;
      }
      __syncthreads();
      if (upd) {
        if (bcol || q == 0 || q == nz - 1) {
          n1q = x0;
          C1[s * RN + t] = n1q;
        } else if (((par + q) & 1) == c1) {
          const T* X = X1 + s * RN;
          n1q = (c0.fc + c0.on * X[t + RX] + NN[s * RN + t - RX] * X[t - RX] +
                 c0.oe * X[t + 1] + EE[s * RN + t - 1] * X[t - 1] + um1 * xm1 + c0.uc * xp1) /
                (c0.oc + c0.cc);
          C1[s * RN + t] = n1q;
        }
      }
      const int k = q - 1;
      if (tile && k >= k0 && k < k1) {
        T v;
        if (((par + k) & 1) == c1) {
          v = n1m1;
        } else {
          const T* R = C1 + sm1 * RN;
          v = (fm1 + NN[sm1 * RN + t] * R[t + RX] + NN[sm1 * RN + t - RX] * R[t - RX] +
               EE[sm1 * RN + t] * R[t + 1] + EE[sm1 * RN + t - 1] * R[t - 1] + um2 * n1m2 +
               um1 * n1q) /
              (om1 + cm1);
        }
        a.xout[(size_t)k * sz + col] = v;
      }
      // slide the window one plane up and fetch the next planes
      um2 = um1;
      fm1 = c0.fc; om1 = c0.oc; cm1 = c0.cc; um1 = c0.uc;
      load_c(q + 3, c0);
      xs[u % 6] = load_x(q + 5);
      n1m2 = n1m1;
      n1m1 = n1q;
      sm1 = s;
      s = (s == 2) ? 0 : s + 1;
    }
  }
}

template <typename T, int TX, int TY>
inline cudaError_t launch_gs7_march(cudaStream_t st, const Gs7Sweep<T>& a0) {
  using S = MarchShape<TX, TY>;
  Gs7Sweep<T> a = a0;
  const Grid g = a.g;
  if (a.kchunk < 1) a.kchunk = 16;
  const size_t smem = (size_t)12 * S::RN * sizeof(T);
  static const cudaError_t attr = cudaFuncSetAttribute(
      k_gs7_march<T, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (attr != cudaSuccess) return attr;
  dim3 grid((g.nx - 2 + TX - 1) / TX, (g.ny - 2 + TY - 1) / TY,
            (g.nz - 2 + a.kchunk - 1) / a.kchunk);
  k_gs7_march<T, TX, TY><<<grid, S::NT, smem, st>>>(a);
  return cudaGetLastError();
}

// The single-pass sweep kernels by PMGB_TUNE_GS7_SWEEP_KERNEL: 0 = ring tiles
// (k_gs7_sweep), 1 = ring tiles staged by cp.async, 2 = column march on 32x16
// tiles (32x8 in FP64, whose window needs more registers), 3 = column march
// on 32x8 tiles, 4 = whole-row pair tiles (k_gs7_sweep_pairs) of up to 768
// threads, 5 = the same with the next plane's coefficients loaded one step
// ahead, 6 and 7 = pair tiles of 4 and 5 rows (2 tile rows and 3, several
// CTAs per SM), 8 and 9 = FP64 pair tiles staged by bulk asynchronous row
// copies (k_gs7_sweep_bulk; 4 x planes and 2 coefficient planes resident, or
// 5 and 3; FP32 runs kernel 4).  A grid the pair
// kernel does not take (even row length, rows of more than 1534 points,
// arrays not pair-aligned) runs the ring-tile kernel.
template <typename T>
inline cudaError_t launch_gs7_sweep_kernel(cudaStream_t st, const Gs7Sweep<T>& a, int kernel) {
  if (kernel == 8 || kernel == 9) {
    cudaError_t e = cudaErrorNotSupported;
    if constexpr (sizeof(T) == 8)
      e = kernel == 8 ? launch_gs7_sweep_bulk<4, 2>(st, a, a.err)
                      : launch_gs7_sweep_bulk<5, 3>(st, a, a.err);
    if (e != cudaErrorNotSupported) return e;
    kernel = 4;
  }
  if (kernel >= 4 && kernel <= 7) {
    const cudaError_t e = kernel == 5   ? launch_gs7_sweep_pairs<T, true>(st, a)
                          : kernel == 6 ? launch_gs7_sweep_pairs<T, false>(st, a, 4)
                          : kernel == 7 ? launch_gs7_sweep_pairs<T, false>(st, a, 5)
                                        : launch_gs7_sweep_pairs<T, false>(st, a);
    if (e != cudaErrorNotSupported) return e;
    kernel = 0;
  }
  switch (kernel) {
    case 1: return launch_gs7_sweep_async<T, 32, 8>(st, a);
    case 2: return sizeof(T) == 8 ? launch_gs7_march<T, 32, 8>(st, a)
                                  : launch_gs7_march<T, 32, 16>(st, a);
    case 3: return launch_gs7_march<T, 32, 8>(st, a);
    default: return launch_gs7_sweep<T, 32, 8>(st, a);
  }
}

}  // namespace pmgb
