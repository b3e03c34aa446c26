// One full red-black Gauss-Seidel sweep of the 7-point operator in a single
// pass, out of place, with every memory access a 16-byte (FP64) or 8-byte
// (FP32) pair load or store.
//
// Restates one iteration of Vgsrb7x (src/pmgc/gsd.c:95-164) exactly as
// k_gs7_sweep does (same expressions, same operand order), so the result is
// bitwise the colour-pass result.
//
// Pairs.  PMG grids have odd nx and ny (c * 2^k + 1 points per axis), so the
// flat index (k*ny + j)*nx + i has the parity of i + j + k: the colour of a
// point is the parity of its flat index.  The aligned pair of flat indices
// (2m, 2m+1) therefore always holds one colour-0 point (element 0) and one
// colour-1 point (element 1).  In row (j, k) with s = (j + k) & 1, pair q
// covers i = 2q - s and 2q - s + 1; (nx + 1) / 2 pairs cover the row (one
// element of the first or last pair lies in the neighbouring row and is left
// alone).  A neighbour of element e in the row or plane next door is element
// 1 - e of pair q - s + e there.
//
// Work split.  A CTA owns whole rows: threadIdx.x is the pair, threadIdx.y
// one of ty tile rows plus a ring row on either side, and it marches up a
// chunk of planes.  At plane P it computes the new colour-c1 values of all
// its rows (ring rows included) into a three-plane shared-memory ring R,
// with the old x values of planes P-1, P, P+1 staged in a second ring XS;
// then the new colour-c2 values of plane P-1 on the tile rows from R.  Old
// values are read only from xin and results go only to xout, so CTAs are
// independent.  Each array is read from HBM once per sweep; the ring rows
// are re-read from L2 by the neighbouring CTA.  The boundary of xout is
// never written: it must hold the same (zero) boundary as xin.
//
// PF = true loads the next plane's coefficient pairs one step ahead.
#pragma once

#include "common.cuh"
#include "gs7_sweep.cuh"

namespace pmgb {

template <typename T> struct PairOf;
template <> struct PairOf<double> { typedef double2 type; };
template <> struct PairOf<float> { typedef float2 type; };

template <int E, typename V>
__device__ __forceinline__ auto pelem(const V& v) -> decltype(v.x) {
  if constexpr (E == 0) return v.x; else return v.y;
}

template <typename V>
__device__ __forceinline__ V pzero() {
  V v;
  v.x = 0;
  v.y = 0;
  return v;
}

template <typename T>
struct PairCoef {
  typename PairOf<T>::type f, o, c, e, n, u;
};

constexpr int kPairThreads = 768;

template <typename T, int C1, bool PF>
__global__ void __launch_bounds__(kPairThreads, 1) k_gs7_sweep_pairs(Gs7Sweep<T> a, int ty) {
  using V = typename PairOf<T>::type;
  constexpr int E1 = C1, E2 = 1 - C1;  // pair element of colour c1 / c2
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int RW = blockDim.x, NY = blockDim.y;
  V* XS = reinterpret_cast<V*>(smem_raw);  // [3][NY][RW] old x
  V* R = XS + 3 * NY * RW;                 // [3][NY][RW] new c1 values, boundary values
  const Grid g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long sy = nx, sz = (long long)nx * ny, N = sz * nz;
  const int W = (nx + 1) / 2;
  const int q = threadIdx.x, y = threadIdx.y;
  const int j = blockIdx.x * ty + y;  // rows j0-1 .. j0+ty with j0 = 1 + blockIdx.x*ty
  const int k0 = 1 + blockIdx.y * a.kchunk;
  const int k1 = min(k0 + a.kchunk, nz - 1);  // tile planes k0 .. k1-1
  const bool on = (j <= ny - 1) && (q < W);
  const bool row_int = (j >= 1) && (j <= ny - 2);
  const bool tile = on && (y >= 1) && (y <= ty) && (j <= ny - 2);
  const T* __restrict__ X = a.xin;
  auto base = [&](int p) -> long long {
    return (long long)p * sz + (long long)j * sy + 2 * q - ((j + p) & 1);
  };
  auto slot = [&](V* ring, int p, int row, int col) -> V& {
    return ring[((p + 3) % 3 * NY + row) * RW + col];
  };
  auto ldx = [&](int p) -> V {
    V v = pzero<V>();
    if (on && p >= 0 && p <= nz - 1) {
      const long long b = base(p);
      if (b + 1 < N) v = __ldg(reinterpret_cast<const V*>(X + b));
      else v.x = X[b];
    }
    return v;
  };
  auto ldc = [&](int p, PairCoef<T>& c) {
    if (on && row_int && p >= 1 && p <= nz - 2) {
      const long long b = base(p);
      c.f = __ldg(reinterpret_cast<const V*>(a.fc + b));
      c.o = __ldg(reinterpret_cast<const V*>(a.oC + b));
      c.c = __ldg(reinterpret_cast<const V*>(a.cc + b));
      c.e = __ldg(reinterpret_cast<const V*>(a.oE + b));
      c.n = __ldg(reinterpret_cast<const V*>(a.oN + b));
      c.u = __ldg(reinterpret_cast<const V*>(a.uC + b));
    }
  };
  // element e of the thread's pair at plane p is an interior point
  auto interior = [&](int p, int e) {
    const int i = 2 * q - ((j + p) & 1) + e;
    return row_int && p >= 1 && p <= nz - 2 && i >= 1 && i <= nx - 2;
  };

  V Xm = ldx(k0 - 2), X0 = ldx(k0 - 1), Xp = ldx(k0);
  if (on) {
    if (k0 - 2 >= 0) slot(XS, k0 - 2, y, q) = Xm;
    slot(XS, k0 - 1, y, q) = X0;
  }
  PairCoef<T> cur{}, nxt{};
  ldc(k0 - 1, cur);
  // colour-c2 data of the previous plane, saved for its update one step later
  T sf = 0, sN = 0, sE = 0, sEw = 0, sU = 0, sD = 1, sc1 = 0;
  for (int P = k0 - 1; P <= k1; P++) {
    // ---- loads of this step (none depends on shared memory) ----
    const V Xn = (P + 2 <= min(k1 + 1, nz - 1)) ? ldx(P + 2) : pzero<V>();
    if (PF) ldc(P + 1, nxt);
    else if (P > k0 - 1) ldc(P, cur);
    const bool doA = on && interior(P, E1);
    const long long ida = base(P) + E1;
    T aNs = 0, aUd = 0, aEw = 0, aXn = 0, aXs = 0;
    if (doA) {
      aNs = a.oN[ida - sy];
      aUd = a.uC[ida - sz];
      if (E1 == 0) aEw = a.oE[ida - 1];
      if (y == NY - 1) aXn = X[ida + sy];
      if (y == 0) aXs = X[ida - sy];
    }
    const int p = P - 1;  // plane of this step's colour-c2 update
    const bool doB = tile && p >= k0 && interior(p, E2);
    const long long idb = base(p) + E2;
    T bNs = 0, bUd = 0, bEw = sEw;
    if (doB) {
      bNs = a.oN[idb - sy];
      bUd = a.uC[idb - sz];
      if (E2 == 0) bEw = a.oE[idb - 1];
    }
    if (on && P + 1 <= nz - 1) slot(XS, P + 1, y, q) = Xp;
    __syncthreads();

    // ---- colour c1 at plane P (tile and ring rows) ----
    if (on) {
      T nv = pelem<E1>(X0);
      if (doA) {
        const int s = (j + P) & 1;
        const int qn = q - s + E1;
        T xe, xw;
        if constexpr (E1 == 0) {
          xe = X0.y;
          xw = slot(XS, P, y, q - 1).y;
        } else {
          xw = X0.x;
          xe = slot(XS, P, y, q + 1).x;
        }
        const T xn = (y + 1 < NY) ? pelem<E2>(slot(XS, P, y + 1, qn)) : aXn;
        const T xs = (y >= 1) ? pelem<E2>(slot(XS, P, y - 1, qn)) : aXs;
        const T xd = pelem<E2>(slot(XS, P - 1, y, qn));
        const T xu = pelem<E2>(slot(XS, P + 1, y, qn));
        const T oEw = (E1 == 1) ? cur.e.x : aEw;
        nv = (pelem<E1>(cur.f) + pelem<E1>(cur.n) * xn + aNs * xs + pelem<E1>(cur.e) * xe +
              oEw * xw + aUd * xd + pelem<E1>(cur.u) * xu) /
             (pelem<E1>(cur.o) + pelem<E1>(cur.c));
      }
      V rv = X0;
      if constexpr (E1 == 0) rv.x = nv; else rv.y = nv;
      slot(R, P, y, q) = rv;
    }
    __syncthreads();

    // ---- colour c2 at plane p = P-1 (tile rows) ----
    if (tile && p >= k0) {
      const bool w1 = interior(p, E1);
      T v = 0;
      if (doB) {
        const int s = (j + p) & 1;
        const int qn = q - s + E2;
        T xe, xw;
        if constexpr (E2 == 0) {
          xe = sc1;
          xw = slot(R, p, y, q - 1).y;
        } else {
          xw = sc1;
          xe = slot(R, p, y, q + 1).x;
        }
        const T xn = pelem<E1>(slot(R, p, y + 1, qn));
        const T xs = pelem<E1>(slot(R, p, y - 1, qn));
        const T xd = pelem<E1>(slot(R, p - 1, y, qn));
        const T xu = pelem<E1>(slot(R, p + 1, y, qn));
        v = (sf + sN * xn + bNs * xs + sE * xe + bEw * xw + bUd * xd + sU * xu) / sD;
      }
      T* out = a.xout + base(p);
      if (w1 && doB) {
        V o;
        if constexpr (E1 == 0) { o.x = sc1; o.y = v; } else { o.x = v; o.y = sc1; }
        *reinterpret_cast<V*>(out) = o;
      } else {
        if (w1) out[E1] = sc1;
        if (doB) out[E2] = v;
      }
    }

    // ---- keep plane P's colour-c2 data for next step, rotate ----
    if (on) {
      sc1 = pelem<E1>(slot(R, P, y, q));
      sf = pelem<E2>(cur.f);
      sN = pelem<E2>(cur.n);
      sE = pelem<E2>(cur.e);
      sU = pelem<E2>(cur.u);
      sD = pelem<E2>(cur.o) + pelem<E2>(cur.c);
      sEw = cur.e.x;  // oE[id-1] of an element-1 point is its own pair's element 0
    }
    if (PF) cur = nxt;
    Xm = X0;
    X0 = Xp;
    Xp = Xn;
  }
}

// Shape of a pair-sweep launch: threads (pairs) per row, rows per CTA.
struct PairShape {
  int rw, ny_blk, ty;
};

inline bool pair_shape(const Grid& g, int rows_cap, PairShape* s) {
  if ((g.nx & 1) == 0 || (g.ny & 1) == 0 || g.nx < 5 || g.ny < 5 || g.nz < 3) return false;
  const int w = (g.nx + 1) / 2;
  s->rw = (w + 31) / 32 * 32;
  s->ny_blk = kPairThreads / s->rw;
  if (rows_cap > 0 && s->ny_blk > rows_cap) s->ny_blk = rows_cap;
  if (s->ny_blk < 3) return false;
  s->ty = s->ny_blk - 2;
  if (s->ty > g.ny - 2) {
    s->ty = g.ny - 2;
    s->ny_blk = s->ty + 2;
  }
  return true;
}

template <typename T>
inline bool pair_aligned(const Gs7Sweep<T>& a) {
  const size_t al = 2 * sizeof(T);
  const void* p[8] = {a.oC, a.oE, a.oN, a.uC, a.cc, a.fc, a.xin, a.xout};
  for (const void* v : p)
    if (reinterpret_cast<uintptr_t>(v) % al) return false;
  return true;
}

// Launches the pair sweep; returns cudaErrorNotSupported (nothing launched)
// when the grid has an even row length, rows too long for one CTA, or
// arrays that are not pair-aligned.  rows_cap > 0 limits the rows of a CTA
// (tile plus ring) so that several CTAs fit on an SM.  The plane chunk is
// chosen so that the CTAs fill the device in one wave.
template <typename T, bool PF>
inline cudaError_t launch_gs7_sweep_pairs(cudaStream_t st, const Gs7Sweep<T>& a0,
                                          int rows_cap = 0) {
  using V = typename PairOf<T>::type;
  PairShape ps;
  if (!pair_shape(a0.g, rows_cap, &ps) || !pair_aligned(a0)) return cudaErrorNotSupported;
  const size_t smem = (size_t)6 * ps.ny_blk * ps.rw * sizeof(V);
  static thread_local int dev_cached = -1, sms = 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev != dev_cached) {
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    for (auto* f : {k_gs7_sweep_pairs<T, 0, PF>, k_gs7_sweep_pairs<T, 1, PF>}) {
      e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(6 * kPairThreads * sizeof(V)));
      if (e != cudaSuccess) return e;
    }
    dev_cached = dev;
  }
  int per_sm = 1;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs7_sweep_pairs<T, 0, PF>,
                                                    ps.rw * ps.ny_blk, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorNotSupported;
  Gs7Sweep<T> a = a0;
  const Grid g = a.g;
  const int rowblocks = (g.ny - 2 + ps.ty - 1) / ps.ty;
  int nchunks = sms * per_sm / rowblocks;
  if (nchunks < 1) nchunks = 1;
  a.kchunk = (g.nz - 2 + nchunks - 1) / nchunks;
  nchunks = (g.nz - 2 + a.kchunk - 1) / a.kchunk;
  dim3 grid(rowblocks, nchunks), block(ps.rw, ps.ny_blk);
  if (a.c1 == 0)
    k_gs7_sweep_pairs<T, 0, PF><<<grid, block, smem, st>>>(a, ps.ty);
  else
    k_gs7_sweep_pairs<T, 1, PF><<<grid, block, smem, st>>>(a, ps.ty);
  return cudaGetLastError();
}

}  // namespace pmgb
