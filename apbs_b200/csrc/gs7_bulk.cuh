// The whole-row pair sweep of gs7_pairs.cuh (FP64) with every plane row
// brought into shared memory by one bulk asynchronous copy
// (cp.async.bulk ... mbarrier::complete_tx) issued planes ahead of its use.
//
// Same arithmetic and operand order as k_gs7_sweep_pairs, so the result is
// bitwise the colour-pass result of Vgsrb7x (src/pmgc/gsd.c:95-164).
//
// A row of pairs starts at an even flat index, so it is a 16-byte-aligned
// run of W = (nx+1)/2 pairs, and consecutive rows start nx - 1 or nx + 1
// elements apart: the rows of a CTA in one plane form one contiguous,
// 16-byte-aligned range, brought in by one copy per array and plane.  Shared
// memory is indexed by the flat offset from the start of that range.  The
// last row of the last plane would run one element past the array and is
// never needed (no update reads it), so it is not copied.
//
// Shared memory: a ring of DX staged planes of x, a ring of DC staged planes
// of the six coefficient arrays (fc, oC, cc, oE, oN, uC), and a four-plane
// ring R of the new colour-c1 values.  Each staged plane has its own
// mbarrier; warp 0 issues the copies of x plane P+DX-2 and coefficient plane
// P+DC-1 at the start of step P, so DX-3 and DC-1 planes of loads are in
// flight while the CTA computes.  One block barrier per plane: phase A
// (colour c1 at plane P) reads only the staged rings and writes R[P]; after
// the barrier phase B (colour c2 at plane P-1) reads R and registers only.
// A stage is refilled only after the barrier that follows its last read.
//
// Every mbarrier wait gives up after 200 ms (it counts itself in *err and no
// later wait of the CTA spins), so a launch always ends; the clock is read
// once per 64 polls.
#pragma once

#include "gs7_pairs.cuh"

namespace pmgb {

constexpr long long kBulkWaitNs = 200LL * 1000 * 1000;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long bulk_now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)),
               "r"(bytes)
               : "memory");
}
// try_wait with a suspend-time hint: a thread whose phase is not complete
// sleeps in hardware (up to about 1 ms) instead of spinning.
__device__ __forceinline__ bool mbar_test(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity), "r"(1000000u)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes,
                                              uint64_t* b) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(b))
      : "memory");
}
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// pairs of one staged plane of one array: rows 0 .. ny_blk-1 from the pair
// base of row 0
inline int bulk_stage_pairs(int ny_blk, int nx) { return ((ny_blk - 1) * nx + 1) / 2 + (nx + 1) / 2; }

template <int DX, int DC>
inline size_t bulk_smem_bytes(int ny_blk, int nx) {
  const int w = (nx + 1) / 2;
  return (size_t)(DX + 6 * DC) * bulk_stage_pairs(ny_blk, nx) * 16 +
         4 * (size_t)ny_blk * w * 8 + (DX + DC) * 8;
}

template <int C1, int DX, int DC>
__global__ void __launch_bounds__(kPairThreads, 1)
    k_gs7_sweep_bulk(Gs7Sweep<double> a, int ty, int* err) {
  using V = double2;
  constexpr int E1 = C1, E2 = 1 - C1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NY = blockDim.y;
  const Grid g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long sy = nx, sz = (long long)nx * ny;
  const int W = (nx + 1) / 2;
  const int SP = ((NY - 1) * nx + 1) / 2 + W;  // pairs per staged plane of one array
  V* XS = reinterpret_cast<V*>(smem_raw);                 // [DX][SP]
  V* CS = XS + DX * SP;                                   // [DC][6][SP]
  double* R = reinterpret_cast<double*>(CS + DC * 6 * SP);  // [4][NY][W]
  uint64_t* bar = reinterpret_cast<uint64_t*>(R + 4 * NY * W);  // [DX + DC]
  const int q = threadIdx.x, y = threadIdx.y;
  const int lane = threadIdx.x & 31;
  const bool warp0 = (y == 0) && (threadIdx.x < 32);
  const int jb = blockIdx.x * ty;  // row of thread row 0
  const int j = jb + y;
  const int k0 = 1 + blockIdx.y * a.kchunk;
  const int k1 = min(k0 + a.kchunk, nz - 1);
  const bool on = (j <= ny - 1) && (q < W);
  const bool row_int = (j >= 1) && (j <= ny - 2);
  const bool tile = on && (y >= 1) && (y <= NY - 2) && (y <= ty) && (j <= ny - 2);
  const int xfirst = max(k0 - 2, 0), xlast = min(k1 + 1, nz - 1);
  const int cfirst = k0 - 1, clast = k1;
  const double* __restrict__ X = a.xin;

  auto base = [&](int p, int jj, int qq) -> long long {
    return (long long)p * sz + (long long)jj * sy + 2 * qq - ((jj + p) & 1);
  };
  auto interior = [&](int p, int e) {
    const int i = 2 * q - ((j + p) & 1) + e;
    return row_int && p >= 1 && p <= nz - 2 && i >= 1 && i <= nx - 2;
  };
  // pair offset of (row, col) in a staged plane p
  auto off = [&](int p, int row, int col) -> int {
    return ((row * nx - ((jb + row + p) & 1) + ((jb + p) & 1)) >> 1) + col;
  };
  auto xs_at = [&](int p, int row, int col) -> const V& {
    return XS[(p - xfirst) % DX * SP + off(p, row, col)];
  };
  auto cs_at = [&](int p, int arr, int row, int col) -> const V& {
    return CS[((p - cfirst) % DC * 6 + arr) * SP + off(p, row, col)];
  };
  auto r_at = [&](int p, int row, int col) -> double& {
    return R[(p % 4 * NY + row) * W + col];
  };
  // warp 0: stage x (narr = 1) or the coefficients (narr = 6) of plane p:
  // rows jb .. jlast (rows of the grid, less the last row of the last plane)
  // as one contiguous range per array
  auto issue = [&](int p, int narr, V* dst, uint64_t* b) {
    int jlast = min(jb + NY - 1, ny - 1);
    if (p == nz - 1 && jlast == ny - 1) jlast--;
    const long long start = base(p, jb, 0);
    const unsigned bytes =
        jlast >= jb ? (unsigned)((base(p, jlast, 0) + 2 * W - start) * 8) : 0u;
    fence_async_shared();
    if (lane == 0) mbar_arrive_tx(b, bytes * narr);
    __syncwarp();
    if (bytes && lane < narr) {
      const double* s0 = narr == 1 ? X
                         : lane == 0 ? a.fc
                         : lane == 1 ? a.oC
                         : lane == 2 ? a.cc
                         : lane == 3 ? a.oE
                         : lane == 4 ? a.oN
                                     : a.uC;
      bulk_copy_g2s(dst + (size_t)lane * SP, s0 + start, bytes, b);
    }
  };
  auto issue_x = [&](int p) {
    if (p < xfirst || p > xlast) return;
    const int sl = (p - xfirst) % DX;
    issue(p, 1, XS + (size_t)sl * SP, bar + sl);
  };
  auto issue_c = [&](int p) {
    if (p < cfirst || p > clast) return;
    const int sl = (p - cfirst) % DC;
    issue(p, 6, CS + (size_t)sl * 6 * SP, bar + DX + sl);
  };
  bool failed = false;
  auto wait = [&](uint64_t* b, unsigned parity) {
    if (failed || mbar_test(b, parity)) return;
    const unsigned long long t0 = bulk_now_ns();
    for (unsigned n = 1; !mbar_test(b, parity); n++) {
      if ((n & 63) == 0 && bulk_now_ns() - t0 > (unsigned long long)kBulkWaitNs) {
        failed = true;
        if (err) atomicAdd(err, 1);
        return;
      }
    }
  };
  auto wait_x = [&](int p) {
    if (p < xfirst || p > xlast) return;
    wait(bar + (p - xfirst) % DX, ((p - xfirst) / DX) & 1);
  };
  auto wait_c = [&](int p) {
    wait(bar + DX + (p - cfirst) % DC, ((p - cfirst) / DC) & 1);
  };

  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int b = 0; b < DX + DC; b++) mbar_init(bar + b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (warp0) {
    for (int p = xfirst; p <= k0 + DX - 4; p++) issue_x(p);
    for (int p = cfirst; p <= k0 + DC - 3; p++) issue_c(p);
  }
  for (int p = xfirst; p < k0; p++) wait_x(p);

  // colour-c2 data of plane P-1 (saved in step P-1 for phase B of step P)
  double sf = 0, sN = 0, sE = 0, sU = 0, sD = 1, sEw = 0, sNs = 0, sc1 = 0;
  double uA = 0;            // uC below the c1 point of pair q at the next plane
  double uB0 = 0, uB1 = 0;  // uC below the c2 point of pair q, one and two planes on
  for (int P = k0 - 1; P <= k1; P++) {
    if (warp0) {
      issue_x(P + DX - 2);
      issue_c(P + DC - 1);
    }
    const bool doA = on && interior(P, E1);
    const long long ida = base(P, j, q) + E1;
    double aXn = 0, aXs = 0, aNs = 0;
    if (doA) {
      if (y == NY - 1) aXn = X[ida + sy];
      if (y == 0) {
        aXs = X[ida - sy];
        aNs = a.oN[ida - sy];
      }
      if (P == k0 - 1) uA = a.uC[ida - sz];
    }
    wait_x(P + 1);
    wait_c(P);

    // ---- phase A: colour c1 at plane P (all rows) ----
    double c1v = 0, nsf = 0, nsN = 0, nsE = 0, nsU = 0, nsD = 1, nsEw = 0, nsNs = 0;
    double nA = 0, nB = 0;
    if (on) {
      // the last row of the last plane is not staged (nothing reads it)
      const V X0 = (j == ny - 1 && P == nz - 1) ? pzero<V>() : xs_at(P, y, q);
      double nv = pelem<E1>(X0);
      const int s = (j + P) & 1;
      if (doA) {
        const int qn = q - s + E1;
        double xe, xw, oEw;
        const V E = cs_at(P, 3, y, q);
        if constexpr (E1 == 0) {
          xe = X0.y;
          xw = xs_at(P, y, q - 1).y;
          oEw = cs_at(P, 3, y, q - 1).y;
        } else {
          xw = X0.x;
          xe = xs_at(P, y, q + 1).x;
          oEw = E.x;
        }
        const double xn = (y + 1 < NY) ? pelem<E2>(xs_at(P, y + 1, qn)) : aXn;
        const double xs = (y >= 1) ? pelem<E2>(xs_at(P, y - 1, qn)) : aXs;
        const double oNs = (y >= 1) ? pelem<E2>(cs_at(P, 4, y - 1, qn)) : aNs;
        const double xd = pelem<E2>(xs_at(P - 1, y, qn));
        const double xu = pelem<E2>(xs_at(P + 1, y, qn));
        nv = (pelem<E1>(cs_at(P, 0, y, q)) + pelem<E1>(cs_at(P, 4, y, q)) * xn + oNs * xs +
              pelem<E1>(E) * xe + oEw * xw + uA * xd + pelem<E1>(cs_at(P, 5, y, q)) * xu) /
             (pelem<E1>(cs_at(P, 1, y, q)) + pelem<E1>(cs_at(P, 2, y, q)));
      }
      r_at(P, y, q) = nv;
      c1v = nv;
      // colour-c2 data of plane P for phase B of the next step
      if (tile && P >= k0 && P <= k1 - 1 && interior(P, E2)) {
        const int qn = q - s + E2;
        nsf = pelem<E2>(cs_at(P, 0, y, q));
        nsN = pelem<E2>(cs_at(P, 4, y, q));
        nsE = pelem<E2>(cs_at(P, 3, y, q));
        nsU = pelem<E2>(cs_at(P, 5, y, q));
        nsD = pelem<E2>(cs_at(P, 1, y, q)) + pelem<E2>(cs_at(P, 2, y, q));
        nsEw = (E2 == 1) ? cs_at(P, 3, y, q).x : cs_at(P, 3, y, q - 1).y;
        nsNs = pelem<E1>(cs_at(P, 4, y - 1, qn));
      }
      // uC at plane P below the points of pair q at plane P+1
      const int s1 = 1 - s;
      if (P + 1 <= k1 && interior(P + 1, E1)) nA = pelem<E2>(cs_at(P, 5, y, q - s1 + E1));
      if (tile && P + 1 <= k1 - 1 && interior(P + 1, E2))
        nB = pelem<E1>(cs_at(P, 5, y, q - s1 + E2));
    }
    __syncthreads();

    // ---- phase B: colour c2 at plane P-1 (tile rows), from R and registers ----
    if (tile && P - 1 >= k0) {
      const int p = P - 1;
      const bool w1 = interior(p, E1);
      const bool doB = interior(p, E2);
      double v = 0;
      if (doB) {
        const int sp = (j + p) & 1;
        const int qn = q - sp + E2;
        double xe, xw;
        if constexpr (E2 == 0) {
          xe = sc1;
          xw = r_at(p, y, q - 1);
        } else {
          xw = sc1;
          xe = r_at(p, y, q + 1);
        }
        const double xn = r_at(p, y + 1, qn);
        const double xs = r_at(p, y - 1, qn);
        const double xd = r_at(p - 1, y, qn);
        const double xu = r_at(p + 1, y, qn);
        v = (sf + sN * xn + sNs * xs + sE * xe + sEw * xw + uB0 * xd + sU * xu) / sD;
      }
      double* out = a.xout + base(p, j, q);
      if (w1 && doB) {
        V o;
        if constexpr (E1 == 0) { o.x = sc1; o.y = v; } else { o.x = v; o.y = sc1; }
        *reinterpret_cast<V*>(out) = o;
      } else {
        if (w1) out[E1] = sc1;
        if (doB) out[E2] = v;
      }
    }
    sf = nsf; sN = nsN; sE = nsE; sU = nsU; sD = nsD; sEw = nsEw; sNs = nsNs; sc1 = c1v;
    uA = nA;
    uB0 = uB1;
    uB1 = nB;
  }
}

// FP64 only.  Returns cudaErrorNotSupported (nothing launched) when the pair
// layout does not apply or the staged rows do not fit in shared memory.
template <int DX, int DC>
inline cudaError_t launch_gs7_sweep_bulk(cudaStream_t st, const Gs7Sweep<double>& a0, int* err) {
  PairShape ps;
  if (!pair_shape(a0.g, 0, &ps) || !pair_aligned(a0)) return cudaErrorNotSupported;
  static thread_local int dev_cached = -1, sms = 0, smem_max = 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev != dev_cached) {
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    for (auto* f : {k_gs7_sweep_bulk<0, DX, DC>, k_gs7_sweep_bulk<1, DX, DC>})
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    if (e != cudaSuccess) return e;
    dev_cached = dev;
  }
  const int nx = a0.g.nx;
  while (ps.ny_blk >= 3 && bulk_smem_bytes<DX, DC>(ps.ny_blk, nx) > (size_t)smem_max) ps.ny_blk--;
  if (ps.ny_blk < 3) return cudaErrorNotSupported;
  ps.ty = ps.ny_blk - 2;
  const size_t smem = bulk_smem_bytes<DX, DC>(ps.ny_blk, nx);
  Gs7Sweep<double> a = a0;
  const Grid g = a.g;
  const int rowblocks = (g.ny - 2 + ps.ty - 1) / ps.ty;
  int nchunks = sms / rowblocks;
  if (nchunks < 1) nchunks = 1;
  a.kchunk = (g.nz - 2 + nchunks - 1) / nchunks;
  nchunks = (g.nz - 2 + a.kchunk - 1) / a.kchunk;
  dim3 grid(rowblocks, nchunks), block(ps.rw, ps.ny_blk);
  if (a.c1 == 0)
    k_gs7_sweep_bulk<0, DX, DC><<<grid, block, smem, st>>>(a, ps.ty, err);
  else
    k_gs7_sweep_bulk<1, DX, DC><<<grid, block, smem, st>>>(a, ps.ty, err);
  return cudaGetLastError();
}

}  // namespace pmgb
