// The single-pass red-black sweep of gs7_rb.cuh with its operands staged in
// shared memory by the bulk-copy engine (cp.async.bulk, completion on
// mbarriers), so a CTA keeps whole plane windows in flight instead of
// relying on warp-level memory parallelism.
//
// The arithmetic, the pair-slot layout and the order of the updates are
// those of k_gs7_rb (one iteration of Vgsrb7x, src/pmgc/gsd.c:95-164); only
// where the operands come from changes, so the results are bitwise those of
// k_gs7_rb and of the two colour passes.
//
// A CTA owns the flat range [c0, c0 + core) of every plane of its chunk
// [k0, k1).  For plane q it keeps a window of each operand array covering
// the in-plane indices [off(q), off(q) + Lw), off(q) being c0 - 2 nx - 2
// rounded down so that the window starts on a 16-byte boundary: that covers
// the widened C1 range [c0 - nx - 1, c0 + core + nx + 1) with its in-plane
// neighbours.  Step t of the march computes the new C1 values of plane t
// (phase A) and, from the C1 values of planes t-2..t, the second colour of
// plane t-1 (phase B), exactly as k_gs7_rb's iteration t-1 does.
//
// Stage j brings the coefficient windows (oE, oN, D, f) of plane j, the uC
// window of plane j and the x window of plane j+1; step t needs stages up to
// t, and stage t+P is issued at the start of step t.  Ring depths follow
// from the live planes of a step: coefficients t-1..t (P+2 slots), uC
// t-2..t (P+3), x t-1..t+1 (P+3).  Windows that would reach outside the
// arrays (the boundary planes; the last planes for small grids) are read
// with guarded plain loads by all threads instead.
//
// Every wait on an mbarrier is bounded: when it gives up, the CTA records
// the failure in *err, waits (bounded) for its copies in flight and
// returns, so a caller sees an error status instead of a hang.
#pragma once

#include "gs7_rb.cuh"

namespace pmgb {

template <typename T>
struct Gs7RbBulk {
  Gs7Rb<T> a;  // arrays, nx, S, nz, core, E, kchunk as for k_gs7_rb
  int Lw;      // window length in elements (a multiple of 16 bytes)
  int* err;    // set to 1 when a wait gives up
};

constexpr unsigned long long kBulkWaitNs = 50ull * 1000 * 1000;  // give up after 50 ms

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* b, unsigned parity) {
  if (mbar_try_wait(b, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(b, parity))
    if (global_ns() - t0 > kBulkWaitNs) return false;
  return true;
}
// global -> shared bulk copy completing on mbarrier b (both addresses 16-byte
// aligned, bytes a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* b) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(b))
      : "memory");
}

// shared-memory bytes of the bulk sweep for a given core (host and device)
template <typename T, int P>
__host__ __device__ constexpr size_t gs7_bulk_smem(int Lw, int E) {
  return 64 + ((size_t)4 * (P + 2) + (P + 3) + (P + 3)) * Lw * sizeof(T) +
         (size_t)3 * E * sizeof(T);
}

template <typename T, int C1, int NT, int P>
__global__ void __launch_bounds__(NT, 1) k_gs7_rb_bulk(Gs7RbBulk<T> b) {
  constexpr int AL = 16 / (int)sizeof(T);  // elements per 16 bytes
  constexpr int NC = P + 2, NU = P + 3, NX = P + 3, NB = P + 1;
  constexpr int C2 = 1 - C1;
  extern __shared__ __align__(16) unsigned char bulk_smem[];
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(bulk_smem);
  const int nx = b.a.nx, S = b.a.S, nz = b.a.nz, E = b.a.E, Lw = b.Lw;
  T* cw = reinterpret_cast<T*>(bulk_smem + 64);  // [NC][4][Lw]: oE, oN, D, f
  T* uw = cw + (size_t)NC * 4 * Lw;              // [NU][Lw]
  T* xw = uw + (size_t)NU * Lw;                  // [NX][Lw]
  T* R = xw + (size_t)NX * Lw;                   // [3][E]: new C1 values by pair slot
  const int c0 = blockIdx.x * b.a.core;
  const int c1e = min(c0 + b.a.core, S);
  const int k0 = 1 + blockIdx.y * b.a.kchunk;
  const int k1 = min(k0 + b.a.kchunk, nz - 1);
  const int t0 = k0 - 1;
  const int ntot = nz * S;

  // in-plane index of window element 0 of plane q
  auto off = [&](int q) -> int {
    const int v = q * S + c0 - 2 * nx - 2;
    const int al = v >= 0 ? (v / AL) * AL : -((-v + AL - 1) / AL) * AL;
    return al - q * S;
  };
  auto cslot = [&](int q, int arr) -> T* { return cw + ((size_t)((q + 4 * NC) % NC) * 4 + arr) * Lw; };
  auto uslot = [&](int q) -> T* { return uw + (size_t)((q + 4 * NU) % NU) * Lw; };
  auto xslot = [&](int q) -> T* { return xw + (size_t)((q + 4 * NX) % NX) * Lw; };

  auto coef_src = [&](int arr) -> const T* {
    return arr == 0 ? b.a.oE : arr == 1 ? b.a.oN : arr == 2 ? b.a.D : b.a.f;
  };
  auto guarded = [&](const T* src, T* dst, int g0) {
    for (int e = threadIdx.x; e < Lw; e += NT) {
      const int g = g0 + e;
      dst[e] = (g >= 0 && g < ntot) ? src[g] : T(0);
    }
  };
  // issue stage j: coefficients of plane j (j >= t0), uC of plane j (j >= t0-1),
  // x of plane j+1 (j+1 >= t0-1); planes outside 0..nz-1 are never read.
  // Windows inside the arrays come by bulk copy, the others by guarded
  // plain loads (read by the consumers after a later barrier).
  auto issue = [&](int j) {
    const int u = j - (t0 - 2);
    unsigned long long* bb = bar + (u % NB);
    const bool has_c = j >= t0 && j >= 0 && j <= nz - 1;
    const bool has_u = j >= t0 - 1 && j >= 0 && j <= nz - 1;
    const bool has_x = j + 1 >= t0 - 1 && j + 1 >= 0 && j + 1 <= nz - 1;
    const int gj = j * S + off(j), gx = (j + 1) * S + off(j + 1);
    const bool bulk_j = gj >= 0 && gj + Lw <= ntot;
    const bool bulk_x = gx >= 0 && gx + Lw <= ntot;
    const unsigned wbytes = (unsigned)(Lw * sizeof(T));
    if (has_c && !bulk_j)
#pragma unroll
      for (int arr = 0; arr < 4; arr++) guarded(coef_src(arr), cslot(j, arr), gj);
    if (has_u && !bulk_j) guarded(b.a.uC, uslot(j), gj);
    if (has_x && !bulk_x) guarded(b.a.xin, xslot(j + 1), gx);
    if (threadIdx.x == 0) {
      const unsigned bytes = ((has_c && bulk_j) ? 4u * wbytes : 0u) +
                             ((has_u && bulk_j) ? wbytes : 0u) + ((has_x && bulk_x) ? wbytes : 0u);
      // the slots were last read through the generic proxy before the
      // barrier that precedes this call
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_expect_tx(bb, bytes);
      if (has_c && bulk_j)
#pragma unroll
        for (int arr = 0; arr < 4; arr++) bulk_g2s(cslot(j, arr), coef_src(arr) + gj, wbytes, bb);
      if (has_u && bulk_j) bulk_g2s(uslot(j), b.a.uC + gj, wbytes, bb);
      if (has_x && bulk_x) bulk_g2s(xslot(j + 1), b.a.xin + gx, wbytes, bb);
    }
  };
  auto wait_stage = [&](int j) -> bool {
    const int u = j - (t0 - 2);
    return mbar_wait_bounded(bar + (u % NB), (unsigned)((u / NB) & 1));
  };
  int last_issued = t0 - 3;
  // give up: record it, wait (bounded) for the stages still in flight, leave
  auto bail = [&](int first_unwaited) {
    if (threadIdx.x == 0) {
      atomicExch(b.err, 1);
      for (int j = first_unwaited; j <= last_issued; j++) (void)wait_stage(j);
    }
    __syncthreads();
  };

  if (threadIdx.x == 0) {
    for (int i = 0; i < NB; i++) mbar_init(bar + i, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // history stages t0-2 and t0-1, then the first P stages of the march
  issue(t0 - 2);
  issue(t0 - 1);
  last_issued = t0 - 1;
  {
    const bool ok = wait_stage(t0 - 2) && wait_stage(t0 - 1);
    if (__syncthreads_or(!ok)) {
      bail(t0 - 2);
      return;
    }
  }
  for (int j = t0; j < t0 + P && j <= k1; j++) {
    issue(j);
    last_issued = j;
  }

  // slot offsets of the C1 neighbours of a second-colour point of pair m
  constexpr int dW = (C2 - C1 - 1) / 2, dE = (C2 - C1 + 1) / 2;
  const int dS = (C2 - C1 - nx) / 2, dN = (C2 - C1 + nx) / 2;
  T* __restrict__ xo = b.a.xout;

  for (int t = t0; t <= k1; t++) {
    if (t + P <= k1) {
      issue(t + P);
      last_issued = t + P;
    }
    {
      const bool ok = wait_stage(t);
      if (__syncthreads_or(!ok)) {
        bail(t);
        return;
      }
    }
    // phase A: new C1 values of plane t on the widened range -> R[t % 3]
    {
      T* Rt = R + (t % 3) * E;
      const int m0 = rb_base(t, S, c0, nx);
      const bool boundary_plane = (t == 0) || (t == nz - 1);
      if (boundary_plane) {
        for (int e = threadIdx.x; e < E; e += NT) Rt[e] = T(0);
      } else {
        const T* cE = cslot(t, 0);
        const T* cN = cslot(t, 1);
        const T* cD = cslot(t, 2);
        const T* cF = cslot(t, 3);
        const T* U0 = uslot(t - 1);
        const T* U1 = uslot(t);
        const T* Xm = xslot(t - 1);
        const T* X0 = xslot(t);
        const T* Xp = xslot(t + 1);
        const int o0 = off(t), om = off(t - 1), op = off(t + 1);
        const int tS = t * S;
        for (int e = threadIdx.x; e < E; e += NT) {
          const int ip = 2 * (m0 + e) + C1 - tS;
          T v = T(0);
          if (ip >= 0 && ip < S) {
            const int l = ip - o0, lm = ip - om, lp = ip - op;
            v = rb_update<T>(cF[l], cN[l], X0[l + nx], cN[l - nx], X0[l - nx], cE[l], X0[l + 1],
                             cE[l - 1], X0[l - 1], U0[lm], Xm[lm], U1[l], Xp[lp], cD[l]);
          }
          Rt[e] = v;
        }
      }
    }
    __syncthreads();
    // phase B: second colour of plane k = t-1 from the C1 values of k-1..k+1
    const int k = t - 1;
    if (k >= k0) {
      const T* Rm = R + ((k + 2) % 3) * E;  // plane k-1
      const T* R0 = R + (k % 3) * E;
      const T* Rp = R + ((k + 1) % 3) * E;
      const int m0 = rb_base(k, S, c0, nx);
      const int dD = m0 + (C2 - C1 - S) / 2 - rb_base(k - 1, S, c0, nx);
      const int dU = m0 + (C2 - C1 + S) / 2 - rb_base(k + 1, S, c0, nx);
      const int lo = k * S + c0, hi = k * S + c1e;
      const T* cE = cslot(k, 0);
      const T* cN = cslot(k, 1);
      const T* cD = cslot(k, 2);
      const T* cF = cslot(k, 3);
      const T* Um = uslot(k - 1);
      const T* U0 = uslot(k);
      const int o0 = off(k), om = off(k - 1);
      const int kS = k * S;
      for (int e = threadIdx.x; e < E; e += NT) {
        const int m = m0 + e;
        const int p2 = 2 * m + C2;
        const int p1 = 2 * m + C1;
        const bool in2 = (p2 >= lo) && (p2 < hi);
        const bool in1 = (p1 >= lo) && (p1 < hi);
        if (!in1 && !in2) continue;
        const T v1 = R0[e];
        T v2 = T(0);
        if (in2) {
          const int l = p2 - kS - o0, lm = p2 - kS - om;
          v2 = rb_update<T>(cF[l], cN[l], R0[e + dN], cN[l - nx], R0[e + dS], cE[l], R0[e + dE],
                            cE[l - 1], R0[e + dW], Um[lm], Rm[e + dD], U0[l], Rp[e + dU], cD[l]);
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
    }
    __syncthreads();  // slots of step t-1 are refilled at the next step's start
  }
}

// Launch geometry of the bulk sweep: the core (even) and plane chunk that
// minimise waves x (kchunk + 2) x Lw, the window volume a CTA streams, with
// the shared memory within smem_max.
struct BulkShape {
  int core, kchunk, Lw, E, nranges, nchunks;
  size_t smem;
};

template <typename T, int P>
inline BulkShape gs7_bulk_shape(int nx, int S, int nz, int sms, size_t smem_max) {
  constexpr int AL = 16 / (int)sizeof(T);
  BulkShape best{};
  double best_cost = 0.0;
  auto lw_of = [&](int core) { return ((core + 4 * nx + 6 + 2 * AL + AL - 1) / AL) * AL; };
  for (int nr = 1; nr <= 4096; nr++) {
    int core = (S + nr - 1) / nr;
    core = (core + 1) & ~1;
    const int Lw = lw_of(core);
    const int E = core / 2 + nx + 3;
    const size_t smem = gs7_bulk_smem<T, P>(Lw, E);
    if (smem > smem_max) continue;
    if ((size_t)(nr - 1) * core >= (size_t)S) continue;  // an empty last range
    const int planes = nz - 2;
    int nc = sms / nr;
    if (nc < 1) nc = 1;
    if (nc > planes) nc = planes;
    const int kchunk = (planes + nc - 1) / nc;
    nc = (planes + kchunk - 1) / kchunk;
    const long long ctas = (long long)nr * nc;
    const long long waves = (ctas + sms - 1) / sms;
    const double cost = (double)waves * (kchunk + 2) * Lw;
    if (best.core == 0 || cost < best_cost) {
      best_cost = cost;
      best = BulkShape{core, kchunk, Lw, E, nr, nc, smem};
    }
    if (core <= 2 * (nx + 2)) break;  // windows mostly halo beyond this
  }
  return best;
}

template <typename T, int NT, int P>
inline cudaError_t launch_gs7_rb_bulk_nt(cudaStream_t st, const Gs7Rb<T>& a0, int c1, int* err,
                                         int sms) {
  constexpr size_t kSmemMax = 220 * 1024;
  Gs7RbBulk<T> b;
  b.a = a0;
  b.err = err;
  const BulkShape sh = gs7_bulk_shape<T, P>(a0.nx, a0.S, a0.nz, sms, kSmemMax);
  if (sh.core == 0) return cudaErrorNotSupported;  // no window fits: the caller falls back
  b.a.core = sh.core;
  b.a.kchunk = sh.kchunk;
  b.a.E = sh.E;
  b.Lw = sh.Lw;
  const dim3 grid(sh.nranges, sh.nchunks);
  if (c1) {
    static const cudaError_t attr = cudaFuncSetAttribute(
        k_gs7_rb_bulk<T, 1, NT, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax);
    if (attr != cudaSuccess) return attr;
    k_gs7_rb_bulk<T, 1, NT, P><<<grid, NT, sh.smem, st>>>(b);
  } else {
    static const cudaError_t attr = cudaFuncSetAttribute(
        k_gs7_rb_bulk<T, 0, NT, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax);
    if (attr != cudaSuccess) return attr;
    k_gs7_rb_bulk<T, 0, NT, P><<<grid, NT, sh.smem, st>>>(b);
  }
  return cudaGetLastError();
}

// One bulk-staged sweep x -> xout.  threads: 0 -> 256, 1 -> 512 per CTA.
template <typename T>
inline cudaError_t launch_gs7_rb_bulk(cudaStream_t st, const Gs7Rb<T>& a, int c1, int threads,
                                      int* err) {
  if ((a.nx & 1) == 0 || (a.S & 1) == 0 || a.nz < 3 ||
      (double)a.S * a.nz * sizeof(T) >= 2147483647.0 || !err)
    return cudaErrorInvalidValue;
  static const int sms = [] {
    int dev = 0, n = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
  }();
  if (threads == 1) return launch_gs7_rb_bulk_nt<T, 512, 2>(st, a, c1, err, sms);
  return launch_gs7_rb_bulk_nt<T, 256, 2>(st, a, c1, err, sms);
}

}  // namespace pmgb
