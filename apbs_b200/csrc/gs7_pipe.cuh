// Temporally blocked 7-point red-black Gauss-Seidel (one cooperative kernel).
//
// Restates nsweep iterations of Vgsrb7x (src/pmgc/gsd.c:95-164), optionally
// followed by the residual of Vmresid7_1s (src/pmgc/matvecd.c:461-489), with
// every point updated by exactly the reference's expression.  Red-black GS
// on a 7-point stencil has no same-colour coupling, so half-sweep h may run
// on a plane as soon as half-sweep h-1 has finished the planes next to it.
// The planes 1..nz-2 are cut into chunks of C planes; in phase p half-sweep h
// works on chunk p-h shifted down by h planes:
//     P_h(p) = [1 + (p-h)*C - h, 1 + (p-h+1)*C - h)
// Chunks of consecutive half-sweeps in one phase are separated by a one-plane
// gap, each reads only planes finished in earlier phases and none writes a
// plane another reads, so phases need just a grid barrier between them.  A
// plane's coefficients are read from HBM by half-sweep 0 and re-read from L2
// by the later half-sweeps a few phases after, which is where the saving
// over separate colour passes comes from.
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"

namespace pmgb {

template <typename T>
struct Gs7Args {
  Grid g;
  const T* oC;
  const T* oE;
  const T* oN;
  const T* uC;
  const T* cc;
  const T* fc;
  T* x;
  T* r;            // residual output (nullptr: no residual phase)
  int nhalf;       // 2 * sweeps
  int first_parity;
  int chunk;       // planes per chunk
};

template <typename T>
__global__ void __launch_bounds__(256) k_gs7_pipe(Gs7Args<T> a) {
  namespace cgr = cooperative_groups;
  cgr::grid_group grid = cgr::this_grid();
  const Grid g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t sy = nx, sz = (size_t)nx * ny;
  const int hr = (nx - 1) / 2;
  const int C = a.chunk;
  const int nphase_items = a.nhalf + (a.r ? 1 : 0);
  // the last pipeline stage is shifted down by (nphase_items - 1) planes, so
  // it needs ceil((nz - 2 + nphase_items - 1) / C) chunks
  const int nphases = (nphase_items - 1) + (nz - 2 + nphase_items - 1 + C - 1) / C;
  const size_t gtid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t nthr = (size_t)gridDim.x * blockDim.x;
  for (int p = 0; p < nphases; p++) {
    int lo[5];
    unsigned cnt[5], total = 0;
    for (int h = 0; h < nphase_items; h++) {
      int l = 1 + (p - h) * C - h, u = l + C;
      if (l < 1) l = 1;
      if (u > nz - 1) u = nz - 1;
      if (p - h < 0 || u <= l) {
        cnt[h] = 0;
        lo[h] = 0;
        continue;
      }
      lo[h] = l;
      const unsigned per_plane = (unsigned)(ny - 2) * (unsigned)((h < a.nhalf) ? hr : (nx - 2));
      cnt[h] = per_plane * (unsigned)(u - l);
      total += cnt[h];
    }
    for (unsigned item = (unsigned)gtid; item < total; item += (unsigned)nthr) {
      int h = 0;
      unsigned rem = item;
      while (rem >= cnt[h]) {
        rem -= cnt[h];
        h++;
      }
      if (h < a.nhalf) {
        const unsigned row = rem / (unsigned)hr;
        const int m = (int)(rem - row * (unsigned)hr);
        const unsigned pl = row / (unsigned)(ny - 2);
        const int j = 1 + (int)(row - pl * (unsigned)(ny - 2));
        const int k = lo[h] + (int)pl;
        const int parity = (a.first_parity + h) & 1;
        const int i = 1 + (((1 + j + k) & 1) != parity) + 2 * m;
        if (i > nx - 2) continue;
        const size_t id = g.idx(i, j, k);
        const T* x = a.x;
        a.x[id] = (a.fc[id] + a.oN[id] * x[id + sy] + a.oN[id - sy] * x[id - sy] +
                   a.oE[id] * x[id + 1] + a.oE[id - 1] * x[id - 1] +
                   a.uC[id - sz] * x[id - sz] + a.uC[id] * x[id + sz]) /
                  (a.oC[id] + a.cc[id]);
      } else {
        const unsigned row = rem / (unsigned)(nx - 2);
        const int i = 1 + (int)(rem - row * (unsigned)(nx - 2));
        const unsigned pl = row / (unsigned)(ny - 2);
        const int j = 1 + (int)(row - pl * (unsigned)(ny - 2));
        const int k = lo[h] + (int)pl;
        const size_t id = g.idx(i, j, k);
        const T* x = a.x;
        a.r[id] = a.fc[id] + a.oN[id] * x[id + sy] + a.oN[id - sy] * x[id - sy] +
                  a.oE[id] * x[id + 1] + a.oE[id - 1] * x[id - 1] +
                  a.uC[id - sz] * x[id - sz] + a.uC[id] * x[id + sz] -
                  (a.oC[id] + a.cc[id]) * x[id];
      }
    }
    grid.sync();
  }
}


// Co-resident grid for the cooperative launch: SMs x min(occupancy limit,
// requested CTAs per SM).
template <typename T>
inline int gs7_pipe_grid(int want) {
  // initialised once, thread-safely (function-local static)
  static const int2 sm_per = [] {
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_gs7_pipe<T>, 256, 0);
    return make_int2(nsm, per < 1 ? 1 : per);
  }();
  const int nsm = sm_per.x, per = sm_per.y;
  int use = (want > 0 && want < per) ? want : per;
  return nsm * use;
}

template <typename T>
inline cudaError_t launch_gs7_pipe(cudaStream_t s, const Gs7Args<T>& a, int blocks_per_sm) {
  Gs7Args<T> arg = a;
  void* params[] = {&arg};
  return cudaLaunchCooperativeKernel((void*)k_gs7_pipe<T>, dim3(gs7_pipe_grid<T>(blocks_per_sm)), dim3(256),
                                     params, 0, s);
}

}  // namespace pmgb
