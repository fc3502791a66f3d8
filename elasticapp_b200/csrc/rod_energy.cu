// Per-rod energies at the current state
// (elastica/Systems/CosseratRods/Utility/Energy.hpp:46-141): one warp per
// rod, lanes stride over the rod's slots, warp-shuffle reduction.  Strains
// and curvatures are recomputed from the current positions and directors.
#include <cuda_runtime.h>

#include "eb_internal.h"
#include "rod_math.cuh"

namespace eb {
namespace {

using D3 = Vec3<double>;

__device__ __forceinline__ D3 ld3(const double* __restrict__ p, int64_t S, int64_t g) {
  return {p[g], p[S + g], p[2 * S + g]};
}

// energies of the rod in slots [o, o + n], lane 0 returns the sums;
// gpot (optional): gravitational potential -sum m g.x is returned too
__device__ __forceinline__ void rod_energy_warp(int64_t o, int64_t n, int64_t S, const double* __restrict__ st,
                                                const double* __restrict__ par, const double* gvec, double& et,
                                                double& er, double& es, double& eb, double& ep) {
  const int lane = threadIdx.x & 31;
  et = 0.0, er = 0.0, es = 0.0, eb = 0.0, ep = 0.0;
  for (int64_t j = lane; j <= n; j += 32) {
    const int64_t g = o + j;
    const D3 v = ld3(st + kStV * S, S, g);
    et += par[kMass * S + g] * (v.x * v.x + v.y * v.y + v.z * v.z);
    if (gvec) {
      const D3 x = ld3(st + kStX * S, S, g);
      ep -= par[kMass * S + g] * (gvec[0] * x.x + gvec[1] * x.y + gvec[2] * x.z);
    }
    if (j < n) {
      const D3 dx = ld3(st + kStX * S, S, g + 1) - ld3(st + kStX * S, S, g);
      const double l = sqrt(dx.x * dx.x + dx.y * dx.y + dx.z * dx.z);
      const double e = l / par[kL0 * S + g];
      const D3 w = ld3(st + kStW * S, S, g);
      const D3 J = ld3(par + kJ * S, S, g);
      er += w.x * (J.x * w.x / e) + w.y * (J.y * w.y / e) + w.z * (J.z * w.z / e);
      double q[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) q[k] = st[(kStQ + k) * S + g];
      const D3 qt = matvec(q, divide(dx, l));
      const D3 s0 = ld3(par + kSig0 * S, S, g);
      const D3 sh = ld3(par + kShear * S, S, g);
      const D3 d = {qt.x * e - s0.x, qt.y * e - s0.y, qt.z * e - 1.0 - s0.z};
      es += (d.x * (sh.x * d.x) + d.y * (sh.y * d.y) + d.z * (sh.z * d.z)) * par[kL0 * S + g];
      if (j + 1 < n) {
        double qn[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) qn[k] = st[(kStQ + k) * S + g + 1];
        const D3 kp = inv_rotate_divide(q, qn, par[kD0 * S + g]);
        const D3 k0 = ld3(par + kKap0 * S, S, g);
        const D3 B = ld3(par + kBend * S, S, g);
        const D3 dk = kp - k0;
        eb += (dk.x * (B.x * dk.x) + dk.y * (B.y * dk.y) + dk.z * (B.z * dk.z)) * par[kD0 * S + g];
      }
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    et += __shfl_down_sync(0xffffffffu, et, off);
    er += __shfl_down_sync(0xffffffffu, er, off);
    es += __shfl_down_sync(0xffffffffu, es, off);
    eb += __shfl_down_sync(0xffffffffu, eb, off);
    ep += __shfl_down_sync(0xffffffffu, ep, off);
  }
}

__global__ void rod_energy_kernel(int64_t n_rods, int64_t S, const int64_t* __restrict__ offsets,
                                  const double* __restrict__ st, const double* __restrict__ par,
                                  double* __restrict__ out) {
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n_rods) return;
  const int64_t o = offsets[warp];
  const int64_t n = offsets[warp + 1] - o - 1;
  double et, er, es, eb, ep;
  rod_energy_warp(o, n, S, st, par, nullptr, et, er, es, eb, ep);
  if (lane == 0) {
    out[4 * warp + 0] = 0.5 * et;
    out[4 * warp + 1] = 0.5 * er;
    out[4 * warp + 2] = 0.5 * es;
    out[4 * warp + 3] = 0.5 * eb;
  }
}

// rods given by their first slot and element count; out[5 r + 4] is the
// gravitational potential -sum m g.x of rod r
__global__ void rod_energy_list_kernel(int64_t n_rods, int64_t S, const int64_t* __restrict__ start,
                                       const int32_t* __restrict__ n_el, const double* __restrict__ st,
                                       const double* __restrict__ par, double g0, double g1, double g2,
                                       double* __restrict__ out) {
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n_rods) return;
  const double gvec[3] = {g0, g1, g2};
  double et, er, es, eb, ep;
  rod_energy_warp(start[warp], n_el[warp], S, st, par, gvec, et, er, es, eb, ep);
  if (lane == 0) {
    out[5 * warp + 0] = 0.5 * et;
    out[5 * warp + 1] = 0.5 * er;
    out[5 * warp + 2] = 0.5 * es;
    out[5 * warp + 3] = 0.5 * eb;
    out[5 * warp + 4] = ep;
  }
}

}  // namespace

cudaError_t launch_rod_energy_list(int64_t n_rods, int64_t stride, const int64_t* start, const int32_t* n_el,
                                   const double* state, const double* params, const double gravity[3], double* out,
                                   cudaStream_t stream) {
  if (n_rods <= 0) return cudaSuccess;
  constexpr int kThreads = 256;
  const unsigned grid = static_cast<unsigned>((n_rods * 32 + kThreads - 1) / kThreads);
  rod_energy_list_kernel<<<grid, kThreads, 0, stream>>>(n_rods, stride, start, n_el, state, params, gravity[0],
                                                        gravity[1], gravity[2], out);
  return cudaGetLastError();
}

cudaError_t launch_rod_energy(int64_t n_rods, int64_t stride, const int64_t* offsets,
                              const double* state, const double* params, double* out,
                              cudaStream_t stream) {
  if (n_rods <= 0) return cudaSuccess;
  constexpr int kThreads = 256;
  const int64_t threads = n_rods * 32;
  const unsigned grid = static_cast<unsigned>((threads + kThreads - 1) / kThreads);
  rod_energy_kernel<<<grid, kThreads, 0, stream>>>(n_rods, stride, offsets, state, params, out);
  return cudaGetLastError();
}

}  // namespace eb
