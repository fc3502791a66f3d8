// Resident multi-step PositionVerlet kernel, mixed precision.
//
// Same structure as rod_block_fp64.cu (whole rods staged in shared memory,
// many steps per launch, both half drifts per step), with the element-local
// arithmetic in FP32 and everything whose stability needs FP64 kept in FP64:
//
//   FP64: positions, velocities, directors and angular velocities (state and
//         their accumulation, including the director's exponential update,
//         whose rounding would otherwise erode the orthonormality the
//         curvature relies on), the position difference of an element, the
//         shear/stretch strain sigma = Q dx / l0 - z of nearly inextensible
//         rods (a cancellation), the curvature's skew products and trace
//         (cancellations between neighbouring directors).
//   FP32: lengths, tangents, dilatations, constitutive products, internal
//         loads and couples, accelerations, the damping factors.
//
// Reformulations (mathematically identical; rounding differs):
//   sigma = (Q t) e - z  =  Q dx / l0 - z         (no normalisation)
//   rate  = (t . dv) / (e l0)  =  (t . dv) / l
//   theta = acos(c) = 2 asin(sqrt((1 - c) / 2)),  sin(theta) = sqrt((1-c)(1+c))
// and the reference's 1e-14 guard inside sin(theta + 1e-14) is dropped (it
// moves the curvature by less than 1e-9 relative at the smallest angle the
// 1e-10 shift of the trace allows); theta / sin(theta) comes from its series
// 1 + y/3 + 2y^2/15 in y = 1 - cos(theta) below y = 1e-3.
#include <cuda_runtime.h>

#include "eb_internal.h"
#include "rod_math.cuh"

namespace eb {
namespace {

using D3 = Vec3<double>;
using F3 = Vec3<float>;

// FP64 rows
enum MixedRowD : int { dX = 0, dV = 3, dQ = 6, dW = 15, dInvL0 = 18, dRowsD = 19 };
// FP32 rows
enum MixedRowF : int {
  fMass = 0, fL0 = 1, fD0 = 2, fSig0 = 3, fKap0 = 6, fShear = 9, fBend = 12, fJ = 15, fJinv = 18,
  fNuF = 21, fNuT = 22,
  fL = 23, fE = 24, fF = 25, fG = 28, fH = 31, fTl = 34, fRowsF = 37
};

template <int kCap>
struct MRows {
  double* d;
  float* f;
  __device__ __forceinline__ double& ad(int r, int s) const { return d[r * kCap + s]; }
  __device__ __forceinline__ float& af(int r, int s) const { return f[r * kCap + s]; }
  __device__ __forceinline__ D3 d3(int r, int s) const { return {ad(r, s), ad(r + 1, s), ad(r + 2, s)}; }
  __device__ __forceinline__ void pd3(int r, int s, D3 v) const {
    ad(r, s) = v.x;
    ad(r + 1, s) = v.y;
    ad(r + 2, s) = v.z;
  }
  __device__ __forceinline__ F3 f3(int r, int s) const { return {af(r, s), af(r + 1, s), af(r + 2, s)}; }
  __device__ __forceinline__ void pf3(int r, int s, F3 v) const {
    af(r, s) = v.x;
    af(r + 1, s) = v.y;
    af(r + 2, s) = v.z;
  }
};

__device__ __forceinline__ F3 tof(D3 a) {
  return {static_cast<float>(a.x), static_cast<float>(a.y), static_cast<float>(a.z)};
}

template <int kCap>
__device__ __forceinline__ void half_drift(const MRows<kCap>& R, int s, uint32_t meta, double hdt) {
  const D3 v = R.d3(dV, s);
  const D3 x = R.d3(dX, s);
  R.pd3(dX, s, D3{x.x + hdt * v.x, x.y + hdt * v.y, x.z + hdt * v.z});
  if (meta & kElem) {
    const D3 w = R.d3(dW, s);
    double q[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) q[k] = R.ad(dQ + k, s);
    so3_update_fast(q, hdt * w.x, hdt * w.y, hdt * w.z);
#pragma unroll
    for (int k = 0; k < 9; ++k) R.ad(dQ + k, s) = q[k];
  }
}

__device__ __forceinline__ int mixed_param_row(int f) {
  switch (f) {
    case kMass: return fMass;
    case kL0: return fL0;
    case kD0: return fD0;
    case kNuF: return fNuF;
    case kNuT: return fNuT;
    default: break;
  }
  if (f >= kSig0 && f < kSig0 + 3) return fSig0 + (f - kSig0);
  if (f >= kKap0 && f < kKap0 + 3) return fKap0 + (f - kKap0);
  if (f >= kShear && f < kShear + 3) return fShear + (f - kShear);
  if (f >= kBend && f < kBend + 3) return fBend + (f - kBend);
  if (f >= kJ && f < kJ + 3) return fJ + (f - kJ);
  if (f >= kJinv && f < kJinv + 3) return fJinv + (f - kJinv);
  return -1;
}

template <int kCap, int kThreads, int kMinBlocks, bool kDamped>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    rod_block_mixed_kernel(const StepArgs a, const int64_t* cta_start, int n_steps) {
  extern __shared__ __align__(128) double smem[];
  const MRows<kCap> R{smem, reinterpret_cast<float*>(smem + dRowsD * kCap)};
  uint32_t* meta_s = reinterpret_cast<uint32_t*>(R.f + fRowsF * kCap);

  const int tid = threadIdx.x;
  const int64_t g0 = cta_start[blockIdx.x];
  const int count = static_cast<int>(cta_start[blockIdx.x + 1] - g0);
  const int64_t S = a.stride;

  for (int s = tid; s < count; s += kThreads) {
    const int64_t g = g0 + s;
    meta_s[s] = a.meta[g];
#pragma unroll 1
    for (int f = 0; f < kStateFields; ++f) R.ad(f, s) = a.in[f * S + g];
    const double l0 = a.par[kL0 * S + g];
    R.ad(dInvL0, s) = 1.0 / l0;
#pragma unroll 1
    for (int f = 0; f < kParamFields; ++f) {
      const int r = mixed_param_row(f);
      if (r < 0 || (!kDamped && (f == kNuF || f == kNuT))) continue;
      R.af(r, s) = static_cast<float>(a.par[f * S + g]);
    }
  }
  __syncthreads();

  const double dt = a.dt, hdt = a.half_dt;
  const float dtf = static_cast<float>(dt);
  const bool any_rod = (a.sim_flags & (kSimClamp | kSimDamper | kSimEndTorque)) != 0;
  const F3 grav = {static_cast<float>(a.gravity[0]), static_cast<float>(a.gravity[1]),
                   static_cast<float>(a.gravity[2])};

  for (int step = 0; step < n_steps; ++step) {
    // ---- first half drift (the second one of the previous step was applied
    // at the end of its update phase) and clamp value constraint
    for (int s = tid; s < count; s += kThreads) {
      const uint32_t meta = meta_s[s];
      half_drift(R, s, meta, hdt);
      if (any_rod && (meta & kFirst)) {
        const RodInfo& ri = a.rods[meta >> kRodShift];
        if (ri.flags & kRodClamp) {
          R.pd3(dX, s, D3{ri.clamp_x[0], ri.clamp_x[1], ri.clamp_x[2]});
#pragma unroll
          for (int k = 0; k < 9; ++k) R.ad(dQ + k, s) = ri.clamp_Q[k];
        }
      }
    }
    __syncthreads();

    // ---- element geometry, internal stress, element-local torque terms
    for (int s = tid; s < count; s += kThreads) {
      const uint32_t meta = meta_s[s];
      F3 f{0.f, 0.f, 0.f}, tl{0.f, 0.f, 0.f};
      float l = 1.f, e = 1.f;
      if (meta & kElem) {
        const D3 dx = R.d3(dX, s + 1) - R.d3(dX, s);
        double qd[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
          qd[k] = R.ad(dQ + 3 * k, s) * dx.x + R.ad(dQ + 3 * k + 1, s) * dx.y + R.ad(dQ + 3 * k + 2, s) * dx.z;
        const double il0 = R.ad(dInvL0, s);
        const F3 s0 = R.f3(fSig0, s);
        const F3 d = {static_cast<float>(qd[0] * il0 - static_cast<double>(s0.x)),
                      static_cast<float>(qd[1] * il0 - static_cast<double>(s0.y)),
                      static_cast<float>((qd[2] * il0 - 1.0) - static_cast<double>(s0.z))};
        l = sqrtf(static_cast<float>(dx.x * dx.x + dx.y * dx.y + dx.z * dx.z));
        const float il = 1.f / l;
        const F3 t = scale(tof(dx), il);
        e = l * static_cast<float>(il0);
        const F3 sh = R.f3(fShear, s);
        const F3 nl = {sh.x * d.x, sh.y * d.y, sh.z * d.z};
        float qf[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) qf[k] = static_cast<float>(R.ad(dQ + k, s));
        const float ie = 1.f / e;
        f = scale(mattranspvec(qf, nl), ie);
        const F3 qt = matvec(qf, t);
        const F3 w = tof(R.d3(dW, s));
        const F3 J = R.f3(fJ, s);
        const F3 jwe = {J.x * w.x * ie, J.y * w.y * ie, J.z * w.z * ie};
        const F3 dv = tof(R.d3(dV, s + 1) - R.d3(dV, s));
        const float rate = dot(t, dv) * il;
        tl = scale(cross(qt, nl), R.af(fL0, s)) + cross(jwe, w) + scale(jwe, rate);
      }
      R.af(fL, s) = l;
      R.af(fE, s) = e;
      R.pf3(fF, s, f);
      R.pf3(fTl, s, tl);
    }
    __syncthreads();

    // ---- Voronoi curvature and couple
    for (int s = tid; s < count; s += kThreads) {
      const uint32_t meta = meta_s[s];
      F3 gg{0.f, 0.f, 0.f}, hh{0.f, 0.f, 0.f};
      if (meta & kVor) {
        double qc[9], qn[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          qc[k] = R.ad(dQ + k, s);
          qn[k] = R.ad(dQ + k, s + 1);
        }
        const double tr = qc[0] * qn[0] + qc[1] * qn[1] + qc[2] * qn[2] + qc[3] * qn[3] + qc[4] * qn[4] +
                          qc[5] * qn[5] + qc[6] * qn[6] + qc[7] * qn[7] + qc[8] * qn[8];
        // 1 - cos(theta) with the reference's 1e-10 shift
        const float y = fmaxf(static_cast<float>((1.5 + 1e-10) - 0.5 * tr), 0.f);
        float ratio;  // theta / sin(theta)
        if (y < 1e-3f) {
          ratio = 1.f + y * (1.f / 3.f + y * (2.f / 15.f));
        } else {
          ratio = 2.f * asinf(sqrtf(0.5f * y)) / sqrtf(y * (2.f - y));
        }
        const float D0 = R.af(fD0, s);
        const float st = 0.5f * ratio / D0;
        const F3 skew = {static_cast<float>(-qc[3] * qn[6] - qc[4] * qn[7] - qc[5] * qn[8] + qc[6] * qn[3] +
                                            qc[7] * qn[4] + qc[8] * qn[5]),
                         static_cast<float>(qc[0] * qn[6] + qc[1] * qn[7] + qc[2] * qn[8] - qc[6] * qn[0] -
                                            qc[7] * qn[1] - qc[8] * qn[2]),
                         static_cast<float>(-qc[0] * qn[3] - qc[1] * qn[4] - qc[2] * qn[5] + qc[3] * qn[0] +
                                            qc[4] * qn[1] + qc[5] * qn[2])};
        const F3 kappa = scale(skew, st);
        const float eps = 0.5f * (R.af(fL, s) + R.af(fL, s + 1)) / D0;
        const float ic = 1.f / (eps * eps * eps);
        const F3 dk = kappa - R.f3(fKap0, s);
        const F3 B = R.f3(fBend, s);
        const F3 tau = {B.x * dk.x, B.y * dk.y, B.z * dk.z};
        gg = scale(tau, ic);
        hh = scale(cross(kappa, tau), ic * D0);
      }
      R.pf3(fG, s, gg);
      R.pf3(fH, s, hh);
    }
    __syncthreads();

    // ---- loads, torques, accelerations, kick, rate constraints, second half drift
    for (int s = tid; s < count; s += kThreads) {
      const uint32_t meta = meta_s[s];
      const bool first = (meta & kFirst) != 0;
      const float m = R.af(fMass, s);
      D3 v = R.d3(dV, s);
      F3 F = R.f3(fF, s);
      if (!first) F = F - R.f3(fF, s - 1);
      if (kDamped) {
        const float cf = m * R.af(fNuF, s);
        const F3 vf = tof(v);
        F = {F.x - cf * vf.x, F.y - cf * vf.y, F.z - cf * vf.z};
      }
      if (a.sim_flags & kSimGravity) F = F + F3{grav.x * m, grav.y * m, grav.z * m};
      const float im = 1.f / m;
      v = {v.x + dt * static_cast<double>(F.x * im), v.y + dt * static_cast<double>(F.y * im),
           v.z + dt * static_cast<double>(F.z * im)};
      D3 w{0.0, 0.0, 0.0};
      const RodInfo* ri = any_rod ? a.rods + (meta >> kRodShift) : nullptr;
      if (meta & kElem) {
        const float e = R.af(fE, s);
        w = R.d3(dW, s);
        F3 T = R.f3(fG, s);
        F3 Q2 = R.f3(fH, s);
        if (!first) {
          T = T - R.f3(fG, s - 1);
          Q2 = Q2 + R.f3(fH, s - 1);
        }
        T = T + scale(Q2, 0.5f) + R.f3(fTl, s);
        if (kDamped) {
          const float ct = 0.5f * (m + R.af(fMass, s + 1)) * R.af(fNuT, s);
          const F3 wf = tof(w);
          T = {T.x - ct * wf.x, T.y - ct * wf.y, T.z - ct * wf.z};
        }
        if (any_rod && (meta & kLastElem) && (ri->flags & kRodEndTorque)) {
          float qf[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) qf[k] = static_cast<float>(R.ad(dQ + k, s));
          T = T + matvec(qf, F3{static_cast<float>(ri->end_torque[0]), static_cast<float>(ri->end_torque[1]),
                                static_cast<float>(ri->end_torque[2])});
        }
        const F3 ji = R.f3(fJinv, s);
        w = {w.x + dt * static_cast<double>(ji.x * T.x * e), w.y + dt * static_cast<double>(ji.y * T.y * e),
             w.z + dt * static_cast<double>(ji.z * T.z * e)};
        if (any_rod && (ri->flags & kRodDamper)) {
          const float mn = R.af(fMass, s + 1);
          float em = 0.5f * (m + mn);
          if (first) em += 0.5f * m;
          if (meta & kLastElem) em += 0.5f * mn;
          const float y = -static_cast<float>(ri->damper_r) * em * dtf * e;
          w = {w.x * static_cast<double>(expf(y * ji.x)), w.y * static_cast<double>(expf(y * ji.y)),
               w.z * static_cast<double>(expf(y * ji.z))};
        }
      }
      if (any_rod) {
        if (first && (ri->flags & kRodClamp)) {
          v = D3{0.0, 0.0, 0.0};
          w = D3{0.0, 0.0, 0.0};
        }
        if (ri->flags & kRodDamper) v = scale(v, ri->damper_t);
      }
      R.pd3(dV, s, v);
      if (meta & kElem) R.pd3(dW, s, w);
      half_drift(R, s, meta, hdt);
    }
    __syncthreads();
  }

  // ---- write-back (the last step's second half drift is already applied)
  for (int s = tid; s < count; s += kThreads) {
    const uint32_t meta = meta_s[s];
    const int64_t g = g0 + s;
#pragma unroll
    for (int f = 0; f < 6; ++f) a.out[f * S + g] = R.ad(f, s);
    if (meta & kElem) {
#pragma unroll
      for (int f = 6; f < kStateFields; ++f) a.out[f * S + g] = R.ad(f, s);
    }
  }
}

template <int kCap, int kThreads, int kMinBlocks>
cudaError_t launch_mixed_cfg(const StepArgs& args, const int64_t* cta_start, int n_ctas, int n_steps, bool damped,
                             cudaStream_t stream) {
  const size_t bytes = size_t(dRowsD) * kCap * sizeof(double) + size_t(fRowsF) * kCap * sizeof(float) +
                       size_t(kCap) * sizeof(uint32_t);
  auto go = [&](auto kern) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e != cudaSuccess) return e;
    kern<<<n_ctas, kThreads, bytes, stream>>>(args, cta_start, n_steps);
    return cudaGetLastError();
  };
  return damped ? go(rod_block_mixed_kernel<kCap, kThreads, kMinBlocks, true>)
                : go(rod_block_mixed_kernel<kCap, kThreads, kMinBlocks, false>);
}

}  // namespace

cudaError_t launch_rod_block_mixed(const StepArgs& args, const int64_t* cta_start, int n_ctas, int n_steps,
                                   int config, bool damped, cudaStream_t stream) {
  if (n_ctas <= 0 || n_steps <= 0) return cudaSuccess;
  // the same capacities as the FP64 resident configurations (0/1: 520 slots,
  // 2/3: 264 slots); the smaller footprint allows two CTAs per SM at 264
  switch (config) {
    case 0: return launch_mixed_cfg<520, 512, 1>(args, cta_start, n_ctas, n_steps, damped, stream);
    case 1: return launch_mixed_cfg<520, 256, 1>(args, cta_start, n_ctas, n_steps, damped, stream);
    case 2: return launch_mixed_cfg<264, 256, 2>(args, cta_start, n_ctas, n_steps, damped, stream);
    case 3: return launch_mixed_cfg<264, 128, 2>(args, cta_start, n_ctas, n_steps, damped, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace eb
