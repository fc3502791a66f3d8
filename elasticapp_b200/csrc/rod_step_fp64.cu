// Fused FP64 PositionVerlet step for a ragged batch of Cosserat rods.
//
// One launch advances every rod by one full step of
// elastica/Time/SymplecticSteppers/Algorithms/PositionVerlet.hpp:49-88 in the
// phase order of elastica/Simulator/Interface/TimeSteppers/
// SymplecticSteppers.hpp:152-216:
//   kinematic half step (x += dt/2 v, Q <- exp(-dt/2 [w]x) Q)
//   value constraints (clamp)
//   internal forces and torques (geometry, strains, curvature, elasticity,
//   explicit damping), gravity and end-torque forcing, update_acceleration
//   dynamic step (v += dt a, w += dt alpha), rate constraints (clamp, damper)
//   kinematic half step
// reading the state once from HBM and writing it once (ping-pong buffers).
//
// Tiling: CTA b owns the slot range [b*kBlock, (b+1)*kBlock) regardless of
// rod boundaries.  Because the step reads the previous state from one buffer
// and writes the other, a tile can recompute its halo (one slot on the left,
// two on the right) redundantly, so rods of any length map onto fixed tiles
// without packing or per-rod launch shapes.  Rod ends need no special code:
// at an end the neighbouring slot holds no element / Voronoi point and
// contributes the zero the reference's ghosts contribute.
#include <cuda_runtime.h>

#include "eb_internal.h"
#include "rod_math.cuh"

namespace eb {
namespace {

constexpr int kBlock = 256;
constexpr int kW = kBlock + 3;  // smem index s <-> slot t0 - 1 + s

using D3 = Vec3<double>;

struct Smem {
  double x[3][kW];  // positions after the first half drift (later: h terms)
  double v[3][kW];  // velocities (later: g terms)
  double q[9][kW];  // directors after the first half drift
  double l[kW];     // element lengths
  double f[3][kW];  // Q^T n_L / e per element (zero where no element)
  double m[kW];     // node masses
};

__device__ __forceinline__ D3 ld3(const double* __restrict__ p, int64_t S, int64_t g) {
  return {p[g], p[S + g], p[2 * S + g]};
}
__device__ __forceinline__ void st3(double* __restrict__ p, int64_t S, int64_t g, D3 a) {
  p[g] = a.x;
  p[S + g] = a.y;
  p[2 * S + g] = a.z;
}
__device__ __forceinline__ D3 sm3(const double (*a)[kW], int s) { return {a[0][s], a[1][s], a[2][s]}; }
__device__ __forceinline__ void ss3(double (*a)[kW], int s, D3 v) {
  a[0][s] = v.x;
  a[1][s] = v.y;
  a[2][s] = v.z;
}

// Phase 1: load a slot, first kinematic half step, clamp value constraint.
__device__ __forceinline__ void phase_load(const StepArgs& a, Smem& sm, int s, int64_t g,
                                           uint32_t meta, bool valid, D3& x, D3& v, double q[9],
                                           D3& w, double& m) {
  const int64_t S = a.stride;
  if (!valid) {
    x = v = w = D3{0.0, 0.0, 0.0};
    m = 1.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) q[k] = 0.0;
  } else {
    const double* __restrict__ in = a.in;
    const double hdt = a.half_dt;
    v = ld3(in + kV * S, S, g);
    const D3 x0 = ld3(in + kX * S, S, g);
    x = {x0.x + hdt * v.x, x0.y + hdt * v.y, x0.z + hdt * v.z};
    m = a.par[kMass * S + g];
    if (meta & kElem) {
#pragma unroll
      for (int k = 0; k < 9; ++k) q[k] = in[(kQ + k) * S + g];
      w = ld3(in + kW * S, S, g);
      so3_update(q, hdt * w.x, hdt * w.y, hdt * w.z);
    } else {
      w = D3{0.0, 0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 9; ++k) q[k] = 0.0;
    }
    if ((a.sim_flags & kSimClamp) && (meta & kFirst)) {
      const RodInfo& ri = a.rods[meta >> kRodShift];
      if (ri.flags & kRodClamp) {
        x = {ri.clamp_x[0], ri.clamp_x[1], ri.clamp_x[2]};
#pragma unroll
        for (int k = 0; k < 9; ++k) q[k] = ri.clamp_Q[k];
      }
    }
  }
  ss3(sm.x, s, x);
  ss3(sm.v, s, v);
#pragma unroll
  for (int k = 0; k < 9; ++k) sm.q[k][s] = q[k];
  sm.m[s] = m;
}

struct ElemOut {
  double l, e;
  D3 t, qt, sigma, nl;
};

// Phase 2: element geometry and internal stress
// (CosseratRodSpanwiseGeometry.hpp:579-644, WithDiagonalLinearHyperElasticModel.hpp:198-238)
__device__ __forceinline__ ElemOut phase_element(const StepArgs& a, Smem& sm, int s, int64_t g,
                                                 uint32_t meta) {
  ElemOut o;
  if (!(meta & kElem)) {
    sm.l[s] = 1.0;
    ss3(sm.f, s, D3{0.0, 0.0, 0.0});
    o.l = o.e = 1.0;
    o.t = o.qt = o.sigma = o.nl = D3{0.0, 0.0, 0.0};
    return o;
  }
  const int64_t S = a.stride;
  const double* __restrict__ par = a.par;
  double q[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) q[k] = sm.q[k][s];
  const D3 dx = sm3(sm.x, s + 1) - sm3(sm.x, s);
  const double l = sqrt(dx.x * dx.x + dx.y * dx.y + dx.z * dx.z);
  const D3 t = divide(dx, l);
  const double e = l / par[kL0 * S + g];
  const D3 qt = matvec(q, t);
  const D3 sigma = {qt.x * e, qt.y * e, qt.z * e - 1.0};
  const D3 s0 = ld3(par + kSig0 * S, S, g);
  const D3 sh = ld3(par + kShear * S, S, g);
  const D3 d = sigma - s0;
  const D3 nl = {sh.x * d.x, sh.y * d.y, sh.z * d.z};
  const D3 f = divide(mattranspvec(q, nl), e);
  sm.l[s] = l;
  ss3(sm.f, s, f);
  o.l = l;
  o.e = e;
  o.t = t;
  o.qt = qt;
  o.sigma = sigma;
  o.nl = nl;
  return o;
}

struct VorOut {
  D3 kappa, tau;
  double eps;
};

// Phase 3: Voronoi curvature and couple
// (CosseratRodSpanwiseGeometry.hpp:652-664, WithDiagonalLinearHyperElasticModel.hpp:293-338)
__device__ __forceinline__ VorOut phase_voronoi(const StepArgs& a, Smem& sm, int s, int64_t g,
                                                uint32_t meta) {
  VorOut o;
  D3 gg{0.0, 0.0, 0.0}, hh{0.0, 0.0, 0.0};
  o.kappa = o.tau = D3{0.0, 0.0, 0.0};
  o.eps = 1.0;
  if (meta & kVor) {
    const int64_t S = a.stride;
    const double* __restrict__ par = a.par;
    double qc[9], qn[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      qc[k] = sm.q[k][s];
      qn[k] = sm.q[k][s + 1];
    }
    const double D0 = par[kD0 * S + g];
    const D3 kappa = inv_rotate_divide(qc, qn, D0);
    const double D = 0.5 * (sm.l[s] + sm.l[s + 1]);
    const double eps = D / D0;
    const double ic = 1.0 / (eps * eps * eps);
    const D3 k0 = ld3(par + kKap0 * S, S, g);
    const D3 B = ld3(par + kBend * S, S, g);
    const D3 dk = kappa - k0;
    const D3 tau = {B.x * dk.x, B.y * dk.y, B.z * dk.z};
    gg = scale(tau, ic);
    hh = scale(cross(kappa, tau), ic * D0);
    o.kappa = kappa;
    o.tau = tau;
    o.eps = eps;
  }
  // g and h reuse the velocity and position rows, free after phase 2
  ss3(sm.v, s, gg);
  ss3(sm.x, s, hh);
  return o;
}

template <bool kDiag, bool kDamped>
__global__ void __launch_bounds__(kBlock) rod_step_fp64_kernel(const StepArgs a) {
  __shared__ Smem sm;
  const int tid = threadIdx.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * kBlock;
  const int64_t S = a.stride;
  const int64_t n_slots = a.n_slots;

  // interior slot of this thread
  const int si = tid + 1;
  const int64_t g = t0 + tid;
  const bool valid = g < n_slots;
  const uint32_t meta = valid ? a.meta[g] : 0u;
  // halo slots: s = 0 (g = t0 - 1), s = kBlock + 1, kBlock + 2
  int hs = -1;
  int64_t hg = 0;
  if (tid < 3) {
    hs = (tid == 0) ? 0 : kBlock + tid;
    hg = t0 - 1 + hs;
  }
  const bool hvalid = (hs >= 0) && hg >= 0 && hg < n_slots;
  const uint32_t hmeta = hvalid ? a.meta[hg] : 0u;

  D3 x, v, w;
  double q[9], m;
  phase_load(a, sm, si, g, meta, valid, x, v, q, w, m);
  if (hs >= 0) {
    D3 hx, hv, hw;
    double hq[9], hm;
    phase_load(a, sm, hs, hg, hmeta, hvalid, hx, hv, hq, hw, hm);
  }
  __syncthreads();

  // element-local quantities; the right-most halo slot (s = kBlock + 2) only
  // supplies its position, so phase 2 covers s in [0, kBlock + 1]
  const ElemOut eo = phase_element(a, sm, si, g, meta);
  if (hs >= 0 && hs <= kBlock + 1) (void)phase_element(a, sm, hs, hg, hmeta);
  // element-local torque terms of the interior element, in the reference's
  // summation order (WithDiagonalLinearHyperElasticModel.hpp:341-384)
  D3 t_shear{0.0, 0.0, 0.0}, t_lag{0.0, 0.0, 0.0}, t_unst{0.0, 0.0, 0.0};
  D3 jwe{0.0, 0.0, 0.0};
  if (meta & kElem) {
    const double l0 = a.par[kL0 * S + g];
    t_shear = scale(cross(eo.qt, eo.nl), l0);
    const D3 J = ld3(a.par + kJ * S, S, g);
    jwe = divide(D3{J.x * w.x, J.y * w.y, J.z * w.z}, eo.e);
    t_lag = cross(jwe, w);
    const D3 dv = sm3(sm.v, si + 1) - sm3(sm.v, si);
    const double rate = dot(eo.t, dv) / (eo.e * l0);
    t_unst = scale(jwe, rate);
  }
  __syncthreads();

  const VorOut vo = phase_voronoi(a, sm, si, g, meta);
  if (hs == 0) (void)phase_voronoi(a, sm, hs, hg, hmeta);
  __syncthreads();

  if (!valid) return;

  // ---- forces on node si
  D3 F = sm3(sm.f, si) - sm3(sm.f, si - 1);
  const double* __restrict__ par = a.par;
  if (kDamped) {
    const double c = m * par[kNuF * S + g];
    F = {F.x - c * v.x, F.y - c * v.y, F.z - c * v.z};
  }
  D3 Fe{0.0, 0.0, 0.0};
  if (a.sim_flags & kSimGravity)
    Fe = {0.0 + a.gravity[0] * m, 0.0 + a.gravity[1] * m, 0.0 + a.gravity[2] * m};
  const double inv_m = 1.0 / m;
  const D3 acc = {(F.x + Fe.x) * inv_m, (F.y + Fe.y) * inv_m, (F.z + Fe.z) * inv_m};

  const RodInfo* ri = nullptr;
  if (a.sim_flags & (kSimClamp | kSimDamper | kSimEndTorque)) ri = a.rods + (meta >> kRodShift);

  // ---- torques on element si
  D3 T{0.0, 0.0, 0.0}, alpha{0.0, 0.0, 0.0};
  double jinv[3] = {0.0, 0.0, 0.0};
  if (meta & kElem) {
    T = sm3(sm.v, si) - sm3(sm.v, si - 1);                  // two-point difference of g
    const D3 h1 = sm3(sm.x, si), h0 = sm3(sm.x, si - 1);    // quadrature of h
    T = T + D3{0.5 * (h1.x + h0.x), 0.5 * (h1.y + h0.y), 0.5 * (h1.z + h0.z)};
    T = T + t_shear;
    T = T + t_lag;
    T = T + t_unst;
    if (kDamped) {
      const double em = 0.5 * (m + sm.m[si + 1]);
      const double c = em * par[kNuT * S + g];
      T = {T.x - c * w.x, T.y - c * w.y, T.z - c * w.z};
    }
    D3 Te{0.0, 0.0, 0.0};
    if ((a.sim_flags & kSimEndTorque) && (meta & kLastElem) && (ri->flags & kRodEndTorque)) {
      const D3 tl = {ri->end_torque[0], ri->end_torque[1], ri->end_torque[2]};
      Te = Te + matvec(q, tl);
    }
    jinv[0] = par[(kJinv + 0) * S + g];
    jinv[1] = par[(kJinv + 1) * S + g];
    jinv[2] = par[(kJinv + 2) * S + g];
    alpha = {(jinv[0] * (T.x + Te.x)) * eo.e, (jinv[1] * (T.y + Te.y)) * eo.e,
             (jinv[2] * (T.z + Te.z)) * eo.e};
  }

  // ---- dynamic step and rate constraints
  const double dt = a.dt;
  v = {v.x + dt * acc.x, v.y + dt * acc.y, v.z + dt * acc.z};
  if (meta & kElem) w = {w.x + dt * alpha.x, w.y + dt * alpha.y, w.z + dt * alpha.z};
  if ((a.sim_flags & kSimClamp) && (meta & kFirst) && (ri->flags & kRodClamp)) {
    v = D3{0.0, 0.0, 0.0};
    w = D3{0.0, 0.0, 0.0};
  }
  if ((a.sim_flags & kSimDamper) && (ri->flags & kRodDamper)) {
    const double tc = ri->damper_t;
    v = {v.x * tc, v.y * tc, v.z * tc};
    if (meta & kElem) {
      double em = 0.5 * (m + sm.m[si + 1]);
      if (meta & kFirst) em += 0.5 * m;
      if (meta & kLastElem) em += 0.5 * sm.m[si + 1];
      const double nur = ri->damper_r;
      const double r0 = exp(-nur * em * jinv[0] * dt);
      const double r1 = exp(-nur * em * jinv[1] * dt);
      const double r2 = exp(-nur * em * jinv[2] * dt);
      w = {w.x * pow(r0, eo.e), w.y * pow(r1, eo.e), w.z * pow(r2, eo.e)};
    }
  }

  // ---- second kinematic half step and store
  const double hdt = a.half_dt;
  x = {x.x + hdt * v.x, x.y + hdt * v.y, x.z + hdt * v.z};
  double* __restrict__ out = a.out;
  st3(out + kX * S, S, g, x);
  st3(out + kV * S, S, g, v);
  if (meta & kElem) {
    so3_update(q, hdt * w.x, hdt * w.y, hdt * w.z);
#pragma unroll
    for (int k = 0; k < 9; ++k) out[(kQ + k) * S + g] = q[k];
    st3(out + kW * S, S, g, w);
  }

  if (kDiag) {
    double* __restrict__ dg = a.diag;
    Fe = F;  // InternalLoads after damping
    st3(dg + kDLoads * S, S, g, Fe);
    st3(dg + kDAccel * S, S, g, acc);
    if (meta & kElem) {
      dg[kDLength * S + g] = eo.e * par[kL0 * S + g];
      dg[kDDil * S + g] = eo.e;
      st3(dg + kDTangent * S, S, g, eo.t);
      st3(dg + kDSigma * S, S, g, eo.sigma);
      st3(dg + kDStress * S, S, g, eo.nl);
      st3(dg + kDTorques * S, S, g, T);
      st3(dg + kDAlpha * S, S, g, alpha);
      dg[kDDim * S + g] = sqrt(M_1_PI * par[kVol * S + g] / eo.l);
    }
    if (meta & kVor) {
      dg[kDVDil * S + g] = vo.eps;
      st3(dg + kDKappa * S, S, g, vo.kappa);
      st3(dg + kDCouple * S, S, g, vo.tau);
    }
  }
}

}  // namespace

// The same source is compiled twice: the default object contracts
// multiply-adds into FMAs; the "strict" object (EB_STRICT_FP64, built with
// --fmad=false) rounds every product and sum separately, as the reference's
// scalar C++ does on a build without FMA contraction.
#ifdef EB_STRICT_FP64
#define EB_FP64_LAUNCHER launch_rod_step_fp64_strict
#else
#define EB_FP64_LAUNCHER launch_rod_step_fp64
#endif

cudaError_t EB_FP64_LAUNCHER(const StepArgs& args, bool diag, bool damped, cudaStream_t stream) {
  if (args.n_slots <= 0) return cudaSuccess;
  const unsigned grid = static_cast<unsigned>((args.n_slots + kBlock - 1) / kBlock);
  if (diag) {
    if (damped)
      rod_step_fp64_kernel<true, true><<<grid, kBlock, 0, stream>>>(args);
    else
      rod_step_fp64_kernel<true, false><<<grid, kBlock, 0, stream>>>(args);
  } else {
    if (damped)
      rod_step_fp64_kernel<false, true><<<grid, kBlock, 0, stream>>>(args);
    else
      rod_step_fp64_kernel<false, false><<<grid, kBlock, 0, stream>>>(args);
  }
  return cudaGetLastError();
}

}  // namespace eb
