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
// Tiling: overlapped fixed windows over the slot array, independent of rod
// boundaries.  CTA b runs kWindow threads over the slots
// [b*kTile - 2, b*kTile - 2 + kWindow); thread k owns slot b*kTile - 2 + k and
// computes every phase for it.  The outputs of the kTile interior slots
// (threads 2 .. kTile+1) are stored; the two slots on the left and on the
// right are recomputed halo (the stencils reach one slot left and two right).
// Because the step reads the previous state from one buffer and writes the
// other, halos can be recomputed redundantly, so rods of any length map onto
// the same tiles without packing.  Rod ends need no special code: at an end
// the neighbouring slot holds no element / Voronoi point and contributes the
// zero that the reference's ghost slots contribute.
#include <cuda_runtime.h>

#include "eb_internal.h"
#include "rod_math.cuh"

namespace eb {
namespace {

constexpr int kWindow = 256;            // threads per CTA = slots per window
constexpr int kTile = kWindow - 4;      // interior slots stored per CTA
constexpr int kLeftHalo = 2;            // window starts 2 slots left of the tile
constexpr int kMinBlocks = 2;           // CTAs per SM the register budget targets

using D3 = Vec3<double>;

struct Smem {
  double x[3][kWindow];  // positions after the first half drift (later: h terms)
  double v[3][kWindow];  // velocities (later: g terms)
  double q[9][kWindow];  // directors after the first half drift
  double l[kWindow];     // element lengths
  double f[3][kWindow];  // Q^T n_L / e per element (zero where no element)
  double m[kWindow];     // node masses
};

__device__ __forceinline__ D3 ld3(const double* __restrict__ p, int64_t S, int64_t g) {
  return {p[g], p[S + g], p[2 * S + g]};
}
__device__ __forceinline__ void st3(double* __restrict__ p, int64_t S, int64_t g, D3 a) {
  p[g] = a.x;
  p[S + g] = a.y;
  p[2 * S + g] = a.z;
}
__device__ __forceinline__ D3 sm3(const double (*a)[kWindow], int s) { return {a[0][s], a[1][s], a[2][s]}; }
__device__ __forceinline__ void ss3(double (*a)[kWindow], int s, D3 v) {
  a[0][s] = v.x;
  a[1][s] = v.y;
  a[2][s] = v.z;
}

template <bool kDiag, bool kDamped>
__global__ void __launch_bounds__(kWindow, kMinBlocks) rod_step_fp64_kernel(const StepArgs a) {
  __shared__ Smem sm;
  const int s = threadIdx.x;
  const int64_t g = static_cast<int64_t>(blockIdx.x) * kTile - kLeftHalo + s;
  const int64_t S = a.stride;
  const bool valid = g >= 0 && g < a.n_slots;
  const bool interior = valid && s >= kLeftHalo && s < kLeftHalo + kTile;
  const uint32_t meta = valid ? a.meta[g] : 0u;
  const double* __restrict__ in = a.in;
  const double* __restrict__ par = a.par;
  const double hdt = a.half_dt;

  // ---- phase 1: load, first kinematic half step, clamp value constraint
  D3 x{0.0, 0.0, 0.0}, v{0.0, 0.0, 0.0}, w{0.0, 0.0, 0.0};
  double q[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) q[k] = 0.0;
  double m = 1.0;
  if (valid) {
    v = ld3(in + kStV * S, S, g);
    const D3 x0 = ld3(in + kStX * S, S, g);
    x = {x0.x + hdt * v.x, x0.y + hdt * v.y, x0.z + hdt * v.z};
    m = par[kMass * S + g];
    if (meta & kElem) {
#pragma unroll
      for (int k = 0; k < 9; ++k) q[k] = in[(kStQ + k) * S + g];
      w = ld3(in + kStW * S, S, g);
      so3_update(q, hdt * w.x, hdt * w.y, hdt * w.z);
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
  __syncthreads();

  // ---- phase 2: element geometry and internal stress
  // (CosseratRodSpanwiseGeometry.hpp:579-644, WithDiagonalLinearHyperElasticModel.hpp:198-238)
  // and the element-local torque terms in the reference's summation order
  // (WithDiagonalLinearHyperElasticModel.hpp:341-384).  The last thread of
  // the window has no right neighbour and only supplies its position.
  const bool elem = (meta & kElem) && s + 1 < kWindow;
  double l = 1.0, e = 1.0;
  D3 t{0.0, 0.0, 0.0}, sigma{0.0, 0.0, 0.0}, nl{0.0, 0.0, 0.0};
  D3 t_shear{0.0, 0.0, 0.0}, t_lag{0.0, 0.0, 0.0}, t_unst{0.0, 0.0, 0.0};
  {
    D3 f{0.0, 0.0, 0.0};
    if (elem) {
      const D3 dx = sm3(sm.x, s + 1) - x;
      l = sqrt(dx.x * dx.x + dx.y * dx.y + dx.z * dx.z);
      t = divide(dx, l);
      const double l0 = par[kL0 * S + g];
      e = l / l0;
      const D3 qt = matvec(q, t);
      sigma = {qt.x * e, qt.y * e, qt.z * e - 1.0};
      const D3 s0 = ld3(par + kSig0 * S, S, g);
      const D3 sh = ld3(par + kShear * S, S, g);
      const D3 d = sigma - s0;
      nl = {sh.x * d.x, sh.y * d.y, sh.z * d.z};
      f = divide(mattranspvec(q, nl), e);
      t_shear = scale(cross(qt, nl), l0);
      const D3 J = ld3(par + kJ * S, S, g);
      const D3 jwe = divide(D3{J.x * w.x, J.y * w.y, J.z * w.z}, e);
      t_lag = cross(jwe, w);
      const D3 dv = sm3(sm.v, s + 1) - v;
      const double rate = dot(t, dv) / (e * l0);
      t_unst = scale(jwe, rate);
    }
    sm.l[s] = l;
    ss3(sm.f, s, f);
  }
  __syncthreads();

  // ---- phase 3: Voronoi curvature and couple
  // (CosseratRodSpanwiseGeometry.hpp:652-664, WithDiagonalLinearHyperElasticModel.hpp:293-338)
  D3 kappa{0.0, 0.0, 0.0}, tau{0.0, 0.0, 0.0};
  double eps = 1.0;
  {
    D3 gg{0.0, 0.0, 0.0}, hh{0.0, 0.0, 0.0};
    if ((meta & kVor) && s + 1 < kWindow) {
      double qn[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) qn[k] = sm.q[k][s + 1];
      const double D0 = par[kD0 * S + g];
      kappa = inv_rotate_divide(q, qn, D0);
      const double D = 0.5 * (l + sm.l[s + 1]);
      eps = D / D0;
      const double ic = 1.0 / (eps * eps * eps);
      const D3 k0 = ld3(par + kKap0 * S, S, g);
      const D3 B = ld3(par + kBend * S, S, g);
      const D3 dk = kappa - k0;
      tau = {B.x * dk.x, B.y * dk.y, B.z * dk.z};
      gg = scale(tau, ic);
      hh = scale(cross(kappa, tau), ic * D0);
    }
    // g and h reuse the velocity and position rows, free after phase 2
    ss3(sm.v, s, gg);
    ss3(sm.x, s, hh);
  }
  __syncthreads();

  if (!interior) return;

  // ---- phase 4: loads, update_acceleration (WithRodKinematics.hpp:684-714)
  D3 F = sm3(sm.f, s) - sm3(sm.f, s - 1);
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

  D3 T{0.0, 0.0, 0.0}, alpha{0.0, 0.0, 0.0};
  double jinv[3] = {0.0, 0.0, 0.0};
  if (meta & kElem) {
    T = sm3(sm.v, s) - sm3(sm.v, s - 1);                  // two-point difference of g
    const D3 h1 = sm3(sm.x, s), h0 = sm3(sm.x, s - 1);    // quadrature of h
    T = T + D3{0.5 * (h1.x + h0.x), 0.5 * (h1.y + h0.y), 0.5 * (h1.z + h0.z)};
    T = T + t_shear;
    T = T + t_lag;
    T = T + t_unst;
    if (kDamped) {
      const double em = 0.5 * (m + sm.m[s + 1]);
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
    alpha = {(jinv[0] * (T.x + Te.x)) * e, (jinv[1] * (T.y + Te.y)) * e, (jinv[2] * (T.z + Te.z)) * e};
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
      // AnalyticalLinearDamper.hpp:40-75: w_k *= exp(y_k)^e with
      // y_k = -nu_r m_e J^-1_k dt.  The reference-rounding build evaluates it
      // as written; the FMA build uses exp(e y_k) (equal up to rounding, one
      // transcendental instead of two).
      double em = 0.5 * (m + sm.m[s + 1]);
      if (meta & kFirst) em += 0.5 * m;
      if (meta & kLastElem) em += 0.5 * sm.m[s + 1];
      const double nur = ri->damper_r;
#ifdef EB_FMA_FP64
      w = {w.x * exp(e * (-nur * em * jinv[0] * dt)), w.y * exp(e * (-nur * em * jinv[1] * dt)),
           w.z * exp(e * (-nur * em * jinv[2] * dt))};
#else
      w = {w.x * pow(exp(-nur * em * jinv[0] * dt), e), w.y * pow(exp(-nur * em * jinv[1] * dt), e),
           w.z * pow(exp(-nur * em * jinv[2] * dt), e)};
#endif
    }
  }

  // ---- second kinematic half step and store
  x = {x.x + hdt * v.x, x.y + hdt * v.y, x.z + hdt * v.z};
  double* __restrict__ out = a.out;
  st3(out + kStX * S, S, g, x);
  st3(out + kStV * S, S, g, v);
  if (meta & kElem) {
    so3_update(q, hdt * w.x, hdt * w.y, hdt * w.z);
#pragma unroll
    for (int k = 0; k < 9; ++k) out[(kStQ + k) * S + g] = q[k];
    st3(out + kStW * S, S, g, w);
  }

  if (kDiag) {
    double* __restrict__ dg = a.diag;
    st3(dg + kDLoads * S, S, g, F);  // InternalLoads include the damping force
    st3(dg + kDAccel * S, S, g, acc);
    if (meta & kElem) {
      dg[kDLength * S + g] = e * par[kL0 * S + g];
      dg[kDDil * S + g] = e;
      st3(dg + kDTangent * S, S, g, t);
      st3(dg + kDSigma * S, S, g, sigma);
      st3(dg + kDStress * S, S, g, nl);
      st3(dg + kDTorques * S, S, g, T);
      st3(dg + kDAlpha * S, S, g, alpha);
      dg[kDDim * S + g] = sqrt(M_1_PI * par[kVol * S + g] / l);
    }
    if (meta & kVor) {
      dg[kDVDil * S + g] = eps;
      st3(dg + kDKappa * S, S, g, kappa);
      st3(dg + kDCouple * S, S, g, tau);
    }
  }
}

}  // namespace

// The same source is compiled twice.  The default object (built with
// --fmad=false) rounds every product and sum separately, as the reference's
// scalar C++ does without FMA contraction, and evaluates the damper as
// written: it tracks the reference to transcendental-rounding level.  The
// EB_FMA_FP64 object contracts multiply-adds into FMAs.
#ifdef EB_FMA_FP64
#define EB_FP64_LAUNCHER launch_rod_step_fp64_fma
#else
#define EB_FP64_LAUNCHER launch_rod_step_fp64
#endif

cudaError_t EB_FP64_LAUNCHER(const StepArgs& args, bool diag, bool damped, cudaStream_t stream) {
  if (args.n_slots <= 0) return cudaSuccess;
  const unsigned grid = static_cast<unsigned>((args.n_slots + kTile - 1) / kTile);
  if (diag) {
    if (damped)
      rod_step_fp64_kernel<true, true><<<grid, kWindow, 0, stream>>>(args);
    else
      rod_step_fp64_kernel<true, false><<<grid, kWindow, 0, stream>>>(args);
  } else {
    if (damped)
      rod_step_fp64_kernel<false, true><<<grid, kWindow, 0, stream>>>(args);
    else
      rod_step_fp64_kernel<false, false><<<grid, kWindow, 0, stream>>>(args);
  }
  return cudaGetLastError();
}

}  // namespace eb
