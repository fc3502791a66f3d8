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
// (threads 2 .. kTile+1) are stored; the two slots on either side are
// recomputed halo (the stencils reach one slot left and two right).  Because
// the step reads the previous state from one buffer and writes the other,
// halos can be recomputed redundantly, so rods of any length map onto the
// same tiles without packing.  Rod ends need no special code: at an end the
// neighbouring slot holds no element / Voronoi point and contributes the zero
// that the reference's ghost slots contribute.
//
// Staging: one thread issues a bulk asynchronous copy (TMA, cp.async.bulk)
// per input field of the window into shared memory, in two stages on two
// mbarriers: the state and the node mass (all the first drift reads), then
// the other parameters, which land while the drift's rotation updates run.
// (Splitting the copies this way took the kernel from 9.97 to 10.9 G
// element-steps/s; a finer split, one stage per phase, lost a third.)  Both
// waits are bounded; the threads vote on them, and a CTA whose copies did
// not land in time records it in the status word, waits for the copies it
// issued and leaves.  The 128-slot windows run 5 CTAs per SM (96 registers a
// thread, 40 KB of shared memory a CTA); a thread keeps its slot's directors
// and angular velocity in registers from phase to phase.  (Re-reading all of
// the slot from shared memory instead, at 80 registers and six CTAs an SM
// with 1 / J formed from J, measured 6% slower; re-reading the directors as
// well as the values below, 2% slower.)  What a thread carries across the barriers is kept
// small: the position, velocity and mass are re-read from their rows in the
// last phase, and in the default build the three element-local torque terms
// travel as one sum; with no register spills left this took the step from
// 0.408 to 0.383 ms on the uneven batch.  Every field row of
// a window is 16-byte aligned in global memory because windows start on an
// even slot and every field array starts on a 256-byte boundary.  The values
// exchanged between neighbouring threads (element lengths, Q^T n_L / e, the
// couple terms) are written over input rows that only their own thread reads
// and has consumed, so shared memory holds one row per staged input field.
#include <cuda_runtime.h>

#include "bulk_copy.cuh"
#include "eb_internal.h"
#include "rod_math.cuh"

namespace eb {
namespace {

// shared-memory row of every staged input field: the 18 state rows, then the
// parameter rows the variant needs (nu_f/nu_t only for explicitly damped
// rods, the volume only when diagnostics are recorded)
template <bool kDamped, bool kDiag>
struct RowMap {
  static constexpr int param(int f) {
    return kStateFields + f - ((!kDamped && f > kNuF) ? 1 : 0) - ((!kDamped && f > kNuT) ? 1 : 0) -
           ((!kDiag && f > kVol) ? 1 : 0);
  }
  static constexpr bool needed(int f) {
    return !((!kDamped && (f == kNuF || f == kNuT)) || (!kDiag && f == kVol));
  }
  static constexpr int rows() { return kStateFields + kParamFields - (kDamped ? 0 : 2) - (kDiag ? 0 : 1); }
};

constexpr uint32_t kMaxPolls = 1u << 22;
// polls of the wait that follows a timeout: far above any copy's duration
// (seconds), so a CTA leaves only once the copies into its shared memory
// are done
constexpr uint32_t kDrainPolls = 1u << 30;

// bounded wait for a barrier phase; a caller-set bound (StepArgs::max_polls)
// polls without blocking, so a small one gives up before copies issued just
// before can land (to exercise the timeout path)
__device__ __forceinline__ bool wait_copies(const StepArgs& a, uint64_t* bar) {
  return a.max_polls ? mbar_test_bounded(bar, 0, a.max_polls) : mbar_wait_bounded(bar, 0, kMaxPolls);
}
using D3 = Vec3<double>;

template <int W>
struct Rows {
  double* base;
  __device__ __forceinline__ double* row(int r) const { return base + r * W; }
  __device__ __forceinline__ double& at(int r, int s) const { return base[r * W + s]; }
  __device__ __forceinline__ D3 get3(int r, int s) const {
    return {base[r * W + s], base[(r + 1) * W + s], base[(r + 2) * W + s]};
  }
  __device__ __forceinline__ void put3(int r, int s, D3 v) const {
    base[r * W + s] = v.x;
    base[(r + 1) * W + s] = v.y;
    base[(r + 2) * W + s] = v.z;
  }
};

__device__ __forceinline__ void st3(double* __restrict__ p, int64_t S, int64_t g, D3 a) {
  p[g] = a.x;
  p[S + g] = a.y;
  p[2 * S + g] = a.z;
}

__device__ __forceinline__ void so3(double q[9], double u0, double u1, double u2) {
#ifdef EB_FAST_FP64
  so3_update_fast(q, u0, u1, u2);
#else
  so3_update(q, u0, u1, u2);
#endif
}

__device__ __forceinline__ D3 curvature(const double qc[9], const double qn[9], double span) {
#ifdef EB_FAST_FP64
  return inv_rotate_divide_fast(qc, qn, span);
#else
  return inv_rotate_divide(qc, qn, span);
#endif
}

// the clamp's value constraint on a slot a clamp holds: the node's position
// and, where the slot holds an element, its directors
__device__ __forceinline__ void clamp_value(const RodInfo& ri, uint32_t hits, uint32_t meta, D3& x, double q[9]) {
  const bool c0 = (hits & kHitClamp0) != 0;
  const double* tx = c0 ? ri.clamp_x : ri.clamp2_x;
  const double* tq = c0 ? ri.clamp_Q : ri.clamp2_Q;
  x = {tx[0], tx[1], tx[2]};
  if (meta & kElem) {
#pragma unroll
    for (int k = 0; k < 9; ++k) q[k] = tq[k];
  }
}

template <int W, bool kDiag, bool kDamped, bool kContact>
__device__ __forceinline__ void rod_step_window(const StepArgs& a, double* smem) {
  using M = RowMap<kDamped, kDiag>;
  constexpr int kTile = W - 4;  // interior slots stored per CTA (even)
  constexpr int kLeftHalo = 2;  // window starts 2 slots left of the tile
  constexpr int kRows = M::rows();
  // rows of the inputs
  constexpr int rX = kStX, rV = kStV, rQ = kStQ, rW = kStW;
  constexpr int rMass = M::param(kMass), rL0 = M::param(kL0), rD0 = M::param(kD0);
  constexpr int rSig0 = M::param(kSig0), rKap0 = M::param(kKap0), rShear = M::param(kShear);
  constexpr int rBend = M::param(kBend), rJ = M::param(kJ), rJinv = M::param(kJinv);
  constexpr int rNuF = M::param(kNuF), rNuT = M::param(kNuT), rVol = M::param(kVol);
  // exchange rows, each over rows only the owning thread reads:
  //   f (written in phase 2) over the angular velocity rows (read in phase 1)
  //   l (phase 2) over the first rest-strain row (read earlier in phase 2)
  //   g, h (phase 3) over the inertia and shear rigidity rows (read in phase 2)
  constexpr int rF = rW, rL = rSig0, rG = rJ, rH = rShear;

  const Rows<W> R{smem};
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kRows * W);

  const int s = threadIdx.x;
  const int64_t g0 = static_cast<int64_t>(blockIdx.x) * kTile - kLeftHalo;
  const int64_t g = g0 + s;
  const int64_t S = a.stride;
  const bool valid = g >= 0 && g < a.n_slots;
  const bool interior = valid && s >= kLeftHalo && s < kLeftHalo + kTile;
  const uint32_t meta = valid ? a.meta[g] : 0u;
  // per-rod constraint data, fetched while the bulk copies are in flight:
  // the slot's hits (which clamp holds it, the torque, the damper) and the
  // damper's constants
  uint32_t hits = 0;
  double damper_t = 1.0, damper_r = 0.0;
  if (valid && (a.sim_flags & (kSimClamp | kSimDamper | kSimEndTorque))) {
    const RodInfo& ri = a.rods[meta >> kRodShift];
    hits = slot_hits(ri, g);
    damper_t = ri.damper_t;
    damper_r = ri.damper_r;
  }

  // ---- stage the window's inputs with bulk copies (issuing them before the
  // loads above, which wait on the metadata word, measured no faster)
  if (s == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (s == 0) {
    const int64_t lo = g0 < 0 ? 0 : g0;
    const int64_t hi = (g0 + W < S) ? g0 + W : S;
    const uint32_t bytes = static_cast<uint32_t>((hi - lo) * sizeof(double));
    const int off = static_cast<int>(lo - g0);
    // the state and the node mass (the first drift's inputs) on bar[0], the
    // other parameters on bar[1], so the drift starts before they land
    mbar_arrive_expect_tx(bar, bytes * static_cast<uint32_t>(kStateFields + 1));
#pragma unroll 1
    for (int f = 0; f < kStateFields; ++f) bulk_g2s(R.row(f) + off, a.in + f * S + lo, bytes, bar);
    bulk_g2s(R.row(M::param(kMass)) + off, a.par + kMass * S + lo, bytes, bar);
    mbar_arrive_expect_tx(bar + 1, bytes * static_cast<uint32_t>(kRows - kStateFields - 1));
#pragma unroll 1
    for (int f = 0; f < kParamFields; ++f)
      if (M::needed(f) && f != kMass) bulk_g2s(R.row(M::param(f)) + off, a.par + f * S + lo, bytes, bar + 1);
  }
  const bool ok0 = wait_copies(a, bar);

  const double hdt = a.drift_pre;

  // ---- phase 1: first kinematic half step and clamp value constraint,
  // in place in shared memory
  D3 x{0.0, 0.0, 0.0}, v{0.0, 0.0, 0.0}, w{0.0, 0.0, 0.0};
  double q[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) q[k] = 0.0;
  double m = 1.0;
  if (ok0 && valid) {
    v = R.get3(rV, s);
    const D3 x0 = R.get3(rX, s);
    x = {x0.x + hdt * v.x, x0.y + hdt * v.y, x0.z + hdt * v.z};
    if (meta & kElem) {
#pragma unroll
      for (int k = 0; k < 9; ++k) q[k] = R.at(rQ + k, s);
      w = R.get3(rW, s);
      so3(q, hdt * w.x, hdt * w.y, hdt * w.z);
    }
    if (hits & (kHitClamp0 | kHitClamp1)) clamp_value(a.rods[meta >> kRodShift], hits, meta, x, q);
    R.put3(rX, s, x);
#pragma unroll
    for (int k = 0; k < 9; ++k) R.at(rQ + k, s) = q[k];
  }
  const bool ok1 = ok0 && wait_copies(a, bar + 1);
  if (!__syncthreads_and(ok1)) {
    // a copy did not land within the bound (every thread agrees): record it,
    // wait for the copies issued into this CTA's shared memory so none is
    // left writing there, and leave
    if (s == 0) atomicOr(a.status, kStatusCopyTimeout);
    (void)mbar_wait_bounded(bar, 0, kDrainPolls);
    (void)mbar_wait_bounded(bar + 1, 0, kDrainPolls);
    return;
  }

  // ---- phase 2: element geometry and internal stress
  // (CosseratRodSpanwiseGeometry.hpp:579-644, WithDiagonalLinearHyperElasticModel.hpp:198-238)
  // and the element-local torque terms in the reference's summation order
  // (WithDiagonalLinearHyperElasticModel.hpp:341-384).  The last thread of
  // the window has no right neighbour and only supplies its position.
  const bool elem = (meta & kElem) && s + 1 < W;
  double l = 1.0, e = 1.0, l0 = 1.0;
  D3 t{0.0, 0.0, 0.0}, sigma{0.0, 0.0, 0.0}, nl{0.0, 0.0, 0.0};
  D3 t_shear{0.0, 0.0, 0.0}, t_lag{0.0, 0.0, 0.0}, t_unst{0.0, 0.0, 0.0};
  {
    D3 f{0.0, 0.0, 0.0};
    if (elem) {
      const D3 dx = R.get3(rX, s + 1) - x;
      l = sqrt(dx.x * dx.x + dx.y * dx.y + dx.z * dx.z);
      l0 = R.at(rL0, s);
      e = l / l0;
#ifdef EB_FAST_FP64
      // one reciprocal each of l and e; the dilatation rate (t . dv) / (e l0)
      // as (t . dv) / l (e l0 = l)
      const double il = 1.0 / l, ie = 1.0 / e;
      t = scale(dx, il);
#else
      t = divide(dx, l);
#endif
      const D3 qt = matvec(q, t);
      sigma = {qt.x * e, qt.y * e, qt.z * e - 1.0};
      const D3 d = sigma - R.get3(rSig0, s);
      const D3 sh = R.get3(rShear, s);
      nl = {sh.x * d.x, sh.y * d.y, sh.z * d.z};
      t_shear = scale(cross(qt, nl), l0);
      const D3 J = R.get3(rJ, s);
      const D3 dv = R.get3(rV, s + 1) - v;
#ifdef EB_FAST_FP64
      f = scale(mattranspvec(q, nl), ie);
      const D3 jwe = scale(D3{J.x * w.x, J.y * w.y, J.z * w.z}, ie);
      const double rate = dot(t, dv) * il;
#else
      f = divide(mattranspvec(q, nl), e);
      const D3 jwe = divide(D3{J.x * w.x, J.y * w.y, J.z * w.z}, e);
      const double rate = dot(t, dv) / (e * l0);
#endif
      t_lag = cross(jwe, w);
      t_unst = scale(jwe, rate);
#ifdef EB_FAST_FP64
      // one vector instead of three carried to phase 4 (the sum is
      // associated differently: a rounding-level change)
      t_shear = t_shear + t_lag + t_unst;
#endif
    }
    R.at(rL, s) = l;
    R.put3(rF, s, f);
  }
  __syncthreads();

  // ---- phase 3: Voronoi curvature and couple
  // (CosseratRodSpanwiseGeometry.hpp:652-664, WithDiagonalLinearHyperElasticModel.hpp:293-338)
  D3 kappa{0.0, 0.0, 0.0}, tau{0.0, 0.0, 0.0};
  double eps = 1.0;
  {
    D3 gg{0.0, 0.0, 0.0}, hh{0.0, 0.0, 0.0};
    if ((meta & kVor) && s + 1 < W) {
      double qn[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) qn[k] = R.at(rQ + k, s + 1);
      const double D0 = R.at(rD0, s);
      kappa = curvature(q, qn, D0);
      const double D = 0.5 * (l + R.at(rL, s + 1));
      eps = D / D0;
#ifdef EB_FAST_FP64
      const double ie = D0 / D;  // 1 / eps
      const double ic = ie * ie * ie;
#else
      const double ic = 1.0 / (eps * eps * eps);
#endif
      const D3 dk = kappa - R.get3(rKap0, s);
      const D3 B = R.get3(rBend, s);
      tau = {B.x * dk.x, B.y * dk.y, B.z * dk.z};
      gg = scale(tau, ic);
      hh = scale(cross(kappa, tau), ic * D0);
    }
    R.put3(rG, s, gg);
    R.put3(rH, s, hh);
  }
  __syncthreads();

  if (!interior) return;
  // the slot's drifted position, velocity and mass from its rows (phase 1
  // left them there), not carried in registers across the barriers
  x = R.get3(rX, s);
  v = R.get3(rV, s);
  m = R.at(rMass, s);

  // ---- phase 4: loads, update_acceleration (WithRodKinematics.hpp:684-714)
  D3 F = R.get3(rF, s) - R.get3(rF, s - 1);
  if (kDamped) {
    const double c = m * R.at(rNuF, s);
    F = {F.x - c * v.x, F.y - c * v.y, F.z - c * v.z};
  }
  D3 Fe{0.0, 0.0, 0.0};
  if (a.sim_flags & kSimGravity)
    Fe = {0.0 + a.gravity[0] * m, 0.0 + a.gravity[1] * m, 0.0 + a.gravity[2] * m};
  if (kContact && a.contact_force) {
    // collision system after gravity: the element before the node, then the
    // element at the node, each adding half its capsule force
    // (Systems/Customization/CosseratRods/Transfer/Common.hpp:32-55)
    const double* __restrict__ cf = a.contact_force;
    if (!(meta & kFirst)) Fe = {Fe.x + 0.5 * cf[g - 1], Fe.y + 0.5 * cf[S + g - 1], Fe.z + 0.5 * cf[2 * S + g - 1]};
    if (meta & kElem) Fe = {Fe.x + 0.5 * cf[g], Fe.y + 0.5 * cf[S + g], Fe.z + 0.5 * cf[2 * S + g]};
  }
  if (kContact && a.joint_force) {
    // connections after the collision system
    const double* __restrict__ jf = a.joint_force;
    Fe = {Fe.x + jf[g], Fe.y + jf[S + g], Fe.z + jf[2 * S + g]};
  }
  const double inv_m = 1.0 / m;
  const D3 acc = {(F.x + Fe.x) * inv_m, (F.y + Fe.y) * inv_m, (F.z + Fe.z) * inv_m};

  D3 T{0.0, 0.0, 0.0}, alpha{0.0, 0.0, 0.0};
  D3 jinv{0.0, 0.0, 0.0};
  if (meta & kElem) {
    T = R.get3(rG, s) - R.get3(rG, s - 1);                // two-point difference of g
    const D3 h1 = R.get3(rH, s), h0 = R.get3(rH, s - 1);  // quadrature of h
    T = T + D3{0.5 * (h1.x + h0.x), 0.5 * (h1.y + h0.y), 0.5 * (h1.z + h0.z)};
    T = T + t_shear;
#ifndef EB_FAST_FP64
    T = T + t_lag;
    T = T + t_unst;
#endif
    if (kDamped) {
      const double em = 0.5 * (m + R.at(rMass, s + 1));
      const double c = em * R.at(rNuT, s);
      T = {T.x - c * w.x, T.y - c * w.y, T.z - c * w.z};
    }
    D3 Te{0.0, 0.0, 0.0};
    if (kContact && a.contact_torque) {
      // the capsule torque recast into the material frame: Q tau
      const double* __restrict__ ct = a.contact_torque;
      Te = Te + matvec(q, D3{ct[g], ct[S + g], ct[2 * S + g]});
    }
    if (kContact && a.joint_torque) {
      // the connections' torque (summed in the lab frame), recast the same way
      const double* __restrict__ jt = a.joint_torque;
      Te = Te + matvec(q, D3{jt[g], jt[S + g], jt[2 * S + g]});
    }
    if (hits & kHitTorque) {
      const RodInfo& ri = a.rods[meta >> kRodShift];
      Te = Te + matvec(q, D3{ri.end_torque[0], ri.end_torque[1], ri.end_torque[2]});
    }
    jinv = R.get3(rJinv, s);
    alpha = {(jinv.x * (T.x + Te.x)) * e, (jinv.y * (T.y + Te.y)) * e, (jinv.z * (T.z + Te.z)) * e};
  }

  // ---- dynamic step and rate constraints
  const double dt = a.kick;
  v = {v.x + dt * acc.x, v.y + dt * acc.y, v.z + dt * acc.z};
  if (meta & kElem) w = {w.x + dt * alpha.x, w.y + dt * alpha.y, w.z + dt * alpha.z};
  if (hits & (kHitClamp0 | kHitClamp1)) {
    v = D3{0.0, 0.0, 0.0};
    w = D3{0.0, 0.0, 0.0};
  }
  if (hits & kHitDamper) {
    // exp(-nu_t dt) for a damper time of dt; another damper time (PEFRL's
    // fractional kicks) scales the exponent
    const double ddt = a.damper_time;
    if (ddt != a.dt) damper_t = exp(log(damper_t) * (ddt / a.dt));
    v = {v.x * damper_t, v.y * damper_t, v.z * damper_t};
    if (meta & kElem) {
      // AnalyticalLinearDamper.hpp:40-75: w_k *= exp(y_k)^e with
      // y_k = -nu_r m_e J^-1_k dt.  The reference-rounding build evaluates it
      // as written; the fast build uses exp(e y_k) (equal up to rounding, one
      // transcendental instead of two).
      const double mn = R.at(rMass, s + 1);
      double em = 0.5 * (m + mn);
      if (meta & kFirst) em += 0.5 * m;
      if (meta & kLastElem) em += 0.5 * mn;
      const double nur = damper_r;
#ifdef EB_FAST_FP64
      w = {w.x * exp(e * (-nur * em * jinv.x * ddt)), w.y * exp(e * (-nur * em * jinv.y * ddt)),
           w.z * exp(e * (-nur * em * jinv.z * ddt))};
#else
      w = {w.x * pow(exp(-nur * em * jinv.x * ddt), e), w.y * pow(exp(-nur * em * jinv.y * ddt), e),
           w.z * pow(exp(-nur * em * jinv.z * ddt), e)};
#endif
    }
  }

  // ---- second kinematic half step and store
  const double hdt2 = a.drift_post;
  x = {x.x + hdt2 * v.x, x.y + hdt2 * v.y, x.z + hdt2 * v.z};
  double* __restrict__ out = a.out;
  st3(out + kStX * S, S, g, x);
  st3(out + kStV * S, S, g, v);
  if (meta & kElem) {
    so3(q, hdt2 * w.x, hdt2 * w.y, hdt2 * w.z);
#pragma unroll
    for (int k = 0; k < 9; ++k) out[(kStQ + k) * S + g] = q[k];
    st3(out + kStW * S, S, g, w);
  }

  if (kDiag) {
    double* __restrict__ dg = a.diag;
    st3(dg + kDLoads * S, S, g, F);  // InternalLoads include the damping force
    st3(dg + kDAccel * S, S, g, acc);
    if (meta & kElem) {
      dg[kDLength * S + g] = e * l0;
      dg[kDDil * S + g] = e;
      st3(dg + kDTangent * S, S, g, t);
      st3(dg + kDSigma * S, S, g, sigma);
      st3(dg + kDStress * S, S, g, nl);
      st3(dg + kDTorques * S, S, g, T);
      st3(dg + kDAlpha * S, S, g, alpha);
      dg[kDDim * S + g] = sqrt(M_1_PI * R.at(rVol, s) / l);
    }
    if (meta & kVor) {
      dg[kDVDil * S + g] = eps;
      st3(dg + kDKappa * S, S, g, kappa);
      st3(dg + kDCouple * S, S, g, tau);
    }
  }
}

template <int W, int MinBlocks, bool kDiag, bool kDamped, bool kContact>
__global__ void __launch_bounds__(W, MinBlocks) rod_step_fp64_kernel(const StepArgs a) {
  extern __shared__ __align__(128) double smem[];
  rod_step_window<W, kDiag, kDamped, kContact>(a, smem);
}

template <int W, int MinBlocks, bool kDiag, bool kDamped, bool kContact>
cudaError_t launch_variant(const StepArgs& args, cudaStream_t stream) {
  constexpr int kTile = W - 4;
  constexpr size_t bytes = size_t(RowMap<kDamped, kDiag>::rows()) * W * sizeof(double) + 16;
  auto kern = rod_step_fp64_kernel<W, MinBlocks, kDiag, kDamped, kContact>;
  // the attribute is per device; setting it on every launch is cheap and
  // keeps multi-device use correct
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  if (e != cudaSuccess) return e;
  const unsigned grid = static_cast<unsigned>((args.n_slots + kTile - 1) / kTile);
  kern<<<grid, W, bytes, stream>>>(args);
  return cudaGetLastError();
}

template <int W, int MinBlocks, bool kContact>
cudaError_t launch_window_c(const StepArgs& args, bool diag, bool damped, cudaStream_t stream) {
  if (diag)
    return damped ? launch_variant<W, MinBlocks, true, true, kContact>(args, stream)
                  : launch_variant<W, MinBlocks, true, false, kContact>(args, stream);
  return damped ? launch_variant<W, MinBlocks, false, true, kContact>(args, stream)
                : launch_variant<W, MinBlocks, false, false, kContact>(args, stream);
}

template <int W, int MinBlocks>
cudaError_t launch_window(const StepArgs& args, bool diag, bool damped, cudaStream_t stream) {
  // the external-load variant: collision system and/or connections
  if ((args.contact_force && args.contact_torque) || (args.joint_force && args.joint_torque))
    return launch_window_c<W, MinBlocks, true>(args, diag, damped, stream);
  return launch_window_c<W, MinBlocks, false>(args, diag, damped, stream);
}

}  // namespace

// The same source is compiled twice.  The default object (EB_FAST_FP64)
// contracts multiply-adds into FMAs and uses the reformulations of
// rod_math.cuh, the damper as exp(e y) and one reciprocal per repeated
// divisor.  The reference-rounding object (built with --fmad=false) rounds
// every product and sum separately, as the reference's scalar C++ does
// without FMA contraction, and evaluates every expression as the reference
// writes it.  Both stay within the same distance of the reference after many
// steps (the rounding of any implementation is amplified alike); the second
// matches the reference's short-horizon golden vectors at its own tolerance.
#ifdef EB_FAST_FP64
#define EB_FP64_LAUNCHER launch_rod_step_fp64
#else
#define EB_FP64_LAUNCHER launch_rod_step_fp64_reference
#endif

// window: slots per CTA: 0 or 128 (the default: 128-slot windows, five CTAs
// an SM), 64 (ten), 96 (six) or 256 (two)
cudaError_t EB_FP64_LAUNCHER(const StepArgs& args, bool diag, bool damped, int window, cudaStream_t stream) {
  if (args.n_slots <= 0) return cudaSuccess;
  // every field row of a window must start on a 16-byte boundary
  if ((args.stride & 1) || (reinterpret_cast<uintptr_t>(args.in) & 15) ||
      (reinterpret_cast<uintptr_t>(args.par) & 15))
    return cudaErrorMisalignedAddress;
  if (window == 256) return launch_window<256, 2>(args, diag, damped, stream);
  if (window == 96) return launch_window<96, 6>(args, diag, damped, stream);
  if (window == 64) return launch_window<64, 10>(args, diag, damped, stream);
  return launch_window<128, 5>(args, diag, damped, stream);
}

}  // namespace eb
