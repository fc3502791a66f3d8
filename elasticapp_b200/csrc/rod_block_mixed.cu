// Resident multi-step PositionVerlet kernel, mixed precision.
//
// Same structure as rod_block_fp64.cu (whole rods staged in shared memory,
// many steps per launch), with the element-local arithmetic in FP32 and
// everything whose stability needs FP64 kept in FP64:
//
//   FP64: positions, velocities, directors and angular velocities (state and
//         their accumulation, including the director's exponential update,
//         whose rounding would otherwise erode the orthonormality the
//         curvature relies on), the position difference of an element, the
//         shear/stretch strain sigma = Q dx / l0 - z of nearly inextensible
//         rods (a cancellation), the differences of neighbouring directors
//         from which the curvature is formed.
//   FP32: lengths, tangents, dilatations, constitutive products, internal
//         loads and couples, accelerations, the damping factors.
//
// The element phase converts the FP64 director and angular velocity it has
// loaded anyway to FP32 (FP32 shadow rows of both, refreshed whenever the
// FP64 values changed, cost 12 shared-memory stores and 12 loads a slot and
// step for the same values and 48 B of shared memory a slot), and the
// divisions of the element math are reciprocal square roots and rounded
// reciprocals (the reciprocals of the masses and Voronoi rest lengths are
// formed each step rather than stored: shared memory per slot, not the
// arithmetic, sets how many slots an SM holds).
//
// Reformulations (mathematically identical; rounding differs):
//   sigma = (Q t) e - z  =  Q dx / l0 - z         (no normalisation)
//   rate  = (t . dv) / (e l0)  =  (t . dv) / l,   1 / e = l0 / l
//   theta = acos(c) = 2 asin(sqrt((1 - c) / 2)),  sin(theta) = sqrt((1-c)(1+c))
//   the curvature's skew products and 1 - cos(theta) from the differences of
//   neighbouring directors (see the Voronoi phase)
//   exp(-[u]x) Q = Q + (sin t / t) [u]x Q + ((1 - cos t) / t^2)(u u^T - t^2) Q,
//   t = |u|, with both coefficients from their Taylor series for t < 0.1
//   (no square root or division)
//   the damper factors exp(x) from their Taylor series for |x| < 0.01
// The reference's 1e-14 guards (in the rotation axis and in sin(theta +
// 1e-14)) are dropped: each moves a director by ~1e-14 per step, far below
// this path's tolerance.  theta / sin(theta) comes from its series in
// y = 1 - cos(theta) through y^7 below y = 0.25 (relative rotations up to
// 0.72 rad a Voronoi point; truncation below 2e-8).  The second half
// drift of a step and the first half drift of the next use the same velocity
// and angular velocity and are applied as one full drift.
//
// A step is two phases with one barrier after each: element and Voronoi
// terms of a slot together (the neighbouring element's length is recomputed
// instead of exchanged), then the kick, the constraints and the drift.
//
// Per-rod constraint data (clamp, damper, end torque flags and the damper's
// constants) is copied into shared memory once per launch, so the step loop
// reads global memory only for the clamp target and end torque of the few
// slots that carry them.
//
// Rod pairs (kPair) as in rod_block_fp64.cu: a rod of up to 1039 elements on
// a cluster of two CTAs, neighbour reads across the split from the partner's
// shared memory, both per-step barriers cluster barriers.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "eb_internal.h"
#include "rod_math.cuh"

namespace eb {
namespace {

using D3 = Vec3<double>;
using F3 = Vec3<float>;

// Shared-memory layout, per slot (kCap entries a row):
//   FP64 rows: position, velocity, angular velocity, 1 / rest length and the
//   rest strain (with the unit axial strain folded in);
//   the director as five double2 rows (Q0 Q1 | Q2 Q3 | Q4 Q5 | Q6 Q7 | Q8 -);
//   FP32 float4 rows, each read or written with one 128-bit access: the
//   element phase's parameters, the kick's parameters and the exchanged terms.
// A warp's 128-bit accesses to one row cover 512 contiguous bytes, so they
// take four wavefronts without bank conflicts, as four 32-bit rows would, in
// a quarter of the instructions.
enum MixedRowD : int { dX = 0, dV = 3, dW = 6, dInvL0 = 9, dSig0 = 10, dRowsD = 13 };
constexpr int kQRows = 5;  // double2 rows of the director
enum MixedRowP : int {
  pA1 = 0,  // rest length, shear rigidity (3)
  pA2 = 1,  // inertia J (3), Voronoi rest length
  pA3 = 2,  // rest curvature (3), -
  pA4 = 3,  // bend rigidity (3), -
  pB1 = 4,  // J^-1 (3), mass
  pB2 = 5,  // damper rate nu_r, 1 - exp(-nu_t dt), explicit damping nu_f, nu_t
  pFE = 6,  // internal load (3), dilatation (exchanged)
  pPP = 7,  // torque terms differenced ahead (3), - (own)
  pMM = 8,  // couple terms differenced behind (3), - (exchanged)
  kRowsP = 9
};
// bytes of shared memory a slot: 13 FP64 rows, 5 double2, 9 float4, two words
constexpr int kMixedSlotBytes = dRowsD * 8 + kQRows * 16 + kRowsP * 16 + 8;

template <int kCap>
struct MRows {
  double* d;
  double2* q;
  float4* p;
  __device__ __forceinline__ double& ad(int r, int s) const { return d[r * kCap + s]; }
  __device__ __forceinline__ D3 d3(int r, int s) const { return {ad(r, s), ad(r + 1, s), ad(r + 2, s)}; }
  __device__ __forceinline__ void pd3(int r, int s, D3 v) const {
    ad(r, s) = v.x;
    ad(r + 1, s) = v.y;
    ad(r + 2, s) = v.z;
  }
  __device__ __forceinline__ void ldq(int s, double o[9]) const {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double2 v = q[k * kCap + s];
      o[2 * k] = v.x;
      o[2 * k + 1] = v.y;
    }
    o[8] = q[4 * kCap + s].x;
  }
  __device__ __forceinline__ void stq(int s, const double o[9]) const {
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k * kCap + s] = make_double2(o[2 * k], o[2 * k + 1]);
    q[4 * kCap + s] = make_double2(o[8], 0.0);
  }
  __device__ __forceinline__ float4 p4(int r, int s) const { return p[r * kCap + s]; }
  __device__ __forceinline__ void sp4(int r, int s, float4 v) const { p[r * kCap + s] = v; }
};

__device__ __forceinline__ F3 tof(D3 a) {
  return {static_cast<float>(a.x), static_cast<float>(a.y), static_cast<float>(a.z)};
}
__device__ __forceinline__ F3 xyz(float4 v) { return {v.x, v.y, v.z}; }

// FP64 director update Q <- exp(-[u]x) Q (Rodrigues' formula of
// Systems/States/Expressions/backends/blaze/SO3PrimitiveAddAssign/Scalar.hpp:41-95),
// written with the unnormalised u: cos t = 1 - a2 t^2, (1 - cos t) uh uh^T =
// a2 u u^T and sin(t) uh = a1 u for uh = u / t.
__device__ __forceinline__ void so3_series(double q[9], double u0, double u1, double u2) {
  const double z = u0 * u0 + u1 * u1 + u2 * u2;
  double a1, a2;  // sin(t) / t and (1 - cos t) / t^2
  if (z < 0.01) {
    a1 = 1.0 + z * (-1.0 / 6.0 + z * (1.0 / 120.0 + z * (-1.0 / 5040.0 + z * (1.0 / 362880.0 - z * (1.0 / 39916800.0)))));
    a2 = 0.5 + z * (-1.0 / 24.0 + z * (1.0 / 720.0 + z * (-1.0 / 40320.0 + z * (1.0 / 3628800.0 - z * (1.0 / 479001600.0)))));
  } else {
    const double t = sqrt(z);
    double s, c;
    sincos(t, &s, &c);
    a1 = s / t;
    a2 = (1.0 - c) / z;
  }
  double out[9];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double com = q[j] * u0 + q[3 + j] * u1 + q[6 + j] * u2;
    out[j] = q[j] + a2 * (u0 * com - z * q[j]) + a1 * (q[3 + j] * u2 - q[6 + j] * u1);
    out[3 + j] = q[3 + j] + a2 * (u1 * com - z * q[3 + j]) + a1 * (q[6 + j] * u0 - q[j] * u2);
    out[6 + j] = q[6 + j] + a2 * (u2 * com - z * q[6 + j]) + a1 * (q[j] * u1 - q[3 + j] * u0);
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) q[k] = out[k];
}

// exp(x), Taylor series below |x| = 0.01 (truncation below 1e-12 relative)
__device__ __forceinline__ float exp_small(float x) {
  if (fabsf(x) < 0.01f) return 1.f + x * (1.f + x * (0.5f + x * (1.f / 6.f + x * (1.f / 24.f))));
  return expf(x);
}

// x += c v; Q <- exp(-c [w]x) Q for element slots
template <int kCap>
__device__ __forceinline__ void drift(const MRows<kCap>& R, int s, uint32_t meta, double c, D3 v, D3 w) {
  const D3 x = R.d3(dX, s);
  R.pd3(dX, s, D3{x.x + c * v.x, x.y + c * v.y, x.z + c * v.z});
  if (meta & kElem) {
    double q[9];
    R.ldq(s, q);
    so3_series(q, c * w.x, c * w.y, c * w.z);
    R.stq(s, q);
  }
}

// the clamp's value constraint on a slot a clamp holds (hits: SlotHits):
// the node's position and, where the slot holds an element, its directors
template <int kCap>
__device__ __forceinline__ void clamp_value(const MRows<kCap>& R, int s, uint32_t meta, uint32_t hits,
                                            const RodInfo& ri) {
  const double* tx = (hits & kHitClamp0) ? ri.clamp_x : ri.clamp2_x;
  const double* tq = (hits & kHitClamp0) ? ri.clamp_Q : ri.clamp2_Q;
  R.pd3(dX, s, D3{tx[0], tx[1], tx[2]});
  if (!(meta & kElem)) return;
  double q[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) q[k] = tq[k];
  R.stq(s, q);
}

// Neighbour access for rod pairs: slot indices at or past `count` continue in
// the partner's first slots (left half), indices below zero in the partner's
// last `pcount` slots (right half).
template <int kCap>
struct MPair {
  MRows<kCap> own, peer;
  int count, pcount;
  __device__ __forceinline__ const MRows<kCap>& rows(int& s) const {
    if (s >= count) {
      s -= count;
      return peer;
    }
    if (s < 0) {
      s += pcount;
      return peer;
    }
    return own;
  }
  __device__ __forceinline__ D3 d3(int r, int s) const {
    const MRows<kCap>& X = rows(s);
    return X.d3(r, s);
  }
  __device__ __forceinline__ void ldq(int s, double o[9]) const {
    const MRows<kCap>& X = rows(s);
    X.ldq(s, o);
  }
  __device__ __forceinline__ float4 p4(int r, int s) const {
    const MRows<kCap>& X = rows(s);
    return X.p4(r, s);
  }
};

// FP32 length of element s from its FP64 position difference (Rows: MRows,
// or MPair for slots that may lie in a pair's partner)
template <class Rows>
__device__ __forceinline__ float element_length(const Rows& R, int s) {
  const F3 dxf = tof(R.d3(dX, s + 1) - R.d3(dX, s));
  const float l2 = dot(dxf, dxf);
  return l2 * rsqrtf(l2);
}

// kServe: the CTA's slot range, step count, time step and environment come
// from serve[blockIdx.x] (serving launches) instead of the work list and the
// launch-wide values
// kGather: cta_start indexes gmap, the list of the CTA's slots (rods that
// need not be neighbours in the slot layout)
// kPair: cluster launch of CTA pairs (see rod_block_fp64_kernel)
template <int kCap, int kThreads, int kMinBlocks, bool kDamped, bool kServe, bool kGather = false, bool kPair = false>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    rod_block_mixed_kernel(const StepArgs a, const int64_t* cta_start, int n_steps_launch, const ServeCta* serve,
                           const int32_t* gmap) {
  extern __shared__ __align__(128) double smem[];
  double2* const qbase = reinterpret_cast<double2*>(smem + dRowsD * kCap);
  float4* const pbase = reinterpret_cast<float4*>(qbase + kQRows * kCap);
  const MRows<kCap> R{smem, qbase, pbase};
  uint32_t* meta_s = reinterpret_cast<uint32_t*>(pbase + kRowsP * kCap);
  uint32_t* rflag_s = meta_s + kCap;

  const int tid = threadIdx.x;
  int64_t g0;
  int count, n_steps = n_steps_launch;
  double dt = a.dt, hdt = a.half_dt;
  uint32_t flags = a.sim_flags;
  double gvec[3] = {a.gravity[0], a.gravity[1], a.gravity[2]};
  if constexpr (kServe) {
    const ServeCta& sc = serve[blockIdx.x];
    g0 = sc.start;
    count = sc.count;
    n_steps = min(n_steps_launch, sc.steps);
    dt = sc.dt;
    hdt = sc.half_dt;
    flags = sc.flags;
    gvec[0] = sc.gravity[0];
    gvec[1] = sc.gravity[1];
    gvec[2] = sc.gravity[2];
  } else {
    g0 = cta_start[blockIdx.x];
    count = static_cast<int>(cta_start[blockIdx.x + 1] - g0);
  }
  if (n_steps <= 0) return;
  const int64_t S = a.stride;
  // partner rows (its own rows for a single CTA) and cluster barriers
  MPair<kCap> N{R, R, count, count};
  bool paired = false;
  if constexpr (kPair) {
    const unsigned partner = blockIdx.x ^ 1u;
    if constexpr (kServe) {
      const ServeCta& sc = serve[blockIdx.x];
      const ServeCta& o = serve[partner];
      paired = sc.pair != 0 && o.pair != 0 && sc.steps == o.steps;
      if (paired) N.pcount = o.count;
    } else {
      paired = true;
      N.pcount = static_cast<int>(cta_start[partner + 1] - cta_start[partner]);
    }
    if (paired) {
      cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
      const unsigned pr = cl.block_rank() ^ 1u;
      N.peer.d = cl.map_shared_rank(R.d, pr);
      N.peer.q = cl.map_shared_rank(R.q, pr);
      N.peer.p = cl.map_shared_rank(R.p, pr);
    }
  }
  // orders a phase's writes before the next phase's neighbour reads
  auto sync_neighbours = [&]() {
    if constexpr (kPair) {
      if (paired) {
        cooperative_groups::this_cluster().sync();
        return;
      }
    }
    __syncthreads();
  };

  // ---- stage state, parameters, reciprocals and rod data
  const bool any_rod = (flags & (kSimClamp | kSimDamper | kSimEndTorque)) != 0;
  for (int s = tid; s < count; s += kThreads) {
    const int64_t g = kGather ? static_cast<int64_t>(gmap[g0 + s]) : g0 + s;
    const uint32_t meta = a.meta[g];
    meta_s[s] = meta;
    uint32_t rf = 0;
    double dtc = 1.0;
    float dr = 0.f;
    if (any_rod) {
      const RodInfo& ri = a.rods[meta >> kRodShift];
      rf = slot_hits(ri, g);
      dtc = ri.damper_t;
      dr = static_cast<float>(ri.damper_r);
    }
    rflag_s[s] = rf;  // the slot's SlotHits
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      R.ad(dX + k, s) = a.in[(kStX + k) * S + g];
      R.ad(dV + k, s) = a.in[(kStV + k) * S + g];
      R.ad(dW + k, s) = a.in[(kStW + k) * S + g];
    }
    double q[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) q[k] = a.in[(kStQ + k) * S + g];
    R.stq(s, q);
    const double il0 = 1.0 / a.par[kL0 * S + g];
    R.ad(dInvL0, s) = il0;
    // the rest strain, with the unit axial strain of sigma = Q dx / l0 - z folded in
    R.ad(dSig0, s) = a.par[kSig0 * S + g];
    R.ad(dSig0 + 1, s) = a.par[(kSig0 + 1) * S + g];
    R.ad(dSig0 + 2, s) = a.par[(kSig0 + 2) * S + g] + 1.0;
    auto pf = [&](int f) { return static_cast<float>(a.par[f * S + g]); };
    R.sp4(pA1, s, make_float4(pf(kL0), pf(kShear), pf(kShear + 1), pf(kShear + 2)));
    R.sp4(pA2, s, make_float4(pf(kJ), pf(kJ + 1), pf(kJ + 2), pf(kD0)));
    R.sp4(pA3, s, make_float4(pf(kKap0), pf(kKap0 + 1), pf(kKap0 + 2), 0.f));
    R.sp4(pA4, s, make_float4(pf(kBend), pf(kBend + 1), pf(kBend + 2), 0.f));
    R.sp4(pB1, s, make_float4(pf(kJinv), pf(kJinv + 1), pf(kJinv + 2), pf(kMass)));
    R.sp4(pB2, s, make_float4(dr, static_cast<float>(1.0 - dtc), kDamped ? pf(kNuF) : 0.f,
                              kDamped ? pf(kNuT) : 0.f));
  }
  __syncthreads();

  const float dtf = static_cast<float>(dt);
  const F3 grav = {static_cast<float>(gvec[0]), static_cast<float>(gvec[1]), static_cast<float>(gvec[2])};

  // ---- first half drift of the first step and the clamp's value constraint
  for (int s = tid; s < count; s += kThreads) {
    const uint32_t meta = meta_s[s];
    drift(R, s, meta, hdt, R.d3(dV, s), R.d3(dW, s));
    const uint32_t hits = rflag_s[s];
    if (hits & (kHitClamp0 | kHitClamp1)) clamp_value(R, s, meta, hits, a.rods[meta >> kRodShift]);
  }
  sync_neighbours();

  // Two phases per step, one barrier after each.  Phase A: element s (strain,
  // internal load, element-local torque terms) and Voronoi s (curvature and
  // couple, with the length of element s + 1 recomputed rather than shared).
  // Phase B: loads, torques, kick, rate constraints, then the merged drift
  // (second half of this step and first half of the next; half on the last
  // step), the value constraint and, on the last step, the write-back.
  for (int step = 0; step < n_steps; ++step) {
    const bool last = step == n_steps - 1;

    for (int s = tid; s < count; s += kThreads) {
      const uint32_t meta = meta_s[s];
      F3 f{0.f, 0.f, 0.f}, p{0.f, 0.f, 0.f}, mm{0.f, 0.f, 0.f};
      float e = 1.f;
      if (meta & kElem) {
        const D3 dx = (kPair ? N.d3(dX, s + 1) : R.d3(dX, s + 1)) - R.d3(dX, s);
        double q[9];
        R.ldq(s, q);
        double qd[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) qd[k] = q[3 * k] * dx.x + q[3 * k + 1] * dx.y + q[3 * k + 2] * dx.z;
        const double il0 = R.ad(dInvL0, s);
        const F3 d = {static_cast<float>(qd[0] * il0 - R.ad(dSig0, s)),
                      static_cast<float>(qd[1] * il0 - R.ad(dSig0 + 1, s)),
                      static_cast<float>(qd[2] * il0 - R.ad(dSig0 + 2, s))};
        const F3 dxf = tof(dx);
        const float l2 = dot(dxf, dxf);
        const float il = rsqrtf(l2);
        const float l = l2 * il;
        const F3 t = scale(dxf, il);
        const float4 a1 = R.p4(pA1, s), a2 = R.p4(pA2, s);
        const float l0 = a1.x;
        e = l * static_cast<float>(il0);
        const float ie = l0 * il;
        const F3 nl = {a1.y * d.x, a1.z * d.y, a1.w * d.z};
        float qf[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) qf[k] = static_cast<float>(q[k]);
        f = scale(mattranspvec(qf, nl), ie);
        const F3 qt = matvec(qf, t);
        const F3 w = tof(R.d3(dW, s));
        const F3 jwe = {a2.x * w.x * ie, a2.y * w.y * ie, a2.z * w.z * ie};
        const F3 dv = tof((kPair ? N.d3(dV, s + 1) : R.d3(dV, s + 1)) - R.d3(dV, s));
        const float rate = dot(t, dv) * il;
        p = scale(cross(qt, nl), l0) + cross(jwe, w) + scale(jwe, rate);

        if (meta & kVor) {
          // With d_k the director rows of element s and dd_k = d_k(s+1) - d_k(s)
          // (FP64 differences), the reference's skew terms are exactly
          //   d3.d2' - d2.d3' = d3.dd2 - d2.dd3 (and cyclic), since d3.d2 = d2.d3,
          // and 1 - cos(theta) = 1.5 - tr/2 = |dd|^2/4 for unit rows (their
          // norms stay within 1e-14 of one, below the reference's 1e-10 shift);
          // both forms are free of the cancellation of the original products.
          double qn[9];
          if constexpr (kPair) N.ldq(s + 1, qn);
          else R.ldq(s + 1, qn);
          float dd[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) dd[k] = static_cast<float>(qn[k] - q[k]);
          float sq = 0.f;
#pragma unroll
          for (int k = 0; k < 9; ++k) sq += dd[k] * dd[k];
          const float y = 0.25f * sq + 1e-10f;
          float ratio;  // theta / sin(theta), theta = acos(1 - y)
          if (y < 0.25f) {
            // its Taylor series in y = 1 - cos(theta) through y^7 (the
            // first omitted term is below 2e-8 for y < 0.25, under FP32's
            // rounding), which covers relative rotations up to 0.72 rad a
            // Voronoi point without the arcsine
            ratio = 1.f + y * (1.f / 3.f + y * (2.f / 15.f + y * (2.f / 35.f + y * (8.f / 315.f +
                    y * (8.f / 693.f + y * (16.f / 3003.f + y * (16.f / 6435.f)))))));
          } else {
            ratio = 2.f * asinf(sqrtf(0.5f * y)) * rsqrtf(y * (2.f - y));
          }
          const float D0 = a2.w;
          const float st = 0.5f * ratio * __frcp_rn(D0);
          const F3 d1{qf[0], qf[1], qf[2]}, d2{qf[3], qf[4], qf[5]}, d3{qf[6], qf[7], qf[8]};
          const F3 e1{dd[0], dd[1], dd[2]}, e2{dd[3], dd[4], dd[5]}, e3{dd[6], dd[7], dd[8]};
          const F3 skew = {dot(d3, e2) - dot(d2, e3), dot(d1, e3) - dot(d3, e1), dot(d2, e1) - dot(d1, e2)};
          const F3 kappa = scale(skew, st);
          // 1 / eps^3 with eps = D / D0, D the mean length of elements s, s + 1
          const float ieps =
              __fdividef(D0, 0.5f * (l + (kPair ? element_length(N, s + 1) : element_length(R, s + 1))));
          const float ic = ieps * ieps * ieps;
          const F3 dk = kappa - xyz(R.p4(pA3, s));
          const F3 B = xyz(R.p4(pA4, s));
          const F3 tau = {B.x * dk.x, B.y * dk.y, B.z * dk.z};
          // the couple's two parts: G = tau / eps^3 (differenced) and
          // H = (kappa x tau) D0 / eps^3 (averaged) enter torque s as
          // (G_s + H_s / 2) - (G_{s-1} - H_{s-1} / 2)
          const F3 gg = scale(tau, ic);
          const F3 hh = scale(cross(kappa, tau), 0.5f * ic * D0);
          p = p + gg + hh;
          mm = gg - hh;
        }
      }
      R.sp4(pFE, s, make_float4(f.x, f.y, f.z, e));
      R.sp4(pPP, s, make_float4(p.x, p.y, p.z, 0.f));
      R.sp4(pMM, s, make_float4(mm.x, mm.y, mm.z, 0.f));
    }
    sync_neighbours();

    for (int s = tid; s < count; s += kThreads) {
      const uint32_t meta = meta_s[s];
      const bool first = (meta & kFirst) != 0;
      const float4 b1 = R.p4(pB1, s);
      const float m = b1.w;
      D3 v = R.d3(dV, s);
      const float4 fe = R.p4(pFE, s);
      F3 F = xyz(fe);
      if (!first) F = F - xyz(kPair ? N.p4(pFE, s - 1) : R.p4(pFE, s - 1));
      const uint32_t rf = rflag_s[s];
      float4 b2 = make_float4(0.f, 0.f, 0.f, 0.f);
      if (kDamped || (rf & kHitDamper)) b2 = R.p4(pB2, s);
      if (kDamped) {
        const float cf = m * b2.z;
        const F3 vf = tof(v);
        F = {F.x - cf * vf.x, F.y - cf * vf.y, F.z - cf * vf.z};
      }
      if (flags & kSimGravity) F = F + F3{grav.x * m, grav.y * m, grav.z * m};
      const float im = __frcp_rn(m);
      v = {v.x + dt * static_cast<double>(F.x * im), v.y + dt * static_cast<double>(F.y * im),
           v.z + dt * static_cast<double>(F.z * im)};
      D3 w{0.0, 0.0, 0.0};
      if (meta & kElem) {
        const float e = fe.w;
        w = R.d3(dW, s);
        F3 T = xyz(R.p4(pPP, s));
        if (!first) T = T - xyz(kPair ? N.p4(pMM, s - 1) : R.p4(pMM, s - 1));
        const float mn = (kDamped || (rf & kHitDamper)) ? (kPair ? N.p4(pB1, s + 1) : R.p4(pB1, s + 1)).w : 0.f;
        if (kDamped) {
          const float ct = 0.5f * (m + mn) * b2.w;
          const F3 wf = tof(w);
          T = {T.x - ct * wf.x, T.y - ct * wf.y, T.z - ct * wf.z};
        }
        if (rf & kHitTorque) {
          const RodInfo& ri = a.rods[meta >> kRodShift];
          double q[9];
          R.ldq(s, q);
          float qf[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) qf[k] = static_cast<float>(q[k]);
          T = T + matvec(qf, F3{static_cast<float>(ri.end_torque[0]), static_cast<float>(ri.end_torque[1]),
                                static_cast<float>(ri.end_torque[2])});
        }
        const F3 ji = xyz(b1);
        w = {w.x + dt * static_cast<double>(ji.x * T.x * e), w.y + dt * static_cast<double>(ji.y * T.y * e),
             w.z + dt * static_cast<double>(ji.z * T.z * e)};
        if (rf & kHitDamper) {
          float em = 0.5f * (m + mn);
          if (first) em += 0.5f * m;
          if (meta & kLastElem) em += 0.5f * mn;
          const float y = -b2.x * em * dtf * e;
          w = {w.x * static_cast<double>(exp_small(y * ji.x)), w.y * static_cast<double>(exp_small(y * ji.y)),
               w.z * static_cast<double>(exp_small(y * ji.z))};
        }
      }
      const bool clamped = (rf & (kHitClamp0 | kHitClamp1)) != 0;
      if (clamped) {
        v = D3{0.0, 0.0, 0.0};
        w = D3{0.0, 0.0, 0.0};
      }
      if (rf & kHitDamper) v = scale(v, 1.0 - static_cast<double>(b2.y));
      R.pd3(dV, s, v);
      if (meta & kElem) R.pd3(dW, s, w);
      drift(R, s, meta, last ? hdt : dt, v, w);
      if (clamped) clamp_value(R, s, meta, rf, a.rods[meta >> kRodShift]);
      if (last) {
        const int64_t g = kGather ? static_cast<int64_t>(gmap[g0 + s]) : g0 + s;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          a.out[(kStX + k) * S + g] = R.ad(dX + k, s);
          a.out[(kStV + k) * S + g] = R.ad(dV + k, s);
        }
        if (meta & kElem) {
          double q[9];
          R.ldq(s, q);
#pragma unroll
          for (int k = 0; k < 9; ++k) a.out[(kStQ + k) * S + g] = q[k];
#pragma unroll
          for (int k = 0; k < 3; ++k) a.out[(kStW + k) * S + g] = R.ad(dW + k, s);
        }
      }
    }
    sync_neighbours();
  }
}

template <int kCap, int kThreads, int kMinBlocks, bool kServe = false, bool kGather = false, bool kPair = false>
cudaError_t launch_mixed_cfg(const StepArgs& args, const int64_t* cta_start, int n_ctas, int n_steps, bool damped,
                             cudaStream_t stream, const ServeCta* serve = nullptr, const int32_t* gmap = nullptr) {
  const size_t bytes = size_t(kMixedSlotBytes) * kCap;
  auto go = [&](auto kern) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e != cudaSuccess) return e;
    if constexpr (kPair) {
      // clusters of two CTAs; the grid is a whole number of clusters
      if (n_ctas % 2 != 0) return cudaErrorInvalidValue;
      cudaLaunchConfig_t lc = {};
      lc.gridDim = dim3(static_cast<unsigned>(n_ctas));
      lc.blockDim = dim3(kThreads);
      lc.dynamicSmemBytes = bytes;
      lc.stream = stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = 2;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      lc.attrs = at;
      lc.numAttrs = 1;
      return cudaLaunchKernelEx(&lc, kern, args, cta_start, n_steps, serve, gmap);
    } else {
      kern<<<n_ctas, kThreads, bytes, stream>>>(args, cta_start, n_steps, serve, gmap);
      return cudaGetLastError();
    }
  };
  return damped ? go(rod_block_mixed_kernel<kCap, kThreads, kMinBlocks, true, kServe, kGather, kPair>)
                : go(rod_block_mixed_kernel<kCap, kThreads, kMinBlocks, false, kServe, kGather, kPair>);
}

}  // namespace

// Serving launches: CTA c runs serve[c] (its request's slot range, time step,
// environment and min(n_steps, serve[c].steps) steps); 520-slot CTAs.
// A cluster launch (n_ctas even) in which entries 2i and 2i + 1 may hold the
// two halves of one rod (ServeCta::pair).  Every serving launch takes this
// form, so a request's arithmetic is the same whatever it is served with.
cudaError_t launch_rod_block_mixed_serve(const StepArgs& args, const ServeCta* serve, int n_ctas, int n_steps,
                                         bool damped, cudaStream_t stream) {
  if (n_ctas <= 0 || n_steps <= 0) return cudaSuccess;
  return launch_mixed_cfg<520, 512, 1, true, false, true>(args, nullptr, n_ctas, n_steps, damped, stream, serve);
}

// Rod pairs on gathered CTAs (see launch_rod_block_fp64_pairs).
cudaError_t launch_rod_block_mixed_pairs(const StepArgs& args, const int64_t* cta_start, const int32_t* gmap,
                                         int n_ctas, int n_steps, int config, bool damped, cudaStream_t stream) {
  if (n_ctas <= 0 || n_steps <= 0) return cudaSuccess;
  switch (config) {
    case 0: return launch_mixed_cfg<520, 512, 1, false, true, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    case 1: return launch_mixed_cfg<520, 256, 1, false, true, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    default: return cudaErrorInvalidValue;
  }
}

// Resident launches: CTA c owns the slots gmap[cta_start[c] .. cta_start[c +
// 1]), whole rods (the host packs them best fit decreasing).  The same
// configurations as the FP64 resident kernel (0/1: 520 slots, 2: 264, 3:
// 320); 304 B of shared memory per slot (312 with explicit damping) allows
// two CTAs per SM at 264 and 320 slots (two of 352 slots on 352 threads
// measured 1% slower than 320 on the mixed batch).
cudaError_t launch_rod_block_mixed_gather(const StepArgs& args, const int64_t* cta_start, const int32_t* gmap,
                                          int n_ctas, int n_steps, int config, bool damped, cudaStream_t stream) {
  if (n_ctas <= 0 || n_steps <= 0) return cudaSuccess;
  switch (config) {
    case 0: return launch_mixed_cfg<520, 512, 1, false, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    case 1: return launch_mixed_cfg<520, 256, 1, false, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    case 2: return launch_mixed_cfg<264, 256, 2, false, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    case 3: return launch_mixed_cfg<320, 320, 2, false, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace eb
