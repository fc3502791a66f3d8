// Resident multi-step PositionVerlet kernel for batches of whole rods.
//
// The streaming step kernel (rod_step_fp64.cu) moves the full state through
// HBM every step.  Rods are independent, so a CTA can instead own a group of
// whole rods, stage their state and parameters into shared memory once, run
// many steps entirely on chip and write the state back once: HBM traffic per
// element-step falls by the number of steps per launch and the step becomes
// arithmetic-bound.
//
// Work list: CTA c owns the slots gmap[cta_start[c] .. cta_start[c + 1]),
// always whole rods (the host packs rods best fit decreasing into CTAs of at
// most kCap slots; serving launches read consecutive slot ranges from a CTA
// table instead).  Every phase loops its threads over the CTA's slots; all
// per-slot data lives in shared-memory rows, so any thread count works.
//
// Step structure: the same substeps as the streaming kernel, including both
// half drifts of every step, in two phases with one barrier after each (see
// the step loop).  (Merging the second half drift of step k with
// the first of step k+1 into one full drift is not an identity here: the
// reference normalises the rotation axis by theta + 1e-14, so one update by
// dt differs from two by dt/2 by ~1e-14 per step, which the stiff rod modes
// amplify into angular-velocity differences far above rounding.  The kernel
// keeps a compile-time switch for it, unused by the configurations below.)
//
// Rod pairs (kPair): a rod of up to 1039 elements runs on a cluster of two
// CTAs, each holding half of its slots.  Reads of a neighbouring slot past
// the left half's end or before the right half's start go to the partner's
// shared memory (distributed shared memory), and the barriers that order a
// phase's writes before the next phase's neighbour reads become cluster
// barriers.  Serving launches mix pairs and single CTAs in one cluster
// launch; a single CTA takes only CTA barriers.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "eb_internal.h"
#include "rod_math.cuh"

namespace eb {
namespace {

using D3 = Vec3<double>;

// shared-memory rows (each kCap doubles)
enum BlockRow : int {
  bX = 0, bV = 3, bQ = 6, bW = 15,  // state (kStateFields rows)
  bMass = 18, bL0 = 19, bD0 = 20, bSig0 = 21, bKap0 = 24, bShear = 27, bBend = 30, bJ = 33, bJinv = 36,
  bE = 39, bF = 40, bG = 43, bH = 46, bTl = 49,  // per-step exchange rows
  bNuF = 52, bNuT = 53              // explicit damping only: the last rows, not allocated otherwise
};

template <int kCap>
struct BRows {
  double* base;
  __device__ __forceinline__ double& at(int r, int s) const { return base[r * kCap + s]; }
  __device__ __forceinline__ D3 get3(int r, int s) const {
    return {base[r * kCap + s], base[(r + 1) * kCap + s], base[(r + 2) * kCap + s]};
  }
  __device__ __forceinline__ void put3(int r, int s, D3 v) const {
    base[r * kCap + s] = v.x;
    base[(r + 1) * kCap + s] = v.y;
    base[(r + 2) * kCap + s] = v.z;
  }
};

// Neighbour access for rod pairs: slot indices at or past `count` continue in
// the partner's first slots (left half), indices below zero in the partner's
// last `pcount` slots (right half).
template <int kCap>
struct BPair {
  BRows<kCap> own, peer;
  int count, pcount;
  __device__ __forceinline__ double at(int r, int s) const {
    if (s >= count) return peer.at(r, s - count);
    if (s < 0) return peer.at(r, s + pcount);
    return own.at(r, s);
  }
  __device__ __forceinline__ D3 get3(int r, int s) const {
    if (s >= count) return peer.get3(r, s - count);
    if (s < 0) return peer.get3(r, s + pcount);
    return own.get3(r, s);
  }
};

// parameter field -> shared row (the rows the resident kernel keeps)
__device__ __forceinline__ int param_row(int f) {
  switch (f) {
    case kMass: return bMass;
    case kL0: return bL0;
    case kD0: return bD0;
    case kNuF: return bNuF;
    case kNuT: return bNuT;
    default: break;
  }
  if (f >= kSig0 && f < kSig0 + 3) return bSig0 + (f - kSig0);
  if (f >= kKap0 && f < kKap0 + 3) return bKap0 + (f - kKap0);
  if (f >= kShear && f < kShear + 3) return bShear + (f - kShear);
  if (f >= kBend && f < kBend + 3) return bBend + (f - kBend);
  if (f >= kJ && f < kJ + 3) return bJ + (f - kJ);
  if (f >= kJinv && f < kJinv + 3) return bJinv + (f - kJinv);
  return -1;  // volume: only read for diagnostics, straight from global memory
}

// kServe: the CTA's slot range, step count, time step and environment come
// from serve[blockIdx.x] (serving launches)
// kGather: cta_start indexes gmap, the list of the CTA's slots (rods that
// need not be neighbours in the slot layout)
// kPair: cluster launch of CTA pairs; with kServe, CTAs 2i and 2i + 1 form a
// pair when both serve entries say so and run the same step count, and are
// single CTAs otherwise; without kServe every cluster is a pair
// kStepper: 0 PositionVerlet, 1 PEFRL (four force evaluations a step), 2
// VelocityVerlet (two: kick dt/2, drift dt, kick dt/2)
// FP64 shared-memory rows per slot
template <bool kDamped>
constexpr int block_rows() { return kDamped ? 54 : 52; }

// two CTAs per SM for the CTAs of at most 264 slots (420 B a slot undamped)
template <int kCap>
constexpr int block_min_ctas() { return kCap <= 264 ? 2 : 1; }

template <int kCap, int kThreads, bool kDamped, bool kSplit, bool kServe, bool kGather = false, bool kPair = false,
          int kStepper = 0>
__global__ void __launch_bounds__(kThreads, block_min_ctas<kCap>()) rod_block_fp64_kernel(const StepArgs a, const int64_t* cta_start,
                                                                    int n_steps_launch, const ServeCta* serve,
                                                                    const int32_t* gmap) {
  extern __shared__ __align__(128) double smem[];
  const BRows<kCap> R{smem};
  uint32_t* meta_s = reinterpret_cast<uint32_t*>(smem + block_rows<kDamped>() * kCap);
  // per slot: which clamp holds it, the torque, the damper (SlotHits)
  uint8_t* hit_s = reinterpret_cast<uint8_t*>(meta_s + kCap);

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
  BPair<kCap> N{R, R, count, count};
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
      N.peer.base = cl.map_shared_rank(smem, cl.block_rank() ^ 1u);
    }
  }
  // orders this phase's writes before the next phase's neighbour reads
  auto sync_neighbours = [&]() {
    if constexpr (kPair) {
      if (paired) {
        cooperative_groups::this_cluster().sync();
        return;
      }
    }
    __syncthreads();
  };
  auto nb3 = [&](int r, int s) -> D3 {
    if constexpr (kPair) return N.get3(r, s);
    return R.get3(r, s);
  };
  auto nb = [&](int r, int s) -> double {
    if constexpr (kPair) return N.at(r, s);
    return R.at(r, s);
  };

  const bool any_rod = (flags & (kSimClamp | kSimDamper | kSimEndTorque)) != 0;

  // ---- stage state, parameters and slot metadata (coalesced loads)
  for (int s = tid; s < count; s += kThreads) {
    const int64_t g = kGather ? static_cast<int64_t>(gmap[g0 + s]) : g0 + s;
    const uint32_t m = a.meta[g];
    meta_s[s] = m;
    hit_s[s] = static_cast<uint8_t>(any_rod ? slot_hits(a.rods[m >> kRodShift], g) : 0u);
#pragma unroll 1
    for (int f = 0; f < kStateFields; ++f) R.at(f, s) = a.in[f * S + g];
#pragma unroll 1
    for (int f = 0; f < kParamFields; ++f) {
      const int r = param_row(f);
      if (r < 0 || (!kDamped && (f == kNuF || f == kNuT))) continue;
      R.at(r, s) = a.par[f * S + g];
    }
  }
  __syncthreads();

  // drift of slot s by c (x += c v, Q <- exp(-c [w]x) Q; c = 0 leaves the
  // slot as it is), then, with `clamp`, the value constraint of the clamp
  // that holds the slot, if any
  auto drift = [&](int s, uint32_t meta, double c, bool clamp) {
    const D3 v = R.get3(bV, s);
    D3 x = R.get3(bX, s);
    x = {x.x + c * v.x, x.y + c * v.y, x.z + c * v.z};
    double q[9];
    if (meta & kElem) {
#pragma unroll
      for (int k = 0; k < 9; ++k) q[k] = R.at(bQ + k, s);
      const D3 w = R.get3(bW, s);
      so3_update_fast(q, c * w.x, c * w.y, c * w.z);
    }
    const uint32_t hit = hit_s[s];
    if (clamp && (hit & (kHitClamp0 | kHitClamp1))) {
      // the clamp's value constraint: the node, and its element if it has one
      const RodInfo& ri = a.rods[meta >> kRodShift];
      const double* tx = (hit & kHitClamp0) ? ri.clamp_x : ri.clamp2_x;
      const double* tq = (hit & kHitClamp0) ? ri.clamp_Q : ri.clamp2_Q;
      x = {tx[0], tx[1], tx[2]};
      if (meta & kElem) {
#pragma unroll
        for (int k = 0; k < 9; ++k) q[k] = tq[k];
      }
    }
    R.put3(bX, s, x);
    if (meta & kElem) {
#pragma unroll
      for (int k = 0; k < 9; ++k) R.at(bQ + k, s) = q[k];
    }
  };
  // length of element s, rounded as written (so the copy a Voronoi point
  // recomputes for its next element equals the element's own)
  auto elem_length = [&](int s) -> double {
    const D3 dx = nb3(bX, s + 1) - nb3(bX, s);
    return sqrt(__fma_rn(dx.z, dx.z, __fma_rn(dx.y, dx.y, __dmul_rn(dx.x, dx.x))));
  };

  // Substeps: PositionVerlet (drift dt/2, kick dt, drift dt/2), or PEFRL's
  // four kicks with their drifts (in units of dt; compile-time constants)
  constexpr bool kPefrl = kStepper == 1, kVelocity = kStepper == 2;
  constexpr int nsub = kPefrl ? 4 : (kVelocity ? 2 : 1);
  auto pefrl_pre = [](int j) -> double {  // drift before force evaluation j
    return j == 0 ? kPefrlXi : (j == 2 ? 1.0 - 2.0 * (kPefrlChi + kPefrlXi) : kPefrlChi);
  };
  auto pefrl_kick = [](int j) -> double {
    return (j == 0 || j == 3) ? 0.5 * (1.0 - 2.0 * kPefrlLambda) : kPefrlLambda;
  };

  // ---- first drift of the first step and the clamp's value constraint
  // (VelocityVerlet starts with a kick: no drift, the clamp's value alone)
  for (int s = tid; s < count; s += kThreads)
    drift(s, meta_s[s], kPefrl ? kPefrlXi * dt : (kVelocity ? 0.0 : hdt), true);
  sync_neighbours();

  // Two phases per force evaluation, one barrier after each: (1) element s
  // (geometry, strain, stress, element-local torque terms) and Voronoi point
  // s (curvature and couple, with the next element's length recomputed
  // rather than exchanged); (2) loads, torques, kick and rate constraints,
  // then the drift before the next force evaluation (after the last kick of
  // a step: its closing drift and the next step's first, kept apart: merging
  // them into one rotation is not an identity under the 1e-14 axis guard).
  for (int step = 0; step < n_steps; ++step)
  for (int sub = 0; sub < nsub; ++sub) {
    const double kc = kPefrl ? pefrl_kick(sub) : (kVelocity ? 0.5 : 1.0);  // this kick, in units of dt
    const double kdt = kc == 1.0 ? dt : kc * dt;
    // the damper's time: the kick's share of dt for PEFRL, the full dt for
    // VelocityVerlet (its constants hold dt and act after each kick)
    const double dc = kVelocity ? 1.0 : kc;
    const double ddt = dc == 1.0 ? dt : kdt;
    for (int s = tid; s < count; s += kThreads) {
      const uint32_t meta = meta_s[s];
      D3 f{0.0, 0.0, 0.0}, tl{0.0, 0.0, 0.0};
      double l = 1.0, e = 1.0;
      double q[9];
      if (meta & kElem) {
#pragma unroll
        for (int k = 0; k < 9; ++k) q[k] = R.at(bQ + k, s);
        const D3 dx = nb3(bX, s + 1) - R.get3(bX, s);
        l = elem_length(s);
        const double il = 1.0 / l;
        const D3 t = {dx.x * il, dx.y * il, dx.z * il};
        const double l0 = R.at(bL0, s);
        e = l / l0;
        const D3 qt = matvec(q, t);
        const D3 sigma = {qt.x * e, qt.y * e, qt.z * e - 1.0};
        const D3 d = sigma - R.get3(bSig0, s);
        const D3 sh = R.get3(bShear, s);
        const D3 nl = {sh.x * d.x, sh.y * d.y, sh.z * d.z};
        const double ie = 1.0 / e;
        f = scale(mattranspvec(q, nl), ie);
        const D3 w = R.get3(bW, s);
        const D3 J = R.get3(bJ, s);
        const D3 jwe = {J.x * w.x * ie, J.y * w.y * ie, J.z * w.z * ie};
        const D3 dv = nb3(bV, s + 1) - R.get3(bV, s);
        const double rate = dot(t, dv) / (e * l0);
        tl = scale(cross(qt, nl), l0) + cross(jwe, w) + scale(jwe, rate);
      }
      R.at(bE, s) = e;
      R.put3(bF, s, f);
      R.put3(bTl, s, tl);
      D3 gg{0.0, 0.0, 0.0}, hh{0.0, 0.0, 0.0};
      if (meta & kVor) {
        double qn[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) qn[k] = nb(bQ + k, s + 1);
        const double D0 = R.at(bD0, s);
        const D3 kappa = inv_rotate_divide_fast(q, qn, D0);
        const double eps = 0.5 * (l + elem_length(s + 1)) / D0;
        const double ic = 1.0 / (eps * eps * eps);
        const D3 dk = kappa - R.get3(bKap0, s);
        const D3 B = R.get3(bBend, s);
        const D3 tau = {B.x * dk.x, B.y * dk.y, B.z * dk.z};
        gg = scale(tau, ic);
        hh = scale(cross(kappa, tau), ic * D0);
      }
      R.put3(bG, s, gg);
      R.put3(bH, s, hh);
    }
    sync_neighbours();

    // ---- loads, torques, accelerations, kick, rate constraints
    for (int s = tid; s < count; s += kThreads) {
      const uint32_t meta = meta_s[s];
      const bool first = (meta & kFirst) != 0;
      const double m = R.at(bMass, s);
      D3 v = R.get3(bV, s);
      D3 F = R.get3(bF, s);
      if (!first) F = F - nb3(bF, s - 1);
      if (kDamped) {
        const double cf = m * R.at(bNuF, s);
        F = {F.x - cf * v.x, F.y - cf * v.y, F.z - cf * v.z};
      }
      if (flags & kSimGravity) F = F + D3{gvec[0] * m, gvec[1] * m, gvec[2] * m};
      const double im = 1.0 / m;
      v = {v.x + kdt * (F.x * im), v.y + kdt * (F.y * im), v.z + kdt * (F.z * im)};
      D3 w{0.0, 0.0, 0.0};
      const uint32_t hit = hit_s[s];
      const RodInfo* ri = any_rod ? a.rods + (meta >> kRodShift) : nullptr;
      if (meta & kElem) {
        const double e = R.at(bE, s);
        w = R.get3(bW, s);
        D3 T = R.get3(bG, s);
        D3 Q2 = R.get3(bH, s);
        if (!first) {
          T = T - nb3(bG, s - 1);
          Q2 = Q2 + nb3(bH, s - 1);
        }
        T = T + scale(Q2, 0.5) + R.get3(bTl, s);
        if (kDamped) {
          const double ct = 0.5 * (m + nb(bMass, s + 1)) * R.at(bNuT, s);
          T = {T.x - ct * w.x, T.y - ct * w.y, T.z - ct * w.z};
        }
        if (hit & kHitTorque) {
          double q[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) q[k] = R.at(bQ + k, s);
          T = T + matvec(q, D3{ri->end_torque[0], ri->end_torque[1], ri->end_torque[2]});
        }
        const D3 ji = R.get3(bJinv, s);
        w = {w.x + kdt * (ji.x * T.x * e), w.y + kdt * (ji.y * T.y * e), w.z + kdt * (ji.z * T.z * e)};
        if (hit & kHitDamper) {
          const double mn = nb(bMass, s + 1);
          double em = 0.5 * (m + mn);
          if (first) em += 0.5 * m;
          if (meta & kLastElem) em += 0.5 * mn;
          const double y = -ri->damper_r * em * ddt * e;
          w = {w.x * exp(y * ji.x), w.y * exp(y * ji.y), w.z * exp(y * ji.z)};
        }
      }
      if (hit & (kHitClamp0 | kHitClamp1)) {
        v = D3{0.0, 0.0, 0.0};
        w = D3{0.0, 0.0, 0.0};
      }
      // exp(-nu_t dt) for a kick of dt; a fractional kick scales the exponent
      if (hit & kHitDamper) v = scale(v, dc == 1.0 ? ri->damper_t : exp(log(ri->damper_t) * dc));
      R.put3(bV, s, v);
      if (meta & kElem) R.put3(bW, s, w);
      if (sub + 1 < nsub) {
        // before the next force evaluation
        drift(s, meta, kVelocity ? dt : pefrl_pre(sub + 1) * dt, true);
      } else if (step + 1 < n_steps) {
        if (kVelocity) {
          drift(s, meta, 0.0, true);  // the next step starts with a kick: the clamp's value alone
        } else if (kPefrl) {
          drift(s, meta, kPefrlXi * dt, false);  // closing drift of this step, own slot
          drift(s, meta, kPefrlXi * dt, true);   // first drift of the next
        } else if (kSplit) {
          drift(s, meta, hdt, false);  // second half of this step, own slot
          drift(s, meta, hdt, true);   // first half of the next
        } else {
          drift(s, meta, dt, true);
        }
      }
    }
    // the next phase reads the neighbours' drifted state; for a pair, the
    // partner must also not leave (and free its rows) while this CTA still
    // reads them
    sync_neighbours();
  }

  // ---- closing drift of the last step and write-back
  const double fin = kPefrl ? kPefrlXi * dt : (kVelocity ? 0.0 : hdt);
  for (int s = tid; s < count; s += kThreads) {
    const uint32_t meta = meta_s[s];
    const int64_t g = kGather ? static_cast<int64_t>(gmap[g0 + s]) : g0 + s;
    const D3 v = R.get3(bV, s);
    D3 x = R.get3(bX, s);
    x = {x.x + fin * v.x, x.y + fin * v.y, x.z + fin * v.z};
    a.out[kStX * S + g] = x.x;
    a.out[(kStX + 1) * S + g] = x.y;
    a.out[(kStX + 2) * S + g] = x.z;
    a.out[kStV * S + g] = v.x;
    a.out[(kStV + 1) * S + g] = v.y;
    a.out[(kStV + 2) * S + g] = v.z;
    if (meta & kElem) {
      double q[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) q[k] = R.at(bQ + k, s);
      const D3 w = R.get3(bW, s);
      so3_update_fast(q, fin * w.x, fin * w.y, fin * w.z);
#pragma unroll
      for (int k = 0; k < 9; ++k) a.out[(kStQ + k) * S + g] = q[k];
      a.out[kStW * S + g] = w.x;
      a.out[(kStW + 1) * S + g] = w.y;
      a.out[(kStW + 2) * S + g] = w.z;
    }
  }
}

template <int kCap, int kThreads, bool kSplit, bool kServe = false, bool kGather = false, bool kPair = false>
cudaError_t launch_block_cfg(const StepArgs& args, const int64_t* cta_start, int n_ctas, int n_steps, bool damped,
                             cudaStream_t stream, const ServeCta* serve = nullptr, const int32_t* gmap = nullptr) {
  const size_t bytes =
      size_t(damped ? block_rows<true>() : block_rows<false>()) * kCap * sizeof(double) +
      size_t(kCap) * (sizeof(uint32_t) + sizeof(uint8_t));
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
  if constexpr (!kServe) {  // serving launches are PositionVerlet
    if (args.n_sub == 4)
      return damped ? go(rod_block_fp64_kernel<kCap, kThreads, true, kSplit, kServe, kGather, kPair, 1>)
                    : go(rod_block_fp64_kernel<kCap, kThreads, false, kSplit, kServe, kGather, kPair, 1>);
    if (args.n_sub == 2)
      return damped ? go(rod_block_fp64_kernel<kCap, kThreads, true, kSplit, kServe, kGather, kPair, 2>)
                    : go(rod_block_fp64_kernel<kCap, kThreads, false, kSplit, kServe, kGather, kPair, 2>);
  }
  return damped ? go(rod_block_fp64_kernel<kCap, kThreads, true, kSplit, kServe, kGather, kPair>)
                : go(rod_block_fp64_kernel<kCap, kThreads, false, kSplit, kServe, kGather, kPair>);
}

}  // namespace

// Configurations offered to the autotuner.  The capacity bounds the longest
// rod a configuration can hold (n + 1 slots).
namespace {
// {slots per CTA, threads per CTA}
constexpr int kBlockConfigs[][2] = {{520, 512}, {520, 256}, {264, 256}, {320, 320}};
constexpr int kNumConfigs = 4;
}  // namespace

int block_config_count() { return kNumConfigs; }

int block_config_capacity(int config) {
  return (config >= 0 && config < kNumConfigs) ? kBlockConfigs[config][0] : 0;
}

int block_config_threads(int config) {
  return (config >= 0 && config < kNumConfigs) ? kBlockConfigs[config][1] : 0;
}

// Serving launches (see launch_rod_block_mixed_serve): 520-slot CTAs in a
// cluster launch (n_ctas even) in which serve entries 2i and 2i + 1 may hold
// the two halves of one rod.
cudaError_t launch_rod_block_fp64_serve(const StepArgs& args, const ServeCta* serve, int n_ctas, int n_steps,
                                        bool damped, cudaStream_t stream) {
  if (n_ctas <= 0 || n_steps <= 0) return cudaSuccess;
  return launch_block_cfg<520, 512, true, true, false, true>(args, nullptr, n_ctas, n_steps, damped, stream, serve);
}

// Rod pairs on gathered CTAs: CTAs 2i and 2i + 1 own the two halves of one
// rod (slots gmap[cta_start[c] .. cta_start[c + 1])); config 0: 512 threads,
// 1: 256 threads per CTA.
cudaError_t launch_rod_block_fp64_pairs(const StepArgs& args, const int64_t* cta_start, const int32_t* gmap,
                                        int n_ctas, int n_steps, int config, bool damped, cudaStream_t stream) {
  if (n_ctas <= 0 || n_steps <= 0) return cudaSuccess;
  switch (config) {
    case 0: return launch_block_cfg<520, 512, true, false, true, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    case 1: return launch_block_cfg<520, 256, true, false, true, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    default: return cudaErrorInvalidValue;
  }
}

// Gathered CTAs: CTA c owns the slots gmap[cta_start[c] .. cta_start[c + 1]),
// whole rods in slot order (the per-size-bucket plans).
cudaError_t launch_rod_block_fp64_gather(const StepArgs& args, const int64_t* cta_start, const int32_t* gmap,
                                         int n_ctas, int n_steps, int config, bool damped, cudaStream_t stream) {
  if (n_ctas <= 0 || n_steps <= 0) return cudaSuccess;
  switch (config) {
    case 0: return launch_block_cfg<520, 512, true, false, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    case 1: return launch_block_cfg<520, 256, true, false, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    case 2: return launch_block_cfg<264, 256, true, false, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    case 3: return launch_block_cfg<320, 320, true, false, true>(args, cta_start, n_ctas, n_steps, damped, stream, nullptr, gmap);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace eb
