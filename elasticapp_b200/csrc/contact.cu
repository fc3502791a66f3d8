// Collision system for rods: capsules, candidate pairs, contact loads.
//
// Every element of a participating rod is a capsule (Systems/Customization/
// CosseratRods/Transfer/Common.hpp:57-93): centre = mid-point of the element's
// nodes, length = dilatation * rest length, radius = the element dimension
// sqrt(V / (pi l)), rotation from the tangent (Utilities/Math/Orthogonal.cpp:
// 118-129), mass-weighted node velocity and the element's angular velocity.
// One evaluation per step, at the state after the first half drift, in
// five stages:
//
//   1. capsule_kernel: capsules and their axis-aligned bounding boxes
//      (Primitives/detail/CapsulePrimitiveBase.cpp:163-180), and the largest
//      box extent (block max, one atomic per CTA).
//   2. cell_kernel + scan + scatter_kernel: a uniform grid with the cell edge
//      just above the largest extent, hashed into a power-of-two table; every
//      capsule is filed under the cell of its box's lower corner (a counting
//      sort by bucket).
//   3. pairs_kernel<0>: every capsule tests the capsules filed in its 27
//      neighbouring cells, then every plane, in one pass, writing up to
//      kFixedPartners partners into its fixed-stride list (sorted) and its
//      count; a capsule with more partners takes a region of the overflow
//      lists (one atomic on their total), and pairs_kernel<1> writes its
//      whole sorted list there.  Two boxes that overlap have lower corners less
//      than one cell apart on each axis, so the candidate set equals the
//      exhaustive search's (Detection/Coarse/ExhaustiveSearch.hpp:322-435,
//      closed intervals of BoundingBox.hpp:532-540), which the reference's
//      hash grids reproduce (tests/.../Test_HashGrids.cpp).
//   4. force_kernel: each capsule evaluates the narrow phase with every
//      partner in ascending id order (RodCapsuleRodCapsule.hpp:70-186,
//      CapsulePlane.hpp:60-113), the pair always oriented with the smaller id
//      as the first body, and sums the spring-dashpot loads
//      (LinearSpringDashpot.cpp:32-85) that act on itself.  Each pair is
//      evaluated by both of its capsules; no atomics, so the loads are
//      deterministic.
//   5. the step kernel adds half the capsule force to each node and the
//      torque, recast as Q tau, to the element (Transfer/Common.hpp:32-55).
//
// This file is compiled without contraction of multiply-adds, so every
// product and sum is rounded as written; the capsules, boxes and candidate
// pairs are then bit-identical to a scalar FP64 evaluation of the same
// expressions.
#include <cuda_runtime.h>

#include <algorithm>

#include "contact.h"
#include "rod_math.cuh"

namespace eb {
namespace {

using D3 = Vec3<double>;

constexpr double kContactThreshold = 1e-8;   // Utilities/Thresholds.hpp:138
constexpr double kParallelThreshold = 1e-8;  // Utilities/Thresholds.hpp:159
constexpr double kFrictionThreshold = 1e-8;  // Utilities/Thresholds.hpp:149
constexpr double kZeroLength = 1e-8;         // is_zero_length bound (Utilities/Math/Zero.hpp:46-49)
constexpr double kCellMargin = 1.0 + 1.0 / 1048576.0;
constexpr double kCellClamp = 1073741824.0;  // 2^30 cells from the origin

constexpr int kThreads = 256;
// the narrow phase: 128-thread CTAs, three per SM at 168 registers a thread
// (12 warps; 256 threads at 192 registers held 8, and a 128-register bound
// spilled 500 bytes a thread): 0.91 -> 0.82 ms a contact step
constexpr int kForceThreads = 128;
constexpr int kForceCtasPerSm = 3;
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanBlock = kScanThreads * kScanItems;

__device__ __forceinline__ D3 ld3(const double* p, int64_t S, int64_t s) { return {p[s], p[S + s], p[2 * S + s]}; }
__device__ __forceinline__ void st3(double* p, int64_t S, int64_t s, D3 a) {
  p[s] = a.x;
  p[S + s] = a.y;
  p[2 * S + s] = a.z;
}
__device__ __forceinline__ D3 mul3(double k, D3 a) { return {k * a.x, k * a.y, k * a.z}; }
__device__ __forceinline__ D3 neg3(D3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ double norm3(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
// blaze::normalize: a * (1 / |a|), a zero vector stays zero
__device__ __forceinline__ D3 normalize3(D3 a) {
  const double len = norm3(a);
  const double il = len != 0.0 ? 1.0 / len : 0.0;
  return {a.x * il, a.y * il, a.z * il};
}

// a capsule's shape (centre, axis, length, radius); its velocity and
// angular velocity are read from the table only where a contact point needs
// them, so they are not held in registers through the closest-point search
// (that took the narrow phase's spills from 108 to 52 B a thread and the
// contact step from 0.71 to 0.69 ms)
struct Capsule {
  D3 c, u;
  double L, r;
};

__device__ __forceinline__ Capsule load_capsule(const double* cap, int64_t S, int64_t s) {
  Capsule k;
  k.c = ld3(cap + kCapC * S, S, s);
  k.L = cap[kCapL * S + s];
  k.r = cap[kCapR * S + s];
  k.u = ld3(cap + kCapU * S, S, s);
  return k;
}

__device__ __forceinline__ bool overlaps(const double alo[3], const double ahi[3], const double blo[3],
                                         const double bhi[3]) {
  return !(blo[0] > ahi[0] || blo[1] > ahi[1] || blo[2] > ahi[2] || bhi[0] < alo[0] || bhi[1] < alo[1] ||
           bhi[2] < alo[2]);
}

__device__ __forceinline__ uint32_t cell_hash(int32_t cx, int32_t cy, int32_t cz) {
  uint64_t h = static_cast<uint64_t>(static_cast<uint32_t>(cx)) * 0x9E3779B97F4A7C15ull ^
               static_cast<uint64_t>(static_cast<uint32_t>(cy)) * 0xC2B2AE3D27D4EB4Full ^
               static_cast<uint64_t>(static_cast<uint32_t>(cz)) * 0x165667B19E3779F9ull;
  h ^= h >> 29;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 32;
  return static_cast<uint32_t>(h);
}

// ---- stage 1: capsules and boxes ------------------------------------------

__global__ void __launch_bounds__(kThreads) capsule_kernel(const ContactArgs a) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
  const int64_t S = a.stride;
  double ext = 0.0;
  bool bad = false;
  if (s < a.n_slots && a.cap_material[s] >= 0) {
    const double* x = a.state + kStX * S;
    const double* v = a.state + kStV * S;
    const double* w = a.state + kStW * S;
    const double c = a.half_dt;
    // positions after the first half drift (PositionVerlet.hpp:60-69) and
    // the clamp's value constraint
    D3 x0 = {x[s] + c * v[s], x[S + s] + c * v[S + s], x[2 * S + s] + c * v[2 * S + s]};
    D3 x1 = {x[s + 1] + c * v[s + 1], x[S + s + 1] + c * v[S + s + 1], x[2 * S + s + 1] + c * v[2 * S + s + 1]};
    const uint32_t meta = a.meta[s];
    if (a.sim_flags & kSimClamp) {
      // either node of the element may be held by a clamp
      const RodInfo& ri = a.rods[meta >> kRodShift];
      double t[3];
      if (clamp_position(ri, s, t)) x0 = {t[0], t[1], t[2]};
      if (clamp_position(ri, s + 1, t)) x1 = {t[0], t[1], t[2]};
    }
    const D3 dx = x1 - x0;
    const double l = norm3(dx);
    const D3 t = {dx.x / l, dx.y / l, dx.z / l};
    const double l0 = a.par[kL0 * S + s];
    const double e = l / l0;
    const double L = e * l0;
    const double r = sqrt(M_1_PI * a.par[kVol * S + s] / l);
    const D3 cen = {0.5 * (x0.x + x1.x), 0.5 * (x0.y + x1.y), 0.5 * (x0.z + x1.z)};
    // Orthogonal.cpp:32-55 with the tangent as the third row
    const D3 v1 = normalize3(t);
    D3 v2 = {0.8, 0.6, 0.0};
    D3 v3 = cross(v1, v2);
    v2 = cross(v3, v1);
    if (dot(v2, v2) < kZeroLength) {
      v2 = {0.6, -0.8, 0.0};
      v3 = normalize3(cross(v1, v2));
      v2 = cross(v3, v1);
    }
    const D3 r0 = normalize3(v2), r1 = normalize3(v3), r2 = v1;
    const double m0 = a.par[kMass * S + s], m1 = a.par[kMass * S + s + 1];
    const D3 va = ld3(v, S, s), vb = ld3(v, S, s + 1);
    const D3 num = mul3(m0, va) + mul3(m1, vb);
    const double den = m0 + m1;
    const D3 vel = {num.x / den, num.y / den, num.z / den};
    const D3 om = ld3(w, S, s);
    const D3 ww = {r0.x * om.x + r1.x * om.y + r2.x * om.z, r0.y * om.x + r1.y * om.y + r2.y * om.z,
                   r0.z * om.x + r1.z * om.y + r2.z * om.z};
    double* cap = a.cap;
    st3(cap + kCapC * S, S, s, cen);
    cap[kCapL * S + s] = L;
    cap[kCapR * S + s] = r;
    st3(cap + kCapU * S, S, s, r2);
    st3(cap + kCapVel * S, S, s, vel);
    st3(cap + kCapW * S, S, s, ww);
    const double ua[3] = {r2.x, r2.y, r2.z}, ca[3] = {cen.x, cen.y, cen.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double len = fabs(ua[d] * L) * 0.5 + r + kContactThreshold;
      const double lo = ca[d] - len, hi = ca[d] + len;
      cap[(kCapLo + d) * S + s] = lo;
      cap[(kCapHi + d) * S + s] = hi;
      const double xt = hi - lo;
      if (!(xt >= 0.0 && xt < 1e300)) bad = true;  // NaN or infinite box
      else ext = fmax(ext, xt);
    }
  }
  // block max of the extents, one atomic per CTA (non-negative doubles order
  // like their bit patterns)
  for (int o = 16; o > 0; o >>= 1) ext = fmax(ext, __shfl_xor_sync(0xffffffffu, ext, o));
  __shared__ double wmax[kThreads / 32];
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = ext;
  if (bad) atomicOr(a.status, kStatusContactNonFinite);
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int i = 0; i < kThreads / 32; ++i) m = fmax(m, wmax[i]);
    if (m > 0.0) atomicMax(a.extent_bits, static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

// ---- stage 2: grid cells, counting sort by bucket --------------------------

__device__ __forceinline__ double inverse_cell(const ContactArgs& a) {
  double h = __longlong_as_double(static_cast<long long>(*a.extent_bits)) * kCellMargin;
  if (!(h > 0.0)) h = 1.0;
  return 1.0 / h;
}

__global__ void __launch_bounds__(kThreads) cell_kernel(const ContactArgs a) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (s == 0) a.pair_offset[a.n_slots] = 0;  // the pair search's overflow total
  if (s >= a.n_slots || a.cap_material[s] < 0) return;
  const int64_t S = a.stride;
  // a capsule whose box is not finite (a diverged state, already flagged by
  // the capsule kernel) takes no part: it would overlap every box
  bool finite = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double lo = a.cap[(kCapLo + d) * S + s], hi = a.cap[(kCapHi + d) * S + s];
    finite = finite && (hi - lo >= 0.0) && (hi - lo < 1e300) && (fabs(lo) < 1e300);
  }
  if (!finite) {
    a.bucket[s] = 0xffffffffu;
    a.pair_count[s] = 0;
    return;
  }
  const double ih = inverse_cell(a);
  int32_t c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double f = floor(a.cap[(kCapLo + d) * S + s] * ih);
    f = fmin(fmax(f, -kCellClamp), kCellClamp);
    c[d] = static_cast<int32_t>(f);
    a.cell[d * S + s] = c[d];
  }
  const uint32_t b = cell_hash(c[0], c[1], c[2]) & a.table_mask;
  a.bucket[s] = b;
  // the capsule's rank in its bucket, kept in its pair count until the
  // scatter has filed it (the pair search then writes the count)
  a.pair_count[s] = atomicAdd(a.bucket_count + b, 1);
}

__global__ void __launch_bounds__(kThreads) scatter_kernel(const ContactArgs a) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (s == 0) *a.extent_bits = 0;  // read only by the cell kernel: zero for the next evaluation
  if (s >= a.n_slots || a.cap_material[s] < 0) return;
  const int64_t S = a.stride;
  const uint32_t b = a.bucket[s];
  if (b > a.table_mask) return;  // excluded (not finite)
  const int32_t pos = a.bucket_start[b] + a.pair_count[s];  // the rank the cell kernel took
  if (pos < 0 || pos >= a.n_caps) {  // cannot happen with consistent counts; never write out of range
    atomicOr(a.status, kStatusContactIndex);
    return;
  }
  double* rec = a.sorted_rec + static_cast<int64_t>(kSortedRecDoubles) * pos;
  *reinterpret_cast<int4*>(rec) = make_int4(a.cell[s], a.cell[S + s], a.cell[2 * S + s], static_cast<int32_t>(s));
  double2* box = reinterpret_cast<double2*>(rec + 2);
  box[0] = make_double2(a.cap[kCapLo * S + s], a.cap[(kCapLo + 1) * S + s]);
  box[1] = make_double2(a.cap[(kCapLo + 2) * S + s], a.cap[kCapHi * S + s]);
  box[2] = make_double2(a.cap[(kCapHi + 1) * S + s], a.cap[(kCapHi + 2) * S + s]);
}

// ---- stage 3: candidate pairs ----------------------------------------------

__device__ __forceinline__ void sort_ids(int32_t* v, int32_t n) {
  for (int32_t i = 1; i < n; ++i) {
    const int32_t x = v[i];
    int32_t j = i - 1;
    while (j >= 0 && v[j] > x) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = x;
  }
}

// The search of one capsule.  kPass 0 (idx: a filed entry, the capsule's
// cell and box from its record) counts the partners and fills the
// fixed-stride list; kPass 1 (idx: a slot, leaving at once unless its
// coalesced count is above kFixedPartners; the cell and box from the
// slot-major rows the records were written from) writes the overflow list of
// a capsule with more partners.  The search is bound by dependent round
// trips to L2: every entry of a neighbouring bucket is one 64-byte record
// read whole before it is tested (its cell, slot and box were three
// dependent loads when kept in separate arrays), and the bucket range of the
// next neighbouring cell is loaded while the current one's entries are
// scanned.
template <int kPass>
__device__ __forceinline__ void search_one(const ContactArgs& a, int32_t n_caps, int64_t idx) {
  int32_t id, cx, cy, cz;
  double lo[3], hi[3];
  int32_t* out;
  if (kPass == 1) {
    const int64_t s = idx;
    // only filed capsules have a count; the others hold zero
    if (s >= a.n_slots || a.pair_count[s] <= kFixedPartners) return;
    const int64_t total = a.pair_offset[a.n_slots];
    if (total > a.capacity) {
      atomicOr(a.status, kStatusPairOverflow);
      atomicMax(a.required, static_cast<unsigned long long>(total));
      return;
    }
    out = a.partners + a.pair_offset[s];  // within [0, capacity)
    const int64_t S = a.stride;
    id = static_cast<int32_t>(s);
    cx = a.cell[s];
    cy = a.cell[S + s];
    cz = a.cell[2 * S + s];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = a.cap[(kCapLo + d) * S + s];
      hi[d] = a.cap[(kCapHi + d) * S + s];
    }
  } else {
    const int32_t e = static_cast<int32_t>(idx);
    if (e >= n_caps) return;
    const double* own = a.sorted_rec + static_cast<int64_t>(kSortedRecDoubles) * e;
    const int4 me = *reinterpret_cast<const int4*>(own);
    id = me.w;
    out = a.fixed + static_cast<int64_t>(id) * kFixedPartners;
    cx = me.x;
    cy = me.y;
    cz = me.z;
    const double2* ob = reinterpret_cast<const double2*>(own + 2);
    const double2 o0 = ob[0], o1 = ob[1], o2 = ob[2];
    lo[0] = o0.x;
    lo[1] = o0.y;
    lo[2] = o1.x;
    hi[0] = o1.y;
    hi[1] = o2.x;
    hi[2] = o2.y;
  }
  int32_t cnt = 0;
  // neighbour cell c: dx = c % 3 - 1 fastest, then dy, then dz
  uint32_t b = cell_hash(cx - 1, cy - 1, cz - 1) & a.table_mask;
  int32_t next0 = a.bucket_start[b], next1 = a.bucket_start[b + 1];
  for (int c = 0; c < 27; ++c) {
    const int32_t nx = cx + c % 3 - 1, ny = cy + (c / 3) % 3 - 1, nz = cz + c / 9 - 1;
    const int32_t k0 = max(next0, 0), k1 = min(next1, n_caps);
    if (c + 1 < 27) {
      b = cell_hash(cx + (c + 1) % 3 - 1, cy + ((c + 1) / 3) % 3 - 1, cz + (c + 1) / 9 - 1) & a.table_mask;
      next0 = a.bucket_start[b];
      next1 = a.bucket_start[b + 1];
    }
    for (int32_t k = k0; k < k1; ++k) {
      const double* r = a.sorted_rec + static_cast<int64_t>(kSortedRecDoubles) * k;
      const int4 h = *reinterpret_cast<const int4*>(r);
      const double2* rb = reinterpret_cast<const double2*>(r + 2);
      const double2 b0 = rb[0], b1 = rb[1], b2 = rb[2];
      // every part of the record is used whatever the cell, so all four
      // loads issue together
      const bool in_cell = (h.x == nx) & (h.y == ny) & (h.z == nz) & (h.w != id);
      const bool apart = (b0.x > hi[0]) | (b0.y > hi[1]) | (b1.x > hi[2]) | (b1.y < lo[0]) | (b2.x < lo[1]) |
                         (b2.y < lo[2]);
      if (!in_cell || apart) continue;
      if (kPass == 1 || cnt < kFixedPartners) out[cnt] = h.w;
      ++cnt;
    }
  }
  for (int32_t p = 0; p < a.n_planes; ++p) {
    if (!overlaps(lo, hi, a.planes[p].lo, a.planes[p].hi)) continue;
    if (kPass == 1 || cnt < kFixedPartners) out[cnt] = static_cast<int32_t>(a.n_slots) + p;
    ++cnt;
  }
  if (kPass == 0) {
    a.pair_count[id] = cnt;
    // a capsule with more partners takes a region of the overflow lists
    // (in whatever order the atomics come; every list is whole and sorted)
    if (cnt > kFixedPartners)
      a.pair_offset[id] = static_cast<int64_t>(atomicAdd(
          reinterpret_cast<unsigned long long*>(a.pair_offset + a.n_slots), static_cast<unsigned long long>(cnt)));
    if (cnt <= kFixedPartners) sort_ids(out, cnt);  // ascending partner order
  } else {
    sort_ids(out, cnt);
  }
}

// a grid of resident CTAs whose threads step through the entries (pass 0) or
// slots (pass 1), as the narrow phase does
template <int kPass>
__global__ void __launch_bounds__(kThreads) pairs_kernel(const ContactArgs a, int32_t n_caps_max) {
  // entries filed this evaluation (the capsules with finite boxes)
  const int32_t n_caps = min(a.bucket_start[a.table_mask + 1], n_caps_max);
  const int64_t n = kPass == 1 ? a.n_slots : n_caps;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kThreads;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride)
    search_one<kPass>(a, n_caps, i);
}

// ---- exclusive scan of int32 counts (out[n] = total), accumulated in Acc ----

template <typename Acc>
__device__ __forceinline__ Acc block_exclusive_scan(Acc v, Acc* total) {
  __shared__ Acc warp_sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Acc x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const Acc y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    Acc ws = warp_sums[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const Acc y = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += y;
    }
    warp_sums[lane] = ws;
  }
  __syncthreads();
  const Acc prefix = (wid > 0 ? warp_sums[wid - 1] : Acc(0)) + x - v;
  *total = warp_sums[kScanThreads / 32 - 1];
  __syncthreads();
  return prefix;
}

template <typename Acc>
__global__ void __launch_bounds__(kScanThreads) scan_partial(int32_t* in, Acc* out, int64_t n, Acc* block_sums,
                                                             bool zero_in) {
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanBlock + static_cast<int64_t>(threadIdx.x) * kScanItems;
  Acc v[kScanItems];
  Acc sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = base + i < n ? static_cast<Acc>(in[base + i]) : Acc(0);
    sum += v[i];
  }
  Acc total;
  Acc run = block_exclusive_scan<Acc>(sum, &total);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) {
      out[base + i] = run;
      if (zero_in) in[base + i] = 0;
    }
    run += v[i];
  }
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

template <typename Acc>
__global__ void __launch_bounds__(kScanThreads) scan_top(Acc* block_sums, int64_t nb, Acc* out, int64_t n) {
  Acc carry = 0;
  for (int64_t base = 0; base < nb; base += kScanThreads) {
    const int64_t i = base + threadIdx.x;
    const Acc v = i < nb ? block_sums[i] : Acc(0);
    Acc total;
    const Acc pre = block_exclusive_scan<Acc>(v, &total);
    if (i < nb) block_sums[i] = carry + pre;
    carry += total;
  }
  if (threadIdx.x == 0) out[n] = carry;
}

template <typename Acc>
__global__ void __launch_bounds__(kScanThreads) scan_add(Acc* out, int64_t n, const Acc* block_sums) {
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanBlock + static_cast<int64_t>(threadIdx.x) * kScanItems;
  const Acc add = block_sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) out[base + i] += add;
}

template <typename Acc>
cudaError_t exclusive_scan(int32_t* in, Acc* out, int64_t n, Acc* block_sums, bool zero_in, cudaStream_t stream,
                           int64_t* launches) {
  const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
  if (nb > 0)
    scan_partial<Acc><<<static_cast<unsigned>(nb), kScanThreads, 0, stream>>>(in, out, n, block_sums, zero_in);
  scan_top<Acc><<<1, kScanThreads, 0, stream>>>(block_sums, nb, out, n);
  if (nb > 0) scan_add<Acc><<<static_cast<unsigned>(nb), kScanThreads, 0, stream>>>(out, n, block_sums);
  *launches += nb > 0 ? 3 : 1;
  return cudaGetLastError();
}

// ---- stage 4: narrow phase and spring-dashpot loads ------------------------

struct ContactPoint {
  D3 pos, n;
  double dist;
};

// Utilities/Geometry/GetClosestLineSegmentPoints.cpp, branch for branch
__device__ void closest_segment_points(D3 a1, D3 a2, D3 b1, D3 b2, D3& cp1, D3& cp2) {
  const D3 a1a2 = a2 - a1, b1b2 = b2 - b1, a1b1 = b1 - a1;
  const double da1 = dot(a1a2, a1b1), db1 = dot(b1b2, a1b1);
  if (da1 <= 0.0 && db1 >= 0.0) {
    cp1 = a1;
    cp2 = b1;
    return;
  }
  const D3 a1b2 = b2 - a1;
  const double da2 = dot(a1a2, a1b2), db2 = dot(b1b2, a1b2);
  if (da2 <= 0.0 && db2 <= 0.0) {
    cp1 = a1;
    cp2 = b2;
    return;
  }
  const D3 a2b1 = b1 - a2;
  const double da3 = dot(a1a2, a2b1), db3 = dot(b1b2, a2b1);
  if (da3 >= 0.0 && db3 >= 0.0) {
    cp1 = a2;
    cp2 = b1;
    return;
  }
  const D3 a2b2 = b2 - a2;
  const double da4 = dot(a1a2, a2b2), db4 = dot(b1b2, a2b2);
  if (da4 >= 0.0 && db4 <= 0.0) {
    cp1 = a2;
    cp2 = b2;
    return;
  }
  const double la = dot(a1a2, a1a2);
  if (da1 >= -kParallelThreshold && da3 <= kParallelThreshold) {
    const D3 k = mul3(da1 / la, a1a2);
    const D3 n = a1b1 - k;
    if (dot(b1b2, n) >= -kParallelThreshold) {
      cp1 = a1 + k;
      cp2 = b1;
      return;
    }
  }
  if (da2 >= -kParallelThreshold && da4 <= kParallelThreshold) {
    const D3 k = mul3(da2 / la, a1a2);
    const D3 n = a1b2 - k;
    if (dot(b1b2, n) <= kParallelThreshold) {
      cp1 = a1 + k;
      cp2 = b2;
      return;
    }
  }
  const double lb = dot(b1b2, b1b2);
  if (db1 <= kParallelThreshold && db2 >= -kParallelThreshold) {
    const D3 k = mul3(-db1 / lb, b1b2);
    const D3 n = neg3(a1b1) - k;
    if (dot(a1a2, n) >= -kParallelThreshold) {
      cp1 = a1;
      cp2 = b1 + k;
      return;
    }
  }
  if (db3 <= kParallelThreshold && db4 >= -kParallelThreshold) {
    const D3 k = mul3(-db3 / lb, b1b2);
    const D3 n = neg3(a2b1) - k;
    if (dot(a1a2, n) <= kParallelThreshold) {
      cp1 = a2;
      cp2 = b1 + k;
      return;
    }
  }
  const double sc = dot(a1a2, b1b2);
  double div = la * lb - sc * sc;
  div = 1.0 / div;
  const double sp = (lb * da1 - sc * db1) * div;
  const double tp = (sc * da1 - la * db1) * div;
  cp1 = a1 + mul3(sp, a1a2);
  cp2 = b1 + mul3(tp, b1b2);
}

// RodCapsuleRodCapsule.hpp:70-186 (c1 has the smaller id)
__device__ __forceinline__ int rod_capsule_contacts(const Capsule& c1, const Capsule& c2, ContactPoint out[2]) {
  const D3 up1 = mul3(0.5 * c1.L, c1.u), up2 = mul3(0.5 * c2.L, c2.u);
  D3 cp1, cp2;
  closest_segment_points(c1.c + up1, c1.c - up1, c2.c + up2, c2.c - up2, cp1, cp2);
  D3 nrm = cp1 - cp2;
  const double ln = norm3(nrm);
  if (ln < kContactThreshold) return 0;
  const double dist = ln - c1.r - c2.r;
  if (!(dist < kContactThreshold)) return 0;
  nrm = normalize3(nrm);
  const double c2x = dot(c1.u, c2.c - c1.c);
  if ((fabs(dot(c1.u, c2.u)) - 1.0) > -kParallelThreshold && fabs(c2x) < c1.L) {
    const double hl1 = 0.5 * c1.L, hl2 = 0.5 * c2.L;
    if (hl1 < c2x + hl2) {
      const double k = c1.r + 0.5 * dist;
      out[0] = {(c1.c + up1) - mul3(k, nrm), nrm, dist};
    } else {
      const double k = c2.r + 0.5 * dist;
      out[0] = {(c2.c + mul3(hl2, c1.u)) + mul3(k, nrm), nrm, dist};
    }
    if (-hl1 > c2x - hl2) {
      const double k = c1.r + 0.5 * dist;
      out[1] = {(c1.c - up1) - mul3(k, nrm), nrm, dist};
    } else {
      const double k = c2.r + 0.5 * dist;
      out[1] = {(c2.c - mul3(hl2, c1.u)) + mul3(k, nrm), nrm, dist};
    }
    return 2;
  }
  const double k = c2.r + 0.5 * dist;
  out[0] = {cp2 + mul3(k, nrm), nrm, dist};
  return 1;
}

// CapsulePlane.hpp:60-113
// (the points are written at constant indices, so they stay in registers)
__device__ __forceinline__ int capsule_plane_contacts(const Capsule& c, const ContactPlane& p, ContactPoint out[2]) {
  const D3 up = mul3(0.5 * c.L, c.u);
  const D3 pu = c.c + up, pl = c.c - up;
  const D3 pp = {p.p[0], p.p[1], p.p[2]}, n = {p.n[0], p.n[1], p.n[2]};
  const double du = fabs(dot(n, pu - pp)) - c.r;
  const double dl = fabs(dot(n, pl - pp)) - c.r;
  const bool hu = du < kContactThreshold, hl = dl < kContactThreshold;
  if (hu) out[0] = {pu - mul3(c.r + du, n), n, du};
  if (hl) {
    const ContactPoint q = {pl - mul3(c.r + dl, n), n, dl};
    if (hu)
      out[1] = q;
    else
      out[0] = q;
  }
  return (hu ? 1 : 0) + (hl ? 1 : 0);
}

// velocity of the material point at pos of capsule s (centre c)
__device__ __forceinline__ D3 point_velocity(const double* cap, int64_t S, int64_t s, D3 c, D3 pos) {
  const D3 vel = ld3(cap + kCapVel * S, S, s), ww = ld3(cap + kCapW * S, S, s);
  return vel + cross(ww, pos - c);
}

// Contact.cpp:150-215 and LinearSpringDashpot.cpp:32-85; false: separated
__device__ bool spring_dashpot(const ContactPoint& ct, D3 rvel, const ContactPair& pm, D3& net) {
  if (!(ct.dist < -kContactThreshold)) return false;
  const D3 n = ct.n;
  const double rvn = dot(n, rvel);
  const double rvt = dot(n, rvel - mul3(rvn, n));
  const double mu = fabs(rvt) > kFrictionThreshold ? pm.mu_d : pm.mu_s;
  const double delta = -ct.dist;
  const double relvn = -dot(n, rvel);
  const D3 relvt = neg3(rvel) - mul3(relvn, n);
  const double fn = fmax(0.0, pm.k * delta + pm.cn * relvn);
  const double ft = fmin(pm.ct * norm3(relvt), mu * fn);
  net = mul3(fn, n) + mul3(ft, normalize3(relvt));
  return true;
}

__device__ __forceinline__ void force_one(const ContactArgs& a, int64_t s) {
  const int32_t mat = a.cap_material[s];
  if (mat < 0) return;
  const int64_t S = a.stride;
  D3 F = {0.0, 0.0, 0.0}, T = {0.0, 0.0, 0.0};
  const int32_t cnt = a.pair_count[s];
  const int32_t* list = a.fixed + s * kFixedPartners;
  bool ok = true;
  if (cnt > kFixedPartners) {
    const int64_t total = a.pair_offset[a.n_slots];
    ok = total <= a.capacity;
    list = a.partners + a.pair_offset[s];
  }
  if (ok) {
    const Capsule me = load_capsule(a.cap, S, s);
    ContactPoint pts[2];
    for (int32_t k = 0; k < cnt; ++k) {
      const int64_t o = list[k];
      if (o >= 0 && o < a.n_slots) {
        const int32_t om = a.cap_material[o];
        if (om < 0) continue;
        const bool first = s < o;
        const Capsule other = load_capsule(a.cap, S, o);
        const Capsule& c1 = first ? me : other;
        const Capsule& c2 = first ? other : me;
        const ContactPair pm = a.pair_table[(first ? mat : om) * a.n_materials + (first ? om : mat)];
        const int np = rod_capsule_contacts(c1, c2, pts);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          if (i >= np) break;
          const D3 rvel = point_velocity(a.cap, S, first ? s : o, c1.c, pts[i].pos) -
                          point_velocity(a.cap, S, first ? o : s, c2.c, pts[i].pos);
          D3 net;
          if (!spring_dashpot(pts[i], rvel, pm, net)) continue;
          // RigidBodyPrimitive.hpp:500-504 add_force_at_position
          const D3 f = first ? net : neg3(net);
          F = F + f;
          T = T + cross(pts[i].pos - me.c, f);
        }
      } else if (o >= a.n_slots && o < a.n_slots + a.n_planes) {
        const ContactPlane& P = a.planes[o - a.n_slots];
        const ContactPair pm = a.pair_table[mat * a.n_materials + P.material];
        const int np = capsule_plane_contacts(me, P, pts);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          if (i >= np) break;
          const D3 rvel = point_velocity(a.cap, S, s, me.c, pts[i].pos) - D3{0.0, 0.0, 0.0};  // the plane is fixed
          D3 net;
          if (!spring_dashpot(pts[i], rvel, pm, net)) continue;
          F = F + net;
          T = T + cross(pts[i].pos - me.c, net);
        }
      }
    }
  }
  st3(a.cf, S, s, F);
  st3(a.ct, S, s, T);
}

// a grid of resident CTAs whose threads step through the slots: the kernel
// has no barrier, so a warp whose capsules had few partners goes on to the
// next ones instead of waiting for the slowest warp of its CTA to finish
// (with the pair search done the same way: 0.691 -> 0.679 ms a contact step)
__global__ void __launch_bounds__(kForceThreads, kForceCtasPerSm) force_kernel(const ContactArgs a) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kForceThreads;
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * kForceThreads + threadIdx.x; s < a.n_slots; s += stride)
    force_one(a, s);
}

}  // namespace

int64_t contact_scan_blocks(int64_t n) { return (n + kScanBlock - 1) / kScanBlock + 1; }

cudaError_t launch_contact(const ContactArgs& a, cudaStream_t stream, int64_t* launches) {
  if (a.n_slots <= 0) return cudaSuccess;
  const unsigned gs = static_cast<unsigned>((a.n_slots + kThreads - 1) / kThreads);
  // the largest box extent and the bucket counts are zero here: allocated
  // zeroed, the extent set back to zero by the scatter once the cell kernel
  // has used it, and each count by the scan as it reads it; the cell kernel
  // zeroes the overflow lists' running total
  cudaError_t e = cudaSuccess;
  const int64_t table = static_cast<int64_t>(a.table_mask) + 1;
  capsule_kernel<<<gs, kThreads, 0, stream>>>(a);
  cell_kernel<<<gs, kThreads, 0, stream>>>(a);
  *launches += 2;
  e = exclusive_scan<int32_t>(a.bucket_count, a.bucket_start, table, reinterpret_cast<int32_t*>(a.scan_blocks), true,
                             stream, launches);
  if (e != cudaSuccess) return e;
  scatter_kernel<<<gs, kThreads, 0, stream>>>(a);
  const unsigned ge = static_cast<unsigned>((a.n_caps + kThreads - 1) / kThreads);
  int pdev = 0, psms = 148;
  if (cudaGetDevice(&pdev) == cudaSuccess) cudaDeviceGetAttribute(&psms, cudaDevAttrMultiProcessorCount, pdev);
  int pper = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pper, pairs_kernel<0>, kThreads, 0);
  const unsigned pblocks = static_cast<unsigned>(std::min<int64_t>(ge, static_cast<int64_t>(psms) * std::max(pper, 1)));
  if (ge > 0) pairs_kernel<0><<<pblocks, kThreads, 0, stream>>>(a, a.n_caps);
  *launches += 2;
  pairs_kernel<1><<<gs, kThreads, 0, stream>>>(a, a.n_caps);
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t fblocks = std::min<int64_t>((a.n_slots + kForceThreads - 1) / kForceThreads,
                                            static_cast<int64_t>(sms) * kForceCtasPerSm);
  force_kernel<<<static_cast<unsigned>(fblocks), kForceThreads, 0, stream>>>(a);
  *launches += 2;
  return cudaGetLastError();
}

}  // namespace eb
