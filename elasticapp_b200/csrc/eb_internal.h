// Internal layout shared by the host side (eb_capi.cu) and the kernels.
//
// Device layout ("slots"): rod r with n_r elements owns n_r + 1 consecutive
// slots starting at offset[r].  Slot offset[r] + j holds node j (j <= n_r),
// element j (j < n_r) and Voronoi point j (j < n_r - 1), so every stagger
// shares one index and one offset table.  The reference instead pads each rod
// with ghost slots (1 node, 2 element, 3 Voronoi ghosts, elastica/Systems/
// CosseratRods/Traits/PlacementTraits/PlacementTraits.hpp:53-56,82-85,124-127)
// to give every stagger the stride n + 2; here the only unused entries are
// the element at j = n and the Voronoi points at j >= n - 1.
//
// Every field is a separate 1-D array of `stride` entries (stride = slot
// count rounded up to 32 so each array starts on a 256-byte boundary);
// component c of a vector field lives at base + c * stride.
#pragma once

#include <cstdint>

namespace eb {

// per-slot metadata word: flag bits | rod id << kRodShift
enum SlotFlags : uint32_t {
  kElem = 1u << 0,      // slot holds an element (j < n)
  kVor = 1u << 1,       // slot holds a Voronoi point (j < n - 1)
  kFirst = 1u << 2,     // j == 0
  kLastNode = 1u << 3,  // j == n
  kLastElem = 1u << 4,  // j == n - 1
};
constexpr int kRodShift = 5;
constexpr uint32_t kFlagMask = (1u << kRodShift) - 1u;

// state arrays (per ping-pong buffer), in units of `stride`
enum StateField : int {
  kStX = 0,   // 3: node positions
  kStV = 3,   // 3: node velocities
  kStQ = 6,   // 9: element directors, Q(k, j) at kStQ + 3k + j
  kStW = 15,  // 3: element angular velocities (material frame)
  kStateFields = 18
};

// parameter arrays, in units of `stride`
enum ParamField : int {
  kMass = 0,    // node mass
  kNuF = 1,     // node force damping rate
  kNuT = 2,     // element torque damping rate
  kL0 = 3,      // element rest length
  kD0 = 4,      // Voronoi rest length
  kVol = 5,     // element volume (read only for the element dimension)
  kSig0 = 6,    // 3: element rest shear/stretch strain
  kKap0 = 9,    // 3: Voronoi rest curvature
  kShear = 12,  // 3: element shear/stretch rigidity diagonal
  kBend = 15,   // 3: Voronoi bend/twist rigidity diagonal
  kJ = 18,      // 3: element mass second moment of inertia diagonal
  kJinv = 21,   // 3: its inverse
  kParamFields = 24
};

// derived (diagnostic) arrays, in units of `stride`
enum DiagField : int {
  kDLength = 0,
  kDDil = 1,
  kDTangent = 2,   // 3
  kDVDil = 5,
  kDSigma = 6,     // 3
  kDKappa = 9,     // 3
  kDStress = 12,   // 3
  kDCouple = 15,   // 3
  kDLoads = 18,    // 3
  kDTorques = 21,  // 3
  kDAccel = 24,    // 3
  kDAlpha = 27,    // 3
  kDDim = 30,
  kDiagFields = 31
};

enum RodFlags : uint32_t { kRodClamp = 1u, kRodEndTorque = 2u, kRodDamper = 4u };

struct RodInfo {
  double clamp_x[3];
  double clamp_Q[9];
  double end_torque[3];  // lab frame
  double damper_t;       // exp(-nu_t dt) for the dt of the current launch
  double damper_r;       // nu_r
  uint32_t flags;
  uint32_t pad;
  // global slots the constraints and the forcing act on (-1: none): clamp
  // 0 (targets clamp_x, clamp_Q) and clamp 1 (targets clamp2_x, clamp2_Q)
  // fix the node at their slot and, where the slot holds one, its element;
  // end_torque acts on the element at torque_slot
  int64_t clamp_slot[2];
  int64_t torque_slot;
  double clamp2_x[3];
  double clamp2_Q[9];
};

// per-slot bits derived from a slot's rod data (kernels keep them with the
// slot): which clamp holds the slot, whether the rod's torque acts on it,
// whether its rod has the damper
enum SlotHits : uint32_t { kHitClamp0 = 1u, kHitClamp1 = 2u, kHitTorque = 4u, kHitDamper = 8u };

// the clamp target of global slot g if one of the rod's clamps holds it
// (returns true and sets x), as the value constraint leaves it
__host__ __device__ __forceinline__ bool clamp_position(const RodInfo& ri, int64_t g, double x[3]) {
  if (!(ri.flags & kRodClamp)) return false;
  const double* t = g == ri.clamp_slot[0] ? ri.clamp_x : (g == ri.clamp_slot[1] ? ri.clamp2_x : nullptr);
  if (!t) return false;
  x[0] = t[0];
  x[1] = t[1];
  x[2] = t[2];
  return true;
}

// (every field is read up front and the test is branch free, so the loads
// go out together)
__host__ __device__ __forceinline__ uint32_t slot_hits(const RodInfo& ri, int64_t g) {
  const uint32_t fl = ri.flags;
  const int64_t c0 = ri.clamp_slot[0], c1 = ri.clamp_slot[1], ts = ri.torque_slot;
  const bool clamp = (fl & kRodClamp) != 0;
  return ((clamp & (g == c0)) ? kHitClamp0 : 0u) | ((clamp & (g == c1)) ? kHitClamp1 : 0u) |
         ((((fl & kRodEndTorque) != 0) & (g == ts)) ? kHitTorque : 0u) | ((fl & kRodDamper) ? kHitDamper : 0u);
}

struct StepArgs {
  int64_t stride;   // array stride (>= n_slots, multiple of 32)
  int64_t n_slots;  // used slots
  const double* in;     // state buffer read this step
  double* out;          // state buffer written this step
  const double* par;    // parameters
  const uint32_t* meta; // slot metadata
  const RodInfo* rods;
  double* diag;         // derived fields, or nullptr
  uint32_t* status;     // device status word (kStatus* bits), never cleared by kernels
  double dt;
  double half_dt;
  // substep times of one streaming launch: drift before the force
  // evaluation, kick, drift after it (PositionVerlet: dt/2, dt, dt/2)
  double drift_pre;
  double kick;
  double drift_post;
  // time the analytical damper's factors of this launch's rate constraint
  // stand for: dt (PositionVerlet; VelocityVerlet, whose damper constants
  // hold the full dt and act after each of its two kicks) or the kick's
  // share of dt (PEFRL)
  double damper_time;
  // force evaluations per step for the resident kernels: 0 or 1 is
  // PositionVerlet, 4 is PEFRL (coefficients below)
  int32_t n_sub;
  double gravity[3];
  uint32_t sim_flags;   // kSim* below
  // capsule contact loads of this step (lab frame, 3 x stride each, per
  // element slot), or nullptr without a collision system
  const double* contact_force;
  const double* contact_torque;
  // connection loads of this step (lab frame, 3 x stride each): forces per
  // node slot, torques per element slot; or nullptr without connections
  const double* joint_force;
  const double* joint_torque;
  // bound on the polls of a bounded wait for bulk copies (0: the built-in
  // bound); a small value exercises the timeout path
  uint32_t max_polls;
};

// Rods longer than one CTA's capacity run on a pair of CTAs (a thread-block
// cluster of two): the left CTA holds the first ceil(W / 2) of the rod's W
// slots, the right CTA the rest, and neighbour reads across the split go to
// the partner's shared memory.
constexpr int kPairMaxSlots = 1040;  // two 520-slot halves

// PEFRL (Omelyan, Mryglod and Folk, Comput. Phys. Commun. 146 (2002)
// 188-202): drifts xi, chi, 1 - 2 (chi + xi), chi, xi around the kicks
// (1 - 2 lambda) / 2, lambda, lambda, (1 - 2 lambda) / 2, in units of dt.
constexpr double kPefrlXi = 0.1786178958448091;
constexpr double kPefrlLambda = -0.2123418310626054;
constexpr double kPefrlChi = -0.06626458266981849;

// Per-CTA work of the serving launches (resident kernels): the CTA's slot
// range, its step count for this launch and the time step and environment of
// the request that owns it.
struct ServeCta {
  int64_t start;  // first slot
  int32_t count;  // slots
  int32_t steps;  // steps to run in this launch (>= 1)
  double dt;
  double half_dt;
  double gravity[3];
  uint32_t flags;  // kSim* bits of the request
  uint32_t pair;   // 1: this CTA and CTA (index ^ 1) hold the two halves of one rod
};

// device status bits reported back to the host
enum StatusBits : uint32_t {
  kStatusCopyTimeout = 1u,
  kStatusPairOverflow = 2u,     // the candidate pair list did not fit its buffer
  kStatusContactNonFinite = 4u, // a capsule had a non-finite bounding box
  kStatusContactIndex = 8u      // a grid index fell outside its table (never expected)
};

enum SimFlags : uint32_t { kSimGravity = 1u, kSimDamper = 2u, kSimEndTorque = 4u, kSimClamp = 8u };

}  // namespace eb
