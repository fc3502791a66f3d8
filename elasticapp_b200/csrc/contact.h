// Device data of the collision system (rod elements as capsules), shared by
// the contact kernels (contact.cu) and the host side (eb_capi.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "eb_internal.h"

namespace eb {

// capsule table rows, in units of stride, indexed by element slot
enum CapsuleRow : int {
  kCapC = 0,     // 3: centre
  kCapL = 3,     // length
  kCapR = 4,     // radius
  kCapU = 5,     // 3: axis (third row of the capsule rotation)
  kCapVel = 8,   // 3: velocity
  kCapW = 11,    // 3: angular velocity taken to the world frame
  kCapLo = 14,   // 3: bounding box lower corner
  kCapHi = 17,   // 3: bounding box upper corner
  kCapRows = 20
};

constexpr int kSortedRecDoubles = 8;

// partners a capsule keeps in its fixed-stride list; a capsule with more
// (a pile-up) gets its whole list in the overflow lists instead
constexpr int kFixedPartners = 32;

struct ContactPlane {
  double p[3];   // point on the plane
  double n[3];   // unit normal
  double lo[3];  // bounding box
  double hi[3];
  int32_t material;
  int32_t pad;
};

// contact parameters of a material pair (series rule for stiffness and
// damping, sum for the friction coefficients)
struct ContactPair {
  double k, cn, ct, mu_s, mu_d;
};

struct ContactArgs {
  int64_t stride;
  int64_t n_slots;
  const double* state;  // state buffer read by the step (slot layout)
  const double* par;
  const uint32_t* meta;
  const RodInfo* rods;
  const int32_t* cap_material;  // per slot: material of the capsule, -1 if none
  double half_dt;
  uint32_t sim_flags;
  double* cap;                       // kCapRows x stride
  unsigned long long* extent_bits;   // largest box extent (bits of a non-negative double)
  int32_t* cell;                     // 3 x stride
  uint32_t* bucket;                  // stride
  uint32_t table_mask;               // hash table size - 1 (power of two)
  int32_t* bucket_count;             // table size (zero between steps)
  int32_t* bucket_start;             // table size + 1
  // the capsules grouped by bucket, one 64-byte record an entry: cell
  // (3 x int32) and slot (int32) in the first 16 bytes, then the box's lower
  // and upper corners (6 doubles)
  double* sorted_rec;                // kSortedRecDoubles per entry
  int32_t* pair_count;               // stride (zero outside capsules): partners per capsule (between
                                     // the cell kernel and the scatter: the capsule's rank in its bucket)
  int32_t* fixed;                    // kFixedPartners x stride: partner lists of up to kFixedPartners
  int64_t* pair_offset;              // n_slots + 1: a capsule's overflow list (if it has more than
                                     // kFixedPartners partners); [n_slots] their total
  int32_t* partners;                 // capacity: overflow lists
  int64_t capacity;
  unsigned long long* required;      // largest pair total seen when over capacity
  const ContactPlane* planes;
  int32_t n_planes;
  int32_t n_materials;
  const ContactPair* pair_table;     // n_materials x n_materials
  double* cf;                        // 3 x stride, capsule force (lab frame)
  double* ct;                        // 3 x stride, capsule torque (lab frame)
  int32_t n_caps;                    // number of capsules (fixed at finalize)
  int64_t* scan_blocks;              // block sums of the scans
  uint32_t* status;
};

// one whole contact evaluation (capsules, candidate pairs, contact loads)
// for the state a.state at the start of a step; launches counted into *launches
cudaError_t launch_contact(const ContactArgs& a, cudaStream_t stream, int64_t* launches);

// scratch sizes of launch_contact's scans
int64_t contact_scan_blocks(int64_t n);

}  // namespace eb
