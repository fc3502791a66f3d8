// Device-side description of the connections between rods (connection.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "eb_internal.h"

namespace eb {

enum JointKind : int32_t { kJointFree = 0, kJointHinge = 1 };

struct JointDev {
  int64_t node_a;  // slot of rod a's node index_a + 1
  int64_t node_b;  // slot of rod b's node index_b
  int32_t kind;    // JointKind
  int32_t pad;
  double k, nu, k_rot;
  double normal[3];
};

struct JointArgs {
  int32_t n_joints;
  const JointDev* joints;
  double* out;  // 6 per joint: force (3), lab-frame torque (3)
  const double* state;
  int64_t stride;
  double pre;  // drift before the force evaluation
  const uint32_t* meta;
  const RodInfo* rods;
  // per loaded slot, the joints acting on it (CSR, connection order)
  int64_t n_force_slots;
  const int64_t* force_slot;
  const int64_t* force_off;
  const int32_t* force_src;
  int64_t n_torque_slots;
  const int64_t* torque_slot;
  const int64_t* torque_off;
  const int32_t* torque_src;
  double* joint_force;   // 3 x stride, node slots
  double* joint_torque;  // 3 x stride, element slots
};

cudaError_t launch_joints(const JointArgs& a, cudaStream_t stream);

}  // namespace eb
