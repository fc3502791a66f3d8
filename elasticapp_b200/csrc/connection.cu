// Connections (joints) between rods.
//
// The reference connects two rods with a user-written force and torque rule
// (simulator->connect(rod_a, at(i)).to(rod_b, at(j)).with(generator),
// elastica/Simulator/Connections/, applied among the pre-dynamic updates
// after the internal loads).  Here the rules are built in: the joint of the
// reference's hinge-joint example (examples/hinge_joint/
// HingeJointCaseStudy.cpp:96-150), with its index conventions:
//
//   force (every joint): d = x_b[j] - x_a[i + 1],
//     F = k d - nu ((v_b[j] - v_a[i + 1]) . u) u,  u = d / |d|
//     (Blaze's normalize multiplies by 1/|d|, or by 0 when |d| = 0),
//     rod a's node i + 1 gains F, rod b's node j loses it;
//   torque (hinge joints): l = x_b[j + 1] - x_b[j], f = -k_rot (l . n) n,
//     tau = l x f; rod a's element i loses Q_a tau and rod b's element j
//     gains Q_b tau (material frame).
//
// Positions are those of the force evaluation: drifted by the substep's
// first drift, with the clamp's value constraint.  Two launches per force
// evaluation: one thread per joint writes its force and torque, then one
// thread per loaded slot sums the joints acting on it in connection order
// (rod a's share before rod b's), so the sums are deterministic.  Torques
// are summed in the lab frame; the step kernel recasts them by the element's
// directors.  Built with --fmad=false, like the CPU restatement.
#include <cuda_runtime.h>

#include "eb_internal.h"
#include "joint.h"

namespace eb {
namespace {

struct P3 {
  double x, y, z;
};

__device__ __forceinline__ P3 node_position(const JointArgs& a, int64_t g) {
  const uint32_t m = a.meta[g];
  double t[3];
  if (clamp_position(a.rods[m >> kRodShift], g, t)) return {t[0], t[1], t[2]};
  const int64_t S = a.stride;
  const double* in = a.state;
  return {in[kStX * S + g] + a.pre * in[kStV * S + g], in[(kStX + 1) * S + g] + a.pre * in[(kStV + 1) * S + g],
          in[(kStX + 2) * S + g] + a.pre * in[(kStV + 2) * S + g]};
}

__device__ __forceinline__ P3 node_velocity(const JointArgs& a, int64_t g) {
  const int64_t S = a.stride;
  return {a.state[kStV * S + g], a.state[(kStV + 1) * S + g], a.state[(kStV + 2) * S + g]};
}

__global__ void joint_eval_kernel(const JointArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n_joints) return;
  const JointDev J = a.joints[c];
  const P3 xa = node_position(a, J.node_a), xb = node_position(a, J.node_b);
  const P3 va = node_velocity(a, J.node_a), vb = node_velocity(a, J.node_b);
  const P3 d = {xb.x - xa.x, xb.y - xa.y, xb.z - xa.z};
  const P3 fel = {J.k * d.x, J.k * d.y, J.k * d.z};
  const double len = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
  const double il = len != 0.0 ? 1.0 / len : len;
  const P3 u = {d.x * il, d.y * il, d.z * il};
  const P3 dv = {vb.x - va.x, vb.y - va.y, vb.z - va.z};
  const double vr = dv.x * u.x + dv.y * u.y + dv.z * u.z;
  const P3 vel = {vr * u.x, vr * u.y, vr * u.z};
  const double mnu = -J.nu;
  double* o = a.out + 6 * static_cast<int64_t>(c);
  o[0] = fel.x + mnu * vel.x;
  o[1] = fel.y + mnu * vel.y;
  o[2] = fel.z + mnu * vel.z;
  P3 tau = {0.0, 0.0, 0.0};
  if (J.kind == kJointHinge) {
    const P3 xb1 = node_position(a, J.node_b + 1);
    const P3 l = {xb1.x - xb.x, xb1.y - xb.y, xb1.z - xb.z};
    const double s = (-J.k_rot) * (l.x * J.normal[0] + l.y * J.normal[1] + l.z * J.normal[2]);
    const P3 f = {s * J.normal[0], s * J.normal[1], s * J.normal[2]};
    tau = {l.y * f.z - l.z * f.y, l.z * f.x - l.x * f.z, l.x * f.y - l.y * f.x};
  }
  o[3] = tau.x;
  o[4] = tau.y;
  o[5] = tau.z;
}

// slots [0, n_force_slots) of the combined index range sum forces, the rest
// torques; entry e of a slot's list is 2 * joint + (1 if subtracted)
__global__ void joint_apply_kernel(const JointArgs a) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool force = t < a.n_force_slots;
  const int64_t k = force ? t : t - a.n_force_slots;
  if (!force && k >= a.n_torque_slots) return;
  const int64_t* slot = force ? a.force_slot : a.torque_slot;
  const int64_t* off = force ? a.force_off : a.torque_off;
  const int32_t* src = force ? a.force_src : a.torque_src;
  double* dst = force ? a.joint_force : a.joint_torque;
  const int col = force ? 0 : 3;
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int64_t e = off[k]; e < off[k + 1]; ++e) {
    const int32_t v = src[e];
    const double* o = a.out + 6 * static_cast<int64_t>(v >> 1) + col;
    if (v & 1) {
      sx = sx - o[0];
      sy = sy - o[1];
      sz = sz - o[2];
    } else {
      sx = sx + o[0];
      sy = sy + o[1];
      sz = sz + o[2];
    }
  }
  const int64_t g = slot[k], S = a.stride;
  dst[g] = sx;
  dst[S + g] = sy;
  dst[2 * S + g] = sz;
}

}  // namespace

cudaError_t launch_joints(const JointArgs& a, cudaStream_t stream) {
  if (a.n_joints <= 0) return cudaSuccess;
  constexpr int kThreads = 128;
  joint_eval_kernel<<<(a.n_joints + kThreads - 1) / kThreads, kThreads, 0, stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int64_t n = a.n_force_slots + a.n_torque_slots;
  joint_apply_kernel<<<static_cast<unsigned>((n + kThreads - 1) / kThreads), kThreads, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace eb
