// Host side of the C-ABI (include/elastica_b200.h): the simulator object,
// rod registry, straight-rod initializer, device buffers and the step loop.
//
// The simulator mirrors the reference's Simulator/Block plugin surface
// (elastica/Simulator/Interface/Simulator/Simulator.hpp,
// elastica/Simulator/Interface/Systems/Module.hpp): rods are emplaced and
// configured on the host, eb_finalize uploads them into the slot layout
// (csrc/eb_internal.h), and eb_step runs the fused step kernels on the
// simulator's own CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/elastica_b200.h"
#include "contact.h"
#include "eb_host.h"
#include "eb_internal.h"
#include "joint.h"

namespace eb {
cudaError_t launch_rod_step_fp64(const StepArgs& args, bool diag, bool damped, int window, cudaStream_t stream);
cudaError_t launch_rod_step_fp64_reference(const StepArgs& args, bool diag, bool damped, int window,
                                           cudaStream_t stream);
int block_config_count();
int block_config_capacity(int config);
int block_config_threads(int config);
cudaError_t launch_rod_block_fp64_gather(const StepArgs& args, const int64_t* cta_start, const int32_t* gmap,
                                         int n_ctas, int n_steps, int config, bool damped, cudaStream_t stream);
cudaError_t launch_rod_block_mixed_gather(const StepArgs& args, const int64_t* cta_start, const int32_t* gmap,
                                          int n_ctas, int n_steps, int config, bool damped, cudaStream_t stream);
cudaError_t launch_rod_block_fp64_pairs(const StepArgs& args, const int64_t* cta_start, const int32_t* gmap,
                                        int n_ctas, int n_steps, int config, bool damped, cudaStream_t stream);
cudaError_t launch_rod_block_mixed_pairs(const StepArgs& args, const int64_t* cta_start, const int32_t* gmap,
                                         int n_ctas, int n_steps, int config, bool damped, cudaStream_t stream);
cudaError_t launch_rod_energy(int64_t n_rods, int64_t stride, const int64_t* offsets,
                              const double* state, const double* params, double* out,
                              cudaStream_t stream);
}  // namespace eb

namespace {

thread_local std::string g_last_error;

eb_status fail(eb_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

#define EB_CUDA(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(EB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

enum Place { kNode = 0, kElement = 1, kVoronoi = 2 };
enum Kind { kState = 0, kParam = 1, kDiag = 2, kContactLoad = 3 };

struct FieldInfo {
  Place place;
  int ncomp;
  Kind kind;
  int offset;  // in units of stride inside its buffer
};

const FieldInfo kFields[EB_FIELD_COUNT] = {
    {kNode, 3, kState, eb::kStX},             // EB_POSITION
    {kNode, 3, kState, eb::kStV},             // EB_VELOCITY
    {kElement, 9, kState, eb::kStQ},          // EB_DIRECTOR
    {kElement, 3, kState, eb::kStW},          // EB_ANGULAR_VELOCITY
    {kNode, 1, kParam, eb::kMass},          // EB_MASS
    {kElement, 1, kParam, eb::kL0},         // EB_REFERENCE_ELEMENT_LENGTH
    {kVoronoi, 1, kParam, eb::kD0},         // EB_REFERENCE_VORONOI_LENGTH
    {kElement, 1, kParam, eb::kVol},        // EB_ELEMENT_VOLUME
    {kElement, 3, kParam, eb::kSig0},       // EB_REFERENCE_SHEAR_STRETCH_STRAIN
    {kVoronoi, 3, kParam, eb::kKap0},       // EB_REFERENCE_CURVATURE
    {kElement, 3, kParam, eb::kShear},      // EB_SHEAR_STRETCH_RIGIDITY_MATRIX
    {kVoronoi, 3, kParam, eb::kBend},       // EB_BENDING_TWIST_RIGIDITY_MATRIX
    {kElement, 3, kParam, eb::kJ},          // EB_MASS_SECOND_MOMENT_OF_INERTIA
    {kElement, 3, kParam, eb::kJinv},       // EB_INV_MASS_SECOND_MOMENT_OF_INERTIA
    {kNode, 1, kParam, eb::kNuF},           // EB_FORCE_DAMPING_RATE
    {kElement, 1, kParam, eb::kNuT},        // EB_TORQUE_DAMPING_RATE
    {kElement, 1, kDiag, eb::kDLength},     // EB_ELEMENT_LENGTH
    {kElement, 1, kDiag, eb::kDDil},        // EB_ELEMENT_DILATATION
    {kElement, 3, kDiag, eb::kDTangent},    // EB_TANGENT
    {kVoronoi, 1, kDiag, eb::kDVDil},       // EB_VORONOI_DILATATION
    {kElement, 3, kDiag, eb::kDSigma},      // EB_SHEAR_STRETCH_STRAIN
    {kVoronoi, 3, kDiag, eb::kDKappa},      // EB_CURVATURE
    {kElement, 3, kDiag, eb::kDStress},     // EB_INTERNAL_STRESS
    {kVoronoi, 3, kDiag, eb::kDCouple},     // EB_INTERNAL_COUPLE
    {kNode, 3, kDiag, eb::kDLoads},         // EB_INTERNAL_LOADS
    {kElement, 3, kDiag, eb::kDTorques},    // EB_INTERNAL_TORQUES
    {kNode, 3, kDiag, eb::kDAccel},         // EB_ACCELERATION
    {kElement, 3, kDiag, eb::kDAlpha},      // EB_ANGULAR_ACCELERATION
    {kElement, 1, kDiag, eb::kDDim},        // EB_ELEMENT_DIMENSION
    {kElement, 3, kContactLoad, 0},         // EB_CONTACT_FORCE
    {kElement, 3, kContactLoad, 3},         // EB_CONTACT_TORQUE
};

int64_t place_count(Place p, int64_t n) { return p == kNode ? n + 1 : (p == kElement ? n : n - 1); }

struct RodHost {
  int64_t n = 0;
  int32_t model = EB_ROD_UNDAMPED;
  // local slot-layout arrays: field f component c at (f + c) * (n + 1) + j
  std::vector<double> state, param, diag;
  eb::RodInfo info{};
  // rod-local index of each clamp (node k, and element k when k < n; -1:
  // none) and the element the torque acts on; the global slots are filled
  // in when the rod table is uploaded
  int64_t clamp_index[2] = {-1, -1};
  int64_t torque_index = -1;
  double damper_nu_t = 0.0;
  int32_t contact_material = -1;  // collision-system material, -1: no contact
};

// device side of the collision system
struct ContactDevice {
  bool on = false;
  int32_t n_caps = 0;
  uint32_t table_mask = 0;
  int64_t capacity = 0;
  double* cap = nullptr;
  int32_t* cap_material = nullptr;
  unsigned long long* extent = nullptr;
  int32_t* cell = nullptr;
  uint32_t* bucket = nullptr;
  int32_t* bucket_count = nullptr;
  int32_t* bucket_start = nullptr;
  double* sorted_rec = nullptr;
  int32_t* pair_count = nullptr;
  int32_t* fixed = nullptr;
  int64_t* pair_offset = nullptr;
  int32_t* partners = nullptr;
  unsigned long long* required = nullptr;
  eb::ContactPlane* planes = nullptr;
  eb::ContactPair* pair_table = nullptr;
  double* loads = nullptr;  // 6 x stride: force rows 0-2, torque rows 3-5
  int64_t* scan_blocks = nullptr;
  double* backup = nullptr;  // state at the start of a step chunk
  bool evaluated = false;
};

// a connection as added, and its device side
struct JointHost {
  int64_t rod_a, index_a, rod_b, index_b;
  eb_joint joint;
};

struct JointDevice {
  bool on = false;
  eb::JointDev* joints = nullptr;
  double* out = nullptr;
  int64_t *force_slot = nullptr, *force_off = nullptr, *torque_slot = nullptr, *torque_off = nullptr;
  int32_t *force_src = nullptr, *torque_src = nullptr;
  int64_t n_force = 0, n_torque = 0;
  double* loads = nullptr;  // 6 x stride: node force rows 0-2, element torque rows 3-5 (lab frame)
};

}  // namespace

struct eb_sim {
  eb_config cfg{};
  bool finalized = false;
  std::vector<RodHost> rods;
  double gravity[3] = {0.0, 0.0, 0.0};
  bool has_gravity = false;
  uint32_t sim_flags = 0;
  bool any_damped = false;
  // device
  cudaStream_t stream = nullptr;
  int64_t n_slots = 0, stride = 0;
  std::vector<int64_t> offsets;
  double* d_state[2] = {nullptr, nullptr};
  double* d_param = nullptr;
  double* d_diag = nullptr;
  uint32_t* d_meta = nullptr;
  eb::RodInfo* d_rods = nullptr;
  int64_t* d_offsets = nullptr;
  double* d_energy = nullptr;
  uint32_t* d_status = nullptr;
  uint32_t max_polls = 0;  // bounded-wait polls of the streaming kernel (0: built in)
  int cur = 0;
  double damper_dt = -1.0;
  int64_t launches = 0;
  // step plan: streaming kernel (one launch per step) or the resident kernel
  // with one of the block configurations, chosen by timing both
  int plan_mode = 0;    // 0 undecided, 1 streaming, 2 resident, 3 resident per size bucket
  int plan_config = -1;
  // the launch length (steps, at most one resident chunk) the plan was timed
  // at, and whether it was chosen by timing (not forced by the flags, the
  // collision system, connections or a configuration)
  int plan_chunk = 0;
  bool plan_timed = false;
  // per-size-bucket plan: bucket 0 holds the rods of at most 263 elements,
  // bucket 1 the rods of 264 to 519, bucket 2 the rods of 520 to 1039 (on
  // CTA pairs); per bucket and configuration a gathered work list (CTA
  // offsets into a list of slots)
  struct Bucket {
    int64_t* d_off[4] = {nullptr, nullptr, nullptr, nullptr};
    int32_t* d_map[4] = {nullptr, nullptr, nullptr, nullptr};
    int n_ctas[4] = {0, 0, 0, 0};
    int64_t rods = 0;
  };
  // bucket 3: buckets 0 and 1 packed together (used in their place when
  // faster; built when the batch also has pair rods)
  Bucket buckets[4];
  int bucket_config[4] = {-1, -1, -1, -1};
  bool bucket_merged = false;
  // whole-batch resident plan, per block configuration (or null): CTA c owns
  // the slots d_gmap[d_cta_start[c] .. d_cta_start[c + 1]); configurations
  // packed the same way share their lists
  std::vector<int64_t*> d_cta_start;
  std::vector<int32_t*> d_gmap;
  std::vector<int> n_ctas;
  float plan_ms[20] = {0};
  // host-state exchange (eb_step_host_state) under a resident plan: the rods
  // split into contiguous slot groups, each packed on its own for the plan
  // (xplan: mode and configuration it was built for), so one group's copies
  // overlap another's launches; per group one work list (whole-batch plan,
  // index 0) or one per size bucket; streams: copies in, copies out,
  // launches of even and of odd groups; events: the start, per group its
  // inputs landed and its steps done, the four streams' ends
  struct XGroup {
    int64_t lo = 0, hi = 0;  // slots [lo, hi)
    int64_t* d_off[4] = {nullptr, nullptr, nullptr, nullptr};
    int32_t* d_map[4] = {nullptr, nullptr, nullptr, nullptr};
    int n_ctas[4] = {0, 0, 0, 0};
  };
  std::vector<XGroup> xgroups;
  int64_t xplan = -1;
  cudaStream_t xs[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> xev;
  // captured streaming steps: per starting buffer parity, for graph_dt
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double graph_dt[2] = {0.0, 0.0};
  // collision system
  std::vector<eb_contact_material> materials;
  std::vector<eb::ContactPlane> planes;
  ContactDevice contact;
  // connections
  std::vector<JointHost> joints;
  JointDevice jd;
};

namespace {

eb_status check_sim(const eb_sim* s) {
  if (!s) return fail(EB_ERR_INVALID_ARGUMENT, "null simulator");
  return EB_OK;
}

eb_status set_device(const eb_sim* s) {
  EB_CUDA(cudaSetDevice(s->cfg.device));
  return EB_OK;
}

double norm3(const double a[3]) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
void cross3(const double m[3], const double v[3], double o[3]) {
  o[0] = m[1] * v[2] - m[2] * v[1];
  o[1] = m[2] * v[0] - m[0] * v[2];
  o[2] = m[0] * v[1] - m[1] * v[0];
}

// StraightCosseratRodInitializer and the component initialize() chains:
// positions by linspace (elastica/Utilities/Generators.hpp:86-119), directors
// from the normal and tangent (elastica/Utilities/Math/Orthogonal.cpp:32-55,
// 98-116), rest geometry (CosseratRodSpanwiseGeometry.hpp:526-545), cross
// section (CosseratRodCrossSectionInterface.hpp:266-307,
// CircleCrossSectionOperations.hpp:84-132), rigidities
// (LinearHyperElasticityFacade.hpp:273-327; Initializers/detail/Elasticity.hpp:
// 54-77) and kinematics (WithRodKinematics.hpp:344-424).
eb_status init_straight_rod(const eb_straight_rod& p, RodHost& r) {
  const int64_t n = p.n_elements;
  if (n < 2) return fail(EB_ERR_INVALID_ARGUMENT, "a rod needs at least 2 elements");
  if (!(p.radius > 0.0) || !(p.length > 0.0) || !(p.density > 0.0))
    return fail(EB_ERR_INVALID_ARGUMENT, "radius, length and density must be positive");
  if (p.model != EB_ROD_DAMPED && p.model != EB_ROD_UNDAMPED)
    return fail(EB_ERR_INVALID_ARGUMENT, "unknown rod model");
  if (p.model == EB_ROD_DAMPED && (p.force_damping_rate < 0.0 || p.torque_damping_rate < 0.0))
    return fail(EB_ERR_INVALID_ARGUMENT, "damping rates must be non-negative");
  const double dn = norm3(p.direction), nn = norm3(p.normal);
  if (dn == 0.0) return fail(EB_ERR_INVALID_ARGUMENT, "direction is zero");
  if (nn == 0.0) return fail(EB_ERR_INVALID_ARGUMENT, "normal is zero");
  const double t[3] = {p.direction[0] / dn, p.direction[1] / dn, p.direction[2] / dn};
  const double nv[3] = {p.normal[0] / nn, p.normal[1] / nn, p.normal[2] / nn};
  if (std::fabs(t[0] * nv[0] + t[1] * nv[1] + t[2] * nv[2]) > 1e-10)
    return fail(EB_ERR_INVALID_ARGUMENT, "the proposed normal and tangent are non-orthogonal");

  r.n = n;
  r.model = p.model;
  const int64_t W = n + 1;
  r.state.assign(static_cast<size_t>(eb::kStateFields * W), 0.0);
  r.param.assign(static_cast<size_t>(eb::kParamFields * W), 0.0);
  r.diag.assign(static_cast<size_t>(eb::kDiagFields * W), 0.0);
  auto S = [&](int f, int64_t j) -> double& { return r.state[static_cast<size_t>(f * W + j)]; };
  auto P = [&](int f, int64_t j) -> double& { return r.param[static_cast<size_t>(f * W + j)]; };

  for (int d = 0; d < 3; ++d) {
    const double stop = p.origin[d] + p.length * t[d];
    const double step = (stop - p.origin[d]) / static_cast<double>(n);
    for (int64_t j = 0; j <= n; ++j) S(eb::kStX + d, j) = p.origin[d] + static_cast<double>(j) * step;
  }
  double v1[3] = {nv[0], nv[1], nv[2]}, v2[3], v3[3], tmp[3];
  cross3(t, nv, v2);
  cross3(v1, v2, v3);
  cross3(v3, v1, tmp);
  std::memcpy(v2, tmp, sizeof(tmp));
  const double n2 = norm3(v2), n3 = norm3(v3);
  const double rows[9] = {v1[0],      v1[1],      v1[2],      v2[0] / n2, v2[1] / n2,
                          v2[2] / n2, v3[0] / n3, v3[1] / n3, v3[2] / n3};
  for (int k = 0; k < 9; ++k)
    for (int64_t i = 0; i < n; ++i) S(eb::kStQ + k, i) = rows[k];

  std::vector<double> l0(n), rad(n);
  for (int64_t i = 0; i < n; ++i) {
    const double dx[3] = {S(eb::kStX, i + 1) - S(eb::kStX, i), S(eb::kStX + 1, i + 1) - S(eb::kStX + 1, i),
                          S(eb::kStX + 2, i + 1) - S(eb::kStX + 2, i)};
    l0[i] = norm3(dx) / 1.0;
    P(eb::kL0, i) = l0[i];
  }
  for (int64_t k = 0; k + 1 < n; ++k) P(eb::kD0, k) = 0.5 * (l0[k] + l0[k + 1]);
  const double A = static_cast<double>(M_PI) * (p.radius * p.radius);
  for (int64_t i = 0; i < n; ++i) {
    P(eb::kVol, i) = A * l0[i];
    rad[i] = std::sqrt(M_1_PI * P(eb::kVol, i) / l0[i]);
    r.diag[static_cast<size_t>(eb::kDDim * W + i)] = rad[i];
  }
  auto I_of = [&](int64_t i, int d) {
    const double Ai = static_cast<double>(M_PI) * (rad[i] * rad[i]);
    const double I1 = (0.25 * M_1_PI) * (Ai * Ai);
    return d == 2 ? 2.0 * I1 : I1;
  };
  const double E = p.youngs_modulus, G = p.shear_modulus;
  const double stiff_b[3] = {E, E, G}, stiff_s[3] = {G, G, E};
  const double alpha_c = 13.5 / 14.0;
  for (int64_t i = 0; i < n; ++i) {
    const double Ai = static_cast<double>(M_PI) * (rad[i] * rad[i]);
    const double eff[3] = {Ai * alpha_c, Ai * alpha_c, Ai};
    for (int d = 0; d < 3; ++d) {
      P(eb::kShear + d, i) = stiff_s[d] * eff[d];
      P(eb::kJ + d, i) = I_of(i, d) * p.density * l0[i];
      P(eb::kJinv + d, i) = 1.0 / (I_of(i, d) * p.density * l0[i]);
    }
  }
  for (int64_t k = 0; k + 1 < n; ++k)
    for (int d = 0; d < 3; ++d)
      P(eb::kBend + d, k) =
          (l0[k] * stiff_b[d] * I_of(k, d) + l0[k + 1] * stiff_b[d] * I_of(k + 1, d)) / (l0[k] + l0[k + 1]);
  for (int64_t j = 0; j <= n; ++j) P(eb::kMass, j) = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double me = p.density * P(eb::kVol, i);
    P(eb::kMass, i) += 0.5 * me;
    P(eb::kMass, i + 1) += 0.5 * me;
  }
  if (p.model == EB_ROD_DAMPED) {
    for (int64_t j = 0; j <= n; ++j) P(eb::kNuF, j) = p.force_damping_rate;
    for (int64_t i = 0; i < n; ++i) P(eb::kNuT, i) = p.torque_damping_rate;
  }
  // benign values in the unused element / Voronoi entries of the last slots
  for (int d = 0; d < 3; ++d) {
    P(eb::kJ + d, n) = 1.0;
    P(eb::kJinv + d, n) = 1.0;
  }
  P(eb::kL0, n) = 1.0;
  P(eb::kD0, n - 1) = 1.0;
  P(eb::kD0, n) = 1.0;
  return EB_OK;
}

eb_status rod_field_check(const eb_sim* s, int64_t rod, int32_t field, int64_t count,
                          const FieldInfo** fi, int64_t* expected) {
  if (field < 0 || field >= EB_FIELD_COUNT) return fail(EB_ERR_INVALID_ARGUMENT, "unknown field");
  if (rod < 0 || rod >= static_cast<int64_t>(s->rods.size()))
    return fail(EB_ERR_NOT_FOUND, "unknown rod id");
  *fi = &kFields[field];
  *expected = (*fi)->ncomp * place_count((*fi)->place, s->rods[rod].n);
  if (count != *expected)
    return fail(EB_ERR_INVALID_ARGUMENT, "value count " + std::to_string(count) + " != " +
                                             std::to_string(*expected));
  return EB_OK;
}

double* device_base(eb_sim* s, const FieldInfo& f) {
  if (f.kind == kContactLoad)
    return s->contact.loads ? s->contact.loads + static_cast<int64_t>(f.offset) * s->stride : nullptr;
  double* base = f.kind == kState ? s->d_state[s->cur] : (f.kind == kParam ? s->d_param : s->d_diag);
  return base ? base + static_cast<int64_t>(f.offset) * s->stride : nullptr;
}

void host_free(eb_sim* s) {
  for (int b = 0; b < 2; ++b)
    if (s->d_state[b]) cudaFree(s->d_state[b]);
  if (s->d_param) cudaFree(s->d_param);
  if (s->d_diag) cudaFree(s->d_diag);
  if (s->d_meta) cudaFree(s->d_meta);
  if (s->d_rods) cudaFree(s->d_rods);
  if (s->d_offsets) cudaFree(s->d_offsets);
  if (s->d_energy) cudaFree(s->d_energy);
  if (s->d_status) cudaFree(s->d_status);
  s->d_status = nullptr;
  {
    std::vector<void*> owned;
    for (auto* p : s->d_cta_start) owned.push_back(p);
    for (auto* p : s->d_gmap) owned.push_back(p);
    std::sort(owned.begin(), owned.end());
    owned.erase(std::unique(owned.begin(), owned.end()), owned.end());
    for (void* p : owned)
      if (p) cudaFree(p);
  }
  s->d_cta_start.clear();
  s->d_gmap.clear();
  {
    JointDevice& j = s->jd;
    void* p[] = {j.joints, j.out, j.force_slot, j.force_off, j.torque_slot, j.torque_off, j.force_src, j.torque_src,
                 j.loads};
    for (void* q : p)
      if (q) cudaFree(q);
    j = JointDevice{};
  }
  for (auto& g : s->xgroups)
    for (int k = 0; k < 4; ++k) {
      if (g.d_off[k]) cudaFree(g.d_off[k]);
      if (g.d_map[k]) cudaFree(g.d_map[k]);
    }
  s->xgroups.clear();
  s->xplan = -1;
  for (auto& b : s->buckets) {
    for (int c = 0; c < 4; ++c) {
      if (b.d_off[c]) cudaFree(b.d_off[c]);
      if (b.d_map[c]) cudaFree(b.d_map[c]);
    }
    b = eb_sim::Bucket{};
  }
  for (auto& g : s->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  ContactDevice& c = s->contact;
  void* cptrs[] = {c.cap, c.cap_material, c.extent, c.cell, c.bucket, c.bucket_count, c.bucket_start,
                   c.sorted_rec, c.pair_count, c.fixed, c.pair_offset,
                   c.partners,
                   c.required, c.planes, c.pair_table, c.loads, c.scan_blocks, c.backup};
  for (void* p : cptrs)
    if (p) cudaFree(p);
  c = ContactDevice{};
  s->d_state[0] = s->d_state[1] = s->d_param = s->d_diag = s->d_energy = nullptr;
  s->d_meta = nullptr;
  s->d_rods = nullptr;
  s->d_offsets = nullptr;
}

// Read the device status word after the stream has drained.
eb_status check_device_status(eb_sim* s) {
  if (!s->d_status) return EB_OK;
  uint32_t st = 0;
  EB_CUDA(cudaMemcpyAsync(&st, s->d_status, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  if (st & eb::kStatusCopyTimeout)
    return fail(EB_ERR_CUDA, "a step kernel gave up waiting for its bulk copies (bounded wait expired)");
  if (st & eb::kStatusContactNonFinite)
    return fail(EB_ERR_NUMERICAL, "a capsule's bounding box was not finite: the state has diverged");
  if (st & eb::kStatusContactIndex)
    return fail(EB_ERR_CUDA, "the contact grid produced an out-of-range index (skipped)");
  return EB_OK;
}

eb_status upload_rod_table(eb_sim* s) {
  std::vector<eb::RodInfo> info(s->rods.size());
  for (size_t r = 0; r < s->rods.size(); ++r) {
    const RodHost& R = s->rods[r];
    info[r] = R.info;
    for (int c = 0; c < 2; ++c)
      info[r].clamp_slot[c] = R.clamp_index[c] >= 0 ? s->offsets[r] + R.clamp_index[c] : -1;
    info[r].torque_slot = R.torque_index >= 0 ? s->offsets[r] + R.torque_index : -1;
  }
  EB_CUDA(cudaMemcpyAsync(s->d_rods, info.data(), info.size() * sizeof(eb::RodInfo),
                          cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return EB_OK;
}

// ---- collision system set-up ------------------------------------------------

struct H3 {
  double x, y, z;
};
H3 h_cross(H3 a, H3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double h_dot(H3 a, H3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// blaze::normalize: a * (1 / |a|), a zero vector stays zero
H3 h_normalize(H3 a) {
  const double len = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  const double il = len != 0.0 ? 1.0 / len : 0.0;
  return {a.x * il, a.y * il, a.z * il};
}

// PlanePrimitive from a normal (PlanePrimitive.cpp:60-130): rotation rows
// from make_orthogonal_bases_from_normal (Utilities/Math/Orthogonal.cpp:32-55,
// 85-96) and the bounding box of the default 1e40 spans (PlanePrimitive.cpp:179-236)
eb::ContactPlane make_plane(const double point[3], const double normal[3], int32_t material) {
  const H3 v1 = h_normalize({normal[0], normal[1], normal[2]});
  H3 v2 = {0.8, 0.6, 0.0};
  H3 v3 = h_cross(v1, v2);
  v2 = h_cross(v3, v1);
  if (h_dot(v2, v2) < 1e-8) {  // is_zero_length with blaze::accuracy
    v2 = {0.6, -0.8, 0.0};
    v3 = h_normalize(h_cross(v1, v2));
    v2 = h_cross(v3, v1);
  }
  const H3 b = h_normalize(v2), t = h_normalize(v3);
  eb::ContactPlane P{};
  const double bb[3] = {b.x, b.y, b.z}, tt[3] = {t.x, t.y, t.z};
  const double n[3] = {v1.x, v1.y, v1.z};
  for (int d = 0; d < 3; ++d) {
    P.p[d] = point[d];
    P.n[d] = n[d];
    const double len = 0.5 * (std::fabs(bb[d] * 1e40) + std::fabs(tt[d] * 1e40)) + 1e-8;
    P.lo[d] = point[d] - len;
    P.hi[d] = point[d] + len;
  }
  P.material = material;
  return P;
}

eb_status setup_contact(eb_sim* s) {
  ContactDevice& c = s->contact;
  const int64_t S = s->stride, nr = static_cast<int64_t>(s->rods.size());
  std::vector<int32_t> cap_mat(static_cast<size_t>(S), -1);
  int64_t n_caps = 0;
  for (int64_t r = 0; r < nr; ++r) {
    const RodHost& R = s->rods[r];
    if (R.contact_material < 0) continue;
    for (int64_t i = 0; i < R.n; ++i) cap_mat[static_cast<size_t>(s->offsets[r] + i)] = R.contact_material;
    n_caps += R.n;
  }
  if (n_caps == 0) return EB_OK;
  if (s->cfg.precision == EB_PRECISION_MIXED)
    return fail(EB_ERR_UNSUPPORTED, "the collision system runs on the FP64 streaming step only");
  if (s->n_slots + static_cast<int64_t>(s->planes.size()) >= (int64_t(1) << 31) - 1)
    return fail(EB_ERR_UNSUPPORTED, "too many slots for the collision system's 32-bit ids");
  c.on = true;
  c.n_caps = static_cast<int32_t>(n_caps);
  int64_t table = 1024;
  // at least four buckets a capsule: every entry of another cell that shares
  // a neighbour's bucket is one more dependent read in the pair search
  // (contact step 0.646 -> 0.633 ms against two a capsule; eight: 0.645 ms)
  while (table < 4 * n_caps) table <<= 1;
  c.table_mask = static_cast<uint32_t>(table - 1);
  c.capacity = std::max<int64_t>(int64_t(1) << 16, 4 * n_caps);  // overflow lists only
  const size_t nm = s->materials.size();
  std::vector<eb::ContactPair> pairs(nm * nm);
  for (size_t i = 0; i < nm; ++i)
    for (size_t j = 0; j < nm; ++j) {
      const eb_contact_material& a = s->materials[i];
      const eb_contact_material& b = s->materials[j];
      pairs[i * nm + j] = {1.0 / (1.0 / a.stiffness + 1.0 / b.stiffness),
                           1.0 / (1.0 / a.normal_damping + 1.0 / b.normal_damping),
                           1.0 / (1.0 / a.tangential_damping + 1.0 / b.tangential_damping),
                           a.static_friction + b.static_friction, a.dynamic_friction + b.dynamic_friction};
    }
  const int64_t scan_blocks = eb::contact_scan_blocks(std::max<int64_t>(table, s->n_slots + 1));
  cudaError_t e = cudaSuccess;
  auto alloc = [&](auto** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, bytes, s->stream);
  };
  alloc(&c.cap, static_cast<size_t>(eb::kCapRows * S) * sizeof(double));
  alloc(&c.cap_material, static_cast<size_t>(S) * sizeof(int32_t));
  alloc(&c.extent, sizeof(unsigned long long));
  alloc(&c.cell, static_cast<size_t>(3 * S) * sizeof(int32_t));
  alloc(&c.bucket, static_cast<size_t>(S) * sizeof(uint32_t));
  alloc(&c.bucket_count, static_cast<size_t>(table) * sizeof(int32_t));
  alloc(&c.bucket_start, static_cast<size_t>(table + 1) * sizeof(int32_t));
  alloc(&c.sorted_rec, static_cast<size_t>(eb::kSortedRecDoubles * n_caps) * sizeof(double));
  alloc(&c.pair_count, static_cast<size_t>(S) * sizeof(int32_t));
  alloc(&c.fixed, static_cast<size_t>(S) * eb::kFixedPartners * sizeof(int32_t));
  alloc(&c.pair_offset, static_cast<size_t>(s->n_slots + 1) * sizeof(int64_t));
  alloc(&c.partners, static_cast<size_t>(c.capacity) * sizeof(int32_t));
  alloc(&c.required, sizeof(unsigned long long));
  alloc(&c.planes, std::max<size_t>(1, s->planes.size()) * sizeof(eb::ContactPlane));
  alloc(&c.pair_table, std::max<size_t>(1, pairs.size()) * sizeof(eb::ContactPair));
  alloc(&c.loads, static_cast<size_t>(6 * S) * sizeof(double));
  alloc(&c.scan_blocks, static_cast<size_t>(scan_blocks) * sizeof(int64_t));
  alloc(&c.backup, static_cast<size_t>(eb::kStateFields * S) * sizeof(double));
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? EB_ERR_OUT_OF_MEMORY : EB_ERR_CUDA,
                std::string("collision system allocation: ") + cudaGetErrorString(e));
  EB_CUDA(cudaMemcpyAsync(c.cap_material, cap_mat.data(), cap_mat.size() * sizeof(int32_t),
                          cudaMemcpyHostToDevice, s->stream));
  if (!s->planes.empty())
    EB_CUDA(cudaMemcpyAsync(c.planes, s->planes.data(), s->planes.size() * sizeof(eb::ContactPlane),
                            cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaMemcpyAsync(c.pair_table, pairs.data(), pairs.size() * sizeof(eb::ContactPair),
                          cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return EB_OK;
}

}  // namespace

namespace eb {
void set_last_error(const std::string& message) { g_last_error = message; }

eb_status host_straight_rod(const eb_straight_rod& p, HostRodData& out) {
  RodHost r;
  if (eb_status st = init_straight_rod(p, r)) return st;
  out.n = r.n;
  out.damped = r.model == EB_ROD_DAMPED;
  out.state = std::move(r.state);
  out.param = std::move(r.param);
  return EB_OK;
}
}  // namespace eb

extern "C" {

EB_API const char* eb_last_error(void) { return g_last_error.c_str(); }
EB_API const char* eb_version(void) { return "elastica_b200 0.1 (sm_100a)"; }

EB_API eb_status eb_sim_create(const eb_config* config, eb_sim** out) {
  if (!out) return fail(EB_ERR_INVALID_ARGUMENT, "null output pointer");
  *out = nullptr;
  eb_config cfg{};
  if (config) cfg = *config;
  if (cfg.precision != EB_PRECISION_FP64 && cfg.precision != EB_PRECISION_MIXED)
    return fail(EB_ERR_INVALID_ARGUMENT, "unknown precision");
  if (cfg.resident_config < 0 || cfg.resident_config > eb::block_config_count())
    return fail(EB_ERR_INVALID_ARGUMENT, "resident_config out of range");
  if (cfg.step_window != 0 && cfg.step_window != 64 && cfg.step_window != 96 && cfg.step_window != 128 &&
      cfg.step_window != 256)
    return fail(EB_ERR_INVALID_ARGUMENT, "step_window must be 0 (default), 64, 96, 128 or 256");
  if (cfg.precision == EB_PRECISION_MIXED && (cfg.flags & (EB_FLAG_REFERENCE_ROUNDING | EB_FLAG_STEP_STREAMING)))
    return fail(EB_ERR_INVALID_ARGUMENT, "mixed precision runs on the resident kernels only");
  if (cfg.stepper != EB_STEPPER_POSITION_VERLET && cfg.stepper != EB_STEPPER_PEFRL &&
      cfg.stepper != EB_STEPPER_VELOCITY_VERLET)
    return fail(EB_ERR_INVALID_ARGUMENT, "unknown time stepper");
  if (cfg.stepper != EB_STEPPER_POSITION_VERLET && cfg.precision == EB_PRECISION_MIXED)
    return fail(EB_ERR_UNSUPPORTED, "PEFRL and VelocityVerlet run in FP64 only");
  if (cfg.flags & ~static_cast<uint32_t>(EB_FLAG_RECORD_DIAGNOSTICS | EB_FLAG_REFERENCE_ROUNDING |
                                          EB_FLAG_STEP_STREAMING | EB_FLAG_STEP_RESIDENT | EB_FLAG_CUDA_GRAPH |
                                          EB_FLAG_STEP_BUCKETED))
    return fail(EB_ERR_INVALID_ARGUMENT, "unknown flag");
  int ndev = 0;
  EB_CUDA(cudaGetDeviceCount(&ndev));
  if (cfg.device < 0 || cfg.device >= ndev) return fail(EB_ERR_INVALID_ARGUMENT, "no such CUDA device");
  eb_sim* s = new eb_sim();
  s->cfg = cfg;
  cudaError_t e = cudaSetDevice(cfg.device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete s;
    return fail(EB_ERR_CUDA, std::string("stream creation: ") + cudaGetErrorString(e));
  }
  *out = s;
  return EB_OK;
}

EB_API eb_status eb_sim_destroy(eb_sim* s) {
  if (!s) return EB_OK;
  cudaSetDevice(s->cfg.device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (cudaStream_t x : s->xs)
    if (x) cudaStreamSynchronize(x);
  host_free(s);
  for (cudaEvent_t e : s->xev) cudaEventDestroy(e);
  for (cudaStream_t x : s->xs)
    if (x) cudaStreamDestroy(x);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return EB_OK;
}

EB_API eb_status eb_emplace_straight_rods(eb_sim* s, const eb_straight_rod* rods, int64_t count,
                                          int64_t* ids_out) {
  if (check_sim(s)) return EB_ERR_INVALID_ARGUMENT;
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "cannot add rods after finalize");
  if (count < 0 || (count > 0 && !rods)) return fail(EB_ERR_INVALID_ARGUMENT, "bad rod array");
  std::vector<RodHost> made(static_cast<size_t>(count));
  for (int64_t i = 0; i < count; ++i) {
    const eb_status st = init_straight_rod(rods[i], made[i]);
    if (st != EB_OK) return st;
  }
  const int64_t first = static_cast<int64_t>(s->rods.size());
  if (first + count >= (int64_t(1) << (32 - eb::kRodShift)))
    return fail(EB_ERR_UNSUPPORTED, "too many rods in one simulator");
  for (auto& r : made) {
    if (r.model == EB_ROD_DAMPED) s->any_damped = true;
    s->rods.push_back(std::move(r));
  }
  if (ids_out)
    for (int64_t i = 0; i < count; ++i) ids_out[i] = first + i;
  return EB_OK;
}

EB_API eb_status eb_rod_count(const eb_sim* s, int64_t* count) {
  if (check_sim(s) || !count) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  *count = static_cast<int64_t>(s->rods.size());
  return EB_OK;
}

EB_API eb_status eb_rod_elements(const eb_sim* s, int64_t rod, int64_t* n) {
  if (check_sim(s) || !n) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (rod < 0 || rod >= static_cast<int64_t>(s->rods.size())) return fail(EB_ERR_NOT_FOUND, "unknown rod id");
  *n = s->rods[rod].n;
  return EB_OK;
}

EB_API eb_status eb_slot_count(const eb_sim* s, int64_t* n_slots) {
  if (check_sim(s) || !n_slots) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  int64_t total = 0;
  for (const auto& r : s->rods) total += r.n + 1;
  *n_slots = total;
  return EB_OK;
}

EB_API eb_status eb_slot_offsets(const eb_sim* s, int64_t* offsets_out, int64_t count) {
  if (check_sim(s) || !offsets_out) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (count != static_cast<int64_t>(s->rods.size()) + 1)
    return fail(EB_ERR_INVALID_ARGUMENT, "offsets need rod_count + 1 entries");
  int64_t total = 0;
  for (size_t r = 0; r < s->rods.size(); ++r) {
    offsets_out[r] = total;
    total += s->rods[r].n + 1;
  }
  offsets_out[s->rods.size()] = total;
  return EB_OK;
}

EB_API eb_status eb_field_size(const eb_sim* s, int64_t rod, int32_t field, int64_t* count) {
  if (check_sim(s) || !count) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (field < 0 || field >= EB_FIELD_COUNT) return fail(EB_ERR_INVALID_ARGUMENT, "unknown field");
  if (rod < 0 || rod >= static_cast<int64_t>(s->rods.size())) return fail(EB_ERR_NOT_FOUND, "unknown rod id");
  *count = kFields[field].ncomp * place_count(kFields[field].place, s->rods[rod].n);
  return EB_OK;
}

EB_API eb_status eb_set_field(eb_sim* s, int64_t rod, int32_t field, const double* values, int64_t count) {
  if (check_sim(s) || !values) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  const FieldInfo* fi;
  int64_t expected;
  if (eb_status st = rod_field_check(s, rod, field, count, &fi, &expected)) return st;
  RodHost& r = s->rods[rod];
  const int64_t per = place_count(fi->place, r.n);
  if (fi->kind == kContactLoad) return fail(EB_ERR_UNSUPPORTED, "contact loads are read only");
  if (!s->finalized) {
    std::vector<double>& buf = fi->kind == kState ? r.state : (fi->kind == kParam ? r.param : r.diag);
    for (int c = 0; c < fi->ncomp; ++c)
      std::memcpy(&buf[static_cast<size_t>((fi->offset + c) * (r.n + 1))], values + c * per,
                  static_cast<size_t>(per) * sizeof(double));
    return EB_OK;
  }
  if (eb_status st = set_device(s)) return st;
  double* base = device_base(s, *fi);
  if (!base) return fail(EB_ERR_UNSUPPORTED, "derived fields need EB_FLAG_RECORD_DIAGNOSTICS");
  EB_CUDA(cudaMemcpy2DAsync(base + s->offsets[rod], s->stride * sizeof(double), values,
                            per * sizeof(double), per * sizeof(double), fi->ncomp,
                            cudaMemcpyHostToDevice, s->stream));
  if (fi->kind == kState) {
    // keep the other ping-pong buffer consistent for the unused slot entries
    double* other = s->d_state[s->cur ^ 1] + static_cast<int64_t>(fi->offset) * s->stride;
    EB_CUDA(cudaMemcpy2DAsync(other + s->offsets[rod], s->stride * sizeof(double), base + s->offsets[rod],
                              s->stride * sizeof(double), per * sizeof(double), fi->ncomp,
                              cudaMemcpyDeviceToDevice, s->stream));
  }
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return EB_OK;
}

EB_API eb_status eb_get_field(eb_sim* s, int64_t rod, int32_t field, double* values, int64_t count) {
  if (check_sim(s) || !values) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  const FieldInfo* fi;
  int64_t expected;
  if (eb_status st = rod_field_check(s, rod, field, count, &fi, &expected)) return st;
  const RodHost& r = s->rods[rod];
  const int64_t per = place_count(fi->place, r.n);
  if (fi->kind == kContactLoad && !s->finalized)
    return fail(EB_ERR_INVALID_STATE, "contact loads exist after eb_finalize");
  if (!s->finalized) {
    const std::vector<double>& buf = fi->kind == kState ? r.state : (fi->kind == kParam ? r.param : r.diag);
    for (int c = 0; c < fi->ncomp; ++c)
      std::memcpy(values + c * per, &buf[static_cast<size_t>((fi->offset + c) * (r.n + 1))],
                  static_cast<size_t>(per) * sizeof(double));
    return EB_OK;
  }
  if (eb_status st = set_device(s)) return st;
  double* base = device_base(s, *fi);
  if (!base)
    return fail(EB_ERR_UNSUPPORTED, fi->kind == kContactLoad ? "no rod takes part in contact"
                                                              : "derived fields need EB_FLAG_RECORD_DIAGNOSTICS");
  EB_CUDA(cudaMemcpy2DAsync(values, per * sizeof(double), base + s->offsets[rod],
                            s->stride * sizeof(double), per * sizeof(double), fi->ncomp,
                            cudaMemcpyDeviceToHost, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_status(s);
}

static eb_status batch_copy(eb_sim* s, int32_t field, int32_t layout, double* host, int64_t count,
                            bool to_device) {
  if (check_sim(s) || !host) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (!s->finalized) return fail(EB_ERR_INVALID_STATE, "batch access needs a finalized simulator");
  if (field < 0 || field >= EB_FIELD_COUNT) return fail(EB_ERR_INVALID_ARGUMENT, "unknown field");
  const FieldInfo& fi = kFields[field];
  if (fi.kind == kContactLoad && to_device) return fail(EB_ERR_UNSUPPORTED, "contact loads are read only");
  if (eb_status st = set_device(s)) return st;
  double* base = device_base(s, fi);
  if (!base) return fail(EB_ERR_UNSUPPORTED, "derived fields need EB_FLAG_RECORD_DIAGNOSTICS");
  const size_t pitch = static_cast<size_t>(s->stride) * sizeof(double);
  if (layout == EB_LAYOUT_SLOTS) {
    if (count != fi.ncomp * s->n_slots)
      return fail(EB_ERR_INVALID_ARGUMENT, "slot layout needs ncomp * slot_count values");
    const size_t w = static_cast<size_t>(s->n_slots) * sizeof(double);
    if (to_device) {
      EB_CUDA(cudaMemcpy2DAsync(base, pitch, host, w, w, fi.ncomp, cudaMemcpyHostToDevice, s->stream));
      if (fi.kind == kState) {
        // the other ping-pong buffer gets the same values on the device (its
        // entries that no step writes must match), not by a second upload
        double* other = s->d_state[s->cur ^ 1] + static_cast<int64_t>(fi.offset) * s->stride;
        EB_CUDA(cudaMemcpy2DAsync(other, pitch, base, pitch, w, fi.ncomp, cudaMemcpyDeviceToDevice, s->stream));
      }
    } else {
      EB_CUDA(cudaMemcpy2DAsync(host, w, base, pitch, w, fi.ncomp, cudaMemcpyDeviceToHost, s->stream));
    }
    EB_CUDA(cudaStreamSynchronize(s->stream));
    return to_device ? EB_OK : check_device_status(s);
  }
  if (layout != EB_LAYOUT_PER_ROD) return fail(EB_ERR_INVALID_ARGUMENT, "unknown layout");
  int64_t total = 0;
  for (const auto& r : s->rods) total += fi.ncomp * place_count(fi.place, r.n);
  if (count != total) return fail(EB_ERR_INVALID_ARGUMENT, "per-rod layout count mismatch");
  // stage through the slot layout; start from the device contents so the
  // unused slot entries keep their values
  std::vector<double> tmp(static_cast<size_t>(fi.ncomp * s->n_slots), 0.0);
  const size_t w = static_cast<size_t>(s->n_slots) * sizeof(double);
  EB_CUDA(cudaMemcpy2DAsync(tmp.data(), w, base, pitch, w, fi.ncomp, cudaMemcpyDeviceToHost, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  int64_t pos = 0;
  for (size_t r = 0; r < s->rods.size(); ++r) {
    const int64_t per = place_count(fi.place, s->rods[r].n);
    for (int c = 0; c < fi.ncomp; ++c) {
      double* slot = tmp.data() + c * s->n_slots + s->offsets[r];
      if (to_device)
        std::memcpy(slot, host + pos, static_cast<size_t>(per) * sizeof(double));
      else
        std::memcpy(host + pos, slot, static_cast<size_t>(per) * sizeof(double));
      pos += per;
    }
  }
  if (!to_device) return EB_OK;
  EB_CUDA(cudaMemcpy2DAsync(base, pitch, tmp.data(), w, w, fi.ncomp, cudaMemcpyHostToDevice, s->stream));
  if (fi.kind == kState) {
    double* other = s->d_state[s->cur ^ 1] + static_cast<int64_t>(fi.offset) * s->stride;
    EB_CUDA(cudaMemcpy2DAsync(other, pitch, base, pitch, w, fi.ncomp, cudaMemcpyDeviceToDevice, s->stream));
  }
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return EB_OK;
}

EB_API eb_status eb_set_field_batch(eb_sim* s, int32_t field, int32_t layout, const double* values,
                                    int64_t count) {
  return batch_copy(s, field, layout, const_cast<double*>(values), count, true);
}

EB_API eb_status eb_get_field_batch(eb_sim* s, int32_t field, int32_t layout, double* values,
                                    int64_t count) {
  return batch_copy(s, field, layout, values, count, false);
}

EB_API eb_status eb_constrain_clamp(eb_sim* s, int64_t rod, int64_t index) {
  if (check_sim(s)) return EB_ERR_INVALID_ARGUMENT;
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "cannot add constraints after finalize");
  if (rod < 0 || rod >= static_cast<int64_t>(s->rods.size())) return fail(EB_ERR_NOT_FOUND, "unknown rod id");
  RodHost& r = s->rods[rod];
  if (index < 0 || index > r.n) return fail(EB_ERR_INVALID_ARGUMENT, "clamp index must name a node of the rod");
  if (index == r.clamp_index[0] || index == r.clamp_index[1])
    return fail(EB_ERR_INVALID_STATE, "this index of the rod is clamped already");
  const int c = r.clamp_index[0] < 0 ? 0 : (r.clamp_index[1] < 0 ? 1 : -1);
  if (c < 0) return fail(EB_ERR_UNSUPPORTED, "at most two clamps per rod");
  // targets: the node's position and the element's directors now (the
  // reference's generator captures them when it is built)
  const int64_t W = r.n + 1;
  double* tx = c == 0 ? r.info.clamp_x : r.info.clamp2_x;
  double* tq = c == 0 ? r.info.clamp_Q : r.info.clamp2_Q;
  const int64_t e = index < r.n ? index : r.n - 1;  // a clamp at node n fixes no element
  for (int d = 0; d < 3; ++d) tx[d] = r.state[static_cast<size_t>((eb::kStX + d) * W + index)];
  for (int k = 0; k < 9; ++k) tq[k] = r.state[static_cast<size_t>((eb::kStQ + k) * W + e)];
  r.clamp_index[c] = index;
  r.info.flags |= eb::kRodClamp;
  s->sim_flags |= eb::kSimClamp;
  return EB_OK;
}

EB_API eb_status eb_add_gravity(eb_sim* s, const double gravity[3]) {
  if (check_sim(s) || !gravity) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "cannot add environments after finalize");
  if (s->has_gravity) return fail(EB_ERR_INVALID_STATE, "the gravity field is a singleton environment");
  for (int d = 0; d < 3; ++d) s->gravity[d] = gravity[d];
  s->has_gravity = true;
  s->sim_flags |= eb::kSimGravity;
  return EB_OK;
}

EB_API eb_status eb_add_element_torque(eb_sim* s, int64_t rod, int64_t element, const double torque_lab[3]) {
  if (check_sim(s) || !torque_lab) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "cannot add forcing after finalize");
  if (rod < 0 || rod >= static_cast<int64_t>(s->rods.size())) return fail(EB_ERR_NOT_FOUND, "unknown rod id");
  RodHost& r = s->rods[rod];
  if (element < 0 || element >= r.n) return fail(EB_ERR_INVALID_ARGUMENT, "element index out of range");
  if (r.torque_index >= 0 && r.torque_index != element)
    return fail(EB_ERR_UNSUPPORTED, "the torques of a rod act on one element");
  for (int d = 0; d < 3; ++d) r.info.end_torque[d] += torque_lab[d];
  r.torque_index = element;
  r.info.flags |= eb::kRodEndTorque;
  s->sim_flags |= eb::kSimEndTorque;
  return EB_OK;
}

EB_API eb_status eb_add_end_torque(eb_sim* s, int64_t rod, const double torque_lab[3]) {
  if (check_sim(s)) return EB_ERR_INVALID_ARGUMENT;
  if (rod < 0 || rod >= static_cast<int64_t>(s->rods.size())) return fail(EB_ERR_NOT_FOUND, "unknown rod id");
  return eb_add_element_torque(s, rod, s->rods[rod].n - 1, torque_lab);
}

EB_API eb_status eb_add_analytical_damper(eb_sim* s, int64_t rod, double translational_rate,
                                          double rotational_rate) {
  if (check_sim(s)) return EB_ERR_INVALID_ARGUMENT;
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "cannot add constraints after finalize");
  if (rod < 0 || rod >= static_cast<int64_t>(s->rods.size())) return fail(EB_ERR_NOT_FOUND, "unknown rod id");
  if (!(translational_rate >= 0.0) || !(rotational_rate >= 0.0))
    return fail(EB_ERR_INVALID_ARGUMENT, "damping rates must be non-negative");
  RodHost& r = s->rods[rod];
  if (r.info.flags & eb::kRodDamper) return fail(EB_ERR_INVALID_STATE, "rod already has a damper");
  r.damper_nu_t = translational_rate;
  r.info.damper_r = rotational_rate;
  r.info.flags |= eb::kRodDamper;
  s->sim_flags |= eb::kSimDamper;
  return EB_OK;
}

EB_API eb_status eb_add_contact_material(eb_sim* s, const eb_contact_material* m, int32_t* material_id) {
  if (check_sim(s) || !m) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "cannot add materials after finalize");
  // Materials.cpp:237-283 argument checks
  if (!(m->stiffness > 0.0) || !std::isfinite(m->stiffness)) return fail(EB_ERR_INVALID_ARGUMENT, "Invalid stiffness");
  if (!(m->normal_damping >= 0.0) || !(m->tangential_damping >= 0.0) || !std::isfinite(m->normal_damping) ||
      !std::isfinite(m->tangential_damping))
    return fail(EB_ERR_INVALID_ARGUMENT, "Invalid damping coefficients");
  if (!(m->static_friction >= 0.0) || !(m->dynamic_friction >= 0.0) || !std::isfinite(m->static_friction) ||
      !std::isfinite(m->dynamic_friction))
    return fail(EB_ERR_INVALID_ARGUMENT, "Invalid coefficient of friction");
  if (s->materials.size() >= 4096) return fail(EB_ERR_UNSUPPORTED, "too many contact materials");
  s->materials.push_back(*m);
  if (material_id) *material_id = static_cast<int32_t>(s->materials.size() - 1);
  return EB_OK;
}

EB_API eb_status eb_add_rod_contact(eb_sim* s, int64_t rod, int32_t material_id) {
  if (check_sim(s)) return EB_ERR_INVALID_ARGUMENT;
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "cannot add contact after finalize");
  if (rod < 0 || rod >= static_cast<int64_t>(s->rods.size())) return fail(EB_ERR_NOT_FOUND, "unknown rod id");
  if (material_id < 0 || material_id >= static_cast<int32_t>(s->materials.size()))
    return fail(EB_ERR_NOT_FOUND, "unknown contact material");
  s->rods[rod].contact_material = material_id;
  return EB_OK;
}

EB_API eb_status eb_add_contact_plane(eb_sim* s, const double point[3], const double normal[3],
                                      int32_t material_id) {
  if (check_sim(s) || !point || !normal) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "cannot add planes after finalize");
  if (material_id < 0 || material_id >= static_cast<int32_t>(s->materials.size()))
    return fail(EB_ERR_NOT_FOUND, "unknown contact material");
  for (int d = 0; d < 3; ++d)
    if (!std::isfinite(point[d]) || !std::isfinite(normal[d]))
      return fail(EB_ERR_INVALID_ARGUMENT, "plane point and normal must be finite");
  if (normal[0] == 0.0 && normal[1] == 0.0 && normal[2] == 0.0)
    return fail(EB_ERR_INVALID_ARGUMENT, "zero plane normal");
  if (s->planes.size() >= 4096) return fail(EB_ERR_UNSUPPORTED, "too many planes");
  s->planes.push_back(make_plane(point, normal, material_id));
  return EB_OK;
}

namespace {

// Device tables of the connections: one entry per joint and, per loaded
// slot, the joints acting on it in connection order (rod a's share first).
eb_status setup_joints(eb_sim* s) {
  JointDevice& j = s->jd;
  if (s->joints.empty()) return EB_OK;
  const int64_t S = s->stride;
  std::vector<eb::JointDev> dev;
  std::map<int64_t, std::vector<int32_t>> fsrc, tsrc;
  for (size_t c = 0; c < s->joints.size(); ++c) {
    const JointHost& h = s->joints[c];
    eb::JointDev d{};
    d.node_a = s->offsets[h.rod_a] + h.index_a + 1;
    d.node_b = s->offsets[h.rod_b] + h.index_b;
    d.kind = h.joint.kind == EB_JOINT_HINGE ? eb::kJointHinge : eb::kJointFree;
    d.k = h.joint.stiffness;
    d.nu = h.joint.damping;
    d.k_rot = h.joint.rotational_stiffness;
    for (int k = 0; k < 3; ++k) d.normal[k] = h.joint.normal[k];
    dev.push_back(d);
    const int32_t id = static_cast<int32_t>(2 * c);
    fsrc[d.node_a].push_back(id);
    fsrc[d.node_b].push_back(id | 1);
    if (d.kind == eb::kJointHinge) {
      tsrc[s->offsets[h.rod_a] + h.index_a].push_back(id | 1);
      tsrc[d.node_b].push_back(id);
    }
  }
  auto csr = [](const std::map<int64_t, std::vector<int32_t>>& m, std::vector<int64_t>& slot,
                std::vector<int64_t>& off, std::vector<int32_t>& src) {
    off.push_back(0);
    for (const auto& kv : m) {
      slot.push_back(kv.first);
      src.insert(src.end(), kv.second.begin(), kv.second.end());
      off.push_back(static_cast<int64_t>(src.size()));
    }
  };
  std::vector<int64_t> fslot, foff, tslot, toff;
  std::vector<int32_t> fs, ts;
  csr(fsrc, fslot, foff, fs);
  csr(tsrc, tslot, toff, ts);
  auto up = [&](auto** p, const auto& v) -> cudaError_t {
    const size_t bytes = std::max<size_t>(1, v.size()) * sizeof(v[0]);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    if (e == cudaSuccess && !v.empty())
      e = cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice, s->stream);
    return e;
  };
  EB_CUDA(up(&j.joints, dev));
  EB_CUDA(up(&j.force_slot, fslot));
  EB_CUDA(up(&j.force_off, foff));
  EB_CUDA(up(&j.force_src, fs));
  EB_CUDA(up(&j.torque_slot, tslot));
  EB_CUDA(up(&j.torque_off, toff));
  EB_CUDA(up(&j.torque_src, ts));
  EB_CUDA(cudaMalloc(reinterpret_cast<void**>(&j.out), dev.size() * 6 * sizeof(double)));
  EB_CUDA(cudaMalloc(reinterpret_cast<void**>(&j.loads), static_cast<size_t>(6 * S) * sizeof(double)));
  EB_CUDA(cudaMemsetAsync(j.loads, 0, static_cast<size_t>(6 * S) * sizeof(double), s->stream));
  j.n_force = static_cast<int64_t>(fslot.size());
  j.n_torque = static_cast<int64_t>(tslot.size());
  j.on = true;
  return EB_OK;
}

eb::JointArgs joint_args(eb_sim* s) {
  const JointDevice& j = s->jd;
  eb::JointArgs a{};
  a.n_joints = static_cast<int32_t>(s->joints.size());
  a.joints = j.joints;
  a.out = j.out;
  a.stride = s->stride;
  a.meta = s->d_meta;
  a.rods = s->d_rods;
  a.n_force_slots = j.n_force;
  a.force_slot = j.force_slot;
  a.force_off = j.force_off;
  a.force_src = j.force_src;
  a.n_torque_slots = j.n_torque;
  a.torque_slot = j.torque_slot;
  a.torque_off = j.torque_off;
  a.torque_src = j.torque_src;
  a.joint_force = j.loads;
  a.joint_torque = j.loads + 3 * s->stride;
  return a;
}

}  // namespace

EB_API eb_status eb_connect(eb_sim* s, int64_t rod_a, int64_t index_a, int64_t rod_b, int64_t index_b,
                            const eb_joint* joint) {
  if (check_sim(s) || !joint) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "cannot add connections after finalize");
  const int64_t nr = static_cast<int64_t>(s->rods.size());
  if (rod_a < 0 || rod_a >= nr || rod_b < 0 || rod_b >= nr) return fail(EB_ERR_NOT_FOUND, "unknown rod");
  if (joint->kind != EB_JOINT_FREE && joint->kind != EB_JOINT_HINGE)
    return fail(EB_ERR_INVALID_ARGUMENT, "unknown joint kind");
  const int64_t na = s->rods[rod_a].n, nb = s->rods[rod_b].n;
  // force on node index_a + 1 of rod a and node index_b of rod b; the hinge
  // also loads element index_a of rod a and element index_b of rod b
  if (index_a < 0 || index_a >= na) return fail(EB_ERR_INVALID_ARGUMENT, "index_a must name an element of rod a");
  if (index_b < 0 || index_b > nb || (joint->kind == EB_JOINT_HINGE && index_b >= nb))
    return fail(EB_ERR_INVALID_ARGUMENT, "index_b must name a node (an element for a hinge) of rod b");
  const double vals[] = {joint->stiffness, joint->damping, joint->rotational_stiffness, joint->normal[0],
                         joint->normal[1], joint->normal[2]};
  for (double v : vals)
    if (!std::isfinite(v)) return fail(EB_ERR_INVALID_ARGUMENT, "joint parameters must be finite");
  if (s->joints.size() >= (size_t(1) << 30)) return fail(EB_ERR_UNSUPPORTED, "too many connections");
  s->joints.push_back({rod_a, index_a, rod_b, index_b, *joint});
  return EB_OK;
}

EB_API eb_status eb_finalize(eb_sim* s) {
  if (check_sim(s)) return EB_ERR_INVALID_ARGUMENT;
  if (s->finalized) return fail(EB_ERR_INVALID_STATE, "already finalized");
  if (s->rods.empty()) return fail(EB_ERR_INVALID_STATE, "no rods");
  if (eb_status st = set_device(s)) return st;
  const int64_t nr = static_cast<int64_t>(s->rods.size());
  s->offsets.assign(static_cast<size_t>(nr + 1), 0);
  for (int64_t r = 0; r < nr; ++r) s->offsets[r + 1] = s->offsets[r] + s->rods[r].n + 1;
  s->n_slots = s->offsets[nr];
  s->stride = (s->n_slots + 31) / 32 * 32;
  const int64_t S = s->stride;
  const bool want_diag = (s->cfg.flags & EB_FLAG_RECORD_DIAGNOSTICS) != 0;

  std::vector<double> hs(static_cast<size_t>(eb::kStateFields * S), 0.0);
  std::vector<double> hp(static_cast<size_t>(eb::kParamFields * S), 0.0);
  std::vector<double> hd;
  if (want_diag) hd.assign(static_cast<size_t>(eb::kDiagFields * S), 0.0);
  std::vector<uint32_t> meta(static_cast<size_t>(S), 0u);
  for (int64_t r = 0; r < nr; ++r) {
    const RodHost& R = s->rods[r];
    const int64_t W = R.n + 1, o = s->offsets[r];
    for (int f = 0; f < eb::kStateFields; ++f)
      std::memcpy(&hs[static_cast<size_t>(f * S + o)], &R.state[static_cast<size_t>(f * W)], W * sizeof(double));
    for (int f = 0; f < eb::kParamFields; ++f)
      std::memcpy(&hp[static_cast<size_t>(f * S + o)], &R.param[static_cast<size_t>(f * W)], W * sizeof(double));
    if (want_diag)
      for (int f = 0; f < eb::kDiagFields; ++f)
        std::memcpy(&hd[static_cast<size_t>(f * S + o)], &R.diag[static_cast<size_t>(f * W)], W * sizeof(double));
    for (int64_t j = 0; j <= R.n; ++j) {
      uint32_t m = static_cast<uint32_t>(r) << eb::kRodShift;
      if (j < R.n) m |= eb::kElem;
      if (j < R.n - 1) m |= eb::kVor;
      if (j == 0) m |= eb::kFirst;
      if (j == R.n) m |= eb::kLastNode;
      if (j == R.n - 1) m |= eb::kLastElem;
      meta[static_cast<size_t>(o + j)] = m;
    }
  }
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  alloc(reinterpret_cast<void**>(&s->d_state[0]), hs.size() * sizeof(double));
  alloc(reinterpret_cast<void**>(&s->d_state[1]), hs.size() * sizeof(double));
  alloc(reinterpret_cast<void**>(&s->d_param), hp.size() * sizeof(double));
  if (want_diag) alloc(reinterpret_cast<void**>(&s->d_diag), hd.size() * sizeof(double));
  alloc(reinterpret_cast<void**>(&s->d_meta), meta.size() * sizeof(uint32_t));
  alloc(reinterpret_cast<void**>(&s->d_rods), static_cast<size_t>(nr) * sizeof(eb::RodInfo));
  alloc(reinterpret_cast<void**>(&s->d_offsets), static_cast<size_t>(nr + 1) * sizeof(int64_t));
  alloc(reinterpret_cast<void**>(&s->d_energy), static_cast<size_t>(4 * nr) * sizeof(double));
  alloc(reinterpret_cast<void**>(&s->d_status), sizeof(uint32_t));
  if (e != cudaSuccess) {
    host_free(s);
    return fail(e == cudaErrorMemoryAllocation ? EB_ERR_OUT_OF_MEMORY : EB_ERR_CUDA,
                std::string("device allocation: ") + cudaGetErrorString(e));
  }
  EB_CUDA(cudaMemcpyAsync(s->d_state[0], hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaMemcpyAsync(s->d_state[1], hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaMemcpyAsync(s->d_param, hp.data(), hp.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  if (want_diag)
    EB_CUDA(cudaMemcpyAsync(s->d_diag, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaMemcpyAsync(s->d_meta, meta.data(), meta.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaMemcpyAsync(s->d_offsets, s->offsets.data(), s->offsets.size() * sizeof(int64_t),
                          cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(uint32_t), s->stream));
  s->cur = 0;
  if (eb_status st = setup_contact(s)) {
    host_free(s);
    return st;
  }
  if (eb_status st = setup_joints(s)) {
    host_free(s);
    return st;
  }
  s->finalized = true;
  if (eb_status st = upload_rod_table(s)) return st;
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return EB_OK;
}

namespace {

constexpr int kResidentChunk = 128;  // steps per launch of the resident kernel
constexpr int kProbeSteps = 8;       // steps per timing probe of the planner

eb::StepArgs step_args(eb_sim* s, double dt) {
  eb::StepArgs a{};
  a.stride = s->stride;
  a.n_slots = s->n_slots;
  a.par = s->d_param;
  a.meta = s->d_meta;
  a.rods = s->d_rods;
  a.dt = dt;
  a.half_dt = 0.5 * dt;
  a.drift_pre = 0.5 * dt;
  a.kick = dt;
  a.drift_post = 0.5 * dt;
  a.damper_time = dt;
  for (int d = 0; d < 3; ++d) a.gravity[d] = s->gravity[d];
  a.sim_flags = s->sim_flags;
  a.status = s->d_status;
  a.max_polls = s->max_polls;
  return a;
}

// the clock after n steps: PositionVerlet takes two TimeUpdate substeps of
// dt/2 a step (PositionVerlet.hpp:52-58), VelocityVerlet one of dt
// (VelocityVerlet.hpp:61-67)
void advance_time(const eb_sim* s, double* time, double dt, int64_t n_steps) {
  if (!time) return;
  for (int64_t k = 0; k < n_steps; ++k) {
    if (s->cfg.stepper == EB_STEPPER_VELOCITY_VERLET) {
      *time += dt;
    } else {
      *time += 0.5 * dt;
      *time += 0.5 * dt;
    }
  }
}

void drop_graphs(eb_sim* s) {
  for (int p = 0; p < 2; ++p)
    if (s->graph[p]) {
      cudaGraphExecDestroy(s->graph[p]);
      s->graph[p] = nullptr;
    }
}


cudaError_t launch_streaming(eb_sim* s, eb::StepArgs& a, bool rec) {
  a.diag = rec ? s->d_diag : nullptr;
  const int window = s->cfg.step_window;  // 0: the persistent kernel
  if (s->cfg.flags & EB_FLAG_REFERENCE_ROUNDING)
    return eb::launch_rod_step_fp64_reference(a, rec, s->any_damped, window, s->stream);
  return eb::launch_rod_step_fp64(a, rec, s->any_damped, window, s->stream);
}

cudaError_t launch_resident(eb_sim* s, eb::StepArgs& a, int config, int steps) {
  if (s->cfg.precision == EB_PRECISION_MIXED)
    return eb::launch_rod_block_mixed_gather(a, s->d_cta_start[config], s->d_gmap[config], s->n_ctas[config], steps,
                                             config, s->any_damped, s->stream);
  return eb::launch_rod_block_fp64_gather(a, s->d_cta_start[config], s->d_gmap[config], s->n_ctas[config], steps,
                                          config, s->any_damped, s->stream);
}

// Pack rods into CTAs of configuration c, best fit decreasing: rods in order
// of decreasing length (ties in rod order), each into the CTA with the least
// room that still holds it, else into a new CTA.  CTAs are filled up to a
// whole number of rounds of the configuration's threads (512 slots with 512
// or 256 threads, 256 with 256, 264 with 288): one slot more would give some
// threads an extra round in every phase.  A rod longer than that gets a CTA
// of its own (up to the configuration's capacity).  off/map: CTA c owns the
// slots map[off[c] .. off[c + 1]), each rod's slots consecutive (its rods in
// slot order).  Best fit fills the CTAs of the 16,384-rod uneven batch to
// 99% against 75% for next fit in rod order, so a launch holds a quarter
// fewer CTAs.  Returns false when a rod is longer than the capacity.
int64_t pack_fill(int config) {
  const int64_t cap = eb::block_config_capacity(config), threads = eb::block_config_threads(config);
  return cap <= threads ? cap : cap / threads * threads;
}

bool pack_best_fit(const eb_sim* s, const std::vector<size_t>& rods, int config, std::vector<int64_t>& off,
                   std::vector<int32_t>& map) {
  const int64_t cap = eb::block_config_capacity(config), fill = pack_fill(config);
  std::vector<size_t> order(rods);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return s->rods[a].n > s->rods[b].n; });
  std::vector<std::vector<size_t>> cta;
  std::multimap<int64_t, size_t> room;  // free slots -> CTA
  for (size_t r : order) {
    const int64_t w = s->rods[r].n + 1;
    if (w > cap) return false;
    auto it = w <= fill ? room.lower_bound(w) : room.end();
    size_t c;
    int64_t left;
    if (it != room.end()) {
      c = it->second;
      left = it->first - w;
      room.erase(it);
    } else {
      c = cta.size();
      cta.emplace_back();
      left = w <= fill ? fill - w : 0;
    }
    cta[c].push_back(r);
    if (left >= 3) room.emplace(left, c);  // a rod takes at least 3 slots
  }
  off.assign(1, 0);
  map.clear();
  for (auto& list : cta) {
    std::sort(list.begin(), list.end());
    for (size_t r : list)
      for (int64_t j = 0; j <= s->rods[r].n; ++j) map.push_back(static_cast<int32_t>(s->offsets[r] + j));
    off.push_back(static_cast<int64_t>(map.size()));
  }
  return true;
}

eb_status build_block_worklists(eb_sim* s) {
  if (!s->d_cta_start.empty()) return EB_OK;
  const int nc = eb::block_config_count();
  s->d_cta_start.assign(static_cast<size_t>(nc), nullptr);
  s->d_gmap.assign(static_cast<size_t>(nc), nullptr);
  s->n_ctas.assign(static_cast<size_t>(nc), 0);
  if (s->n_slots > INT32_MAX) return EB_OK;  // the slot lists hold 32-bit slot indices: streaming only
  std::vector<size_t> all(s->rods.size());
  for (size_t r = 0; r < all.size(); ++r) all[r] = r;
  std::vector<int64_t> off;
  std::vector<int32_t> map;
  for (int c = 0; c < nc; ++c) {
    const int64_t cap = eb::block_config_capacity(c);
    int same = -1;  // an earlier configuration packed the same way
    for (int k = 0; k < c; ++k)
      if (eb::block_config_capacity(k) == cap && pack_fill(k) == pack_fill(c)) same = k;
    if (same >= 0) {
      s->d_cta_start[c] = s->d_cta_start[same];
      s->d_gmap[c] = s->d_gmap[same];
      s->n_ctas[c] = s->n_ctas[same];
      continue;
    }
    if (!pack_best_fit(s, all, c, off, map)) continue;
    EB_CUDA(cudaMalloc(reinterpret_cast<void**>(&s->d_cta_start[c]), off.size() * sizeof(int64_t)));
    EB_CUDA(cudaMalloc(reinterpret_cast<void**>(&s->d_gmap[c]), map.size() * sizeof(int32_t)));
    EB_CUDA(cudaMemcpyAsync(s->d_cta_start[c], off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                            s->stream));
    EB_CUDA(cudaMemcpyAsync(s->d_gmap[c], map.data(), map.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                            s->stream));
    s->n_ctas[c] = static_cast<int>(off.size() - 1);
  }
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return EB_OK;
}

// Substeps of one step as (drift before, kick, drift after, damper time) in
// units of dt: PositionVerlet (PositionVerlet.hpp:49-88) fuses its two half
// drifts around one kick; VelocityVerlet (VelocityVerlet.hpp:49-87) kicks by
// 1/2, drifts by 1, kicks by 1/2, with the damper's full-dt factors after
// each kick; PEFRL (Omelyan, Mryglod and Folk 2002) is four kicks with the
// drifts xi, chi, 1 - 2 (chi + xi), chi, xi between them and the damper's
// factors for each kick's share of dt.
struct Substep {
  double pre, kick, post, damper;
};
using eb::kPefrlChi;
using eb::kPefrlLambda;
using eb::kPefrlXi;
const Substep kVerlet[1] = {{0.5, 1.0, 0.5, 1.0}};
const Substep kVelocityVerlet[2] = {{0.0, 0.5, 1.0, 1.0}, {0.0, 0.5, 0.0, 1.0}};
const Substep kPefrl[4] = {{kPefrlXi, 0.5 * (1.0 - 2.0 * kPefrlLambda), 0.0, 0.5 * (1.0 - 2.0 * kPefrlLambda)},
                           {kPefrlChi, kPefrlLambda, 0.0, kPefrlLambda},
                           {1.0 - 2.0 * (kPefrlChi + kPefrlXi), kPefrlLambda, 0.0, kPefrlLambda},
                           {kPefrlChi, 0.5 * (1.0 - 2.0 * kPefrlLambda), kPefrlXi, 0.5 * (1.0 - 2.0 * kPefrlLambda)}};

int substeps(const eb_sim* s, const Substep** table);

// the stepper's force evaluations per step, for the resident kernels
void set_substeps(const eb_sim* s, eb::StepArgs& a) {
  const Substep* sub;
  a.n_sub = substeps(s, &sub);
}

int substeps(const eb_sim* s, const Substep** table) {
  if (s->cfg.stepper == EB_STEPPER_PEFRL) {
    *table = kPefrl;
    return 4;
  }
  if (s->cfg.stepper == EB_STEPPER_VELOCITY_VERLET) {
    *table = kVelocityVerlet;
    return 2;
  }
  *table = kVerlet;
  return 1;
}

// One step on the streaming kernel: one launch per substep.
cudaError_t stream_one_step(eb_sim* s, eb::StepArgs& a, double dt, bool rec) {
  const Substep* sub;
  const int ns = substeps(s, &sub);
  for (int k = 0; k < ns; ++k) {
    if (ns == 1) {
      a.drift_pre = 0.5 * dt;  // PositionVerlet: bit-identical to half_dt
      a.kick = dt;
      a.drift_post = 0.5 * dt;
      a.damper_time = dt;
    } else {
      a.drift_pre = sub[k].pre * dt;
      a.kick = sub[k].kick * dt;
      a.drift_post = sub[k].post * dt;
      a.damper_time = sub[k].damper * dt;
    }
    a.in = s->d_state[s->cur];
    a.out = s->d_state[s->cur ^ 1];
    cudaError_t e = launch_streaming(s, a, rec && k == ns - 1);
    if (e != cudaSuccess) return e;
    s->cur ^= 1;
    ++s->launches;
  }
  return cudaSuccess;
}

constexpr int64_t kGraphSteps = 32;  // steps per captured graph (an even launch count)

// Replay (capturing first if needed) the graph of kGraphSteps streaming steps
// that starts from the current buffer parity.
eb_status graph_steps(eb_sim* s, double dt) {
  const int p = s->cur;
  if (!s->graph[p] || s->graph_dt[p] != dt) {
    if (s->graph[p]) {
      cudaGraphExecDestroy(s->graph[p]);
      s->graph[p] = nullptr;
    }
    eb::StepArgs a = step_args(s, dt);
    const int64_t launches0 = s->launches;
    EB_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (int64_t k = 0; k < kGraphSteps && e == cudaSuccess; ++k) e = stream_one_step(s, a, dt, false);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
    // capture only recorded the launches: restore the parity and the count
    s->cur = p;
    s->launches = launches0;
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return fail(EB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    const cudaError_t e3 = cudaGraphInstantiate(&s->graph[p], g, 0);
    cudaGraphDestroy(g);
    EB_CUDA(e3);
    s->graph_dt[p] = dt;
  }
  EB_CUDA(cudaGraphLaunch(s->graph[p], s->stream));
  const Substep* sub;
  const int64_t per = substeps(s, &sub);
  s->launches += per * kGraphSteps;
  if ((per * kGraphSteps) & 1) s->cur ^= 1;
  return EB_OK;
}

// Per-size-bucket work lists: the rods of each bucket packed best fit
// decreasing into CTAs of each configuration's capacity; a CTA's slots are
// listed in a gather map, so its rods need not be neighbours in the layout.
// Rods of the pair bucket each take a cluster of two CTAs: the first
// ceil(W / 2) slots on the even CTA, the rest on the odd one.
constexpr int64_t kShortRodSlots = 264;
constexpr int kPairConfigs = 2;  // 512 or 256 threads per CTA
int bucket_of(int64_t w) {
  if (w <= kShortRodSlots) return 0;
  if (w <= 520) return 1;
  if (w <= eb::kPairMaxSlots) return 2;
  return -1;
}

eb_status build_bucket_worklists(eb_sim* s) {
  if (s->buckets[0].rods + s->buckets[1].rods + s->buckets[2].rods > 0) return EB_OK;  // built already
  int64_t count[3] = {0, 0, 0};
  for (const auto& r : s->rods) {
    const int b = bucket_of(r.n + 1);
    if (b >= 0) ++count[b];
  }
  const bool merge = count[0] > 0 && count[1] > 0 && count[2] > 0;
  for (int b = 0; b < 4; ++b) {
    if (b == 3 && !merge) continue;
    std::vector<size_t> rods;
    for (size_t r = 0; r < s->rods.size(); ++r) {
      const int rb = bucket_of(s->rods[r].n + 1);
      if (rb == b || (b == 3 && (rb == 0 || rb == 1))) rods.push_back(r);
    }
    s->buckets[b].rods = static_cast<int64_t>(rods.size());
    if (rods.empty()) continue;
    if (b == 2) {
      std::vector<int64_t> off{0};
      std::vector<int32_t> map;
      for (size_t r : rods) {
        const int64_t w = s->rods[r].n + 1, h = (w + 1) / 2;
        for (int64_t j = 0; j < w; ++j) map.push_back(static_cast<int32_t>(s->offsets[r] + j));
        off.push_back(off.back() + h);
        off.push_back(off.back() + (w - h));
      }
      eb_sim::Bucket& B = s->buckets[2];
      for (int c = 0; c < kPairConfigs; ++c) {  // one list, shared by both configurations
        if (c == 0) {
          EB_CUDA(cudaMalloc(reinterpret_cast<void**>(&B.d_off[0]), off.size() * sizeof(int64_t)));
          EB_CUDA(cudaMalloc(reinterpret_cast<void**>(&B.d_map[0]), map.size() * sizeof(int32_t)));
          EB_CUDA(cudaMemcpyAsync(B.d_off[0], off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                                  s->stream));
          EB_CUDA(cudaMemcpyAsync(B.d_map[0], map.data(), map.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                  s->stream));
        }
        B.n_ctas[c] = static_cast<int>(off.size() - 1);
      }
      continue;
    }
    for (int c = 0; c < eb::block_config_count(); ++c) {
      std::vector<int64_t> off;
      std::vector<int32_t> map;
      if (!pack_best_fit(s, rods, c, off, map)) continue;
      eb_sim::Bucket& B = s->buckets[b];
      EB_CUDA(cudaMalloc(reinterpret_cast<void**>(&B.d_off[c]), off.size() * sizeof(int64_t)));
      EB_CUDA(cudaMalloc(reinterpret_cast<void**>(&B.d_map[c]), map.size() * sizeof(int32_t)));
      EB_CUDA(cudaMemcpyAsync(B.d_off[c], off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                              s->stream));
      EB_CUDA(cudaMemcpyAsync(B.d_map[c], map.data(), map.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                              s->stream));
      B.n_ctas[c] = static_cast<int>(off.size() - 1);
    }
  }
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return EB_OK;
}

cudaError_t launch_bucket(eb_sim* s, eb::StepArgs& a, int b, int config, int steps) {
  const eb_sim::Bucket& B = s->buckets[b];
  if (b == 2) {
    if (s->cfg.precision == EB_PRECISION_MIXED)
      return eb::launch_rod_block_mixed_pairs(a, B.d_off[0], B.d_map[0], B.n_ctas[config], steps, config,
                                              s->any_damped, s->stream);
    return eb::launch_rod_block_fp64_pairs(a, B.d_off[0], B.d_map[0], B.n_ctas[config], steps, config,
                                           s->any_damped, s->stream);
  }
  if (s->cfg.precision == EB_PRECISION_MIXED)
    return eb::launch_rod_block_mixed_gather(a, B.d_off[config], B.d_map[config], B.n_ctas[config], steps, config,
                                             s->any_damped, s->stream);
  return eb::launch_rod_block_fp64_gather(a, B.d_off[config], B.d_map[config], B.n_ctas[config], steps, config,
                                          s->any_damped, s->stream);
}

// Predicted time of kProbeSteps steps of a resident launch sequence when it
// runs in launches of `chunk` steps: runs of kProbeSteps and 3 kProbeSteps
// steps (after a warm-up) give the per-step cost and the fixed cost of a
// launch (staging the state and writing it back), so a probe of a few steps
// does not charge a 128-step launch with its staging eight times over.
extern "C++" {
template <class Launch>
eb_status time_resident(eb_sim* s, cudaEvent_t e0, cudaEvent_t e1, int chunk, Launch launch, float* ms_out) {
  float t[2] = {0.0f, 0.0f};
  const int steps[2] = {kProbeSteps, 3 * kProbeSteps};
  EB_CUDA(launch(kProbeSteps));  // warm-up
  for (int i = 0; i < 2; ++i) {
    EB_CUDA(cudaEventRecord(e0, s->stream));
    EB_CUDA(launch(steps[i]));
    EB_CUDA(cudaEventRecord(e1, s->stream));
    EB_CUDA(cudaEventSynchronize(e1));
    EB_CUDA(cudaEventElapsedTime(&t[i], e0, e1));
  }
  const float per = std::max(0.0f, (t[1] - t[0]) / static_cast<float>(steps[1] - steps[0]));
  const float fixed = std::max(0.0f, t[0] - per * static_cast<float>(steps[0]));
  *ms_out = per * kProbeSteps + fixed * static_cast<float>(kProbeSteps) / static_cast<float>(std::max(1, chunk));
  return EB_OK;
}
}  // extern "C++"

// Per-size-bucket plan: when the batch has rods of two or more buckets, or
// rods of 520 to 1039 elements (and none longer), time every configuration on
// each bucket alone for kProbeSteps steps into the spare buffer; *total_ms =
// the sum of the buckets' best times, or -1 when the plan does not apply.
eb_status probe_buckets(eb_sim* s, const eb::StepArgs& args, cudaEvent_t e0, cudaEvent_t e1, int chunk,
                        float* total_ms) {
  *total_ms = -1.0f;
  if (s->n_slots > INT32_MAX) return EB_OK;  // the gathered slot lists hold 32-bit slot indices
  for (const auto& r : s->rods)
    if (bucket_of(r.n + 1) < 0) return EB_OK;
  if (eb_status st = build_bucket_worklists(s)) return st;
  const int used = (s->buckets[0].rods > 0) + (s->buckets[1].rods > 0) + (s->buckets[2].rods > 0);
  if (used < 2 && s->buckets[2].rods == 0) return EB_OK;
  eb::StepArgs a = args;
  float best_of[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int b = 0; b < 4; ++b) {
    s->bucket_config[b] = -1;
    if (s->buckets[b].rods == 0) continue;
    float best = 0.0f;
    const int n_cfg = b == 2 ? kPairConfigs : eb::block_config_count();
    for (int c = 0; c < n_cfg; ++c) {
      if (!s->buckets[b].d_off[b == 2 ? 0 : c]) continue;
      float ms = 0.0f;
      if (eb_status st = time_resident(s, e0, e1, chunk, [&](int k) { return launch_bucket(s, a, b, c, k); }, &ms))
        return st;
      s->plan_ms[b == 3 ? 16 + c : 5 + 4 * b + c] = ms;
      if (s->bucket_config[b] < 0 || ms < best) {
        best = ms;
        s->bucket_config[b] = c;
      }
    }
    if (s->bucket_config[b] < 0 && b != 3) return EB_OK;
    best_of[b] = best;
  }
  // buckets 0 and 1 apart, or packed together (bucket 3) when that is faster
  const float apart = best_of[0] + best_of[1];
  s->bucket_merged = s->bucket_config[3] >= 0 && best_of[3] < apart;
  *total_ms = best_of[2] + (s->bucket_merged ? best_of[3] : apart);
  return EB_OK;
}

// bucket configurations as one number: c0 + 4 c1 + 16 c2, plus 64 (c3 + 1)
// when buckets 0 and 1 run packed together (c0 = c1 = 0 then)
int bucket_plan_config(const eb_sim* s) {
  if (s->bucket_merged) return 16 * std::max(0, s->bucket_config[2]) + 64 * (s->bucket_config[3] + 1);
  int c = 0;
  for (int b = 2; b >= 0; --b) c = 4 * c + std::max(0, s->bucket_config[b]);
  return c;
}

// Choose between the streaming kernel and the resident configurations by
// timing each for kProbeSteps steps from the current state into the spare
// buffer (the current state is left untouched).
// chunk: steps per resident launch the first call would run (its step count,
// at most kResidentChunk); the resident probes are compared at that length.
eb_status plan_steps(eb_sim* s, double dt, int chunk) {
  // contact needs a global exchange every step, PEFRL four force evaluations
  // a step: the streaming kernel
  const bool force_stream = (s->cfg.flags & (EB_FLAG_STEP_STREAMING | EB_FLAG_REFERENCE_ROUNDING)) != 0 ||
                            s->contact.on || s->jd.on;
  if (force_stream) {
    s->plan_mode = 1;
    return EB_OK;
  }
  if (eb_status st = build_block_worklists(s)) return st;
  const int want = s->cfg.resident_config - 1;
  if (want >= 0) {
    if (s->d_cta_start[want]) {
      s->plan_mode = 2;
      s->plan_config = want;
    } else {
      s->plan_mode = 1;  // the rods do not fit this configuration
    }
    return EB_OK;
  }
  cudaEvent_t e0, e1;
  EB_CUDA(cudaEventCreate(&e0));
  EB_CUDA(cudaEventCreate(&e1));
  eb::StepArgs a = step_args(s, dt);
  set_substeps(s, a);  // the resident kernels take the stepper's substeps
  a.in = s->d_state[s->cur];
  a.out = s->d_state[s->cur ^ 1];
  float best = 0.0f;
  int best_mode = 1, best_cfg = -1;
  float bucket_ms = -1.0f;
  bool bucket_done = false;
  if (s->cfg.flags & EB_FLAG_STEP_BUCKETED) {
    bucket_done = true;
    if (eb_status st = probe_buckets(s, a, e0, e1, chunk, &bucket_ms)) return st;
    if (bucket_ms >= 0.0f) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      s->plan_mode = 3;
      s->plan_config = bucket_plan_config(s);
      return check_device_status(s);
    }
  }
  // mixed precision exists only on the resident kernels: the streaming FP64
  // kernel is then a fallback for rods too long for any configuration
  const bool force_resident =
      (s->cfg.flags & EB_FLAG_STEP_RESIDENT) != 0 || s->cfg.precision == EB_PRECISION_MIXED;
  for (int c = -1; c < eb::block_config_count(); ++c) {
    if (c >= 0 && !s->d_cta_start[c]) continue;
    if (c < 0 && force_resident) continue;
    float ms = 0.0f;
    if (c < 0) {
      // whole steps: one launch per substep (four for PEFRL)
      const Substep* sub;
      const int ns = substeps(s, &sub);
      for (int rep = 0; rep < 2; ++rep) {  // first repetition warms up
        EB_CUDA(cudaEventRecord(e0, s->stream));
        for (int k = 0; k < kProbeSteps; ++k)
          for (int j = 0; j < ns; ++j) {
            eb::StepArgs b = a;
            b.drift_pre = sub[j].pre * dt;
            b.kick = sub[j].kick * dt;
            b.drift_post = sub[j].post * dt;
            b.damper_time = sub[j].damper * dt;
            EB_CUDA(launch_streaming(s, b, false));
          }
        EB_CUDA(cudaEventRecord(e1, s->stream));
        EB_CUDA(cudaEventSynchronize(e1));
      }
      EB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    } else if (eb_status st = time_resident(s, e0, e1, chunk, [&](int k) { return launch_resident(s, a, c, k); },
                                            &ms)) {
      return st;
    }
    s->plan_ms[c + 1] = ms;
    if (best_cfg == -1 && best_mode == 1 && best == 0.0f) {
      best = ms;
      best_mode = c < 0 ? 1 : 2;
      best_cfg = c;
    } else if (ms < best) {
      best = ms;
      best_mode = c < 0 ? 1 : 2;
      best_cfg = c;
    }
  }
  if (best_mode == 2 && best_cfg < 0) best_mode = 1;
  // per size bucket: keep the best pair if it beats the plans above
  if (!bucket_done) {
    if (eb_status st = probe_buckets(s, a, e0, e1, chunk, &bucket_ms)) return st;
    // (mixed precision: the streaming kernel was not timed, so any bucket
    // plan beats the FP64 fallback)
    const bool have_best = best_cfg >= 0 || !force_resident;
    if (bucket_ms >= 0.0f && (!have_best || bucket_ms < best)) {
      best_mode = 3;
      best_cfg = bucket_plan_config(s);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s->plan_mode = best_mode;
  s->plan_config = best_cfg;
  s->plan_timed = true;
  return check_device_status(s);
}

constexpr int64_t kContactChunk = 32;  // steps between checks of the pair buffer

eb::ContactArgs contact_args(eb_sim* s, double dt) {
  ContactDevice& c = s->contact;
  eb::ContactArgs a{};
  a.stride = s->stride;
  a.n_slots = s->n_slots;
  a.par = s->d_param;
  a.meta = s->d_meta;
  a.rods = s->d_rods;
  a.cap_material = c.cap_material;
  a.half_dt = 0.5 * dt;
  a.sim_flags = s->sim_flags;
  a.cap = c.cap;
  a.extent_bits = c.extent;
  a.cell = c.cell;
  a.bucket = c.bucket;
  a.table_mask = c.table_mask;
  a.bucket_count = c.bucket_count;
  a.bucket_start = c.bucket_start;
  a.sorted_rec = c.sorted_rec;
  a.pair_count = c.pair_count;
  a.fixed = c.fixed;
  a.pair_offset = c.pair_offset;
  a.partners = c.partners;
  a.capacity = c.capacity;
  a.required = c.required;
  a.planes = c.planes;
  a.n_planes = static_cast<int32_t>(s->planes.size());
  a.n_materials = static_cast<int32_t>(s->materials.size());
  a.pair_table = c.pair_table;
  a.cf = c.loads;
  a.ct = c.loads + 3 * s->stride;
  a.n_caps = c.n_caps;
  a.scan_blocks = c.scan_blocks;
  a.status = s->d_status;
  return a;
}

// Streaming steps with external loads evaluated at every force evaluation's
// drifted state: the collision system (in chunks of kContactChunk steps,
// rerun with a larger pair buffer on overflow) and/or the connections.
eb_status step_with_contact(eb_sim* s, double dt, int64_t n_steps, bool diag) {
  ContactDevice& c = s->contact;
  const bool contact = c.on;
  const size_t state_bytes = static_cast<size_t>(eb::kStateFields * s->stride) * sizeof(double);
  eb::StepArgs a = step_args(s, dt);
  if (contact) {
    a.contact_force = c.loads;
    a.contact_torque = c.loads + 3 * s->stride;
  }
  eb::JointArgs ja{};
  if (s->jd.on) {
    ja = joint_args(s);
    a.joint_force = ja.joint_force;
    a.joint_torque = ja.joint_torque;
  }
  int64_t done = 0;
  int regrowths = 0;
  while (done < n_steps) {
    const int64_t k = contact ? std::min<int64_t>(kContactChunk, n_steps - done) : n_steps - done;
    const int c0 = s->cur;
    const Substep* sub;
    const int ns = substeps(s, &sub);
    // the chunk's starting state is kept for a rerun; a chunk of one launch
    // leaves it untouched in the buffer the launch reads
    const bool keep = contact && k * ns > 1;
    if (keep)
      EB_CUDA(cudaMemcpyAsync(c.backup, s->d_state[c0], state_bytes, cudaMemcpyDeviceToDevice, s->stream));
    eb::ContactArgs ca{};
    if (contact) ca = contact_args(s, dt);
    for (int64_t i = 0; i < k; ++i) {
      for (int j = 0; j < ns; ++j) {
        // one contact evaluation per force evaluation, at its drifted state
        if (ns > 1) {
          a.drift_pre = sub[j].pre * dt;
          a.kick = sub[j].kick * dt;
          a.drift_post = sub[j].post * dt;
          ca.half_dt = a.drift_pre;
        }
        if (contact) {
          ca.state = s->d_state[s->cur];
          EB_CUDA(eb::launch_contact(ca, s->stream, &s->launches));
        }
        if (s->jd.on) {
          ja.state = s->d_state[s->cur];
          ja.pre = a.drift_pre;
          EB_CUDA(eb::launch_joints(ja, s->stream));
          s->launches += 2;
        }
        a.in = s->d_state[s->cur];
        a.out = s->d_state[s->cur ^ 1];
        EB_CUDA(launch_streaming(s, a, diag && done + i == n_steps - 1 && j == ns - 1));
        s->cur ^= 1;
        ++s->launches;
      }
    }
    if (!contact) {
      done += k;
      continue;
    }
    uint32_t st = 0;
    EB_CUDA(cudaMemcpyAsync(&st, s->d_status, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
    EB_CUDA(cudaStreamSynchronize(s->stream));
    if (st & eb::kStatusPairOverflow) {
      // the pair total the lists needed, read only when they did not fit
      unsigned long long req = 0;
      EB_CUDA(cudaMemcpyAsync(&req, c.required, sizeof(req), cudaMemcpyDeviceToHost, s->stream));
      EB_CUDA(cudaStreamSynchronize(s->stream));
      if (++regrowths > 8) return fail(EB_ERR_OUT_OF_MEMORY, "candidate pair buffer keeps overflowing");
      const int64_t want = std::max<int64_t>(2 * c.capacity, static_cast<int64_t>(req) + req / 2);
      if (want >= (int64_t(1) << 31)) return fail(EB_ERR_UNSUPPORTED, "more than 2^31 candidate pairs");
      EB_CUDA(cudaFree(c.partners));
      c.partners = nullptr;
      EB_CUDA(cudaMalloc(reinterpret_cast<void**>(&c.partners), static_cast<size_t>(want) * sizeof(int32_t)));
      EB_CUDA(cudaMemsetAsync(c.partners, 0, static_cast<size_t>(want) * sizeof(int32_t), s->stream));
      c.capacity = want;
      const uint32_t cleared = st & ~static_cast<uint32_t>(eb::kStatusPairOverflow);
      EB_CUDA(cudaMemcpyAsync(s->d_status, &cleared, sizeof(cleared), cudaMemcpyHostToDevice, s->stream));
      EB_CUDA(cudaMemsetAsync(c.required, 0, sizeof(unsigned long long), s->stream));
      if (keep)
        EB_CUDA(cudaMemcpyAsync(s->d_state[c0], c.backup, state_bytes, cudaMemcpyDeviceToDevice, s->stream));
      EB_CUDA(cudaStreamSynchronize(s->stream));
      s->cur = c0;
      continue;
    }
    c.evaluated = true;
    if (st) return check_device_status(s);
    done += k;
  }
  return EB_OK;
}

// the reference builds the damper's exponential constants once for the
// simulation's dt (AnalyticalLinearDamper.hpp:40-57)
eb_status damper_for_dt(eb_sim* s, double dt) {
  if (!(s->sim_flags & eb::kSimDamper) || dt == s->damper_dt) return EB_OK;
  for (auto& r : s->rods)
    if (r.info.flags & eb::kRodDamper) r.info.damper_t = std::exp(-r.damper_nu_t * dt);
  if (eb_status st = upload_rod_table(s)) return st;
  s->damper_dt = dt;
  return EB_OK;
}

// Slot groups of the host-state exchange for the resident plan (mode 2: the
// whole-batch configuration; mode 3: each size bucket's): the rods in order
// cut into contiguous runs of about equal slot counts, each packed on its own
// the way the plan packs the whole batch (a group's CTAs touch only its
// slots, so its launches need only its copies).  The first group's upload and
// the last one's download overlap no launch, so the groups are small at
// either end and larger in between (1, 2, then about 4 waves of 512-slot
// CTAs each, then 2 and 1): against equal groups of six waves, at most eight,
// that took the uneven batch's exchange from 13.5 to 14.5 G element-steps/s
// (14.1 G with equal groups of three waves, 14.3 G of two).  A single group
// means no overlap and the exchange runs its copies and steps in sequence.
eb_status upload_list(eb_sim* s, const std::vector<int64_t>& off, const std::vector<int32_t>& map, int64_t** d_off,
                      int32_t** d_map) {
  EB_CUDA(cudaMalloc(reinterpret_cast<void**>(d_off), off.size() * sizeof(int64_t)));
  EB_CUDA(cudaMalloc(reinterpret_cast<void**>(d_map), map.size() * sizeof(int32_t)));
  EB_CUDA(cudaMemcpyAsync(*d_off, off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaMemcpyAsync(*d_map, map.data(), map.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return EB_OK;
}

// the buckets a bucketed plan launches
bool bucket_launched(const eb_sim* s, int b) {
  return s->buckets[b].rods > 0 && !(s->bucket_merged ? (b == 0 || b == 1) : b == 3);
}

eb_status build_exchange_groups(eb_sim* s) {
  const int64_t plan = 1000 * s->plan_mode + (s->plan_mode == 2 ? s->plan_config : bucket_plan_config(s));
  if (s->xplan == plan && !s->xgroups.empty()) return EB_OK;
  for (auto& g : s->xgroups)
    for (int k = 0; k < 4; ++k) {
      if (g.d_off[k]) EB_CUDA(cudaFree(g.d_off[k]));
      if (g.d_map[k]) EB_CUDA(cudaFree(g.d_map[k]));
    }
  s->xgroups.clear();
  s->xplan = plan;
  int sms = 0;
  EB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->cfg.device));
  // group sizes in waves of 512-slot CTAs: 1 and 2 at either end (their
  // copies overlap no launch), equal groups of about four in between
  const double units = static_cast<double>(s->n_slots) / (static_cast<double>(std::max(sms, 1)) * 512.0);
  if (units < 2.0 || s->rods.size() < 2) return EB_OK;
  std::vector<double> wts;
  if (units >= 12.0) {
    const double mid = units - 6.0;
    const int m = std::max(1, static_cast<int>(std::llround(mid / 4.0)));
    wts = {1.0, 2.0};
    for (int i = 0; i < m; ++i) wts.push_back(mid / m);
    wts.push_back(2.0);
    wts.push_back(1.0);
  } else {
    wts.assign(static_cast<size_t>(units / 2.0), 1.0);
  }
  const int64_t n_groups = static_cast<int64_t>(wts.size());
  if (n_groups < 2) return EB_OK;
  std::vector<int64_t> bound(1, 0);
  {
    double tot = 0.0, acc = 0.0;
    for (double w : wts) tot += w;
    for (double w : wts) {
      acc += w;
      bound.push_back(static_cast<int64_t>(static_cast<double>(s->n_slots) * (acc / tot)));
    }
  }
  std::vector<std::vector<size_t>> members(1);
  std::vector<int64_t> cut(1, 0);
  for (size_t r = 0; r < s->rods.size(); ++r) {
    const int64_t j = static_cast<int64_t>(members.size());
    if (!members.back().empty() && j < n_groups && s->offsets[r] >= bound[static_cast<size_t>(j)]) {
      members.emplace_back();
      cut.push_back(s->offsets[r]);
    }
    members.back().push_back(r);
  }
  cut.push_back(s->n_slots);
  if (members.size() < 2) return EB_OK;
  std::vector<int64_t> off;
  std::vector<int32_t> map;
  for (size_t g = 0; g < members.size(); ++g) {
    s->xgroups.emplace_back();  // owned from here on (freed with the simulator)
    eb_sim::XGroup& X = s->xgroups.back();
    X.lo = cut[g];
    X.hi = cut[g + 1];
    for (int b = 0; b < 4; ++b) {
      std::vector<size_t> rods;
      if (s->plan_mode == 2) {
        if (b > 0) break;
        rods = members[g];
      } else {
        if (!bucket_launched(s, b)) continue;
        for (size_t r : members[g]) {
          const int rb = bucket_of(s->rods[r].n + 1);
          if (rb == b || (b == 3 && (rb == 0 || rb == 1))) rods.push_back(r);
        }
      }
      if (rods.empty()) continue;
      if (s->plan_mode == 3 && b == 2) {
        // rod pairs: the first half of each rod's slots on the even CTA
        off.assign(1, 0);
        map.clear();
        for (size_t r : rods) {
          const int64_t w = s->rods[r].n + 1, h = (w + 1) / 2;
          for (int64_t k = 0; k < w; ++k) map.push_back(static_cast<int32_t>(s->offsets[r] + k));
          off.push_back(off.back() + h);
          off.push_back(off.back() + (w - h));
        }
      } else {
        const int c = s->plan_mode == 2 ? s->plan_config : s->bucket_config[b];
        if (!pack_best_fit(s, rods, c, off, map)) return fail(EB_ERR_INVALID_STATE, "exchange group does not pack");
      }
      if (eb_status st = upload_list(s, off, map, &X.d_off[b], &X.d_map[b])) return st;
      X.n_ctas[b] = static_cast<int>(off.size() - 1);
    }
  }
  if (!s->xs[0])
    for (auto& x : s->xs) EB_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
  const size_t n_ev = 2 * s->xgroups.size() + 5;
  while (s->xev.size() < n_ev) {
    cudaEvent_t e;
    EB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    s->xev.push_back(e);
  }
  return EB_OK;
}

// One resident launch of `steps` steps over slot group X.
cudaError_t launch_exchange_group(eb_sim* s, eb::StepArgs& a, const eb_sim::XGroup& X, int steps, cudaStream_t L,
                                  int64_t* launches) {
  const bool mixed = s->cfg.precision == EB_PRECISION_MIXED;
  for (int b = 0; b < 4; ++b) {
    if (X.n_ctas[b] == 0) continue;
    const int c = s->plan_mode == 2 ? s->plan_config : s->bucket_config[b];
    cudaError_t e;
    if (s->plan_mode == 3 && b == 2)
      e = mixed ? eb::launch_rod_block_mixed_pairs(a, X.d_off[b], X.d_map[b], X.n_ctas[b], steps, c, s->any_damped, L)
                : eb::launch_rod_block_fp64_pairs(a, X.d_off[b], X.d_map[b], X.n_ctas[b], steps, c, s->any_damped, L);
    else
      e = mixed ? eb::launch_rod_block_mixed_gather(a, X.d_off[b], X.d_map[b], X.n_ctas[b], steps, c, s->any_damped, L)
                : eb::launch_rod_block_fp64_gather(a, X.d_off[b], X.d_map[b], X.n_ctas[b], steps, c, s->any_damped, L);
    if (e != cudaSuccess) return e;
    ++*launches;
  }
  return cudaSuccess;
}

}  // namespace

EB_API eb_status eb_step(eb_sim* s, double* time, double dt, int64_t n_steps) {
  if (check_sim(s)) return EB_ERR_INVALID_ARGUMENT;
  if (!s->finalized) return fail(EB_ERR_INVALID_STATE, "finalize before stepping");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(EB_ERR_INVALID_ARGUMENT, "dt must be positive and finite");
  if (n_steps < 0) return fail(EB_ERR_INVALID_ARGUMENT, "negative step count");
  if (n_steps == 0) return EB_OK;
  if (eb_status st = set_device(s)) return st;
  if (eb_status st = damper_for_dt(s, dt)) return st;
  {
    // plan at the first call; plan again when a call's launches would be
    // much longer than the ones the plan was timed at (a first call of a
    // few steps favours the streaming kernel, whose launches carry no
    // staging cost, for every later call)
    const int chunk = static_cast<int>(std::min<int64_t>(n_steps, kResidentChunk));
    if (s->plan_mode == 0 || (s->plan_timed && chunk >= 4 * s->plan_chunk)) {
      if (eb_status st = plan_steps(s, dt, chunk)) return st;
      s->plan_chunk = chunk;
    }
  }
  const bool diag = s->d_diag != nullptr;
  if (s->contact.on || s->jd.on) {
    if (eb_status st = step_with_contact(s, dt, n_steps, diag)) return st;
    advance_time(s, time, dt, n_steps);
    return EB_OK;
  }
  eb::StepArgs a = step_args(s, dt);
  set_substeps(s, a);  // the resident kernels take the stepper's substeps
  int64_t done = 0;
  if (s->plan_mode == 2 || s->plan_mode == 3) {
    // resident kernel in chunks; the last step of a call that records
    // diagnostics runs on the streaming kernel, which writes them
    const int64_t resident_steps = diag ? n_steps - 1 : n_steps;
    const int c = s->plan_config;
    while (done < resident_steps) {
      const int k = static_cast<int>(std::min<int64_t>(kResidentChunk, resident_steps - done));
      a.in = s->d_state[s->cur];
      a.out = s->d_state[s->cur ^ 1];
      if (s->plan_mode == 2) {
        EB_CUDA(launch_resident(s, a, c, k));
        ++s->launches;
      } else {
        // one launch per size bucket over the same buffers
        for (int b = 0; b < 4; ++b) {
          if (s->buckets[b].rods == 0) continue;
          if (s->bucket_merged ? (b == 0 || b == 1) : b == 3) continue;
          EB_CUDA(launch_bucket(s, a, b, s->bucket_config[b], k));
          ++s->launches;
        }
      }
      s->cur ^= 1;
      done += k;
    }
  }
  if (s->cfg.flags & EB_FLAG_CUDA_GRAPH) {
    // whole graphs of kGraphSteps steps; a recorded last step stays outside
    while (n_steps - done - (diag ? 1 : 0) >= kGraphSteps) {
      if (eb_status st = graph_steps(s, dt)) return st;
      done += kGraphSteps;
    }
  }
  for (; done < n_steps; ++done) EB_CUDA(stream_one_step(s, a, dt, diag && done == n_steps - 1));
  advance_time(s, time, dt, n_steps);
  return EB_OK;
}

// The state fields the exchange moves, in eb_host_state's order.
constexpr int32_t kExchangeFields[4] = {EB_POSITION, EB_VELOCITY, EB_DIRECTOR, EB_ANGULAR_VELOCITY};

EB_API eb_status eb_step_host_state(eb_sim* s, double* time, double dt, int64_t n_steps,
                                    const eb_host_state* host) {
  if (check_sim(s) || !host) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (!s->finalized) return fail(EB_ERR_INVALID_STATE, "finalize before stepping");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(EB_ERR_INVALID_ARGUMENT, "dt must be positive and finite");
  if (n_steps < 0) return fail(EB_ERR_INVALID_ARGUMENT, "negative step count");
  const double* in[4] = {host->position_in, host->velocity_in, host->director_in, host->angular_velocity_in};
  double* out[4] = {host->position_out, host->velocity_out, host->director_out, host->angular_velocity_out};
  bool any_out = false;
  for (double* o : out) any_out = any_out || o;
  if (eb_status st = set_device(s)) return st;
  // the plan is chosen by the first step; contact, connections and recorded
  // diagnostics step the whole batch together
  bool overlap = n_steps > 0 && (s->plan_mode == 2 || s->plan_mode == 3) && !s->contact.on && !s->jd.on && !s->d_diag;
  if (overlap) {
    if (eb_status st = build_exchange_groups(s)) return st;
    overlap = !s->xgroups.empty();
  }
  if (!overlap) {
    for (int f = 0; f < 4; ++f)
      if (in[f])
        if (eb_status st = batch_copy(s, kExchangeFields[f], EB_LAYOUT_SLOTS, const_cast<double*>(in[f]),
                                      kFields[kExchangeFields[f]].ncomp * s->n_slots, true))
          return st;
    if (eb_status st = eb_step(s, time, dt, n_steps)) return st;
    for (int f = 0; f < 4; ++f)
      if (out[f])
        if (eb_status st = batch_copy(s, kExchangeFields[f], EB_LAYOUT_SLOTS, out[f],
                                      kFields[kExchangeFields[f]].ncomp * s->n_slots, false))
          return st;
    return EB_OK;
  }
  if (eb_status st = damper_for_dt(s, dt)) return st;
  eb::StepArgs a = step_args(s, dt);
  set_substeps(s, a);
  const int64_t S = s->stride;
  const size_t pitch = static_cast<size_t>(S) * sizeof(double);
  const size_t hpitch = static_cast<size_t>(s->n_slots) * sizeof(double);
  const int64_t chunks = (n_steps + kResidentChunk - 1) / kResidentChunk;
  const int c0 = s->cur, c1 = static_cast<int>((c0 + chunks) & 1);
  const size_t G = s->xgroups.size();
  cudaEvent_t* ev = s->xev.data();  // [0] start, [1, G] inputs landed, [G+1, 2G] steps done, [2G+1, 2G+4] ends
  EB_CUDA(cudaEventRecord(ev[0], s->stream));
  for (cudaStream_t x : s->xs) EB_CUDA(cudaStreamWaitEvent(x, ev[0], 0));
  for (size_t g = 0; g < G; ++g) {
    const eb_sim::XGroup& X = s->xgroups[g];
    const size_t w = static_cast<size_t>(X.hi - X.lo) * sizeof(double);
    cudaStream_t L = s->xs[2 + (g & 1)];
    // inputs into the current buffer, then the same values into the other
    // one on the device (as eb_set_field_batch: entries no step writes match)
    for (int f = 0; f < 4; ++f) {
      if (!in[f]) continue;
      const FieldInfo& fi = kFields[kExchangeFields[f]];
      EB_CUDA(cudaMemcpy2DAsync(s->d_state[c0] + fi.offset * S + X.lo, pitch, in[f] + X.lo, hpitch, w, fi.ncomp,
                                cudaMemcpyHostToDevice, s->xs[0]));
    }
    EB_CUDA(cudaEventRecord(ev[1 + g], s->xs[0]));
    EB_CUDA(cudaStreamWaitEvent(L, ev[1 + g], 0));
    for (int f = 0; f < 4; ++f) {
      if (!in[f]) continue;
      const FieldInfo& fi = kFields[kExchangeFields[f]];
      EB_CUDA(cudaMemcpy2DAsync(s->d_state[c0 ^ 1] + fi.offset * S + X.lo, pitch, s->d_state[c0] + fi.offset * S + X.lo,
                                pitch, w, fi.ncomp, cudaMemcpyDeviceToDevice, L));
    }
    int cur = c0;
    for (int64_t done = 0; done < n_steps;) {
      const int k = static_cast<int>(std::min<int64_t>(kResidentChunk, n_steps - done));
      a.in = s->d_state[cur];
      a.out = s->d_state[cur ^ 1];
      EB_CUDA(launch_exchange_group(s, a, X, k, L, &s->launches));
      cur ^= 1;
      done += k;
    }
    EB_CUDA(cudaEventRecord(ev[1 + G + g], L));
    EB_CUDA(cudaStreamWaitEvent(s->xs[1], ev[1 + G + g], 0));
    for (int f = 0; f < 4; ++f) {
      if (!out[f]) continue;
      const FieldInfo& fi = kFields[kExchangeFields[f]];
      EB_CUDA(cudaMemcpy2DAsync(out[f] + X.lo, hpitch, s->d_state[c1] + fi.offset * S + X.lo, pitch, w, fi.ncomp,
                                cudaMemcpyDeviceToHost, s->xs[1]));
    }
  }
  for (int k = 0; k < 4; ++k) {
    EB_CUDA(cudaEventRecord(ev[1 + 2 * G + k], s->xs[k]));
    EB_CUDA(cudaStreamWaitEvent(s->stream, ev[1 + 2 * G + k], 0));
  }
  s->cur = c1;
  advance_time(s, time, dt, n_steps);
  if (!any_out) return EB_OK;
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_status(s);
}

EB_API eb_status eb_contact_pairs(eb_sim* s, int64_t* pairs, int64_t capacity, int64_t* count) {
  if (check_sim(s) || !count) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (capacity > 0 && !pairs) return fail(EB_ERR_INVALID_ARGUMENT, "null pair buffer");
  const ContactDevice& c = s->contact;
  if (!c.on) return fail(EB_ERR_UNSUPPORTED, "no rod takes part in contact");
  if (!c.evaluated) return fail(EB_ERR_INVALID_STATE, "no contact evaluation yet: step first");
  if (eb_status st = set_device(s)) return st;
  const size_t n = static_cast<size_t>(s->n_slots);
  std::vector<int32_t> cnt(n), fixed(n * eb::kFixedPartners);
  std::vector<int64_t> off(n + 1);
  EB_CUDA(cudaMemcpyAsync(cnt.data(), c.pair_count, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
  EB_CUDA(cudaMemcpyAsync(fixed.data(), c.fixed, fixed.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
  EB_CUDA(cudaMemcpyAsync(off.data(), c.pair_offset, off.size() * sizeof(int64_t), cudaMemcpyDeviceToHost,
                          s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  const int64_t total = off[n];
  if (total > c.capacity) return fail(EB_ERR_INVALID_STATE, "the last evaluation overflowed the pair buffer");
  std::vector<int32_t> part(static_cast<size_t>(std::max<int64_t>(total, 1)));
  if (total > 0)
    EB_CUDA(cudaMemcpyAsync(part.data(), c.partners, static_cast<size_t>(total) * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  int64_t m = 0;
  for (size_t a = 0; a < n; ++a) {
    const int32_t k = cnt[a];
    const int32_t* list = k <= eb::kFixedPartners ? &fixed[a * eb::kFixedPartners] : &part[static_cast<size_t>(off[a])];
    for (int32_t j = 0; j < k; ++j) {
      const int64_t b = list[j];
      if (b <= static_cast<int64_t>(a)) continue;
      if (m < capacity) {
        pairs[2 * m] = static_cast<int64_t>(a);
        pairs[2 * m + 1] = b;
      }
      ++m;
    }
  }
  *count = m;
  return check_device_status(s);
}

EB_API eb_status eb_step_plan(const eb_sim* s, int32_t* mode, int32_t* config, float* probe_ms, int32_t count) {
  if (check_sim(s) || !mode || !config) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  *mode = s->plan_mode;
  *config = s->plan_config;
  if (probe_ms)
    for (int i = 0; i < count && i < 20; ++i) probe_ms[i] = s->plan_ms[i];
  return EB_OK;
}

EB_API eb_status eb_synchronize(eb_sim* s) {
  if (check_sim(s)) return EB_ERR_INVALID_ARGUMENT;
  if (!s->stream) return EB_OK;
  if (eb_status st = set_device(s)) return st;
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_status(s);
}

EB_API eb_status eb_energy(eb_sim* s, double* out, int64_t count) {
  if (check_sim(s) || !out) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (!s->finalized) return fail(EB_ERR_INVALID_STATE, "finalize first");
  const int64_t nr = static_cast<int64_t>(s->rods.size());
  if (count != 4 * nr) return fail(EB_ERR_INVALID_ARGUMENT, "energy needs 4 values per rod");
  if (eb_status st = set_device(s)) return st;
  EB_CUDA(eb::launch_rod_energy(nr, s->stride, s->d_offsets, s->d_state[s->cur], s->d_param,
                                s->d_energy, s->stream));
  ++s->launches;
  EB_CUDA(cudaMemcpyAsync(out, s->d_energy, static_cast<size_t>(4 * nr) * sizeof(double),
                          cudaMemcpyDeviceToHost, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_status(s);
}

// ---- snapshots ------------------------------------------------------------
// Layout: SnapshotHeader, n per rod (int64), the current state rows
// (kStateFields x n_slots doubles), the parameter rows (kParamFields x
// n_slots doubles), the per-rod constraint and forcing table (RodInfo per
// rod).  The configuration hash covers what must match for a load: the
// rods' sizes and models, contact membership, the connections, precision,
// stepper, environment flags and gravity.
namespace {
struct SnapshotHeader {
  char magic[8];
  uint32_t version;
  uint32_t sim_flags;
  int64_t n_rods;
  int64_t n_slots;
  uint64_t config_hash;
  double gravity[3];
};
constexpr char kSnapshotMagic[8] = {'E', 'B', 'S', 'N', 'A', 'P', '0', '1'};

uint64_t snapshot_hash(const eb_sim* s) {
  uint64_t h = 1469598103934665603ull;  // FNV-1a over the configuration words
  auto mix = [&](uint64_t v) {
    for (int b = 0; b < 8; ++b) {
      h ^= (v >> (8 * b)) & 0xffu;
      h *= 1099511628211ull;
    }
  };
  mix(static_cast<uint64_t>(s->cfg.precision));
  mix(static_cast<uint64_t>(s->cfg.stepper));
  mix(s->sim_flags);
  for (const RodHost& r : s->rods) {
    mix(static_cast<uint64_t>(r.n));
    mix(static_cast<uint64_t>(r.model));
    mix(static_cast<uint64_t>(static_cast<int64_t>(r.contact_material)));
  }
  for (const JointHost& j : s->joints) {
    mix(static_cast<uint64_t>(j.rod_a));
    mix(static_cast<uint64_t>(j.index_a));
    mix(static_cast<uint64_t>(j.rod_b));
    mix(static_cast<uint64_t>(j.index_b));
    mix(static_cast<uint64_t>(j.joint.kind));
  }
  return h;
}

uint64_t snapshot_bytes(const eb_sim* s) {
  const uint64_t nr = s->rods.size(), ns = static_cast<uint64_t>(s->n_slots);
  return sizeof(SnapshotHeader) + nr * sizeof(int64_t) +
         ns * (eb::kStateFields + eb::kParamFields) * sizeof(double) + nr * sizeof(eb::RodInfo);
}
}  // namespace

EB_API eb_status eb_snapshot_size(const eb_sim* s, uint64_t* bytes) {
  if (check_sim(s) || !bytes) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (!s->finalized) return fail(EB_ERR_INVALID_STATE, "a snapshot needs a finalized simulator");
  *bytes = snapshot_bytes(s);
  return EB_OK;
}

EB_API eb_status eb_snapshot_save(eb_sim* s, void* buffer, uint64_t bytes) {
  if (check_sim(s) || !buffer) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (!s->finalized) return fail(EB_ERR_INVALID_STATE, "a snapshot needs a finalized simulator");
  if (bytes != snapshot_bytes(s)) return fail(EB_ERR_INVALID_ARGUMENT, "buffer size differs from eb_snapshot_size");
  if (eb_status st = set_device(s)) return st;
  unsigned char* p = static_cast<unsigned char*>(buffer);
  SnapshotHeader h{};
  std::memcpy(h.magic, kSnapshotMagic, 8);
  h.version = 1;
  h.sim_flags = s->sim_flags;
  h.n_rods = static_cast<int64_t>(s->rods.size());
  h.n_slots = s->n_slots;
  h.config_hash = snapshot_hash(s);
  for (int d = 0; d < 3; ++d) h.gravity[d] = s->gravity[d];
  std::memcpy(p, &h, sizeof(h));
  p += sizeof(h);
  for (const RodHost& r : s->rods) {
    std::memcpy(p, &r.n, sizeof(int64_t));
    p += sizeof(int64_t);
  }
  const size_t pitch = static_cast<size_t>(s->stride) * sizeof(double);
  const size_t w = static_cast<size_t>(s->n_slots) * sizeof(double);
  EB_CUDA(cudaMemcpy2DAsync(p, w, s->d_state[s->cur], pitch, w, eb::kStateFields, cudaMemcpyDeviceToHost,
                            s->stream));
  p += w * eb::kStateFields;
  EB_CUDA(cudaMemcpy2DAsync(p, w, s->d_param, pitch, w, eb::kParamFields, cudaMemcpyDeviceToHost, s->stream));
  p += w * eb::kParamFields;
  EB_CUDA(cudaMemcpyAsync(p, s->d_rods, s->rods.size() * sizeof(eb::RodInfo), cudaMemcpyDeviceToHost, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_status(s);
}

EB_API eb_status eb_snapshot_load(eb_sim* s, const void* buffer, uint64_t bytes) {
  if (check_sim(s) || !buffer) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  if (!s->finalized) return fail(EB_ERR_INVALID_STATE, "loading a snapshot needs a finalized simulator");
  if (bytes < sizeof(SnapshotHeader)) return fail(EB_ERR_INVALID_ARGUMENT, "not a snapshot (too short)");
  const unsigned char* p = static_cast<const unsigned char*>(buffer);
  SnapshotHeader h;
  std::memcpy(&h, p, sizeof(h));
  if (std::memcmp(h.magic, kSnapshotMagic, 8) != 0 || h.version != 1)
    return fail(EB_ERR_INVALID_ARGUMENT, "not a snapshot of this format");
  if (bytes != snapshot_bytes(s) || h.n_rods != static_cast<int64_t>(s->rods.size()) || h.n_slots != s->n_slots ||
      h.config_hash != snapshot_hash(s) || h.sim_flags != s->sim_flags ||
      std::memcmp(h.gravity, s->gravity, sizeof(h.gravity)) != 0)
    return fail(EB_ERR_INVALID_ARGUMENT, "the snapshot was taken from a differently configured simulator");
  p += sizeof(h);
  for (const RodHost& r : s->rods) {
    int64_t n = 0;
    std::memcpy(&n, p, sizeof(n));
    p += sizeof(int64_t);
    if (n != r.n) return fail(EB_ERR_INVALID_ARGUMENT, "the snapshot's rods differ from this simulator's");
  }
  if (eb_status st = set_device(s)) return st;
  const size_t pitch = static_cast<size_t>(s->stride) * sizeof(double);
  const size_t w = static_cast<size_t>(s->n_slots) * sizeof(double);
  EB_CUDA(cudaMemcpy2DAsync(s->d_state[s->cur], pitch, p, w, w, eb::kStateFields, cudaMemcpyHostToDevice,
                            s->stream));
  p += w * eb::kStateFields;
  EB_CUDA(cudaMemcpy2DAsync(s->d_param, pitch, p, w, w, eb::kParamFields, cudaMemcpyHostToDevice, s->stream));
  p += w * eb::kParamFields;
  EB_CUDA(cudaMemcpyAsync(s->d_rods, p, s->rods.size() * sizeof(eb::RodInfo), cudaMemcpyHostToDevice, s->stream));
  EB_CUDA(cudaStreamSynchronize(s->stream));
  s->damper_dt = -1.0;  // the damper factors are refreshed for the next step's dt
  return check_device_status(s);
}

EB_API eb_status eb_debug_set_wait_bound(eb_sim* s, uint32_t polls) {
  if (check_sim(s)) return EB_ERR_INVALID_ARGUMENT;
  s->max_polls = polls;
  drop_graphs(s);  // captured launches hold the bound
  return EB_OK;
}

EB_API eb_status eb_get_stream(const eb_sim* s, void** stream) {
  if (check_sim(s) || !stream) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  *stream = static_cast<void*>(s->stream);
  return EB_OK;
}

EB_API eb_status eb_launch_count(const eb_sim* s, int64_t* count) {
  if (check_sim(s) || !count) return fail(EB_ERR_INVALID_ARGUMENT, "null argument");
  *count = s->launches;
  return EB_OK;
}

}  // extern "C"
