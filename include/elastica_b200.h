/* elastica_b200.h — C-ABI of the B200-native Cosserat-rod step.
 *
 * This is the drop-in boundary for the rod-block update of Elastica++
 * (GazzolaLab/elasticapp).  Each entry point names the reference interface it
 * replaces (paths relative to the reference repository).  All entry points
 * are plain C: pointers and sizes, no C++ or torch types, no exceptions.
 *
 * Conventions
 * - Every function returns an eb_status; on failure eb_last_error() returns
 *   a message for the calling thread.  The reference throws std::logic_error
 *   for use after finalize (elastica/Simulator/Interface/Simulator/
 *   Simulator.hpp:485-509) and std::domain_error for bad parameters
 *   (elastica/Systems/CosseratRods/Initializers/detail/Elasticity.hpp:106-116);
 *   those become EB_ERR_INVALID_STATE and EB_ERR_INVALID_ARGUMENT.
 * - The simulator owns all device memory; the caller owns host buffers.
 * - Calls on one simulator must be serialised by the caller; several
 *   simulators may coexist (one CUDA stream each).
 * - Frames and layouts are the reference's (CosseratRodTraits.hpp:450-468):
 *   per rod, vector fields are 3 x N row-major (row = x, y, z), the director
 *   is 3 x 3 x N page-major (Q[k][j][i] = component j of director d_k of
 *   element i), scalars are N.  Loads are lab frame on nodes; torques,
 *   couples and angular velocities are material frame on elements.
 */
#ifndef ELASTICA_B200_H
#define ELASTICA_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define EB_API __attribute__((visibility("default")))
#else
#define EB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum eb_status {
  EB_OK = 0,
  EB_ERR_INVALID_ARGUMENT = 1,
  EB_ERR_INVALID_STATE = 2,
  EB_ERR_UNSUPPORTED = 3,
  EB_ERR_OUT_OF_MEMORY = 4,
  EB_ERR_CUDA = 5,
  EB_ERR_NOT_FOUND = 6,
  EB_ERR_NUMERICAL = 7
} eb_status;

typedef enum eb_precision {
  /* all arithmetic and state in FP64, as the reference (real_t = double,
   * elastica/Utilities/DefineTypes.h:6) */
  EB_PRECISION_FP64 = 0,
  /* element-local arithmetic in FP32, state accumulation in FP64 */
  EB_PRECISION_MIXED = 1
} eb_precision;

/* eb_config.flags */
#define EB_FLAG_RECORD_DIAGNOSTICS 0x1u /* keep the derived per-element fields
                                           (strains, curvature, loads, ...) of
                                           the last step of every eb_step call */
#define EB_FLAG_REFERENCE_ROUNDING 0x2u /* FP64 step that evaluates every
                                           expression as the reference's
                                           scalar C++ code does, without fused
                                           multiply-adds.  The default build
                                           contracts multiply-adds and uses
                                           rounding-level reformulations
                                           (reciprocals, small-angle series) */

#define EB_FLAG_STEP_STREAMING 0x4u    /* always use the streaming step kernel
                                           (one launch per step, state through
                                           HBM every step) */
#define EB_FLAG_STEP_RESIDENT 0x8u     /* always use a resident configuration
                                           (whole rods kept on chip for up to
                                           128 steps per launch) when the rods
                                           fit; by default the first eb_step
                                           times both and keeps the faster */
#define EB_FLAG_CUDA_GRAPH 0x10u       /* streaming steps (without contact or
                                           connections)
                                           replayed from a captured CUDA graph
                                           of 32 steps: one graph launch
                                           instead of 32 (128 with PEFRL)
                                           kernel launches */
#define EB_FLAG_STEP_BUCKETED 0x20u    /* always use the per-size-bucket
                                           resident plan (rods of at most 263
                                           elements, of 264 to 519 and of 520
                                           to 1039 in separate launches, each
                                           with its fastest configuration)
                                           when the batch has rods of two
                                           sizes, or rods of 520 to 1039
                                           elements, and none longer */

typedef struct eb_config {
  int32_t device;          /* CUDA device ordinal */
  int32_t precision;       /* eb_precision */
  uint32_t flags;          /* EB_FLAG_* */
  int32_t step_window;     /* streaming kernel, slots per CTA: 0 (default) or 128, or 64, 96, 256 */
  int32_t resident_config; /* 0: chosen by timing; c > 0: resident configuration c - 1 */
  int32_t stepper;         /* eb_stepper (0: PositionVerlet) */
} eb_config;

/* Time steppers (elastica/Time/SymplecticSteppers/Algorithms/Types.hpp:31).
 * PositionVerlet follows PositionVerlet.hpp:49-88.  PEFRL is declared but not
 * implemented in the reference; here it is the position-extended
 * Forest-Ruth-like integrator of Omelyan, Mryglod and Folk (Comput. Phys.
 * Commun. 146, 188-202, 2002): four force evaluations per step with
 * xi = 0.1786178958448091, lambda = -0.2123418310626054,
 * chi = -0.06626458266981849, value constraints after every drift and rate
 * constraints after every kick (the damper's factors for the kick's share of
 * dt).  PEFRL runs in FP64, on the streaming kernel (four launches a step)
 * or on the resident kernels (four force evaluations a step on chip), as the
 * step plan chooses. */
typedef enum eb_stepper {
  EB_STEPPER_POSITION_VERLET = 0,
  EB_STEPPER_PEFRL = 1,
  /* VelocityVerlet.hpp:49-87: kick dt/2, drift dt, kick dt/2 (two force
   * evaluations a step), value constraints before and rate constraints
   * after each kick; the analytical damper multiplies by its full-dt factors
   * after each kick, as the reference's rate constraint does.  FP64, on the
   * streaming kernel (two launches a step). */
  EB_STEPPER_VELOCITY_VERLET = 2
} eb_stepper;

/* Rod models (elastica/Systems/CosseratRods/Aliases/CosseratRod.hpp:33-40 and
 * Aliases/CosseratRodWithoutDamping.hpp). */
typedef enum eb_rod_model {
  EB_ROD_DAMPED = 0,  /* CosseratRod: explicit force/torque damping */
  EB_ROD_UNDAMPED = 1 /* CosseratRodWithoutDamping */
} eb_rod_model;

/* Parameters of StraightCosseratRodInitializer
 * (elastica/Systems/CosseratRods/Initializers/StraightCosseratRod.hpp,
 * Initializers/detail/Geometry.hpp:110-214) plus the material entries the
 * rod reads (elastica/Simulator/Materials/Materials.hpp:436-449). */
typedef struct eb_straight_rod {
  int64_t n_elements;
  int32_t model; /* eb_rod_model */
  int32_t reserved;
  double density;
  double youngs_modulus;
  double shear_modulus;
  double radius;
  double length;
  double origin[3];
  double direction[3];
  double normal[3]; /* must be orthogonal to direction */
  double force_damping_rate;  /* EB_ROD_DAMPED only */
  double torque_damping_rate; /* EB_ROD_DAMPED only */
} eb_straight_rod;

/* Rod variables, named after elastica::tags (elastica/Systems/CosseratRods/
 * Tags.hpp).  Shapes per rod with n elements: N = nodes (n+1), E = elements
 * (n), V = Voronoi points (n-1).
 * Settable state and parameters: */
typedef enum eb_field {
  EB_POSITION = 0,                        /* 3 x N */
  EB_VELOCITY = 1,                        /* 3 x N */
  EB_DIRECTOR = 2,                        /* 3 x 3 x E */
  EB_ANGULAR_VELOCITY = 3,                /* 3 x E */
  EB_MASS = 4,                            /* N */
  EB_REFERENCE_ELEMENT_LENGTH = 5,        /* E */
  EB_REFERENCE_VORONOI_LENGTH = 6,        /* V */
  EB_ELEMENT_VOLUME = 7,                  /* E */
  EB_REFERENCE_SHEAR_STRETCH_STRAIN = 8,  /* 3 x E */
  EB_REFERENCE_CURVATURE = 9,             /* 3 x V */
  EB_SHEAR_STRETCH_RIGIDITY_MATRIX = 10,  /* 3 x E (diagonal) */
  EB_BENDING_TWIST_RIGIDITY_MATRIX = 11,  /* 3 x V (diagonal) */
  EB_MASS_SECOND_MOMENT_OF_INERTIA = 12,  /* 3 x E (diagonal) */
  EB_INV_MASS_SECOND_MOMENT_OF_INERTIA = 13, /* 3 x E (diagonal) */
  EB_FORCE_DAMPING_RATE = 14,             /* N (EB_ROD_DAMPED) */
  EB_TORQUE_DAMPING_RATE = 15,            /* E (EB_ROD_DAMPED) */
  /* Derived per-step fields (mid-step values of the last step; need
   * EB_FLAG_RECORD_DIAGNOSTICS).  Setting them is allowed, as in the
   * reference, but the next step overwrites them. */
  EB_ELEMENT_LENGTH = 16,        /* E */
  EB_ELEMENT_DILATATION = 17,    /* E */
  EB_TANGENT = 18,               /* 3 x E */
  EB_VORONOI_DILATATION = 19,    /* V */
  EB_SHEAR_STRETCH_STRAIN = 20,  /* 3 x E */
  EB_CURVATURE = 21,             /* 3 x V */
  EB_INTERNAL_STRESS = 22,       /* 3 x E */
  EB_INTERNAL_COUPLE = 23,       /* 3 x V */
  EB_INTERNAL_LOADS = 24,        /* 3 x N */
  EB_INTERNAL_TORQUES = 25,      /* 3 x E */
  EB_ACCELERATION = 26,          /* 3 x N */
  EB_ANGULAR_ACCELERATION = 27,  /* 3 x E */
  EB_ELEMENT_DIMENSION = 28,     /* E */
  /* collision system (after eb_add_rod_contact), read only: the capsule
   * loads of the last step's contact evaluation, lab frame, per element */
  EB_CONTACT_FORCE = 29,         /* 3 x E */
  EB_CONTACT_TORQUE = 30,        /* 3 x E */
  EB_FIELD_COUNT = 31
} eb_field;

/* Layout of the batch accessors. */
typedef enum eb_layout {
  /* rods concatenated in id order, each in the per-rod layout above */
  EB_LAYOUT_PER_ROD = 0,
  /* the device layout: component-major over slots, component c of slot s at
   * c * eb_slot_count() + s; rod r owns slots [offset[r], offset[r] + n_r] */
  EB_LAYOUT_SLOTS = 1
} eb_layout;

/* --- lifecycle: elastica::make_simulator (Simulator.hpp:1087-1093) ----- */
EB_API eb_status eb_sim_create(const eb_config* config, struct eb_sim** out);
EB_API eb_status eb_sim_destroy(struct eb_sim* sim);
EB_API const char* eb_last_error(void);
EB_API const char* eb_version(void);

/* --- systems: simulator->emplace_back<CosseratRod>(initializer)
 * (elastica/Simulator/Interface/Systems/Module.hpp:898-955).  ids_out
 * receives stable rod handles (0, 1, 2, ... in insertion order). ---------- */
EB_API eb_status eb_emplace_straight_rods(struct eb_sim* sim, const eb_straight_rod* rods,
                                          int64_t count, int64_t* ids_out);
EB_API eb_status eb_rod_count(const struct eb_sim* sim, int64_t* count);
EB_API eb_status eb_rod_elements(const struct eb_sim* sim, int64_t rod, int64_t* n_elements);
EB_API eb_status eb_slot_count(const struct eb_sim* sim, int64_t* n_slots);
/* offsets_out has rod_count + 1 entries */
EB_API eb_status eb_slot_offsets(const struct eb_sim* sim, int64_t* offsets_out, int64_t count);
/* Number of doubles eb_get_field/eb_set_field expect for this rod. */
EB_API eb_status eb_field_size(const struct eb_sim* sim, int64_t rod, int32_t field, int64_t* count);

/* --- variable access: blocks::get<tags::X>(rod_slice) = values
 * (elastica/Systems/Block, used by the reference's golden tests,
 * tests/Unit/Systems/CosseratRods/FullRodTest/Test_PerturbedRodStep.cpp:115-142).
 * Allowed before and after eb_finalize. -------------------------------- */
EB_API eb_status eb_set_field(struct eb_sim* sim, int64_t rod, int32_t field,
                              const double* values, int64_t count);
EB_API eb_status eb_get_field(struct eb_sim* sim, int64_t rod, int32_t field, double* values,
                              int64_t count);
/* All rods at once (after eb_finalize), in the given eb_layout.  For
 * EB_LAYOUT_SLOTS the transfer is one host<->device copy per field; pinned
 * host memory makes it asynchronous-speed. */
EB_API eb_status eb_set_field_batch(struct eb_sim* sim, int32_t field, int32_t layout,
                                    const double* values, int64_t count);
EB_API eb_status eb_get_field_batch(struct eb_sim* sim, int32_t field, int32_t layout,
                                    double* values, int64_t count);

/* --- constraints: simulator->constrain(rod).at(index).with(clamp), the
 * value constraint fixing node index's position x_k and, for index < n,
 * element index's directors Q_k, and the rate constraint zeroing v_k and
 * w_k (elastica/Simulator/Constraints/MakeConstraint.hpp:130-151, 458-494;
 * the generator of examples/dynamic_cantilever/
 * DynamicCantileverCaseStudy.cpp:73-89 applied at .at(index)).  index is a
 * node index, 0..n.  The targets are the node's position and the element's
 * directors at the time of this call (the reference's generator captures
 * them when it is built).  A rod takes at most two clamps (a beam clamped
 * at both ends: indices 0 and n); a third is EB_ERR_UNSUPPORTED, the same
 * index twice EB_ERR_INVALID_STATE. */
EB_API eb_status eb_constrain_clamp(struct eb_sim* sim, int64_t rod, int64_t index);

/* --- environments: GravityField, F_ext += g m
 * (elastica/Simulator/Environments/GravityField/GravityField.hpp:239-246). */
EB_API eb_status eb_add_gravity(struct eb_sim* sim, const double gravity[3]);

/* --- forcing: simulator->force(rod).at(element).with(make_forcing(...))
 * with a constant lab-frame torque applied at one element in the material
 * frame as Q T (elastica/Simulator/Forcing/MakeForcing.hpp:74-165,
 * Forcing.hpp:737-749; examples/axial_stretching/
 * AxialStretchingCaseStudy.cpp:125-134).  Torques added to one rod sum;
 * they act on one element per rod (another element is EB_ERR_UNSUPPORTED).
 * eb_add_end_torque is the same at the last element (n - 1). */
EB_API eb_status eb_add_element_torque(struct eb_sim* sim, int64_t rod, int64_t element,
                                       const double torque_lab[3]);
EB_API eb_status eb_add_end_torque(struct eb_sim* sim, int64_t rod, const double torque_lab[3]);

/* --- rate constraint: the analytical linear damper
 * (examples/fish_swimming/FishModel/Dissipations/AnalyticalLinearDamper.hpp:
 * 15-76): v *= exp(-nu_t dt); w_k *= exp(-nu_r m_e J^-1_k dt)^e. */
EB_API eb_status eb_add_analytical_damper(struct eb_sim* sim, int64_t rod,
                                          double translational_rate, double rotational_rate);

/* --- environments: the collision system (elastica/Simulator/Environments/
 * CollisionSystem, resolved once per dynamic substep, DEMSolver.hpp:701-727).
 * Every element of a participating rod is a capsule (Systems/Customization/
 * CosseratRods/Transfer/Common.hpp:57-93); candidate pairs are the capsule
 * pairs and capsule-plane pairs whose closed bounding boxes overlap
 * (Detection/Coarse/HashGrids.hpp, ExhaustiveSearch.hpp:322-435); the narrow
 * phase is RodCapsuleRodCapsule.hpp:70-186 and CapsulePlane.hpp:60-113; the
 * response is the linear spring-dashpot (Response/DEMForces/
 * LinearSpringDashpot.cpp:32-85); the capsule loads go back to the nodes
 * (half each) and, recast as Q tau, to the element (Transfer/Common.hpp:
 * 32-55), after gravity.  Contact runs on the FP64 streaming step only. */

/* Contact parameters of one material (elastica::create_material,
 * Simulator/Materials/Materials.cpp:237-372).  A pair of materials uses
 * 1 / (1 / a + 1 / b) for stiffness and both dampings and a + b for the
 * friction coefficients (Materials.hpp:1131-1137). */
typedef struct eb_contact_material {
  double stiffness;           /* > 0 */
  double normal_damping;      /* >= 0 */
  double tangential_damping;  /* >= 0 */
  double static_friction;     /* >= 0 */
  double dynamic_friction;    /* >= 0 */
} eb_contact_material;

/* create_material: returns the material id (0, 1, 2, ... in order). */
EB_API eb_status eb_add_contact_material(struct eb_sim* sim, const eb_contact_material* material,
                                         int32_t* material_id);
/* The rod takes part in the collision system with this material (the
 * RodInitializer::Material of the reference's rods). */
EB_API eb_status eb_add_rod_contact(struct eb_sim* sim, int64_t rod, int32_t material_id);
/* An infinite, fixed, double-sided plane through `point` with `normal`
 * (PlanePrimitive, Simulator/Environments/Primitives/PlanePrimitive.cpp:60-130). */
EB_API eb_status eb_add_contact_plane(struct eb_sim* sim, const double point[3], const double normal[3],
                                      int32_t material_id);
/* --- connections (joints) between rods --------------------------------------
 * The reference joins two rods with simulator->connect(rod_a, at(i)).to(rod_b,
 * at(j)).with(generator), the generator holding a user-written force and
 * torque rule applied among the pre-dynamic updates
 * (elastica/Simulator/Connections/Connection.hpp, MakeConnection.hpp).  The
 * rules here are built in, those of the reference's hinge-joint example
 * (examples/hinge_joint/HingeJointCaseStudy.cpp:96-150) with its indices:
 *   every joint: d = x_b[j] - x_a[i + 1], u = d / |d| (0 for d = 0),
 *     F = k d - nu ((v_b[j] - v_a[i + 1]) . u) u; node i + 1 of rod a gains F,
 *     node j of rod b loses it;
 *   EB_JOINT_HINGE also: l = x_b[j + 1] - x_b[j], f = -k_rot (l . n) n,
 *     tau = l x f; element i of rod a loses Q_a tau, element j of rod b gains
 *     Q_b tau (material frame).
 * i must name an element of rod a; j a node of rod b (an element for a
 * hinge).  Connections are evaluated at every force evaluation's drifted
 * state (as the collision system), after gravity and contact; several
 * connections on one node or element are summed in the order they were
 * added.  A simulator with connections steps on the streaming kernel. */
typedef enum eb_joint_kind { EB_JOINT_FREE = 0, EB_JOINT_HINGE = 1 } eb_joint_kind;
typedef struct eb_joint {
  int32_t kind;                /* eb_joint_kind */
  int32_t reserved;
  double stiffness;            /* k */
  double damping;              /* nu, along the separation */
  double rotational_stiffness; /* k_rot (hinge) */
  double normal[3];            /* n (hinge): the direction the hinge resists */
} eb_joint;
EB_API eb_status eb_connect(struct eb_sim* sim, int64_t rod_a, int64_t index_a, int64_t rod_b, int64_t index_b,
                            const eb_joint* joint);

/* Candidate pairs of the last step's contact evaluation: pairs[2 k], pairs[2 k + 1]
 * = (a, b), a < b, sorted; a capsule's id is its element slot (rod r's element
 * i is eb_slot_offsets()[r] + i) and plane p is eb_slot_count() + p.  Writes
 * up to `capacity` pairs and sets *count to the total (the set the
 * reference's coarse detection produces, Detection/Coarse/ExhaustiveSearch.hpp:
 * 322-435).  EB_ERR_INVALID_STATE before the first step. */
EB_API eb_status eb_contact_pairs(struct eb_sim* sim, int64_t* pairs, int64_t capacity, int64_t* count);

/* --- simulator->finalize() (Simulator.hpp:538-578): allocates device
 * memory and uploads the rods.  No rods or constraints may be added after. */
EB_API eb_status eb_finalize(struct eb_sim* sim);

/* --- simulator->step(PositionVerlet, t, dt) repeated n_steps times
 * (elastica/Simulator/Interface/TimeSteppers/SymplecticSteppers.hpp:133-217;
 * elastica/Time/SymplecticSteppers/Algorithms/PositionVerlet.hpp:49-88).
 * *time is advanced by n_steps * dt.  Asynchronous on the simulator's
 * stream; eb_get_* and eb_synchronize wait for it. */
EB_API eb_status eb_step(struct eb_sim* sim, double* time, double dt, int64_t n_steps);
EB_API eb_status eb_synchronize(struct eb_sim* sim);

/* --- one cycle of a host-driven loop: the state set from host memory, then
 * the reference's CaseStudy run_for and communicate()
 * (elastica/Utilities/AppSupport/Python/CaseStudyPybind.hpp:40-110).  Uploads
 * every non-null input (slot layout, ncomp x slot_count doubles, as
 * eb_set_field_batch with EB_LAYOUT_SLOTS), runs n_steps as eb_step and reads
 * every non-null output back (as eb_get_field_batch); the result is the same
 * as those calls in sequence, bit for bit.  An output may be the same buffer
 * as its input.  Under a resident plan (eb_step_plan mode 2 or 3; no contact,
 * connections or recorded diagnostics) the rods are cut into contiguous slot
 * groups whose copies overlap the other groups' launches; with pinned host
 * buffers the cycle then costs about the steps plus one group's copies
 * instead of the steps plus all copies.  Otherwise, and on the call that
 * chooses the plan, the copies and steps run in sequence.  Returns once the
 * outputs are written (asynchronous when there are none). */
typedef struct eb_host_state {
  const double* position_in;         /* 3 x slot_count, or NULL */
  const double* velocity_in;         /* 3 x slot_count, or NULL */
  const double* director_in;         /* 9 x slot_count, or NULL */
  const double* angular_velocity_in; /* 3 x slot_count, or NULL */
  double* position_out;
  double* velocity_out;
  double* director_out;
  double* angular_velocity_out;
} eb_host_state;
EB_API eb_status eb_step_host_state(struct eb_sim* sim, double* time, double dt, int64_t n_steps,
                                    const eb_host_state* host);

/* --- energies (elastica/Systems/CosseratRods/Utility/Energy.hpp:46-141) at
 * the current state: out[4 r + {0,1,2,3}] = translational, rotational,
 * shear/stretch, bend/twist energy of rod r. */
EB_API eb_status eb_energy(struct eb_sim* sim, double* out, int64_t count);

/* The cudaStream_t every kernel and copy of this simulator is issued on, for
 * callers that order their own work or timing events against it. */
EB_API eb_status eb_get_stream(const struct eb_sim* sim, void** stream);

/* --- snapshots (checkpoint / restart) --------------------------------------
 * The reference serialises a finalized simulator (its systems' variables and
 * modules) into an archive and loads it into an identically configured one
 * (elastica/Simulator/Interface/Simulator/Serialize.hpp:19-92).  Here a
 * snapshot is one host buffer: a header, the rods' sizes, the device state and
 * parameter arrays and the per-rod constraint and forcing table.  Loading
 * needs a finalized simulator built with the same rods (sizes, models,
 * contact membership), connections, precision, stepper and environment;
 * anything else is
 * EB_ERR_INVALID_ARGUMENT.  The time is the caller's (eb_step's t). */
EB_API eb_status eb_snapshot_size(const struct eb_sim* sim, uint64_t* bytes);
EB_API eb_status eb_snapshot_save(struct eb_sim* sim, void* buffer, uint64_t bytes);
EB_API eb_status eb_snapshot_load(struct eb_sim* sim, const void* buffer, uint64_t bytes);

/* The step plan chosen by the first eb_step: mode 1 = streaming kernel,
 * 2 = resident kernel with block configuration `config`, 3 = resident kernel
 * per size bucket, one launch per bucket that holds rods: bucket 0 (rods of
 * at most 263 elements) with configuration config % 4, bucket 1 (264 to 519)
 * with (config / 4) % 4, bucket 2 (520 to 1039 elements, each rod on a
 * cluster of two CTAs) with (config / 16) % 4 (0: 512, 1: 256 threads per
 * CTA); config >= 64 means buckets 0 and 1 run packed together, with
 * configuration config / 64 - 1, because that timed faster.
 * probe_ms[0] is the time of 8 streaming steps; probe_ms[1 + c] the predicted
 * time of 8 steps of configuration c on the whole batch, and probe_ms[5 + 4 b
 * + c] on bucket b alone and probe_ms[16 + c] on buckets 0 and 1 together,
 * when run in launches of the first eb_step call's
 * step count (at most 128): resident runs of 8 and 24 steps separate the
 * per-step cost from the launch's fixed staging cost (up to count entries;
 * untimed entries are 0). */
EB_API eb_status eb_step_plan(const struct eb_sim* sim, int32_t* mode, int32_t* config, float* probe_ms,
                              int32_t count);

/* Debug only: the number of polls after which the streaming step kernel's
 * waits for its bulk copies give up (polled without blocking) (0 restores the built-in bound, millions
 * of polls).  A kernel that gives up records it in the simulator's status,
 * waits for the copies it issued and returns; the next call that reads the
 * status (eb_get_field, eb_synchronize, ...) returns EB_ERR_CUDA and the
 * simulator's state is no longer valid.  A bound of 1 makes the first wait
 * run out: it exists to exercise that path without a fault.  No counterpart
 * in the reference. */
EB_API eb_status eb_debug_set_wait_bound(struct eb_sim* sim, uint32_t polls);

/* Number of kernel launches this simulator has issued (diagnostic). */
EB_API eb_status eb_launch_count(const struct eb_sim* sim, int64_t* count);

/* --- multi-GPU: k-way partition of rods by element count (the largest
 * differencing method of elastica/Utilities/KarmarkarKarpPartition.hpp:
 * 332-422), for sharding one batch across GPUs.  part_of[i] in [0, n_parts)
 * receives item i's part; deterministic (ties by creation order). */
EB_API eb_status eb_partition_rods(const int64_t* weights, int64_t n, int32_t n_parts, int32_t* part_of);

/* --- serving: continuous batching of rod-assembly simulations.  No
 * counterpart in the reference (its simulator runs one case study at a time);
 * this is the serving form of the same step.  Requests arrive at any time,
 * are admitted into a device pool of 520-slot bins sized from an HBM budget
 * as bins free up, and every tick advances all admitted requests with one
 * launch of the resident step kernel per precision (steps_per_launch steps
 * each, counted from the request's own admission, so a result does not depend
 * on the other requests).  A finished request's state and energies are copied
 * to host memory on the server's stream and its bins are reused at once;
 * eb_server_poll reports completions without blocking.  Mixed-precision
 * requests whose mechanical energy (kinetic + elastic + gravitational) grows
 * by more than energy_tolerance times a scale (the sum of the initial energy
 * magnitudes plus m |g| L of every rod), or turns non-finite, are rerun in
 * FP64 from their initial conditions.  Rods of
 * a request hold at most 519 elements (one bin). */
typedef struct eb_server_config {
  int32_t device;
  int32_t precision;          /* EB_PRECISION_MIXED (with FP64 fallback) or EB_PRECISION_FP64 */
  int32_t steps_per_launch;   /* 0: 128 */
  uint32_t flags;             /* EB_SERVER_* */
  double hbm_budget_bytes;    /* device pool; 0: 40e9 */
  double energy_tolerance;    /* 0: 1e-3 */
} eb_server_config;

/* every mixed-precision result is treated as failing the energy check (for
 * exercising the FP64 fallback) */
#define EB_SERVER_FORCE_FALLBACK 0x1u

#define EB_REQUEST_CLAMP 0x1u   /* clamp node 0 / element 0 of every rod */
#define EB_REQUEST_DAMPER 0x2u  /* analytical linear damper on every rod */
#define EB_REQUEST_GRAVITY 0x4u /* uniform gravity */

typedef struct eb_request {
  const eb_straight_rod* rods;
  int64_t n_rods;
  const double* velocities;   /* NULL, or per rod 3 x (n + 1) node velocities, concatenated */
  double dt;
  int64_t n_steps;
  double gravity[3];
  uint32_t options;           /* EB_REQUEST_* */
  uint32_t reserved;
  double damper_translational;
  double damper_rotational;
} eb_request;

typedef struct eb_completion {
  int64_t request_id;
  int32_t precision;          /* precision of the delivered result */
  int32_t fell_back;          /* 1: the mixed run failed the energy check and was rerun in FP64 */
  double latency_s;           /* submission to observed completion */
  double energy_initial;
  double energy_final;
  int64_t elements;
  int64_t steps;
  double queued_s;            /* submission to first admission (time spent waiting for bins) */
} eb_completion;

typedef struct eb_server_stats {
  int64_t queued, active, finishing, completed, fallbacks, bins_total, bins_used, ticks;
  double element_steps;
  double kernel_seconds; /* device time of the ticks' step launches that have completed */
} eb_server_stats;

EB_API eb_status eb_server_create(const eb_server_config* config, struct eb_server** out);
EB_API eb_status eb_server_destroy(struct eb_server* server);
EB_API eb_status eb_server_submit(struct eb_server* server, const eb_request* request, int64_t* request_id);
/* admit what fits, launch one tick, enqueue the retirement of the requests it
 * finishes; *in_flight (optional) = queued + active + finishing requests */
EB_API eb_status eb_server_tick(struct eb_server* server, int64_t* in_flight);
EB_API eb_status eb_server_poll(struct eb_server* server, eb_completion* out, int32_t capacity, int32_t* count);
/* final state of rod `rod` of a completed request: EB_POSITION, EB_VELOCITY,
 * EB_DIRECTOR or EB_ANGULAR_VELOCITY, in the per-rod layout of eb_get_field */
EB_API eb_status eb_server_result(struct eb_server* server, int64_t request_id, int64_t rod, int32_t field,
                                  double* values, int64_t count);
EB_API eb_status eb_server_release(struct eb_server* server, int64_t request_id);
EB_API eb_status eb_server_get_stats(const struct eb_server* server, eb_server_stats* out);
/* where a request is: *state 0 queued (not yet admitted), 1 active,
 * 2 finishing, 3 done; *age_s (optional) the time since submission (the
 * latency once done); *queued_s (optional) the time from submission to its
 * first admission, or since submission while it is still queued (a lower
 * bound on its queueing delay) */
#define EB_REQUEST_QUEUED 0
#define EB_REQUEST_ACTIVE 1
#define EB_REQUEST_FINISHING 2
#define EB_REQUEST_DONE 3
EB_API eb_status eb_server_request_status(const struct eb_server* server, int64_t request_id, int32_t* state,
                                          double* age_s, double* queued_s);

/* --- candidate pairs of caller-provided boxes, allocating nothing.  No
 * counterpart in the reference: it is the collision system's broad phase
 * (the search behind eb_contact_pairs) for callers that cannot allocate device
 * memory, for example operators inside a host framework that reserves the
 * whole GPU memory pool and hands them their buffers, or loops that cannot
 * take the device-wide synchronisation of cudaMalloc / cudaFree.  Its working
 * memory is a fixed 16 MiB device array inside the library, held by every GPU
 * that loads it until the process exits.
 *
 * boxes: device pointer, n_boxes boxes of 6 doubles (lo x, lo y, lo z,
 * hi x, hi y, hi z), closed intervals, finite, hi >= lo.  n_boxes <= 131072
 * (larger counts are rejected with EB_ERR_INVALID_ARGUMENT).  The grid's cell
 * edge is the largest box extent: with very uneven extents (one box spanning
 * the others) most boxes share a cell and the search costs up to O(n^2)
 * overlap tests; each box's partners are then sorted in place by one thread,
 * O(cnt^2) for a box with cnt partners.  pairs: device
 * pointer to capacity pairs of int64 (i, j), i < j; the overlapping pairs are
 * written sorted by i then j.  *count (host) receives their number; when it
 * exceeds capacity nothing is written and EB_ERR_INVALID_ARGUMENT is
 * returned.  stream: a cudaStream_t of the current device (NULL = default
 * stream); the call returns after its work on the stream has finished.
 * The first call on a device finds the device address of the working array
 * and keeps it for later calls.  Every call shares that array:
 * calls whose GPU work overlaps (other streams or host threads) race and must
 * be serialised by the caller. */
EB_API eb_status eb_box_pairs_noalloc(const double* boxes, int64_t n_boxes, int64_t* pairs, int64_t capacity,
                                      int64_t* count, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ELASTICA_B200_H */
