/* CPU FP64 oracle for the Cosserat-rod PositionVerlet step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain C++ restatement of the
 * reference's scalar kernels (GazzolaLab/elasticapp, "Elastica++"), used by
 * tests/ as the parity checker and by bench.py as the timed CPU baseline.
 * The product (elasticapp_b200, libelastica_b200.so) never links or calls it.
 *
 * Parity pin: tests/test_oracle_golden.py checks this code against the
 * reference's own hex-exact golden vectors (PyElastica FP64 state embedded in
 * tests/Unit/Systems/CosseratRods/FullRodTest/Test_PerturbedRodStep*.cpp),
 * extracted by tests/golden/make_golden.py.
 *
 * Slot layout (shared with the device code, but restated here independently):
 * rod r owns slots [offset[r], offset[r+1]) with offset[r+1]-offset[r] = n_r+1.
 * Node j, element i and Voronoi point k of rod r all live at slot
 * offset[r]+j / +i / +k.  Every field is component-major: component c of a
 * vector field at slot s is field[c*n_slots + s]; director Q(k,j) (director
 * k, lab component j) is Q[(3k+j)*n_slots + s].
 */
#ifndef ELASTICA_B200_ROD_ORACLE_H
#define ELASTICA_B200_ROD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcRods {
  int64_t n_rods;
  int64_t n_slots;
  const int64_t* offset; /* n_rods + 1 */

  /* state (read-write) */
  double* x; /* 3 * S, nodes      */
  double* v; /* 3 * S, nodes      */
  double* Q; /* 9 * S, elements   */
  double* w; /* 3 * S, elements (material frame) */

  /* parameters (read-only) */
  const double* mass;         /* S, nodes            */
  const double* rest_length;  /* S, elements  (l0)   */
  const double* rest_voronoi; /* S, Voronoi   (D0)   */
  const double* volume;       /* S, elements         */
  const double* rest_sigma;   /* 3*S, elements       */
  const double* rest_kappa;   /* 3*S, Voronoi        */
  const double* shear_diag;   /* 3*S, elements  (S)  */
  const double* bend_diag;    /* 3*S, Voronoi   (B)  */
  const double* inertia_diag; /* 3*S, elements  (J diagonal)    */
  const double* inv_inertia;  /* 3*S, elements  (J^-1 diagonal) */
  const double* nu_force;     /* S nodes, NULL => undamped model */
  const double* nu_torque;    /* S elements, NULL => undamped model */

  /* per-rod environment, forcing and constraints (may be NULL) */
  const uint8_t* clamp;       /* n_rods: clamp node 0 / element 0 */
  const double* clamp_x;      /* 3*n_rods  (rod-major: [3r+c])   */
  const double* clamp_Q;      /* 9*n_rods  (rod-major: [9r+3k+j])*/
  const double* end_torque;   /* 3*n_rods lab-frame torque applied at element n-1 */
  const double* damper_nu;    /* 2*n_rods analytical damper (translational, rotational);
                                 both zero => off */
  double gravity[3];

  /* optional diagnostics (mid-step values of the last step; NULL => skip) */
  double* d_length;       /* S elements (reset to e*l0 like the reference) */
  double* d_dilatation;   /* S elements */
  double* d_tangent;      /* 3*S elements */
  double* d_vdilatation;  /* S Voronoi */
  double* d_sigma;        /* 3*S elements */
  double* d_kappa;        /* 3*S Voronoi */
  double* d_stress;       /* 3*S elements (InternalStress n_L) */
  double* d_couple;       /* 3*S Voronoi  (InternalCouple tau_L) */
  double* d_loads;        /* 3*S nodes    (InternalLoads) */
  double* d_torques;      /* 3*S elements (InternalTorques) */
  double* d_accel;        /* 3*S nodes */
  double* d_alpha;        /* 3*S elements */
  double* d_dimension;    /* S elements (radius) */

  /* where the constraints and the forcing act (may be NULL: the clamp at
   * node 0 / element 0 and the torque at element n - 1).  A clamp at index k
   * fixes node k's position and, for k < n, element k's directors
   * (value constraint), and zeroes their velocity and angular velocity
   * (rate constraint), the pattern of DynamicCantileverCaseStudy.cpp:73-89
   * applied at .at(k) (Simulator/Constraints/MakeConstraint.hpp:130-151). */
  const int64_t* clamp_index;  /* 2*n_rods: index of clamp 0 (targets clamp_x, clamp_Q) and of
                                  clamp 1 (targets clamp2_x, clamp2_Q); -1: none */
  const double* clamp2_x;      /* 3*n_rods */
  const double* clamp2_Q;      /* 9*n_rods */
  const int64_t* torque_index; /* n_rods: element end_torque acts on; -1: element n - 1 */
} OrcRods;

/* Advance every rod by n_steps PositionVerlet steps of size dt.
 * n_threads <= 0 uses all OpenMP threads. */
int orc_step(const OrcRods* rods, double dt, int64_t n_steps, int n_threads);

/* n_steps PEFRL steps (declared, not implemented, in the reference;
 * Omelyan, Mryglod and Folk 2002): four force evaluations per step. */
int orc_step_pefrl(const OrcRods* rods, double dt, int64_t n_steps, int n_threads);
/* VelocityVerlet steps (elastica/Time/SymplecticSteppers/Algorithms/VelocityVerlet.hpp:49-87) */
int orc_step_velocity_verlet(const OrcRods* rods, double dt, int64_t n_steps, int n_threads);

/* One force evaluation without any time update (the reference's
 * compute_internal_forces + compute_internal_torques + update_acceleration),
 * writing the diagnostics. */
int orc_force_eval(const OrcRods* rods, int n_threads);

/* Energies of each rod at the current state: out[4*r + {0..3}] =
 * translational, rotational, shear/stretch, bend/twist. */
int orc_energy(const OrcRods* rods, double* out, int n_threads);

/* ---- rod-rod and rod-plane contact (capsule collision system) ----------
 *
 * Every element of a participating rod is a capsule (centre = mid-point of
 * its nodes, length = dilatation * rest length, radius = the element
 * dimension, axis = the tangent).  Capsule ids are element slot indices;
 * plane p has id n_slots + p in pair lists.  Pair lists hold (a, b) with
 * a < b, sorted. */
typedef struct OrcContactMaterial {
  double stiffness, normal_damping, tangential_damping, static_friction, dynamic_friction;
} OrcContactMaterial;

typedef struct OrcContact {
  int32_t n_materials;
  const OrcContactMaterial* materials;
  const int32_t* rod_material; /* n_rods; < 0 => the rod takes no part */
  int32_t n_planes;
  const double* plane_point;   /* 3 * n_planes (row-major [3p+c]) */
  const double* plane_normal;  /* 3 * n_planes */
  const int32_t* plane_material;
  /* per element slot, lab frame, of the last force evaluation (NULL => skip) */
  double* capsule_force;  /* 3*S */
  double* capsule_torque; /* 3*S */
} OrcContact;

/* PositionVerlet steps with the collision system resolved inside every
 * dynamic substep (after the internal forces, after gravity). */
int orc_step_contact(const OrcRods* rods, const OrcContact* contact, double dt, int64_t n_steps,
                     int n_threads);

/* ---- connections (joints) between rods -----------------------------------
 * Connection c joins rod_a at index_a to rod_b at index_b with the joint of
 * the reference's hinge-joint example: kind 0 = translational spring (k) and
 * dashpot along the separation (nu) between node index_a + 1 of rod a and
 * node index_b of rod b; kind 1 adds the rotational spring (k_rot) that
 * penalises the component of rod b's element index_b along `normal`, as a
 * torque on element index_a of rod a and element index_b of rod b. */
typedef struct OrcConnections {
  int64_t n;
  const int64_t* rod_a;
  const int64_t* index_a;
  const int64_t* rod_b;
  const int64_t* index_b;
  const int32_t* kind;
  const double* k;
  const double* nu;
  const double* k_rot;
  const double* normal; /* 3 * n */
} OrcConnections;

/* PositionVerlet steps with the collision system (contact, may be NULL) and
 * the connections (may be NULL) evaluated at the drifted state of every
 * dynamic substep; external loads in the order gravity, contact,
 * connections (forces) and contact, connections, end torque (torques). */
int orc_step_loads(const OrcRods* rods, const OrcContact* contact, const OrcConnections* connections, double dt,
                   int64_t n_steps, int n_threads);

/* Capsules of the current state after a kinematic drift of half_dt (0: as
 * is) and the clamp's value constraint, the way one step would build them:
 * out[k*S + s] for k = 0..14 = centre(3), length, radius, axis(3), AABB
 * min(3), AABB max(3); non-capsule slots are left untouched. */
int orc_contact_capsules(const OrcRods* rods, const OrcContact* contact, double half_dt, double* out);

/* Candidate pairs (closed AABB overlap) of those capsules, from an
 * exhaustive search (exhaustive != 0) or a uniform grid.  Writes up to
 * capacity pairs as (a, b) int64 couples and returns the total count, or -1. */
int64_t orc_contact_pairs(const OrcRods* rods, const OrcContact* contact, double half_dt, int exhaustive,
                          int64_t* pairs, int64_t capacity);

/* Single-pair kernels for the reference's fine-detection and response
 * tests.  A capsule is described by 14 doubles: centre(3), axis(3), radius,
 * length, velocity(3), angular velocity(3) (body frame of the rotation built
 * from the axis); a plane by point(3), normal(3).  Contacts are written as 7
 * doubles each: position(3), normal(3), distance; the return value is their
 * count.  orc_fine_pair_loads applies the spring-dashpot model with pair
 * parameters pm = {k, c_n, c_t, mu_static, mu_dynamic} to every contact of
 * the pair and writes force1(3), torque1(3), force2(3), torque2(3). */
int orc_fine_capsule_capsule(const double* a, const double* b, double* contacts);
int orc_fine_capsule_plane(const double* capsule, const double* plane, double* contacts);
int orc_fine_pair_loads(const double* a, const double* b, const double* pm, double* out);

/* Element kernels of the step, exposed for the reference's kernel tests.
 * A director matrix is 9 doubles q[3 k + j] = component j of director d_k.
 * orc_so3_add_assign: q <- exp(-[u]x) q (SO3PrimitiveAddAssign/Scalar.hpp).
 * orc_inv_rotate_divide: curvature between directors qc and qn divided by
 * span, out[3] (InvRotateDivide/Scalar.hpp). */
int orc_so3_add_assign(double* q, const double* u);
int orc_inv_rotate_divide(const double* qc, const double* qn, double span, double* out);

/* Straight-rod initializer (reference Initializers/detail/Geometry.hpp and the
 * component initialize() chains).  Fills one rod of n elements:
 * x[3*(n+1)], Q[9*n], l0[n], D0[n-1], V[n], radius[n], mass[n+1],
 * J[3*n], Jinv[3*n], S[3*n], B[3*(n-1)], all component-major with stride
 * n (+1 for nodes).  Returns 0, or -1 for invalid input. */
int orc_straight_rod(int64_t n, const double origin[3], const double direction[3],
                     const double normal[3], double length, double radius,
                     double density, double youngs, double shear_modulus,
                     double* x, double* Q, double* l0, double* D0, double* V,
                     double* radius_out, double* mass, double* J, double* Jinv,
                     double* S, double* B);

#ifdef __cplusplus
}
#endif

#endif
