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
} OrcRods;

/* Advance every rod by n_steps PositionVerlet steps of size dt.
 * n_threads <= 0 uses all OpenMP threads. */
int orc_step(const OrcRods* rods, double dt, int64_t n_steps, int n_threads);

/* One force evaluation without any time update (the reference's
 * compute_internal_forces + compute_internal_torques + update_acceleration),
 * writing the diagnostics. */
int orc_force_eval(const OrcRods* rods, int n_threads);

/* Energies of each rod at the current state: out[4*r + {0..3}] =
 * translational, rotational, shear/stretch, bend/twist. */
int orc_energy(const OrcRods* rods, double* out, int n_threads);

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
