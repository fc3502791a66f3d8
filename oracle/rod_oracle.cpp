// CPU FP64 oracle for the Cosserat-rod PositionVerlet step.
//
// TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); the
// product library never links it.  Every function restates one piece of the
// reference (GazzolaLab/elasticapp) and cites the file:line it follows.
// Paths are relative to the reference's repository root.
//
// Arithmetic follows the reference's *scalar* backends operation by
// operation (same association order), compiled with -ffp-contract=off so no
// fused multiply-adds change the rounding.  Where the reference evaluates a
// quantity over a ghost-padded "block", this code evaluates the same formula
// per rod with explicit zero padding at the rod ends; the reference's ghost
// values (zeroed dummy vectors, zeroed curvature ghosts) make the two equal.
#include "rod_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 {
  double x, y, z;
};

inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }

// elastica/Utilities/Math/BlazeDetail/BlazeLinearAlgebra.hpp (batch_norm):
// sqrt of the component-wise sum of squares.
inline double norm(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

// Traits/Operations/BlazeBackend/LinearAlgebra/CrossProduct/Operation.hpp:58-81
inline V3 cross(V3 m, V3 v) {
  return {m.y * v.z - m.z * v.y, m.z * v.x - m.x * v.z, m.x * v.y - m.y * v.x};
}

// Traits/Operations/BlazeBackend/LinearAlgebra/MatVec/Operation.hpp:24-30 and
// KernelGenerators/MatVec/Scalar.hpp:27-59: out_k = Q(k,0)v0+Q(k,1)v1+Q(k,2)v2.
inline V3 matvec(const double q[9], V3 v) {
  return {q[0] * v.x + q[1] * v.y + q[2] * v.z, q[3] * v.x + q[4] * v.y + q[5] * v.z,
          q[6] * v.x + q[7] * v.y + q[8] * v.z};
}

// Traits/Operations/BlazeBackend/OpsTraits.hpp:166-188 (batch_mattranspvec,
// non-patched branch): out_i = sum over k of Q(k,i) * v_k, summed k = 0,1,2.
inline V3 mattranspvec(const double q[9], V3 v) {
  return {q[0] * v.x + q[3] * v.y + q[6] * v.z, q[1] * v.x + q[4] * v.y + q[7] * v.z,
          q[2] * v.x + q[5] * v.y + q[8] * v.z};
}

struct Field {
  const double* p;
  int64_t S;
  V3 get(int64_t s) const { return {p[s], p[S + s], p[2 * S + s]}; }
};
struct MField {
  double* p;
  int64_t S;
  V3 get(int64_t s) const { return {p[s], p[S + s], p[2 * S + s]}; }
  void set(int64_t s, V3 a) const {
    p[s] = a.x;
    p[S + s] = a.y;
    p[2 * S + s] = a.z;
  }
};

inline void load_q(const double* Q, int64_t S, int64_t s, double q[9]) {
  for (int c = 0; c < 9; ++c) q[c] = Q[c * S + s];
}
inline void store_q(double* Q, int64_t S, int64_t s, const double q[9]) {
  for (int c = 0; c < 9; ++c) Q[c * S + s] = q[c];
}

// Systems/States/Expressions/backends/blaze/SO3PrimitiveAddAssign/Scalar.hpp:41-95
// Q <- exp(-[u]x) Q by Rodrigues' formula with the reference's 1e-14 guard.
// q[3k+j] = Q(k, j).
inline void so3_add_assign(double q[9], V3 uu) {
  double u[3] = {uu.x, uu.y, uu.z};
  const double theta = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  const double c_alpha = std::cos(theta);
  const double alpha = 1.0 - c_alpha;
  const double beta = std::sin(theta);
  for (int d = 0; d < 3; ++d) u[d] /= (theta + 1e-14);
  double out[9];
  for (int j = 0; j < 3; ++j) {
    const double com = q[j] * u[0] + q[3 + j] * u[1] + q[6 + j] * u[2];
    out[j] = c_alpha * q[j] + alpha * u[0] * com + beta * (q[3 + j] * u[2] - q[6 + j] * u[1]);
    out[3 + j] =
        c_alpha * q[3 + j] + alpha * u[1] * com + beta * (q[6 + j] * u[0] - q[j] * u[2]);
    out[6 + j] =
        c_alpha * q[6 + j] + alpha * u[2] * com + beta * (q[j] * u[1] - q[3 + j] * u[0]);
  }
  std::memcpy(q, out, sizeof(out));
}

// Traits/Operations/BlazeBackend/InvRotateDivide/Scalar.hpp:80-105
// Curvature of the Voronoi point between directors qc (element i) and qn
// (element i+1), divided by the rest Voronoi length.
inline V3 inv_rotate_divide(const double qc[9], const double qn[9], double span) {
  const double tr = qc[0] * qn[0] + qc[1] * qn[1] + qc[2] * qn[2] + qc[3] * qn[3] +
                    qc[4] * qn[4] + qc[5] * qn[5] + qc[6] * qn[6] + qc[7] * qn[7] +
                    qc[8] * qn[8];
  const double rest = 0.5 + 1e-10;
  const double theta = std::acos(0.5 * tr - rest);
  const double st = 0.5 * theta / std::sin(theta + 1e-14) / span;
  return {st * (-qc[3] * qn[6] - qc[4] * qn[7] - qc[5] * qn[8] + qc[6] * qn[3] +
                qc[7] * qn[4] + qc[8] * qn[5]),
          st * (qc[0] * qn[6] + qc[1] * qn[7] + qc[2] * qn[8] - qc[6] * qn[0] -
                qc[7] * qn[1] - qc[8] * qn[2]),
          st * (-qc[0] * qn[3] - qc[1] * qn[4] - qc[2] * qn[5] + qc[3] * qn[0] +
                qc[4] * qn[1] + qc[5] * qn[2])};
}

// Per-thread scratch for one rod.
struct Scratch {
  std::vector<double> len, dil, vlen, vdil, sig, kap, stress, couple, fl, tq, g, h, dil_rate;
  std::vector<double> tan;
  void resize(int64_t n) {
    const size_t ne = static_cast<size_t>(n) + 1;
    len.assign(ne, 0.0);
    dil.assign(ne, 0.0);
    vlen.assign(ne, 0.0);
    vdil.assign(ne, 0.0);
    dil_rate.assign(ne, 0.0);
    tan.assign(3 * ne, 0.0);
    sig.assign(3 * ne, 0.0);
    kap.assign(3 * ne, 0.0);
    stress.assign(3 * ne, 0.0);
    couple.assign(3 * ne, 0.0);
    fl.assign(3 * ne, 0.0);
    tq.assign(3 * ne, 0.0);
    g.assign(3 * ne, 0.0);
    h.assign(3 * ne, 0.0);
  }
};

inline V3 getv(const std::vector<double>& a, int64_t i) {
  return {a[3 * i], a[3 * i + 1], a[3 * i + 2]};
}
inline void setv(std::vector<double>& a, int64_t i, V3 v) {
  a[3 * i] = v.x;
  a[3 * i + 1] = v.y;
  a[3 * i + 2] = v.z;
}

// PositionVerlet.hpp:60-69 kinematic substep: x += (0.5 dt) v and the SO3
// exponential update of the directors with u = (0.5 dt) w.
void kinematic_half(const OrcRods& R, int64_t r, double dt) {
  const int64_t S = R.n_slots, o = R.offset[r], n = R.offset[r + 1] - o - 1;
  const double c = 0.5 * dt;
  for (int64_t j = 0; j <= n; ++j) {
    const int64_t s = o + j;
    for (int d = 0; d < 3; ++d) R.x[d * S + s] = R.x[d * S + s] + c * R.v[d * S + s];
  }
  for (int64_t i = 0; i < n; ++i) {
    const int64_t s = o + i;
    double q[9];
    load_q(R.Q, S, s, q);
    so3_add_assign(q, {c * R.w[s], c * R.w[S + s], c * R.w[2 * S + s]});
    store_q(R.Q, S, s, q);
  }
}

// drift by c: x += c v, Q <- exp(-c [w]x) Q (the kinematic substep of a
// symplectic stepper with coefficient c / dt)
void kinematic(const OrcRods& R, int64_t r, double c) {
  const int64_t S = R.n_slots, o = R.offset[r], n = R.offset[r + 1] - o - 1;
  for (int64_t j = 0; j <= n; ++j) {
    const int64_t s = o + j;
    for (int d = 0; d < 3; ++d) R.x[d * S + s] = R.x[d * S + s] + c * R.v[d * S + s];
  }
  for (int64_t i = 0; i < n; ++i) {
    const int64_t s = o + i;
    double q[9];
    load_q(R.Q, S, s, q);
    so3_add_assign(q, {c * R.w[s], c * R.w[S + s], c * R.w[2 * S + s]});
    store_q(R.Q, S, s, q);
  }
}

// index (within the rod) of clamp c of rod r, or -1
int64_t clamp_at(const OrcRods& R, int64_t r, int c) {
  if (!R.clamp || !R.clamp[r]) return -1;
  if (!R.clamp_index) return c == 0 ? 0 : -1;
  return R.clamp_index[2 * r + c];
}

// Value constraint of the clamps (examples/dynamic_cantilever/
// DynamicCantileverCaseStudy.cpp:73-89 at .at(k), applied post-kinematic,
// Simulator/Interface/TimeSteppers/SymplecticSteppers.hpp:174): node k's
// position and, for k < n, element k's directors.
void clamp_values(const OrcRods& R, int64_t r) {
  const int64_t S = R.n_slots, o = R.offset[r], n = R.offset[r + 1] - o - 1;
  for (int c = 0; c < 2; ++c) {
    const int64_t k = clamp_at(R, r, c);
    if (k < 0) continue;
    const double* tx = c == 0 ? R.clamp_x : R.clamp2_x;
    const double* tq = c == 0 ? R.clamp_Q : R.clamp2_Q;
    for (int d = 0; d < 3; ++d) R.x[d * S + o + k] = tx[3 * r + d];
    if (k < n)
      for (int q = 0; q < 9; ++q) R.Q[q * S + o + k] = tq[9 * r + q];
  }
}

// Internal forces and torques of one rod (ElasticityInterface.hpp:360-365),
// then external loads and update_acceleration.  Fills sc.fl (loads, nodes)
// and sc.tq (torques, elements) and the per-element dilatation sc.dil.
// cf, ct: capsule contact force and torque (lab frame, per element slot,
// 3*S) transferred to the rod as in
// Systems/Customization/CosseratRods/Transfer/Common.hpp:32-55, or NULL.
// nf, nt: connection loads (lab frame; node forces and element torques,
// 3*S each), added after the contact loads, or NULL.
void compute_dynamics(const OrcRods& R, int64_t r, Scratch& sc, double* acc, double* alpha,
                      const double* cf = nullptr, const double* ct = nullptr, const double* nf = nullptr,
                      const double* nt = nullptr) {
  const int64_t S = R.n_slots, o = R.offset[r], n = R.offset[r + 1] - o - 1;
  const Field x{R.x, S}, v{R.v, S}, w{R.w, S};
  sc.resize(n);

  // -- compute_shear_strains (CosseratRodCrossSectionInterface.hpp:492-502):
  // update_spanwise_variables (CosseratRodSpanwiseGeometry.hpp:579-622)
  for (int64_t i = 0; i < n; ++i) {
    const V3 dx = sub(x.get(o + i + 1), x.get(o + i));
    const double l = norm(dx);
    sc.len[i] = l;
    // batch_division_matvec: tangent = dx / l (VecScalarDiv/Operation.hpp)
    setv(sc.tan, i, {dx.x / l, dx.y / l, dx.z / l});
    sc.dil[i] = l / R.rest_length[o + i];
  }
  for (int64_t k = 0; k + 1 < n; ++k) {
    // average_kernel (OpsTraits.hpp:262-269): 0.5 * (a_k + a_{k+1})
    sc.vlen[k] = 0.5 * (sc.len[k] + sc.len[k + 1]);
    sc.vdil[k] = sc.vlen[k] / R.rest_voronoi[o + k];
  }
  // compute_cross_sectional_variables (CircleCrossSectionOperations.hpp:110-117)
  if (R.d_dimension)
    for (int64_t i = 0; i < n; ++i)
      R.d_dimension[o + i] = std::sqrt(M_1_PI * R.volume[o + i] / sc.len[i]);
  // update_shear_stretch_strain (CosseratRodSpanwiseGeometry.hpp:630-644):
  // sigma = (Q t) * e - z   (batch_matvec_scale + batch_subtract_z_unit)
  for (int64_t i = 0; i < n; ++i) {
    double q[9];
    load_q(R.Q, S, o + i, q);
    const V3 qt = matvec(q, getv(sc.tan, i));
    const double e = sc.dil[i];
    setv(sc.sig, i, {qt.x * e, qt.y * e, qt.z * e - 1.0});
  }

  // -- compute_internal_modeled_loads_impl
  // (WithDiagonalLinearHyperElasticModel.hpp:198-238)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t s = o + i;
    const V3 sg = getv(sc.sig, i);
    const V3 d = {sg.x - R.rest_sigma[s], sg.y - R.rest_sigma[S + s], sg.z - R.rest_sigma[2 * S + s]};
    const V3 nl = {R.shear_diag[s] * d.x, R.shear_diag[S + s] * d.y, R.shear_diag[2 * S + s] * d.z};
    setv(sc.stress, i, nl);
    double q[9];
    load_q(R.Q, S, s, q);
    const V3 t = mattranspvec(q, nl);
    const double e = sc.dil[i];
    setv(sc.g, i, {t.x / e, t.y / e, t.z / e});  // cosserat internal stress
  }
  // two_point_difference_kernel (Calculus/KernelGenerators/Scalar.hpp:24-60),
  // zero padded at both rod ends.
  for (int64_t j = 0; j <= n; ++j) {
    const V3 a = (j < n) ? getv(sc.g, j) : V3{0.0, 0.0, 0.0};
    const V3 b = (j > 0) ? getv(sc.g, j - 1) : V3{0.0, 0.0, 0.0};
    setv(sc.fl, j, sub(a, b));
  }
  // explicit damping of forces (ExplicitDampingAdapterFacade.hpp:181-200):
  // F -= (m * nu_f) * v
  if (R.nu_force) {
    for (int64_t j = 0; j <= n; ++j) {
      const int64_t s = o + j;
      const double c = R.mass[s] * R.nu_force[s];
      const V3 vv = v.get(s);
      const V3 f = getv(sc.fl, j);
      setv(sc.fl, j, {f.x - c * vv.x, f.y - c * vv.y, f.z - c * vv.z});
    }
  }

  // -- compute_internal_modeled_torques_impl
  // (WithDiagonalLinearHyperElasticModel.hpp:247-391)
  for (int64_t k = 0; k + 1 < n; ++k) {
    double qc[9], qn[9];
    load_q(R.Q, S, o + k, qc);
    load_q(R.Q, S, o + k + 1, qn);
    setv(sc.kap, k, inv_rotate_divide(qc, qn, R.rest_voronoi[o + k]));
  }
  std::vector<double>& cc = sc.h;  // (kappa x couple) * inv_cube * D0
  for (int64_t k = 0; k + 1 < n; ++k) {
    const int64_t s = o + k;
    const V3 kp = getv(sc.kap, k);
    const V3 d = {kp.x - R.rest_kappa[s], kp.y - R.rest_kappa[S + s], kp.z - R.rest_kappa[2 * S + s]};
    const V3 tau = {R.bend_diag[s] * d.x, R.bend_diag[S + s] * d.y, R.bend_diag[2 * S + s] * d.z};
    setv(sc.couple, k, tau);
    const double ed = sc.vdil[k];
    const double ic = 1.0 / (ed * ed * ed);  // OpsTraits.hpp:100-105 inverse_cube
    setv(sc.g, k, {tau.x * ic, tau.y * ic, tau.z * ic});
    const V3 kt = cross(kp, tau);
    const double icd = ic * R.rest_voronoi[s];
    setv(cc, k, {kt.x * icd, kt.y * icd, kt.z * icd});
  }
  for (int64_t i = 0; i < n; ++i) {
    const int64_t s = o + i;
    // two_point_difference of couple * inv_cube (zero padded)
    const V3 a = (i < n - 1) ? getv(sc.g, i) : V3{0.0, 0.0, 0.0};
    const V3 b = (i > 0) ? getv(sc.g, i - 1) : V3{0.0, 0.0, 0.0};
    V3 T = sub(a, b);
    // quadrature_kernel (Calculus/Quadrature/Operation.hpp:23-27): 0.5*(a+b)
    const V3 qa = (i < n - 1) ? getv(cc, i) : V3{0.0, 0.0, 0.0};
    const V3 qb = (i > 0) ? getv(cc, i - 1) : V3{0.0, 0.0, 0.0};
    const V3 qd = {0.5 * (qa.x + qb.x), 0.5 * (qa.y + qb.y), 0.5 * (qa.z + qb.z)};
    T = {T.x + qd.x, T.y + qd.y, T.z + qd.z};
    // shear/stretch couple: (Q t) x n_L * l0
    double q[9];
    load_q(R.Q, S, s, q);
    const V3 qt = matvec(q, getv(sc.tan, i));
    const V3 sc3 = cross(qt, getv(sc.stress, i));
    const double l0 = R.rest_length[s];
    T = {T.x + sc3.x * l0, T.y + sc3.y * l0, T.z + sc3.z * l0};
    // lagrangian transport: (J w / e) x w  (J diagonal)
    const V3 om = w.get(s);
    const double e = sc.dil[i];
    const V3 jw = {R.inertia_diag[s] * om.x, R.inertia_diag[S + s] * om.y,
                   R.inertia_diag[2 * S + s] * om.z};
    const V3 jwe = {jw.x / e, jw.y / e, jw.z / e};
    const V3 lt = cross(jwe, om);
    T = {T.x + lt.x, T.y + lt.y, T.z + lt.z};
    // unsteady dilatation: (J w / e) * (t . dv) / (e * l0)
    const V3 dv = sub(v.get(s + 1), v.get(s));
    const V3 t = getv(sc.tan, i);
    const double rate = (t.x * dv.x + t.y * dv.y + t.z * dv.z) / (e * l0);
    T = {T.x + jwe.x * rate, T.y + jwe.y * rate, T.z + jwe.z * rate};
    // explicit torque damping (ExplicitDampingAdapterFacade.hpp:210-235):
    // T -= (avg(m) * nu_t) * w
    if (R.nu_torque) {
      const double em = 0.5 * (R.mass[s] + R.mass[s + 1]);
      const double c = em * R.nu_torque[s];
      T = {T.x - c * om.x, T.y - c * om.y, T.z - c * om.z};
    }
    setv(sc.tq, i, T);
  }

  // -- external loads (pre-dynamic): gravity
  // (Simulator/Environments/GravityField/GravityField.hpp:239-246) and the
  // end torque forcing (applied in the material frame as Q T_lab,
  // Simulator/Forcing/MakeForcing.hpp), then update_acceleration
  // (Components/Kinematics/WithRodKinematics.hpp:684-714).
  V3 tend = {0.0, 0.0, 0.0};
  const int64_t tk = (R.torque_index && R.torque_index[r] >= 0) ? R.torque_index[r] : n - 1;
  if (R.end_torque) {
    double q[9];
    load_q(R.Q, S, o + tk, q);
    tend = matvec(q, {R.end_torque[3 * r], R.end_torque[3 * r + 1], R.end_torque[3 * r + 2]});
  }
  for (int64_t j = 0; j <= n; ++j) {
    const int64_t s = o + j;
    const double m = R.mass[s];
    V3 fe = {0.0 + R.gravity[0] * m, 0.0 + R.gravity[1] * m, 0.0 + R.gravity[2] * m};
    if (cf) {
      // element j-1 adds half its force to node j first, then element j
      if (j > 0) fe = {fe.x + 0.5 * cf[s - 1], fe.y + 0.5 * cf[S + s - 1], fe.z + 0.5 * cf[2 * S + s - 1]};
      if (j < n) fe = {fe.x + 0.5 * cf[s], fe.y + 0.5 * cf[S + s], fe.z + 0.5 * cf[2 * S + s]};
    }
    if (nf) fe = {fe.x + nf[s], fe.y + nf[S + s], fe.z + nf[2 * S + s]};
    const V3 f = getv(sc.fl, j);
    const double im = 1.0 / m;  // InvMass, WithRodKinematics.hpp:411-424
    const V3 a = {(f.x + fe.x) * im, (f.y + fe.y) * im, (f.z + fe.z) * im};
    acc[3 * j] = a.x;
    acc[3 * j + 1] = a.y;
    acc[3 * j + 2] = a.z;
  }
  for (int64_t i = 0; i < n; ++i) {
    const int64_t s = o + i;
    V3 te = {0.0, 0.0, 0.0};
    if (ct) {
      // the capsule torque recast into the material frame: Q tau
      double q[9];
      load_q(R.Q, S, s, q);
      const V3 tc = matvec(q, {ct[s], ct[S + s], ct[2 * S + s]});
      te = {te.x + tc.x, te.y + tc.y, te.z + tc.z};
    }
    if (nt) {
      // the connections' torque, summed in the lab frame, recast the same way
      double q[9];
      load_q(R.Q, S, s, q);
      const V3 tc = matvec(q, {nt[s], nt[S + s], nt[2 * S + s]});
      te = {te.x + tc.x, te.y + tc.y, te.z + tc.z};
    }
    if (i == tk) te = {te.x + tend.x, te.y + tend.y, te.z + tend.z};
    const V3 T = getv(sc.tq, i);
    const double e = sc.dil[i];
    alpha[3 * i] = (R.inv_inertia[s] * (T.x + te.x)) * e;
    alpha[3 * i + 1] = (R.inv_inertia[S + s] * (T.y + te.y)) * e;
    alpha[3 * i + 2] = (R.inv_inertia[2 * S + s] * (T.z + te.z)) * e;
  }
}

void write_diagnostics(const OrcRods& R, int64_t r, const Scratch& sc, const double* acc,
                       const double* alpha) {
  const int64_t S = R.n_slots, o = R.offset[r], n = R.offset[r + 1] - o - 1;
  auto put3 = [&](double* dst, int64_t s, const double* src) {
    if (!dst) return;
    dst[s] = src[0];
    dst[S + s] = src[1];
    dst[2 * S + s] = src[2];
  };
  for (int64_t i = 0; i < n; ++i) {
    const int64_t s = o + i;
    // the reference resets element_length = dilatation * rest length at the
    // end of the torque computation (WithDiagonalLinearHyperElasticModel.hpp:386-389)
    if (R.d_length) R.d_length[s] = sc.dil[i] * R.rest_length[s];
    if (R.d_dilatation) R.d_dilatation[s] = sc.dil[i];
    put3(R.d_tangent, s, &sc.tan[3 * i]);
    put3(R.d_sigma, s, &sc.sig[3 * i]);
    put3(R.d_stress, s, &sc.stress[3 * i]);
    put3(R.d_torques, s, &sc.tq[3 * i]);
    put3(R.d_alpha, s, &alpha[3 * i]);
  }
  for (int64_t k = 0; k + 1 < n; ++k) {
    const int64_t s = o + k;
    if (R.d_vdilatation) R.d_vdilatation[s] = sc.vdil[k];
    put3(R.d_kappa, s, &sc.kap[3 * k]);
    put3(R.d_couple, s, &sc.couple[3 * k]);
  }
  for (int64_t j = 0; j <= n; ++j) {
    put3(R.d_loads, o + j, &sc.fl[3 * j]);
    put3(R.d_accel, o + j, &acc[3 * j]);
  }
}

// PositionVerlet.hpp:71-77 dynamic substep v += dt a, w += dt alpha, followed
// by the post-dynamic rate constraints: the clamps (v_k = w_k = 0 at each
// clamp index k) and the analytical damper (examples/fish_swimming/
// FishModel/Dissipations/AnalyticalLinearDamper.hpp:15-76, "physical
// version").  damper_dt: the time step the damper's constants were formed
// with (its rate constraint multiplies by exp(-nu damper_dt) after every
// dynamic substep); negative: dt
void dynamic_update(const OrcRods& R, int64_t r, double dt, const Scratch& sc, const double* acc,
                    const double* alpha, double damper_dt = -1.0) {
  const double ddt = damper_dt < 0.0 ? dt : damper_dt;
  const int64_t S = R.n_slots, o = R.offset[r], n = R.offset[r + 1] - o - 1;
  for (int64_t j = 0; j <= n; ++j)
    for (int d = 0; d < 3; ++d) R.v[d * S + o + j] = R.v[d * S + o + j] + dt * acc[3 * j + d];
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) R.w[d * S + o + i] = R.w[d * S + o + i] + dt * alpha[3 * i + d];
  for (int c = 0; c < 2; ++c) {
    const int64_t k = clamp_at(R, r, c);
    if (k < 0) continue;
    for (int d = 0; d < 3; ++d) {
      R.v[d * S + o + k] = 0.0;
      if (k < n) R.w[d * S + o + k] = 0.0;
    }
  }
  if (R.damper_nu && (R.damper_nu[2 * r] != 0.0 || R.damper_nu[2 * r + 1] != 0.0)) {
    const double nut = R.damper_nu[2 * r], nur = R.damper_nu[2 * r + 1];
    const double tcoef = std::exp(-nut * ddt);
    for (int64_t j = 0; j <= n; ++j)
      for (int d = 0; d < 3; ++d) R.v[d * S + o + j] *= tcoef;
    for (int64_t i = 0; i < n; ++i) {
      const int64_t s = o + i;
      double em = 0.5 * (R.mass[s] + R.mass[s + 1]);
      if (i == 0) em += 0.5 * R.mass[s];
      if (i == n - 1) em += 0.5 * R.mass[s + 1];
      for (int d = 0; d < 3; ++d) {
        const double rc = std::exp(-nur * em * R.inv_inertia[d * S + s] * ddt);
        R.w[d * S + s] *= std::pow(rc, sc.dil[i]);
      }
    }
  }
}

int check(const OrcRods* R) {
  if (!R || !R->offset || R->n_rods < 0) return -1;
  for (int64_t r = 0; r < R->n_rods; ++r)
    if (R->offset[r + 1] - R->offset[r] < 3) return -1;  // n >= 2 elements
  return 0;
}

// ---------------------------------------------------------------------------
// Collision system (Simulator/Environments/CollisionSystem): every element of
// a participating rod becomes a capsule, candidate pairs are the capsule
// pairs (and capsule-plane pairs) whose closed axis-aligned bounding boxes
// overlap, the narrow phase generates contact points, a linear
// spring-dashpot turns them into forces and torques on the capsules, and the
// capsule loads are transferred back to the rods' external loads.

constexpr double kContactThreshold = 1e-8;   // Utilities/Thresholds.hpp:138
constexpr double kParallelThreshold = 1e-8;  // Utilities/Thresholds.hpp:159
constexpr double kFrictionThreshold = 1e-8;  // Utilities/Thresholds.hpp:149
// blaze::accuracy for double (Blaze's Limits<double>::accuracy()), the bound
// of is_zero_length (Utilities/Math/Zero.hpp:46-49)
constexpr double kZeroLength = 1e-8;
// default plane spans (Simulator/Environments/Primitives/PlanePrimitive.cpp:63-66)
constexpr double kPlaneSpan = 1e40;

inline double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 add3(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 mul3(double k, V3 a) { return {k * a.x, k * a.y, k * a.z}; }
inline V3 neg3(V3 a) { return {-a.x, -a.y, -a.z}; }
// blaze::normalize: a * (1 / |a|); a zero vector stays zero
inline V3 normalize3(V3 a) {
  const double len = norm(a);
  const double il = len != 0.0 ? 1.0 / len : 0.0;
  return {a.x * il, a.y * il, a.z * il};
}

struct Basis {
  V3 r0, r1, r2;  // rows of the rotation matrix
};

// Utilities/Math/Orthogonal.cpp:32-55 (make_orthogonal_bases_impl): returns
// {v1, normalize(v2), normalize(v3)} for the normalised input v1.
inline void orthogonal_bases(V3 vec, V3& v1, V3& v2n, V3& v3n) {
  v1 = normalize3(vec);
  V3 v2 = {0.8, 0.6, 0.0};
  V3 v3 = cross(v1, v2);
  v2 = cross(v3, v1);
  if (dot3(v2, v2) < kZeroLength) {
    v2 = {0.6, -0.8, 0.0};
    v3 = normalize3(cross(v1, v2));
    v2 = cross(v3, v1);
  }
  v2n = normalize3(v2);
  v3n = normalize3(v3);
}

// Orthogonal.cpp:118-129 make_orthogonal_bases_from_tangent: rows permuted
// {1, 2, 0}, so the tangent is the third row.
inline Basis bases_from_tangent(V3 t) {
  V3 a, b, c;
  orthogonal_bases(t, a, b, c);
  return {b, c, a};
}

// Orthogonal.cpp:85-96 make_orthogonal_bases_from_normal: rows in order.
inline Basis bases_from_normal(V3 n) {
  V3 a, b, c;
  orthogonal_bases(n, a, b, c);
  return {a, b, c};
}

struct Capsule {
  V3 c;       // centre
  double L;   // length
  double r;   // radius
  V3 u;       // axis (third row of the rotation)
  V3 vel;     // translational velocity
  V3 ww;      // angular velocity taken to the world frame, trans(R) w
  double lo[3], hi[3];
  int32_t material;
};

struct Plane {
  V3 p, n;
  double lo[3], hi[3];
  int32_t material;
};

// Rod -> capsule transfer (Systems/Customization/CosseratRods/Transfer/
// Common.hpp:57-93, CapsuleFromRodPrimitive::transfer) and the capsule
// bounding box (Primitives/detail/CapsulePrimitiveBase.cpp:163-180).  x0, x1
// are the (drifted) nodes of the element at slot s.
Capsule make_capsule(const OrcRods& R, int64_t s, V3 x0, V3 x1, int32_t material) {
  const int64_t S = R.n_slots;
  Capsule k;
  const V3 dx = sub(x1, x0);
  const double l = norm(dx);
  const V3 t = {dx.x / l, dx.y / l, dx.z / l};
  const double l0 = R.rest_length[s];
  const double e = l / l0;
  k.L = e * l0;  // element_length = dilatation * rest length after the torques
  k.r = std::sqrt(M_1_PI * R.volume[s] / l);
  k.c = {0.5 * (x0.x + x1.x), 0.5 * (x0.y + x1.y), 0.5 * (x0.z + x1.z)};
  const Basis B = bases_from_tangent(t);
  k.u = B.r2;
  const double m0 = R.mass[s], m1 = R.mass[s + 1];
  const V3 v0 = {R.v[s], R.v[S + s], R.v[2 * S + s]};
  const V3 v1 = {R.v[s + 1], R.v[S + s + 1], R.v[2 * S + s + 1]};
  const V3 num = add3(mul3(m0, v0), mul3(m1, v1));
  const double den = m0 + m1;
  k.vel = {num.x / den, num.y / den, num.z / den};
  const V3 w = {R.w[s], R.w[S + s], R.w[2 * S + s]};
  // RigidBodyPrimitive.hpp:382-393 from_body_FOR_to_world_FOR: trans(Q) * w
  k.ww = {B.r0.x * w.x + B.r1.x * w.y + B.r2.x * w.z, B.r0.y * w.x + B.r1.y * w.y + B.r2.y * w.z,
          B.r0.z * w.x + B.r1.z * w.y + B.r2.z * w.z};
  const double ua[3] = {k.u.x, k.u.y, k.u.z}, ca[3] = {k.c.x, k.c.y, k.c.z};
  for (int d = 0; d < 3; ++d) {
    const double len = std::fabs(ua[d] * k.L) * 0.5 + k.r + kContactThreshold;
    k.lo[d] = ca[d] - len;
    k.hi[d] = ca[d] + len;
  }
  k.material = material;
  return k;
}

// PlanePrimitive.cpp:88-130 (rotation from the normal) and :179-236 (its
// bounding box with the default spans).
Plane make_plane(V3 point, V3 normal, int32_t material) {
  Plane P;
  const Basis B = bases_from_normal(normal);
  P.p = point;
  P.n = B.r0;
  const double b[3] = {B.r1.x, B.r1.y, B.r1.z}, t[3] = {B.r2.x, B.r2.y, B.r2.z};
  const double pa[3] = {point.x, point.y, point.z};
  for (int d = 0; d < 3; ++d) {
    const double len = 0.5 * (std::fabs(b[d] * kPlaneSpan) + std::fabs(t[d] * kPlaneSpan)) + kContactThreshold;
    P.lo[d] = pa[d] - len;
    P.hi[d] = pa[d] + len;
  }
  P.material = material;
  return P;
}

// Detection/Coarse/BoundingBox.hpp:532-540 (closed intervals)
inline bool overlaps(const double alo[3], const double ahi[3], const double blo[3], const double bhi[3]) {
  return !(blo[0] > ahi[0] || blo[1] > ahi[1] || blo[2] > ahi[2] || bhi[0] < alo[0] || bhi[1] < alo[1] ||
           bhi[2] < alo[2]);
}

// Utilities/Geometry/GetClosestLineSegmentPoints.cpp (closest points of the
// segments a1-a2 and b1-b2), branch for branch.
void closest_segment_points(V3 a1, V3 a2, V3 b1, V3 b2, V3& cp1, V3& cp2) {
  const V3 a1a2 = sub(a2, a1), b1b2 = sub(b2, b1), a1b1 = sub(b1, a1);
  const double da1 = dot3(a1a2, a1b1), db1 = dot3(b1b2, a1b1);
  if (da1 <= 0.0 && db1 >= 0.0) {
    cp1 = a1;
    cp2 = b1;
    return;
  }
  const V3 a1b2 = sub(b2, a1);
  const double da2 = dot3(a1a2, a1b2), db2 = dot3(b1b2, a1b2);
  if (da2 <= 0.0 && db2 <= 0.0) {
    cp1 = a1;
    cp2 = b2;
    return;
  }
  const V3 a2b1 = sub(b1, a2);
  const double da3 = dot3(a1a2, a2b1), db3 = dot3(b1b2, a2b1);
  if (da3 >= 0.0 && db3 >= 0.0) {
    cp1 = a2;
    cp2 = b1;
    return;
  }
  const V3 a2b2 = sub(b2, a2);
  const double da4 = dot3(a1a2, a2b2), db4 = dot3(b1b2, a2b2);
  if (da4 >= 0.0 && db4 <= 0.0) {
    cp1 = a2;
    cp2 = b2;
    return;
  }
  const double la = dot3(a1a2, a1a2);
  if (da1 >= -kParallelThreshold && da3 <= kParallelThreshold) {
    const V3 k = mul3(da1 / la, a1a2);
    const V3 n = sub(a1b1, k);
    if (dot3(b1b2, n) >= -kParallelThreshold) {
      cp1 = add3(a1, k);
      cp2 = b1;
      return;
    }
  }
  if (da2 >= -kParallelThreshold && da4 <= kParallelThreshold) {
    const V3 k = mul3(da2 / la, a1a2);
    const V3 n = sub(a1b2, k);
    if (dot3(b1b2, n) <= kParallelThreshold) {
      cp1 = add3(a1, k);
      cp2 = b2;
      return;
    }
  }
  const double lb = dot3(b1b2, b1b2);
  if (db1 <= kParallelThreshold && db2 >= -kParallelThreshold) {
    const V3 k = mul3(-db1 / lb, b1b2);
    const V3 n = sub(neg3(a1b1), k);
    if (dot3(a1a2, n) >= -kParallelThreshold) {
      cp1 = a1;
      cp2 = add3(b1, k);
      return;
    }
  }
  if (db3 <= kParallelThreshold && db4 >= -kParallelThreshold) {
    const V3 k = mul3(-db3 / lb, b1b2);
    const V3 n = sub(neg3(a2b1), k);
    if (dot3(a1a2, n) <= kParallelThreshold) {
      cp1 = a2;
      cp2 = add3(b1, k);
      return;
    }
  }
  const double scale = dot3(a1a2, b1b2);
  double div = la * lb - scale * scale;
  div = 1.0 / div;
  const double sp = (lb * da1 - scale * db1) * div;
  const double tp = (scale * da1 - la * db1) * div;
  cp1 = add3(a1, mul3(sp, a1a2));
  cp2 = add3(b1, mul3(tp, b1b2));
}

struct ContactPoint {
  V3 pos, n;
  double dist;
};

// Detection/Fine/Kernels/RodCapsuleRodCapsule.hpp:70-186; c1 is the capsule
// with the smaller id.  Returns the number of contact points (0, 1 or 2).
int rod_capsule_contacts(const Capsule& c1, const Capsule& c2, ContactPoint out[2]) {
  const V3 up1 = mul3(0.5 * c1.L, c1.u), up2 = mul3(0.5 * c2.L, c2.u);
  V3 cp1, cp2;
  closest_segment_points(add3(c1.c, up1), sub(c1.c, up1), add3(c2.c, up2), sub(c2.c, up2), cp1, cp2);
  V3 nrm = sub(cp1, cp2);
  const double ln = norm(nrm);
  if (ln < kContactThreshold) return 0;
  const double dist = ln - c1.r - c2.r;
  if (!(dist < kContactThreshold)) return 0;
  nrm = normalize3(nrm);
  const double c2x = dot3(c1.u, sub(c2.c, c1.c));
  if ((std::fabs(dot3(c1.u, c2.u)) - 1.0) > -kParallelThreshold && std::fabs(c2x) < c1.L) {
    const double hl1 = 0.5 * c1.L, hl2 = 0.5 * c2.L;
    if (hl1 < c2x + hl2) {
      const double k = c1.r + 0.5 * dist;
      out[0] = {sub(add3(c1.c, up1), mul3(k, nrm)), nrm, dist};
    } else {
      const double k = c2.r + 0.5 * dist;
      out[0] = {add3(add3(c2.c, mul3(hl2, c1.u)), mul3(k, nrm)), nrm, dist};
    }
    if (-hl1 > c2x - hl2) {
      const double k = c1.r + 0.5 * dist;
      out[1] = {sub(sub(c1.c, up1), mul3(k, nrm)), nrm, dist};
    } else {
      const double k = c2.r + 0.5 * dist;
      out[1] = {add3(sub(c2.c, mul3(hl2, c1.u)), mul3(k, nrm)), nrm, dist};
    }
    return 2;
  }
  const double k = c2.r + 0.5 * dist;
  out[0] = {add3(cp2, mul3(k, nrm)), nrm, dist};
  return 1;
}

// Detection/Fine/Kernels/CapsulePlane.hpp:60-113
int capsule_plane_contacts(const Capsule& c, const Plane& p, ContactPoint out[2]) {
  const V3 up = mul3(0.5 * c.L, c.u);
  const V3 pu = add3(c.c, up), pl = sub(c.c, up);
  const double du = std::fabs(dot3(p.n, sub(pu, p.p))) - c.r;
  const double dl = std::fabs(dot3(p.n, sub(pl, p.p))) - c.r;
  int k = 0;
  if (du < kContactThreshold) out[k++] = {sub(pu, mul3(c.r + du, p.n)), p.n, du};
  if (dl < kContactThreshold) out[k++] = {sub(pl, mul3(c.r + dl, p.n)), p.n, dl};
  return k;
}

struct PairMaterial {
  double k, cn, ct, mu_s, mu_d;
};

// Simulator/Materials/Materials.hpp:1131-1137 and the damping analogues
// (series rule), Materials.cpp:346-372 (pair friction = sum of the two)
PairMaterial pair_material(const OrcContact& C, int32_t m1, int32_t m2) {
  const OrcContactMaterial& a = C.materials[m1];
  const OrcContactMaterial& b = C.materials[m2];
  PairMaterial pm;
  pm.k = 1.0 / (1.0 / a.stiffness + 1.0 / b.stiffness);
  pm.cn = 1.0 / (1.0 / a.normal_damping + 1.0 / b.normal_damping);
  pm.ct = 1.0 / (1.0 / a.tangential_damping + 1.0 / b.tangential_damping);
  pm.mu_s = a.static_friction + b.static_friction;
  pm.mu_d = a.dynamic_friction + b.dynamic_friction;
  return pm;
}

// velocity of a capsule's material point at pos (RigidBodyPrimitive.hpp:451-465)
inline V3 point_velocity(const Capsule& k, V3 pos) { return add3(k.vel, cross(k.ww, sub(pos, k.c))); }

// Contact.cpp:150-215 (relative velocity, friction coefficient choice) and
// Response/DEMForces/LinearSpringDashpot.cpp:32-85.  rvel is the relative
// velocity of body 1 against body 2 at the contact point.  Returns false for
// a separated contact (no force).
bool spring_dashpot(const ContactPoint& ct, V3 rvel, const PairMaterial& pm, V3& net) {
  if (!(ct.dist < -kContactThreshold)) return false;
  const V3 n = ct.n;
  const double rvn = dot3(n, rvel);
  const double rvt = dot3(n, sub(rvel, mul3(rvn, n)));
  const double mu = std::fabs(rvt) > kFrictionThreshold ? pm.mu_d : pm.mu_s;
  const double delta = -ct.dist;
  const double relvn = -dot3(n, rvel);
  const V3 relv = neg3(rvel);
  const V3 relvt = sub(relv, mul3(relvn, n));
  const double fn = std::max(0.0, pm.k * delta + pm.cn * relvn);
  const V3 fN = mul3(fn, n);
  const double ft = std::min(pm.ct * norm(relvt), mu * fn);
  const V3 fT = mul3(ft, normalize3(relvt));
  net = add3(fN, fT);
  return true;
}

struct ContactWorld {
  std::vector<Capsule> caps;      // by slot (only element slots of participating rods used)
  std::vector<uint8_t> is_cap;    // by slot
  std::vector<int64_t> cap_ids;   // participating element slots, ascending
  std::vector<Plane> planes;
};

// capsules of the current R.x (already drifted) for every participating rod
void build_capsules(const OrcRods& R, const OrcContact& C, ContactWorld& W, const double* x) {
  const int64_t S = R.n_slots;
  W.caps.resize(S);
  W.is_cap.assign(S, 0);
  W.cap_ids.clear();
  for (int64_t r = 0; r < R.n_rods; ++r) {
    const int32_t mat = C.rod_material ? C.rod_material[r] : -1;
    if (mat < 0) continue;
    const int64_t o = R.offset[r], n = R.offset[r + 1] - o - 1;
    for (int64_t i = 0; i < n; ++i) {
      const int64_t s = o + i;
      const V3 x0 = {x[s], x[S + s], x[2 * S + s]};
      const V3 x1 = {x[s + 1], x[S + s + 1], x[2 * S + s + 1]};
      W.caps[s] = make_capsule(R, s, x0, x1, mat);
      W.is_cap[s] = 1;
      W.cap_ids.push_back(s);
    }
  }
  W.planes.clear();
  for (int32_t p = 0; p < C.n_planes; ++p)
    W.planes.push_back(make_plane({C.plane_point[3 * p], C.plane_point[3 * p + 1], C.plane_point[3 * p + 2]},
                                  {C.plane_normal[3 * p], C.plane_normal[3 * p + 1], C.plane_normal[3 * p + 2]},
                                  C.plane_material[p]));
}

// Exhaustive search (Detection/Coarse/ExhaustiveSearch.hpp:322-435) over the
// capsules in id order, then every capsule against every plane.
void pairs_exhaustive(const OrcRods& R, const ContactWorld& W, std::vector<int64_t>& pairs) {
  pairs.clear();
  const size_t N = W.cap_ids.size();
  for (size_t i = 0; i < N; ++i) {
    const Capsule& a = W.caps[W.cap_ids[i]];
    for (size_t j = i + 1; j < N; ++j) {
      const Capsule& b = W.caps[W.cap_ids[j]];
      if (overlaps(a.lo, a.hi, b.lo, b.hi)) {
        pairs.push_back(W.cap_ids[i]);
        pairs.push_back(W.cap_ids[j]);
      }
    }
    for (size_t p = 0; p < W.planes.size(); ++p)
      if (overlaps(a.lo, a.hi, W.planes[p].lo, W.planes[p].hi)) {
        pairs.push_back(W.cap_ids[i]);
        pairs.push_back(R.n_slots + static_cast<int64_t>(p));
      }
  }
}

// The same pair set from a uniform grid: cell edge above the largest box
// extent, each capsule filed under the cell of its box's lower corner, every
// capsule tested against the capsules of its 27 neighbouring cells.  Two
// overlapping boxes have lower corners less than one cell apart on every
// axis, so the set equals the exhaustive one (the property the reference
// tests for its hash grids, Test_HashGrids.cpp).
void pairs_grid(const OrcRods& R, const ContactWorld& W, std::vector<int64_t>& pairs) {
  pairs.clear();
  const size_t N = W.cap_ids.size();
  double h = 0.0;
  for (int64_t s : W.cap_ids)
    for (int d = 0; d < 3; ++d) h = std::max(h, W.caps[s].hi[d] - W.caps[s].lo[d]);
  h = h * (1.0 + 1.0 / 1048576.0);
  if (!(h > 0.0)) h = 1.0;
  const double ih = 1.0 / h;
  auto cell = [&](const Capsule& k, int d) {
    double c = std::floor(k.lo[d] * ih);
    c = std::min(std::max(c, -1073741824.0), 1073741824.0);
    return static_cast<int64_t>(c);
  };
  auto key = [](int64_t a, int64_t b, int64_t c) {
    return (static_cast<uint64_t>(a + (1ll << 31)) << 42) ^ (static_cast<uint64_t>(b + (1ll << 31)) << 21) ^
           static_cast<uint64_t>(c + (1ll << 31));
  };
  std::vector<std::array<int64_t, 3>> cells(N);
  std::unordered_map<uint64_t, std::vector<int64_t>> grid;
  grid.reserve(2 * N + 1);
  for (size_t i = 0; i < N; ++i) {
    const Capsule& k = W.caps[W.cap_ids[i]];
    cells[i] = {cell(k, 0), cell(k, 1), cell(k, 2)};
  }
  for (size_t i = 0; i < N; ++i) grid[key(cells[i][0], cells[i][1], cells[i][2])].push_back(static_cast<int64_t>(i));
  std::vector<int64_t> found;
  for (size_t i = 0; i < N; ++i) {
    const Capsule& a = W.caps[W.cap_ids[i]];
    found.clear();
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int64_t cx = cells[i][0] + dx, cy = cells[i][1] + dy, cz = cells[i][2] + dz;
          auto it = grid.find(key(cx, cy, cz));
          if (it == grid.end()) continue;
          for (int64_t j : it->second) {
            if (static_cast<size_t>(j) <= i) continue;
            if (cells[j][0] != cx || cells[j][1] != cy || cells[j][2] != cz) continue;
            const Capsule& b = W.caps[W.cap_ids[j]];
            if (overlaps(a.lo, a.hi, b.lo, b.hi)) found.push_back(W.cap_ids[j]);
          }
        }
    std::sort(found.begin(), found.end());
    for (int64_t b : found) {
      pairs.push_back(W.cap_ids[i]);
      pairs.push_back(b);
    }
    for (size_t p = 0; p < W.planes.size(); ++p)
      if (overlaps(a.lo, a.hi, W.planes[p].lo, W.planes[p].hi)) {
        pairs.push_back(W.cap_ids[i]);
        pairs.push_back(R.n_slots + static_cast<int64_t>(p));
      }
  }
}

// Narrow phase and response for every capsule over its partners in
// ascending id order (capsules, then planes), each pair evaluated with the
// smaller id as the first body; then the loads per capsule (lab frame).
void contact_loads(const OrcRods& R, const OrcContact& C, const ContactWorld& W, const std::vector<int64_t>& pairs,
                   double* cf, double* ct, int nt) {
  const int64_t S = R.n_slots;
  std::vector<std::vector<int64_t>> adj(S);
  for (size_t k = 0; k < pairs.size(); k += 2) {
    adj[pairs[k]].push_back(pairs[k + 1]);
    if (pairs[k + 1] < S) adj[pairs[k + 1]].push_back(pairs[k]);
  }
  for (int64_t s = 0; s < S; ++s) std::sort(adj[s].begin(), adj[s].end());
  const int64_t nc = static_cast<int64_t>(W.cap_ids.size());
  (void)nt;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt)
#endif
  for (int64_t q = 0; q < nc; ++q) {
    const int64_t s = W.cap_ids[q];
    const Capsule& me = W.caps[s];
    V3 F = {0.0, 0.0, 0.0}, T = {0.0, 0.0, 0.0};
    ContactPoint pts[2];
    for (int64_t o : adj[s]) {
      if (o < S) {
        const bool first = s < o;
        const Capsule& c1 = first ? me : W.caps[o];
        const Capsule& c2 = first ? W.caps[o] : me;
        const PairMaterial pm = pair_material(C, c1.material, c2.material);
        const int np = rod_capsule_contacts(c1, c2, pts);
        for (int k = 0; k < np; ++k) {
          const V3 rvel = sub(point_velocity(c1, pts[k].pos), point_velocity(c2, pts[k].pos));
          V3 net;
          if (!spring_dashpot(pts[k], rvel, pm, net)) continue;
          // Primitives/RigidBodyPrimitive.hpp:500-504 add_force_at_position
          const V3 f = first ? net : neg3(net);
          F = add3(F, f);
          T = add3(T, cross(sub(pts[k].pos, me.c), f));
        }
      } else {
        const Plane& P = W.planes[o - S];
        const PairMaterial pm = pair_material(C, me.material, P.material);
        const int np = capsule_plane_contacts(me, P, pts);
        for (int k = 0; k < np; ++k) {
          // the plane is fixed: zero velocity
          const V3 rvel = sub(point_velocity(me, pts[k].pos), V3{0.0, 0.0, 0.0});
          V3 net;
          if (!spring_dashpot(pts[k], rvel, pm, net)) continue;
          F = add3(F, net);
          T = add3(T, cross(sub(pts[k].pos, me.c), net));
        }
      }
    }
    cf[s] = F.x;
    cf[S + s] = F.y;
    cf[2 * S + s] = F.z;
    ct[s] = T.x;
    ct[S + s] = T.y;
    ct[2 * S + s] = T.z;
  }
}

int check_contact(const OrcRods& R, const OrcContact* C) {
  if (!C) return -1;
  if (C->n_materials < 0 || (C->n_materials > 0 && !C->materials)) return -1;
  if (C->n_planes < 0 || (C->n_planes > 0 && (!C->plane_point || !C->plane_normal || !C->plane_material)))
    return -1;
  for (int64_t r = 0; r < R.n_rods; ++r)
    if (C->rod_material && C->rod_material[r] >= C->n_materials) return -1;
  for (int32_t p = 0; p < C->n_planes; ++p)
    if (C->plane_material[p] < 0 || C->plane_material[p] >= C->n_materials) return -1;
  return 0;
}

// ---- connections between rods -------------------------------------------
// The joints of the reference's hinge-joint example
// (examples/hinge_joint/HingeJointCaseStudy.cpp:96-150), connecting rod a at
// index i to rod b at index j:
//   force:  d = x_b[j] - x_a[i + 1];  F = k d - nu ((v_b[j] - v_a[i + 1]) . u) u,
//           u = d / |d| (Blaze's normalize: d times 1/|d|, or d times 0 for
//           |d| = 0);  rod a's node i + 1 gains F, rod b's node j loses it;
//   torque (hinge only): l = x_b[j + 1] - x_b[j];  f = -k_rot (l . n) n;
//           tau = l x f;  rod a's element i loses Q_a tau, rod b's element j
//           gains Q_b tau (material frame).
// Loads are summed per slot in connection order, each connection adding to
// rod a before rod b; torques are summed in the lab frame and recast by the
// element's directors in compute_dynamics.
void connection_loads(const OrcRods& R, const OrcConnections& C, double* nf, double* nt) {
  const int64_t S = R.n_slots;
  std::fill(nf, nf + 3 * S, 0.0);
  std::fill(nt, nt + 3 * S, 0.0);
  const Field x{R.x, S}, v{R.v, S};
  auto add = [&](double* a, int64_t s, V3 f, bool minus) {
    if (minus) {
      a[s] = a[s] - f.x;
      a[S + s] = a[S + s] - f.y;
      a[2 * S + s] = a[2 * S + s] - f.z;
    } else {
      a[s] = a[s] + f.x;
      a[S + s] = a[S + s] + f.y;
      a[2 * S + s] = a[2 * S + s] + f.z;
    }
  };
  for (int64_t c = 0; c < C.n; ++c) {
    const int64_t na = R.offset[C.rod_a[c]] + C.index_a[c] + 1, nb = R.offset[C.rod_b[c]] + C.index_b[c];
    const V3 d = sub(x.get(nb), x.get(na));
    const double k = C.k[c], nu = C.nu[c];
    const V3 fel = {k * d.x, k * d.y, k * d.z};
    const double len = std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
    const double il = len != 0.0 ? 1.0 / len : len;
    const V3 u = {d.x * il, d.y * il, d.z * il};
    const V3 dv = sub(v.get(nb), v.get(na));
    const double vr = dv.x * u.x + dv.y * u.y + dv.z * u.z;
    const V3 vel = {vr * u.x, vr * u.y, vr * u.z};
    const double mnu = -nu;
    const V3 F = {fel.x + mnu * vel.x, fel.y + mnu * vel.y, fel.z + mnu * vel.z};
    add(nf, na, F, false);
    add(nf, nb, F, true);
    if (C.kind[c] == 1) {
      const V3 l = sub(x.get(nb + 1), x.get(nb));
      const V3 n = {C.normal[3 * c], C.normal[3 * c + 1], C.normal[3 * c + 2]};
      const double s = (-C.k_rot[c]) * (l.x * n.x + l.y * n.y + l.z * n.z);
      const V3 f = {s * n.x, s * n.y, s * n.z};
      const V3 tau = {l.y * f.z - l.z * f.y, l.z * f.x - l.x * f.z, l.x * f.y - l.y * f.x};
      add(nt, na - 1, tau, true);
      add(nt, nb, tau, false);
    }
  }
}

int check_connections(const OrcRods& R, const OrcConnections* C) {
  if (!C) return 0;
  for (int64_t c = 0; c < C->n; ++c) {
    const int64_t ra = C->rod_a[c], rb = C->rod_b[c];
    if (ra < 0 || ra >= R.n_rods || rb < 0 || rb >= R.n_rods) return -1;
    const int64_t na = R.offset[ra + 1] - R.offset[ra] - 1, nb = R.offset[rb + 1] - R.offset[rb] - 1;
    if (C->index_a[c] < 0 || C->index_a[c] >= na || C->index_b[c] < 0) return -1;
    if (C->kind[c] == 1 ? C->index_b[c] >= nb : C->index_b[c] > nb) return -1;
  }
  return 0;
}

// positions after a drift of c and the clamp's value constraint (a copy)
std::vector<double> drifted_positions(const OrcRods& R, double c) {
  const int64_t S = R.n_slots;
  std::vector<double> x(R.x, R.x + 3 * S);
  for (int64_t i = 0; i < 3 * S; ++i) x[i] = x[i] + c * R.v[i];
  for (int64_t r = 0; r < R.n_rods; ++r)
    for (int c = 0; c < 2; ++c) {
      const int64_t k = clamp_at(R, r, c);
      if (k < 0) continue;
      const double* tx = c == 0 ? R.clamp_x : R.clamp2_x;
      for (int d = 0; d < 3; ++d) x[d * S + R.offset[r] + k] = tx[3 * r + d];
    }
  return x;
}

}  // namespace

extern "C" int orc_step(const OrcRods* rods, double dt, int64_t n_steps, int n_threads) {
  if (check(rods) != 0) return -1;
  const OrcRods& R = *rods;
#ifdef _OPENMP
  const int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
  {
    Scratch sc;
    std::vector<double> acc, alpha;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int64_t r = 0; r < R.n_rods; ++r) {
      const int64_t n = R.offset[r + 1] - R.offset[r] - 1;
      acc.assign(3 * (n + 1), 0.0);
      alpha.assign(3 * (n + 1), 0.0);
      // Simulator::step substep order (SymplecticSteppers.hpp:152-216):
      // [Kinematic(1/2), t+=dt/2, Dynamic, t+=dt/2, Kinematic(1/2)]
      for (int64_t step = 0; step < n_steps; ++step) {
        kinematic_half(R, r, dt);
        clamp_values(R, r);
        compute_dynamics(R, r, sc, acc.data(), alpha.data());
        if (step == n_steps - 1) write_diagnostics(R, r, sc, acc.data(), alpha.data());
        dynamic_update(R, r, dt, sc, acc.data(), alpha.data());
        kinematic_half(R, r, dt);
      }
    }
  }
  (void)n_threads;
  return 0;
}

extern "C" int orc_step_contact(const OrcRods* rods, const OrcContact* contact, double dt, int64_t n_steps,
                                int n_threads) {
  if (!contact) return -1;
  return orc_step_loads(rods, contact, nullptr, dt, n_steps, n_threads);
}

extern "C" int orc_step_loads(const OrcRods* rods, const OrcContact* contact, const OrcConnections* conns,
                              double dt, int64_t n_steps, int n_threads) {
  if (check(rods) != 0) return -1;
  const OrcRods& R = *rods;
  if (contact && check_contact(R, contact) != 0) return -1;
  if (check_connections(R, conns) != 0) return -1;
  const bool has_conn = conns && conns->n > 0;
#ifdef _OPENMP
  const int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#else
  const int nt = 1;
#endif
  const int64_t S = R.n_slots;
  std::vector<double> cf(3 * S, 0.0), ct(3 * S, 0.0), jf, jt;  // contact; connection loads
  if (has_conn) {
    jf.assign(3 * S, 0.0);
    jt.assign(3 * S, 0.0);
  }
  ContactWorld W;
  std::vector<int64_t> pairs;
  for (int64_t step = 0; step < n_steps; ++step) {
    // kinematic half step and value constraints of every rod first: the
    // collision system sees all rods at the drifted state
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt)
#endif
    for (int64_t r = 0; r < R.n_rods; ++r) {
      kinematic_half(R, r, dt);
      clamp_values(R, r);
    }
    if (contact) {
      const OrcContact& C = *contact;
      build_capsules(R, C, W, R.x);
      pairs_grid(R, W, pairs);
      contact_loads(R, C, W, pairs, cf.data(), ct.data(), nt);
      if (step == n_steps - 1 && C.capsule_force && C.capsule_torque) {
        std::copy(cf.begin(), cf.end(), C.capsule_force);
        std::copy(ct.begin(), ct.end(), C.capsule_torque);
      }
    }
    if (has_conn) connection_loads(R, *conns, jf.data(), jt.data());
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
    {
      Scratch sc;
      std::vector<double> acc, alpha;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
      for (int64_t r = 0; r < R.n_rods; ++r) {
        const int64_t n = R.offset[r + 1] - R.offset[r] - 1;
        acc.assign(3 * (n + 1), 0.0);
        alpha.assign(3 * (n + 1), 0.0);
        compute_dynamics(R, r, sc, acc.data(), alpha.data(), contact ? cf.data() : nullptr,
                         contact ? ct.data() : nullptr, has_conn ? jf.data() : nullptr,
                         has_conn ? jt.data() : nullptr);
        if (step == n_steps - 1) write_diagnostics(R, r, sc, acc.data(), alpha.data());
        dynamic_update(R, r, dt, sc, acc.data(), alpha.data());
        kinematic_half(R, r, dt);
      }
    }
  }
  return 0;
}

extern "C" int orc_contact_capsules(const OrcRods* rods, const OrcContact* contact, double half_dt, double* out) {
  if (check(rods) != 0 || !out) return -1;
  const OrcRods& R = *rods;
  if (check_contact(R, contact) != 0) return -1;
  const int64_t S = R.n_slots;
  const std::vector<double> x = drifted_positions(R, half_dt);
  ContactWorld W;
  build_capsules(R, *contact, W, x.data());
  for (int64_t s : W.cap_ids) {
    const Capsule& k = W.caps[s];
    const double vals[15] = {k.c.x, k.c.y, k.c.z, k.L, k.r, k.u.x, k.u.y, k.u.z,
                             k.lo[0], k.lo[1], k.lo[2], k.hi[0], k.hi[1], k.hi[2], 0.0};
    for (int f = 0; f < 14; ++f) out[f * S + s] = vals[f];
  }
  return 0;
}

extern "C" int64_t orc_contact_pairs(const OrcRods* rods, const OrcContact* contact, double half_dt, int exhaustive,
                                     int64_t* pairs, int64_t capacity) {
  if (check(rods) != 0) return -1;
  const OrcRods& R = *rods;
  if (check_contact(R, contact) != 0) return -1;
  const std::vector<double> x = drifted_positions(R, half_dt);
  ContactWorld W;
  build_capsules(R, *contact, W, x.data());
  std::vector<int64_t> p;
  if (exhaustive)
    pairs_exhaustive(R, W, p);
  else
    pairs_grid(R, W, p);
  const int64_t n = static_cast<int64_t>(p.size() / 2);
  for (int64_t k = 0; k < std::min(n, capacity); ++k) {
    pairs[2 * k] = p[2 * k];
    pairs[2 * k + 1] = p[2 * k + 1];
  }
  return n;
}

namespace {
Capsule capsule_from_desc(const double* d) {
  Capsule k;
  k.c = {d[0], d[1], d[2]};
  const Basis B = bases_from_tangent({d[3], d[4], d[5]});
  k.u = B.r2;
  k.r = d[6];
  k.L = d[7];
  k.vel = {d[8], d[9], d[10]};
  const V3 w = {d[11], d[12], d[13]};
  k.ww = {B.r0.x * w.x + B.r1.x * w.y + B.r2.x * w.z, B.r0.y * w.x + B.r1.y * w.y + B.r2.y * w.z,
          B.r0.z * w.x + B.r1.z * w.y + B.r2.z * w.z};
  k.material = 0;
  return k;
}
void put_contacts(const ContactPoint* pts, int n, double* out) {
  for (int i = 0; i < n; ++i) {
    const double v[7] = {pts[i].pos.x, pts[i].pos.y, pts[i].pos.z, pts[i].n.x, pts[i].n.y, pts[i].n.z,
                         pts[i].dist};
    for (int k = 0; k < 7; ++k) out[7 * i + k] = v[k];
  }
}
}  // namespace

/* Single-element kernels for the reference's own kernel tests
 * (tests/Unit/Systems/States/Expressions/SO3/Test_SO3PrimitiveAddAssign.cpp,
 * tests/Unit/Systems/CosseratRods/Traits/Operations/BlazeBackend/Test_InvRotateDivide_Scalar.cpp):
 * the same so3_add_assign and inv_rotate_divide the step uses. */
extern "C" int orc_so3_add_assign(double* q, const double* u) {
  so3_add_assign(q, {u[0], u[1], u[2]});
  return 0;
}

extern "C" int orc_inv_rotate_divide(const double* qc, const double* qn, double span, double* out) {
  const V3 k = inv_rotate_divide(qc, qn, span);
  out[0] = k.x;
  out[1] = k.y;
  out[2] = k.z;
  return 0;
}

extern "C" int orc_fine_capsule_capsule(const double* a, const double* b, double* contacts) {
  ContactPoint pts[2];
  const int n = rod_capsule_contacts(capsule_from_desc(a), capsule_from_desc(b), pts);
  if (contacts) put_contacts(pts, n, contacts);
  return n;
}

extern "C" int orc_fine_capsule_plane(const double* capsule, const double* plane, double* contacts) {
  ContactPoint pts[2];
  const Plane P = make_plane({plane[0], plane[1], plane[2]}, {plane[3], plane[4], plane[5]}, 0);
  const int n = capsule_plane_contacts(capsule_from_desc(capsule), P, pts);
  if (contacts) put_contacts(pts, n, contacts);
  return n;
}

extern "C" int orc_fine_pair_loads(const double* a, const double* b, const double* pmv, double* out) {
  const Capsule c1 = capsule_from_desc(a), c2 = capsule_from_desc(b);
  const PairMaterial pm = {pmv[0], pmv[1], pmv[2], pmv[3], pmv[4]};
  ContactPoint pts[2];
  const int n = rod_capsule_contacts(c1, c2, pts);
  V3 F1 = {0.0, 0.0, 0.0}, T1 = F1, F2 = F1, T2 = F1;
  for (int k = 0; k < n; ++k) {
    const V3 rvel = sub(point_velocity(c1, pts[k].pos), point_velocity(c2, pts[k].pos));
    V3 net;
    if (!spring_dashpot(pts[k], rvel, pm, net)) continue;
    F2 = add3(F2, neg3(net));
    T2 = add3(T2, cross(sub(pts[k].pos, c2.c), neg3(net)));
    F1 = add3(F1, net);
    T1 = add3(T1, cross(sub(pts[k].pos, c1.c), net));
  }
  const V3 all[4] = {F1, T1, F2, T2};
  for (int i = 0; i < 4; ++i) {
    out[3 * i] = all[i].x;
    out[3 * i + 1] = all[i].y;
    out[3 * i + 2] = all[i].z;
  }
  return n;
}

// PEFRL (Omelyan, Mryglod and Folk, Comput. Phys. Commun. 146 (2002)
// 188-202): drifts xi, chi, 1 - 2 (chi + xi), chi, xi around four kicks
// (1 - 2 lambda)/2, lambda, lambda, (1 - 2 lambda)/2, each kick followed by
// the rate constraints for its share of dt, each drift by the value
// constraints.  The reference declares this stepper without implementing it.
extern "C" int orc_step_pefrl(const OrcRods* rods, double dt, int64_t n_steps, int n_threads) {
  if (check(rods) != 0) return -1;
  const OrcRods& R = *rods;
  const double xi = 0.1786178958448091, lambda = -0.2123418310626054, chi = -0.06626458266981849;
  const double pre[4] = {xi, chi, 1.0 - 2.0 * (chi + xi), chi};
  const double kick[4] = {0.5 * (1.0 - 2.0 * lambda), lambda, lambda, 0.5 * (1.0 - 2.0 * lambda)};
#ifdef _OPENMP
  const int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
  {
    Scratch sc;
    std::vector<double> acc, alpha;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int64_t r = 0; r < R.n_rods; ++r) {
      const int64_t n = R.offset[r + 1] - R.offset[r] - 1;
      acc.assign(3 * (n + 1), 0.0);
      alpha.assign(3 * (n + 1), 0.0);
      for (int64_t step = 0; step < n_steps; ++step)
        for (int k = 0; k < 4; ++k) {
          kinematic(R, r, pre[k] * dt);
          clamp_values(R, r);
          compute_dynamics(R, r, sc, acc.data(), alpha.data());
          if (step == n_steps - 1 && k == 3) write_diagnostics(R, r, sc, acc.data(), alpha.data());
          dynamic_update(R, r, kick[k] * dt, sc, acc.data(), alpha.data());
          if (k == 3) {
            kinematic(R, r, xi * dt);
            clamp_values(R, r);
          }
        }
    }
  }
  (void)n_threads;
  return 0;
}

// VelocityVerlet (elastica/Time/SymplecticSteppers/Algorithms/
// VelocityVerlet.hpp:49-87): substeps [Dynamic(dt/2), Kinematic(dt),
// TimeUpdate(dt), Dynamic(dt/2)] walked as in Simulator::step
// (SymplecticSteppers.hpp:152-216): every dynamic substep first applies the
// value constraints, evaluates the loads at the current state, kicks by
// dt/2 and applies the rate constraints.  The analytical damper's constants
// are formed with the full dt at construction, so each of the two rate
// constraint passes multiplies by exp(-nu dt).
extern "C" int orc_step_velocity_verlet(const OrcRods* rods, double dt, int64_t n_steps, int n_threads) {
  if (check(rods) != 0) return -1;
  const OrcRods& R = *rods;
#ifdef _OPENMP
  const int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
  {
    Scratch sc;
    std::vector<double> acc, alpha;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int64_t r = 0; r < R.n_rods; ++r) {
      const int64_t n = R.offset[r + 1] - R.offset[r] - 1;
      acc.assign(3 * (n + 1), 0.0);
      alpha.assign(3 * (n + 1), 0.0);
      for (int64_t step = 0; step < n_steps; ++step) {
        clamp_values(R, r);
        compute_dynamics(R, r, sc, acc.data(), alpha.data());
        dynamic_update(R, r, 0.5 * dt, sc, acc.data(), alpha.data(), dt);
        kinematic(R, r, dt);
        clamp_values(R, r);
        compute_dynamics(R, r, sc, acc.data(), alpha.data());
        if (step == n_steps - 1) write_diagnostics(R, r, sc, acc.data(), alpha.data());
        dynamic_update(R, r, 0.5 * dt, sc, acc.data(), alpha.data(), dt);
      }
    }
  }
  (void)n_threads;
  return 0;
}

extern "C" int orc_force_eval(const OrcRods* rods, int n_threads) {
  if (check(rods) != 0) return -1;
  const OrcRods& R = *rods;
  (void)n_threads;
  Scratch sc;
  std::vector<double> acc, alpha;
  for (int64_t r = 0; r < R.n_rods; ++r) {
    const int64_t n = R.offset[r + 1] - R.offset[r] - 1;
    acc.assign(3 * (n + 1), 0.0);
    alpha.assign(3 * (n + 1), 0.0);
    compute_dynamics(R, r, sc, acc.data(), alpha.data());
    write_diagnostics(R, r, sc, acc.data(), alpha.data());
  }
  return 0;
}

// Systems/CosseratRods/Utility/Energy.hpp:46-141, evaluated at the current
// state (strains and curvatures recomputed from x and Q).
extern "C" int orc_energy(const OrcRods* rods, double* out, int n_threads) {
  if (check(rods) != 0 || !out) return -1;
  const OrcRods& R = *rods;
  const int64_t S = R.n_slots;
  (void)n_threads;
  for (int64_t r = 0; r < R.n_rods; ++r) {
    const int64_t o = R.offset[r], n = R.offset[r + 1] - o - 1;
    const Field x{R.x, S}, v{R.v, S}, w{R.w, S};
    double et = 0.0, er = 0.0, es = 0.0, eb = 0.0;
    for (int64_t j = 0; j <= n; ++j) {
      const V3 vv = v.get(o + j);
      et += R.mass[o + j] * (vv.x * vv.x + vv.y * vv.y + vv.z * vv.z);
    }
    std::vector<double> len(n), dil(n);
    for (int64_t i = 0; i < n; ++i) {
      const int64_t s = o + i;
      const V3 dx = sub(x.get(s + 1), x.get(s));
      len[i] = norm(dx);
      dil[i] = len[i] / R.rest_length[s];
      const V3 om = w.get(s);
      const double e = dil[i];
      er += om.x * (R.inertia_diag[s] * om.x / e) + om.y * (R.inertia_diag[S + s] * om.y / e) +
            om.z * (R.inertia_diag[2 * S + s] * om.z / e);
      double q[9];
      load_q(R.Q, S, s, q);
      const V3 t = {dx.x / len[i], dx.y / len[i], dx.z / len[i]};
      const V3 qt = matvec(q, t);
      const V3 d = {qt.x * e - R.rest_sigma[s], qt.y * e - R.rest_sigma[S + s],
                    qt.z * e - 1.0 - R.rest_sigma[2 * S + s]};
      es += (d.x * (R.shear_diag[s] * d.x) + d.y * (R.shear_diag[S + s] * d.y) +
             d.z * (R.shear_diag[2 * S + s] * d.z)) *
            R.rest_length[s];
    }
    for (int64_t k = 0; k + 1 < n; ++k) {
      const int64_t s = o + k;
      double qc[9], qn[9];
      load_q(R.Q, S, s, qc);
      load_q(R.Q, S, s + 1, qn);
      const V3 kp = inv_rotate_divide(qc, qn, R.rest_voronoi[s]);
      const V3 d = {kp.x - R.rest_kappa[s], kp.y - R.rest_kappa[S + s], kp.z - R.rest_kappa[2 * S + s]};
      eb += (d.x * (R.bend_diag[s] * d.x) + d.y * (R.bend_diag[S + s] * d.y) +
             d.z * (R.bend_diag[2 * S + s] * d.z)) *
            R.rest_voronoi[s];
    }
    out[4 * r] = 0.5 * et;
    out[4 * r + 1] = 0.5 * er;
    out[4 * r + 2] = 0.5 * es;
    out[4 * r + 3] = 0.5 * eb;
  }
  return 0;
}

// Straight rod: Initializers/detail/Geometry.hpp:143-211 (linspace positions
// from Utilities/Generators.hpp:86-119, directors from
// Utilities/Math/Orthogonal.cpp:32-55,98-116), cross section and volume
// (CosseratRodCrossSectionInterface.hpp:266-307, CircleCrossSectionOperations.hpp:84-132),
// reference geometry (CosseratRodSpanwiseGeometry.hpp:526-545), rigidities
// (LinearHyperElasticityFacade.hpp:273-327, Initializers/detail/Elasticity.hpp:54-77)
// and kinematics (WithRodKinematics.hpp:344-424).
extern "C" int orc_straight_rod(int64_t n, const double origin[3], const double direction[3],
                                const double normal[3], double length, double radius,
                                double density, double youngs, double shear_modulus, double* x,
                                double* Q, double* l0, double* D0, double* V, double* radius_out,
                                double* mass, double* J, double* Jinv, double* S, double* B) {
  if (n < 2 || !(length > 0.0) || !(radius > 0.0)) return -1;
  const V3 dr = {direction[0], direction[1], direction[2]};
  const V3 nr = {normal[0], normal[1], normal[2]};
  const double dn = norm(dr), nn = norm(nr);
  if (dn == 0.0 || nn == 0.0) return -1;
  const V3 t = {dr.x / dn, dr.y / dn, dr.z / dn};
  const V3 nv = {nr.x / nn, nr.y / nn, nr.z / nn};
  if (std::fabs(t.x * nv.x + t.y * nv.y + t.z * nv.z) > 1e-10) return -1;
  const int64_t nn1 = n + 1;
  // positions: start + index * step, step = (stop - start) / n
  const double o3[3] = {origin[0], origin[1], origin[2]};
  const double tv[3] = {t.x, t.y, t.z};
  for (int d = 0; d < 3; ++d) {
    const double stop = o3[d] + length * tv[d];
    const double step = (stop - o3[d]) / static_cast<double>(n);
    for (int64_t j = 0; j <= n; ++j) x[d * nn1 + j] = o3[d] + static_cast<double>(j) * step;
  }
  // directors: rows (v1, v2, v3) = (normal, (t x n)-based binormal, tangent)
  const V3 v1 = nv;
  V3 v2 = cross(t, nv);  // proposed_tangent % proposed_normal
  V3 v3 = cross(v1, v2);
  v2 = cross(v3, v1);
  const double n2 = norm(v2), n3 = norm(v3);
  v2 = {v2.x / n2, v2.y / n2, v2.z / n2};
  v3 = {v3.x / n3, v3.y / n3, v3.z / n3};
  const double rows[9] = {v1.x, v1.y, v1.z, v2.x, v2.y, v2.z, v3.x, v3.y, v3.z};
  for (int c = 0; c < 9; ++c)
    for (int64_t i = 0; i < n; ++i) Q[c * n + i] = rows[c];
  // reference geometry: l0 = |dx| / e (e = 1), D0 = average(l0)
  for (int64_t i = 0; i < n; ++i) {
    const V3 dx = {x[i + 1] - x[i], x[nn1 + i + 1] - x[nn1 + i], x[2 * nn1 + i + 1] - x[2 * nn1 + i]};
    l0[i] = norm(dx) / 1.0;
  }
  for (int64_t k = 0; k + 1 < n; ++k) D0[k] = 0.5 * (l0[k] + l0[k + 1]);
  // cross section: A = pi r^2, V = A l0, dimension = sqrt(V / pi / l0)
  const double A = static_cast<double>(M_PI) * (radius * radius);
  const double I1 = (0.25 * M_1_PI) * (A * A);
  const double Ivec[3] = {I1, I1, 2.0 * I1};
  for (int64_t i = 0; i < n; ++i) {
    V[i] = A * l0[i];
    radius_out[i] = std::sqrt(M_1_PI * V[i] / l0[i]);
  }
  // second moment of area uses the element dimension (the updated radius)
  auto I_of = [&](int64_t i, int d) {
    const double Ai = static_cast<double>(M_PI) * (radius_out[i] * radius_out[i]);
    const double I1i = (0.25 * M_1_PI) * (Ai * Ai);
    return d == 2 ? 2.0 * I1i : I1i;
  };
  (void)Ivec;
  const double stiff_b[3] = {youngs, youngs, shear_modulus};
  const double stiff_s[3] = {shear_modulus, shear_modulus, youngs};
  const double alpha_c = 13.5 / 14.0;
  for (int64_t i = 0; i < n; ++i) {
    const double Ai = static_cast<double>(M_PI) * (radius_out[i] * radius_out[i]);
    const double eff[3] = {Ai * alpha_c, Ai * alpha_c, Ai};
    for (int d = 0; d < 3; ++d) S[d * n + i] = stiff_s[d] * eff[d];
  }
  for (int64_t k = 0; k + 1 < n; ++k)
    for (int d = 0; d < 3; ++d)
      B[d * (n - 1) + k] = (l0[k] * stiff_b[d] * I_of(k, d) + l0[k + 1] * stiff_b[d] * I_of(k + 1, d)) /
                           (l0[k] + l0[k + 1]);
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      J[d * n + i] = I_of(i, d) * density * l0[i];
      Jinv[d * n + i] = 1.0 / (I_of(i, d) * density * l0[i]);
    }
  for (int64_t j = 0; j <= n; ++j) mass[j] = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double me = density * V[i];
    mass[i] += 0.5 * me;
    mass[i + 1] += 0.5 * me;
  }
  return 0;
}
