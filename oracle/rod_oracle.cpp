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

#include <cmath>
#include <cstring>
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

// Value constraint of the clamp (examples/dynamic_cantilever/
// DynamicCantileverCaseStudy.cpp:73-89, applied post-kinematic,
// Simulator/Interface/TimeSteppers/SymplecticSteppers.hpp:174).
void clamp_values(const OrcRods& R, int64_t r) {
  if (!R.clamp || !R.clamp[r]) return;
  const int64_t S = R.n_slots, s = R.offset[r];
  for (int d = 0; d < 3; ++d) R.x[d * S + s] = R.clamp_x[3 * r + d];
  for (int c = 0; c < 9; ++c) R.Q[c * S + s] = R.clamp_Q[9 * r + c];
}

// Internal forces and torques of one rod (ElasticityInterface.hpp:360-365),
// then external loads and update_acceleration.  Fills sc.fl (loads, nodes)
// and sc.tq (torques, elements) and the per-element dilatation sc.dil.
void compute_dynamics(const OrcRods& R, int64_t r, Scratch& sc, double* acc, double* alpha) {
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
  if (R.end_torque) {
    double q[9];
    load_q(R.Q, S, o + n - 1, q);
    tend = matvec(q, {R.end_torque[3 * r], R.end_torque[3 * r + 1], R.end_torque[3 * r + 2]});
  }
  for (int64_t j = 0; j <= n; ++j) {
    const int64_t s = o + j;
    const double m = R.mass[s];
    const V3 fe = {0.0 + R.gravity[0] * m, 0.0 + R.gravity[1] * m, 0.0 + R.gravity[2] * m};
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
    if (i == n - 1) te = {te.x + tend.x, te.y + tend.y, te.z + tend.z};
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
// by the post-dynamic rate constraints: clamp (v0 = w0 = 0) and the
// analytical damper (examples/fish_swimming/FishModel/Dissipations/
// AnalyticalLinearDamper.hpp:15-76, "physical version").
void dynamic_update(const OrcRods& R, int64_t r, double dt, const Scratch& sc, const double* acc,
                    const double* alpha) {
  const int64_t S = R.n_slots, o = R.offset[r], n = R.offset[r + 1] - o - 1;
  for (int64_t j = 0; j <= n; ++j)
    for (int d = 0; d < 3; ++d) R.v[d * S + o + j] = R.v[d * S + o + j] + dt * acc[3 * j + d];
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) R.w[d * S + o + i] = R.w[d * S + o + i] + dt * alpha[3 * i + d];
  if (R.clamp && R.clamp[r]) {
    for (int d = 0; d < 3; ++d) {
      R.v[d * S + o] = 0.0;
      R.w[d * S + o] = 0.0;
    }
  }
  if (R.damper_nu && (R.damper_nu[2 * r] != 0.0 || R.damper_nu[2 * r + 1] != 0.0)) {
    const double nut = R.damper_nu[2 * r], nur = R.damper_nu[2 * r + 1];
    const double tcoef = std::exp(-nut * dt);
    for (int64_t j = 0; j <= n; ++j)
      for (int d = 0; d < 3; ++d) R.v[d * S + o + j] *= tcoef;
    for (int64_t i = 0; i < n; ++i) {
      const int64_t s = o + i;
      double em = 0.5 * (R.mass[s] + R.mass[s + 1]);
      if (i == 0) em += 0.5 * R.mass[s];
      if (i == n - 1) em += 0.5 * R.mass[s + 1];
      for (int d = 0; d < 3; ++d) {
        const double rc = std::exp(-nur * em * R.inv_inertia[d * S + s] * dt);
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
