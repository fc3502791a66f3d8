// Device-side rod arithmetic shared by the step kernels.
//
// Each helper restates one scalar kernel of the reference (GazzolaLab/
// elasticapp) with the same association order, so that the FP64 path tracks
// the reference to rounding level.  Templated on the arithmetic type so the
// mixed-precision path can instantiate the element-local math in float.
#pragma once

#include <cuda_runtime.h>

namespace eb {

template <typename T>
struct Vec3 {
  T x, y, z;
};

template <typename T>
__device__ __forceinline__ Vec3<T> v3(T x, T y, T z) {
  return Vec3<T>{x, y, z};
}
template <typename T>
__device__ __forceinline__ Vec3<T> operator-(Vec3<T> a, Vec3<T> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename T>
__device__ __forceinline__ Vec3<T> operator+(Vec3<T> a, Vec3<T> b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <typename T>
__device__ __forceinline__ Vec3<T> scale(Vec3<T> a, T s) {
  return {a.x * s, a.y * s, a.z * s};
}
template <typename T>
__device__ __forceinline__ Vec3<T> divide(Vec3<T> a, T s) {
  return {a.x / s, a.y / s, a.z / s};
}
template <typename T>
__device__ __forceinline__ T dot(Vec3<T> a, Vec3<T> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
// LinearAlgebra/CrossProduct/Operation.hpp:58-81
template <typename T>
__device__ __forceinline__ Vec3<T> cross(Vec3<T> m, Vec3<T> v) {
  return {m.y * v.z - m.z * v.y, m.z * v.x - m.x * v.z, m.x * v.y - m.y * v.x};
}
// MatVec/Operation.hpp:24-30: (Q v)_k = Q(k,0) v0 + Q(k,1) v1 + Q(k,2) v2
template <typename T>
__device__ __forceinline__ Vec3<T> matvec(const T q[9], Vec3<T> v) {
  return {q[0] * v.x + q[1] * v.y + q[2] * v.z, q[3] * v.x + q[4] * v.y + q[5] * v.z,
          q[6] * v.x + q[7] * v.y + q[8] * v.z};
}
// OpsTraits.hpp:166-188: (Q^T v)_i = sum_k Q(k,i) v_k
template <typename T>
__device__ __forceinline__ Vec3<T> mattranspvec(const T q[9], Vec3<T> v) {
  return {q[0] * v.x + q[3] * v.y + q[6] * v.z, q[1] * v.x + q[4] * v.y + q[7] * v.z,
          q[2] * v.x + q[5] * v.y + q[8] * v.z};
}

__device__ __forceinline__ void sincos_t(double a, double* s, double* c) { sincos(a, s, c); }
__device__ __forceinline__ void sincos_t(float a, float* s, float* c) { sincosf(a, s, c); }

// Systems/States/Expressions/backends/blaze/SO3PrimitiveAddAssign/Scalar.hpp:41-95
// Q <- exp(-[u]x) Q (Rodrigues), theta = |u|, axis u / (theta + 1e-14).
template <typename T>
__device__ __forceinline__ void so3_update(T q[9], T u0, T u1, T u2) {
  const T theta = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
  T s, c;
  sincos_t(theta, &s, &c);
  const T alpha = T(1) - c;
  const T den = theta + T(1e-14);
  u0 /= den;
  u1 /= den;
  u2 /= den;
  T out[9];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const T com = q[j] * u0 + q[3 + j] * u1 + q[6 + j] * u2;
    out[j] = c * q[j] + alpha * u0 * com + s * (q[3 + j] * u2 - q[6 + j] * u1);
    out[3 + j] = c * q[3 + j] + alpha * u1 * com + s * (q[6 + j] * u0 - q[j] * u2);
    out[6 + j] = c * q[6 + j] + alpha * u2 * com + s * (q[j] * u1 - q[3 + j] * u0);
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) q[k] = out[k];
}

// Traits/Operations/BlazeBackend/InvRotateDivide/Scalar.hpp:80-105
template <typename T>
__device__ __forceinline__ Vec3<T> inv_rotate_divide(const T qc[9], const T qn[9], T span) {
  const T tr = qc[0] * qn[0] + qc[1] * qn[1] + qc[2] * qn[2] + qc[3] * qn[3] + qc[4] * qn[4] +
               qc[5] * qn[5] + qc[6] * qn[6] + qc[7] * qn[7] + qc[8] * qn[8];
  const T rest = T(0.5) + T(1e-10);
  const T theta = acos(T(0.5) * tr - rest);
  const T st = T(0.5) * theta / sin(theta + T(1e-14)) / span;
  return {st * (-qc[3] * qn[6] - qc[4] * qn[7] - qc[5] * qn[8] + qc[6] * qn[3] + qc[7] * qn[4] +
                qc[8] * qn[5]),
          st * (qc[0] * qn[6] + qc[1] * qn[7] + qc[2] * qn[8] - qc[6] * qn[0] - qc[7] * qn[1] -
                qc[8] * qn[2]),
          st * (-qc[0] * qn[3] - qc[1] * qn[4] - qc[2] * qn[5] + qc[3] * qn[0] + qc[4] * qn[1] +
                qc[5] * qn[2])};
}

// ---- rounding-level reformulations used by the fast FP64 build -------------
// Each is mathematically identical to the helper above it and changes the
// result only by rounding.

// Q <- exp(-[u]x) Q with sin(theta) and 1 - cos(theta) from their Taylor
// series for theta < 0.1 (truncation below 1e-21 relative), which also avoids
// the cancellation of 1 - cos(theta) at small angles, and one reciprocal for
// the axis normalisation.
__device__ __forceinline__ void so3_update_fast(double q[9], double u0, double u1, double u2) {
  const double z = u0 * u0 + u1 * u1 + u2 * u2;
  const double theta = sqrt(z);
  double s, alpha;
  if (theta < 0.1) {
    s = theta * (1.0 + z * (-1.0 / 6.0 + z * (1.0 / 120.0 + z * (-1.0 / 5040.0 +
                                                           z * (1.0 / 362880.0 - z * (1.0 / 39916800.0))))));
    alpha = z * (0.5 + z * (-1.0 / 24.0 + z * (1.0 / 720.0 + z * (-1.0 / 40320.0 + z * (1.0 / 3628800.0)))));
  } else {
    double c;
    sincos(theta, &s, &c);
    alpha = 1.0 - c;
  }
  const double c = 1.0 - alpha;
  const double r = 1.0 / (theta + 1e-14);
  u0 *= r;
  u1 *= r;
  u2 *= r;
  double out[9];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double com = q[j] * u0 + q[3 + j] * u1 + q[6 + j] * u2;
    out[j] = c * q[j] + alpha * u0 * com + s * (q[3 + j] * u2 - q[6 + j] * u1);
    out[3 + j] = c * q[3 + j] + alpha * u1 * com + s * (q[6 + j] * u0 - q[j] * u2);
    out[6 + j] = c * q[6 + j] + alpha * u2 * com + s * (q[j] * u1 - q[3 + j] * u0);
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) q[k] = out[k];
}

// Curvature with sin(acos(c) + d) = sqrt((1 - c)(1 + c)) cos d + c sin d,
// d = 1e-14 (cos d rounds to 1, sin d to d).
__device__ __forceinline__ Vec3<double> inv_rotate_divide_fast(const double qc[9], const double qn[9],
                                                               double span) {
  const double tr = qc[0] * qn[0] + qc[1] * qn[1] + qc[2] * qn[2] + qc[3] * qn[3] + qc[4] * qn[4] +
                    qc[5] * qn[5] + qc[6] * qn[6] + qc[7] * qn[7] + qc[8] * qn[8];
  const double cth = 0.5 * tr - (0.5 + 1e-10);
  const double theta = acos(cth);
  const double sin_shifted = sqrt((1.0 - cth) * (1.0 + cth)) + cth * 1e-14;
  const double st = (0.5 * theta) / (sin_shifted * span);
  return {st * (-qc[3] * qn[6] - qc[4] * qn[7] - qc[5] * qn[8] + qc[6] * qn[3] + qc[7] * qn[4] +
                qc[8] * qn[5]),
          st * (qc[0] * qn[6] + qc[1] * qn[7] + qc[2] * qn[8] - qc[6] * qn[0] - qc[7] * qn[1] -
                qc[8] * qn[2]),
          st * (-qc[0] * qn[3] - qc[1] * qn[4] - qc[2] * qn[5] + qc[3] * qn[0] + qc[4] * qn[1] +
                qc[5] * qn[2])};
}

}  // namespace eb
