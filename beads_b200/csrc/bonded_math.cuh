// bonded_math.cuh -- harmonic bond / angle / dihedral forces written once
// over a scalar type, so the adjoint can evaluate them on forward-mode dual
// numbers: Dual<K> carries a value and K directional derivatives, and the
// derivative parts of a term's force, energy and virial are then exact
// directional derivatives (Jacobian-vector products, parameter derivatives).
//
// The term conventions are the step kernels' (kernels.cu, bond_forces /
// angle_forces / dihedral_forces, after native/src/forcefield/bond/
// bond_harmonic.cu:24-99, angle/angle_harmonic.cu:54-178 and
// dihedral/dihedral_harmonic.cu:65-227): arms are minimum-image differences
// of member positions, cos clamped to [-1, 1], sin floored at 1e-3, singular
// geometry contributing energy only.  Branches test values only, so on a
// branch the derivative is that of the branch taken.
#pragma once

#include <cuda_runtime.h>

namespace bb {

template <int K>
struct Dual {
  float v;
  float d[K];
};

template <int K>
__device__ __forceinline__ Dual<K> dconst(float x) {
  Dual<K> r;
  r.v = x;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = 0.f;
  return r;
}

template <int K>
__device__ __forceinline__ Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(const Dual<K>& a) {
  Dual<K> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator*(float a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a * b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a * b.d[k];
  return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  const float inv = 1.0f / b.v;
  r.v = a.v * inv;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
  return r;
}
template <int K>
__device__ __forceinline__ Dual<K> dsqrt(const Dual<K>& a) {
  Dual<K> r;
  r.v = sqrtf(a.v);
  const float h = r.v > 0.f ? 0.5f / r.v : 0.f;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * h;
  return r;
}
template <int K>
__device__ __forceinline__ Dual<K> dacos(const Dual<K>& a) {
  Dual<K> r;
  r.v = acosf(a.v);
  const float s = 1.0f - a.v * a.v;
  const float h = s > 0.f ? -1.0f / sqrtf(s) : 0.f;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * h;
  return r;
}
template <int K>
__device__ __forceinline__ Dual<K> dcos(const Dual<K>& a) {
  Dual<K> r;
  float s, c;
  sincosf(a.v, &s, &c);
  r.v = c;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = -s * a.d[k];
  return r;
}
template <int K>
__device__ __forceinline__ Dual<K> dsin(const Dual<K>& a) {
  Dual<K> r;
  float s, c;
  sincosf(a.v, &s, &c);
  r.v = s;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = c * a.d[k];
  return r;
}

template <typename S>
struct V3T {
  S x, y, z;
};
template <typename S>
__device__ __forceinline__ S tdot(const V3T<S>& a, const V3T<S>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename S>
__device__ __forceinline__ V3T<S> tcross(const V3T<S>& a, const V3T<S>& b) {
  return V3T<S>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename S>
__device__ __forceinline__ V3T<S> tscale(const S& a, const V3T<S>& x) {
  return V3T<S>{a * x.x, a * x.y, a * x.z};
}
template <typename S>
__device__ __forceinline__ V3T<S> tadd(const V3T<S>& a, const V3T<S>& b) {
  return V3T<S>{a.x + b.x, a.y + b.y, a.z + b.z};
}
template <typename S>
__device__ __forceinline__ V3T<S> tsub(const V3T<S>& a, const V3T<S>& b) {
  return V3T<S>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename S>
__device__ __forceinline__ V3T<S> tneg(const V3T<S>& a) {
  return V3T<S>{-a.x, -a.y, -a.z};
}

// U = 0.5 k (r - r0)^2; d = x_i - x_j; force on member `role` (0: i, 1: j).
template <int K>
__device__ V3T<Dual<K>> dual_bond(const V3T<Dual<K>>& d, const Dual<K>& k, const Dual<K>& r0,
                                  uint32_t role, Dual<K>& energy, Dual<K>& virial) {
  const Dual<K> r2 = tdot(d, d);
  const Dual<K> r = dsqrt(r2);
  const Dual<K> s = r - r0;
  energy = 0.5f * (k * s * s);
  if (r.v == 0.0f) {
    virial = dconst<K>(0.f);
    const Dual<K> z = dconst<K>(0.f);
    return V3T<Dual<K>>{z, z, z};
  }
  const Dual<K> sc = -(k * s) / r;
  virial = sc * r2;
  return tscale(role == 0u ? sc : -sc, d);
}

// U = 0.5 k (theta - theta0)^2 (theta0 in radians); a1 = x_i - x_j,
// a2 = x_k - x_j; force on member `role` (0: i, 1: j, 2: k).
template <int K>
__device__ V3T<Dual<K>> dual_angle(const V3T<Dual<K>>& a1, const V3T<Dual<K>>& a2,
                                   const Dual<K>& k, const Dual<K>& theta0, uint32_t role,
                                   Dual<K>& energy, Dual<K>& virial) {
  const Dual<K> q1 = tdot(a1, a1);
  const Dual<K> q2 = tdot(a2, a2);
  const Dual<K> z = dconst<K>(0.f);
  if (q1.v == 0.0f || q2.v == 0.0f) {
    energy = 0.5f * (k * theta0 * theta0);
    virial = z;
    return V3T<Dual<K>>{z, z, z};
  }
  const Dual<K> r1 = dsqrt(q1);
  const Dual<K> r2 = dsqrt(q2);
  Dual<K> cs = tdot(a1, a2) / (r1 * r2);
  if (cs.v > 1.0f) cs = dconst<K>(1.0f);
  if (cs.v < -1.0f) cs = dconst<K>(-1.0f);
  const Dual<K> theta = cs.v == 1.0f ? dconst<K>(0.0f)
                        : (cs.v == -1.0f ? dconst<K>(3.14159265358979323846f) : dacos(cs));
  const Dual<K> dth = theta - theta0;
  energy = 0.5f * (k * dth * dth);
  const Dual<K> s2 = dconst<K>(1.0f) - cs * cs;
  const Dual<K> sn = s2.v <= 1.0e-6f ? dconst<K>(1.0e-3f) : dsqrt(s2);
  const Dual<K> a = -(k * dth) / sn;
  const Dual<K> c11 = a * cs / q1;
  const Dual<K> c12 = -a / (r1 * r2);
  const Dual<K> c22 = a * cs / q2;
  const V3T<Dual<K>> fi = tadd(tscale(c12, a2), tscale(c11, a1));
  const V3T<Dual<K>> fk = tadd(tscale(c12, a1), tscale(c22, a2));
  virial = tdot(a1, fi) + tdot(a2, fk);
  if (role == 0u) return fi;
  if (role == 2u) return fk;
  return tneg(tadd(fi, fk));
}

// U = k (1 + d cos(n phi)), signed phi; b0 = x_i - x_j, b1 = x_k - x_j,
// b2 = x_k - x_l; force on member `role` (0..3 = i, j, k, l).
template <int K>
__device__ V3T<Dual<K>> dual_dihedral(const V3T<Dual<K>>& b0, const V3T<Dual<K>>& b1,
                                      const V3T<Dual<K>>& b2, const Dual<K>& k, int dd, int nn,
                                      uint32_t role, Dual<K>& energy, Dual<K>& virial) {
  const V3T<Dual<K>> m = tcross(b0, b1);
  const V3T<Dual<K>> n = tcross(b1, b2);
  const Dual<K> q1 = tdot(b1, b1);
  const Dual<K> qm = tdot(m, m);
  const Dual<K> qn = tdot(n, n);
  const Dual<K> z = dconst<K>(0.f);
  if (q1.v == 0.0f || qm.v == 0.0f || qn.v == 0.0f) {
    energy = nn == 0 ? (1.0f + (float)dd) * k : k;
    virial = z;
    return V3T<Dual<K>>{z, z, z};
  }
  Dual<K> cs = tdot(m, n) / dsqrt(qm * qn);
  if (cs.v > 1.0f) cs = dconst<K>(1.0f);
  if (cs.v < -1.0f) cs = dconst<K>(-1.0f);
  Dual<K> phi = cs.v == 1.0f ? dconst<K>(0.0f)
                : (cs.v == -1.0f ? dconst<K>(3.14159265358979323846f) : dacos(cs));
  if (tdot(b0, n).v < 0.0f) phi = -phi;
  const Dual<K> arg = (float)nn * phi;
  energy = k * (dconst<K>(1.0f) + (float)dd * dcos(arg));
  const Dual<K> de = -((float)dd * (float)nn) * (k * dsin(arg));
  const Dual<K> l1 = dsqrt(q1);
  const V3T<Dual<K>> fi = tscale(-(de * l1) / qm, m);
  const V3T<Dual<K>> fl = tscale((de * l1) / qn, n);
  const Dual<K> p0 = tdot(b0, b1) / q1;
  const Dual<K> p2 = tdot(b2, b1) / q1;
  const V3T<Dual<K>> s = tsub(tscale(p0, fi), tscale(p2, fl));
  const V3T<Dual<K>> fj = tsub(s, fi);
  const V3T<Dual<K>> fk = tneg(tadd(s, fl));
  const V3T<Dual<K>> lj = tsub(b1, b2);
  virial = tdot(b0, fi) + tdot(b1, fk) + tdot(lj, fl);
  switch (role) {
    case 0u: return fi;
    case 1u: return fj;
    case 2u: return fk;
    default: return fl;
  }
}

}  // namespace bb
