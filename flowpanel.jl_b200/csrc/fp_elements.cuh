// Influence kernels of FLOWPanel.jl (src/FLOWPanel_elements.jl) as device
// functions, templated on the arithmetic type. The formulas, their order and
// their regularisations (core offset, cutoff, sign(z), dtheta, nR0) are the
// reference's; the only rewrites are algebraic identities that leave each term
// within an ulp: x/y -> x*(1/y) where one reciprocal serves several terms, and
// node-distance terms shared by the two edges that meet at a node computed once.
#pragma once
#include <cuda_runtime.h>

#include "fp_common.cuh"

namespace fpb {

template <class T> struct Vec3 { T x, y, z; };

template <class T> __device__ __forceinline__ T dsqrt(T a);
template <> __device__ __forceinline__ double dsqrt<double>(double a) { return sqrt(a); }
template <> __device__ __forceinline__ float dsqrt<float>(float a) { return sqrtf(a); }

template <class T> __device__ __forceinline__ T drcp(T a);
template <> __device__ __forceinline__ double drcp<double>(double a) { return 1.0 / a; }
template <> __device__ __forceinline__ float drcp<float>(float a) { return __frcp_rn(a); }

// ---------------------------------------------------------------------------
// Vortex ring (== constant doublet velocity), dotted with a unit normal:
// sum over the NN edges of U_boundvortex (src/FLOWPanel_elements.jl:345-428,
// 442-467). Node vectors r_k = X - p_k and 1/(|r_k| + offset) are shared by
// the two edges meeting at node k. NN is a template parameter so that every
// index is static and the node arrays live in registers.
template <class T, int NN>
__device__ __forceinline__ T ring_dot_n(const T* __restrict__ p, T X, T Y, T Z, T n1, T n2, T n3,
                                        T offset, T cutoff2, T offset2) {
  T rx[NN], ry[NN], rz[NN], inv[NN];
#pragma unroll
  for (int k = 0; k < NN; ++k) {
    rx[k] = X - p[3 * k];
    ry[k] = Y - p[3 * k + 1];
    rz[k] = Z - p[3 * k + 2];
    inv[k] = drcp<T>(dsqrt<T>(rx[k] * rx[k] + ry[k] * ry[k] + rz[k] * rz[k]) + offset);
  }
  T acc = T(0);
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int b = (a + 1) % NN;
    T rij1 = p[3 * b] - p[3 * a], rij2 = p[3 * b + 1] - p[3 * a + 1], rij3 = p[3 * b + 2] - p[3 * a + 2];
    T c1 = ry[a] * rz[b] - rz[a] * ry[b];
    T c2 = rz[a] * rx[b] - rx[a] * rz[b];
    T c3 = rx[a] * ry[b] - ry[a] * rx[b];
    T dot = c1 * c1 + c2 * c2 + c3 * c3;
    T rd = rij1 * (rx[a] * inv[a] - rx[b] * inv[b]) + rij2 * (ry[a] * inv[a] - ry[b] * inv[b]) +
           rij3 * (rz[a] * inv[a] - rz[b] * inv[b]);
    if (dot > cutoff2) {
      T aux = rd / (T(kFourPi) * (dot + offset2));
      acc += aux * (c1 * n1 + c2 * n2 + c3 * n3);
    }
  }
  return acc;
}

template <class T>
__device__ __forceinline__ T ring_dot(const T* __restrict__ p, int nn, T X, T Y, T Z, T n1, T n2,
                                      T n3, T offset, T cutoff2, T offset2) {
  return nn == 4 ? ring_dot_n<T, 4>(p, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2)
                 : ring_dot_n<T, 3>(p, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2);
}

// Same ring, full velocity vector times strength (for field evaluation).
template <class T, int NN>
__device__ __forceinline__ void ring_vel_n(const T* __restrict__ p, T s, T X, T Y, T Z, T offset,
                                           T cutoff2, T offset2, T& u, T& v, T& w) {
  T rx[NN], ry[NN], rz[NN], inv[NN];
#pragma unroll
  for (int k = 0; k < NN; ++k) {
    rx[k] = X - p[3 * k];
    ry[k] = Y - p[3 * k + 1];
    rz[k] = Z - p[3 * k + 2];
    inv[k] = drcp<T>(dsqrt<T>(rx[k] * rx[k] + ry[k] * ry[k] + rz[k] * rz[k]) + offset);
  }
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int b = (a + 1) % NN;
    T rij1 = p[3 * b] - p[3 * a], rij2 = p[3 * b + 1] - p[3 * a + 1], rij3 = p[3 * b + 2] - p[3 * a + 2];
    T c1 = ry[a] * rz[b] - rz[a] * ry[b];
    T c2 = rz[a] * rx[b] - rx[a] * rz[b];
    T c3 = rx[a] * ry[b] - ry[a] * rx[b];
    T dot = c1 * c1 + c2 * c2 + c3 * c3;
    T rd = rij1 * (rx[a] * inv[a] - rx[b] * inv[b]) + rij2 * (ry[a] * inv[a] - ry[b] * inv[b]) +
           rij3 * (rz[a] * inv[a] - rz[b] * inv[b]);
    if (dot > cutoff2) {
      T aux = s * rd / (T(kFourPi) * (dot + offset2));
      u += aux * c1;
      v += aux * c2;
      w += aux * c3;
    }
  }
}

template <class T>
__device__ __forceinline__ void ring_vel(const T* __restrict__ p, int nn, T s, T X, T Y, T Z,
                                         T offset, T cutoff2, T offset2, T& u, T& v, T& w) {
  if (nn == 4) ring_vel_n<T, 4>(p, s, X, Y, Z, offset, cutoff2, offset2, u, v, w);
  else ring_vel_n<T, 3>(p, s, X, Y, Z, offset, cutoff2, offset2, u, v, w);
}

// One bound filament pa -> pb (U_boundvortex, :345-428), accumulating
// strength * U into (u, v, w).
template <class T>
__device__ __forceinline__ void filament(T pa1, T pa2, T pa3, T pb1, T pb2, T pb3, T s, T X, T Y,
                                         T Z, T offset, T cutoff2, T offset2, T& u, T& v, T& w) {
  T rij1 = pb1 - pa1, rij2 = pb2 - pa2, rij3 = pb3 - pa3;
  T ri1 = X - pa1, ri2 = Y - pa2, ri3 = Z - pa3;
  T rj1 = X - pb1, rj2 = Y - pb2, rj3 = Z - pb3;
  T c1 = ri2 * rj3 - ri3 * rj2;
  T c2 = ri3 * rj1 - ri1 * rj3;
  T c3 = ri1 * rj2 - ri2 * rj1;
  T dot = c1 * c1 + c2 * c2 + c3 * c3;
  T ia = drcp<T>(dsqrt<T>(ri1 * ri1 + ri2 * ri2 + ri3 * ri3) + offset);
  T ib = drcp<T>(dsqrt<T>(rj1 * rj1 + rj2 * rj2 + rj3 * rj3) + offset);
  T rd = rij1 * (ri1 * ia - rj1 * ib) + rij2 * (ri2 * ia - rj2 * ib) + rij3 * (ri3 * ia - rj3 * ib);
  if (dot > cutoff2) {
    T aux = s * rd / (T(kFourPi) * (dot + offset2));
    u += aux * c1;
    v += aux * c2;
    w += aux * c3;
  }
}

// Semi-infinite vortex from p along unit d (U_semiinfinite_vortex, :480-628):
// bound part p -> p0 (foot point of X) plus the infinite part.
template <class T>
__device__ __forceinline__ void semiinf(T p1, T p2, T p3, T d1, T d2, T d3, T s, T X, T Y, T Z,
                                        T offset, T cutoff2, T offset2, T& u, T& v, T& w) {
  T xmpdotd = (X - p1) * d1 + (Y - p2) * d2 + (Z - p3) * d3;
  T p01 = p1 + xmpdotd * d1;
  T p02 = p2 + xmpdotd * d2;
  T p03 = p3 + xmpdotd * d3;
  T e1 = p01 - p1, e2 = p02 - p2, e3 = p03 - p3;
  if (e1 * e1 + e2 * e2 + e3 * e3 > offset2) {
    filament<T>(p1, p2, p3, p01, p02, p03, s, X, Y, Z, offset, cutoff2, offset2, u, v, w);
  }
  T h1 = X - p01, h2 = Y - p02, h3 = Z - p03;
  T hsqr = h1 * h1 + h2 * h2 + h3 * h3;
  T m1 = d2 * h3 - d3 * h2;
  T m2 = d3 * h1 - d1 * h3;
  T m3 = d1 * h2 - d2 * h1;
  if (hsqr > cutoff2) {
    T aux = s / (T(kFourPi) * (hsqr + offset2));
    u += aux * m1;
    v += aux * m2;
    w += aux * m3;
  }
}

// Semi-infinite horseshoe (da at pa, db at pb) (U_semiinfinite_horseshoe, :692-730).
template <class T>
__device__ __forceinline__ void horseshoe(const T* pa, const T* pb, const T* da, const T* db, T s,
                                          T X, T Y, T Z, T offset, T cutoff2, T offset2, T& u,
                                          T& v, T& w) {
  semiinf<T>(pa[0], pa[1], pa[2], da[0], da[1], da[2], -s, X, Y, Z, offset, cutoff2, offset2, u, v, w);
  filament<T>(pa[0], pa[1], pa[2], pb[0], pb[1], pb[2], s, X, Y, Z, offset, cutoff2, offset2, u, v, w);
  semiinf<T>(pb[0], pb[1], pb[2], db[0], db[1], db[2], s, X, Y, Z, offset, cutoff2, offset2, u, v, w);
}

// Dotted forms (out[ti] += aux * (c . n) per sub-element, as with dot_with):
// they accumulate into acc in the reference's order.
template <class T>
__device__ __forceinline__ void filament_dot(T pa1, T pa2, T pa3, T pb1, T pb2, T pb3, T s, T X,
                                             T Y, T Z, T n1, T n2, T n3, T offset, T cutoff2,
                                             T offset2, T& acc) {
  T rij1 = pb1 - pa1, rij2 = pb2 - pa2, rij3 = pb3 - pa3;
  T ri1 = X - pa1, ri2 = Y - pa2, ri3 = Z - pa3;
  T rj1 = X - pb1, rj2 = Y - pb2, rj3 = Z - pb3;
  T c1 = ri2 * rj3 - ri3 * rj2;
  T c2 = ri3 * rj1 - ri1 * rj3;
  T c3 = ri1 * rj2 - ri2 * rj1;
  T dot = c1 * c1 + c2 * c2 + c3 * c3;
  T ia = drcp<T>(dsqrt<T>(ri1 * ri1 + ri2 * ri2 + ri3 * ri3) + offset);
  T ib = drcp<T>(dsqrt<T>(rj1 * rj1 + rj2 * rj2 + rj3 * rj3) + offset);
  T rd = rij1 * (ri1 * ia - rj1 * ib) + rij2 * (ri2 * ia - rj2 * ib) + rij3 * (ri3 * ia - rj3 * ib);
  if (dot > cutoff2) {
    T aux = s * rd / (T(kFourPi) * (dot + offset2));
    acc += aux * (c1 * n1 + c2 * n2 + c3 * n3);
  }
}

template <class T>
__device__ __forceinline__ void semiinf_dot(T p1, T p2, T p3, T d1, T d2, T d3, T s, T X, T Y,
                                            T Z, T n1, T n2, T n3, T offset, T cutoff2,
                                            T offset2, T& acc) {
  T xmpdotd = (X - p1) * d1 + (Y - p2) * d2 + (Z - p3) * d3;
  T p01 = p1 + xmpdotd * d1;
  T p02 = p2 + xmpdotd * d2;
  T p03 = p3 + xmpdotd * d3;
  T e1 = p01 - p1, e2 = p02 - p2, e3 = p03 - p3;
  if (e1 * e1 + e2 * e2 + e3 * e3 > offset2) {
    filament_dot<T>(p1, p2, p3, p01, p02, p03, s, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2, acc);
  }
  T h1 = X - p01, h2 = Y - p02, h3 = Z - p03;
  T hsqr = h1 * h1 + h2 * h2 + h3 * h3;
  T m1 = d2 * h3 - d3 * h2;
  T m2 = d3 * h1 - d1 * h3;
  T m3 = d1 * h2 - d2 * h1;
  if (hsqr > cutoff2) {
    T aux = s / (T(kFourPi) * (hsqr + offset2));
    acc += aux * (m1 * n1 + m2 * n2 + m3 * n3);
  }
}

template <class T>
__device__ __forceinline__ void horseshoe_dot(const T* pa, const T* pb, const T* da, const T* db,
                                              T s, T X, T Y, T Z, T n1, T n2, T n3, T offset,
                                              T cutoff2, T offset2, T& acc) {
  semiinf_dot<T>(pa[0], pa[1], pa[2], da[0], da[1], da[2], -s, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2, acc);
  filament_dot<T>(pa[0], pa[1], pa[2], pb[0], pb[1], pb[2], s, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2, acc);
  semiinf_dot<T>(pb[0], pb[1], pb[2], db[0], db[1], db[2], s, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2, acc);
}

// ---------------------------------------------------------------------------
// Constant source (U_constant_source, :29-141). The panel frame, the local
// node coordinates and the per-edge dij/Sij/Cij do not depend on the target;
// they are computed once per panel (same formulas, same values) into a record.
struct SourceRec {
  double O[3];          // origin node
  double t[3], o[3], n[3];  // flipped frame (o, t, -n) of :51-56
  double xs[4], ys[4], zs[4];
  double dij[4], S[4], Cc[4];
  int nn;
  int pad;
};

__device__ __forceinline__ void source_vel(const SourceRec& R, double X1, double X2, double X3,
                                           double offset, double& u, double& v, double& w) {
  const double dx = X1 - R.O[0], dy = X2 - R.O[1], dz = X3 - R.O[2];
  const double x = R.t[0] * dx + R.t[1] * dy + R.t[2] * dz;
  const double y = R.o[0] * dx + R.o[1] * dy + R.o[2] * dz;
  const double z = R.n[0] * dx + R.n[1] * dy + R.n[2] * dz;
  double V1 = 0, V2 = 0, V3 = 0;
  double dtheta = 2 * kPi;
  int nR0 = 0;
  const int nn = R.nn;
  for (int i = 0; i < nn; ++i) {
    const int j = (i + 1 == nn) ? 0 : i + 1;
    const double xi = R.xs[i], yi = R.ys[i], zi = R.zs[i];
    const double xj = R.xs[j], yj = R.ys[j], zj = R.zs[j];
    const double dij = R.dij[i];
    const double ri = sqrt((x - xi) * (x - xi) + (y - yi) * (y - yi) + (z - zi) * (z - zi));
    const double rj = sqrt((x - xj) * (x - xj) + (y - yj) * (y - yj) + (z - zj) * (z - zj));
    const double Qij = log((ri + rj + dij) / (ri + rj - dij + offset));
    const double Sij = R.S[i];
    const double Cij = R.Cc[i];
    const double siji = (xi - x) * Cij + (yi - y) * Sij;
    const double sijj = (xj - x) * Cij + (yj - y) * Sij;
    const double Rij = (x - xi) * Sij - (y - yi) * Cij;
    const double Jij = atan2(Rij * fabs(z) * (ri * sijj - rj * siji), ri * rj * Rij * Rij + z * z * sijj * siji);
    V1 -= Sij * Qij;
    V2 += Cij * Qij;
    V3 -= Jij;
    dtheta *= (Rij >= 0);
    nR0 += (Rij == 0);
  }
  V3 += dtheta;
  V3 *= (z > 0) ? 1.0 : ((z < 0) ? -1.0 : 0.0);
  V3 *= (double)!(nR0 > 1);
  V1 *= 1 / (4 * kPi);
  V2 *= 1 / (4 * kPi);
  V3 *= 1 / (4 * kPi);
  u = V1 * R.t[0] + V2 * R.o[0] + V3 * R.n[0];
  v = V1 * R.t[1] + V2 * R.o[1] + V3 * R.n[1];
  w = V1 * R.t[2] + V2 * R.o[2] + V3 * R.n[2];
}

}  // namespace fpb
