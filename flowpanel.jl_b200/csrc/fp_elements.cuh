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
template <> __device__ __forceinline__ double drcp<double>(double a) { return __drcp_rn(a); }
template <> __device__ __forceinline__ float drcp<float>(float a) { return __frcp_rn(a); }

// ---------------------------------------------------------------------------
// Vortex ring (== constant doublet velocity), dotted with a unit normal:
// sum over the NN edges of U_boundvortex (src/FLOWPanel_elements.jl:345-428,
// 442-467). Node vectors r_k = X - p_k and 1/(|r_k| + offset) are shared by
// the two edges meeting at node k. NN is a template parameter so that every
// index is static and the node arrays live in registers. The edge's factor
// rd / (4 pi (|c|^2 + offset^2)) is formed as rd times the correctly rounded
// reciprocal (one rounding more than the reference's division, 13 % less
// FP64-pipe time for the assembly).
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
      T aux = rd * drcp<T>(T(kFourPi) * (dot + offset2));
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
      T aux = s * rd * drcp<T>(T(kFourPi) * (dot + offset2));
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

// ---------------------------------------------------------------- potentials
// All in FP64 and in the panel's flipped frame (o, t, -n) held by SourceRec;
// unit strength, the caller scales.

// Constant-source potential (src/FLOWPanel_elements.jl:152-241, Hess & Smith).
__device__ __forceinline__ double source_phi(const SourceRec& R, double X1, double X2, double X3, double offset) {
  const double dx = X1 - R.O[0], dy = X2 - R.O[1], dz = X3 - R.O[2];
  const double x = R.t[0] * dx + R.t[1] * dy + R.t[2] * dz;
  const double y = R.o[0] * dx + R.o[1] * dy + R.o[2] * dz;
  const double z = R.n[0] * dx + R.n[1] * dy + R.n[2] * dz;
  const double az = fabs(z);
  double phi = 0, dtheta = 2 * kPi;
  const int nn = R.nn;
  for (int i = 0; i < nn; ++i) {
    const int j = (i + 1 == nn) ? 0 : i + 1;
    const double xi = R.xs[i], yi = R.ys[i], zi = R.zs[i];
    const double xj = R.xs[j], yj = R.ys[j], zj = R.zs[j];
    const double dij = R.dij[i];
    const double ri = sqrt((x - xi) * (x - xi) + (y - yi) * (y - yi) + (z - zi) * (z - zi));
    const double rj = sqrt((x - xj) * (x - xj) + (y - yj) * (y - yj) + (z - zj) * (z - zj));
    const double Qij = log((ri + rj + dij) / (ri + rj - dij + offset));
    const double Sij = R.S[i], Cij = R.Cc[i];
    const double siji = (xi - x) * Cij + (yi - y) * Sij;
    const double sijj = (xj - x) * Cij + (yj - y) * Sij;
    const double Rij = (x - xi) * Sij - (y - yi) * Cij;
    const double Jij = atan2(Rij * az * (ri * sijj - rj * siji), ri * rj * Rij * Rij + z * z * sijj * siji);
    phi -= Rij * Qij + az * Jij;
    dtheta *= (Rij >= 0);
  }
  phi += az * dtheta;
  return phi * (1 / (4 * kPi));
}

// Hess-Smith solid angle over a polygon in local coordinates (xs, ys, zs) at
// local (x, y, z): the doublet potential's kernel (src/FLOWPanel_elements.jl:796-833).
template <int NNMAX>
__device__ __forceinline__ double solid_angle(double x, double y, double z, const double* xs, const double* ys,
                                              const double* zs, const double* dijs, const double* Ss,
                                              const double* Cs, int nn) {
  double V3 = 0, dtheta = 2 * kPi;
  int nR0 = 0;
#pragma unroll
  for (int i = 0; i < NNMAX; ++i) {
    if (i >= nn) break;
    const int j = (i + 1 == nn) ? 0 : i + 1;
    const double xi = xs[i], yi = ys[i], zi = zs[i];
    const double xj = xs[j], yj = ys[j], zj = zs[j];
    double dij, Sij, Cij;
    if (dijs) {
      dij = dijs[i]; Sij = Ss[i]; Cij = Cs[i];
    } else {
      dij = sqrt((xj - xi) * (xj - xi) + (yj - yi) * (yj - yi) + (zj - zi) * (zj - zi));
      Sij = (yj - yi) / dij;
      Cij = (xj - xi) / dij;
    }
    const double ri = sqrt((x - xi) * (x - xi) + (y - yi) * (y - yi) + (z - zi) * (z - zi));
    const double rj = sqrt((x - xj) * (x - xj) + (y - yj) * (y - yj) + (z - zj) * (z - zj));
    const double siji = (xi - x) * Cij + (yi - y) * Sij;
    const double sijj = (xj - x) * Cij + (yj - y) * Sij;
    const double Rij = (x - xi) * Sij - (y - yi) * Cij;
    const double Jij = atan2(Rij * fabs(z) * (ri * sijj - rj * siji), ri * rj * Rij * Rij + z * z * sijj * siji);
    V3 -= Jij;
    dtheta *= (Rij >= 0);
    nR0 += (Rij == 0);
  }
  V3 += dtheta;
  V3 *= (z > 0) ? 1.0 : ((z < 0) ? -1.0 : 0.0);
  V3 *= (double)!(nR0 > 1);
  return V3 * (1 / (4 * kPi));
}

// Constant-doublet potential (src/FLOWPanel_elements.jl:751-847).
__device__ __forceinline__ double doublet_phi(const SourceRec& R, double X1, double X2, double X3) {
  const double dx = X1 - R.O[0], dy = X2 - R.O[1], dz = X3 - R.O[2];
  const double x = R.t[0] * dx + R.t[1] * dy + R.t[2] * dz;
  const double y = R.o[0] * dx + R.o[1] * dy + R.o[2] * dz;
  const double z = R.n[0] * dx + R.n[1] * dy + R.n[2] * dz;
  return solid_angle<4>(x, y, z, R.xs, R.ys, R.zs, R.dij, R.S, R.Cc, R.nn);
}

// Semi-infinite doublet potential along one direction d from the shedding
// edge (p_i, p_j) (src/FLOWPanel_elements.jl:959-1092, Moran App. F): the
// bound triangle (p_a, p_i, p_j), p_a the foot of p_j on the line through
// p_i along d, plus the semi-infinite strip from (p_a, p_j).
__device__ __forceinline__ double semiinf_doublet_phi(const double* p_i, const double* p_j, const double* d,
                                                      double X1, double X2, double X3) {
  const double pijdotd = (p_j[0] - p_i[0]) * d[0] + (p_j[1] - p_i[1]) * d[1] + (p_j[2] - p_i[2]) * d[2];
  const double pa[3] = {p_i[0] + pijdotd * d[0], p_i[1] + pijdotd * d[1], p_i[2] + pijdotd * d[2]};
  const double nrm = sqrt((p_j[0] - pa[0]) * (p_j[0] - pa[0]) + (p_j[1] - pa[1]) * (p_j[1] - pa[1]) +
                          (p_j[2] - pa[2]) * (p_j[2] - pa[2]));
  const double ex[3] = {d[0], d[1], d[2]};
  const double ey[3] = {(p_j[0] - pa[0]) / nrm, (p_j[1] - pa[1]) / nrm, (p_j[2] - pa[2]) / nrm};
  const double ez[3] = {ex[1] * ey[2] - ex[2] * ey[1], ex[2] * ey[0] - ex[0] * ey[2], ex[0] * ey[1] - ex[1] * ey[0]};
  auto loc = [&](const double* e, double a, double b, double c) {
    return e[0] * (a - p_i[0]) + e[1] * (b - p_i[1]) + e[2] * (c - p_i[2]);
  };
  const double xs[3] = {loc(ex, pa[0], pa[1], pa[2]), loc(ex, p_i[0], p_i[1], p_i[2]), loc(ex, p_j[0], p_j[1], p_j[2])};
  const double ys[3] = {loc(ey, pa[0], pa[1], pa[2]), loc(ey, p_i[0], p_i[1], p_i[2]), loc(ey, p_j[0], p_j[1], p_j[2])};
  const double zs[3] = {loc(ez, pa[0], pa[1], pa[2]), loc(ez, p_i[0], p_i[1], p_i[2]), loc(ez, p_j[0], p_j[1], p_j[2])};
  const double xa = xs[0], ya = ys[0], yb = ys[2];
  const double x = loc(ex, X1, X2, X3), y = loc(ey, X1, X2, X3), z = loc(ez, X1, X2, X3);
  double phi = 0;
  if (fabs(pijdotd) > 2 * 2.220446049250313e-16)
    phi += solid_angle<3>(x, y, z, xs, ys, zs, nullptr, nullptr, nullptr, 3);
  double val = atan((yb - y) / z) + atan((yb - y) * (x - xa) / (z * sqrt((x - xa) * (x - xa) + (yb - y) * (yb - y) + z * z)));
  val -= atan((ya - y) / z) + atan((ya - y) * (x - xa) / (z * sqrt((x - xa) * (x - xa) + (ya - y) * (ya - y) + z * z)));
  return phi + val * (1 / (4 * kPi));
}

// Semi-infinite doublet with directions (da, db) (src/FLOWPanel_elements.jl:1110-1244):
// the da part, plus, when db differs, the triangle (p_b + L da, p_b, p_b + L db)
// with L = infinitelength.
__device__ __forceinline__ double semiinf_doublet_phi2(const double* p_a, const double* p_b, const double* da,
                                                       const double* db, double X1, double X2, double X3,
                                                       double L) {
  double phi = semiinf_doublet_phi(p_a, p_b, da, X1, X2, X3);
  const double e2 = 2 * 2.220446049250313e-16;
  if (fabs(da[0] - db[0]) > e2 || fabs(da[1] - db[1]) > e2 || fabs(da[2] - db[2]) > e2) {
    const double pda[3] = {p_b[0] + L * da[0], p_b[1] + L * da[1], p_b[2] + L * da[2]};
    const double pdb[3] = {p_b[0] + L * db[0], p_b[1] + L * db[1], p_b[2] + L * db[2]};
    double ez[3] = {da[1] * db[2] - da[2] * db[1], da[2] * db[0] - da[0] * db[2], da[0] * db[1] - da[1] * db[0]};
    const double nz = sqrt(ez[0] * ez[0] + ez[1] * ez[1] + ez[2] * ez[2]);
    ez[0] = ez[0] / nz; ez[1] = ez[1] / nz; ez[2] = ez[2] / nz;
    const double ex[3] = {da[0], da[1], da[2]};
    const double ey[3] = {ez[1] * ex[2] - ez[2] * ex[1], ez[2] * ex[0] - ez[0] * ex[2], ez[0] * ex[1] - ez[1] * ex[0]};
    auto loc = [&](const double* e, double a, double b, double c) {
      return e[0] * (a - p_b[0]) + e[1] * (b - p_b[1]) + e[2] * (c - p_b[2]);
    };
    const double xs[3] = {loc(ex, pda[0], pda[1], pda[2]), loc(ex, p_b[0], p_b[1], p_b[2]), loc(ex, pdb[0], pdb[1], pdb[2])};
    const double ys[3] = {loc(ey, pda[0], pda[1], pda[2]), loc(ey, p_b[0], p_b[1], p_b[2]), loc(ey, pdb[0], pdb[1], pdb[2])};
    const double zs[3] = {loc(ez, pda[0], pda[1], pda[2]), loc(ez, p_b[0], p_b[1], p_b[2]), loc(ez, pdb[0], pdb[1], pdb[2])};
    phi += solid_angle<3>(loc(ex, X1, X2, X3), loc(ey, X1, X2, X3), loc(ez, X1, X2, X3), xs, ys, zs, nullptr,
                          nullptr, nullptr, 3);
  }
  return phi;
}

}  // namespace fpb
