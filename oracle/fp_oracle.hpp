// ORACLE — test infrastructure only.
//
// CPU restatement of the FLOWPanel.jl v1.2.1 panel-method hot path, used by the
// tests, the smoke check and the CPU-baseline leg of the benchmark as the
// checker. It is never the measured or shipped path: the product is the CUDA
// library under flowpanel.jl_b200/csrc, which fails loudly without a GPU.
//
// Every function follows the reference operation by operation (same formulas,
// same order, same regularisations) and cites the reference file:line it
// restates. The kernels are templated on the scalar type so that the same code
// runs in double (the oracle), in a forward dual number (stands in for
// ForwardDiff in the reference's grad(phi) == u known-answer tests), and in an
// operation counter (pins the per-interaction operation counts that the
// roofline uses).
//
// Pinning: the reference cannot run here (it is Julia; no Julia binary exists
// on either machine). The restatement is pinned against the reference's own
// known-answer tests (test/runtests_elements.jl:37-315,
// test/runtests_semiinfiniteelements.jl:28-241), the analytic sphere Cp
// (examples/sphere.jl:86-87) and the swept-wing CL tolerance of
// test/runtests_solvers.jl:165-174, all re-run by tests/test_oracle_*.py.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

namespace fpo {

using std::abs;
using std::atan2;
using std::log;
using std::sqrt;

constexpr double PI = 3.14159265358979323846;

// ---------------------------------------------------------------- scalar helpers
template <class T> inline T sq(const T& a) { return a * a; }
inline double value_of(double a) { return a; }

// Julia's sign(): -1, 0 or +1 (sign(0) == 0).
template <class T> inline double jsign(const T& a) {
  double v = value_of(a);
  return (v > 0) ? 1.0 : ((v < 0) ? -1.0 : 0.0);
}

// ---------------------------------------------------------------- forward dual
// Minimal forward-mode dual number with K partials; stands in for ForwardDiff.
template <int K> struct Dual {
  double v;
  double d[K];
  Dual() : v(0) { for (int i = 0; i < K; ++i) d[i] = 0; }
  Dual(double a) : v(a) { for (int i = 0; i < K; ++i) d[i] = 0; }
  Dual& operator+=(const Dual& b) { v += b.v; for (int i = 0; i < K; ++i) d[i] += b.d[i]; return *this; }
  Dual& operator-=(const Dual& b) { v -= b.v; for (int i = 0; i < K; ++i) d[i] -= b.d[i]; return *this; }
  Dual& operator*=(const Dual& b) {
    for (int i = 0; i < K; ++i) d[i] = d[i] * b.v + v * b.d[i];
    v *= b.v; return *this;
  }
};
template <int K> inline double value_of(const Dual<K>& a) { return a.v; }
template <int K> inline Dual<K> operator+(Dual<K> a, const Dual<K>& b) { return a += b; }
template <int K> inline Dual<K> operator-(Dual<K> a, const Dual<K>& b) { return a -= b; }
template <int K> inline Dual<K> operator-(const Dual<K>& a) { Dual<K> r; r.v = -a.v; for (int i = 0; i < K; ++i) r.d[i] = -a.d[i]; return r; }
template <int K> inline Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r; r.v = a.v * b.v; for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r;
}
template <int K> inline Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r; r.v = a.v / b.v;
  for (int i = 0; i < K; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v);
  return r;
}
template <int K> inline Dual<K> operator+(const Dual<K>& a, double b) { return a + Dual<K>(b); }
template <int K> inline Dual<K> operator+(double a, const Dual<K>& b) { return Dual<K>(a) + b; }
template <int K> inline Dual<K> operator-(const Dual<K>& a, double b) { return a - Dual<K>(b); }
template <int K> inline Dual<K> operator-(double a, const Dual<K>& b) { return Dual<K>(a) - b; }
template <int K> inline Dual<K> operator*(const Dual<K>& a, double b) { return a * Dual<K>(b); }
template <int K> inline Dual<K> operator*(double a, const Dual<K>& b) { return Dual<K>(a) * b; }
template <int K> inline Dual<K> operator/(const Dual<K>& a, double b) { return a / Dual<K>(b); }
template <int K> inline Dual<K> operator/(double a, const Dual<K>& b) { return Dual<K>(a) / b; }
template <int K> inline bool operator>(const Dual<K>& a, double b) { return a.v > b; }
template <int K> inline bool operator>(const Dual<K>& a, const Dual<K>& b) { return a.v > b.v; }
template <int K> inline bool operator>=(const Dual<K>& a, double b) { return a.v >= b; }
template <int K> inline bool operator==(const Dual<K>& a, double b) { return a.v == b; }
template <int K> inline Dual<K> sqrt(const Dual<K>& a) {
  Dual<K> r; r.v = std::sqrt(a.v); for (int i = 0; i < K; ++i) r.d[i] = a.d[i] / (2 * r.v); return r;
}
template <int K> inline Dual<K> log(const Dual<K>& a) {
  Dual<K> r; r.v = std::log(a.v); for (int i = 0; i < K; ++i) r.d[i] = a.d[i] / a.v; return r;
}
template <int K> inline Dual<K> abs(const Dual<K>& a) {
  Dual<K> r; double s = a.v >= 0 ? 1.0 : -1.0; r.v = std::abs(a.v);
  for (int i = 0; i < K; ++i) r.d[i] = s * a.d[i]; return r;
}
template <int K> inline Dual<K> atan2(const Dual<K>& y, const Dual<K>& x) {
  Dual<K> r; r.v = std::atan2(y.v, x.v); double den = x.v * x.v + y.v * y.v;
  for (int i = 0; i < K; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) / den; return r;
}
template <int K> inline Dual<K> atan(const Dual<K>& a) {
  Dual<K> r; r.v = std::atan(a.v);
  for (int i = 0; i < K; ++i) r.d[i] = a.d[i] / (1 + a.v * a.v); return r;
}
using std::atan;

// ---------------------------------------------------------------- operation counter
// Counts floating-point operations as written in the reference: +,-,*,/ and
// each of sqrt, log, atan/atan2, abs as one operation. Comparisons are free.
struct OpCount {
  double v;
  OpCount() : v(0) {}
  OpCount(double a) : v(a) {}
  static long long& n() { static long long c = 0; return c; }
};
inline double value_of(const OpCount& a) { return a.v; }
inline OpCount operator+(const OpCount& a, const OpCount& b) { ++OpCount::n(); return OpCount(a.v + b.v); }
inline OpCount operator-(const OpCount& a, const OpCount& b) { ++OpCount::n(); return OpCount(a.v - b.v); }
inline OpCount operator*(const OpCount& a, const OpCount& b) { ++OpCount::n(); return OpCount(a.v * b.v); }
inline OpCount operator/(const OpCount& a, const OpCount& b) { ++OpCount::n(); return OpCount(a.v / b.v); }
inline OpCount operator-(const OpCount& a) { return OpCount(-a.v); }
inline OpCount operator+(const OpCount& a, double b) { return a + OpCount(b); }
inline OpCount operator+(double a, const OpCount& b) { return OpCount(a) + b; }
inline OpCount operator-(const OpCount& a, double b) { return a - OpCount(b); }
inline OpCount operator-(double a, const OpCount& b) { return OpCount(a) - b; }
inline OpCount operator*(const OpCount& a, double b) { return a * OpCount(b); }
inline OpCount operator*(double a, const OpCount& b) { return OpCount(a) * b; }
inline OpCount operator/(const OpCount& a, double b) { return a / OpCount(b); }
inline OpCount operator/(double a, const OpCount& b) { return OpCount(a) / b; }
inline OpCount& operator+=(OpCount& a, const OpCount& b) { a = a + b; return a; }
inline OpCount& operator-=(OpCount& a, const OpCount& b) { a = a - b; return a; }
inline OpCount& operator*=(OpCount& a, const OpCount& b) { a = a * b; return a; }
inline bool operator>(const OpCount& a, double b) { return a.v > b; }
inline bool operator>(const OpCount& a, const OpCount& b) { return a.v > b.v; }
inline bool operator>=(const OpCount& a, double b) { return a.v >= b; }
inline bool operator==(const OpCount& a, double b) { return a.v == b; }
inline OpCount sqrt(const OpCount& a) { ++OpCount::n(); return OpCount(std::sqrt(a.v)); }
inline OpCount log(const OpCount& a) { ++OpCount::n(); return OpCount(std::log(a.v)); }
inline OpCount abs(const OpCount& a) { ++OpCount::n(); return OpCount(std::abs(a.v)); }
inline OpCount atan2(const OpCount& y, const OpCount& x) { ++OpCount::n(); return OpCount(std::atan2(y.v, x.v)); }
inline OpCount atan(const OpCount& a) { ++OpCount::n(); return OpCount(std::atan(a.v)); }

// ---------------------------------------------------------------- mesh views
// nodes: 3 x nnodes, column-major (x0,y0,z0,x1,...). A panel is a list of
// 0-based node indices (3 or more nodes, planar polygon).
template <class T> struct NodeRef {
  const T* nodes;
  inline const T& c(int k, int ni) const { return nodes[3 * (int64_t)ni + k]; }
};

// Panel unit vectors t, o, n as documented in docs/src/elements/paneldefinition.md:15-35
// (GeometricTools _calc_t*/_calc_o*/_calc_n*, unvendored): t = (p2-p1)/|p2-p1|,
// n = (p2-p1)x(p3-p1)/|.|, o = n x t.
template <class T>
inline void panel_frame(const T* nodes, const int* panel, T t[3], T o[3], T n[3]) {
  NodeRef<T> N{nodes};
  int a = panel[0], b = panel[1], c = panel[2];
  T e1 = N.c(0, b) - N.c(0, a), e2 = N.c(1, b) - N.c(1, a), e3 = N.c(2, b) - N.c(2, a);
  T f1 = N.c(0, c) - N.c(0, a), f2 = N.c(1, c) - N.c(1, a), f3 = N.c(2, c) - N.c(2, a);
  T ne = sqrt(e1 * e1 + e2 * e2 + e3 * e3);
  t[0] = e1 / ne; t[1] = e2 / ne; t[2] = e3 / ne;
  T c1 = e2 * f3 - e3 * f2, c2 = e3 * f1 - e1 * f3, c3 = e1 * f2 - e2 * f1;
  T nc = sqrt(c1 * c1 + c2 * c2 + c3 * c3);
  n[0] = c1 / nc; n[1] = c2 / nc; n[2] = c3 / nc;
  o[0] = n[1] * t[2] - n[2] * t[1];
  o[1] = n[2] * t[0] - n[0] * t[2];
  o[2] = n[0] * t[1] - n[1] * t[0];
}

// ================================================================ SOURCE
// U_constant_source: src/FLOWPanel_elements.jl:29-141 (Hess & Smith 1967).
// If dot_with != nullptr, out[ti] += strength * U . dot_with[:, ti]
// otherwise out[3ti+k] += strength * U_k.
template <class T>
void U_constant_source(const T* nodes, const int* panel, int nn, T strength,
                       const T* targets, int64_t nt, T* out, const T* dot_with,
                       double offset) {
  NodeRef<T> N{nodes};
  T tt[3], oo[3], nnv[3];
  panel_frame(nodes, panel, tt, oo, nnv);
  // :51-56 flip: (t, o, n) <- (o, t, -n)
  T t1 = oo[0], t2 = oo[1], t3 = oo[2];
  T o1 = tt[0], o2 = tt[1], o3 = tt[2];
  T n1 = -nnv[0], n2 = -nnv[1], n3 = -nnv[2];
  int Oi = panel[0];
  for (int64_t ti = 0; ti < nt; ++ti) {
    const T* X = targets + 3 * ti;
    T x = t1 * (X[0] - N.c(0, Oi)) + t2 * (X[1] - N.c(1, Oi)) + t3 * (X[2] - N.c(2, Oi));
    T y = o1 * (X[0] - N.c(0, Oi)) + o2 * (X[1] - N.c(1, Oi)) + o3 * (X[2] - N.c(2, Oi));
    T z = n1 * (X[0] - N.c(0, Oi)) + n2 * (X[1] - N.c(1, Oi)) + n3 * (X[2] - N.c(2, Oi));
    T V1(0.0), V2(0.0), V3(0.0);
    double dtheta = 2 * PI;
    int nR0 = 0;
    for (int i = 0; i < nn; ++i) {
      int pi = panel[i], pj = panel[(i + 1) % nn];
      T xi = t1 * (N.c(0, pi) - N.c(0, Oi)) + t2 * (N.c(1, pi) - N.c(1, Oi)) + t3 * (N.c(2, pi) - N.c(2, Oi));
      T yi = o1 * (N.c(0, pi) - N.c(0, Oi)) + o2 * (N.c(1, pi) - N.c(1, Oi)) + o3 * (N.c(2, pi) - N.c(2, Oi));
      T zi = n1 * (N.c(0, pi) - N.c(0, Oi)) + n2 * (N.c(1, pi) - N.c(1, Oi)) + n3 * (N.c(2, pi) - N.c(2, Oi));
      T xj = t1 * (N.c(0, pj) - N.c(0, Oi)) + t2 * (N.c(1, pj) - N.c(1, Oi)) + t3 * (N.c(2, pj) - N.c(2, Oi));
      T yj = o1 * (N.c(0, pj) - N.c(0, Oi)) + o2 * (N.c(1, pj) - N.c(1, Oi)) + o3 * (N.c(2, pj) - N.c(2, Oi));
      T zj = n1 * (N.c(0, pj) - N.c(0, Oi)) + n2 * (N.c(1, pj) - N.c(1, Oi)) + n3 * (N.c(2, pj) - N.c(2, Oi));
      T dij = sqrt(sq(xj - xi) + sq(yj - yi) + sq(zj - zi));
      T ri = sqrt(sq(x - xi) + sq(y - yi) + sq(z - zi));
      T rj = sqrt(sq(x - xj) + sq(y - yj) + sq(z - zj));
      T Qij = log((ri + rj + dij) / (ri + rj - dij + offset));
      T Sij = (yj - yi) / dij;
      T Cij = (xj - xi) / dij;
      T siji = (xi - x) * Cij + (yi - y) * Sij;
      T sijj = (xj - x) * Cij + (yj - y) * Sij;
      T Rij = (x - xi) * Sij - (y - yi) * Cij;
      T Jij = atan2(Rij * abs(z) * (ri * sijj - rj * siji), ri * rj * sq(Rij) + sq(z) * sijj * siji);
      V1 -= Sij * Qij;
      V2 += Cij * Qij;
      V3 -= Jij;
      dtheta *= (value_of(Rij) >= 0);
      nR0 += (value_of(Rij) == 0);
    }
    V3 += T(dtheta);
    V3 *= T(jsign(z));
    V3 *= T((double)!(nR0 > 1));
    V1 *= T(1 / (4 * PI));
    V2 *= T(1 / (4 * PI));
    V3 *= T(1 / (4 * PI));
    if (dot_with) {
      const T* D = dot_with + 3 * ti;
      out[ti] += strength * (V1 * t1 + V2 * o1 + V3 * n1) * D[0];
      out[ti] += strength * (V1 * t2 + V2 * o2 + V3 * n2) * D[1];
      out[ti] += strength * (V1 * t3 + V2 * o3 + V3 * n3) * D[2];
    } else {
      out[3 * ti + 0] += strength * (V1 * t1 + V2 * o1 + V3 * n1);
      out[3 * ti + 1] += strength * (V1 * t2 + V2 * o2 + V3 * n2);
      out[3 * ti + 2] += strength * (V1 * t3 + V2 * o3 + V3 * n3);
    }
  }
}

// phi_constant_source: src/FLOWPanel_elements.jl:152-241 (Hess & Smith p. 53).
template <class T>
void phi_constant_source(const T* nodes, const int* panel, int nn, T strength,
                         const T* targets, int64_t nt, T* out, double offset) {
  NodeRef<T> N{nodes};
  T tt[3], oo[3], nnv[3];
  panel_frame(nodes, panel, tt, oo, nnv);
  T t1 = oo[0], t2 = oo[1], t3 = oo[2];
  T o1 = tt[0], o2 = tt[1], o3 = tt[2];
  T n1 = -nnv[0], n2 = -nnv[1], n3 = -nnv[2];
  int Oi = panel[0];
  for (int64_t ti = 0; ti < nt; ++ti) {
    const T* X = targets + 3 * ti;
    T x = t1 * (X[0] - N.c(0, Oi)) + t2 * (X[1] - N.c(1, Oi)) + t3 * (X[2] - N.c(2, Oi));
    T y = o1 * (X[0] - N.c(0, Oi)) + o2 * (X[1] - N.c(1, Oi)) + o3 * (X[2] - N.c(2, Oi));
    T z = n1 * (X[0] - N.c(0, Oi)) + n2 * (X[1] - N.c(1, Oi)) + n3 * (X[2] - N.c(2, Oi));
    double dtheta = 2 * PI;
    for (int i = 0; i < nn; ++i) {
      int pi = panel[i], pj = panel[(i + 1) % nn];
      T xi = t1 * (N.c(0, pi) - N.c(0, Oi)) + t2 * (N.c(1, pi) - N.c(1, Oi)) + t3 * (N.c(2, pi) - N.c(2, Oi));
      T yi = o1 * (N.c(0, pi) - N.c(0, Oi)) + o2 * (N.c(1, pi) - N.c(1, Oi)) + o3 * (N.c(2, pi) - N.c(2, Oi));
      T zi = n1 * (N.c(0, pi) - N.c(0, Oi)) + n2 * (N.c(1, pi) - N.c(1, Oi)) + n3 * (N.c(2, pi) - N.c(2, Oi));
      T xj = t1 * (N.c(0, pj) - N.c(0, Oi)) + t2 * (N.c(1, pj) - N.c(1, Oi)) + t3 * (N.c(2, pj) - N.c(2, Oi));
      T yj = o1 * (N.c(0, pj) - N.c(0, Oi)) + o2 * (N.c(1, pj) - N.c(1, Oi)) + o3 * (N.c(2, pj) - N.c(2, Oi));
      T zj = n1 * (N.c(0, pj) - N.c(0, Oi)) + n2 * (N.c(1, pj) - N.c(1, Oi)) + n3 * (N.c(2, pj) - N.c(2, Oi));
      T dij = sqrt(sq(xj - xi) + sq(yj - yi) + sq(zj - zi));
      T ri = sqrt(sq(x - xi) + sq(y - yi) + sq(z - zi));
      T rj = sqrt(sq(x - xj) + sq(y - yj) + sq(z - zj));
      T Qij = log((ri + rj + dij) / (ri + rj - dij + offset));
      T Sij = (yj - yi) / dij;
      T Cij = (xj - xi) / dij;
      T siji = (xi - x) * Cij + (yi - y) * Sij;
      T sijj = (xj - x) * Cij + (yj - y) * Sij;
      T Rij = (x - xi) * Sij - (y - yi) * Cij;
      T Jij = atan2(Rij * abs(z) * (ri * sijj - rj * siji), ri * rj * sq(Rij) + sq(z) * sijj * siji);
      out[ti] -= strength / (4 * PI) * (Rij * Qij + abs(z) * Jij);
      dtheta *= (value_of(Rij) >= 0);
    }
    out[ti] += strength / (4 * PI) * abs(z) * T(dtheta);
  }
}

// ================================================================ VORTEX FILAMENTS
// U_boundvortex: src/FLOWPanel_elements.jl:345-428. One target.
template <class T>
inline void U_boundvortex_one(const T& pa1, const T& pa2, const T& pa3,
                              const T& pb1, const T& pb2, const T& pb3,
                              const T& strength, const T* X, T* out3, T* outdot,
                              const T* D, double cutoff, double offset) {
  T rij1 = pb1 - pa1, rij2 = pb2 - pa2, rij3 = pb3 - pa3;
  T ri1 = X[0] - pa1, ri2 = X[1] - pa2, ri3 = X[2] - pa3;
  T rj1 = X[0] - pb1, rj2 = X[1] - pb2, rj3 = X[2] - pb3;
  T rixrj1 = ri2 * rj3 - ri3 * rj2;
  T rixrj2 = ri3 * rj1 - ri1 * rj3;
  T rixrj3 = ri1 * rj2 - ri2 * rj1;
  T dotrixrj = sq(rixrj1) + sq(rixrj2) + sq(rixrj3);
  T normri = sqrt(sq(ri1) + sq(ri2) + sq(ri3)) + offset;
  T normrj = sqrt(sq(rj1) + sq(rj2) + sq(rj3)) + offset;
  T rijdothat = rij1 * (ri1 / normri - rj1 / normrj) + rij2 * (ri2 / normri - rj2 / normrj) +
                rij3 * (ri3 / normri - rj3 / normrj);
  if (value_of(dotrixrj) > cutoff * cutoff) {
    T aux = strength * rijdothat / (4 * PI * (dotrixrj + offset * offset));
    if (outdot) {
      *outdot += aux * (rixrj1 * D[0] + rixrj2 * D[1] + rixrj3 * D[2]);
    } else {
      out3[0] += aux * rixrj1;
      out3[1] += aux * rixrj2;
      out3[2] += aux * rixrj3;
    }
  }
}

template <class T>
void U_boundvortex(const T& pa1, const T& pa2, const T& pa3, const T& pb1, const T& pb2,
                   const T& pb3, T strength, const T* targets, int64_t nt, T* out,
                   const T* dot_with, double cutoff, double offset) {
  for (int64_t ti = 0; ti < nt; ++ti) {
    if (dot_with)
      U_boundvortex_one(pa1, pa2, pa3, pb1, pb2, pb3, strength, targets + 3 * ti, (T*)nullptr,
                        out + ti, dot_with + 3 * ti, cutoff, offset);
    else
      U_boundvortex_one(pa1, pa2, pa3, pb1, pb2, pb3, strength, targets + 3 * ti, out + 3 * ti,
                        (T*)nullptr, (const T*)nullptr, cutoff, offset);
  }
}

// U_vortexring == U_constant_doublet: src/FLOWPanel_elements.jl:442-467,740.
template <class T>
void U_vortexring(const T* nodes, const int* panel, int nn, T strength, const T* targets,
                  int64_t nt, T* out, const T* dot_with, double cutoff, double offset) {
  NodeRef<T> N{nodes};
  for (int i = 0; i < nn; ++i) {
    int pi = panel[i], pj = panel[(i + 1) % nn];
    U_boundvortex(N.c(0, pi), N.c(1, pi), N.c(2, pi), N.c(0, pj), N.c(1, pj), N.c(2, pj),
                  strength, targets, nt, out, dot_with, cutoff, offset);
  }
}

// U_semiinfinite_vortex: src/FLOWPanel_elements.jl:480-628. One target.
template <class T>
inline void U_semiinfinite_vortex_one(const T& p1, const T& p2, const T& p3, const T& d1,
                                      const T& d2, const T& d3, const T& strength, const T* X,
                                      T* out3, T* outdot, const T* D, double cutoff,
                                      double offset) {
  T xmpdotd = (X[0] - p1) * d1 + (X[1] - p2) * d2 + (X[2] - p3) * d3;
  T p01 = p1 + xmpdotd * d1;
  T p02 = p2 + xmpdotd * d2;
  T p03 = p3 + xmpdotd * d3;
  // bound section :513-577
  if (value_of(sq(p01 - p1) + sq(p02 - p2) + sq(p03 - p3)) > offset * offset) {
    T rij1 = p01 - p1, rij2 = p02 - p2, rij3 = p03 - p3;
    T ri1 = X[0] - p1, ri2 = X[1] - p2, ri3 = X[2] - p3;
    T rj1 = X[0] - p01, rj2 = X[1] - p02, rj3 = X[2] - p03;
    T rixrj1 = ri2 * rj3 - ri3 * rj2;
    T rixrj2 = ri3 * rj1 - ri1 * rj3;
    T rixrj3 = ri1 * rj2 - ri2 * rj1;
    T dotrixrj = sq(rixrj1) + sq(rixrj2) + sq(rixrj3);
    T normri = sqrt(sq(ri1) + sq(ri2) + sq(ri3)) + offset;
    T normrj = sqrt(sq(rj1) + sq(rj2) + sq(rj3)) + offset;
    T rijdothat = rij1 * (ri1 / normri - rj1 / normrj) + rij2 * (ri2 / normri - rj2 / normrj) +
                  rij3 * (ri3 / normri - rj3 / normrj);
    if (value_of(dotrixrj) > cutoff * cutoff) {
      T aux = strength * rijdothat / (4 * PI * (dotrixrj + offset * offset));
      if (outdot) {
        *outdot += aux * (rixrj1 * D[0] + rixrj2 * D[1] + rixrj3 * D[2]);
      } else {
        out3[0] += aux * rixrj1;
        out3[1] += aux * rixrj2;
        out3[2] += aux * rixrj3;
      }
    }
  }
  // semi-infinite section :582-624
  T hsqr = sq(X[0] - p01) + sq(X[1] - p02) + sq(X[2] - p03);
  T h1 = X[0] - p01, h2 = X[1] - p02, h3 = X[2] - p03;
  T n1 = d2 * h3 - d3 * h2;
  T n2 = d3 * h1 - d1 * h3;
  T n3 = d1 * h2 - d2 * h1;
  if (value_of(hsqr) > cutoff * cutoff) {
    T aux = strength / (4 * PI * (hsqr + offset * offset));
    if (outdot) {
      *outdot += aux * (n1 * D[0] + n2 * D[1] + n3 * D[2]);
    } else {
      out3[0] += aux * n1;
      out3[1] += aux * n2;
      out3[2] += aux * n3;
    }
  }
}

// Unit-direction check of src/FLOWPanel_elements.jl:495-498 (abs(|d|^2-1) > 2eps -> error).
inline bool is_unit(double d1, double d2, double d3) {
  return !(std::abs(d1 * d1 + d2 * d2 + d3 * d3 - 1) > 2 * 2.220446049250313e-16);
}

// U_semiinfinite_horseshoe with (da, db): src/FLOWPanel_elements.jl:692-730.
// pa = nodes[:, TE0], pb = nodes[:, TE1]. One target.
template <class T>
inline void U_semiinfinite_horseshoe_one(const T* nodes, int TE0, int TE1, const T& da1,
                                         const T& da2, const T& da3, const T& db1,
                                         const T& db2, const T& db3, const T& strength,
                                         const T* X, T* out3, T* outdot, const T* D,
                                         double cutoff, double offset) {
  NodeRef<T> N{nodes};
  U_semiinfinite_vortex_one(N.c(0, TE0), N.c(1, TE0), N.c(2, TE0), da1, da2, da3, -strength, X,
                            out3, outdot, D, cutoff, offset);
  U_boundvortex_one(N.c(0, TE0), N.c(1, TE0), N.c(2, TE0), N.c(0, TE1), N.c(1, TE1),
                    N.c(2, TE1), strength, X, out3, outdot, D, cutoff, offset);
  U_semiinfinite_vortex_one(N.c(0, TE1), N.c(1, TE1), N.c(2, TE1), db1, db2, db3, strength, X,
                            out3, outdot, D, cutoff, offset);
}

// The reference applies each sub-element to all targets before the next
// sub-element (:706-729); per target the accumulation order is the same as
// applying the three sub-elements in turn, which is what _one does.
template <class T>
void U_semiinfinite_horseshoe(const T* nodes, int TE0, int TE1, T da1, T da2, T da3, T db1,
                              T db2, T db3, T strength, const T* targets, int64_t nt, T* out,
                              const T* dot_with, double cutoff, double offset) {
  for (int64_t ti = 0; ti < nt; ++ti) {
    if (dot_with)
      U_semiinfinite_horseshoe_one(nodes, TE0, TE1, da1, da2, da3, db1, db2, db3, strength,
                                   targets + 3 * ti, (T*)nullptr, out + ti, dot_with + 3 * ti,
                                   cutoff, offset);
    else
      U_semiinfinite_horseshoe_one(nodes, TE0, TE1, da1, da2, da3, db1, db2, db3, strength,
                                   targets + 3 * ti, out + 3 * ti, (T*)nullptr,
                                   (const T*)nullptr, cutoff, offset);
  }
}

// ================================================================ DOUBLET POTENTIALS
// Shared Hess-Smith solid-angle term used by phi_constant_doublet and the
// bound part of phi_semiinfinite_doublet (src/FLOWPanel_elements.jl:796-833,1025-1061).
template <class T>
inline T hs_solid_angle(const T& x, const T& y, const T& z, const T* xs, const T* ys,
                        const T* zs, int nn) {
  T V3(0.0);
  double dtheta = 2 * PI;
  int nR0 = 0;
  for (int i = 0; i < nn; ++i) {
    int j = (i + 1) % nn;
    const T &xi = xs[i], &yi = ys[i], &zi = zs[i], &xj = xs[j], &yj = ys[j], &zj = zs[j];
    T dij = sqrt(sq(xj - xi) + sq(yj - yi) + sq(zj - zi));
    T ri = sqrt(sq(x - xi) + sq(y - yi) + sq(z - zi));
    T rj = sqrt(sq(x - xj) + sq(y - yj) + sq(z - zj));
    T Sij = (yj - yi) / dij;
    T Cij = (xj - xi) / dij;
    T siji = (xi - x) * Cij + (yi - y) * Sij;
    T sijj = (xj - x) * Cij + (yj - y) * Sij;
    T Rij = (x - xi) * Sij - (y - yi) * Cij;
    T Jij = atan2(Rij * abs(z) * (ri * sijj - rj * siji), ri * rj * sq(Rij) + sq(z) * sijj * siji);
    V3 -= Jij;
    dtheta *= (value_of(Rij) >= 0);
    nR0 += (value_of(Rij) == 0);
  }
  V3 += T(dtheta);
  V3 *= T(jsign(z));
  V3 *= T((double)!(nR0 > 1));
  V3 *= T(1 / (4 * PI));
  return V3;
}

// phi_constant_doublet: src/FLOWPanel_elements.jl:751-847.
template <class T>
void phi_constant_doublet(const T* nodes, const int* panel, int nn, T strength,
                          const T* targets, int64_t nt, T* out) {
  NodeRef<T> N{nodes};
  T tt[3], oo[3], nnv[3];
  panel_frame(nodes, panel, tt, oo, nnv);
  T t1 = oo[0], t2 = oo[1], t3 = oo[2];
  T o1 = tt[0], o2 = tt[1], o3 = tt[2];
  T n1 = -nnv[0], n2 = -nnv[1], n3 = -nnv[2];
  int Oi = panel[0];
  std::vector<T> xs(nn), ys(nn), zs(nn);
  for (int i = 0; i < nn; ++i) {
    int p = panel[i];
    xs[i] = t1 * (N.c(0, p) - N.c(0, Oi)) + t2 * (N.c(1, p) - N.c(1, Oi)) + t3 * (N.c(2, p) - N.c(2, Oi));
    ys[i] = o1 * (N.c(0, p) - N.c(0, Oi)) + o2 * (N.c(1, p) - N.c(1, Oi)) + o3 * (N.c(2, p) - N.c(2, Oi));
    zs[i] = n1 * (N.c(0, p) - N.c(0, Oi)) + n2 * (N.c(1, p) - N.c(1, Oi)) + n3 * (N.c(2, p) - N.c(2, Oi));
  }
  for (int64_t ti = 0; ti < nt; ++ti) {
    const T* X = targets + 3 * ti;
    T x = t1 * (X[0] - N.c(0, Oi)) + t2 * (X[1] - N.c(1, Oi)) + t3 * (X[2] - N.c(2, Oi));
    T y = o1 * (X[0] - N.c(0, Oi)) + o2 * (X[1] - N.c(1, Oi)) + o3 * (X[2] - N.c(2, Oi));
    T z = n1 * (X[0] - N.c(0, Oi)) + n2 * (X[1] - N.c(1, Oi)) + n3 * (X[2] - N.c(2, Oi));
    T V3 = hs_solid_angle(x, y, z, xs.data(), ys.data(), zs.data(), nn);
    out[ti] += strength * V3;
  }
}

// phi_semiinfinite_doublet (single direction d): src/FLOWPanel_elements.jl:959-1092
// (Moran 1984, App. F). Returns false on a non-unit direction.
template <class T>
bool phi_semiinfinite_doublet(const T* nodes, int TE0, int TE1, T d1, T d2, T d3, T strength,
                              const T* targets, int64_t nt, T* out) {
  if (!is_unit(value_of(d1), value_of(d2), value_of(d3))) return false;
  NodeRef<T> N{nodes};
  T p_i1 = N.c(0, TE0), p_i2 = N.c(1, TE0), p_i3 = N.c(2, TE0);
  T p_j1 = N.c(0, TE1), p_j2 = N.c(1, TE1), p_j3 = N.c(2, TE1);
  T pijdotd = (p_j1 - p_i1) * d1 + (p_j2 - p_i2) * d2 + (p_j3 - p_i3) * d3;
  T pa1 = p_i1 + pijdotd * d1, pa2 = p_i2 + pijdotd * d2, pa3 = p_i3 + pijdotd * d3;
  T x1 = d1, x2 = d2, x3 = d3;
  T nrmpbpa = sqrt(sq(p_j1 - pa1) + sq(p_j2 - pa2) + sq(p_j3 - pa3));
  T y1 = (p_j1 - pa1) / nrmpbpa, y2 = (p_j2 - pa2) / nrmpbpa, y3 = (p_j3 - pa3) / nrmpbpa;
  T z1 = x2 * y3 - x3 * y2, z2 = x3 * y1 - x1 * y3, z3 = x1 * y2 - x2 * y1;
  T O1 = p_i1, O2 = p_i2, O3 = p_i3;
  auto lx = [&](const T& a, const T& b, const T& c) { return x1 * (a - O1) + x2 * (b - O2) + x3 * (c - O3); };
  auto ly = [&](const T& a, const T& b, const T& c) { return y1 * (a - O1) + y2 * (b - O2) + y3 * (c - O3); };
  auto lz = [&](const T& a, const T& b, const T& c) { return z1 * (a - O1) + z2 * (b - O2) + z3 * (c - O3); };
  // bound triangle (p_a, p_i, p_j) in local coordinates
  T xs[3] = {lx(pa1, pa2, pa3), lx(p_i1, p_i2, p_i3), lx(p_j1, p_j2, p_j3)};
  T ys[3] = {ly(pa1, pa2, pa3), ly(p_i1, p_i2, p_i3), ly(p_j1, p_j2, p_j3)};
  T zs[3] = {lz(pa1, pa2, pa3), lz(p_i1, p_i2, p_i3), lz(p_j1, p_j2, p_j3)};
  T xa = xs[0], ya = ys[0];
  T yb = ly(p_j1, p_j2, p_j3);
  for (int64_t ti = 0; ti < nt; ++ti) {
    const T* X = targets + 3 * ti;
    T x = lx(X[0], X[1], X[2]);
    T y = ly(X[0], X[1], X[2]);
    T z = lz(X[0], X[1], X[2]);
    if (std::abs(value_of(pijdotd)) > 2 * 2.220446049250313e-16) {
      T V3 = hs_solid_angle(x, y, z, xs, ys, zs, 3);
      out[ti] += strength * V3;
    }
    T val(0.0);
    val += atan((yb - y) / z) + atan((yb - y) * (x - xa) / (z * sqrt(sq(x - xa) + sq(yb - y) + sq(z))));
    val -= atan((ya - y) / z) + atan((ya - y) * (x - xa) / (z * sqrt(sq(x - xa) + sq(ya - y) + sq(z))));
    out[ti] += strength / (4 * PI) * val;
  }
  return true;
}

// phi_semiinfinite_doublet (da, db): src/FLOWPanel_elements.jl:1110-1244.
template <class T>
bool phi_semiinfinite_doublet2(const T* nodes, int TE0, int TE1, T da1, T da2, T da3, T db1,
                               T db2, T db3, T strength, const T* targets, int64_t nt, T* out,
                               double infinitelength) {
  if (!is_unit(value_of(da1), value_of(da2), value_of(da3))) return false;
  if (!is_unit(value_of(db1), value_of(db2), value_of(db3))) return false;
  if (value_of(da1 * db1 + da2 * db2 + da3 * db3) <= 0) return false;
  phi_semiinfinite_doublet(nodes, TE0, TE1, da1, da2, da3, strength, targets, nt, out);
  const double e2 = 2 * 2.220446049250313e-16;
  if (std::abs(value_of(da1 - db1)) > e2 || std::abs(value_of(da2 - db2)) > e2 ||
      std::abs(value_of(da3 - db3)) > e2) {
    NodeRef<T> N{nodes};
    T pb1 = N.c(0, TE1), pb2 = N.c(1, TE1), pb3 = N.c(2, TE1);
    T pda1 = pb1 + infinitelength * da1, pda2 = pb2 + infinitelength * da2, pda3 = pb3 + infinitelength * da3;
    T pdb1 = pb1 + infinitelength * db1, pdb2 = pb2 + infinitelength * db2, pdb3 = pb3 + infinitelength * db3;
    T x1 = da1, x2 = da2, x3 = da3;
    T z1 = da2 * db3 - da3 * db2, z2 = da3 * db1 - da1 * db3, z3 = da1 * db2 - da2 * db1;
    T nrmz = sqrt(z1 * z1 + z2 * z2 + z3 * z3);
    z1 = z1 / nrmz; z2 = z2 / nrmz; z3 = z3 / nrmz;
    T y1 = z2 * x3 - z3 * x2, y2 = z3 * x1 - z1 * x3, y3 = z1 * x2 - z2 * x1;
    T O1 = pb1, O2 = pb2, O3 = pb3;
    auto lx = [&](const T& a, const T& b, const T& c) { return x1 * (a - O1) + x2 * (b - O2) + x3 * (c - O3); };
    auto ly = [&](const T& a, const T& b, const T& c) { return y1 * (a - O1) + y2 * (b - O2) + y3 * (c - O3); };
    auto lz = [&](const T& a, const T& b, const T& c) { return z1 * (a - O1) + z2 * (b - O2) + z3 * (c - O3); };
    // triangle (pda, pb, pdb) :1201-1210
    T xs[3] = {lx(pda1, pda2, pda3), lx(pb1, pb2, pb3), lx(pdb1, pdb2, pdb3)};
    T ys[3] = {ly(pda1, pda2, pda3), ly(pb1, pb2, pb3), ly(pdb1, pdb2, pdb3)};
    T zs[3] = {lz(pda1, pda2, pda3), lz(pb1, pb2, pb3), lz(pdb1, pdb2, pdb3)};
    for (int64_t ti = 0; ti < nt; ++ti) {
      const T* X = targets + 3 * ti;
      T x = lx(X[0], X[1], X[2]);
      T y = ly(X[0], X[1], X[2]);
      T z = lz(X[0], X[1], X[2]);
      out[ti] += strength * hs_solid_angle(x, y, z, xs, ys, zs, 3);
    }
  }
  return true;
}

// ================================================================ GEOMETRY
// Control point, normal, area and characteristic length of each panel.
// _calc_normals!: src/FLOWPanel_abstractbody.jl:738-755.
// _calc_controlpoints!: src/FLOWPanel_abstractbody.jl:635-694 (vertex mean, in-plane
// centroid correction, then + off * l * n).
// _calc_areas!: src/FLOWPanel_abstractbody.jl:905-917 with GeometricTools' polygon area
// (unvendored): restated as the fan of triangles from the first node.
template <class T>
void panel_normal(const T* nodes, const int* panel, T n[3]) {
  T t[3], o[3];
  panel_frame(nodes, panel, t, o, n);
}

template <class T>
void panel_controlpoint(const T* nodes, const int* panel, int nn, const T n[3], double off,
                        double l, T cp[3]) {
  NodeRef<T> N{nodes};
  T c1(0.0), c2(0.0), c3(0.0);
  for (int k = 0; k < nn; ++k) {
    c1 += N.c(0, panel[k]); c2 += N.c(1, panel[k]); c3 += N.c(2, panel[k]);
  }
  c1 = c1 / T((double)nn); c2 = c2 / T((double)nn); c3 = c3 / T((double)nn);
  T t[3], o[3], nn_[3];
  panel_frame(nodes, panel, t, o, nn_);
  T x(0.0), y(0.0);
  for (int k = 0; k < nn; ++k) {
    int ni = panel[k];
    x += (N.c(0, ni) - c1) * t[0]; x += (N.c(1, ni) - c2) * t[1]; x += (N.c(2, ni) - c3) * t[2];
    y += (N.c(0, ni) - c1) * o[0]; y += (N.c(1, ni) - c2) * o[1]; y += (N.c(2, ni) - c3) * o[2];
  }
  x = x / T((double)nn); y = y / T((double)nn);
  c1 += x * t[0] + y * o[0];
  c2 += x * t[1] + y * o[1];
  c3 += x * t[2] + y * o[2];
  c1 += off * l * n[0];
  c2 += off * l * n[1];
  c3 += off * l * n[2];
  cp[0] = c1; cp[1] = c2; cp[2] = c3;
}

template <class T>
T panel_area(const T* nodes, const int* panel, int nn) {
  NodeRef<T> N{nodes};
  T a(0.0);
  int p0 = panel[0];
  for (int k = 1; k + 1 < nn; ++k) {
    int p1 = panel[k], p2 = panel[k + 1];
    T e1 = N.c(0, p1) - N.c(0, p0), e2 = N.c(1, p1) - N.c(1, p0), e3 = N.c(2, p1) - N.c(2, p0);
    T f1 = N.c(0, p2) - N.c(0, p0), f2 = N.c(1, p2) - N.c(1, p0), f3 = N.c(2, p2) - N.c(2, p0);
    T c1 = e2 * f3 - e3 * f2, c2 = e3 * f1 - e1 * f3, c3 = e1 * f2 - e2 * f1;
    a += 0.5 * sqrt(c1 * c1 + c2 * c2 + c3 * c3);
  }
  return a;
}

}  // namespace fpo
