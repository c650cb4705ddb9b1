// ORACLE — test infrastructure only (see fp_oracle.hpp). C entry points for
// ctypes. Arrays are column-major 3 x n doubles; panels are CSR
// (offsets[npanels+1], node indices 0-based); shedding is 6 x nsh int32
// (pi, nia, nib, pj, nja, njb), 0-based, pj == -1 for no lower side.
#include <omp.h>

#include <cstring>

#include "fp_oracle.hpp"

using namespace fpo;

namespace {
template <class T, class S>
std::vector<T> cast_vec(const S* a, int64_t n) {
  std::vector<T> r(n);
  for (int64_t i = 0; i < n; ++i) r[i] = T(a[i]);
  return r;
}
}  // namespace

extern "C" {

// ------------------------------------------------------------------ elements
void fpo_U_constant_source(const double* nodes, const int* panel, int nn, double strength,
                           const double* targets, long long nt, double* out,
                           const double* dot_with, double offset) {
  U_constant_source<double>(nodes, panel, nn, strength, targets, nt, out, dot_with, offset);
}
void fpo_phi_constant_source(const double* nodes, const int* panel, int nn, double strength,
                             const double* targets, long long nt, double* out, double offset) {
  phi_constant_source<double>(nodes, panel, nn, strength, targets, nt, out, offset);
}
void fpo_U_vortexring(const double* nodes, const int* panel, int nn, double strength,
                      const double* targets, long long nt, double* out, const double* dot_with,
                      double cutoff, double offset) {
  U_vortexring<double>(nodes, panel, nn, strength, targets, nt, out, dot_with, cutoff, offset);
}
void fpo_phi_constant_doublet(const double* nodes, const int* panel, int nn, double strength,
                              const double* targets, long long nt, double* out) {
  phi_constant_doublet<double>(nodes, panel, nn, strength, targets, nt, out);
}
void fpo_U_boundvortex(const double* pa, const double* pb, double strength,
                       const double* targets, long long nt, double* out,
                       const double* dot_with, double cutoff, double offset) {
  U_boundvortex<double>(pa[0], pa[1], pa[2], pb[0], pb[1], pb[2], strength, targets, nt, out,
                        dot_with, cutoff, offset);
}
// returns 0, or 1 when a direction is not unit (src/FLOWPanel_elements.jl:495-498)
int fpo_U_semiinfinite_vortex(const double* p, const double* d, double strength,
                              const double* targets, long long nt, double* out,
                              const double* dot_with, double cutoff, double offset) {
  if (!is_unit(d[0], d[1], d[2])) return 1;
  for (long long ti = 0; ti < nt; ++ti)
    U_semiinfinite_vortex_one<double>(p[0], p[1], p[2], d[0], d[1], d[2], strength,
                                      targets + 3 * ti, dot_with ? nullptr : out + 3 * ti,
                                      dot_with ? out + ti : nullptr,
                                      dot_with ? dot_with + 3 * ti : nullptr, cutoff, offset);
  return 0;
}
int fpo_U_semiinfinite_horseshoe(const double* nodes, int TE0, int TE1, const double* da,
                                 const double* db, double strength, const double* targets,
                                 long long nt, double* out, const double* dot_with,
                                 double cutoff, double offset) {
  if (!is_unit(da[0], da[1], da[2]) || !is_unit(db[0], db[1], db[2])) return 1;
  U_semiinfinite_horseshoe<double>(nodes, TE0, TE1, da[0], da[1], da[2], db[0], db[1], db[2],
                                   strength, targets, nt, out, dot_with, cutoff, offset);
  return 0;
}
int fpo_phi_semiinfinite_doublet(const double* nodes, int TE0, int TE1, const double* d,
                                 double strength, const double* targets, long long nt,
                                 double* out) {
  return phi_semiinfinite_doublet<double>(nodes, TE0, TE1, d[0], d[1], d[2], strength, targets,
                                          nt, out) ? 0 : 1;
}
int fpo_phi_semiinfinite_doublet2(const double* nodes, int TE0, int TE1, const double* da,
                                  const double* db, double strength, const double* targets,
                                  long long nt, double* out, double infinitelength) {
  return phi_semiinfinite_doublet2<double>(nodes, TE0, TE1, da[0], da[1], da[2], db[0], db[1],
                                           db[2], strength, targets, nt, out, infinitelength)
             ? 0 : 1;
}

// ------------------------------------------------------------------ dual-number derivatives
// grad phi at one target X (3), and the Jacobian dU_i/dX_j (row-major 3x3) at X.
// kind: 0 = constant source, 1 = constant doublet (ring), 2 = semi-infinite doublet (d)
void fpo_grad_phi(int kind, const double* nodes, int nnodes, const int* panel, int nn,
                  const double* d, double strength, const double* X, double offset,
                  double* grad) {
  typedef Dual<3> D3;
  std::vector<D3> N = cast_vec<D3>(nodes, 3 * (int64_t)nnodes);
  D3 XT[3];
  for (int k = 0; k < 3; ++k) { XT[k] = D3(X[k]); XT[k].d[k] = 1.0; }
  D3 out(0.0);
  if (kind == 0) phi_constant_source<D3>(N.data(), panel, nn, D3(strength), XT, 1, &out, offset);
  else if (kind == 1) phi_constant_doublet<D3>(N.data(), panel, nn, D3(strength), XT, 1, &out);
  else phi_semiinfinite_doublet<D3>(N.data(), panel[0], panel[1], D3(d[0]), D3(d[1]), D3(d[2]),
                                    D3(strength), XT, 1, &out);
  for (int k = 0; k < 3; ++k) grad[k] = out.d[k];
}

// kind: 0 = constant source, 1 = vortex ring, 2 = semi-infinite horseshoe (single d)
void fpo_jac_U(int kind, const double* nodes, int nnodes, const int* panel, int nn,
               const double* d, double strength, const double* X, double cutoff,
               double offset, double* U, double* J) {
  typedef Dual<3> D3;
  std::vector<D3> N = cast_vec<D3>(nodes, 3 * (int64_t)nnodes);
  D3 XT[3];
  for (int k = 0; k < 3; ++k) { XT[k] = D3(X[k]); XT[k].d[k] = 1.0; }
  D3 out[3] = {D3(0.0), D3(0.0), D3(0.0)};
  if (kind == 0)
    U_constant_source<D3>(N.data(), panel, nn, D3(strength), XT, 1, out, nullptr, offset);
  else if (kind == 1)
    U_vortexring<D3>(N.data(), panel, nn, D3(strength), XT, 1, out, nullptr, cutoff, offset);
  else
    U_semiinfinite_horseshoe<D3>(N.data(), panel[0], panel[1], D3(d[0]), D3(d[1]), D3(d[2]),
                                 D3(d[0]), D3(d[1]), D3(d[2]), D3(strength), XT, 1, out,
                                 nullptr, cutoff, offset);
  for (int i = 0; i < 3; ++i) {
    U[i] = out[i].v;
    for (int j = 0; j < 3; ++j) J[3 * i + j] = out[i].d[j];
  }
}

// ------------------------------------------------------------------ geometry
// off[i] and l[i] per panel (CPoffset * sign flips and characteristic length are
// resolved by the caller, as MultiBody does in src/FLOWPanel_multibody.jl:658-680).
void fpo_geometry(const double* nodes, const int* offsets, const int* pnodes, long long npanels,
                  const double* off, const double* l, double* normals, double* cps,
                  double* areas) {
  for (long long p = 0; p < npanels; ++p) {
    const int* panel = pnodes + offsets[p];
    int nn = offsets[p + 1] - offsets[p];
    double n[3];
    panel_normal<double>(nodes, panel, n);
    if (normals) { normals[3 * p] = n[0]; normals[3 * p + 1] = n[1]; normals[3 * p + 2] = n[2]; }
    if (cps) panel_controlpoint<double>(nodes, panel, nn, n, off ? off[p] : 0.0, l ? l[p] : 1.0, cps + 3 * p);
    if (areas) areas[p] = panel_area<double>(nodes, panel, nn);
  }
}

// ------------------------------------------------------------------ assembly
// Vortex-ring AIC with Kutta wake columns: src/FLOWPanel_liftingbody.jl:455-572.
// G is ncp x npanels column-major (leading dimension ncp). Returns 1 on a
// non-unit wake direction.
int fpo_assemble_vortexring(const double* nodes, const int* offsets, const int* pnodes,
                            long long npanels, const double* cps, const double* normals,
                            long long ncp, const int* shedding, long long nsh,
                            const double* Das, const double* Dbs, double offset,
                            double cutoff, double* G, int nthreads) {
  for (long long e = 0; e < nsh; ++e)
    if (!is_unit(Das[3 * e], Das[3 * e + 1], Das[3 * e + 2]) ||
        !is_unit(Dbs[3 * e], Dbs[3 * e + 1], Dbs[3 * e + 2]))
      return 1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  // HOT LOOP 1, threaded over panels like :476-503
#pragma omp parallel for schedule(static)
  for (long long pj = 0; pj < npanels; ++pj) {
    const int* panel = pnodes + offsets[pj];
    int nn = offsets[pj + 1] - offsets[pj];
    U_vortexring<double>(nodes, panel, nn, 1.0, cps, ncp, G + pj * ncp, normals, cutoff, offset);
  }
  // HOT LOOP 2, wake columns :508-567; different edges may touch the same
  // column, so this loop is serial to keep the reference's per-column order.
  for (long long e = 0; e < nsh; ++e) {
    const int* s = shedding + 6 * e;
    int pi = s[0], nia = s[1], nib = s[2], pj = s[3], nja = s[4], njb = s[5];
    const int* pan = pnodes + offsets[pi];
    const double* da = Das + 3 * e;
    const double* db = Dbs + 3 * e;
    U_semiinfinite_horseshoe<double>(nodes, pan[nia], pan[nib], da[0], da[1], da[2], db[0],
                                     db[1], db[2], 1.0, cps, ncp, G + (long long)pi * ncp,
                                     normals, cutoff, offset);
    if (pj != -1) {
      const int* panj = pnodes + offsets[pj];
      U_semiinfinite_horseshoe<double>(nodes, panj[nja], panj[njb], db[0], db[1], db[2], da[0],
                                       da[1], da[2], 1.0, cps, ncp, G + (long long)pj * ncp,
                                       normals, cutoff, offset);
    }
  }
  return 0;
}

// Constant-source AIC: src/FLOWPanel_nonliftingbody.jl:141-186.
void fpo_assemble_source(const double* nodes, const int* offsets, const int* pnodes,
                         long long npanels, const double* cps, const double* normals,
                         long long ncp, double offset, double* G, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (long long pj = 0; pj < npanels; ++pj) {
    const int* panel = pnodes + offsets[pj];
    int nn = offsets[pj + 1] - offsets[pj];
    U_constant_source<double>(nodes, panel, nn, 1.0, cps, ncp, G + pj * ncp, normals, offset);
  }
}

// ------------------------------------------------------------------ induced velocity
// _Uvortexring!: src/FLOWPanel_liftingbody.jl:576-661. out (3 x nt) accumulates.
// Parallel over target chunks: each target sees the panels (then the wake) in
// the reference's order, so the per-target sums are the reference's.
int fpo_uind_vortexring(const double* nodes, const int* offsets, const int* pnodes,
                        long long npanels, const double* strength, const int* shedding,
                        long long nsh, const double* Das, const double* Dbs, double offset,
                        double cutoff, const double* targets, long long nt, double* out,
                        int nthreads) {
  for (long long e = 0; e < nsh; ++e)
    if (!is_unit(Das[3 * e], Das[3 * e + 1], Das[3 * e + 2]) ||
        !is_unit(Dbs[3 * e], Dbs[3 * e + 1], Dbs[3 * e + 2]))
      return 1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const long long CH = 64;
#pragma omp parallel for schedule(dynamic)
  for (long long t0 = 0; t0 < nt; t0 += CH) {
    long long n = (nt - t0 < CH) ? nt - t0 : CH;
    const double* T = targets + 3 * t0;
    double* O = out + 3 * t0;
    for (long long i = 0; i < npanels; ++i) {
      const int* panel = pnodes + offsets[i];
      int nn = offsets[i + 1] - offsets[i];
      U_vortexring<double>(nodes, panel, nn, strength[i], T, n, O, nullptr, cutoff, offset);
    }
    for (long long e = 0; e < nsh; ++e) {
      const int* s = shedding + 6 * e;
      int pi = s[0], nia = s[1], nib = s[2], pj = s[3], nja = s[4], njb = s[5];
      // _get_wakestrength_mu: src/FLOWPanel_liftingbody.jl:1078-1082
      double si = strength[pi], sj = (pj != -1) ? strength[pj] : 0.0;
      const int* pan = pnodes + offsets[pi];
      const double* da = Das + 3 * e;
      const double* db = Dbs + 3 * e;
      U_semiinfinite_horseshoe<double>(nodes, pan[nia], pan[nib], da[0], da[1], da[2], db[0],
                                       db[1], db[2], si, T, n, O, nullptr, cutoff, offset);
      if (pj != -1) {
        const int* panj = pnodes + offsets[pj];
        U_semiinfinite_horseshoe<double>(nodes, panj[nja], panj[njb], db[0], db[1], db[2],
                                         da[0], da[1], da[2], sj, T, n, O, nullptr, cutoff,
                                         offset);
      }
    }
  }
  return 0;
}

// Source-body _Uind!: src/FLOWPanel_nonliftingbody.jl:188-218.
void fpo_uind_source(const double* nodes, const int* offsets, const int* pnodes,
                     long long npanels, const double* strength, double offset,
                     const double* targets, long long nt, double* out, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const long long CH = 64;
#pragma omp parallel for schedule(dynamic)
  for (long long t0 = 0; t0 < nt; t0 += CH) {
    long long n = (nt - t0 < CH) ? nt - t0 : CH;
    for (long long i = 0; i < npanels; ++i) {
      const int* panel = pnodes + offsets[i];
      int nn = offsets[i + 1] - offsets[i];
      U_constant_source<double>(nodes, panel, nn, strength[i], targets + 3 * t0, n,
                                out + 3 * t0, nullptr, offset);
    }
  }
}

// ------------------------------------------------------------------ operation counts
// Per-interaction operation counts of the reference formulas (sqrt, log, atan2,
// abs and division counted as one operation each), measured by running the
// restatement on an operation-counting scalar. which: 0 filament, 1 ring of nn
// edges, 2 semi-infinite vortex, 3 horseshoe, 4 constant source of nn edges
// (dot_with form, panel-frame set-up excluded).
long long fpo_opcount(int which, int nn) {
  typedef OpCount C;
  double nodes_d[12] = {0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0};
  std::vector<C> nodes = cast_vec<C>(nodes_d, 12);
  int panel[4] = {0, 1, 2, 3};
  C X[3] = {C(0.3), C(0.4), C(0.5)};
  C D[3] = {C(0.0), C(0.0), C(1.0)};
  C out(0.0);
  C d[3] = {C(1.0), C(0.0), C(0.0)};
  long long base;
  switch (which) {
    case 0:
      OpCount::n() = 0;
      U_boundvortex_one<C>(nodes[0], nodes[1], nodes[2], nodes[3], nodes[4], nodes[5], C(1.0),
                           X, nullptr, &out, D, 1e-14, 1e-8);
      return OpCount::n();
    case 1:
      OpCount::n() = 0;
      U_vortexring<C>(nodes.data(), panel, nn, C(1.0), X, 1, &out, D, 1e-14, 1e-8);
      return OpCount::n();
    case 2:
      OpCount::n() = 0;
      U_semiinfinite_vortex_one<C>(nodes[0], nodes[1], nodes[2], d[0], d[1], d[2], C(1.0), X,
                                   nullptr, &out, D, 1e-14, 1e-8);
      return OpCount::n();
    case 3:
      OpCount::n() = 0;
      U_semiinfinite_horseshoe_one<C>(nodes.data(), 0, 1, d[0], d[1], d[2], d[0], d[1], d[2],
                                      C(1.0), X, nullptr, &out, D, 1e-14, 1e-8);
      return OpCount::n();
    case 4: {
      // total minus the per-panel frame set-up (measured with zero targets)
      OpCount::n() = 0;
      U_constant_source<C>(nodes.data(), panel, nn, C(1.0), X, 0, &out, D, 1e-8);
      base = OpCount::n();
      OpCount::n() = 0;
      U_constant_source<C>(nodes.data(), panel, nn, C(1.0), X, 1, &out, D, 1e-8);
      return OpCount::n() - base;
    }
  }
  return -1;
}

// ------------------------------------------------------------------ forward-mode derivatives
// Directional derivatives with Dual<1> (the stand-in for ForwardDiff through
// the reference's CPU path), the oracle of the reverse-mode kernels.
namespace {
typedef Dual<1> D1;
std::vector<D1> seed(const double* v, const double* dv, int64_t n) {
  std::vector<D1> r(n);
  for (int64_t i = 0; i < n; ++i) {
    r[i] = D1(v[i]);
    r[i].d[0] = dv ? dv[i] : 0.0;
  }
  return r;
}
// out[3t..] (or out[t] with normals) += velocity of the rings (strengths s)
// and of the wake horseshoes (s_pi, s_pj) at targets t0..t0+nt-1, in the
// reference's per-target order (src/FLOWPanel_liftingbody.jl:576-661).
void body_velocity(const std::vector<D1>& N, const int* offsets, const int* pnodes,
                   long long npanels, const std::vector<D1>& s, const int* shedding,
                   long long nsh, const std::vector<D1>& Da, const std::vector<D1>& Db,
                   const D1* T, long long nt, D1* out, const D1* normals, double cutoff,
                   double offset) {
  for (long long j = 0; j < npanels; ++j) {
    const int* panel = pnodes + offsets[j];
    const int nn = offsets[j + 1] - offsets[j];
    U_vortexring<D1>(N.data(), panel, nn, s[j], T, nt, out, normals, cutoff, offset);
  }
  for (long long e = 0; e < nsh; ++e) {
    const int* sh = shedding + 6 * e;
    const int pi = sh[0], nia = sh[1], nib = sh[2], pj = sh[3], nja = sh[4], njb = sh[5];
    const int* pan = pnodes + offsets[pi];
    const D1* da = Da.data() + 3 * e;
    const D1* db = Db.data() + 3 * e;
    U_semiinfinite_horseshoe<D1>(N.data(), pan[nia], pan[nib], da[0], da[1], da[2], db[0], db[1],
                                 db[2], s[pi], T, nt, out, normals, cutoff, offset);
    if (pj != -1) {
      const int* panj = pnodes + offsets[pj];
      U_semiinfinite_horseshoe<D1>(N.data(), panj[nja], panj[njb], db[0], db[1], db[2], da[0],
                                   da[1], da[2], s[pj], T, nt, out, normals, cutoff, offset);
    }
  }
}
}  // namespace

// F = sum_i lambda_i (b_i - (A gamma)_i), b_i = -Uinf_i . n_i, A the vortex-ring
// AIC with Kutta wake columns (src/FLOWPanel_liftingbody.jl:455-572,
// src/FLOWPanel_linearsolver.jl:297-312); F and its derivative along the
// given directions (any direction pointer may be NULL = 0); optionally the
// residual vector r = b - A gamma and its derivative dr (lambda may be NULL).
void fpo_residual_jvp(const double* nodes, const double* dnodes, long long nnodes,
                      const int* offsets, const int* pnodes, long long npanels, const double* cps,
                      const double* dcps, const double* normals, const double* dnormals,
                      const int* shedding, long long nsh, const double* Das, const double* dDas,
                      const double* Dbs, const double* dDbs, const double* Uinfs,
                      const double* dUinfs, const double* lambda, const double* gamma,
                      double offset, double cutoff, double* F, double* dF, double* r,
                      double* dr, int nthreads) {
  const std::vector<D1> N = seed(nodes, dnodes, 3 * nnodes);
  const std::vector<D1> X = seed(cps, dcps, 3 * npanels);
  const std::vector<D1> Nr = seed(normals, dnormals, 3 * npanels);
  const std::vector<D1> Da = seed(Das, dDas, 3 * nsh), Db = seed(Dbs, dDbs, 3 * nsh);
  const std::vector<D1> U = seed(Uinfs, dUinfs, 3 * npanels);
  const std::vector<D1> s = seed(gamma, nullptr, npanels);
  std::vector<D1> AG(npanels, D1(0.0));
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const long long CH = 16;
#pragma omp parallel for schedule(dynamic)
  for (long long t0 = 0; t0 < npanels; t0 += CH) {
    const long long nt = (npanels - t0 < CH) ? npanels - t0 : CH;
    body_velocity(N, offsets, pnodes, npanels, s, shedding, nsh, Da, Db, X.data() + 3 * t0, nt,
                  AG.data() + t0, Nr.data() + 3 * t0, cutoff, offset);
  }
  D1 acc(0.0);
  for (long long i = 0; i < npanels; ++i) {
    const D1 b = -(U[3 * i] * Nr[3 * i] + U[3 * i + 1] * Nr[3 * i + 1] + U[3 * i + 2] * Nr[3 * i + 2]);
    const D1 ri = b - AG[i];
    if (r) r[i] = ri.v;
    if (dr) dr[i] = ri.d[0];
    if (lambda) acc += D1(lambda[i]) * ri;
  }
  *F = acc.v;
  *dF = acc.d[0];
}

// F = sum_i wbar_i . Uind(targets_i) of the vortex-ring body with strengths;
// F and its derivative along (dnodes, dtargets, dstrengths, dDas, dDbs);
// optionally the velocities U (3 x m) and their derivatives dU (wbar may be NULL).
void fpo_uind_jvp(const double* nodes, const double* dnodes, long long nnodes, const int* offsets,
                  const int* pnodes, long long npanels, const double* strengths,
                  const double* dstrengths, const int* shedding, long long nsh, const double* Das,
                  const double* dDas, const double* Dbs, const double* dDbs,
                  const double* targets, const double* dtargets, long long m, const double* wbar,
                  double offset, double cutoff, double* F, double* dF, double* U, double* dU,
                  int nthreads) {
  const std::vector<D1> N = seed(nodes, dnodes, 3 * nnodes);
  const std::vector<D1> X = seed(targets, dtargets, 3 * m);
  const std::vector<D1> Da = seed(Das, dDas, 3 * nsh), Db = seed(Dbs, dDbs, 3 * nsh);
  const std::vector<D1> s = seed(strengths, dstrengths, npanels);
  std::vector<D1> Uo(3 * m, D1(0.0));
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const long long CH = 16;
#pragma omp parallel for schedule(dynamic)
  for (long long t0 = 0; t0 < m; t0 += CH) {
    const long long nt = (m - t0 < CH) ? m - t0 : CH;
    body_velocity(N, offsets, pnodes, npanels, s, shedding, nsh, Da, Db, X.data() + 3 * t0, nt,
                  Uo.data() + 3 * t0, nullptr, cutoff, offset);
  }
  D1 acc(0.0);
  for (long long i = 0; i < 3 * m; ++i) {
    if (U) U[i] = Uo[i].v;
    if (dU) dU[i] = Uo[i].d[0];
    if (wbar) acc += D1(wbar[i]) * Uo[i];
  }
  *F = acc.v;
  *dF = acc.d[0];
}

}  // extern "C"
