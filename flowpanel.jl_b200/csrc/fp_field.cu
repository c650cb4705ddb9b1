// Induced velocity (Uind!) and potential (phi!) of a solved body at arbitrary
// targets. The velocity sums vortex rings with their strengths plus the wake
// horseshoes with (Gamma_pi, Gamma_pj) (src/FLOWPanel_liftingbody.jl:576-661),
// or constant sources (src/FLOWPanel_nonliftingbody.jl:188-218); the
// potential is k_phi below.
//
// One thread per target, panels staged through shared memory; each target
// adds the panels in the reference's order (panels, then shedding edges) on
// top of the value already in out. Compute-bound (FP64 or FP32 pipe).
#include "fp_internal.cuh"

namespace fpb {

constexpr int kFieldThreads = 128;
constexpr int kFieldTile = 64;

template <class T>
__global__ void __launch_bounds__(kFieldThreads)
k_uind_ring(const PanelRec* __restrict__ panels, const double* __restrict__ strength, int64_t n,
            const WakeRec* __restrict__ wake, int64_t nsh, const double* __restrict__ targets,
            int64_t m, double* __restrict__ out, double offset, double cutoff2, double offset2) {
  __shared__ T sp[kFieldTile][14];   // 12 coordinates, strength, node count
  const int64_t t = (int64_t)blockIdx.x * kFieldThreads + threadIdx.x;
  const bool live = t < m;
  const T X = live ? (T)targets[3 * t] : T(0);
  const T Y = live ? (T)targets[3 * t + 1] : T(0);
  const T Z = live ? (T)targets[3 * t + 2] : T(0);
  T u = live ? (T)out[3 * t] : T(0);
  T v = live ? (T)out[3 * t + 1] : T(0);
  T w = live ? (T)out[3 * t + 2] : T(0);
  const T off = (T)offset, c2 = (T)cutoff2, o2 = (T)offset2;
  for (int64_t j0 = 0; j0 < n; j0 += kFieldTile) {
    const int nt = (int)imin64(kFieldTile, n - j0);
    __syncthreads();
    for (int q = threadIdx.x; q < nt * 14; q += kFieldThreads) {
      const int jj = q / 14, e = q % 14;
      const PanelRec& P = panels[j0 + jj];
      double val;
      if (e < 12) val = P.p[e];
      else if (e == 12) val = strength[j0 + jj];
      else val = P.nn;
      sp[jj][e] = (T)val;
    }
    __syncthreads();
    if (live) {
      for (int jj = 0; jj < nt; ++jj)
        ring_vel<T>(sp[jj], (int)sp[jj][13], sp[jj][12], X, Y, Z, off, c2, o2, u, v, w);
    }
  }
  if (!live) return;
  for (int64_t e = 0; e < nsh; ++e) {
    const WakeRec& wr = wake[e];
    const T si = (T)strength[wr.pi];
    T pa[3] = {(T)wr.pa[0], (T)wr.pa[1], (T)wr.pa[2]};
    T pb[3] = {(T)wr.pb[0], (T)wr.pb[1], (T)wr.pb[2]};
    T da[3] = {(T)wr.da[0], (T)wr.da[1], (T)wr.da[2]};
    T db[3] = {(T)wr.db[0], (T)wr.db[1], (T)wr.db[2]};
    horseshoe<T>(pa, pb, da, db, si, X, Y, Z, off, c2, o2, u, v, w);
    if (wr.pj >= 0) {
      const T sj = (T)strength[wr.pj];
      T qa[3] = {(T)wr.qa[0], (T)wr.qa[1], (T)wr.qa[2]};
      T qb[3] = {(T)wr.qb[0], (T)wr.qb[1], (T)wr.qb[2]};
      horseshoe<T>(qa, qb, db, da, sj, X, Y, Z, off, c2, o2, u, v, w);
    }
  }
  out[3 * t] = (double)u;
  out[3 * t + 1] = (double)v;
  out[3 * t + 2] = (double)w;
}

__global__ void __launch_bounds__(kFieldThreads)
k_uind_source(const SourceRec* __restrict__ recs, const double* __restrict__ strength, int64_t n,
              const double* __restrict__ targets, int64_t m, double* __restrict__ out,
              double offset) {
  const int64_t t = (int64_t)blockIdx.x * kFieldThreads + threadIdx.x;
  if (t >= m) return;
  const double X = targets[3 * t], Y = targets[3 * t + 1], Z = targets[3 * t + 2];
  double a = out[3 * t], b = out[3 * t + 1], c = out[3 * t + 2];
  for (int64_t j = 0; j < n; ++j) {
    double u, v, w;
    source_vel(recs[j], X, Y, Z, offset, u, v, w);
    const double s = strength[j];
    a += s * u;
    b += s * v;
    c += s * w;
  }
  out[3 * t] = a;
  out[3 * t + 1] = b;
  out[3 * t + 2] = c;
}

// Potential phi! of a solved body (one thread per target, FP64): for each
// panel in order, its source and/or doublet potential scaled by its
// strengths (sigma, mu), then, for a lifting body, each shedding edge's
// semi-infinite doublets, (da, db) from the upper panel's TE nodes with mu_pi
// and (db, da) from the lower's with mu_pj (src/FLOWPanel_liftingbody.jl:664-742).
__global__ void __launch_bounds__(kFieldThreads)
k_phi(const SourceRec* __restrict__ recs, const double* __restrict__ sigma, const double* __restrict__ mu,
      int64_t n, const WakeRec* __restrict__ wake, int64_t nsh, const double* __restrict__ targets, int64_t m,
      double* __restrict__ out, double offset) {
  const int64_t t = (int64_t)blockIdx.x * kFieldThreads + threadIdx.x;
  if (t >= m) return;
  const double X = targets[3 * t], Y = targets[3 * t + 1], Z = targets[3 * t + 2];
  double phi = out[t];
  for (int64_t j = 0; j < n; ++j) {
    const SourceRec& R = recs[j];
    if (sigma) phi += sigma[j] * source_phi(R, X, Y, Z, offset);
    if (mu) phi += mu[j] * doublet_phi(R, X, Y, Z);
  }
  for (int64_t e = 0; mu && e < nsh; ++e) {
    const WakeRec& wr = wake[e];
    phi += mu[wr.pi] * semiinf_doublet_phi2(wr.pa, wr.pb, wr.da, wr.db, X, Y, Z, 1e12);
    if (wr.pj >= 0) phi += mu[wr.pj] * semiinf_doublet_phi2(wr.qa, wr.qb, wr.db, wr.da, X, Y, Z, 1e12);
  }
  out[t] = phi;
}

int launch_phi(fp_ctx* c, const double* d_sigma, const double* d_mu, const double* d_targets, int64_t m,
               double* d_out, bool wake) {
  const unsigned g = (unsigned)((m + kFieldThreads - 1) / kFieldThreads);
  k_phi<<<g, kFieldThreads, 0, c->stream>>>(c->d_src, d_sigma, d_mu, c->N, c->d_wake, wake ? c->nsh : 0, d_targets,
                                              m, d_out, c->kern_offset);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

int launch_uind_ring(fp_ctx* c, const double* d_strength, const double* d_targets, int64_t m,
                     double* d_out, bool fp32) {
  const unsigned g = (unsigned)((m + kFieldThreads - 1) / kFieldThreads);
  const double off = c->kern_offset, cut2 = c->kern_cutoff * c->kern_cutoff, off2 = off * off;
  if (fp32)
    k_uind_ring<float><<<g, kFieldThreads, 0, c->stream>>>(c->d_panels, d_strength, c->N, c->d_wake, c->nsh, d_targets, m, d_out, off, cut2, off2);
  else
    k_uind_ring<double><<<g, kFieldThreads, 0, c->stream>>>(c->d_panels, d_strength, c->N, c->d_wake, c->nsh, d_targets, m, d_out, off, cut2, off2);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

int launch_uind_source(fp_ctx* c, const double* d_strength, const double* d_targets, int64_t m,
                       double* d_out) {
  const unsigned g = (unsigned)((m + kFieldThreads - 1) / kFieldThreads);
  k_uind_source<<<g, kFieldThreads, 0, c->stream>>>(c->d_src, d_strength, c->N, d_targets, m, d_out, c->kern_offset);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

}  // namespace fpb
