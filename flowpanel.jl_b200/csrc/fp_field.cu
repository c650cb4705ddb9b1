// Induced velocity (Uind!) and potential (phi!) of a solved body at arbitrary
// targets. The velocity sums vortex rings with their strengths plus the wake
// horseshoes with (Gamma_pi, Gamma_pj) (src/FLOWPanel_liftingbody.jl:576-661),
// or constant sources (src/FLOWPanel_nonliftingbody.jl:188-218); the
// potential is k_phi below.
//
// One thread per target, panels staged through shared memory; each target
// adds the panels in the reference's order (panels, then shedding edges) on
// top of the value already in out. Compute-bound (FP64 or FP32 pipe). The
// FP32 form serves off-body probes: its error grows near the panels, where
// single-precision positions carry a larger share of the distances. With
// few targets (the body's own control points) the panels are split in
// gridDim.y chunks so that the grid fills the device: each chunk writes its
// partial sum, the last chunk also the shedding edges, and k_uind_reduce adds
// them to out in chunk order.
#include "fp_internal.cuh"

namespace fpb {

constexpr int kFieldThreads = 128;
constexpr int kFieldTile = 64;

template <class T>
__global__ void __launch_bounds__(kFieldThreads)
k_uind_ring(const PanelRec* __restrict__ panels, const double* __restrict__ strength, int64_t n,
            const WakeRec* __restrict__ wake, int64_t nsh, const double* __restrict__ targets,
            int64_t m, double* __restrict__ out, double offset, double cutoff2, double offset2,
            double* __restrict__ partial) {
  __shared__ T sp[kFieldTile][14];   // 12 coordinates, strength, node count
  const int64_t t = (int64_t)blockIdx.x * kFieldThreads + threadIdx.x;
  const bool live = t < m;
  const int64_t per = (n + gridDim.y - 1) / gridDim.y;
  const int64_t jb = imin64(n, (int64_t)blockIdx.y * per), je = imin64(n, jb + per);
  const bool last = blockIdx.y == gridDim.y - 1;
  const T X = live ? (T)targets[3 * t] : T(0);
  const T Y = live ? (T)targets[3 * t + 1] : T(0);
  const T Z = live ? (T)targets[3 * t + 2] : T(0);
  T u = live && !partial ? (T)out[3 * t] : T(0);
  T v = live && !partial ? (T)out[3 * t + 1] : T(0);
  T w = live && !partial ? (T)out[3 * t + 2] : T(0);
  const T off = (T)offset, c2 = (T)cutoff2, o2 = (T)offset2;
  for (int64_t j0 = jb; j0 < je; j0 += kFieldTile) {
    const int nt = (int)imin64(kFieldTile, je - j0);
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
  for (int64_t e = 0; last && e < nsh; ++e) {
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
  double* dst = partial ? partial + 3 * ((int64_t)blockIdx.y * m + t) : out + 3 * t;
  dst[0] = (double)u;
  dst[1] = (double)v;
  dst[2] = (double)w;
}

__global__ void __launch_bounds__(kFieldThreads)
k_uind_source(const SourceRec* __restrict__ recs, const double* __restrict__ strength, int64_t n,
              const double* __restrict__ targets, int64_t m, double* __restrict__ out,
              double offset, double* __restrict__ partial) {
  const int64_t t = (int64_t)blockIdx.x * kFieldThreads + threadIdx.x;
  if (t >= m) return;
  const int64_t per = (n + gridDim.y - 1) / gridDim.y;
  const int64_t jb = imin64(n, (int64_t)blockIdx.y * per), je = imin64(n, jb + per);
  const double X = targets[3 * t], Y = targets[3 * t + 1], Z = targets[3 * t + 2];
  double a = partial ? 0.0 : out[3 * t], b = partial ? 0.0 : out[3 * t + 1], c = partial ? 0.0 : out[3 * t + 2];
  for (int64_t j = jb; j < je; ++j) {
    double u, v, w;
    source_vel(recs[j], X, Y, Z, offset, u, v, w);
    const double s = strength[j];
    a += s * u;
    b += s * v;
    c += s * w;
  }
  double* dst = partial ? partial + 3 * ((int64_t)blockIdx.y * m + t) : out + 3 * t;
  dst[0] = a;
  dst[1] = b;
  dst[2] = c;
}

// out += the chunks' partial sums, in chunk order
__global__ void __launch_bounds__(256)
k_uind_reduce(const double* __restrict__ partial, int nchunk, int64_t m, double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (i >= 3 * m) return;
  double s = out[i];
  for (int k = 0; k < nchunk; ++k) s += partial[(int64_t)k * 3 * m + i];
  out[i] = s;
}

// Panel chunks for m targets: enough blocks for four per SM, chunks of at
// least 512 panels, at most 16.
int uind_chunks(int64_t m, int64_t n) {
  const int64_t blocks = (m + kFieldThreads - 1) / kFieldThreads;
  const int64_t want = 4 * (int64_t)num_sms();
  if (blocks >= want) return 1;
  int64_t s = (want + blocks - 1) / blocks;
  s = imin64(s, imin64(16, n / 512));
  return (int)std::max<int64_t>(s, 1);
}

int ensure_uind_scratch(fp_ctx* c, size_t n) {
  if (n <= c->cap_uscr) return FP_OK;
  if (c->d_uscr) cudaFree(c->d_uscr);
  c->d_uscr = nullptr;
  c->cap_uscr = 0;
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_uscr, n * sizeof(double)));
  c->cap_uscr = n;
  return FP_OK;
}

int reduce_chunks(fp_ctx* c, int nchunk, int64_t m, double* d_out) {
  k_uind_reduce<<<(unsigned)((3 * m + 255) / 256), 256, 0, c->stream>>>(c->d_uscr, nchunk, m, d_out);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
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
  const int nchunk = uind_chunks(m, c->N);
  if (nchunk > 1 && ensure_uind_scratch(c, (size_t)nchunk * 3 * m)) return FP_ECUDA;
  double* part = nchunk > 1 ? c->d_uscr : nullptr;
  const dim3 g((unsigned)((m + kFieldThreads - 1) / kFieldThreads), nchunk);
  const double off = c->kern_offset, cut2 = c->kern_cutoff * c->kern_cutoff, off2 = off * off;
  if (fp32)
    k_uind_ring<float><<<g, kFieldThreads, 0, c->stream>>>(c->d_panels, d_strength, c->N, c->d_wake, c->nsh,
                                                           d_targets, m, d_out, off, cut2, off2, part);
  else
    k_uind_ring<double><<<g, kFieldThreads, 0, c->stream>>>(c->d_panels, d_strength, c->N, c->d_wake, c->nsh,
                                                            d_targets, m, d_out, off, cut2, off2, part);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return nchunk > 1 ? reduce_chunks(c, nchunk, m, d_out) : FP_OK;
}

int launch_uind_source(fp_ctx* c, const double* d_strength, const double* d_targets, int64_t m,
                       double* d_out) {
  const int nchunk = uind_chunks(m, c->N);
  if (nchunk > 1 && ensure_uind_scratch(c, (size_t)nchunk * 3 * m)) return FP_ECUDA;
  double* part = nchunk > 1 ? c->d_uscr : nullptr;
  const dim3 g((unsigned)((m + kFieldThreads - 1) / kFieldThreads), nchunk);
  k_uind_source<<<g, kFieldThreads, 0, c->stream>>>(c->d_src, d_strength, c->N, d_targets, m, d_out, c->kern_offset,
                                                    part);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return nchunk > 1 ? reduce_chunks(c, nchunk, m, d_out) : FP_OK;
}

}  // namespace fpb
