// Dense AIC and RHS assembly on sm_100a.
//
// G[i, j] = unit-strength normal velocity of panel j at control point i,
// column-major with leading dimension ld (HBM layout: FP64 G for residuals,
// optional FP32 copy for the factorisation, written by the same pass).
//
// Roofline: compute-bound on the FP64 pipe (plus the MUFU-seeded sqrt and
// reciprocal sequences); the G write is 8 B per entry against ~250 FP64
// operations per entry.
#include "fp_internal.cuh"

namespace fpb {

constexpr int kAsmThreads = 128;   // targets per CTA (one per thread)
constexpr int kAsmPanels = 32;     // panels per CTA (smem tile)

// HOT LOOP 1 of _G_Uvortexring! (src/FLOWPanel_liftingbody.jl:476-503): every
// (control point, panel) pair. Targets on threads (coalesced column writes),
// panel records staged in shared memory and broadcast to the CTA.
template <bool W32>
__global__ void __launch_bounds__(kAsmThreads)
k_asm_ring(const PanelRec* __restrict__ panels, int64_t n, const double* __restrict__ tgt,
           int64_t ld, double offset, double cutoff2, double offset2, double* __restrict__ G,
           float* __restrict__ G32) {
  __shared__ PanelRec sp[kAsmPanels];
  __shared__ int quads;   // every panel of the tile has 4 nodes
  const int64_t j0 = (int64_t)blockIdx.y * kAsmPanels;
  const int npt = (int)imin64(kAsmPanels, n - j0);
  {
    const double* src = reinterpret_cast<const double*>(panels + j0);
    double* dst = reinterpret_cast<double*>(sp);
    for (int q = threadIdx.x; q < npt * 16; q += kAsmThreads) dst[q] = src[q];
  }
  if (threadIdx.x < 32) {
    const bool q4 = threadIdx.x >= npt || (int)panels[j0 + threadIdx.x].nn == 4;
    const unsigned all = __all_sync(0xffffffffu, q4);
    if (threadIdx.x == 0) quads = (int)all;
  }
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * kAsmThreads + threadIdx.x;
  if (i >= n) return;
  const double X = tgt[i], Y = tgt[n + i], Z = tgt[2 * n + i];
  const double n1 = tgt[3 * n + i], n2 = tgt[4 * n + i], n3 = tgt[5 * n + i];
  if (quads) {
    // two panels a step, no per-panel branch on the node count: the two
    // entries' sqrt / reciprocal chains are independent and interleave
    int jj = 0;
    for (; jj + 1 < npt; jj += 2) {
      const double g0 = ring_dot_n<double, 4>(sp[jj].p, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2);
      const double g1 = ring_dot_n<double, 4>(sp[jj + 1].p, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2);
      const int64_t idx = (j0 + jj) * ld + i;
      G[idx] = g0;
      G[idx + ld] = g1;
      if (W32) {
        G32[idx] = (float)g0;
        G32[idx + ld] = (float)g1;
      }
    }
    if (jj < npt) {
      const double g = ring_dot_n<double, 4>(sp[jj].p, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2);
      const int64_t idx = (j0 + jj) * ld + i;
      G[idx] = g;
      if (W32) G32[idx] = (float)g;
    }
    return;
  }
  for (int jj = 0; jj < npt; ++jj) {
    const PanelRec& P = sp[jj];
    const double g = ring_dot<double>(P.p, (int)P.nn, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2);
    const int64_t idx = (j0 + jj) * ld + i;
    G[idx] = g;
    if (W32) G32[idx] = (float)g;
  }
}

// HOT LOOP 2 (src/FLOWPanel_liftingbody.jl:508-567): Kutta wake columns. For
// shedding edge e, the upper panel pi gets the horseshoe (da, db) and the
// lower panel pj the horseshoe over its own TE nodes with (db, da) swapped,
// both added on top of the ring part already in the column. With disjoint
// columns every (target, edge) pair runs in parallel; otherwise one thread
// per target walks the edges in order.
template <bool W32>
__global__ void __launch_bounds__(kAsmThreads)
k_asm_wake(const WakeRec* __restrict__ wake, int64_t nsh, int64_t n, const double* __restrict__ tgt,
           int64_t ld, double offset, double cutoff2, double offset2, double* __restrict__ G,
           float* __restrict__ G32, bool serial) {
  const int64_t i = (int64_t)blockIdx.x * kAsmThreads + threadIdx.x;
  if (i >= n) return;
  const double X = tgt[i], Y = tgt[n + i], Z = tgt[2 * n + i];
  const double n1 = tgt[3 * n + i], n2 = tgt[4 * n + i], n3 = tgt[5 * n + i];
  const int64_t e0 = serial ? 0 : blockIdx.y;
  const int64_t e1 = serial ? nsh : blockIdx.y + 1;
  for (int64_t e = e0; e < e1; ++e) {
    const WakeRec& w = wake[e];
    {
      const int64_t idx = (int64_t)w.pi * ld + i;
      double acc = G[idx];
      horseshoe_dot<double>(w.pa, w.pb, w.da, w.db, 1.0, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2, acc);
      G[idx] = acc;
      if (W32) G32[idx] = (float)acc;
    }
    if (w.pj >= 0) {
      const int64_t idx = (int64_t)w.pj * ld + i;
      double acc = G[idx];
      horseshoe_dot<double>(w.qa, w.qb, w.db, w.da, 1.0, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2, acc);
      G[idx] = acc;
      if (W32) G32[idx] = (float)acc;
    }
  }
}

// Constant-source columns (src/FLOWPanel_nonliftingbody.jl:169-185): with
// dot_with the three components are added one by one (:127-130).
template <bool W32>
__global__ void __launch_bounds__(kAsmThreads)
k_asm_source(const SourceRec* __restrict__ recs, int64_t n, const double* __restrict__ tgt,
             int64_t ld, double offset, double* __restrict__ G, float* __restrict__ G32) {
  __shared__ SourceRec sr[kAsmPanels];
  const int64_t j0 = (int64_t)blockIdx.y * kAsmPanels;
  const int npt = (int)imin64(kAsmPanels, n - j0);
  {
    const int words = sizeof(SourceRec) / 4;
    const int* src = reinterpret_cast<const int*>(recs + j0);
    int* dst = reinterpret_cast<int*>(sr);
    for (int q = threadIdx.x; q < npt * words; q += kAsmThreads) dst[q] = src[q];
  }
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * kAsmThreads + threadIdx.x;
  if (i >= n) return;
  const double X = tgt[i], Y = tgt[n + i], Z = tgt[2 * n + i];
  const double n1 = tgt[3 * n + i], n2 = tgt[4 * n + i], n3 = tgt[5 * n + i];
  for (int jj = 0; jj < npt; ++jj) {
    double u, v, w;
    source_vel(sr[jj], X, Y, Z, offset, u, v, w);
    double g = 0.0;
    g += u * n1;
    g += v * n2;
    g += w * n3;
    const int64_t idx = (j0 + jj) * ld + i;
    G[idx] = g;
    if (W32) G32[idx] = (float)g;
  }
}

// The FP32 AIC alone, for the FP32 factorisation of the mixed forms: each
// panel in coordinates local to its vertex mean (FP64 differences rounded
// once to FP32), so that near and far entries keep FP32 relative accuracy
// (no large absolute coordinates cancel in FP32); the same ring formula in
// FP32. The FP64 AIC of the refinement residuals is written by k_asm_ring
// on a background stream meanwhile.
struct PanelLocal {
  double c[3];
  float p[12];
  int nn, pad;
};

__global__ void __launch_bounds__(kAsmThreads)
k_asm_ring32(const PanelRec* __restrict__ panels, int64_t n, const double* __restrict__ tgt, int64_t ld,
             float offset, float cutoff2, float offset2, float* __restrict__ G32) {
  __shared__ PanelLocal sp[kAsmPanels];
  const int64_t j0 = (int64_t)blockIdx.y * kAsmPanels;
  const int npt = (int)imin64(kAsmPanels, n - j0);
  if (threadIdx.x < npt) {
    const PanelRec& P = panels[j0 + threadIdx.x];
    const int nn = (int)P.nn;
    double c0 = 0.0, c1 = 0.0, c2 = 0.0;
    for (int k = 0; k < nn; ++k) { c0 += P.p[3 * k]; c1 += P.p[3 * k + 1]; c2 += P.p[3 * k + 2]; }
    c0 /= nn; c1 /= nn; c2 /= nn;
    PanelLocal& L = sp[threadIdx.x];
    L.c[0] = c0; L.c[1] = c1; L.c[2] = c2;
    for (int k = 0; k < 4; ++k) {
      const bool in = k < nn;
      L.p[3 * k] = in ? (float)(P.p[3 * k] - c0) : 0.f;
      L.p[3 * k + 1] = in ? (float)(P.p[3 * k + 1] - c1) : 0.f;
      L.p[3 * k + 2] = in ? (float)(P.p[3 * k + 2] - c2) : 0.f;
    }
    L.nn = nn;
  }
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * kAsmThreads + threadIdx.x;
  if (i >= n) return;
  const double X = tgt[i], Y = tgt[n + i], Z = tgt[2 * n + i];
  const float n1 = (float)tgt[3 * n + i], n2 = (float)tgt[4 * n + i], n3 = (float)tgt[5 * n + i];
  for (int jj = 0; jj < npt; ++jj) {
    const PanelLocal& P = sp[jj];
    const float x = (float)(X - P.c[0]), y = (float)(Y - P.c[1]), z = (float)(Z - P.c[2]);
    G32[(j0 + jj) * ld + i] = ring_dot<float>(P.p, P.nn, x, y, z, n1, n2, n3, offset, cutoff2, offset2);
  }
}

// The Kutta wake columns of the FP32 AIC: the horseshoes in FP64 (2 nsh
// columns), added to the ring part in G32 (the same row walk as k_asm_wake).
__global__ void __launch_bounds__(kAsmThreads)
k_asm_wake32(const WakeRec* __restrict__ wake, int64_t nsh, int64_t n, const double* __restrict__ tgt,
             int64_t ld, double offset, double cutoff2, double offset2, float* __restrict__ G32, bool serial) {
  const int64_t i = (int64_t)blockIdx.x * kAsmThreads + threadIdx.x;
  if (i >= n) return;
  const double X = tgt[i], Y = tgt[n + i], Z = tgt[2 * n + i];
  const double n1 = tgt[3 * n + i], n2 = tgt[4 * n + i], n3 = tgt[5 * n + i];
  const int64_t e0 = serial ? 0 : blockIdx.y;
  const int64_t e1 = serial ? nsh : blockIdx.y + 1;
  for (int64_t e = e0; e < e1; ++e) {
    const WakeRec& w = wake[e];
    {
      const int64_t idx = (int64_t)w.pi * ld + i;
      double acc = G32[idx];
      horseshoe_dot<double>(w.pa, w.pb, w.da, w.db, 1.0, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2, acc);
      G32[idx] = (float)acc;
    }
    if (w.pj >= 0) {
      const int64_t idx = (int64_t)w.pj * ld + i;
      double acc = G32[idx];
      horseshoe_dot<double>(w.qa, w.qb, w.db, w.da, 1.0, X, Y, Z, n1, n2, n3, offset, cutoff2, offset2, acc);
      G32[idx] = (float)acc;
    }
  }
}

int launch_assemble_ring32(fp_ctx* c, double offset, double cutoff) {
  const int64_t n = c->N;
  dim3 grid((unsigned)((n + kAsmThreads - 1) / kAsmThreads), (unsigned)((n + kAsmPanels - 1) / kAsmPanels));
  const double cut2 = cutoff * cutoff, off2 = offset * offset;
  k_asm_ring32<<<grid, kAsmThreads, 0, c->stream>>>(c->d_panels, n, c->d_tgt, c->ld, (float)offset, (float)cut2,
                                                     (float)off2, c->d_G32);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  if (c->nsh > 0) {
    const bool serial = !c->wake_disjoint;
    dim3 g2((unsigned)((n + kAsmThreads - 1) / kAsmThreads), serial ? 1u : (unsigned)c->nsh);
    k_asm_wake32<<<g2, kAsmThreads, 0, c->stream>>>(c->d_wake, c->nsh, n, c->d_tgt, c->ld, offset, cut2, off2,
                                                     c->d_G32, serial);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
  }
  return FP_OK;
}

// RHS_i = -U_i . n_i (src/FLOWPanel_linearsolver.jl:297-312), k right-hand sides.
__global__ void k_rhs(const double* __restrict__ U, int64_t n, int64_t k,
                      const double* __restrict__ tgt, double* __restrict__ rhs, int64_t ld) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * k) return;
  const int64_t i = t % n, q = t / n;
  const double* u = U + 3 * (q * n + i);
  const double d = u[0] * tgt[3 * n + i] + u[1] * tgt[4 * n + i] + u[2] * tgt[5 * n + i];
  rhs[q * ld + i] = -d;
}

int launch_assemble_ring(fp_ctx* c, double offset, double cutoff, bool write32, cudaStream_t s) {
  const int64_t n = c->N;
  cudaStream_t st = s ? s : c->stream;
  dim3 grid((unsigned)((n + kAsmThreads - 1) / kAsmThreads), (unsigned)((n + kAsmPanels - 1) / kAsmPanels));
  const double cut2 = cutoff * cutoff, off2 = offset * offset;
  if (write32)
    k_asm_ring<true><<<grid, kAsmThreads, 0, st>>>(c->d_panels, n, c->d_tgt, c->ld, offset, cut2, off2, c->d_G, c->d_G32);
  else
    k_asm_ring<false><<<grid, kAsmThreads, 0, st>>>(c->d_panels, n, c->d_tgt, c->ld, offset, cut2, off2, c->d_G, nullptr);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  if (c->nsh > 0) {
    const bool serial = !c->wake_disjoint;
    dim3 g2((unsigned)((n + kAsmThreads - 1) / kAsmThreads), serial ? 1u : (unsigned)c->nsh);
    if (write32)
      k_asm_wake<true><<<g2, kAsmThreads, 0, st>>>(c->d_wake, c->nsh, n, c->d_tgt, c->ld, offset, cut2, off2, c->d_G, c->d_G32, serial);
    else
      k_asm_wake<false><<<g2, kAsmThreads, 0, st>>>(c->d_wake, c->nsh, n, c->d_tgt, c->ld, offset, cut2, off2, c->d_G, nullptr, serial);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
  }
  return FP_OK;
}

int launch_assemble_source(fp_ctx* c, double offset, bool write32) {
  const int64_t n = c->N;
  dim3 grid((unsigned)((n + kAsmThreads - 1) / kAsmThreads), (unsigned)((n + kAsmPanels - 1) / kAsmPanels));
  if (write32)
    k_asm_source<true><<<grid, kAsmThreads, 0, c->stream>>>(c->d_src, n, c->d_tgt, c->ld, offset, c->d_G, c->d_G32);
  else
    k_asm_source<false><<<grid, kAsmThreads, 0, c->stream>>>(c->d_src, n, c->d_tgt, c->ld, offset, c->d_G, nullptr);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

int launch_rhs(fp_ctx* c, const double* d_U, int64_t k) {
  const int64_t tot = c->N * k;
  k_rhs<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(d_U, c->N, k, c->d_tgt, c->d_rhs, c->ld);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

}  // namespace fpb
