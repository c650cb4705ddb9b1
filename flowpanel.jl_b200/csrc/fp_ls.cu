// Least-squares solve of watertight vortex-ring bodies
// (RigidWakeBody{VortexRing, 2} / MultiBody{VortexRing, 2},
// src/FLOWPanel_liftingbody.jl:236-447, src/FLOWPanel_multibody.jl:373-617):
// with the AIC G (wake columns included) and RHS = -Uinf . n,
//   r = RHS - sum_p val_p G[:, el_p]          (prescribed strengths moved right)
//   Gred = G without the prescribed columns
//   (Gred^T Gred) Gamma_red = Gred^T r         (normal equations, FP64)
// solved with the FP64 LU (solve_ludiv!, the reference's default solver), and
// Gamma scattered back around the prescribed values (set_solution).
//
// Gred is never formed: cmap[j] is the column of G behind column j of Gred.
// The Gram matrix is symmetric: k_gram_dmma (the FP64 tensor path) or k_gram
// (SIMT, FP_TUNE_FP64_DMMA 0) computes the tiles on and below the diagonal and
// writes each off-diagonal tile twice. FP64 throughout: the normal equations
// square the condition number, so they are formed in FP64 as the reference
// forms them on the CPU.
#include <algorithm>
#include <vector>

#include "fp_internal.cuh"

namespace fpb {

constexpr int kGramT = 64, kGramK = 32, kGramThreads = 256;

// Gls (nr x nr, leading dimension ldl) = Gred^T Gred over the m rows of G.
__global__ void __launch_bounds__(kGramThreads)
k_gram(const double* __restrict__ G, int64_t ldg, int64_t m, const int* __restrict__ cmap, int64_t nr,
       double* __restrict__ Gls, int64_t ldl) {
  __shared__ double As[kGramK][kGramT + 1], Bs[kGramK][kGramT + 1];
  __shared__ int ca[kGramT], cb[kGramT];
  // tile (bi, bj), bj <= bi, from the linear index t = bi (bi + 1) / 2 + bj
  const int64_t t = blockIdx.x;
  int64_t bi = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) / 2.0);
  while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while (bi * (bi + 1) / 2 > t) --bi;
  const int64_t bj = t - bi * (bi + 1) / 2;
  const int64_t r0 = bi * kGramT, c0 = bj * kGramT;
  const int tid = threadIdx.x, tr = tid & 15, tc = tid >> 4;   // rows 4 tr.., columns 4 tc..
  if (tid < kGramT) {
    ca[tid] = (r0 + tid < nr) ? cmap[r0 + tid] : -1;
    cb[tid] = (c0 + tid < nr) ? cmap[c0 + tid] : -1;
  }
  __syncthreads();
  double acc[4][4] = {};
  for (int64_t k0 = 0; k0 < m; k0 += kGramK) {
    for (int e = tid; e < kGramK * kGramT; e += kGramThreads) {
      const int kk = e % kGramK, j = e / kGramK;   // rows of G fastest: coalesced columns
      const int64_t row = k0 + kk;
      As[kk][j] = (row < m && ca[j] >= 0) ? G[(int64_t)ca[j] * ldg + row] : 0.0;
      Bs[kk][j] = (row < m && cb[j] >= 0) ? G[(int64_t)cb[j] * ldg + row] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kGramK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = As[kk][4 * tr + i];
        b[i] = Bs[kk][4 * tc + i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int l = 0; l < 4; ++l) acc[i][l] += a[i] * b[l];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const int64_t r = r0 + 4 * tr + i, c = c0 + 4 * tc + l;
      if (r < nr && c < nr) {
        Gls[c * ldl + r] = acc[i][l];
        if (bi != bj) Gls[r * ldl + c] = acc[i][l];
      }
    }
}

// The same Gram matrix on the FP64 tensor path (mma.sync m8n8k4 .f64):
// 128 x 128 tiles on and below the diagonal, 32 warps of 32 x 16, 32-deep K
// slices through a 3-stage cp.async ring. Both operands are columns of G
// (K-contiguous), staged [column][k] with 36-double rows (the fragment loads
// of 8 columns x 4 k cover the banks in two wavefronts). Fragments as in the
// LU's update (PTX ISA, mma m8n8k4 .f64): lane = 4 g + t; A(8x4) element
// (g, t); B(4x8) element (t, g); C(8x8) elements (g, 2t), (g, 2t+1).
namespace gd {
constexpr int T = 128, BK = 32, BP = BK + 4, STAGES = 3, NT = 1024, MF = 4, NF = 2;
__host__ __device__ constexpr size_t stage_doubles() { return 2 * (size_t)T * BP; }
constexpr size_t smem() { return STAGES * stage_doubles() * sizeof(double) + 2 * T * sizeof(int); }
}  // namespace gd

__device__ __forceinline__ void cp_async16_sz_ls(void* smem, const void* gmem, int bytes) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}

__global__ void __launch_bounds__(gd::NT, 1)
k_gram_dmma(const double* __restrict__ G, int64_t ldg, int64_t m, const int* __restrict__ cmap, int64_t nr,
            double* __restrict__ Gls, int64_t ldl) {
  using namespace gd;
  extern __shared__ __align__(16) unsigned char gsm[];
  double* const ring = reinterpret_cast<double*>(gsm);
  int* ca = reinterpret_cast<int*>(gsm + STAGES * stage_doubles() * sizeof(double));
  int* cb = ca + T;
  const int64_t t = blockIdx.x;   // tile (bi, bj), bj <= bi
  int64_t bi = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) / 2.0);
  while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while (bi * (bi + 1) / 2 > t) --bi;
  const int64_t bj = t - bi * (bi + 1) / 2;
  const int64_t r0 = bi * T, c0 = bj * T;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  constexpr int WARPS_M = T / (8 * MF);
  const int wm = (warp % WARPS_M) * 8 * MF, wn = (warp / WARPS_M) * 8 * NF;
  if (tid < T) {
    ca[tid] = (r0 + tid < nr) ? cmap[r0 + tid] : -1;
    cb[tid] = (c0 + tid < nr) ? cmap[c0 + tid] : -1;
  }
  __syncthreads();
  const int nk = (int)((m + BK - 1) / BK);
  // one K slice into stage s: per operand 128 columns x 16 pieces of 16 bytes
  auto issue = [&](int kb, int s) {
    double* As = ring + (size_t)s * stage_doubles();
    double* Bs = As + (size_t)T * BP;
    const int64_t k0 = (int64_t)kb * BK;
#pragma unroll
    for (int u = 0; u < (T * BK / 2) / NT; ++u) {
      const int q = tid + u * NT;
      const int j = q / (BK / 2), kq = (q % (BK / 2)) * 2;
      const int64_t row = k0 + kq;
      const int ks = row < m ? (int)((m - row) < 2 ? (m - row) : 2) : 0;
      const int a = ca[j], b = cb[j];
      cp_async16_sz_ls(As + j * BP + kq, (a >= 0 && ks > 0) ? G + (int64_t)a * ldg + row : G, (a >= 0) ? ks * 8 : 0);
      cp_async16_sz_ls(Bs + j * BP + kq, (b >= 0 && ks > 0) ? G + (int64_t)b * ldg + row : G, (b >= 0) ? ks * 8 : 0);
    }
  };
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) issue(s, s);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  double acc[MF][NF][2];
#pragma unroll
  for (int a = 0; a < MF; ++a)
#pragma unroll
    for (int b = 0; b < NF; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll 1
  for (int kb = 0; kb < nk; ++kb) {
    asm volatile("cp.async.wait_group %0;" ::"n"(STAGES - 2) : "memory");
    __syncthreads();   // slice kb has landed for every thread; slot (kb - 1) % STAGES is free
    if (kb + STAGES - 1 < nk) issue(kb + STAGES - 1, (kb + STAGES - 1) % STAGES);
    asm volatile("cp.async.commit_group;" ::: "memory");
    const double* As = ring + (size_t)(kb % STAGES) * stage_doubles();
    const double* Bs = As + (size_t)T * BP;
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      double av[MF], bv[NF];
#pragma unroll
      for (int mi = 0; mi < MF; ++mi) av[mi] = As[(wm + mi * 8 + g) * BP + k4 + tq];
#pragma unroll
      for (int ni = 0; ni < NF; ++ni) bv[ni] = Bs[(wn + ni * 8 + g) * BP + k4 + tq];
#pragma unroll
      for (int mi = 0; mi < MF; ++mi)
#pragma unroll
        for (int ni = 0; ni < NF; ++ni)
          asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                       : "+d"(acc[mi][ni][0]), "+d"(acc[mi][ni][1])
                       : "d"(av[mi]), "d"(bv[ni]));
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
#pragma unroll
  for (int ni = 0; ni < NF; ++ni)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int64_t cc = c0 + wn + ni * 8 + 2 * tq + e;
      if (cc >= nr) continue;
#pragma unroll
      for (int mi = 0; mi < MF; ++mi) {
        const int64_t r = r0 + wm + mi * 8 + g;
        if (r < nr) {
          Gls[cc * ldl + r] = acc[mi][ni][e];
          if (bi != bj) Gls[r * ldl + cc] = acc[mi][ni][e];
        }
      }
    }
}

// r = rhs - sum_p val_p G[:, el_p]
__global__ void k_ls_fold(const double* __restrict__ G, int64_t ldg, int64_t m, const double* __restrict__ rhs,
                          const int* __restrict__ el, const double* __restrict__ val, int npres,
                          double* __restrict__ r) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double v = rhs[i];
  for (int p = 0; p < npres; ++p) v -= val[p] * G[(int64_t)el[p] * ldg + i];
  r[i] = v;
}

// y[j] = G[:, cmap[j]] . r, one warp per j
__global__ void k_ls_atb(const double* __restrict__ G, int64_t ldg, int64_t m, const int* __restrict__ cmap,
                         int64_t nr, const double* __restrict__ r, double* __restrict__ y) {
  const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= nr) return;
  const double* col = G + (int64_t)cmap[j] * ldg;
  double s = 0;
  for (int64_t i = lane; i < m; i += 32) s += col[i] * r[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[j] = s;
}

int ls_solve(fp_ctx* c, const int* h_el, const double* h_val, int npres, double* h_gamma_red) {
  const int64_t n = c->N, ld = c->ld, nr = n - npres;
  const int64_t ldl = round_up(nr, 64);
  std::vector<int> cmap;
  cmap.reserve(nr);
  for (int64_t j = 0, p = 0; j < n; ++j) {
    if (p < npres && h_el[p] == j) { ++p; continue; }
    cmap.push_back((int)j);
  }
  // small device arrays: column map, prescribed indices and values (staging)
  const size_t bytes = cmap.size() * sizeof(int) + (size_t)npres * (sizeof(int) + sizeof(double)) + 64;
  if (int rc = ensure_stage(c, (bytes + 7) / 8)) return rc;
  char* st = reinterpret_cast<char*>(c->d_stage);
  double* d_val = reinterpret_cast<double*>(st);
  int* d_el = reinterpret_cast<int*>(st + (size_t)npres * sizeof(double));
  int* d_cmap = d_el + npres;
  if (npres > 0) {
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_val, h_val, npres * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_el, h_el, npres * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  }
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_cmap, cmap.data(), cmap.size() * sizeof(int), cudaMemcpyHostToDevice,
                                      c->stream));
  k_ls_fold<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->d_G, ld, n, c->d_rhs, d_el, d_val, npres, c->d_r);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_x, 0, ldl * sizeof(double), c->stream));
  k_ls_atb<<<(unsigned)((nr * 32 + 255) / 256), 256, 0, c->stream>>>(c->d_G, ld, n, d_cmap, nr, c->d_r, c->d_x);
  ++c->nlaunch;
  // the FP64 tensor path needs 16-byte aligned column starts (ld even)
  if (c->fp64_dmma && (ld % 2) == 0) {
    static SmemAttr attr;
    FP_CUDA_TRY(c->err, attr.ensure(k_gram_dmma, (int)gd::smem()));
    const int64_t nt = (nr + gd::T - 1) / gd::T;
    k_gram_dmma<<<(unsigned)(nt * (nt + 1) / 2), gd::NT, gd::smem(), c->stream>>>(c->d_G, ld, n, d_cmap, nr, c->d_LU,
                                                                                   ldl);
  } else {
    const int64_t nt = (nr + kGramT - 1) / kGramT;
    k_gram<<<(unsigned)(nt * (nt + 1) / 2), kGramThreads, 0, c->stream>>>(c->d_G, ld, n, d_cmap, nr, c->d_LU, ldl);
  }
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  if (int rc = lu_factor<double>(c, c->d_LU, nr, ldl, c->d_ipiv, c->d_cert)) return rc;
  if (int rc = lu_diag_inverses<double>(c, c->d_LU, nr, ldl)) return rc;
  if (int rc = lu_solve<double>(c, c->d_LU, nr, ldl, c->d_ipiv, c->d_x, ldl, 1, false)) return rc;
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(h_gamma_red, c->d_x, nr * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

}  // namespace fpb
