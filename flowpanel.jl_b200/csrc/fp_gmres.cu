// GMRES on the FP64 AIC (solve_gmres!, src/FLOWPanel_linearsolver.jl:110-157:
// Krylov.jl 0.9's gmres with memory=50, atol=rtol=sqrt(eps), restart=false),
// and GMRES-IR: restarted GMRES right-preconditioned by the FP32 LU factors,
// started from the refined iterate, for the mixed-precision form.
//
// Arnoldi uses classical Gram-Schmidt applied twice (two fused passes of
// dot products and updates per step instead of j sequential MGS steps); the
// small Hessenberg least-squares problem (Givens rotations) runs on the host.
// Stop test as Krylov.jl: the residual estimate <= atol + rtol ||r0||.
#include <cmath>
#include <vector>

#include "fp_internal.cuh"

namespace fpb {

constexpr int kDotThreads = 256;

// h[i] = V_i . w, i < nv
__global__ void k_dots(const double* __restrict__ V, int64_t ld, int nv, const double* __restrict__ w,
                       int64_t n, double* __restrict__ h) {
  __shared__ double red[kDotThreads / 32];
  const int i = blockIdx.x;
  double s = 0.0;
  for (int64_t r = threadIdx.x; r < n; r += kDotThreads) s += V[(int64_t)i * ld + r] * w[r];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < kDotThreads / 32; ++q) t += red[q];
    h[i] = t;
  }
}

// w -= sum_i h[i] V_i ; acc[i] += h[i]
__global__ void k_sub_Vh(const double* __restrict__ V, int64_t ld, int nv, const double* __restrict__ h,
                         double* __restrict__ w, int64_t n) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double s = w[r];
  for (int i = 0; i < nv; ++i) s -= h[i] * V[(int64_t)i * ld + r];
  w[r] = s;
}

// u = V y (nv columns)
__global__ void k_Vy(const double* __restrict__ V, int64_t ld, int nv, const double* __restrict__ y,
                     double* __restrict__ u, int64_t n) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double s = 0.0;
  for (int i = 0; i < nv; ++i) s += y[i] * V[(int64_t)i * ld + r];
  u[r] = s;
}

__global__ void k_scale(const double* __restrict__ a, double alpha, double* __restrict__ b, int64_t n) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) b[r] = alpha * a[r];
}

__global__ void k_add(double* __restrict__ x, const double* __restrict__ u, int64_t n) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) x[r] += u[r];
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) b[r] = (float)a[r];
}
__global__ void k_to_f64(const float* __restrict__ a, double* __restrict__ b, int64_t n) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) b[r] = (double)a[r];
}

int colnorm2(fp_ctx* c, const double* a, int64_t n, int64_t lda, int64_t k, double* d_out);

namespace {
struct Gm {
  fp_ctx* c;
  int64_t n, ld;
  unsigned g1;
  int norm2(const double* a, double* out) {
    if (int rc = colnorm2(c, a, n, ld, 1, c->d_h)) return rc;
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(out, c->d_h, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
    return FP_OK;
  }
  // u <- M^-1 u with the context's factors (FP64 in place, or the FP32 ones)
  int precond(double* u) {
    if (c->factored == FP_PREC_FP64) return lu_solve<double>(c, c->d_LU, n, ld, c->d_ipiv, u, ld, 1, false);
    k_to_f32<<<g1, 256, 0, c->stream>>>(u, c->d_w32, n);
    ++c->nlaunch;
    if (int rc = lu_solve<float>(c, c->d_G32, n, ld, c->d_ipiv, c->d_w32, ld, 1, false)) return rc;
    k_to_f64<<<g1, 256, 0, c->stream>>>(c->d_w32, u, n);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
    return FP_OK;
  }
};

// Device buffers for a basis of `cap` vectors: d_V holds the work vector w,
// the correction u, then V_0 .. V_cap (cap + 3 columns of ld); d_h holds the
// norms, two projection vectors of cap + 1 entries and y. `keep` columns of
// the old basis (w and u included) are carried over when it grows.
int ensure_basis(fp_ctx* c, int cap, int keep) {
  if (c->cap_gmres_m >= cap) return FP_OK;
  const int64_t ld = c->ld;
  double* V = nullptr;
  double* h = nullptr;
  FP_CUDA_TRY(c->err, cudaMalloc(&V, (size_t)(cap + 3) * ld * sizeof(double)));
  FP_CUDA_TRY(c->err, cudaMalloc(&h, (size_t)(3 * (cap + 1) + 16) * sizeof(double)));
  if (c->d_V && keep > 0)
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(V, c->d_V, (size_t)keep * ld * sizeof(double), cudaMemcpyDeviceToDevice,
                                        c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  if (c->d_V) cudaFree(c->d_V);
  if (c->d_h) cudaFree(c->d_h);
  c->d_V = V;
  c->d_h = h;
  c->cap_gmres_m = cap;
  return FP_OK;
}
}  // namespace

// GMRES for k right-hand sides, one after the other (as gmres(A, b::AbstractMatrix)
// does, src/FLOWPanel_linearsolver.jl:151-157), each from x = 0 unless
// `precondition` (GMRES-IR: from the refined iterate, right-preconditioned by
// the context's LU factors: the FP32 ones, or FP64 factors whose block-local
// pivots are not certified).
//  * Default (the reference's Krylov.jl 0.9 gmres with restart = false): one
//    Arnoldi process whose basis grows past `memory` (a storage hint) until
//    the Givens estimate of the residual norm falls to atol + rtol ||r0|| or
//    itmax steps (2N) are taken; a breakdown (h_{j+1,j} <= eps^(3/4)) ends it.
//  * gmres_restart != 0, and GMRES-IR: GMRES(memory), restarted from the true
//    residual, which must itself meet the tolerance.
int gmres_solve(fp_ctx* c, const double* b, double* x, int64_t k, const fp_solve_opts& o,
                bool precondition, int* iters, double* relres) {
  const int64_t n = c->N, ld = c->ld;
  const int mem = o.gmres_memory > 0 ? o.gmres_memory : 50;
  const bool restart = precondition || o.gmres_restart != 0;
  const double eps = 2.220446049250313e-16;
  const double btol = std::pow(eps, 0.75);
  const double atol = o.gmres_atol >= 0 ? o.gmres_atol : std::sqrt(eps);
  const double rtol = o.gmres_rtol >= 0 ? o.gmres_rtol : std::sqrt(eps);
  const int64_t itmax = o.gmres_itmax > 0 ? o.gmres_itmax : 2 * n;
  if (precondition && c->factored != FP_PREC_MIXED && c->factored != FP_PREC_FP64)
    return c->err.set(FP_ESTATE, "GMRES-IR needs LU factors");
  if (int rc = ensure_basis(c, (int)std::min<int64_t>(mem, itmax), 0)) return rc;
  if (!c->d_part) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_part, (size_t)kGemvSplitHost * 4 * c->capN * sizeof(double)));
  Gm G{c, n, ld, (unsigned)((n + 255) / 256)};
  int total = 0;
  double worst = 0.0;
  bool all_conv = true;
  // host side of the Arnoldi process: column j of the rotated Hessenberg
  // matrix (j + 2 entries), the rotations and the rotated right-hand side
  std::vector<std::vector<double>> H;
  std::vector<double> cs, sn, g, h, h2, y;
  for (int64_t q = 0; q < k; ++q) {
    const double* bq = b + q * ld;
    double* xq = x + q * ld;
    if (!precondition) FP_CUDA_TRY(c->err, cudaMemsetAsync(xq, 0, n * sizeof(double), c->stream));
    double bn2 = 0;
    if (int rc = G.norm2(bq, &bn2)) return rc;
    const double bnorm = std::sqrt(bn2);
    // Krylov.jl: eps = atol + rtol ||r0||, with r0 = b from x = 0; GMRES-IR
    // measures against ||b|| too
    const double target = atol + rtol * bnorm;
    // r = b - A x in w
    if (int rc = gemv_residual(c, c->d_G, n, ld, xq, bq, c->d_V, 1)) return rc;
    double beta2 = 0;
    if (int rc = G.norm2(c->d_V, &beta2)) return rc;
    double beta = std::sqrt(beta2);
    int it = 0;
    bool conv = beta <= target;
    while (!conv && it < itmax) {
      k_scale<<<G.g1, 256, 0, c->stream>>>(c->d_V, 1.0 / beta, c->d_V + 2 * ld, n);
      ++c->nlaunch;
      H.clear(); cs.clear(); sn.clear();
      g.assign(1, beta);
      int kd = 0;
      bool solved = false;
      for (int j = 0; it < itmax; ++j) {
        if (restart && j >= mem) break;
        double* const w = c->d_V;
        double* const u = c->d_V + ld;
        double* const V = c->d_V + 2 * ld;
        double* const dh = c->d_h + 8;
        double* vj = V + (size_t)j * ld;
        const double* src = vj;
        if (precondition) {
          FP_CUDA_TRY(c->err, cudaMemcpyAsync(u, vj, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
          if (int rc = G.precond(u)) return rc;
          src = u;
        }
        // w = A src  (residual form with b = 0: w = -(A src); negate via scale)
        FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_r, 0, n * sizeof(double), c->stream));
        if (int rc = gemv_residual(c, c->d_G, n, ld, src, c->d_r, w, 1)) return rc;
        k_scale<<<G.g1, 256, 0, c->stream>>>(w, -1.0, w, n);
        ++c->nlaunch;
        // classical Gram-Schmidt, twice
        h.resize(j + 1);
        h2.resize(j + 1);
        k_dots<<<j + 1, kDotThreads, 0, c->stream>>>(V, ld, j + 1, w, n, dh);
        ++c->nlaunch;
        k_sub_Vh<<<G.g1, 256, 0, c->stream>>>(V, ld, j + 1, dh, w, n);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaMemcpyAsync(h.data(), dh, (j + 1) * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        k_dots<<<j + 1, kDotThreads, 0, c->stream>>>(V, ld, j + 1, w, n, dh + c->cap_gmres_m + 1);
        ++c->nlaunch;
        k_sub_Vh<<<G.g1, 256, 0, c->stream>>>(V, ld, j + 1, dh + c->cap_gmres_m + 1, w, n);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaMemcpyAsync(h2.data(), dh + c->cap_gmres_m + 1, (j + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                                            c->stream));
        double hn2 = 0;
        if (int rc = G.norm2(w, &hn2)) return rc;   // syncs the stream
        const double hn = std::sqrt(hn2);
        H.emplace_back(j + 2);
        std::vector<double>& Hj = H.back();
        for (int i = 0; i <= j; ++i) Hj[i] = h[i] + h2[i];
        Hj[j + 1] = hn;
        const bool breakdown = hn <= btol;
        if (!breakdown) {
          if (j + 1 > c->cap_gmres_m) {   // the basis outgrows its storage hint: room for V_{j+1}
            const int cap2 = (int)std::min<int64_t>(2 * (int64_t)c->cap_gmres_m, itmax);
            if (int rc = ensure_basis(c, std::max(cap2, j + 1), j + 3)) return rc;
          }
          k_scale<<<G.g1, 256, 0, c->stream>>>(c->d_V, 1.0 / hn, c->d_V + 2 * ld + (size_t)(j + 1) * ld, n);
          ++c->nlaunch;
        }
        FP_CUDA_TRY(c->err, cudaGetLastError());
        // Givens rotations
        for (int i = 0; i < j; ++i) {
          const double t = cs[i] * Hj[i] + sn[i] * Hj[i + 1];
          Hj[i + 1] = -sn[i] * Hj[i] + cs[i] * Hj[i + 1];
          Hj[i] = t;
        }
        const double den = std::hypot(Hj[j], Hj[j + 1]);
        cs.push_back(den > 0 ? Hj[j] / den : 1.0);
        sn.push_back(den > 0 ? Hj[j + 1] / den : 0.0);
        Hj[j] = den;
        Hj[j + 1] = 0.0;
        g.push_back(-sn[j] * g[j]);
        g[j] = cs[j] * g[j];
        ++it;
        kd = j + 1;
        solved = std::fabs(g[j + 1]) <= target;
        if (solved || breakdown) break;
      }
      // y = R^-1 g (upper triangular kd x kd), x += V y (preconditioned)
      y.assign(kd, 0.0);
      for (int i = kd - 1; i >= 0; --i) {
        double s = g[i];
        for (int l = i + 1; l < kd; ++l) s -= H[l][i] * y[l];
        y[i] = s / H[i][i];
      }
      double* const w = c->d_V;
      double* const u = c->d_V + ld;
      double* const V = c->d_V + 2 * ld;
      double* const dh = c->d_h + 8;
      FP_CUDA_TRY(c->err, cudaMemcpyAsync(dh, y.data(), kd * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      k_Vy<<<G.g1, 256, 0, c->stream>>>(V, ld, kd, dh, u, n);
      ++c->nlaunch;
      if (precondition)
        if (int rc = G.precond(u)) return rc;
      k_add<<<G.g1, 256, 0, c->stream>>>(xq, u, n);
      ++c->nlaunch;
      FP_CUDA_TRY(c->err, cudaGetLastError());
      if (int rc = gemv_residual(c, c->d_G, n, ld, xq, bq, w, 1)) return rc;
      if (int rc = G.norm2(w, &beta2)) return rc;
      beta = std::sqrt(beta2);
      // restarted: the true residual decides; one Arnoldi process: its estimate
      conv = restart ? beta <= target : solved;
      if (!restart) break;
    }
    total += it;
    worst = std::max(worst, bnorm > 0 ? beta / bnorm : beta);
    all_conv = all_conv && conv;
  }
  *iters = total;
  *relres = worst;
  if (!all_conv) return c->err.set(FP_ENOCONV, "GMRES did not reach its tolerance");
  return FP_OK;
}

}  // namespace fpb
