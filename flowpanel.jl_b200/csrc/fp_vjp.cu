// Reverse mode of the vortex-ring and wake-horseshoe velocity kernels (FP64).
//
// The reference differentiates its solve with ForwardDiff duals pushed
// through _G_Uvortexring! / _Uvortexring! and the ImplicitAD rule of the
// linear solve (src/FLOWPanel_linearsolver.jl:73,128). Here the pair kernels
// are differentiated by hand in reverse mode, so that one pass over the
// (target, panel) pairs gives the gradient with respect to every vertex,
// target, wake direction and strength.
//
// For a target X with cotangent vector w (for the assembly w_i = -lambda_i n_i,
// for a field evaluation the caller's dF/dU_i) and element strengths s_j, the
// scalar being differentiated is F = sum_i w_i . sum_j s_j U_j(X_i).
//
// Bound filament a -> b (U_boundvortex, src/FLOWPanel_elements.jl:345-428):
//   r_a = X - a, r_b = X - b, l = |r|, i = 1/(l + offset), c = r_a x r_b,
//   rd = (b - a) . (r_a i_a - r_b i_b), q = 1/(4 pi (|c|^2 + offset^2)),
//   f = s rd (c . w) q  (zero when |c|^2 <= cutoff^2).
//   df/dr_a = s q [ (c.w) (i_a r_ab - i_a^2 (r_ab . r_a)/l_a r_a) + rd (r_b x w) ]
//             - 2 s rd (c.w) q / (|c|^2 + offset^2) (r_b x c)
//   df/dr_b = s q [ (c.w) (-i_b r_ab + i_b^2 (r_ab . r_b)/l_b r_b) + rd (w x r_a) ]
//             - 2 s rd (c.w) q / (|c|^2 + offset^2) (c x r_a)
//   df/dr_ab = s (c.w) q (r_a i_a - r_b i_b), with r_ab = b - a.
// Semi-infinite vortex from p along d (U_semiinfinite_vortex, :480-628): the
// foot point p0 = p + ((X - p).d) d, a bound filament p -> p0 (when
// |p0 - p|^2 > offset^2) and the infinite part f = s ((d x h).w) q_h with
// h = X - p0, q_h = 1/(4 pi (|h|^2 + offset^2)) (zero when |h|^2 <= cutoff^2);
// p0's gradient is carried back to X, p and d.
#include "fp_internal.cuh"

namespace fpb {

namespace {

struct D3 { double x, y, z; };
__device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return d3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
  return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ void acc3(D3& a, D3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }

// Per-node quantities of a target: r = X - p, l = |r|, i = 1/(l + offset).
struct NodeQ { D3 r; double l, i; };
__device__ __forceinline__ NodeQ nodeq(D3 X, D3 p, double offset) {
  NodeQ q;
  q.r = X - p;
  q.l = sqrt(dot3(q.r, q.r));
  q.i = 1.0 / (q.l + offset);
  return q;
}

// Reverse of one filament edge given its node quantities and r_ab = b - a.
// Adds df/dr_a to ga, df/dr_b to gb, df/dr_ab to gab, s * U to U and
// df/ds to gs.
__device__ __forceinline__ void edge_rev(const NodeQ& A, const NodeQ& B, D3 rab, D3 w, double s,
                                         double cutoff2, double offset2, D3& ga, D3& gb, D3& gab,
                                         D3& U, double& gs) {
  const D3 c = cross3(A.r, B.r);
  const double cc = dot3(c, c);
  if (!(cc > cutoff2)) return;
  const D3 u = A.i * A.r - B.i * B.r;
  const double rd = dot3(rab, u);
  const double den = cc + offset2;
  const double q = 1.0 / (kFourPi * den);
  const double g = dot3(c, w);
  const double Arq = rd * q;             // velocity per unit strength is Arq * c
  acc3(U, (s * Arq) * c);
  gs += Arq * g;
  const double Ard = s * g * q;          // df/drd
  const double Ag = s * Arq;             // df/d(c.w)
  const double Ac = -2.0 * s * rd * g * q / den;   // df/dc via |c|^2, times 1/2 of d|c|^2/dc
  const double ta = A.l > 0.0 ? A.i * A.i * dot3(rab, A.r) / A.l : 0.0;
  const double tb = B.l > 0.0 ? B.i * B.i * dot3(rab, B.r) / B.l : 0.0;
  acc3(ga, Ard * (A.i * rab - ta * A.r) + Ag * cross3(B.r, w) + Ac * cross3(B.r, c));
  acc3(gb, Ard * (tb * B.r - B.i * rab) + Ag * cross3(w, A.r) + Ac * cross3(c, A.r));
  acc3(gab, Ard * u);
}

// Reverse of a free filament pa -> pb of strength s.
__device__ __forceinline__ void filament_rev(D3 pa, D3 pb, double s, D3 X, D3 w, double offset,
                                             double cutoff2, double offset2, D3& gpa, D3& gpb,
                                             D3& gX, D3& U, double& gs) {
  const NodeQ A = nodeq(X, pa, offset), B = nodeq(X, pb, offset);
  D3 ga = d3(0, 0, 0), gb = d3(0, 0, 0), gab = d3(0, 0, 0);
  edge_rev(A, B, pb - pa, w, s, cutoff2, offset2, ga, gb, gab, U, gs);
  acc3(gX, ga + gb);
  gpa = gpa - ga - gab;
  gpb = gpb - gb + gab;
}

// Reverse of the semi-infinite vortex from p along d (strength s).
__device__ __forceinline__ void semiinf_rev(D3 p, D3 d, double s, D3 X, D3 w, double offset,
                                            double cutoff2, double offset2, D3& gp, D3& gd, D3& gX,
                                            D3& U, double& gs) {
  const D3 xmp = X - p;
  const double t = dot3(xmp, d);
  const D3 p0 = p + t * d;
  const D3 e = p0 - p;
  D3 gp0 = d3(0, 0, 0);
  if (dot3(e, e) > offset2) filament_rev(p, p0, s, X, w, offset, cutoff2, offset2, gp, gp0, gX, U, gs);
  const D3 h = X - p0;
  const double hsqr = dot3(h, h);
  if (hsqr > cutoff2) {
    const D3 m = cross3(d, h);
    const double den = hsqr + offset2;
    const double qh = 1.0 / (kFourPi * den);
    const double mw = dot3(m, w);
    acc3(U, (s * qh) * m);
    gs += mw * qh;
    const D3 Gh = (s * qh) * cross3(w, d) - (2.0 * s * mw * qh / den) * h;
    acc3(gd, (s * qh) * cross3(h, w));
    acc3(gX, Gh);
    gp0 = gp0 - Gh;
  }
  const double gt = dot3(gp0, d);
  acc3(gp, gp0 - gt * d);
  acc3(gX, gt * d);
  acc3(gd, t * gp0 + gt * xmp);
}

// Reverse of a ring of NN nodes (one pair): vertex gradients into gv, the
// target gradient and velocity into gX, U, df/ds into gs.
template <int NN>
__device__ __forceinline__ void ring_rev(const double* __restrict__ p, double s, D3 X, D3 w,
                                         double offset, double cutoff2, double offset2, D3* gv,
                                         D3& gX, D3& U, double& gs) {
  NodeQ q[NN];
#pragma unroll
  for (int k = 0; k < NN; ++k) q[k] = nodeq(X, d3(p[3 * k], p[3 * k + 1], p[3 * k + 2]), offset);
  D3 gr[NN];
#pragma unroll
  for (int k = 0; k < NN; ++k) gr[k] = d3(0, 0, 0);
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    const int b = (a + 1) % NN;
    const D3 rab = d3(p[3 * b] - p[3 * a], p[3 * b + 1] - p[3 * a + 1], p[3 * b + 2] - p[3 * a + 2]);
    D3 gab = d3(0, 0, 0);
    edge_rev(q[a], q[b], rab, w, s, cutoff2, offset2, gr[a], gr[b], gab, U, gs);
    acc3(gv[b], gab);
    gv[a] = gv[a] - gab;
  }
#pragma unroll
  for (int k = 0; k < NN; ++k) {
    acc3(gX, gr[k]);
    gv[k] = gv[k] - gr[k];
  }
}

// Warp reduce-scatter of 8 values: on return, lane l with (l & 3) == 0 holds
// the warp sum of value (l >> 2) in the return value.
__device__ __forceinline__ double warp_reduce_scatter8(const double v[8], int lane) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  double a[4], c[2];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double send = b4 ? v[k] : v[k + 4];
    const double keep = b4 ? v[k + 4] : v[k];
    a[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double send = b3 ? a[k] : a[k + 2];
    const double keep = b3 ? a[k + 2] : a[k];
    c[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  double e;
  {
    const double send = b2 ? c[0] : c[1];
    const double keep = b2 ? c[1] : c[0];
    e = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  e += __shfl_xor_sync(0xffffffffu, e, 2);
  e += __shfl_xor_sync(0xffffffffu, e, 1);
  return e;
}

constexpr int kVjpThreads = 128;   // panels per CTA (one per thread)
constexpr int kVjpTile = 32;       // targets staged per tile
constexpr int kVjpChunk = 512;     // targets per CTA

// One thread per panel, targets broadcast from shared memory. Per-panel sums
// (12 vertex components, strength) stay in registers over the CTA's target
// chunk; per-target sums (gradient, velocity) are reduced over the CTA's
// panels by a warp reduce-scatter and shared memory, then added to global
// memory with atomics (the other CTAs on the same targets add theirs).
__global__ void __launch_bounds__(kVjpThreads)
k_vjp_ring(const PanelRec* __restrict__ panels, const double* __restrict__ strength, int64_t n,
           const double* __restrict__ tx, const double* __restrict__ tw, int64_t m, double offset,
           double cutoff2, double offset2, double* __restrict__ gX, double* __restrict__ Uo,
           double* __restrict__ gvert, double* __restrict__ gs_out) {
  __shared__ double st[kVjpTile][6];
  __shared__ double red[kVjpThreads / 32][kVjpTile][8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t j = (int64_t)blockIdx.x * kVjpThreads + tid;
  const bool valid = j < n;
  double p[12];
  int nn = 4;
  double s = 0.0;
  if (valid) {
    const PanelRec& P = panels[j];
#pragma unroll
    for (int k = 0; k < 12; ++k) p[k] = P.p[k];
    nn = (int)P.nn;
    s = strength[j];
  } else {
#pragma unroll
    for (int k = 0; k < 12; ++k) p[k] = 0.0;
  }
  D3 gv[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) gv[k] = d3(0, 0, 0);
  double gs = 0.0;
  const int64_t t0 = (int64_t)blockIdx.y * kVjpChunk;
  const int64_t t1 = imin64(m, t0 + kVjpChunk);
  for (int64_t tb = t0; tb < t1; tb += kVjpTile) {
    const int nt = (int)imin64(kVjpTile, t1 - tb);
    __syncthreads();
    for (int e = tid; e < kVjpTile * 6; e += kVjpThreads) {
      const int t = e % kVjpTile, c = e / kVjpTile;
      double v = 0.0;
      if (t < nt) v = (c < 3) ? tx[c * m + tb + t] : tw[(c - 3) * m + tb + t];
      st[t][c] = v;
    }
    __syncthreads();
    for (int t = 0; t < nt; ++t) {
      const D3 X = d3(st[t][0], st[t][1], st[t][2]);
      const D3 w = d3(st[t][3], st[t][4], st[t][5]);
      D3 gx = d3(0, 0, 0), U = d3(0, 0, 0);
      if (valid) {
        if (nn == 4) ring_rev<4>(p, s, X, w, offset, cutoff2, offset2, gv, gx, U, gs);
        else ring_rev<3>(p, s, X, w, offset, cutoff2, offset2, gv, gx, U, gs);
      }
      const double v[8] = {gx.x, gx.y, gx.z, U.x, U.y, U.z, 0.0, 0.0};
      const double r = warp_reduce_scatter8(v, lane);
      if ((lane & 3) == 0) red[warp][t][lane >> 2] = r;
    }
    __syncthreads();
    for (int e = tid; e < nt * 6; e += kVjpThreads) {
      const int t = e / 6, c = e % 6;
      double a = 0.0;
#pragma unroll
      for (int w = 0; w < kVjpThreads / 32; ++w) a += red[w][t][c];
      if (c < 3) atomicAdd(&gX[c * m + tb + t], a);
      else if (Uo) atomicAdd(&Uo[(c - 3) * m + tb + t], a);
    }
  }
  if (valid) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < nn) {
        atomicAdd(&gvert[12 * j + 3 * k], gv[k].x);
        atomicAdd(&gvert[12 * j + 3 * k + 1], gv[k].y);
        atomicAdd(&gvert[12 * j + 3 * k + 2], gv[k].z);
      }
    }
    atomicAdd(&gs_out[j], gs);
  }
}

// Wake horseshoes: one thread per target, kWakeEdges shedding edges per CTA
// row; the per-edge sums (TE nodes of both sides, both directions, both
// strengths: 20 values) are reduced over the warp and added with atomics,
// the per-target sums once per CTA.
constexpr int kVjpWakeThreads = 128;
constexpr int kWakeEdges = 8;
constexpr int kWakeGrad = 20;   // pa, pb, qa, qb, da, db (3 each), s_pi, s_pj

__global__ void __launch_bounds__(kVjpWakeThreads)
k_vjp_wake(const WakeRec* __restrict__ wake, int64_t nsh, const double* __restrict__ strength,
           const double* __restrict__ tx, const double* __restrict__ tw, int64_t m, double offset,
           double cutoff2, double offset2, double* __restrict__ gX, double* __restrict__ Uo,
           double* __restrict__ gwake) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * kVjpWakeThreads + threadIdx.x;
  const bool valid = i < m;
  D3 X = d3(0, 0, 0), w = d3(0, 0, 0);
  if (valid) {
    X = d3(tx[i], tx[m + i], tx[2 * m + i]);
    w = d3(tw[i], tw[m + i], tw[2 * m + i]);
  }
  D3 gx = d3(0, 0, 0), U = d3(0, 0, 0);
  const int64_t e0 = (int64_t)blockIdx.y * kWakeEdges, e1 = imin64(nsh, e0 + kWakeEdges);
  for (int64_t e = e0; e < e1; ++e) {
    const WakeRec& R = wake[e];
    const D3 pa = d3(R.pa[0], R.pa[1], R.pa[2]), pb = d3(R.pb[0], R.pb[1], R.pb[2]);
    const D3 da = d3(R.da[0], R.da[1], R.da[2]), db = d3(R.db[0], R.db[1], R.db[2]);
    D3 gpa = d3(0, 0, 0), gpb = d3(0, 0, 0), gqa = d3(0, 0, 0), gqb = d3(0, 0, 0);
    D3 gda = d3(0, 0, 0), gdb = d3(0, 0, 0);
    double gsi = 0.0, gsj = 0.0;
    if (valid) {
      // upper side: horseshoe over (pa, pb) with (da, db), strength s_pi
      // (U_semiinfinite_horseshoe, src/FLOWPanel_elements.jl:692-730)
      const double si = strength[R.pi];
      double g1 = 0.0, g2 = 0.0, g3 = 0.0;
      semiinf_rev(pa, da, -si, X, w, offset, cutoff2, offset2, gpa, gda, gx, U, g1);
      filament_rev(pa, pb, si, X, w, offset, cutoff2, offset2, gpa, gpb, gx, U, g2);
      semiinf_rev(pb, db, si, X, w, offset, cutoff2, offset2, gpb, gdb, gx, U, g3);
      gsi = -g1 + g2 + g3;
      if (R.pj >= 0) {
        // lower side: its own TE nodes with the directions swapped (db, da)
        // (src/FLOWPanel_liftingbody.jl:540-567), strength s_pj
        const D3 qa = d3(R.qa[0], R.qa[1], R.qa[2]), qb = d3(R.qb[0], R.qb[1], R.qb[2]);
        const double sj = strength[R.pj];
        double h1 = 0.0, h2 = 0.0, h3 = 0.0;
        semiinf_rev(qa, db, -sj, X, w, offset, cutoff2, offset2, gqa, gdb, gx, U, h1);
        filament_rev(qa, qb, sj, X, w, offset, cutoff2, offset2, gqa, gqb, gx, U, h2);
        semiinf_rev(qb, da, sj, X, w, offset, cutoff2, offset2, gqb, gda, gx, U, h3);
        gsj = -h1 + h2 + h3;
      }
    }
    double v[kWakeGrad] = {gpa.x, gpa.y, gpa.z, gpb.x, gpb.y, gpb.z, gqa.x, gqa.y, gqa.z, gqb.x,
                           gqb.y, gqb.z, gda.x, gda.y, gda.z, gdb.x, gdb.y, gdb.z, gsi, gsj};
#pragma unroll
    for (int k = 0; k < kWakeGrad; ++k) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < kWakeGrad; ++k) atomicAdd(&gwake[kWakeGrad * e + k], v[k]);
    }
  }
  if (valid) {
    atomicAdd(&gX[i], gx.x);
    atomicAdd(&gX[m + i], gx.y);
    atomicAdd(&gX[2 * m + i], gx.z);
    if (Uo) {
      atomicAdd(&Uo[i], U.x);
      atomicAdd(&Uo[m + i], U.y);
      atomicAdd(&Uo[2 * m + i], U.z);
    }
  }
}

__global__ void k_vjp_cotangent(const double* __restrict__ lambda, const double* __restrict__ tgt,
                                int64_t n, double* __restrict__ w) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double l = lambda[i];
  w[i] = -l * tgt[3 * n + i];
  w[n + i] = -l * tgt[4 * n + i];
  w[2 * n + i] = -l * tgt[5 * n + i];
}

}  // namespace

// Gradient of F = sum_i w_i . sum_j s_j U_j(X_i) over the body's rings and
// wake horseshoes. All outputs are accumulated (the caller zeroes them):
// gX, U 3 x m (SoA), gvert N x 12 (per panel, node k at 3k..3k+2), gs N,
// gwake nsh x 20.
int launch_pair_vjp(fp_ctx* c, const double* d_strength, const double* d_x, const double* d_w,
                    int64_t m, double* d_gX, double* d_U, double* d_gvert, double* d_gs,
                    double* d_gwake) {
  const int64_t n = c->N;
  const double offset = c->kern_offset, cut2 = c->kern_cutoff * c->kern_cutoff, off2 = offset * offset;
  dim3 g((unsigned)((n + kVjpThreads - 1) / kVjpThreads), (unsigned)((m + kVjpChunk - 1) / kVjpChunk));
  k_vjp_ring<<<g, kVjpThreads, 0, c->stream>>>(c->d_panels, d_strength, n, d_x, d_w, m, offset, cut2, off2,
                                               d_gX, d_U, d_gvert, d_gs);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  if (c->nsh > 0) {
    dim3 g2((unsigned)((m + kVjpWakeThreads - 1) / kVjpWakeThreads),
            (unsigned)((c->nsh + kWakeEdges - 1) / kWakeEdges));
    k_vjp_wake<<<g2, kVjpWakeThreads, 0, c->stream>>>(c->d_wake, c->nsh, d_strength, d_x, d_w, m, offset, cut2,
                                                      off2, d_gX, d_U, d_gwake);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
  }
  return FP_OK;
}

int launch_vjp_cotangent(fp_ctx* c, const double* d_lambda, double* d_w) {
  const int64_t n = c->N;
  k_vjp_cotangent<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(d_lambda, c->d_tgt, n, d_w);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

}  // namespace fpb
