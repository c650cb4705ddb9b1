// Surface post-processing of a solved body on the device:
//
//   * the surface velocity from the gradient of the doublet strength,
//     calcfield_Ugradmu! with its cell scheme (Green-Gauss with the
//     inverse-distance face value, the trailing-edge cells' face terms added
//     back) and node scheme (linear gradient of area-weighted nodal values),
//     combined per cell (src/FLOWPanel_postprocess.jl:139-1042);
//   * the pressure coefficient with the trailing-edge Kutta average
//     (calcfield_Cp!, :1059-1112), the panel forces with their trailing-edge
//     override (calcfield_F!, :1199-1307) and their sum projected on lift,
//     drag and sideslip (calcfield_LDS!, :1615-1652).
//
// The reference asks three questions of GeometricTools (unvendored); they are
// answered here as follows:
//   neighbor(grid, ni, ci; preserveEdge=true) -> the cell across the edge from
//       the cell's local node ni to ni%3+1, none at a free edge;
//   get_nodal_data(grid, data; areas)          -> per node, the area-weighted
//       mean of the data of the cells around it;
//   project_3d_2d! + get_tri_gradient!         -> the in-plane gradient of the
//       linear interpolant of the three nodal values.
//
// The topology (neighbours, cells around each node, areas) is built once per
// geometry on the host from a hash of the edges. The schemes run one thread
// per cell in FP64 (a few hundred flops per cell: latency and launch bound at
// these sizes). The Kutta averages are a recurrence over the shedding rows in
// the reference (a row reads values an earlier row may have written); one CTA
// runs it in shared memory, then sums the forces.
#include "fp_internal.cuh"

#include <cmath>
#include <string>
#include <unordered_map>
#include <vector>

namespace fpb {

namespace {

constexpr int kPostThreads = 128;
constexpr int kKuttaThreads = 512;
constexpr int kForcedCell = 1 << 16;     // teflag bit: cell value forced on the node scheme (pi, pi+1, pj, pj-1)
constexpr int kTeUpper = 1 << 17;        // teflag bit: an upper trailing-edge cell (pi, pi+1) of the sharp-TE node scheme
constexpr int kTeLower = 1 << 18;        // teflag bit: a lower trailing-edge cell (pj, pj-1)
constexpr size_t kKuttaSmemMax = 48 * 1024;

template <class T> void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

struct PostArgs {
  const PanelRec* panels;
  const double* tgt;       // 6 x N SoA: control points, normals
  int64_t N;
  const double* area;
  const int32_t* nb;       // 3N neighbours, then 3N node indices
  const int32_t* teflag;
  const double* sgn;       // sign(CPoffset) per cell (1 where 0)
  const double* g;         // strengths (the Gammai column)
  const double* nodal;     // nodal values (node scheme)
  int sharpte;             // node scheme: trailing-edge cells take their side's nodal values at TE nodes
  const int32_t* teslot;   // node -> trailing-edge slot, -1 if none
  const double* nodal_te;  // 2 x nte: the upper, then the lower nodal values of the TE nodes
  int64_t nte;
  int mode;                // FP_UGRADMU_* or -1 for none
  int force_cellTE;
  double cosang;
  double maxgrad;
  double* out;             // 3N AoS
  double* out_cell;
  double* out_node;
  // surface loads fused behind the scheme (optional)
  const double* U;         // 3N velocity at the control points (freestream + induced)
  double Uref;
  const double* Cp0;       // N values Cp is added to (calcfield_Cp! adds to `out`), or null
  double qneg;             // (-0.5 rho) * Uinf^2
  double* Utot;            // 3N, U + Ugradmu
  double* Cp;              // N
  double* F;               // 3N
};

// One Green-Gauss face term of the cell scheme, already scaled by
// 0.5*sign(CPoffset): (postprocess.jl:189-247) for the edge from local node k
// to k+1 of the triangle P with neighbour control point cpn and strength gn.
__device__ __forceinline__ void gg_term(const double* P, int k, const double* nc, const double* cpc,
                                        const double* cpn, double gc, double gn, double area, double hs,
                                        double* t) {
  const int ei = k, ej = (k + 1) % 3;
  const double r1 = P[3 * ej] - P[3 * ei];
  const double r2 = P[3 * ej + 1] - P[3 * ei + 1];
  const double r3 = P[3 * ej + 2] - P[3 * ei + 2];
  double d1 = r2 * nc[2] - r3 * nc[1];
  double d2 = r3 * nc[0] - r1 * nc[2];
  double d3 = r1 * nc[1] - r2 * nc[0];
  const double dmag = sqrt(d1 * d1 + d2 * d2 + d3 * d3);
  d1 /= dmag;
  d2 /= dmag;
  d3 /= dmag;
  const double m1 = P[3 * ei] - cpc[0], m2 = P[3 * ei + 1] - cpc[1], m3 = P[3 * ei + 2] - cpc[2];
  const double n1 = P[3 * ei] - cpn[0], n2 = P[3 * ei + 1] - cpn[1], n3 = P[3 * ei + 2] - cpn[2];
  const double a1 = m2 * r3 - m3 * r2, a2 = m3 * r1 - m1 * r3, a3 = m1 * r2 - m2 * r1;
  const double b1 = n2 * r3 - n3 * r2, b2 = n3 * r1 - n1 * r3, b3 = n1 * r2 - n2 * r1;
  const double dMain = sqrt(a1 * a1 + a2 * a2 + a3 * a3);
  const double dNear = sqrt(b1 * b1 + b2 * b2 + b3 * b3);
  const double f = dNear / (dMain + dNear);
  const double face = f * gc + (1.0 - f) * gn;
  const double mag = face * sqrt(r1 * r1 + r2 * r2 + r3 * r3) / area;
  t[0] = hs * d1 * mag;
  t[1] = hs * d2 * mag;
  t[2] = hs * d3 * mag;
}

// In-plane gradient of the linear function through (P_k, v_k), k = 0..2.
__device__ __forceinline__ void tri_gradient(const double* P, double v1, double v2, double v3, double* g) {
  double e1[3] = {P[3] - P[0], P[4] - P[1], P[5] - P[2]};
  const double x2 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
  e1[0] /= x2; e1[1] /= x2; e1[2] /= x2;
  const double w[3] = {P[6] - P[0], P[7] - P[1], P[8] - P[2]};
  const double x3 = w[0] * e1[0] + w[1] * e1[1] + w[2] * e1[2];
  double e2[3] = {w[0] - x3 * e1[0], w[1] - x3 * e1[1], w[2] - x3 * e1[2]};
  const double y3 = sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
  e2[0] /= y3; e2[1] /= y3; e2[2] /= y3;
  const double gx = (v2 - v1) / x2;
  const double gy = (v3 - v1 - gx * x3) / y3;
  for (int d = 0; d < 3; ++d) g[d] = gx * e1[d] + gy * e2[d];
}

__global__ void __launch_bounds__(kPostThreads)
k_nodal(const int32_t* __restrict__ voff, const int32_t* __restrict__ vcell, const double* __restrict__ area,
        const double* __restrict__ g, int64_t nn, double* __restrict__ nodal) {
  const int64_t v = (int64_t)blockIdx.x * kPostThreads + threadIdx.x;
  if (v >= nn) return;
  double num = 0.0, den = 0.0;
  for (int32_t k = voff[v]; k < voff[v + 1]; ++k) {
    const int32_t c = vcell[k];
    num += area[c] * g[c];
    den += area[c];
  }
  nodal[v] = den > 0.0 ? num / den : 0.0;
}

__global__ void __launch_bounds__(kPostThreads) k_ugradmu(PostArgs a) {
  const int64_t c = (int64_t)blockIdx.x * kPostThreads + threadIdx.x;
  if (c >= a.N) return;
  const int64_t N = a.N;
  double res[3] = {0.0, 0.0, 0.0};
  if (a.mode >= 0) {
    double P[9];
    for (int i = 0; i < 9; ++i) P[i] = a.panels[c].p[i];
    const double s = a.sgn[c];
    const double nc[3] = {a.tgt[3 * N + c], a.tgt[4 * N + c], a.tgt[5 * N + c]};
    int nbk[3];
    for (int k = 0; k < 3; ++k) nbk[k] = a.nb[3 * c + k];
    double oc[3] = {0.0, 0.0, 0.0}, on[3] = {0.0, 0.0, 0.0};
    if (a.mode == FP_UGRADMU_COMBINED || a.mode == FP_UGRADMU_CELL) {
      if (a.mode == FP_UGRADMU_CELL)   // the cell scheme alone adds to `out`
        for (int d = 0; d < 3; ++d) oc[d] = a.out[3 * c + d];
      const double cpc[3] = {a.tgt[c], a.tgt[N + c], a.tgt[2 * N + c]};
      const double gc = a.g[c], ar = a.area[c], hs = 0.5 * s;
      double t[3][3];
      for (int k = 0; k < 3; ++k) {
        if (nbk[k] < 0) continue;
        const int64_t n = nbk[k];
        const double cpn[3] = {a.tgt[n], a.tgt[N + n], a.tgt[2 * N + n]};
        gg_term(P, k, nc, cpc, cpn, gc, a.g[n], ar, hs, t[k]);
        for (int d = 0; d < 3; ++d) oc[d] -= t[k][d];
      }
      // trailing-edge cells: the face terms added back once per appearance
      // as pi or pj in the shedding rows (postprocess.jl:391-474)
      const int te = a.teflag[c] & 0xffff;
      for (int r = 0; r < te; ++r)
        for (int k = 0; k < 3; ++k)
          if (nbk[k] >= 0)
            for (int d = 0; d < 3; ++d) oc[d] += t[k][d];
      if (a.mode == FP_UGRADMU_CELL) {
        const double nrm = sqrt(oc[0] * oc[0] + oc[1] * oc[1] + oc[2] * oc[2]);
        if (nrm >= a.maxgrad) oc[0] = oc[1] = oc[2] = 0.0;
      }
    }
    if (a.mode == FP_UGRADMU_COMBINED || a.mode == FP_UGRADMU_NODE) {
      const int32_t* tri = a.nb + 3 * N + 3 * c;
      double nv[3];
      const int side = (a.teflag[c] & kTeLower) ? 1 : 0;   // a cell of both sides ends with the lower values
      const bool te_cell = a.sharpte && (a.teflag[c] & (kTeUpper | kTeLower));
      for (int k = 0; k < 3; ++k) {
        const int32_t t = te_cell ? a.teslot[tri[k]] : -1;
        nv[k] = t >= 0 ? a.nodal_te[side * a.nte + t] : a.nodal[tri[k]];
      }
      double g[3];
      tri_gradient(P, s * nv[0], s * nv[1], s * nv[2], g);
      for (int d = 0; d < 3; ++d) on[d] = -0.5 * g[d];
    }
    if (a.mode == FP_UGRADMU_COMBINED) {
      if (a.force_cellTE && (a.teflag[c] & kForcedCell))
        for (int d = 0; d < 3; ++d) on[d] = oc[d];
      bool use_node = false;
      for (int k = 0; k < 3 && !use_node; ++k) {
        if (nbk[k] < 0) { use_node = true; break; }
        const int64_t n = nbk[k];
        const double cosang = nc[0] * a.tgt[3 * N + n] + nc[1] * a.tgt[4 * N + n] + nc[2] * a.tgt[5 * N + n];
        if (cosang < a.cosang) use_node = true;
      }
      for (int d = 0; d < 3; ++d) res[d] = use_node ? on[d] : oc[d];
      if (a.out)
        for (int d = 0; d < 3; ++d) a.out[3 * c + d] += res[d];
    } else if (a.mode == FP_UGRADMU_CELL) {
      for (int d = 0; d < 3; ++d) res[d] = oc[d];
      if (a.out)
        for (int d = 0; d < 3; ++d) a.out[3 * c + d] = oc[d];
    } else {
      for (int d = 0; d < 3; ++d) res[d] = on[d];
      if (a.out)
        for (int d = 0; d < 3; ++d) a.out[3 * c + d] = on[d];
    }
    if (a.out_cell)
      for (int d = 0; d < 3; ++d) a.out_cell[3 * c + d] = oc[d];
    if (a.out_node)
      for (int d = 0; d < 3; ++d) a.out_node[3 * c + d] = on[d];
  }
  if (a.Cp) {
    // addfields("Ugradmu" -> "U"), calcfield_Cp! before its Kutta average,
    // calcfield_F! before its trailing-edge override
    double U[3];
    for (int d = 0; d < 3; ++d) U[d] = a.U[3 * c + d] + res[d];
    if (a.Utot)
      for (int d = 0; d < 3; ++d) a.Utot[3 * c + d] = U[d];
    const double q = sqrt(U[0] * U[0] + U[1] * U[1] + U[2] * U[2]) / a.Uref;
    const double cp = (a.Cp0 ? a.Cp0[c] : 0.0) + (1.0 - q * q);
    a.Cp[c] = cp;
    const double s = a.sgn[c];
    const double val = a.qneg * cp * a.area[c];
    for (int d = 0; d < 3; ++d) a.F[3 * c + d] = 0.0 + val * (a.tgt[(3 + d) * N + c] * s);
  }
}

// The trailing-edge nodes' nodal values from one side's cells only: the
// area-weighted mean over the upper (then the lower) cells that contain the
// node (GeometricTools' get_nodal_data_TEcells, restated in the weighting of
// k_nodal). csr: [up offsets][up cells][lo offsets][lo cells].
__global__ void __launch_bounds__(kPostThreads)
k_nodal_te(const int32_t* __restrict__ csr, int64_t nte, int64_t nup, const double* __restrict__ area,
           const double* __restrict__ g, double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * kPostThreads + threadIdx.x;
  if (i >= 2 * nte) return;
  const int side = (int)(i / nte);
  const int64_t t = i % nte;
  const int32_t* off = csr + (side ? (nte + 1 + nup) : 0);
  const int32_t* cells = off + nte + 1;
  double num = 0.0, den = 0.0;
  for (int32_t k = off[t]; k < off[t + 1]; ++k) {
    const int32_t c = cells[k];
    num += area[c] * g[c];
    den += area[c];
  }
  out[i] = den > 0.0 ? num / den : 0.0;
}

// smoothPass / smoothRows of the cell scheme (postprocess.jl:501-526): passes
// times, each listed cell in order takes the mean of its neighbours' current
// values (in place, so later cells see the earlier ones' new values); one
// thread, as the recurrence is sequential.
__global__ void k_smooth(const int32_t* __restrict__ nb, const int32_t* __restrict__ cells, int64_t ncells,
                         int passes, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int p = 0; p < passes; ++p)
    for (int64_t q = 0; q < ncells; ++q) {
      const int32_t c = cells[q];
      double acc[3] = {0.0, 0.0, 0.0};
      int cnt = 0;
      for (int k = 0; k < 3; ++k) {
        const int32_t n = nb[3 * c + k];
        if (n < 0) continue;
        ++cnt;
        for (int d = 0; d < 3; ++d) acc[d] += out[3 * n + d];
      }
      for (int d = 0; d < 3; ++d) out[3 * c + d] = acc[d] / cnt;
    }
}

// the cell scheme's maxgrad cut, after the smoothing
__global__ void __launch_bounds__(kPostThreads) k_maxgrad(double* __restrict__ out, int64_t N, double maxgrad) {
  const int64_t c = (int64_t)blockIdx.x * kPostThreads + threadIdx.x;
  if (c >= N) return;
  const double n = sqrt(out[3 * c] * out[3 * c] + out[3 * c + 1] * out[3 * c + 1] + out[3 * c + 2] * out[3 * c + 2]);
  if (n >= maxgrad) out[3 * c] = out[3 * c + 1] = out[3 * c + 2] = 0.0;
}

struct KuttaArgs {
  int64_t N, nsh, nk;
  const int32_t* krow;     // nsh x 4
  const int32_t* kcell;    // nk
  const int32_t* klast;    // nk
  double* kwork;           // nk doubles of global scratch when shared memory is too small
  double* Cp;              // N, Kutta-averaged in place when cp_kutta
  const double* Cpf;       // N, the Cp field the force override reads (may equal Cp)
  double* F;               // 3N
  const double* area;
  const double* tgt;
  const double* sgn;
  double q;                // 0.5 rho Uinf^2
  int cp_kutta, f_kutta, use_smem;
  double* lds;             // 9 (column-major L, D, S), or null
  const double* hats;      // 9: Lhat, Dhat, Shat
  const double* Fsum;      // 3N forces to sum (F, or the caller's)
};

__global__ void __launch_bounds__(kKuttaThreads) k_kutta_lds(KuttaArgs a) {
  extern __shared__ double sm[];
  double* kc = a.use_smem ? sm : a.kwork;
  int32_t* krow_s = a.use_smem ? reinterpret_cast<int32_t*>(sm + a.nk) : nullptr;
  const int32_t* krow = a.use_smem ? krow_s : a.krow;
  const int tid = threadIdx.x;
  if (a.nsh > 0 && (a.cp_kutta || a.f_kutta)) {
    const double* src = a.cp_kutta ? a.Cp : a.Cpf;
    for (int64_t i = tid; i < a.nk; i += kKuttaThreads) kc[i] = src[a.kcell[i]];
    if (a.use_smem)
      for (int64_t i = tid; i < 4 * a.nsh; i += kKuttaThreads) krow_s[i] = a.krow[i];
    __syncthreads();
    if (a.cp_kutta) {
      if (tid == 0) {
        // the reference's loop over the shedding rows, in order
        for (int64_t r = 0; r < a.nsh; ++r) {
          const int32_t* s = krow + 4 * r;
          if (s[2] >= 0) {
            const double ave = (kc[s[0]] + kc[s[1]] + kc[s[2]] + kc[s[3]]) / 4;
            kc[s[0]] = ave; kc[s[1]] = ave; kc[s[2]] = ave; kc[s[3]] = ave;
          } else {
            const double ave = (kc[s[0]] + kc[s[1]]) / 2;
            kc[s[0]] = ave; kc[s[1]] = ave;
          }
        }
      }
      __syncthreads();
      for (int64_t i = tid; i < a.nk; i += kKuttaThreads) a.Cp[a.kcell[i]] = kc[i];
    }
    if (a.f_kutta) {
      // rows read the (final) Cp field only, so they run in parallel; a cell
      // on several rows takes the value of the last one, as in the loop
      for (int64_t r = tid; r < a.nsh; r += kKuttaThreads) {
        const int32_t* s = krow + 4 * r;
        const int nslot = s[2] >= 0 ? 4 : 2;
        const double ave = nslot == 4 ? (kc[s[0]] + kc[s[1]] + kc[s[2]] + kc[s[3]]) / 4
                                      : (kc[s[0]] + kc[s[1]]) / 2;
        for (int j = 0; j < nslot; ++j) {
          if (a.klast[s[j]] != r) continue;
          const int64_t c = a.kcell[s[j]];
          const double sg = a.sgn[c];
          for (int d = 0; d < 3; ++d)
            a.F[3 * c + d] = -ave * a.q * a.area[c] * (a.tgt[(3 + d) * a.N + c] * sg);
        }
      }
    }
    __syncthreads();
  }
  if (!a.lds) return;
  // Ftot = sum of the forces, then the projections of calcfield_LDS!
  double f[3] = {0.0, 0.0, 0.0};
  for (int64_t c = tid; c < a.N; c += kKuttaThreads)
    for (int d = 0; d < 3; ++d) f[d] += a.Fsum[3 * c + d];
  __shared__ double red[3][kKuttaThreads / 32];
  for (int d = 0; d < 3; ++d) {
    double v = f[d];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) red[d][tid >> 5] = v;
  }
  __syncthreads();
  if (tid == 0) {
    double ft[3];
    for (int d = 0; d < 3; ++d) {
      double v = 0.0;
      for (int w = 0; w < kKuttaThreads / 32; ++w) v += red[d][w];
      ft[d] = a.lds[6 + d] + v;
    }
    for (int col = 0; col < 3; ++col) {
      const double* h = a.hats + 3 * col;
      const double dot = ft[0] * h[0] + ft[1] * h[1] + ft[2] * h[2];
      for (int d = 0; d < 3; ++d) a.lds[3 * col + d] = h[d] * dot;
    }
  }
}

int ensure_post(fp_ctx* c, size_t n) {
  if (n <= c->cap_post) return FP_OK;
  dfree(c->d_post);
  c->cap_post = 0;
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_post, n * sizeof(double)));
  c->cap_post = n;
  return FP_OK;
}

// Neighbours, node indices, cells around each node and areas of a
// triangular body.
int build_topology(fp_ctx* c) {
  if (c->topo_valid) return FP_OK;
  const int64_t N = c->N;
  const std::vector<int32_t>& off = c->h_offsets;
  const std::vector<int32_t>& pn = c->h_pnodes;
  const int64_t nn = (int64_t)c->h_nodes.size() / 3;
  for (int64_t p = 0; p < N; ++p)
    if (off[p + 1] - off[p] != 3)
      return c->err.set(FP_EINVAL, "fp_ugradmu: the grad(mu) schemes need triangular panels (panel " +
                                       std::to_string(p) + " has " + std::to_string(off[p + 1] - off[p]) +
                                       " nodes)");
  std::vector<int32_t> nbtri(6 * N, -1);
  for (int64_t p = 0; p < N; ++p)
    for (int k = 0; k < 3; ++k) nbtri[3 * N + 3 * p + k] = pn[off[p] + k];
  std::unordered_map<uint64_t, int64_t> edge;
  edge.reserve((size_t)(3 * N));
  for (int64_t p = 0; p < N; ++p)
    for (int k = 0; k < 3; ++k) {
      const uint32_t u = (uint32_t)pn[off[p] + k], v = (uint32_t)pn[off[p] + (k + 1) % 3];
      const uint64_t key = ((uint64_t)std::min(u, v) << 32) | std::max(u, v);
      auto it = edge.find(key);
      if (it == edge.end()) {
        edge.emplace(key, 3 * p + k);
      } else if (it->second < 0) {
        return c->err.set(FP_EINVAL, "fp_ugradmu: an edge of panel " + std::to_string(p) +
                                         " is shared by more than two panels");
      } else {
        const int64_t o = it->second;
        nbtri[o] = (int32_t)p;
        nbtri[3 * p + k] = (int32_t)(o / 3);
        it->second = -1;
      }
    }
  std::vector<int32_t> voff(nn + 1, 0), vcell(3 * N);
  for (int64_t p = 0; p < N; ++p)
    for (int k = 0; k < 3; ++k) ++voff[pn[off[p] + k] + 1];
  for (int64_t v = 0; v < nn; ++v) voff[v + 1] += voff[v];
  {
    std::vector<int32_t> fill(voff.begin(), voff.end() - 1);
    for (int64_t p = 0; p < N; ++p)
      for (int k = 0; k < 3; ++k) vcell[fill[pn[off[p] + k]]++] = (int32_t)p;
  }
  std::vector<double> area(N);
  const double* X = c->h_nodes.data();
  for (int64_t p = 0; p < N; ++p) {
    const double* p0 = X + 3 * (int64_t)pn[off[p]];
    const double* p1 = X + 3 * (int64_t)pn[off[p] + 1];
    const double* p2 = X + 3 * (int64_t)pn[off[p] + 2];
    const double e1 = p1[0] - p0[0], e2 = p1[1] - p0[1], e3 = p1[2] - p0[2];
    const double f1 = p2[0] - p0[0], f2 = p2[1] - p0[1], f3 = p2[2] - p0[2];
    const double c1 = e2 * f3 - e3 * f2, c2 = e3 * f1 - e1 * f3, c3 = e1 * f2 - e2 * f1;
    area[p] = 0.5 * std::sqrt(c1 * c1 + c2 * c2 + c3 * c3);
  }
  dfree(c->d_nb); dfree(c->d_voff); dfree(c->d_vcell); dfree(c->d_area);
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_nb, 6 * N * sizeof(int32_t)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_voff, (nn + 1) * sizeof(int32_t)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_vcell, 3 * N * sizeof(int32_t)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_area, N * sizeof(double)));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_nb, nbtri.data(), 6 * N * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_voff, voff.data(), (nn + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_vcell, vcell.data(), 3 * N * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_area, area.data(), N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  c->topo_nnodes = nn;
  c->topo_valid = true;
  return FP_OK;
}

// Areas of any body (fan of triangles from the first node), for the loads
// of bodies that are not triangulated.
int build_areas(fp_ctx* c) {
  if (c->topo_valid) return FP_OK;
  const int64_t N = c->N;
  std::vector<double> area(N, 0.0);
  const double* X = c->h_nodes.data();
  for (int64_t p = 0; p < N; ++p) {
    const int32_t* pn = c->h_pnodes.data() + c->h_offsets[p];
    const int nv = c->h_offsets[p + 1] - c->h_offsets[p];
    const double* p0 = X + 3 * (int64_t)pn[0];
    double a = 0.0;
    for (int k = 1; k + 1 < nv; ++k) {
      const double* p1 = X + 3 * (int64_t)pn[k];
      const double* p2 = X + 3 * (int64_t)pn[k + 1];
      const double e1 = p1[0] - p0[0], e2 = p1[1] - p0[1], e3 = p1[2] - p0[2];
      const double f1 = p2[0] - p0[0], f2 = p2[1] - p0[1], f3 = p2[2] - p0[2];
      const double c1 = e2 * f3 - e3 * f2, c2 = e3 * f1 - e1 * f3, c3 = e1 * f2 - e2 * f1;
      a += 0.5 * std::sqrt(c1 * c1 + c2 * c2 + c3 * c3);
    }
    area[p] = a;
  }
  dfree(c->d_area);
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_area, N * sizeof(double)));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_area, area.data(), N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

// Trailing-edge tables from the shedding rows: the times each cell is pi or
// pj and the forced cells (for the schemes), the Kutta rows as slots of the
// distinct cells they touch and the last row that writes each cell's force.
int build_kutta(fp_ctx* c) {
  if (c->kutta_valid) return FP_OK;
  const int64_t N = c->N, nsh = c->nsh;
  std::vector<int32_t> te(N, 0), krow(4 * std::max<int64_t>(nsh, 1), -1), slot(N, -1), kcell, klast;
  for (int64_t r = 0; r < nsh; ++r) {
    const int32_t* s = c->h_shed.data() + 6 * r;
    const int32_t pi = s[0], pj = s[3];
    if (pi + 1 >= N || (pj != -1 && pj < 1))
      return c->err.set(FP_EINVAL, "shedding row " + std::to_string(r) +
                                       ": the Kutta average needs panels pi+1 and pj-1 to exist");
    // the low 16 bits count the rows a cell is pi or pj of; bit 16 (forced
    // cell value) may already be set by another row's pi+1 or pj-1
    auto bump = [&](int32_t p) {
      if ((te[p] & 0xffff) == 0xffff) return false;
      ++te[p];
      return true;
    };
    if (!bump(pi) || (pj >= 0 && !bump(pj)))
      return c->err.set(FP_EINVAL, "fp_ugradmu: a panel appears in too many shedding rows");
    const int32_t cells[4] = {pi, pi + 1, pj, pj - 1};
    const int ncell = pj != -1 ? 4 : 2;
    for (int j = 0; j < ncell; ++j) {
      const int32_t cc = cells[j];
      te[cc] |= kForcedCell;
      if (slot[cc] < 0) {
        slot[cc] = (int32_t)kcell.size();
        kcell.push_back(cc);
        klast.push_back(0);
      }
      krow[4 * r + j] = slot[cc];
      klast[slot[cc]] = (int32_t)r;
    }
  }
  // sharp trailing edge: the upper cells pi, pi+1 and lower cells pj, pj-1,
  // the TE nodes (the upper edge's nodes) and, per TE node, the cells of
  // each side that contain it
  const int64_t nnodes = (int64_t)c->h_nodes.size() / 3;
  std::vector<int32_t> up, lo, tenodes, teslot(nnodes, -1);
  for (int64_t r = 0; r < nsh; ++r) {
    const int32_t* s = c->h_shed.data() + 6 * r;
    const int32_t pi = s[0], pj = s[3];
    for (int32_t cc : {pi, pi + 1})
      if (cc >= 0 && cc < N && !(te[cc] & kTeUpper)) { te[cc] |= kTeUpper; up.push_back(cc); }
    if (pj != -1)
      for (int32_t cc : {pj, pj - 1})
        if (cc >= 0 && cc < N && !(te[cc] & kTeLower)) { te[cc] |= kTeLower; lo.push_back(cc); }
    for (int k : {s[1], s[2]}) {
      const int32_t v = c->h_pnodes[c->h_offsets[pi] + k];
      if (v >= 0 && v < nnodes && teslot[v] < 0) {
        teslot[v] = (int32_t)tenodes.size();
        tenodes.push_back(v);
      }
    }
  }
  const int64_t nte = (int64_t)tenodes.size();
  std::vector<int32_t> csr;
  int64_t nup = 0;
  for (const std::vector<int32_t>* side : {&up, &lo}) {
    std::vector<std::vector<int32_t>> lists(nte);
    for (int32_t cc : *side)
      for (int k = c->h_offsets[cc]; k < c->h_offsets[cc + 1]; ++k) {
        const int32_t t = teslot[c->h_pnodes[k]];
        if (t >= 0) lists[t].push_back(cc);
      }
    const size_t base = csr.size();
    csr.resize(base + nte + 1);
    csr[base] = 0;
    for (int64_t t = 0; t < nte; ++t) csr[base + t + 1] = csr[base + t] + (int32_t)lists[t].size();
    for (int64_t t = 0; t < nte; ++t) csr.insert(csr.end(), lists[t].begin(), lists[t].end());
    if (side == &up) nup = csr[base + nte];
  }
  dfree(c->d_teslot); dfree(c->d_tecsr);
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_teslot, std::max<int64_t>(nnodes, 1) * sizeof(int32_t)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_tecsr, csr.size() * sizeof(int32_t)));
  if (nnodes > 0)
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_teslot, teslot.data(), nnodes * sizeof(int32_t), cudaMemcpyHostToDevice,
                                        c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_tecsr, csr.data(), csr.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                      c->stream));
  c->nte = nte;
  c->te_up_cells = nup;
  const int64_t nk = (int64_t)kcell.size();
  dfree(c->d_teflag); dfree(c->d_krow); dfree(c->d_kcell); dfree(c->d_klast);
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_teflag, N * sizeof(int32_t)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_krow, krow.size() * sizeof(int32_t)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_kcell, std::max<int64_t>(nk, 1) * sizeof(int32_t)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_klast, std::max<int64_t>(nk, 1) * sizeof(int32_t)));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_teflag, te.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_krow, krow.data(), krow.size() * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  if (nk > 0) {
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_kcell, kcell.data(), nk * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_klast, klast.data(), nk * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  }
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  c->nkcell = nk;
  c->kutta_valid = true;
  return FP_OK;
}

unsigned grid_of(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// sign(CPoffset) per cell (1 where it is 0 or not given)
void signs_of(const double* cp_offset, int64_t N, std::vector<double>& s) {
  s.assign(N, 1.0);
  if (cp_offset)
    for (int64_t i = 0; i < N; ++i) s[i] = cp_offset[i] < 0 ? -1.0 : 1.0;
}

// The scheme on device data: d_g strengths, d_sgn signs; writes the fields
// selected in `a` (out, out_cell, out_node and/or the fused loads).
int launch_scheme(fp_ctx* c, PostArgs& a, double* d_nodal) {
  if (a.mode == FP_UGRADMU_COMBINED || a.mode == FP_UGRADMU_NODE) {
    k_nodal<<<grid_of(c->topo_nnodes, kPostThreads), kPostThreads, 0, c->stream>>>(
        c->d_voff, c->d_vcell, c->d_area, a.g, c->topo_nnodes, d_nodal);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
  }
  a.nodal = d_nodal;
  k_ugradmu<<<grid_of(c->N, kPostThreads), kPostThreads, 0, c->stream>>>(a);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

int launch_kutta(fp_ctx* c, KuttaArgs& k, double* d_kwork) {
  const size_t smem = (size_t)c->nkcell * sizeof(double) + 4 * (size_t)c->nsh * sizeof(int32_t);
  k.use_smem = smem <= kKuttaSmemMax;
  k.kwork = d_kwork;
  k.nk = c->nkcell;
  k.krow = c->d_krow;
  k.kcell = c->d_kcell;
  k.klast = c->d_klast;
  k_kutta_lds<<<1, kKuttaThreads, k.use_smem ? smem : 0, c->stream>>>(k);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

// calcfield_F!'s panel loop on a given Cp field: F += ((-0.5 rho Uinf^2) Cp A) n,
// n flipped by sign(CPoffset)
__global__ void __launch_bounds__(kPostThreads)
k_panel_forces(const double* __restrict__ Cp, const double* __restrict__ sgn, const double* __restrict__ area,
               const double* __restrict__ tgt, int64_t N, double qneg, double* __restrict__ F) {
  const int64_t c = (int64_t)blockIdx.x * kPostThreads + threadIdx.x;
  if (c >= N) return;
  const double val = qneg * Cp[c] * area[c];
  const double s = sgn[c];
  for (int d = 0; d < 3; ++d) F[3 * c + d] += val * (tgt[(3 + d) * N + c] * s);
}

int launch_panel_forces(fp_ctx* c, const double* d_cp, const double* d_sgn, double qneg, double* d_F) {
  k_panel_forces<<<grid_of(c->N, kPostThreads), kPostThreads, 0, c->stream>>>(d_cp, d_sgn, c->d_area, c->d_tgt,
                                                                               c->N, qneg, d_F);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

int ev_begin(fp_ctx* c) {
  FP_CUDA_TRY(c->err, cudaEventRecord(c->ev0, c->stream));
  return FP_OK;
}

int ev_end(fp_ctx* c, double* ms) {
  FP_CUDA_TRY(c->err, cudaEventRecord(c->ev1, c->stream));
  FP_CUDA_TRY(c->err, cudaEventSynchronize(c->ev1));
  float f = 0.f;
  FP_CUDA_TRY(c->err, cudaEventElapsedTime(&f, c->ev0, c->ev1));
  *ms = f;
  return FP_OK;
}

bool unit(const double* v) {
  return std::fabs(std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - 1) <= 2 * 2.220446049250313e-16;
}

}  // namespace

void post_free(fp_ctx* c) {
  dfree(c->d_nb); dfree(c->d_voff); dfree(c->d_vcell); dfree(c->d_area);
  dfree(c->d_teflag); dfree(c->d_krow); dfree(c->d_kcell); dfree(c->d_klast);
  dfree(c->d_teslot); dfree(c->d_tecsr);
  dfree(c->d_post);
  c->cap_post = 0;
  dfree(c->d_uscr);
  c->cap_uscr = 0;
  c->topo_valid = c->kutta_valid = false;
}

}  // namespace fpb

using namespace fpb;

int fp_ugradmu(fp_ctx* c, int scheme, const double* strength, const double* cp_offset, double anglecrit,
               int force_cellTE, double maxgrad, double* out, double* out_cell, double* out_node) {
  return fp_ugradmu_ex(c, scheme, strength, cp_offset, anglecrit, force_cellTE, maxgrad, 0, nullptr, 0, 0, out,
                       out_cell, out_node);
}

int fp_ugradmu_ex(fp_ctx* c, int scheme, const double* strength, const double* cp_offset, double anglecrit,
                  int force_cellTE, double maxgrad, int sharpTE, const int32_t* smooth_cells, int64_t nsmooth,
                  int smooth_pass, double* out, double* out_cell, double* out_node) {
  if (!c) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_ugradmu: no geometry");
  if (scheme < FP_UGRADMU_COMBINED || scheme > FP_UGRADMU_NODE || !strength || !out)
    return c->err.set(FP_EINVAL, "fp_ugradmu: bad arguments");
  if (scheme != FP_UGRADMU_COMBINED && (out_cell || out_node))
    return c->err.set(FP_EINVAL, "fp_ugradmu: out_cell/out_node belong to the combined scheme");
  if (nsmooth < 0 || smooth_pass < 0 || (nsmooth > 0 && !smooth_cells))
    return c->err.set(FP_EINVAL, "fp_ugradmu: bad smoothing arguments");
  for (int64_t q = 0; q < nsmooth; ++q)
    if (smooth_cells[q] < 0 || smooth_cells[q] >= c->N)
      return c->err.set(FP_EINVAL, "fp_ugradmu: smoothing cell index out of range");
  const bool smooth = scheme == FP_UGRADMU_CELL && nsmooth > 0 && smooth_pass > 0;
  int rc;
  if ((rc = build_topology(c)) || (rc = build_kutta(c))) return rc;
  const int64_t N = c->N, nn = c->topo_nnodes;
  const int64_t nte = c->nte;
  if ((rc = ensure_post(c, (size_t)(2 * N + nn + 9 * N + 2 * nte + (nsmooth + 1) / 2 + 1)))) return rc;
  double* d_g = c->d_post;
  double* d_sgn = d_g + N;
  double* d_nodal = d_sgn + N;
  double* d_out = d_nodal + nn;
  double* d_oc = d_out + 3 * N;
  double* d_on = d_oc + 3 * N;
  double* d_nte = d_on + 3 * N;
  int32_t* d_smooth = reinterpret_cast<int32_t*>(d_nte + 2 * nte);
  std::vector<double> sg;
  signs_of(cp_offset, N, sg);
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_g, strength, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_sgn, sg.data(), N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_out, out, 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  PostArgs a{};
  a.panels = c->d_panels; a.tgt = c->d_tgt; a.N = N; a.area = c->d_area; a.nb = c->d_nb;
  a.teflag = c->d_teflag; a.sgn = d_sgn; a.g = d_g; a.mode = scheme; a.force_cellTE = force_cellTE;
  // cosd(anglecrit) with the degree-to-radian factor applied first
  a.cosang = std::cos(anglecrit * (M_PI / 180.0));
  a.maxgrad = smooth ? INFINITY : maxgrad;   // with smoothing, the cut follows it
  a.out = d_out;
  a.out_cell = out_cell ? d_oc : nullptr;
  a.out_node = out_node ? d_on : nullptr;
  a.sharpte = sharpTE && nte > 0 && scheme != FP_UGRADMU_CELL;
  a.teslot = c->d_teslot;
  a.nodal_te = d_nte;
  a.nte = nte;
  if (smooth)
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_smooth, smooth_cells, nsmooth * sizeof(int32_t), cudaMemcpyHostToDevice,
                                        c->stream));
  if (ev_begin(c)) return FP_ECUDA;
  if (a.sharpte) {
    k_nodal_te<<<grid_of(2 * nte, kPostThreads), kPostThreads, 0, c->stream>>>(c->d_tecsr, nte, c->te_up_cells,
                                                                                c->d_area, d_g, d_nte);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
  }
  if ((rc = launch_scheme(c, a, d_nodal))) return rc;
  if (smooth) {
    k_smooth<<<1, 32, 0, c->stream>>>(c->d_nb, d_smooth, nsmooth, smooth_pass, d_out);
    ++c->nlaunch;
    if (std::isfinite(maxgrad)) {
      k_maxgrad<<<grid_of(N, kPostThreads), kPostThreads, 0, c->stream>>>(d_out, N, maxgrad);
      ++c->nlaunch;
    }
    FP_CUDA_TRY(c->err, cudaGetLastError());
  }
  double ms = 0;
  if (ev_end(c, &ms)) return FP_ECUDA;
  c->kms[FP_STAGE_POST] = ms;
  c->klaunch[FP_STAGE_POST] = scheme == FP_UGRADMU_CELL ? 1 : 2;
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(out, d_out, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (out_cell)
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(out_cell, d_oc, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (out_node)
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(out_node, d_on, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

int fp_calcfield_cp(fp_ctx* c, const double* Us, double Uref, int correct_kutta, double* out) {
  if (!c) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_calcfield_cp: no geometry");
  if (!Us || !out) return c->err.set(FP_EINVAL, "fp_calcfield_cp: bad arguments");
  int rc;
  if ((rc = build_kutta(c)) || (rc = c->topo_valid ? FP_OK : build_areas(c))) return rc;
  const int64_t N = c->N;
  if ((rc = ensure_post(c, (size_t)(N + 3 * N + N + 3 * N + c->nkcell + 1)))) return rc;
  double* d_sgn = c->d_post;
  double* d_U = d_sgn + N;
  double* d_cp = d_U + 3 * N;
  double* d_F = d_cp + N;
  double* d_kw = d_F + 3 * N;
  std::vector<double> sg(N, 1.0);
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_sgn, sg.data(), N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_U, Us, 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_cp, out, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  PostArgs a{};
  a.panels = c->d_panels; a.tgt = c->d_tgt; a.N = N; a.area = c->d_area; a.sgn = d_sgn; a.mode = -1;
  a.U = d_U; a.Uref = Uref; a.Cp0 = d_cp; a.qneg = 0.0; a.Cp = d_cp; a.F = d_F;
  if ((rc = launch_scheme(c, a, nullptr))) return rc;
  if (correct_kutta && c->nsh > 0) {
    KuttaArgs k{};
    k.N = N; k.nsh = c->nsh; k.Cp = d_cp; k.Cpf = d_cp; k.cp_kutta = 1; k.f_kutta = 0;
    if ((rc = launch_kutta(c, k, d_kw))) return rc;
  }
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(out, d_cp, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

int fp_calcfield_f(fp_ctx* c, const double* Cps, const double* cp_offset, double Uinf, double rho,
                   int correct_kutta, double* out) {
  if (!c) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_calcfield_f: no geometry");
  if (!Cps || !out) return c->err.set(FP_EINVAL, "fp_calcfield_f: bad arguments");
  int rc;
  if ((rc = build_kutta(c)) || (rc = c->topo_valid ? FP_OK : build_areas(c))) return rc;
  const int64_t N = c->N;
  if ((rc = ensure_post(c, (size_t)(N + N + 3 * N + c->nkcell + 1)))) return rc;
  double* d_sgn = c->d_post;
  double* d_cp = d_sgn + N;
  double* d_F = d_cp + N;
  double* d_kw = d_F + 3 * N;
  std::vector<double> sg;
  signs_of(cp_offset, N, sg);
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_sgn, sg.data(), N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_cp, Cps, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_F, out, 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if ((rc = launch_panel_forces(c, d_cp, d_sgn, -0.5 * rho * (Uinf * Uinf), d_F))) return rc;
  if (correct_kutta && c->nsh > 0) {
    KuttaArgs k{};
    k.N = N; k.nsh = c->nsh; k.Cp = d_cp; k.Cpf = d_cp; k.F = d_F; k.area = c->d_area;
    k.tgt = c->d_tgt; k.sgn = d_sgn; k.q = 0.5 * rho * (Uinf * Uinf); k.cp_kutta = 0; k.f_kutta = 1;
    if ((rc = launch_kutta(c, k, d_kw))) return rc;
  }
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(out, d_F, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

int fp_calcfield_lds(fp_ctx* c, const double* Fs, const double* Lhat, const double* Dhat, const double* Shat,
                     double* out) {
  if (!c) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_calcfield_lds: no geometry");
  if (!Fs || !Lhat || !Dhat || !Shat || !out) return c->err.set(FP_EINVAL, "fp_calcfield_lds: bad arguments");
  if (!unit(Lhat)) return c->err.set(FP_EINVAL, "Lhat is not a unitary vector");
  if (!unit(Dhat)) return c->err.set(FP_EINVAL, "Dhat is not a unitary vector");
  if (!unit(Shat)) return c->err.set(FP_EINVAL, "Shat is not a unitary vector");
  int rc;
  const int64_t N = c->N;
  if ((rc = ensure_post(c, (size_t)(3 * N + 18)))) return rc;
  double* d_F = c->d_post;
  double* d_lds = d_F + 3 * N;
  double* d_hats = d_lds + 9;
  double hats[9] = {Lhat[0], Lhat[1], Lhat[2], Dhat[0], Dhat[1], Dhat[2], Shat[0], Shat[1], Shat[2]};
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_F, Fs, 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_lds, out, 9 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_hats, hats, 9 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  KuttaArgs k{};
  k.N = N; k.nsh = 0; k.lds = d_lds; k.hats = d_hats; k.Fsum = d_F;
  k_kutta_lds<<<1, kKuttaThreads, 0, c->stream>>>(k);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(out, d_lds, 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

int fp_surface_loads(fp_ctx* c, int element, const double* strengths, const double* Uinfs,
                     const double* cp_offset, double kerneloffset, double kernelcutoff, int ugradmu,
                     double Uref, double rho, const double* Lhat, const double* Dhat, const double* Shat,
                     int correct_kutta, double* U, double* Cp, double* F, double* LDS) {
  if (!c) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_surface_loads: no geometry");
  if (!strengths || !Uinfs || !Lhat || !Dhat || !Shat || !Cp || !F || !LDS ||
      element < FP_ELEMENT_SOURCE || element > FP_ELEMENT_SOURCE_DOUBLET || Uref == 0.0)
    return c->err.set(FP_EINVAL, "fp_surface_loads: bad arguments");
  if (!unit(Lhat)) return c->err.set(FP_EINVAL, "Lhat is not a unitary vector");
  if (!unit(Dhat)) return c->err.set(FP_EINVAL, "Dhat is not a unitary vector");
  if (!unit(Shat)) return c->err.set(FP_EINVAL, "Shat is not a unitary vector");
  if (ugradmu && element == FP_ELEMENT_SOURCE)
    return c->err.set(FP_EINVAL, "fp_surface_loads: a source body has no doublet strength for grad(mu)");
  int rc;
  if (ugradmu) {
    if ((rc = build_topology(c))) return rc;
  } else if (!c->topo_valid && (rc = build_areas(c))) {
    return rc;
  }
  if ((rc = build_kutta(c))) return rc;
  const int64_t N = c->N, nn = ugradmu ? c->topo_nnodes : 0;
  const int64_t ns = element == FP_ELEMENT_SOURCE_DOUBLET ? 2 * N : N;
  // work: strengths, signs, control points (AoS), U, U total, Cp, F, nodal, Kutta scratch, L/D/S
  const size_t need = (size_t)(ns + N + 3 * N + 3 * N + 3 * N + N + 3 * N + nn + c->nkcell + 18);
  if ((rc = ensure_post(c, need))) return rc;
  double* d_s = c->d_post;
  double* d_sgn = d_s + ns;
  double* d_cps = d_sgn + N;
  double* d_U = d_cps + 3 * N;
  double* d_Ut = d_U + 3 * N;
  double* d_cp = d_Ut + 3 * N;
  double* d_F = d_cp + N;
  double* d_nodal = d_F + 3 * N;
  double* d_kw = d_nodal + nn;
  double* d_lds = d_kw + c->nkcell;
  double* d_hats = d_lds + 9;
  std::vector<double> sg, cps(3 * N);
  signs_of(cp_offset, N, sg);
  for (int64_t i = 0; i < N; ++i)
    for (int d = 0; d < 3; ++d) cps[3 * i + d] = c->h_tgt[d * N + i];
  const double zero9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double hats[9] = {Lhat[0], Lhat[1], Lhat[2], Dhat[0], Dhat[1], Dhat[2], Shat[0], Shat[1], Shat[2]};
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_s, strengths, ns * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_sgn, sg.data(), N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_cps, cps.data(), 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_U, Uinfs, 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_lds, zero9, 9 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(d_hats, hats, 9 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  c->kern_offset = kerneloffset;
  c->kern_cutoff = kernelcutoff;
  const int64_t launches0 = c->nlaunch;
  if (ev_begin(c)) return FP_ECUDA;
  // calcfield_U: U = Uinf + Uind at the control points (postprocess.jl:28-110)
  if (element == FP_ELEMENT_VORTEXRING) {
    rc = launch_uind_ring(c, d_s, d_cps, N, d_U, false);
  } else if (element == FP_ELEMENT_SOURCE_DOUBLET) {
    const int64_t nsh = c->nsh;
    c->nsh = 0;
    rc = launch_uind_source(c, d_s, d_cps, N, d_U);
    if (!rc) rc = launch_uind_ring(c, d_s + N, d_cps, N, d_U, false);
    c->nsh = nsh;
  } else {
    rc = launch_uind_source(c, d_s, d_cps, N, d_U);
  }
  if (rc) return rc;
  // grad(mu) (doublet strengths: the ring strengths, or the second column)
  PostArgs a{};
  a.panels = c->d_panels; a.tgt = c->d_tgt; a.N = N; a.area = c->d_area; a.nb = c->d_nb;
  a.teflag = c->d_teflag; a.sgn = d_sgn;
  a.g = element == FP_ELEMENT_SOURCE_DOUBLET ? d_s + N : d_s;
  a.mode = ugradmu ? FP_UGRADMU_COMBINED : -1;
  a.force_cellTE = 1;
  a.cosang = std::cos(30.0 * (M_PI / 180.0));
  a.maxgrad = INFINITY;
  a.U = d_U; a.Uref = Uref; a.qneg = -0.5 * rho * (Uref * Uref); a.Utot = d_Ut; a.Cp = d_cp; a.F = d_F;
  if ((rc = launch_scheme(c, a, d_nodal))) return rc;
  KuttaArgs k{};
  k.N = N; k.nsh = correct_kutta ? c->nsh : 0; k.Cp = d_cp; k.Cpf = d_cp; k.F = d_F; k.area = c->d_area;
  k.tgt = c->d_tgt; k.sgn = d_sgn; k.q = 0.5 * rho * (Uref * Uref); k.cp_kutta = 1; k.f_kutta = 1;
  k.lds = d_lds; k.hats = d_hats; k.Fsum = d_F;
  if ((rc = launch_kutta(c, k, d_kw))) return rc;
  double ms = 0;
  if (ev_end(c, &ms)) return FP_ECUDA;
  c->kms[FP_STAGE_POST] = ms;
  c->klaunch[FP_STAGE_POST] = (int)(c->nlaunch - launches0);
  if (U) FP_CUDA_TRY(c->err, cudaMemcpyAsync(U, d_Ut, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(Cp, d_cp, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(F, d_F, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(LDS, d_lds, 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}
