// C ABI of the B200 panel-method library: context, geometry, orchestration.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fp_internal.cuh"

using namespace fpb;

namespace fpb {
int num_sms() {   // of the current device, cached per device
  static std::atomic<int> cache[64];
  int dev = 0;
  cudaGetDevice(&dev);
  std::atomic<int>& slot = cache[dev & 63];
  int sms = slot.load(std::memory_order_relaxed);
  if (sms <= 0) {
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
    slot.store(sms, std::memory_order_relaxed);
  }
  return sms;
}

// Device staging buffer of at least n doubles, kept across calls (no
// allocation in the steady state of repeated solves / field evaluations).
int ensure_stage(fp_ctx* c, size_t n) {
  if (n <= c->cap_stage) return FP_OK;
  if (c->d_stage) cudaFree(c->d_stage);
  c->d_stage = nullptr;
  c->cap_stage = 0;
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_stage, n * sizeof(double)));
  c->cap_stage = n;
  return FP_OK;
}
}  // namespace fpb

namespace {

template <class T> void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

int check_ctx(fp_ctx* c) { return c ? FP_OK : FP_EINVAL; }

// Device status bits -> FP_* status (and reset the word).
int consume_status(fp_ctx* c) {
  int st = 0;
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  if (st) {
    FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
    if (st & DEV_TIMEOUT) return c->err.set(FP_ETIMEOUT, "a bounded device-side wait ran out");
    if (st & DEV_ZERO_PIVOT) return c->err.set(FP_ESINGULAR, "zero pivot in the LU factorisation");
  }
  return FP_OK;
}

// Panel unit vectors of docs/src/elements/paneldefinition.md:15-35.
void frame(const double* nodes, const int32_t* pn, double t[3], double o[3], double n[3]) {
  const double* a = nodes + 3 * (int64_t)pn[0];
  const double* b = nodes + 3 * (int64_t)pn[1];
  const double* c = nodes + 3 * (int64_t)pn[2];
  double e[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double f[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double ne = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
  for (int k = 0; k < 3; ++k) t[k] = e[k] / ne;
  double cr[3] = {e[1] * f[2] - e[2] * f[1], e[2] * f[0] - e[0] * f[2], e[0] * f[1] - e[1] * f[0]};
  double nc = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  for (int k = 0; k < 3; ++k) n[k] = cr[k] / nc;
  o[0] = n[1] * t[2] - n[2] * t[1];
  o[1] = n[2] * t[0] - n[0] * t[2];
  o[2] = n[0] * t[1] - n[1] * t[0];
}

int ensure_rhs(fp_ctx* c, int64_t k) {
  if (k <= c->cap_rhs) return FP_OK;
  dfree(c->d_rhs); dfree(c->d_x); dfree(c->d_r); dfree(c->d_w32); dfree(c->d_norms);
  const size_t n = (size_t)c->ld * k;
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_rhs, n * sizeof(double)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_x, n * sizeof(double)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_r, n * sizeof(double)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_w32, n * sizeof(float)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_norms, 2 * k * sizeof(double)));
  c->cap_rhs = k;
  return FP_OK;
}


int time_begin(fp_ctx* c) {
  FP_CUDA_TRY(c->err, cudaEventRecord(c->ev0, c->stream));
  return FP_OK;
}
int time_end(fp_ctx* c, double* ms) {
  FP_CUDA_TRY(c->err, cudaEventRecord(c->ev1, c->stream));
  FP_CUDA_TRY(c->err, cudaEventSynchronize(c->ev1));
  float f = 0.f;
  FP_CUDA_TRY(c->err, cudaEventElapsedTime(&f, c->ev0, c->ev1));
  *ms = f;
  return FP_OK;
}

void free_matrices(fp_ctx* c) {
  if (c->stream_bg) cudaStreamSynchronize(c->stream_bg);   // a background pass may still write G
  c->g64_pending = false;
  dfree(c->d_G); dfree(c->d_LU); dfree(c->d_G32); dfree(c->d_ipiv);
  dfree(c->d_dinv64); dfree(c->d_dinv32); dfree(c->d_flags); dfree(c->d_mbox); dfree(c->d_part);
  dfree(c->d_dinv128_64); dfree(c->d_dinv128_32); dfree(c->d_mprev64); dfree(c->d_mprev32);
  dfree(c->d_mq32); dfree(c->d_ms32); dfree(c->d_zbox);
  c->trs2_ready = false;
  if (c->d_minv) { cudaFree(c->d_minv); c->d_minv = nullptr; }
  dfree(c->d_rhs); dfree(c->d_x); dfree(c->d_r); dfree(c->d_w32); dfree(c->d_norms);
  dfree(c->d_V); dfree(c->d_h);
  dfree(c->d_ab); dfree(c->d_ax); dfree(c->d_ar); dfree(c->d_aw32); dfree(c->d_anorms);
  c->cap_adj = 0;
  dfree(c->d_vjp);
  c->cap_vjp = 0;
  dfree(c->d_stage);
  c->cap_stage = 0;
  for (int s = 0; s < 2; ++s) {
    for (int i = 0; i < 4; ++i) dfree(c->d_tc[s][i]);
    c->tc_cap[s] = 0;
  }
  c->cap_rhs = 0; c->cap_gmres_m = 0;
  c->assembled = -1; c->factored = -1; c->nrhs = 0;
  if (c->lu_graph) cudaGraphExecDestroy(c->lu_graph);
  c->lu_graph = nullptr;
  c->lu_graph_key.clear();
  c->lu_graph_seen.clear();
}

}  // namespace

extern "C" {

int fp_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int fp_ctx_create(int device, fp_ctx** out) {
  if (!out) return FP_EINVAL;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return FP_ECUDA;
  if (device < 0 || device >= n) return FP_EINVAL;
  fp_ctx* c = new fp_ctx();
  c->device = device;
  // the context's stream carries the factorisation's critical path (panels):
  // give it the highest priority; stream2 (the bulk trailing update) the lowest
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->stream2, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->stream3, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->stream4, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_top, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_u12r, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_pinv, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_u12n, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_tcr, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_l21t, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->stream_bg, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_g64, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_diag, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_asm, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_panel, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_rest, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess || cudaMalloc(&c->d_cert, sizeof(float)) != cudaSuccess ||
      cudaMalloc(&c->d_ticket, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(c->d_status, 0, sizeof(int)) != cudaSuccess || cudaMemset(c->d_ticket, 0, sizeof(unsigned)) != cudaSuccess) {
    delete c;
    return FP_ECUDA;
  }
  *out = c;
  return FP_OK;
}

int fp_ctx_destroy(fp_ctx* c) {
  if (!c) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->stream2) cudaStreamSynchronize(c->stream2);
  if (c->stream3) cudaStreamSynchronize(c->stream3);
  if (c->stream4) cudaStreamSynchronize(c->stream4);
  if (c->stream_bg) cudaStreamSynchronize(c->stream_bg);
  free_matrices(c);
  post_free(c);
  dfree(c->d_panels); dfree(c->d_src); dfree(c->d_tgt); dfree(c->d_wake);
  dfree(c->d_status); dfree(c->d_cert); dfree(c->d_ticket);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (cudaEvent_t e : c->ktimer.pool) cudaEventDestroy(e);
  for (cudaEvent_t e : c->trace.pool) cudaEventDestroy(e);
  if (c->ev_panel) cudaEventDestroy(c->ev_panel);
  if (c->ev_rest) cudaEventDestroy(c->ev_rest);
  if (c->ev_g64) cudaEventDestroy(c->ev_g64);
  if (c->ev_diag) cudaEventDestroy(c->ev_diag);
  if (c->ev_asm) cudaEventDestroy(c->ev_asm);
  if (c->ev_pinv) cudaEventDestroy(c->ev_pinv);
  if (c->ev_u12n) cudaEventDestroy(c->ev_u12n);
  if (c->ev_tcr) cudaEventDestroy(c->ev_tcr);
  if (c->ev_l21t) cudaEventDestroy(c->ev_l21t);
  if (c->ev_top) cudaEventDestroy(c->ev_top);
  if (c->ev_u12r) cudaEventDestroy(c->ev_u12r);
  if (c->stream4) cudaStreamDestroy(c->stream4);
  if (c->stream3) cudaStreamDestroy(c->stream3);
  if (c->stream_bg) cudaStreamDestroy(c->stream_bg);
  if (c->stream2) cudaStreamDestroy(c->stream2);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return FP_OK;
}

const char* fp_last_error(const fp_ctx* c) { return c ? c->err.msg.c_str() : "null context"; }

int fp_set_geometry(fp_ctx* c, const double* nodes, int64_t nnodes, const int32_t* offsets,
                    const int32_t* pnodes, int64_t npanels, const double* cps,
                    const double* normals, const double* cp_offset) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (!nodes || !offsets || !pnodes || nnodes <= 0 || npanels <= 0)
    return c->err.set(FP_EINVAL, "fp_set_geometry: empty mesh or null pointer");
  // a background assembly pass may still read the panels it may free
  if (c->g64_pending) {
    FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream_bg));
    c->g64_pending = false;
  }
  if (offsets[0] != 0) return c->err.set(FP_EINVAL, "fp_set_geometry: panel_offsets[0] must be 0");
  for (int64_t p = 0; p < npanels; ++p) {
    const int nn = offsets[p + 1] - offsets[p];
    if (nn < 3 || nn > 4)
      return c->err.set(FP_EINVAL, "fp_set_geometry: panel " + std::to_string(p) + " has " +
                                       std::to_string(nn) + " nodes (3 or 4 supported)");
    for (int k = 0; k < nn; ++k) {
      const int32_t ni = pnodes[offsets[p] + k];
      if (ni < 0 || ni >= nnodes)
        return c->err.set(FP_EINVAL, "fp_set_geometry: node index out of range in panel " + std::to_string(p));
    }
  }
  for (int64_t i = 0; i < 3 * nnodes; ++i)
    if (!std::isfinite(nodes[i])) return c->err.set(FP_EINVAL, "fp_set_geometry: non-finite node coordinate");
  // device buffers only grow: a smaller body reuses them (leading dimension
  // unchanged), so a sequence of bodies allocates for the largest only
  if (npanels > c->capN) {
    free_matrices(c);
    c->capN = npanels;
    c->ld = round_up(npanels, 64);
  }
  c->N = npanels;
  c->h_nodes.assign(nodes, nodes + 3 * nnodes);
  c->h_offsets.assign(offsets, offsets + npanels + 1);
  c->h_pnodes.assign(pnodes, pnodes + offsets[npanels]);
  c->assembled = -1;
  c->factored = -1;

  std::vector<PanelRec> pr(npanels);
  std::vector<SourceRec> sr(npanels);
  std::vector<double> tgt(6 * npanels);
  for (int64_t p = 0; p < npanels; ++p) {
    const int32_t* pn = pnodes + offsets[p];
    const int nn = offsets[p + 1] - offsets[p];
    PanelRec& r = pr[p];
    std::memset(&r, 0, sizeof(r));
    for (int k = 0; k < nn; ++k)
      for (int d = 0; d < 3; ++d) r.p[3 * k + d] = nodes[3 * (int64_t)pn[k] + d];
    r.nn = nn;
    double t[3], o[3], n[3];
    frame(nodes, pn, t, o, n);
    // source record: flipped frame (o, t, -n) of src/FLOWPanel_elements.jl:51-56
    SourceRec& s = sr[p];
    std::memset(&s, 0, sizeof(s));
    s.nn = nn;
    const double* O = nodes + 3 * (int64_t)pn[0];
    for (int d = 0; d < 3; ++d) { s.O[d] = O[d]; s.t[d] = o[d]; s.o[d] = t[d]; s.n[d] = -n[d]; }
    for (int k = 0; k < nn; ++k) {
      const double* P = nodes + 3 * (int64_t)pn[k];
      s.xs[k] = s.t[0] * (P[0] - O[0]) + s.t[1] * (P[1] - O[1]) + s.t[2] * (P[2] - O[2]);
      s.ys[k] = s.o[0] * (P[0] - O[0]) + s.o[1] * (P[1] - O[1]) + s.o[2] * (P[2] - O[2]);
      s.zs[k] = s.n[0] * (P[0] - O[0]) + s.n[1] * (P[1] - O[1]) + s.n[2] * (P[2] - O[2]);
    }
    for (int k = 0; k < nn; ++k) {
      const int j = (k + 1) % nn;
      const double dx = s.xs[j] - s.xs[k], dy = s.ys[j] - s.ys[k], dz = s.zs[j] - s.zs[k];
      s.dij[k] = std::sqrt(dx * dx + dy * dy + dz * dz);
      s.S[k] = (s.ys[j] - s.ys[k]) / s.dij[k];
      s.Cc[k] = (s.xs[j] - s.xs[k]) / s.dij[k];
    }
    // control point and normal
    double cp[3], nr[3];
    if (normals) { for (int d = 0; d < 3; ++d) nr[d] = normals[3 * p + d]; }
    else { for (int d = 0; d < 3; ++d) nr[d] = n[d]; }
    if (cps) {
      for (int d = 0; d < 3; ++d) cp[d] = cps[3 * p + d];
    } else {
      // _calc_controlpoints!: vertex mean, in-plane centroid correction, + off*l*n (l = 1)
      double cc[3] = {0, 0, 0};
      for (int k = 0; k < nn; ++k)
        for (int d = 0; d < 3; ++d) cc[d] += nodes[3 * (int64_t)pn[k] + d];
      for (int d = 0; d < 3; ++d) cc[d] /= nn;
      double x = 0, y = 0;
      for (int k = 0; k < nn; ++k) {
        const double* P = nodes + 3 * (int64_t)pn[k];
        for (int d = 0; d < 3; ++d) x += (P[d] - cc[d]) * t[d];
        for (int d = 0; d < 3; ++d) y += (P[d] - cc[d]) * o[d];
      }
      x /= nn; y /= nn;
      const double off = cp_offset ? cp_offset[p] : 1e-14;
      for (int d = 0; d < 3; ++d) cp[d] = cc[d] + x * t[d] + y * o[d] + off * 1.0 * nr[d];
    }
    for (int d = 0; d < 3; ++d) {
      tgt[d * npanels + p] = cp[d];
      tgt[(3 + d) * npanels + p] = nr[d];
    }
  }
  if (npanels > c->cap_geom) {
    dfree(c->d_panels); dfree(c->d_src); dfree(c->d_tgt);
    c->cap_geom = 0;
    FP_CUDA_TRY(c->err, cudaMalloc(&c->d_panels, npanels * sizeof(PanelRec)));
    FP_CUDA_TRY(c->err, cudaMalloc(&c->d_src, npanels * sizeof(SourceRec)));
    FP_CUDA_TRY(c->err, cudaMalloc(&c->d_tgt, 6 * npanels * sizeof(double)));
    c->cap_geom = npanels;
  }
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_panels, pr.data(), npanels * sizeof(PanelRec), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_src, sr.data(), npanels * sizeof(SourceRec), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_tgt, tgt.data(), 6 * npanels * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  c->h_tgt = tgt;
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  c->has_geometry = true;
  c->nsh = 0;
  c->h_shed.clear();
  c->topo_valid = false;
  c->kutta_valid = false;
  return FP_OK;
}

int fp_set_wake(fp_ctx* c, const int32_t* shedding, int64_t nsh, const double* Das,
                const double* Dbs) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_set_wake: call fp_set_geometry first");
  if (nsh < 0 || (nsh > 0 && (!shedding || !Das || !Dbs)))
    return c->err.set(FP_EINVAL, "fp_set_wake: bad arguments");
  // a background assembly pass may still read the wake records it may free
  if (c->g64_pending) {
    FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream_bg));
    c->g64_pending = false;
  }
  const double tol = 2 * 2.220446049250313e-16;
  std::vector<WakeRec> w(nsh);
  std::vector<int> touched(c->N, 0);
  bool disjoint = true;
  int64_t opposite = -1;   // first edge whose da, db are opposite or orthogonal
  for (int64_t e = 0; e < nsh; ++e) {
    const int32_t* s = shedding + 6 * e;
    const double* da = Das + 3 * e;
    const double* db = Dbs + 3 * e;
    // non-unit direction check of src/FLOWPanel_elements.jl:495-498
    if (std::fabs(da[0] * da[0] + da[1] * da[1] + da[2] * da[2] - 1) > tol ||
        std::fabs(db[0] * db[0] + db[1] * db[1] + db[2] * db[2] - 1) > tol)
      return c->err.set(FP_EINVAL, "Found non-unitary semi-infinite direction at shedding edge " + std::to_string(e));
    const int pi = s[0], pj = s[3];
    if (pi < 0 || pi >= c->N || pj < -1 || pj >= c->N)
      return c->err.set(FP_EINVAL, "fp_set_wake: panel index out of range at edge " + std::to_string(e));
    auto node_of = [&](int panel, int local, double* out3) -> bool {
      const int nn = c->h_offsets[panel + 1] - c->h_offsets[panel];
      if (local < 0 || local >= nn) return false;
      const int ni = c->h_pnodes[c->h_offsets[panel] + local];
      for (int d = 0; d < 3; ++d) out3[d] = c->h_nodes[3 * (int64_t)ni + d];
      return true;
    };
    WakeRec& r = w[e];
    std::memset(&r, 0, sizeof(r));
    if (!node_of(pi, s[1], r.pa) || !node_of(pi, s[2], r.pb))
      return c->err.set(FP_EINVAL, "fp_set_wake: local node index out of range at edge " + std::to_string(e));
    if (pj >= 0 && (!node_of(pj, s[4], r.qa) || !node_of(pj, s[5], r.qb)))
      return c->err.set(FP_EINVAL, "fp_set_wake: local node index out of range at edge " + std::to_string(e));
    for (int d = 0; d < 3; ++d) { r.da[d] = da[d]; r.db[d] = db[d]; }
    r.pi = pi;
    r.pj = pj;
    if (da[0] * db[0] + da[1] * db[1] + da[2] * db[2] <= 0 && opposite < 0) opposite = e;
    if (touched[pi]++) disjoint = false;
    if (pj >= 0 && touched[pj]++) disjoint = false;
  }
  if (nsh > c->cap_wake) {
    dfree(c->d_wake);
    c->cap_wake = 0;
    FP_CUDA_TRY(c->err, cudaMalloc(&c->d_wake, nsh * sizeof(WakeRec)));
    c->cap_wake = nsh;
  }
  if (nsh > 0) {
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_wake, w.data(), nsh * sizeof(WakeRec), cudaMemcpyHostToDevice, c->stream));
    FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  }
  c->h_shed.assign(shedding, shedding + 6 * nsh);
  c->h_Da.assign(Das, Das + 3 * nsh);
  c->h_Db.assign(Dbs, Dbs + 3 * nsh);
  c->wake_opposite = opposite;
  c->nsh = nsh;
  c->kutta_valid = false;
  c->wake_disjoint = disjoint;
  c->assembled = -1;
  c->factored = -1;
  return FP_OK;
}

int fp_assemble(fp_ctx* c, int element, double kerneloffset, double kernelcutoff, int precision) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_assemble: no geometry");
  if (element != FP_ELEMENT_SOURCE && element != FP_ELEMENT_VORTEXRING)
    return c->err.set(FP_EINVAL, "fp_assemble: unknown element");
  if (precision != FP_PREC_FP64 && precision != FP_PREC_MIXED && precision != FP_PREC_MIXED_GEPP &&
      precision != FP_PREC_BF16)
    return c->err.set(FP_EINVAL, "fp_assemble: unknown precision");
  // the previous assembly's background pass must be done before G is written again
  if (int rc = sync_g64(c)) return rc;
  const size_t elems = (size_t)c->ld * c->capN;   // for the largest body the buffers hold
  if (!c->d_G) {
    FP_CUDA_TRY(c->err, cudaMalloc(&c->d_G, elems * sizeof(double)));
    FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_G, 0, elems * sizeof(double), c->stream));
  }
  // the FP32 copy for the FP32 factorisations (the BF16 form rounds its copy from G at fp_factor)
  const bool w32 = precision == FP_PREC_MIXED || precision == FP_PREC_MIXED_GEPP;
  if (w32 && !c->d_G32) {
    FP_CUDA_TRY(c->err, cudaMalloc(&c->d_G32, elems * sizeof(float)));
    FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_G32, 0, elems * sizeof(float), c->stream));
  }
  c->kern_offset = kerneloffset;
  c->kern_cutoff = kernelcutoff;
  if (time_begin(c)) return FP_ECUDA;
  int rc;
  if (element == FP_ELEMENT_VORTEXRING && w32 && c->asm32) {
    // the FP32 AIC on the critical path; the FP64 AIC (read only by the
    // refinement residuals) on the background stream under the factorisation
    if ((rc = launch_assemble_ring32(c, kerneloffset, kernelcutoff))) return rc;
    FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_asm, c->stream));
    FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream_bg, c->ev_asm, 0));
    if ((rc = launch_assemble_ring(c, kerneloffset, kernelcutoff, false, c->stream_bg))) return rc;
    FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_g64, c->stream_bg));
    c->g64_pending = true;
  } else {
    rc = element == FP_ELEMENT_VORTEXRING ? launch_assemble_ring(c, kerneloffset, kernelcutoff, w32)
                                          : launch_assemble_source(c, kerneloffset, w32);
    if (rc) return rc;
  }
  if (time_end(c, &c->ms_assemble)) return FP_ECUDA;
  c->kms[FP_STAGE_ASSEMBLE] = c->ms_assemble;
  c->klaunch[FP_STAGE_ASSEMBLE] = (element == FP_ELEMENT_VORTEXRING && c->nsh > 0) ? 2 : 1;
  c->assembled = element;
  c->assembled_prec = precision;
  c->factored = -1;
  return FP_OK;
}

int fp_get_aic(fp_ctx* c, double* G) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (c->assembled < 0) return c->err.set(FP_ESTATE, "fp_get_aic: nothing assembled");
  if (int rc = sync_g64(c)) return rc;
  FP_CUDA_TRY(c->err, cudaMemcpy2DAsync(G, c->N * sizeof(double), c->d_G, c->ld * sizeof(double),
                                        c->N * sizeof(double), c->N, cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

int fp_set_rhs(fp_ctx* c, const double* Uinfs, int64_t k) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_set_rhs: no geometry");
  if (!Uinfs || k <= 0) return c->err.set(FP_EINVAL, "fp_set_rhs: bad arguments");
  if (int rc = ensure_rhs(c, k)) return rc;
  const size_t elems = 3 * (size_t)c->N * k;
  if (int rc = ensure_stage(c, elems)) return rc;
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_stage, Uinfs, elems * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (int rc = launch_rhs(c, c->d_stage, k)) return rc;
  c->nrhs = k;
  return FP_OK;
}

// Sized for capN (the largest problem the context's buffers hold), so that
// any later body of up to capN unknowns reuses them.
static int alloc_factor_buffers(fp_ctx* c, int precision) {
  const int64_t N = c->capN;
  const size_t elems = (size_t)c->ld * N;
  const int64_t nblk = (N + kLuNB - 1) / kLuNB;
  if (!c->d_ipiv) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_ipiv, N * sizeof(int32_t)));
  if (!c->d_flags) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_flags, (nblk + 2) * sizeof(unsigned int)));
  if (!c->d_mbox) {
    const size_t words = (size_t)((N + 127) / 128) * 128;
    FP_CUDA_TRY(c->err, cudaMalloc(&c->d_mbox, words * sizeof(unsigned long long)));
    FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_mbox, 0, words * sizeof(unsigned long long), c->stream));
  }
  if (!c->d_zbox) {
    const size_t words = (size_t)((N + 127) / 128) * 128;
    FP_CUDA_TRY(c->err, cudaMalloc(&c->d_zbox, words * sizeof(unsigned long long)));
    FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_zbox, 0, words * sizeof(unsigned long long), c->stream));
  }
  if (!c->d_part) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_part, (size_t)kGemvSplitHost * 4 * N * sizeof(double)));
  if (!c->d_minv) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_minv, kMinvBytes + (size_t)2 * kPanelSlots * kLuNB * sizeof(int)));
  if (precision == FP_PREC_FP64) {
    if (!c->d_LU) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_LU, elems * sizeof(double)));
    if (!c->d_dinv64) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_dinv64, nblk * 2 * kLuNB * kLuNB * sizeof(double)));
    if (!c->d_dinv128_64)
      FP_CUDA_TRY(c->err, cudaMalloc(&c->d_dinv128_64, ((N + 127) / 128) * 2 * 128 * 128 * sizeof(double)));
    if (!c->d_mprev64)
      FP_CUDA_TRY(c->err, cudaMalloc(&c->d_mprev64, ((N + 127) / 128) * 2 * 128 * 128 * sizeof(double)));
  } else {
    if (!c->d_G32) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_G32, elems * sizeof(float)));
    if (!c->d_dinv32) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_dinv32, nblk * 2 * kLuNB * kLuNB * sizeof(float)));
    if (!c->d_dinv128_32)
      FP_CUDA_TRY(c->err, cudaMalloc(&c->d_dinv128_32, ((N + 127) / 128) * 2 * 128 * 128 * sizeof(float)));
    if (!c->d_mprev32)
      FP_CUDA_TRY(c->err, cudaMalloc(&c->d_mprev32, ((N + 127) / 128) * 2 * 128 * 128 * sizeof(float)));
    if (!c->d_mq32) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_mq32, ((N + 127) / 128) * 2 * 128 * 128 * sizeof(float)));
    if (!c->d_ms32) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_ms32, ((N + 127) / 128) * 2 * 128 * 128 * sizeof(float)));
  }
  return FP_OK;
}

// The static-order factorisation (lu_factor_static + the diagonal-block
// inverses of the solves) on c->stream, replayed from a CUDA graph when the
// same problem (sizes, buffers, form, tuning) was factored before.
static int factor_static_graph(fp_ctx* c, bool bf16) {
  auto run = [&]() -> int {
    int rc = lu_factor_static(c, c->d_G32, c->N, c->ld, c->d_ipiv, c->d_cert, bf16);
    if (!rc) rc = lu_diag_inverses<float>(c, c->d_G32, c->N, c->ld);
    return rc;
  };
  if (!c->use_graph || c->trace.on || c->ktimer.on) return run();
  std::vector<uintptr_t> key = {(uintptr_t)c->N, (uintptr_t)c->ld, (uintptr_t)c->d_G32, (uintptr_t)c->d_ipiv,
                                (uintptr_t)c->d_cert, (uintptr_t)c->d_status, (uintptr_t)c->d_minv,
                                (uintptr_t)bf16, (uintptr_t)c->tc_stages, (uintptr_t)c->tc_tiles, (uintptr_t)c->tc_smem,
                                (uintptr_t)c->tc_split, (uintptr_t)c->tc_red, (uintptr_t)c->tc_narrow_stages,
                                (uintptr_t)c->lu_overlap, (uintptr_t)c->use_tc, (uintptr_t)c->panel_gemm,
                                (uintptr_t)c->tc_x3, (uintptr_t)c->tc_prefetch, (uintptr_t)c->lu_split,
                                (uintptr_t)c->lu_fuse, (uintptr_t)c->u12_wide, (uintptr_t)c->l21_async,
                                (uintptr_t)c->u12_async, (uintptr_t)c->pdl, (uintptr_t)c->rest_split,
                                (uintptr_t)c->pdiag_linv};
  for (int s = 0; s < 2; ++s)
    for (int i = 0; i < 4; ++i) key.push_back((uintptr_t)c->d_tc[s][i]);
  key.push_back((uintptr_t)c->d_dinv32);
  key.push_back((uintptr_t)c->d_dinv128_32);
  key.push_back((uintptr_t)c->d_mprev32);
  if (c->lu_graph && key == c->lu_graph_key) {
    FP_CUDA_TRY(c->err, cudaGraphLaunch(c->lu_graph, c->stream));
    return FP_OK;
  }
  if (key != c->lu_graph_seen) {   // first time: direct launches (buffers grow here)
    c->lu_graph_seen = key;
    return run();
  }
  if (c->lu_graph) {
    cudaGraphExecDestroy(c->lu_graph);
    c->lu_graph = nullptr;
  }
  FP_CUDA_TRY(c->err, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = run();
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return c->err.set(FP_ECUDA, std::string("capture of the factorisation: ") + cudaGetErrorString(e));
  const cudaError_t ei = cudaGraphInstantiate(&c->lu_graph, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    c->lu_graph = nullptr;
    return c->err.set(FP_ECUDA, std::string("instantiating the factorisation graph: ") + cudaGetErrorString(ei));
  }
  c->lu_graph_key = key;
  FP_CUDA_TRY(c->err, cudaGraphLaunch(c->lu_graph, c->stream));
  return FP_OK;
}

int fp_factor(fp_ctx* c, int precision) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (c->assembled < 0) return c->err.set(FP_ESTATE, "fp_factor: assemble first");
  if (precision != FP_PREC_FP64 && precision != FP_PREC_MIXED && precision != FP_PREC_MIXED_GEPP &&
      precision != FP_PREC_BF16)
    return c->err.set(FP_EINVAL, "fp_factor: unknown precision");
  if (int rc = alloc_factor_buffers(c, precision)) return rc;
  // every factorisation but the FP32 ones of an FP32-assembled AIC reads G
  if (precision == FP_PREC_FP64 || precision == FP_PREC_BF16 ||
      (c->assembled_prec != FP_PREC_MIXED && c->assembled_prec != FP_PREC_MIXED_GEPP))
    if (int rc = sync_g64(c)) return rc;
  if (time_begin(c)) return FP_ECUDA;
  int rc;
  double ms_static = 0;
  c->static_order = false;
  if (precision == FP_PREC_FP64) {
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_LU, c->d_G, (size_t)c->ld * c->N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    rc = lu_factor<double>(c, c->d_LU, c->N, c->ld, c->d_ipiv, c->d_cert);
    if (!rc) rc = lu_diag_inverses<double>(c, c->d_LU, c->N, c->ld);
  } else {
    const bool bf16 = precision == FP_PREC_BF16;
    if (bf16) {   // the AIC the factorisation starts from is the BF16-rounded one
      rc = convert_f64_bf16(c, c->d_G, c->d_G32, c->N, c->N, c->ld, c->ld);
      if (rc) return rc;
    } else if (c->assembled_prec != FP_PREC_MIXED && c->assembled_prec != FP_PREC_MIXED_GEPP) {
      rc = convert_f64_f32(c, c->d_G, c->d_G32, c->N, c->N, c->ld, c->ld);
      if (rc) return rc;
    }
    bool pivoted = precision == FP_PREC_MIXED_GEPP;
    if (!pivoted) {
      // static row order; a zero or non-finite pivot falls back to the pivoted
      // factorisation of a fresh FP32 copy of the AIC
      rc = factor_static_graph(c, bf16);
      if (rc) return rc;
      if (time_end(c, &ms_static)) return FP_ECUDA;
      int st = 0;
      FP_CUDA_TRY(c->err, cudaMemcpy(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
      if (st & DEV_ZERO_PIVOT) {
        FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
        if (time_begin(c)) return FP_ECUDA;
        if ((rc = sync_g64(c))) return rc;
        if ((rc = convert_f64_f32(c, c->d_G, c->d_G32, c->N, c->N, c->ld, c->ld))) return rc;
        pivoted = true;
      } else {
        c->static_order = true;
      }
    }
    if (pivoted) {
      rc = lu_factor<float>(c, c->d_G32, c->N, c->ld, c->d_ipiv, c->d_cert);
      if (!rc) rc = lu_diag_inverses<float>(c, c->d_G32, c->N, c->ld);
    }
    c->assembled_prec = -2;   // the FP32 copy now holds factors
  }
  if (rc) return rc;
  if (c->static_order) {
    c->ms_factor = ms_static;
  } else {
    if (time_end(c, &c->ms_factor)) return FP_ECUDA;
    c->ms_factor += ms_static;
  }
  kt_collect(c);
  tr_collect(c);
  c->kms[FP_STAGE_FACTOR] = c->ms_factor;
  if ((rc = consume_status(c))) return rc;
  float cert = 0.f;
  FP_CUDA_TRY(c->err, cudaMemcpy(&cert, c->d_cert, sizeof(float), cudaMemcpyDeviceToHost));
  c->last.max_abs_L = cert;
  c->last.gepp_certified = cert <= 1.0f;
  c->last.ms_factor = c->ms_factor;
  c->factored = precision == FP_PREC_FP64 ? FP_PREC_FP64 : FP_PREC_MIXED;   // both FP32 forms
  return FP_OK;
}

static void default_opts(fp_solve_opts& o) {
  o.solver = FP_SOLVER_LU;
  o.precision = FP_PREC_FP64;
  o.ir_tol = 1e-12;
  o.ir_maxiter = 10;
  o.gmres_memory = 50;
  o.gmres_atol = -1;
  o.gmres_rtol = -1;
  o.gmres_itmax = 0;
  o.gmres_restart = 0;
}

static void normalize_opts(fp_solve_opts& o) {
  if (o.ir_tol <= 0) o.ir_tol = 1e-12;
  if (o.ir_maxiter <= 0) o.ir_maxiter = 10;
  if (o.gmres_memory <= 0) o.gmres_memory = 50;
}

// max over RHS of ||r_q|| / ||b_q||
static int residual_ratio(fp_ctx* c, const double* r, const double* b, int64_t k, double* out,
                          bool need_b, double* norms = nullptr) {
  if (!norms) norms = c->d_norms;
  if (int rc = colnorm2(c, r, c->N, c->ld, k, norms)) return rc;
  if (need_b)
    if (int rc = colnorm2(c, b, c->N, c->ld, k, norms + k)) return rc;
  std::vector<double> h(2 * k);
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(h.data(), norms, 2 * k * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  double m = 0;
  for (int64_t q = 0; q < k; ++q) {
    const double bn = std::sqrt(h[k + q]);
    const double rn = std::sqrt(h[q]);
    m = std::max(m, bn > 0 ? rn / bn : rn);
  }
  *out = m;
  return FP_OK;
}

// FP64 factors whose certificate failed (a block-local pivot differs from
// partial pivoting over the whole column, so growth is not bounded as
// LAPACK's is): refine x against the FP64 AIC, r = b - G x, x += LU^-1 r,
// until the relative residual stops halving (the FP64 level) or reaches
// 1e-15; if it is then above opts.ir_tol, GMRES-IR preconditioned by the same
// factors takes over. Statistics as for the mixed form.
static int refine_fp64(fp_ctx* c, int64_t k, const fp_solve_opts& o) {
  const int64_t n = c->N, ld = c->ld;
  double prev = 1e300, rr = 0;
  int rc;
  for (int it = 0; it <= o.ir_maxiter; ++it) {
    if ((rc = gemv_residual(c, c->d_G, n, ld, c->d_x, c->d_rhs, c->d_r, k))) return rc;
    if ((rc = residual_ratio(c, c->d_r, c->d_rhs, k, &rr, it == 0))) return rc;
    if ((rc = consume_status(c))) return rc;
    if (rr <= 1e-15 || rr > 0.5 * prev || it == o.ir_maxiter) break;
    prev = rr;
    if ((rc = lu_solve<double>(c, c->d_LU, n, ld, c->d_ipiv, c->d_r, ld, k, false))) return rc;
    if ((rc = axpy_f64(c, c->d_r, c->d_x, n, k, ld))) return rc;
    c->last.ir_iters = it + 1;
  }
  c->last.rel_residual = rr;
  if (rr <= o.ir_tol) return FP_OK;
  int it = 0;
  fp_solve_opts g = o;
  g.gmres_atol = 0.0;
  g.gmres_rtol = o.ir_tol;
  rc = gmres_solve(c, c->d_rhs, c->d_x, k, g, true, &it, &rr);
  c->last.gmres_iters = it;
  c->last.used_gmres = 1;
  c->last.rel_residual = rr;
  return rc;
}

// Mixed-precision iterative refinement with the FP32 factors: x0 = A32^-1 b;
// r = b - A x (FP64, on the stored FP64 AIC); x += A32^-1 r, until
// ||r||/||b|| <= opts.ir_tol; when the residual stops halving, GMRES-IR
// (right-preconditioned by the same factors) takes over.
static int refine_mixed(fp_ctx* c, int64_t k, const fp_solve_opts& o) {
  const int64_t n = c->N, ld = c->ld;
  int rc;
  FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_x, 0, ld * k * sizeof(double), c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_r, c->d_rhs, ld * k * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  double prev = 1e300, rr = 0;
  bool converged = false, first = true;
  for (int it = 0; it < o.ir_maxiter; ++it) {
    if ((rc = convert_f64_f32(c, c->d_r, c->d_w32, n, k, ld, ld))) return rc;
    if ((rc = lu_solve<float>(c, c->d_G32, n, ld, c->d_ipiv, c->d_w32, ld, k, false))) return rc;
    if ((rc = axpy_f32_to_f64(c, c->d_w32, c->d_x, n, k, ld))) return rc;
    if ((rc = gemv_residual(c, c->d_G, n, ld, c->d_x, c->d_rhs, c->d_r, k))) return rc;
    if ((rc = residual_ratio(c, c->d_r, c->d_rhs, k, &rr, first))) return rc;
    if ((rc = consume_status(c))) return rc;
    first = false;
    c->last.ir_iters = it + 1;
    if (rr <= o.ir_tol) { converged = true; break; }
    if (!(rr <= 0.5 * prev)) break;   // stagnating, diverging or not finite: hand over to GMRES-IR
    prev = rr;
  }
  c->last.rel_residual = rr;
  if (converged) return FP_OK;
  int it = 0;
  fp_solve_opts g = o;
  g.gmres_atol = 0.0;
  g.gmres_rtol = o.ir_tol;
  rc = gmres_solve(c, c->d_rhs, c->d_x, k, g, true, &it, &rr);
  c->last.gmres_iters = it;
  c->last.used_gmres = 1;
  c->last.rel_residual = rr;
  return rc;
}

int fp_solve(fp_ctx* c, double* x, int64_t k, const fp_solve_opts* opts, fp_stats* stats) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  fp_solve_opts o;
  default_opts(o);
  if (opts) o = *opts;
  normalize_opts(o);
  if (k <= 0 || k > c->nrhs) return c->err.set(FP_EINVAL, "fp_solve: k must be in 1..(number of RHS set)");
  if (c->assembled < 0) return c->err.set(FP_ESTATE, "fp_solve: assemble first");
  const int64_t n = c->N, ld = c->ld;
  c->last.ir_iters = 0;
  c->last.gmres_iters = 0;
  c->last.used_gmres = 0;
  int rc;
  if (time_begin(c)) return FP_ECUDA;
  if ((rc = sync_g64(c))) return rc;   // the residuals read the FP64 AIC
  if (o.solver == FP_SOLVER_GMRES) {
    int it = 0;
    double rr = 0;
    rc = gmres_solve(c, c->d_rhs, c->d_x, k, o, false, &it, &rr);
    if (rc && rc != FP_ENOCONV) return rc;
    c->last.gmres_iters = it;
    c->last.used_gmres = 1;
    c->last.rel_residual = rr;
    if (rc == FP_ENOCONV) {
      time_end(c, &c->ms_solve);
      return rc;
    }
  } else if (o.precision == FP_PREC_FP64) {
    if (c->factored != FP_PREC_FP64) return c->err.set(FP_ESTATE, "fp_solve: no FP64 factors (call fp_factor)");
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_x, c->d_rhs, ld * k * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if ((rc = lu_solve<double>(c, c->d_LU, n, ld, c->d_ipiv, c->d_x, ld, k, false))) return rc;
    if (!c->last.gepp_certified && (rc = refine_fp64(c, k, o))) {
      time_end(c, &c->ms_solve);
      return rc;
    }
  } else {
    if (c->factored != FP_PREC_MIXED) return c->err.set(FP_ESTATE, "fp_solve: no FP32 factors (call fp_factor)");
    rc = refine_mixed(c, k, o);
    if (rc == FP_ENOCONV && c->static_order) {
      // the statically ordered FP32 factors were not good enough even for
      // GMRES-IR: factor again with pivoting and refine once more
      double ms_first = 0;
      time_end(c, &ms_first);
      if ((rc = fp_factor(c, FP_PREC_MIXED_GEPP))) return rc;
      c->last.ir_iters = 0;
      c->last.gmres_iters = 0;
      c->last.used_gmres = 0;
      if (time_begin(c)) return FP_ECUDA;
      rc = refine_mixed(c, k, o);
    }
    if (rc) { time_end(c, &c->ms_solve); return rc; }
  }
  if (time_end(c, &c->ms_solve)) return FP_ECUDA;
  c->kms[FP_STAGE_SOLVE] = c->ms_solve;
  if ((rc = consume_status(c))) return rc;
  if (o.solver == FP_SOLVER_LU && o.precision == FP_PREC_FP64) {
    // residual of the FP64 solve, for the statistics
    if ((rc = gemv_residual(c, c->d_G, n, ld, c->d_x, c->d_rhs, c->d_r, k))) return rc;
    double rr = 0;
    if ((rc = residual_ratio(c, c->d_r, c->d_rhs, k, &rr, true))) return rc;
    c->last.rel_residual = rr;
  }
  if (x) {
    FP_CUDA_TRY(c->err, cudaMemcpy2DAsync(x, n * sizeof(double), c->d_x, ld * sizeof(double), n * sizeof(double), k,
                                          cudaMemcpyDeviceToHost, c->stream));
    FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  }
  c->last.ms_assemble = c->ms_assemble;
  c->last.ms_factor = c->ms_factor;
  c->last.ms_solve = c->ms_solve;
  if (stats) *stats = c->last;
  return FP_OK;
}

// The knob values of one configuration, in FP_TUNE_* order.
static std::vector<int> current_knobs(const fp_ctx* c) {
  return {c->tc_stages, c->lu_overlap ? 1 : 0, c->tc_tiles, c->use_graph ? 1 : 0, c->tc_smem, c->fp64_dmma,
          c->tc_split, c->tc_red ? 1 : 0, c->asm32 ? 1 : 0, c->tc_narrow_stages};
}

int fp_autotune(fp_ctx* c, int precision, int reps, int* knobs_out) {
  if (check_ctx(c)) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (precision != FP_PREC_FP64 && precision != FP_PREC_MIXED && precision != FP_PREC_BF16)
    return c->err.set(FP_EINVAL, "fp_autotune: precision must be FP_PREC_FP64, FP_PREC_MIXED or FP_PREC_BF16");
  reps = std::max(1, std::min(reps, 16));
  const uint64_t key = ((uint64_t)c->N << 8) | (uint64_t)precision;
  auto hit = c->tuned.find(key);
  if (hit == c->tuned.end()) {
    if (c->assembled < 0) return c->err.set(FP_ESTATE, "fp_autotune: assemble first");
    if (precision == FP_PREC_MIXED && c->assembled_prec != FP_PREC_MIXED && c->assembled_prec != FP_PREC_MIXED_GEPP)
      return c->err.set(FP_ESTATE, "fp_autotune: FP_PREC_MIXED needs an AIC assembled for it");
    // candidates: (knob, value) settings over the defaults; each is timed by
    // its median factorisation (device time) on the assembled AIC
    std::vector<std::vector<std::pair<int, int>>> cand;
    if (precision == FP_PREC_FP64) {
      for (int v : {6, 5, 4, 3, 0}) cand.push_back({{FP_TUNE_FP64_DMMA, v}});
    } else if (precision == FP_PREC_MIXED && c->tc_x3 && c->panel_gemm > 0) {
      // the BF16-pair update has one epilogue and ring; only the narrow ring varies
      for (int narrow : {6, 0}) cand.push_back({{FP_TUNE_TC_NARROW, narrow}});
    } else {
      for (int red : {1, 0})
        for (int stages : {2, 3})
          for (int tiles : {0, 4}) {
            if (tiles && stages == 3) continue;   // the multi-tile kernel has its own ring
            for (int narrow : {6, 0}) {
              if (narrow && !red) continue;   // the deep narrow ring is a red.global kernel
              cand.push_back({{FP_TUNE_TC_RED, red}, {FP_TUNE_TC_STAGES, stages}, {FP_TUNE_TC_TILES, tiles},
                              {FP_TUNE_TC_NARROW, narrow}});
            }
          }
    }
    const std::vector<int> saved = current_knobs(c);
    const int element = c->assembled, aprec = c->assembled_prec;
    const double off = c->kern_offset, cut = c->kern_cutoff;
    // on an error the caller's knobs come back before the status is returned
    auto fail = [&](int rc) {
      const std::string msg = c->err.msg;
      for (int k = 0; k < (int)saved.size(); ++k) fp_set_tuning(c, k, saved[k]);
      return c->err.set(rc, msg);
    };
    double best = 1e300;
    std::vector<int> best_knobs = saved;
    for (const auto& cfg : cand) {
      for (int k = 0; k < (int)saved.size(); ++k) fp_set_tuning(c, k, saved[k]);
      for (const auto& kv : cfg) fp_set_tuning(c, kv.first, kv.second);
      std::vector<double> ms;
      for (int r = 0; r < reps + 1; ++r) {   // the first run warms the kernels up
        // the FP32 factorisations work in place on the FP32 AIC: assemble it again
        if (precision != FP_PREC_FP64 && precision != FP_PREC_BF16)
          if (int rc = fp_assemble(c, element, off, cut, aprec)) return fail(rc);
        if (int rc = fp_factor(c, precision)) return fail(rc);
        if (r > 0) ms.push_back(c->ms_factor);
      }
      std::sort(ms.begin(), ms.end());
      const double med = ms[ms.size() / 2];
      if (med < best) { best = med; best_knobs = current_knobs(c); }
    }
    hit = c->tuned.emplace(key, best_knobs).first;
    // leave the context assembled, not factored
    if (int rc = fp_assemble(c, element, off, cut, aprec)) return fail(rc);
  }
  for (int k = 0; k < (int)hit->second.size(); ++k) fp_set_tuning(c, k, hit->second[k]);
  if (knobs_out)
    for (int k = 0; k < (int)hit->second.size(); ++k) knobs_out[k] = hit->second[k];
  return FP_OK;
}

int fp_set_tuning(fp_ctx* c, int knob, int value) {
  if (check_ctx(c)) return FP_EINVAL;
  switch (knob) {
    case FP_TUNE_TC_STAGES:
      if (value != 2 && value != 3) return c->err.set(FP_EINVAL, "fp_set_tuning: FP_TUNE_TC_STAGES is 2 or 3");
      c->tc_stages = value;
      return FP_OK;
    case FP_TUNE_LU_OVERLAP:
      c->lu_overlap = value != 0;
      return FP_OK;
    case FP_TUNE_TC_TILES:
      if (value < 0 || value > 64) return c->err.set(FP_EINVAL, "fp_set_tuning: FP_TUNE_TC_TILES is 0..64");
      c->tc_tiles = value;
      return FP_OK;
    case FP_TUNE_GRAPH:
      c->use_graph = value != 0;
      return FP_OK;
    case FP_TUNE_FP64_DMMA:
      if (value < 0 || value > 6) return c->err.set(FP_EINVAL, "fp_set_tuning: FP_TUNE_FP64_DMMA is 0..6");
      c->fp64_dmma = value;
      return FP_OK;
    case FP_TUNE_TRS2:
      c->trs_skip2 = value != 0;
      if (!c->trs_skip2) c->trs2_ready = false;
      return FP_OK;
    case FP_TUNE_PANEL_GEMM:
      if (value < 0 || value > 2) return c->err.set(FP_EINVAL, "fp_set_tuning: FP_TUNE_PANEL_GEMM is 0..2");
      c->panel_gemm = value;
      return FP_OK;
    case FP_TUNE_TC_BF16X3:
      c->tc_x3 = value != 0;
      return FP_OK;
    case FP_TUNE_TC_PREFETCH:
      c->tc_prefetch = value != 0;
      return FP_OK;
    case FP_TUNE_PDL:
      c->pdl = value != 0;
      return FP_OK;
    case FP_TUNE_LU_SPLIT:
      c->lu_split = value != 0;
      return FP_OK;
    case FP_TUNE_LU_FUSE:
      c->lu_fuse = value != 0;
      return FP_OK;
    case FP_TUNE_U12_WIDE:
      c->u12_wide = value != 0;
      return FP_OK;
    case FP_TUNE_L21_ASYNC:
      c->l21_async = value != 0;
      return FP_OK;
    case FP_TUNE_U12_ASYNC:
      c->u12_async = value != 0;
      return FP_OK;
    case FP_TUNE_PDIAG_LINV:
      c->pdiag_linv = value != 0;
      return FP_OK;
    case FP_TUNE_REST_SPLIT:
      if (value < 0 || value > 2) return c->err.set(FP_EINVAL, "fp_set_tuning: FP_TUNE_REST_SPLIT is 0, 1 or 2");
      c->rest_split = value;
      return FP_OK;
    case FP_TUNE_TC_NARROW:
      if (value != 0 && value != 6) return c->err.set(FP_EINVAL, "fp_set_tuning: FP_TUNE_TC_NARROW is 0 or 6");
      c->tc_narrow_stages = value;
      return FP_OK;
    case FP_TUNE_ASM32:
      c->asm32 = value != 0;
      return FP_OK;
    case FP_TUNE_TC_RED:
      c->tc_red = value != 0;
      return FP_OK;
    case FP_TUNE_TC_SPLIT:
      if (value < 0 || value > 3) return c->err.set(FP_EINVAL, "fp_set_tuning: FP_TUNE_TC_SPLIT is 0..3");
      c->tc_split = value;
      return FP_OK;
    case FP_TUNE_TC_SMEM:
      if (value < 0 || value > kTcSmemMax)
        return c->err.set(FP_EINVAL, "fp_set_tuning: FP_TUNE_TC_SMEM is 0.." + std::to_string(kTcSmemMax));
      c->tc_smem = value;
      return FP_OK;
    default:
      return c->err.set(FP_EINVAL, "fp_set_tuning: unknown knob");
  }
}

int fp_lu_solve_noalloc(fp_ctx* c, double* B, int64_t ldb, int64_t k) {
  if (check_ctx(c)) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (!B || k <= 0 || ldb < c->N) return c->err.set(FP_EINVAL, "fp_lu_solve_noalloc: B must be N x k with ldb >= N");
  if (c->factored != FP_PREC_FP64)
    return c->err.set(FP_ESTATE, "fp_lu_solve_noalloc: no FP64 factors (call fp_factor with FP_PREC_FP64)");
  if (!c->last.gepp_certified)
    return c->err.set(FP_ESTATE, "fp_lu_solve_noalloc: the FP64 factors are not certified (a block-local pivot "
                                 "differs from partial pivoting); fp_solve refines such factors");
  if (int rc = lu_solve_noalloc(c, B, ldb, k)) return rc;
  return consume_status(c);
}

int fp_solve_body(fp_ctx* c, int element, double kerneloffset, double kernelcutoff,
                  const double* Uinfs, int64_t k, const fp_solve_opts* opts, double* x,
                  fp_stats* stats) {
  if (check_ctx(c)) return FP_EINVAL;
  fp_solve_opts o;
  default_opts(o);
  if (opts) o = *opts;
  int rc;
  const int prec = (o.solver == FP_SOLVER_LU) ? o.precision : FP_PREC_FP64;
  if ((rc = fp_assemble(c, element, kerneloffset, kernelcutoff, prec))) return rc;
  if ((rc = fp_set_rhs(c, Uinfs, k))) return rc;
  if (o.solver == FP_SOLVER_LU || o.precision != FP_PREC_FP64)
    if ((rc = fp_factor(c, o.precision))) return rc;
  return fp_solve(c, x, k, &o, stats);
}

int fp_uind(fp_ctx* c, int element, const double* strengths, const double* targets, int64_t m,
            double* out, int precision, double kerneloffset, double kernelcutoff) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_uind: no geometry");
  if (!strengths || (m > 0 && (!targets || !out)) || m < 0)
    return c->err.set(FP_EINVAL, "fp_uind: bad arguments");
  if (m == 0) return FP_OK;
  c->kern_offset = kerneloffset;
  c->kern_cutoff = kernelcutoff;
  const int64_t ns = element == FP_ELEMENT_SOURCE_DOUBLET ? 2 * c->N : c->N;
  if (int rc = ensure_stage(c, (size_t)ns + 6 * (size_t)m)) return rc;
  double* ds = c->d_stage;
  double* dt = ds + ns;
  double* dout = dt + 3 * m;
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(ds, strengths, ns * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(dt, targets, 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(dout, out, 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (time_begin(c)) return FP_ECUDA;
  int rc;
  if (element == FP_ELEMENT_VORTEXRING) {
    rc = launch_uind_ring(c, ds, dt, m, dout, precision != FP_PREC_FP64);
  } else if (element == FP_ELEMENT_SOURCE_DOUBLET) {   // sources, then doublets (rings without wake)
    const int64_t nsh = c->nsh;
    c->nsh = 0;
    rc = launch_uind_source(c, ds, dt, m, dout);
    if (!rc) rc = launch_uind_ring(c, ds + c->N, dt, m, dout, false);
    c->nsh = nsh;
  } else {
    rc = launch_uind_source(c, ds, dt, m, dout);
  }
  if (rc) return rc;
  if (time_end(c, &c->ms_uind)) return FP_ECUDA;
  c->kms[FP_STAGE_UIND] = c->ms_uind;
  c->klaunch[FP_STAGE_UIND] = 1;
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(out, dout, 3 * m * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

int fp_solve_ls(fp_ctx* c, double kerneloffset, double kernelcutoff, const double* Uinfs, int64_t npres,
                const int64_t* el_index, const double* el_value, double* x, fp_stats* stats) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_solve_ls: no geometry");
  if (int rc = sync_g64(c)) return rc;
  if (!Uinfs || !x || npres < 0 || npres >= c->N || (npres > 0 && (!el_index || !el_value)))
    return c->err.set(FP_EINVAL, "fp_solve_ls: bad arguments");
  // prescribed elements sorted by index (src/FLOWPanel_liftingbody.jl:399)
  std::vector<std::pair<int64_t, double>> pres(npres);
  for (int64_t p = 0; p < npres; ++p) pres[p] = {el_index[p], el_value[p]};
  std::sort(pres.begin(), pres.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  std::vector<int> el(npres);
  std::vector<double> val(npres);
  for (int64_t p = 0; p < npres; ++p) {
    if (pres[p].first < 0 || pres[p].first >= c->N || (p > 0 && pres[p].first == pres[p - 1].first))
      return c->err.set(FP_EINVAL, "fp_solve_ls: prescribed element indices must be distinct and in 0..N-1");
    el[p] = (int)pres[p].first;
    val[p] = pres[p].second;
  }
  int rc;
  if ((rc = fp_assemble(c, FP_ELEMENT_VORTEXRING, kerneloffset, kernelcutoff, FP_PREC_FP64))) return rc;
  if ((rc = fp_set_rhs(c, Uinfs, 1))) return rc;
  if ((rc = alloc_factor_buffers(c, FP_PREC_FP64))) return rc;
  FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_cert, 0, sizeof(float), c->stream));
  std::vector<double> g(c->N - npres);
  if (time_begin(c)) return FP_ECUDA;
  if ((rc = ls_solve(c, el.data(), val.data(), (int)npres, g.data()))) return rc;
  if (time_end(c, &c->ms_factor)) return FP_ECUDA;
  c->factored = -1;   // the FP64 factor buffer now holds the normal equations' factors
  c->nrhs = 0;
  if ((rc = consume_status(c))) return rc;
  // set_solution: the reduced strengths around the prescribed values
  for (int64_t j = 0, p = 0, q = 0; j < c->N; ++j) {
    if (p < npres && el[p] == j) x[j] = val[p++];
    else x[j] = g[q++];
  }
  float cert = 0.f;
  FP_CUDA_TRY(c->err, cudaMemcpy(&cert, c->d_cert, sizeof(float), cudaMemcpyDeviceToHost));
  c->last = fp_stats{};
  c->last.ms_assemble = c->ms_assemble;
  c->last.ms_factor = c->ms_factor;
  c->last.max_abs_L = cert;
  c->last.gepp_certified = cert <= 1.0f;
  if (stats) *stats = c->last;
  return FP_OK;
}

int fp_phi(fp_ctx* c, int element, const double* strengths, const double* targets, int64_t m, double* out,
           double kerneloffset) {
  if (check_ctx(c)) return FP_EINVAL;
  cudaSetDevice(c->device);
  if (!c->has_geometry) return c->err.set(FP_ESTATE, "fp_phi: no geometry");
  if (element != FP_ELEMENT_SOURCE && element != FP_ELEMENT_VORTEXRING && element != FP_ELEMENT_SOURCE_DOUBLET)
    return c->err.set(FP_EINVAL, "fp_phi: unknown element");
  if (!strengths || (m > 0 && (!targets || !out)) || m < 0) return c->err.set(FP_EINVAL, "fp_phi: bad arguments");
  const bool wake = element == FP_ELEMENT_VORTEXRING && c->nsh > 0;
  if (wake && c->wake_opposite >= 0) {
    const double* da = c->h_Da.data() + 3 * c->wake_opposite;
    const double* db = c->h_Db.data() + 3 * c->wake_opposite;
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "Invalid semi-infinite directions: da=[%g, %g, %g] is opposite or orthogonal to db=[%g, %g, %g]",
                  da[0], da[1], da[2], db[0], db[1], db[2]);
    return c->err.set(FP_EINVAL, msg);
  }
  if (m == 0) return FP_OK;
  c->kern_offset = kerneloffset;
  const int64_t ns = element == FP_ELEMENT_SOURCE_DOUBLET ? 2 * c->N : c->N;
  if (int rc = ensure_stage(c, (size_t)ns + 4 * (size_t)m)) return rc;
  double* ds = c->d_stage;
  double* dt = ds + ns;
  double* dout = dt + 3 * m;
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(ds, strengths, ns * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(dt, targets, 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(dout, out, m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  const double* sigma = element == FP_ELEMENT_VORTEXRING ? nullptr : ds;
  const double* mu = element == FP_ELEMENT_SOURCE ? nullptr : (element == FP_ELEMENT_SOURCE_DOUBLET ? ds + c->N : ds);
  double ms = 0;
  if (time_begin(c)) return FP_ECUDA;
  if (int rc = launch_phi(c, sigma, mu, dt, m, dout, wake)) return rc;
  if (time_end(c, &ms)) return FP_ECUDA;
  c->kms[FP_STAGE_PHI] = ms;
  c->klaunch[FP_STAGE_PHI] = 1;
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(out, dout, m * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

static int ensure_adjoint(fp_ctx* c, int64_t k) {
  if (k <= c->cap_adj) return FP_OK;
  dfree(c->d_ab); dfree(c->d_ax); dfree(c->d_ar); dfree(c->d_aw32);
  c->cap_adj = 0;
  const size_t n = (size_t)c->ld * k;
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_ab, n * sizeof(double)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_ax, n * sizeof(double)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_ar, n * sizeof(double)));
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_aw32, n * sizeof(float)));
  dfree(c->d_anorms);
  FP_CUDA_TRY(c->err, cudaMalloc(&c->d_anorms, 2 * k * sizeof(double)));
  c->cap_adj = k;
  return FP_OK;
}

// A^T lambda = ybar on the device with the saved factors; the solution stays
// in d_ax. FP64 factors: one transposed LU solve. FP32 factors: iterative
// refinement with the transposed FP32 solve and the FP64 residual
// ybar - A^T lambda on the stored FP64 AIC, to a relative residual of 1e-12.
static int adjoint_device(fp_ctx* c, int64_t k) {
  const int64_t n = c->N, ld = c->ld;
  int rc;
  c->adj_iters = 0;
  c->adj_relres = 0;
  if (c->factored == FP_PREC_FP64) {
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_ax, c->d_ab, ld * k * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if ((rc = lu_solve<double>(c, c->d_LU, n, ld, c->d_ipiv, c->d_ax, ld, k, true))) return rc;
    if (c->last.gepp_certified) return FP_OK;
    // uncertified block-local pivots: refine against the FP64 AIC (transposed)
    double rr = 0, prev = 1e300;
    for (int it = 0;; ++it) {
      if ((rc = gemvT_residual(c, c->d_G, n, ld, c->d_ax, c->d_ab, c->d_ar, k))) return rc;
      if ((rc = residual_ratio(c, c->d_ar, c->d_ab, k, &rr, it == 0, c->d_anorms))) return rc;
      c->adj_relres = rr;
      if (rr <= 1e-15 || rr > 0.5 * prev || it == 10) break;
      prev = rr;
      if ((rc = lu_solve<double>(c, c->d_LU, n, ld, c->d_ipiv, c->d_ar, ld, k, true))) return rc;
      if ((rc = axpy_f64(c, c->d_ar, c->d_ax, n, k, ld))) return rc;
      c->adj_iters = it + 1;
    }
    if (rr <= 1e-12) return FP_OK;
    return c->err.set(FP_ENOCONV, "fp_adjoint_solve: refinement of the uncertified FP64 factors stalled at "
                                  "relative residual " + std::to_string(rr));
  }
  const double tol = 1e-12;
  const int maxit = 10;
  FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_ax, 0, ld * k * sizeof(double), c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(c->d_ar, c->d_ab, ld * k * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  double rr = 0, prev = 1e300;
  bool first = true;
  for (int it = 0; it < maxit; ++it) {
    if ((rc = convert_f64_f32(c, c->d_ar, c->d_aw32, n, k, ld, ld))) return rc;
    if ((rc = lu_solve<float>(c, c->d_G32, n, ld, c->d_ipiv, c->d_aw32, ld, k, true))) return rc;
    if ((rc = axpy_f32_to_f64(c, c->d_aw32, c->d_ax, n, k, ld))) return rc;
    if ((rc = gemvT_residual(c, c->d_G, n, ld, c->d_ax, c->d_ab, c->d_ar, k))) return rc;
    if ((rc = residual_ratio(c, c->d_ar, c->d_ab, k, &rr, first, c->d_anorms))) return rc;
    first = false;
    c->adj_iters = it + 1;
    c->adj_relres = rr;
    if (rr <= tol) return FP_OK;
    if (rr > 0.5 * prev) break;
    prev = rr;
  }
  return c->err.set(FP_ENOCONV, "fp_adjoint_solve: refinement with the FP32 factors stalled at relative residual " +
                                    std::to_string(rr));
}

int fp_adjoint_solve(fp_ctx* c, const double* ybar, int64_t k, double* lambda) {
  if (check_ctx(c)) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (!ybar || !lambda || k <= 0) return c->err.set(FP_EINVAL, "fp_adjoint_solve: bad arguments");
  if (c->factored < 0) return c->err.set(FP_ESTATE, "fp_adjoint_solve: no factors (call fp_factor)");
  const int64_t n = c->N, ld = c->ld;
  int rc;
  if ((rc = sync_g64(c))) return rc;   // the adjoint's residuals read the FP64 AIC
  if ((rc = ensure_adjoint(c, k))) return rc;
  FP_CUDA_TRY(c->err, cudaMemcpy2DAsync(c->d_ab, ld * sizeof(double), ybar, n * sizeof(double), n * sizeof(double), k,
                                        cudaMemcpyHostToDevice, c->stream));
  if (time_begin(c)) return FP_ECUDA;
  rc = adjoint_device(c, k);
  double ms = 0;
  if (time_end(c, &ms)) return FP_ECUDA;
  c->kms[FP_STAGE_ADJOINT] = ms;
  if (rc) return rc;
  if ((rc = consume_status(c))) return rc;
  FP_CUDA_TRY(c->err, cudaMemcpy2DAsync(lambda, n * sizeof(double), c->d_ax, ld * sizeof(double), n * sizeof(double), k,
                                        cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamSynchronize(c->stream));
  return FP_OK;
}

// Device workspace of the reverse pass for m targets.
struct VjpBufs {
  double *x, *w, *gX, *U, *gvert, *gs, *gwake, *lam, *gam;
  size_t zero_count;   // gX .. gwake are contiguous and zeroed before a pass
};
static int vjp_buffers(fp_ctx* c, int64_t m, VjpBufs& b) {
  const size_t n = (size_t)c->N, nsh = (size_t)c->nsh;
  const size_t need = 3 * m + 3 * m + 3 * m + 3 * m + 12 * n + n + kWakeGradHost * nsh + n + n;
  if (need > c->cap_vjp) {
    dfree(c->d_vjp);
    c->cap_vjp = 0;
    FP_CUDA_TRY(c->err, cudaMalloc(&c->d_vjp, need * sizeof(double)));
    c->cap_vjp = need;
  }
  double* p = c->d_vjp;
  b.x = p; p += 3 * m;
  b.w = p; p += 3 * m;
  b.gX = p; p += 3 * m;
  b.U = p; p += 3 * m;
  b.gvert = p; p += 12 * n;
  b.gs = p; p += n;
  b.gwake = p; p += kWakeGradHost * nsh;
  b.lam = p; p += n;
  b.gam = p;
  b.zero_count = 3 * m + 3 * m + 12 * n + n + kWakeGradHost * nsh;
  return FP_OK;
}

// Adds the per-panel vertex gradients (N x 12) and the wake TE-node
// gradients to dnodes (3 x nnodes), and writes dDas / dDbs.
static void scatter_vjp(fp_ctx* c, const std::vector<double>& gvert, const std::vector<double>& gwake,
                        double* dnodes, double* dDas, double* dDbs) {
  const int64_t nnodes = (int64_t)c->h_nodes.size() / 3;
  if (dnodes) {
    std::fill(dnodes, dnodes + 3 * nnodes, 0.0);
    for (int64_t j = 0; j < c->N; ++j) {
      const int o = c->h_offsets[j], nn = c->h_offsets[j + 1] - o;
      for (int k = 0; k < nn; ++k) {
        const int64_t ni = c->h_pnodes[o + k];
        for (int d = 0; d < 3; ++d) dnodes[3 * ni + d] += gvert[12 * j + 3 * k + d];
      }
    }
  }
  for (int64_t e = 0; e < c->nsh; ++e) {
    const int32_t* s = c->h_shed.data() + 6 * e;
    const double* g = gwake.data() + kWakeGradHost * e;
    if (dnodes) {
      auto add = [&](int panel, int local, const double* gg) {
        const int64_t ni = c->h_pnodes[c->h_offsets[panel] + local];
        for (int d = 0; d < 3; ++d) dnodes[3 * ni + d] += gg[d];
      };
      add(s[0], s[1], g + 0);
      add(s[0], s[2], g + 3);
      if (s[3] >= 0) {
        add(s[3], s[4], g + 6);
        add(s[3], s[5], g + 9);
      }
    }
    if (dDas) for (int d = 0; d < 3; ++d) dDas[3 * e + d] = g[12 + d];
    if (dDbs) for (int d = 0; d < 3; ++d) dDbs[3 * e + d] = g[15 + d];
  }
}

int fp_assembly_vjp(fp_ctx* c, const double* lambda, const double* gamma, const double* Uinfs,
                    double* dnodes, double* dcps, double* dnormals, double* dUinfs, double* dDas,
                    double* dDbs) {
  if (check_ctx(c)) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (c->assembled != FP_ELEMENT_VORTEXRING)
    return c->err.set(FP_ESTATE, "fp_assembly_vjp: assemble a vortex-ring body first");
  if (!lambda && c->cap_adj < 1)
    return c->err.set(FP_ESTATE, "fp_assembly_vjp: no lambda given and no fp_adjoint_solve result on the device");
  if (!gamma && c->cap_rhs < 1)
    return c->err.set(FP_ESTATE, "fp_assembly_vjp: no gamma given and no fp_solve result on the device");
  if ((dnormals || dUinfs) && !Uinfs)
    return c->err.set(FP_EINVAL, "fp_assembly_vjp: dnormals / dUinfs need Uinfs");
  const int64_t n = c->N;
  VjpBufs b;
  int rc;
  if ((rc = vjp_buffers(c, n, b))) return rc;
  if (time_begin(c)) return FP_ECUDA;
  const double* dl = c->d_ax;
  const double* dg = c->d_x;
  if (lambda) {
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(b.lam, lambda, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    dl = b.lam;
  }
  if (gamma) {
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(b.gam, gamma, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    dg = b.gam;
  }
  FP_CUDA_TRY(c->err, cudaMemsetAsync(b.gX, 0, b.zero_count * sizeof(double), c->stream));
  if ((rc = launch_vjp_cotangent(c, dl, b.w))) return rc;
  if ((rc = launch_pair_vjp(c, dg, c->d_tgt, b.w, n, b.gX, b.U, b.gvert, b.gs, b.gwake))) return rc;
  std::vector<double> hX(3 * n), hU(3 * n), hv(12 * n), hw(kWakeGradHost * c->nsh), hl(n);
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(hX.data(), b.gX, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(hU.data(), b.U, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(hv.data(), b.gvert, 12 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (c->nsh > 0)
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(hw.data(), b.gwake, kWakeGradHost * c->nsh * sizeof(double),
                                        cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(hl.data(), dl, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  double ms = 0;
  if (time_end(c, &ms)) return FP_ECUDA;
  c->kms[FP_STAGE_VJP] = ms;
  // residual r = b - A Gamma with b_i = -Uinf_i . n_i: d(lambda^T r)/dn_i =
  // -lambda_i (U_i + Uinf_i), d/dUinf_i = -lambda_i n_i, d/dX_i from the kernel
  const double* T = c->h_tgt.data();
  for (int64_t i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) {
      if (dcps) dcps[3 * i + d] = hX[d * n + i];
      if (dnormals) dnormals[3 * i + d] = -hl[i] * (hU[d * n + i] + Uinfs[3 * i + d]);
      if (dUinfs) dUinfs[3 * i + d] = -hl[i] * T[(3 + d) * n + i];
    }
  }
  scatter_vjp(c, hv, hw, dnodes, dDas, dDbs);
  return FP_OK;
}

int fp_uind_vjp(fp_ctx* c, const double* strengths, const double* targets, int64_t m, const double* wbar,
                double* dtargets, double* dstrengths, double* dnodes, double* dDas, double* dDbs) {
  if (check_ctx(c)) return FP_EINVAL;
  FP_CUDA_TRY(c->err, cudaSetDevice(c->device));
  if (c->assembled != FP_ELEMENT_VORTEXRING)
    return c->err.set(FP_ESTATE, "fp_uind_vjp: assemble a vortex-ring body first");
  if (!strengths || !targets || !wbar || m <= 0) return c->err.set(FP_EINVAL, "fp_uind_vjp: bad arguments");
  const int64_t n = c->N;
  VjpBufs b;
  int rc;
  if ((rc = vjp_buffers(c, m, b))) return rc;
  // targets and cotangents arrive 3 x m (point-major); the kernels read SoA
  std::vector<double> hx(3 * m), hwv(3 * m);
  for (int64_t i = 0; i < m; ++i)
    for (int d = 0; d < 3; ++d) {
      hx[d * m + i] = targets[3 * i + d];
      hwv[d * m + i] = wbar[3 * i + d];
    }
  if (time_begin(c)) return FP_ECUDA;
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(b.x, hx.data(), 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(b.w, hwv.data(), 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(b.gam, strengths, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FP_CUDA_TRY(c->err, cudaMemsetAsync(b.gX, 0, b.zero_count * sizeof(double), c->stream));
  if ((rc = launch_pair_vjp(c, b.gam, b.x, b.w, m, b.gX, nullptr, b.gvert, b.gs, b.gwake))) return rc;
  std::vector<double> hX(3 * m), hv(12 * n), hs(n), hw(kWakeGradHost * c->nsh);
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(hX.data(), b.gX, 3 * m * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(hv.data(), b.gvert, 12 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FP_CUDA_TRY(c->err, cudaMemcpyAsync(hs.data(), b.gs, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (c->nsh > 0)
    FP_CUDA_TRY(c->err, cudaMemcpyAsync(hw.data(), b.gwake, kWakeGradHost * c->nsh * sizeof(double),
                                        cudaMemcpyDeviceToHost, c->stream));
  double ms = 0;
  if (time_end(c, &ms)) return FP_ECUDA;
  c->kms[FP_STAGE_VJP] = ms;
  if (dtargets)
    for (int64_t i = 0; i < m; ++i)
      for (int d = 0; d < 3; ++d) dtargets[3 * i + d] = hX[d * m + i];
  if (dstrengths) {
    for (int64_t j = 0; j < n; ++j) dstrengths[j] = hs[j];
    // wake strengths are Gamma_pi (upper) and Gamma_pj (lower)
    for (int64_t e = 0; e < c->nsh; ++e) {
      const int32_t* s = c->h_shed.data() + 6 * e;
      dstrengths[s[0]] += hw[kWakeGradHost * e + 18];
      if (s[3] >= 0) dstrengths[s[3]] += hw[kWakeGradHost * e + 19];
    }
  }
  scatter_vjp(c, hv, hw, dnodes, dDas, dDbs);
  return FP_OK;
}

int fp_kernel_timing(fp_ctx* c, int enable) {
  if (check_ctx(c)) return FP_EINVAL;
  KernelTimer& t = c->ktimer;
  t.on = enable != 0;
  t.used = 0;
  t.work.clear();
  t.launches = 0;
  t.ms = 0;
  t.flops = 0;
  t.units = 0;
  t.elems.clear();
  return FP_OK;
}

int fp_kernel_timing_read(fp_ctx* c, int64_t* launches, double* ms, double* flops, double* elems) {
  if (check_ctx(c)) return FP_EINVAL;
  if (launches) *launches = c->ktimer.launches;
  if (ms) *ms = c->ktimer.ms;
  if (flops) *flops = c->ktimer.flops;
  if (elems) *elems = c->ktimer.units;
  return FP_OK;
}

int fp_trace(fp_ctx* c, int enable) {
  if (check_ctx(c)) return FP_EINVAL;
  c->trace.on = enable != 0;
  c->trace.recs.clear();
  c->trace.used = 0;
  c->trace.base = -1;
  return FP_OK;
}

int fp_trace_read(fp_ctx* c, int64_t cap, int* tags, int* streams, float* t0, float* t1, int64_t* count) {
  if (check_ctx(c) || !count) return FP_EINVAL;
  const Trace& t = c->trace;
  *count = (int64_t)t.t0.size();
  for (int64_t i = 0; i < std::min<int64_t>(cap, *count); ++i) {
    if (tags) tags[i] = t.tags[i];
    if (streams) streams[i] = t.streams[i];
    if (t0) t0[i] = t.t0[i];
    if (t1) t1[i] = t.t1[i];
  }
  return FP_OK;
}

int fp_kernel_launches(fp_ctx* c, int64_t* count) {
  if (check_ctx(c) || !count) return FP_EINVAL;
  *count = c->nlaunch;
  return FP_OK;
}

int fp_last_kernel_ms(fp_ctx* c, int stage, double* ms, int* launches) {
  if (check_ctx(c) || stage < 0 || stage > FP_STAGE_PHI) return FP_EINVAL;
  if (ms) *ms = c->kms[stage];
  if (launches) *launches = c->klaunch[stage];
  return FP_OK;
}

}  // extern "C"
