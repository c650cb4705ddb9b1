// Context and internal launchers of the B200 panel-method library.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <string>
#include <vector>

#include "fp_common.cuh"
#include "fp_elements.cuh"

// Wake record: both horseshoes of one shedding edge, node coordinates resolved.
struct WakeRec {
  double pa[3], pb[3];   // upper: TE[1], TE[2] of panel pi
  double qa[3], qb[3];   // lower: TE[1], TE[2] of panel pj (unused if pj < 0)
  double da[3], db[3];
  int pi, pj;
};

// Opt-in per-launch timing of one kernel (CUDA events on the context's stream
// around each launch), for the roofline of the factorisation's trailing update.
struct KernelTimer {
  bool on = false;
  std::vector<cudaEvent_t> pool;   // pairs (start, stop), reused
  size_t used = 0;                 // events recorded since the last collect
  std::vector<double> work;        // algorithmic flops of each timed launch
  std::vector<double> elems;       // output elements (m x n) of each timed launch
  int64_t launches = 0;
  double ms = 0, flops = 0, units = 0;
};

// Opt-in timeline of the factorisation: CUDA events around every launch of
// lu_factor on either stream, tagged by kernel; times relative to a base event
// at the start of the factorisation (fp_trace / fp_trace_read).
struct TraceRec { int tag, stream, slot; };
struct Trace {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  std::vector<TraceRec> recs;
  size_t used = 0;
  int base = -1;
  std::vector<float> t0, t1;   // collected, ms from the base event
  std::vector<int> tags, streams;
};

struct fp_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  fpb::ErrorSink err;

  // sizes
  int64_t N = 0;        // panels == unknowns == control points
  int64_t ld = 0;       // leading dimension of the device matrices (>= N, set by capN)
  int64_t capN = 0;     // matrix buffers hold problems of up to capN unknowns (grow-only)
  int64_t cap_geom = 0; // panel records allocated
  int64_t cap_wake = 0; // wake records allocated
  int64_t nsh = 0;
  int64_t wake_opposite = -1;           // first shedding edge with da . db <= 0, or -1
  bool wake_disjoint = true;   // every wake column touched by one edge only
  bool has_geometry = false;
  int assembled = -1;          // element kind of the assembled G, -1 none
  int assembled_prec = -1;
  int factored = -1;           // FP_PREC_FP64 or FP_PREC_MIXED (either FP32 form) of the factors, -1 none
  bool static_order = false;   // the FP32 factors were formed without pivot search (fp_lu_static.cu)
  int64_t nrhs = 0;
  double kern_offset = 1e-8;   // kerneloffset of the assembled body
  double kern_cutoff = 1e-14;  // kernelcutoff of the assembled body

  // host copies needed for post-processing calls
  std::vector<int32_t> h_offsets, h_pnodes;
  std::vector<double> h_nodes;
  std::vector<int32_t> h_shed;
  std::vector<double> h_Da, h_Db;
  std::vector<double> h_tgt;            // 6 x N SoA copy of d_tgt

  // device buffers
  fpb::PanelRec* d_panels = nullptr;    // N records
  fpb::SourceRec* d_src = nullptr;      // N records (source bodies)
  double* d_tgt = nullptr;              // 6 x N SoA: cx, cy, cz, nx, ny, nz
  WakeRec* d_wake = nullptr;            // nsh records
  double* d_G = nullptr;                // FP64 AIC, ld x N
  double* d_LU = nullptr;               // FP64 factors, ld x N
  float* d_G32 = nullptr;               // FP32 AIC copy / FP32 factors, ld x N
  int32_t* d_ipiv = nullptr;            // N
  double* d_rhs = nullptr;              // N x k (ld)
  double* d_x = nullptr;                // N x k
  double* d_r = nullptr;                // N x k residual (FP64)
  float* d_w32 = nullptr;               // N x k FP32 work
  int* d_status = nullptr;              // device status word(s)
  unsigned int* d_flags = nullptr;      // triangular-solve flags
  unsigned long long* d_mbox = nullptr; // per 128-row block, 128 (epoch, FP32 value) words of the single-RHS sweep
  unsigned trs_epoch = 0;               // epoch of the last sweep launched
  float* d_cert = nullptr;              // max |L| certificate
  unsigned* d_ticket = nullptr;         // ticket of the factorisation's block launches (zero between launches)
  double* d_dinv64 = nullptr;           // inverses of the FP64 diagonal blocks
  float* d_dinv32 = nullptr;            // inverses of the FP32 diagonal blocks
  double* d_dinv128_64 = nullptr;       // inverses of the 128-row diagonal blocks (FP64 factors)
  float* d_dinv128_32 = nullptr;        // inverses of the 128-row diagonal blocks (FP32 factors)
  double* d_mprev64 = nullptr;          // inv(D_bb) T(b, p) of each 128-row block's predecessor, per sweep (FP64)
  float* d_mprev32 = nullptr;           // the same for the FP32 factors
  float* d_mq32 = nullptr;              // two-block sweep chain: R_b = Q_b - P_b P_{b-1} per block and sweep (FP32)
  float* d_ms32 = nullptr;              // S_b = P_b Q_{b-1}
  unsigned long long* d_zbox = nullptr; // the sweeps' second mailbox: z_b words (epoch, value)
  bool trs_skip2 = false;               // FP32 sweeps: the two-block chain (FP_TUNE_TRS2)
  int panel_gemm = 2;                   // static-order FP32 LU: 1 both panel inverses, GEMM-form L21 / U12; 2: inv(L) only, beside k_l21 (FP_TUNE_PANEL_GEMM)
  bool tc_x3 = true;                    // FP32 form: the update from BF16 pairs, three MMAs (FP_TUNE_TC_BF16X3)
  int tc_prefetch = 1;                  // red.global updates: idle warps prefetch the C tile into L2 (FP_TUNE_TC_PREFETCH)
  bool lu_split = true;                 // static-order LU: split panel chain (FP_TUNE_LU_SPLIT)
  bool l21_async = true;                // static-order LU: k_l21 with asynchronous column-major staging (FP_TUNE_L21_ASYNC)
  bool u12_async = false;               // static-order LU: k_u12g stages A12 column-major by cp.async (FP_TUNE_U12_ASYNC)
  bool u12_wide = false;                // static-order LU: U12 of the columns beyond, 64 columns a CTA (FP_TUNE_U12_WIDE)
  bool lu_fuse = false;                 // split chain: U12 and the diagonal tile's update in one kernel (FP_TUNE_LU_FUSE)
  int rest_split = 0;                   // split chain: the trailing update in two row ranges, U12 of the columns beyond on stream4 (FP_TUNE_REST_SPLIT; 2: the first range on stream4 too)
  bool pdl = true;                      // static-order LU: programmatic dependent launch of its kernels (FP_TUNE_PDL)
  bool pdiag_linv = false;              // static-order LU: k_pdiag forms the full inv(L), no k_pinv (FP_TUNE_PDIAG_LINV)
  bool trs2_ready = false;              // R and S formed for the current FP32 factors
  double* d_part = nullptr;             // GEMV partial sums
  void* d_minv = nullptr;               // per block of a panel: M' = inv(L11) P11 (NB x NB, FP64 size), then the row order (NB ints)
  double* d_norms = nullptr;            // column norms (2 x cap_rhs)
  int64_t cap_rhs = 0;                  // allocated RHS columns
  size_t cap_flags = 0;

  // adjoint solves (kept apart from the primal RHS and solution)
  double* d_ab = nullptr;               // N x k adjoint right-hand sides (ld)
  double* d_ax = nullptr;               // N x k adjoint solutions
  double* d_ar = nullptr;               // N x k adjoint residuals
  float* d_aw32 = nullptr;              // N x k FP32 work
  double* d_anorms = nullptr;           // column norms (2 x cap_adj)
  int64_t cap_adj = 0;

  // persistent staging of per-call inputs (fp_set_rhs, fp_uind)
  double* d_stage = nullptr;
  size_t cap_stage = 0;                 // doubles

  // reverse-mode workspace (fp_assembly_vjp / fp_uind_vjp)
  double* d_vjp = nullptr;
  size_t cap_vjp = 0;                   // doubles

  // GMRES workspace
  double* d_V = nullptr;                // (m+1) x ld Krylov basis
  double* d_h = nullptr;                // small vectors
  int cap_gmres_m = 0;

  // timing
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double ms_assemble = 0, ms_factor = 0, ms_solve = 0, ms_uind = 0;
  double kms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int klaunch[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int adj_iters = 0;                    // refinement steps of the last adjoint solve
  double adj_relres = 0;                // its relative residual
  fp_stats last{};
  int64_t nlaunch = 0;          // kernels launched by this context
  KernelTimer ktimer;           // trailing-update launches of fp_factor
  Trace trace;                  // timeline of fp_factor (off by default)
  bool use_tc = true;           // tcgen05 3xTF32 trailing update for the FP32 factors
  int tc_stages = 2;            // ring depth of that update in the static-order LU (fp_set_tuning)
  int tc_tiles = 0;             // static-order LU: output tiles per CTA of the multi-tile update, 0 = one-tile kernel
  int tc_smem = 0;              // static-order LU: shared memory reserved by each one-tile update CTA (0 = its own)
  int tc_split = 0;             // static-order LU: 0 pre-split operands; 1..3 split in shared memory (3, 4, 6 x stages)
  bool tc_red = true;           // static-order LU: the update's epilogue adds to C by red.global instead of TMA
  int tc_narrow_stages = 6;     // ring depth of the update of one column of tiles (6, or 0: as the others)
  int fp64_dmma = 6;            // FP64 LU update: 0 SIMT; FP64 tensor path, variants 1..6 (fp_set_tuning)
  bool lu_overlap = true;       // static-order LU: trailing update on the second stream (fp_set_tuning)
  // The static-order FP32 factorisation replayed as a CUDA graph (both streams,
  // the diagonal-block inverses included): captured on the second call with
  // the same key (the first runs the launches directly and grows the scratch
  // buffers), replayed while the key holds. Off while tracing or timing.
  bool use_graph = false;
  cudaGraphExec_t lu_graph = nullptr;
  std::vector<uintptr_t> lu_graph_key, lu_graph_seen;
  // split operands (Ah, Al, Bh, Bl) of the tensor-core update, one set per
  // stream of the look-ahead factorisation (slot 0: c->stream, 1: stream2)
  float* d_tc[2][4] = {{nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}};
  size_t tc_cap[2] = {0, 0};
  int tc_slot = 0;                      // scratch set of the current launches
  cudaStream_t stream2 = nullptr;       // second stream of the look-ahead factorisation
  cudaStream_t stream3 = nullptr;       // third stream (high priority): the static-order LU's inv(L) beside k_l21
  cudaStream_t stream4 = nullptr;       // fourth stream (high priority): U12 of the columns beyond, beside the trailing update
  cudaStream_t stream_bg = nullptr;     // lowest priority: the FP64 AIC pass under the FP32 factorisation
  cudaEvent_t ev_g64 = nullptr;         // that pass done (stream_bg -> stream)
  cudaEvent_t ev_asm = nullptr;         // assembly inputs ready (stream -> stream_bg)
  bool g64_pending = false;             // the FP64 AIC is still being written on stream_bg
  bool asm32 = false;                   // mixed forms: FP32 AIC pass first, FP64 pass in the background
  std::map<uint64_t, std::vector<int>> tuned;   // fp_autotune: (N, precision) -> knob values
  cudaEvent_t ev_panel = nullptr;       // panel factored (stream -> stream2)
  cudaEvent_t ev_diag = nullptr;        // static-order LU: diagonal block factored (stream -> stream2)
  cudaEvent_t ev_rest = nullptr;        // trailing update done (stream2 -> stream)
  cudaEvent_t ev_pinv = nullptr;        // static-order LU: inv(L) formed (stream3 -> stream, stream2)
  cudaEvent_t ev_u12n = nullptr;        // split panel chain: the next panel's U12 formed (stream -> stream3)
  cudaEvent_t ev_tcr = nullptr;         // split panel chain: the rows below the next panel updated (stream3 -> stream)
  cudaEvent_t ev_l21t = nullptr;        // split panel chain: L21 of the rows below the next panel (stream3 -> stream2)
  cudaEvent_t ev_top = nullptr;         // trailing update of the next panel's rows done (stream2 -> stream, stream4)
  cudaEvent_t ev_u12r = nullptr;        // U12 of the columns beyond formed (stream4 -> stream2)

  // surface post-processing (fp_post.cu). The mesh topology of a triangular
  // body is built on first use after fp_set_geometry, the Kutta-average
  // tables on first use after fp_set_wake.
  bool topo_valid = false;
  bool kutta_valid = false;
  int64_t topo_nnodes = 0;
  int32_t* d_nb = nullptr;              // 3 x N (AoS): cell across edge k (local nodes k -> k+1), -1 at a free edge
  int32_t* d_voff = nullptr;            // nnodes + 1: CSR of the cells around each node (ascending)
  int32_t* d_vcell = nullptr;           // 3N
  double* d_area = nullptr;             // N panel areas
  int32_t* d_teflag = nullptr;          // N: times the cell is a shedding pi/pj (low 16 bits), bit 16 = forced cell value
  int32_t* d_krow = nullptr;            // nsh x 4 slots of (pi, pi+1, pj, pj-1) in d_kcell, -1 absent
  // sharp trailing edge (node scheme): the trailing-edge node slot of each
  // node (-1 if none), and per slot the upper (pi, pi+1) and lower (pj, pj-1)
  // cells that contain it, as two CSR lists
  int32_t* d_teslot = nullptr;          // topo_nnodes
  int32_t* d_tecsr = nullptr;           // [up offsets (nte+1)] [up cells] [lo offsets (nte+1)] [lo cells]
  int64_t nte = 0, te_up_cells = 0, te_lo_cells = 0;
  int32_t* d_kcell = nullptr;           // distinct cells of the Kutta rows
  int32_t* d_klast = nullptr;           // per distinct cell: the last row that overwrites its force
  int64_t nkcell = 0;
  double* d_post = nullptr;             // post-processing work (fields of N cells and the nodes)
  double* d_uscr = nullptr;             // partial sums of the chunked induced-velocity kernels
  size_t cap_uscr = 0;                  // doubles
  size_t cap_post = 0;                  // doubles
};

namespace fpb {

// assembly (fp_assembly.cu)
int launch_assemble_ring(fp_ctx* c, double offset, double cutoff, bool write32, cudaStream_t s = nullptr);
// the FP32 AIC (G32) alone, the ring in panel-local FP32 coordinates
int launch_assemble_ring32(fp_ctx* c, double offset, double cutoff);
int launch_assemble_source(fp_ctx* c, double offset, bool write32);
int launch_rhs(fp_ctx* c, const double* d_U, int64_t k);

// dense linear algebra (fp_lu.cu)
template <class T>
int lu_factor(fp_ctx* c, T* A, int64_t n, int64_t lda, int32_t* ipiv, float* cert_max_L);
template <class T>
int lu_solve(fp_ctx* c, const T* LU, int64_t n, int64_t lda, const int32_t* ipiv, T* B,
             int64_t ldb, int64_t k, bool transpose);
int gemv_residual(fp_ctx* c, const double* A, int64_t n, int64_t lda, const double* x,
                  const double* b, double* r, int64_t k);
// r = b - A^T x (FP64); x, b, r share the leading dimension lda
int gemvT_residual(fp_ctx* c, const double* A, int64_t n, int64_t lda, const double* x,
                   const double* b, double* r, int64_t k);
int convert_f64_f32(fp_ctx* c, const double* a, float* b, int64_t n, int64_t k, int64_t lda,
                    int64_t ldb);
int axpy_f32_to_f64(fp_ctx* c, const float* d, double* x, int64_t n, int64_t k, int64_t ld);
int axpy_f64(fp_ctx* c, const double* d, double* x, int64_t n, int64_t k, int64_t ld);
template <class T>
int lu_diag_inverses(fp_ctx* c, const T* LU, int64_t n, int64_t lda);
// FP64 solve with the context's factors on caller memory, flags of the
// triangular solves in a static device array (no device allocation)
int lu_solve_noalloc(fp_ctx* c, double* B, int64_t ldb, int64_t k);
int colnorm2(fp_ctx* c, const double* a, int64_t n, int64_t lda, int64_t k, double* d_out);
constexpr int kLuNB = 64;        // block size of the factorisation and the solves
constexpr int kOuterPanel = 256;  // columns per outer panel of the factorisation
constexpr int kPanelSlots = kOuterPanel / kLuNB;   // blocks per outer panel
// two sets of the pivoted LU's block inverses, or two panel slots of the
// static-order LU (its 32 x 32 inverses and the full 128 x 128 inverses)
constexpr size_t kMinvBytes = std::max((size_t)2 * kPanelSlots * kLuNB * kLuNB * sizeof(double),
                                       (size_t)2 * (8 * 32 * 32 + 2 * 128 * 128) * sizeof(float));
// split-operand scratch of the tensor-core update for scratch set `slot` (fp_tc.cu)
int ensure_tc_scratch(fp_ctx* c, int slot, int64_t rows_max);
constexpr int kGemvSplitHost = 16;
// FP32 LU with a static row order (no pivot search) for the mixed form
// (fp_lu_static.cu): panels of kStaticPanel columns, identity ipiv, max|L| in
// cert; DEV_ZERO_PIVOT in the status word on a zero or non-finite pivot
constexpr int kStaticPanel = 128;
// bf16: the trailing update multiplies BF16 operands (kind::f16, FP32 accumulation)
int lu_factor_static(fp_ctx* c, float* A, int64_t n, int64_t lda, int32_t* ipiv, float* cert, bool bf16 = false);
bool tc_gemm_sub_bf16(fp_ctx* c, const void* Ah, const void* Bh, int ldk, float* C, int64_t ldc, int64_t m,
                      int64_t nn, int kk);
bool tc_gemm_sub_bf16x3(fp_ctx* c, const void* Ah, const void* Al, const void* Bh, const void* Bl, int ldk, float* C,
                        int64_t ldc, int64_t m, int64_t nn, int kk);
// b = FP32 copy of the FP64 a rounded to BF16 values
int convert_f64_bf16(fp_ctx* c, const double* a, float* b, int64_t n, int64_t k, int64_t lda, int64_t ldb);
// FP32 trailing update on tensor cores (fp_tc.cu); returns false if the
// shape is not supported, in which case the SIMT kernel runs.
bool tc_gemm_sub_f32(fp_ctx* c, const float* A, const float* B, float* C, int64_t lda, int64_t m,
                     int64_t nn, int kk);
// The same from operands already split into 3xTF32 hi / lo parts, K-major
// with ldk floats per row (Ah, Al: m rows; Bh, Bl: nn columns); C column-major (ldc).
bool tc_gemm_sub_presplit(fp_ctx* c, const float* Ah, const float* Al, const float* Bh, const float* Bl, int ldk,
                          float* C, int64_t ldc, int64_t m, int64_t nn, int kk);
// C -= A B from unsplit FP32 K-major operands (Ax: m rows, Bx: nn columns,
// ldk floats a row); the 3xTF32 split is done in shared memory
bool tc_gemm_sub_xsplit(fp_ctx* c, const float* Ax, const float* Bx, int ldk, float* C, int64_t ldc, int64_t m,
                        int64_t nn, int kk);
// C -= A B on the SIMT pipe (FP32), all three blocks of one matrix (lda)
int gemm_sub_simt_f32(fp_ctx* c, const float* A, const float* B, float* C, int64_t lda, int64_t m, int64_t nn,
                      int kk);

// induced velocity (fp_field.cu)
int launch_uind_ring(fp_ctx* c, const double* d_strength, const double* d_targets, int64_t m,
                     double* d_out, bool fp32);
int ensure_stage(fp_ctx* c, size_t n);   // the staging buffer holds at least n doubles
// least squares of a watertight vortex-ring body (fp_ls.cu): Gamma_red of the
// normal equations with the prescribed columns (sorted, distinct) removed
int ls_solve(fp_ctx* c, const int* h_el, const double* h_val, int npres, double* h_gamma_red);
int launch_phi(fp_ctx* c, const double* d_sigma, const double* d_mu, const double* d_targets, int64_t m,
               double* d_out, bool wake);
int launch_uind_source(fp_ctx* c, const double* d_strength, const double* d_targets, int64_t m,
                       double* d_out);
// surface post-processing (fp_post.cu)
void post_free(fp_ctx* c);

// reverse mode of the pair kernels (fp_vjp.cu)
int launch_pair_vjp(fp_ctx* c, const double* d_strength, const double* d_x, const double* d_w,
                    int64_t m, double* d_gX, double* d_U, double* d_gvert, double* d_gs,
                    double* d_gwake);
int launch_vjp_cotangent(fp_ctx* c, const double* d_lambda, double* d_w);
constexpr int kWakeGradHost = 20;   // per shedding edge: pa, pb, qa, qb, da, db, s_pi, s_pj

// GMRES (fp_gmres.cu)
int gmres_solve(fp_ctx* c, const double* b, double* x, int64_t k, const fp_solve_opts& o,
                bool precondition, int* iters, double* relres);

int num_sms();

// Raises a kernel's dynamic shared-memory limit once per device. Thread-safe:
// a repeated call from a racing thread only sets the same value again.
constexpr int kTcSmemMax = 232448;   // the opt-in shared memory of one CTA on sm_100

// Orders the context's stream after the background FP64 assembly pass, once;
// every reader of the FP64 AIC (or writer of a new one) calls it first.
inline int sync_g64(fp_ctx* c);

struct SmemAttr {
  std::atomic<unsigned long long> done{0};
  template <class K>
  cudaError_t ensure(K* kernel, int bytes) {
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_release);
    return e;
  }
};

// Launches kernel on stream s, with programmatic dependent launch when pdl:
// the launch may begin before the stream's previous kernel has finished, and
// the kernel's griddep_wait() holds it until that kernel's results are
// visible. Only kernels that call griddep_wait() before reading what their
// predecessors wrote may be launched with pdl.
template <class... KArgs, class... Args>
inline cudaError_t launch_k(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? at : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Routes the launches of a section to stream s (tensor-core scratch unchanged).
struct OnStream {
  fp_ctx* c;
  cudaStream_t s0;
  OnStream(fp_ctx* c_, cudaStream_t s) : c(c_), s0(c_->stream) { c->stream = s; }
  ~OnStream() { c->stream = s0; }
};

// Routes the launches of a section to stream2 and its tensor-core scratch.
struct OnStream2 {
  fp_ctx* c;
  cudaStream_t s0;
  int slot0;
  explicit OnStream2(fp_ctx* c_) : c(c_), s0(c_->stream), slot0(c_->tc_slot) {
    c->stream = c->stream2;
    c->tc_slot = 1;
  }
  ~OnStream2() {
    c->stream = s0;
    c->tc_slot = slot0;
  }
};

// KernelTimer: kt_begin records the start event of a launch (returns its
// slot, or -1 when timing is off or an event cannot be made), kt_end the stop
// event and the launch's algorithmic flops; kt_collect sums the elapsed times
// after the stream has been synchronised.
inline int kt_begin(fp_ctx* c) {
  KernelTimer& t = c->ktimer;
  if (!t.on) return -1;
  while (t.pool.size() < t.used + 2) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    t.pool.push_back(e);
  }
  const int slot = (int)t.used;
  cudaEventRecord(t.pool[slot], c->stream);
  t.used += 2;
  return slot;
}
inline void kt_end(fp_ctx* c, int slot, double flops, double elems) {
  if (slot < 0) return;
  cudaEventRecord(c->ktimer.pool[slot + 1], c->stream);
  c->ktimer.work.push_back(flops);
  c->ktimer.elems.push_back(elems);
}
inline void kt_collect(fp_ctx* c) {
  KernelTimer& t = c->ktimer;
  for (size_t s = 0; s + 1 < t.used; s += 2) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, t.pool[s], t.pool[s + 1]) == cudaSuccess) t.ms += ms;
    t.flops += t.work[s / 2];
    t.units += t.elems[s / 2];
    ++t.launches;
  }
  t.used = 0;
  t.work.clear();
  t.elems.clear();
}

// Trace: tr_event records one event on the current stream and returns its
// slot (-1 when tracing is off); TraceScope brackets one launch.
enum TraceTag { TR_DIAG = 0, TR_L21 /* k_blk */, TR_U12 /* k_pfix */, TR_STRIP, TR_GEMM_TC, TR_SPLIT_A, TR_SPLIT_B, TR_GEMM_SIMT, TR_PINV };
inline int tr_event(fp_ctx* c) {
  Trace& t = c->trace;
  if (!t.on) return -1;
  if (t.pool.size() < t.used + 1) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    t.pool.push_back(e);
  }
  const int s = (int)t.used++;
  cudaEventRecord(t.pool[s], c->stream);
  return s;
}
struct TraceScope {
  fp_ctx* c;
  int tag, s;
  TraceScope(fp_ctx* c_, int tag_) : c(c_), tag(tag_), s(tr_event(c_)) {}
  ~TraceScope() {
    if (s < 0) return;
    const int e = tr_event(c);
    if (e < 0) return;
    c->trace.recs.push_back(TraceRec{tag, c->stream == c->stream2 ? 1 : (c->stream == c->stream3 ? 2 : (c->stream == c->stream4 ? 3 : 0)), s});
  }
};
inline void tr_collect(fp_ctx* c) {
  Trace& t = c->trace;
  t.t0.clear(); t.t1.clear(); t.tags.clear(); t.streams.clear();
  if (!t.on || t.base < 0) return;
  for (const TraceRec& r : t.recs) {
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, t.pool[t.base], t.pool[r.slot]);
    cudaEventElapsedTime(&b, t.pool[t.base], t.pool[r.slot + 1]);
    t.t0.push_back(a); t.t1.push_back(b); t.tags.push_back(r.tag); t.streams.push_back(r.stream);
  }
  t.recs.clear();
  t.used = 0;
  t.base = -1;
}
inline int sync_g64(fp_ctx* c) {
  if (!c->g64_pending) return FP_OK;
  c->g64_pending = false;
  FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_g64, 0));
  return FP_OK;
}

}  // namespace fpb
