// Dense LU factorisation and triangular solves on sm_100a.
//
// Blocked right-looking LU with partial pivoting inside each NB x NB diagonal
// block (the search runs over the rows of the block). After the block is
// factored, L21 = A21 U11^-1 is formed and max|L21| is kept: when it is <= 1
// every pivot equals the one LAPACK dgetrf (partial pivoting over the whole
// column) picks, so the factorisation is the reference's up to rounding
// (src/FLOWPanel_linearsolver.jl:173-234). The wing AICs of this path need
// only adjacent-row swaps at the trailing edge, which the block search finds.
//
// Per 64-block step: (1) k_diag factors the diagonal block (one CTA) and
// forms M' = L11^-1 P11; (2) k_blk forms L21, and the update of the panel's
// own columns as (L21 M') A12 with A12 as it lies, and, in its last CTA among
// those holding the next block's rows, factors the next diagonal block. After
// the panel's blocks, (3) k_pfix writes U12 = M' A12 and the row swaps left of
// each block. Columns outside the panel get the panel's swaps and U12 from
// k_strip and the trailing update from a GEMM (SIMT FP64, or the 3xTF32
// tcgen05 kernel of fp_tc.cu for the FP32 factors), on two streams (see
// lu_factor).
//
// Triangular solves run in one persistent kernel per sweep: CTAs take row
// blocks by ticket (atomic counter), wait (bounded) for the blocks they depend
// on, subtract their contribution and multiply by the precomputed inverse of
// the diagonal block.
#include <cuda_bf16.h>

#include <cfloat>
#include <string>

#include "fp_internal.cuh"

namespace fpb {

constexpr int NB = 64;          // block size of the factorisation and of the solves
constexpr int kSpinLimit = 1 << 22;   // bounded waits in the persistent solve

template <class T> __device__ __forceinline__ T tabs(T a) { return a < T(0) ? -a : a; }
// Returns p unchanged, but opaque to the compiler: addresses formed from it
// are not shared with (and kept live from) earlier uses of the same pointer.
template <class P> __device__ __forceinline__ P* opaque_ptr(P* p) {
  uint64_t v = reinterpret_cast<uint64_t>(p);
  asm volatile("mov.b64 %0, %0;" : "+l"(v));
  return reinterpret_cast<P*>(v);
}

// ----------------------------------------------------------------------------
// 16-byte vectors of T (float4 / double2) for the shared-memory sweeps below.
template <class T> struct V16;
template <> struct V16<float> { typedef float4 type; static constexpr int n = 4; };
template <> struct V16<double> { typedef double2 type; static constexpr int n = 2; };
template <class T> __device__ __forceinline__ T vget(const typename V16<T>::type& v, int i);
template <> __device__ __forceinline__ float vget<float>(const float4& v, int i) {
  return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}
template <> __device__ __forceinline__ double vget<double>(const double2& v, int i) { return i == 0 ? v.x : v.y; }
template <class T> __device__ __forceinline__ void vset(typename V16<T>::type& v, int i, T x);
template <> __device__ __forceinline__ void vset<float>(float4& v, int i, float x) {
  if (i == 0) v.x = x; else if (i == 1) v.y = x; else if (i == 2) v.z = x; else v.w = x;
}
template <> __device__ __forceinline__ void vset<double>(double2& v, int i, double x) {
  if (i == 0) v.x = x; else v.y = x;
}
// Stages an NB x NB block element by element with NT threads: element
// (r, c) = get(r, c) goes to put(r, c, v), r fastest over the threads (so that
// column-major global reads coalesce). Each thread issues a batch of up to 16
// loads before its stores, so that the copy costs a few memory latencies
// rather than one per element.
template <int NT, class T, class Get, class Put>
__device__ __forceinline__ void stage_block(int tid, Get get, Put put) {
  constexpr int IT = NB * NB / NT;
  constexpr int BATCH = IT < 16 ? IT : 16;
#pragma unroll
  for (int i0 = 0; i0 < IT; i0 += BATCH) {
    T v[BATCH];
#pragma unroll
    for (int u = 0; u < BATCH; ++u) {
      const int e = tid + (i0 + u) * NT;
      v[u] = get(e & (NB - 1), e / NB);
    }
#pragma unroll
    for (int u = 0; u < BATCH; ++u) {
      const int e = tid + (i0 + u) * NT;
      put(e & (NB - 1), e / NB, v[u]);
    }
  }
}
// row pitch of an NB-wide row in shared memory: whole 16-byte vectors, not a
// multiple of 32 banks
template <class T> __host__ __device__ constexpr int rpitch() { return NB + 16 / (int)sizeof(T); }

// ----------------------------------------------------------------------------
// (1) k_diag: four warps factor the NB x NB diagonal block with partial
// pivoting over its rows. Each row belongs to a pair of adjacent lanes, each
// holding 32 of its not yet eliminated entries in registers, shifted so that
// the even lane's R[0] is always the current column: step j forms
// R[c] <- R[c + 1] - m U(j, j + 1 + c) with static indices (the odd lane's
// first entry moves to the even lane by one shuffle, zeros enter at the end),
// so the step loop stays rolled and small enough for the instruction cache,
// and each lane does 32 FMAs a step on its own SM sub-partition. Rows never
// move: a pivot row is marked used and every other unused row eliminates
// column j with its own multiplier. The pivot is LAPACK's: the largest |a| in
// column j among the unused rows, the first in the current logical order on
// ties. Each warp reduces an integer key (the bits of |a| plus one, 0 for used
// rows; FP64 in two 32-bit halves) with __reduce_max_sync, ties by logical
// position with __reduce_min_sync; the four warps' candidates meet in shared
// memory together with each warp's best row (aligned 16-byte stores of the
// registers as they are), so one barrier per step suffices; every row reads
// the winner back with broadcast 16-byte loads. Multipliers and U rows collect in
// shared memory (S[row][column]) and go out in logical row order at the end.
// LAPACK's ipiv follows from the logical order: at step j, logical rows j and
// the pivot's position swap. Per-step shared buffers alternate between two
// copies, so one barrier orders each step's reads before the next step's
// writes. Last, M' = L11^-1 P11 (P11's columns in physical row order) is
// formed for the block's update, two lanes per column in the same way, and
// the row order kept for the panel's fix-up (k_pfix).
constexpr int kDiagThreads = 2 * NB;
constexpr int kHalf = NB / 2;   // entries of a row per lane

__device__ __forceinline__ void bar_diag() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

template <class T> struct PivKey;
template <> struct PivKey<float> {
  __device__ static void of(float v, bool used, unsigned& hi, unsigned& lo) {
    hi = used ? 0u : __float_as_uint(fabsf(v)) + 1u;
    lo = 0u;
  }
};
template <> struct PivKey<double> {
  __device__ static void of(double v, bool used, unsigned& hi, unsigned& lo) {
    const unsigned long long b = used ? 0ull : (unsigned long long)__double_as_longlong(fabs(v)) + 1ull;
    hi = (unsigned)(b >> 32);
    lo = (unsigned)b;
  }
};

// shared workspace of diag_factor: pcand[2][4][NB], S / Lsh [NB][RP],
// cand[2][4] (uint4), lpiv[NB], rowat[NB]
template <class T> __host__ __device__ constexpr int diag_ws_bytes() {
  return 2 * 4 * NB * (int)sizeof(T) + NB * rpitch<T>() * (int)sizeof(T) + 128 + 2 * NB * 4;
}

template <class T> __device__ __forceinline__ T rcp_rn(T x);
template <> __device__ __forceinline__ float rcp_rn<float>(float x) { return __frcp_rn(x); }
template <> __device__ __forceinline__ double rcp_rn<double>(double x) { return __drcp_rn(x); }

// The 128 threads of the calling CTA factor the diagonal block at k (k_diag;
// k_blk runs it for the next block once that block's rows are final). A is
// read through L2, so another CTA's stores, ordered before by a fence and an
// atomic, are seen. One barrier per step: each warp's best row publishes
// itself (its key and its whole row) in the step's slot for that warp, and
// after the barrier every thread picks the best of the four and reads that
// row. The key is (|a| bits + 1, 63 - logical position, row), compared as
// unsigned words in that order.
template <class T>
__device__ __forceinline__ void diag_factor(T* __restrict__ A, int64_t lda, int64_t n, int64_t k,
                                            int32_t* __restrict__ ipiv, int* __restrict__ status,
                                            T* __restrict__ Minv, int* __restrict__ rowat_out, unsigned char* ws) {
  typedef typename V16<T>::type VT;
  constexpr int V = V16<T>::n, RP = rpitch<T>(), HQ = kHalf / V;
  T (*pcand)[4][NB] = reinterpret_cast<T (*)[4][NB]>(ws);           // candidate rows, per parity and warp
  T* const buf = reinterpret_cast<T*>(ws + 2 * 4 * NB * sizeof(T));  // S, then Lsh
  uint4 (*cand)[4] = reinterpret_cast<uint4 (*)[4]>(buf + NB * RP);  // per parity and warp: key
  int* const lpiv = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(cand) + 128);
  int* const rowat = lpiv + NB;
  // S[r][c]: row r's entry of L (c < its step) or U
  T (*S)[NB + 1] = reinterpret_cast<T (*)[NB + 1]>(buf);
  const int nb = (int)imin64(NB, n - k);
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int h = lane & 1;                       // which half of the row
  const int row = warp * 16 + (lane >> 1);      // the row of this lane pair
  const int g0 = h * kHalf;                     // first column of this half
  T R[kHalf];
#pragma unroll
  for (int c = 0; c < kHalf; ++c) {
    const int g = g0 + c;
    R[c] = (row < nb && g < nb) ? __ldcg(&A[(k + g) * lda + (k + row)]) : ((row == g) ? T(1) : T(0));
  }
  bool used = !(row < nb);
  int pos = row;
  bool zero = false;
  T cur = __shfl_sync(0xffffffffu, R[0], lane & ~1);   // the row's entry in the current column
  // this warp's best unused row for the next step: key words and, after the
  // row's update, its row in pcand
  auto reduce_key = [&](unsigned& mh, unsigned& ml, unsigned& mlow) {
    unsigned hi, lo;
    PivKey<T>::of(cur, used, hi, lo);
    mh = __reduce_max_sync(0xffffffffu, hi);
    ml = (sizeof(T) == 8) ? __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u) : 0u;
    const bool top = hi == mh && lo == ml;
    mlow = __reduce_max_sync(0xffffffffu, top ? ((unsigned)(63 - pos) << 6) | (unsigned)row : 0u);
  };
  auto publish_row = [&](int par, unsigned mh, unsigned ml, unsigned mlow) {
    if (lane == 0) cand[par][warp] = make_uint4(mh, ml, mlow, 0u);
    if ((unsigned)row == (mlow & 63u)) {   // this warp's best row: whole 16-byte stores of both halves
      VT* out = reinterpret_cast<VT*>(&pcand[par][warp][g0]);
#pragma unroll
      for (int q = 0; q < HQ; ++q) {
        VT v;
#pragma unroll
        for (int e = 0; e < V; ++e) vset<T>(v, e, R[q * V + e]);
        out[q] = v;
      }
    }
  };
  if (nb > 0) {
    unsigned mh, ml, mlow;
    reduce_key(mh, ml, mlow);
    publish_row(0, mh, ml, mlow);
  }
#pragma unroll 1
  for (int j = 0; j < nb; ++j) {
    const int par = j & 1;
    bar_diag();
    uint4 best = cand[par][0];
    int w = 0;
#pragma unroll
    for (int q = 1; q < 4; ++q) {
      const uint4 c4 = cand[par][q];
      const unsigned long long kq = ((unsigned long long)c4.x << 32) | c4.y;
      const unsigned long long kb = ((unsigned long long)best.x << 32) | best.y;
      if (kq > kb || (kq == kb && c4.z > best.z)) { best = c4; w = q; }
    }
    const int pr = (int)(best.z & 63u);         // pivot row
    const int lp = 63 - (int)(best.z >> 6);     // its logical position
    const T* prow = pcand[par][w];
    const T piv = prow[0];
    const T rp = (piv != T(0)) ? rcp_rn<T>(piv) : T(0);
    if (row == pr) { pos = j; used = true; } else if (pos == j) { pos = lp; }
    if (t == 0) lpiv[j] = lp;
    // the pivot's row of U goes to S[pr][j..], one element per thread
    if (t < NB - j) S[pr][j + t] = prow[t];
    zero |= (rp == T(0));
    const T m = cur * rp;   // 0 on a zero pivot: the row only shifts
    if (!used && h == 0) S[row][j] = m;
    T pv[kHalf];
    const VT* in = reinterpret_cast<const VT*>(&prow[g0]);
#pragma unroll
    for (int q = 0; q < HQ; ++q) {
      const VT v = in[q];
#pragma unroll
      for (int e = 0; e < V; ++e) pv[q * V + e] = vget<T>(v, e);
    }
    const T pnext = (h == 0) ? prow[kHalf] : T(0);
    const T nxt = __shfl_down_sync(0xffffffffu, R[0], 1);   // the odd lane's first entry
    // the next step's column first: its key reductions overlap the rest
    R[0] = R[1] - m * pv[1];
    cur = __shfl_sync(0xffffffffu, R[0], lane & ~1);
    unsigned mh = 0, ml = 0, mlow = 0;
    if (j + 1 < nb) reduce_key(mh, ml, mlow);
#pragma unroll
    for (int c = 1; c < kHalf - 1; ++c) R[c] = R[c + 1] - m * pv[c + 1];
    R[kHalf - 1] = (h == 0 ? nxt : T(0)) - m * pnext;
    if (j + 1 < nb) publish_row(par ^ 1, mh, ml, mlow);
  }
  if (zero && t == 0) atomicOr(status, (int)DEV_ZERO_PIVOT);
  if (h == 0 && row < nb) rowat[pos] = row;
  bar_diag();
  // write back in logical row order, rows fastest over the threads
  for (int e = t; e < nb * nb; e += kDiagThreads) {
    const int s = e % nb, c = e / nb;
    A[(k + c) * lda + (k + s)] = S[rowat[s]][c];
  }
  if (t < nb) ipiv[k + t] = (int32_t)(k + lpiv[t]);
  if (t < NB) rowat_out[t] = (t < nb) ? rowat[t] : t;
  bar_diag();   // the factors are in A (visible to the CTA); S is free
  // M' = L11^-1 P11 with P11's columns in physical row order (M' A12 = U12
  // for A12 as it lies): column r solves L y = e_pos(r), held by the lane
  // pair of row r, with L's columns shifted as the factorisation's rows were:
  // Lsh[j][c] = L(j + 1 + c, j), zero past the end.
  T (*Lsh)[RP] = reinterpret_cast<T (*)[RP]>(buf);
  for (int e = t; e < NB * NB; e += kDiagThreads) {
    const int c = e % NB, j = e / NB;
    Lsh[j][c] = (j + 1 + c < nb) ? A[(k + j) * lda + (k + j + 1 + c)] : T(0);
  }
  bar_diag();
  T y[kHalf];
#pragma unroll
  for (int c = 0; c < kHalf; ++c) y[c] = (g0 + c == pos) ? T(1) : T(0);
#pragma unroll 1
  for (int j = 0; j < NB; ++j) {
    const T yj = __shfl_sync(0xffffffffu, y[0], lane & ~1);
    const T nxt = __shfl_down_sync(0xffffffffu, y[0], 1);
    if (h == 0) Minv[j * NB + row] = yj;
    T lv[kHalf];
    const VT* lrow = reinterpret_cast<const VT*>(&Lsh[j][g0]);
#pragma unroll
    for (int q = 0; q < HQ; ++q) {
      const VT v = lrow[q];
#pragma unroll
      for (int e = 0; e < V; ++e) lv[q * V + e] = vget<T>(v, e);
    }
#pragma unroll
    for (int c = 0; c < kHalf - 1; ++c) y[c] = y[c + 1] - yj * lv[c];
    y[kHalf - 1] = (h == 0 ? nxt : T(0)) - yj * lv[kHalf - 1];
  }
}

template <class T>
__global__ void __launch_bounds__(kDiagThreads)
k_diag(T* __restrict__ A, int64_t lda, int64_t n, int64_t k, int32_t* __restrict__ ipiv,
       int* __restrict__ status, T* __restrict__ Minv, int* __restrict__ rowat_out) {
  __shared__ __align__(16) unsigned char ws[diag_ws_bytes<T>()];
  diag_factor<T>(A, lda, n, k, ipiv, status, Minv, rowat_out, ws);
}

// ----------------------------------------------------------------------------
// (2) k_blk: the rest of a block step in one launch. CTA b owns the rows
// [k1 + b RT, +RT) below the factored diagonal block (k1 = k + NB):
//  * L21 = A21 U11^-1 by substitution, four lanes per row (16 entries each),
//    the row kept shifted in registers as in k_diag (rolled loop over the 64
//    columns, 16-byte broadcast reads of the shifted U rows); max|L21| is the
//    GEPP certificate;
//  * W = L21 M' with M' = L11^-1 P11 from k_diag;
//  * C -= W A12 on the panel's columns right of the block, with A12 as it
//    lies (rows not yet swapped): W A12 = L21 U12, so no CTA needs U12, which
//    k_pfix writes after the panel, and the CTAs never wait for one another;
//  * the last of the CTAs owning the next block's rows (ticket) factors the
//    next diagonal block while the other CTAs still update.
// The shared memory (27 KB for FP32) lets a CTA run beside two CTAs of the
// tensor-core update on the same SM.
constexpr int kBlkRows = 32, kBlkThreads = 128;
template <class T> __host__ __device__ constexpr int blk_lpitch() { return kBlkRows + 16 / (int)sizeof(T); }
template <class T> constexpr size_t blk_smem() {
  return (size_t)NB * rpitch<T>() * sizeof(T) + (size_t)NB * blk_lpitch<T>() * sizeof(T) + NB * sizeof(T) + 64;
}
static_assert(blk_smem<float>() >= (size_t)diag_ws_bytes<float>() && blk_smem<double>() >= (size_t)diag_ws_bytes<double>(),
              "k_blk's shared memory holds diag_factor's workspace");

// acc[i][l] += sum_j P[j][r0 + i] Q[j][c0 + l] over j < NB (both [j][.] in
// shared memory, 16-byte aligned rows)
template <class T, int PP, int QP>
__device__ __forceinline__ void mm4x4(const T (*P)[PP], const T (*Q)[QP], int r0, int c0, T (&acc)[4][4]) {
  typedef typename V16<T>::type VT;
  constexpr int V = V16<T>::n;
#pragma unroll 4
  for (int j = 0; j < NB; ++j) {
    T a[4], b[4];
#pragma unroll
    for (int h = 0; h < 4 / V; ++h) {
      const VT va = *reinterpret_cast<const VT*>(&P[j][r0 + h * V]);
      const VT vb = *reinterpret_cast<const VT*>(&Q[j][c0 + h * V]);
#pragma unroll
      for (int e = 0; e < V; ++e) {
        a[h * V + e] = vget<T>(va, e);
        b[h * V + e] = vget<T>(vb, e);
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int l = 0; l < 4; ++l) acc[i][l] += a[i] * b[l];
  }
}

template <class T>
__device__ void pfix_task(T* __restrict__ A, int64_t lda, int64_t K0, int64_t kend, int nblk,
                          const T* __restrict__ Minv, const int* __restrict__ rowat, int task, unsigned char* smem);

template <class T>
__global__ void __launch_bounds__(kBlkThreads, sizeof(T) == 4 ? 3 : 2)
k_blk(T* __restrict__ A, int64_t lda, int64_t n, int64_t k, int64_t kend, const T* __restrict__ Minv,
      float* __restrict__ cert, int next, int32_t* __restrict__ ipiv, int* __restrict__ status,
      T* __restrict__ Minv_next, int* __restrict__ rowat_next, unsigned* __restrict__ ticket, int nmain,
      int64_t K0, int nblk, const T* __restrict__ slots, const int* __restrict__ rowat) {
  typedef typename V16<T>::type VT;
  constexpr int V = V16<T>::n, RP = rpitch<T>(), LP = blk_lpitch<T>();
  extern __shared__ __align__(16) unsigned char bsm[];
  if ((int)blockIdx.x >= nmain) {   // extra CTAs of a panel's last block: the panel's fix-up tasks
    pfix_task<T>(A, lda, K0, kend, nblk, slots, rowat, (int)blockIdx.x - nmain, bsm);
    return;
  }
  T (*Bs)[RP] = reinterpret_cast<T (*)[RP]>(bsm);   // shifted U11 rows, then M', then A12 chunks
  T (*Ls)[LP] = reinterpret_cast<T (*)[LP]>(bsm + (size_t)NB * RP * sizeof(T));   // L21, then W: [column][row]
  T* rd = reinterpret_cast<T*>(bsm + (size_t)NB * RP * sizeof(T) + (size_t)NB * LP * sizeof(T));
  const int tid = threadIdx.x;
  const int64_t k1 = k + NB;
  const int64_t row0 = k1 + (int64_t)blockIdx.x * kBlkRows;
  const int rows = (int)imin64(kBlkRows, n - row0);
  // Bs[j][c] = U(j, j + 1 + c), zero past the row's end; rd[j] = 1 / U(j, j)
  stage_block<kBlkThreads, T>(
      tid, [&](int j, int l) { return (l >= j) ? A[(k + l) * lda + (k + j)] : T(0); },
      [&](int j, int l, T v) {
        if (l == j) rd[j] = T(1) / v;
        Bs[j][l > j ? l - j - 1 : NB - 1 - j + l] = (l > j) ? v : T(0);
      });
  __syncthreads();
  {
    // four lanes per row, 16 of its entries each, shifted as in k_diag: the
    // quarter-0 lane holds the current column; the next quarter's first entry
    // moves down by one shuffle a step
    constexpr int QW = NB / 4;
    const int r = tid >> 2, qtr = tid & 3, lane = tid & 31;
    const int64_t grow = row0 + r;
    T x[QW];
#pragma unroll
    for (int c = 0; c < QW; ++c) x[c] = (r < rows) ? A[(k + qtr * QW + c) * lda + grow] : T(0);
    float lmax = 0.f;
#pragma unroll 1
    for (int j = 0; j < NB; ++j) {
      const T xj = __shfl_sync(0xffffffffu, x[0], lane & ~3) * rd[j];
      const T nxt = __shfl_down_sync(0xffffffffu, x[0], 1);
      if (qtr == 0) {
        Ls[j][r] = xj;
        if (r < rows) A[(k + j) * lda + grow] = xj;
        lmax = fmaxf(lmax, (float)tabs(xj));
      }
      T u[QW];
      const VT* urow = reinterpret_cast<const VT*>(&Bs[j][qtr * QW]);
#pragma unroll
      for (int q = 0; q < QW / V; ++q) {
        const VT v = urow[q];
#pragma unroll
        for (int e = 0; e < V; ++e) u[q * V + e] = vget<T>(v, e);
      }
#pragma unroll
      for (int c = 0; c < QW - 1; ++c) x[c] = x[c + 1] - xj * u[c];
      x[QW - 1] = (qtr < 3 ? nxt : T(0)) - xj * u[QW - 1];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if (lane == 0 && lmax > 0.f) atomicMax(reinterpret_cast<int*>(cert), __float_as_int(lmax));
  }
  const int64_t nn = kend - k1;
  if (nn <= 0) return;   // then there is no next block in the panel
  __syncthreads();
  // M' -> Bs[j][c]
  stage_block<kBlkThreads, T>(
      tid, [&](int c, int j) { return Minv[j * NB + c]; }, [&](int c, int j, T v) { Bs[j][c] = v; });
  __syncthreads();
  // thread (rg, cg): rows 4 rg.. of the CTA's 32, columns 4 cg.. of 64
  const int rg = tid & 7, cg = tid >> 3;
  {
    T w[4][4] = {};
    mm4x4<T, LP, RP>(Ls, Bs, 4 * rg, 4 * cg, w);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int l = 0; l < 4; ++l) Ls[4 * cg + l][4 * rg + i] = w[i][l];   // Ls[j][r] = W(r, j)
  }
  for (int64_t c0 = 0; c0 < nn; c0 += NB) {
    const int nc = (int)imin64(NB, nn - c0);
    __syncthreads();
    // A12 chunk as it lies: Bs[j][cc] = A(k + j, k1 + c0 + cc)
    stage_block<kBlkThreads, T>(
        tid, [&](int j, int cc) { return (cc < nc) ? A[(k1 + c0 + cc) * lda + (k + j)] : T(0); },
        [&](int j, int cc, T v) { Bs[j][cc] = v; });
    __syncthreads();
    T acc[4][4] = {};
    mm4x4<T, LP, RP>(Ls, Bs, 4 * rg, 4 * cg, acc);
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const int cc = 4 * cg + l;
      if (cc >= nc) continue;
      T* col = A + (k1 + c0 + cc) * lda + row0 + 4 * rg;
      if (4 * rg + 4 <= rows) {
#pragma unroll
        for (int h = 0; h < 4 / V; ++h) {
          VT v = reinterpret_cast<VT*>(col)[h];
#pragma unroll
          for (int e = 0; e < V; ++e) vset<T>(v, e, vget<T>(v, e) - acc[h * V + e][l]);
          reinterpret_cast<VT*>(col)[h] = v;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (4 * rg + i < rows) col[i] -= acc[i][l];
      }
    }
  }
  // The next block's diagonal block (rows and columns k1..k1+63, inside the
  // panel) is final once the CTAs owning its rows are done: the last of them
  // (ticket) factors it while the other CTAs still update, so the next
  // block's step can start as soon as this launch ends.
  const unsigned owners = (unsigned)imin64(NB / kBlkRows, nmain);
  if (!next || blockIdx.x >= owners) return;
  __shared__ unsigned last;
  __threadfence();   // this CTA's stores, visible device-wide before its ticket
  __syncthreads();
  if (tid == 0) {
    const unsigned got = atomicAdd(ticket, 1u);
    last = (got == owners - 1);
    if (last) {
      *ticket = 0u;   // every owner has taken its ticket: ready for the next launch
      __threadfence();
    }
  }
  __syncthreads();
  if (!last) return;
  static_assert(kDiagThreads == kBlkThreads, "the whole CTA factors the next diagonal block");
  diag_factor<T>(A, lda, n, k1, ipiv, status, Minv_next, rowat_next, bsm);
}

// ----------------------------------------------------------------------------
// (3) k_pfix: after a panel's blocks, for each block b of the panel, its row
// swaps on the panel's columns left of it and U12 = M'_b A12 on the columns
// right of it, in place (nothing reads these parts before: the blocks' own
// steps use L21 and A12 as they lie). Task t of nblk (nblk - 1): block
// b = t / (nblk - 1), i = t % (nblk - 1); i < b: left chunk i, else right
// chunk i - b; 64 columns per task. The panel's last k_blk runs these tasks
// in extra CTAs (its own work touches none of these parts); k_pfix runs them
// when that block has no rows below it (the matrix's last block).
constexpr int kPfixThreads = 128;
constexpr int kPfixKC = 16;   // rows of M' staged at a time
template <class T> __host__ __device__ constexpr size_t pfix_smem() {
  return (size_t)(NB + kPfixKC) * rpitch<T>() * sizeof(T) + 64;
}

template <class T>
__device__ void pfix_task(T* __restrict__ A, int64_t lda, int64_t K0, int64_t kend, int nblk,
                          const T* __restrict__ Minv, const int* __restrict__ rowat, int task, unsigned char* smem) {
  constexpr int RP = rpitch<T>();
  T (*X)[RP] = reinterpret_cast<T (*)[RP]>(smem);                                 // X[row j][column]
  T (*Ms)[RP] = reinterpret_cast<T (*)[RP]>(smem + (size_t)NB * RP * sizeof(T));   // Ms[jj][r] = M'(r, j0 + jj)
  const int tid = threadIdx.x;
  const int b = task / (nblk - 1), i = task % (nblk - 1);
  const int64_t kb = K0 + (int64_t)b * NB;
  const int nbb = (int)imin64(NB, kend - kb);
  const bool left = i < b;
  const int64_t c0 = left ? K0 + (int64_t)i * NB : kb + NB + (int64_t)(i - b) * NB;
  const int nc = (int)imin64(NB, (left ? kb : kend) - c0);
  if (nc <= 0) return;
  stage_block<kPfixThreads, T>(
      tid, [&](int j, int cc) { return (j < nbb && cc < nc) ? A[(c0 + cc) * lda + (kb + j)] : T(0); },
      [&](int j, int cc, T v) { X[j][cc] = v; });
  if (left) {
    const int* ra = rowat + b * NB;
    __syncthreads();
    for (int e = tid; e < NB * NB; e += kPfixThreads) {
      const int s = e & (NB - 1), cc = e / NB;
      if (s < nbb && cc < nc) A[(c0 + cc) * lda + (kb + s)] = X[ra[s]][cc];
    }
    return;
  }
  const T* M = Minv + (size_t)b * NB * NB;
  const int rg = tid & 15, cg = tid >> 4;   // rows 4 rg.., columns 8 cg..
  T acc[4][8] = {};
  for (int j0 = 0; j0 < NB; j0 += kPfixKC) {
    __syncthreads();
    for (int e = tid; e < kPfixKC * NB; e += kPfixThreads) {
      const int jj = e % kPfixKC, r = e / kPfixKC;
      Ms[jj][r] = M[r * NB + j0 + jj];
    }
    __syncthreads();
#pragma unroll 4
    for (int jj = 0; jj < kPfixKC; ++jj) {
      T a[4], q[8];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = Ms[jj][4 * rg + u];
#pragma unroll
      for (int l = 0; l < 8; ++l) q[l] = X[j0 + jj][8 * cg + l];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int l = 0; l < 8; ++l) acc[u][l] += a[u] * q[l];
    }
  }
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    const int cc = 8 * cg + l;
    if (cc >= nc) continue;
#pragma unroll
    for (int u = 0; u < 4; ++u) A[(c0 + cc) * lda + (kb + 4 * rg + u)] = acc[u][l];
  }
}

static_assert(kPfixThreads == kBlkThreads && pfix_smem<float>() <= blk_smem<float>() &&
                  pfix_smem<double>() <= blk_smem<double>(),
              "the extra CTAs of k_blk run pfix_task");

template <class T>
__global__ void __launch_bounds__(kPfixThreads)
k_pfix(T* __restrict__ A, int64_t lda, int64_t K0, int64_t kend, int nblk, const T* __restrict__ Minv,
       const int* __restrict__ rowat) {
  extern __shared__ __align__(16) unsigned char psm[];
  pfix_task<T>(A, lda, K0, kend, nblk, Minv, rowat, (int)blockIdx.x, psm);
}

// ----------------------------------------------------------------------------
// (2b) k_strip: a strip of columns outside a factored panel (the panel's w
// rows from K0, w <= kStripRows, in nblk 64-row blocks). On the columns
// [cl0, cl1) it puts each block's rows in their logical order; on [cr0, cr1)
// it forms U12 = L_panel^-1 P_panel A12 block by block,
//     U_b = L_bb^-1 (P_b X_b - sum_{b' < b} L_bb' U_b'),
// with L_bb^-1 = M'_b P_b^T (M' of k_diag, columns taken in logical order)
// and L_bb' the panel's L (k_pfix left it in logical row order); each U_b is
// written in place and read back by the later blocks. Every product is a
// 64 x 64 x 32 tile product from shared memory with a rolled K loop, so the
// code stays small. One CTA owns 32 columns.
constexpr int kStripRows = kOuterPanel;
constexpr int kStripCols = 32;
constexpr int kStripThreads = 256;
template <class T> __host__ __device__ constexpr int strip_qpitch() { return kStripCols + 16 / (int)sizeof(T); }
template <class T> constexpr size_t strip_smem() {
  return (size_t)NB * rpitch<T>() * sizeof(T) + (size_t)NB * strip_qpitch<T>() * sizeof(T) + 64;
}

// acc[i][l] += sum_j P[j][r0 + i] Q[j][c0 + l], 4 rows x 2 columns
template <class T, int PP, int QP>
__device__ __forceinline__ void mm4x2(const T (*P)[PP], const T (*Q)[QP], int r0, int c0, T (&acc)[4][2]) {
  typedef typename V16<T>::type VT;
  constexpr int V = V16<T>::n;
#pragma unroll 4
  for (int j = 0; j < NB; ++j) {
    T a[4];
#pragma unroll
    for (int h = 0; h < 4 / V; ++h) {
      const VT va = *reinterpret_cast<const VT*>(&P[j][r0 + h * V]);
#pragma unroll
      for (int e = 0; e < V; ++e) a[h * V + e] = vget<T>(va, e);
    }
    const T b0 = Q[j][c0], b1 = Q[j][c0 + 1];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      acc[i][0] += a[i] * b0;
      acc[i][1] += a[i] * b1;
    }
  }
}

template <class T>
__global__ void __launch_bounds__(kStripThreads)
k_strip(T* __restrict__ A, int64_t lda, int64_t K0, int w, const T* __restrict__ Minv,
        const int* __restrict__ rowat, int64_t cl0, int64_t cl1, int64_t cr0, int64_t cr1) {
  constexpr int RP = rpitch<T>(), QP = strip_qpitch<T>();
  extern __shared__ __align__(16) unsigned char ssm[];
  T (*Pt)[RP] = reinterpret_cast<T (*)[RP]>(ssm);                                 // Pt[j][r]
  T (*Q)[QP] = reinterpret_cast<T (*)[QP]>(ssm + (size_t)NB * RP * sizeof(T));   // Q[j][c]
  const int tid = threadIdx.x;
  const int nblk = (w + NB - 1) / NB;
  const int64_t nl = cl1 - cl0;
  const int64_t gl = (nl + kStripCols - 1) / kStripCols;
  const bool right = (int64_t)blockIdx.x >= gl;
  const int64_t c0 = right ? cr0 + ((int64_t)blockIdx.x - gl) * kStripCols : cl0 + (int64_t)blockIdx.x * kStripCols;
  const int nc = (int)imin64(kStripCols, right ? cr1 - c0 : cl1 - c0);
  if (!right) {
    // each block's rows in logical order: row s <- row rowat[s]
    for (int b = 0; b < nblk; ++b) {
      const int nbb = min(NB, w - b * NB);
      const int* ra = rowat + b * NB;
      const int64_t rb = K0 + (int64_t)b * NB;
      int moved = 0;
      for (int s = tid; s < nbb; s += kStripThreads) moved |= (ra[s] != s);
      if (!__syncthreads_or(moved)) continue;
      for (int e = tid; e < NB * kStripCols; e += kStripThreads) {
        const int s = e & (NB - 1), cc = e / NB;
        if (s < nbb && cc < nc) Q[s][cc] = A[(c0 + cc) * lda + rb + s];
      }
      __syncthreads();
      for (int e = tid; e < NB * kStripCols; e += kStripThreads) {
        const int s = e & (NB - 1), cc = e / NB;
        if (s < nbb && cc < nc) A[(c0 + cc) * lda + rb + s] = Q[ra[s]][cc];
      }
      __syncthreads();
    }
    return;
  }
  const int rg = tid & 15, cg = tid >> 4;   // rows 4 rg.., columns 2 cg..
  for (int b = 0; b < nblk; ++b) {
    const int nbb = min(NB, w - b * NB);
    const int* ra = rowat + b * NB;
    const int64_t rb = K0 + (int64_t)b * NB;
    T acc[4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int l = 0; l < 2; ++l) {
        const int r = 4 * rg + i, cc = 2 * cg + l;
        acc[i][l] = (r < nbb && cc < nc) ? A[(c0 + cc) * lda + rb + ra[r]] : T(0);
      }
    for (int b2 = 0; b2 < b; ++b2) {
      const int64_t rb2 = K0 + (int64_t)b2 * NB;
      __syncthreads();
      stage_block<kStripThreads, T>(
          tid, [&](int r, int j) { return (r < nbb) ? A[(rb2 + j) * lda + rb + r] : T(0); },
          [&](int r, int j, T v) { Pt[j][r] = v; });   // Pt[j][r] = L(b row r, b2 column j)
      for (int e = tid; e < NB * kStripCols; e += kStripThreads) {
        const int j = e & (NB - 1), cc = e / NB;
        Q[j][cc] = (cc < nc) ? A[(c0 + cc) * lda + rb2 + j] : T(0);   // U_b2
      }
      __syncthreads();
      T d[4][2] = {};
      mm4x2<T, RP, QP>(Pt, Q, 4 * rg, 2 * cg, d);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int l = 0; l < 2; ++l) acc[i][l] -= d[i][l];
    }
    __syncthreads();
    // Y -> Q[r][c]; Pt[s][r] = L_bb^-1(r, s) = M'(r, rowat[s])
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int l = 0; l < 2; ++l) Q[4 * rg + i][2 * cg + l] = acc[i][l];
    const T* M = Minv + (size_t)b * NB * NB;
    stage_block<kStripThreads, T>(
        tid, [&](int r, int s) { return M[r * NB + ra[s]]; }, [&](int r, int s, T v) { Pt[s][r] = v; });
    __syncthreads();
    T u[4][2] = {};
    mm4x2<T, RP, QP>(Pt, Q, 4 * rg, 2 * cg, u);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int l = 0; l < 2; ++l) {
        const int r = 4 * rg + i, cc = 2 * cg + l;
        if (r < nbb && cc < nc) A[(c0 + cc) * lda + rb + r] = u[i][l];
      }
  }
}

// ----------------------------------------------------------------------------
// (3) trailing update C -= A B, SIMT register tiles (the FP64 path). The C tile
// is fetched into shared memory with cp.async when the CTA starts, so its
// latency overlaps the K loop; global loads of the next K slice go to
// registers while the current slice is multiplied from shared memory (double
// buffer). Consecutive threads own consecutive rows (coalesced C accesses).
template <class T, int BM, int BN, int BK, int TM, int TN>
constexpr size_t gemm_smem() {
  return (size_t)2 * BK * (BM + 2) * sizeof(T) + (size_t)2 * BK * (BN + 2) * sizeof(T) + (size_t)BM * BN * sizeof(T);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}

template <class T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
k_gemm_sub(const T* __restrict__ Am, const T* __restrict__ Bm, T* __restrict__ Cm, int64_t lda,
           int64_t m, int64_t nn, int kk, bool pre) {
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int LA = BK * BM / NT;
  constexpr int LB = BK * BN / NT;
  constexpr int TX = BM / TM;
  constexpr int V16 = 16 / sizeof(T);   // elements per 16-byte copy
  extern __shared__ __align__(16) unsigned char gsm[];
  T (*As)[BK][BM + 2] = reinterpret_cast<T (*)[BK][BM + 2]>(gsm);
  T (*Bs)[BK][BN + 2] = reinterpret_cast<T (*)[BK][BN + 2]>(gsm + (size_t)2 * BK * (BM + 2) * sizeof(T));
  T (*Cs)[BM] = reinterpret_cast<T (*)[BM]>(gsm + (size_t)2 * BK * (BM + 2) * sizeof(T) +
                                            (size_t)2 * BK * (BN + 2) * sizeof(T));   // Cs[col][row]
  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  const int64_t i0 = (int64_t)blockIdx.x * BM, j0 = (int64_t)blockIdx.y * BN;
  // C tile -> shared memory (asynchronous); whole 16-byte pieces of rows < m
  // only (i0 and lda keep them aligned), the rest is zero and never stored
  if (pre) {
    for (int e = tid; e < BM * BN / V16; e += NT) {
      const int col = e / (BM / V16), rv = (e % (BM / V16)) * V16;
      const int64_t gi = i0 + rv, gj = j0 + col;
      const bool ok = (gj < nn) && (gi + V16 <= m);
      cp_async16(&Cs[col][rv], ok ? (const void*)(Cm + gj * lda + gi) : (const void*)Cm, ok);
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  T acc[TM][TN];
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TN; ++b) acc[a][b] = T(0);
  T ra[LA], rb[LB];
  auto gload = [&](int k0) {
#pragma unroll
    for (int u = 0; u < LA; ++u) {
      const int q = tid + u * NT;
      const int ii = q % BM, kq = q / BM;
      const int64_t gi = i0 + ii;
      ra[u] = (gi < m && k0 + kq < kk) ? Am[(int64_t)(k0 + kq) * lda + gi] : T(0);
    }
#pragma unroll
    for (int u = 0; u < LB; ++u) {
      const int q = tid + u * NT;
      const int kq = q % BK, jj = q / BK;
      const int64_t gj = j0 + jj;
      rb[u] = (gj < nn && k0 + kq < kk) ? Bm[gj * lda + k0 + kq] : T(0);
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int u = 0; u < LA; ++u) {
      const int q = tid + u * NT;
      As[buf][q / BM][q % BM] = ra[u];
    }
#pragma unroll
    for (int u = 0; u < LB; ++u) {
      const int q = tid + u * NT;
      Bs[buf][q % BK][q / BK] = rb[u];
    }
  };
  gload(0);
  sstore(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < kk; k0 += BK) {
    const bool more = k0 + BK < kk;
    if (more) gload(k0 + BK);
#pragma unroll
    for (int kq = 0; kq < BK; ++kq) {
      T a[TM], b[TN];
#pragma unroll
      for (int u = 0; u < TM; ++u) a[u] = As[buf][kq][tx + u * TX];
#pragma unroll
      for (int v = 0; v < TN; ++v) b[v] = Bs[buf][kq][ty + v * (BN / TN)];
#pragma unroll
      for (int u = 0; u < TM; ++u)
#pragma unroll
        for (int v = 0; v < TN; ++v) acc[u][v] += a[u] * b[v];
    }
    if (more) sstore(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  const bool full_rows = pre && i0 + BM <= m;
#pragma unroll
  for (int v = 0; v < TN; ++v) {
    const int col = ty + v * (BN / TN);
    const int64_t gj = j0 + col;
    if (gj >= nn) continue;
#pragma unroll
    for (int u = 0; u < TM; ++u) {
      const int row = tx + u * TX;
      const int64_t gi = i0 + row;
      if (gi >= m) continue;
      // rows of a partial 16-byte piece were not prefetched: read them directly
      const T cv = (full_rows || (pre && (row / V16) * V16 + V16 + i0 <= m)) ? Cs[col][row] : Cm[gj * lda + gi];
      Cm[gj * lda + gi] = cv - acc[u][v];
    }
  }
}


// ----------------------------------------------------------------------------
// FP64 trailing update C -= A B: 128 x 128 tiles, 256 threads with 8 x 8
// register tiles, 16-deep K slices streamed by cp.async through a 3-stage
// shared-memory ring (the next two slices are in flight while one is
// multiplied), C read and written once at the end. A slice of A is 16
// columns of 128 rows (Asm[k][row]); a slice of B is 16 rows of 128 columns,
// kept column by column (Bsm[col][k]), so both come in 16-byte pieces of the
// column-major matrix.
namespace d64 {
constexpr int BM = 128, BN = 128, BK = 16, TM = 8, TN = 8, STAGES = 3, NT = (BM / TM) * (BN / TN);
constexpr int BP = BK + 2;   // row pitch of Bsm (doubles): 16-byte rows
__host__ __device__ constexpr size_t stage_doubles() { return (size_t)BK * BM + (size_t)BN * BP; }
constexpr size_t smem() { return STAGES * stage_doubles() * sizeof(double); }
}  // namespace d64

__device__ __forceinline__ void cp_async16_sz(void* smem, const void* gmem, int bytes) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}

__global__ void __launch_bounds__(d64::NT, 1)
k_gemm_sub_f64(const double* __restrict__ Am, const double* __restrict__ Bm, double* __restrict__ Cm, int64_t lda,
               int64_t m, int64_t nn, int kk) {
  using namespace d64;
  extern __shared__ __align__(16) unsigned char gsm[];
  double* const ring = reinterpret_cast<double*>(gsm);
  const int tid = threadIdx.x;
  const int tx = tid % (BM / TM), ty = tid / (BM / TM);
  const int64_t i0 = (int64_t)blockIdx.x * BM, j0 = (int64_t)blockIdx.y * BN;
  const int nk = (kk + BK - 1) / BK;
  // one K slice into stage s: 1024 16-byte pieces of A and 1024 of B, 4 + 4 per thread
  auto issue = [&](int kb, int s) {
    double* As = ring + (size_t)s * stage_doubles();
    double* Bs = As + BK * BM;
    const int k0 = kb * BK;
#pragma unroll
    for (int u = 0; u < (BK * BM / 2) / NT; ++u) {
      const int q = tid + u * NT;
      const int kq = q / (BM / 2), ii = (q % (BM / 2)) * 2;
      const int64_t gi = i0 + ii;
      const bool kin = k0 + kq < kk;
      const int rows = kin ? (int)imin64(2, m - gi) : 0;
      const double* src = (rows > 0) ? Am + (int64_t)(k0 + kq) * lda + gi : Am;
      cp_async16_sz(As + kq * BM + ii, src, rows > 0 ? rows * 8 : 0);
    }
#pragma unroll
    for (int u = 0; u < (BK * BN / 2) / NT; ++u) {
      const int q = tid + u * NT;
      const int jj = q / (BK / 2), kq = (q % (BK / 2)) * 2;
      const int64_t gj = j0 + jj;
      const int ks = (gj < nn) ? (int)imin64(2, kk - (k0 + kq)) : 0;
      const double* src = (ks > 0) ? Bm + gj * lda + k0 + kq : Bm;
      cp_async16_sz(Bs + jj * BP + kq, src, ks > 0 ? ks * 8 : 0);
    }
  };
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) issue(s, s);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  double acc[TM][TN];
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TN; ++b) acc[a][b] = 0.0;
#pragma unroll 1
  for (int kb = 0; kb < nk; ++kb) {
    asm volatile("cp.async.wait_group %0;" ::"n"(STAGES - 2) : "memory");
    __syncthreads();   // slice kb has landed for every thread; slot (kb - 1) % STAGES is free
    if (kb + STAGES - 1 < nk) issue(kb + STAGES - 1, (kb + STAGES - 1) % STAGES);
    asm volatile("cp.async.commit_group;" ::: "memory");
    const double* As = ring + (size_t)(kb % STAGES) * stage_doubles();
    const double* Bs = As + BK * BM;
#pragma unroll
    for (int kq = 0; kq < BK; ++kq) {
      double a[TM], b[TN];
#pragma unroll
      for (int u = 0; u < TM; ++u) a[u] = As[kq * BM + tx + u * (BM / TM)];
#pragma unroll
      for (int v = 0; v < TN; ++v) b[v] = Bs[(ty + v * (BN / TN)) * BP + kq];
#pragma unroll
      for (int u = 0; u < TM; ++u)
#pragma unroll
        for (int v = 0; v < TN; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
#pragma unroll
  for (int v = 0; v < TN; ++v) {
    const int64_t gj = j0 + ty + v * (BN / TN);
    if (gj >= nn) continue;
#pragma unroll
    for (int u = 0; u < TM; ++u) {
      const int64_t gi = i0 + tx + u * (BM / TM);
      if (gi < m) Cm[gj * lda + gi] -= acc[u][v];
    }
  }
}

// The same FP64 update on the FP64 tensor path (mma.sync m8n8k4 .f64, the
// DMMA instruction; tcgen05 has no FP64 kind): 128 x 128 CTA tiles, NT/32
// warps, each a (8 MF) x (8 NF) warp tile of MF x NF fragments of 8 x 8 with
// the accumulators in registers (256 threads: 2 x 4 warps of 64 x 32; 512
// threads: 4 x 4 warps of 32 x 32); 16-deep K slices through a 3-stage
// cp.async ring. Shared-memory pitches keep the fragment loads free of bank
// conflicts: A slices [k][row] with 136-double rows (the 4 k rows a fragment
// reads start 64 bytes apart in the bank space), B slices [col][k] with
// 20-double rows (the 8 columns a fragment reads cover all banks).
// Fragments (PTX ISA, mma m8n8k4 .f64): lane = 4 g + t; A(8x4, row) element
// (g, t); B(4x8, col) element (t, g); C(8x8) elements (g, 2t) and (g, 2t+1).
namespace dm {
constexpr int BM = 128, AP = BM + 8;
template <int BK> __host__ __device__ constexpr int bp() { return BK + 4; }
template <int BK, int BN = 128> __host__ __device__ constexpr size_t stage_doubles() {
  return (size_t)BK * AP + (size_t)BN * bp<BK>();
}
template <int BK, int STAGES, int BN = 128> constexpr size_t smem() {
  return STAGES * stage_doubles<BK, BN>() * sizeof(double);
}
}  // namespace dm

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int NT, int MF, int NF, int BK = 16, int STAGES = 3, int BN = 128, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB)
k_gemm_sub_dmma(const double* __restrict__ Am, const double* __restrict__ Bm, double* __restrict__ Cm, int64_t lda,
                int64_t m, int64_t nn, int kk, int pf) {
  using namespace dm;
  constexpr int BP = bp<BK>();
  constexpr int WARPS_M = BM / (8 * MF);
  static_assert(WARPS_M * (BN / (8 * NF)) * 32 == NT, "the warp tiles cover the CTA tile");
  extern __shared__ __align__(16) unsigned char gsm[];
  double* const ring = reinterpret_cast<double*>(gsm);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp % WARPS_M) * 8 * MF, wn = (warp / WARPS_M) * 8 * NF;
  const int64_t i0 = (int64_t)blockIdx.x * BM, j0 = (int64_t)blockIdx.y * BN;
  const int nk = (kk + BK - 1) / BK;
  if (pf && tid < BN && j0 + tid < nn) {
    // the epilogue reads the C tile once: bring it into L2 (one bulk prefetch
    // of up to BM doubles a column) while the K loop runs
    const uint32_t bytes = (uint32_t)(imin64(BM, m - i0) * 8) & ~15u;
    if (bytes)
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(Cm + (j0 + tid) * lda + i0), "r"(bytes) : "memory");
  }
  // one K slice into stage s: 1024 16-byte pieces of A and 1024 of B
  auto issue = [&](int kb, int s) {
    double* As = ring + (size_t)s * stage_doubles<BK, BN>();
    double* Bs = As + BK * AP;
    const int k0 = kb * BK;
#pragma unroll
    for (int u = 0; u < (BK * BM / 2) / NT; ++u) {
      const int q = tid + u * NT;
      const int kq = q / (BM / 2), ii = (q % (BM / 2)) * 2;
      const int64_t gi = i0 + ii;
      const bool kin = k0 + kq < kk;
      const int rows = kin ? (int)imin64(2, m - gi) : 0;
      const double* src = (rows > 0) ? Am + (int64_t)(k0 + kq) * lda + gi : Am;
      cp_async16_sz(As + kq * AP + ii, src, rows > 0 ? rows * 8 : 0);
    }
#pragma unroll
    for (int u = 0; u < (BK * BN / 2) / NT; ++u) {
      const int q = tid + u * NT;
      const int jj = q / (BK / 2), kq = (q % (BK / 2)) * 2;
      const int64_t gj = j0 + jj;
      const int ks = (gj < nn) ? (int)imin64(2, kk - (k0 + kq)) : 0;
      const double* src = (ks > 0) ? Bm + gj * lda + k0 + kq : Bm;
      cp_async16_sz(Bs + jj * BP + kq, src, ks > 0 ? ks * 8 : 0);
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
    const double* As = ring + (size_t)(kb % STAGES) * stage_doubles<BK, BN>();
    const double* Bs = As + BK * AP;
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      double a[MF], b[NF];
#pragma unroll
      for (int mi = 0; mi < MF; ++mi) a[mi] = As[(k4 + t) * AP + wm + mi * 8 + g];
#pragma unroll
      for (int ni = 0; ni < NF; ++ni) b[ni] = Bs[(wn + ni * 8 + g) * BP + k4 + t];
#pragma unroll
      for (int mi = 0; mi < MF; ++mi)
#pragma unroll
        for (int ni = 0; ni < NF; ++ni) dmma(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
#pragma unroll
  for (int ni = 0; ni < NF; ++ni)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int64_t gj = j0 + wn + ni * 8 + 2 * t + e;
      if (gj >= nn) continue;
#pragma unroll
      for (int mi = 0; mi < MF; ++mi) {
        const int64_t gi = i0 + wm + mi * 8 + g;
        if (gi < m) Cm[gj * lda + gi] -= acc[mi][ni][e];
      }
    }
}

// C (m x nn) -= A (m x kk) B (kk x nn); all three are sub-blocks of one
// column-major matrix with leading dimension lda.
template <class T>
static int gemm_sub(fp_ctx* c, const T* Am, const T* Bm, T* Cm, int64_t lda, int64_t m, int64_t nn,
                    int kk) {
  if (m <= 0 || nn <= 0 || kk <= 0) return FP_OK;
  if constexpr (sizeof(T) == 4) {
    if (tc_gemm_sub_f32(c, (const float*)Am, (const float*)Bm, (float*)Cm, lda, m, nn, kk)) return FP_OK;
    return gemm_sub_simt_f32(c, (const float*)Am, (const float*)Bm, (float*)Cm, lda, m, nn, kk);
  } else {
    // cp.async moves 16-byte pieces: the blocks' row offsets and lda must keep them aligned
    const uintptr_t mis = (reinterpret_cast<uintptr_t>(Am) | reinterpret_cast<uintptr_t>(Bm) |
                           (uintptr_t)(lda * sizeof(T))) & 15;
    const int slot = kt_begin(c);
    TraceScope tr(c, TR_GEMM_SIMT);
    if (mis == 0 && c->fp64_dmma) {
      static SmemAttr attr8, attr16, attr32, attr32k, attr2c, attr2k;
      constexpr int sm16 = (int)dm::smem<16, 3>(), sm32 = (int)dm::smem<32, 3>();
      FP_CUDA_TRY(c->err, attr8.ensure(k_gemm_sub_dmma<256, 8, 4>, sm16));
      FP_CUDA_TRY(c->err, attr16.ensure(k_gemm_sub_dmma<512, 4, 4>, sm16));
      FP_CUDA_TRY(c->err, attr32.ensure(k_gemm_sub_dmma<1024, 4, 2>, sm16));
      FP_CUDA_TRY(c->err, attr32k.ensure(k_gemm_sub_dmma<1024, 4, 2, 32, 3>, sm32));
      constexpr int sm64 = (int)dm::smem<16, 3, 64>();
      FP_CUDA_TRY(c->err, attr2c.ensure(k_gemm_sub_dmma<512, 4, 2, 16, 3, 64, 2>, sm64));
      constexpr int sm64k = (int)dm::smem<32, 2, 64>();
      FP_CUDA_TRY(c->err, attr2k.ensure(k_gemm_sub_dmma<512, 4, 2, 32, 2, 64, 2>, sm64k));
      dim3 g((unsigned)((m + dm::BM - 1) / dm::BM), (unsigned)((nn + 127) / 128));
      const double* Ad = (const double*)Am;
      const double* Bd = (const double*)Bm;
      double* Cd = (double*)Cm;
      if (c->fp64_dmma == 6) {   // 128 x 64 tiles, two CTAs an SM, 32-deep K slices in 2 stages
        dim3 g2((unsigned)((m + dm::BM - 1) / dm::BM), (unsigned)((nn + 63) / 64));
        k_gemm_sub_dmma<512, 4, 2, 32, 2, 64, 2><<<g2, 512, sm64k, c->stream>>>(Ad, Bd, Cd, lda, m, nn, kk, c->tc_prefetch);
      } else if (c->fp64_dmma == 5) {   // 128 x 64 tiles, two CTAs an SM
        dim3 g2((unsigned)((m + dm::BM - 1) / dm::BM), (unsigned)((nn + 63) / 64));
        k_gemm_sub_dmma<512, 4, 2, 16, 3, 64, 2><<<g2, 512, sm64, c->stream>>>(Ad, Bd, Cd, lda, m, nn, kk, c->tc_prefetch);
      } else if (c->fp64_dmma == 4)
        k_gemm_sub_dmma<1024, 4, 2, 32, 3><<<g, 1024, sm32, c->stream>>>(Ad, Bd, Cd, lda, m, nn, kk, c->tc_prefetch);
      else if (c->fp64_dmma == 3)
        k_gemm_sub_dmma<1024, 4, 2><<<g, 1024, sm16, c->stream>>>(Ad, Bd, Cd, lda, m, nn, kk, c->tc_prefetch);
      else if (c->fp64_dmma == 2)
        k_gemm_sub_dmma<512, 4, 4><<<g, 512, sm16, c->stream>>>(Ad, Bd, Cd, lda, m, nn, kk, c->tc_prefetch);
      else
        k_gemm_sub_dmma<256, 8, 4><<<g, 256, sm16, c->stream>>>(Ad, Bd, Cd, lda, m, nn, kk, c->tc_prefetch);
    } else if (mis == 0) {
      static SmemAttr attr;
      FP_CUDA_TRY(c->err, attr.ensure(k_gemm_sub_f64, (int)d64::smem()));
      dim3 g((unsigned)((m + d64::BM - 1) / d64::BM), (unsigned)((nn + d64::BN - 1) / d64::BN));
      k_gemm_sub_f64<<<g, d64::NT, d64::smem(), c->stream>>>((const double*)Am, (const double*)Bm, (double*)Cm, lda, m,
                                                             nn, kk);
    } else {
      constexpr int BM = 128, BN = 128, BK = 8, TM = 8, TN = 8;
      constexpr size_t sm = gemm_smem<T, BM, BN, BK, TM, TN>();
      static SmemAttr attr;
      FP_CUDA_TRY(c->err, attr.ensure(k_gemm_sub<T, BM, BN, BK, TM, TN>, (int)sm));
      dim3 g((unsigned)((m + BM - 1) / BM), (unsigned)((nn + BN - 1) / BN));
      const bool pre = ((reinterpret_cast<uintptr_t>(Cm) | (uintptr_t)(lda * sizeof(T))) & 15) == 0;
      k_gemm_sub<T, BM, BN, BK, TM, TN><<<g, (BM / TM) * (BN / TN), sm, c->stream>>>(Am, Bm, Cm, lda, m, nn, kk, pre);
    }
    kt_end(c, slot, 2.0 * (double)m * (double)nn * (double)kk, (double)m * (double)nn);
    ++c->nlaunch;
  }
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

int gemm_sub_simt_f32(fp_ctx* c, const float* A, const float* B, float* C, int64_t lda, int64_t m, int64_t nn,
                      int kk) {
  constexpr int BM = 128, BN = 128, BK = 16, TM = 8, TN = 8;
  constexpr size_t sm = gemm_smem<float, BM, BN, BK, TM, TN>();
  static SmemAttr attr;
  FP_CUDA_TRY(c->err, attr.ensure(k_gemm_sub<float, BM, BN, BK, TM, TN>, (int)sm));
  dim3 g((unsigned)((m + BM - 1) / BM), (unsigned)((nn + BN - 1) / BN));
  const bool pre = ((reinterpret_cast<uintptr_t>(C) | (uintptr_t)(lda * sizeof(float))) & 15) == 0;
  k_gemm_sub<float, BM, BN, BK, TM, TN><<<g, (BM / TM) * (BN / TN), sm, c->stream>>>(A, B, C, lda, m, nn, kk, pre);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

// Two-level blocked right-looking LU with look-ahead. Outer panels of
// kOuterNB columns; inside a panel, NB-wide blocks are factored (pivots local
// to the diagonal block), their L21 formed, and the update applied to the
// panel's own columns only. Two streams share the work of each panel P:
//  * c->stream (high priority, the critical path): factor P; then, once the
//    previous panel's trailing update is done, the row swaps and U12 of P's
//    rows in the next panel's columns and the update of those columns
//    (K = kOuterNB), so that the next panel can start;
//  * c->stream2 (after P is factored): the row swaps of P in the columns left
//    of P, its U12 rows in the columns beyond the next panel, and the
//    trailing update of those columns, which overlaps the next panel.
// Row swaps stay inside 64-row blocks, so the swaps of different blocks
// commute, and a row update (C_r -= L_r U) commutes with a swap of the rows
// of both C and L. Step (1) leaves P's L rows swapped by all of P's blocks,
// so a strip of columns outside P first receives all of P's swaps and only
// then the per-block substitutions and updates (k_strip). Columns are split between the
// streams so that no element is written by both at once.
constexpr int kOuterNB = kOuterPanel;

template <class T>
int lu_factor(fp_ctx* c, T* A, int64_t n, int64_t lda, int32_t* ipiv, float* cert) {
  FP_CUDA_TRY(c->err, cudaMemsetAsync(cert, 0, sizeof(float), c->stream));
  static SmemAttr attr_blk, attr_pfix;
  FP_CUDA_TRY(c->err, attr_blk.ensure(k_blk<T>, (int)blk_smem<T>()));
  FP_CUDA_TRY(c->err, attr_pfix.ensure(k_pfix<T>, (int)pfix_smem<T>()));
  // M' and the row order of each block of a panel, two sets of slots
  static_assert(kOuterNB / NB <= kPanelSlots, "one scratch slot per block of a panel");
  T* const minv = reinterpret_cast<T*>(c->d_minv);
  int* const rowat = reinterpret_cast<int*>(reinterpret_cast<char*>(c->d_minv) + kMinvBytes);
  if (sizeof(T) == 4 && c->use_tc) {   // both scratch sets before any concurrent launch
    if (int rc = ensure_tc_scratch(c, 0, n)) return rc;
    if (int rc = ensure_tc_scratch(c, 1, n)) return rc;
  }
  auto at = [&](int64_t r, int64_t col) { return A + col * lda + r; };
  static_assert(kOuterNB == kStripRows, "a strip holds one outer panel's rows");
  static SmemAttr attr_strip;
  FP_CUDA_TRY(c->err, attr_strip.ensure(k_strip<T>, (int)strip_smem<T>()));
  // slots of the panel starting at K0 (two sets: stream2's strip of panel P
  // reads its set while panel P + 1 fills the other)
  auto pminv = [&](int64_t K0) { return minv + ((K0 / kOuterNB) & 1) * kPanelSlots * NB * NB; };
  auto prowat = [&](int64_t K0) { return rowat + ((K0 / kOuterNB) & 1) * kPanelSlots * NB; };
  auto strip = [&](int64_t K0, int w, int64_t cl0, int64_t cl1, int64_t cr0, int64_t cr1) -> int {
    const int64_t g = (cl1 - cl0 + kStripCols - 1) / kStripCols + (cr1 - cr0 + kStripCols - 1) / kStripCols;
    if (g <= 0) return FP_OK;
    TraceScope tr(c, TR_STRIP);
    k_strip<T><<<(unsigned)g, kStripThreads, strip_smem<T>(), c->stream>>>(A, lda, K0, w, pminv(K0), prowat(K0), cl0,
                                                                           cl1, cr0, cr1);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
    return FP_OK;
  };
  c->trace.base = tr_event(c);
  // stream2 starts after everything already queued on c->stream
  FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_rest, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream2, c->ev_rest, 0));
  for (int64_t K0 = 0; K0 < n; K0 += kOuterNB) {
    const int64_t kend = std::min<int64_t>(K0 + kOuterNB, n);
    const int64_t knext = std::min<int64_t>(kend + kOuterNB, n);   // next panel: columns [kend, knext)
    // (1) factor the panel's columns, full height
    const int nblk = (int)((kend - K0 + NB - 1) / NB);
    bool fixed = false;   // the panel's fix-up ran in its last k_blk
    for (int64_t k = K0; k < kend; k += NB) {
      const int nb = (int)std::min<int64_t>(NB, n - k);
      const int64_t below = n - k - nb;
      const int slot = (int)((k - K0) / NB);
      T* const mv = pminv(K0);
      int* const ra = prowat(K0);
      if (k == K0) {   // later blocks of the panel are factored at the end of the previous k_blk
        TraceScope tr(c, TR_DIAG);
        k_diag<T><<<1, kDiagThreads, 0, c->stream>>>(A, lda, n, k, ipiv, c->d_status, mv + slot * NB * NB,
                                                     ra + slot * NB);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaGetLastError());
      }
      if (below > 0) {   // then nb == NB
        const int nmain = (int)((below + kBlkRows - 1) / kBlkRows);
        const int next = k + NB < kend;
        // the panel's last block also runs the panel's fix-up tasks
        const int fix = (!next && nblk > 1) ? nblk * (nblk - 1) : 0;
        if (fix) fixed = true;
        const unsigned g = (unsigned)(nmain + fix);
        TraceScope tr(c, TR_L21);
        k_blk<T><<<g, kBlkThreads, blk_smem<T>(), c->stream>>>(A, lda, n, k, kend, mv + slot * NB * NB, cert, next,
                                                               ipiv, c->d_status, mv + (slot + 1) * NB * NB,
                                                               ra + (slot + 1) * NB, c->d_ticket, nmain, K0, nblk,
                                                               mv, ra);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaGetLastError());
      }
    }
    if (nblk > 1 && !fixed) {
      TraceScope tr(c, TR_U12);
      k_pfix<T><<<(unsigned)(nblk * (nblk - 1)), kPfixThreads, pfix_smem<T>(), c->stream>>>(A, lda, K0, kend, nblk,
                                                                                          pminv(K0), prowat(K0));
      ++c->nlaunch;
      FP_CUDA_TRY(c->err, cudaGetLastError());
    }
    FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_panel, c->stream));
    // (2) the next panel's columns: P's swaps and U12 rows, then their update
    if (knext > kend) {
      FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_rest, 0));
      if (int rc = strip(K0, (int)(kend - K0), 0, 0, kend, knext)) return rc;
      if (int rc = gemm_sub<T>(c, at(kend, K0), at(K0, kend), at(kend, kend), lda, n - kend, knext - kend,
                               (int)(kend - K0)))
        return rc;
    }
    // (3) on stream2: swaps left of P, U12 rows beyond the next panel, their update
    {
      OnStream2 on2(c);
      FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_panel, 0));
      if (int rc = strip(K0, (int)(kend - K0), 0, K0, knext, n)) return rc;
      if (n > knext)
        if (int rc = gemm_sub<T>(c, at(kend, K0), at(K0, knext), at(kend, knext), lda, n - kend, n - knext,
                                 (int)(kend - K0)))
          return rc;
      FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_rest, c->stream));
    }
  }
  // join: c->stream continues after the last work on stream2
  FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_rest, 0));
  return FP_OK;
}

// ----------------------------------------------------------------------------
// Inverses of the diagonal blocks (unit-lower and upper), for the solves.
// Dinv[b][0] = inv(L_bb), Dinv[b][1] = inv(U_bb), NB x NB column-major each.
template <class T>
__global__ void __launch_bounds__(NB)
k_diag_inv(const T* __restrict__ A, int64_t lda, int64_t n, T* __restrict__ Dinv) {
  __shared__ T Ls[NB][NB + 1];   // [c][r]
  const int64_t b = blockIdx.x;
  const int64_t k = b * NB;
  const int nb = (int)imin64(NB, n - k);
  const int t = threadIdx.x;   // column of the inverse
  for (int q = t; q < NB * NB; q += NB) {
    const int r = q % NB, cc = q / NB;
    Ls[cc][r] = (r < nb && cc < nb) ? A[(k + cc) * lda + (k + r)] : ((r == cc) ? T(1) : T(0));
  }
  __syncthreads();
  T* Li = Dinv + b * 2 * NB * NB;
  T* Ui = Li + NB * NB;
  // inv(L): column t solves L x = e_t (unit diagonal)
  {
    T x[NB];
#pragma unroll
    for (int r = 0; r < NB; ++r) x[r] = (r == t) ? T(1) : T(0);
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const T xj = x[j];
#pragma unroll
      for (int r = j + 1; r < NB; ++r) x[r] -= Ls[j][r] * xj;
    }
#pragma unroll
    for (int r = 0; r < NB; ++r) Li[t * NB + r] = x[r];
  }
  // inv(U): column t solves U x = e_t
  {
    T x[NB];
#pragma unroll
    for (int r = 0; r < NB; ++r) x[r] = (r == t) ? T(1) : T(0);
#pragma unroll
    for (int j = NB - 1; j >= 0; --j) {
      const T xj = x[j] / Ls[j][j];
      x[j] = xj;
#pragma unroll
      for (int r = 0; r < j; ++r) x[r] -= Ls[j][r] * xj;
    }
#pragma unroll
    for (int r = 0; r < NB; ++r) Ui[t * NB + r] = x[r];
  }
}

// Row swaps of the block-local pivots on k right-hand sides (forward order),
// or their inverse (reverse order).
template <class T>
__global__ void k_apply_piv(T* __restrict__ B, int64_t ldb, int64_t n, int64_t k,
                            const int32_t* __restrict__ ipiv, bool reverse) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nblk = (n + NB - 1) / NB;
  if (t >= nblk * k) return;
  const int64_t b = t % nblk, q = t / nblk;
  const int64_t k0 = b * NB;
  const int nb = (int)imin64(NB, n - k0);
  T* col = B + q * ldb;
  if (!reverse) {
    for (int j = 0; j < nb; ++j) {
      const int64_t p = ipiv[k0 + j];
      if (p != k0 + j) { const T a = col[k0 + j]; col[k0 + j] = col[p]; col[p] = a; }
    }
  } else {
    for (int j = nb - 1; j >= 0; --j) {
      const int64_t p = ipiv[k0 + j];
      if (p != k0 + j) { const T a = col[k0 + j]; col[k0 + j] = col[p]; col[p] = a; }
    }
  }
}

// Persistent blocked triangular solve (one sweep), KR right-hand sides.
// LOWER (the forward sweep over blocks): L y = b (unit lower) or, with TRANS,
// U^T z = b; otherwise the backward sweep: U x = y, or with TRANS L^T v = z.
// TRANS reads the dependency tiles A(c, b) instead of A(b, c) and the
// transposed inverse of the diagonal block.
// The solution overwrites B. flags[b] = 1 once block b is final.
// Every dependency tile of the factors is final before the solve starts, so a
// CTA issues the loads of the next tile into shared memory before it waits for
// the flag of the block whose solution it multiplies.
constexpr int kTrsThreads = 256;
template <class T, bool LOWER, int KR, bool TRANS = false>
__global__ void __launch_bounds__(kTrsThreads)
k_trs(const T* __restrict__ A, int64_t lda, int64_t n, const T* __restrict__ Dinv,
      T* __restrict__ B, int64_t ldb, unsigned int* __restrict__ flags,
      unsigned int* __restrict__ ticket, int* __restrict__ status) {
  __shared__ T tile[NB][NB + 1];   // tile[l][r] = A(k0 + r, c0 + l)
  __shared__ T acc[KR][NB];
  __shared__ T y[KR][NB];
  __shared__ int blk_s, stop_s;
  constexpr int PER = NB * NB / kTrsThreads;   // tile elements per thread
  const int64_t nblk = (n + NB - 1) / NB;
  const int tid = threadIdx.x;
  const int r = tid % NB;          // row within the block
  const int qg = tid / NB;         // RHS lane group
  constexpr int QG = kTrsThreads / NB;
  for (;;) {
    if (tid == 0) { blk_s = (int)atomicAdd(ticket, 1u); stop_s = 0; }
    __syncthreads();
    const int64_t tk = blk_s;
    if (tk >= nblk) return;
    const int64_t b = LOWER ? tk : nblk - 1 - tk;
    const int64_t k0 = b * NB;
    const int nb = (int)imin64(NB, n - k0);
    for (int q = qg; q < KR; q += QG) acc[q][r] = (r < nb) ? B[q * ldb + k0 + r] : T(0);
    for (int64_t s = 0; s < tk; ++s) {
      const int64_t cb = LOWER ? s : nblk - 1 - s;
      const int64_t c0 = cb * NB;
      const int cn = (int)imin64(NB, n - c0);
      T v[PER];
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const int e = tid + u * kTrsThreads;
        if (TRANS) {   // tile[l][r] = A(c0 + l, k0 + r), l fastest over threads
          const int ll = e % NB, rr = e / NB;
          v[u] = (rr < nb && ll < cn) ? A[(k0 + rr) * lda + c0 + ll] : T(0);
        } else {
          const int rr = e % NB, ll = e / NB;
          v[u] = (rr < nb && ll < cn) ? A[(c0 + ll) * lda + k0 + rr] : T(0);
        }
      }
      if (tid == 0) {
        int spins = 0;
        while (atomicAdd(&flags[cb], 0u) == 0u) {
          if (++spins > kSpinLimit) { atomicOr(status, (int)DEV_TIMEOUT); stop_s = 1; break; }
          __nanosleep(64);
        }
      }
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const int e = tid + u * kTrsThreads;
        if (TRANS) tile[e % NB][e / NB] = v[u];
        else tile[e / NB][e % NB] = v[u];
      }
      __syncthreads();
      if (stop_s) return;
      for (int q = qg; q < KR; q += QG) y[q][r] = (r < cn) ? __ldcg(&B[q * ldb + c0 + r]) : T(0);
      __syncthreads();
      for (int q = qg; q < KR; q += QG) {
        T s0 = T(0);
#pragma unroll 16
        for (int l = 0; l < NB; ++l) s0 += tile[l][r] * y[q][l];
        acc[q][r] -= s0;
      }
      __syncthreads();
    }
    // x_b = inv(D_bb) acc
    {
      const T* Di = Dinv + b * 2 * NB * NB + ((LOWER != TRANS) ? 0 : NB * NB);
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const int e = tid + u * kTrsThreads;
        // Di column-major: e = l*NB + rr; TRANS uses Di^T
        if (TRANS) tile[e % NB][e / NB] = Di[e];
        else tile[e / NB][e % NB] = Di[e];
      }
      __syncthreads();
      for (int q = qg; q < KR; q += QG) {
        T s0 = T(0);
#pragma unroll 16
        for (int l = 0; l < NB; ++l) s0 += tile[l][r] * acc[q][l];
        if (r < nb) B[q * ldb + k0 + r] = s0;
      }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicExch(&flags[b], 1u);
  }
}

// ----------------------------------------------------------------------------
// Single-RHS sweep over 128-row blocks (k_trs1): block b needs y_s of every
// earlier block s (in sweep order); a CTA streams the row block's tiles with
// 16-byte loads issued before it waits, each warp reading the flags of up to
// 32 upcoming blocks with one acquire load per lane and consuming every block
// already complete, partial sums per thread (4 rows x 16 columns of a tile),
// reduced once. The blocks before the predecessor p (b - 1 forward, b + 1
// backward) give x' = inv(D_bb) (b_b - sum) before p is done; then
// x_b = x' - Mprev_b y_p with Mprev_b = inv(D_bb) T(b, p) (k_mprev, once per
// factorisation), so the step on the chain of n/128 dependent blocks is one
// tile product and one reduction. The flag is published with a release store
// after the barrier that orders the CTA's stores of x_b. With FP32 factors
// no block waits for a flag: every x_b value also goes to the block's mailbox
// as one 64-bit word (the sweep's epoch, the value's bits), which is valid on
// its own once its epoch matches, so each later block polls the 16 values a
// warp needs directly (one L2 round trip per dependency instead of the
// stores' release, the flag and a second load).
constexpr int SB = 128;
constexpr int kTrs1Threads = 256;
template <class T> constexpr size_t trs1_smem() {
  return (size_t)SB * (SB + 1) * sizeof(T) + (size_t)8 * SB * sizeof(T) + (size_t)3 * SB * sizeof(T) + 64;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned int* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ float ld_cg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }

// this thread's 4 rows x 16 columns of an SB x SB column-major tile (leading
// dimension ld) at rows 4 rg.., columns ph + 8 i; zero outside rows < nr,
// columns < nc
template <class T>
__device__ __forceinline__ void load_tile4x16(const T* __restrict__ src, int64_t ld, int rg, int ph, int nr, int nc,
                                              T (&a)[16][4]) {
  const bool rows_full = 4 * rg + 4 <= nr;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int col = ph + 8 * i;
    if (col < nc && rows_full) {
      const T* s = src + col * ld + 4 * rg;
      if (sizeof(T) == 4) {
        const float4 v = *reinterpret_cast<const float4*>(s);
        a[i][0] = v.x; a[i][1] = v.y; a[i][2] = v.z; a[i][3] = v.w;
      } else {
        const double2 v0 = *reinterpret_cast<const double2*>(s);
        const double2 v1 = *reinterpret_cast<const double2*>(s + 2);
        a[i][0] = v0.x; a[i][1] = v0.y; a[i][2] = v1.x; a[i][3] = v1.y;
      }
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) a[i][j] = (col < nc && 4 * rg + j < nr) ? src[col * ld + 4 * rg + j] : T(0);
    }
  }
}

// SKIP2 (FP32 sweeps): the chain of dependent blocks runs two blocks at a
// time. With P_b = inv(D_bb) T(b, b-1) (Mprev), Q_b = inv(D_bb) T(b, b-2)
// (sweep order), z_b = inv(D_bb)(b_b - sum over s <= b-3 of T(b, s) y_s):
//   y_b = z_b - P_b z_{b-1} + S_b y_{b-3} - R_b y_{b-2},
//   R_b = Q_b - P_b P_{b-1} (Mq), S_b = P_b Q_{b-1} (Ms), formed once per
// factorisation (k_mprev with distance 2, k_mprod). Block b publishes z_b to
// the second mailbox zbox as soon as it has it; only R_b y_{b-2} waits for a
// block's immediate chain, so the chain has n/256 steps instead of n/128.
template <class T, bool LOWER, bool SKIP2 = false>
__global__ void __launch_bounds__(kTrs1Threads)
k_trs1(const T* __restrict__ A, int64_t lda, int64_t n, const T* __restrict__ Dinv128, const T* __restrict__ Mprev,
       T* __restrict__ B, unsigned int* __restrict__ flags, unsigned int* __restrict__ ticket,
       int* __restrict__ status, unsigned long long* __restrict__ mbox, unsigned epoch,
       const T* __restrict__ Mq = nullptr, const T* __restrict__ Ms = nullptr,
       unsigned long long* __restrict__ zbox = nullptr) {
  static_assert(!SKIP2 || sizeof(T) == 4, "the two-block chain is for the FP32 sweeps");
  extern __shared__ __align__(16) unsigned char tsm[];
  T (*Ds)[SB + 1] = reinterpret_cast<T (*)[SB + 1]>(tsm);                    // Ds[l][r] = inv(D)(r, l)
  T (*red)[SB] = reinterpret_cast<T (*)[SB]>(tsm + (size_t)SB * (SB + 1) * sizeof(T));   // per phase
  T* accs = reinterpret_cast<T*>(tsm + (size_t)SB * (SB + 1) * sizeof(T) + (size_t)8 * SB * sizeof(T));
  T* xpart = accs + SB;
  T* xfin = xpart + SB;
  __shared__ int blk_s, stop_s;
  const int64_t nblk = (n + SB - 1) / SB;
  const int tid = threadIdx.x, lane = tid & 31;
  const int rg = tid & 31, ph = tid >> 5;   // rows 4rg..4rg+3, columns ph, ph+8, ...
  for (;;) {
    if (tid == 0) { blk_s = (int)atomicAdd(ticket, 1u); stop_s = 0; }
    __syncthreads();
    const int64_t tk = blk_s;
    if (tk >= nblk) return;
    const int64_t b = LOWER ? tk : nblk - 1 - tk;
    const int64_t k0 = b * SB;
    const int nb = (int)imin64(SB, n - k0);
    const T* Di = Dinv128 + b * 2 * SB * SB + (LOWER ? 0 : SB * SB);
    for (int e = tid; e < SB * SB; e += kTrs1Threads) Ds[e / SB][e % SB] = Di[e];   // Di column-major: e = l*SB + r
    // this block's right-hand side, written only by this CTA: fetched now,
    // off the chain of dependent blocks
    const T rhs = (tid < nb) ? B[k0 + tid] : T(0);
    T sum[4] = {T(0), T(0), T(0), T(0)};
    int64_t ready = 0;   // dependencies known complete (this warp)
    if constexpr (sizeof(T) == 4) {
      // every earlier block but the predecessor (but the last two with
      // SKIP2), its values from its mailbox: lanes 0..15 poll the words of
      // columns ph + 8 lane (spinning first, then backing off), the warp
      // shares them by shuffles
      for (int64_t s = 0; s + (SKIP2 ? 2 : 1) < tk; ++s) {
        const int64_t cb = LOWER ? s : nblk - 1 - s;
        const int64_t c0 = cb * SB;
        const int cn = (int)imin64(SB, n - c0);
        T a[16][4];
        load_tile4x16<T>(A + c0 * lda + k0, lda, rg, ph, nb, cn, a);
        float yl = 0.f;
        const int col = ph + 8 * lane;
        if (lane < 16 && col < cn) {
          int spins = 0;
          for (;;) {
            const unsigned long long w = ld_relaxed_u64(&mbox[c0 + col]);
            if ((unsigned)(w >> 32) == epoch) { yl = __uint_as_float((unsigned)w); break; }
            if (++spins > kSpinLimit) { atomicOr(status, (int)DEV_TIMEOUT); stop_s = 1; break; }
            if (spins > 64) __nanosleep(32);
          }
        }
        __syncwarp();
        if (stop_s) break;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const T yv = __shfl_sync(0xffffffffu, yl, i);
#pragma unroll
          for (int j = 0; j < 4; ++j) sum[j] += a[i][j] * yv;
        }
      }
    } else {
      for (int64_t s = 0; s + 1 < tk; ++s) {   // every earlier block but the predecessor
        const int64_t cb = LOWER ? s : nblk - 1 - s;
        const int64_t c0 = cb * SB;
        const int cn = (int)imin64(SB, n - c0);
        T a[16][4];
        load_tile4x16<T>(A + c0 * lda + k0, lda, rg, ph, nb, cn, a);
        if (s >= ready) {   // read the flags of up to 32 blocks at once
          int spins = 0;
          for (;;) {
            const int64_t sq = s + lane;
            const int64_t fb = LOWER ? sq : nblk - 1 - sq;
            const unsigned f = (sq < tk) ? ld_acquire(&flags[fb]) : 0u;
            const unsigned m = __ballot_sync(0xffffffffu, f != 0u);
            const int cnt = __ffs(~m) - 1;   // consecutive ready blocks from s
            if (m == 0xffffffffu) { ready = s + 32; break; }
            if (cnt > 0) { ready = s + cnt; break; }
            if (++spins > kSpinLimit) { atomicOr(status, (int)DEV_TIMEOUT); stop_s = 1; break; }
            __nanosleep(32);
          }
          __syncwarp();
          if (stop_s) break;
        }
  #pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int col = ph + 8 * i;
          const T yv = (col < cn) ? ld_cg(&B[c0 + col]) : T(0);
  #pragma unroll
          for (int j = 0; j < 4; ++j) sum[j] += a[i][j] * yv;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) red[ph][4 * rg + j] = sum[j];
    __syncthreads();
    if (stop_s) return;
    if (tid < SB) {
      T s0 = T(0);
#pragma unroll
      for (int q = 0; q < 8; ++q) s0 += red[q][tid];
      accs[tid] = (tid < nb) ? rhs - s0 : T(0);
    }
    __syncthreads();
    const int r = tid % SB, h = tid / SB;
    {   // x' = inv(D) acc: thread (r, half) sums half of the columns
      T s0 = T(0);
#pragma unroll 8
      for (int l = h * (SB / 2); l < (h + 1) * (SB / 2); ++l) s0 += Ds[l][r] * accs[l];
      if (h == 1) xpart[r] = s0;
      __syncthreads();
      if (h == 0) xfin[r] = s0 + xpart[r];
    }
    if constexpr (SKIP2) {
      // z_b for the next block in sweep order; then
      // y_b = z_b - (P_b z_{b-1} - S_b y_{b-3} + R_b y_{b-2}), the R_b term last
      if (h == 0 && r < nb)
        st_relaxed_u64(&zbox[k0 + r], ((unsigned long long)epoch << 32) | __float_as_uint(xfin[r]));
      T s2[4] = {T(0), T(0), T(0), T(0)};
      // s2 += sign M v over this thread's 4 rows x 16 columns, v the 128 words
      // of block vb in box (lanes 0..15 poll columns ph + 8 lane)
      auto add_mv = [&](const T* Mt, int64_t vb, const unsigned long long* box, T sign) {
        const int64_t v0 = vb * SB;
        const int nv = (int)imin64(SB, n - v0);
        T mt[16][4];
        load_tile4x16<T>(Mt, SB, rg, ph, nb, nv, mt);
        float yl = 0.f;
        const int col = ph + 8 * lane;
        if (lane < 16 && col < nv) {
          int spins = 0;
          for (;;) {
            const unsigned long long w = ld_relaxed_u64(&box[v0 + col]);
            if ((unsigned)(w >> 32) == epoch) { yl = __uint_as_float((unsigned)w); break; }
            if (++spins > kSpinLimit) { atomicOr(status, (int)DEV_TIMEOUT); stop_s = 1; break; }
          }
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const T yv = sign * __shfl_sync(0xffffffffu, yl, i);
#pragma unroll
          for (int j = 0; j < 4; ++j) s2[j] += mt[i][j] * yv;
        }
      };
      const int64_t dir = LOWER ? -1 : 1;
      const int64_t tile = (b * 2 + (LOWER ? 0 : 1)) * SB * SB;
      if (tk >= 1) add_mv(Mprev + tile, b + dir, zbox, T(1));
      if (tk >= 3) add_mv(Ms + tile, b + 3 * dir, mbox, T(-1));
      if (tk >= 2) add_mv(Mq + tile, b + 2 * dir, mbox, T(1));   // on the chain
#pragma unroll
      for (int j = 0; j < 4; ++j) red[ph][4 * rg + j] = s2[j];
      __syncthreads();
      if (stop_s) return;
      if (h == 0 && r < nb) {
        T s0 = T(0);
#pragma unroll
        for (int q = 0; q < 8; ++q) s0 += red[q][r];
        const T xv = xfin[r] - s0;
        st_relaxed_u64(&mbox[k0 + r], ((unsigned long long)epoch << 32) | __float_as_uint(xv));
        B[k0 + r] = xv;
      }
    } else if (tk > 0) {   // x_b = x' - Mprev_b y_p, on the chain
      // the predecessor's tile Mprev_b, loaded before the wait
      const int64_t pb = LOWER ? b - 1 : b + 1;
      const int np = (int)imin64(SB, n - pb * SB);
      T mp[16][4];
      load_tile4x16<T>(Mprev + (b * 2 + (LOWER ? 0 : 1)) * SB * SB, SB, rg, ph, nb, np, mp);
      T s2[4] = {T(0), T(0), T(0), T(0)};
      const int64_t p0 = pb * SB;
      if constexpr (sizeof(T) == 4) {
        // lanes 0..15 poll the mailbox words of columns ph + 8 lane
        float yl = 0.f;
        const int col = ph + 8 * lane;
        if (lane < 16 && col < np) {
          int spins = 0;
          for (;;) {
            const unsigned long long w = ld_relaxed_u64(&mbox[p0 + col]);
            if ((unsigned)(w >> 32) == epoch) { yl = __uint_as_float((unsigned)w); break; }
            if (++spins > kSpinLimit) { atomicOr(status, (int)DEV_TIMEOUT); stop_s = 1; break; }
          }
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const T yv = __shfl_sync(0xffffffffu, yl, i);
#pragma unroll
          for (int j = 0; j < 4; ++j) s2[j] += mp[i][j] * yv;
        }
      } else {
        if (lane == 0) {
          int spins = 0;
          while (!ld_acquire(&flags[pb])) {
            if (++spins > kSpinLimit) { atomicOr(status, (int)DEV_TIMEOUT); stop_s = 1; break; }
            __nanosleep(32);
          }
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int col = ph + 8 * i;
          const T yv = (col < np) ? ld_cg(&B[p0 + col]) : T(0);
#pragma unroll
          for (int j = 0; j < 4; ++j) s2[j] += mp[i][j] * yv;
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) red[ph][4 * rg + j] = s2[j];
      __syncthreads();
      if (stop_s) return;
      if (h == 0 && r < nb) {
        T s0 = T(0);
#pragma unroll
        for (int q = 0; q < 8; ++q) s0 += red[q][r];
        const T xv = xfin[r] - s0;
        if constexpr (sizeof(T) == 4)
          st_relaxed_u64(&mbox[k0 + r], ((unsigned long long)epoch << 32) | __float_as_uint(xv));
        B[k0 + r] = xv;
      }
    } else {
      __syncthreads();
      if (h == 0 && r < nb) {
        const T xv = xfin[r];
        if constexpr (sizeof(T) == 4)
          st_relaxed_u64(&mbox[k0 + r], ((unsigned long long)epoch << 32) | __float_as_uint(xv));
        B[k0 + r] = xv;
      }
    }
    // publish: the barrier orders the CTA's stores of x_b before thread 0's
    // release store of the flag
    __syncthreads();
    if (tid == 0) st_release(&flags[b], 1u);
  }
}

// Mprev_b = inv(D_bb) T(b, p) for the predecessor p of block b in each sweep
// (forward: p = b - 1, T = L; backward: p = b + 1, T = U), SB x SB
// column-major per block and sweep (zero past the matrix's rows and
// columns). blockIdx.y: 0 forward, 1 backward.
template <class T>
__global__ void __launch_bounds__(256)
k_mprev(const T* __restrict__ LU, int64_t lda, int64_t n, const T* __restrict__ Dinv128, T* __restrict__ Mprev,
        int dist = 1) {
  constexpr int KC = sizeof(T) == 4 ? 32 : 16;
  __shared__ __align__(16) T Dsh[KC][SB + 4];   // Dsh[l][r] = inv(D)(r, l0 + l)
  __shared__ __align__(16) T Tsh[KC][SB + 4];   // Tsh[l][c] = T(l0 + l, c)
  const int64_t nblk = (n + SB - 1) / SB;
  const int64_t b = blockIdx.x;
  const bool lower = blockIdx.y == 0;
  const int64_t p = lower ? b - dist : b + dist;
  if (p < 0 || p >= nblk) return;   // the sweep's first blocks have no such predecessor
  const int64_t k0 = b * SB, p0 = p * SB;
  const int nb = (int)imin64(SB, n - k0), np = (int)imin64(SB, n - p0);
  const T* Di = Dinv128 + b * 2 * SB * SB + (lower ? 0 : SB * SB);
  T* out = Mprev + (b * 2 + (lower ? 0 : 1)) * SB * SB;
  const int tid = threadIdx.x;
  const int r0 = 8 * (tid & 15), c0 = 8 * (tid >> 4);
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = T(0);
  for (int l0 = 0; l0 < SB; l0 += KC) {
    __syncthreads();
    for (int e = tid; e < KC * SB; e += 256) {
      const int r = e % SB, l = e / SB;
      Dsh[l][r] = Di[(l0 + l) * SB + r];
      const int ll = e % KC, c = e / KC;
      Tsh[ll][c] = (l0 + ll < nb && c < np) ? LU[(p0 + c) * lda + k0 + l0 + ll] : T(0);
    }
    __syncthreads();
#pragma unroll 4
    for (int l = 0; l < KC; ++l) {
      T x[8], y[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) { x[i] = Dsh[l][r0 + i]; y[i] = Tsh[l][c0 + i]; }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] += x[i] * y[j];
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int i = 0; i < 8; ++i) out[(c0 + j) * SB + r0 + i] = acc[i][j];
}

// The products of the two-block sweep chain, per 128-row block b and sweep
// (sweep order: p1, p2 = the blocks one and two before b):
//   job 0: Ms_b = P_b Q_{p1}            (b at sweep position >= 3)
//   job 1: Mq_b = Q_b - P_b P_{p1}       (b at sweep position >= 2, in place)
// P = Mprev, Q = Mq as k_mprev left it (distance 2); SB x SB column-major
// tiles whose columns beyond a partial block are zero. Job 0 runs before
// job 1 (it reads Q_{p1}).
template <class T>
__global__ void __launch_bounds__(256)
k_mprod(const T* __restrict__ P, T* __restrict__ Q, T* __restrict__ S, int64_t n, int job) {
  constexpr int KC = sizeof(T) == 4 ? 32 : 16;
  __shared__ __align__(16) T Ysh[KC][SB + 4];   // Ysh[l][r] = P_b(r, l0 + l)
  __shared__ __align__(16) T Zsh[KC][SB + 4];   // Zsh[l][c] = Z(l0 + l, c)
  const int64_t nblk = (n + SB - 1) / SB;
  const int64_t b = blockIdx.x;
  const bool lower = blockIdx.y == 0;
  const int64_t tk = lower ? b : nblk - 1 - b;
  if (tk < (job == 0 ? 3 : 2)) return;
  const int64_t p1 = lower ? b - 1 : b + 1;
  const int64_t tb = (b * 2 + (lower ? 0 : 1)) * SB * SB, tp = (p1 * 2 + (lower ? 0 : 1)) * SB * SB;
  const T* Y = P + tb;
  const T* Z = job == 0 ? Q + tp : P + tp;
  T* out = job == 0 ? S + tb : Q + tb;
  const int tid = threadIdx.x;
  const int r0 = 8 * (tid & 15), c0 = 8 * (tid >> 4);
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = T(0);
  for (int l0 = 0; l0 < SB; l0 += KC) {
    __syncthreads();
    for (int e = tid; e < KC * SB; e += 256) {
      const int r = e % SB, l = e / SB;
      Ysh[l][r] = Y[(l0 + l) * SB + r];
      const int ll = e % KC, c = e / KC;
      Zsh[ll][c] = Z[c * SB + l0 + ll];
    }
    __syncthreads();
#pragma unroll 4
    for (int l = 0; l < KC; ++l) {
      T x[8], y[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) { x[i] = Ysh[l][r0 + i]; y[i] = Zsh[l][c0 + i]; }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] += x[i] * y[j];
    }
  }
  __syncthreads();   // job 1 overwrites Q_b, which no other block of this launch reads
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int64_t o = (int64_t)(c0 + j) * SB + r0 + i;
      out[o] = job == 0 ? acc[i][j] : out[o] - acc[i][j];
    }
}

// Inverses of the 128-row diagonal blocks from those of the 64-row blocks:
// inv(L_B) = [[Li0, 0], [-Li1 L21 Li0, Li1]], inv(U_B) = [[Ui0, -Ui0 U12 Ui1],
// [0, Ui1]]; Dinv128[B] = inv(L_B), inv(U_B), SB x SB column-major each.
template <class T> constexpr size_t dinv128_smem() { return (size_t)4 * NB * (NB + 1) * sizeof(T); }

template <class T>
__global__ void __launch_bounds__(256)
k_dinv128(const T* __restrict__ LU, int64_t lda, int64_t n, const T* __restrict__ Dinv64, T* __restrict__ Dinv128) {
  extern __shared__ __align__(16) unsigned char dsm3[];
  T (*X)[NB + 1] = reinterpret_cast<T (*)[NB + 1]>(dsm3);   // [r][c]
  T (*Y)[NB + 1] = X + NB;
  T (*Z)[NB + 1] = X + 2 * NB;
  T (*W)[NB + 1] = X + 3 * NB;
  const int tid = threadIdx.x;
  const int64_t B = blockIdx.x;
  const int64_t i0 = 2 * B, k0 = B * SB;
  const bool two = k0 + NB < n;
  const int n1 = two ? (int)imin64(NB, n - k0 - NB) : 0;
  T* outL = Dinv128 + B * 2 * SB * SB;
  T* outU = outL + SB * SB;
  for (int e = tid; e < SB * SB; e += 256) { outL[e] = T(0); outU[e] = T(0); }
  __syncthreads();
  // diagonal quadrants: the 64-row inverses (identity for a missing second block)
  for (int e = tid; e < NB * NB; e += 256) {
    const int r = e % NB, c = e / NB;
    const T* L0 = Dinv64 + i0 * 2 * NB * NB;
    outL[c * SB + r] = L0[e];
    outU[c * SB + r] = L0[NB * NB + e];
    T l1 = (r == c) ? T(1) : T(0), u1 = l1;
    if (two) {
      const T* L1 = Dinv64 + (i0 + 1) * 2 * NB * NB;
      l1 = L1[e];
      u1 = L1[NB * NB + e];
    }
    outL[(NB + c) * SB + NB + r] = l1;
    outU[(NB + c) * SB + NB + r] = u1;
  }
  if (!two) return;
  auto mm = [&](T (*C)[NB + 1], T (*P)[NB + 1], T (*Q)[NB + 1], T sgn) {   // C = sgn * P Q
    for (int e = tid; e < NB * NB; e += 256) {
      const int r = e % NB, c = e / NB;
      T s = T(0);
      for (int l = 0; l < NB; ++l) s += P[r][l] * Q[l][c];
      C[r][c] = sgn * s;
    }
  };
  const T* L0 = Dinv64 + i0 * 2 * NB * NB;
  const T* L1 = Dinv64 + (i0 + 1) * 2 * NB * NB;
  // lower: X = L21, Y = Li0 -> Z = L21 Li0; Y = Li1 -> W = -Li1 Z
  for (int e = tid; e < NB * NB; e += 256) {
    const int r = e % NB, c = e / NB;
    X[r][c] = (r < n1) ? LU[(k0 + c) * lda + k0 + NB + r] : T(0);
    Y[r][c] = L0[e];
  }
  __syncthreads();
  mm(Z, X, Y, T(1));
  __syncthreads();
  for (int e = tid; e < NB * NB; e += 256) Y[e % NB][e / NB] = L1[e];
  __syncthreads();
  mm(W, Y, Z, T(-1));
  __syncthreads();
  for (int e = tid; e < NB * NB; e += 256) {
    const int r = e % NB, c = e / NB;
    outL[c * SB + NB + r] = W[r][c];
  }
  // upper: X = U12, Y = Ui1 -> Z = U12 Ui1; Y = Ui0 -> W = -Ui0 Z
  __syncthreads();
  for (int e = tid; e < NB * NB; e += 256) {
    const int r = e % NB, c = e / NB;
    X[r][c] = (c < n1) ? LU[(k0 + NB + c) * lda + k0 + r] : T(0);
    Y[r][c] = L1[NB * NB + e];
  }
  __syncthreads();
  mm(Z, X, Y, T(1));
  __syncthreads();
  for (int e = tid; e < NB * NB; e += 256) Y[e % NB][e / NB] = L0[NB * NB + e];
  __syncthreads();
  mm(W, Y, Z, T(-1));
  __syncthreads();
  for (int e = tid; e < NB * NB; e += 256) {
    const int r = e % NB, c = e / NB;
    outU[(NB + c) * SB + r] = W[r][c];
  }
}

template <class T, bool LOWER>
static int run_trs1(fp_ctx* c, const T* A, int64_t n, int64_t lda, const T* Dinv128, const T* Mprev, T* B) {
  const int64_t nblk = (n + SB - 1) / SB;
  FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_flags, 0, (nblk + 1) * sizeof(unsigned int), c->stream));
  const unsigned grid = (unsigned)std::min<int64_t>(nblk, 2 * num_sms());
  if (++c->trs_epoch == 0) ++c->trs_epoch;   // epoch 0 marks words never written
  if constexpr (sizeof(T) == 4) {
    if (c->trs_skip2 && c->trs2_ready) {
      k_trs1<float, LOWER, true><<<grid, kTrs1Threads, trs1_smem<T>(), c->stream>>>(
          A, lda, n, Dinv128, Mprev, B, c->d_flags, c->d_flags + nblk, c->d_status, c->d_mbox, c->trs_epoch,
          c->d_mq32, c->d_ms32, c->d_zbox);
      ++c->nlaunch;
      FP_CUDA_TRY(c->err, cudaGetLastError());
      return FP_OK;
    }
  }
  k_trs1<T, LOWER><<<grid, kTrs1Threads, trs1_smem<T>(), c->stream>>>(A, lda, n, Dinv128, Mprev, B, c->d_flags,
                                                                      c->d_flags + nblk, c->d_status, c->d_mbox,
                                                                      c->trs_epoch);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

template <class T, bool LOWER, int KR, bool TRANS = false>
static int run_trs(fp_ctx* c, const T* A, int64_t n, int64_t lda, const T* Dinv, T* B,
                   int64_t ldb) {
  const int64_t nblk = (n + NB - 1) / NB;
  FP_CUDA_TRY(c->err, cudaMemsetAsync(c->d_flags, 0, (nblk + 1) * sizeof(unsigned int), c->stream));
  const unsigned grid = (unsigned)std::min<int64_t>(nblk, 2 * num_sms());
  k_trs<T, LOWER, KR, TRANS><<<grid, kTrsThreads, 0, c->stream>>>(A, lda, n, Dinv, B, ldb, c->d_flags,
                                                                  c->d_flags + nblk, c->d_status);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

template <class T, bool TRANS = false>
static int solve_group(fp_ctx* c, const T* LU, int64_t n, int64_t lda, const T* Dinv, T* B,
                       int64_t ldb, int kr) {
  int rc;
#define FP_TRS_CASE(KR)                                                               \
  case KR:                                                                            \
    if ((rc = run_trs<T, true, KR, TRANS>(c, LU, n, lda, Dinv, B, ldb))) return rc;   \
    return run_trs<T, false, KR, TRANS>(c, LU, n, lda, Dinv, B, ldb);
  switch (kr) {
    FP_TRS_CASE(1)
    FP_TRS_CASE(2)
    FP_TRS_CASE(4)
    FP_TRS_CASE(8)
  }
#undef FP_TRS_CASE
  return c->err.set(FP_EINVAL, "unsupported RHS group");
}

// Dinv buffer and flags are sized by the caller (fp_capi.cu) for n.
// P A = L U. Plain: B <- P B, L y = B, U x = y. Transposed (A^T x = B):
// U^T z = B, L^T v = z, x = P^T v (the swaps in reverse order).
template <class T>
int lu_solve(fp_ctx* c, const T* LU, int64_t n, int64_t lda, const int32_t* ipiv, T* B,
             int64_t ldb, int64_t k, bool transpose) {
  const int64_t nblk = (n + NB - 1) / NB;
  T* Dinv = reinterpret_cast<T*>(sizeof(T) == 8 ? (void*)c->d_dinv64 : (void*)c->d_dinv32);
  // the static-order FP32 factors have the identity row order: no swaps
  const bool identity_piv = sizeof(T) == 4 && c->static_order;
  if (transpose) {
    for (int64_t q0 = 0; q0 < k;) {
      const int64_t left = k - q0;
      const int kr = left >= 8 ? 8 : left >= 4 ? 4 : left >= 2 ? 2 : 1;
      int rc = solve_group<T, true>(c, LU, n, lda, Dinv, B + q0 * ldb, ldb, kr);
      if (rc) return rc;
      q0 += kr;
    }
    if (identity_piv) return FP_OK;
    const int64_t t = nblk * k;
    k_apply_piv<T><<<(unsigned)((t + 127) / 128), 128, 0, c->stream>>>(B, ldb, n, k, ipiv, true);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
    return FP_OK;
  }
  if (!identity_piv) {
    const int64_t t = nblk * k;
    k_apply_piv<T><<<(unsigned)((t + 127) / 128), 128, 0, c->stream>>>(B, ldb, n, k, ipiv, false);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
  }
  if (k == 1) {   // one right-hand side: the 128-row streaming sweeps
    const T* D128 = reinterpret_cast<const T*>(sizeof(T) == 8 ? (void*)c->d_dinv128_64 : (void*)c->d_dinv128_32);
    const T* Mp = reinterpret_cast<const T*>(sizeof(T) == 8 ? (void*)c->d_mprev64 : (void*)c->d_mprev32);
    static SmemAttr attr_lo, attr_up;
    FP_CUDA_TRY(c->err, attr_lo.ensure(k_trs1<T, true>, (int)trs1_smem<T>()));
    FP_CUDA_TRY(c->err, attr_up.ensure(k_trs1<T, false>, (int)trs1_smem<T>()));
    if constexpr (sizeof(T) == 4) {
      static SmemAttr attr_lo2, attr_up2;
      FP_CUDA_TRY(c->err, attr_lo2.ensure(k_trs1<float, true, true>, (int)trs1_smem<T>()));
      FP_CUDA_TRY(c->err, attr_up2.ensure(k_trs1<float, false, true>, (int)trs1_smem<T>()));
    }
    if (int rc = run_trs1<T, true>(c, LU, n, lda, D128, Mp, B)) return rc;
    return run_trs1<T, false>(c, LU, n, lda, D128, Mp, B);
  }
  for (int64_t q0 = 0; q0 < k;) {
    const int64_t left = k - q0;
    const int kr = left >= 8 ? 8 : left >= 4 ? 4 : left >= 2 ? 2 : 1;
    int rc = solve_group<T>(c, LU, n, lda, Dinv, B + q0 * ldb, ldb, kr);
    if (rc) return rc;
    q0 += kr;
  }
  return FP_OK;
}

template <class T>
int lu_diag_inverses(fp_ctx* c, const T* LU, int64_t n, int64_t lda) {
  const int64_t nblk = (n + NB - 1) / NB;
  T* Dinv = reinterpret_cast<T*>(sizeof(T) == 8 ? (void*)c->d_dinv64 : (void*)c->d_dinv32);
  k_diag_inv<T><<<(unsigned)nblk, NB, 0, c->stream>>>(LU, lda, n, Dinv);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  T* D128 = reinterpret_cast<T*>(sizeof(T) == 8 ? (void*)c->d_dinv128_64 : (void*)c->d_dinv128_32);
  static SmemAttr attr;
  FP_CUDA_TRY(c->err, attr.ensure(k_dinv128<T>, (int)dinv128_smem<T>()));
  k_dinv128<T><<<(unsigned)((n + SB - 1) / SB), 256, dinv128_smem<T>(), c->stream>>>(LU, lda, n, Dinv, D128);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  T* Mp = reinterpret_cast<T*>(sizeof(T) == 8 ? (void*)c->d_mprev64 : (void*)c->d_mprev32);
  const dim3 gm((unsigned)((n + SB - 1) / SB), 2);
  k_mprev<T><<<gm, 256, 0, c->stream>>>(LU, lda, n, D128, Mp);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  if constexpr (sizeof(T) == 4) {
    // the two-block chain of the FP32 sweeps: Q (distance 2), then S = P Q_p1,
    // then R = Q - P P_p1 in place of Q
    c->trs2_ready = false;
    if (c->trs_skip2 && c->d_mq32 && c->d_ms32 && c->d_zbox) {
      k_mprev<float><<<gm, 256, 0, c->stream>>>(LU, lda, n, D128, c->d_mq32, 2);
      k_mprod<float><<<gm, 256, 0, c->stream>>>(c->d_mprev32, c->d_mq32, c->d_ms32, n, 0);
      k_mprod<float><<<gm, 256, 0, c->stream>>>(c->d_mprev32, c->d_mq32, c->d_ms32, n, 1);
      c->nlaunch += 3;
      FP_CUDA_TRY(c->err, cudaGetLastError());
      c->trs2_ready = true;
    }
  }
  return FP_OK;
}

// ----------------------------------------------------------------------------
// r = b - A x (FP64), k right-hand sides, split over column ranges.
constexpr int kGemvRows = 128;
constexpr int kGemvSplit = 16;
template <int KR>
__global__ void __launch_bounds__(kGemvRows)
k_gemv_partial(const double* __restrict__ A, int64_t lda, int64_t n, const double* __restrict__ x,
               int64_t ldx, double* __restrict__ part) {
  const int64_t i = (int64_t)blockIdx.x * kGemvRows + threadIdx.x;
  const int64_t cs = (n + kGemvSplit - 1) / kGemvSplit;
  const int64_t c0 = blockIdx.y * cs, c1 = imin64(n, c0 + cs);
  double s[KR];
#pragma unroll
  for (int q = 0; q < KR; ++q) s[q] = 0.0;
  if (i < n) {
    for (int64_t j = c0; j < c1; ++j) {
      const double a = A[j * lda + i];
#pragma unroll
      for (int q = 0; q < KR; ++q) s[q] += a * __ldg(&x[q * ldx + j]);
    }
#pragma unroll
    for (int q = 0; q < KR; ++q) part[((int64_t)blockIdx.y * KR + q) * n + i] = s[q];
  }
}

template <int KR>
__global__ void k_gemv_finish(const double* __restrict__ part, int64_t n, const double* __restrict__ b,
                              int64_t ldb, double* __restrict__ r, int64_t ldr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int q = 0; q < KR; ++q) {
    double s = 0.0;
    for (int p = 0; p < kGemvSplit; ++p) s += part[((int64_t)p * KR + q) * n + i];
    r[q * ldr + i] = b[q * ldb + i] - s;
  }
}

int gemv_residual(fp_ctx* c, const double* A, int64_t n, int64_t lda, const double* x,
                  const double* b, double* r, int64_t k) {
  for (int64_t q0 = 0; q0 < k;) {
    const int64_t left = k - q0;
    const int kr = left >= 4 ? 4 : left >= 2 ? 2 : 1;
    dim3 g((unsigned)((n + kGemvRows - 1) / kGemvRows), kGemvSplit);
    const unsigned gf = (unsigned)((n + 255) / 256);
    const double* xq = x + q0 * lda;
    if (kr == 4) {
      k_gemv_partial<4><<<g, kGemvRows, 0, c->stream>>>(A, lda, n, xq, lda, c->d_part);
      ++c->nlaunch;
      k_gemv_finish<4><<<gf, 256, 0, c->stream>>>(c->d_part, n, b + q0 * lda, lda, r + q0 * lda, lda);
      ++c->nlaunch;
    } else if (kr == 2) {
      k_gemv_partial<2><<<g, kGemvRows, 0, c->stream>>>(A, lda, n, xq, lda, c->d_part);
      ++c->nlaunch;
      k_gemv_finish<2><<<gf, 256, 0, c->stream>>>(c->d_part, n, b + q0 * lda, lda, r + q0 * lda, lda);
      ++c->nlaunch;
    } else {
      k_gemv_partial<1><<<g, kGemvRows, 0, c->stream>>>(A, lda, n, xq, lda, c->d_part);
      ++c->nlaunch;
      k_gemv_finish<1><<<gf, 256, 0, c->stream>>>(c->d_part, n, b + q0 * lda, lda, r + q0 * lda, lda);
      ++c->nlaunch;
    }
    FP_CUDA_TRY(c->err, cudaGetLastError());
    q0 += kr;
  }
  return FP_OK;
}

// ----------------------------------------------------------------------------
// r = b - A^T x (FP64), k right-hand sides: one warp per column j of A (the
// column is contiguous, read with 16-byte loads when aligned), x read through
// L1; the dot product reduced by shuffles. HBM-bound: 8 N^2 bytes per pass.
constexpr int kGemvTThreads = 256;
template <int KR>
__global__ void __launch_bounds__(kGemvTThreads)
k_gemvT_residual(const double* __restrict__ A, int64_t lda, int64_t n, const double* __restrict__ x,
                 const double* __restrict__ b, double* __restrict__ r, int64_t ldx, bool vec) {
  const int lane = threadIdx.x & 31;
  const int64_t j = (int64_t)blockIdx.x * (kGemvTThreads / 32) + (threadIdx.x >> 5);
  if (j >= n) return;
  const double* col = A + j * lda;
  double s[KR];
#pragma unroll
  for (int q = 0; q < KR; ++q) s[q] = 0.0;
  int64_t i0 = 0;
  if (vec) {
    const int64_t n2 = n & ~int64_t(63);
    for (int64_t i = 2 * lane; i < n2; i += 64) {
      const double2 a = *reinterpret_cast<const double2*>(col + i);
#pragma unroll
      for (int q = 0; q < KR; ++q) {
        const double2 xv = __ldg(reinterpret_cast<const double2*>(x + q * ldx + i));
        s[q] += a.x * xv.x;
        s[q] += a.y * xv.y;
      }
    }
    i0 = n2;
  }
  for (int64_t i = i0 + lane; i < n; i += 32) {
    const double a = col[i];
#pragma unroll
    for (int q = 0; q < KR; ++q) s[q] += a * __ldg(&x[q * ldx + i]);
  }
#pragma unroll
  for (int q = 0; q < KR; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < KR; ++q) r[q * ldx + j] = b[q * ldx + j] - s[q];
  }
}

int gemvT_residual(fp_ctx* c, const double* A, int64_t n, int64_t lda, const double* x,
                   const double* b, double* r, int64_t k) {
  const bool vec = ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(x) |
                     (uintptr_t)(lda * sizeof(double))) & 15) == 0;
  const unsigned g = (unsigned)((n + kGemvTThreads / 32 - 1) / (kGemvTThreads / 32));
  for (int64_t q0 = 0; q0 < k;) {
    const int64_t left = k - q0;
    const int kr = left >= 4 ? 4 : left >= 2 ? 2 : 1;
    const int64_t o = q0 * lda;
    if (kr == 4) k_gemvT_residual<4><<<g, kGemvTThreads, 0, c->stream>>>(A, lda, n, x + o, b + o, r + o, lda, vec);
    else if (kr == 2) k_gemvT_residual<2><<<g, kGemvTThreads, 0, c->stream>>>(A, lda, n, x + o, b + o, r + o, lda, vec);
    else k_gemvT_residual<1><<<g, kGemvTThreads, 0, c->stream>>>(A, lda, n, x + o, b + o, r + o, lda, vec);
    ++c->nlaunch;
    FP_CUDA_TRY(c->err, cudaGetLastError());
    q0 += kr;
  }
  return FP_OK;
}

// ----------------------------------------------------------------------------
__global__ void k_f64_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n,
                             int64_t k, int64_t lda, int64_t ldb) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * k) return;
  const int64_t i = t % n, q = t / n;
  b[q * ldb + i] = (float)a[q * lda + i];
}
__global__ void k_axpy_f32(const float* __restrict__ d, double* __restrict__ x, int64_t n,
                           int64_t k, int64_t ld) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * k) return;
  const int64_t i = t % n, q = t / n;
  x[q * ld + i] += (double)d[q * ld + i];
}

int convert_f64_f32(fp_ctx* c, const double* a, float* b, int64_t n, int64_t k, int64_t lda,
                    int64_t ldb) {
  const int64_t t = n * k;
  k_f64_to_f32<<<(unsigned)((t + 255) / 256), 256, 0, c->stream>>>(a, b, n, k, lda, ldb);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}
__global__ void k_f64_to_bf16f32(const double* __restrict__ a, float* __restrict__ b, int64_t n, int64_t k,
                                 int64_t lda, int64_t ldb) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * k) return;
  const int64_t i = t % n, q = t / n;
  b[q * ldb + i] = __bfloat162float(__float2bfloat16_rn((float)a[q * lda + i]));
}
int convert_f64_bf16(fp_ctx* c, const double* a, float* b, int64_t n, int64_t k, int64_t lda, int64_t ldb) {
  const int64_t t = n * k;
  k_f64_to_bf16f32<<<(unsigned)((t + 255) / 256), 256, 0, c->stream>>>(a, b, n, k, lda, ldb);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}
int axpy_f32_to_f64(fp_ctx* c, const float* d, double* x, int64_t n, int64_t k, int64_t ld) {
  const int64_t t = n * k;
  k_axpy_f32<<<(unsigned)((t + 255) / 256), 256, 0, c->stream>>>(d, x, n, k, ld);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}
__global__ void k_axpy_f64(const double* __restrict__ d, double* __restrict__ x, int64_t n, int64_t k, int64_t ld) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * k) return;
  const int64_t i = t % n, q = t / n;
  x[q * ld + i] += d[q * ld + i];
}
int axpy_f64(fp_ctx* c, const double* d, double* x, int64_t n, int64_t k, int64_t ld) {
  const int64_t t = n * k;
  k_axpy_f64<<<(unsigned)((t + 255) / 256), 256, 0, c->stream>>>(d, x, n, k, ld);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

// column norms ||a_q||_2^2 for q < k (one CTA per column)
__global__ void k_colnorm2(const double* __restrict__ a, int64_t n, int64_t lda, double* __restrict__ out) {
  __shared__ double red[256 / 32];
  const int64_t q = blockIdx.x;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) { const double v = a[q * lda + i]; s += v * v; }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 256 / 32; ++w) t += red[w];
    out[q] = t;
  }
}
int colnorm2(fp_ctx* c, const double* a, int64_t n, int64_t lda, int64_t k, double* d_out) {
  k_colnorm2<<<(unsigned)k, 256, 0, c->stream>>>(a, n, lda, d_out);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

// ----------------------------------------------------------------------------
// Allocation-free solve with the FP64 factors of a context
// (fp_lu_solve_noalloc). Some callers cannot let a library allocate device
// memory while they solve: a host program that hands every byte of the device
// to its own pool or arena (a Julia session whose CUDA.jl pool holds the
// device memory, a service with a fixed memory budget), or one that re-solves
// inside a time-stepping or design loop where a cudaMalloc may synchronise the
// device or fail once the pool is full. For them the ready flags and the
// ticket counter of k_trs live in the file-scope array below instead of a
// context buffer; everything else the solve touches (factors, inverses of the
// diagonal blocks, pivots, status word) was allocated by fp_factor, and the
// right-hand sides are the caller's.
//
// The array holds one flag per 64-row block plus the ticket, so n is limited
// to kNoAllocMaxN unknowns (4 KiB per device). Every flag and the ticket must
// be zero when a sweep starts; each sweep clears them itself with
// cudaMemsetAsync on the context's stream, so callers initialise nothing.
// There is one array per device, shared by every context on that device:
// calls that overlap in time on one device (from several host threads) race
// on it and return wrong results or FP_ETIMEOUT, so they must be serialised.
constexpr int64_t kNoAllocMaxN = 65536;
constexpr int64_t kNoAllocMaxBlocks = kNoAllocMaxN / NB;
static __device__ __align__(256) unsigned int g_trs_scratch[kNoAllocMaxBlocks + 1];

// Device address of g_trs_scratch on the context's device, which must be the
// current device, resolved on every call with cudaGetSymbolAddress: that
// allocates nothing once this library's device code is loaded on the device
// (the first call may load it), and it follows the module when a device reset
// (cudaDeviceReset, CUDA.device_reset!) reloads it at another address.
static int trs_scratch_address(fp_ctx* c, unsigned int** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_trs_scratch);
  if (e != cudaSuccess)
    return c->err.set(FP_ECUDA, std::string("cudaGetSymbolAddress(g_trs_scratch): ") + cudaGetErrorString(e));
  *out = static_cast<unsigned int*>(p);
  return FP_OK;
}

template <bool LOWER, int KR>
static int run_trs_static(fp_ctx* c, int64_t n, double* B, int64_t ldb, unsigned int* flags) {
  const int64_t nblk = (n + NB - 1) / NB;
  FP_CUDA_TRY(c->err, cudaMemsetAsync(flags, 0, (nblk + 1) * sizeof(unsigned int), c->stream));
  const unsigned grid = (unsigned)std::min<int64_t>(nblk, 2 * num_sms());
  k_trs<double, LOWER, KR><<<grid, kTrsThreads, 0, c->stream>>>(c->d_LU, c->ld, n, c->d_dinv64, B, ldb, flags,
                                                                flags + nblk, c->d_status);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  return FP_OK;
}

int lu_solve_noalloc(fp_ctx* c, double* B, int64_t ldb, int64_t k) {
  const int64_t n = c->N;
  if (n > kNoAllocMaxN)
    return c->err.set(FP_EINVAL, "fp_lu_solve_noalloc: " + std::to_string(n) +
                                     " unknowns exceed the static scratch limit of " +
                                     std::to_string(kNoAllocMaxN));
  unsigned int* flags = nullptr;
  if (int rc = trs_scratch_address(c, &flags)) return rc;
  const int64_t nblk = (n + NB - 1) / NB;
  k_apply_piv<double><<<(unsigned)((nblk * k + 127) / 128), 128, 0, c->stream>>>(B, ldb, n, k, c->d_ipiv, false);
  ++c->nlaunch;
  FP_CUDA_TRY(c->err, cudaGetLastError());
  for (int64_t q0 = 0; q0 < k;) {
    const int64_t left = k - q0;
    const int kr = left >= 8 ? 8 : left >= 4 ? 4 : left >= 2 ? 2 : 1;
    double* Bq = B + q0 * ldb;
    int rc;
    switch (kr) {
      case 8: rc = run_trs_static<true, 8>(c, n, Bq, ldb, flags); if (!rc) rc = run_trs_static<false, 8>(c, n, Bq, ldb, flags); break;
      case 4: rc = run_trs_static<true, 4>(c, n, Bq, ldb, flags); if (!rc) rc = run_trs_static<false, 4>(c, n, Bq, ldb, flags); break;
      case 2: rc = run_trs_static<true, 2>(c, n, Bq, ldb, flags); if (!rc) rc = run_trs_static<false, 2>(c, n, Bq, ldb, flags); break;
      default: rc = run_trs_static<true, 1>(c, n, Bq, ldb, flags); if (!rc) rc = run_trs_static<false, 1>(c, n, Bq, ldb, flags); break;
    }
    if (rc) return rc;
    q0 += kr;
  }
  return FP_OK;
}

template int lu_factor<double>(fp_ctx*, double*, int64_t, int64_t, int32_t*, float*);
template int lu_factor<float>(fp_ctx*, float*, int64_t, int64_t, int32_t*, float*);
template int lu_solve<double>(fp_ctx*, const double*, int64_t, int64_t, const int32_t*, double*, int64_t, int64_t, bool);
template int lu_solve<float>(fp_ctx*, const float*, int64_t, int64_t, const int32_t*, float*, int64_t, int64_t, bool);
template int lu_diag_inverses<double>(fp_ctx*, const double*, int64_t, int64_t);
template int lu_diag_inverses<float>(fp_ctx*, const float*, int64_t, int64_t);

}  // namespace fpb
