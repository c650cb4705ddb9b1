// FP32 LU with a static row order, the factorisation of the mixed-precision
// form (FP_PREC_MIXED).
//
// The FP32 factors only have to be good enough for FP64 iterative refinement
// (and GMRES-IR behind it) to recover the FP64 solution, so no pivot search
// runs at factorisation time: the rows keep the order of the panels (static
// pivoting). The panel AICs of this path have their column maxima on or next
// to the diagonal, and unpivoted elimination keeps the multipliers of order
// one; max|L| is recorded (when it is <= 1 the factors are the ones partial
// pivoting would give). A zero or non-finite pivot sets DEV_ZERO_PIVOT and the
// caller falls back to the pivoted factorisation of fp_lu.cu.
//
// Without a pivot search the 128 x 128 diagonal block of a panel is the only
// sequential work; everything else is tile products:
//   K1 k_pdiag  one CTA factors the diagonal block in shared memory (32-wide
//               inner blocks: one warp eliminates a 32 x 32 block in
//               registers, two warps invert its L and U, all 16 warps form
//               the inner L / U blocks and the update as register-tiled
//               products) and keeps the inverses of the four 32 x 32 diagonal
//               blocks of L and U;
//   K6 k_l21    L21 = A21 U^-1 for the rows below, 64 rows per CTA, by block
//               substitution with those inverses; writes L21 in place and its
//               3xTF32 split (hi, lo; K-major) for the tensor-core update;
//   K2 k_u12    U12 = L^-1 A12 for a range of columns, likewise, in place and
//               split;
//   K3/K5       the trailing update C -= L21 U12 on tcgen05 (fp_tc.cu) from
//               the split operands, with no separate split pass.
// Look-ahead on two streams (lu_factor_static): the panel stream runs K1, K6,
// then (after the previous panel's trailing update) K2 and K3 on the next
// panel's columns; the second stream runs K2 and K5 on the columns beyond.
// The panel width equals the triangular solves' 128-row blocks.
#include <cuda_bf16.h>

#include <cfloat>

#include "fp_internal.cuh"

namespace fpb {
namespace st {

constexpr int PW = kStaticPanel;   // panel width (128)
constexpr int IB = 32;             // inner block of the diagonal factor
constexpr int NIB = PW / IB;       // inner blocks per panel
constexpr int SP = PW + 4;         // shared row pitch (floats) of 128-wide rows: 16-byte rows, not 32 banks
constexpr int kDiagThreads = 256;
constexpr unsigned FULL = 0xffffffffu;

// dinv layout per panel: [t][0] = inv(L_tt) (unit lower), [t][1] = inv(U_tt),
// each IB x IB row-major
constexpr int kDinvFloats = NIB * 2 * IB * IB;
__host__ __device__ constexpr int dinv_off(int t, int which) { return (t * 2 + which) * IB * IB; }

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  return __uint_as_float(h);
}

// 1/x from the special-function unit (relative error ~1e-7): the FP32
// factors only precondition FP64 refinement, so correct rounding buys nothing
__device__ __forceinline__ float rcp_fast(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void atomic_max_pos(float* addr, float v) {
  if (v > 0.f) atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

// Staging helpers: global <-> shared copies of column-major blocks with
// 16-byte loads, all of a thread's loads issued before its shared stores.
// Column c of the block starts at g + c * ld (rows contiguous); element
// (r, c) goes to or comes from s(r, c). Rows past `rows` / columns past
// `cols` read as zero (or `pad(r, c)`) and are not written.
// Piece q covers rows r..r+3 of column c. With 16 or more columns, a warp's
// 32 pieces are two row quads x 16 columns, so that the transposing shared
// accesses of a row-major copy (pitch = 4 mod 32 floats) hit 32 distinct
// banks and each 32-byte sector of global memory is read by one pair of lanes.
template <int ROWS, int COLS>
__device__ __forceinline__ void piece(int q, int& r, int& c) {
  constexpr int R4 = ROWS / 4;
  if constexpr (COLS % 16 == 0 && R4 % 2 == 0) {
    const int h = q & 1, cl = (q >> 1) & 15, rest = q >> 5;
    const int g = rest % (R4 / 2), cb = rest / (R4 / 2);
    r = (2 * g + h) * 4;
    c = cb * 16 + cl;
  } else {
    c = q / R4;
    r = (q % R4) * 4;
  }
}
// A block in flight: fetch() issues all of a thread's 16-byte loads, put()
// stores them to shared memory, so that a kernel can issue the loads of all
// its blocks before the first store (one round trip to L2 / HBM, not one a
// block).
template <int NT, int ROWS, int COLS>
struct Staged {
  static constexpr int R4 = ROWS / 4, NV = R4 * COLS, PER = (NV + NT - 1) / NT;
  float4 v[PER];
  template <class Pad>
  __device__ __forceinline__ void fetch(const float* __restrict__ g, int64_t ld, int rows, int cols, Pad pad, int tid) {
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int q = tid + u * NT;
      int r, c;
      piece<ROWS, COLS>(q, r, c);
      if (q < NV && c < cols && r + 4 <= rows) {
        v[u] = __ldcg(reinterpret_cast<const float4*>(g + (int64_t)c * ld + r));
      } else if (q < NV) {
        float t[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) t[i] = (c < cols && r + i < rows) ? __ldcg(g + (int64_t)c * ld + r + i) : pad(r + i, c);
        v[u] = make_float4(t[0], t[1], t[2], t[3]);
      }
    }
  }
  template <class S>
  __device__ __forceinline__ void put(S s, int tid) const {
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int q = tid + u * NT;
      if (q < NV) {
        int r, c;
        piece<ROWS, COLS>(q, r, c);
        s(r, c, v[u].x); s(r + 1, c, v[u].y); s(r + 2, c, v[u].z); s(r + 3, c, v[u].w);
      }
    }
  }
};
// The four IB x IB inverses of one kind (which = 0: L, 1: U) of a panel's
// dinv into dst (inverse t's row r at dst[t * IB + r]) by asynchronous
// 16-byte copies (cp.async: no registers, all in flight at once); the caller
// waits with cp_async_wait_all() before its __syncthreads.
template <int NT, int P>
__device__ __forceinline__ void copy_inv_async(float (*dst)[P], const float* __restrict__ dinv, int which, int tid) {
  constexpr int NV = NIB * IB * IB / 4;
  static_assert(P % 4 == 0, "16-byte rows");
#pragma unroll
  for (int u = 0; u < (NV + NT - 1) / NT; ++u) {
    const int e = tid + u * NT;
    if (e < NV) {
      const int t = e / (IB * IB / 4), r = (e / (IB / 4)) % IB, c = (e % (IB / 4)) * 4;
      const uint32_t d = (uint32_t)__cvta_generic_to_shared(&dst[t * IB + r][c]);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(&dinv[dinv_off(t, which) + r * IB + c])
                   : "memory");
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <int NT, int ROWS, int COLS, class S, class Pad>
__device__ __forceinline__ void load_block(const float* __restrict__ g, int64_t ld, int rows, int cols, S s, Pad pad,
                                           int tid) {
  Staged<NT, ROWS, COLS> b;
  b.fetch(g, ld, rows, cols, pad, tid);
  b.put(s, tid);
}
template <int NT, int ROWS, int COLS, class S>
__device__ __forceinline__ void store_block(float* __restrict__ g, int64_t ld, int rows, int cols, S s, int tid) {
  constexpr int R4 = ROWS / 4, NV = R4 * COLS, PER = (NV + NT - 1) / NT;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int q = tid + u * NT;
    int r, c;
    piece<ROWS, COLS>(q, r, c);
    if (q >= NV || c >= cols) continue;
    if (r + 4 <= rows) {
      *reinterpret_cast<float4*>(g + (int64_t)c * ld + r) = make_float4(s(r, c), s(r + 1, c), s(r + 2, c), s(r + 3, c));
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (r + i < rows) g[(int64_t)c * ld + r + i] = s(r + i, c);
    }
  }
}

// ---------------------------------------------------------------------------
// K1: the PW x PW diagonal block at (k, k), factored in place (unit L below,
// U on and above the diagonal); the inverses of its IB x IB diagonal blocks
// of L and U go to dinv. Rows and columns past n are padded with the identity.
// 256 threads and 85 KB of shared memory, so that the CTA fits on an SM
// beside two CTAs of the tensor-core update of the second stream.
//
// Per inner block kb (columns k0 .. k0 + 31):
//   (a) warp 0 eliminates the IB x IB diagonal block (eliminate);
//   (b) warps 2..7 form the block's L rows below (one thread per row,
//       substitution with U_kk) and U columns right (one thread per column,
//       substitution with L_kk) while warps 0 and 1 invert L_kk and U_kk for
//       the other panel kernels (invert);
//   (c) all warps update the rest of the block; the next diagonal block's
//       tiles come first, so that warp 0 eliminates it while warps 1..7
//       update the rest.
constexpr size_t pdiag_smem(bool linv = false) {
  return (size_t)PW * SP * sizeof(float)        // As
         + (size_t)IB * SP * sizeof(float)      // LT: the inner block's L columns, transposed
         + (size_t)2 * IB * sizeof(float)       // pivot row, two buffers
         + (linv ? (size_t)PW * (IB + 4) * sizeof(float) : 0);   // Dl: the four inv(L_kk) (full inv(L) only)
}

// Warp 0: the IB x IB block at (k0, k0) of As factored in place. Lane i
// holds row i; the step loop is unrolled, so every register index is static
// and step j touches only columns j.. (the triangle of the work); the pivot
// row goes to the other lanes through a shared buffer (two, alternating, one
// __syncwarp a step). Each lane keeps its multipliers in place, so its
// registers end as its row of L and U.
__device__ __forceinline__ void eliminate(float (*As)[SP], float* pbuf, int k0, int lane, float& lmax, int* status) {
  float Rw[IB];
  const float4* rp = reinterpret_cast<const float4*>(&As[k0 + lane][k0]);
#pragma unroll
  for (int q = 0; q < IB / 4; ++q) {
    const float4 v = rp[q];
    Rw[4 * q] = v.x; Rw[4 * q + 1] = v.y; Rw[4 * q + 2] = v.z; Rw[4 * q + 3] = v.w;
  }
  bool bad = false;
#pragma unroll
  for (int j = 0; j < IB; ++j) {
    float4* pb = reinterpret_cast<float4*>(pbuf + (j & 1) * IB);
    if (lane == j)
#pragma unroll
      for (int q = j / 4; q < IB / 4; ++q) pb[q] = make_float4(Rw[4 * q], Rw[4 * q + 1], Rw[4 * q + 2], Rw[4 * q + 3]);
    __syncwarp();
    float pv[IB];
#pragma unroll
    for (int q = j / 4; q < IB / 4; ++q) {
      const float4 v = pb[q];
      pv[4 * q] = v.x; pv[4 * q + 1] = v.y; pv[4 * q + 2] = v.z; pv[4 * q + 3] = v.w;
    }
    bad |= !(fabsf(pv[j]) > 0.f && fabsf(pv[j]) <= FLT_MAX);
    const float rpiv = rcp_fast(pv[j]);
    if (lane > j) {
      const float l = Rw[j] * rpiv;
      Rw[j] = l;
      lmax = fmaxf(lmax, fabsf(l));
#pragma unroll
      for (int c = j + 1; c < IB; ++c) Rw[c] = fmaf(-l, pv[c], Rw[c]);
    }
  }
  float4* wp = reinterpret_cast<float4*>(&As[k0 + lane][k0]);
#pragma unroll
  for (int q = 0; q < IB / 4; ++q) wp[q] = make_float4(Rw[4 * q], Rw[4 * q + 1], Rw[4 * q + 2], Rw[4 * q + 3]);
  if (bad && lane == 0) atomicOr(status, (int)DEV_ZERO_PIVOT);
}

// Warp 0: inv(U_kk) -> dinv[.., 1]; warp 1: inv(L_kk) -> dinv[.., 0]; lane c
// forms column c by substitution in registers (constant loop bounds, so the
// loops unroll and the column stays in registers), four partial sums.
__device__ __forceinline__ void invert(const float (*As)[SP], float* __restrict__ dinv, int kb, int warp, int lane,
                                       float (*Dl)[IB + 4]) {
  const int k0 = kb * IB;
  if (warp == 0) {
    float x[IB];
#pragma unroll
    for (int i = IB - 1; i >= 0; --i) {
      float s[4] = {(lane == i) ? 1.f : 0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int g = 0; g < IB / 4; ++g) {
        if (4 * g + 3 <= i) continue;
        const float4 a = *reinterpret_cast<const float4*>(&As[k0 + i][k0 + 4 * g]);
        const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4 * g + e > i) s[e] = fmaf(-av[e], x[4 * g + e], s[e]);
      }
      x[i] = ((s[0] + s[1]) + (s[2] + s[3])) * rcp_fast(As[k0 + i][k0 + i]);
    }
#pragma unroll
    for (int i = 0; i < IB; ++i) dinv[dinv_off(kb, 1) + i * IB + lane] = x[i];
  } else if (warp == 1) {
    float y[IB];
#pragma unroll
    for (int i = 0; i < IB; ++i) {
      float s[4] = {(lane == i) ? 1.f : 0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int g = 0; g < IB / 4; ++g) {
        if (4 * g >= i) continue;
        const float4 a = *reinterpret_cast<const float4*>(&As[k0 + i][k0 + 4 * g]);
        const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4 * g + e < i) s[e] = fmaf(-av[e], y[4 * g + e], s[e]);
      }
      y[i] = (s[0] + s[1]) + (s[2] + s[3]);
    }
#pragma unroll
    for (int i = 0; i < IB; ++i) dinv[dinv_off(kb, 0) + i * IB + lane] = y[i];
    if (Dl != nullptr)
#pragma unroll
      for (int i = 0; i < IB; ++i) Dl[kb * IB + i][lane] = y[i];
  }
}

// (b) task `task` of 2R: task < R is row i = k1 + task of L(., kb) =
// A(i, kb) inv(U_kk), by right-looking substitution (row s of U_kk is
// contiguous); else column j = k1 + task - R of U(kb, .) = inv(L_kk) A(kb, j),
// by left-looking substitution (row t of L_kk is contiguous). Each thread
// owns its row or column, so results go straight back to As (and L's
// transpose to LT).
__device__ __forceinline__ void substitute(float (*As)[SP], float (*LT)[SP], int k0, int R, int task, float& lmax) {
  const int k1 = k0 + IB;
  float x[IB];
  if (task < R) {
    const int i = k1 + task;
#pragma unroll
    for (int q = 0; q < IB / 4; ++q) {
      const float4 v = *reinterpret_cast<const float4*>(&As[i][k0 + 4 * q]);
      x[4 * q] = v.x; x[4 * q + 1] = v.y; x[4 * q + 2] = v.z; x[4 * q + 3] = v.w;
    }
#pragma unroll
    for (int s = 0; s < IB; ++s) {
      x[s] *= rcp_fast(As[k0 + s][k0 + s]);
#pragma unroll
      for (int g = 0; g < IB / 4; ++g) {
        if (4 * g + 3 <= s) continue;
        const float4 u = *reinterpret_cast<const float4*>(&As[k0 + s][k0 + 4 * g]);
        const float uv[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4 * g + e > s) x[4 * g + e] = fmaf(-x[s], uv[e], x[4 * g + e]);
      }
    }
#pragma unroll
    for (int q = 0; q < IB / 4; ++q)
      *reinterpret_cast<float4*>(&As[i][k0 + 4 * q]) = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
#pragma unroll
    for (int t = 0; t < IB; ++t) {
      LT[t][i] = x[t];
      lmax = fmaxf(lmax, fabsf(x[t]));
    }
  } else {
    const int j = k1 + task - R;
#pragma unroll
    for (int t = 0; t < IB; ++t) {
      float s[4] = {As[k0 + t][j], 0.f, 0.f, 0.f};
#pragma unroll
      for (int g = 0; g < IB / 4; ++g) {
        if (4 * g >= t) continue;
        const float4 l = *reinterpret_cast<const float4*>(&As[k0 + t][k0 + 4 * g]);
        const float lv[4] = {l.x, l.y, l.z, l.w};
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4 * g + e < t) s[e] = fmaf(-lv[e], x[4 * g + e], s[e]);
      }
      x[t] = (s[0] + s[1]) + (s[2] + s[3]);
    }
#pragma unroll
    for (int t = 0; t < IB; ++t) As[k0 + t][j] = x[t];
  }
}

// (c) for the 4 x 4 tiles [first, last) of the update of the block after the
// inner block k0 (R x R from row and column k1 = k0 + IB), in an order where
// the next diagonal block's 64 tiles come first:
// As(i, j) -= sum_t LT(t, i) As(k0 + t, j).
__device__ __forceinline__ void update_tiles(float (*As)[SP], const float (*LT)[SP], int k0, int R, int first,
                                             int last, int stride) {
  const int k1 = k0 + IB, RQ = R / 4;
  for (int tile = first; tile < last; tile += stride) {
    int iq, jq;
    if (tile < 64) {   // the next diagonal block
      iq = tile >> 3; jq = tile & 7;
    } else {           // the rest, row quad by row quad
      const int t = tile - 64;
      const int rest_cols = RQ - 8;
      if (t < 8 * rest_cols) { iq = t / rest_cols; jq = 8 + t % rest_cols; }
      else { const int u = t - 8 * rest_cols; iq = 8 + u / RQ; jq = u % RQ; }
    }
    const int i0 = k1 + 4 * iq, j0 = k1 + 4 * jq;
    float acc[4][4] = {};
#pragma unroll 8
    for (int t = 0; t < IB; ++t) {
      const float4 l = *reinterpret_cast<const float4*>(&LT[t][i0]);
      const float4 u = *reinterpret_cast<const float4*>(&As[k0 + t][j0]);
      const float lv[4] = {l.x, l.y, l.z, l.w}, uv[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(lv[i], uv[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float4* p = reinterpret_cast<float4*>(&As[i0 + i][j0]);
      float4 v = *p;
      v.x -= acc[i][0]; v.y -= acc[i][1]; v.z -= acc[i][2]; v.w -= acc[i][3];
      *p = v;
    }
  }
}

// The full inv(L) of the factored block in As (with linvt, in place of a
// separate k_pinv launch), by block rows: X_ii = D_i = inv(L_ii) (kept in Dl
// by invert), X_ij = -D_i sum_{m=j}^{i-1} L_im X_mj for j < i. As is free
// once the factors are stored: row block i of it still holds L when X_i. is
// formed (the sums T_ij go to LT), the rows above already hold X. Written as
// k_pinv writes it: linvt[c * PW + q] = inv(L)(q, c) for q in or below the
// block row of c, 0 above.
__device__ __forceinline__ void full_linv(float (*As)[SP], float (*LT)[SP], const float (*Dl)[IB + 4],
                                          float* __restrict__ linvt, int tid) {
  __syncthreads();   // every thread has read As for the store
  for (int e = tid; e < NIB * IB * IB; e += kDiagThreads) {   // X_ii = D_i
    const int b = e / (IB * IB), r = (e / IB) % IB, c = e % IB;
    As[b * IB + r][b * IB + c] = Dl[b * IB + r][c];
  }
  __syncthreads();
  const int r = tid >> 3, c4 = (tid & 7) * 4;   // a 1 x 4 piece of a 32 x 32 block
#pragma unroll 1
  for (int i = 1; i < NIB; ++i) {
#pragma unroll 1
    for (int j = 0; j < i; ++j) {   // T_ij = sum_m L(i IB + r, m) X(m, j IB + c4 ..)
      float t[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
      for (int m = j * IB; m < i * IB; ++m) {
        const float a = As[i * IB + r][m];
        const float4 x = *reinterpret_cast<const float4*>(&As[m][j * IB + c4]);
        t[0] = fmaf(a, x.x, t[0]); t[1] = fmaf(a, x.y, t[1]); t[2] = fmaf(a, x.z, t[2]); t[3] = fmaf(a, x.w, t[3]);
      }
      *reinterpret_cast<float4*>(&LT[r][j * IB + c4]) = make_float4(t[0], t[1], t[2], t[3]);
    }
    __syncthreads();
#pragma unroll 1
    for (int j = 0; j < i; ++j) {   // X_ij = -D_i T_ij
      float y[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 8
      for (int q = 0; q < IB; ++q) {
        const float d = Dl[i * IB + r][q];
        const float4 x = *reinterpret_cast<const float4*>(&LT[q][j * IB + c4]);
        y[0] = fmaf(d, x.x, y[0]); y[1] = fmaf(d, x.y, y[1]); y[2] = fmaf(d, x.z, y[2]); y[3] = fmaf(d, x.w, y[3]);
      }
      *reinterpret_cast<float4*>(&As[i * IB + r][j * IB + c4]) = make_float4(-y[0], -y[1], -y[2], -y[3]);
    }
    __syncthreads();
  }
  for (int e = tid; e < PW * PW / 4; e += kDiagThreads) {   // lanes over q: coalesced stores
    const int q = e % PW, c0 = (e / PW) * 4;
    const bool below = q / IB >= c0 / IB;   // the four columns share a block column
    const float4 v = below ? *reinterpret_cast<const float4*>(&As[q][c0]) : make_float4(0.f, 0.f, 0.f, 0.f);
    linvt[(size_t)(c0 + 0) * PW + q] = v.x;
    linvt[(size_t)(c0 + 1) * PW + q] = v.y;
    linvt[(size_t)(c0 + 2) * PW + q] = v.z;
    linvt[(size_t)(c0 + 3) * PW + q] = v.w;
  }
}

__global__ void __launch_bounds__(kDiagThreads, 1)
k_pdiag(float* __restrict__ A, int64_t lda, int64_t n, int64_t k, float* __restrict__ dinv,
        float* __restrict__ cert, int* __restrict__ status, float* __restrict__ linvt) {
  griddep_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  float (*As)[SP] = reinterpret_cast<float (*)[SP]>(smem);
  float (*LT)[SP] = reinterpret_cast<float (*)[SP]>(smem + (size_t)PW * SP * sizeof(float));
  float* pbuf = reinterpret_cast<float*>(LT + IB);
  float (*Dl)[IB + 4] = linvt != nullptr ? reinterpret_cast<float (*)[IB + 4]>(pbuf + 2 * IB) : nullptr;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nb = (int)imin64(PW, n - k);
  load_block<kDiagThreads, PW, PW>(
      A + k * lda + k, lda, nb, nb, [&](int r, int c, float v) { As[r][c] = v; },
      [](int r, int c) { return r == c ? 1.f : 0.f; }, tid);
  __syncthreads();
  float lmax = 0.f;
  if (warp == 0) eliminate(As, pbuf, 0, lane, lmax, status);
  __syncthreads();
#pragma unroll 1
  for (int kb = 0; kb < NIB; ++kb) {
    const int k0 = kb * IB, R = PW - k0 - IB;   // R rows (and columns) after the inner block
    if (warp < 2) invert(As, dinv, kb, warp, lane, Dl);
    else if (tid - 64 < 2 * R) substitute(As, LT, k0, R, tid - 64, lmax);
    if (R == 0) break;
    __syncthreads();
    const int tiles = (R / 4) * (R / 4);
    update_tiles(As, LT, k0, R, tid, 64, kDiagThreads);
    __syncthreads();
    if (warp == 0) eliminate(As, pbuf, k0 + IB, lane, lmax, status);
    else update_tiles(As, LT, k0, R, 64 + (tid - 32), tiles, kDiagThreads - 32);
    __syncthreads();
  }
  __syncthreads();
  griddep_launch();
  // write the factors back (16-byte stores down the columns)
  store_block<kDiagThreads, PW, PW>(A + k * lda + k, lda, nb, nb, [&](int r, int c) { return As[r][c]; }, tid);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(FULL, lmax, o));
  if (lane == 0) atomic_max_pos(cert, lmax);
  if (linvt != nullptr && nb == PW) full_linv(As, LT, Dl, linvt, tid);
}

// The split of four consecutive K values of a K-major operand at o (element
// offset), by split mode SM: kSplitTf32 TF32 hi / lo (unsplit FP32 when lo is
// null), kSplitBf16 BF16 (the BF16 form; no lo), kSplitBf16x2 BF16 hi / lo
// (lo = the BF16 rounding of the remainder).
constexpr int kSplitTf32 = 0, kSplitBf16 = 1, kSplitBf16x2 = 2;
template <int SM>
__device__ __forceinline__ void put_split(float* __restrict__ hi, float* __restrict__ lo, int64_t o, const float v[4]) {
  if (SM == kSplitBf16) {
    __nv_bfloat162* d = reinterpret_cast<__nv_bfloat162*>(reinterpret_cast<__nv_bfloat16*>(hi) + o);
    d[0] = __floats2bfloat162_rn(v[0], v[1]);
    d[1] = __floats2bfloat162_rn(v[2], v[3]);
  } else if (SM == kSplitBf16x2) {
    __nv_bfloat162* dh = reinterpret_cast<__nv_bfloat162*>(reinterpret_cast<__nv_bfloat16*>(hi) + o);
    __nv_bfloat162* dl = reinterpret_cast<__nv_bfloat162*>(reinterpret_cast<__nv_bfloat16*>(lo) + o);
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * p], v[2 * p + 1]);
      dh[p] = h;
      dl[p] = __floats2bfloat162_rn(v[2 * p] - __low2float(h), v[2 * p + 1] - __high2float(h));
    }
  } else if (lo) {
    float h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) { h[i] = tf32_rna(v[i]); l[i] = v[i] - h[i]; }
    *reinterpret_cast<float4*>(hi + o) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(lo + o) = make_float4(l[0], l[1], l[2], l[3]);
  } else {
    *reinterpret_cast<float4*>(hi + o) = make_float4(v[0], v[1], v[2], v[3]);
  }
}

// ---------------------------------------------------------------------------
// K6: L21 = A21 U^-1 for the rows [rbeg + 32 b, +32) (rows [r0, n) below the
// panel at k, the split operand indexed from r0) by
// block substitution over the four inner column blocks t:
//   Y_t = A21_t - sum_{s < t} L_s U(s, t),   L_t = Y_t inv(U_tt).
// The row block, the panel's U above the diagonal blocks and the four
// inverses are staged once (one round of loads), then the four steps run from
// shared memory. Writes L21 in place and its split Ah = rna_tf32(L21),
// Al = L21 - Ah (K-major: row (r - r0) of ldk = PW floats); max|L21| into
// cert. Thread tile: 2 rows x 4 columns of the 32 x 32 block.
constexpr int L21_ROWS = 32, L21_THREADS = 128;
constexpr int XP = PW + 4;   // row pitch of the row block
constexpr int UP = IB + 4;   // row pitch of the 32-wide blocks
constexpr int UBP = PW - IB + 4;   // row pitch of U(0..95, 32..127)
constexpr size_t l21_smem() {
  return (size_t)L21_ROWS * XP * sizeof(float) + (size_t)(PW - IB) * UBP * sizeof(float) +
         (size_t)NIB * IB * UP * sizeof(float);
}

template <int SM>
__global__ void __launch_bounds__(L21_THREADS)
k_l21(float* __restrict__ A, int64_t lda, int64_t n, int64_t k, int64_t r0, int64_t rbeg, const float* __restrict__ dinv,
      float* __restrict__ Ah, float* __restrict__ Al, float* __restrict__ cert) {
  griddep_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  float (*X)[XP] = reinterpret_cast<float (*)[XP]>(smem);
  // Ub[s][c - IB] = U(s, c) for s < 96, c >= 32 (entries below the diagonal blocks are not read)
  float (*Ub)[UBP] = reinterpret_cast<float (*)[UBP]>(smem + (size_t)L21_ROWS * XP * sizeof(float));
  float (*Ut)[UP] = reinterpret_cast<float (*)[UP]>(reinterpret_cast<unsigned char*>(Ub) +
                                                     (size_t)(PW - IB) * UBP * sizeof(float));   // inv(U_tt), 4 x 32 rows
  const int tid = threadIdx.x;
  const int64_t row0 = rbeg + (int64_t)blockIdx.x * L21_ROWS;   // rows [rbeg, n); the split is indexed from r0
  const int rows = (int)imin64(L21_ROWS, n - row0);
  {   // all loads in flight before the first store
    const auto zero = [](int, int) { return 0.f; };
    Staged<L21_THREADS, L21_ROWS, PW> xs;
    Staged<L21_THREADS, PW - IB, PW - IB> us;
    copy_inv_async<L21_THREADS>(Ut, dinv, 1, tid);
    xs.fetch(A + k * lda + row0, lda, rows, PW, zero, tid);
    us.fetch(A + (k + IB) * lda + k, lda, PW - IB, PW - IB, zero, tid);
    xs.put([&](int r, int c, float v) { X[r][c] = v; }, tid);
    us.put([&](int r, int c, float v) { Ub[r][c] = v; }, tid);
    cp_async_wait_all();
  }
  __syncthreads();
  const int rg = tid & 15, cg = tid >> 4;   // 16 row pairs x 8 column quads = 32 x 32
#pragma unroll 1
  for (int t = 0; t < NIB; ++t) {
    const int c0 = t * IB;
    float y[2][4] = {};
#pragma unroll 4
    for (int s = 0; s < c0; ++s) {   // sum_s L_s U(s, t): X's columns < c0 hold L
      const float4 q = *reinterpret_cast<const float4*>(&Ub[s][c0 - IB + 4 * cg]);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const float p = X[2 * rg + i][s];
#pragma unroll
        for (int j = 0; j < 4; ++j) y[i][j] = fmaf(p, qv[j], y[i][j]);
      }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)   // each thread owns its 2 x 4 entries of block t: no other thread reads them yet
#pragma unroll
      for (int j = 0; j < 4; ++j) X[2 * rg + i][c0 + 4 * cg + j] -= y[i][j];
    __syncthreads();
    float l[2][4] = {};
#pragma unroll 4
    for (int s = 0; s < IB; ++s) {   // L_t = Y_t inv(U_tt)
      const float4 q = *reinterpret_cast<const float4*>(&Ut[t * IB + s][4 * cg]);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const float p = X[2 * rg + i][c0 + s];
#pragma unroll
        for (int j = 0; j < 4; ++j) l[i][j] = fmaf(p, qv[j], l[i][j]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) X[2 * rg + i][c0 + 4 * cg + j] = l[i][j];
    __syncthreads();
  }
  griddep_launch();
  store_block<L21_THREADS, L21_ROWS, PW>(A + k * lda + row0, lda, rows, PW, [&](int r, int c) { return X[r][c]; },
                                        tid);
  float lmax = 0.f;
  constexpr int C4 = PW / 4;
  for (int e = tid; e < rows * C4; e += L21_THREADS) {   // K-major split: 16-byte stores along each row
    const int r = e / C4, c = (e % C4) * 4;
    const float4 v = *reinterpret_cast<const float4*>(&X[r][c]);
    const float vv[4] = {v.x, v.y, v.z, v.w};
    put_split<SM>(Ah, Al, (row0 - r0 + r) * (int64_t)PW + c, vv);
    lmax = fmaxf(lmax, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(FULL, lmax, o));
  if ((tid & 31) == 0) atomic_max_pos(cert, lmax);
}

// ---------------------------------------------------------------------------
// K2: U12 = L^-1 A12 for the panel's rows [k, k + PW) and the columns
// [c0 + CW b, +CW) of [c0, c1), by block substitution over the four inner row
// blocks t:  Z_t = A12_t - sum_{s < t} L(t, s) U12_s,  U12_t = inv(L_tt) Z_t.
// The column block, the panel's L below the diagonal blocks and the four
// inverses are staged once. Writes U12 in place and its split Bh, Bl (column
// j - c0 holds its PW values contiguously). Thread tile: RT rows of block t
// x 4 columns.
template <int CW, int RT>
struct U12Cfg {
  static constexpr int THREADS = (IB / RT) * (CW / 4);
  static constexpr int ZP = CW + 4;   // row pitch of the column block
  static constexpr int LP = PW - IB + 4;
  static constexpr size_t smem() {
    return (size_t)PW * ZP * sizeof(float) + (size_t)(PW - IB) * LP * sizeof(float) +
           (size_t)NIB * IB * UP * sizeof(float);
  }
};

template <int CW, int RT, bool BF16>
__global__ void __launch_bounds__(U12Cfg<CW, RT>::THREADS)
k_u12(float* __restrict__ A, int64_t lda, int64_t k, int64_t c0, int64_t c1, const float* __restrict__ dinv,
      float* __restrict__ Bh, float* __restrict__ Bl) {
  griddep_wait();
  typedef U12Cfg<CW, RT> Cfg;
  constexpr int T = Cfg::THREADS, ZP = Cfg::ZP, LP = Cfg::LP;
  extern __shared__ __align__(16) unsigned char smem[];
  float (*Z)[ZP] = reinterpret_cast<float (*)[ZP]>(smem);                                    // PW x CW
  // Lb[r - IB][s] = L(r, s) for r >= 32, s < 96 (entries right of the diagonal blocks are not read)
  float (*Lb)[LP] = reinterpret_cast<float (*)[LP]>(smem + (size_t)PW * ZP * sizeof(float));
  float (*Lt)[UP] = reinterpret_cast<float (*)[UP]>(reinterpret_cast<unsigned char*>(Lb) +
                                                     (size_t)(PW - IB) * LP * sizeof(float));   // inv(L_tt), 4 x 32 rows
  const int tid = threadIdx.x;
  const int64_t col0 = c0 + (int64_t)blockIdx.x * CW;
  const int cols = (int)imin64(CW, c1 - col0);
  {   // all loads in flight before the first store
    const auto zero = [](int, int) { return 0.f; };
    Staged<T, PW, CW> zs;
    Staged<T, PW - IB, PW - IB> ls;
    copy_inv_async<T>(Lt, dinv, 0, tid);
    zs.fetch(A + col0 * lda + k, lda, PW, cols, zero, tid);
    ls.fetch(A + k * lda + k + IB, lda, PW - IB, PW - IB, zero, tid);
    zs.put([&](int r, int c, float v) { Z[r][c] = v; }, tid);
    ls.put([&](int r, int s, float v) { Lb[r][s] = v; }, tid);
    cp_async_wait_all();
  }
  __syncthreads();
  constexpr int CQ = CW / 4;
  const int cq = tid % CQ, rq = tid / CQ;   // rq < IB / RT
#pragma unroll 1
  for (int t = 0; t < NIB; ++t) {
    const int t0 = t * IB;
    float z[RT][4] = {};
#pragma unroll 4
    for (int s = 0; s < t0; ++s) {
      const float4 q = *reinterpret_cast<const float4*>(&Z[s][4 * cq]);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int i = 0; i < RT; ++i) {
        const float p = Lb[t0 - IB + RT * rq + i][s];
#pragma unroll
        for (int j = 0; j < 4; ++j) z[i][j] = fmaf(p, qv[j], z[i][j]);
      }
    }
#pragma unroll
    for (int i = 0; i < RT; ++i)   // own entries of block t: nothing else reads them yet
#pragma unroll
      for (int j = 0; j < 4; ++j) Z[t0 + RT * rq + i][4 * cq + j] -= z[i][j];
    __syncthreads();
    float u[RT][4] = {};
#pragma unroll 4
    for (int s = 0; s < IB; ++s) {
      const float4 q = *reinterpret_cast<const float4*>(&Z[t0 + s][4 * cq]);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int i = 0; i < RT; ++i) {
        const float p = Lt[t * IB + RT * rq + i][s];
#pragma unroll
        for (int j = 0; j < 4; ++j) u[i][j] = fmaf(p, qv[j], u[i][j]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) Z[t0 + RT * rq + i][4 * cq + j] = u[i][j];
    __syncthreads();
  }
  griddep_launch();
  store_block<T, PW, CW>(A + col0 * lda + k, lda, PW, cols, [&](int r, int c) { return Z[r][c]; }, tid);
  constexpr int R4 = PW / 4;
  for (int e = tid; e < cols * R4; e += T) {   // the split, K-major: column j - c0 holds its PW values
    const int c = e / R4, r = (e % R4) * 4;
    const float v[4] = {Z[r][c], Z[r + 1][c], Z[r + 2][c], Z[r + 3][c]};
    const int64_t o = (col0 - c0 + c) * (int64_t)PW + r;
    if (BF16) {
      __nv_bfloat162* d = reinterpret_cast<__nv_bfloat162*>(reinterpret_cast<__nv_bfloat16*>(Bh) + o);
      d[0] = __floats2bfloat162_rn(v[0], v[1]);
      d[1] = __floats2bfloat162_rn(v[2], v[3]);
    } else if (Bl) {
      float h[4], lo[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) { h[i] = tf32_rna(v[i]); lo[i] = v[i] - h[i]; }
      *reinterpret_cast<float4*>(&Bh[o]) = make_float4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<float4*>(&Bl[o]) = make_float4(lo[0], lo[1], lo[2], lo[3]);
    } else {   // unsplit: the update splits in shared memory
      *reinterpret_cast<float4*>(&Bh[o]) = make_float4(v[0], v[1], v[2], v[3]);
    }
  }
}

// ---------------------------------------------------------------------------
// The GEMM form of K6 / K2 (FP_TUNE_PANEL_GEMM 1, 2). K1b k_pinv forms the
// full inverses of the diagonal block's factors once a panel; L21 = A21 inv(U)
// and U12 = inv(L) A12 are then one triangular product each: one K loop a
// thread, no dependent steps and no barriers between them.
//
// Per panel slot of the scratch, after dinv: inv(L)^T (PW x PW; row s holds
// column s of inv(L)) and inv(U) (PW x PW, row-major), both written whole
// (zeros outside the triangle).
constexpr int kInvFloats = PW * PW;
constexpr int kSlotFloats = kDinvFloats + 2 * kInvFloats;
constexpr int kLinvtOff = kDinvFloats, kUinvOff = kDinvFloats + kInvFloats;
constexpr int GP = PW + 4;   // pitch of 128-float rows in shared memory (16-byte rows, 4 banks apart)
constexpr int DP = IB + 4;   // pitch of 32-float rows

// One 16-byte asynchronous copy global -> shared; bytes < 16 copies that many
// and zero-fills the rest (bytes = 0: no global read).
__device__ __forceinline__ void cp16(void* sdst, const float* gsrc, int bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc), "r"(bytes) : "memory");
}
// PW x PW floats, row-major at g with pitch PW, into dst (pitch GP)
template <int NT>
__device__ __forceinline__ void copy_square_async(float (*dst)[GP], const float* __restrict__ g, int tid) {
#pragma unroll
  for (int u = 0; u < PW * PW / 4 / NT; ++u) {
    const int e = tid + u * NT, r = e / (PW / 4), c = (e % (PW / 4)) * 4;
    cp16(&dst[r][c], g + (size_t)r * PW + c, 16);
  }
}

// K6 with asynchronous staging (FP_TUNE_L21_ASYNC): the same substitution as
// k_l21, but the row block and U are kept column-major in shared memory, as
// they lie in global memory, so that every staging copy is a cp.async (all
// of a CTA's loads in flight at once, no registers): XT[c][r] = A21(r, c),
// UbT[c][s] = U(s, IB + c). Thread tile: rows 2 rg, 2 rg + 1 x 4 columns.
constexpr int XTP = L21_ROWS + 4;   // pitch of XT (32 rows)
constexpr int UTP = PW - IB + 4;    // pitch of UbT (96 rows)
constexpr size_t l21a_smem() {
  return ((size_t)PW * XTP + (size_t)(PW - IB) * UTP + (size_t)NIB * IB * UP) * sizeof(float);
}
template <int SM>
__global__ void __launch_bounds__(L21_THREADS)
k_l21a(float* __restrict__ A, int64_t lda, int64_t n, int64_t k, int64_t r0, int64_t rbeg,
       const float* __restrict__ dinv, float* __restrict__ Ah, float* __restrict__ Al, float* __restrict__ cert) {
  griddep_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  float (*XT)[XTP] = reinterpret_cast<float (*)[XTP]>(smem);
  float (*UbT)[UTP] = reinterpret_cast<float (*)[UTP]>(smem + (size_t)PW * XTP * sizeof(float));
  float (*Ut)[UP] = reinterpret_cast<float (*)[UP]>(reinterpret_cast<unsigned char*>(UbT) +
                                                     (size_t)(PW - IB) * UTP * sizeof(float));
  const int tid = threadIdx.x;
  const int64_t row0 = rbeg + (int64_t)blockIdx.x * L21_ROWS;
  const int rows = (int)imin64(L21_ROWS, n - row0);
#pragma unroll
  for (int u = 0; u < PW * (L21_ROWS / 4) / L21_THREADS; ++u) {   // XT: 128 columns x 8 chunks of 4 rows
    const int e = tid + u * L21_THREADS, c = e / (L21_ROWS / 4), q = (e % (L21_ROWS / 4)) * 4;
    const int bytes = 4 * max(0, min(4, rows - q));
    const float* col = A + (k + c) * lda;
    cp16(&XT[c][q], bytes ? col + row0 + q : col, bytes);
  }
#pragma unroll
  for (int u = 0; u < (PW - IB) * ((PW - IB) / 4) / L21_THREADS; ++u) {   // UbT: 96 columns x 24 chunks
    const int e = tid + u * L21_THREADS, c = e / ((PW - IB) / 4), q = (e % ((PW - IB) / 4)) * 4;
    cp16(&UbT[c][q], A + (k + IB + c) * lda + k + q, 16);
  }
  copy_inv_async<L21_THREADS>(Ut, dinv, 1, tid);
  cp_async_wait_all();
  __syncthreads();
  const int rg = tid & 15, cg = tid >> 4;   // 16 row pairs x 8 column quads = 32 x 32
#pragma unroll 1
  for (int t = 0; t < NIB; ++t) {
    const int c0 = t * IB;
    float y[2][4] = {};
#pragma unroll 2
    for (int s = 0; s < c0; s += 4) {   // sum_s L_s U(s, t): XT's columns < c0 hold L
      float4 uq[4];   // U(s .. s+3, c0 + 4 cg + j)
#pragma unroll
      for (int j = 0; j < 4; ++j) uq[j] = *reinterpret_cast<const float4*>(&UbT[c0 - IB + 4 * cg + j][s]);
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        const float2 x = *reinterpret_cast<const float2*>(&XT[s + d][2 * rg]);
        const float uv[4] = {(&uq[0].x)[d], (&uq[1].x)[d], (&uq[2].x)[d], (&uq[3].x)[d]};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          y[0][j] = fmaf(x.x, uv[j], y[0][j]);
          y[1][j] = fmaf(x.y, uv[j], y[1][j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {   // own entries of block t: nothing else reads them yet
      float2* p = reinterpret_cast<float2*>(&XT[c0 + 4 * cg + j][2 * rg]);
      float2 v = *p;
      v.x -= y[0][j]; v.y -= y[1][j];
      *p = v;
    }
    __syncthreads();
    float l[2][4] = {};
#pragma unroll 4
    for (int s = 0; s < IB; ++s) {   // L_t = Y_t inv(U_tt)
      const float4 q = *reinterpret_cast<const float4*>(&Ut[t * IB + s][4 * cg]);
      const float2 x = *reinterpret_cast<const float2*>(&XT[c0 + s][2 * rg]);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        l[0][j] = fmaf(x.x, qv[j], l[0][j]);
        l[1][j] = fmaf(x.y, qv[j], l[1][j]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j)
      *reinterpret_cast<float2*>(&XT[c0 + 4 * cg + j][2 * rg]) = make_float2(l[0][j], l[1][j]);
    __syncthreads();
  }
  griddep_launch();
  // L21 in place (column-major, as staged) and its split (K-major rows)
#pragma unroll
  for (int u = 0; u < PW * (L21_ROWS / 4) / L21_THREADS; ++u) {
    const int e = tid + u * L21_THREADS, c = e / (L21_ROWS / 4), q = (e % (L21_ROWS / 4)) * 4;
    float* const g = A + (k + c) * lda + row0 + q;
    const float4 v = *reinterpret_cast<const float4*>(&XT[c][q]);
    if (q + 4 <= rows) {
      *reinterpret_cast<float4*>(g) = v;
    } else {
      const float vv[4] = {v.x, v.y, v.z, v.w};
      for (int i = 0; i < 4; ++i)
        if (q + i < rows) g[i] = vv[i];
    }
  }
  float lmax = 0.f;
  constexpr int C4 = PW / 4;
  for (int e = tid; e < L21_ROWS * C4; e += L21_THREADS) {   // lanes over rows: conflict-free column reads
    const int r = e % L21_ROWS, c = (e / L21_ROWS) * 4;
    if (r >= rows) continue;
    const float v[4] = {XT[c][r], XT[c + 1][r], XT[c + 2][r], XT[c + 3][r]};
    put_split<SM>(Ah, Al, (row0 - r0 + r) * (int64_t)PW + c, v);
    lmax = fmaxf(lmax, fmaxf(fmaxf(fabsf(v[0]), fabsf(v[1])), fmaxf(fabsf(v[2]), fabsf(v[3]))));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(FULL, lmax, o));
  if ((tid & 31) == 0) atomic_max_pos(cert, lmax);
}

// K1b: 2 NIB CTAs. CTA b < NIB forms block column j = b of inv(L), CTA
// b >= NIB block column j = b - NIB of inv(U^T) = inv(U)^T; both are the
// inverse of a lower-triangular M from its diagonal-block inverses D_i:
//   X_jj = D_j,   X_ij = -D_i sum_{m=j}^{i-1} M_im X_mj   (i = j+1 .. NIB-1),
// with M = L, D_i = inv(L_ii), or M = U^T, D_i = inv(U_ii)^T. Block (i, j) of
// X goes to out[IB j + c][IB i + r] = X_ij(r, c): out is inv(L)^T for L and
// inv(U) for U. Launched only for full panels (rows below exist); a grid of
// NIB CTAs forms inv(L) alone. The factored block is staged whole:
// G[p][q] = column p, row q of it; the D_i come from the slot's dinv (k_pdiag).
constexpr int PI_THREADS = 256;
constexpr size_t pinv_smem() {
  return ((size_t)PW * GP + (size_t)NIB * IB * DP + (size_t)PW * DP + (size_t)IB * DP) * sizeof(float);
}
__global__ void __launch_bounds__(PI_THREADS)
k_pinv(const float* __restrict__ A, int64_t lda, int64_t k, float* __restrict__ slot) {
  griddep_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  float (*G)[GP] = reinterpret_cast<float (*)[GP]>(smem);
  float (*Ds)[DP] = reinterpret_cast<float (*)[DP]>(smem + (size_t)PW * GP * sizeof(float));
  float (*Xs)[DP] = Ds + NIB * IB;   // block column j of X, rows 0 .. PW - 1 (those below IB j used)
  float (*Ts)[DP] = Xs + PW;
  const int tid = threadIdx.x;
  const bool upper = blockIdx.x >= NIB;
  const int j = upper ? blockIdx.x - NIB : blockIdx.x;
#pragma unroll
  for (int u = 0; u < PW * PW / 4 / PI_THREADS; ++u) {
    const int e = tid + u * PI_THREADS, p = e / (PW / 4), q = (e % (PW / 4)) * 4;
    cp16(&G[p][q], A + (k + p) * lda + k + q, 16);
  }
  copy_inv_async<PI_THREADS>(Ds, slot, upper ? 1 : 0, tid);
  cp_async_wait_all();
  __syncthreads();
  // M(r, m) and D_i(r, m) of the triangle being inverted
  const auto Mx = [&](int r, int m) { return upper ? G[r][m] : G[m][r]; };
  const auto Dx = [&](int i, int r, int m) { return upper ? Ds[i * IB + m][r] : Ds[i * IB + r][m]; };
  const int r = tid >> 3, c = (tid & 7) * 4;   // this thread's 1 x 4 piece of a 32 x 32 block
#pragma unroll
  for (int e = 0; e < 4; ++e) Xs[IB * j + r][c + e] = Dx(j, r, c + e);
  __syncthreads();
#pragma unroll 1
  for (int i = j + 1; i < NIB; ++i) {
    float t[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
    for (int m = IB * j; m < IB * i; ++m) {
      const float a = Mx(IB * i + r, m);
      const float4 x = *reinterpret_cast<const float4*>(&Xs[m][c]);
      t[0] = fmaf(a, x.x, t[0]); t[1] = fmaf(a, x.y, t[1]); t[2] = fmaf(a, x.z, t[2]); t[3] = fmaf(a, x.w, t[3]);
    }
    *reinterpret_cast<float4*>(&Ts[r][c]) = make_float4(t[0], t[1], t[2], t[3]);
    __syncthreads();
    float y[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 8
    for (int m = 0; m < IB; ++m) {
      const float d = Dx(i, r, m);
      const float4 x = *reinterpret_cast<const float4*>(&Ts[m][c]);
      y[0] = fmaf(d, x.x, y[0]); y[1] = fmaf(d, x.y, y[1]); y[2] = fmaf(d, x.z, y[2]); y[3] = fmaf(d, x.w, y[3]);
    }
    *reinterpret_cast<float4*>(&Xs[IB * i + r][c]) = make_float4(-y[0], -y[1], -y[2], -y[3]);
    __syncthreads();
  }
  griddep_launch();
  // out[IB j + cc][q] = X(q, cc) for q >= IB j, 0 above
  float* const out = slot + (upper ? kUinvOff : kLinvtOff);
#pragma unroll
  for (int u = 0; u < IB * PW / 4 / PI_THREADS; ++u) {
    const int e = tid + u * PI_THREADS, cc = e / (PW / 4), q = (e % (PW / 4)) * 4;
    float v[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) v[h] = (q + h >= IB * j) ? Xs[q + h][cc] : 0.f;
    *reinterpret_cast<float4*>(out + (size_t)(IB * j + cc) * PW + q) = make_float4(v[0], v[1], v[2], v[3]);
  }
}

// K6g: L21 = A21 inv(U) for the rows [r0 + 32 b, +32) below the panel at k.
// 8 warps, warp w owns the columns [16 w, +16) (inv(U) is upper triangular:
// its K loop stops at 16 w + 16), a 4 x 4 piece a lane. Writes L21 in place
// and its split (K-major, as k_l21), max|L21| into cert.
constexpr int L21G_THREADS = 256;
constexpr size_t l21g_smem() { return ((size_t)PW * DP + (size_t)PW * GP) * sizeof(float); }
template <int SM>
__global__ void __launch_bounds__(L21G_THREADS)
k_l21g(float* __restrict__ A, int64_t lda, int64_t n, int64_t k, int64_t r0, const float* __restrict__ slot,
       float* __restrict__ Ah, float* __restrict__ Al, float* __restrict__ cert) {
  griddep_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  float (*XT)[DP] = reinterpret_cast<float (*)[DP]>(smem);   // XT[s][r] = A21(r, s)
  float (*Us)[GP] = reinterpret_cast<float (*)[GP]>(smem + (size_t)PW * DP * sizeof(float));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t row0 = r0 + (int64_t)blockIdx.x * L21_ROWS;
  const int rows = (int)imin64(L21_ROWS, n - row0);
#pragma unroll
  for (int u = 0; u < PW * L21_ROWS / 4 / L21G_THREADS; ++u) {
    const int e = tid + u * L21G_THREADS, s = e / (L21_ROWS / 4), q = (e % (L21_ROWS / 4)) * 4;
    const int bytes = 4 * max(0, min(4, rows - q));
    const float* col = A + (k + s) * lda;
    cp16(&XT[s][q], bytes ? col + row0 + q : col, bytes);
  }
  copy_square_async<L21G_THREADS>(Us, slot + kUinvOff, tid);
  cp_async_wait_all();
  __syncthreads();
  const int cq = lane & 3, rq = lane >> 2;
  const int cb = 16 * warp + 4 * cq, rb = 4 * rq;
  float acc[4][4] = {};
  const int send = 16 * warp + 16;
#pragma unroll 4
  for (int s = 0; s < send; ++s) {
    const float4 x = *reinterpret_cast<const float4*>(&XT[s][rb]);
    const float4 u = *reinterpret_cast<const float4*>(&Us[s][cb]);
    const float xv[4] = {x.x, x.y, x.z, x.w}, uv[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = fmaf(xv[a], uv[b], acc[a][b]);
  }
  griddep_launch();
  float lmax = 0.f;
#pragma unroll
  for (int b = 0; b < 4; ++b) {   // L21 in place: column k + cb + b, rows row0 + rb ..
    float* const g = A + (k + cb + b) * lda + row0 + rb;
    if (rb + 4 <= rows) {
      *reinterpret_cast<float4*>(g) = make_float4(acc[0][b], acc[1][b], acc[2][b], acc[3][b]);
    } else {
#pragma unroll
      for (int a = 0; a < 4; ++a)
        if (rb + a < rows) g[a] = acc[a][b];
    }
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {   // the split: row (row0 - r0 + rb + a), K values cb .. cb + 3
    if (rb + a < rows) {
      put_split<SM>(Ah, Al, (row0 - r0 + rb + a) * (int64_t)PW + cb, acc[a]);
#pragma unroll
      for (int b = 0; b < 4; ++b) lmax = fmaxf(lmax, fabsf(acc[a][b]));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(FULL, lmax, o));
  if (lane == 0) atomic_max_pos(cert, lmax);
}

// K2g: U12 = inv(L) A12 for the panel's rows [k, k + PW) and the columns
// [c0 + CW b, +CW) of [c0, c1). A 4 x 4 piece a lane; a warp's piece is
// WR = 512 / CW rows x CW columns, and its K loop stops at its last row
// (inv(L) is lower triangular). Writes U12 in place and its split (K-major:
// column j - c0 holds its PW values), as k_u12.
// DIAG (the split panel chain): then also the next diagonal tile's update,
// A(kd + r, j) -= sum_s L21(kd + r, k + s) U12(k + s, j) for r < PW and the
// CTA's columns j, in FP32 on the FMA pipe: U12 from the registers through
// shared memory, the 128 x 128 block of L21 (written before this launch)
// staged where inv(L) was.
template <int CW>
struct U12gCfg {
  static constexpr int THREADS = 8 * CW;
  static constexpr int WR = 512 / CW;
  static constexpr int ZP = CW + 4;
  // the A12 block row-major (Z[s][c], through registers) or column-major
  // (ZT[c][s], by cp.async: FP_TUNE_U12_ASYNC), whichever is larger
  static constexpr size_t smem() {
    return ((size_t)PW * GP + std::max((size_t)PW * ZP, (size_t)CW * GP)) * sizeof(float);
  }
};
template <int CW, int SM, bool DIAG = false>
__global__ void __launch_bounds__(U12gCfg<CW>::THREADS)
k_u12g(float* __restrict__ A, int64_t lda, int64_t k, int64_t c0, int64_t c1, const float* __restrict__ slot,
       float* __restrict__ Bh, float* __restrict__ Bl, int64_t kd, int zasync) {
  griddep_wait();
  typedef U12gCfg<CW> Cfg;
  constexpr int T = Cfg::THREADS, ZP = Cfg::ZP, CQ = CW / 4;
  extern __shared__ __align__(16) unsigned char smem[];
  float (*LT)[GP] = reinterpret_cast<float (*)[GP]>(smem);   // LT[s][i] = inv(L)(i, s)
  float (*Z)[ZP] = reinterpret_cast<float (*)[ZP]>(smem + (size_t)PW * GP * sizeof(float));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t col0 = c0 + (int64_t)blockIdx.x * CW;
  const int cols = (int)imin64(CW, c1 - col0);
  float (*ZT)[GP] = reinterpret_cast<float (*)[GP]>(Z);   // async staging: ZT[c][s] = A12(s, c)
  copy_square_async<T>(LT, slot + kLinvtOff, tid);
  if (zasync) {
#pragma unroll
    for (int u = 0; u < CW * (PW / 4) / T; ++u) {   // column c of the block: PW contiguous floats
      const int e = tid + u * T, c = e / (PW / 4), q = (e % (PW / 4)) * 4;
      const float* col = A + (col0 + c) * lda + k;
      cp16(&ZT[c][q], c < cols ? col + q : A + col0 * lda + k, c < cols ? 16 : 0);
    }
  } else {
    Staged<T, PW, CW> zs;
    zs.fetch(A + col0 * lda + k, lda, PW, cols, [](int, int) { return 0.f; }, tid);
    zs.put([&](int r, int c, float v) { Z[r][c] = v; }, tid);
  }
  cp_async_wait_all();
  __syncthreads();
  const int cq = lane % CQ, rq = lane / CQ;
  const int ib = Cfg::WR * warp + 4 * rq, cb = 4 * cq;
  float acc[4][4] = {};
  const int send = Cfg::WR * (warp + 1);
  if (zasync) {
#pragma unroll 2
    for (int s = 0; s < send; s += 4) {   // 4 K values a step: inv(L) rows and A12 columns as float4
      float4 zq[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) zq[b] = *reinterpret_cast<const float4*>(&ZT[cb + b][s]);
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        const float4 l = *reinterpret_cast<const float4*>(&LT[s + d][ib]);
        const float lv[4] = {l.x, l.y, l.z, l.w};
        const float zv[4] = {(&zq[0].x)[d], (&zq[1].x)[d], (&zq[2].x)[d], (&zq[3].x)[d]};
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = fmaf(lv[a], zv[b], acc[a][b]);
      }
    }
  } else {
#pragma unroll 4
    for (int s = 0; s < send; ++s) {
      const float4 l = *reinterpret_cast<const float4*>(&LT[s][ib]);
      const float4 z = *reinterpret_cast<const float4*>(&Z[s][cb]);
      const float lv[4] = {l.x, l.y, l.z, l.w}, zv[4] = {z.x, z.y, z.z, z.w};
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fmaf(lv[a], zv[b], acc[a][b]);
    }
  }
  griddep_launch();
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    if (cb + b >= cols) break;
    const float v[4] = {acc[0][b], acc[1][b], acc[2][b], acc[3][b]};
    *reinterpret_cast<float4*>(A + (col0 + cb + b) * lda + k + ib) = make_float4(v[0], v[1], v[2], v[3]);
    put_split<SM>(Bh, Bl, (col0 - c0 + cb + b) * (int64_t)PW + ib, v);
  }
  if constexpr (DIAG) {
    __syncthreads();   // every warp is done with inv(L) and the A12 block
#pragma unroll
    for (int u = 0; u < PW * PW / 4 / T; ++u) {   // LT[s][r] = L21(kd + r, k + s)
      const int e = tid + u * T, sc = e / (PW / 4), q = (e % (PW / 4)) * 4;
      cp16(&LT[sc][q], A + (k + sc) * lda + kd + q, 16);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) Z[ib + a][cb + b] = acc[a][b];
    cp_async_wait_all();
    __syncthreads();
    float upd[4][4] = {};
#pragma unroll 4
    for (int s = 0; s < PW; ++s) {
      const float4 l = *reinterpret_cast<const float4*>(&LT[s][ib]);
      const float4 z = *reinterpret_cast<const float4*>(&Z[s][cb]);
      const float lv[4] = {l.x, l.y, l.z, l.w}, zv[4] = {z.x, z.y, z.z, z.w};
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) upd[a][b] = fmaf(lv[a], zv[b], upd[a][b]);
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      if (cb + b >= cols) break;
      float4* const g = reinterpret_cast<float4*>(A + (col0 + cb + b) * lda + kd + ib);
      float4 v = *g;
      v.x -= upd[0][b]; v.y -= upd[1][b]; v.z -= upd[2][b]; v.w -= upd[3][b];
      *g = v;
    }
  }
}

__global__ void k_iota(int32_t* __restrict__ ipiv, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ipiv[i] = (int32_t)i;
}

}  // namespace st

// Host side of the look-ahead factorisation (see the head of this file). The
// scratch: per panel parity, the 32 x 32 inverses (in c->d_minv) and the
// split operands Ah, Al (rows below the panel) and Bh, Bl (columns right of
// it) in the tensor-core scratch set of that parity.
int lu_factor_static(fp_ctx* c, float* A, int64_t n, int64_t lda, int32_t* ipiv, float* cert, bool bf16) {
  using namespace st;
  static_assert((size_t)2 * kSlotFloats * sizeof(float) <= kMinvBytes, "inverse slots fit the panel scratch");
  FP_CUDA_TRY(c->err, cudaMemsetAsync(cert, 0, sizeof(float), c->stream));
  typedef U12Cfg<16, 1> CfgN;   // the next panel's columns: many small CTAs
  typedef U12Cfg<32, 2> CfgR;   // the columns beyond
  static SmemAttr attr_d, attr_l, attr_lx, attr_un, attr_ur, attr_lb, attr_unb, attr_urb, attr_la[3];
  FP_CUDA_TRY(c->err, attr_la[0].ensure(k_l21a<kSplitTf32>, (int)l21a_smem()));
  FP_CUDA_TRY(c->err, attr_la[1].ensure(k_l21a<kSplitBf16x2>, (int)l21a_smem()));
  FP_CUDA_TRY(c->err, attr_la[2].ensure(k_l21a<kSplitBf16>, (int)l21a_smem()));
  static SmemAttr attr_pi, attr_lg[2], attr_ugn[2], attr_ugr[2], attr_ugd[2], attr_ugw[2];
  // the GEMM form of the panel kernels, for the FP32 form (the BF16 form keeps
  // block substitution: with BF16 updates its GMRES-IR needed more iterations)
  const bool pg = c->panel_gemm > 0 && !bf16;   // U12 = inv(L) A12
  // 2: L21 by block substitution on the panel stream, inv(L) alone on the
  // third stream beside it; 1: both inverses on the panel stream, L21 = A21 inv(U)
  const bool lside = pg && c->panel_gemm == 2;
  // FP_TUNE_PDIAG_LINV: k_pdiag forms the full inv(L) too (no k_pinv), and
  // with the split chain L21 of the next panel's rows moves to the third
  // stream, beside U12 of the next panel's columns on the panel stream
  const bool dl = lside && c->pdiag_linv;
  const bool lg = pg && !lside;
  typedef U12gCfg<16> GCfgN;
  typedef U12gCfg<32> GCfgR;
  typedef U12gCfg<64> GCfgW;   // FP_TUNE_U12_WIDE: 64 columns a CTA for the columns beyond
  if (pg) {
    FP_CUDA_TRY(c->err, attr_pi.ensure(k_pinv, (int)pinv_smem()));
    FP_CUDA_TRY(c->err, attr_lg[0].ensure(k_l21g<kSplitTf32>, (int)l21g_smem()));
    FP_CUDA_TRY(c->err, attr_lg[1].ensure(k_l21g<kSplitBf16x2>, (int)l21g_smem()));
    FP_CUDA_TRY(c->err, attr_ugn[0].ensure(k_u12g<16, kSplitTf32>, (int)GCfgN::smem()));
    FP_CUDA_TRY(c->err, attr_ugn[1].ensure(k_u12g<16, kSplitBf16x2>, (int)GCfgN::smem()));
    FP_CUDA_TRY(c->err, attr_ugd[0].ensure(k_u12g<16, kSplitTf32, true>, (int)GCfgN::smem()));
    FP_CUDA_TRY(c->err, attr_ugd[1].ensure(k_u12g<16, kSplitBf16x2, true>, (int)GCfgN::smem()));
    FP_CUDA_TRY(c->err, attr_ugr[0].ensure(k_u12g<32, kSplitTf32>, (int)GCfgR::smem()));
    FP_CUDA_TRY(c->err, attr_ugr[1].ensure(k_u12g<32, kSplitBf16x2>, (int)GCfgR::smem()));
    FP_CUDA_TRY(c->err, attr_ugw[0].ensure(k_u12g<64, kSplitTf32>, (int)GCfgW::smem()));
    FP_CUDA_TRY(c->err, attr_ugw[1].ensure(k_u12g<64, kSplitBf16x2>, (int)GCfgW::smem()));
  }
  // the FP32 form's update from BF16 pairs (needs the GEMM-form panel kernels)
  const bool x3 = !bf16 && pg && c->tc_x3 && c->use_tc;
  FP_CUDA_TRY(c->err, attr_d.ensure(k_pdiag, (int)pdiag_smem(true)));
  FP_CUDA_TRY(c->err, attr_l.ensure(k_l21<kSplitTf32>, (int)l21_smem()));
  FP_CUDA_TRY(c->err, attr_lx.ensure(k_l21<kSplitBf16x2>, (int)l21_smem()));
  FP_CUDA_TRY(c->err, attr_un.ensure(k_u12<16, 1, false>, (int)CfgN::smem()));
  FP_CUDA_TRY(c->err, attr_ur.ensure(k_u12<32, 2, false>, (int)CfgR::smem()));
  FP_CUDA_TRY(c->err, attr_lb.ensure(k_l21<kSplitBf16>, (int)l21_smem()));
  FP_CUDA_TRY(c->err, attr_unb.ensure(k_u12<16, 1, true>, (int)CfgN::smem()));
  FP_CUDA_TRY(c->err, attr_urb.ensure(k_u12<32, 2, true>, (int)CfgR::smem()));
  if (int rc = ensure_tc_scratch(c, 0, n)) return rc;
  if (int rc = ensure_tc_scratch(c, 1, n)) return rc;
  // the tensor-core update splits the operands in shared memory: L21 and U12
  // are written unsplit (the FP32 form; the BF16 form has no lo part)
  const bool xsplit = !bf16 && c->tc_split > 0 && c->use_tc;
  st::k_iota<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(ipiv, n);
  ++c->nlaunch;
  float* const dinv_base = reinterpret_cast<float*>(c->d_minv);
  auto at = [&](int64_t r, int64_t col) { return A + col * lda + r; };
  c->trace.base = tr_event(c);
  FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_rest, c->stream));
  if (c->rest_split) FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_top, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream2, c->ev_rest, 0));
  // C -= L21 U12 on the rows [kend, n) and columns [cb, ce): tensor cores from
  // the split operands, or the SIMT kernel on the factors in place
  // (rows [kend + roff, kend + roff + mrows), mrows < 0: to n; roff rows into the L21 operand)
  auto update = [&](int slot, int64_t kend, int64_t K0, int64_t cb, int64_t ce, int64_t boff, int64_t roff = 0,
                    int64_t mrows = -1) -> int {
    const int64_t r0 = kend + roff;
    const int64_t m = mrows < 0 ? n - r0 : std::min<int64_t>(mrows, n - r0), nn = ce - cb;
    if (m <= 0 || nn <= 0) return FP_OK;
    float* const* s = c->d_tc[slot];
    const int kk = (int)std::min<int64_t>(PW, n - K0);
    const int64_t ao = roff * PW;   // the L21 operand's rows are PW elements apart (bf16 or float)
    if (bf16) {
      const __nv_bfloat16* ah = reinterpret_cast<const __nv_bfloat16*>(s[0]) + ao;
      const __nv_bfloat16* bh = reinterpret_cast<const __nv_bfloat16*>(s[2]) + boff * PW;
      if (c->use_tc && tc_gemm_sub_bf16(c, ah, bh, PW, at(r0, cb), lda, m, nn, kk)) return FP_OK;
    } else if (x3) {
      const __nv_bfloat16* ah = reinterpret_cast<const __nv_bfloat16*>(s[0]) + ao;
      const __nv_bfloat16* al = reinterpret_cast<const __nv_bfloat16*>(s[1]) + ao;
      const __nv_bfloat16* bh = reinterpret_cast<const __nv_bfloat16*>(s[2]) + boff * PW;
      const __nv_bfloat16* bl = reinterpret_cast<const __nv_bfloat16*>(s[3]) + boff * PW;
      if (tc_gemm_sub_bf16x3(c, ah, al, bh, bl, PW, at(r0, cb), lda, m, nn, kk)) return FP_OK;
    } else if (xsplit) {
      if (c->use_tc && tc_gemm_sub_xsplit(c, s[0] + ao, s[2] + boff * PW, PW, at(r0, cb), lda, m, nn, kk)) return FP_OK;
    } else if (c->use_tc && tc_gemm_sub_presplit(c, s[0] + ao, s[1] + ao, s[2] + boff * PW, s[3] + boff * PW, PW,
                                                 at(r0, cb), lda, m, nn, kk)) {
      return FP_OK;
    }
    FP_CUDA_TRY(c->err, cudaGetLastError());
    return gemm_sub_simt_f32(c, at(r0, K0), at(K0, cb), at(r0, cb), lda, m, nn, (int)std::min<int64_t>(PW, n - K0));
  };
  bool prev_split = false;   // the previous panel's rows below the next one were left to the third stream
  for (int64_t K0 = 0; K0 < n; K0 += PW) {
    const int64_t kend = std::min<int64_t>(K0 + PW, n);
    const int64_t knext = std::min<int64_t>(kend + PW, n);
    const int slot = (int)((K0 / PW) & 1);
    float* const dinv = dinv_base + (size_t)slot * kSlotFloats;   // then inv(L)^T, inv(U) (GEMM form)
    float* const* s = c->d_tc[slot];
    {
      TraceScope tr(c, TR_DIAG);
      float* const linvt = (dl && kend < n) ? dinv + kLinvtOff : nullptr;
      launch_k(c->pdl, k_pdiag, 1, kDiagThreads, pdiag_smem(linvt != nullptr), c->stream, A, lda, n, K0, dinv, cert,
               c->d_status, linvt);
      ++c->nlaunch;
      FP_CUDA_TRY(c->err, cudaGetLastError());
    }
    if (lg && kend < n) {   // the full inverses (a full panel: rows below exist)
      TraceScope tr(c, TR_PINV);
      launch_k(c->pdl, k_pinv, 2 * NIB, PI_THREADS, pinv_smem(), c->stream, A, lda, K0, dinv);
      ++c->nlaunch;
      FP_CUDA_TRY(c->err, cudaGetLastError());
    }
    // the columns beyond the next panel need only the diagonal block's
    // inverses for their U12: the second stream starts them beside k_l21
    FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_diag, c->stream));
    if (dl && kend < n) FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_pinv, c->stream));   // inv(L) came with k_pdiag
    if (lside && !dl && kend < n) {   // inv(L) (the first NIB CTAs of k_pinv) on the third stream, beside k_l21
      OnStream on3(c, c->stream3);
      FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_diag, 0));
      {
        TraceScope tr(c, TR_PINV);
        launch_k(c->pdl, k_pinv, NIB, PI_THREADS, pinv_smem(), c->stream, A, lda, K0, dinv);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaGetLastError());
      }
      FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_pinv, c->stream));
    }
    // split: the panel stream keeps only what the next diagonal block needs
    // (L21 and the next-panel update of the next panel's 128 rows); the
    // third stream does the rows below, beside the next k_pdiag
    const bool sp = c->lu_split && lside && c->lu_overlap && kend + PW < n;
    // rest split: the trailing update of the columns beyond runs as the next
    // panel's rows (T), then the rows below (B); the next panel's U12 kernels
    // read only T's rows, so they wait for T (ev_top) and U12 of the columns
    // beyond runs on the fourth stream beside B; what reads B's rows waits
    // for ev_rest
    const bool rs = sp && c->rest_split;
    // 2: T on the fourth stream after U12 of the columns beyond, so that B
    // starts as soon as that U12 is done; T waits for B of the previous
    // panel (the same rows), which keeps the additions to a row in order
    const bool rs2 = rs && c->rest_split == 2;
    // the rows below this panel's diagonal block were last updated on the third stream
    if (prev_split && kend < n) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_tcr, 0));
    if (sp) {
      float* const al = s[1];
      // with the full inv(L) from k_pdiag both L21 launches run on the third
      // stream, the next panel's rows first
      OnStream on3h(c, dl ? c->stream3 : c->stream);
      if (dl) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_diag, 0));
      {
        TraceScope tr(c, TR_L21);
        const int64_t he = kend + PW;   // the next panel's rows
        if (x3)
          launch_k(c->pdl, c->l21_async ? k_l21a<kSplitBf16x2> : k_l21<kSplitBf16x2>, (unsigned)(PW / L21_ROWS), L21_THREADS, c->l21_async ? l21a_smem() : l21_smem(), c->stream, A, lda,
                   he, K0, kend, kend, dinv, s[0], s[1], cert);
        else
          launch_k(c->pdl, c->l21_async ? k_l21a<kSplitTf32> : k_l21<kSplitTf32>, (unsigned)(PW / L21_ROWS), L21_THREADS, c->l21_async ? l21a_smem() : l21_smem(), c->stream, A, lda, he,
                   K0, kend, kend, dinv, s[0], xsplit ? nullptr : al, cert);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaGetLastError());
      }
      if (dl) FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_panel, c->stream));
      OnStream on3(c, c->stream3);
      {
        TraceScope tr(c, TR_L21);
        const unsigned g = (unsigned)((n - kend - PW + L21_ROWS - 1) / L21_ROWS);
        if (x3)
          launch_k(c->pdl, c->l21_async ? k_l21a<kSplitBf16x2> : k_l21<kSplitBf16x2>, g, L21_THREADS, c->l21_async ? l21a_smem() : l21_smem(), c->stream, A, lda, n, K0, kend, kend + PW,
                   dinv, s[0], s[1], cert);
        else
          launch_k(c->pdl, c->l21_async ? k_l21a<kSplitTf32> : k_l21<kSplitTf32>, g, L21_THREADS, c->l21_async ? l21a_smem() : l21_smem(), c->stream, A, lda, n, K0, kend, kend + PW, dinv,
                   s[0], xsplit ? nullptr : al, cert);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaGetLastError());
      }
      FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_l21t, c->stream));
    } else if (kend < n) {
      TraceScope tr(c, TR_L21);
      const unsigned g = (unsigned)((n - kend + L21_ROWS - 1) / L21_ROWS);
      float* const al = bf16 ? s[1] : (xsplit ? nullptr : s[1]);
      if (lg) {
        if (x3) launch_k(c->pdl, k_l21g<kSplitBf16x2>, g, L21G_THREADS, l21g_smem(), c->stream, A, lda, n, K0, kend, dinv, s[0], s[1], cert);
        else launch_k(c->pdl, k_l21g<kSplitTf32>, g, L21G_THREADS, l21g_smem(), c->stream, A, lda, n, K0, kend, dinv, s[0], al, cert);
      } else if (bf16) {
        launch_k(c->pdl, c->l21_async ? k_l21a<kSplitBf16> : k_l21<kSplitBf16>, g, L21_THREADS, c->l21_async ? l21a_smem() : l21_smem(), c->stream, A, lda, n, K0, kend, kend, dinv, s[0], al, cert);
      } else if (x3) {
        launch_k(c->pdl, c->l21_async ? k_l21a<kSplitBf16x2> : k_l21<kSplitBf16x2>, g, L21_THREADS, c->l21_async ? l21a_smem() : l21_smem(), c->stream, A, lda, n, K0, kend, kend, dinv, s[0], s[1], cert);
      } else {
        launch_k(c->pdl, c->l21_async ? k_l21a<kSplitTf32> : k_l21<kSplitTf32>, g, L21_THREADS, c->l21_async ? l21a_smem() : l21_smem(), c->stream, A, lda, n, K0, kend, kend, dinv, s[0], al, cert);
      }
      ++c->nlaunch;
      FP_CUDA_TRY(c->err, cudaGetLastError());
    }
    if (!(dl && sp)) FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_panel, c->stream));
    if (knext > kend) {
      // split: U12 of the next panel's columns and the update of its diagonal
      // tile in one launch (k_u12g<16, ., true>)
      const bool fused = sp && c->lu_fuse;
      // the next panel's columns: after the previous panel's trailing update
      // (rest split: its rows of this panel, unless the launch also updates
      // the diagonal tile below them)
      FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->rest_split && !fused ? c->ev_top : c->ev_rest, 0));
      if (lside && kend < n) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_pinv, 0));
      if (fused) {
        if (dl) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_panel, 0));   // L21 of the next panel's rows
        TraceScope tr(c, TR_U12);
        const unsigned g = (unsigned)((knext - kend + 15) / 16);
        if (x3)
          launch_k(c->pdl, k_u12g<16, kSplitBf16x2, true>, g, GCfgN::THREADS, GCfgN::smem(), c->stream, A, lda, K0, kend,
                   knext, dinv, s[2], s[3], kend, (int)c->u12_async);
        else
          launch_k(c->pdl, k_u12g<16, kSplitTf32, true>, g, GCfgN::THREADS, GCfgN::smem(), c->stream, A, lda, K0, kend,
                   knext, dinv, s[2], xsplit ? nullptr : s[3], kend, (int)c->u12_async);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaGetLastError());
      } else {
        TraceScope tr(c, TR_U12);
        const unsigned g = (unsigned)((knext - kend + 15) / 16);
        if (x3)
          launch_k(c->pdl, k_u12g<16, kSplitBf16x2>, g, GCfgN::THREADS, GCfgN::smem(), c->stream, A, lda, K0, kend, knext, dinv, s[2], s[3], (int64_t)0, (int)c->u12_async);
        else if (pg)
          launch_k(c->pdl, k_u12g<16, kSplitTf32>, g, GCfgN::THREADS, GCfgN::smem(), c->stream, A, lda, K0, kend, knext, dinv, s[2],
                                                                                     xsplit ? nullptr : s[3], (int64_t)0, (int)c->u12_async);
        else if (bf16)
          launch_k(c->pdl, k_u12<16, 1, true>, g, CfgN::THREADS, CfgN::smem(), c->stream, A, lda, K0, kend, knext, dinv, s[2], s[3]);
        else
          launch_k(c->pdl, k_u12<16, 1, false>, g, CfgN::THREADS, CfgN::smem(), c->stream, A, lda, K0, kend, knext, dinv, s[2],
                                                                              xsplit ? nullptr : s[3]);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaGetLastError());
      }
      if (sp) {
        FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_u12n, c->stream));
        if (!fused) {
          if (c->rest_split) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_rest, 0));
          if (dl) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_panel, 0));   // L21 of these rows
          if (int rc = update(slot, kend, K0, kend, knext, 0, 0, PW)) return rc;   // the next diagonal block's rows
        }
        OnStream on3(c, c->stream3);
        FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_u12n, 0));
        if (c->rest_split) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_rest, 0));
        if (int rc = update(slot, kend, K0, kend, knext, 0, PW)) return rc;      // the rows below
        FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_tcr, c->stream));
      } else {
        if (c->rest_split) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_rest, 0));
        if (int rc = update(slot, kend, K0, kend, knext, 0)) return rc;
      }
    }
    prev_split = sp;
    // the columns beyond the next panel: on the second stream (look-ahead), or
    // after the panel's own work on the same stream
    auto rest = [&]() -> int {
      if (n > knext) {
        {   // rest split: U12 of the columns beyond on the fourth stream, after T of the previous panel
          OnStream on4(c, rs ? c->stream4 : c->stream);
          if (rs) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_top, 0));
          if (lside) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_pinv, 0));   // inv(L)
          {
            TraceScope tr(c, TR_STRIP);
            const unsigned g = (unsigned)((n - knext + 31) / 32);
            // the B operand of the columns beyond starts (knext - kend) columns in (bf16 or float elements)
            const auto b16 = [&](float* p) {
              return reinterpret_cast<float*>(reinterpret_cast<__nv_bfloat16*>(p) + (knext - kend) * PW);
            };
            float* bh = (bf16 || x3) ? b16(s[2]) : s[2] + (knext - kend) * PW;
            const unsigned gw = (unsigned)((n - knext + 63) / 64);
            if (x3 && c->u12_wide)
              launch_k(c->pdl, k_u12g<64, kSplitBf16x2>, gw, GCfgW::THREADS, GCfgW::smem(), c->stream, A, lda, K0, knext, n,
                       dinv, bh, b16(s[3]), (int64_t)0, (int)c->u12_async);
            else if (x3)
              launch_k(c->pdl, k_u12g<32, kSplitBf16x2>, g, GCfgR::THREADS, GCfgR::smem(), c->stream, A, lda, K0, knext, n, dinv, bh,
                                                                                          b16(s[3]), (int64_t)0, (int)c->u12_async);
            else if (pg)
              launch_k(c->pdl, k_u12g<32, kSplitTf32>, g, GCfgR::THREADS, GCfgR::smem(), c->stream, 
                  A, lda, K0, knext, n, dinv, bh, xsplit ? nullptr : s[3] + (knext - kend) * PW, (int64_t)0, (int)c->u12_async);
            else if (bf16)
              launch_k(c->pdl, k_u12<32, 2, true>, g, CfgR::THREADS, CfgR::smem(), c->stream, A, lda, K0, knext, n, dinv, bh, nullptr);
            else
              launch_k(c->pdl, k_u12<32, 2, false>, g, CfgR::THREADS, CfgR::smem(), c->stream, 
                  A, lda, K0, knext, n, dinv, bh, xsplit ? nullptr : s[3] + (knext - kend) * PW);
            ++c->nlaunch;
            FP_CUDA_TRY(c->err, cudaGetLastError());
          }
          if (rs) FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_u12r, c->stream));
          if (rs2) {
            FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_panel, 0));   // L21 of these rows
            FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_rest, 0));    // B of the previous panel
            if (int rc = update(slot, kend, K0, knext, n, knext - kend, 0, PW)) return rc;   // T
            FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_top, c->stream));
          }
        }
        if (rs) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_u12r, 0));
        // the update reads L21 (the panel stream's k_l21, and the third stream's when split)
        if (c->lu_overlap) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_panel, 0));
        if (rs) {
          if (!rs2) {
            if (int rc = update(slot, kend, K0, knext, n, knext - kend, 0, PW)) return rc;   // T: the next panel's rows
            FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_top, c->stream));
          }
          FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_l21t, 0));
          if (int rc = update(slot, kend, K0, knext, n, knext - kend, PW)) return rc;      // B: the rows below
          return FP_OK;
        }
        if (sp) FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_l21t, 0));
        if (int rc = update(slot, kend, K0, knext, n, knext - kend)) return rc;
      }
      return FP_OK;
    };
    if (c->lu_overlap) {
      OnStream2 on2(c);
      FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_diag, 0));
      if (int rc = rest()) return rc;
      if (c->rest_split && !rs) FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_top, c->stream));
      FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_rest, c->stream));
    } else {
      if (int rc = rest()) return rc;
      if (c->rest_split) FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_top, c->stream));
      FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_rest, c->stream));
    }
  }
  FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_rest, 0));
  return FP_OK;
}

}  // namespace fpb
