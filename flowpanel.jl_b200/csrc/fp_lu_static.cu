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
#include <cfloat>

#include "fp_internal.cuh"

namespace fpb {
namespace st {

constexpr int PW = kStaticPanel;   // panel width (128)
constexpr int IB = 32;             // inner block of the diagonal factor
constexpr int NIB = PW / IB;       // inner blocks per panel
constexpr int SP = PW + 4;         // shared row pitch (floats) of 128-wide rows: 16-byte rows, not 32 banks
constexpr int DP = IB + 4;         // pitch of the 32 x 32 inverses (16-byte rows for float4 reads)
constexpr int kDiagThreads = 512;
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

__device__ __forceinline__ void atomic_max_pos(float* addr, float v) {
  if (v > 0.f) atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

// ---------------------------------------------------------------------------
// K1: the PW x PW diagonal block at (k, k), factored in place (unit L below,
// U on and above the diagonal); the inverses of its IB x IB diagonal blocks
// of L and U go to dinv. Rows and columns past n are padded with the identity.
constexpr size_t pdiag_smem() {
  return (size_t)PW * SP * sizeof(float)        // As
         + (size_t)IB * SP * sizeof(float)      // LT: the inner block's L columns, transposed
         + (size_t)2 * IB * DP * sizeof(float); // inverses of the current inner block
}

__global__ void __launch_bounds__(kDiagThreads, 1)
k_pdiag(float* __restrict__ A, int64_t lda, int64_t n, int64_t k, float* __restrict__ dinv,
        float* __restrict__ cert, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  float (*As)[SP] = reinterpret_cast<float (*)[SP]>(smem);
  float (*LT)[SP] = reinterpret_cast<float (*)[SP]>(smem + (size_t)PW * SP * sizeof(float));
  float (*Li)[DP] = reinterpret_cast<float (*)[DP]>(smem + (size_t)(PW + IB) * SP * sizeof(float));
  float (*Ui)[DP] = Li + IB;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nb = (int)imin64(PW, n - k);
  for (int e = tid; e < PW * PW; e += kDiagThreads) {
    const int r = e % PW, c = e / PW;   // rows fastest: coalesced column reads
    As[r][c] = (r < nb && c < nb) ? __ldcg(&A[(k + c) * lda + k + r]) : (r == c ? 1.f : 0.f);
  }
  __syncthreads();
  float lmax = 0.f;
#pragma unroll 1
  for (int kb = 0; kb < NIB; ++kb) {
    const int k0 = kb * IB, k1 = k0 + IB, R = PW - k1;   // R rows (and columns) after the inner block
    // (a) warp 0 eliminates the IB x IB block. Lane i holds row i shifted so
    // that R[0] is the current column (static register indices, rolled step
    // loop); a row stops shifting once it is the pivot row, so at the end lane
    // i holds U(i, i..) and writes it; each step's multipliers go to As.
    if (warp == 0) {
      float Rw[IB];
      const float4* rp = reinterpret_cast<const float4*>(&As[k0 + lane][k0]);
#pragma unroll
      for (int q = 0; q < IB / 4; ++q) {
        const float4 v = rp[q];
        Rw[4 * q] = v.x; Rw[4 * q + 1] = v.y; Rw[4 * q + 2] = v.z; Rw[4 * q + 3] = v.w;
      }
      bool bad = false;
#pragma unroll 1
      for (int j = 0; j < IB; ++j) {
        float pv[IB];
#pragma unroll
        for (int c = 0; c < IB; ++c) pv[c] = __shfl_sync(FULL, Rw[c], j);
        bad |= !(fabsf(pv[0]) > 0.f && fabsf(pv[0]) <= FLT_MAX);
        if (lane > j) {
          const float l = Rw[0] / pv[0];
          As[k0 + lane][k0 + j] = l;
          lmax = fmaxf(lmax, fabsf(l));
#pragma unroll
          for (int c = 0; c < IB - 1; ++c) Rw[c] = fmaf(-l, pv[c + 1], Rw[c + 1]);
          Rw[IB - 1] = 0.f;
        }
      }
#pragma unroll
      for (int c = 0; c < IB; ++c)
        if (c < IB - lane) As[k0 + lane][k0 + lane + c] = Rw[c];
      if (bad && lane == 0) atomicOr(status, (int)DEV_ZERO_PIVOT);
    }
    __syncthreads();
    // (a2) warp 0: inv(U_kk), warp 1: inv(L_kk); lane c forms column c by
    // substitution, its entries kept in the inverse's own column
    if (warp == 0) {
#pragma unroll 1
      for (int i = IB - 1; i >= 0; --i) {
        float s0 = (lane == i) ? 1.f : 0.f, s1 = 0.f;
        int t = i + 1;
#pragma unroll 1
        for (; t + 1 < IB; t += 2) {
          s0 = fmaf(-As[k0 + i][k0 + t], Ui[t][lane], s0);
          s1 = fmaf(-As[k0 + i][k0 + t + 1], Ui[t + 1][lane], s1);
        }
        if (t < IB) s0 = fmaf(-As[k0 + i][k0 + t], Ui[t][lane], s0);
        Ui[i][lane] = (s0 + s1) / As[k0 + i][k0 + i];
      }
    } else if (warp == 1) {
#pragma unroll 1
      for (int i = 0; i < IB; ++i) {
        float s0 = (lane == i) ? 1.f : 0.f, s1 = 0.f;
        int t = 0;
#pragma unroll 1
        for (; t + 1 < i; t += 2) {
          s0 = fmaf(-As[k0 + i][k0 + t], Li[t][lane], s0);
          s1 = fmaf(-As[k0 + i][k0 + t + 1], Li[t + 1][lane], s1);
        }
        if (t < i) s0 = fmaf(-As[k0 + i][k0 + t], Li[t][lane], s0);
        Li[i][lane] = s0 + s1;
      }
    }
    __syncthreads();
    for (int e = tid; e < 2 * IB * IB; e += kDiagThreads) {   // keep both inverses for the panel's products
      const int which = e / (IB * IB), r = (e / IB) % IB, c = e % IB;
      dinv[dinv_off(kb, which) + r * IB + c] = which ? Ui[r][c] : Li[r][c];
    }
    if (R == 0) break;
    // (b) rows below: L(i, kb) = A(i, kb) inv(U_kk) into LT (transposed);
    // columns right: U(kb, j) = inv(L_kk) A(kb, j) into registers. Both read
    // parts of As that the other part's results replace, so As is written
    // after the barrier.
    {
      if (tid < (R / 4) * 8) {   // (row quad, 4-column group)
        const int tg = tid & 7, iq = tid >> 3;
        const int t0 = 4 * tg, i0 = k1 + 4 * iq;
        float acc[4][4] = {};
        for (int s = 0; s <= t0 + 3; ++s) {
          const float4 u = *reinterpret_cast<const float4*>(&Ui[s][t0]);   // inv(U)[s][t] = 0 for s > t
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float a = As[i0 + i][k0 + s];
            acc[i][0] = fmaf(a, u.x, acc[i][0]);
            acc[i][1] = fmaf(a, u.y, acc[i][1]);
            acc[i][2] = fmaf(a, u.z, acc[i][2]);
            acc[i][3] = fmaf(a, u.w, acc[i][3]);
          }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int c = 0; c < 4; ++c) LT[t0 + c][i0 + i] = acc[i][c];
      }
      // (32-column group, inner row quad): at most 24 tasks, so two per warp
      constexpr int NW = kDiagThreads / 32;
      const int ntask_c = (R / 32) * 8;
      float uc[2][4] = {};
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int task = warp + q * NW;
        if (task < ntask_c) {
          const int tq = task & 7, jg = task >> 3;
          const int j = k1 + 32 * jg + lane, t0 = 4 * tq;
          for (int s = 0; s <= t0 + 3; ++s) {
            const float a = As[k0 + s][j];
#pragma unroll
            for (int i = 0; i < 4; ++i) uc[q][i] = fmaf(Li[t0 + i][s], a, uc[q][i]);   // inv(L)[t][s] = 0 for s > t
          }
        }
      }
      __syncthreads();
      for (int e = tid; e < R * IB; e += kDiagThreads) {
        const int i = e / IB, t = e % IB;
        const float v = LT[t][k1 + i];
        As[k1 + i][k0 + t] = v;
        lmax = fmaxf(lmax, fabsf(v));
      }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int task = warp + q * NW;
        if (task < ntask_c) {
          const int tq = task & 7, jg = task >> 3;
#pragma unroll
          for (int i = 0; i < 4; ++i) As[k0 + 4 * tq + i][k1 + 32 * jg + lane] = uc[q][i];
        }
      }
    }
    __syncthreads();
    // (c) trailing update of the block: As(i, j) -= sum_t LT(t, i) As(k0 + t, j), i, j >= k1;
    // thread tile 4 x 4
    {
      const int tiles = (R / 4) * (R / 4);
      for (int tile = tid; tile < tiles; tile += kDiagThreads) {
        const int jq = tile % (R / 4), iq = tile / (R / 4);
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
    __syncthreads();
  }
  // write the factors back (rows fastest: coalesced)
  for (int e = tid; e < nb * nb; e += kDiagThreads) {
    const int r = e % nb, c = e / nb;
    A[(k + c) * lda + k + r] = As[r][c];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(FULL, lmax, o));
  if (lane == 0) atomic_max_pos(cert, lmax);
}

// ---------------------------------------------------------------------------
// Register-tiled product over shared memory: acc[i][j] += sum_{s < K}
// P[r0 + i][s] Q[s][c0 + j] (P row pitch PP, Q row pitch QP; 4 x 4 tile).
template <int PP, int QP>
__device__ __forceinline__ void tile4x4(const float (*P)[PP], const float (*Q)[QP], int r0, int c0, int K,
                                        float (&acc)[4][4]) {
#pragma unroll 4
  for (int s = 0; s < K; ++s) {
    const float4 q = *reinterpret_cast<const float4*>(&Q[s][c0]);
    const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float p = P[r0 + i][s];
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(p, qv[j], acc[i][j]);
    }
  }
}

// ---------------------------------------------------------------------------
// K6: L21 = A21 U^-1 for the rows [r0 + 64 b, +64) below the panel at k, by
// block substitution over the four inner column blocks t:
//   Y_t = A21_t - sum_{s < t} L_s U(s, t),   L_t = Y_t inv(U_tt).
// Writes L21 in place and its split Ah = rna_tf32(L21), Al = L21 - Ah
// (K-major: row (r - r0) of ldk = PW floats); max|L21| into cert.
constexpr int L21_ROWS = 64, L21_THREADS = 128;   // 16 x 8 thread tiles of 4 x 4 over 64 x 32
constexpr int XP = PW + 4;   // row pitch of the row block
constexpr size_t l21_smem() {
  return (size_t)L21_ROWS * XP * sizeof(float) + (size_t)(PW - IB) * (IB + 4) * sizeof(float) +
         (size_t)IB * (IB + 4) * sizeof(float);
}

__global__ void __launch_bounds__(L21_THREADS)
k_l21(float* __restrict__ A, int64_t lda, int64_t n, int64_t k, int64_t r0, const float* __restrict__ dinv,
      float* __restrict__ Ah, float* __restrict__ Al, float* __restrict__ cert) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int UP = IB + 4;
  float (*X)[XP] = reinterpret_cast<float (*)[XP]>(smem);
  float (*Ub)[UP] = reinterpret_cast<float (*)[UP]>(smem + (size_t)L21_ROWS * XP * sizeof(float));   // U(s-blocks, t)
  float (*Ut)[UP] = Ub + (PW - IB);                                                                     // inv(U_tt)
  const int tid = threadIdx.x;
  const int64_t row0 = r0 + (int64_t)blockIdx.x * L21_ROWS;
  const int rows = (int)imin64(L21_ROWS, n - row0);
  for (int e = tid; e < L21_ROWS * PW; e += L21_THREADS) {
    const int r = e % L21_ROWS, c = e / L21_ROWS;
    X[r][c] = (r < rows) ? __ldcg(&A[(k + c) * lda + row0 + r]) : 0.f;
  }
  const int rg = tid & 15, cg = tid >> 4;   // 16 row quads x 8 column quads = 64 x 32
#pragma unroll 1
  for (int t = 0; t < NIB; ++t) {
    const int c0 = t * IB;
    // U(0..c0-1, c0..c0+31) and inv(U_tt)
    for (int e = tid; e < c0 * IB; e += L21_THREADS) {
      const int s = e % c0, c = e / c0;
      Ub[s][c] = __ldcg(&A[(k + c0 + c) * lda + k + s]);
    }
    for (int e = tid; e < IB * IB; e += L21_THREADS) Ut[e / IB][e % IB] = dinv[dinv_off(t, 1) + e];
    __syncthreads();
    float y[4][4] = {};
    if (c0 > 0) tile4x4<XP, UP>(X, Ub, 4 * rg, 4 * cg, c0, y);   // sum_s L_s U(s, t) (X's columns < c0 hold L)
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) X[4 * rg + i][c0 + 4 * cg + j] -= y[i][j];
    __syncthreads();
    float l[4][4] = {};
    // L_t = Y_t inv(U_tt): P = X's column block t (pitch XP, offset c0)
#pragma unroll 4
    for (int s = 0; s < IB; ++s) {
      const float4 q = *reinterpret_cast<const float4*>(&Ut[s][4 * cg]);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float p = X[4 * rg + i][c0 + s];
#pragma unroll
        for (int j = 0; j < 4; ++j) l[i][j] = fmaf(p, qv[j], l[i][j]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) X[4 * rg + i][c0 + 4 * cg + j] = l[i][j];
    __syncthreads();
  }
  float lmax = 0.f;
  for (int e = tid; e < rows * PW; e += L21_THREADS) {
    const int r = e % rows, c = e / rows;   // rows fastest: coalesced column stores
    A[(k + c) * lda + row0 + r] = X[r][c];
  }
  for (int e = tid; e < rows * PW; e += L21_THREADS) {
    const int r = e / PW, c = e % PW;       // columns fastest: K-major split
    const float v = X[r][c];
    const float h = tf32_rna(v);
    const int64_t o = (row0 - r0 + r) * (int64_t)PW + c;
    Ah[o] = h;
    Al[o] = v - h;
    lmax = fmaxf(lmax, fabsf(v));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(FULL, lmax, o));
  if ((tid & 31) == 0) atomic_max_pos(cert, lmax);
}

// ---------------------------------------------------------------------------
// K2: U12 = L^-1 A12 for the panel's rows [k, k + PW) and the columns
// [c0 + CW b, +CW) of [c0, c1), by block substitution over the four inner row
// blocks t:  Z_t = A12_t - sum_{s < t} L(t, s) U12_s,  U12_t = inv(L_tt) Z_t.
// Writes U12 in place and its split Bh, Bl (column j - c0 holds its PW
// values contiguously). Thread tile: RT rows of block t x 4 columns.
template <int CW, int RT>
struct U12Cfg {
  static constexpr int THREADS = (IB / RT) * (CW / 4);
  static constexpr int ZP = CW + 4;   // row pitch of the column block
  static constexpr size_t smem() {
    return (size_t)PW * ZP * sizeof(float) + (size_t)IB * (PW - IB + 4) * sizeof(float) +
           (size_t)IB * (IB + 4) * sizeof(float);
  }
};

template <int CW, int RT>
__global__ void __launch_bounds__(U12Cfg<CW, RT>::THREADS)
k_u12(float* __restrict__ A, int64_t lda, int64_t k, int64_t c0, int64_t c1, const float* __restrict__ dinv,
      float* __restrict__ Bh, float* __restrict__ Bl) {
  constexpr int T = U12Cfg<CW, RT>::THREADS, ZP = U12Cfg<CW, RT>::ZP, LP = PW - IB + 4, IP = IB + 4;
  extern __shared__ __align__(16) unsigned char smem[];
  float (*Z)[ZP] = reinterpret_cast<float (*)[ZP]>(smem);                                    // PW x CW
  float (*Lb)[LP] = reinterpret_cast<float (*)[LP]>(smem + (size_t)PW * ZP * sizeof(float));  // L(t, 0..t0-1)
  float (*Lt)[IP] = reinterpret_cast<float (*)[IP]>(reinterpret_cast<unsigned char*>(Lb) +
                                                     (size_t)IB * LP * sizeof(float));        // inv(L_tt)
  const int tid = threadIdx.x;
  const int64_t col0 = c0 + (int64_t)blockIdx.x * CW;
  const int cols = (int)imin64(CW, c1 - col0);
  for (int e = tid; e < PW * CW; e += T) {
    const int r = e % PW, c = e / PW;
    Z[r][c] = (c < cols) ? __ldcg(&A[(col0 + c) * lda + k + r]) : 0.f;
  }
  constexpr int CQ = CW / 4;
  const int cq = tid % CQ, rq = tid / CQ;   // rq < IB / RT
#pragma unroll 1
  for (int t = 0; t < NIB; ++t) {
    const int t0 = t * IB;
    for (int e = tid; e < IB * t0; e += T) {
      const int r = e % IB, s = e / IB;
      Lb[r][s] = __ldcg(&A[(k + s) * lda + k + t0 + r]);
    }
    for (int e = tid; e < IB * IB; e += T) Lt[e / IB][e % IB] = dinv[dinv_off(t, 0) + e];
    __syncthreads();
    float z[RT][4] = {};
#pragma unroll 4
    for (int s = 0; s < t0; ++s) {
      const float4 q = *reinterpret_cast<const float4*>(&Z[s][4 * cq]);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int i = 0; i < RT; ++i) {
        const float p = Lb[RT * rq + i][s];
#pragma unroll
        for (int j = 0; j < 4; ++j) z[i][j] = fmaf(p, qv[j], z[i][j]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RT; ++i)
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
        const float p = Lt[RT * rq + i][s];
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
  for (int e = tid; e < PW * cols; e += T) {
    const int r = e % PW, c = e / PW;   // rows fastest: coalesced, and K-major for the split
    const float v = Z[r][c];
    A[(col0 + c) * lda + k + r] = v;
    const float h = tf32_rna(v);
    const int64_t o = (col0 - c0 + c) * (int64_t)PW + r;
    Bh[o] = h;
    Bl[o] = v - h;
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
int lu_factor_static(fp_ctx* c, float* A, int64_t n, int64_t lda, int32_t* ipiv, float* cert) {
  using namespace st;
  static_assert((size_t)2 * kDinvFloats * sizeof(float) <= kMinvBytes, "inverse slots fit the panel scratch");
  FP_CUDA_TRY(c->err, cudaMemsetAsync(cert, 0, sizeof(float), c->stream));
  typedef U12Cfg<8, 1> CfgN;    // the next panel's columns: many small CTAs
  typedef U12Cfg<32, 2> CfgR;   // the columns beyond
  static SmemAttr attr_d, attr_l, attr_un, attr_ur;
  FP_CUDA_TRY(c->err, attr_d.ensure(k_pdiag, (int)pdiag_smem()));
  FP_CUDA_TRY(c->err, attr_l.ensure(k_l21, (int)l21_smem()));
  FP_CUDA_TRY(c->err, attr_un.ensure(k_u12<8, 1>, (int)CfgN::smem()));
  FP_CUDA_TRY(c->err, attr_ur.ensure(k_u12<32, 2>, (int)CfgR::smem()));
  if (int rc = ensure_tc_scratch(c, 0, n)) return rc;
  if (int rc = ensure_tc_scratch(c, 1, n)) return rc;
  st::k_iota<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(ipiv, n);
  ++c->nlaunch;
  float* const dinv_base = reinterpret_cast<float*>(c->d_minv);
  auto at = [&](int64_t r, int64_t col) { return A + col * lda + r; };
  c->trace.base = tr_event(c);
  FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_rest, c->stream));
  FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream2, c->ev_rest, 0));
  // C -= L21 U12 on the rows [kend, n) and columns [cb, ce): tensor cores from
  // the split operands, or the SIMT kernel on the factors in place
  auto update = [&](int slot, int64_t kend, int64_t K0, int64_t cb, int64_t ce, int64_t boff) -> int {
    const int64_t m = n - kend, nn = ce - cb;
    if (m <= 0 || nn <= 0) return FP_OK;
    float* const* s = c->d_tc[slot];
    if (c->use_tc && tc_gemm_sub_presplit(c, s[0], s[1], s[2] + boff * PW, s[3] + boff * PW, PW, at(kend, cb), lda, m,
                                          nn, (int)(std::min<int64_t>(PW, n - K0))))
      return FP_OK;
    FP_CUDA_TRY(c->err, cudaGetLastError());
    return gemm_sub_simt_f32(c, at(kend, K0), at(K0, cb), at(kend, cb), lda, m, nn, (int)std::min<int64_t>(PW, n - K0));
  };
  for (int64_t K0 = 0; K0 < n; K0 += PW) {
    const int64_t kend = std::min<int64_t>(K0 + PW, n);
    const int64_t knext = std::min<int64_t>(kend + PW, n);
    const int slot = (int)((K0 / PW) & 1);
    float* const dinv = dinv_base + (size_t)slot * kDinvFloats;
    float* const* s = c->d_tc[slot];
    {
      TraceScope tr(c, TR_DIAG);
      k_pdiag<<<1, kDiagThreads, pdiag_smem(), c->stream>>>(A, lda, n, K0, dinv, cert, c->d_status);
      ++c->nlaunch;
      FP_CUDA_TRY(c->err, cudaGetLastError());
    }
    if (kend < n) {
      TraceScope tr(c, TR_L21);
      k_l21<<<(unsigned)((n - kend + L21_ROWS - 1) / L21_ROWS), L21_THREADS, l21_smem(), c->stream>>>(
          A, lda, n, K0, kend, dinv, s[0], s[1], cert);
      ++c->nlaunch;
      FP_CUDA_TRY(c->err, cudaGetLastError());
    }
    FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_panel, c->stream));
    if (knext > kend) {
      // the next panel's columns: after the previous panel's trailing update
      FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_rest, 0));
      {
        TraceScope tr(c, TR_U12);
        k_u12<8, 1><<<(unsigned)((knext - kend + 7) / 8), CfgN::THREADS, CfgN::smem(), c->stream>>>(
            A, lda, K0, kend, knext, dinv, s[2], s[3]);
        ++c->nlaunch;
        FP_CUDA_TRY(c->err, cudaGetLastError());
      }
      if (int rc = update(slot, kend, K0, kend, knext, 0)) return rc;
    }
    {
      OnStream2 on2(c);
      FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_panel, 0));
      if (n > knext) {
        {
          TraceScope tr(c, TR_STRIP);
          k_u12<32, 2><<<(unsigned)((n - knext + 31) / 32), CfgR::THREADS, CfgR::smem(), c->stream>>>(
              A, lda, K0, knext, n, dinv, s[2] + (knext - kend) * PW, s[3] + (knext - kend) * PW);
          ++c->nlaunch;
          FP_CUDA_TRY(c->err, cudaGetLastError());
        }
        if (int rc = update(slot, kend, K0, knext, n, knext - kend)) return rc;
      }
      FP_CUDA_TRY(c->err, cudaEventRecord(c->ev_rest, c->stream));
    }
  }
  FP_CUDA_TRY(c->err, cudaStreamWaitEvent(c->stream, c->ev_rest, 0));
  return FP_OK;
}

}  // namespace fpb
