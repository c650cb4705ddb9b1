// FP32 trailing update C -= A B of the mixed-precision LU on the 5th-generation
// tensor cores (tcgen05, kind::tf32), with the 3xTF32 split
//     A B ~= Ah Bh + Ah Bl + Al Bh,   Ah = rna_tf32(A), Al = A - Ah (same for B)
// which keeps the product at FP32-level accuracy (a single TF32 product
// would leave kappa * u_tf32 ~ 10 on the wing AIC and refinement would not
// converge).
//
// Data flow per 128 x 128 output tile (one CTA, 4 warps):
//   * split kernels write Ah, Al (K-major copies of the L21 panel) and Bh, Bl
//     (K-major copies of the U12 panel) to scratch in HBM;
//   * warp 0 / lane 0 streams 16-wide K blocks of the four operands into a
//     3-stage shared-memory ring with TMA (SWIZZLE_64B, no multicast); the
//     ring (96 KB) leaves room for a second CTA on the SM, whose epilogue
//     overlaps this one's MMAs;
//   * warp 1 / lane 0 issues 3 x 4 tcgen05.mma (M=128, N=128, K=8) per K block
//     into a 128-column TMEM accumulator and frees each stage with
//     tcgen05.commit;
//   * all four warps read the accumulator back with tcgen05.ld (warp w owns
//     TMEM lanes 32w..32w+31 = tile rows), stage -D in the drained ring and
//     add it to C with one TMA reduce-add per warp (cp.reduce.async.bulk.tensor
//     .add), so no C value passes through registers and the kernel keeps few
//     registers: a panel kernel of the factorisation fits beside two of these
//     CTAs on an SM.
// Every mbarrier wait is bounded; on a timeout the kernel records DEV_TIMEOUT,
// drains its own copies, frees TMEM and returns.
#include <cuda.h>

#include <cstring>

#include "fp_internal.cuh"

namespace fpb {
namespace tc {

constexpr int BM = 128, BN = 128, BK = 16, THREADS = 128;
constexpr int TILE_A = BM * BK * 4;                 // 8 KB
constexpr int TILE_B = BN * BK * 4;                 // 8 KB
constexpr int STAGE_BYTES = 2 * TILE_A + 2 * TILE_B;
// the ring's depth: 3 stages (96 KB) for the pivoted factorisation's K = 256
// panels, 2 (64 KB, still room for the epilogue's 64 KB staging) where
// the panel kernels of the static-order factorisation must fit beside two
// of these CTAs on an SM
template <int STAGES> constexpr int smem_bytes() { return STAGES * STAGE_BYTES + 1024 + 256; }
static_assert(2 * STAGE_BYTES >= 4 * 32 * BN * 4, "the drained ring holds the epilogue's staging");
constexpr uint32_t TMEM_COLS = 128;
constexpr int kWaitLimit = 1 << 22;
// instruction descriptor: D f32 (bits 4-5 = 1), A/B tf32 (bits 7-9, 10-12 = 2),
// both K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (int i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
// K-major shared-memory matrix descriptor for BK-float (BK * 4-byte) rows
// with the matching swizzle (tile base 1024-B aligned): start address >> 4,
// LBO 16 B (unused), SBO = one 8-row swizzle atom (8 x BK * 4 bytes),
// version 1, layout 64B swizzle (4) for 64-byte rows, 128B swizzle (2) for
// 128-byte rows.
constexpr uint32_t ROW_BYTES = BK * 4;
constexpr uint32_t SWZ_LAYOUT = ROW_BYTES == 64 ? 4u : 2u;
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)((8u * ROW_BYTES) >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)SWZ_LAYOUT << 61;
  return d;
}
// C[y.., x..] += box at src (fp32 add in L2), tracked by the bulk group
__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* tm, const void* src, int x, int y) {
  asm volatile("cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(tm)),
               "r"(smem_u32(src)), "r"(x), "r"(y)
               : "memory");
}
__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  return __uint_as_float(h);
}

// kind::f16 instruction descriptor: D f32, A/B bf16 (1), both K-major, N >> 3, M >> 4
constexpr uint32_t IDESC_BF16 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                ((uint32_t)(BM >> 4) << 24);
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(IDESC_BF16), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// RED: the epilogue adds -D to C with red.global.add.f32 straight from the
// registers (lane = row, 128-byte coalesced per column; Cp / ldc address C)
// instead of staging it for a TMA reduce-add.
// BF16: BF16 operands (tmAh, tmBh only; kind::f16, one MMA per 16-deep
// step, 32-deep K blocks of 64-byte rows: 16 KB a stage).
// X3 (with BF16): each operand as a BF16 pair hi + lo, C -= Ah Bl + Al Bh +
// Ah Bh (three kind::f16 MMAs per 16-deep step, 32 KB a stage): half the
// operand bytes and MMA time of 3xTF32 a K element, 16-bit operand splits.
template <int STAGES, bool RED = false, bool BF16 = false, bool X3 = false>
__global__ void __launch_bounds__(THREADS, 2)
k_tc_gemm_sub(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
              const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBl,
              const __grid_constant__ CUtensorMap tmC, int m, int n, int K, int* __restrict__ status,
              float* __restrict__ Cp = nullptr, int64_t ldc = 0, int pf = 0) {
  constexpr int SB = BF16 ? (X3 ? 4 : 2) * TILE_A : STAGE_BYTES;   // bytes a stage
  static_assert(!X3 || BF16, "X3 splits BF16 operands");
  constexpr int KB = BF16 ? 32 : BK;                    // K elements a stage
  static_assert(RED || STAGES * SB >= 4 * 32 * BN * 4, "the drained ring holds the epilogue's staging");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * SB);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int nk = (K + KB - 1) / KB;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (RED && pf && warp >= 2) {
    // warps 2 and 3 only wait for the accumulator during the main loop:
    // meanwhile they bring the CTA's C tile into L2 (one bulk prefetch of up
    // to 512 bytes a column), so that the epilogue's reductions find it there
    const uint32_t bytes = (uint32_t)(min(BM, m - m0) * 4) & ~15u;
    if (bytes)
      for (int cc = threadIdx.x - 64; cc < BN && n0 + cc < n; cc += 64)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(Cp + (int64_t)(n0 + cc) * ldc + m0), "r"(bytes)
                     : "memory");
  }
  griddep_wait();   // the operands and C come from the stream's earlier kernels
  if (warp == 0 && lane == 0) {
    // producer
    int issued = 0;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (kb >= STAGES && !mbar_wait(&empty[s], ((kb / STAGES) - 1) & 1)) { *abort_flag = 1; break; }
      if (*(volatile int*)abort_flag) break;
      mbar_expect_tx(&full[s], SB);
      uint8_t* base = smem + s * SB;
      if (BF16 && X3) {
        tma_load_2d(base, &tmAh, kb * KB, m0, &full[s]);
        tma_load_2d(base + TILE_A, &tmAl, kb * KB, m0, &full[s]);
        tma_load_2d(base + 2 * TILE_A, &tmBh, kb * KB, n0, &full[s]);
        tma_load_2d(base + 3 * TILE_A, &tmBl, kb * KB, n0, &full[s]);
      } else if (BF16) {
        tma_load_2d(base, &tmAh, kb * KB, m0, &full[s]);
        tma_load_2d(base + TILE_A, &tmBh, kb * KB, n0, &full[s]);
      } else {
        tma_load_2d(base, &tmAh, kb * BK, m0, &full[s]);
        tma_load_2d(base + TILE_A, &tmAl, kb * BK, m0, &full[s]);
        tma_load_2d(base + 2 * TILE_A, &tmBh, kb * BK, n0, &full[s]);
        tma_load_2d(base + 2 * TILE_A + TILE_B, &tmBl, kb * BK, n0, &full[s]);
      }
      ++issued;
    }
    if (*(volatile int*)abort_flag) {
      // drain the copies this CTA issued before leaving
      for (int kb = (issued > STAGES ? issued - STAGES : 0); kb < issued; ++kb)
        mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    bool ok = true;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(&full[s], (kb / STAGES) & 1)) { ok = false; *abort_flag = 1; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(smem + s * SB);
      if (BF16 && X3) {
        const uint64_t dAh = sdesc(base), dAl = sdesc(base + TILE_A);
        const uint64_t dBh = sdesc(base + 2 * TILE_A), dBl = sdesc(base + 3 * TILE_A);
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {   // 16 bf16 = 32 bytes along K per MMA
          const uint64_t off = (uint64_t)((kk * 32) >> 4);
          umma_bf16(tmem, dAh + off, dBl + off, (kb | kk) != 0 ? 1u : 0u);
          umma_bf16(tmem, dAl + off, dBh + off, 1u);
          umma_bf16(tmem, dAh + off, dBh + off, 1u);
        }
      } else if (BF16) {
        const uint64_t dA = sdesc(base), dB = sdesc(base + TILE_A);
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {   // 16 bf16 = 32 bytes along K per MMA
          const uint64_t off = (uint64_t)((kk * 32) >> 4);
          umma_bf16(tmem, dA + off, dB + off, (kb | kk) != 0 ? 1u : 0u);
        }
      } else {
        const uint64_t dAh = sdesc(base), dAl = sdesc(base + TILE_A);
        const uint64_t dBh = sdesc(base + 2 * TILE_A), dBl = sdesc(base + 2 * TILE_A + TILE_B);
#pragma unroll
        for (int kk = 0; kk < BK / 8; ++kk) {
          const uint64_t off = (uint64_t)((kk * 32) >> 4);   // 8 tf32 = 32 bytes along K
          umma_tf32(tmem, dAh + off, dBl + off, (kb | kk) != 0 ? 1u : 0u);
          umma_tf32(tmem, dAl + off, dBh + off, 1u);
          umma_tf32(tmem, dAh + off, dBh + off, 1u);
        }
      }
      umma_commit(&empty[s]);
    }
    if (ok) umma_commit(done);
  }
  __syncwarp();
  // epilogue: every warp waits for the accumulator, stages -D for its 32 rows
  // column by column ([column][row], 32 rows = 128 B per column) in the ring,
  // whose operands the MMAs have all consumed, and adds it to C with TMA
  // warp-uniform: the epilogue's tcgen05.ld is a .sync.aligned warp instruction
  const bool ok = __all_sync(0xffffffffu, mbar_wait(done, 0));
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  griddep_launch();
  if (ok && RED) {
    const int64_t row = (int64_t)m0 + warp * 32 + lane;
    float* cp = Cp + (int64_t)n0 * ldc + row;
#pragma unroll 1
    for (int cc = 0; cc < BN; cc += 8) {
      uint32_t r[8];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cc;
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                   : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < m) {
        const int nc = n - (n0 + cc);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (j < nc) asm volatile("red.global.add.f32 [%0], %1;" ::"l"(cp), "f"(-__uint_as_float(r[j])) : "memory");
          cp += ldc;
        }
      } else {
        cp += 8 * ldc;
      }
    }
  } else if (ok) {
    float* stg = reinterpret_cast<float*>(smem) + warp * 32 * BN;
#pragma unroll 1
    for (int cc = 0; cc < BN; cc += 32) {
      uint32_t r[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cc;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
            "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) stg[(cc + j) * 32 + lane] = -__uint_as_float(r[j]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0 && m0 + warp * 32 < m) {
      tma_reduce_add_2d(&tmC, stg, m0 + warp * 32, n0);
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
      // the CTA may leave once the copy has read the staging buffer; its adds complete in L2
      asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
  } else if (threadIdx.x == 0) {
    atomicOr(status, (int)DEV_TIMEOUT);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------------------
// The same one-tile update from unsplit FP32 operands (K-major x copies of
// the L21 panel and of the U12 rows): the split into hi = rna_tf32(x) and
// lo = x - hi is done in shared memory, so a K block moves 16 KB by TMA
// instead of 32 KB and more K blocks are in flight for the same shared
// memory (XS stages of x, LB buffers of lo). 4 warps:
//   warp 0 / lane 0   TMA producer: x of A and B into stage kb % XS;
//   warps 2..3        converters: wait for the stage, write hi over x and lo
//                     into buffer kb % LB (once the MMAs that read its last
//                     contents are done), make the writes visible to the
//                     tensor core (fence.proxy.async), one arrival;
//   warp 1 / lane 0   MMA issuer: 3 x 2 tcgen05.mma (K = 8) per K block into
//                     the 128-column TMEM accumulator; one commit frees the x
//                     stage, one the lo buffer;
//   all four warps    epilogue as k_tc_gemm_sub (the drained stages and lo
//                     buffers, at least 64 KB, hold the staging).
// Bounded waits as k_tc_gemm_sub.
namespace xs {
constexpr int XBYTES = TILE_A + TILE_B;   // one K block of x (A then B)
constexpr int CT = 64;                    // converter threads
template <int XS, int LB> constexpr int smem_bytes() { return (XS + LB) * XBYTES + 1024 + 256; }
}  // namespace xs

template <int XS, int LB>
__global__ void __launch_bounds__(THREADS)
k_tc_gemm_sub_xs(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const __grid_constant__ CUtensorMap tmC, int m, int n, int K, int* __restrict__ status) {
  using namespace xs;
  static_assert((XS + LB) * XBYTES >= 4 * 32 * BN * 4, "the drained stages hold the epilogue's staging");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint8_t* lo_base = smem + XS * XBYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (XS + LB) * XBYTES);
  uint64_t* xempty = full + XS;
  uint64_t* cvt = xempty + XS;
  uint64_t* loempty = cvt + LB;
  uint64_t* done = loempty + LB;
  uint64_t* drain = done + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  volatile int* cvt_fail = abort_flag + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int nk = (K + BK - 1) / BK;

  if (threadIdx.x == 0) {
    *cvt_fail = 0;
    for (int q = 0; q < XS; ++q) { mbar_init(&full[q], 1); mbar_init(&xempty[q], 1); }
    for (int q = 0; q < LB; ++q) { mbar_init(&cvt[q], 1); mbar_init(&loempty[q], 1); }
    mbar_init(done, 1);
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {   // producer
      int issued = 0;
      for (int kb = 0; kb < nk; ++kb) {
        const int st = kb % XS;
        if (kb >= XS && !mbar_wait(&xempty[st], ((kb / XS) - 1) & 1)) { *abort_flag = 1; break; }
        if (*(volatile int*)abort_flag) break;
        mbar_expect_tx(&full[st], XBYTES);
        uint8_t* base = smem + st * XBYTES;
        tma_load_2d(base, &tmA, kb * BK, m0, &full[st]);
        tma_load_2d(base + TILE_A, &tmB, kb * BK, n0, &full[st]);
        issued = kb + 1;
      }
      if (*(volatile int*)abort_flag)   // drain the copies this CTA issued before leaving
        for (int kb = (issued > XS ? issued - XS : 0); kb < issued; ++kb) mbar_wait(&full[kb % XS], (kb / XS) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {   // MMA issuer
      int issued = 0;
      bool ok = true;
      for (int kb = 0; kb < nk; ++kb) {
        const int st = kb % XS, b = kb % LB;
        if (!mbar_wait(&cvt[b], (kb / LB) & 1)) { ok = false; *abort_flag = 1; break; }
        if (*(volatile int*)abort_flag) { ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t xb = smem_u32(smem + st * XBYTES), lb = smem_u32(lo_base + b * XBYTES);
        const uint64_t dAh = sdesc(xb), dBh = sdesc(xb + TILE_A);
        const uint64_t dAl = sdesc(lb), dBl = sdesc(lb + TILE_A);
#pragma unroll
        for (int kk = 0; kk < BK / 8; ++kk) {
          const uint64_t off = (uint64_t)((kk * 32) >> 4);   // 8 tf32 = 32 bytes along K
          umma_tf32(tmem, dAh + off, dBl + off, (kb | kk) != 0 ? 1u : 0u);
          umma_tf32(tmem, dAl + off, dBh + off, 1u);
          umma_tf32(tmem, dAh + off, dBh + off, 1u);
        }
        umma_commit(&xempty[st]);
        umma_commit(&loempty[b]);
        issued = kb + 1;
      }
      if (ok) umma_commit(done);
      else if (issued > 0) {   // MMAs still in flight must finish before TMEM is freed
        umma_commit(drain);
        mbar_wait(drain, 0);
      }
    }
  } else {   // converters
    // every converter thread reaches both named barriers of every K block:
    // failures are written before the first, read between the two, so the
    // 64 threads leave the loop together
    const int ct = threadIdx.x - 64;
    for (int kb = 0; kb < nk; ++kb) {
      const int st = kb % XS, b = kb % LB;
      bool ok = mbar_wait(&full[st], (kb / XS) & 1);
      if (ok && kb >= LB) ok = mbar_wait(&loempty[b], ((kb / LB) - 1) & 1);
      if (!ok) { *cvt_fail = 1; *(volatile int*)abort_flag = 1; }
      asm volatile("bar.sync 1, %0;" ::"n"(CT) : "memory");
      const int stop = *cvt_fail;
      asm volatile("bar.sync 1, %0;" ::"n"(CT) : "memory");
      if (stop) break;
      float4* x = reinterpret_cast<float4*>(smem + st * XBYTES);
      float4* lo = reinterpret_cast<float4*>(lo_base + b * XBYTES);
#pragma unroll 4
      for (int q = ct; q < XBYTES / 16; q += CT) {
        const float4 v = x[q];
        const float4 h = make_float4(tf32_rna(v.x), tf32_rna(v.y), tf32_rna(v.z), tf32_rna(v.w));
        x[q] = h;
        lo[q] = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("bar.sync 1, %0;" ::"n"(CT) : "memory");
      if (ct == 0) mbar_arrive(&cvt[b]);
    }
  }
  __syncwarp();
  // warp-uniform: the epilogue's tcgen05.ld is a .sync.aligned warp instruction
  const bool ok = __all_sync(0xffffffffu, !*(volatile int*)abort_flag && mbar_wait(done, 0));
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    float* stg = reinterpret_cast<float*>(smem) + warp * 32 * BN;
#pragma unroll 1
    for (int cc = 0; cc < BN; cc += 32) {
      uint32_t r[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cc;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
            "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) stg[(cc + j) * 32 + lane] = -__uint_as_float(r[j]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0 && m0 + warp * 32 < m) {
      tma_reduce_add_2d(&tmC, stg, m0 + warp * 32, n0);
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
      asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
  } else if (threadIdx.x == 0) {
    atomicOr(status, (int)DEV_TIMEOUT);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------------------
// The same update with several output tiles per CTA and the accumulator
// double-buffered in TMEM (2 x 128 columns), so that the epilogue of one tile
// overlaps the MMAs of the next. Warp-specialised, 192 threads:
//   warp 0 / lane 0   TMA producer: 16-wide K blocks of Ah, Al, Bh, Bl into a
//                     3-stage ring (full / empty mbarriers);
//   warp 1 / lane 0   MMA issuer: 3 x 2 tcgen05.mma per K block into
//                     accumulator t & 1 (after the epilogue has released it),
//                     tcgen05.commit frees each stage and, after a tile's
//                     last block, marks the accumulator full;
//   warps 2..5        epilogue: warp w reads TMEM lanes 32 (w % 4).., i.e.
//                     the tile's rows 32 (w % 4).., 32 columns at a time,
//                     stages -D in one of two 4 KB buffers and adds it to C
//                     by a TMA reduce-add of a 32 x 32 box (the buffer is
//                     reused once the bulk copy two boxes back has read it),
//                     then releases the accumulator.
// A CTA takes tiles_per_cta consecutive tiles (columns fastest within a row
// of tiles), so CTAs still retire during a long update and the panel kernels
// of the other stream get SMs. 128 KB of shared memory. Bounded waits as in
// k_tc_gemm_sub: on a timeout the kernel records DEV_TIMEOUT, each role
// stops, drains what it issued and the TMEM is freed.
// With BF16 operands (kind::f16, one MMA per 16-deep step, no lo parts) a
// K block is 32 elements (the same 64-byte rows) and a stage holds Ah and Bh.
namespace mt {
constexpr int STAGES = 3, THREADS = 192;
constexpr int STG_BYTES = 32 * 32 * 4;   // one epilogue box
template <bool BF16> __host__ __device__ constexpr int stage_bytes() { return BF16 ? 2 * BM * 64 : STAGE_BYTES; }
template <bool BF16> __host__ __device__ constexpr int kblock() { return BF16 ? 32 : BK; }
template <bool BF16> __host__ __device__ constexpr int smem() { return STAGES * stage_bytes<BF16>() + 4 * 2 * STG_BYTES + 1024 + 256; }
constexpr uint32_t TMEM_COLS = 2 * BN;
}  // namespace mt



template <bool BF16, bool RED = false>
__global__ void __launch_bounds__(mt::THREADS, 1)
k_tc_gemm_multi(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
                const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBl,
                const __grid_constant__ CUtensorMap tmC, int m, int n, int K, int tiles_per_cta,
                int* __restrict__ status, float* __restrict__ Cp = nullptr, int64_t ldc = 0) {
  using namespace mt;
  constexpr int SB = stage_bytes<BF16>(), KB = kblock<BF16>();
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  float* stage_out = reinterpret_cast<float*>(smem + STAGES * SB);   // [4 warps][2][32 x 32]
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * SB + 4 * 2 * STG_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* accf = empty + STAGES;
  uint64_t* acce = accf + 2;
  uint64_t* drain = acce + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (K + KB - 1) / KB;
  const int mt_ = (m + BM - 1) / BM, nt_ = (n + BN - 1) / BN;
  const int ntiles = mt_ * nt_;
  const int t0 = blockIdx.x * tiles_per_cta;
  const int t1 = min(ntiles, t0 + tiles_per_cta);
  auto tile_mn = [&](int t, int& m0, int& n0) {   // columns fastest: a CTA's tiles share their rows of A
    m0 = (t / nt_) * BM;
    n0 = (t % nt_) * BN;
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    for (int b = 0; b < 2; ++b) { mbar_init(&accf[b], 1); mbar_init(&acce[b], 4); }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(mt::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {   // producer
      int it = 0, issued = 0;
      for (int t = t0; t < t1 && !*(volatile int*)abort_flag; ++t) {
        int m0, n0;
        tile_mn(t, m0, n0);
        for (int kb = 0; kb < nk; ++kb, ++it) {
          const int s = it % STAGES;
          if (it >= STAGES && !mbar_wait(&empty[s], ((it / STAGES) - 1) & 1)) { *abort_flag = 1; break; }
          if (*(volatile int*)abort_flag) break;
          mbar_expect_tx(&full[s], SB);
          uint8_t* base = smem + s * SB;
          if (BF16) {
            tma_load_2d(base, &tmAh, kb * KB, m0, &full[s]);
            tma_load_2d(base + SB / 2, &tmBh, kb * KB, n0, &full[s]);
          } else {
            tma_load_2d(base, &tmAh, kb * BK, m0, &full[s]);
            tma_load_2d(base + TILE_A, &tmAl, kb * BK, m0, &full[s]);
            tma_load_2d(base + 2 * TILE_A, &tmBh, kb * BK, n0, &full[s]);
            tma_load_2d(base + 2 * TILE_A + TILE_B, &tmBl, kb * BK, n0, &full[s]);
          }
          issued = it + 1;
        }
      }
      if (*(volatile int*)abort_flag)   // drain the copies this CTA issued before leaving
        for (int q = (issued > STAGES ? issued - STAGES : 0); q < issued; ++q)
          mbar_wait(&full[q % STAGES], (q / STAGES) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {   // MMA issuer
      int it = 0, u = 0;
      for (int t = t0; t < t1 && !*(volatile int*)abort_flag; ++t, ++u) {
        const int b = u & 1;
        if (u >= 2 && !mbar_wait(&acce[b], ((u >> 1) - 1) & 1)) { *abort_flag = 1; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(b * BN);
        bool ok = true;
        for (int kb = 0; kb < nk; ++kb, ++it) {
          const int s = it % STAGES;
          if (!mbar_wait(&full[s], (it / STAGES) & 1)) { ok = false; *abort_flag = 1; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t base = smem_u32(smem + s * SB);
          if (BF16) {
            const uint64_t dA = sdesc(base), dB = sdesc(base + SB / 2);
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {   // 16 bf16 = 32 bytes along K per MMA
              const uint64_t off = (uint64_t)((kk * 32) >> 4);
              umma_bf16(acc, dA + off, dB + off, (kb | kk) != 0 ? 1u : 0u);
            }
          } else {
            const uint64_t dAh = sdesc(base), dAl = sdesc(base + TILE_A);
            const uint64_t dBh = sdesc(base + 2 * TILE_A), dBl = sdesc(base + 2 * TILE_A + TILE_B);
#pragma unroll
            for (int kk = 0; kk < BK / 8; ++kk) {
              const uint64_t off = (uint64_t)((kk * 32) >> 4);   // 8 tf32 = 32 bytes along K
              umma_tf32(acc, dAh + off, dBl + off, (kb | kk) != 0 ? 1u : 0u);
              umma_tf32(acc, dAl + off, dBh + off, 1u);
              umma_tf32(acc, dAh + off, dBh + off, 1u);
            }
          }
          umma_commit(&empty[s]);
        }
        if (!ok) break;
        umma_commit(&accf[b]);
      }
      if (*(volatile int*)abort_flag && it > 0) {   // MMAs still in flight must finish before TMEM is freed
        umma_commit(drain);
        mbar_wait(drain, 0);
      }
    }
  } else {   // epilogue warps 2..5
    const int q = warp & 3;   // TMEM lanes 32 q .. 32 q + 31 = tile rows
    float* stg0 = stage_out + (size_t)(warp - 2) * 2 * (STG_BYTES / 4);
    int u = 0, sb = 0;
    bool ok = true;
    for (int t = t0; t < t1 && ok; ++t, ++u) {
      const int b = u & 1;
      int m0, n0;
      tile_mn(t, m0, n0);
      // warp-uniform: tcgen05.ld is a .sync.aligned warp instruction
      if (!__all_sync(0xffffffffu, mbar_wait(&accf[b], (u >> 1) & 1))) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (RED) {   // -D added to C with red.global straight from the registers (lane = row)
        const int64_t row = (int64_t)m0 + q * 32 + lane;
        float* cp = Cp + (int64_t)n0 * ldc + row;
#pragma unroll 1
        for (int cc = 0; cc < BN; cc += 8) {
          uint32_t r[8];
          const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + cc);
          asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                       : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                         "=r"(r[7])
                       : "r"(taddr));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (row < m) {
            const int nc = n - (n0 + cc);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              if (j < nc) asm volatile("red.global.add.f32 [%0], %1;" ::"l"(cp), "f"(-__uint_as_float(r[j])) : "memory");
              cp += ldc;
            }
          } else {
            cp += 8 * ldc;
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&acce[b]);
        continue;
      }
#pragma unroll 1
      for (int cc = 0; cc < BN; cc += 32) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + cc);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        // the bulk copy that last read this staging buffer (two boxes back) is done
        if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
        __syncwarp();
        float* stg = stg0 + sb * (STG_BYTES / 4);
#pragma unroll
        for (int j = 0; j < 32; ++j) stg[j * 32 + lane] = -__uint_as_float(r[j]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          if (m0 + q * 32 < m && n0 + cc < n) tma_reduce_add_2d(&tmC, stg, m0 + q * 32, n0 + cc);
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
        sb ^= 1;
      }
      // every TMEM read of this accumulator has completed: release it to the MMA warp
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[b]);
    }
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    if (!ok && lane == 0) { *(volatile int*)abort_flag = 1; }
  }
  __syncwarp();
  if (threadIdx.x == 0 && *(volatile int*)abort_flag) atomicOr(status, (int)DEV_TIMEOUT);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(mt::TMEM_COLS) : "memory");
}


// L21 panel (m x K, column-major, lda) -> K-major copies Ah, Al (m x ldk, row-major).
__global__ void k_split_A(const float* __restrict__ A, int64_t lda, int m, int K, int ldk,
                          float* __restrict__ Ah, float* __restrict__ Al) {
  __shared__ float t[32][33];
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8
  for (int j = ty; j < 32; j += 8) {
    const int i = i0 + tx, k = k0 + j;
    t[j][tx] = (i < m && k < K) ? A[(int64_t)k * lda + i] : 0.f;
  }
  __syncthreads();
  for (int j = ty; j < 32; j += 8) {
    const int i = i0 + j, k = k0 + tx;
    if (i < m && k < ldk) {
      const float v = t[tx][j];
      const float h = tf32_rna(v);
      Ah[(int64_t)i * ldk + k] = h;
      Al[(int64_t)i * ldk + k] = v - h;
    }
  }
}

// U12 panel (K x n, column-major, lda) -> Bh, Bl (K x n, column-major, ldk).
__global__ void k_split_B(const float* __restrict__ B, int64_t lda, int K, int n, int ldk,
                          float* __restrict__ Bh, float* __restrict__ Bl) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)ldk * n) return;
  const int k = (int)(t % ldk);
  const int64_t j = t / ldk;
  const float v = (k < K) ? B[j * lda + k] : 0.f;
  const float h = tf32_rna(v);
  Bh[t] = h;
  Bl[t] = v - h;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn resolve_encode_fn() {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    return reinterpret_cast<EncodeTiledFn>(p);
  return nullptr;
}
static EncodeTiledFn encode_fn() {
  static const EncodeTiledFn fn = resolve_encode_fn();   // initialised once, thread-safe
  return fn;
}

// 2-D fp32 map over a K-major matrix: inner dim K (extent kext, row pitch ldk
// floats), outer dim rows; box BK x box_rows, swizzle of BK * 4-byte rows,
// zero fill.
static bool make_map(CUtensorMap* tm, const float* base, int kext, int64_t rows, int ldk, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kext, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ldk * 4};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, ROW_BYTES == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2-D fp32 map over the column-major block C (m rows x n columns, column
// pitch ldc floats) for the epilogue's reduce-add: inner dim the rows, box
// 32 rows x box_cols columns, no swizzle.
static bool make_map_c(CUtensorMap* tm, float* C, int64_t m, int64_t n, int64_t ldc, int box_cols = BN) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)n};
  cuuint64_t strides[1] = {(cuuint64_t)ldc * 4};
  cuuint32_t box[2] = {32u, (cuuint32_t)box_cols};
  cuuint32_t es[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace tc

// Scratch for the split operands: 4 x N x kOuterPanel floats.
int ensure_tc_scratch(fp_ctx* c, int slot, int64_t rows_max) {
  const size_t need = (size_t)rows_max * kOuterPanel;
  if (c->tc_cap[slot] >= need) return FP_OK;
  for (int i = 0; i < 4; ++i) {
    if (c->d_tc[slot][i]) cudaFree(c->d_tc[slot][i]);
    c->d_tc[slot][i] = nullptr;
  }
  c->tc_cap[slot] = 0;
  for (int i = 0; i < 4; ++i) FP_CUDA_TRY(c->err, cudaMalloc(&c->d_tc[slot][i], need * sizeof(float)));
  c->tc_cap[slot] = need;
  return FP_OK;
}

bool tc_gemm_sub_f32(fp_ctx* c, const float* A, const float* B, float* C, int64_t lda, int64_t m,
                     int64_t nn, int kk) {
  if (!c->use_tc || kk <= 0 || kk > kOuterPanel || m <= 0 || nn <= 0) return false;
  if (!tc::encode_fn()) return false;
  // the reduce-add needs a 16-byte aligned C and column pitch
  if (((reinterpret_cast<uintptr_t>(C) | (uintptr_t)(lda * 4)) & 15) != 0) return false;
  static SmemAttr attr;
  if (attr.ensure(tc::k_tc_gemm_sub<3>, kTcSmemMax) != cudaSuccess) return false;
  const int slot = c->tc_slot;
  if (ensure_tc_scratch(c, slot, std::max<int64_t>(m, nn)) != FP_OK) return false;
  const int ldk = (int)round_up(kk, 32);
  float *Ah = c->d_tc[slot][0], *Al = c->d_tc[slot][1], *Bh = c->d_tc[slot][2], *Bl = c->d_tc[slot][3];
  {
    dim3 g((unsigned)((m + 31) / 32), (unsigned)((ldk + 31) / 32));
    {
      TraceScope tr(c, TR_SPLIT_A);
      tc::k_split_A<<<g, dim3(32, 8), 0, c->stream>>>(A, lda, (int)m, kk, ldk, Ah, Al);
    }
    ++c->nlaunch;
    const int64_t t = (int64_t)ldk * nn;
    {
      TraceScope tr(c, TR_SPLIT_B);
      tc::k_split_B<<<(unsigned)((t + 255) / 256), 256, 0, c->stream>>>(B, lda, kk, (int)nn, ldk, Bh, Bl);
    }
    ++c->nlaunch;
  }
  CUtensorMap mAh, mAl, mBh, mBl, mC;
  if (!tc::make_map(&mAh, Ah, kk, m, ldk, tc::BM) || !tc::make_map(&mAl, Al, kk, m, ldk, tc::BM) ||
      !tc::make_map(&mBh, Bh, kk, nn, ldk, tc::BN) || !tc::make_map(&mBl, Bl, kk, nn, ldk, tc::BN) ||
      !tc::make_map_c(&mC, C, m, nn, lda))
    return false;
  dim3 grid((unsigned)((m + tc::BM - 1) / tc::BM), (unsigned)((nn + tc::BN - 1) / tc::BN));
  const int ev = kt_begin(c);
  TraceScope tr(c, TR_GEMM_TC);
  tc::k_tc_gemm_sub<3><<<grid, tc::THREADS, tc::smem_bytes<3>(), c->stream>>>(mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk,
                                                                       c->d_status);
  kt_end(c, ev, 2.0 * (double)m * (double)nn * (double)kk, (double)m * (double)nn);
  ++c->nlaunch;
  return cudaGetLastError() == cudaSuccess;
}

bool tc_gemm_sub_presplit(fp_ctx* c, const float* Ah, const float* Al, const float* Bh, const float* Bl, int ldk,
                          float* C, int64_t ldc, int64_t m, int64_t nn, int kk) {
  if (kk <= 0 || kk > ldk || m <= 0 || nn <= 0 || (ldk & 3) != 0) return false;
  if (!tc::encode_fn()) return false;
  // TMA: 16-byte aligned bases and pitches
  if (((reinterpret_cast<uintptr_t>(C) | (uintptr_t)(ldc * 4) | reinterpret_cast<uintptr_t>(Ah) |
        reinterpret_cast<uintptr_t>(Al) | reinterpret_cast<uintptr_t>(Bh) | reinterpret_cast<uintptr_t>(Bl)) &
       15) != 0)
    return false;
  static SmemAttr attr2, attr3, attrm, attr2r, attr3r, attr6r, attrmr;
  if (attr3r.ensure(tc::k_tc_gemm_sub<3, true>, kTcSmemMax) != cudaSuccess) return false;
  if (attr6r.ensure(tc::k_tc_gemm_sub<6, true>, kTcSmemMax) != cudaSuccess) return false;
  if (attrmr.ensure(tc::k_tc_gemm_multi<false, true>, tc::mt::smem<false>()) != cudaSuccess) return false;
  if (attr2.ensure(tc::k_tc_gemm_sub<2>, kTcSmemMax) != cudaSuccess) return false;
  if (attr3.ensure(tc::k_tc_gemm_sub<3>, kTcSmemMax) != cudaSuccess) return false;
  if (attr2r.ensure(tc::k_tc_gemm_sub<2, true>, kTcSmemMax) != cudaSuccess) return false;
  if (attrm.ensure(tc::k_tc_gemm_multi<false>, tc::mt::smem<false>()) != cudaSuccess) return false;
  const bool multi = c->tc_tiles > 0;
  CUtensorMap mAh, mAl, mBh, mBl, mC;
  if (!tc::make_map(&mAh, Ah, kk, m, ldk, tc::BM) || !tc::make_map(&mAl, Al, kk, m, ldk, tc::BM) ||
      !tc::make_map(&mBh, Bh, kk, nn, ldk, tc::BN) || !tc::make_map(&mBl, Bl, kk, nn, ldk, tc::BN) ||
      !tc::make_map_c(&mC, C, m, nn, ldc, multi ? 32 : tc::BN))
    return false;
  dim3 grid((unsigned)((m + tc::BM - 1) / tc::BM), (unsigned)((nn + tc::BN - 1) / tc::BN));
  const int ev = kt_begin(c);
  TraceScope tr(c, TR_GEMM_TC);
  if (multi) {
    const int tiles = (int)(grid.x * grid.y);
    const unsigned ctas = (unsigned)((tiles + c->tc_tiles - 1) / c->tc_tiles);
    if (c->tc_red)
      tc::k_tc_gemm_multi<false, true><<<ctas, tc::mt::THREADS, tc::mt::smem<false>(), c->stream>>>(
          mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk, c->tc_tiles, c->d_status, C, ldc);
    else
      tc::k_tc_gemm_multi<false><<<ctas, tc::mt::THREADS, tc::mt::smem<false>(), c->stream>>>(
          mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk, c->tc_tiles, c->d_status);
  } else if (c->tc_red && c->tc_narrow_stages == 6 && grid.y == 1 && (int)grid.x <= num_sms())
    // one column of tiles (the next panel's update, on the factorisation's
    // critical path): at most one CTA an SM, so a 6-stage ring costs no
    // occupancy and puts 6 of the 8 K blocks in flight at once
    tc::k_tc_gemm_sub<6, true><<<grid, tc::THREADS, tc::smem_bytes<6>(), c->stream>>>(
        mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk, c->d_status, C, ldc, c->tc_prefetch);
  else if (c->tc_red && c->tc_stages == 3)
    tc::k_tc_gemm_sub<3, true><<<grid, tc::THREADS, std::max(tc::smem_bytes<3>(), c->tc_smem), c->stream>>>(
        mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk, c->d_status, C, ldc, c->tc_prefetch);
  else if (c->tc_red)
    tc::k_tc_gemm_sub<2, true><<<grid, tc::THREADS, std::max(tc::smem_bytes<2>(), c->tc_smem), c->stream>>>(
        mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk, c->d_status, C, ldc, c->tc_prefetch);
  else if (c->tc_stages == 2)
    tc::k_tc_gemm_sub<2><<<grid, tc::THREADS, std::max(tc::smem_bytes<2>(), c->tc_smem), c->stream>>>(
        mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk, c->d_status);
  else
    tc::k_tc_gemm_sub<3><<<grid, tc::THREADS, std::max(tc::smem_bytes<3>(), c->tc_smem), c->stream>>>(
        mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk, c->d_status);
  kt_end(c, ev, 2.0 * (double)m * (double)nn * (double)kk, (double)m * (double)nn);
  ++c->nlaunch;
  return cudaGetLastError() == cudaSuccess;
}

// C -= A B from unsplit FP32 operands (K-major, ldk floats a row), the split
// done in shared memory by k_tc_gemm_sub_xs (x stages by c->tc_split: 1 -> 3,
// 2 -> 4, 3 -> 6; one lo buffer).
bool tc_gemm_sub_xsplit(fp_ctx* c, const float* Ax, const float* Bx, int ldk, float* C, int64_t ldc, int64_t m,
                        int64_t nn, int kk) {
  if (kk <= 0 || kk > ldk || m <= 0 || nn <= 0 || (ldk & 3) != 0) return false;
  if (!tc::encode_fn()) return false;
  if (((reinterpret_cast<uintptr_t>(C) | (uintptr_t)(ldc * 4) | reinterpret_cast<uintptr_t>(Ax) |
        reinterpret_cast<uintptr_t>(Bx)) & 15) != 0)
    return false;
  static SmemAttr a3, a4, a6;
  if (a3.ensure(tc::k_tc_gemm_sub_xs<3, 1>, kTcSmemMax) != cudaSuccess) return false;
  if (a4.ensure(tc::k_tc_gemm_sub_xs<4, 1>, kTcSmemMax) != cudaSuccess) return false;
  if (a6.ensure(tc::k_tc_gemm_sub_xs<6, 1>, kTcSmemMax) != cudaSuccess) return false;
  CUtensorMap mA, mB, mC;
  if (!tc::make_map(&mA, Ax, kk, m, ldk, tc::BM) || !tc::make_map(&mB, Bx, kk, nn, ldk, tc::BN) ||
      !tc::make_map_c(&mC, C, m, nn, ldc, tc::BN))
    return false;
  dim3 grid((unsigned)((m + tc::BM - 1) / tc::BM), (unsigned)((nn + tc::BN - 1) / tc::BN));
  const int ev = kt_begin(c);
  TraceScope tr(c, TR_GEMM_TC);
  if (c->tc_split >= 3)
    tc::k_tc_gemm_sub_xs<6, 1><<<grid, tc::THREADS, std::max(tc::xs::smem_bytes<6, 1>(), c->tc_smem), c->stream>>>(
        mA, mB, mC, (int)m, (int)nn, kk, c->d_status);
  else if (c->tc_split == 2)
    tc::k_tc_gemm_sub_xs<4, 1><<<grid, tc::THREADS, std::max(tc::xs::smem_bytes<4, 1>(), c->tc_smem), c->stream>>>(
        mA, mB, mC, (int)m, (int)nn, kk, c->d_status);
  else
    tc::k_tc_gemm_sub_xs<3, 1><<<grid, tc::THREADS, std::max(tc::xs::smem_bytes<3, 1>(), c->tc_smem), c->stream>>>(
        mA, mB, mC, (int)m, (int)nn, kk, c->d_status);
  kt_end(c, ev, 2.0 * (double)m * (double)nn * (double)kk, (double)m * (double)nn);
  ++c->nlaunch;
  return cudaGetLastError() == cudaSuccess;
}

// C -= A B from BF16 pairs (Ah + Al: m rows, Bh + Bl: nn columns, K-major
// with ldk bf16 elements a row; kk <= ldk): three kind::f16 MMAs a 16-deep
// step, red.global epilogue; the update of one column of tiles (at most one
// CTA an SM) uses a 6-stage ring, the others 2 stages (two CTAs an SM).
bool tc_gemm_sub_bf16x3(fp_ctx* c, const void* Ah, const void* Al, const void* Bh, const void* Bl, int ldk, float* C,
                        int64_t ldc, int64_t m, int64_t nn, int kk) {
  if (kk <= 0 || kk > ldk || m <= 0 || nn <= 0 || (ldk & 7) != 0) return false;
  if (!tc::encode_fn()) return false;
  if (((reinterpret_cast<uintptr_t>(C) | (uintptr_t)(ldc * 4) | reinterpret_cast<uintptr_t>(Ah) |
        reinterpret_cast<uintptr_t>(Al) | reinterpret_cast<uintptr_t>(Bh) | reinterpret_cast<uintptr_t>(Bl)) &
       15) != 0)
    return false;
  static SmemAttr a2, a6;
  if (a2.ensure(tc::k_tc_gemm_sub<2, true, true, true>, kTcSmemMax) != cudaSuccess) return false;
  if (a6.ensure(tc::k_tc_gemm_sub<6, true, true, true>, kTcSmemMax) != cudaSuccess) return false;
  auto map16 = [&](CUtensorMap* tm, const void* base, int64_t rows) {
    cuuint64_t dims[2] = {(cuuint64_t)kk, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ldk * 2};
    cuuint32_t box[2] = {32u, (cuuint32_t)tc::BM};
    cuuint32_t es[2] = {1, 1};
    return tc::encode_fn()(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  CUtensorMap mAh, mAl, mBh, mBl, mC;
  if (!map16(&mAh, Ah, m) || !map16(&mAl, Al, m) || !map16(&mBh, Bh, nn) || !map16(&mBl, Bl, nn) ||
      !tc::make_map_c(&mC, C, m, nn, ldc, 32))
    return false;
  dim3 grid((unsigned)((m + tc::BM - 1) / tc::BM), (unsigned)((nn + tc::BN - 1) / tc::BN));
  const int ev = kt_begin(c);
  TraceScope tr(c, TR_GEMM_TC);
  if (c->tc_narrow_stages == 6 && grid.y == 1 && (int)grid.x <= num_sms())
    launch_k(c->pdl, tc::k_tc_gemm_sub<6, true, true, true>, grid, dim3(tc::THREADS), tc::smem_bytes<6>(), c->stream,
             mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk, c->d_status, C, ldc, c->tc_prefetch);
  else
    launch_k(c->pdl, tc::k_tc_gemm_sub<2, true, true, true>, grid, dim3(tc::THREADS),
             std::max(tc::smem_bytes<2>(), c->tc_smem), c->stream, mAh, mAl, mBh, mBl, mC, (int)m, (int)nn, kk,
             c->d_status, C, ldc, c->tc_prefetch);
  kt_end(c, ev, 2.0 * (double)m * (double)nn * (double)kk, (double)m * (double)nn);
  ++c->nlaunch;
  return cudaGetLastError() == cudaSuccess;
}

// C -= A B from BF16 operands (Ah: m rows, Bh: nn columns, K-major with ldk
// elements a row), FP32 accumulation, on the multi-tile kernel.
bool tc_gemm_sub_bf16(fp_ctx* c, const void* Ah, const void* Bh, int ldk, float* C, int64_t ldc, int64_t m,
                      int64_t nn, int kk) {
  if (kk <= 0 || kk > ldk || m <= 0 || nn <= 0 || (ldk & 7) != 0) return false;
  if (!tc::encode_fn()) return false;
  if (((reinterpret_cast<uintptr_t>(C) | (uintptr_t)(ldc * 4) | reinterpret_cast<uintptr_t>(Ah) |
        reinterpret_cast<uintptr_t>(Bh)) & 15) != 0)
    return false;
  static SmemAttr attr, attr1;
  if (attr.ensure(tc::k_tc_gemm_multi<true>, tc::mt::smem<true>()) != cudaSuccess) return false;
  if (attr1.ensure(tc::k_tc_gemm_sub<4, true, true>, kTcSmemMax) != cudaSuccess) return false;
  auto map16 = [&](CUtensorMap* tm, const void* base, int64_t rows) {
    cuuint64_t dims[2] = {(cuuint64_t)kk, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ldk * 2};
    cuuint32_t box[2] = {32u, (cuuint32_t)tc::BM};
    cuuint32_t es[2] = {1, 1};
    return tc::encode_fn()(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  CUtensorMap mA, mB, mC;
  if (!map16(&mA, Ah, m) || !map16(&mB, Bh, nn) || !tc::make_map_c(&mC, C, m, nn, ldc, 32)) return false;
  const int tiles = (int)(((m + tc::BM - 1) / tc::BM) * ((nn + tc::BN - 1) / tc::BN));
  const int ev = kt_begin(c);
  TraceScope tr(c, TR_GEMM_TC);
  if (c->tc_red && c->tc_tiles == 0) {
    // one tile a CTA, 4-stage ring of 16 KB stages, red.global epilogue
    dim3 grid((unsigned)((m + tc::BM - 1) / tc::BM), (unsigned)((nn + tc::BN - 1) / tc::BN));
    constexpr int sb = 4 * 2 * tc::TILE_A + 1024 + 256;
    tc::k_tc_gemm_sub<4, true, true><<<grid, tc::THREADS, std::max(sb, c->tc_smem), c->stream>>>(
        mA, mA, mB, mB, mC, (int)m, (int)nn, kk, c->d_status, C, ldc, c->tc_prefetch);
  } else {
    const int tpc = c->tc_tiles > 0 ? c->tc_tiles : 4;
    tc::k_tc_gemm_multi<true><<<(unsigned)((tiles + tpc - 1) / tpc), tc::mt::THREADS, tc::mt::smem<true>(),
                                c->stream>>>(mA, mA, mB, mB, mC, (int)m, (int)nn, kk, tpc, c->d_status);
  }
  kt_end(c, ev, 2.0 * (double)m * (double)nn * (double)kk, (double)m * (double)nn);
  ++c->nlaunch;
  return cudaGetLastError() == cudaSuccess;
}

// ---------------------------------------------------------------------------
// Self-test: C0 - A B for random A (m x k), B (k x n), C0 (m x n) by the
// tensor-core kernel, by the SIMT kernel and in FP64; errors relative to
// k * max|a| * max|b| (= k).
__global__ void k_fill_rand(float* a, int64_t n, uint32_t seed) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t h = (uint32_t)t * 2654435761u ^ seed;
  h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
  a[t] = (float)((double)h / 4294967296.0 * 2.0 - 1.0);
}
__global__ void k_ref_f64(const float* A, const float* B, const float* C0, double* R, int64_t ld, int m, int n,
                          int k) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)m * n) return;
  const int i = (int)(t % m), j = (int)(t / m);
  double s = C0[(int64_t)j * ld + i];
  for (int l = 0; l < k; ++l) s -= (double)A[(int64_t)l * ld + i] * (double)B[(int64_t)j * ld + l];
  R[(int64_t)j * m + i] = s;
}
__global__ void k_maxerr(const float* C, const double* R, int64_t ld, int m, int n, unsigned long long* out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)m * n) return;
  const int i = (int)(t % m), j = (int)(t / m);
  const double e = fabs((double)C[(int64_t)j * ld + i] - R[(int64_t)j * m + i]);
  atomicMax(out, (unsigned long long)__double_as_longlong(e));
}

int gemm_sub_simt_f32(fp_ctx* c, const float* A, const float* B, float* C, int64_t lda, int64_t m, int64_t nn,
                      int kk);

}  // namespace fpb

extern "C" int fp_tc_selftest(int device, int64_t m, int64_t n, int k, double* err_tc, double* err_simt,
                              double* ms_tc) {
  using namespace fpb;
  if (m <= 0 || n <= 0 || k <= 0 || k > kOuterPanel || !err_tc || !err_simt || !ms_tc) return FP_EINVAL;
  fp_ctx* c = nullptr;
  if (int rc = fp_ctx_create(device, &c)) return rc;
  const int64_t ld = round_up(std::max<int64_t>(m, k), 64);
  const int64_t cols = std::max<int64_t>(n, k);
  float *A = nullptr, *B = nullptr, *C1 = nullptr, *C2 = nullptr;
  double* R = nullptr;
  unsigned long long* e = nullptr;
  int rc = FP_OK;
  auto fail = [&](int code) { rc = code; };
  if (cudaMalloc(&A, ld * cols * 4) || cudaMalloc(&B, ld * cols * 4) || cudaMalloc(&C1, ld * cols * 4) ||
      cudaMalloc(&C2, ld * cols * 4) || cudaMalloc(&R, m * n * 8) || cudaMalloc(&e, 16)) {
    fail(FP_ECUDA);
  } else {
    const int64_t tot = ld * cols;
    const unsigned g = (unsigned)((tot + 255) / 256);
    k_fill_rand<<<g, 256, 0, c->stream>>>(A, tot, 1u);
    k_fill_rand<<<g, 256, 0, c->stream>>>(B, tot, 2u);
    k_fill_rand<<<g, 256, 0, c->stream>>>(C1, tot, 3u);
    cudaMemcpyAsync(C2, C1, tot * 4, cudaMemcpyDeviceToDevice, c->stream);
    const unsigned gr = (unsigned)((m * n + 255) / 256);
    k_ref_f64<<<gr, 256, 0, c->stream>>>(A, B, C1, R, ld, (int)m, (int)n, k);
    cudaEventRecord(c->ev0, c->stream);
    const bool used = tc_gemm_sub_f32(c, A, B, C1, ld, m, n, k);
    cudaEventRecord(c->ev1, c->stream);
    if (!used) fail(FP_EINVAL);
    if (gemm_sub_simt_f32(c, A, B, C2, ld, m, n, k)) fail(FP_ECUDA);
    double h[2] = {0, 0};
    for (int w = 0; w < 2; ++w) {
      cudaMemsetAsync(e, 0, 8, c->stream);
      k_maxerr<<<gr, 256, 0, c->stream>>>(w == 0 ? C1 : C2, R, ld, (int)m, (int)n, e);
      unsigned long long v = 0;
      cudaMemcpyAsync(&v, e, 8, cudaMemcpyDeviceToHost, c->stream);
      cudaStreamSynchronize(c->stream);
      double d;
      std::memcpy(&d, &v, 8);
      h[w] = d / k;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    *err_tc = h[0];
    *err_simt = h[1];
    *ms_tc = ms;
    int st = 0;
    cudaMemcpy(&st, c->d_status, 4, cudaMemcpyDeviceToHost);
    if (st & DEV_TIMEOUT) fail(FP_ETIMEOUT);
    if (cudaGetLastError() != cudaSuccess) fail(FP_ECUDA);
  }
  cudaFree(A); cudaFree(B); cudaFree(C1); cudaFree(C2); cudaFree(R); cudaFree(e);
  fp_ctx_destroy(c);
  return rc;
}
