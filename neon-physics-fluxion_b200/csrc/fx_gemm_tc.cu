// fx_gemm_tc.cu -- tensor-core (tcgen05) NT GEMMs for the DCT stage.
//
// D[i][j] = sum_k A[i][k] * B[j][k] for G x G row-major f32/bf16 matrices,
// both operands K-major. One CTA computes a 128 x 128 tile of D:
//   * warp 0 (one elected thread) streams 128 x 128-byte K slices of A and B
//     into a ring of shared-memory stages with TMA (128B swizzle, no
//     multicast), signalling a per-stage mbarrier with the transaction bytes;
//   * warp 1 (one thread) issues tcgen05.mma (M = 128, N = 128, K = 32 bytes
//     per instruction) into a 128-column TMEM accumulator and releases each
//     stage with tcgen05.commit;
//   * warp 2 owns the TMEM allocation;
//   * all four warps drain TMEM with tcgen05.ld (warp w holds rows 32w..32w+31)
//     and apply the optional element-wise scale S before storing.
// Precisions: TF32 (kind::tf32, one product), BF16 (kind::f16 with bf16
// operands, one product) and FP32 as 3xTF32: A = Ah + Al, B = Bh + Bl with the
// heads rounded to TF32, D = Ah Bh + Ah Bl + Al Bh accumulated in FP32 (the
// Al Bl term is below f32 resolution).
// Every mbarrier wait is bounded: on expiry the CTA records an error, waits
// (bounded) for its own TMA copies, frees TMEM and returns.
#include <cuda.h>

#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "fx_internal.h"
#include "fx_gemm.cuh"

namespace fx {

constexpr int kTcBM = 128, kTcBN = 128, kTcThreads = 128;
constexpr int kTileBytes = 128 * 128;  // one 128-row x 128-byte operand tile
constexpr uint32_t kWaitLimit = 1u << 22;

// ---- PTX helpers ----------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of the given parity; false on expiry.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map,
                                            uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// K-major operand tile, 128-byte rows packed, 128B swizzle: SBO = 1024 bytes
// (8-row swizzle atoms), LBO unused (16), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3ffffu) >> 4);
  d |= (uint64_t)(16u >> 4) << 16;
  d |= (uint64_t)(1024u >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
template <int KIND>
__device__ __forceinline__ void umma(uint32_t tmem, uint64_t a, uint64_t b,
                                     uint32_t idesc, uint32_t accum) {
  if (KIND == 0)
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          bar)
      : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, "
      "%9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, "
      "%24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
        "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
        "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]),
        "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// PREC: 0 = 3xTF32, 1 = TF32, 2 = BF16.
template <int PREC>
struct TcCfg {
  static constexpr int kKind = PREC == 2 ? 1 : 0;          // 0 tf32, 1 f16
  static constexpr int kElem = PREC == 2 ? 2 : 4;          // operand bytes
  static constexpr int kKBlock = 128 / kElem;              // elements per slice
  static constexpr int kTiles = PREC == 0 ? 4 : 2;         // tiles per stage
  static constexpr int kStages = PREC == 0 ? 3 : 6;
  static constexpr int kStageBytes = kTiles * kTileBytes;
  static constexpr uint32_t kFmt = PREC == 2 ? 1u : 2u;    // bf16 : tf32
  static constexpr uint32_t kIdesc = (1u << 4) | (kFmt << 7) | (kFmt << 10) |
                                     ((uint32_t)(kTcBN >> 3) << 17) |
                                     ((uint32_t)(kTcBM >> 4) << 24);
  static constexpr int kSmem = 1024 + kStages * kStageBytes + 256;
};

template <int PREC>
__global__ void __launch_bounds__(kTcThreads, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tA,
               const __grid_constant__ CUtensorMap tAlo,
               const __grid_constant__ CUtensorMap tB,
               const __grid_constant__ CUtensorMap tBlo, int G, int K, int a_batch_rows,
               int b_batch_rows, const float *__restrict__ S, float *__restrict__ D,
               float *__restrict__ Dlo, uint16_t *__restrict__ Dbf,
               float *__restrict__ part, unsigned int *__restrict__ err) {
  using Cfg = TcCfg<PREC>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;  // 1024-aligned stages
  const uint32_t bar0 = base + Cfg::kStages * Cfg::kStageBytes;
  // barriers: full[s] at bar0 + 8s, empty[s] at bar0 + 64 + 8s, done at +128
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 64u + 8u * s; };
  const uint32_t done_bar = bar0 + 128u;
  const uint32_t tmem_slot = bar0 + 136u;
  const uint32_t abort_slot = bar0 + 140u;
  uint8_t *gen_base = smem_raw + (base - raw);
  volatile uint32_t *tmem_ptr = (volatile uint32_t *)(gen_base + (tmem_slot - base));
  volatile uint32_t *abort_flag = (volatile uint32_t *)(gen_base + (abort_slot - base));

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bm = blockIdx.y * kTcBM, bn = blockIdx.x * kTcBN;
  // batch z (half GEMMs): operand rows offset by z * a_batch_rows / b_batch_rows
  const int am = bm + (int)blockIdx.z * a_batch_rows, bnz = bn + (int)blockIdx.z * b_batch_rows;
  const int KB = K / Cfg::kKBlock;

  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::kStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0u;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tmem_slot),
                 "r"(kTcBN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_ptr;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer --------------------------------------------------------
    int issued = 0;
    for (int kb = 0; kb < KB; ++kb) {
      const int s = kb % Cfg::kStages;
      const uint32_t ph = (uint32_t)(kb / Cfg::kStages) & 1u;
      if (kb >= Cfg::kStages && !mbar_wait(empty_bar(s), ph ^ 1u)) {
        *abort_flag = 1u;
        atomicOr(err, 2u);
        break;
      }
      if (*abort_flag) break;
      const uint32_t st = base + s * Cfg::kStageBytes;
      mbar_expect_tx(full_bar(s), Cfg::kStageBytes);
      const int x = kb * Cfg::kKBlock;
      tma_load_2d(st, &tA, full_bar(s), x, am);
      tma_load_2d(st + kTileBytes, &tB, full_bar(s), x, bnz);
      if (PREC == 0) {
        tma_load_2d(st + 2 * kTileBytes, &tAlo, full_bar(s), x, am);
        tma_load_2d(st + 3 * kTileBytes, &tBlo, full_bar(s), x, bnz);
      }
      issued = kb + 1;
    }
    // Before leaving, make sure none of this CTA's copies is still in flight.
    const int first = issued > Cfg::kStages ? issued - Cfg::kStages : 0;
    for (int kb = first; kb < issued; ++kb)
      mbar_wait(full_bar(kb % Cfg::kStages), (uint32_t)(kb / Cfg::kStages) & 1u);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----------------------------------------------------------
    bool ok = true;
    for (int kb = 0; kb < KB; ++kb) {
      const int s = kb % Cfg::kStages;
      const uint32_t ph = (uint32_t)(kb / Cfg::kStages) & 1u;
      if (!mbar_wait(full_bar(s), ph) || *abort_flag) {
        *abort_flag = 1u;
        atomicOr(err, 2u);
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t st = base + s * Cfg::kStageBytes;
      const uint64_t a = umma_desc(st), b = umma_desc(st + kTileBytes);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
        umma<Cfg::kKind>(tmem, a + 2u * k, b + 2u * k, Cfg::kIdesc, acc);
        if (PREC == 0) {
          const uint64_t alo = umma_desc(st + 2 * kTileBytes);
          const uint64_t blo = umma_desc(st + 3 * kTileBytes);
          umma<Cfg::kKind>(tmem, a + 2u * k, blo + 2u * k, Cfg::kIdesc, 1u);
          umma<Cfg::kKind>(tmem, alo + 2u * k, b + 2u * k, Cfg::kIdesc, 1u);
        }
      }
      umma_commit(empty_bar(s));
    }
    umma_commit(done_bar);
    (void)ok;
  }
  // ---- epilogue: all warps ------------------------------------------------------
  // tcgen05.ld is warp-collective: lane 0 waits and the warp follows its
  // verdict.
  __syncwarp();
  uint32_t go = 0u;
  if (lane == 0) {
    const bool done_ok = mbar_wait(done_bar, 0u);
    if (!done_ok) {
      *abort_flag = 1u;
      atomicOr(err, 2u);
    }
    go = (done_ok && !*abort_flag) ? 1u : 0u;
  }
  go = __shfl_sync(0xffffffffu, go, 0);
  tc_fence_after();
  if (go) {
    const int r = bm + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < kTcBN; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      const size_t o = (size_t)r * G + bn + c0;
      if (part) {  // raw partial of batch z: rows gridDim.y * 128, stride G
        float *pz = part + (size_t)blockIdx.z * gridDim.y * kTcBM * G;
#pragma unroll
        for (int j = 0; j < 32; ++j) pz[o + j] = __uint_as_float(v[j]);
        continue;
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        float x = __uint_as_float(v[j]);
        if (S) x *= S[o + j];
        store_operand(x, o + j, D, Dlo, Dbf);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcBN));
  }
}

// ---- FX_DCT_I8: FP32-accurate products from exact 8-bit slices ---------------------
// An operand row r is split under a power-of-two scale 2^e (the smallest with
// every |x| < 2^e) into kI8Slices = 6 signed 8-bit slices:
// x = 2^e sum_t s_t 2^(-7t), t = 1..6, exact for every x >= 2^(e-18) (42 bits
// cover the 24-bit significand of entries down to 2^-18 of the row's
// largest; the DCT spectra span about that within a row) and within
// 2^(e-42) below. A product of two rows is sum_w 2^(-7w) sum_{t+u=w}
// s_t . s'_u; the weight classes w = 2..7 (21 slice pairs) keep every pair
// above 2^-49 of the row scales. The operator A is stored with its slices in
// order [s1 .. s6] along K, the data operand B reversed [s6 .. s1], so class
// c = w - 2 is one GEMM over A columns [0, (c+1)K) and B columns
// [(5-c)K, 6K). tcgen05 kind::i8 accumulates the classes exactly in six
// 64-column int32 TMEM accumulators (|partial| <= 6K 127^2 < 2^31 for
// K <= 8192); the epilogue adds them in FP64, applies the row and column
// scales and rounds once to f32. The tensor cores' own accumulation
// rounding, which makes 3xTF32 lose accuracy with K, does not arise.
// Tiles are 128 x 64 (M x N), so a 1024-wide grid gives 128 CTAs. Each slice
// block crosses L2 once: per 128-byte K block, the six B slices stay in
// shared memory (double-buffered) while the six A slices stream through a
// ring, and A slice t meets every B slice u with t + u <= 7 (classes
// c = t + u - 2), 84 MMAs per K block.
constexpr int kI8Slices = 6;
constexpr int kI8BN = 64;
constexpr int kI8AStages = 6;                      // A slice ring
constexpr int kI8BTile = kI8BN * 128;              // one B slice block (64 rows x 128 B)
constexpr int kI8BBuf = kI8Slices * kI8BTile;      // the six B slices of one K block
constexpr int kI8Smem = 1024 + kI8AStages * kTileBytes + 2 * kI8BBuf + 256;
constexpr int kI8Cols = 512;                       // six 64-column accumulators (384 used)
// kind::i8 instruction descriptor: D s32 (2), A and B s8 (1), N / 8, M / 16
constexpr uint32_t kI8Idesc = (2u << 4) | (1u << 7) | (1u << 10) |
                              ((uint32_t)(kI8BN >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
static_assert(kI8Slices * kI8BN <= kI8Cols, "accumulators exceed the TMEM allocation");
static_assert(kI8Smem <= 227 * 1024, "shared memory");

__device__ __forceinline__ void umma_i8(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accum));
}

// Batch z (blockIdx.z; the even/odd half products) reads A rows from
// z a_rows, B rows from z b_rows and writes D from z d_elems on; D has G
// columns.
__global__ void __launch_bounds__(kTcThreads, 1)
tc_i8_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB,
             int G, int K, int a_rows, int b_rows, size_t d_elems,
             const float *__restrict__ sa, const float *__restrict__ sb,
             const float *__restrict__ S, float *__restrict__ D, unsigned int *__restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;    // 1024-aligned tiles
  const uint32_t bbuf0 = base + kI8AStages * kTileBytes;
  const uint32_t bar0 = bbuf0 + 2 * kI8BBuf;
  // barriers: afull[s] at bar0 + 8s, aempty[s] at +64 + 8s, bfull[j] at
  // +112 + 8j, bempty[j] at +128 + 8j, done at +144; then the TMEM address
  // and the abort flag
  auto afull = [&](int s) { return bar0 + 8u * s; };
  auto aempty = [&](int s) { return bar0 + 64u + 8u * s; };
  auto bfull = [&](int j) { return bar0 + 112u + 8u * j; };
  auto bempty = [&](int j) { return bar0 + 128u + 8u * j; };
  const uint32_t done_bar = bar0 + 144u;
  const uint32_t tmem_slot = bar0 + 152u;
  const uint32_t abort_slot = bar0 + 156u;
  uint8_t *gen_base = smem_raw + (base - raw);
  volatile uint32_t *tmem_ptr = (volatile uint32_t *)(gen_base + (tmem_slot - base));
  volatile uint32_t *abort_flag = (volatile uint32_t *)(gen_base + (abort_slot - base));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bm = blockIdx.y * kTcBM, bn = blockIdx.x * kI8BN;
  const int am = bm + (int)blockIdx.z * a_rows, bnz = bn + (int)blockIdx.z * b_rows;
  D += (size_t)blockIdx.z * d_elems;
  const int KB = K / 128;  // 128-byte blocks of one slice

  if (threadIdx.x == 0) {
    for (int s = 0; s < kI8AStages; ++s) {
      mbar_init(afull(s), 1);
      mbar_init(aempty(s), 1);
    }
    for (int j = 0; j < 2; ++j) {
      mbar_init(bfull(j), 1);
      mbar_init(bempty(j), 1);
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0u;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tmem_slot),
                 "r"(kI8Cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_ptr;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ------------------------------------------------------------
    int a_issued = 0, b_issued = 0;
    bool stop = false;
    for (int kb = 0; kb < KB && !stop; ++kb) {
      const int j = kb & 1;
      if (kb >= 2 && !mbar_wait(bempty(j), ((uint32_t)(kb >> 1) & 1u) ^ 1u)) {
        *abort_flag = 1u;
        atomicOr(err, 2u);
        break;
      }
      if (*abort_flag) break;
      const uint32_t bb = bbuf0 + j * kI8BBuf;
      mbar_expect_tx(bfull(j), kI8BBuf);
      for (int v = 0; v < kI8Slices; ++v)  // B layout position v holds slice 6 - v
        tma_load_2d(bb + v * kI8BTile, &tB, bfull(j), v * K + kb * 128, bnz);
      b_issued = kb + 1;
      for (int t = 0; t < kI8Slices; ++t) {
        const int i = kb * kI8Slices + t;
        const int s = i % kI8AStages;
        const uint32_t ph = (uint32_t)(i / kI8AStages) & 1u;
        if (i >= kI8AStages && !mbar_wait(aempty(s), ph ^ 1u)) {
          *abort_flag = 1u;
          atomicOr(err, 2u);
          stop = true;
          break;
        }
        if (*abort_flag) {
          stop = true;
          break;
        }
        mbar_expect_tx(afull(s), kTileBytes);
        tma_load_2d(base + s * kTileBytes, &tA, afull(s), t * K + kb * 128, am);
        a_issued = i + 1;
      }
    }
    // Before leaving, make sure none of this CTA's copies is still in flight.
    for (int i = a_issued > kI8AStages ? a_issued - kI8AStages : 0; i < a_issued; ++i)
      mbar_wait(afull(i % kI8AStages), (uint32_t)(i / kI8AStages) & 1u);
    for (int q = b_issued > 2 ? b_issued - 2 : 0; q < b_issued; ++q)
      mbar_wait(bfull(q & 1), (uint32_t)(q >> 1) & 1u);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: A slice t (value 2^-7(t+1)) x B slice u into class t + u --
    bool ok = true;
    for (int kb = 0; kb < KB && ok; ++kb) {
      const int j = kb & 1;
      if (!mbar_wait(bfull(j), (uint32_t)(kb >> 1) & 1u) || *abort_flag) {
        *abort_flag = 1u;
        atomicOr(err, 2u);
        break;
      }
      const uint32_t bb = bbuf0 + j * kI8BBuf;
      for (int t = 0; t < kI8Slices; ++t) {
        const int i = kb * kI8Slices + t;
        const int s = i % kI8AStages;
        if (!mbar_wait(afull(s), (uint32_t)(i / kI8AStages) & 1u) || *abort_flag) {
          *abort_flag = 1u;
          atomicOr(err, 2u);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t a = umma_desc(base + s * kTileBytes);
        for (int u = 0; u < kI8Slices - t; ++u) {
          const uint64_t b = umma_desc(bb + (kI8Slices - 1 - u) * kI8BTile);
          const uint32_t acc_col = (uint32_t)(kI8BN * (t + u));
#pragma unroll
          for (int k = 0; k < 4; ++k)  // 32 bytes of K per instruction
            umma_i8(tmem + acc_col, a + 2u * k, b + 2u * k, kI8Idesc,
                    (kb > 0 || t > 0 || k > 0) ? 1u : 0u);
        }
        umma_commit(aempty(s));
      }
      if (ok) umma_commit(bempty(j));
    }
    umma_commit(done_bar);
  }
  // ---- epilogue: all warps --------------------------------------------------------
  __syncwarp();
  uint32_t go = 0u;
  if (lane == 0) {
    const bool done_ok = mbar_wait(done_bar, 0u);
    if (!done_ok) {
      *abort_flag = 1u;
      atomicOr(err, 2u);
    }
    go = (done_ok && !*abort_flag) ? 1u : 0u;
  }
  go = __shfl_sync(0xffffffffu, go, 0);
  tc_fence_after();
  if (go) {
    const int r = bm + warp * 32 + lane;
    const double sr = (double)sa[am + warp * 32 + lane];
    const float *sbz = sb + (size_t)blockIdx.z * b_rows;
#pragma unroll 1
    for (int c0 = 0; c0 < kI8BN; c0 += 32) {
      double acc[32];
#pragma unroll
      for (int jj = 0; jj < 32; ++jj) acc[jj] = 0.0;
#pragma unroll 1
      for (int c = 0; c < kI8Slices; ++c) {
        uint32_t v[32];
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(kI8BN * c + c0), v);
        const double wgt = ldexp(1.0, -7 * (c + 2));
#pragma unroll
        for (int jj = 0; jj < 32; ++jj) acc[jj] += (double)(int32_t)v[jj] * wgt;
      }
      const size_t o = (size_t)r * G + bn + c0;
#pragma unroll
      for (int jj = 0; jj < 32; ++jj) {
        float x = (float)(acc[jj] * sr * (double)sbz[bn + c0 + jj]);
        if (S) x *= S[o + jj];
        D[o + jj] = x;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kI8Cols));
  }
}

// Slices of a data operand (rows x K f32, row-major) in the reversed order
// [s6 .. s1] along 6K columns, and each row's scale 2^e. One warp per row.
// Every step is exact in f32: scaling by powers of two, truncation, and the
// remainder of a truncation.
__global__ void i8_slice_kernel(const float *__restrict__ X, int rows, int K,
                                int8_t *__restrict__ out, float *__restrict__ scale) {
  const int lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += (gridDim.x * blockDim.x) >> 5) {
    const float *x = X + (size_t)r * K;
    float m = 0.f;
    for (int k = lane; k < K; k += 32) m = fmaxf(m, fabsf(x[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    int e = 0;
    if (m > 0.f) frexpf(m, &e);  // m = f 2^e, f in [0.5, 1): every |x| < 2^e
    if (lane == 0) scale[r] = ldexpf(1.f, e);
    int8_t *o8 = out + (size_t)r * kI8Slices * K;
    for (int k = lane; k < K; k += 32) {
      float a = ldexpf(x[k], -e);
#pragma unroll
      for (int t = 0; t < kI8Slices; ++t) {
        const float q = a * 128.f;
        const float w = truncf(q);
        o8[(size_t)(kI8Slices - 1 - t) * K + k] = (int8_t)(int)w;
        a = q - w;
      }
    }
  }
}

// ---- host: tensor maps -------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t,
                                  void *, const cuuint64_t *, const cuuint64_t *,
                                  const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  });
  return fn;
}

// A rows x cols row-major operand of esz-byte elements (4: f32, 2: bf16,
// 1: int8 slices) as a 2-D tensor map with 128 x 128-byte boxes.
static int make_map(const void *ptr, int cols, int rows, int esz, CUtensorMap *out,
                    int box_rows = 128) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is unavailable");
    return FX_ECUDA;
  }
  if (((uintptr_t)ptr & 15u) != 0) {
    set_error("tensor map base not 16-byte aligned");
    return FX_EINVAL;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * esz};
  const cuuint32_t box[2] = {(cuuint32_t)(128 / esz), (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r =
      fn(out,
         esz == 1   ? CU_TENSOR_MAP_DATA_TYPE_UINT8
         : esz == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                    : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
         2,
         const_cast<void *>(ptr), dims, strides, box, estr,
         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return FX_ECUDA;
  }
  return FX_OK;
}

struct MapKey {
  const void *p;
  int cols, rows;
  int esz, box_rows;
  bool operator==(const MapKey &o) const {
    return p == o.p && cols == o.cols && rows == o.rows && esz == o.esz &&
           box_rows == o.box_rows;
  }
};
struct MapKeyHash {
  size_t operator()(const MapKey &k) const {
    return std::hash<const void *>()(k.p) ^ ((size_t)k.cols << 1) ^ ((size_t)k.rows << 21) ^
           (size_t)k.esz ^ ((size_t)k.box_rows << 8);
  }
};

static int get_map(const void *ptr, int cols, int rows, int esz, CUtensorMap *out,
                   int box_rows = 128) {
  static std::mutex mu;
  static std::unordered_map<MapKey, CUtensorMap, MapKeyHash> cache;
  std::lock_guard<std::mutex> g(mu);
  const MapKey k{ptr, cols, rows, esz, box_rows};
  auto it = cache.find(k);
  if (it != cache.end()) {
    *out = it->second;
    return FX_OK;
  }
  FX_TRY(make_map(ptr, cols, rows, esz, out, box_rows));
  if (cache.size() >= 4096) cache.clear();  // bounded: designs come and go
  cache.emplace(k, *out);
  return FX_OK;
}

// half == false: D = A B^T on G x G operands (epilogue: S, formats).
// half == true: the two (G/2) x G x (G/2) products of the even/odd halves
// (A: 2 x (G/2) x (G/2), B: 2 x G x (G/2)) as raw partials in `part`.
template <int PREC>
static int launch(fx_ctx *ctx, int G, const GemmOperands &A, const GemmOperands &B,
                  const float *S, const GemmOperands &D, cudaStream_t s, bool half = false,
                  float *part = nullptr) {
  using Cfg = TcCfg<PREC>;
  const bool bf = PREC == 2;
  CUtensorMap ta, talo, tb, tblo;
  const void *pa = bf ? (const void *)A.bf : (const void *)A.f32;
  const void *pb = bf ? (const void *)B.bf : (const void *)B.f32;
  if (!pa || !pb || (PREC == 0 && (!A.lo || !B.lo))) {
    set_error("gemm_nt: operand format missing for precision %d", PREC);
    return FX_EINVAL;
  }
  const int h = G / 2;
  const int kc = half ? h : G, ar = half ? 2 * h : G, br = half ? 2 * G : G;
  FX_TRY(get_map(pa, kc, ar, bf ? 2 : 4, &ta));
  FX_TRY(get_map(pb, kc, br, bf ? 2 : 4, &tb));
  if (PREC == 0) {
    FX_TRY(get_map(A.lo, kc, ar, 4, &talo));
    FX_TRY(get_map(B.lo, kc, br, 4, &tblo));
  } else {
    talo = ta;
    tblo = tb;
  }
  FX_TRY(raise_smem_limit(reinterpret_cast<const void *>(tc_gemm_kernel<PREC>), Cfg::kSmem));
  unsigned int *err = ctx->tc_err;
  if (half) {
    dim3 grid(G / kTcBN, h / kTcBM, 2);
    tc_gemm_kernel<PREC><<<grid, kTcThreads, Cfg::kSmem, s>>>(
        ta, talo, tb, tblo, G, h, h, G, nullptr, nullptr, nullptr, nullptr, part, err);
  } else {
    dim3 grid(G / kTcBN, G / kTcBM);
    tc_gemm_kernel<PREC><<<grid, kTcThreads, Cfg::kSmem, s>>>(
        ta, talo, tb, tblo, G, G, 0, 0, S, D.f32, D.lo, D.bf, nullptr, err);
  }
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

int gemm_nt_tc(fx_ctx *ctx, int precision, int G, const GemmOperands &A,
               const GemmOperands &B, const float *S, const GemmOperands &D,
               cudaStream_t s) {
  switch (precision) {
    case FX_DCT_FP32: return launch<0>(ctx, G, A, B, S, D, s);
    case FX_DCT_TF32: return launch<1>(ctx, G, A, B, S, D, s);
    case FX_DCT_BF16: return launch<2>(ctx, G, A, B, S, D, s);
  }
  set_error("gemm_nt: unknown precision %d", precision);
  return FX_EINVAL;
}

int gemm_half_tc(fx_ctx *ctx, int precision, int G, const GemmOperands &Ah,
                 const GemmOperands &Bh, float *part, cudaStream_t s) {
  const GemmOperands none{nullptr, nullptr, nullptr};
  switch (precision) {
    case FX_DCT_FP32: return launch<0>(ctx, G, Ah, Bh, nullptr, none, s, true, part);
    case FX_DCT_TF32: return launch<1>(ctx, G, Ah, Bh, nullptr, none, s, true, part);
    case FX_DCT_BF16: return launch<2>(ctx, G, Ah, Bh, nullptr, none, s, true, part);
  }
  set_error("gemm_half: unknown precision %d", precision);
  return FX_EINVAL;
}

// D = A B^T (times S) from the slices of A (operator, [s1..s6]) and of B
// (data, [s6..s1]), each G x 6G int8 with a scale per row; D in f32.
int gemm_nt_i8(fx_ctx *ctx, int G, const int8_t *A8, const float *sa, const int8_t *B8,
               const float *sb, const float *S, float *D, cudaStream_t s) {
  if (G % 128 != 0 || G > 8192) {
    set_error("gemm_nt_i8: G = %d must be a multiple of 128 up to 8192", G);
    return FX_EINVAL;
  }
  CUtensorMap ta, tb;
  FX_TRY(get_map(A8, kI8Slices * G, G, 1, &ta));
  FX_TRY(get_map(B8, kI8Slices * G, G, 1, &tb, kI8BN));
  FX_TRY(raise_smem_limit(reinterpret_cast<const void *>(tc_i8_kernel), kI8Smem));
  dim3 grid(G / kI8BN, G / kTcBM);
  tc_i8_kernel<<<grid, kTcThreads, kI8Smem, s>>>(ta, tb, G, G, 0, 0, 0, sa, sb, S, D,
                                                 ctx->tc_err);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

// The even/odd halves (G a multiple of 256, h = G / 2): two products
// part[z] (h x G) = A_z (h x h) B_z^T (G x h) in one launch, from A8
// (2h x 6h: the two operator halves' slices) and B8 (2G x 6h: the two halves
// of the folded or split data operand), as raw f32 partials.
int gemm_half_i8_tc(fx_ctx *ctx, int G, const int8_t *A8, const float *sa, const int8_t *B8,
                    const float *sb, float *part, cudaStream_t s) {
  const int h = G / 2;
  if (G % 256 != 0 || G > 8192) {
    set_error("gemm_half_i8: G = %d must be a multiple of 256 up to 8192", G);
    return FX_EINVAL;
  }
  CUtensorMap ta, tb;
  FX_TRY(get_map(A8, kI8Slices * h, 2 * h, 1, &ta));
  FX_TRY(get_map(B8, kI8Slices * h, 2 * G, 1, &tb, kI8BN));
  FX_TRY(raise_smem_limit(reinterpret_cast<const void *>(tc_i8_kernel), kI8Smem));
  dim3 grid(G / kI8BN, h / kTcBM, 2);
  tc_i8_kernel<<<grid, kTcThreads, kI8Smem, s>>>(ta, tb, G, h, h, G, (size_t)h * G, sa, sb,
                                                 nullptr, part, ctx->tc_err);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

int i8_slices() { return kI8Slices; }

int i8_slice(fx_ctx *ctx, const float *X, int rows, int K, int8_t *out, float *scale,
             cudaStream_t s) {
  const int blocks = std::min((rows + 7) / 8, ctx->num_sms * 8);
  i8_slice_kernel<<<blocks, 256, 0, s>>>(X, rows, K, out, scale);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

// Error word of the context's tensor-core GEMMs (bit 1: a bounded wait
// expired). A set word is reported once and cleared, so one expired wait
// does not fail every later call of the context.
int gemm_tc_error(fx_ctx *ctx, unsigned int *out, cudaStream_t s) {
  *out = 0;
  FX_CHECK_CUDA(cudaMemcpyAsync(out, ctx->tc_err, 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (*out) {
    FX_CHECK_CUDA(cudaMemsetAsync(ctx->tc_err, 0, 4, s));
    FX_CHECK_CUDA(cudaStreamSynchronize(s));
  }
  return FX_OK;
}

}  // namespace fx
