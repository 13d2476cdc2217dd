// fx_gemm.cuh -- NT GEMM interface used by the DCT Poisson stage.
#pragma once
#include <cstdint>
#include <cstring>

#include <cuda_bf16.h>

namespace fx {

// One GEMM operand in every format a precision path may read or write:
//   f32 -- full values (SIMT, TF32) or the TF32 head (3xTF32 split),
//   lo  -- residual f32 - head (3xTF32 only),
//   bf  -- bfloat16 copy (BF16 only).
struct GemmOperands {
  float *f32;
  float *lo;
  uint16_t *bf;
};

// Round-to-nearest-even to TF32 (10 explicit mantissa bits). A value whose
// low 13 bits are zero is read exactly by the tensor cores whatever their
// rounding of f32 inputs.
__host__ __device__ inline float tf32_round(float v) {
  uint32_t u;
  memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) {
    u += 0xfffu + ((u >> 13) & 1u);
    u &= 0xffffe000u;
  }
  float r;
  memcpy(&r, &u, 4);
  return r;
}

inline float tf32_hi_host(float v) { return tf32_round(v); }

inline uint16_t bf16_host(float v) {
  uint32_t u;
  memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

// Writes v in the formats requested by the non-null pointers: with `lo` the
// head goes to f32 and the exact residual to lo.
__device__ __forceinline__ void store_operand(float v, size_t i, float *f32,
                                              float *lo, uint16_t *bf) {
  if (lo) {
    const float h = tf32_round(v);
    f32[i] = h;
    lo[i] = v - h;
  } else if (f32) {
    f32[i] = v;
  }
  if (bf) {
    __nv_bfloat16 b = __float2bfloat16_rn(v);
    bf[i] = *reinterpret_cast<uint16_t *>(&b);
  }
}

// D[i][j] = sum_k A[i][k] * B[j][k] (* S[i][j] when S != nullptr) for G x G
// row-major matrices, written to D in the formats of `precision`.
// split_ws: SIMT split-K workspace of sgemm_splits(G, sms) * G * G floats, or
// nullptr for no split.
int gemm_nt(fx_ctx *ctx, int precision, int G, const GemmOperands &A,
            const GemmOperands &B, const float *S, const GemmOperands &D,
            cudaStream_t s, float *split_ws = nullptr);
int sgemm_splits(int G, int num_sms);

// Even/odd halves of a DCT-stage GEMM (G a multiple of 256), on the CUDA
// cores (FX_DCT_SIMT) or the tensor cores: Ah holds two (G/2) x (G/2)
// operator halves, Bh the two G x (G/2) halves of the folded or split data
// operand, each in the formats of `precision`; kHalfRows interleaves the
// results as even/odd rows, kHalfPair writes rows r and G-1-r as E + O and
// sign (E - O); D gets f32 values. part: half_splits(G, sms) * G * G floats
// (SIMT split-K partials) or G * G (tensor cores).
constexpr int kHalfRows = 0, kHalfPair = 1;
int half_splits(int G, int num_sms);
int gemm_half(fx_ctx *ctx, int precision, int G, const GemmOperands &Ah,
              const GemmOperands &Bh, int mode, float sign, const float *S, float *D,
              float *part, cudaStream_t s);

// FX_DCT_I8 (fx_gemm_tc.cu): D = A B^T (times S) from 8-bit slices: A8 the
// operator's G x (i8_slices() G) slices [s1 ..] with row scales sa, B8 the
// data operand's [.. s1] with row scales sb (i8_slice writes those).
int i8_slices();
int gemm_nt_i8(fx_ctx *ctx, int G, const int8_t *A8, const float *sa, const int8_t *B8,
               const float *sb, const float *S, float *D, cudaStream_t s);
int i8_slice(fx_ctx *ctx, const float *X, int rows, int K, int8_t *out, float *scale,
             cudaStream_t s);
int gemm_half_i8_tc(fx_ctx *ctx, int G, const int8_t *A8, const float *sa, const int8_t *B8,
                    const float *sb, float *part, cudaStream_t s);
// gemm_half for FX_DCT_I8: slices Bh (2G x G/2 f32) into b8 / bsc, then the
// two half products from the operator halves' slices (A8, sa) and the
// placing reduce (mode, sign, S as gemm_half).
int gemm_half_i8(fx_ctx *ctx, int G, const int8_t *A8, const float *sa, const float *Bh,
                 int mode, float sign, const float *S, float *D, float *part, int8_t *b8,
                 float *bsc, cudaStream_t s);

}  // namespace fx
