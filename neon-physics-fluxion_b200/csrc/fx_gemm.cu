// fx_gemm.cu -- NT GEMM dispatch for the DCT stage and the FP32 CUDA-core
// (SIMT) variant. The tensor-core variants live in fx_gemm_tc.cu.
#include "fx_internal.h"
#include "fx_gemm.cuh"

namespace fx {

int gemm_nt_tc(fx_ctx *ctx, int precision, int G, const GemmOperands &A,
               const GemmOperands &B, const float *S, const GemmOperands &D,
               cudaStream_t s);
int gemm_half_tc(fx_ctx *ctx, int precision, int G, const GemmOperands &Ah,
                 const GemmOperands &Bh, float *part, cudaStream_t s);

constexpr int kBM = 128, kBN = 128, kBK = 16;

// 128 x 128 tile per CTA, 8 x 8 outputs per thread in two 4-wide strips per
// axis (conflict-free shared reads), K staged 16 at a time and stored
// k-major in shared memory. With `part` the CTA covers K range
// [z*Ks, (z+1)*Ks) of split z = blockIdx.z and writes its raw partial tile to
// part[z]; sgemm_reduce_kernel then adds the splits in order.
__global__ void __launch_bounds__(256)
sgemm_nt_kernel(const float *__restrict__ A, const float *__restrict__ B,
                int G, int Ks, const float *__restrict__ S, float *__restrict__ D,
                float *__restrict__ Dlo, uint16_t *__restrict__ Dbf,
                float *__restrict__ part) {
  __shared__ __align__(16) float As[kBK][kBM + 4];
  __shared__ __align__(16) float Bs[kBK][kBN + 4];
  const int t = threadIdx.x;
  const int bm = blockIdx.y * kBM, bn = blockIdx.x * kBN;
  const int lr = t >> 2, lk = (t & 3) * 4;
  const int tx = t & 15, ty = t >> 4;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
  const int kb = blockIdx.z * Ks;
  const float *a0 = A + (size_t)(bm + lr) * G + kb + lk;
  const float *a1 = a0 + (size_t)64 * G;
  const float *b0 = B + (size_t)(bn + lr) * G + kb + lk;
  const float *b1 = b0 + (size_t)64 * G;
  float4 ra0 = *(const float4 *)a0, ra1 = *(const float4 *)a1;
  float4 rb0 = *(const float4 *)b0, rb1 = *(const float4 *)b1;
  for (int k0 = 0; k0 < Ks; k0 += kBK) {
    As[lk + 0][lr] = ra0.x; As[lk + 1][lr] = ra0.y;
    As[lk + 2][lr] = ra0.z; As[lk + 3][lr] = ra0.w;
    As[lk + 0][lr + 64] = ra1.x; As[lk + 1][lr + 64] = ra1.y;
    As[lk + 2][lr + 64] = ra1.z; As[lk + 3][lr + 64] = ra1.w;
    Bs[lk + 0][lr] = rb0.x; Bs[lk + 1][lr] = rb0.y;
    Bs[lk + 2][lr] = rb0.z; Bs[lk + 3][lr] = rb0.w;
    Bs[lk + 0][lr + 64] = rb1.x; Bs[lk + 1][lr + 64] = rb1.y;
    Bs[lk + 2][lr + 64] = rb1.z; Bs[lk + 3][lr + 64] = rb1.w;
    __syncthreads();
    if (k0 + kBK < Ks) {
      ra0 = *(const float4 *)(a0 + k0 + kBK);
      ra1 = *(const float4 *)(a1 + k0 + kBK);
      rb0 = *(const float4 *)(b0 + k0 + kBK);
      rb1 = *(const float4 *)(b1 + k0 + kBK);
    }
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      const float4 x0 = *(const float4 *)&As[kk][ty * 4];
      const float4 x1 = *(const float4 *)&As[kk][64 + ty * 4];
      const float4 y0 = *(const float4 *)&Bs[kk][tx * 4];
      const float4 y1 = *(const float4 *)&Bs[kk][64 + tx * 4];
      const float a[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
      const float b[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = bm + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = bn + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
      const size_t o = (size_t)r * G + c;
      float v = acc[i][j];
      if (part) {
        part[(size_t)blockIdx.z * G * G + o] = v;
        continue;
      }
      if (S) v *= S[o];
      store_operand(v, o, D, Dlo, Dbf);
    }
  }
}

// Adds the split-K partial tiles in split order, then the epilogue.
__global__ void sgemm_reduce_kernel(const float *__restrict__ part, int splits, int G,
                                    const float *__restrict__ S, float *__restrict__ D,
                                    float *__restrict__ Dlo, uint16_t *__restrict__ Dbf) {
  const size_t cells = (size_t)G * G;
  for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < cells;
       o += (size_t)gridDim.x * blockDim.x) {
    float v = part[o];
    for (int z = 1; z < splits; ++z) v += part[z * cells + o];
    if (S) v *= S[o];
    store_operand(v, o, D, Dlo, Dbf);
  }
}

// Split-K factor of the SIMT GEMM: the largest power of two (<= 8) whose
// CTAs still fit in one wave (two 256-thread CTAs are resident per SM), K
// per split a multiple of 16.
int sgemm_splits(int G, int num_sms) {
  const int tiles = (G / kBM) * (G / kBN);
  int s = 1;
  while (tiles * 2 * s <= 2 * num_sms && s < 8 && (G / (2 * s)) % kBK == 0) s *= 2;
  return s;
}

// ---- even/odd halves of the DCT GEMMs (SIMT) --------------------------------
// Two GEMMs of (G/2) x G x (G/2) in one launch: z = b * splits + split,
//   part[z][r][c] = sum_{k in split} A_b[r][k] B_b[c][k],
// with A_b = A + b (G/2)^2 and B_b = B + b G (G/2), row stride G/2.
__global__ void __launch_bounds__(256)
sgemm_half_kernel(const float *__restrict__ A, const float *__restrict__ B, int G, int splits,
                  float *__restrict__ part) {
  __shared__ __align__(16) float As[kBK][kBM + 4];
  __shared__ __align__(16) float Bs[kBK][kBN + 4];
  const int h = G >> 1, Ks = h / splits;
  const int bt = blockIdx.z / splits, sp = blockIdx.z - bt * splits;
  const float *Ab = A + (size_t)bt * h * h, *Bb = B + (size_t)bt * G * h;
  const int t = threadIdx.x;
  const int bm = blockIdx.y * kBM, bn = blockIdx.x * kBN;
  const int lr = t >> 2, lk = (t & 3) * 4;
  const int tx = t & 15, ty = t >> 4;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
  const int kb = sp * Ks;
  const float *a0 = Ab + (size_t)(bm + lr) * h + kb + lk;
  const float *a1 = a0 + (size_t)64 * h;
  const float *b0 = Bb + (size_t)(bn + lr) * h + kb + lk;
  const float *b1 = b0 + (size_t)64 * h;
  float4 ra0 = *(const float4 *)a0, ra1 = *(const float4 *)a1;
  float4 rb0 = *(const float4 *)b0, rb1 = *(const float4 *)b1;
  for (int k0 = 0; k0 < Ks; k0 += kBK) {
    As[lk + 0][lr] = ra0.x; As[lk + 1][lr] = ra0.y;
    As[lk + 2][lr] = ra0.z; As[lk + 3][lr] = ra0.w;
    As[lk + 0][lr + 64] = ra1.x; As[lk + 1][lr + 64] = ra1.y;
    As[lk + 2][lr + 64] = ra1.z; As[lk + 3][lr + 64] = ra1.w;
    Bs[lk + 0][lr] = rb0.x; Bs[lk + 1][lr] = rb0.y;
    Bs[lk + 2][lr] = rb0.z; Bs[lk + 3][lr] = rb0.w;
    Bs[lk + 0][lr + 64] = rb1.x; Bs[lk + 1][lr + 64] = rb1.y;
    Bs[lk + 2][lr + 64] = rb1.z; Bs[lk + 3][lr + 64] = rb1.w;
    __syncthreads();
    if (k0 + kBK < Ks) {
      ra0 = *(const float4 *)(a0 + k0 + kBK);
      ra1 = *(const float4 *)(a1 + k0 + kBK);
      rb0 = *(const float4 *)(b0 + k0 + kBK);
      rb1 = *(const float4 *)(b1 + k0 + kBK);
    }
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      const float4 x0 = *(const float4 *)&As[kk][ty * 4];
      const float4 x1 = *(const float4 *)&As[kk][64 + ty * 4];
      const float4 y0 = *(const float4 *)&Bs[kk][tx * 4];
      const float4 y1 = *(const float4 *)&Bs[kk][64 + tx * 4];
      const float a[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
      const float b[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  float *pz = part + (size_t)blockIdx.z * h * G;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = bm + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = bn + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
      pz[(size_t)r * G + c] = acc[i][j];
    }
  }
}

// Adds each half's split-K partials in split order, then places the halves:
// kHalfRows: even and odd output rows (2r, 2r + 1) of a C-type product;
// kHalfPair: rows r and G-1-r as E + O and sign (E - O) of a C^T-type one.
__global__ void sgemm_half_reduce_kernel(const float *__restrict__ part, int splits, int G,
                                         int mode, float sign, const float *__restrict__ S,
                                         float *__restrict__ D, float *__restrict__ Dlo,
                                         uint16_t *__restrict__ Dbf) {
  const int h = G >> 1;
  const size_t half = (size_t)h * G;
  for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < half;
       o += (size_t)gridDim.x * blockDim.x) {
    float e = part[o], q = part[(size_t)splits * half + o];
    for (int z = 1; z < splits; ++z) {
      e += part[(size_t)z * half + o];
      q += part[(size_t)(splits + z) * half + o];
    }
    const size_t r = o / (size_t)G, c = o - r * (size_t)G;
    size_t o0, o1;
    float v0, v1;
    if (mode == kHalfRows) {
      o0 = (2 * r) * G + c;
      o1 = (2 * r + 1) * G + c;
      v0 = e;
      v1 = q;
    } else {
      o0 = r * G + c;
      o1 = ((size_t)G - 1 - r) * G + c;
      v0 = e + q;
      v1 = sign * (e - q);
    }
    if (S) {
      v0 *= S[o0];
      v1 *= S[o1];
    }
    store_operand(v0, o0, D, Dlo, Dbf);
    store_operand(v1, o1, D, Dlo, Dbf);
  }
}

// Split-K of the half GEMMs: the largest power of two (<= 8) that keeps the
// launch to one 256-thread CTA per SM. A CTA holds half an SM's registers, so
// the Barnes-Hut kernels that run beside the density stage still find room.
int half_splits(int G, int num_sms) {
  const int h = G / 2, tiles = 2 * (h / kBM) * (G / kBN);
  int s = 1;
  while (tiles * 2 * s <= num_sms && s < 8 && (h / (2 * s)) % kBK == 0) s *= 2;
  return s;
}

int gemm_half(fx_ctx *ctx, int precision, int G, const GemmOperands &Ah,
              const GemmOperands &Bh, int mode, float sign, const float *S, float *D,
              float *part, cudaStream_t s) {
  if (G % 256 != 0) {
    set_error("gemm_half: G=%d is not a multiple of 256", G);
    return FX_EINVAL;
  }
  int splits = 1;
  if (precision == FX_DCT_SIMT) {
    splits = half_splits(G, ctx->num_sms);
    dim3 grid(G / kBN, (G / 2) / kBM, 2 * splits);
    sgemm_half_kernel<<<grid, 256, 0, s>>>(Ah.f32, Bh.f32, G, splits, part);
    ctx->launches += 1;
  } else {
    FX_TRY(gemm_half_tc(ctx, precision, G, Ah, Bh, part, s));
  }
  sgemm_half_reduce_kernel<<<ctx->num_sms * 8, 256, 0, s>>>(part, splits, G, mode, sign, S, D,
                                                            nullptr, nullptr);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

int gemm_half_i8(fx_ctx *ctx, int G, const int8_t *A8, const float *sa, const float *Bh,
                 int mode, float sign, const float *S, float *D, float *part, int8_t *b8,
                 float *bsc, cudaStream_t s) {
  FX_TRY(i8_slice(ctx, Bh, 2 * G, G / 2, b8, bsc, s));
  FX_TRY(gemm_half_i8_tc(ctx, G, A8, sa, b8, bsc, part, s));
  sgemm_half_reduce_kernel<<<ctx->num_sms * 8, 256, 0, s>>>(part, 1, G, mode, sign, S, D,
                                                            nullptr, nullptr);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

int gemm_nt(fx_ctx *ctx, int precision, int G, const GemmOperands &A,
            const GemmOperands &B, const float *S, const GemmOperands &D,
            cudaStream_t s, float *split_ws) {
  if (G % 128 != 0) {
    set_error("gemm_nt: G=%d is not a multiple of 128", G);
    return FX_EINVAL;
  }
  if (precision == FX_DCT_SIMT) {
    const int splits = split_ws ? sgemm_splits(G, ctx->num_sms) : 1;
    dim3 grid(G / kBN, G / kBM, splits);
    sgemm_nt_kernel<<<grid, 256, 0, s>>>(A.f32, B.f32, G, G / splits, S, D.f32, D.lo, D.bf,
                                         splits > 1 ? split_ws : nullptr);
    if (splits > 1)
      sgemm_reduce_kernel<<<ctx->num_sms * 8, 256, 0, s>>>(split_ws, splits, G, S, D.f32,
                                                           D.lo, D.bf);
    FX_CHECK_LAUNCH();
    ctx->launches += splits > 1 ? 2 : 1;
    return FX_OK;
  }
  return gemm_nt_tc(ctx, precision, G, A, B, S, D, s);
}

}  // namespace fx
