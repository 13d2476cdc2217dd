// fx_density.cu -- row C: DCT-II Poisson density force as dense GEMM stages.
//
// Follows ElectrostaticSmoothingForce (O/src/python/fluxion/
// force_electrostatic.py):
//   density      rho[r,c] += area / (bw*bh), point-in-bin      (:47-60)
//   charge       rho - rho_target                                (:122-123)
//   spectrum     rho_hat = DCT-II_ortho(rho) = C rho C^T         (:69)
//   eigenvalues  (wx cos(pi kx/nx) - wx)^2 + (wy cos(pi ky/ny) - wy)^2,
//                [0,0] := 1, phi_hat = -rho_hat / lambda, phi_hat[0,0] := 0
//                                                                (:72-86)
//   potential    phi = IDCT_ortho(phi_hat) = C^T phi_hat C       (:89)
//   field        centred differences inside, one-sided at edges  (:91-103),
//                applied as the operator products Dx C^T / Dy C^T
//   force        F_i = area_i * E[row, col] * weight             (:134-150)
// C is the orthonormal DCT-II matrix (G x G). The transforms are NT GEMMs
// D = A * B^T with A a constant operator and B the data produced by the
// previous GEMM (see density_run).
// Bin areas are accumulated as 64-bit fixed point so the density is exact
// and independent of the scatter order.
#include <algorithm>
#include <cmath>

#include "fx_internal.h"
#include "fx_device.cuh"
#include "fx_gemm.cuh"

namespace fx {

int gemm_tc_error(fx_ctx *ctx, unsigned int *out, cudaStream_t s);

constexpr double kAreaScale = 4294967296.0;  // 2^32

// numpy's int(clip(v / bin, 0, G-1)) (force_electrostatic.py:55-56) with the
// division in f32.
__device__ __forceinline__ int bin_at(float v, float bin, int G) {
  const float q = __fdiv_rn(v, bin);
  if (!(q >= 1.0f)) return 0;
  if (q >= (float)(G - 1)) return G - 1;
  return (int)q;
}

__global__ void dens_scatter_kernel(const float *__restrict__ x,
                                    const float *__restrict__ y,
                                    const float *__restrict__ area, int n,
                                    int G, float bw, float bh,
                                    unsigned long long *__restrict__ acc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const int c = bin_at(x[i], bw, G), r = bin_at(y[i], bh, G);
    const unsigned long long a =
        (unsigned long long)llrint((double)area[i] * kAreaScale);
    atomicAdd(acc + (size_t)r * G + c, a);
  }
}

// Charge grid rho - rho_target in f32 (and the operand formats the chosen
// GEMM path reads); re-arms the accumulator.
// Four consecutive bins per thread: two 16-byte loads in flight per thread
// and one pass over the grid (a grid-stride loop waited out one DRAM round
// trip per bin).
__global__ void dens_charge_kernel(unsigned long long *__restrict__ acc,
                                   int cells, double inv_bin_area,
                                   float target, float *__restrict__ rho,
                                   float *__restrict__ rho_lo,
                                   uint16_t *__restrict__ rho_bf) {
  const int i0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (i0 >= cells) return;
  unsigned long long q[4];
  if (i0 + 3 < cells) {
    const ulonglong2 a = reinterpret_cast<const ulonglong2 *>(acc)[i0 >> 1];
    const ulonglong2 b = reinterpret_cast<const ulonglong2 *>(acc)[(i0 >> 1) + 1];
    q[0] = a.x; q[1] = a.y; q[2] = b.x; q[3] = b.y;
    reinterpret_cast<ulonglong2 *>(acc)[i0 >> 1] = make_ulonglong2(0ull, 0ull);
    reinterpret_cast<ulonglong2 *>(acc)[(i0 >> 1) + 1] = make_ulonglong2(0ull, 0ull);
  } else {
    for (int r = 0; r < 4; ++r) {
      q[r] = i0 + r < cells ? acc[i0 + r] : 0ull;
      if (i0 + r < cells) acc[i0 + r] = 0ull;
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    if (i0 + r >= cells) break;
    const double a = (double)q[r] * (1.0 / kAreaScale) * inv_bin_area;
    store_operand((float)(a - (double)target), i0 + r, rho, rho_lo, rho_bf);
  }
}

// Even/odd halves of a data operand B (G x G, row-major), each G x (G/2):
// fold (for products with C, whose columns mirror as C[i][G-1-k] =
// (-1)^i C[i][k]): B[j][k] + B[j][G-1-k] and B[j][k] - B[j][G-1-k];
// split (for C^T-type operators, whose rows mirror): B[j][2m] and B[j][2m+1].
// Outputs go out in the operand formats of the GEMM path (f32 or TF32 head,
// 3xTF32 residual, bf16), as store_operand writes them.
__global__ void dct_fold_kernel(const float *__restrict__ B, int G, float *__restrict__ out,
                                float *__restrict__ out_lo, uint16_t *__restrict__ out_bf) {
  const int h = G >> 1;
  const size_t half = (size_t)G * h;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < half;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t j = i / (size_t)h, k = i - j * (size_t)h;
    const float a = B[j * G + k], b = B[j * G + (G - 1 - k)];
    store_operand(a + b, i, out, out_lo, out_bf);
    store_operand(a - b, half + i, out, out_lo, out_bf);
  }
}

__global__ void dct_split_kernel(const float *__restrict__ B, int G, float *__restrict__ out,
                                 float *__restrict__ out_lo, uint16_t *__restrict__ out_bf) {
  const int h = G >> 1;
  const size_t half = (size_t)G * h;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < half;
       i += (size_t)gridDim.x * blockDim.x) {
    const float2 v = reinterpret_cast<const float2 *>(B)[i];  // B[j][2m], B[j][2m+1]
    store_operand(v.x, i, out, out_lo, out_bf);
    store_operand(v.y, half + i, out, out_lo, out_bf);
  }
}

// Per-gate force and the FP64 energy 0.5 * sum q * phi (force_electrostatic.
// py:134-150).
__global__ void dens_gather_kernel(const float *__restrict__ x,
                                   const float *__restrict__ y,
                                   const float *__restrict__ area, int n,
                                   int G, float bw, float bh, float weight,
                                   const float *__restrict__ ex,
                                   const float *__restrict__ ey,
                                   const float *__restrict__ phi,
                                   float2 *__restrict__ force,
                                   double *__restrict__ partial,
                                   unsigned int *__restrict__ done,
                                   double *__restrict__ energy) {
  double e = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const int c = bin_at(x[i], bw, G), r = bin_at(y[i], bh, G);
    const size_t b = (size_t)r * G + c;
    const float q = area[i];
    force[i] = make_float2(__fmul_rn(__fmul_rn(q, ex[b]), weight),
                           __fmul_rn(__fmul_rn(q, ey[b]), weight));
    e += 0.5 * (double)q * (double)phi[b];
  }
  last_block_sum(block_sum_double(e) * (double)weight, partial, done, energy);
}

// Uploads a constant G x G operand computed in FP64 in the formats of
// `precision`: f32 values (SIMT, TF32), TF32 head + residual (3xTF32), bf16.
static int upload_operand(const std::vector<double> &m, int precision, float *f32,
                          float *lo, uint16_t *bf, cudaStream_t s) {
  const size_t cells = m.size();
  std::vector<float> hi(cells), rl;
  std::vector<uint16_t> hb;
  if (precision == FX_DCT_FP32) rl.resize(cells);
  if (precision == FX_DCT_BF16) hb.resize(cells);
  for (size_t i = 0; i < cells; ++i) {
    const float v = (float)m[i];
    if (precision == FX_DCT_FP32) {
      hi[i] = tf32_hi_host(v);
      rl[i] = v - hi[i];
    } else {
      hi[i] = v;
    }
    if (precision == FX_DCT_BF16) hb[i] = bf16_host(v);
  }
  FX_CHECK_CUDA(cudaMemcpyAsync(f32, hi.data(), cells * 4, cudaMemcpyHostToDevice, s));
  if (lo) FX_CHECK_CUDA(cudaMemcpyAsync(lo, rl.data(), cells * 4, cudaMemcpyHostToDevice, s));
  if (bf) FX_CHECK_CUDA(cudaMemcpyAsync(bf, hb.data(), cells * 2, cudaMemcpyHostToDevice, s));
  return cudaStreamSynchronize(s) == cudaSuccess ? FX_OK : FX_ECUDA;
}

// Host: DCT matrix C, the inverse eigenvalues and the field operators
// Dx C^T, Dy C^T, in FP64 then rounded. Dx is the reference's x stencil
// (force_electrostatic.py:96-103) as a matrix on a row of phi:
// E_x[r][c] = sum_c' phi[r][c'] Dx[c][c'] with -wx/2 (phi[c+1] - phi[c-1])
// inside and -wx (phi[1] - phi[0]), -wx (phi[G-1] - phi[G-2]) at the edges;
// Dy likewise on columns. Since phi = C^T phi_hat C, the field is
//   E_x = C^T (phi_hat (Dx C^T)^T),   E_y = (Dy C^T) (phi_hat C),
// the same linear map as differencing phi, without forming the difference
// of a large smooth potential in f32.
static int dens_setup(fx_design *d, int G, int precision, cudaStream_t s) {
  DensityWork &w = d->dens;
  if (w.G == G && w.precision == precision && w.cmat.p) return FX_OK;
  const size_t cells = (size_t)G * G;
  FX_TRY(w.area_fx.alloc(cells));
  FX_TRY(w.cmat.alloc(cells));
  FX_TRY(w.cmat_t.alloc(cells));
  FX_TRY(w.dxct.alloc(cells));
  FX_TRY(w.dyct.alloc(cells));
  FX_TRY(w.inv_eig.alloc(cells));
  for (int i = 0; i < 5; ++i) FX_TRY(w.buf[i].alloc(cells));
  FX_TRY(w.ex.alloc(cells));
  FX_TRY(w.ey.alloc(cells));
  FX_TRY(w.energy.alloc(4096 + 8));
  FX_TRY(w.force.alloc((size_t)d->n));
  // The GEMMs are halved by the DCT's even/odd symmetry when G is a multiple
  // of 256 (tiles of 128 on each half). Not for 3xTF32: rows G-1-i come out
  // as E - O, and that difference magnifies the tensor cores' accumulation
  // error (2.1e-4 instead of 5e-5 at G = 256).
  w.halves = G % 256 == 0 && precision != FX_DCT_FP32;
  {
    int sp = precision == FX_DCT_SIMT ? sgemm_splits(G, d->ctx->num_sms) : 1;
    if (w.halves && precision == FX_DCT_SIMT) sp = std::max(sp, half_splits(G, d->ctx->num_sms));
    if (sp > 1 || w.halves) FX_TRY(w.split_ws.alloc((size_t)sp * cells));
  }
  const bool split_fmt = precision == FX_DCT_FP32, bf_fmt = precision == FX_DCT_BF16;
  if (w.halves) {
    FX_TRY(w.c_h.alloc(cells / 2));
    FX_TRY(w.ct_h.alloc(cells / 2));
    FX_TRY(w.dx_h.alloc(cells / 2));
    FX_TRY(w.dy_h.alloc(cells / 2));
    for (int i = 0; i < 3; ++i) FX_TRY(w.hw[i].alloc(cells));
    if (split_fmt) {
      FX_TRY(w.c_h_lo.alloc(cells / 2));
      FX_TRY(w.ct_h_lo.alloc(cells / 2));
      FX_TRY(w.dx_h_lo.alloc(cells / 2));
      FX_TRY(w.dy_h_lo.alloc(cells / 2));
      for (int i = 0; i < 3; ++i) FX_TRY(w.hw_lo[i].alloc(cells));
    }
    if (bf_fmt) {
      FX_TRY(w.c_h_bf.alloc(cells / 2));
      FX_TRY(w.ct_h_bf.alloc(cells / 2));
      FX_TRY(w.dx_h_bf.alloc(cells / 2));
      FX_TRY(w.dy_h_bf.alloc(cells / 2));
      for (int i = 0; i < 3; ++i) FX_TRY(w.hw_bf[i].alloc(cells));
    }
  }
  const bool split = precision == FX_DCT_FP32, half = precision == FX_DCT_BF16;
  if (split) {
    FX_TRY(w.cmat_lo.alloc(cells));
    FX_TRY(w.cmat_t_lo.alloc(cells));
    FX_TRY(w.dxct_lo.alloc(cells));
    FX_TRY(w.dyct_lo.alloc(cells));
    for (int i = 0; i < 4; ++i) FX_TRY(w.lo[i].alloc(cells));
  }
  if (half) {
    FX_TRY(w.cmat_bf.alloc(cells));
    FX_TRY(w.cmat_t_bf.alloc(cells));
    FX_TRY(w.dxct_bf.alloc(cells));
    FX_TRY(w.dyct_bf.alloc(cells));
    for (int i = 0; i < 3; ++i) FX_TRY(w.bf[i].alloc(cells));
  }
  const double pi = 3.14159265358979323846;
  std::vector<double> c(cells), ct(cells), dx(cells), dy(cells);
  for (int k = 0; k < G; ++k) {
    const double sk = k == 0 ? std::sqrt(1.0 / G) : std::sqrt(2.0 / G);
    for (int n = 0; n < G; ++n) {
      const double v = sk * std::cos(pi * (2.0 * n + 1.0) * k / (2.0 * G));
      c[(size_t)k * G + n] = v;
      ct[(size_t)n * G + k] = v;
    }
  }
  // wx = 1/bw with bw = die/G (force_electrostatic.py:126-128).
  const double bw = (double)(d->chip_w / (float)G), bh = (double)(d->chip_h / (float)G);
  const double wx = 1.0 / bw, wy = 1.0 / bh;
  // (D C^T)[i][k] = sum_j D[i][j] C[k][j] with the two-point stencils.
  auto stencil = [&](double wgt, std::vector<double> &out) {
    for (int i = 0; i < G; ++i)
      for (int k = 0; k < G; ++k) {
        const double *ck = &c[(size_t)k * G];
        double v;
        if (i == 0)
          v = -(ck[1] - ck[0]) * wgt;
        else if (i == G - 1)
          v = -(ck[G - 1] - ck[G - 2]) * wgt;
        else
          v = -(ck[i + 1] - ck[i - 1]) * wgt * 0.5;
        out[(size_t)i * G + k] = v;
      }
  };
  stencil(wx, dx);
  stencil(wy, dy);
  std::vector<float> ie(cells);
  for (int ky = 0; ky < G; ++ky)
    for (int kx = 0; kx < G; ++kx) {
      const double ax = wx * std::cos(pi * kx / G) - wx;
      const double ay = wy * std::cos(pi * ky / G) - wy;
      double lam = ax * ax + ay * ay;
      if (kx == 0 && ky == 0) lam = 1.0;
      ie[(size_t)ky * G + kx] = (kx == 0 && ky == 0) ? 0.0f : (float)(-1.0 / lam);
    }
  FX_CHECK_CUDA(cudaMemcpyAsync(w.inv_eig.p, ie.data(), cells * 4, cudaMemcpyHostToDevice, s));
  // FX_DCT_I8: the operators' 8-bit slices, cut from their FP64 values (7
  // bits of each row's scale per slice), in the order [s1 ..] along NS K
  // columns, for rows x K operators (the full G x G ones, or the 2 x (G/2) x
  // (G/2) half operators below)
  auto slice_op = [&](const std::vector<double> &m, int rows, int K, int o) -> int {
    const int NS = i8_slices();
    std::vector<int8_t> sl((size_t)NS * rows * K);
    std::vector<float> sc(rows);
    for (int i = 0; i < rows; ++i) {
      double mx = 0.0;
      for (int k = 0; k < K; ++k) mx = std::max(mx, std::fabs(m[(size_t)i * K + k]));
      int e = 0;
      if (mx > 0.0) std::frexp(mx, &e);
      sc[i] = std::ldexp(1.0f, e);
      for (int k = 0; k < K; ++k) {
        double a = std::ldexp(m[(size_t)i * K + k], -e);
        for (int t = 0; t < NS; ++t) {
          const double q = a * 128.0;
          const double tr = std::trunc(q);
          sl[(size_t)i * NS * K + (size_t)t * K + k] = (int8_t)tr;
          a = q - tr;
        }
      }
    }
    FX_TRY(w.op8[o].alloc(sl.size()));
    FX_TRY(w.op_sc[o].alloc(rows));
    FX_CHECK_CUDA(cudaMemcpyAsync(w.op8[o].p, sl.data(), sl.size(), cudaMemcpyHostToDevice, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(w.op_sc[o].p, sc.data(), (size_t)rows * 4,
                                  cudaMemcpyHostToDevice, s));
    FX_CHECK_CUDA(cudaStreamSynchronize(s));  // sl and sc go out of scope
    return FX_OK;
  };
  if (precision == FX_DCT_I8) {
    for (int i = 0; i < 2; ++i) {  // data slices: G x NS G (or 2G x NS G/2)
      FX_TRY(w.d8[i].alloc((size_t)i8_slices() * cells));
      FX_TRY(w.d_sc[i].alloc(2 * (size_t)G));
    }
    if (!w.halves) {
      FX_TRY(slice_op(c, G, G, 0));
      FX_TRY(slice_op(ct, G, G, 1));
      FX_TRY(slice_op(dx, G, G, 2));
      FX_TRY(slice_op(dy, G, G, 3));
    }
  }
  FX_TRY(upload_operand(c, precision, w.cmat.p, split ? w.cmat_lo.p : nullptr,
                        half ? w.cmat_bf.p : nullptr, s));
  FX_TRY(upload_operand(ct, precision, w.cmat_t.p, split ? w.cmat_t_lo.p : nullptr,
                        half ? w.cmat_t_bf.p : nullptr, s));
  FX_TRY(upload_operand(dx, precision, w.dxct.p, split ? w.dxct_lo.p : nullptr,
                        half ? w.dxct_bf.p : nullptr, s));
  FX_TRY(upload_operand(dy, precision, w.dyct.p, split ? w.dyct_lo.p : nullptr,
                        half ? w.dyct_bf.p : nullptr, s));
  if (w.halves) {
    // [rows 2r | rows 2r+1] of C, first G/2 columns (C's columns mirror);
    // [columns 2m | columns 2m+1] of C^T, Dx C^T, Dy C^T, first G/2 rows
    // (their rows mirror): exact slices of the FP64 operators
    const int h = G / 2;
    const size_t hh = (size_t)h * h;
    std::vector<double> chh(2 * hh), cth(2 * hh), dxh(2 * hh), dyh(2 * hh);
    for (int r = 0; r < h; ++r)
      for (int k = 0; k < h; ++k) {
        chh[(size_t)r * h + k] = c[(size_t)(2 * r) * G + k];
        chh[hh + (size_t)r * h + k] = c[(size_t)(2 * r + 1) * G + k];
        cth[(size_t)r * h + k] = ct[(size_t)r * G + 2 * k];
        cth[hh + (size_t)r * h + k] = ct[(size_t)r * G + 2 * k + 1];
        dxh[(size_t)r * h + k] = dx[(size_t)r * G + 2 * k];
        dxh[hh + (size_t)r * h + k] = dx[(size_t)r * G + 2 * k + 1];
        dyh[(size_t)r * h + k] = dy[(size_t)r * G + 2 * k];
        dyh[hh + (size_t)r * h + k] = dy[(size_t)r * G + 2 * k + 1];
      }
    FX_TRY(upload_operand(chh, precision, w.c_h.p, split_fmt ? w.c_h_lo.p : nullptr,
                          bf_fmt ? w.c_h_bf.p : nullptr, s));
    FX_TRY(upload_operand(cth, precision, w.ct_h.p, split_fmt ? w.ct_h_lo.p : nullptr,
                          bf_fmt ? w.ct_h_bf.p : nullptr, s));
    FX_TRY(upload_operand(dxh, precision, w.dx_h.p, split_fmt ? w.dx_h_lo.p : nullptr,
                          bf_fmt ? w.dx_h_bf.p : nullptr, s));
    FX_TRY(upload_operand(dyh, precision, w.dy_h.p, split_fmt ? w.dy_h_lo.p : nullptr,
                          bf_fmt ? w.dy_h_bf.p : nullptr, s));
    if (precision == FX_DCT_I8) {  // the two halves of each, as 2h rows of h
      FX_TRY(slice_op(chh, 2 * h, h, 0));
      FX_TRY(slice_op(cth, 2 * h, h, 1));
      FX_TRY(slice_op(dxh, 2 * h, h, 2));
      FX_TRY(slice_op(dyh, 2 * h, h, 3));
    }
  }
  FX_CHECK_CUDA(cudaMemsetAsync(w.area_fx.p, 0, cells * 8, s));
  FX_CHECK_CUDA(cudaMemsetAsync(w.energy.p, 0, (4096 + 8) * 8, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  w.G = G;
  w.precision = precision;
  return FX_OK;
}

// Scatter of the given positions into the area accumulator.
int density_scatter(fx_ctx *ctx, fx_design *d, const float *x, const float *y,
                    int G, int precision, cudaStream_t s) {
  FX_TRY(dens_setup(d, G, precision, s));
  // The accumulator may still hold the scatter of a previous call's final
  // positions: start from zero.
  FX_CHECK_CUDA(cudaMemsetAsync(d->dens.area_fx.p, 0, (size_t)G * G * 8, s));
  const float bw = d->chip_w / (float)G, bh = d->chip_h / (float)G;
  int nb = (d->n + 255) / 256;
  if (nb > ctx->num_sms * 8) nb = ctx->num_sms * 8;
  dens_scatter_kernel<<<nb, 256, 0, s>>>(x, y, d->area.p, d->n, G, bw, bh,
                                         d->dens.area_fx.p);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

// Charge grid -> spectrum -> field (and the potential when need_phi), from
// the accumulated areas (which are consumed and re-armed). Seven NT GEMMs
// D = A B^T on G x G matrices, A always a constant operator:
//   T1^T = C rho^T ; phi_hat = (C T1) * (-1/lambda) ;
//   T3^T = C^T phi_hat^T ; E_y = (Dy C^T) T3 ;
//   T4^T = (Dx C^T) phi_hat^T ; E_x = C^T T4 ; [phi = C^T T3].
int density_run(fx_ctx *ctx, fx_design *d, int G, float target, float weight,
                int precision, bool need_phi, cudaStream_t s) {
  (void)weight;
  FX_TRY(dens_setup(d, G, precision, s));
  DensityWork &w = d->dens;
  const int cells = G * G;
  const float bw = d->chip_w / (float)G, bh = d->chip_h / (float)G;
  const double inv_bin_area = 1.0 / ((double)bw * (double)bh);
  cudaEvent_t ev;
  timer_begin(ctx, FX_STAGE_DENSITY, s, &ev);
  const int eb = ctx->num_sms * 8;
  // Split (3xTF32) and bf16 operand copies exist only for their precision.
  const bool split = precision == FX_DCT_FP32, half = precision == FX_DCT_BF16;
  auto LO = [&](int i) { return split ? w.lo[i].p : nullptr; };
  auto BF = [&](int i) { return half ? w.bf[i].p : nullptr; };
  auto K = [&](float *f, float *l, uint16_t *b) {
    return GemmOperands{f, split ? l : nullptr, half ? b : nullptr};
  };
  dens_charge_kernel<<<(cells + 1023) / 1024, 256, 0, s>>>(
      w.area_fx.p, cells, inv_bin_area, target, w.buf[0].p, LO(2), BF(0));
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  float *WS = precision == FX_DCT_SIMT ? w.split_ws.p : nullptr;
  if (precision == FX_DCT_I8 && !w.halves) {
    // the same seven products; each data operand is sliced once and kept
    // while later products read it (phat and T3 twice)
    float *rho = w.buf[0].p, *t1 = w.buf[1].p, *phat = w.buf[2].p, *t3 = w.buf[1].p;
    float *t4 = w.buf[4].p;
    auto slice = [&](const float *X, int i) {
      return i8_slice(ctx, X, G, G, w.d8[i].p, w.d_sc[i].p, s);
    };
    auto mm = [&](int op, int i, const float *S, float *D) {
      return gemm_nt_i8(ctx, G, w.op8[op].p, w.op_sc[op].p, w.d8[i].p, w.d_sc[i].p, S, D, s);
    };
    FX_TRY(slice(rho, 0));
    FX_TRY(mm(0, 0, nullptr, t1));              // T1^T = C rho^T
    FX_TRY(slice(t1, 0));
    FX_TRY(mm(0, 0, w.inv_eig.p, phat));        // phi_hat = (C T1) * (-1/lambda)
    FX_TRY(slice(phat, 1));
    FX_TRY(mm(1, 1, nullptr, t3));              // T3^T = C^T phi_hat^T
    FX_TRY(slice(t3, 0));
    FX_TRY(mm(3, 0, nullptr, w.ey.p));          // E_y = (Dy C^T) T3
    if (need_phi) FX_TRY(mm(1, 0, nullptr, w.buf[3].p));  // phi = C^T T3
    FX_TRY(mm(2, 1, nullptr, t4));              // T4^T = (Dx C^T) phi_hat^T
    FX_TRY(slice(t4, 0));
    FX_TRY(mm(1, 0, nullptr, w.ex.p));          // E_x = C^T T4
    timer_end(ctx, FX_STAGE_DENSITY, s, ev);
    return FX_OK;
  }
  if (w.halves) {
    // each product as two half-size GEMMs on the folded or split operand;
    // products come back as f32 and the folds write the GEMM formats
    auto H = [&](int i) {
      return GemmOperands{w.hw[i].p, split ? w.hw_lo[i].p : nullptr,
                          half ? w.hw_bf[i].p : nullptr};
    };
    auto fold = [&](const float *B, const GemmOperands &o) {
      dct_fold_kernel<<<eb, 256, 0, s>>>(B, G, o.f32, o.lo, o.bf);
      ctx->launches += 1;
    };
    auto split_k = [&](const float *B, const GemmOperands &o) {
      dct_split_kernel<<<eb, 256, 0, s>>>(B, G, o.f32, o.lo, o.bf);
      ctx->launches += 1;
    };
    const GemmOperands Ch = K(w.c_h.p, w.c_h_lo.p, w.c_h_bf.p);
    const GemmOperands Cth = K(w.ct_h.p, w.ct_h_lo.p, w.ct_h_bf.p);
    const GemmOperands Dxh = K(w.dx_h.p, w.dx_h_lo.p, w.dx_h_bf.p);
    const GemmOperands Dyh = K(w.dy_h.p, w.dy_h_lo.p, w.dy_h_bf.p);
    float *rho = w.buf[0].p, *t1 = w.buf[1].p, *phat = w.buf[2].p, *t3 = w.buf[1].p;
    float *t4 = w.buf[4].p, *phi = w.buf[3].p;
    float *P = w.split_ws.p;
    if (precision == FX_DCT_I8) {
      // the same products from 8-bit slices; each folded or split operand
      // is sliced by its product (into d8[0] / d_sc[0])
      auto hm = [&](int op, int i, int mode, float sign, const float *S, float *D) {
        return gemm_half_i8(ctx, G, w.op8[op].p, w.op_sc[op].p, w.hw[i].p, mode, sign, S, D, P,
                            w.d8[0].p, w.d_sc[0].p, s);
      };
      fold(rho, H(0));
      FX_TRY(hm(0, 0, kHalfRows, 1.f, nullptr, t1));
      fold(t1, H(0));
      FX_TRY(hm(0, 0, kHalfRows, 1.f, w.inv_eig.p, phat));
      split_k(phat, H(1));
      FX_TRY(hm(1, 1, kHalfPair, 1.f, nullptr, t3));
      split_k(t3, H(2));
      FX_TRY(hm(3, 2, kHalfPair, -1.f, nullptr, w.ey.p));
      if (need_phi) FX_TRY(hm(1, 2, kHalfPair, 1.f, nullptr, phi));
      FX_TRY(hm(2, 1, kHalfPair, -1.f, nullptr, t4));
      split_k(t4, H(0));
      FX_TRY(hm(1, 0, kHalfPair, 1.f, nullptr, w.ex.p));
      FX_CHECK_LAUNCH();
      timer_end(ctx, FX_STAGE_DENSITY, s, ev);
      return FX_OK;
    }
    fold(rho, H(0));
    FX_TRY(gemm_half(ctx, precision, G, Ch, H(0), kHalfRows, 1.f, nullptr, t1, P, s));
    fold(t1, H(0));
    FX_TRY(gemm_half(ctx, precision, G, Ch, H(0), kHalfRows, 1.f, w.inv_eig.p, phat, P, s));
    split_k(phat, H(1));
    FX_TRY(gemm_half(ctx, precision, G, Cth, H(1), kHalfPair, 1.f, nullptr, t3, P, s));
    split_k(t3, H(2));
    FX_TRY(gemm_half(ctx, precision, G, Dyh, H(2), kHalfPair, -1.f, nullptr, w.ey.p, P, s));
    if (need_phi)
      FX_TRY(gemm_half(ctx, precision, G, Cth, H(2), kHalfPair, 1.f, nullptr, phi, P, s));
    FX_TRY(gemm_half(ctx, precision, G, Dxh, H(1), kHalfPair, -1.f, nullptr, t4, P, s));
    split_k(t4, H(0));
    FX_TRY(gemm_half(ctx, precision, G, Cth, H(0), kHalfPair, 1.f, nullptr, w.ex.p, P, s));
    FX_CHECK_LAUNCH();
    timer_end(ctx, FX_STAGE_DENSITY, s, ev);
    return FX_OK;
  }
  const GemmOperands C = K(w.cmat.p, w.cmat_lo.p, w.cmat_bf.p);
  const GemmOperands Ct = K(w.cmat_t.p, w.cmat_t_lo.p, w.cmat_t_bf.p);
  const GemmOperands DxCt = K(w.dxct.p, w.dxct_lo.p, w.dxct_bf.p);
  const GemmOperands DyCt = K(w.dyct.p, w.dyct_lo.p, w.dyct_bf.p);
  const GemmOperands rho{w.buf[0].p, LO(2), BF(0)};
  const GemmOperands t1{w.buf[1].p, LO(1), BF(1)};
  const GemmOperands phat{w.buf[2].p, LO(0), BF(0)};
  const GemmOperands t3{w.buf[1].p, LO(1), BF(1)};
  const GemmOperands t4{w.buf[4].p, LO(3), BF(2)};
  const GemmOperands ex{w.ex.p, nullptr, nullptr};
  const GemmOperands ey{w.ey.p, nullptr, nullptr};
  const GemmOperands phi{w.buf[3].p, nullptr, nullptr};
  FX_TRY(gemm_nt(ctx, precision, G, C, rho, nullptr, t1, s, WS));
  FX_TRY(gemm_nt(ctx, precision, G, C, t1, w.inv_eig.p, phat, s, WS));
  FX_TRY(gemm_nt(ctx, precision, G, Ct, phat, nullptr, t3, s, WS));
  FX_TRY(gemm_nt(ctx, precision, G, DyCt, t3, nullptr, ey, s, WS));
  if (need_phi) FX_TRY(gemm_nt(ctx, precision, G, Ct, t3, nullptr, phi, s, WS));
  FX_TRY(gemm_nt(ctx, precision, G, DxCt, phat, nullptr, t4, s, WS));
  FX_TRY(gemm_nt(ctx, precision, G, Ct, t4, nullptr, ex, s, WS));
  timer_end(ctx, FX_STAGE_DENSITY, s, ev);
  return FX_OK;
}

int density_gather(fx_ctx *ctx, fx_design *d, const float *x, const float *y,
                   int G, float weight, cudaStream_t s) {
  DensityWork &w = d->dens;
  const float bw = d->chip_w / (float)G, bh = d->chip_h / (float)G;
  int nb = (d->n + 255) / 256;
  if (nb > 4096) nb = 4096;
  dens_gather_kernel<<<nb, 256, 0, s>>>(x, y, d->area.p, d->n, G, bw, bh,
                                        weight, w.ex.p, w.ey.p, w.buf[3].p,
                                        w.force.p, w.energy.p, (unsigned int *)(w.energy.p + 4096),
                                        w.energy.p + 4097);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

}  // namespace fx

using namespace fx;

extern "C" int fx_stage_density(fx_ctx *ctx, fx_design *d, int32_t bins,
                                float target_density, float weight,
                                int32_t precision, float *out_fx,
                                float *out_fy, float *out_rho, float *out_phi,
                                float *out_ex, float *out_ey,
                                double *out_energy) {
  if (!ctx || !d || bins < 128 || bins % 128 != 0 || bins > 8192 ||
      precision < FX_DCT_FP32 || precision > FX_DCT_I8) {
    set_error("fx_stage_density: invalid arguments (bins must be a multiple of 128)");
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream;
  const float *x = d->x[d->cur].p, *y = d->y[d->cur].p;
  FX_TRY(density_scatter(ctx, d, x, y, bins, precision, s));
  FX_TRY(density_run(ctx, d, bins, target_density, weight, precision, true, s));
  FX_TRY(density_gather(ctx, d, x, y, bins, weight, s));
  DensityWork &w = d->dens;
  const size_t cells = (size_t)bins * bins, n = (size_t)d->n;
  std::vector<float2> f(n);
  double e = 0.0;
  FX_CHECK_CUDA(cudaMemcpyAsync(f.data(), w.force.p, n * 8, cudaMemcpyDeviceToHost, s));
  std::vector<float> rho_lo;
  if (out_rho) FX_CHECK_CUDA(cudaMemcpyAsync(out_rho, w.buf[0].p, cells * 4, cudaMemcpyDeviceToHost, s));
  if (out_rho && precision == FX_DCT_FP32) {
    rho_lo.resize(cells);
    FX_CHECK_CUDA(cudaMemcpyAsync(rho_lo.data(), w.lo[2].p, cells * 4, cudaMemcpyDeviceToHost, s));
  }
  if (out_phi) FX_CHECK_CUDA(cudaMemcpyAsync(out_phi, w.buf[3].p, cells * 4, cudaMemcpyDeviceToHost, s));
  if (out_ex) FX_CHECK_CUDA(cudaMemcpyAsync(out_ex, w.ex.p, cells * 4, cudaMemcpyDeviceToHost, s));
  if (out_ey) FX_CHECK_CUDA(cudaMemcpyAsync(out_ey, w.ey.p, cells * 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(&e, w.energy.p + 4097, 8, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  unsigned int tc_err = 0;
  FX_TRY(gemm_tc_error(ctx, &tc_err, s));
  if (tc_err) {
    set_error("tensor-core GEMM: a bounded wait expired (error word %u)", tc_err);
    return FX_ETIMEOUT;
  }
  for (size_t i = 0; i < n; ++i) {
    if (out_fx) out_fx[i] = f[i].x;
    if (out_fy) out_fy[i] = f[i].y;
  }
  for (size_t i = 0; i < rho_lo.size(); ++i) out_rho[i] += rho_lo[i];
  if (out_energy) *out_energy = e;
  return FX_OK;
}
