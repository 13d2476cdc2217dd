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
//   field        centred differences inside, one-sided at edges  (:91-103)
//   force        F_i = area_i * E[row, col] * weight             (:134-150)
// C is the orthonormal DCT-II matrix (G x G). The four transforms are NT
// GEMMs D = A * B^T with A in {C, C^T} (constant) and B the data produced by
// the previous stage:
//   T1^T = C * rho^T ; rho_hat = C * T1 (epilogue: * -1/lambda) ;
//   T3^T = C^T * phi_hat^T ; phi = C^T * T3.
// Bin areas are accumulated as 64-bit fixed point so the density is exact
// and independent of the scatter order.
#include <cmath>

#include "fx_internal.h"
#include "fx_device.cuh"
#include "fx_gemm.cuh"

namespace fx {

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
__global__ void dens_charge_kernel(unsigned long long *__restrict__ acc,
                                   int cells, double inv_bin_area,
                                   float target, float *__restrict__ rho,
                                   float *__restrict__ rho_lo,
                                   uint16_t *__restrict__ rho_bf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cells;
       i += gridDim.x * blockDim.x) {
    const double a = (double)acc[i] * (1.0 / kAreaScale) * inv_bin_area;
    const float v = (float)(a - (double)target);
    acc[i] = 0ull;
    store_operand(v, i, rho, rho_lo, rho_bf);
  }
}

// E = -grad(phi) with the reference's stencils (force_electrostatic.py:
// 96-103), evaluated in f32 in the same operation order.
__global__ void dens_field_kernel(const float *__restrict__ phi, int G,
                                  float wx, float wy, float *__restrict__ ex,
                                  float *__restrict__ ey) {
  const int cells = G * G;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cells;
       i += gridDim.x * blockDim.x) {
    const int r = i / G, c = i - r * G;
    float e;
    if (c == 0)
      e = -__fmul_rn(__fsub_rn(phi[i + 1], phi[i]), wx);
    else if (c == G - 1)
      e = -__fmul_rn(__fsub_rn(phi[i], phi[i - 1]), wx);
    else
      e = __fmul_rn(__fmul_rn(-__fsub_rn(phi[i + 1], phi[i - 1]), wx), 0.5f);
    ex[i] = e;
    if (r == 0)
      e = -__fmul_rn(__fsub_rn(phi[i + G], phi[i]), wy);
    else if (r == G - 1)
      e = -__fmul_rn(__fsub_rn(phi[i], phi[i - G]), wy);
    else
      e = __fmul_rn(__fmul_rn(-__fsub_rn(phi[i + G], phi[i - G]), wy), 0.5f);
    ey[i] = e;
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

// Host: DCT matrices and the inverse eigenvalues, in FP64 then rounded.
static int dens_setup(fx_design *d, int G, int precision, cudaStream_t s) {
  DensityWork &w = d->dens;
  if (w.G == G && w.precision == precision && w.cmat.p) return FX_OK;
  const size_t cells = (size_t)G * G;
  FX_TRY(w.area_fx.alloc(cells));
  FX_TRY(w.cmat.alloc(cells));
  FX_TRY(w.cmat_t.alloc(cells));
  FX_TRY(w.inv_eig.alloc(cells));
  for (int i = 0; i < 4; ++i) FX_TRY(w.buf[i].alloc(cells));
  FX_TRY(w.ex.alloc(cells));
  FX_TRY(w.ey.alloc(cells));
  FX_TRY(w.energy.alloc(4096 + 8));
  FX_TRY(w.force.alloc((size_t)d->n));
  if (precision == FX_DCT_FP32) {
    FX_TRY(w.cmat_lo.alloc(cells));
    FX_TRY(w.cmat_t_lo.alloc(cells));
    for (int i = 0; i < 3; ++i) FX_TRY(w.lo[i].alloc(cells));
  }
  if (precision == FX_DCT_BF16) {
    FX_TRY(w.cmat_bf.alloc(cells));
    FX_TRY(w.cmat_t_bf.alloc(cells));
    FX_TRY(w.bf[0].alloc(cells));
    FX_TRY(w.bf[1].alloc(cells));
  }
  std::vector<float> c(cells), ct(cells), ie(cells);
  std::vector<float> clo, ctlo;
  std::vector<uint16_t> cbf, ctbf;
  const double pi = 3.14159265358979323846;
  for (int k = 0; k < G; ++k) {
    const double sk = k == 0 ? std::sqrt(1.0 / G) : std::sqrt(2.0 / G);
    for (int n = 0; n < G; ++n) {
      const float v = (float)(sk * std::cos(pi * (2.0 * n + 1.0) * k / (2.0 * G)));
      c[(size_t)k * G + n] = v;
      ct[(size_t)n * G + k] = v;
    }
  }
  // wx = 1/bw with bw = die/G (force_electrostatic.py:126-128).
  const double bw = (double)(d->chip_w / (float)G), bh = (double)(d->chip_h / (float)G);
  const double wx = 1.0 / bw, wy = 1.0 / bh;
  for (int ky = 0; ky < G; ++ky)
    for (int kx = 0; kx < G; ++kx) {
      const double ax = wx * std::cos(pi * kx / G) - wx;
      const double ay = wy * std::cos(pi * ky / G) - wy;
      double lam = ax * ax + ay * ay;
      if (kx == 0 && ky == 0) lam = 1.0;
      ie[(size_t)ky * G + kx] = (kx == 0 && ky == 0) ? 0.0f : (float)(-1.0 / lam);
    }
  FX_CHECK_CUDA(cudaMemcpyAsync(w.cmat.p, c.data(), cells * 4, cudaMemcpyHostToDevice, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(w.cmat_t.p, ct.data(), cells * 4, cudaMemcpyHostToDevice, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(w.inv_eig.p, ie.data(), cells * 4, cudaMemcpyHostToDevice, s));
  if (precision == FX_DCT_FP32) {
    // 3xTF32: cmat holds the TF32 head of C, cmat_lo the exact residual.
    clo.resize(cells);
    ctlo.resize(cells);
    for (int k = 0; k < G; ++k)
      for (int n = 0; n < G; ++n) {
        const float v = c[(size_t)k * G + n];
        const float h = tf32_hi_host(v);
        c[(size_t)k * G + n] = h;
        ct[(size_t)n * G + k] = h;
        clo[(size_t)k * G + n] = v - h;
        ctlo[(size_t)n * G + k] = v - h;
      }
    FX_CHECK_CUDA(cudaMemcpyAsync(w.cmat.p, c.data(), cells * 4, cudaMemcpyHostToDevice, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(w.cmat_t.p, ct.data(), cells * 4, cudaMemcpyHostToDevice, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(w.cmat_lo.p, clo.data(), cells * 4, cudaMemcpyHostToDevice, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(w.cmat_t_lo.p, ctlo.data(), cells * 4, cudaMemcpyHostToDevice, s));
  }
  if (precision == FX_DCT_BF16) {
    cbf.resize(cells);
    ctbf.resize(cells);
    for (size_t i = 0; i < cells; ++i) {
      cbf[i] = bf16_host(c[i]);
      ctbf[i] = bf16_host(ct[i]);
    }
    FX_CHECK_CUDA(cudaMemcpyAsync(w.cmat_bf.p, cbf.data(), cells * 2, cudaMemcpyHostToDevice, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(w.cmat_t_bf.p, ctbf.data(), cells * 2, cudaMemcpyHostToDevice, s));
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

// Charge grid -> phi -> field, from the accumulated areas (which are
// consumed and re-armed).
int density_run(fx_ctx *ctx, fx_design *d, int G, float target, float weight,
                int precision, cudaStream_t s) {
  (void)weight;
  FX_TRY(dens_setup(d, G, precision, s));
  DensityWork &w = d->dens;
  const int cells = G * G;
  const float bw = d->chip_w / (float)G, bh = d->chip_h / (float)G;
  const double inv_bin_area = 1.0 / ((double)bw * (double)bh);
  cudaEvent_t ev;
  timer_begin(ctx, FX_STAGE_DENSITY, s, &ev);
  const int eb = ctx->num_sms * 8;
  float *rho = w.buf[0].p, *t1 = w.buf[1].p, *phat = w.buf[2].p, *t3 = w.buf[1].p;
  float *phi = w.buf[3].p;
  // Split (3xTF32) and bf16 operand copies exist only for their precision.
  const bool split = precision == FX_DCT_FP32, half = precision == FX_DCT_BF16;
  auto LO = [&](int i) { return split ? w.lo[i].p : nullptr; };
  auto BF = [&](int i) { return half ? w.bf[i].p : nullptr; };
  dens_charge_kernel<<<eb, 256, 0, s>>>(w.area_fx.p, cells, inv_bin_area, target,
                                        rho, LO(2), BF(0));
  FX_CHECK_LAUNCH();
  GemmOperands A{w.cmat.p, split ? w.cmat_lo.p : nullptr, half ? w.cmat_bf.p : nullptr};
  GemmOperands At{w.cmat_t.p, split ? w.cmat_t_lo.p : nullptr,
                  half ? w.cmat_t_bf.p : nullptr};
  GemmOperands B0{rho, LO(2), BF(0)};
  GemmOperands B1{t1, LO(1), BF(1)};
  GemmOperands B2{phat, LO(0), BF(0)};
  GemmOperands B3{t3, LO(1), BF(1)};
  // T1^T = C rho^T
  FX_TRY(gemm_nt(ctx, precision, G, A, B0, nullptr, B1, s));
  // rho_hat = C T1, epilogue * (-1/lambda) -> phi_hat
  FX_TRY(gemm_nt(ctx, precision, G, A, B1, w.inv_eig.p, B2, s));
  // T3^T = C^T phi_hat^T
  FX_TRY(gemm_nt(ctx, precision, G, At, B2, nullptr, B3, s));
  // phi = C^T T3
  GemmOperands P{phi, nullptr, nullptr};
  FX_TRY(gemm_nt(ctx, precision, G, At, B3, nullptr, P, s));
  dens_field_kernel<<<eb, 256, 0, s>>>(phi, G, (float)(1.0 / (double)bw),
                                       (float)(1.0 / (double)bh), w.ex.p, w.ey.p);
  FX_CHECK_LAUNCH();
  ctx->launches += 2;
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
      precision < FX_DCT_FP32 || precision > FX_DCT_SIMT) {
    set_error("fx_stage_density: invalid arguments (bins must be a multiple of 128)");
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const float *x = d->x[d->cur].p, *y = d->y[d->cur].p;
  FX_TRY(density_scatter(ctx, d, x, y, bins, precision, s));
  FX_TRY(density_run(ctx, d, bins, target_density, weight, precision, s));
  FX_TRY(density_gather(ctx, d, x, y, bins, weight, s));
  DensityWork &w = d->dens;
  const size_t cells = (size_t)bins * bins, n = (size_t)d->n;
  std::vector<float2> f(n);
  double e = 0.0;
  FX_CHECK_CUDA(cudaMemcpyAsync(f.data(), w.force.p, n * 8, cudaMemcpyDeviceToHost, s));
  if (out_rho) FX_CHECK_CUDA(cudaMemcpyAsync(out_rho, w.buf[0].p, cells * 4, cudaMemcpyDeviceToHost, s));
  if (out_phi) FX_CHECK_CUDA(cudaMemcpyAsync(out_phi, w.buf[3].p, cells * 4, cudaMemcpyDeviceToHost, s));
  if (out_ex) FX_CHECK_CUDA(cudaMemcpyAsync(out_ex, w.ex.p, cells * 4, cudaMemcpyDeviceToHost, s));
  if (out_ey) FX_CHECK_CUDA(cudaMemcpyAsync(out_ey, w.ey.p, cells * 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(&e, w.energy.p + 4097, 8, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  for (size_t i = 0; i < n; ++i) {
    if (out_fx) out_fx[i] = f[i].x;
    if (out_fy) out_fy[i] = f[i].y;
  }
  if (out_energy) *out_energy = e;
  return FX_OK;
}
