// fx_attract.cu -- rows A + E: net-spring attraction as a CSR segmented
// reduction, fused with the Barnes-Hut and density forces and the damped
// Euler step; plus the plain composite iteration driver.
//
// Attraction follows place_gates_in_leaf (H/src/algorithm/placer.rs:243-255)
// over the full deduplicated adjacency (circuit.rs:154-171):
//   F_i = k * sum_{j in adj(i)} (p_j - p_i).
// Eight lanes own one gate: they read its adjacency row with coalesced
// loads, gather neighbour positions (L2-resident) and combine their partial
// sums with a fixed shuffle tree, so no float atomics are involved and the
// result does not depend on scheduling.
// The step follows placer.rs:275-280 exactly (no contraction):
//   v = (v + F*dt) * damping ; p = clamp(p + v*dt, lo, hi).
#include "fx_internal.h"
#include "fx_device.cuh"

namespace fx {

int bh_bbox(fx_ctx *ctx, fx_design *d, const float *x, const float *y,
            cudaStream_t s);
int density_scatter(fx_ctx *ctx, fx_design *d, const float *x, const float *y,
                    int G, int precision, cudaStream_t s);

constexpr int kLanes = 8;
constexpr int kStepThreads = 256;

template <int L>
__device__ __forceinline__ float2 spring_sum(const int32_t *__restrict__ adj_ptr,
                                             const int32_t *__restrict__ adj_idx,
                                             const float *__restrict__ x,
                                             const float *__restrict__ y,
                                             int g, bool valid, int sub) {
  float sx = 0.f, sy = 0.f;
  if (valid) {
    const float xi = x[g], yi = y[g];
    const int b = __ldg(adj_ptr + g), e = __ldg(adj_ptr + g + 1);
    for (int q = b + sub; q < e; q += L) {
      const int j = __ldg(adj_idx + q);
      sx += __fsub_rn(__ldg(x + j), xi);
      sy += __fsub_rn(__ldg(y + j), yi);
    }
  }
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o, L);
    sy += __shfl_xor_sync(0xffffffffu, sy, o, L);
  }
  return make_float2(sx, sy);
}

__global__ void __launch_bounds__(kStepThreads)
attract_kernel(const int32_t *__restrict__ adj_ptr,
               const int32_t *__restrict__ adj_idx, const float *__restrict__ x,
               const float *__restrict__ y, int n, float k,
               float2 *__restrict__ out) {
  const int per_block = kStepThreads / kLanes;
  const int sub = threadIdx.x % kLanes;
  for (int base = blockIdx.x * per_block; base < n; base += gridDim.x * per_block) {
    const int g = base + threadIdx.x / kLanes;
    const bool valid = g < n;
    const float2 s = spring_sum<kLanes>(adj_ptr, adj_idx, x, y, g, valid, sub);
    if (valid && sub == 0) out[g] = make_float2(__fmul_rn(k, s.x), __fmul_rn(k, s.y));
  }
}

struct StepArgs {
  const int32_t *adj_ptr, *adj_idx;
  const float *x, *y;
  float *xn, *yn, *vx, *vy;
  int n;
  float k;
  const float2 *fbh;  // Barnes-Hut force or null
  // density force (ex == null: off)
  const float *ex, *ey, *phi, *area;
  int G;
  float bw, bh, dweight;
  // integrate
  float dt, damp, xlo, ylo, xhi, yhi;
  // bookkeeping for the next iteration
  unsigned int *bbox;
  unsigned long long *dens_acc;
  double *epart;
  unsigned int *edone;
  double *energy;
};

__device__ __forceinline__ int bin_of(float v, float bin, int G) {
  const float q = __fdiv_rn(v, bin);
  if (!(q >= 1.0f)) return 0;
  if (q >= (float)(G - 1)) return G - 1;
  return (int)q;
}

__device__ __forceinline__ float clampf_ref(float v, float lo, float hi) {
  // Rust f32::clamp: NaN passes through.
  if (v < lo) v = lo;
  if (v > hi) v = hi;
  return v;
}

__global__ void __launch_bounds__(kStepThreads)
fused_step_kernel(StepArgs a) {
  const int per_block = kStepThreads / kLanes;
  const int sub = threadIdx.x % kLanes;
  const int lane = threadIdx.x & 31;
  double e_acc = 0.0;
  for (int base = blockIdx.x * per_block; base < a.n; base += gridDim.x * per_block) {
    const int g = base + threadIdx.x / kLanes;
    const bool valid = g < a.n;
    const float2 s = spring_sum<kLanes>(a.adj_ptr, a.adj_idx, a.x, a.y, g, valid, sub);
    float nx = FLT_MAX, ny = FLT_MAX;
    bool lead = valid && sub == 0;
    if (lead) {
      const float px = a.x[g], py = a.y[g];
      float fx = __fmul_rn(a.k, s.x), fy = __fmul_rn(a.k, s.y);
      if (a.fbh) {
        const float2 b = a.fbh[g];
        fx = __fadd_rn(fx, b.x);
        fy = __fadd_rn(fy, b.y);
      }
      if (a.ex) {
        const int c = bin_of(px, a.bw, a.G), r = bin_of(py, a.bh, a.G);
        const size_t bi = (size_t)r * a.G + c;
        const float q = a.area[g];
        fx = __fadd_rn(fx, __fmul_rn(__fmul_rn(q, a.ex[bi]), a.dweight));
        fy = __fadd_rn(fy, __fmul_rn(__fmul_rn(q, a.ey[bi]), a.dweight));
        e_acc += 0.5 * (double)q * (double)a.phi[bi] * (double)a.dweight;
      }
      float vx = __fmul_rn(__fadd_rn(a.vx[g], __fmul_rn(fx, a.dt)), a.damp);
      float vy = __fmul_rn(__fadd_rn(a.vy[g], __fmul_rn(fy, a.dt)), a.damp);
      nx = clampf_ref(__fadd_rn(px, __fmul_rn(vx, a.dt)), a.xlo, a.xhi);
      ny = clampf_ref(__fadd_rn(py, __fmul_rn(vy, a.dt)), a.ylo, a.yhi);
      a.vx[g] = vx;
      a.vy[g] = vy;
      a.xn[g] = nx;
      a.yn[g] = ny;
      if (a.dens_acc) {
        const int c = bin_of(nx, a.bw, a.G), r = bin_of(ny, a.bh, a.G);
        atomicAdd(a.dens_acc + (size_t)r * a.G + c,
                  (unsigned long long)llrint((double)a.area[g] * 4294967296.0));
      }
    }
    if (a.bbox) {
      float mnx = lead ? nx : FLT_MAX, mny = lead ? ny : FLT_MAX;
      float mxx = lead ? nx : -FLT_MAX, mxy = lead ? ny : -FLT_MAX;
#pragma unroll
      for (int o = 16; o >= kLanes; o >>= 1) {
        mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
      }
      if (lane == 0) {
        atomicMin(a.bbox + 0, f2ord(mnx));
        atomicMin(a.bbox + 1, f2ord(mny));
        atomicMax(a.bbox + 2, f2ord(mxx));
        atomicMax(a.bbox + 3, f2ord(mxy));
      }
    }
  }
  if (a.energy) last_block_sum(block_sum_double(e_acc), a.epart, a.edone, a.energy);
}

int attraction_run(fx_ctx *ctx, fx_design *d, float k, float2 *out,
                   cudaStream_t s) {
  int nb = (d->n + (kStepThreads / kLanes) - 1) / (kStepThreads / kLanes);
  if (nb > ctx->num_sms * 16) nb = ctx->num_sms * 16;
  attract_kernel<<<nb, kStepThreads, 0, s>>>(d->adj_ptr.p, d->adj_idx.p,
                                             d->x[d->cur].p, d->y[d->cur].p,
                                             d->n, k, out);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

static int validate_cfg(const fx_design *d, const fx_iter_cfg &c) {
  if (!(c.dt > 0.f) || !(c.damping >= 0.f) || !(c.min_dist > 0.f) ||
      !(c.theta >= 0.f) || c.density_bins < 0 || c.cong_cols < 0 ||
      c.cong_rows < 0 || (c.cong_cols == 0) != (c.cong_rows == 0)) {
    set_error("fx_iter_cfg: invalid values");
    return FX_EINVAL;
  }
  if (c.density_bins && (c.density_bins % 128 != 0 || c.density_bins > 8192)) {
    set_error("fx_iter_cfg: density_bins must be a multiple of 128 (<= 8192)");
    return FX_EINVAL;
  }
  if (c.dct_precision < FX_DCT_FP32 || c.dct_precision > FX_DCT_SIMT) {
    set_error("fx_iter_cfg: unknown dct_precision %d", c.dct_precision);
    return FX_EINVAL;
  }
  (void)d;
  return FX_OK;
}

}  // namespace fx

using namespace fx;

extern "C" int fx_iter_cfg_default(fx_iter_cfg *c) {
  if (!c) return FX_EINVAL;
  c->attract_weight = 1.0f;
  c->repel_weight = 0.5f;
  c->min_dist = 0.1f;
  c->theta = 0.5f;
  c->density_weight = 1.0e-4f;
  c->target_density = 0.7f;
  c->density_bins = 1024;
  c->dct_precision = FX_DCT_SIMT;
  c->cong_cols = 512;
  c->cong_rows = 512;
  c->damping = 0.9f;
  c->dt = 0.1f;
  return FX_OK;
}

extern "C" int fx_stage_attraction(fx_ctx *ctx, fx_design *d, float k,
                                   float *out_fx, float *out_fy) {
  if (!ctx || !d) return FX_EINVAL;
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  FX_TRY(attraction_run(ctx, d, k, d->fattr.p, s));
  std::vector<float2> f((size_t)d->n);
  FX_CHECK_CUDA(cudaMemcpyAsync(f.data(), d->fattr.p, (size_t)d->n * 8,
                                cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < d->n; ++i) {
    if (out_fx) out_fx[i] = f[i].x;
    if (out_fy) out_fy[i] = f[i].y;
  }
  return FX_OK;
}

namespace fx {
int density_run(fx_ctx *ctx, fx_design *d, int G, float target, float weight,
                int precision, cudaStream_t s);
}

extern "C" int fx_force_iterate(fx_ctx *ctx, fx_design *d,
                                const fx_iter_cfg *cfg, int32_t iters, float *x,
                                float *y, fx_iter_stats *stats) {
  if (!ctx || !d || !cfg || iters < 0 || (x == nullptr) != (y == nullptr)) {
    set_error("fx_force_iterate: invalid arguments");
    return FX_EINVAL;
  }
  const fx_iter_cfg c = *cfg;
  FX_TRY(validate_cfg(d, c));
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream, s2 = ctx->stream2;
  if (x) FX_TRY(fx_design_set_positions(d, x, y));
  const bool use_bh = c.repel_weight != 0.f;
  const bool use_dens = c.density_bins > 0 && c.density_weight != 0.f;
  const bool use_cong = c.cong_cols > 0;
  const int G = c.density_bins;
  // Bounding box / density of the starting positions; each step then
  // prepares both for the positions it writes.
  if (use_bh) {
    FX_TRY(bh_bbox(ctx, d, d->x[d->cur].p, d->y[d->cur].p, s));
    FX_CHECK_CUDA(cudaMemsetAsync(d->bh.bbox.p + 4, 0, 4, s));
  }
  if (use_dens) FX_TRY(density_scatter(ctx, d, d->x[d->cur].p, d->y[d->cur].p, G,
                                       c.dct_precision, s));
  for (int it = 0; it < iters; ++it) {
    if (use_dens) {
      FX_CHECK_CUDA(cudaEventRecord(ctx->fork, s));
      FX_CHECK_CUDA(cudaStreamWaitEvent(s2, ctx->fork, 0));
      FX_TRY(density_run(ctx, d, G, c.target_density, c.density_weight,
                         c.dct_precision, s2));
      FX_CHECK_CUDA(cudaEventRecord(ctx->join, s2));
    }
    if (use_bh) FX_TRY(bh_run(ctx, d, c.repel_weight, c.theta, c.min_dist, s));
    if (use_dens) FX_CHECK_CUDA(cudaStreamWaitEvent(s, ctx->join, 0));
    const int nxt = d->cur ^ 1;
    StepArgs a{};
    a.adj_ptr = d->adj_ptr.p;
    a.adj_idx = d->adj_idx.p;
    a.x = d->x[d->cur].p;
    a.y = d->y[d->cur].p;
    a.xn = d->x[nxt].p;
    a.yn = d->y[nxt].p;
    a.vx = d->vx.p;
    a.vy = d->vy.p;
    a.n = d->n;
    a.k = c.attract_weight;
    a.fbh = use_bh ? d->bh.force.p : nullptr;
    if (use_dens) {
      a.ex = d->dens.ex.p;
      a.ey = d->dens.ey.p;
      a.phi = d->dens.buf[3].p;
      a.area = d->area.p;
      a.G = G;
      a.bw = d->chip_w / (float)G;
      a.bh = d->chip_h / (float)G;
      a.dweight = c.density_weight;
      a.dens_acc = d->dens.area_fx.p;
      a.epart = d->dens.energy.p;
      a.edone = (unsigned int *)(d->dens.energy.p + 4096);
      a.energy = d->dens.energy.p + 4098;
    }
    a.dt = c.dt;
    a.damp = c.damping;
    a.xlo = 0.f;
    a.ylo = 0.f;
    a.xhi = d->chip_w;
    a.yhi = d->chip_h;
    a.bbox = use_bh ? d->bh.bbox.p : nullptr;
    cudaEvent_t ev;
    timer_begin(ctx, FX_STAGE_ATTRACT_INTEGRATE, s, &ev);
    int nb = (d->n + (kStepThreads / kLanes) - 1) / (kStepThreads / kLanes);
    if (nb > ctx->num_sms * 16) nb = ctx->num_sms * 16;
    fused_step_kernel<<<nb, kStepThreads, 0, s>>>(a);
    FX_CHECK_LAUNCH();
    ctx->launches += 1;
    timer_end(ctx, FX_STAGE_ATTRACT_INTEGRATE, s, ev);
    d->cur = nxt;
    if (use_cong)
      FX_TRY(congestion_run(ctx, d, d->x[d->cur].p, d->y[d->cur].p, c.cong_cols,
                            c.cong_rows, s));
  }
  fx_iter_stats st{};
  st.iterations = iters;
  if (use_cong && iters > 0) {
    double res[2];
    FX_CHECK_CUDA(cudaMemcpyAsync(res, d->cong.result.p, 16, cudaMemcpyDeviceToHost, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(&st.max_overflow, d->cong.result_max.p, 4,
                                  cudaMemcpyDeviceToHost, s));
    FX_CHECK_CUDA(cudaStreamSynchronize(s));
    st.hpwl = res[0];
    st.total_overflow = res[1];
  }
  if (use_dens && iters > 0)
    FX_CHECK_CUDA(cudaMemcpyAsync(&st.density_energy, d->dens.energy.p + 4098, 8,
                                  cudaMemcpyDeviceToHost, s));
  if (use_bh && iters > 0) {
    unsigned int err = 0;
    FX_CHECK_CUDA(cudaMemcpyAsync(&err, d->bh.bbox.p + 4, 4, cudaMemcpyDeviceToHost, s));
    FX_CHECK_CUDA(cudaStreamSynchronize(s));
    if (err) {
      set_error("Barnes-Hut walk stack overflow");
      return FX_EINVAL;
    }
    st.bh_nodes = d->n - 1;
  }
  if (x) FX_TRY(fx_design_get_positions(d, x, y));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (stats) *stats = st;
  return FX_OK;
}
