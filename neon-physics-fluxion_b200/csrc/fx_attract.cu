// fx_attract.cu -- rows A + E: net-spring attraction as a CSR segmented
// reduction, fused with the Barnes-Hut and density forces and the damped
// Euler step; plus the plain composite iteration driver.
//
// Attraction follows place_gates_in_leaf (H/src/algorithm/placer.rs:243-255)
// over the full deduplicated adjacency (circuit.rs:154-171):
//   F_i = sum_{j in adj(i)} k * (p_j - p_i),
// added in adjacency order in f32 exactly as the reference does. A block owns
// 256 consecutive gates; their adjacency rows form one contiguous CSR range,
// which the block stages through shared memory with coalesced index loads and
// neighbour-position gathers, then each thread walks its own row in order.
// No float atomics are involved and the result is bit-identical to the
// reference's sequential sum.
// The step follows placer.rs:275-280 exactly (no contraction):
//   v = (v + F*dt) * damping ; p = clamp(p + v*dt, lo, hi).
#include <algorithm>
#include <cstring>
#include <vector>

#include "fx_internal.h"
#include "fx_device.cuh"

namespace fx {

int bh_bbox(fx_ctx *ctx, fx_design *d, const float *x, const float *y,
            cudaStream_t s);
int density_scatter(fx_ctx *ctx, fx_design *d, const float *x, const float *y,
                    int G, int precision, cudaStream_t s);

constexpr int kGates = 256;   // gates (threads) per block
constexpr int kChunk = 2048;  // adjacency entries staged per round

// Block-cooperative spring sum: every thread of the block must call it.
__device__ __forceinline__ float2 spring_block(const int32_t *__restrict__ adj_ptr,
                                               const int32_t *__restrict__ adj_idx,
                                               const float *__restrict__ x,
                                               const float *__restrict__ y,
                                               int n, int g0, float k,
                                               float xi, float yi) {
  __shared__ float2 sh[kChunk];
  const int t = threadIdx.x, g = g0 + t;
  const bool valid = g < n;
  const int gend = min(g0 + kGates, n);
  const int A0 = __ldg(adj_ptr + g0), A1 = __ldg(adj_ptr + gend);
  const int b = valid ? __ldg(adj_ptr + g) : 0;
  const int e = valid ? __ldg(adj_ptr + g + 1) : 0;
  float ax = 0.f, ay = 0.f;
  constexpr int kPer = kChunk / kGates;  // staged entries per thread and chunk
  for (int c0 = A0; c0 < A1; c0 += kChunk) {
    const int c1 = min(c0 + kChunk, A1);
    // all of a thread's index loads, then all of its gathers, so that
    // 3 x kPer independent loads are in flight instead of a chain per entry
    int jj[kPer];
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
      const int q = c0 + t + r * kGates;
      jj[r] = q < c1 ? __ldg(adj_idx + q) : -1;
    }
    float2 pv[kPer];
#pragma unroll
    for (int r = 0; r < kPer; ++r)
      pv[r] = jj[r] >= 0 ? make_float2(__ldg(x + jj[r]), __ldg(y + jj[r]))
                         : make_float2(0.f, 0.f);
#pragma unroll
    for (int r = 0; r < kPer; ++r)
      if (jj[r] >= 0) sh[t + r * kGates] = pv[r];
    __syncthreads();
    const int lo = max(b, c0), hi = min(e, c1);
    for (int q = lo; q < hi; ++q) {
      const float2 pj = sh[q - c0];
      ax = __fadd_rn(ax, __fmul_rn(k, __fsub_rn(pj.x, xi)));
      ay = __fadd_rn(ay, __fmul_rn(k, __fsub_rn(pj.y, yi)));
    }
    __syncthreads();
  }
  return make_float2(ax, ay);
}

__global__ void __launch_bounds__(kGates)
attract_kernel(const int32_t *__restrict__ adj_ptr,
               const int32_t *__restrict__ adj_idx, const float *__restrict__ x,
               const float *__restrict__ y, int n, float k,
               float2 *__restrict__ out) {
  const int g0 = blockIdx.x * kGates, g = g0 + threadIdx.x;
  const bool valid = g < n;
  const float xi = valid ? x[g] : 0.f, yi = valid ? y[g] : 0.f;
  const float2 f = spring_block(adj_ptr, adj_idx, x, y, n, g0, k, xi, yi);
  if (valid) out[g] = f;
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
  unsigned int *bbox;          // box of the new positions (ordered ints) or null
  unsigned long long *dens_acc;  // density accumulator for the new positions
  float4 *bbox_part;
  double *e_part;
  unsigned int *done;
  double *energy;
  float *trace;  // or null: {F_x, F_y, x, y, v_x, v_y} of every gate (6 x n)
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

// One gate per thread: F = attraction + Barnes-Hut + density (f32, in this
// order), the damped step, then the new positions' density scatter and box.
__global__ void __launch_bounds__(kGates)
fused_step_kernel(StepArgs a) {
  const int g0 = blockIdx.x * kGates, g = g0 + threadIdx.x;
  const bool valid = g < a.n;
  const float px = valid ? a.x[g] : 0.f, py = valid ? a.y[g] : 0.f;
  const float2 s = spring_block(a.adj_ptr, a.adj_idx, a.x, a.y, a.n, g0, a.k, px, py);
  float nx = px, ny = py;
  double e_acc = 0.0;
  long long dbin = -1;
  unsigned long long dval = 0;
  if (valid) {
    float fx = s.x, fy = s.y;
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
      if (a.phi) e_acc = 0.5 * (double)q * (double)a.phi[bi] * (double)a.dweight;
    }
    const float vx0 = a.vx[g], vy0 = a.vy[g];
    if (a.trace) {
      const size_t n = (size_t)a.n;
      a.trace[g] = fx;
      a.trace[n + g] = fy;
      a.trace[2 * n + g] = px;
      a.trace[3 * n + g] = py;
      a.trace[4 * n + g] = vx0;
      a.trace[5 * n + g] = vy0;
    }
    const float vx = __fmul_rn(__fadd_rn(vx0, __fmul_rn(fx, a.dt)), a.damp);
    const float vy = __fmul_rn(__fadd_rn(vy0, __fmul_rn(fy, a.dt)), a.damp);
    nx = clampf_ref(__fadd_rn(px, __fmul_rn(vx, a.dt)), a.xlo, a.xhi);
    ny = clampf_ref(__fadd_rn(py, __fmul_rn(vy, a.dt)), a.ylo, a.yhi);
    a.vx[g] = vx;
    a.vy[g] = vy;
    a.xn[g] = nx;
    a.yn[g] = ny;
    if (a.dens_acc) {
      const int c = bin_of(nx, a.bw, a.G), r = bin_of(ny, a.bh, a.G);
      dbin = (long long)r * a.G + c;
      dval = (unsigned long long)llrint((double)a.area[g] * 4294967296.0);
    }
  }
  if (a.dens_acc) agg_add_u64(a.dens_acc, dbin, dval);
  // Box of the new positions and density energy: per-block values, then the
  // last block combines them in block order.
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float mnx = valid ? nx : FLT_MAX, mny = valid ? ny : FLT_MAX;
  float mxx = valid ? nx : -FLT_MAX, mxy = valid ? ny : -FLT_MAX;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
  }
  __shared__ float4 wbox[kGates / 32];
  if (lane == 0) wbox[w] = make_float4(mnx, mny, mxx, mxy);
  const double esum = block_sum_double(e_acc);  // contains __syncthreads
  __shared__ bool last;
  if (threadIdx.x == 0) {
    float4 bb = wbox[0];
    for (int q = 1; q < kGates / 32; ++q) {
      bb.x = fminf(bb.x, wbox[q].x);
      bb.y = fminf(bb.y, wbox[q].y);
      bb.z = fmaxf(bb.z, wbox[q].z);
      bb.w = fmaxf(bb.w, wbox[q].w);
    }
    a.bbox_part[blockIdx.x] = bb;
    a.e_part[blockIdx.x] = esum;
    __threadfence();
    last = atomicAdd(a.done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  float4 bb = make_float4(FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX);
  double et = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kGates) {
    const float4 q = __ldcg(a.bbox_part + i);
    bb.x = fminf(bb.x, q.x);
    bb.y = fminf(bb.y, q.y);
    bb.z = fmaxf(bb.z, q.z);
    bb.w = fmaxf(bb.w, q.w);
    et += __ldcg(a.e_part + i);
  }
  et = block_sum_double(et);
  bb.x = -block_max_float(-bb.x);
  bb.y = -block_max_float(-bb.y);
  bb.z = block_max_float(bb.z);
  bb.w = block_max_float(bb.w);
  if (threadIdx.x == 0) {
    if (a.bbox) {
      a.bbox[0] = f2ord(bb.x);
      a.bbox[1] = f2ord(bb.y);
      a.bbox[2] = f2ord(bb.z);
      a.bbox[3] = f2ord(bb.w);
    }
    if (a.energy) *a.energy = et;
    *a.done = 0u;
  }
}

int attraction_run(fx_ctx *ctx, fx_design *d, float k, float2 *out,
                   cudaStream_t s) {
  const int nb = (d->n + kGates - 1) / kGates;
  attract_kernel<<<nb, kGates, 0, s>>>(d->adj_ptr.p, d->adj_idx.p,
                                       d->x[d->cur].p, d->y[d->cur].p, d->n, k,
                                       out);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

static int step_alloc(fx_design *d, cudaStream_t s) {
  StepWork &w = d->step;
  const size_t nb = ((size_t)d->n + kGates - 1) / kGates;
  if (w.bbox_part.p && w.bbox_part.n >= nb) return FX_OK;
  FX_TRY(w.bbox_part.alloc(nb));
  FX_TRY(w.e_part.alloc(nb));
  FX_TRY(w.done.alloc(4));
  FX_TRY(w.energy.alloc(4));
  FX_CHECK_CUDA(cudaMemsetAsync(w.done.p, 0, 16, s));
  FX_CHECK_CUDA(cudaMemsetAsync(w.energy.p, 0, 32, s));
  return FX_OK;
}

static int validate_cfg(const fx_iter_cfg &c) {
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
  if (c.bh_walk != FX_BH_FAST && c.bh_walk != FX_BH_EXACT) {
    set_error("fx_iter_cfg: unknown bh_walk %d", c.bh_walk);
    return FX_EINVAL;
  }
  if (c.dct_precision < FX_DCT_FP32 || c.dct_precision > FX_DCT_I8) {
    set_error("fx_iter_cfg: unknown dct_precision %d", c.dct_precision);
    return FX_EINVAL;
  }
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
  c->dct_precision = FX_DCT_I8;  // FP32-accurate on the tensor cores; second stream
  c->cong_cols = 512;
  c->cong_rows = 512;
  c->damping = 0.9f;
  c->dt = 0.1f;
  c->bh_walk = FX_BH_FAST;
  return FX_OK;
}

extern "C" int fx_stage_attraction(fx_ctx *ctx, fx_design *d, float k,
                                   float *out_fx, float *out_fy) {
  if (!ctx || !d) return FX_EINVAL;
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
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
                int precision, bool need_phi, cudaStream_t s);

// A run's statistics and error words, written by one thread straight into
// the context's pinned readback block: one launch before the final
// synchronisation instead of a copy per value (and a second round trip for
// the tensor-core error word).
__global__ void iter_stats_kernel(const double *__restrict__ cong_res,
                                  const float *__restrict__ cong_max,
                                  const double *__restrict__ energy,
                                  const unsigned int *__restrict__ bh_err,
                                  const unsigned int *__restrict__ tc_err,
                                  IterReadback *__restrict__ out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  IterReadback r{};
  if (cong_res) {
    r.res[0] = cong_res[0];
    r.res[1] = cong_res[1];
    r.max_overflow = cong_max[0];
  }
  if (energy) r.energy = energy[0];
  if (bh_err) r.err = bh_err[0];
  if (tc_err) r.tc_err = tc_err[0];
  *out = r;
}
}

// What a captured single-iteration graph depends on: the configuration, the
// context (the tensor-core error word its GEMMs write), the starting parity,
// the in-die flag (from which the host decides whether the tree build
// launches its deep-key kernels), and the address and size of every buffer
// of the design and its workspaces.
static std::vector<uint64_t> iter_graph_key(fx_ctx *ctx, fx_design *d, const fx_iter_cfg &c,
                                            int cur, bool box) {
  std::vector<uint64_t> k;
  k.reserve(320);
  const unsigned char *cb = reinterpret_cast<const unsigned char *>(&c);
  for (size_t i = 0; i < sizeof c; i += 8) {
    uint64_t w = 0;
    std::memcpy(&w, cb + i, std::min<size_t>(8, sizeof c - i));
    k.push_back(w);
  }
  k.push_back((uint64_t)(uintptr_t)ctx);
  k.push_back((uint64_t)(uintptr_t)ctx->tc_err);
  k.push_back((uint64_t)cur);
  k.push_back(box ? 1u : 0u);
  auto add = [&k](auto &b) {
    k.push_back((uint64_t)(uintptr_t)b.p);
    k.push_back((uint64_t)b.n);
  };
  add(d->net_ptr);
  add(d->net_gate);
  add(d->adj_ptr);
  add(d->adj_idx);
  add(d->area);
  for (int i = 0; i < 2; ++i) {
    add(d->x[i]);
    add(d->y[i]);
  }
  add(d->vx);
  add(d->vy);
  d->bh.for_each(add);
  d->dens.for_each(add);
  d->cong.for_each(add);
  d->step.for_each(add);
  k.push_back((uint64_t)d->dens.halves);
  k.push_back((uint64_t)(uint32_t)d->dens.G);
  k.push_back((uint64_t)(uint32_t)d->dens.precision);
  k.push_back((uint64_t)(uint32_t)d->cong.cols);
  k.push_back((uint64_t)(uint32_t)d->cong.rows);
  k.push_back((uint64_t)(uint32_t)d->bh.n);
  k.push_back(ctx->timer.enabled ? 1u + (uint64_t)ctx->timer.mask : 0u);
  return k;
}

extern "C" int fx_force_iterate(fx_ctx *ctx, fx_design *d,
                                const fx_iter_cfg *cfg, int32_t iters, float *x,
                                float *y, fx_iter_stats *stats) {
  if (!ctx || !d || !cfg || iters < 0 || (x == nullptr) != (y == nullptr)) {
    set_error("fx_force_iterate: invalid arguments");
    return FX_EINVAL;
  }
  const fx_iter_cfg c = *cfg;
  FX_TRY(validate_cfg(c));
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream, s2 = ctx->stream2;
  if (x) FX_TRY(fx_design_set_positions(d, x, y));
  FX_TRY(step_alloc(d, s));
  if (d->trace_on) FX_TRY(d->trace.alloc((size_t)d->n * 6));
  const bool use_bh = c.repel_weight != 0.f;
  const bool use_dens = c.density_bins > 0 && c.density_weight != 0.f;
  const bool use_cong = c.cong_cols > 0;
  const int G = c.density_bins;
  // Bounding box / density of the starting positions; each step then
  // prepares both for the positions it writes.
  auto prologue = [&]() -> int {
    if (use_bh) FX_TRY(bh_bbox(ctx, d, d->x[d->cur].p, d->y[d->cur].p, s));
    if (use_dens)
      FX_TRY(density_scatter(ctx, d, d->x[d->cur].p, d->y[d->cur].p, G,
                             c.dct_precision, s));
    if (use_cong) FX_TRY(congestion_alloc(d, c.cong_cols, c.cong_rows, s));
    return FX_OK;
  };
  const int nb = (d->n + kGates - 1) / kGates;
  bool copied_out = false;  // positions already on their way to x, y
  // The congestion of the positions a step writes only feeds the statistics
  // (the last step's are returned), so it runs at the start of the next
  // step on the second stream, beside that step's Barnes-Hut chain; the last
  // step runs its own on the primary stream. Same kernels, inputs and order
  // on the scratch as running each right after its step.
  bool cong_pending = false;
  // One iteration; `last` adds the potential (energy statistic).
  auto step = [&](bool last) -> int {
    // The Barnes-Hut chain (the critical path) is issued first, so the GPU
    // starts it while the host still issues the side work; the previous
    // step's congestion and the density solve fork from the same point of
    // the primary stream and run beside it, joined before the step kernel
    // (which writes the other position buffer).
    const bool side = use_dens || cong_pending;
    if (side) FX_CHECK_CUDA(cudaEventRecord(ctx->fork, s));
    if (use_bh) FX_TRY(bh_run(ctx, d, c.repel_weight, c.theta, c.min_dist, c.bh_walk, s));
    if (side) {
      FX_CHECK_CUDA(cudaStreamWaitEvent(s2, ctx->fork, 0));
      if (cong_pending) {
        FX_TRY(congestion_run(ctx, d, d->x[d->cur].p, d->y[d->cur].p, c.cong_cols,
                              c.cong_rows, s2));
        cong_pending = false;
      }
      // the potential only feeds the energy statistic of the last step
      if (use_dens)
        FX_TRY(density_run(ctx, d, G, c.target_density, c.density_weight,
                           c.dct_precision, last, s2));
      FX_CHECK_CUDA(cudaEventRecord(ctx->join, s2));
      FX_CHECK_CUDA(cudaStreamWaitEvent(s, ctx->join, 0));
    }
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
      a.phi = last ? d->dens.buf[3].p : nullptr;
      a.area = d->area.p;
      a.G = G;
      a.bw = d->chip_w / (float)G;
      a.bh = d->chip_h / (float)G;
      a.dweight = c.density_weight;
      a.dens_acc = d->dens.area_fx.p;
    }
    a.dt = c.dt;
    a.damp = c.damping;
    a.xlo = 0.f;
    a.ylo = 0.f;
    a.xhi = d->chip_w;
    a.yhi = d->chip_h;
    a.bbox = use_bh ? d->bh.bbox.p : nullptr;
    a.bbox_part = d->step.bbox_part.p;
    a.e_part = d->step.e_part.p;
    a.done = d->step.done.p;
    a.energy = d->step.energy.p;
    a.trace = d->trace_on ? d->trace.p : nullptr;
    cudaEvent_t ev;
    timer_begin(ctx, FX_STAGE_ATTRACT_INTEGRATE, s, &ev);
    fused_step_kernel<<<nb, kGates, 0, s>>>(a);
    FX_CHECK_LAUNCH();
    ctx->launches += 1;
    timer_end(ctx, FX_STAGE_ATTRACT_INTEGRATE, s, ev);
    d->cur = nxt;
    d->pos_in_box = true;  // the step clamps every position to the die
    if (last && x) {
      // the final positions go to the caller's buffers on the second stream
      // while the congestion of the same positions runs on the first
      const size_t bytes = (size_t)d->n * 4;
      FX_CHECK_CUDA(cudaEventRecord(ctx->fork, s));
      FX_CHECK_CUDA(cudaStreamWaitEvent(s2, ctx->fork, 0));
      FX_CHECK_CUDA(cudaMemcpyAsync(x, d->x[d->cur].p, bytes, cudaMemcpyDeviceToHost, s2));
      FX_CHECK_CUDA(cudaMemcpyAsync(y, d->y[d->cur].p, bytes, cudaMemcpyDeviceToHost, s2));
      copied_out = true;
    }
    if (use_cong) {
      if (last)
        FX_TRY(congestion_run(ctx, d, d->x[d->cur].p, d->y[d->cur].p, c.cong_cols,
                              c.cong_rows, s));
      else
        cong_pending = true;
    }
    return FX_OK;
  };
  // A single iteration on the resident positions (the common call of a
  // host loop that restores or edits state between calls) replays a cached
  // graph of the whole call: the prologue and the step. A call whose key
  // matches what the previous eager call of the same parity left behind is
  // captured; a changed configuration, context, buffer or state flag makes
  // the key differ and the call run eagerly.
  int it = 0;
  bool replayed = false;
  const fx_design::IterGraph *timed_graph = nullptr;  // its stage events to read
  // With stage timing on, the graph carries the timed stages' events as
  // event record nodes, read after each replay (the key holds the timer's
  // state, so turning timing on or off captures another graph).
  if (iters == 1 && !x && !d->trace_on) {
    const int cur_start = d->cur;
    const bool box_start = d->pos_in_box;
    fx_design::IterGraph &g = d->g1[cur_start];
    std::vector<uint64_t> key = iter_graph_key(ctx, d, c, cur_start, box_start);
    if (g.exec && g.key == key) {
      FX_CHECK_CUDA(cudaGraphLaunch(g.exec, s));
      ctx->launches += g.launches;
      d->cur ^= 1;
      d->pos_in_box = true;  // the step clamps every position to the die
      replayed = true;
      if (!g.timing.empty()) timed_graph = &g;
    } else {
      g.reset();
      if (g.seen == key && g.failed != key) {
        const int64_t l0 = ctx->launches;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        int rc = FX_OK;
        auto drop_captured = [&]() {
          for (auto &t : ctx->timer.captured) {
            cudaEventDestroy(t.a);
            cudaEventDestroy(t.b);
          }
          ctx->timer.captured.clear();
        };
        drop_captured();
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
          rc = prologue();
          if (rc == FX_OK) rc = step(true);
          const cudaError_t e = cudaStreamEndCapture(s, &graph);
          if (e != cudaSuccess || rc != FX_OK ||
              cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
            exec = nullptr;
        }
        cudaGetLastError();  // a failed capture leaves an error: run eagerly
        if (graph) cudaGraphDestroy(graph);
        const int64_t per_call = ctx->launches - l0;
        ctx->launches = l0;
        d->cur = cur_start;
        d->pos_in_box = box_start;
        if (exec) {
          g.exec = exec;
          g.key = key;
          g.launches = per_call;
          g.timing.swap(ctx->timer.captured);
          if (!g.timing.empty()) timed_graph = &g;
        }
        drop_captured();
        if (exec) {
          FX_CHECK_CUDA(cudaGraphLaunch(g.exec, s));
          ctx->launches += per_call;
          d->cur ^= 1;
          d->pos_in_box = true;
          replayed = true;
        } else {
          g.failed = key;  // this key runs eagerly from now on
        }
      }
    }
    if (!replayed) {
      FX_TRY(prologue());
      const int rc = step(true);
      if (rc != FX_OK) return rc;
      // this call's start state with the buffers it ended with: the next
      // call of this parity with the same key is captured
      g.seen = iter_graph_key(ctx, d, c, cur_start, box_start);
      replayed = true;
    }
    it = iters;
  } else {
    FX_TRY(prologue());
  }
  // Long runs replay a CUDA graph of two iterations (one per ping-pong
  // parity) after an eager first iteration has sized every buffer; the last
  // iteration runs eagerly. Same kernels and arguments, same results; not
  // used while stage timing is on (its events are per launch).
  if (!ctx->timer.enabled && iters >= 8) {
    FX_TRY(step(false));
    ++it;
    const int cur0 = d->cur;
    const bool pending0 = cong_pending;
    const int64_t l0 = ctx->launches;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = FX_OK;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      rc = step(false);
      if (rc == FX_OK) rc = step(false);
      const cudaError_t e = cudaStreamEndCapture(s, &graph);
      if (e == cudaSuccess && rc == FX_OK &&
          cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
        exec = nullptr;
    }
    cudaGetLastError();  // a failed capture leaves an error: fall back to eager
    d->cur = cur0;
    // a pair of steps leaves a congestion pending exactly as it found one
    cong_pending = pending0;
    const int64_t per_pair = ctx->launches - l0;
    ctx->launches = l0;
    if (exec) {
      for (; it + 2 <= iters - 1; it += 2) {
        FX_CHECK_CUDA(cudaGraphLaunch(exec, s));
        ctx->launches += per_pair;
      }
      cudaGraphExecDestroy(exec);
    }
    if (graph) cudaGraphDestroy(graph);
  }
  for (; it < iters; ++it) {
    const int rc = step(it == iters - 1);
    if (rc != FX_OK) {
      // never return while a copy into the caller's buffers is in flight
      if (copied_out) cudaStreamSynchronize(s2);
      return rc;
    }
  }
  fx_iter_stats st{};
  st.iterations = iters;
  // the statistics come back through the context's pinned buffer (truly
  // asynchronous copies; pageable ones would stage through the driver)
  IterReadback &rb = *ctx->readback;
  rb = IterReadback{};
  const bool tc = use_dens && c.dct_precision != FX_DCT_SIMT;
  if (iters > 0) {
    iter_stats_kernel<<<1, 32, 0, s>>>(use_cong ? d->cong.result.p : nullptr,
                                       use_cong ? d->cong.result_max.p : nullptr,
                                       use_dens ? d->step.energy.p : nullptr,
                                       use_bh ? d->bh.bbox.p + 4 : nullptr,
                                       tc ? ctx->tc_err : nullptr, ctx->readback_dev);
    FX_CHECK_LAUNCH();
    ctx->launches += 1;
  }
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (timed_graph) ctx->timer.add_elapsed(timed_graph->timing);
  const double res[2] = {rb.res[0], rb.res[1]};
  const unsigned int err = rb.err;
  st.max_overflow = rb.max_overflow;
  st.density_energy = rb.energy;
  if (copied_out) FX_CHECK_CUDA(cudaStreamSynchronize(s2));
  FX_TRY(bh_error(err));
  if (rb.tc_err) {
    const unsigned int tc_err = rb.tc_err;
    // cleared so that the context's next GEMMs report only their own waits
    FX_CHECK_CUDA(cudaMemsetAsync(ctx->tc_err, 0, 4, s));
    FX_CHECK_CUDA(cudaStreamSynchronize(s));
    set_error("tensor-core GEMM: a bounded wait expired (error word %u)", tc_err);
    return FX_ETIMEOUT;
  }
  st.hpwl = res[0];
  st.total_overflow = res[1];
  st.bh_nodes = use_bh ? d->n - 1 : 0;
  if (x && !copied_out) FX_TRY(fx_design_get_positions(d, x, y));
  if (stats) *stats = st;
  return FX_OK;
}

extern "C" int fx_design_trace(fx_design *d, int enable) {
  if (!d) return FX_EINVAL;
  d->trace_on = enable != 0;
  return FX_OK;
}

extern "C" int fx_design_trace_get(fx_design *d, float *out_fx, float *out_fy, float *out_x,
                                   float *out_y, float *out_vx, float *out_vy) {
  if (!d || !d->ctx) return FX_EINVAL;
  if (!d->trace.p || d->trace.n < (size_t)d->n * 6) {
    set_error("fx_design_trace_get: no traced iteration (enable fx_design_trace, then "
              "run fx_force_iterate)");
    return FX_EINVAL;
  }
  fx_ctx *ctx = d->ctx;
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  float *outs[6] = {out_fx, out_fy, out_x, out_y, out_vx, out_vy};
  const size_t n = (size_t)d->n;
  for (int i = 0; i < 6; ++i)
    if (outs[i])
      FX_CHECK_CUDA(cudaMemcpyAsync(outs[i], d->trace.p + i * n, n * 4,
                                    cudaMemcpyDeviceToHost, ctx->stream));
  FX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return FX_OK;
}
