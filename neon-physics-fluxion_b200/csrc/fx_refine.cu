// fx_refine.cu -- the congestion refinement loop (refine_placement,
// H/src/algorithm/refiner.rs:34-126) on the device.
//
// Each iteration: congestion counts (rows D+F kernels), the total overflow as
// the reference's f32 running sum over cells in row-major order (one warp
// stages tiles, one lane adds them in order: the stop and stall rules compare
// this exact value), then every gate whose
// cell is hot (overflow > threshold, gates_in_hot_cells, congestion.rs:77-93)
// moves toward the first least-congested cell within radius 3
// (move_gate_from_hot_cell, refiner.rs:92-126; Iterator::min_by keeps the
// first minimum in (dr, dc) order). A move reads only the gate's own position
// and the grid frozen at the start of the iteration, so all gates move in
// parallel with the reference's sequential result.
#include <cmath>

#include "fx_internal.h"
#include "fx_device.cuh"

namespace fx {

__device__ __forceinline__ float rclampf(float v, float lo, float hi) {
  if (v < lo) v = lo;
  if (v > hi) v = hi;
  return v;
}

// grid.rs:86-91 total_overflow: f32 running sum, row-major. One warp: the
// lanes compute a tile of overflows into shared memory, then lane 0 adds the
// tile in cell order (the loads from shared memory run ahead of the adds, so
// the fold costs about one add latency per cell). The maximum is order-free.
constexpr int kTotalTile = 4096;

__global__ void __launch_bounds__(32)
refine_total_kernel(const uint32_t *__restrict__ counts, int cells, float cap,
                    float *__restrict__ out) {
  __shared__ float tile[kTotalTile];
  const int lane = threadIdx.x;
  float t = 0.0f, mx = 0.0f;
  for (int base = 0; base < cells; base += kTotalTile) {
    const int m = min(kTotalTile, cells - base);
    for (int i = lane; i < m; i += 32) {
      const float c = (float)counts[base + i];
      const float ov = fmaxf(__fsub_rn(__fadd_rn(c, c), cap), 0.0f);
      tile[i] = ov;
      mx = fmaxf(mx, ov);
    }
    __syncwarp();
    if (lane == 0) {
#pragma unroll 16
      for (int i = 0; i < m; ++i) t = __fadd_rn(t, tile[i]);
    }
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) {
    out[0] = t;
    out[1] = mx;
  }
}

__global__ void refine_move_kernel(float *__restrict__ x, float *__restrict__ y, int n,
                                   const uint32_t *__restrict__ counts, int cols,
                                   int rows, float cw, float ch, float cap,
                                   float threshold, float max_move, float chip_w,
                                   float chip_h, unsigned int *__restrict__ moved) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const float gx = x[g], gy = y[g];
  const int col = cell_at(gx, cw, cols), row = cell_at(gy, ch, rows);
  const float c0 = (float)counts[(size_t)row * cols + col];
  const float ov = fmaxf(__fsub_rn(__fadd_rn(c0, c0), cap), 0.0f);
  if (!(ov > threshold)) return;
  bool found = false;
  int bc = 0, br = 0;
  float best = 0.0f;
  for (int dr = -3; dr <= 3; ++dr)
    for (int dc = -3; dc <= 3; ++dc) {
      if (dr == 0 && dc == 0) continue;
      const int nc = col + dc, nr = row + dr;
      if (nc < 0 || nc >= cols || nr < 0 || nr >= rows) continue;
      const float c = (float)counts[(size_t)nr * cols + nc];
      const float tot = __fadd_rn(c, c);
      if (!found || tot < best) {
        found = true;
        best = tot;
        bc = nc;
        br = nr;
      }
    }
  if (!found) return;
  const float tx = __fmul_rn(__fadd_rn((float)bc, 0.5f), cw);
  const float ty = __fmul_rn(__fadd_rn((float)br, 0.5f), ch);
  const float dx = rclampf(__fsub_rn(tx, gx), -max_move, max_move);
  const float dy = rclampf(__fsub_rn(ty, gy), -max_move, max_move);
  x[g] = rclampf(__fadd_rn(gx, dx), 0.0f, chip_w);
  y[g] = rclampf(__fadd_rn(gy, dy), 0.0f, chip_h);
  if (moved) atomicAdd(moved, 1u);
}

}  // namespace fx

using namespace fx;

extern "C" int fx_refine_cfg_default(fx_refine_cfg *c) {
  if (!c) return FX_EINVAL;
  c->max_iterations = 100;
  c->move_distance = 5.0f;
  c->overflow_threshold = 1.0f;
  c->grid_cols = 256;
  c->grid_rows = 256;
  c->reserved0 = 0;
  return FX_OK;
}

extern "C" int fx_refine(fx_ctx *ctx, fx_design *d, const fx_refine_cfg *cfg,
                         float *x, float *y, fx_refine_stats *stats,
                         uint32_t *out_counts) {
  if (!ctx || !d || !cfg || (x == nullptr) != (y == nullptr) || cfg->grid_cols <= 0 ||
      cfg->grid_rows <= 0 || cfg->max_iterations < 0 ||
      (int64_t)cfg->grid_cols * cfg->grid_rows > (int64_t)1 << 26) {
    set_error("fx_refine: invalid arguments");
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream;
  if (x) FX_TRY(fx_design_set_positions(d, x, y));
  const int cols = cfg->grid_cols, rows = cfg->grid_rows, cells = cols * rows;
  // RoutingGrid::new (grid.rs:25-32)
  const float cw = d->chip_w / (float)cols, ch = d->chip_h / (float)rows;
  const float cap = (cw + ch) * 0.5f;
  float *px = d->x[d->cur].p, *py = d->y[d->cur].p;
  d->pos_in_box = false;  // moved positions are not re-checked against the die
  DevBuf<float> tot;
  DevBuf<unsigned int> moved;
  FX_TRY(tot.alloc(2));
  FX_TRY(moved.alloc(1));
  FX_CHECK_CUDA(cudaMemsetAsync(moved.p, 0, 4, s));  // moves summed over iterations
  float prev = 3.40282347e+38f;
  int stall = 0, iters = 0;
  int64_t moves = 0;
  for (int it = 0; it < cfg->max_iterations; ++it) {
    FX_TRY(congestion_run(ctx, d, px, py, cols, rows, s));
    refine_total_kernel<<<1, 32, 0, s>>>(d->cong.counts.p, cells, cap, tot.p);
    float h[2];
    FX_CHECK_CUDA(cudaMemcpyAsync(h, tot.p, 8, cudaMemcpyDeviceToHost, s));
    FX_CHECK_CUDA(cudaStreamSynchronize(s));
    ctx->launches += 1;
    const float total = h[0];
    if (total <= cfg->overflow_threshold) break;
    if (std::fabs(prev - total) < 0.01f * std::fmax(prev, 1.0f)) {
      if (++stall >= 10) break;
    } else {
      stall = 0;
    }
    prev = total;
    refine_move_kernel<<<(d->n + 255) / 256, 256, 0, s>>>(
        px, py, d->n, d->cong.counts.p, cols, rows, cw, ch, cap, cfg->overflow_threshold,
        cfg->move_distance, d->chip_w, d->chip_h, moved.p);
    FX_CHECK_LAUNCH();
    ctx->launches += 1;
    ++iters;
  }
  FX_TRY(congestion_run(ctx, d, px, py, cols, rows, s));
  refine_total_kernel<<<1, 32, 0, s>>>(d->cong.counts.p, cells, cap, tot.p);
  ctx->launches += 1;
  float h[2];
  double hp = 0.0;
  FX_CHECK_CUDA(cudaMemcpyAsync(h, tot.p, 8, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(&hp, d->cong.result.p, 8, cudaMemcpyDeviceToHost, s));
  unsigned int mv = 0;
  FX_CHECK_CUDA(cudaMemcpyAsync(&mv, moved.p, 4, cudaMemcpyDeviceToHost, s));
  if (out_counts)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_counts, d->cong.counts.p, (size_t)cells * 4,
                                  cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (x) FX_TRY(fx_design_get_positions(d, x, y));
  moves = mv;
  if (stats) {
    stats->iterations = iters;
    stats->moves = moves;
    stats->total_overflow = h[0];
    stats->max_overflow = h[1];
    stats->hpwl = hp;
  }
  return FX_OK;
}
