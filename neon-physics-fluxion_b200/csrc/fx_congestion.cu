// fx_congestion.cu -- rows D + F: net bounding boxes -> integer congestion
// counts (2-D difference array + 2-D prefix sum) and FP64 HPWL.
//
// Semantics follow compute_congestion_cpu (H/src/algorithm/congestion.rs:
// 11-62), RoutingGrid::new / cell_at (H/src/data/grid.rs:25-62) and
// Placement::compute_hpwl (H/src/data/placement.rs:48-74). The reference adds
// 1.0f to every covered cell of two identical f32 grids; counts stay below
// 2^24, so one exact uint32 grid carries both.
#include <mutex>

#include "fx_internal.h"
#include "fx_device.cuh"

namespace fx {

constexpr int kNetThreads = 256;
constexpr int kMaxNetBlocks = 148 * 16;

// One thread per net: f32 bounding box with Rust's NaN-ignoring min/max,
// cell_at on both corners, four corner increments of the difference array
// (warp-aggregated: lanes hitting the same element add once), and the net's
// HPWL term in FP64. Warps step through the nets together so every lane
// takes part in the aggregation.
__global__ void __launch_bounds__(kNetThreads)
cong_nets_kernel(const int32_t *__restrict__ net_ptr,
                 const int32_t *__restrict__ net_gate,
                 const float *__restrict__ x, const float *__restrict__ y,
                 int M, float cw, float ch, int cols, int rows,
                 int32_t *__restrict__ diff, double *__restrict__ partial,
                 unsigned int *__restrict__ done, double *__restrict__ result) {
  double acc = 0.0;
  const long long ld = cols + 1;
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  for (int w0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); w0 < M; w0 += stride) {
    const int e = w0 + lane;
    int b = 0, t = 0;
    if (e < M) {
      b = __ldg(net_ptr + e);
      t = __ldg(net_ptr + e + 1);
    }
    long long i00 = -1, i01 = -1, i10 = -1, i11 = -1;
    if (t - b >= 2) {
      float mnx = FLT_MAX, mxx = -FLT_MAX, mny = FLT_MAX, mxy = -FLT_MAX;
      for (int q = b; q < t; ++q) {
        const int g = __ldg(net_gate + q);
        const float px = __ldg(x + g), py = __ldg(y + g);
        mnx = fminf(mnx, px);
        mxx = fmaxf(mxx, px);
        mny = fminf(mny, py);
        mxy = fmaxf(mxy, py);
      }
      acc += ((double)mxx - (double)mnx) + ((double)mxy - (double)mny);
      const int c0 = cell_at(mnx, cw, cols), c1 = cell_at(mxx, cw, cols);
      const int r0 = cell_at(mny, ch, rows), r1 = cell_at(mxy, ch, rows);
      if (c0 <= c1 && r0 <= r1) {
        i00 = (long long)r0 * ld + c0;
        i01 = (long long)r0 * ld + c1 + 1;
        i10 = (long long)(r1 + 1) * ld + c0;
        i11 = (long long)(r1 + 1) * ld + c1 + 1;
      }
    }
    if (diff) {
      agg_add_const_i32(diff, i00, 1);
      agg_add_const_i32(diff, i01, -1);
      agg_add_const_i32(diff, i10, -1);
      agg_add_const_i32(diff, i11, 1);
    }
  }
  const double s = block_sum_double(acc);
  last_block_sum(s, partial, done, result);
}

// In-place inclusive scan of each difference-array row over columns.
__global__ void __launch_bounds__(1024)
cong_scan_rows_kernel(int32_t *__restrict__ diff, int cols, int rows) {
  const int r = blockIdx.x;
  if (r >= rows) return;
  int32_t *row = diff + (size_t)r * (cols + 1);
  __shared__ int32_t warp_tot[32];
  int carry = 0;
  for (int base = 0; base < cols; base += blockDim.x) {
    const int c = base + threadIdx.x;
    int v = c < cols ? row[c] : 0;
    // warp inclusive scan
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    if (lane == 31) warp_tot[w] = v;
    __syncthreads();
    if (w == 0) {
      const int nw = blockDim.x >> 5;
      int t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int u = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += u;
      }
      if (lane < nw) warp_tot[lane] = t;
    }
    __syncthreads();
    const int off = (w > 0 ? warp_tot[w - 1] : 0) + carry;
    if (c < cols) row[c] = v + off;
    carry += warp_tot[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
}

// Column scan over 32-column stripes: produces the counts, zeroes the
// difference array for the next call, and reduces the overflow
// max(0, h + v - capacity) (grid.rs:71-91) as an FP64 sum and an f32 max.
__global__ void __launch_bounds__(1024)
cong_scan_cols_kernel(int32_t *__restrict__ diff, uint32_t *__restrict__ counts,
                      int cols, int rows, float cap,
                      double *__restrict__ partial, float *__restrict__ pmax,
                      unsigned int *__restrict__ done, double *__restrict__ result,
                      float *__restrict__ result_max) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int c = blockIdx.x * 32 + tx;
  const int ld = cols + 1;
  const int chunk = (rows + 31) / 32;
  const int r0 = ty * chunk, r1 = min(rows, r0 + chunk);
  __shared__ int32_t part[32][33];
  int s = 0;
  if (c < cols)
    for (int r = r0; r < r1; ++r) s += diff[(size_t)r * ld + c];
  part[ty][tx] = s;
  __syncthreads();
  int run = 0;
  for (int yy = 0; yy < ty; ++yy) run += part[yy][tx];
  double ov_sum = 0.0;
  float ov_max = 0.f;
  if (c < cols) {
    for (int r = r0; r < r1; ++r) {
      const size_t i = (size_t)r * ld + c;
      run += diff[i];
      diff[i] = 0;
      counts[(size_t)r * cols + c] = (uint32_t)run;
      const float cf = (float)run;
      const float ov = fmaxf(__fsub_rn(__fadd_rn(cf, cf), cap), 0.f);
      ov_sum += (double)ov;
      ov_max = fmaxf(ov_max, ov);
    }
    if (ty == 0) diff[(size_t)rows * ld + c] = 0;
  }
  if (blockIdx.x == 0) {
    const int t = ty * 32 + tx;
    for (int r = t; r <= rows; r += 1024) diff[(size_t)r * ld + cols] = 0;
  }
  // FP64 sum and f32 max over the block, then across blocks.
  const double bs = block_sum_double(ov_sum);
  const float bm = block_max_float(ov_max);
  __shared__ bool last;
  const int lin = ty * 32 + tx;
  if (lin == 0) {
    partial[blockIdx.x] = bs;
    pmax[blockIdx.x] = bm;
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double a = 0.0;
    float m = 0.f;
    for (int i = lin; i < (int)gridDim.x; i += 1024) {
      a += ((volatile double *)partial)[i];
      m = fmaxf(m, ((volatile float *)pmax)[i]);
    }
    a = block_sum_double(a);
    m = block_max_float(m);
    if (lin == 0) {
      result[1] = a;
      result_max[0] = m;
      *done = 0;
    }
  }
}

int congestion_alloc(fx_design *d, int cols, int rows, cudaStream_t s) {
  CongWork &w = d->cong;
  if ((int64_t)(cols + 1) * (rows + 1) > (int64_t)INT32_MAX) {  // corner indexes are 31-bit
    set_error("congestion grid %d x %d too large", cols, rows);
    return FX_EINVAL;
  }
  if (w.cols != cols || w.rows != rows || !w.diff.p) {
    const size_t cells1 = (size_t)(cols + 1) * (rows + 1);
    FX_TRY(w.diff.alloc(cells1));
    FX_TRY(w.counts.alloc((size_t)cols * rows));
    FX_TRY(w.partial.alloc(kMaxNetBlocks + 4096));
    FX_TRY(w.partial_max.alloc(4096));
    FX_TRY(w.done.alloc(4));
    FX_TRY(w.result.alloc(4));
    FX_TRY(w.result_max.alloc(4));
    FX_CHECK_CUDA(cudaMemsetAsync(w.diff.p, 0, cells1 * 4, s));
    FX_CHECK_CUDA(cudaMemsetAsync(w.done.p, 0, 16, s));
    w.cols = cols;
    w.rows = rows;
  }
  return FX_OK;
}

int congestion_run(fx_ctx *ctx, fx_design *d, const float *dx,
                   const float *dy, int cols, int rows, cudaStream_t s) {
  CongWork &w = d->cong;
  FX_TRY(congestion_alloc(d, cols, rows, s));
  // RoutingGrid::new (grid.rs:27-31): f32 cell size and capacity.
  const float cw = d->chip_w / (float)cols;
  const float ch = d->chip_h / (float)rows;
  const float cap = (cw + ch) * 0.5f;
  cudaEvent_t ev;
  timer_begin(ctx, FX_STAGE_CONGESTION, s, &ev);
  int nb = (d->m + kNetThreads - 1) / kNetThreads;
  if (nb > kMaxNetBlocks) nb = kMaxNetBlocks;
  if (nb < 1) nb = 1;
  cong_nets_kernel<<<nb, kNetThreads, 0, s>>>(
      d->net_ptr.p, d->net_gate.p, dx, dy, d->m, cw, ch, cols, rows, w.diff.p,
      w.partial.p, w.done.p, w.result.p);
  FX_CHECK_LAUNCH();
  cong_scan_rows_kernel<<<rows, 1024, 0, s>>>(w.diff.p, cols, rows);
  FX_CHECK_LAUNCH();
  const int cb = (cols + 31) / 32;
  if (cb > 4096) {
    set_error("congestion grid too wide (%d columns)", cols);
    return FX_EINVAL;
  }
  cong_scan_cols_kernel<<<cb, dim3(32, 32), 0, s>>>(
      w.diff.p, w.counts.p, cols, rows, cap, w.partial.p + kMaxNetBlocks,
      w.partial_max.p, w.done.p + 1, w.result.p, w.result_max.p);
  FX_CHECK_LAUNCH();
  ctx->launches += 3;
  timer_end(ctx, FX_STAGE_CONGESTION, s, ev);
  return FX_OK;
}

}  // namespace fx

using namespace fx;

extern "C" int fx_congestion(fx_ctx *ctx, fx_design *d, const float *x,
                             const float *y, int32_t cols, int32_t rows,
                             uint32_t *out_counts, double *out_hpwl,
                             double *out_total_overflow,
                             float *out_max_overflow) {
  if (!ctx || !d || cols <= 0 || rows <= 0 || (x == nullptr) != (y == nullptr)) {
    set_error("fx_congestion: invalid arguments");
    return FX_EINVAL;
  }
  if ((int64_t)cols * rows > (int64_t)1 << 28 || cols > 4096 * 32) {
    set_error("fx_congestion: grid %d x %d too large", cols, rows);
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream;
  const float *dx = d->x[d->cur].p, *dy = d->y[d->cur].p;
  if (x) {
    // Stage host positions in the inactive ping-pong buffer.
    const int o = d->cur ^ 1;
    FX_CHECK_CUDA(cudaMemcpyAsync(d->x[o].p, x, (size_t)d->n * 4,
                                  cudaMemcpyHostToDevice, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(d->y[o].p, y, (size_t)d->n * 4,
                                  cudaMemcpyHostToDevice, s));
    dx = d->x[o].p;
    dy = d->y[o].p;
  }
  FX_TRY(congestion_run(ctx, d, dx, dy, cols, rows, s));
  CongWork &w = d->cong;
  double res[2] = {0, 0};
  float mx = 0.f;
  if (out_counts)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_counts, w.counts.p,
                                  (size_t)cols * rows * 4,
                                  cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(res, w.result.p, 16, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(&mx, w.result_max.p, 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (out_hpwl) *out_hpwl = res[0];
  if (out_total_overflow) *out_total_overflow = res[1];
  if (out_max_overflow) *out_max_overflow = mx;
  return FX_OK;
}

// ---- congestion without allocation --------------------------------------------
// fx_congestion sizes its workspace on first use and again whenever the grid
// changes. Some callers may not allocate device memory at that point: a host
// framework whose own pool already holds the HBM (a fresh cudaMalloc can then
// fail mid-run), or a loop that cannot accept the device-wide wait that
// cudaFree implies while other streams are busy. fx_congestion_noalloc runs
// the same three kernels with all their scratch in one fixed array declared
// below, and writes its results to device buffers the caller already owns.
namespace fx {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Layout of the scratch array (byte offsets, each 256-aligned):
//   [0]      two last-block counters        -- must be zero when a call starts
//   [256]    result slots for NULL outputs  (2 doubles + 1 float)
//   [512]    FP64 block partials            (kMaxNetBlocks + 4096 doubles)
//   [..]     f32 block maxima               (4096 floats)
//   [..]     difference array               -- must be zero when a call starts
// Each successful call leaves both zero-required regions zero again: the
// column scan clears every difference entry it reads and the last block of
// each reduction resets its counter. The first call on a device zeroes the
// whole array; a call that fails after launching marks the device so the
// next call zeroes it again before use.
constexpr size_t kNaDone = 0;
constexpr size_t kNaResult = 256;
constexpr size_t kNaPartial = 512;
constexpr size_t kNaPartialMax = kNaPartial + (size_t)(kMaxNetBlocks + 4096) * 8;
constexpr size_t kNaDiff = kNaPartialMax + 4096 * 4;
constexpr size_t kNaDiffEntries = (kNoAllocScratchBytes - kNaDiff) / 4;
static_assert(kNaPartialMax % 256 == 0 && kNaDiff % 256 == 0, "scratch alignment");

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mu;
unsigned char *g_na_ptr[kNaMaxDevices] = {};
bool g_na_dirty[kNaMaxDevices] = {};

// Once per device: the device address of the scratch array, zeroed. The
// zeroing runs on the calling context's stream (non-blocking, so it would
// not wait for a legacy-stream memset) and set-up waits for it, so this
// call's kernels and every later call see a zero array.
int noalloc_scratch(int device, cudaStream_t s, unsigned char **out) {
  if (device < 0 || device >= kNaMaxDevices) {
    set_error("fx_congestion_noalloc: device %d out of range", device);
    return FX_EINVAL;
  }
  if (!g_na_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error("fx_congestion_noalloc: cudaGetSymbolAddress failed: %s",
                cudaGetErrorString(e));
      return FX_ECUDA;
    }
    FX_CHECK_CUDA(cudaMemsetAsync(p, 0, kNoAllocScratchBytes, s));
    FX_CHECK_CUDA(cudaStreamSynchronize(s));
    g_na_ptr[device] = static_cast<unsigned char *>(p);
    g_na_dirty[device] = false;
  }
  *out = g_na_ptr[device];
  return FX_OK;
}

}  // namespace
}  // namespace fx

extern "C" int fx_congestion_noalloc(fx_ctx *ctx, const fx_design *d, const float *d_x,
                                     const float *d_y, int32_t cols, int32_t rows,
                                     uint32_t *d_counts, double *d_hpwl_overflow,
                                     float *d_max_overflow) {
  if (!ctx || !d || !d_counts || cols <= 0 || rows <= 0 ||
      (d_x == nullptr) != (d_y == nullptr)) {
    set_error("fx_congestion_noalloc: invalid arguments");
    return FX_EINVAL;
  }
  const int64_t entries = (int64_t)(cols + 1) * (rows + 1);
  if (entries > (int64_t)kNaDiffEntries || (cols + 31) / 32 > 4096) {
    set_error("fx_congestion_noalloc: a %d x %d grid needs %lld bytes of scratch, the "
              "fixed array holds %zu; use fx_congestion for this grid",
              cols, rows, (long long)(entries * 4), (size_t)(kNaDiffEntries * 4));
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lock(g_na_mu);
  unsigned char *sc = nullptr;
  cudaStream_t s = ctx->stream;
  FX_TRY(noalloc_scratch(ctx->device, s, &sc));
  if (g_na_dirty[ctx->device]) {
    FX_CHECK_CUDA(cudaMemsetAsync(sc, 0, kNoAllocScratchBytes, s));
    g_na_dirty[ctx->device] = false;
  }
  unsigned int *done = reinterpret_cast<unsigned int *>(sc + kNaDone);
  double *partial = reinterpret_cast<double *>(sc + kNaPartial);
  float *pmax = reinterpret_cast<float *>(sc + kNaPartialMax);
  int32_t *diff = reinterpret_cast<int32_t *>(sc + kNaDiff);
  double *result = d_hpwl_overflow ? d_hpwl_overflow
                                   : reinterpret_cast<double *>(sc + kNaResult);
  float *result_max = d_max_overflow ? d_max_overflow
                                     : reinterpret_cast<float *>(sc + kNaResult + 16);
  const float *px = d_x ? d_x : d->x[d->cur].p;
  const float *py = d_y ? d_y : d->y[d->cur].p;
  // RoutingGrid::new (grid.rs:27-31), as in congestion_run
  const float cw = d->chip_w / (float)cols;
  const float ch = d->chip_h / (float)rows;
  const float cap = (cw + ch) * 0.5f;
  int nb = (d->m + kNetThreads - 1) / kNetThreads;
  if (nb > kMaxNetBlocks) nb = kMaxNetBlocks;
  if (nb < 1) nb = 1;
  cong_nets_kernel<<<nb, kNetThreads, 0, s>>>(d->net_ptr.p, d->net_gate.p, px, py, d->m,
                                               cw, ch, cols, rows, diff, partial, done,
                                               result);
  cong_scan_rows_kernel<<<rows, 1024, 0, s>>>(diff, cols, rows);
  cong_scan_cols_kernel<<<(cols + 31) / 32, dim3(32, 32), 0, s>>>(
      diff, d_counts, cols, rows, cap, partial + kMaxNetBlocks, pmax, done + 1, result,
      result_max);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_na_dirty[ctx->device] = true;
    set_error("fx_congestion_noalloc: launch failed: %s", cudaGetErrorString(e));
    return FX_ECUDA;
  }
  ctx->launches += 3;
  return FX_OK;
}
