// fx_bh.cu -- row B: Barnes-Hut repulsion on the device.
//
// Tree semantics follow the reference quadtree (O/src/cpp/BarnesHutTree.cpp):
//   * root square: bounding box grown by a margin of 1.0, side = the larger
//     extent, centred on the box (BarnesHutTree.cpp:24-46);
//   * quadrant rule: a point on a midline goes west/south (`px <= mx`,
//     BarnesHutTree.cpp:107-123). The quantised key uses ceil(t) - 1, which
//     maps (k, k+1] to cell k, so a point exactly on a boundary falls in the
//     lower cell;
//   * opening rule: a node is replaced by its centre of mass when it is a
//     single point or size / max(d, min_dist) < theta (BarnesHutTree.cpp:
//     151-166); the law is k * q * Q / d^2 along the unit vector
//     (placer.rs:258-272, q = 1).
// Instead of pointer insertion the tree is built from sorted 30-bit Morton
// keys (15 bits per axis): a binary radix tree (Karras 2012) whose nodes are
// mapped back to quadtree cells. A binary node whose prefix length is
// delta, under a parent of prefix length delta_p, holds exactly the points of
// every quad cell of level l with delta_p < 2l <= delta; those cells share
// one centre of mass, so the walk tests only the smallest (level
// floor(delta/2)). Nodes that stand for no quad level (delta_p and delta in
// the same level) are always opened. Points that share all 30 key bits form
// a bucket (a cell of level 15): it is accepted as a whole by the same rule,
// otherwise each of its points interacts directly.
// Deep keys: the distance in the opening rule is clamped to min_dist, so a
// cell smaller than theta * min_dist is accepted by every point. When a
// level-15 cell is not (size^2 >= theta^2 min_dist^2, decided on the device
// from the root square), each point also gets the 24-bit key of its sub-cell
// within its level-15 cell (12 more levels, computed in f64), the points are
// sorted by (key, sub-key, index), and the tree has 27 levels: its buckets
// are then accepted whole by every point, and a crowded cell costs log k per
// point instead of k. The host skips these kernels when the positions lie in
// the die and (die + 2) / 2^15 < theta * min_dist.
//
// Every value is fixed by the sorted keys alone: node mass sums are added in
// tree order (left + right, FP64) by a bottom-up sweep, decisions and forces
// use IEEE f32 operations without contraction (the inverse square root is a
// fixed bit-level estimate plus Newton steps), and each point adds its terms
// in a fixed order. The result is bit-identical run to run and to a sequential
// restatement of the same rules.
#include <algorithm>
#include <climits>
#include <cstdlib>

#include "fx_internal.h"
#include "fx_device.cuh"

namespace fx {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys
constexpr int kWalkWarps = 8;
constexpr int kStack = 64;       // walk stack of a 15-level tree (<= 3 * 15 + 4)
constexpr int kStackDeep = 96;   // of a 27-level tree (<= 3 * 27 + 4)
constexpr int kDeepLevels = 12;  // levels below 15 in deep mode
constexpr int kKeyBits = 30, kDeepBits = kKeyBits + 2 * kDeepLevels;

// ---- bounding box and root square ----------------------------------------
__global__ void bh_bbox_kernel(const float *__restrict__ x,
                               const float *__restrict__ y, int n,
                               unsigned int *__restrict__ bbox) {
  float mnx = FLT_MAX, mny = FLT_MAX, mxx = -FLT_MAX, mxy = -FLT_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const float px = x[i], py = y[i];
    mnx = fminf(mnx, px);
    mxx = fmaxf(mxx, px);
    mny = fminf(mny, py);
    mxy = fmaxf(mxy, py);
  }
  __shared__ float red[4][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
  }
  if (lane == 0) {
    red[0][w] = mnx;
    red[1][w] = mny;
    red[2][w] = mxx;
    red[3][w] = mxy;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
      mnx = fminf(mnx, red[0][q]);
      mny = fminf(mny, red[1][q]);
      mxx = fmaxf(mxx, red[2][q]);
      mxy = fmaxf(mxy, red[3][q]);
    }
    atomicMin(bbox + 0, f2ord(mnx));
    atomicMin(bbox + 1, f2ord(mny));
    atomicMax(bbox + 2, f2ord(mxx));
    atomicMax(bbox + 3, f2ord(mxy));
  }
}

// Root square from the box (BarnesHutTree.cpp:24-46, in f32 without
// contraction), then re-arms the box for the next accumulation.
__global__ void bh_root_kernel(unsigned int *__restrict__ bbox,
                               float *__restrict__ root, float th2, float md2) {
  float mnx = ord2f(bbox[0]), mny = ord2f(bbox[1]);
  float mxx = ord2f(bbox[2]), mxy = ord2f(bbox[3]);
  mnx = __fsub_rn(mnx, 1.0f);
  mxx = __fadd_rn(mxx, 1.0f);
  mny = __fsub_rn(mny, 1.0f);
  mxy = __fadd_rn(mxy, 1.0f);
  const float size = fmaxf(__fsub_rn(mxx, mnx), __fsub_rn(mxy, mny));
  const float cx = __fmul_rn(__fadd_rn(mnx, mxx), 0.5f);
  const float cy = __fmul_rn(__fadd_rn(mny, mxy), 0.5f);
  const float half = __fmul_rn(size, 0.5f);
  root[0] = __fsub_rn(cx, half);
  root[1] = __fsub_rn(cy, half);
  root[2] = size;
  // deep keys when a level-15 cell is not always accepted
  const float s15 = ldexpf(size, -15);
  root[3] = __fmul_rn(s15, s15) >= __fmul_rn(th2, md2) ? 1.0f : 0.0f;
  bbox[0] = 0xffffffffu;
  bbox[1] = 0xffffffffu;
  bbox[2] = 0u;
  bbox[3] = 0u;
}

__device__ __forceinline__ uint32_t quantize15(float p, float o, float size) {
  const float t = __fmul_rn(__fdiv_rn(__fsub_rn(p, o), size), 32768.0f);
  if (!(t > 0.0f)) return 0u;
  const float c = ceilf(t);
  if (c >= 32768.0f) return 32767u;
  return (uint32_t)c - 1u;
}

__device__ __forceinline__ uint32_t spread15(uint32_t v) {
  v &= 0x7fffu;
  v = (v | (v << 8)) & 0x00ff00ffu;
  v = (v | (v << 4)) & 0x0f0f0f0fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

// Sub-cell (0..4095) of p within its level-15 cell c15, in f64 without
// contraction; a point the f32 quantisation put in c15 but that lies just
// outside it is clamped to the edge sub-cell, so cells nest.
__device__ __forceinline__ uint32_t quantize_sub(float p, float o, float size, uint32_t c15) {
  const double w = __ddiv_rn((double)size, 32768.0);
  const double o15 = __dadd_rn((double)o, __dmul_rn((double)c15, w));
  const double t = __dmul_rn(__ddiv_rn(__dsub_rn((double)p, o15), w), 4096.0);
  if (!(t > 0.0)) return 0u;
  const double c = ceil(t);
  if (c >= 4096.0) return 4095u;
  return (uint32_t)c - 1u;
}

// Keys (and identity indices); with klo, also the 24-bit sub-cell keys and
// the deep sort's inputs.
__global__ void bh_keys_kernel(const float *__restrict__ x,
                               const float *__restrict__ y, int n,
                               const float *__restrict__ root,
                               uint32_t *__restrict__ keys,
                               int32_t *__restrict__ idx, uint32_t *__restrict__ klo,
                               uint32_t *__restrict__ kl0, int32_t *__restrict__ il0) {
  const float ox = root[0], oy = root[1], size = root[2];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const uint32_t qx = quantize15(x[i], ox, size);
    const uint32_t qy = quantize15(y[i], oy, size);
    keys[i] = (spread15(qx) << 1) | spread15(qy);
    idx[i] = i;
    if (klo) {
      const uint32_t lo = (spread15(quantize_sub(x[i], ox, size, qx)) << 1) |
                          spread15(quantize_sub(y[i], oy, size, qy));
      klo[i] = lo;
      kl0[i] = lo;
      il0[i] = i;
    }
  }
}

// Deep mode only (root[3] set): the primary keys and indices in the order of
// the sub-key sort (gather into buffer 1, then copy back to buffer 0), and
// the sub-keys in the final sorted order.
__global__ void bh_deep_gather_kernel(const float *__restrict__ root, int n,
                                      const uint32_t *__restrict__ keys0,
                                      const int32_t *__restrict__ il1,
                                      uint32_t *__restrict__ keys1,
                                      int32_t *__restrict__ idx1) {
  if (!(root[3] > 0.f)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int g = il1[i];
    keys1[i] = keys0[g];
    idx1[i] = g;
  }
}

__global__ void bh_deep_copy_kernel(const float *__restrict__ root, int n,
                                    const uint32_t *__restrict__ keys1,
                                    const int32_t *__restrict__ idx1,
                                    uint32_t *__restrict__ keys0, int32_t *__restrict__ idx0) {
  if (!(root[3] > 0.f)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    keys0[i] = keys1[i];
    idx0[i] = idx1[i];
  }
}

__global__ void bh_deep_slo_kernel(const float *__restrict__ root, int n,
                                   const uint32_t *__restrict__ klo,
                                   const int32_t *__restrict__ idx0,
                                   uint32_t *__restrict__ slo) {
  if (!(root[3] > 0.f)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    slo[i] = klo[idx0[i]];
}

// ---- stable LSD radix sort (8-bit digits) ------------------------------------
__global__ void __launch_bounds__(kSortThreads)
radix_hist_kernel(const uint32_t *__restrict__ keys, int n, int shift,
                  uint32_t *__restrict__ tile_hist, int T,
                  const float *__restrict__ gate = nullptr) {
  if (gate && !(gate[3] > 0.f)) return;  // a deep-key pass outside deep mode
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * kSortTile;
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int i = base + r * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  tile_hist[(size_t)threadIdx.x * T + blockIdx.x] = h[threadIdx.x];
}

// Per-digit exclusive scan of the digit-major tile histogram: block d scans
// the T tile counts of digit d and records the digit's total.
__global__ void __launch_bounds__(256)
radix_scan_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                  uint32_t *__restrict__ digit_total, int T,
                  const float *__restrict__ gate = nullptr) {
  if (gate && !(gate[3] > 0.f)) return;
  __shared__ uint32_t ws[8];
  const int d = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
  const uint32_t *row = in + (size_t)d * T;
  uint32_t *orow = out + (size_t)d * T;
  const int per = (T + 255) / 256;
  const int b = min(T, t * per), e = min(T, b + per);
  uint32_t s = 0;
  for (int i = b; i < e; ++i) s += row[i];
  uint32_t v = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) ws[w] = v;
  __syncthreads();
  uint32_t run = v - s;
  for (int q = 0; q < w; ++q) run += ws[q];
  for (int i = b; i < e; ++i) {
    const uint32_t c = row[i];
    orow[i] = run;
    run += c;
  }
  if (t == 255) digit_total[d] = run;
}

// Stable scatter: within a tile, warp w ranks its 256 keys in order
// (__match_any_sync groups lanes with equal digits), warps are ordered by a
// per-digit prefix over the warp counts, tiles by the per-digit scan and
// digits by the scan of the digit totals.
__global__ void __launch_bounds__(kSortThreads)
radix_scatter_kernel(const uint32_t *__restrict__ kin,
                     const int32_t *__restrict__ iin,
                     uint32_t *__restrict__ kout, int32_t *__restrict__ iout,
                     int n, int shift, const uint32_t *__restrict__ tile_scan,
                     const uint32_t *__restrict__ digit_total, int T,
                     const float *__restrict__ gate = nullptr) {
  if (gate && !(gate[3] > 0.f)) return;
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t cnt[kWarps][256];
  __shared__ uint32_t doff[256];
  __shared__ uint32_t ws[kWarps];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  for (int i = t; i < kWarps * 256; i += kSortThreads) (&cnt[0][0])[i] = 0;
  {
    const uint32_t s = digit_total[t];
    uint32_t v = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    if (lane == 31) ws[w] = v;
    __syncthreads();
    uint32_t off = v - s;
    for (int q = 0; q < w; ++q) off += ws[q];
    doff[t] = off;
  }
  __syncthreads();
  const int base = blockIdx.x * kSortTile + w * (32 * kSortItems);
  const unsigned lt_mask = (1u << lane) - 1u;
  uint32_t k[kSortItems];
  int32_t v[kSortItems];
  uint32_t rank[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int i = base + r * 32 + lane;
    const bool valid = i < n;
    k[r] = valid ? kin[i] : 0u;
    v[r] = valid ? iin[i] : 0;
    const uint32_t dg = valid ? ((k[r] >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, dg);
    const int leader = __ffs(peers) - 1;
    const uint32_t old = valid ? cnt[w][dg] : 0u;
    __syncwarp();
    if (valid && lane == leader) cnt[w][dg] = old + __popc(peers);
    __syncwarp();
    rank[r] = old + __popc(peers & lt_mask);
  }
  __syncthreads();
  // thread t = digit t: offsets of the warps within the digit, and the
  // digit's start within the tile (exclusive scan over digits)
  __shared__ uint32_t tstart[256];
  __shared__ uint32_t gbase[256];
  {
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < kWarps; ++ww) {
      const uint32_t c = cnt[ww][t];
      cnt[ww][t] = run;
      run += c;
    }
    uint32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    __syncthreads();
    if (lane == 31) ws[w] = x;
    __syncthreads();
    uint32_t st = x - run;
    for (int q = 0; q < w; ++q) st += ws[q];
    tstart[t] = st;
    // output index of tile position j of digit t: gbase[t] + j
    gbase[t] = doff[t] + tile_scan[(size_t)t * T + blockIdx.x] - st;
  }
  __syncthreads();
  // stage the tile in sorted order, then write it out: consecutive threads
  // cover consecutive positions of a digit's run, so the stores coalesce
  __shared__ uint32_t sk[kSortTile];
  __shared__ int32_t sv[kSortTile];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int i = base + r * 32 + lane;
    if (i < n) {
      const uint32_t dg = (k[r] >> shift) & 255u;
      const uint32_t j = tstart[dg] + cnt[w][dg] + rank[r];
      sk[j] = k[r];
      sv[j] = v[r];
    }
  }
  __syncthreads();
  const int m = min(kSortTile, n - (int)(blockIdx.x * kSortTile));
  for (int j = t; j < m; j += kSortThreads) {
    const uint32_t key = sk[j];
    const uint32_t pos = gbase[(key >> shift) & 255u] + (uint32_t)j;
    kout[pos] = key;
    iout[pos] = sv[j];
  }
}

// Stable LSD sort of (key, value) pairs on the low 8*passes key bits. The
// pairs start in (k[0], v[0]); the result is in (k[passes & 1], v[passes & 1]).
// Workspace: tile_hist / tile_scan of 256 * radix_sort_tiles(n) words each
// and digit_total of 256 words.
int radix_sort_pairs(uint32_t *k[2], int32_t *v[2], int n, int passes,
                     uint32_t *tile_hist, uint32_t *tile_scan, uint32_t *digit_total,
                     cudaStream_t s) {
  if (n <= 0) return FX_OK;
  const int T = (n + kSortTile - 1) / kSortTile;
  for (int pass = 0; pass < passes; ++pass) {
    const int src = pass & 1, dst = src ^ 1;
    radix_hist_kernel<<<T, kSortThreads, 0, s>>>(k[src], n, 8 * pass, tile_hist, T);
    radix_scan_kernel<<<256, 256, 0, s>>>(tile_hist, tile_scan, digit_total, T);
    radix_scatter_kernel<<<T, kSortThreads, 0, s>>>(k[src], v[src], k[dst], v[dst], n,
                                                    8 * pass, tile_scan, digit_total, T);
  }
  FX_CHECK_LAUNCH();
  return FX_OK;
}

int radix_sort_tiles(int n) { return (n + kSortTile - 1) / kSortTile; }

// ---- one-sweep LSD radix sort (the Barnes-Hut keys) ----------------------------
// The same stable sort in 1 + passes launches instead of 3 per pass: one
// kernel counts every pass's digits at once; then each pass is one kernel in
// which a block takes the next tile (an atomic ticket, so tiles start in
// order), ranks its keys stably as radix_scatter_kernel does, publishes its
// per-digit counts and finds the counts of all earlier tiles by a look-back
// over their published words (decoupled look-back). A block waits only on
// tiles whose blocks have started and publish their own counts before they
// wait, so every wait ends; each is still bounded, and an expired wait sets
// bit 4 of the error word (the host turns it into FX_ETIMEOUT).
constexpr uint32_t kOsAgg = 1u << 30, kOsInc = 2u << 30, kOsVal = (1u << 30) - 1u;
constexpr uint32_t kOsSpin = 1u << 22;
constexpr int kOsWin = 16;  // earlier tiles read per look-back step
// 4096-key tiles: the look-back chain (one round trip per kOsWin tiles
// whose predecessors have not finished) is half as long as with 2048.
constexpr int kOsItems = 16;
constexpr int kOsTile = kSortThreads * kOsItems;
static int os_tiles(int n) { return (n + kOsTile - 1) / kOsTile; }

__global__ void __launch_bounds__(kSortThreads)
os_hist_kernel(const uint32_t *__restrict__ keys, int n, int passes,
               uint32_t *__restrict__ hist) {
  __shared__ uint32_t h[4][256];
  for (int i = threadIdx.x; i < 4 * 256; i += kSortThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  for (int i = blockIdx.x * kSortThreads + threadIdx.x; i < n; i += gridDim.x * kSortThreads) {
    const uint32_t k = keys[i];
    for (int q = 0; q < passes; ++q) atomicAdd(&h[q][(k >> (8 * q)) & 255u], 1u);
  }
  __syncthreads();
  for (int q = 0; q < passes; ++q) {
    const uint32_t c = h[q][threadIdx.x];
    if (c) atomicAdd(hist + q * 256 + threadIdx.x, c);
  }
}

__global__ void __launch_bounds__(kSortThreads, 3)
os_pass_kernel(const uint32_t *__restrict__ kin, const int32_t *__restrict__ iin,
               uint32_t *__restrict__ kout, int32_t *__restrict__ iout, int n, int shift,
               const uint32_t *__restrict__ hist, uint32_t *__restrict__ status,
               unsigned int *__restrict__ ticket, unsigned int *__restrict__ err,
               const float *__restrict__ px, const float *__restrict__ py,
               float2 *__restrict__ spos) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t cnt[kWarps][256];
  __shared__ uint32_t tstart[256], gbase[256], ws[kWarps];
  __shared__ int tile_s;
  __shared__ uint32_t sk[kOsTile];
  __shared__ int32_t sv[kOsTile];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t == 0) tile_s = (int)atomicAdd(ticket, 1u);
  for (int i = t; i < kWarps * 256; i += kSortThreads) (&cnt[0][0])[i] = 0;
  __syncthreads();
  const int tile = tile_s;
  // base of every digit: exclusive scan of this pass's digit counts
  uint32_t dbase;
  {
    const uint32_t c = hist[t];
    uint32_t v = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    if (lane == 31) ws[w] = v;
    __syncthreads();
    dbase = v - c;
    for (int q = 0; q < w; ++q) dbase += ws[q];
    __syncthreads();
  }
  // stable ranks within the tile: per warp by __match_any_sync, then warps
  // in order (as radix_scatter_kernel)
  const int base = tile * kOsTile + w * (32 * kOsItems);
  const unsigned lt_mask = (1u << lane) - 1u;
  uint32_t k[kOsItems];
  int32_t v[kOsItems];
  uint32_t rank[kOsItems];
#pragma unroll
  for (int r = 0; r < kOsItems; ++r) {
    const int i = base + r * 32 + lane;
    const bool valid = i < n;
    k[r] = valid ? kin[i] : 0u;
    v[r] = valid ? iin[i] : 0;
    const uint32_t dg = valid ? ((k[r] >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, dg);
    const int leader = __ffs(peers) - 1;
    const uint32_t old = valid ? cnt[w][dg] : 0u;
    __syncwarp();
    if (valid && lane == leader) cnt[w][dg] = old + __popc(peers);
    __syncwarp();
    rank[r] = old + __popc(peers & lt_mask);
  }
  __syncthreads();
  // thread t = digit t: warp offsets within the digit, the digit's count in
  // this tile, and its start within the tile
  uint32_t local;
  {
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < kWarps; ++ww) {
      const uint32_t c = cnt[ww][t];
      cnt[ww][t] = run;
      run += c;
    }
    local = run;
    uint32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    uint32_t st = x - run;
    for (int q = 0; q < w; ++q) st += ws[q];
    tstart[t] = st;
  }
  // decoupled look-back for digit t
  {
    volatile uint32_t *stv = status;
    uint32_t *my = status + (size_t)tile * 256 + t;
    if (tile == 0) {
      atomicExch(my, kOsInc | local);
      gbase[t] = dbase - tstart[t];
    } else {
      atomicExch(my, kOsAgg | local);
      // The words of the kOsWin nearest earlier tiles are loaded together
      // (independent loads, one round trip) and added from the nearest on,
      // up to the first inclusive one; a tile that has not published yet is
      // waited for (bounded), then the window restarts from it.
      uint32_t prefix = 0;
      uint32_t spin = 0;
      for (int p = tile - 1; p >= 0;) {
        uint32_t wv[kOsWin];
#pragma unroll
        for (int q = 0; q < kOsWin; ++q)
          wv[q] = p - q >= 0 ? (uint32_t)stv[(size_t)(p - q) * 256 + t] : (uint32_t)(2u << 30);  // before tile 0: inclusive 0
        int q = 0;
        bool done = false;
#pragma unroll
        for (int r = 0; r < kOsWin; ++r) {
          if (done || q < r) continue;  // stopped at an earlier entry
          const uint32_t flag = wv[r] & ~kOsVal;
          if (flag == 0u) break;         // not published yet: q == r
          prefix += wv[r] & kOsVal;
          q = r + 1;
          if (flag == kOsInc) done = true;
        }
        if (done) break;
        p -= q;
        if (q < kOsWin && p >= 0) {  // wait for tile p to publish
          while ((stv[(size_t)p * 256 + t] & ~kOsVal) == 0u && spin < kOsSpin) ++spin;
          if (spin >= kOsSpin) {  // expired: record it and stop
            atomicOr(err, 4u);
            break;
          }
        }
      }
      __threadfence();
      atomicExch(my, kOsInc | (prefix + local));
      gbase[t] = dbase + prefix - tstart[t];
    }
  }
  __syncthreads();
  // stage the tile in sorted order, then write it out coalesced
#pragma unroll
  for (int r = 0; r < kOsItems; ++r) {
    const int i = base + r * 32 + lane;
    if (i < n) {
      const uint32_t dg = (k[r] >> shift) & 255u;
      const uint32_t j = tstart[dg] + cnt[w][dg] + rank[r];
      sk[j] = k[r];
      sv[j] = v[r];
    }
  }
  __syncthreads();
  const int m = min(kOsTile, n - tile * kOsTile);
  for (int j = t; j < m; j += kSortThreads) {
    const uint32_t key = sk[j];
    const uint32_t pos = gbase[(key >> shift) & 255u] + (uint32_t)j;
    const int32_t g = sv[j];
    kout[pos] = key;
    iout[pos] = g;
    if (spos) spos[pos] = make_float2(px[g], py[g]);
  }
}

// Stable LSD sort of (key, value) pairs on the low 8*passes (<= 4) key bits,
// in 1 + passes launches. With spos, the last pass also writes
// spos[i] = (px[v], py[v]) for the sorted values v. Pairs start in (k[0], v[0]); the result is in
// (k[passes & 1], v[passes & 1]). Workspace `ws`: os_sort_words(n, passes)
// words, cleared here.
size_t os_sort_words(int n, int passes) {
  return (size_t)passes * 256 + (size_t)passes * os_tiles(n) * 256 + 4;
}

int radix_sort_onesweep(uint32_t *k[2], int32_t *v[2], int n, int passes, uint32_t *ws,
                        unsigned int *err, cudaStream_t s, const float *px,
                        const float *py, float2 *spos) {
  if (n <= 0) return FX_OK;
  if (passes > 4 || n >= (int)kOsVal) {
    set_error("radix_sort_onesweep: %d keys / %d passes out of range", n, passes);
    return FX_EINVAL;
  }
  const int T = os_tiles(n);
  uint32_t *hist = ws, *status = ws + passes * 256,
           *ticket = status + (size_t)passes * T * 256;
  FX_CHECK_CUDA(cudaMemsetAsync(ws, 0, os_sort_words(n, passes) * 4, s));
  const int hb = std::min(T, 2 * 148);
  os_hist_kernel<<<hb, kSortThreads, 0, s>>>(k[0], n, passes, hist);
  for (int pass = 0; pass < passes; ++pass) {
    const int src = pass & 1, dst = src ^ 1;
    const bool last = pass == passes - 1;
    os_pass_kernel<<<T, kSortThreads, 0, s>>>(k[src], v[src], k[dst], v[dst], n, 8 * pass,
                                              hist + 256 * pass,
                                              status + (size_t)pass * T * 256, ticket + pass,
                                              err, px, py, last ? spos : nullptr);
  }
  FX_CHECK_LAUNCH();
  return FX_OK;
}

// ---- radix tree (Karras 2012) -----------------------------------------------
// Common prefix length of the keys at sorted positions i and j: 30-bit key,
// then (deep mode, lo != null) the 24-bit sub-key, then the index.
__device__ __forceinline__ int bh_delta(const uint32_t *__restrict__ keys,
                                        const uint32_t *__restrict__ lo,
                                        int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t a = keys[i], b = keys[j];
  if (a != b) return __clz(a ^ b) - 2;
  if (lo) {
    const uint32_t la = lo[i], lb = lo[j];
    if (la != lb) return kKeyBits + __clz(la ^ lb) - 8;
    return kDeepBits + __clz((uint32_t)(i ^ j));
  }
  return kKeyBits + __clz((uint32_t)(i ^ j));
}

__global__ void bh_tree_kernel(const uint32_t *__restrict__ keys,
                               const uint32_t *__restrict__ slo,
                               const float *__restrict__ root, int n,
                               int32_t *__restrict__ child,
                               int32_t *__restrict__ range,
                               int32_t *__restrict__ dnode,
                               int32_t *__restrict__ dparent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const uint32_t *sub = (slo && root[3] > 0.f) ? slo : nullptr;
  const int dr = bh_delta(keys, sub, n, i, i + 1), dl = bh_delta(keys, sub, n, i, i - 1);
  const int d = (dr - dl) >= 0 ? 1 : -1;
  const int dmin = bh_delta(keys, sub, n, i, i - d);
  int lmax = 2;
  while (bh_delta(keys, sub, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (bh_delta(keys, sub, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dn = bh_delta(keys, sub, n, i, j);
  int s = 0;
  for (int div = 2;; div *= 2) {
    const int t = (l + div - 1) / div;
    if (bh_delta(keys, sub, n, i, i + (s + t) * d) > dn) s += t;
    if (t == 1) break;
  }
  const int gamma = i + s * d + min(d, 0);
  const int lo = min(i, j), hi = max(i, j);
  const int left = (lo == gamma) ? ~gamma : gamma;
  const int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
  child[2 * i] = left;
  child[2 * i + 1] = right;
  range[2 * i] = lo;
  range[2 * i + 1] = hi;
  dnode[i] = dn;
  if (left >= 0) dparent[left] = dn;
  if (right >= 0) dparent[right] = dn;
  if (i == 0) dparent[0] = -1;
}

// ---- exact prefix sums of the sorted positions ---------------------------------
// Every position becomes the 128-bit integer trunc(v * 2^64) (exact for
// |v| >= 2^-41; smaller magnitudes lose their bits below 2^-64, non-finite
// values count as 0). Integer sums do not depend on the order of addition,
// so the prefix is computed tile-parallel and a node's sum, a prefix
// difference, is exact. Its centre of mass is then
//   ((double)hi * 2^64 + (double)lo) * 2^-64 / count
// with hi/lo the upper (signed) and lower (unsigned) 64 bits, each step
// rounded to nearest.
constexpr int kFixThreads = 256, kFixItems = 8, kFixTile = kFixThreads * kFixItems;

__device__ __forceinline__ __int128 fixed64(float v) {
  const uint32_t u = __float_as_uint(v);
  const int e = (int)((u >> 23) & 255u);
  if (e == 0 || e == 255) return 0;
  const unsigned long long m = (u & 0x7fffffu) | 0x800000u;  // v = m * 2^(e - 150)
  const int sh = e - 86;                                     // v * 2^64 = m * 2^(e - 86)
  unsigned __int128 r = 0;
  if (sh >= 0) r = (unsigned __int128)m << sh;
  else if (sh > -64) r = m >> (-sh);
  return (u >> 31) ? -(__int128)r : (__int128)r;
}

__device__ __forceinline__ ulonglong2 pack128(__int128 v) {
  return make_ulonglong2((unsigned long long)v, (unsigned long long)((unsigned __int128)v >> 64));
}
__device__ __forceinline__ __int128 unpack128(ulonglong2 p) {
  return (__int128)(((unsigned __int128)p.y << 64) | p.x);
}
__device__ __forceinline__ __int128 shfl_up128(__int128 v, int d) {
  const ulonglong2 p = pack128(v);
  return unpack128(make_ulonglong2(__shfl_up_sync(0xffffffffu, p.x, d),
                                   __shfl_up_sync(0xffffffffu, p.y, d)));
}

// Inclusive scan of one int128 per thread over the block; also returns the
// block total.
__device__ __forceinline__ __int128 block_scan128(__int128 v, __int128 &total) {
  __shared__ ulonglong2 wtot[kFixThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const __int128 u = shfl_up128(v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) wtot[w] = pack128(v);
  __syncthreads();
  __int128 off = 0, tot = 0;
  for (int q = 0; q < kFixThreads / 32; ++q) {
    const __int128 t = unpack128(wtot[q]);
    if (q < w) off += t;
    tot += t;
  }
  __syncthreads();
  total = tot;
  return v + off;
}

// Pass 1: the (x, y) sums of each tile of kFixTile sorted points.
__global__ void __launch_bounds__(kFixThreads)
fix_tile_kernel(const float2 *__restrict__ spos, int n, ulonglong4 *__restrict__ tile_sum) {
  const int b0 = blockIdx.x * kFixTile + threadIdx.x * kFixItems;
  __int128 sx = 0, sy = 0;
#pragma unroll
  for (int k = 0; k < kFixItems; ++k) {
    const int i = b0 + k;
    if (i < n) {
      const float2 p = spos[i];
      sx += fixed64(p.x);
      sy += fixed64(p.y);
    }
  }
  __int128 tx, ty;
  block_scan128(sx, tx);
  block_scan128(sy, ty);
  if (threadIdx.x == 0) {
    const ulonglong2 a = pack128(tx), c = pack128(ty);
    tile_sum[blockIdx.x] = make_ulonglong4(a.x, a.y, c.x, c.y);
  }
}

// Pass 2: exclusive offsets of the tiles (one block, kFixThreads tiles at a
// time, carrying the running total; exact, so the grouping is free).
__global__ void __launch_bounds__(kFixThreads)
fix_top_kernel(ulonglong4 *__restrict__ tile_sum, int tiles) {
  __int128 cx = 0, cy = 0;
  for (int base = 0; base < tiles; base += kFixThreads) {
    const int t = base + threadIdx.x;
    __int128 vx = 0, vy = 0;
    if (t < tiles) {
      const ulonglong4 v = tile_sum[t];
      vx = unpack128(make_ulonglong2(v.x, v.y));
      vy = unpack128(make_ulonglong2(v.z, v.w));
    }
    __int128 tx, ty;
    const __int128 ix = block_scan128(vx, tx);
    const __int128 iy = block_scan128(vy, ty);
    if (t < tiles) {
      const ulonglong2 a = pack128(cx + ix - vx), c = pack128(cy + iy - vy);
      tile_sum[t] = make_ulonglong4(a.x, a.y, c.x, c.y);
    }
    cx += tx;
    cy += ty;
  }
}

// Pass 3: inclusive prefix of every point (x lo/hi, y lo/hi).
__global__ void __launch_bounds__(kFixThreads)
fix_prefix_kernel(const float2 *__restrict__ spos, int n,
                  const ulonglong4 *__restrict__ tile_off, ulonglong4 *__restrict__ prefix) {
  const int b0 = blockIdx.x * kFixTile + threadIdx.x * kFixItems;
  __int128 sx = 0, sy = 0;
#pragma unroll
  for (int k = 0; k < kFixItems; ++k) {
    const int i = b0 + k;
    if (i < n) {
      const float2 p = spos[i];
      sx += fixed64(p.x);
      sy += fixed64(p.y);
    }
  }
  __int128 tx, ty;
  const ulonglong4 to = tile_off[blockIdx.x];
  __int128 rx = block_scan128(sx, tx) - sx + unpack128(make_ulonglong2(to.x, to.y));
  __int128 ry = block_scan128(sy, ty) - sy + unpack128(make_ulonglong2(to.z, to.w));
  for (int k = 0; k < kFixItems; ++k) {  // the points again (cached), in order
    const int i = b0 + k;
    if (i >= n) break;
    const float2 p = spos[i];
    rx += fixed64(p.x);
    ry += fixed64(p.y);
    const ulonglong2 a = pack128(rx), c = pack128(ry);
    prefix[i] = make_ulonglong4(a.x, a.y, c.x, c.y);
  }
}

// ((double)hi * 2^64 + (double)lo) * 2^-64, each step rounded to nearest.
__device__ __forceinline__ double fixed_to_double(__int128 v) {
  const long long hi = (long long)(v >> 64);
  const unsigned long long lo = (unsigned long long)v;
  return __dmul_rn(__dadd_rn(__dmul_rn(__ll2double_rn(hi), 18446744073709551616.0),
                             __ull2double_rn(lo)),
                   5.42101086242752217003726400434970855712890625e-20);
}

// Walk record of every internal node (two float4):
//   r0 = {cx_hi, cy_hi, cx_lo, cy_lo}  centre of mass as an f32 hi/lo pair
//   r1 = {count (negative: bucket), size^2 (negative: no quad level),
//         first, last (as int bits)}
__device__ __forceinline__ void bh_qchild(int i, const int32_t *__restrict__ child,
                                          const int32_t *__restrict__ dnode, int kb,
                                          int4 *__restrict__ qchild);

// Also writes the node's quad children (bh_qchild below).
__global__ void bh_node_kernel(int n, const int32_t *__restrict__ range,
                               const int32_t *__restrict__ dnode,
                               const int32_t *__restrict__ dparent,
                               const ulonglong4 *__restrict__ prefix,
                               const float *__restrict__ root, int deep_ok,
                               float4 *__restrict__ node,
                               const int32_t *__restrict__ child,
                               int4 *__restrict__ qchild) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  bh_qchild(i, child, dnode, (deep_ok && root[3] > 0.f) ? kDeepBits : kKeyBits, qchild);
  const bool deep = deep_ok && root[3] > 0.f;
  const int kb = deep ? kDeepBits : kKeyBits;  // prefix length of a bucket
  const int f = range[2 * i], l = range[2 * i + 1];
  const int cnt = l - f + 1;
  const ulonglong4 pl = prefix[l];
  __int128 sx = unpack128(make_ulonglong2(pl.x, pl.y));
  __int128 sy = unpack128(make_ulonglong2(pl.z, pl.w));
  if (f > 0) {
    const ulonglong4 pf = prefix[f - 1];
    sx -= unpack128(make_ulonglong2(pf.x, pf.y));
    sy -= unpack128(make_ulonglong2(pf.z, pf.w));
  }
  const double cx = __ddiv_rn(fixed_to_double(sx), (double)cnt);
  const double cy = __ddiv_rn(fixed_to_double(sy), (double)cnt);
  const float hx = (float)cx, hy = (float)cy;
  node[2 * i] = make_float4(hx, hy, (float)(cx - (double)hx), (float)(cy - (double)hy));
  const int dn = dnode[i], dp = dparent[i];
  const float rs = root[2];
  float c, s2;
  if (dn >= kb) {
    const float sz = ldexpf(rs, -(kb >> 1));
    c = -(float)cnt;
    s2 = __fmul_rn(sz, sz);
  } else {
    const int lmax = dn >> 1;
    c = (float)cnt;
    if (dp >= 0 && (dp >> 1) == lmax) {
      s2 = -1.0f;
    } else {
      const float sz = ldexpf(rs, -lmax);
      s2 = __fmul_rn(sz, sz);
    }
  }
  node[2 * i + 1] = make_float4(c, s2, __int_as_float(f), __int_as_float(l));
}

// Quad children: a node that stands for no quad level (at most one such level
// separates two quad cells) is replaced by its own two children, so every
// node lists up to four children, in key order. kNone marks empty slots.
constexpr int kNone = INT_MIN;

__device__ __forceinline__ void bh_qchild(int i, const int32_t *__restrict__ child,
                                          const int32_t *__restrict__ dnode, int kb,
                                          int4 *__restrict__ qchild) {
  int out[4] = {kNone, kNone, kNone, kNone};
  int k = 0;
  const int lv = dnode[i] >> 1;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int c = child[2 * i + h];
    if (c >= 0 && dnode[c] < kb && (dnode[c] >> 1) == lv) {
      out[k++] = child[2 * c];
      out[k++] = child[2 * c + 1];
    } else {
      out[k++] = c;
    }
  }
  qchild[i] = make_int4(out[0], out[1], out[2], out[3]);
}

// ---- warp-cooperative walk ----------------------------------------------------
// Each warp owns 32 consecutive sorted points (spatially close), split into
// groups of kWalkGroup lanes. Each group walks the quadtree with its own
// shared stack of (node, lane mask) entries, each an opened cell; the groups
// of a warp pop in lockstep, so one pass of the loop serves up to 32/kWalkGroup
// cells. Popping a cell evaluates all its children for the lanes in the mask:
// every lane applies the reference opening rule to its own point, so
// interaction lists are exactly per point. A lane adds, per opened cell, the
// terms of its children in order (single points, accepted cells, opened
// buckets point by point), and then descends into the children it opened, in
// order. A group's stack holds the union of its points' opened cells, which
// near the leaves is much smaller than the union over the whole warp.

// 1/sqrt(x) for x >= min_dist^2 > 0: the bit-level estimate of Lomont
// ("Fast inverse square root", 2003; constant 0x5f375a86) refined by three
// Newton steps y <- y * fma(-(x/2) * y, y, 1.5) in IEEE f32. Integer ops,
// correctly rounded products and fused multiply-adds only (each written out
// explicitly, nothing left to contraction), so a sequential restatement with
// fmaf reproduces it bit for bit; the result is within a couple of ulp of the
// exact value.
__device__ __forceinline__ float bh_rsqrt(float x) {
  float y = __int_as_float(0x5f375a86 - (__float_as_int(x) >> 1));
  const float h = __fmul_rn(0.5f, x);
#pragma unroll
  for (int i = 0; i < 3; ++i)
    y = __fmul_rn(y, __fmaf_rn(-__fmul_rn(h, y), y, 1.5f));
  return y;
}

// The law k*Q/d^2 along (dx, dy)/d with d = max(|r|, min_dist), in f32:
// inv = rsqrt(max(r2, md^2)), f = ((kQ * inv) * inv) * inv,
// F = fma(f, r, F); r2 = fma(dx, dx, dy * dy).
template <bool Fast>
__device__ __forceinline__ void bh_term(float dx, float dy, float r2c, float kq,
                                        float &fx, float &fy) {
  const float inv = Fast ? rsqrtf(r2c) : bh_rsqrt(r2c);
  const float f = __fmul_rn(__fmul_rn(__fmul_rn(kq, inv), inv), inv);
  fx = __fmaf_rn(f, dx, fx);
  fy = __fmaf_rn(f, dy, fy);
}

template <bool Fast>
__device__ __forceinline__ void bh_direct(float px, float py, float2 q,
                                          float kq, float md2, float &fx,
                                          float &fy) {
  const float dx = __fsub_rn(px, q.x), dy = __fsub_rn(py, q.y);
  const float r2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
  bh_term<Fast>(dx, dy, fmaxf(r2, md2), kq, fx, fy);
}

// Applies the opening rule of child c (an internal node when `cell`) to the
// lane's point when `in`; adds accepted-cell, single-point and bucket terms
// (Fast: with the hardware rsqrt; Count: counting them in `terms`).
// Called by all 32 lanes together (the ballot); returns the lanes that open
// c as a cell to descend into.
template <bool Fast, bool Count>
__device__ __forceinline__ unsigned bh_eval(int c, bool in, bool cell, int s,
                                            float2 p, float k, float th2,
                                            float md2,
                                            const float4 *__restrict__ node,
                                            const float2 *__restrict__ spos,
                                            float &fx, float &fy, int &terms) {
  bool op = false;
  if (in) {
    if (!cell) {  // single point ~c
      if (~c != s) {
        bh_direct<Fast>(p.x, p.y, spos[~c], k, md2, fx, fy);
        if (Count) ++terms;
      }
    } else {
      const float4 r0 = node[2 * c], r1 = node[2 * c + 1];
      const float dx = __fsub_rn(__fsub_rn(p.x, r0.x), r0.z);
      const float dy = __fsub_rn(__fsub_rn(p.y, r0.y), r0.w);
      const float r2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
      const float r2c = fmaxf(r2, md2);
      // size^2 < 0 (a node standing for no quad level) is always opened
      if (r1.y >= 0.f && r1.y < __fmul_rn(th2, r2c)) {
        bh_term<Fast>(dx, dy, r2c, __fmul_rn(k, fabsf(r1.x)), fx, fy);
        if (Count) ++terms;
      } else if (r1.x > 0.f) {
        op = true;
      } else {  // bucket: point by point
        const int b = __float_as_int(r1.z), e = __float_as_int(r1.w);
        for (int t = b; t <= e; ++t)
          if (t != s) {
            bh_direct<Fast>(p.x, p.y, spos[t], k, md2, fx, fy);
            if (Count) ++terms;
          }
      }
    }
  }
  return __ballot_sync(0xffffffffu, op);
}

constexpr int kWalkGroup = 8;                    // lanes per group
constexpr int kWalkGroups = 32 / kWalkGroup;     // groups per warp

// The walk of the 32 points of one warp (sorted positions base .. base + 31),
// groups of kWalkGroup lanes each with their own stack in st_node / st_mask
// (this warp's [kWalkGroups][Stack + 1] arrays). Fast: FX_BH_FAST, the same
// cells and term order with the hardware rsqrt (a few ulp) instead of the
// reproducible one; Count: also each point's number of terms.
template <int Stack, bool Fast, bool Count>
__device__ __forceinline__ void bh_group_walk(
    int base, int n, const float2 *__restrict__ spos, const int32_t *__restrict__ perm,
    const int4 *__restrict__ qchild, const float4 *__restrict__ node, float k, float th2,
    float md2, float2 *__restrict__ force, unsigned int *__restrict__ err,
    int32_t *__restrict__ term_count, int32_t (*st_node)[Stack + 1],
    unsigned (*st_mask)[Stack + 1]) {
  const int lane = threadIdx.x & 31;
  const int g = lane / kWalkGroup;
  const bool leader = (lane % kWalkGroup) == 0;
  const unsigned gmask = (kWalkGroup == 32 ? 0xffffffffu
                                           : ((1u << kWalkGroup) - 1u) << (g * kWalkGroup));
  const int s = base + lane;
  const bool valid = s < n;
  const float2 p = valid ? spos[s] : make_float2(0.f, 0.f);
  float fx = 0.f, fy = 0.f;
  int sp = 0;  // this group's stack depth (uniform in the group)
  int terms = 0;
  auto eval = [&](int c, bool in, bool cell) -> unsigned {
    return bh_eval<Fast, Count>(c, in, cell, s, p, k, th2, md2, node, spos, fx, fy, terms);
  };
  if (n >= 2) {
    const unsigned open = eval(0, valid, true) & gmask;
    if (open) {
      if (leader) {
        st_node[g][0] = 0;
        st_mask[g][0] = open;
      }
      sp = 1;
    }
  }
  __syncwarp();
  while (__any_sync(0xffffffffu, sp > 0)) {
    const bool has = sp > 0;
    int nd = 0;
    unsigned mask = 0u;
    if (has) {
      --sp;
      nd = st_node[g][sp];
      mask = st_mask[g][sp];
    }
    __syncwarp();
    int4 q = make_int4(kNone, kNone, kNone, kNone);
    if (has) q = qchild[nd];
    const int qc[4] = {q.x, q.y, q.z, q.w};
    const bool in = (mask >> lane) & 1u;
    unsigned om[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int c = qc[h];
      om[h] = eval(c, in && c != kNone, c >= 0) & gmask;
    }
    const int np = (om[0] != 0u) + (om[1] != 0u) + (om[2] != 0u) + (om[3] != 0u);
    if (sp + np > Stack) {
      if (leader) atomicOr(err, 1u);
    } else {
      // push the opened children in reverse so the first one is popped first
#pragma unroll
      for (int h = 3; h >= 0; --h) {
        if (om[h] != 0u) {
          if (leader) {
            st_node[g][sp] = qc[h];
            st_mask[g][sp] = om[h];
          }
          ++sp;
        }
      }
    }
    __syncwarp();
  }
  if (valid) {
    force[perm[s]] = make_float2(fx, fy);
    if (Count) term_count[perm[s]] = terms;
  }
}

template <int Stack, bool Fast = false, bool Count = false>
__global__ void __launch_bounds__(kWalkWarps * 32, 8)
bh_walk_kernel(int n, const float2 *__restrict__ spos,
               const int32_t *__restrict__ perm,
               const int4 *__restrict__ qchild,
               const float4 *__restrict__ node, float k, float th2, float md2,
               float2 *__restrict__ force, unsigned int *__restrict__ err,
               int32_t *__restrict__ term_count = nullptr) {
  // one stack per group; the odd stride puts the groups' tops (often at the
  // same depth) in different banks
  __shared__ int32_t st_node[kWalkWarps][kWalkGroups][Stack + 1];
  __shared__ unsigned st_mask[kWalkWarps][kWalkGroups][Stack + 1];
  const int w = threadIdx.x >> 5;
  const int base = (blockIdx.x * kWalkWarps + w) * 32;
  if (base >= n) return;  // warp-uniform
  bh_group_walk<Stack, Fast, Count>(base, n, spos, perm, qchild, node, k, th2, md2, force,
                                    err, term_count, st_node[w], st_mask[w]);
}

// ---- batched walk (FX_BH_FAST) ----------------------------------------------
// The same cells, decisions and terms as the group walk, organised by cell
// instead of by point. Each warp owns 32 consecutive sorted points and a
// stack of (cell, lane mask) entries: the cells opened by at least one of
// its points, with the lanes that must evaluate them. A pass pops up to 32
// entries, one per lane; each lane loads its entry's walk record into shared
// memory, then every lane evaluates all popped entries for its own point
// (broadcast reads), adds the accepted terms and votes which lanes open each
// entry. Opened cells push their quad children with that vote as the mask;
// opened buckets are walked point by point. Every lane does the same work in
// every step (no divergence between cells, points and buckets), and a cell
// is loaded once per warp instead of once per group. Per point the
// interaction list is exactly the group walk's (the same opening rule with
// the same f32 operations); the terms are added in another order.
// The stack holds kBatchStack entries (the 1M-gate uniform placement peaks at
// 219; clustered, line and radial sets of 20k-200k points at 160-224 in a CPU
// model of this walk): a warp whose stack would overflow starts over with
// the group walk, whose stacks are bounded, in the same shared memory.
// The hardware reciprocal square root without the subnormal handling of
// rsqrtf (the argument here is at least min_dist^2).
__device__ __forceinline__ float rsqrt_approx_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr int kBatchWarps = 8;
constexpr int kBatchStack = 400;
static_assert(kBatchStack * sizeof(int2) >= 2 * kWalkGroups * (kStackDeep + 1) * sizeof(int32_t),
              "the group walk's stacks must fit in a warp's batch stack");

// The stack entries a warp may use (kBatchStack; less when the environment
// variable FLUXION_BH_BATCH_STACK asks for it, a test setting that sends more
// warps down the group-walk path).
static int batch_stack_cap() {
  static const int cap = [] {
    const char *e = std::getenv("FLUXION_BH_BATCH_STACK");
    const int v = e ? std::atoi(e) : kBatchStack;
    return std::min(kBatchStack, std::max(4, v));
  }();
  return cap;
}

template <int Stack, bool Count>
__global__ void __launch_bounds__(kBatchWarps * 32, 5)
bh_batch_walk_kernel(int n, const float2 *__restrict__ spos, const int32_t *__restrict__ perm,
                     const int4 *__restrict__ qchild, const float4 *__restrict__ node,
                     float k, float th2, float md2, float2 *__restrict__ force,
                     unsigned int *__restrict__ err, int32_t *__restrict__ term_count,
                     int stack_cap) {
  __shared__ int2 st[kBatchWarps][kBatchStack];
  __shared__ float4 rec_a[kBatchWarps][32];  // cx_hi, cy_hi, cx_lo, cy_lo
  __shared__ float4 rec_b[kBatchWarps][32];  // k*mass, size^2 rule, lane mask, self
  __shared__ unsigned open_s[kBatchWarps][32];  // per popped entry: the lanes opening it
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool lane0 = lane == 0;
  const int base = (blockIdx.x * kBatchWarps + w) * 32;
  if (base >= n) return;  // warp-uniform
  const int s = base + lane;
  const bool valid = s < n;
  const unsigned lanebit = 1u << lane;
  const float2 p = valid ? spos[s] : make_float2(0.f, 0.f);
  float fx = 0.f, fy = 0.f;
  int terms = 0;
  int sp = 0;  // stack depth (warp-uniform)
  if (n >= 2) {
    const unsigned vm = __ballot_sync(full, valid);
    if (lane == 0) st[w][0] = make_int2(0, (int)vm);
    sp = 1;
  }
  __syncwarp();
  bool overflow = false;
  while (sp > 0) {
    const int cnt = min(sp, 32);
    sp -= cnt;
    int c = kNone, bf = 0, bl = -1;
    bool bucket = false;
    if (lane < cnt) {
      const int2 e = st[w][sp + lane];
      c = e.x;
      float4 a, b;
      if (c >= 0) {
        a = node[2 * c];
        const float4 r1 = node[2 * c + 1];
        // size^2 < 0 (a node standing for no quad level): never accepted
        b = make_float4(__fmul_rn(k, fabsf(r1.x)), r1.y >= 0.f ? r1.y : __int_as_float(0x7f800000),
                        __int_as_float(e.y), __int_as_float(-1));
        bucket = !(r1.x > 0.f);
        bf = __float_as_int(r1.z);
        bl = __float_as_int(r1.w);
      } else {  // single point ~c: always accepted
        const float2 q = spos[~c];
        a = make_float4(q.x, q.y, 0.f, 0.f);
        b = make_float4(k, -1.f, __int_as_float(e.y), __int_as_float(~c));
      }
      rec_a[w][lane] = a;
      rec_b[w][lane] = b;
    }
    __syncwarp();
#pragma unroll 4
    for (int j = 0; j < cnt; ++j) {
      const float4 a = rec_a[w][j];
      const float4 b = rec_b[w][j];
      const float dx = __fsub_rn(__fsub_rn(p.x, a.x), a.z);
      const float dy = __fsub_rn(__fsub_rn(p.y, a.y), a.w);
      const float r2c = fmaxf(__fmaf_rn(dx, dx, __fmul_rn(dy, dy)), md2);
      const bool in = (__float_as_uint(b.z) & lanebit) != 0u;
      const bool acc = b.y < __fmul_rn(th2, r2c);
      const unsigned om = __ballot_sync(full, in && !acc);
      if (lane0) open_s[w][j] = om;
      const float inv = rsqrt_approx_ftz(r2c);  // r2c >= md2 > 0: never subnormal
      const float f = __fmul_rn(__fmul_rn(__fmul_rn(b.x, inv), inv), inv);
      const float fu = (in && acc) ? f : 0.f;
      fx = __fmaf_rn(fu, dx, fx);
      fy = __fmaf_rn(fu, dy, fy);
      if (Count) terms += (in && acc && __float_as_int(b.w) != s) ? 1 : 0;
    }
    __syncwarp();
    const unsigned myopen = lane < cnt ? open_s[w][lane] : 0u;
    // opened buckets: their points one by one
    unsigned bk = __ballot_sync(full, bucket && myopen != 0u);
    while (bk) {
      const int j = __ffs(bk) - 1;
      bk &= bk - 1u;
      const unsigned om = __shfl_sync(full, myopen, j);
      const int f = __shfl_sync(full, bf, j), l = __shfl_sync(full, bl, j);
      const bool in = (om & lanebit) != 0u;
      for (int t = f; t <= l; ++t) {
        const float2 q = spos[t];
        if (in && t != s) {
          bh_direct<true>(p.x, p.y, q, k, md2, fx, fy);
          if (Count) ++terms;
        }
      }
    }
    // opened cells: push their quad children with the opening lanes as mask
    const bool op = myopen != 0u && c >= 0 && !bucket;
    int4 q = make_int4(kNone, kNone, kNone, kNone);
    if (op) q = qchild[c];
    const int nc = (q.x != kNone) + (q.y != kNone) + (q.z != kNone) + (q.w != kNone);
    int incl = nc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(full, incl, 31);
    if (sp + total > stack_cap) {  // stack_cap <= kBatchStack
      overflow = true;
      break;
    }
    int pos = sp + incl - nc;
    const int qc[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int h = 0; h < 4; ++h)
      if (qc[h] != kNone) st[w][pos++] = make_int2(qc[h], (int)myopen);
    sp += total;
    __syncwarp();
  }
  if (overflow) {  // warp-uniform: start over with the bounded group walk
    __syncwarp();
    int32_t *mem = reinterpret_cast<int32_t *>(&st[w][0]);
    bh_group_walk<Stack, true, Count>(
        base, n, spos, perm, qchild, node, k, th2, md2, force, err, term_count,
        reinterpret_cast<int32_t(*)[Stack + 1]>(mem),
        reinterpret_cast<unsigned(*)[Stack + 1]>(mem + kWalkGroups * (Stack + 1)));
    return;
  }
  if (valid) {
    force[perm[s]] = make_float2(fx, fy);
    if (Count) term_count[perm[s]] = terms;
  }
}

static int bh_alloc(fx_design *d) {
  BHWork &b = d->bh;
  const int n = d->n;
  if (b.n == n && b.node.p) return FX_OK;
  const int T = (n + kSortTile - 1) / kSortTile;
  const size_t ni = n > 1 ? (size_t)n - 1 : 1;
  for (int i = 0; i < 2; ++i) {
    FX_TRY(b.keys[i].alloc(n));
    FX_TRY(b.idx[i].alloc(n));
  }
  FX_TRY(b.tile_hist.alloc((size_t)256 * T));
  FX_TRY(b.tile_scan.alloc((size_t)256 * T));
  FX_TRY(b.digit_total.alloc(256));
  FX_TRY(b.spos.alloc(n));
  FX_TRY(b.child.alloc(2 * ni));
  FX_TRY(b.range.alloc(2 * ni));
  FX_TRY(b.dnode.alloc(ni));
  FX_TRY(b.dparent.alloc(ni));
  FX_TRY(b.qchild.alloc(ni));
  FX_TRY(b.tile_fix.alloc((size_t)(n + kFixTile - 1) / kFixTile));
  FX_TRY(b.prefix.alloc(n));
  FX_TRY(b.node.alloc(2 * ni));
  FX_TRY(b.root.alloc(4));
  FX_TRY(b.bbox.alloc(8));
  FX_TRY(b.force.alloc(n));
  FX_TRY(b.os_ws.alloc(os_sort_words(n, 4)));
  b.n = n;
  return FX_OK;
}

static int bh_alloc_deep(fx_design *d) {
  BHWork &b = d->bh;
  const size_t n = (size_t)d->n;
  if (b.klo.p && b.klo.n >= n) return FX_OK;
  FX_TRY(b.klo.alloc(n));
  FX_TRY(b.kl[0].alloc(n));
  FX_TRY(b.kl[1].alloc(n));
  FX_TRY(b.il[0].alloc(n));
  FX_TRY(b.il[1].alloc(n));
  FX_TRY(b.slo.alloc(n));
  return FX_OK;
}

// Whether the deep-key kernels can be needed: unless the positions are known
// to lie in the die and a level-15 cell of the largest possible root square,
// (die + 2) / 2^15, is accepted by every point (margins cover f32 rounding).
static bool bh_maybe_deep(const fx_design *d, float th2, float md2) {
  if (!d->pos_in_box) return true;
  const double rb = ((double)std::max(d->chip_w, d->chip_h) + 2.0) * (1.0 + 1e-6);
  const double s15 = rb / 32768.0;
  return s15 * s15 >= (double)th2 * (double)md2 * (1.0 - 1e-6);
}

// The walk's and the sort's error word (bh.bbox[4]) as a status.
int bh_error(unsigned int err) {
  if (err & 4u) {
    set_error("Barnes-Hut key sort: a bounded look-back wait expired");
    return FX_ETIMEOUT;
  }
  if (err) {
    set_error("Barnes-Hut walk stack overflow");
    return FX_EINVAL;
  }
  return FX_OK;
}

// Bounding box of the given positions into bh.bbox (re-armed first).
int bh_bbox(fx_ctx *ctx, fx_design *d, const float *x, const float *y,
            cudaStream_t s) {
  FX_TRY(bh_alloc(d));
  // {0xffffffff, 0xffffffff, 0, 0, 0}: min/max seeds of the ordered box and
  // a clear error word (memsets: no host buffer to stage)
  FX_CHECK_CUDA(cudaMemsetAsync(d->bh.bbox.p, 0xff, 8, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d->bh.bbox.p + 2, 0, 12, s));
  int nb = (d->n + 255) / 256;
  if (nb > ctx->num_sms * 8) nb = ctx->num_sms * 8;
  bh_bbox_kernel<<<nb, 256, 0, s>>>(x, y, d->n, d->bh.bbox.p);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

// Full Barnes-Hut force evaluation on the current positions; bh.bbox must
// hold their bounding box. Result: bh.force (original gate order).
int bh_run(fx_ctx *ctx, fx_design *d, float k, float theta, float min_dist, int walk,
           cudaStream_t s, int32_t *term_count) {
  FX_TRY(bh_alloc(d));
  BHWork &b = d->bh;
  const int n = d->n;
  const float *x = d->x[d->cur].p, *y = d->y[d->cur].p;
  const int T = (n + kSortTile - 1) / kSortTile;
  unsigned int *err = b.bbox.p + 4;
  const float th2 = theta * theta, md2 = min_dist * min_dist;
  const bool deep = bh_maybe_deep(d, th2, md2);  // launch the deep-key kernels
  if (deep) FX_TRY(bh_alloc_deep(d));
  cudaEvent_t ev;
  const int gb = (n + 255) / 256;
  int launches = 0;
  timer_begin(ctx, FX_STAGE_BH_KEYS, s, &ev);
  bh_root_kernel<<<1, 1, 0, s>>>(b.bbox.p, b.root.p, th2, md2);
  FX_CHECK_LAUNCH();
  bh_keys_kernel<<<gb, 256, 0, s>>>(x, y, n, b.root.p, b.keys[0].p, b.idx[0].p,
                                    deep ? b.klo.p : nullptr, deep ? b.kl[0].p : nullptr,
                                    deep ? b.il[0].p : nullptr);
  FX_CHECK_LAUNCH();
  launches += 2;
  timer_end(ctx, FX_STAGE_BH_KEYS, s, ev);
  timer_begin(ctx, FX_STAGE_BH_SORT, s, &ev);
  const float *gate = b.root.p;
  if (deep) {
    // stable sort by the 24-bit sub-key (3 passes; no-ops unless root[3]),
    // then the primary keys and indices in that order into buffer 0
    for (int pass = 0; pass < 3; ++pass) {
      const int src = pass & 1, dst = src ^ 1;
      radix_hist_kernel<<<T, kSortThreads, 0, s>>>(b.kl[src].p, n, 8 * pass, b.tile_hist.p, T,
                                                   gate);
      radix_scan_kernel<<<256, 256, 0, s>>>(b.tile_hist.p, b.tile_scan.p, b.digit_total.p, T,
                                            gate);
      radix_scatter_kernel<<<T, kSortThreads, 0, s>>>(
          b.kl[src].p, b.il[src].p, b.kl[dst].p, b.il[dst].p, n, 8 * pass, b.tile_scan.p,
          b.digit_total.p, T, gate);
    }
    bh_deep_gather_kernel<<<gb, 256, 0, s>>>(gate, n, b.keys[0].p, b.il[1].p, b.keys[1].p,
                                             b.idx[1].p);
    bh_deep_copy_kernel<<<gb, 256, 0, s>>>(gate, n, b.keys[1].p, b.idx[1].p, b.keys[0].p,
                                           b.idx[0].p);
    FX_CHECK_LAUNCH();
    launches += 9 + 2;
  }
  {
    uint32_t *kk[2] = {b.keys[0].p, b.keys[1].p};
    int32_t *vv[2] = {b.idx[0].p, b.idx[1].p};
    // result in buffer 0; the last pass also gathers the sorted positions
    FX_TRY(radix_sort_onesweep(kk, vv, n, 4, b.os_ws.p, err, s, x, y, b.spos.p));
  }
  launches += 5;
  if (deep) {
    bh_deep_slo_kernel<<<gb, 256, 0, s>>>(gate, n, b.klo.p, b.idx[0].p, b.slo.p);
    ++launches;
  }
  FX_CHECK_LAUNCH();
  timer_end(ctx, FX_STAGE_BH_SORT, s, ev);
  timer_begin(ctx, FX_STAGE_BH_TREE, s, &ev);
  if (n >= 2) {
    const int tb = (n - 1 + 255) / 256;
    bh_tree_kernel<<<tb, 256, 0, s>>>(b.keys[0].p, deep ? b.slo.p : nullptr, b.root.p, n,
                                      b.child.p, b.range.p, b.dnode.p, b.dparent.p);
    // exact prefix sums: tile sums, tile offsets, point prefixes
    const int tiles = (n + kFixTile - 1) / kFixTile;
    fix_tile_kernel<<<tiles, kFixThreads, 0, s>>>(b.spos.p, n, b.tile_fix.p);
    fix_top_kernel<<<1, kFixThreads, 0, s>>>(b.tile_fix.p, tiles);
    fix_prefix_kernel<<<tiles, kFixThreads, 0, s>>>(b.spos.p, n, b.tile_fix.p, b.prefix.p);
    bh_node_kernel<<<tb, 256, 0, s>>>(n, b.range.p, b.dnode.p, b.dparent.p,
                                      b.prefix.p, b.root.p, deep ? 1 : 0, b.node.p, b.child.p,
                                      b.qchild.p);
    launches += 5;
  }
  FX_CHECK_LAUNCH();
  timer_end(ctx, FX_STAGE_BH_TREE, s, ev);
  timer_begin(ctx, FX_STAGE_BH_WALK, s, &ev);
  if (walk == FX_BH_EXACT) {
    const int wb = (n + kWalkWarps * 32 - 1) / (kWalkWarps * 32);
    if (deep)
      bh_walk_kernel<kStackDeep><<<wb, kWalkWarps * 32, 0, s>>>(
          n, b.spos.p, b.idx[0].p, b.qchild.p, b.node.p, k, th2, md2, b.force.p, err);
    else
      bh_walk_kernel<kStack><<<wb, kWalkWarps * 32, 0, s>>>(
          n, b.spos.p, b.idx[0].p, b.qchild.p, b.node.p, k, th2, md2, b.force.p, err);
  } else {
    const int wb = (n + kBatchWarps * 32 - 1) / (kBatchWarps * 32);
#define FX_FAST_WALK(ST, CNT)                                                             \
  bh_batch_walk_kernel<ST, CNT><<<wb, kBatchWarps * 32, 0, s>>>(                          \
      n, b.spos.p, b.idx[0].p, b.qchild.p, b.node.p, k, th2, md2, b.force.p, err, term_count, \
      batch_stack_cap())
    if (deep) {
      if (term_count) FX_FAST_WALK(kStackDeep, true);
      else FX_FAST_WALK(kStackDeep, false);
    } else {
      if (term_count) FX_FAST_WALK(kStack, true);
      else FX_FAST_WALK(kStack, false);
    }
#undef FX_FAST_WALK
  }
  FX_CHECK_LAUNCH();
  ++launches;
  timer_end(ctx, FX_STAGE_BH_WALK, s, ev);
  ctx->launches += launches;
  return FX_OK;
}

}  // namespace fx

using namespace fx;

extern "C" int fx_stage_barnes_hut_walk(fx_ctx *ctx, fx_design *d, float k, float theta,
                                        float min_dist, int32_t walk, float *out_fx,
                                        float *out_fy, uint32_t *out_keys, int32_t *out_perm,
                                        float *out_root, int32_t *out_terms) {
  if (!ctx || !d || !(theta >= 0.f) || !(min_dist > 0.f) ||
      (walk != FX_BH_FAST && walk != FX_BH_EXACT) || (out_terms && walk != FX_BH_FAST)) {
    set_error("fx_stage_barnes_hut: invalid arguments");
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream;
  const size_t n = (size_t)d->n;
  DevBuf<int32_t> terms;
  if (out_terms) FX_TRY(terms.alloc(n));
  FX_TRY(bh_bbox(ctx, d, d->x[d->cur].p, d->y[d->cur].p, s));
  FX_TRY(bh_run(ctx, d, k, theta, min_dist, walk, s, out_terms ? terms.p : nullptr));
  if (out_terms)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_terms, terms.p, n * 4, cudaMemcpyDeviceToHost, s));
  std::vector<float2> f(n);
  std::vector<uint32_t> skeys(n);
  std::vector<int32_t> perm(n);
  unsigned int err = 0;
  FX_CHECK_CUDA(cudaMemcpyAsync(f.data(), d->bh.force.p, n * 8, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(skeys.data(), d->bh.keys[0].p, n * 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(perm.data(), d->bh.idx[0].p, n * 4, cudaMemcpyDeviceToHost, s));
  if (out_root)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_root, d->bh.root.p, 12, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(&err, d->bh.bbox.p + 4, 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  FX_TRY(bh_error(err));
  for (size_t i = 0; i < n; ++i) {
    if (out_fx) out_fx[i] = f[i].x;
    if (out_fy) out_fy[i] = f[i].y;
  }
  // keys in gate order; perm maps sorted position -> gate
  if (out_keys)
    for (size_t i = 0; i < n; ++i) out_keys[perm[i]] = skeys[i];
  if (out_perm) std::copy(perm.begin(), perm.end(), out_perm);
  return FX_OK;
}

extern "C" int fx_stage_barnes_hut(fx_ctx *ctx, fx_design *d, float k, float theta,
                                   float min_dist, float *out_fx, float *out_fy,
                                   uint32_t *out_keys, int32_t *out_perm, float *out_root) {
  return fx_stage_barnes_hut_walk(ctx, d, k, theta, min_dist, FX_BH_EXACT, out_fx, out_fy,
                                  out_keys, out_perm, out_root, nullptr);
}
