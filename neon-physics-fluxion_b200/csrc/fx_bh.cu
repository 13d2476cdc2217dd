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
#include "fx_internal.h"
#include "fx_device.cuh"

namespace fx {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys
constexpr int kScanBlock = 1024;                        // prefix-sum block
constexpr int kWalkWarps = 8;
constexpr int kStack = 64;

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
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(bbox + 0, f2ord(mnx));
    atomicMin(bbox + 1, f2ord(mny));
    atomicMax(bbox + 2, f2ord(mxx));
    atomicMax(bbox + 3, f2ord(mxy));
  }
}

// Root square from the box (BarnesHutTree.cpp:24-46, in f32 without
// contraction), then re-arms the box for the next accumulation.
__global__ void bh_root_kernel(unsigned int *__restrict__ bbox,
                               float *__restrict__ root) {
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

__global__ void bh_keys_kernel(const float *__restrict__ x,
                               const float *__restrict__ y, int n,
                               const float *__restrict__ root,
                               uint32_t *__restrict__ keys,
                               int32_t *__restrict__ idx) {
  const float ox = root[0], oy = root[1], size = root[2];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const uint32_t qx = quantize15(x[i], ox, size);
    const uint32_t qy = quantize15(y[i], oy, size);
    keys[i] = (spread15(qx) << 1) | spread15(qy);
    idx[i] = i;
  }
}

// ---- stable LSD radix sort (8-bit digits) ------------------------------------
__global__ void __launch_bounds__(kSortThreads)
radix_hist_kernel(const uint32_t *__restrict__ keys, int n, int shift,
                  uint32_t *__restrict__ tile_hist, int T) {
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

// Exclusive scan of the digit-major tile histogram (single block).
__global__ void __launch_bounds__(1024)
radix_scan_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                  int count) {
  __shared__ uint32_t ws[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int per = (count + 1023) / 1024;
  const int b = t * per, e = min(count, b + per);
  uint32_t s = 0;
  for (int i = b; i < e; ++i) s += in[i];
  uint32_t v = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    uint32_t u = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t q = __shfl_up_sync(0xffffffffu, u, o);
      if (lane >= o) u += q;
    }
    ws[lane] = u;
  }
  __syncthreads();
  uint32_t run = v - s + (w > 0 ? ws[w - 1] : 0u);
  for (int i = b; i < e; ++i) {
    const uint32_t c = in[i];
    out[i] = run;
    run += c;
  }
}

// Stable scatter: within a tile, warp w ranks its 256 keys in order
// (__match_any_sync groups lanes with equal digits), then warps are ordered
// by a per-digit prefix over the warp counts.
__global__ void __launch_bounds__(kSortThreads)
radix_scatter_kernel(const uint32_t *__restrict__ kin,
                     const int32_t *__restrict__ iin,
                     uint32_t *__restrict__ kout, int32_t *__restrict__ iout,
                     int n, int shift, const uint32_t *__restrict__ tile_scan,
                     int T) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t cnt[kWarps][256];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  for (int i = t; i < kWarps * 256; i += kSortThreads) (&cnt[0][0])[i] = 0;
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
  if (t < 256) {
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < kWarps; ++ww) {
      const uint32_t c = cnt[ww][t];
      cnt[ww][t] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int i = base + r * 32 + lane;
    if (i < n) {
      const uint32_t dg = (k[r] >> shift) & 255u;
      const uint32_t pos =
          tile_scan[(size_t)dg * T + blockIdx.x] + cnt[w][dg] + rank[r];
      kout[pos] = k[r];
      iout[pos] = v[r];
    }
  }
}

// ---- sorted positions and FP64 prefix sums -------------------------------------
__global__ void __launch_bounds__(256)
bh_gather_kernel(const float *__restrict__ x, const float *__restrict__ y,
                 const int32_t *__restrict__ perm, int n,
                 float2 *__restrict__ spos, double2 *__restrict__ bsum) {
  const int base = blockIdx.x * kScanBlock;
  double sx = 0.0, sy = 0.0;
  for (int i = base + threadIdx.x; i < min(n, base + kScanBlock); i += 256) {
    const int g = perm[i];
    const float2 p = make_float2(x[g], y[g]);
    spos[i] = p;
    sx += (double)p.x;
    sy += (double)p.y;
  }
  sx = block_sum_double(sx);
  sy = block_sum_double(sy);
  if (threadIdx.x == 0) bsum[blockIdx.x] = make_double2(sx, sy);
}

// Exclusive scan of the block sums (single block, sequential per thread).
__global__ void __launch_bounds__(1024)
bh_bsum_scan_kernel(double2 *__restrict__ bsum, int nb) {
  __shared__ double2 part[1024];
  const int t = threadIdx.x;
  const int per = (nb + 1023) / 1024;
  const int b = t * per, e = min(nb, b + per);
  double sx = 0.0, sy = 0.0;
  for (int i = b; i < e; ++i) {
    sx += bsum[i].x;
    sy += bsum[i].y;
  }
  part[t] = make_double2(sx, sy);
  __syncthreads();
  if (t == 0) {
    double ax = 0.0, ay = 0.0;
    for (int i = 0; i < 1024; ++i) {
      const double2 q = part[i];
      part[i] = make_double2(ax, ay);
      ax += q.x;
      ay += q.y;
    }
  }
  __syncthreads();
  double ax = part[t].x, ay = part[t].y;
  for (int i = b; i < e; ++i) {
    const double2 q = bsum[i];
    bsum[i] = make_double2(ax, ay);
    ax += q.x;
    ay += q.y;
  }
}

// Inclusive prefix of the sorted positions within each block plus the block
// offset. Sequential per thread over 4 consecutive items, then a warp/block
// scan of the thread totals.
__global__ void __launch_bounds__(256)
bh_prefix_kernel(const float2 *__restrict__ spos, int n,
                 const double2 *__restrict__ bsum,
                 double2 *__restrict__ prefix) {
  __shared__ double2 ws[8];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int base = blockIdx.x * kScanBlock + t * 4;
  double px[4], py[4];
  double sx = 0.0, sy = 0.0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int i = base + j;
    const float2 p = i < n ? spos[i] : make_float2(0.f, 0.f);
    sx += (double)p.x;
    sy += (double)p.y;
    px[j] = sx;
    py[j] = sy;
  }
  double vx = sx, vy = sy;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double ux = __shfl_up_sync(0xffffffffu, vx, o);
    const double uy = __shfl_up_sync(0xffffffffu, vy, o);
    if (lane >= o) {
      vx += ux;
      vy += uy;
    }
  }
  if (lane == 31) ws[w] = make_double2(vx, vy);
  __syncthreads();
  double ox = bsum[blockIdx.x].x, oy = bsum[blockIdx.x].y;
  for (int q = 0; q < w; ++q) {
    ox += ws[q].x;
    oy += ws[q].y;
  }
  ox += vx - sx;
  oy += vy - sy;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int i = base + j;
    if (i < n) prefix[i] = make_double2(ox + px[j], oy + py[j]);
  }
}

// ---- radix tree (Karras 2012) -----------------------------------------------
__device__ __forceinline__ int bh_delta(const uint32_t *__restrict__ keys,
                                        int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t a = keys[i], b = keys[j];
  if (a != b) return __clz(a ^ b) - 2;
  return 30 + __clz((uint32_t)(i ^ j));
}

__global__ void bh_tree_kernel(const uint32_t *__restrict__ keys, int n,
                               int32_t *__restrict__ child,
                               int32_t *__restrict__ range,
                               int32_t *__restrict__ delta_node,
                               int32_t *__restrict__ delta_parent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int dr = bh_delta(keys, n, i, i + 1), dl = bh_delta(keys, n, i, i - 1);
  const int d = (dr - dl) >= 0 ? 1 : -1;
  const int dmin = bh_delta(keys, n, i, i - d);
  int lmax = 2;
  while (bh_delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (bh_delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dn = bh_delta(keys, n, i, j);
  int s = 0;
  for (int div = 2;; div *= 2) {
    const int t = (l + div - 1) / div;
    if (bh_delta(keys, n, i, i + (s + t) * d) > dn) s += t;
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
  delta_node[i] = dn;
  if (left >= 0) delta_parent[left] = dn;
  if (right >= 0) delta_parent[right] = dn;
  if (i == 0) delta_parent[0] = -1;
}

// Centre of mass (FP64 prefix difference, stored as an f32 hi/lo pair) and
// the node's opening size: meta = {count, size^2}; size^2 < 0 marks a node
// that stands for no quad level (always opened); count < 0 marks a bucket.
__global__ void bh_finalize_kernel(int n, const int32_t *__restrict__ range,
                                   const int32_t *__restrict__ delta_node,
                                   const int32_t *__restrict__ delta_parent,
                                   const double2 *__restrict__ prefix,
                                   const float *__restrict__ root,
                                   float4 *__restrict__ com,
                                   float2 *__restrict__ meta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int first = range[2 * i], last = range[2 * i + 1];
  const int cnt = last - first + 1;
  double2 hi2 = prefix[last];
  if (first > 0) {
    const double2 lo2 = prefix[first - 1];
    hi2.x -= lo2.x;
    hi2.y -= lo2.y;
  }
  const double cx = hi2.x / (double)cnt, cy = hi2.y / (double)cnt;
  const float hx = (float)cx, hy = (float)cy;
  com[i] = make_float4(hx, hy, (float)(cx - (double)hx), (float)(cy - (double)hy));
  const int dn = delta_node[i], dp = delta_parent[i];
  const float rs = root[2];
  float2 m;
  if (dn >= 30) {
    const float s = ldexpf(rs, -15);
    m = make_float2(-(float)cnt, __fmul_rn(s, s));
  } else {
    const int lmax = dn >> 1;
    if (dp >= 0 && (dp >> 1) == lmax) {
      m = make_float2((float)cnt, -1.0f);
    } else {
      const float s = ldexpf(rs, -lmax);
      m = make_float2((float)cnt, __fmul_rn(s, s));
    }
  }
  meta[i] = m;
}

// ---- warp-cooperative walk ----------------------------------------------------
// Each warp owns 32 consecutive sorted points (spatially close). It walks the
// tree once with a shared stack of (node, lane mask): every lane applies the
// reference opening rule to its own point, lanes that accept a node take its
// centre-of-mass term, and the children are pushed only for the lanes that
// opened it. Interaction lists are therefore exactly per point.
__device__ __forceinline__ void bh_direct(float px, float py, float2 q,
                                          float kq, float md2, float &fx,
                                          float &fy) {
  const float dx = __fsub_rn(px, q.x), dy = __fsub_rn(py, q.y);
  const float r2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  const float inv = rsqrtf(fmaxf(r2, md2));
  const float f = kq * inv * inv * inv;
  fx += f * dx;
  fy += f * dy;
}

__global__ void __launch_bounds__(kWalkWarps * 32)
bh_walk_kernel(int n, const float2 *__restrict__ spos,
               const int32_t *__restrict__ perm,
               const int32_t *__restrict__ child,
               const int32_t *__restrict__ range,
               const float4 *__restrict__ com, const float2 *__restrict__ meta,
               float k, float th2, float md2, float2 *__restrict__ force,
               unsigned int *__restrict__ err) {
  __shared__ int32_t st_node[kWalkWarps][kStack];
  __shared__ unsigned st_mask[kWalkWarps][kStack];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int s = (blockIdx.x * kWalkWarps + w) * 32 + lane;
  const bool valid = s < n;
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  if (active == 0) return;
  const float2 p = valid ? spos[s] : make_float2(0.f, 0.f);
  float fx = 0.f, fy = 0.f;
  int sp = 0;
  if (n >= 2) {
    if (lane == 0) {
      st_node[w][0] = 0;
      st_mask[w][0] = active;
    }
    sp = 1;
  }
  __syncwarp();
  while (sp > 0) {
    --sp;
    const int node = st_node[w][sp];
    const unsigned mask = st_mask[w][sp];
    __syncwarp();
    const bool in = (mask >> lane) & 1u;
    if (node < 0) {  // single point
      const int t = ~node;
      if (in && t != s) bh_direct(p.x, p.y, spos[t], k, md2, fx, fy);
      continue;
    }
    const float2 m = meta[node];
    unsigned open;
    if (m.y < 0.f) {
      open = mask;
    } else {
      const float4 c = com[node];
      const float dx = __fsub_rn(__fsub_rn(p.x, c.x), c.z);
      const float dy = __fsub_rn(__fsub_rn(p.y, c.y), c.w);
      const float r2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
      const float r2c = fmaxf(r2, md2);
      const bool accept = in && (m.y < __fmul_rn(th2, r2c));
      if (accept) {
        const float inv = rsqrtf(r2c);
        const float f = k * fabsf(m.x) * inv * inv * inv;
        fx += f * dx;
        fy += f * dy;
      }
      open = __ballot_sync(0xffffffffu, in && !accept);
      if (open == 0) continue;
      if (m.x < 0.f) {  // bucket: direct terms for the lanes that opened it
        const bool mine = (open >> lane) & 1u;
        const int b = range[2 * node], e = range[2 * node + 1];
        for (int t = b; t <= e; ++t) {
          const float2 q = spos[t];
          if (mine && t != s) bh_direct(p.x, p.y, q, k, md2, fx, fy);
        }
        continue;
      }
    }
    if (sp + 2 > kStack) {
      if (lane == 0) atomicOr(err, 1u);
      continue;
    }
    if (lane == 0) {
      st_node[w][sp] = child[2 * node + 1];
      st_mask[w][sp] = open;
      st_node[w][sp + 1] = child[2 * node];
      st_mask[w][sp + 1] = open;
    }
    sp += 2;
    __syncwarp();
  }
  if (valid) force[perm[s]] = make_float2(fx, fy);
}

static int bh_alloc(fx_design *d) {
  BHWork &b = d->bh;
  const int n = d->n;
  if (b.n == n && b.com.p) return FX_OK;
  const int T = (n + kSortTile - 1) / kSortTile;
  const int NB = (n + kScanBlock - 1) / kScanBlock;
  const size_t ni = n > 1 ? (size_t)n - 1 : 1;
  for (int i = 0; i < 2; ++i) {
    FX_TRY(b.keys[i].alloc(n));
    FX_TRY(b.idx[i].alloc(n));
  }
  FX_TRY(b.tile_hist.alloc((size_t)256 * T));
  FX_TRY(b.tile_scan.alloc((size_t)256 * T + (size_t)2 * NB * 2));
  FX_TRY(b.spos.alloc(n));
  FX_TRY(b.prefix.alloc(n));
  FX_TRY(b.child.alloc(2 * ni + 2 * ni + 2 * ni + 4));  // child, delta_node, delta_parent
  FX_TRY(b.range.alloc(2 * ni));
  FX_TRY(b.com.alloc(ni));
  FX_TRY(b.meta.alloc(ni));
  FX_TRY(b.root.alloc(4));
  FX_TRY(b.bbox.alloc(8));
  FX_TRY(b.force.alloc(n));
  b.n = n;
  return FX_OK;
}

// Bounding box of the given positions into bh.bbox (re-armed first).
int bh_bbox(fx_ctx *ctx, fx_design *d, const float *x, const float *y,
            cudaStream_t s) {
  FX_TRY(bh_alloc(d));
  const unsigned int init[4] = {0xffffffffu, 0xffffffffu, 0u, 0u};
  FX_CHECK_CUDA(cudaMemcpyAsync(d->bh.bbox.p, init, 16, cudaMemcpyHostToDevice, s));
  int nb = (d->n + 255) / 256;
  if (nb > ctx->num_sms * 8) nb = ctx->num_sms * 8;
  bh_bbox_kernel<<<nb, 256, 0, s>>>(x, y, d->n, d->bh.bbox.p);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

// Full Barnes-Hut force evaluation on the current positions; bh.bbox must
// hold their bounding box. Result: bh.force (original gate order).
int bh_run(fx_ctx *ctx, fx_design *d, float k, float theta, float min_dist,
           cudaStream_t s) {
  FX_TRY(bh_alloc(d));
  BHWork &b = d->bh;
  const int n = d->n;
  const float *x = d->x[d->cur].p, *y = d->y[d->cur].p;
  const int T = (n + kSortTile - 1) / kSortTile;
  const int NB = (n + kScanBlock - 1) / kScanBlock;
  int32_t *delta_node = b.child.p + 2 * (size_t)(n > 1 ? n - 1 : 1);
  int32_t *delta_parent = delta_node + (n > 1 ? n - 1 : 1);
  unsigned int *err = b.bbox.p + 4;
  cudaEvent_t ev;
  const int gb = (n + 255) / 256;
  timer_begin(ctx, FX_STAGE_BH_KEYS, s, &ev);
  bh_root_kernel<<<1, 1, 0, s>>>(b.bbox.p, b.root.p);
  FX_CHECK_LAUNCH();
  bh_keys_kernel<<<gb, 256, 0, s>>>(x, y, n, b.root.p, b.keys[0].p, b.idx[0].p);
  FX_CHECK_LAUNCH();
  timer_end(ctx, FX_STAGE_BH_KEYS, s, ev);
  timer_begin(ctx, FX_STAGE_BH_SORT, s, &ev);
  for (int pass = 0; pass < 4; ++pass) {
    const int src = pass & 1, dst = src ^ 1;
    radix_hist_kernel<<<T, kSortThreads, 0, s>>>(b.keys[src].p, n, 8 * pass,
                                                 b.tile_hist.p, T);
    radix_scan_kernel<<<1, 1024, 0, s>>>(b.tile_hist.p, b.tile_scan.p, 256 * T);
    radix_scatter_kernel<<<T, kSortThreads, 0, s>>>(
        b.keys[src].p, b.idx[src].p, b.keys[dst].p, b.idx[dst].p, n, 8 * pass,
        b.tile_scan.p, T);
  }
  FX_CHECK_LAUNCH();
  timer_end(ctx, FX_STAGE_BH_SORT, s, ev);
  timer_begin(ctx, FX_STAGE_BH_TREE, s, &ev);
  double2 *bsum = (double2 *)(b.tile_scan.p + (size_t)256 * T);
  bh_gather_kernel<<<NB, 256, 0, s>>>(x, y, b.idx[0].p, n, b.spos.p, bsum);
  bh_bsum_scan_kernel<<<1, 1024, 0, s>>>(bsum, NB);
  bh_prefix_kernel<<<NB, 256, 0, s>>>(b.spos.p, n, bsum, b.prefix.p);
  if (n >= 2) {
    const int tb = (n - 1 + 255) / 256;
    bh_tree_kernel<<<tb, 256, 0, s>>>(b.keys[0].p, n, b.child.p, b.range.p,
                                      delta_node, delta_parent);
    bh_finalize_kernel<<<tb, 256, 0, s>>>(n, b.range.p, delta_node,
                                          delta_parent, b.prefix.p, b.root.p,
                                          b.com.p, b.meta.p);
  }
  FX_CHECK_LAUNCH();
  timer_end(ctx, FX_STAGE_BH_TREE, s, ev);
  timer_begin(ctx, FX_STAGE_BH_WALK, s, &ev);
  const int wb = (n + kWalkWarps * 32 - 1) / (kWalkWarps * 32);
  bh_walk_kernel<<<wb, kWalkWarps * 32, 0, s>>>(
      n, b.spos.p, b.idx[0].p, b.child.p, b.range.p, b.com.p, b.meta.p, k,
      theta * theta, min_dist * min_dist, b.force.p, err);
  FX_CHECK_LAUNCH();
  timer_end(ctx, FX_STAGE_BH_WALK, s, ev);
  ctx->launches += 2 + 12 + 3 + (n >= 2 ? 2 : 0) + 1;
  return FX_OK;
}

}  // namespace fx

using namespace fx;

extern "C" int fx_stage_barnes_hut(fx_ctx *ctx, fx_design *d, float k,
                                   float theta, float min_dist, float *out_fx,
                                   float *out_fy, uint32_t *out_keys,
                                   int32_t *out_perm, float *out_root) {
  if (!ctx || !d || !(theta >= 0.f) || !(min_dist > 0.f)) {
    set_error("fx_stage_barnes_hut: invalid arguments");
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  FX_TRY(bh_bbox(ctx, d, d->x[d->cur].p, d->y[d->cur].p, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d->bh.bbox.p + 4, 0, 4, s));
  FX_TRY(bh_run(ctx, d, k, theta, min_dist, s));
  const size_t n = (size_t)d->n;
  std::vector<float2> f(n);
  unsigned int err = 0;
  FX_CHECK_CUDA(cudaMemcpyAsync(f.data(), d->bh.force.p, n * 8, cudaMemcpyDeviceToHost, s));
  if (out_keys)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_keys, d->bh.keys[0].p, n * 4, cudaMemcpyDeviceToHost, s));
  if (out_perm)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_perm, d->bh.idx[0].p, n * 4, cudaMemcpyDeviceToHost, s));
  if (out_root)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_root, d->bh.root.p, 12, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(&err, d->bh.bbox.p + 4, 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (err) {
    set_error("Barnes-Hut walk stack overflow");
    return FX_EINVAL;
  }
  for (size_t i = 0; i < n; ++i) {
    if (out_fx) out_fx[i] = f[i].x;
    if (out_fy) out_fy[i] = f[i].y;
  }
  return FX_OK;
}
