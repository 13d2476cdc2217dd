// fx_attention.cu -- (f.4) attention scores between the clusters of one
// hierarchy level (compute_level_attention, H/src/algorithm/attention.rs:
// 50-88):
//   score(A -> B) = |nets touching A and B| / |nets touching A|,  A != B
// and, per cluster, the top_k clusters by score (descending, ties by index,
// as the stable sort_by of :81-82; zero scores dropped).
//
// The reference forms the dense n x n matrix from per-cluster net sets
// (nets_touching_gates, :90-99). Here every net finds its distinct clusters
// (a warp per net with __match_any_sync up to 32 pins; a block per larger net
// over a shared-memory bitmap of the level's clusters), emits each ordered
// pair of them once, and a radix sort + run-length count of the pair keys
// gives the shared-net counts of the pairs that have any: the work follows
// the pins and the pairs, not n^2, and a high-fanout net costs no more than
// its pairs. Scans are three-phase tile scans of 1024 elements. All counts
// are integers, so the f32 scores are those of the reference formula (shared
// as f32 / total as f32, rounded to nearest).
#include <algorithm>
#include <vector>

#include "fx_internal.h"

namespace fx {
namespace {

// gate -> cluster for the level's CSR (one thread per listed gate); cl starts
// at -1. bad[0] |= 1 for a gate out of range, 2 for a gate in two clusters.
__global__ void attn_map_kernel(int n, int G, int n_gates, const int32_t *__restrict__ cptr,
                                const int32_t *__restrict__ cgate, int32_t *__restrict__ cl,
                                int32_t *__restrict__ bad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G) return;
  int lo = 0, hi = n;  // the cluster c with cptr[c] <= q < cptr[c + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (cptr[mid] <= q) lo = mid; else hi = mid;
  }
  const int g = cgate[q];
  if (g < 0 || g >= n_gates) {
    atomicOr(bad, 1);
    return;
  }
  if (atomicCAS(cl + g, -1, lo) != -1) atomicOr(bad, 2);
}

// ---- exclusive scan in place: tile sums, scan of the sums, tile scans ------
constexpr int kScanThreads = 256, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

// Exclusive scan of one value per thread across the block; returns the
// block total through *total.
template <typename T>
__device__ __forceinline__ T block_exclusive(T v, T *total) {
  __shared__ T warp_sum[kScanThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_sum[w] = inc;
  __syncthreads();
  T before = 0, all = 0;
  for (int k = 0; k < kScanThreads / 32; ++k) {
    if (k < w) before += warp_sum[k];
    all += warp_sum[k];
  }
  __syncthreads();  // warp_sum is reused by the next call
  *total = all;
  return before + inc - v;
}

template <typename T>
__global__ void scan_sum_kernel(const T *__restrict__ a, long long n, T *__restrict__ tsum) {
  const long long base = (long long)blockIdx.x * kScanTile + threadIdx.x * kScanPer;
  T v = 0;
  for (int k = 0; k < kScanPer; ++k)
    if (base + k < n) v += a[base + k];
  T total;
  block_exclusive(v, &total);
  if (threadIdx.x == 0) tsum[blockIdx.x] = total;
}

template <typename T>
__global__ void scan_top_kernel(T *__restrict__ tsum, int tiles) {
  T carry = 0;
  for (int base = 0; base < tiles; base += kScanThreads) {
    const int i = base + threadIdx.x;
    const T v = i < tiles ? tsum[i] : T(0);
    T total;
    const T ex = block_exclusive(v, &total);
    if (i < tiles) tsum[i] = carry + ex;
    carry += total;
  }
}

template <typename T>
__global__ void scan_apply_kernel(T *__restrict__ a, long long n, const T *__restrict__ tsum) {
  const long long base = (long long)blockIdx.x * kScanTile + threadIdx.x * kScanPer;
  T v[kScanPer], t = 0;
  for (int k = 0; k < kScanPer; ++k) {
    v[k] = base + k < n ? a[base + k] : T(0);
    t += v[k];
  }
  T total;
  T run = block_exclusive(t, &total) + tsum[blockIdx.x];
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < n) a[base + k] = run;
    run += v[k];
  }
}

int scan_tiles(long long n) { return (int)((n + kScanTile - 1) / kScanTile); }

// In-place exclusive scan of a[0..n) on stream s; tsum holds scan_tiles(n).
template <typename T>
int exclusive_scan(T *a, long long n, T *tsum, cudaStream_t s) {
  if (n <= 0) return FX_OK;
  const int tiles = scan_tiles(n);
  scan_sum_kernel<T><<<tiles, kScanThreads, 0, s>>>(a, n, tsum);
  scan_top_kernel<T><<<1, kScanThreads, 0, s>>>(tsum, tiles);
  scan_apply_kernel<T><<<tiles, kScanThreads, 0, s>>>(a, n, tsum);
  FX_CHECK_LAUNCH();
  return FX_OK;
}

// ---- distinct clusters of every net ---------------------------------------
// For net e with pins [b, t): its c distinct clusters go to dc[b .. b+c) in
// first-pin order, dn[b + k] = e for k < c and -1 beyond, cnt[e] = c,
// npairs[e] = c (c - 1), and touch[a] += 1 for each (|nets touching a|).
constexpr int kSmallNet = 32;
constexpr int kMaxClusters = 65535;
constexpr int kBitmapWords = (kMaxClusters + 31) / 32;
constexpr int kBigThreads = 256;

// The distinct clusters of net e by one warp (at most 32 pins).
__device__ __forceinline__ void dedupe_warp_net(int e, int lane,
                                                const int32_t *__restrict__ net_ptr,
                                                const int32_t *__restrict__ net_gate,
                                                const int32_t *__restrict__ cl,
                                                int32_t *__restrict__ dc,
                                                int32_t *__restrict__ dn,
                                                int32_t *__restrict__ cnt,
                                                unsigned long long *__restrict__ npairs,
                                                int32_t *__restrict__ touch) {
  const int b = net_ptr[e], deg = net_ptr[e + 1] - b;
  // lanes past the net's pins get distinct negative tags, pins of no cluster -1
  const int c = lane < deg ? cl[net_gate[b + lane]] : -2 - lane;
  const unsigned same = __match_any_sync(0xffffffffu, c);
  const bool first = c >= 0 && (__ffs(same) - 1) == lane;
  const unsigned firsts = __ballot_sync(0xffffffffu, first);
  const int k = __popc(firsts);
  if (first) {
    const int pos = __popc(firsts & ((1u << lane) - 1u));
    dc[b + pos] = c;
    atomicAdd(touch + c, 1);
  }
  if (lane < deg) dn[b + lane] = lane < k ? e : -1;
  if (lane == 0) {
    cnt[e] = k;
    npairs[e] = (unsigned long long)k * (unsigned long long)(k > 0 ? k - 1 : 0);
  }
}

constexpr int kThreadNet = 16;

// Appends e to list[] for every lane with `take`, one atomic per warp.
__device__ __forceinline__ void warp_push(bool take, int e, int32_t *__restrict__ list,
                                          int32_t *__restrict__ count) {
  const unsigned mask = __ballot_sync(0xffffffffu, take);
  if (!mask) return;
  const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (take) list[base + __popc(mask & ((1u << lane) - 1u))] = e;
}

// One thread per net of at most 16 pins, deduplicated in registers; nets of
// 17..32 pins are listed in mid[], larger ones in big[]. The touches of a
// warp's nets are added once per distinct cluster and pin slot
// (__match_any_sync), which keeps the few counters of shallow levels from
// serialising the kernel.
__global__ void __launch_bounds__(256)
attn_dedupe_thread_kernel(int m, const int32_t *__restrict__ net_ptr,
                          const int32_t *__restrict__ net_gate, const int32_t *__restrict__ cl,
                          int32_t *__restrict__ dc, int32_t *__restrict__ dn,
                          int32_t *__restrict__ cnt, unsigned long long *__restrict__ npairs,
                          int32_t *__restrict__ touch, int32_t *__restrict__ mid,
                          int32_t *__restrict__ n_mid, int32_t *__restrict__ big,
                          int32_t *__restrict__ n_big) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool active = e < m;  // no early return: the warp votes below
  int b = 0, deg = 0;
  if (active) {
    b = net_ptr[e];
    deg = net_ptr[e + 1] - b;
  }
  const bool small = active && deg <= kThreadNet;
  warp_push(active && deg > kThreadNet && deg <= kSmallNet, e, mid, n_mid);
  warp_push(active && deg > kSmallNet, e, big, n_big);
  int cc[kThreadNet];
#pragma unroll
  for (int i = 0; i < kThreadNet; ++i) cc[i] = (small && i < deg) ? cl[net_gate[b + i]] : -1;
  unsigned firsts = 0;
  int k = 0;
#pragma unroll
  for (int i = 0; i < kThreadNet; ++i) {
    bool f = cc[i] >= 0;
#pragma unroll
    for (int j = 0; j < i; ++j) f = f && cc[j] != cc[i];
    if (f) {
      dc[b + k] = cc[i];
      ++k;
      firsts |= 1u << i;
    }
  }
  if (small) {
    for (int q = 0; q < deg; ++q) dn[b + q] = q < k ? e : -1;
    cnt[e] = k;
    npairs[e] = (unsigned long long)k * (unsigned long long)(k > 0 ? k - 1 : 0);
  }
  const int maxdeg = __reduce_max_sync(0xffffffffu, small ? deg : 0);
#pragma unroll
  for (int i = 0; i < kThreadNet; ++i) {
    if (i >= maxdeg) break;  // uniform across the warp
    const int c = (firsts >> i) & 1u ? cc[i] : -1;
    const unsigned same = __match_any_sync(0xffffffffu, c);
    if (c >= 0 && (__ffs(same) - 1) == lane) atomicAdd(touch + c, __popc(same));
  }
}

// One warp per listed net of 17..32 pins (grid-stride over *n_mid).
__global__ void attn_dedupe_warp_kernel(const int32_t *__restrict__ mid,
                                        const int32_t *__restrict__ n_mid,
                                        const int32_t *__restrict__ net_ptr,
                                        const int32_t *__restrict__ net_gate,
                                        const int32_t *__restrict__ cl,
                                        int32_t *__restrict__ dc, int32_t *__restrict__ dn,
                                        int32_t *__restrict__ cnt,
                                        unsigned long long *__restrict__ npairs,
                                        int32_t *__restrict__ touch) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int nm = *n_mid;
  for (int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < nm; i += warps)
    dedupe_warp_net(mid[i], lane, net_ptr, net_gate, cl, dc, dn, cnt, npairs, touch);
}
// One block per listed net (grid-stride over *n_big); the bitmap holds the
// clusters seen so far in the net and is cleared pin by pin afterwards.
__global__ void __launch_bounds__(kBigThreads)
attn_dedupe_big_kernel(const int32_t *__restrict__ big, const int32_t *__restrict__ n_big,
                       const int32_t *__restrict__ net_ptr,
                       const int32_t *__restrict__ net_gate, const int32_t *__restrict__ cl,
                       int n, int32_t *__restrict__ dc, int32_t *__restrict__ dn,
                       int32_t *__restrict__ cnt, unsigned long long *__restrict__ npairs,
                       int32_t *__restrict__ touch) {
  __shared__ uint32_t seen[kBitmapWords];
  const int words = (n + 31) >> 5;
  for (int w = threadIdx.x; w < words; w += blockDim.x) seen[w] = 0u;
  __syncthreads();
  const int nb = *n_big;
  for (int i = blockIdx.x; i < nb; i += gridDim.x) {
    const int e = big[i];
    const int b = net_ptr[e], t = net_ptr[e + 1];
    int base = 0;
    for (int q0 = b; q0 < t; q0 += blockDim.x) {  // uniform trip count
      const int q = q0 + threadIdx.x;
      const int c = q < t ? cl[net_gate[q]] : -1;
      int first = 0;
      if (c >= 0) {
        const uint32_t bit = 1u << (c & 31);
        first = (atomicOr(seen + (c >> 5), bit) & bit) == 0u;
      }
      int total;
      const int pos = base + block_exclusive(first, &total);
      if (first) {
        dc[b + pos] = c;
        atomicAdd(touch + c, 1);
      }
      base += total;
    }
    for (int q = b + threadIdx.x; q < t; q += blockDim.x) dn[q] = q - b < base ? e : -1;
    if (threadIdx.x == 0) {
      cnt[e] = base;
      npairs[e] = (unsigned long long)base * (unsigned long long)(base > 0 ? base - 1 : 0);
    }
    __syncthreads();  // every bit of this net is set before any is cleared
    for (int q = b + threadIdx.x; q < t; q += blockDim.x) {
      const int c = cl[net_gate[q]];
      if (c >= 0) seen[c >> 5] = 0u;
    }
    __syncthreads();
  }
}

// Record slot q of net e (dn[q] = e) emits (a, a_k) for every other distinct
// cluster k of e, as keys a * n + a_k, at off[e] + j (c - 1), j = q - b.
__global__ void attn_emit_kernel(int pins, int n, const int32_t *__restrict__ net_ptr,
                                 const int32_t *__restrict__ dn, const int32_t *__restrict__ dc,
                                 const int32_t *__restrict__ cnt,
                                 const unsigned long long *__restrict__ off,
                                 uint32_t *__restrict__ keys) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= pins) return;
  const int e = dn[q];
  if (e < 0) return;
  const int b = net_ptr[e], c = cnt[e], j = q - b;
  unsigned long long o = off[e] + (unsigned long long)j * (unsigned long long)(c - 1);
  const uint32_t row = (uint32_t)dc[q] * (uint32_t)n;
  for (int k = 0; k < c; ++k)
    if (k != j) keys[o++] = row + (uint32_t)dc[b + k];
}

// ---- run-length count of the sorted pair keys ------------------------------
// head[i] = 1 where a run of equal keys starts; head[p] = 0 (after the scan
// it holds the number of runs).
__global__ void attn_head_kernel(const uint32_t *__restrict__ key, int p,
                                 uint32_t *__restrict__ head) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > p) return;
  head[i] = (i < p && (i == 0 || key[i] != key[i - 1])) ? 1u : 0u;
}

// The first key of every run and where the run starts, at the run's index.
__global__ void attn_compact_kernel(const uint32_t *__restrict__ key, int p,
                                    const uint32_t *__restrict__ idx,
                                    uint32_t *__restrict__ ukey, int32_t *__restrict__ ustart) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p) return;
  if (idx[i + 1] != idx[i]) {  // a run starts at i
    ukey[idx[i]] = key[i];
    ustart[idx[i]] = i;
  }
}

// Scores of the pairs with shared nets (count = length of the key's run),
// and the dense matrix when asked. *nu = number of runs.
__global__ void attn_score_kernel(int p, int n, const uint32_t *__restrict__ nu,
                                  const uint32_t *__restrict__ ukey,
                                  const int32_t *__restrict__ ustart,
                                  const int32_t *__restrict__ touch,
                                  float *__restrict__ score, float *__restrict__ dense) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int u = (int)*nu;
  if (i >= u) return;
  const int cnt = (i + 1 < u ? ustart[i + 1] : p) - ustart[i];
  const uint32_t a = ukey[i] / (uint32_t)n, b = ukey[i] % (uint32_t)n;
  const float s = __fdiv_rn((float)cnt, (float)touch[a]);
  score[i] = s;
  if (dense) dense[(size_t)a * n + b] = s;
}

// One warp per cluster a: its pairs are the run of sorted keys in
// [a n, (a + 1) n), by ascending b. Round r picks the best entry below the
// previous pick in the order (score descending, b ascending) -- the stable
// descending sort of the reference -- as the warp maximum of the 64-bit key
// (score bits, ~b); positive f32 scores order like their bit patterns.
__device__ __forceinline__ int lower_bound_u32(const uint32_t *__restrict__ a, int u,
                                               uint32_t v) {
  int lo = 0, hi = u;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void attn_topk_kernel(int n, const uint32_t *__restrict__ nu, int top_k,
                                 const uint32_t *__restrict__ ukey,
                                 const float *__restrict__ score, int32_t *__restrict__ out) {
  const int a = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (a >= n) return;  // uniform per warp
  const int u = nu ? (int)*nu : 0;
  const uint32_t row = (uint32_t)a * (uint32_t)n;
  const int lo = lower_bound_u32(ukey, u, row);
  const int hi = lower_bound_u32(ukey, u, row + (uint32_t)n);  // (n - 1) n + n < 2^32
  int32_t *o = out + (size_t)a * top_k;
  unsigned long long last = ~0ull;
  int r = 0;
  for (; r < top_k; ++r) {
    unsigned long long best = 0;
    for (int i = lo + lane; i < hi; i += 32) {
      const unsigned long long key =
          ((unsigned long long)__float_as_uint(score[i]) << 32) | (0xFFFFFFFFu - (ukey[i] - row));
      if (key < last && key > best) best = key;
    }
    for (int off = 16; off > 0; off >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, off);
      best = other > best ? other : best;
    }
    if (best == 0) break;  // the row has no entry left
    if (lane == 0) o[r] = (int32_t)(0xFFFFFFFFu - (uint32_t)best);
    last = best;
  }
  for (int rr = r + lane; rr < top_k; rr += 32) o[rr] = -1;
}

}  // namespace
}  // namespace fx

using namespace fx;

extern "C" int fx_attention(fx_ctx *ctx, fx_design *d, int32_t n_clusters,
                            const int32_t *cluster_ptr, const int32_t *cluster_gate,
                            int32_t top_k, int32_t *out_topk, float *out_scores) {
  if (!ctx || !d || n_clusters < 0 || top_k < 0 || top_k > 1024 ||
      (n_clusters > 0 && !cluster_ptr)) {
    set_error("fx_attention: invalid arguments");
    return FX_EINVAL;
  }
  if (n_clusters > 65535) {
    set_error("fx_attention: %d clusters; at most 65535 per level", n_clusters);
    return FX_EINVAL;
  }
  const int n = n_clusters;
  if (n == 0) return FX_OK;
  if (cluster_ptr[0] != 0) {
    set_error("fx_attention: cluster_ptr[0] must be 0");
    return FX_EINVAL;
  }
  for (int c = 0; c < n; ++c)
    if (cluster_ptr[c + 1] < cluster_ptr[c]) {
      set_error("fx_attention: cluster_ptr decreases at %d", c);
      return FX_EINVAL;
    }
  const int G = cluster_ptr[n];
  if (G > 0 && !cluster_gate) {
    set_error("fx_attention: cluster_gate is NULL");
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream;
  const int m = d->m;
  if (d->p >= INT32_MAX) {
    set_error("fx_attention: %lld pins exceed the buffer limit", (long long)d->p);
    return FX_EINVAL;
  }
  const int pins = m > 0 ? (int)d->p : 0;
  const size_t nk = top_k > 0 ? (size_t)n * top_k : 1;
  int launches = 0;
  const size_t pp = (size_t)pins + 1, mm = (size_t)m + 1;
  DevBuf<int32_t> d_cl, d_cptr, d_cgate, d_bad, touch, dc, dn, cnt, mid, big, out;
  DevBuf<unsigned long long> npairs, psum;
  DevBuf<float> score, dense;
  FX_TRY(d_cl.alloc(d->n));
  FX_TRY(d_cptr.alloc((size_t)n + 1));
  FX_TRY(d_cgate.alloc(G > 0 ? (size_t)G : 1));
  FX_TRY(d_bad.alloc(3));  // [0] error flags, [1] nets of > 32 pins, [2] of 17..32
  FX_TRY(touch.alloc(n));
  FX_TRY(dc.alloc(pp));
  FX_TRY(dn.alloc(pp));
  FX_TRY(cnt.alloc(mm));
  FX_TRY(mid.alloc(mm));
  FX_TRY(big.alloc(mm));
  FX_TRY(npairs.alloc(mm));
  FX_TRY(psum.alloc(scan_tiles((long long)mm)));
  FX_CHECK_CUDA(cudaMemcpyAsync(d_cptr.p, cluster_ptr, ((size_t)n + 1) * 4,
                                cudaMemcpyHostToDevice, s));
  if (G > 0)
    FX_CHECK_CUDA(cudaMemcpyAsync(d_cgate.p, cluster_gate, (size_t)G * 4,
                                  cudaMemcpyHostToDevice, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d_cl.p, 0xFF, (size_t)d->n * 4, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d_bad.p, 0, 12, s));
  FX_CHECK_CUDA(cudaMemsetAsync(touch.p, 0, (size_t)n * 4, s));
  FX_CHECK_CUDA(cudaMemsetAsync(npairs.p + m, 0, 8, s));  // the total's slot
  cudaEvent_t t0;  // device time of the level, both halves around the host read
  timer_begin(ctx, FX_STAGE_ATTENTION, s, &t0);
  if (G > 0) {
    attn_map_kernel<<<(G + 255) / 256, 256, 0, s>>>(n, G, d->n, d_cptr.p, d_cgate.p, d_cl.p,
                                                    d_bad.p);
    FX_CHECK_LAUNCH();
    ++launches;
  }
  if (m > 0) {
    attn_dedupe_thread_kernel<<<(m + 255) / 256, 256, 0, s>>>(
        m, d->net_ptr.p, d->net_gate.p, d_cl.p, dc.p, dn.p, cnt.p, npairs.p, touch.p, mid.p,
        d_bad.p + 2, big.p, d_bad.p + 1);
    attn_dedupe_warp_kernel<<<4 * ctx->num_sms, 256, 0, s>>>(
        mid.p, d_bad.p + 2, d->net_ptr.p, d->net_gate.p, d_cl.p, dc.p, dn.p, cnt.p, npairs.p,
        touch.p);
    attn_dedupe_big_kernel<<<4 * ctx->num_sms, kBigThreads, 0, s>>>(
        big.p, d_bad.p + 1, d->net_ptr.p, d->net_gate.p, d_cl.p, n, dc.p, dn.p, cnt.p,
        npairs.p, touch.p);
    FX_CHECK_LAUNCH();
    launches += 3;
  }
  // exclusive offsets of the pairs; the extra (zero) slot becomes the total
  FX_TRY(exclusive_scan(npairs.p, (long long)mm, psum.p, s));
  launches += 3;
  timer_end(ctx, FX_STAGE_ATTENTION, s, t0);
  unsigned long long total = 0;
  int32_t bad = 0;
  FX_CHECK_CUDA(cudaMemcpyAsync(&total, npairs.p + m, 8, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(&bad, d_bad.p, 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (bad) {
    set_error("fx_attention: %s", (bad & 1) ? "a cluster gate is out of range"
                                            : "a gate is listed in two clusters");
    return FX_EINVAL;
  }
  if (total >= (unsigned long long)INT32_MAX) {
    set_error("fx_attention: %llu cluster pairs exceed the buffer limit", total);
    return FX_EINVAL;
  }
  const int P = (int)total;
  const size_t pc = (size_t)P + 1;
  DevBuf<uint32_t> keys[2], head, hsum;
  DevBuf<int32_t> vals[2];
  FX_TRY(keys[0].alloc(pc));
  FX_TRY(keys[1].alloc(pc));
  FX_TRY(vals[0].alloc(pc));
  FX_TRY(vals[1].alloc(pc));
  FX_TRY(head.alloc(pc));
  FX_TRY(hsum.alloc(scan_tiles((long long)pc)));
  FX_TRY(score.alloc(pc));
  FX_TRY(out.alloc(nk));
  DevBuf<uint32_t> kh, ks, dt;
  FX_TRY(kh.alloc((size_t)256 * radix_sort_tiles(P > 0 ? P : 1)));
  FX_TRY(ks.alloc((size_t)256 * radix_sort_tiles(P > 0 ? P : 1)));
  FX_TRY(dt.alloc(256));
  if (out_scores) {
    FX_TRY(dense.alloc((size_t)n * n));
    FX_CHECK_CUDA(cudaMemsetAsync(dense.p, 0, (size_t)n * n * 4, s));
  }
  cudaEvent_t t1;
  timer_begin(ctx, FX_STAGE_ATTENTION, s, &t1);
  if (P > 0) {
    attn_emit_kernel<<<(pins + 255) / 256, 256, 0, s>>>(pins, n, d->net_ptr.p, dn.p, dc.p,
                                                        cnt.p, npairs.p, keys[0].p);
    FX_CHECK_LAUNCH();
    // keys < n^2: as many 8-bit passes as n^2 - 1 has bytes
    const uint32_t kmax = (uint32_t)n * (uint32_t)n - 1u;
    int kp = 0;
    while (kp < 4 && (kmax >> (8 * kp)) != 0) ++kp;
    uint32_t *kk[2] = {keys[0].p, keys[1].p};
    int32_t *vv[2] = {vals[0].p, vals[1].p};
    FX_TRY(radix_sort_pairs(kk, vv, P, kp, kh.p, ks.p, dt.p, s));
    const uint32_t *skey = keys[kp & 1].p;
    uint32_t *ukey = keys[(kp & 1) ^ 1].p;
    // runs of equal keys: run index by a scan of the run heads
    attn_head_kernel<<<(P + 256) / 256, 256, 0, s>>>(skey, P, head.p);
    FX_CHECK_LAUNCH();
    FX_TRY(exclusive_scan(head.p, (long long)P + 1, hsum.p, s));
    attn_compact_kernel<<<(P + 255) / 256, 256, 0, s>>>(skey, P, head.p, ukey, vals[0].p);
    attn_score_kernel<<<(P + 255) / 256, 256, 0, s>>>(P, n, head.p + P, ukey, vals[0].p,
                                                      touch.p, score.p,
                                                      out_scores ? dense.p : nullptr);
    FX_CHECK_LAUNCH();
    launches += 1 + 3 * kp + 1 + 3 + 2;
    if (top_k > 0) {
      attn_topk_kernel<<<(n + 7) / 8, 256, 0, s>>>(n, head.p + P, top_k, ukey, score.p,
                                                   out.p);
      FX_CHECK_LAUNCH();
      ++launches;
    }
  } else if (top_k > 0) {
    attn_topk_kernel<<<(n + 7) / 8, 256, 0, s>>>(n, nullptr, top_k, keys[0].p, score.p,
                                                 out.p);
    FX_CHECK_LAUNCH();
    ++launches;
  }
  timer_end(ctx, FX_STAGE_ATTENTION, s, t1);
  if (top_k > 0 && out_topk)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_topk, out.p, nk * 4, cudaMemcpyDeviceToHost, s));
  if (out_scores)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_scores, dense.p, (size_t)n * n * 4,
                                  cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  ctx->launches += launches;
  return FX_OK;
}
