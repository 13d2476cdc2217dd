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
#include <functional>
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

// A level's gate -> cluster map from the gate -> leaf map and the level's
// leaf -> cluster index (-1: a leaf above the level).
__global__ void attn_level_map_kernel(int n_gates, const int32_t *__restrict__ gate_leaf,
                                      const int32_t *__restrict__ leaf_cluster,
                                      int32_t *__restrict__ cl) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n_gates;
       g += gridDim.x * blockDim.x) {
    const int l = gate_leaf[g];
    cl[g] = l >= 0 ? leaf_cluster[l] : -1;
  }
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
// 17..32 pins are listed in mid[], larger ones in big[]. Grid-stride over the
// nets. The touches of a warp's nets are added once per distinct cluster and
// pin slot (__match_any_sync), into a per-block shared histogram when the
// level has at most kHist clusters (flushed at the end): the few counters of
// shallow levels would otherwise serialise the kernel.
constexpr int kHist = 4096;

__global__ void __launch_bounds__(256)
attn_dedupe_thread_kernel(int m, int n, const int32_t *__restrict__ net_ptr,
                          const int32_t *__restrict__ net_gate, const int32_t *__restrict__ cl,
                          int32_t *__restrict__ dc, int32_t *__restrict__ dn,
                          int32_t *__restrict__ cnt, unsigned long long *__restrict__ npairs,
                          int32_t *__restrict__ touch, int32_t *__restrict__ mid,
                          int32_t *__restrict__ n_mid, int32_t *__restrict__ big,
                          int32_t *__restrict__ n_big) {
  __shared__ int32_t hist[kHist];
  const bool shared_hist = n <= kHist;
  if (shared_hist) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) hist[i] = 0;
    __syncthreads();
  }
  int32_t *tgt = shared_hist ? hist : touch;
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < m; base += gridDim.x * blockDim.x) {
    const int e = base + threadIdx.x;
    const bool active = e < m;  // no early exit: the warp votes below
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
      if (c >= 0 && (__ffs(same) - 1) == lane) atomicAdd(tgt + c, __popc(same));
    }
  }
  if (shared_hist) {
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      if (hist[i]) atomicAdd(touch + i, hist[i]);
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

// ---- shared-net counts, n <= kDenseMax: an n x n matrix per block ---------
// Each block adds the pairs of its nets into a shared n x n count matrix
// (a thread per net of <= 16 pins, a warp per listed larger net) and flushes
// it into the global matrix gm.
constexpr int kDenseMax = 128;

__global__ void __launch_bounds__(256)
attn_dense_count_kernel(int m, int n, const int32_t *__restrict__ net_ptr,
                        const int32_t *__restrict__ dc, const int32_t *__restrict__ cnt,
                        const int32_t *__restrict__ mid, const int32_t *__restrict__ n_mid,
                        const int32_t *__restrict__ big, const int32_t *__restrict__ n_big,
                        int32_t *__restrict__ gm) {
  extern __shared__ int32_t sm[];
  const int nn = n * n;
  for (int i = threadIdx.x; i < nn; i += blockDim.x) sm[i] = 0;
  __syncthreads();
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    const int b = net_ptr[e], deg = net_ptr[e + 1] - b;
    if (deg > kThreadNet) continue;  // listed: a warp takes it below
    const int c = cnt[e];
    int cc[kThreadNet];
#pragma unroll
    for (int i = 0; i < kThreadNet; ++i) cc[i] = i < c ? dc[b + i] : 0;
#pragma unroll
    for (int i = 0; i < kThreadNet; ++i) {
      if (i >= c) break;
#pragma unroll
      for (int j = 0; j < kThreadNet; ++j) {
        if (j >= c) break;
        if (j != i) atomicAdd(sm + cc[i] * n + cc[j], 1);
      }
    }
  }
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = stride >> 5;
  const int nm = *n_mid, nb = *n_big;
  for (int i = warp; i < nm + nb; i += warps) {
    const int e = i < nm ? mid[i] : big[i - nm];
    const int b = net_ptr[e], c = cnt[e];
    for (int t = lane; t < c * c; t += 32) {
      const int u = t / c, v = t - u * c;
      if (u != v) atomicAdd(sm + dc[b + u] * n + dc[b + v], 1);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nn; i += blockDim.x)
    if (sm[i]) atomicAdd(gm + i, sm[i]);
}

// One warp per row a of the n x n counts: scores, dense row, top-k rounds.
__device__ __forceinline__ unsigned long long rank_key(float score, int b) {
  return ((unsigned long long)__float_as_uint(score) << 32) | (0xFFFFFFFFu - (uint32_t)b);
}

__global__ void attn_dense_rows_kernel(int n, int top_k, const int32_t *__restrict__ gm,
                                       const int32_t *__restrict__ touch,
                                       float *__restrict__ dense, int32_t *__restrict__ out) {
  const int a = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (a >= n) return;  // uniform per warp
  const int32_t *row = gm + (size_t)a * n;
  const float tot = (float)touch[a];
  if (dense)
    for (int b = lane; b < n; b += 32)
      dense[(size_t)a * n + b] = row[b] ? __fdiv_rn((float)row[b], tot) : 0.0f;
  int32_t *o = out + (size_t)a * top_k;
  unsigned long long last = ~0ull;
  int r = 0;
  for (; r < top_k; ++r) {
    unsigned long long best = 0;
    for (int b = lane; b < n; b += 32) {
      if (!row[b]) continue;
      const unsigned long long key = rank_key(__fdiv_rn((float)row[b], tot), b);
      if (key < last && key > best) best = key;
    }
    for (int off = 16; off > 0; off >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, off);
      best = other > best ? other : best;
    }
    if (best == 0) break;
    if (lane == 0) o[r] = (int32_t)(0xFFFFFFFFu - (uint32_t)best);
    last = best;
  }
  for (int rr = r + lane; rr < top_k; rr += 32) o[rr] = -1;
}

// ---- shared-net counts, n <= kRowMax: one block per row -------------------
// The distinct (net, cluster) records are bucketed by cluster (rnet, by
// rp); the block of row a walks the nets touching a and counts the clusters
// of each in shared memory, listing each cluster on its first count.
constexpr int kRowMax = 16384;
constexpr int kRowThreads = 256;
constexpr int kKeyRegs = 4;

// Counting sort of the record slots by cluster, one contiguous chunk of
// slots per block: a shared histogram, one global reservation per (block,
// cluster), then the scatter through shared cursors.
constexpr int kBucketThreads = 512;

__global__ void __launch_bounds__(kBucketThreads)
attn_bucket_kernel(int pins, int n, const int32_t *__restrict__ dn,
                   const int32_t *__restrict__ dc, int32_t *__restrict__ cursor,
                   int32_t *__restrict__ rnet) {
  extern __shared__ int32_t sm[];
  int32_t *hist = sm, *base = sm + n;
  const int chunk = (pins + gridDim.x - 1) / gridDim.x;
  const int q0 = blockIdx.x * chunk, q1 = min(pins, q0 + chunk);
  for (int i = threadIdx.x; i < n; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x)
    if (dn[q] >= 0) atomicAdd(hist + dc[q], 1);
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (hist[i]) base[i] = atomicAdd(cursor + i, hist[i]);
    hist[i] = 0;
  }
  __syncthreads();
  for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    const int e = dn[q];
    if (e < 0) continue;
    const int a = dc[q];
    rnet[base[a] + atomicAdd(hist + a, 1)] = e;
  }
}

__global__ void __launch_bounds__(kRowThreads)
attn_rows_kernel(int n, int top_k, const int32_t *__restrict__ rp,
                 const int32_t *__restrict__ rnet, const int32_t *__restrict__ net_ptr,
                 const int32_t *__restrict__ dc, const int32_t *__restrict__ cnt,
                 const int32_t *__restrict__ touch, float *__restrict__ dense,
                 int32_t *__restrict__ out) {
  extern __shared__ int32_t sm[];
  int32_t *count = sm;                                        // [n]
  uint16_t *list = reinterpret_cast<uint16_t *>(sm + n);      // [n]
  __shared__ int list_n;
  __shared__ unsigned long long wbest[2 * (kRowThreads / 32)];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < n; i += blockDim.x) count[i] = 0;
  for (int a = blockIdx.x; a < n; a += gridDim.x) {
    if (tid == 0) list_n = 0;
    __syncthreads();
    const int lo = rp[a], hi = rp[a + 1];
    for (int r = lo + tid; r < hi; r += blockDim.x) {  // a record per thread
      const int e = rnet[r];
      const int b0 = net_ptr[e], c = cnt[e];
      for (int k = 0; k < c; ++k) {
        const int b = dc[b0 + k];
        if (b != a && atomicAdd(count + b, 1) == 0) list[atomicAdd(&list_n, 1)] = (uint16_t)b;
      }
    }
    __syncthreads();
    const int L = list_n;
    const float tot = (float)touch[a];
    if (dense)
      for (int i = tid; i < L; i += blockDim.x) {
        const int b = list[i];
        dense[(size_t)a * n + b] = __fdiv_rn((float)count[b], tot);
      }
    // rank keys held in registers when the row has at most kKeyRegs * threads
    // entries, else recomputed every round
    unsigned long long kr[kKeyRegs];
    const bool in_regs = L <= kKeyRegs * kRowThreads;
#pragma unroll
    for (int j = 0; j < kKeyRegs; ++j) {
      const int i = tid + j * kRowThreads;
      kr[j] = 0;
      if (in_regs && i < L) kr[j] = rank_key(__fdiv_rn((float)count[list[i]], tot), list[i]);
    }
    unsigned long long last = ~0ull;
    int r = 0;
    for (; r < top_k; ++r) {
      unsigned long long best = 0;
      if (in_regs) {
#pragma unroll
        for (int j = 0; j < kKeyRegs; ++j)
          if (kr[j] < last && kr[j] > best) best = kr[j];
      } else {
        for (int i = tid; i < L; i += blockDim.x) {
          const int b = list[i];
          const unsigned long long key = rank_key(__fdiv_rn((float)count[b], tot), b);
          if (key < last && key > best) best = key;
        }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, off);
        best = other > best ? other : best;
      }
      // double-buffered: round r + 1 writes the other half, and round r + 2
      // comes after the barrier of round r + 1
      unsigned long long *wb = wbest + (r & 1) * (kRowThreads / 32);
      if (lane == 0) wb[warp] = best;
      __syncthreads();
      best = 0;
      for (int w = 0; w < kRowThreads / 32; ++w) best = wb[w] > best ? wb[w] : best;
      if (best == 0) break;  // the same for every thread
      if (tid == 0) out[(size_t)a * top_k + r] = (int32_t)(0xFFFFFFFFu - (uint32_t)best);
      last = best;
    }
    for (int rr = r + tid; rr < top_k; rr += blockDim.x) out[(size_t)a * top_k + rr] = -1;
    for (int i = tid; i < L; i += blockDim.x) count[list[i]] = 0;
    __syncthreads();
  }
}

// ---- shared-net counts in a hash table of the pair keys -------------------
// Open addressing with linear probing over T = 2^log_t >= 2 P slots (key
// kEmpty = free); counts are added to the key's slot. The table's order is
// irrelevant: rows are bucketed afterwards and the top-k order is total.
constexpr uint32_t kEmpty = 0xFFFFFFFFu;  // a * n + b < n^2 <= 65535^2 < kEmpty

__device__ __forceinline__ uint32_t pair_slot(uint32_t key, int log_t) {
  return (uint32_t)(((unsigned long long)key * 0x9E3779B97F4A7C15ull) >> (64 - log_t));
}

// Record slot q of net e (dn[q] = e, j = q - net_ptr[e]) adds the pairs
// (a_j, a_k), k != j, of the net's c distinct clusters. Lanes with the same
// key in one round add once (__match_any_sync). bad[0] |= 4 if a probe ever
// went round the whole table (it cannot at load factor <= 1/2).
__global__ void __launch_bounds__(256)
attn_pairs_kernel(int pins, int n, const int32_t *__restrict__ net_ptr,
                  const int32_t *__restrict__ dn, const int32_t *__restrict__ dc,
                  const int32_t *__restrict__ cnt, int log_t, uint32_t *__restrict__ tkey,
                  uint32_t *__restrict__ tcnt, int32_t *__restrict__ bad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  int e = -1, b = 0, c = 0, j = 0;
  if (q < pins) e = dn[q];
  if (e >= 0) {
    b = net_ptr[e];
    c = cnt[e];
    j = q - b;
  }
  const uint32_t row = e >= 0 ? (uint32_t)dc[q] * (uint32_t)n : 0u;
  const uint32_t mask = (1u << log_t) - 1u;
  const int rounds = __reduce_max_sync(0xffffffffu, c);
  for (int t = 0; t < rounds; ++t) {
    const uint32_t key = (t < c && t != j) ? row + (uint32_t)dc[b + t] : kEmpty;
    const unsigned same = __match_any_sync(0xffffffffu, key);
    if (key == kEmpty || (__ffs(same) - 1) != lane) continue;
    uint32_t h = pair_slot(key, log_t);
    bool done = false;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      const uint32_t prev = atomicCAS(tkey + h, kEmpty, key);
      if (prev == kEmpty || prev == key) {
        atomicAdd(tcnt + h, (uint32_t)__popc(same));
        done = true;
        break;
      }
      h = (h + 1u) & mask;
    }
    if (!done) atomicOr(bad, 4);
  }
}

// Entries per row (cluster a), counted over the table.
__global__ void attn_row_count_kernel(uint32_t T, int n, const uint32_t *__restrict__ tkey,
                                      int32_t *__restrict__ rowcnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t key = i < T ? tkey[i] : kEmpty;
  const int a = key != kEmpty ? (int)(key / (uint32_t)n) : -1;
  const unsigned same = __match_any_sync(0xffffffffu, a);
  if (a >= 0 && (__ffs(same) - 1) == (int)(threadIdx.x & 31))
    atomicAdd(rowcnt + a, __popc(same));
}

// Each entry to its row's bucket (rowcur starts at the row offsets) with its
// score shared / |nets touching a| in f32, and to the dense matrix if asked.
__global__ void attn_row_fill_kernel(uint32_t T, int n, const uint32_t *__restrict__ tkey,
                                     const uint32_t *__restrict__ tcnt,
                                     const int32_t *__restrict__ touch,
                                     int32_t *__restrict__ rowcur, int32_t *__restrict__ rb,
                                     float *__restrict__ rs, float *__restrict__ dense) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  const uint32_t key = tkey[i];
  if (key == kEmpty) return;
  const uint32_t a = key / (uint32_t)n, b = key % (uint32_t)n;
  const float sc = __fdiv_rn((float)tcnt[i], (float)touch[a]);
  const int pos = atomicAdd(rowcur + a, 1);
  rb[pos] = (int32_t)b;
  rs[pos] = sc;
  if (dense) dense[(size_t)a * n + b] = sc;
}

// One warp per cluster a over its bucket [rowptr[a], rowptr[a+1]) (any
// order). Round r picks the best entry below the previous pick in the order
// (score descending, b ascending) -- the stable descending sort of the
// reference -- as the warp maximum of the 64-bit key (score bits, ~b);
// positive f32 scores order like their bit patterns.
__global__ void attn_topk_kernel(int n, int top_k, const int32_t *__restrict__ rowptr,
                                 const int32_t *__restrict__ rb, const float *__restrict__ rs,
                                 int32_t *__restrict__ out) {
  const int a = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (a >= n) return;  // uniform per warp
  const int lo = rowptr[a], hi = rowptr[a + 1];
  int32_t *o = out + (size_t)a * top_k;
  unsigned long long last = ~0ull;
  int r = 0;
  for (; r < top_k; ++r) {
    unsigned long long best = 0;
    for (int i = lo + lane; i < hi; i += 32) {
      const unsigned long long key =
          ((unsigned long long)__float_as_uint(rs[i]) << 32) | (0xFFFFFFFFu - (uint32_t)rb[i]);
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

// One level's scores and top-k. build_map enqueues on ctx->stream the
// kernels that fill the gate -> cluster map d_cl (preset to -1) and may set
// bad[0] (1: a gate out of range, 2: a gate in two clusters).
using MapBuilder = std::function<int(int32_t *d_cl, int32_t *bad, int *launches)>;

static int level_attention(fx_ctx *ctx, fx_design *d, int n, const MapBuilder &build_map,
                           int top_k, int32_t *out_topk, float *out_scores) {
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
  DevBuf<int32_t> d_cl, d_bad, touch, dc, dn, cnt, mid, big, out;
  DevBuf<unsigned long long> npairs, psum;
  DevBuf<float> dense;
  FX_TRY(d_cl.alloc(d->n));
  FX_TRY(d_bad.alloc(3));  // [0] error flags, [1] nets of > 32 pins, [2] of 17..32
  FX_TRY(touch.alloc(n));
  FX_TRY(dc.alloc(pp));
  FX_TRY(dn.alloc(pp));
  FX_TRY(cnt.alloc(mm));
  FX_TRY(mid.alloc(mm));
  FX_TRY(big.alloc(mm));
  FX_TRY(npairs.alloc(mm));
  FX_TRY(psum.alloc(scan_tiles((long long)mm)));
  FX_CHECK_CUDA(cudaMemsetAsync(d_cl.p, 0xFF, (size_t)d->n * 4, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d_bad.p, 0, 12, s));
  FX_CHECK_CUDA(cudaMemsetAsync(touch.p, 0, (size_t)n * 4, s));
  FX_CHECK_CUDA(cudaMemsetAsync(npairs.p + m, 0, 8, s));  // the total's slot
  cudaEvent_t t0;  // device time of the level, both halves around the host read
  timer_begin(ctx, FX_STAGE_ATTENTION, s, &t0);
  FX_TRY(build_map(d_cl.p, d_bad.p, &launches));
  if (m > 0) {
    const int tb = std::min((m + 255) / 256, 4 * ctx->num_sms);
    attn_dedupe_thread_kernel<<<tb, 256, 0, s>>>(m, n, d->net_ptr.p, d->net_gate.p, d_cl.p,
                                                 dc.p, dn.p, cnt.p, npairs.p, touch.p, mid.p,
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
  if (n <= kRowMax) {  // shared-memory counts, no pair list
    FX_TRY(out.alloc(nk));
    if (out_scores) {
      FX_TRY(dense.alloc((size_t)n * n));
      FX_CHECK_CUDA(cudaMemsetAsync(dense.p, 0, (size_t)n * n * 4, s));
    }
    DevBuf<int32_t> gm, rp, rcur, rsum, rnet;
    if (n <= kDenseMax) {
      // the whole level's counts as an n x n matrix
      FX_TRY(gm.alloc((size_t)n * n));
      FX_CHECK_CUDA(cudaMemsetAsync(gm.p, 0, (size_t)n * n * 4, s));
      const int smem = n * n * 4;
      FX_TRY(raise_smem_limit(reinterpret_cast<const void *>(attn_dense_count_kernel), smem));
      if (m > 0) {
        attn_dense_count_kernel<<<ctx->num_sms, 256, smem, s>>>(
            m, n, d->net_ptr.p, dc.p, cnt.p, mid.p, d_bad.p + 2, big.p, d_bad.p + 1, gm.p);
        FX_CHECK_LAUNCH();
        ++launches;
      }
      if (top_k > 0 || out_scores) {
        attn_dense_rows_kernel<<<(n + 7) / 8, 256, 0, s>>>(n, top_k, gm.p, touch.p,
                                                           out_scores ? dense.p : nullptr,
                                                           out.p);
        FX_CHECK_LAUNCH();
        ++launches;
      }
    } else {
      // records bucketed by cluster, then one block per row
      FX_TRY(rp.alloc((size_t)n + 1));
      FX_TRY(rcur.alloc((size_t)n + 1));
      FX_TRY(rsum.alloc(scan_tiles((long long)n + 1)));
      FX_TRY(rnet.alloc(pp));
      FX_CHECK_CUDA(cudaMemcpyAsync(rp.p, touch.p, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
      FX_CHECK_CUDA(cudaMemsetAsync(rp.p + n, 0, 4, s));
      FX_TRY(exclusive_scan(rp.p, (long long)n + 1, rsum.p, s));
      FX_CHECK_CUDA(cudaMemcpyAsync(rcur.p, rp.p, ((size_t)n + 1) * 4,
                                    cudaMemcpyDeviceToDevice, s));
      launches += 3;
      if (pins > 0) {
        const int bsm = 2 * n * 4;
        FX_TRY(raise_smem_limit(reinterpret_cast<const void *>(attn_bucket_kernel), bsm));
        attn_bucket_kernel<<<ctx->num_sms, kBucketThreads, bsm, s>>>(pins, n, dn.p, dc.p,
                                                                     rcur.p, rnet.p);
        FX_CHECK_LAUNCH();
        ++launches;
      }
      const int smem = n * 4 + ((n * 2 + 15) & ~15);
      FX_TRY(raise_smem_limit(reinterpret_cast<const void *>(attn_rows_kernel), smem));
      int per_sm = 1;
      FX_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, attn_rows_kernel,
                                                                  kRowThreads, smem));
      attn_rows_kernel<<<std::min(n, std::max(1, per_sm) * ctx->num_sms), kRowThreads, smem,
                         s>>>(
          n, top_k, rp.p, rnet.p, d->net_ptr.p, dc.p, cnt.p, touch.p,
          out_scores ? dense.p : nullptr, out.p);
      FX_CHECK_LAUNCH();
      ++launches;
    }
    timer_end(ctx, FX_STAGE_ATTENTION, s, t0);
    int32_t bad = 0;
    FX_CHECK_CUDA(cudaMemcpyAsync(&bad, d_bad.p, 4, cudaMemcpyDeviceToHost, s));
    FX_CHECK_CUDA(cudaStreamSynchronize(s));
    if (bad) {
      set_error("fx_attention: %s", (bad & 1) ? "a cluster gate is out of range"
                                              : "a gate is listed in two clusters");
      return FX_EINVAL;
    }
    if (top_k > 0 && out_topk)
      FX_CHECK_CUDA(cudaMemcpyAsync(out_topk, out.p, nk * 4, cudaMemcpyDeviceToHost, s));
    if (out_scores)
      FX_CHECK_CUDA(cudaMemcpyAsync(out_scores, dense.p, (size_t)n * n * 4,
                                    cudaMemcpyDeviceToHost, s));
    FX_CHECK_CUDA(cudaStreamSynchronize(s));
    ctx->launches += launches;
    return FX_OK;
  }
  // n > kRowMax: pair keys counted in a hash table
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
  int log_t = 10;
  while (log_t < 31 && (1ull << log_t) < 2ull * (unsigned long long)P) ++log_t;
  const uint32_t T = 1u << log_t;
  DevBuf<uint32_t> tkey, tcnt;
  DevBuf<int32_t> rowptr, rowcur, rb, rsum;
  DevBuf<float> rs;
  FX_TRY(tkey.alloc(T));
  FX_TRY(tcnt.alloc(T));
  FX_TRY(rowptr.alloc((size_t)n + 1));
  FX_TRY(rowcur.alloc((size_t)n + 1));
  FX_TRY(rsum.alloc(scan_tiles((long long)n + 1)));
  FX_TRY(rb.alloc((size_t)P + 1));
  FX_TRY(rs.alloc((size_t)P + 1));
  FX_TRY(out.alloc(nk));
  if (out_scores) {
    FX_TRY(dense.alloc((size_t)n * n));
    FX_CHECK_CUDA(cudaMemsetAsync(dense.p, 0, (size_t)n * n * 4, s));
  }
  FX_CHECK_CUDA(cudaMemsetAsync(rowptr.p, 0, ((size_t)n + 1) * 4, s));
  if (P > 0) {
    FX_CHECK_CUDA(cudaMemsetAsync(tkey.p, 0xFF, (size_t)T * 4, s));
    FX_CHECK_CUDA(cudaMemsetAsync(tcnt.p, 0, (size_t)T * 4, s));
  }
  cudaEvent_t t1;
  timer_begin(ctx, FX_STAGE_ATTENTION, s, &t1);
  if (P > 0) {
    attn_pairs_kernel<<<(pins + 255) / 256, 256, 0, s>>>(pins, n, d->net_ptr.p, dn.p, dc.p,
                                                         cnt.p, log_t, tkey.p, tcnt.p, d_bad.p);
    attn_row_count_kernel<<<(T + 255) / 256, 256, 0, s>>>(T, n, tkey.p, rowptr.p);
    FX_CHECK_LAUNCH();
    FX_TRY(exclusive_scan(rowptr.p, (long long)n + 1, rsum.p, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(rowcur.p, rowptr.p, ((size_t)n + 1) * 4,
                                  cudaMemcpyDeviceToDevice, s));
    attn_row_fill_kernel<<<(T + 255) / 256, 256, 0, s>>>(T, n, tkey.p, tcnt.p, touch.p,
                                                         rowcur.p, rb.p, rs.p,
                                                         out_scores ? dense.p : nullptr);
    FX_CHECK_LAUNCH();
    launches += 2 + 3 + 1;
  }
  if (top_k > 0) {
    attn_topk_kernel<<<(n + 7) / 8, 256, 0, s>>>(n, top_k, rowptr.p, rb.p, rs.p, out.p);
    FX_CHECK_LAUNCH();
    ++launches;
  }
  timer_end(ctx, FX_STAGE_ATTENTION, s, t1);
  int32_t bad2 = 0;
  FX_CHECK_CUDA(cudaMemcpyAsync(&bad2, d_bad.p, 4, cudaMemcpyDeviceToHost, s));
  if (top_k > 0 && out_topk)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_topk, out.p, nk * 4, cudaMemcpyDeviceToHost, s));
  if (out_scores)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_scores, dense.p, (size_t)n * n * 4,
                                  cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  ctx->launches += launches;
  if (bad2 & 4) {
    set_error("fx_attention: the pair table overflowed");
    return FX_ECUDA;
  }
  return FX_OK;
}

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
  return level_attention(
      ctx, d, n,
      [&](int32_t *d_cl, int32_t *bad, int *launches) -> int {
        cudaStream_t s = ctx->stream;
        DevBuf<int32_t> d_cptr, d_cgate;  // freed in stream order after the map
        FX_TRY(d_cptr.alloc((size_t)n + 1));
        FX_TRY(d_cgate.alloc(G > 0 ? (size_t)G : 1));
        FX_CHECK_CUDA(cudaMemcpyAsync(d_cptr.p, cluster_ptr, ((size_t)n + 1) * 4,
                                      cudaMemcpyHostToDevice, s));
        if (G > 0) {
          FX_CHECK_CUDA(cudaMemcpyAsync(d_cgate.p, cluster_gate, (size_t)G * 4,
                                        cudaMemcpyHostToDevice, s));
          attn_map_kernel<<<(G + 255) / 256, 256, 0, s>>>(n, G, d->n, d_cptr.p, d_cgate.p,
                                                          d_cl, bad);
          FX_CHECK_LAUNCH();
          ++*launches;
        }
        return FX_OK;
      },
      top_k, out_topk, out_scores);
}

// All levels of a hierarchy given by its leaves in DFS order and their depths
// (every internal node has two children, so the depths fix the tree):
// compute_all_attention (H/src/algorithm/attention.rs:33-48), the levels with
// at least two clusters in depth order. The leaf lists go up once; each level
// then needs only its leaf -> cluster index.
extern "C" int fx_attention_tree(fx_ctx *ctx, fx_design *d, int32_t n_leaves,
                                 const int32_t *leaf_ptr, const int32_t *leaf_gate,
                                 const int32_t *leaf_depth, int32_t top_k, int32_t max_levels,
                                 int32_t *out_n_levels, int32_t *out_level_depth,
                                 int32_t *out_level_clusters, int64_t topk_capacity,
                                 int32_t *out_topk) {
  if (!ctx || !d || n_leaves < 0 || top_k < 0 || top_k > 1024 || max_levels < 0 ||
      !out_n_levels || (n_leaves > 0 && (!leaf_ptr || !leaf_depth)) ||
      (max_levels > 0 && (!out_level_depth || !out_level_clusters))) {
    set_error("fx_attention_tree: invalid arguments");
    return FX_EINVAL;
  }
  *out_n_levels = 0;
  const int L = n_leaves;
  if (L == 0) return FX_OK;
  if (leaf_ptr[0] != 0) {
    set_error("fx_attention_tree: leaf_ptr[0] must be 0");
    return FX_EINVAL;
  }
  int dmax = 0;
  for (int l = 0; l < L; ++l) {
    if (leaf_ptr[l + 1] < leaf_ptr[l] || leaf_depth[l] < 0 || leaf_depth[l] > 62) {
      set_error("fx_attention_tree: leaf %d: bad range or depth (0..62)", l);
      return FX_EINVAL;
    }
    dmax = std::max(dmax, (int)leaf_depth[l]);
  }
  const int G = leaf_ptr[L];
  if (G > 0 && !leaf_gate) {
    set_error("fx_attention_tree: leaf_gate is NULL");
    return FX_EINVAL;
  }
  // path of each leaf as a dmax-free binary code (0 = first child); the
  // depths form a full binary tree iff the codes count up to 2^d - 1
  std::vector<uint64_t> code((size_t)L, 0);
  for (int l = 1; l < L; ++l) {
    uint64_t c = code[l - 1] + 1;
    const int dp = leaf_depth[l - 1], dl = leaf_depth[l];
    if (dl >= dp) {
      c <<= (dl - dp);
    } else {
      const int k = dp - dl;
      if (c & ((1ull << k) - 1ull)) {
        set_error("fx_attention_tree: leaf depths do not form a full binary tree");
        return FX_EINVAL;
      }
      c >>= k;
    }
    code[l] = c;
  }
  if (code[L - 1] + 1 != (1ull << leaf_depth[L - 1])) {
    set_error("fx_attention_tree: leaf depths do not form a full binary tree");
    return FX_EINVAL;
  }
  // per depth: the leaf -> cluster index and the cluster count
  std::vector<std::vector<int32_t>> lc;
  std::vector<int32_t> depth, count;
  int64_t need = 0;
  for (int t = 0; t <= dmax; ++t) {
    std::vector<int32_t> m((size_t)L, -1);
    int nt = 0;
    uint64_t prev = 0;
    bool any = false;
    for (int l = 0; l < L; ++l) {
      if (leaf_depth[l] < t) continue;
      const uint64_t pre = code[l] >> (leaf_depth[l] - t);
      if (!any || pre != prev) ++nt;
      any = true;
      prev = pre;
      m[l] = nt - 1;
    }
    if (nt < 2) continue;
    if (nt > 65535) {
      set_error("fx_attention_tree: %d clusters at depth %d; at most 65535", nt, t);
      return FX_EINVAL;
    }
    lc.push_back(std::move(m));
    depth.push_back(t);
    count.push_back(nt);
    need += (int64_t)nt * top_k;
  }
  const int nl = (int)depth.size();
  if (nl > max_levels || (out_topk && need > topk_capacity)) {
    set_error("fx_attention_tree: needs %d levels and %lld top-k slots", nl, (long long)need);
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream;
  // gate -> leaf, once (the same checks as a level's clusters)
  DevBuf<int32_t> gate_leaf, d_lp, d_lg, d_err, d_lc;
  FX_TRY(gate_leaf.alloc(d->n));
  FX_TRY(d_lp.alloc((size_t)L + 1));
  FX_TRY(d_lg.alloc(G > 0 ? (size_t)G : 1));
  FX_TRY(d_err.alloc(1));
  FX_TRY(d_lc.alloc((size_t)L));
  FX_CHECK_CUDA(cudaMemsetAsync(gate_leaf.p, 0xFF, (size_t)d->n * 4, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d_err.p, 0, 4, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(d_lp.p, leaf_ptr, ((size_t)L + 1) * 4, cudaMemcpyHostToDevice, s));
  if (G > 0) {
    FX_CHECK_CUDA(cudaMemcpyAsync(d_lg.p, leaf_gate, (size_t)G * 4, cudaMemcpyHostToDevice, s));
    attn_map_kernel<<<(G + 255) / 256, 256, 0, s>>>(L, G, d->n, d_lp.p, d_lg.p, gate_leaf.p,
                                                    d_err.p);
    FX_CHECK_LAUNCH();
    ctx->launches += 1;
  }
  int32_t err = 0;
  FX_CHECK_CUDA(cudaMemcpyAsync(&err, d_err.p, 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (err) {
    set_error("fx_attention_tree: %s", (err & 1) ? "a leaf gate is out of range"
                                                 : "a gate is listed in two leaves");
    return FX_EINVAL;
  }
  int64_t off = 0;
  for (int v = 0; v < nl; ++v) {
    const std::vector<int32_t> &m = lc[v];
    FX_TRY(level_attention(
        ctx, d, count[v],
        [&](int32_t *d_cl, int32_t *, int *launches) -> int {
          FX_CHECK_CUDA(cudaMemcpyAsync(d_lc.p, m.data(), (size_t)L * 4,
                                        cudaMemcpyHostToDevice, s));
          attn_level_map_kernel<<<std::min((d->n + 255) / 256, 8 * ctx->num_sms), 256, 0, s>>>(
              d->n, gate_leaf.p, d_lc.p, d_cl);
          FX_CHECK_LAUNCH();
          ++*launches;
          return FX_OK;
        },
        top_k, out_topk ? out_topk + off : nullptr, nullptr));
    out_level_depth[v] = depth[v];
    out_level_clusters[v] = count[v];
    off += (int64_t)count[v] * top_k;
  }
  *out_n_levels = nl;
  return FX_OK;
}
