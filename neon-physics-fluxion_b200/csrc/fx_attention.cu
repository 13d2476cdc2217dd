// fx_attention.cu -- (f.4) attention scores between the clusters of one
// hierarchy level (compute_level_attention, H/src/algorithm/attention.rs:
// 50-88):
//   score(A -> B) = |nets touching A and B| / |nets touching A|,  A != B
// and, per cluster, the top_k clusters by score (descending, ties by index,
// as the stable sort_by of :81-82; zero scores dropped).
//
// The reference forms the dense n x n matrix from per-cluster net sets
// (nets_touching_gates, :90-99). Here the pins, tagged with their gate's
// cluster, are radix sorted by (net, cluster); the distinct records are the
// (net, cluster) incidences. Every net emits each ordered pair of its distinct
// clusters once, and a radix sort + run-length count of the pair keys gives
// the shared-net counts of the pairs that have any: the work follows the pins
// and the pairs, not n^2, and a high-fanout net costs no more than its
// pairs. Scans are three-phase tile scans of 1024 elements. All counts are integers, so the f32
// scores are those of the reference formula (shared as f32 / total as f32,
// rounded to nearest).
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

// One record per pin: its gate's cluster (kNoCluster when the gate is in no
// cluster of the level) and its net.
constexpr uint32_t kNoCluster = 0xFFFFu;  // cluster ids are < 65535

__global__ void attn_pin_kernel(int m, const int32_t *__restrict__ net_ptr,
                                const int32_t *__restrict__ net_gate,
                                const int32_t *__restrict__ cl, uint32_t *__restrict__ pc,
                                int32_t *__restrict__ pn) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m) return;
  for (int q = net_ptr[e]; q < net_ptr[e + 1]; ++q) {
    const int a = cl[net_gate[q]];
    pc[q] = a >= 0 ? (uint32_t)a : kNoCluster;
    pn[q] = e;
  }
}

// Records sorted by (net, cluster): head[i] = 1 where a distinct (net,
// cluster) pair with a real cluster starts; head[p] = 0.
__global__ void attn_rec_head_kernel(const int32_t *__restrict__ rn,
                                     const int32_t *__restrict__ rc, int p,
                                     uint32_t *__restrict__ head) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > p) return;
  head[i] = (i < p && (uint32_t)rc[i] != kNoCluster &&
             (i == 0 || rn[i] != rn[i - 1] || rc[i] != rc[i - 1])) ? 1u : 0u;
}

// Distinct records in order (dn = net, dc = cluster); each is one net
// touching one cluster, so touch[a] = |nets touching a|.
__global__ void attn_rec_compact_kernel(const int32_t *__restrict__ rn,
                                        const int32_t *__restrict__ rc, int p,
                                        const uint32_t *__restrict__ idx,
                                        int32_t *__restrict__ dn, int32_t *__restrict__ dc,
                                        int32_t *__restrict__ touch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p || idx[i + 1] == idx[i]) return;
  dn[idx[i]] = rn[i];
  dc[idx[i]] = rc[i];
  atomicAdd(touch + rc[i], 1);
}

// Sorting by net keeps every net's pins at [net_ptr[e], net_ptr[e+1]), so
// its distinct clusters are [idx[net_ptr[e]], idx[net_ptr[e+1]]): c of them,
// c (c - 1) ordered pairs.
__global__ void attn_net_pairs_kernel(int m, const int32_t *__restrict__ net_ptr,
                                      const uint32_t *__restrict__ idx,
                                      unsigned long long *__restrict__ npairs) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m) return;
  const unsigned long long c = idx[net_ptr[e + 1]] - idx[net_ptr[e]];
  npairs[e] = c * (c > 0 ? c - 1 : 0);
}

// Distinct record j of net e emits (a_j, a_k) for every other distinct
// cluster k of e, as keys a_j * n + a_k, at off[e] + (j - s) (c - 1).
__global__ void attn_emit_kernel(int D, int n, const int32_t *__restrict__ net_ptr,
                                 const uint32_t *__restrict__ idx,
                                 const int32_t *__restrict__ dn, const int32_t *__restrict__ dc,
                                 const unsigned long long *__restrict__ off,
                                 uint32_t *__restrict__ keys) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= D) return;
  const int e = dn[j];
  const int s = (int)idx[net_ptr[e]], t = (int)idx[net_ptr[e + 1]];
  unsigned long long o = off[e] + (unsigned long long)(j - s) * (unsigned long long)(t - s - 1);
  const uint32_t row = (uint32_t)dc[j] * (uint32_t)n;
  for (int k = s; k < t; ++k)
    if (k != j) keys[o++] = row + (uint32_t)dc[k];
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

// Per cluster: its pairs are a contiguous run of the sorted keys (ascending
// b); keep the top_k by score, ties by smaller b (stable descending sort).
__global__ void attn_topk_kernel(int n, const uint32_t *__restrict__ nu, int top_k,
                                 const uint32_t *__restrict__ ukey,
                                 const float *__restrict__ score, int32_t *__restrict__ best_b,
                                 float *__restrict__ best_s, int32_t *__restrict__ out) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const int u = nu ? (int)*nu : 0;
  // first key >= a * n
  const uint32_t lo_key = (uint32_t)a * (uint32_t)n;
  int lo = 0, hi = u;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ukey[mid] < lo_key) lo = mid + 1; else hi = mid;
  }
  int32_t *bb = best_b + (size_t)a * top_k;
  float *bs = best_s + (size_t)a * top_k;
  int have = 0;
  for (int i = lo; i < u && ukey[i] / (uint32_t)n == (uint32_t)a; ++i) {
    const float s = score[i];
    const int32_t b = (int32_t)(ukey[i] % (uint32_t)n);
    // entries come by ascending b, so an equal score never displaces one
    int pos = have;
    while (pos > 0 && bs[pos - 1] < s) --pos;
    if (pos >= top_k) continue;
    const int last = have < top_k ? have : top_k - 1;
    for (int r = last; r > pos; --r) {
      bs[r] = bs[r - 1];
      bb[r] = bb[r - 1];
    }
    bs[pos] = s;
    bb[pos] = b;
    if (have < top_k) ++have;
  }
  for (int r = 0; r < top_k; ++r) out[(size_t)a * top_k + r] = r < have ? bb[r] : -1;
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
  const int mb = (m + 255) / 256;
  int launches = 0;
  DevBuf<int32_t> d_cl, touch, bb, out, dn, dc;
  DevBuf<unsigned long long> npairs, psum;
  DevBuf<uint32_t> rc[2], idx, isum;
  DevBuf<int32_t> rn[2];
  DevBuf<float> bs, score, dense;
  const size_t pp = (size_t)pins + 1;
  DevBuf<int32_t> d_cptr, d_cgate, d_bad;
  FX_TRY(d_cl.alloc(d->n));
  FX_TRY(d_cptr.alloc((size_t)n + 1));
  FX_TRY(d_cgate.alloc(G > 0 ? (size_t)G : 1));
  FX_TRY(d_bad.alloc(1));
  FX_TRY(touch.alloc(n));
  FX_TRY(npairs.alloc((size_t)m + 1));
  FX_TRY(psum.alloc(scan_tiles((long long)m + 1)));
  FX_TRY(rc[0].alloc(pp));
  FX_TRY(rc[1].alloc(pp));
  FX_TRY(rn[0].alloc(pp));
  FX_TRY(rn[1].alloc(pp));
  FX_TRY(idx.alloc(pp));
  FX_TRY(isum.alloc(scan_tiles((long long)pp)));
  FX_TRY(dn.alloc(pp));
  FX_TRY(dc.alloc(pp));
  DevBuf<uint32_t> th, ts, dt;
  FX_TRY(th.alloc((size_t)256 * radix_sort_tiles(pins > 0 ? pins : 1)));
  FX_TRY(ts.alloc((size_t)256 * radix_sort_tiles(pins > 0 ? pins : 1)));
  FX_TRY(dt.alloc(256));
  FX_CHECK_CUDA(cudaMemcpyAsync(d_cptr.p, cluster_ptr, ((size_t)n + 1) * 4,
                                cudaMemcpyHostToDevice, s));
  if (G > 0)
    FX_CHECK_CUDA(cudaMemcpyAsync(d_cgate.p, cluster_gate, (size_t)G * 4,
                                  cudaMemcpyHostToDevice, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d_cl.p, 0xFF, (size_t)d->n * 4, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d_bad.p, 0, 4, s));
  FX_CHECK_CUDA(cudaMemsetAsync(touch.p, 0, (size_t)n * 4, s));
  FX_CHECK_CUDA(cudaMemsetAsync(npairs.p, 0, ((size_t)m + 1) * 8, s));
  cudaEvent_t t0;  // device time of the level, both halves around the host read
  timer_begin(ctx, FX_STAGE_ATTENTION, s, &t0);
  if (G > 0) {
    attn_map_kernel<<<(G + 255) / 256, 256, 0, s>>>(n, G, d->n, d_cptr.p, d_cgate.p, d_cl.p,
                                                    d_bad.p);
    FX_CHECK_LAUNCH();
    ++launches;
  }
  if (pins > 0) {
    attn_pin_kernel<<<mb, 256, 0, s>>>(m, d->net_ptr.p, d->net_gate.p, d_cl.p, rc[0].p,
                                       rn[0].p);
    FX_CHECK_LAUNCH();
    // (net, cluster) order: stable by cluster (16 bits), then stable by net
    uint32_t *k1[2] = {rc[0].p, rc[1].p};
    int32_t *v1[2] = {rn[0].p, rn[1].p};
    FX_TRY(radix_sort_pairs(k1, v1, pins, 2, th.p, ts.p, dt.p, s));  // result in buffer 0
    int net_passes = 0;
    while (net_passes < 4 && ((uint32_t)(m - 1) >> (8 * net_passes)) != 0) ++net_passes;
    uint32_t *k2[2] = {reinterpret_cast<uint32_t *>(rn[0].p),
                       reinterpret_cast<uint32_t *>(rn[1].p)};
    int32_t *v2[2] = {reinterpret_cast<int32_t *>(rc[0].p),
                      reinterpret_cast<int32_t *>(rc[1].p)};
    FX_TRY(radix_sort_pairs(k2, v2, pins, net_passes, th.p, ts.p, dt.p, s));
    const int rb = net_passes & 1;  // buffer holding the sorted records
    const int32_t *rnet = rn[rb].p;
    const int32_t *rcl = reinterpret_cast<const int32_t *>(rc[rb].p);
    attn_rec_head_kernel<<<(pins + 256) / 256, 256, 0, s>>>(rnet, rcl, pins, idx.p);
    FX_CHECK_LAUNCH();
    FX_TRY(exclusive_scan(idx.p, (long long)pp, isum.p, s));
    attn_rec_compact_kernel<<<(pins + 255) / 256, 256, 0, s>>>(rnet, rcl, pins, idx.p, dn.p,
                                                               dc.p, touch.p);
    attn_net_pairs_kernel<<<mb, 256, 0, s>>>(m, d->net_ptr.p, idx.p, npairs.p);
    FX_CHECK_LAUNCH();
    launches += 1 + 3 * 2 + 3 * net_passes + 1 + 3 + 2;
  }
  // exclusive offsets of the pairs; the extra (zero) slot becomes the total
  FX_TRY(exclusive_scan(npairs.p, (long long)m + 1, psum.p, s));
  if (m > 0) launches += 3;
  timer_end(ctx, FX_STAGE_ATTENTION, s, t0);
  unsigned long long total = 0;
  uint32_t distinct = 0;
  FX_CHECK_CUDA(cudaMemcpyAsync(&total, npairs.p + m, 8, cudaMemcpyDeviceToHost, s));
  int32_t bad = 0;
  if (pins > 0)
    FX_CHECK_CUDA(cudaMemcpyAsync(&distinct, idx.p + pins, 4, cudaMemcpyDeviceToHost, s));
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
  const int P = (int)total, D = (int)distinct;
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
  FX_TRY(bb.alloc(nk));
  FX_TRY(bs.alloc(nk));
  FX_TRY(out.alloc(nk));
  DevBuf<uint32_t> kh, ks;
  FX_TRY(kh.alloc((size_t)256 * radix_sort_tiles(P > 0 ? P : 1)));
  FX_TRY(ks.alloc((size_t)256 * radix_sort_tiles(P > 0 ? P : 1)));
  if (out_scores) {
    FX_TRY(dense.alloc((size_t)n * n));
    FX_CHECK_CUDA(cudaMemsetAsync(dense.p, 0, (size_t)n * n * 4, s));
  }
  cudaEvent_t t1;
  timer_begin(ctx, FX_STAGE_ATTENTION, s, &t1);
  if (P > 0) {
    attn_emit_kernel<<<(D + 255) / 256, 256, 0, s>>>(D, n, d->net_ptr.p, idx.p, dn.p, dc.p,
                                                     npairs.p, keys[0].p);
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
      attn_topk_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, head.p + P, top_k, ukey, score.p,
                                                       bb.p, bs.p, out.p);
      FX_CHECK_LAUNCH();
      ++launches;
    }
  } else if (top_k > 0) {
    attn_topk_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, nullptr, top_k, keys[0].p, score.p,
                                                     bb.p, bs.p, out.p);
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
