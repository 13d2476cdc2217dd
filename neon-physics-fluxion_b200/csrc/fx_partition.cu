// fx_partition.cu -- (f.2) the hierarchy build: recursive spectral bisection
// (build_hierarchy, H/src/algorithm/partitioner.rs:36-100) on the device,
// plus the region pass of hapr_placement (H/src/algorithm/placer.rs:40-63,
// 111-141).
//
// The shape of the tree depends only on cluster sizes: a cluster of n gates
// is a leaf when n <= max_leaf_size or n <= min_cluster_size (:75), otherwise
// it splits at clamp(n/2, ceil(n*balance), n - ceil(n*balance)) (:197-212)
// into two halves. The host therefore lays out the whole tree up front; the
// device decides which gates go where. All clusters of one depth are
// processed together:
//   * every cluster is a contiguous segment of a gate permutation, left child
//     before right child, so the leaves come out in HierarchyTree::leaves()
//     order (hierarchy.rs:176-190);
//   * the power iteration runs on all clusters of the depth at once, on the
//     induced Laplacians (in-cluster adjacency entries in reference order);
//   * a stable segmented sort by Fiedler value (slice::sort_by with
//     partial_cmp, under which -0.0 == +0.0) reorders each segment, and the
//     split index cuts it into its two children.
// Two arithmetic modes:
//   FX_PART_EXACT  the reference's f32 iteration: v0 = sin(i * 2.71828) from
//                  the host's libm (the reference's f32::sin calls it too),
//                  sums of lv and lv^2 as sequential f32 folds (one warp per
//                  cluster, one lane adding), f32 mean / sqrt / divide:
//                  identical leaves.
//   FX_PART_FP64   f32 SpMV, FP64 chunked reductions (mean, norm, Rayleigh
//                  quotient), per-cluster stop once the Rayleigh quotient
//                  changes by <= tol (relative), at most power_iterations.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fx_internal.h"

namespace fx {
namespace {

constexpr int kPartChunk = 4096;

// Index of the last entry of the sorted array a[0..C) that is <= x.
__device__ __forceinline__ int last_le(const int32_t *__restrict__ a, int C, int x) {
  int lo = 0, hi = C - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Cluster of every position and gate at this depth (-1: not split here).
__global__ void part_fill_kernel(int n, const int32_t *__restrict__ perm,
                                 const int32_t *__restrict__ beg,
                                 const int32_t *__restrict__ end, int C,
                                 int32_t *__restrict__ clp, int32_t *__restrict__ clg) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int c = last_le(beg, C, p);
  const int cl = (beg[c] <= p && p < end[c]) ? c : -1;
  clp[p] = cl;
  clg[perm[p]] = cl;
}

// Degrees of the induced Laplacian (partitioner.rs:124-137: +1.0 per
// in-cluster adjacency entry) and the start vector v_i = sin(i * 2.71828).
__global__ void part_init_kernel(int n, const int32_t *__restrict__ perm,
                                 const int32_t *__restrict__ adj_ptr,
                                 const int32_t *__restrict__ adj_idx,
                                 const int32_t *__restrict__ clp,
                                 const int32_t *__restrict__ clg,
                                 const int32_t *__restrict__ beg,
                                 const float *__restrict__ sin_tab,
                                 float *__restrict__ deg, float *__restrict__ v) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int c = clp[p];
  if (c < 0) return;
  const int g = perm[p];
  int cnt = 0;
  for (int e = adj_ptr[g]; e < adj_ptr[g + 1]; ++e) cnt += clg[adj_idx[e]] == c;
  deg[p] = (float)cnt;
  v[p] = sin_tab[p - beg[c]];
}

// The depth's induced Laplacians as one CSR in position order: row p lists
// the positions of p's in-cluster neighbours in adjacency order, so the 30
// products of a depth read only in-cluster entries, row after row, instead
// of every adjacency entry through three gathers. Row lengths are the
// degrees part_init_kernel counted (0 outside the depth's clusters); an
// exclusive scan gives the row starts.
constexpr int kScanItems = 8, kScanTile = 256 * kScanItems;

__global__ void __launch_bounds__(256)
part_scan_tile_kernel(int n, const int32_t *__restrict__ clp, const float *__restrict__ deg,
                      int32_t *__restrict__ rp, int32_t *__restrict__ tsum) {
  __shared__ int32_t wsum[8];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int base = blockIdx.x * kScanTile + t * kScanItems;
  int c[kScanItems];
  int run = 0;
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    const int p = base + r;
    c[r] = p < n && clp[p] >= 0 ? (int)deg[p] : 0;
    run += c[r];
  }
  int x = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += u;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  int before = x - run;
  for (int q = 0; q < w; ++q) before += wsum[q];
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    const int p = base + r;
    if (p < n) rp[p] = before;
    before += c[r];
  }
  if (t == 255) tsum[blockIdx.x] = before;  // the tile's total
}

// Exclusive scan of the T tile totals in place (one block); tsum[T] = total.
__global__ void __launch_bounds__(1024)
part_scan_top_kernel(int T, int32_t *__restrict__ tsum) {
  __shared__ int32_t wsum[32];
  __shared__ int32_t carry_s;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t == 0) carry_s = 0;
  __syncthreads();
  for (int b0 = 0; b0 < T; b0 += 1024) {
    const int i = b0 + t;
    const int v = i < T ? tsum[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      int y = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) y += u;
      }
      wsum[lane] = y;
    }
    __syncthreads();
    const int carry = carry_s;
    const int excl = carry + (w > 0 ? wsum[w - 1] : 0) + x - v;
    if (i < T) tsum[i] = excl;
    __syncthreads();
    if (t == 1023) carry_s = excl + v;
    __syncthreads();
  }
  if (t == 0) tsum[T] = carry_s;
}

__global__ void part_scan_add_kernel(int n, int T, const int32_t *__restrict__ tsum,
                                     int32_t *__restrict__ rp) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) rp[p] += tsum[p / kScanTile];
  if (p == 0) rp[n] = tsum[T];
}

__global__ void part_csr_kernel(int n, const int32_t *__restrict__ perm,
                                const int32_t *__restrict__ pos_of,
                                const int32_t *__restrict__ adj_ptr,
                                const int32_t *__restrict__ adj_idx,
                                const int32_t *__restrict__ clp,
                                const int32_t *__restrict__ clg,
                                const int32_t *__restrict__ rp, int32_t *__restrict__ col) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int c = clp[p];
  if (c < 0) return;
  const int g = perm[p];
  int k = rp[p];
  for (int e = adj_ptr[g]; e < adj_ptr[g + 1]; ++e) {
    const int j = adj_idx[e];
    if (clg[j] == c) col[k++] = pos_of[j];
  }
}

// lv = deg * v - A v in the reference's f32 order per row: deg*v first,
// then minus each in-cluster neighbour in adjacency order
// (partitioner.rs:158-165), over the depth's CSR.
__global__ void part_spmv_csr_kernel(int n, const int32_t *__restrict__ rp,
                                     const int32_t *__restrict__ col,
                                     const int32_t *__restrict__ clp,
                                     const int32_t *__restrict__ active,
                                     const float *__restrict__ deg,
                                     const float *__restrict__ v, float *__restrict__ lv) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int c = clp[p];
  if (c < 0 || !active[c]) return;
  float l = __fmul_rn(deg[p], v[p]);
  const int e1 = rp[p + 1];
  for (int e = rp[p]; e < e1; ++e) l = __fsub_rn(l, v[col[e]]);
  lv[p] = l;
}

}  // namespace

// FX_PART_EXACT reductions: sequential f32 folds in position order
// (Iterator::sum), one warp per cluster. The warp stages tiles of x in
// shared memory with coalesced loads and lane 0 folds each tile in order, so
// the fold is bound by the add latency rather than by global loads. With
// `deflate`: mean = sum(x) / n and x -= mean in place (:167-171); then
// norm = sqrt(sum(x*x)), kept as the divisor only when norm > 1e-10
// (:151-156, :174-180).
constexpr int kSeqTile = 2048;

__global__ void __launch_bounds__(32)
part_seq_kernel(int C, const int32_t *__restrict__ beg, const int32_t *__restrict__ end,
                float *__restrict__ x, int deflate, float *__restrict__ nrm) {
  __shared__ float tile[kSeqTile];
  const int c = blockIdx.x, lane = threadIdx.x;
  if (c >= C) return;
  const int b = beg[c], e = end[c];
  float mean = 0.f;
  if (deflate) {
    float s = 0.f;
    for (int t0 = b; t0 < e; t0 += kSeqTile) {
      const int m = min(kSeqTile, e - t0);
      for (int i = lane; i < m; i += 32) tile[i] = x[t0 + i];
      __syncwarp();
      if (lane == 0) {
#pragma unroll 16
        for (int i = 0; i < m; ++i) s = __fadd_rn(s, tile[i]);
      }
      __syncwarp();
    }
    mean = __fdiv_rn(__shfl_sync(0xffffffffu, s, 0), (float)(e - b));
  }
  float q = 0.f;
  for (int t0 = b; t0 < e; t0 += kSeqTile) {
    const int m = min(kSeqTile, e - t0);
    for (int i = lane; i < m; i += 32) tile[i] = x[t0 + i];
    __syncwarp();
    if (lane == 0) {
      if (deflate) {
#pragma unroll 16
        for (int i = 0; i < m; ++i) {
          const float y = __fsub_rn(tile[i], mean);
          tile[i] = y;
          q = __fadd_rn(q, __fmul_rn(y, y));
        }
      } else {
#pragma unroll 16
        for (int i = 0; i < m; ++i) q = __fadd_rn(q, __fmul_rn(tile[i], tile[i]));
      }
    }
    __syncwarp();
    if (deflate)
      for (int i = lane; i < m; i += 32) x[t0 + i] = tile[i];
    __syncwarp();
  }
  if (lane == 0) {
    const float norm = __fsqrt_rn(q);
    nrm[c] = norm > 1e-10f ? norm : 0.f;
  }
}

namespace {

// v = (x - mean) / norm, or without the division when the norm was too
// small, for the active clusters. x may be v.
__global__ void part_div_kernel(int n, const int32_t *__restrict__ clp,
                                const int32_t *__restrict__ active, const float *x,
                                const float *__restrict__ mean,
                                const float *__restrict__ nrm, float *v) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int c = clp[p];
  if (c < 0 || !active[c]) return;
  float y = x[p];
  if (mean) y = __fsub_rn(y, mean[c]);
  const float r = nrm[c];
  v[p] = r > 0.f ? __fdiv_rn(y, r) : y;
}

// FX_PART_FP64: one warp per chunk (<= kPartChunk positions of one cluster)
// sums x, x^2 and v.x in FP64; one thread per cluster then adds its chunks
// in order, so the reductions are deterministic.
__global__ void part_chunk_kernel(int K, const int32_t *__restrict__ ck_beg,
                                  const int32_t *__restrict__ ck_end,
                                  const int32_t *__restrict__ ck_cl,
                                  const int32_t *__restrict__ active,
                                  const float *__restrict__ x, const float *__restrict__ v,
                                  double *__restrict__ part) {
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (k >= K || !active[ck_cl[k]]) return;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int p = ck_beg[k] + lane; p < ck_end[k]; p += 32) {
    const double a = (double)x[p];
    s1 += a;
    s2 += a * a;
    if (v) s3 += (double)v[p] * a;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
    s3 += __shfl_down_sync(0xffffffffu, s3, o);
  }
  if (lane == 0) {
    part[3 * k] = s1;
    part[3 * k + 1] = s2;
    part[3 * k + 2] = s3;
  }
}

// Mean and norm per cluster (|x - mean|^2 = sum(x^2) - n mean^2: 1^T L v = 0,
// so no cancellation), the Rayleigh quotient v.Lv of the unit v, and the
// stop test. Without `deflate` (the start vector): norm only.
__global__ void part_combine_kernel(int C, const int32_t *__restrict__ beg,
                                    const int32_t *__restrict__ end,
                                    const int32_t *__restrict__ cl_ck,
                                    const double *__restrict__ part, int deflate,
                                    double tol, int32_t *__restrict__ active,
                                    float *__restrict__ mean, float *__restrict__ nrm,
                                    double *__restrict__ lambda,
                                    int32_t *__restrict__ iters) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C || !active[c]) return;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int k = cl_ck[c]; k < cl_ck[c + 1]; ++k) {
    s1 += part[3 * k];
    s2 += part[3 * k + 1];
    s3 += part[3 * k + 2];
  }
  const double n = (double)(end[c] - beg[c]);
  const double m = deflate ? s1 / n : 0.0;
  const double var = deflate ? fmax(s2 - s1 * m, 0.0) : s2;
  const double norm = sqrt(var);
  mean[c] = (float)m;
  nrm[c] = norm > 1e-10 ? (float)norm : 0.f;
  if (!deflate) return;
  const double prev = lambda[c];
  lambda[c] = s3;
  iters[c] += 1;
  if (tol > 0.0 && iters[c] > 1 && fabs(s3 - prev) <= tol * fabs(s3))
    active[c] = 2;  // converged: this update is the last
}

__global__ void part_retire_kernel(int C, int32_t *__restrict__ active,
                                   int32_t *__restrict__ any) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  if (active[c] == 2) active[c] = 0;
  if (active[c]) atomicOr(any, 1);
}

// Sort input for the A positions of the bisected clusters, packed cluster
// by cluster (slot t of cluster c <-> position beg[c] + t - off[c]): the
// Fiedler value as an order-preserving uint32 (-0.0 read as +0.0, so equal
// values keep their order), the slot as the value.
__global__ void part_keys_kernel(int A, int C, const int32_t *__restrict__ beg,
                                 const int32_t *__restrict__ off,
                                 const float *__restrict__ v, uint32_t *__restrict__ key,
                                 int32_t *__restrict__ slot_pos, int32_t *__restrict__ val) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A) return;
  const int c = last_le(off, C, t);
  const int p = beg[c] + (t - off[c]);
  float f = v[p];
  if (f == 0.f) f = 0.f;
  const uint32_t u = __float_as_uint(f);
  key[t] = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
  slot_pos[t] = p;
  val[t] = t;
}

// After the value sort: the cluster of each slot's source, as the next key.
__global__ void part_major_kernel(int A, int C, const int32_t *__restrict__ val,
                                  const int32_t *__restrict__ off,
                                  uint32_t *__restrict__ key) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A) return;
  key[t] = (uint32_t)last_le(off, C, val[t]);
}

// Slot t now holds source slot val[t]: that gate moves to slot t's position.
__global__ void part_apply_kernel(int A, const int32_t *__restrict__ val,
                                  const int32_t *__restrict__ slot_pos,
                                  const int32_t *__restrict__ perm_in,
                                  int32_t *__restrict__ perm_out,
                                  int32_t *__restrict__ pos_of) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A) return;
  const int dst = slot_pos[t];
  const int g = perm_in[slot_pos[val[t]]];
  perm_out[dst] = g;
  pos_of[g] = dst;
}

struct PNode {
  int32_t beg, end, depth, left = -1, right = -1;
  float cx = 0.f, cy = 0.f, w = 0.f, h = 0.f;
};

// The tree of sizes (recursive_bisect, partitioner.rs:64-100), nodes in
// pre-order (the reference's next_id order).
int32_t build_shape(std::vector<PNode> &nodes, int32_t beg, int32_t end, int32_t depth,
                    const fx_part_cfg &cfg) {
  const int32_t id = (int32_t)nodes.size();
  PNode nd;
  nd.beg = beg;
  nd.end = end;
  nd.depth = depth;
  nodes.push_back(nd);
  const int32_t n = end - beg;
  if (n <= cfg.max_leaf_size || n <= cfg.min_cluster_size) return id;
  // split_by_fiedler (:197-212): min_size = (n as f32 * balance).ceil() as usize
  const float fm = std::ceil((float)n * cfg.balance_factor);
  const int64_t min_size = fm > 0.f ? (int64_t)fm : 0;
  int64_t split = n / 2;
  split = std::max<int64_t>(split, min_size);
  split = std::min<int64_t>(split, (int64_t)n - min_size);
  if (split <= 0 || split >= n) return id;  // an empty half: the cluster stays a leaf
  const int32_t l = build_shape(nodes, beg, beg + (int32_t)split, depth + 1, cfg);
  const int32_t r = build_shape(nodes, beg + (int32_t)split, end, depth + 1, cfg);
  nodes[id].left = l;
  nodes[id].right = r;
  return id;
}

// place_level_recursive (placer.rs:111-141) for two children: cols =
// ceil(sqrt(2)) = 2 and rows = 1, so each child gets one column of its
// parent, in the reference's f32 operations.
void place_regions(std::vector<PNode> &nodes, int32_t id) {
  const PNode nd = nodes[id];
  if (nd.left < 0) return;
  const int32_t kids[2] = {nd.left, nd.right};
  const size_t cnt = 2;
  const float half_w = nd.w / 2.0f, half_h = nd.h / 2.0f;
  const float ox = nd.cx - half_w, oy = nd.cy - half_h;
  const size_t cols = (size_t)std::ceil(std::sqrt((float)cnt));
  const size_t rows = (cnt + cols - 1) / cols;
  for (size_t i = 0; i < cnt; ++i) {
    const size_t col = i % cols, row = i / cols;
    const float cw = nd.w / (float)cols;
    const float ch = nd.h / (float)rows;
    PNode &c = nodes[kids[i]];
    c.cx = ox + ((float)col + 0.5f) * cw;
    c.cy = oy + ((float)row + 0.5f) * ch;
    c.w = cw;
    c.h = ch;
  }
  place_regions(nodes, nd.left);
  place_regions(nodes, nd.right);
}

template <class T>
int upload(DevBuf<T> &d, const std::vector<T> &h, cudaStream_t s) {
  FX_TRY(d.alloc(h.empty() ? 1 : h.size()));
  if (!h.empty())
    FX_CHECK_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T),
                                  cudaMemcpyHostToDevice, s));
  return FX_OK;
}

}  // namespace
}  // namespace fx

using namespace fx;

extern "C" int fx_part_cfg_default(fx_part_cfg *c) {
  if (!c) return FX_EINVAL;
  // PartitionConfig::default (partitioner.rs:24-32) with the power-iteration
  // count main.rs:80 passes; the FP64 mode's tolerance.
  c->max_leaf_size = 64;
  c->min_cluster_size = 8;
  c->balance_factor = 0.4f;
  c->power_iterations = 30;
  c->mode = FX_PART_EXACT;
  c->reserved0 = 0;
  c->tol = 1e-6;
  return FX_OK;
}

extern "C" int fx_partition(fx_ctx *ctx, fx_design *d, const fx_part_cfg *cfg,
                            int32_t leaf_capacity, int32_t *out_leaf_ptr,
                            int32_t *out_leaf_gate, float *out_region,
                            int32_t *out_leaf_depth, fx_part_stats *out_stats) {
  if (!ctx || !d || !cfg || cfg->max_leaf_size < 1 || cfg->min_cluster_size < 0 ||
      !(cfg->balance_factor >= 0.f && cfg->balance_factor <= 0.5f) ||
      cfg->power_iterations < 0 ||
      (cfg->mode != FX_PART_EXACT && cfg->mode != FX_PART_FP64) || !(cfg->tol >= 0.0) ||
      leaf_capacity < 0) {
    set_error("fx_partition: invalid arguments");
    return FX_EINVAL;
  }
  const int32_t N = d->n;
  std::vector<PNode> nodes;
  if (N > 0) build_shape(nodes, 0, N, 0, *cfg);
  int32_t max_depth = 0, n_leaves = 0, levels = 0, max_active = 0;
  for (const PNode &nd : nodes) {
    if (nd.left < 0) {
      ++n_leaves;
      max_depth = std::max(max_depth, nd.depth);
    } else {
      levels = std::max(levels, nd.depth + 1);
      max_active = std::max(max_active, nd.end - nd.beg);
    }
  }
  if (n_leaves > leaf_capacity && (out_leaf_ptr || out_region || out_leaf_depth)) {
    set_error("fx_partition: the tree has %d leaves, capacity %d", n_leaves, leaf_capacity);
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream;
  const bool exact = cfg->mode == FX_PART_EXACT;
  int64_t total_iters = 0;
  DevBuf<int32_t> perm[2], pos_of;
  int cur = 0;
  if (N > 0) {
    std::vector<int32_t> iota((size_t)N);
    for (int32_t i = 0; i < N; ++i) iota[i] = i;
    FX_TRY(upload(perm[0], iota, s));
    FX_TRY(upload(pos_of, iota, s));
    FX_TRY(perm[1].alloc(N));
  }
  if (levels > 0) {
    // the reference's start vector, from the host libm (as f32::sin)
    std::vector<float> sin_tab((size_t)max_active);
    for (int32_t i = 0; i < max_active; ++i) sin_tab[i] = std::sin((float)i * 2.71828f);
    DevBuf<float> d_sin, deg, v, lv, mean, nrm;
    DevBuf<int32_t> clp, clg, beg, end, off, act, iters, any, ck_beg, ck_end, ck_cl, cl_ck;
    DevBuf<double> part, lambda;
    DevBuf<uint32_t> keys[2], th, ts, dt;
    DevBuf<int32_t> vals[2], slot_pos;
    FX_TRY(upload(d_sin, sin_tab, s));
    FX_TRY(clp.alloc(N));
    FX_TRY(clg.alloc(N));
    FX_TRY(deg.alloc(N));
    FX_TRY(v.alloc(N));
    FX_TRY(lv.alloc(N));
    FX_TRY(keys[0].alloc(N));
    FX_TRY(keys[1].alloc(N));
    FX_TRY(vals[0].alloc(N));
    FX_TRY(vals[1].alloc(N));
    FX_TRY(slot_pos.alloc(N));
    FX_TRY(th.alloc((size_t)256 * radix_sort_tiles(N)));
    FX_TRY(ts.alloc((size_t)256 * radix_sort_tiles(N)));
    FX_TRY(dt.alloc(256));
    FX_TRY(any.alloc(1));
    const int nb = (N + 255) / 256;
    // the depth's in-cluster CSR: row starts, tile totals, neighbour positions
    const int st = (N + kScanTile - 1) / kScanTile;
    DevBuf<int32_t> rp, tsum, col;
    FX_TRY(rp.alloc((size_t)N + 1));
    FX_TRY(tsum.alloc((size_t)st + 1));
    FX_TRY(col.alloc(std::max<size_t>(d->adj_idx.n, 1)));
    for (int32_t depth = 0; depth < levels; ++depth) {
      // the clusters bisected at this depth, in position order (pre-order
      // lists them left to right within a depth)
      std::vector<int32_t> hb, he, hoff;
      int32_t A = 0;
      for (const PNode &nd : nodes)
        if (nd.depth == depth && nd.left >= 0) {
          hb.push_back(nd.beg);
          he.push_back(nd.end);
          hoff.push_back(A);
          A += nd.end - nd.beg;
        }
      const int C = (int)hb.size();
      if (C == 0) continue;
      FX_TRY(upload(beg, hb, s));
      FX_TRY(upload(end, he, s));
      FX_TRY(upload(off, hoff, s));
      FX_TRY(upload(act, std::vector<int32_t>((size_t)C, 1), s));
      FX_TRY(mean.alloc(C));
      FX_TRY(nrm.alloc(C));
      FX_TRY(lambda.alloc(C));
      FX_TRY(iters.alloc(C));
      FX_CHECK_CUDA(cudaMemsetAsync(lambda.p, 0, (size_t)C * 8, s));
      FX_CHECK_CUDA(cudaMemsetAsync(iters.p, 0, (size_t)C * 4, s));
      int K = 0;
      if (!exact) {
        std::vector<int32_t> hcb, hce, hcc, hclck((size_t)C + 1, 0);
        for (int c = 0; c < C; ++c) {
          for (int32_t p = hb[c]; p < he[c]; p += kPartChunk) {
            hcb.push_back(p);
            hce.push_back(std::min(p + kPartChunk, he[c]));
            hcc.push_back(c);
          }
          hclck[(size_t)c + 1] = (int32_t)hcb.size();
        }
        K = (int)hcb.size();
        FX_TRY(upload(ck_beg, hcb, s));
        FX_TRY(upload(ck_end, hce, s));
        FX_TRY(upload(ck_cl, hcc, s));
        FX_TRY(upload(cl_ck, hclck, s));
        FX_TRY(part.alloc((size_t)3 * K));
      }
      const int cb = (C + 63) / 64, kb = (K * 32 + 255) / 256;
      part_fill_kernel<<<nb, 256, 0, s>>>(N, perm[cur].p, beg.p, end.p, C, clp.p, clg.p);
      part_init_kernel<<<nb, 256, 0, s>>>(N, perm[cur].p, d->adj_ptr.p, d->adj_idx.p, clp.p,
                                          clg.p, beg.p, d_sin.p, deg.p, v.p);
      part_scan_tile_kernel<<<st, 256, 0, s>>>(N, clp.p, deg.p, rp.p, tsum.p);
      part_scan_top_kernel<<<1, 1024, 0, s>>>(st, tsum.p);
      part_scan_add_kernel<<<nb, 256, 0, s>>>(N, st, tsum.p, rp.p);
      part_csr_kernel<<<nb, 256, 0, s>>>(N, perm[cur].p, pos_of.p, d->adj_ptr.p, d->adj_idx.p,
                                         clp.p, clg.p, rp.p, col.p);
      ctx->launches += 4;
      // normalise the start vector (:151-156)
      if (exact) {
        part_seq_kernel<<<C, 32, 0, s>>>(C, beg.p, end.p, v.p, 0, nrm.p);
      } else {
        part_chunk_kernel<<<kb, 256, 0, s>>>(K, ck_beg.p, ck_end.p, ck_cl.p, act.p, v.p,
                                             nullptr, part.p);
        part_combine_kernel<<<cb, 64, 0, s>>>(C, beg.p, end.p, cl_ck.p, part.p, 0, 0.0, act.p,
                                              mean.p, nrm.p, lambda.p, iters.p);
      }
      part_div_kernel<<<nb, 256, 0, s>>>(N, clp.p, act.p, v.p, nullptr, nrm.p, v.p);
      FX_CHECK_LAUNCH();
      ctx->launches += exact ? 4 : 5;
      int it = 0;
      while (it < cfg->power_iterations) {
        part_spmv_csr_kernel<<<nb, 256, 0, s>>>(N, rp.p, col.p, clp.p, act.p, deg.p, v.p,
                                                lv.p);
        ++it;
        if (exact) {
          // deflate and norm in place in lv, then v = lv / norm (v = lv, :182)
          part_seq_kernel<<<C, 32, 0, s>>>(C, beg.p, end.p, lv.p, 1, nrm.p);
          part_div_kernel<<<nb, 256, 0, s>>>(N, clp.p, act.p, lv.p, nullptr, nrm.p, v.p);
          FX_CHECK_LAUNCH();
          ctx->launches += 3;
          continue;
        }
        part_chunk_kernel<<<kb, 256, 0, s>>>(K, ck_beg.p, ck_end.p, ck_cl.p, act.p, lv.p, v.p,
                                             part.p);
        part_combine_kernel<<<cb, 64, 0, s>>>(C, beg.p, end.p, cl_ck.p, part.p, 1, cfg->tol,
                                              act.p, mean.p, nrm.p, lambda.p, iters.p);
        part_div_kernel<<<nb, 256, 0, s>>>(N, clp.p, act.p, lv.p, mean.p, nrm.p, v.p);
        FX_CHECK_LAUNCH();
        ctx->launches += 4;
        if (cfg->tol <= 0.0) continue;  // fixed iteration count: nothing converges early
        FX_CHECK_CUDA(cudaMemsetAsync(any.p, 0, 4, s));
        part_retire_kernel<<<cb, 64, 0, s>>>(C, act.p, any.p);
        FX_CHECK_LAUNCH();
        ctx->launches += 1;
        if ((it & 7) == 0) {  // every 8 iterations: all converged?
          int32_t h_any = 0;
          FX_CHECK_CUDA(cudaMemcpyAsync(&h_any, any.p, 4, cudaMemcpyDeviceToHost, s));
          FX_CHECK_CUDA(cudaStreamSynchronize(s));
          if (!h_any) break;
        }
      }
      if (exact) {
        total_iters += (int64_t)it * C;
      } else {
        std::vector<int32_t> hit((size_t)C);
        FX_CHECK_CUDA(cudaMemcpyAsync(hit.data(), iters.p, (size_t)C * 4,
                                      cudaMemcpyDeviceToHost, s));
        FX_CHECK_CUDA(cudaStreamSynchronize(s));
        for (int32_t x : hit) total_iters += x;
      }
      // stable segmented sort: by value (4 passes), then stably by cluster
      const int ab = (A + 255) / 256;
      part_keys_kernel<<<ab, 256, 0, s>>>(A, C, beg.p, off.p, v.p, keys[0].p, slot_pos.p,
                                          vals[0].p);
      FX_CHECK_LAUNCH();
      uint32_t *kk[2] = {keys[0].p, keys[1].p};
      int32_t *vv[2] = {vals[0].p, vals[1].p};
      FX_TRY(radix_sort_pairs(kk, vv, A, 4, th.p, ts.p, dt.p, s));  // result in buffer 0
      int rb = 0;
      if (C > 1) {
        part_major_kernel<<<ab, 256, 0, s>>>(A, C, vals[0].p, off.p, keys[0].p);
        FX_CHECK_LAUNCH();
        const int passes = C <= 256 ? 1 : (C <= 65536 ? 2 : 3);
        FX_TRY(radix_sort_pairs(kk, vv, A, passes, th.p, ts.p, dt.p, s));
        rb = passes & 1;
      }
      FX_CHECK_CUDA(cudaMemcpyAsync(perm[cur ^ 1].p, perm[cur].p, (size_t)N * 4,
                                    cudaMemcpyDeviceToDevice, s));
      part_apply_kernel<<<ab, 256, 0, s>>>(A, vals[rb].p, slot_pos.p, perm[cur].p,
                                           perm[cur ^ 1].p, pos_of.p);
      FX_CHECK_LAUNCH();
      ctx->launches += 3;
      cur ^= 1;
      FX_CHECK_CUDA(cudaStreamSynchronize(s));
    }
  }
  // outputs: leaves in position order, with their regions
  if (!nodes.empty()) {
    nodes[0].cx = d->chip_w / 2.0f;
    nodes[0].cy = d->chip_h / 2.0f;
    nodes[0].w = d->chip_w;
    nodes[0].h = d->chip_h;
    place_regions(nodes, 0);
  }
  if (out_leaf_gate && N > 0)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_leaf_gate, perm[cur].p, (size_t)N * 4,
                                  cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  int32_t l = 0;
  for (const PNode &nd : nodes) {
    if (nd.left >= 0) continue;
    if (out_leaf_ptr) out_leaf_ptr[l] = nd.beg;
    if (out_region) {
      out_region[4 * l + 0] = nd.cx;
      out_region[4 * l + 1] = nd.cy;
      out_region[4 * l + 2] = nd.w;
      out_region[4 * l + 3] = nd.h;
    }
    if (out_leaf_depth) out_leaf_depth[l] = nd.depth;
    ++l;
  }
  if (out_leaf_ptr) out_leaf_ptr[n_leaves] = N;
  if (out_stats) {
    out_stats->n_leaves = n_leaves;
    out_stats->n_nodes = (int32_t)nodes.size();
    out_stats->max_depth = max_depth;
    out_stats->levels = levels;
    out_stats->power_iterations = total_iters;
  }
  return FX_OK;
}
