// fx_leaf.cu -- row H: batched leaf placement (place_gates_in_leaf for
// thousands of independent leaf clusters in one persistent launch).
//
// Semantics are those of place_gates_in_leaf (H/src/algorithm/placer.rs:
// 210-287), reproduced bit for bit:
//   * init (placer.rs:226-227): x_i = min_x + (i/n) w,
//     y_i = min_y + ((7i mod n)/n) h, velocities 0;
//   * attraction (:243-255): for each neighbour of gate i in adjacency order
//     that lies in the leaf, F_i += k (p_j - p_i); a gate listed more than
//     once gets all its listings' springs on its last slot (the HashMap
//     index), and the positions go out slot by slot, so the last slot wins;
//   * repulsion (:258-272): the reference walks pairs i < j and adds the pair
//     force to i and subtracts it from j, so gate j receives its terms in
//     partner order m = 0..n-1. Each thread owns one gate and adds, in that
//     order, f_jm = force * (p_j - p_m) / dist, which equals the reference's
//     "-= fx_ij" exactly (IEEE subtraction of t equals addition of -t, and the
//     products are sign-symmetric); sqrt and divisions are IEEE as in Rust;
//   * damped step with clamp to the leaf box (:275-280).
// Schedules: a group of T threads (T = 32, 64, 128 or 256) owns one leaf at a
// time, looping over gates when n > T; groups pull leaves (largest first)
// from an atomic work counter until the batch is done, running all
// iterations of a leaf in shared memory. The pair-triangle schedules (leaves
// of at most 128 gates, below) compute each pair's term once instead of once
// per gate. Every schedule gives identical results, so the autotuner is free
// to pick the fastest.
#include <algorithm>
#include <numeric>
#include <unordered_map>

#include <mutex>
#include <system_error>
#include <thread>

#include "fx_internal.h"

namespace fx {

constexpr int kLeafMax = 512;  // gates per leaf held in shared memory
constexpr int kLeafArrays = 6;  // x, y, vx, vy, fx, fy
constexpr int kPairUnroll = 4;  // partners whose repulsion terms are in flight at once

struct LeafBatch {
  const int32_t *gptr;     // [L+1] offsets into the gate list (leaf order)
  const int32_t *gate;     // [G] global gate ids; ~gate for a slot whose gate a
                           // later slot of the batch writes again
  const int32_t *aptr;     // [G+1] in-leaf adjacency row offsets
  const int16_t *aidx;     // in-leaf neighbour local indices (reference order)
  const float4 *region;    // [L] (cx, cy, w, h)
  const int32_t *order;    // [L] leaves in processing order
  int n_leaves;
  int iters;
  float k, repel, damping, dt;
  float *out_x, *out_y;    // global positions (written for leaf gates)
  unsigned int *counter;   // work counter
  float2 *trace;           // or null: each slot's total force of the first iteration
};

// The repulsion term of a pair from positions a and b (placer.rs:258-272):
// force * (a - b) / dist with dist = max(|a - b|, 0.1), force = repel / dist^2.
// IEEE: the reference's rounding steps (sqrt, three divisions), bit for bit.
// Fast (FX_LEAF_FAST): repel * (a - b) * rsqrt(max(d^2, 0.1^2))^3 with the
// hardware rsqrt, equal to f32 rounding.
template <bool Fast>
__device__ __forceinline__ float2 leaf_pair_force(float ax, float ay, float bx, float by,
                                                  float repel) {
  const float dx = __fsub_rn(ax, bx), dy = __fsub_rn(ay, by);
  if (Fast) {
    const float inv = rsqrtf(fmaxf(__fmaf_rn(dx, dx, __fmul_rn(dy, dy)), 0.1f * 0.1f));
    const float f = __fmul_rn(__fmul_rn(__fmul_rn(repel, inv), inv), inv);
    return make_float2(__fmul_rn(f, dx), __fmul_rn(f, dy));
  }
  const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  const float dist = fmaxf(__fsqrt_rn(d2), 0.1f);
  const float force = __fdiv_rn(repel, __fmul_rn(dist, dist));
  return make_float2(__fdiv_rn(__fmul_rn(force, dx), dist),
                     __fdiv_rn(__fmul_rn(force, dy), dist));
}

__device__ __forceinline__ float rclamp(float v, float lo, float hi) {
  if (v < lo) v = lo;
  if (v > hi) v = hi;
  return v;
}

// Barrier of one T-thread group: the warp, the whole block, or a named
// barrier (ids 1.. per group) for intermediate sizes.
template <int T>
__device__ __forceinline__ void group_sync(int id) {
  if (T == 32)
    __syncwarp();
  else if (T == 256)
    __syncthreads();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(T) : "memory");
}

// One leaf on a group of T threads (tid in [0, T)); sm: the group's shared
// arrays x, y, vx, vy, fx, fy (kLeafMax each).
template <int T, bool Fast>
__device__ void place_leaf(const LeafBatch &b, int leaf, int tid, float *sm, int sid) {
  float *sx = sm, *sy = sm + kLeafMax, *svx = sm + 2 * kLeafMax;
  float *svy = sm + 3 * kLeafMax, *sfx = sm + 4 * kLeafMax, *sfy = sm + 5 * kLeafMax;
  const int g0 = b.gptr[leaf];
  const int n = b.gptr[leaf + 1] - g0;
  if (n <= 0) return;
  const float4 r = b.region[leaf];
  const float half_w = r.z / 2.0f, half_h = r.w / 2.0f;
  const float min_x = __fsub_rn(r.x, half_w), min_y = __fsub_rn(r.y, half_h);
  const float max_x = __fadd_rn(min_x, r.z), max_y = __fadd_rn(min_y, r.w);
  const float nf = (float)n;
  for (int i = tid; i < n; i += T) {
    sx[i] = __fadd_rn(min_x, __fmul_rn(__fdiv_rn((float)i, nf), r.z));
    sy[i] = __fadd_rn(min_y, __fmul_rn(__fdiv_rn((float)((i * 7) % n), nf), r.w));
    svx[i] = 0.f;
    svy[i] = 0.f;
  }
  group_sync<T>(sid);
  for (int it = 0; it < b.iters; ++it) {
    for (int i = tid; i < n; i += T) {
      const float xi = sx[i], yi = sy[i];
      float ax = 0.f, ay = 0.f;
      const int a0 = b.aptr[g0 + i], a1 = b.aptr[g0 + i + 1];
      for (int e = a0; e < a1; ++e) {
        const int j = b.aidx[e];
        ax = __fadd_rn(ax, __fmul_rn(b.k, __fsub_rn(sx[j], xi)));
        ay = __fadd_rn(ay, __fmul_rn(b.k, __fsub_rn(sy[j], yi)));
      }
      // partners in order m = 0..n-1; four partners' terms are computed
      // independently (their sqrt and divisions overlap), then added in order
      int m = 0;
      for (; m + kPairUnroll <= n; m += kPairUnroll) {
        float tx[kPairUnroll], ty[kPairUnroll];
#pragma unroll
        for (int u = 0; u < kPairUnroll; ++u) {
          const float2 t = leaf_pair_force<Fast>(xi, yi, sx[m + u], sy[m + u], b.repel);
          tx[u] = t.x;
          ty[u] = t.y;
        }
#pragma unroll
        for (int u = 0; u < kPairUnroll; ++u)
          if (m + u != i) {
            ax = __fadd_rn(ax, tx[u]);
            ay = __fadd_rn(ay, ty[u]);
          }
      }
      for (; m < n; ++m) {
        if (m == i) continue;
        const float2 t = leaf_pair_force<Fast>(xi, yi, sx[m], sy[m], b.repel);
        ax = __fadd_rn(ax, t.x);
        ay = __fadd_rn(ay, t.y);
      }
      sfx[i] = ax;
      sfy[i] = ay;
      if (b.trace && it == 0) b.trace[g0 + i] = make_float2(ax, ay);
    }
    group_sync<T>(sid);
    for (int i = tid; i < n; i += T) {
      const float vx = __fmul_rn(__fadd_rn(svx[i], __fmul_rn(sfx[i], b.dt)), b.damping);
      const float vy = __fmul_rn(__fadd_rn(svy[i], __fmul_rn(sfy[i], b.dt)), b.damping);
      svx[i] = vx;
      svy[i] = vy;
      sx[i] = rclamp(__fadd_rn(sx[i], __fmul_rn(vx, b.dt)), min_x, max_x);
      sy[i] = rclamp(__fadd_rn(sy[i], __fmul_rn(vy, b.dt)), min_y, max_y);
    }
    group_sync<T>(sid);
  }
  for (int i = tid; i < n; i += T) {
    const int g = b.gate[g0 + i];  // ~gate: a later slot of the batch writes this gate
    if (g >= 0) {
      b.out_x[g] = sx[i];
      b.out_y[g] = sy[i];
    }
  }
  group_sync<T>(sid);
}

// T threads per leaf; the 256-thread block holds 256 / T groups.
template <int T, bool Fast>
__global__ void __launch_bounds__(256)
leaf_batch_kernel(LeafBatch b, int per_cluster_leaf) {
  extern __shared__ float lsm[];
  constexpr int kGroups = 256 / T;
  const int grp = threadIdx.x / T, tid = threadIdx.x % T;
  float *sm = lsm + grp * kLeafArrays * kLeafMax;
  const int sid = 1 + grp;
  if (per_cluster_leaf >= 0) {  // the one-launch-per-leaf baseline
    if (grp == 0) place_leaf<T, Fast>(b, per_cluster_leaf, tid, sm, sid);
    return;
  }
  __shared__ int next[kGroups];
  while (true) {
    if (tid == 0) {
      const unsigned int w = atomicAdd(b.counter, 1u);
      next[grp] = w < (unsigned)b.n_leaves ? b.order[w] : -1;
    }
    group_sync<T>(sid);
    const int leaf = next[grp];
    group_sync<T>(sid);
    if (leaf < 0) break;
    place_leaf<T, Fast>(b, leaf, tid, sm, sid);
  }
}

// ---------------------------------------------------------------------------
// Pair-triangle schedules (leaves of at most kPairMax gates). The reference's
// pair loop computes each pair's force once and applies it to both gates; so
// do these. Phase 1 spreads the n(n-1)/2 pair terms t(r, c) = force *
// (p_r - p_c) / dist (r < c) over every thread of the group; phase 2 has each
// gate add its terms in partner order m = 0..n-1: -t(m, j) for m < j (the
// reference's "-= f"), t(j, m) for m > j. The per-gate sums are unchanged, so
// the results are those of the other schedules bit for bit.
//
// The triangle is folded into a rectangle of U = n/2 rows of stride s:
// triangle row r < U sits at rect row r, columns c - r - 1; row r >= U at
// rect row n - 2 - r, column c (rows r and n-2-r together hold n entries).
// Phase 1 walks the rectangle in order (contiguous stores). In phase 2 the
// lanes of a warp read either one triangle row (contiguous) or one column
// (step s - 1 or -s): s is the least value >= n with s = 2 (mod 4), which
// keeps those reads to at most two wavefronts per half-warp.
constexpr int kPairMax = 128;
constexpr int kMidUnroll = 8;  // mixed-segment partners loaded ahead of their adds

__host__ __device__ __forceinline__ int pair_rows(int n) { return n >> 1; }
__host__ __device__ __forceinline__ int pair_stride(int n) { return ((n + 1) | 3) - 1; }

__host__ __device__ __forceinline__ size_t pair_smem_bytes(int nmax) {
  const size_t b = (size_t)pair_rows(nmax) * pair_stride(nmax) * sizeof(float2) +
                   (size_t)kLeafArrays * nmax * sizeof(float);
  return (b + 15) & ~(size_t)15;
}

// Barrier of a G-thread group: the whole block, or named barrier id (1, 2)
// of one half.
template <int G, int kBar>
__device__ __forceinline__ void pair_sync() {
  if (kBar == 0)
    __syncthreads();
  else
    asm volatile("bar.sync %0, %1;" ::"n"(kBar), "n"(G) : "memory");
}

// Repulsion term of the pair (r, c), r < c, from their positions.
template <bool Fast>
__device__ __forceinline__ float2 pair_term(float2 pr, float2 pc, float repel) {
  return leaf_pair_force<Fast>(pr.x, pr.y, pc.x, pc.y, repel);
}

// One leaf on a group of T threads (tid in [0, T); the block with kBar = 0,
// or one half of it with named barrier kBar). tri: the folded triangle; pos:
// positions (x, y) in two buffers of nmax float2 (double-buffered across
// iterations), then velocities (nmax float2).
template <int T, int kBar, bool Fast>
__device__ void place_leaf_pairs(const LeafBatch &b, int leaf, int nmax, float2 *tri,
                                 float *pos, int tid) {
  const int g0 = b.gptr[leaf];
  const int n = b.gptr[leaf + 1] - g0;
  if (n <= 0) return;
  float2 *xy = reinterpret_cast<float2 *>(pos);  // buffer p at xy + p nmax
  float2 *sv = xy + 2 * nmax;
  const float4 r4 = b.region[leaf];
  const float half_w = r4.z / 2.0f, half_h = r4.w / 2.0f;
  const float min_x = __fsub_rn(r4.x, half_w), min_y = __fsub_rn(r4.y, half_h);
  const float max_x = __fadd_rn(min_x, r4.z), max_y = __fadd_rn(min_y, r4.w);
  const float nf = (float)n;
  for (int i = tid; i < n; i += T) {
    xy[i] = make_float2(__fadd_rn(min_x, __fmul_rn(__fdiv_rn((float)i, nf), r4.z)),
                        __fadd_rn(min_y, __fmul_rn(__fdiv_rn((float)((i * 7) % n), nf), r4.w)));
    sv[i] = make_float2(0.f, 0.f);
  }
  const int U = pair_rows(n), s = pair_stride(n);
  const int npairs = n * (n - 1) / 2;
  const int qd = T / n, qm = T % n;    // rect (row, col) advance per stride of T
  const int dat = qd * s + qm;         // rect address advance (before a row wrap)
  const int u0 = tid / n, c0 = tid % n;
  pair_sync<T, kBar>();
  for (int it = 0; it < b.iters; ++it) {
    const float2 *sxy = xy + (it & 1) * nmax;
    float2 *nxy = xy + ((it & 1) ^ 1) * nmax;
    // attraction of the gates this thread owns (it reads only this
    // iteration's positions, so its load chain runs while every warp is busy
    // with phase 1); phase 2 continues these sums with the pair terms
    constexpr int kOwn = (kPairMax + T - 1) / T;
    float atx[kOwn], aty[kOwn];
#pragma unroll
    for (int g = 0; g < kOwn; ++g) {
      const int j = tid + g * T;
      float ax = 0.f, ay = 0.f;
      if (j < n) {
        const float2 pj = sxy[j];
        const int a0 = b.aptr[g0 + j], a1 = b.aptr[g0 + j + 1];
        for (int e = a0; e < a1; ++e) {
          const float2 po = sxy[b.aidx[e]];
          ax = __fadd_rn(ax, __fmul_rn(b.k, __fsub_rn(po.x, pj.x)));
          ay = __fadd_rn(ay, __fmul_rn(b.k, __fsub_rn(po.y, pj.y)));
        }
      }
      atx[g] = ax;
      aty[g] = ay;
    }
    // phase 1: pair terms, kPairUnroll rect entries per thread in flight.
    // Entry q = (u, col) = (q / n, q % n): c1 = u + 1 + col < n puts it in the
    // first segment (r = u, c = c1), else the second (r = n-2-u, c = col).
    // The n(n-1)/2 valid entries are exactly q < npairs (for even n the
    // unused half of the last rect row comes last). Whole batches of
    // kPairUnroll entries need no bounds test; the last partial one does.
    int u = u0, col = c0, at = u0 * s + c0;
    auto advance = [&]() {
      col += qm;
      u += qd;
      at += dat;
      if (col >= n) {
        col -= n;
        ++u;
        at += s - n;
      }
    };
    int q = tid;
    for (; q + (kPairUnroll - 1) * T < npairs; q += kPairUnroll * T) {
      float2 t[kPairUnroll];
      int at_k[kPairUnroll];
#pragma unroll
      for (int k = 0; k < kPairUnroll; ++k) {
        const int c1 = u + 1 + col;
        const bool first = c1 < n;
        at_k[k] = at;
        t[k] = pair_term<Fast>(sxy[first ? u : n - 2 - u], sxy[first ? c1 : col], b.repel);
        advance();
      }
#pragma unroll
      for (int k = 0; k < kPairUnroll; ++k) tri[at_k[k]] = t[k];
    }
    for (; q < npairs; q += T) {
      const int c1 = u + 1 + col;
      const bool first = c1 < n;
      tri[at] = pair_term<Fast>(sxy[first ? u : n - 2 - u], sxy[first ? c1 : col], b.repel);
      advance();
    }
    pair_sync<T, kBar>();
    // phase 2: the pair terms in partner order after the attraction; damped step
#pragma unroll
    for (int g = 0; g < kOwn; ++g) {
      const int j = tid + g * T;
      if (j >= n) break;
      const float2 pj = sxy[j];
      float ax = atx[g], ay = aty[g];
      // Partner m < j adds -t(m, j) (row m), m > j adds t(j, m) (row j);
      // a + (-t) is a - t. The warp's gates are w..w+31, so partners below w
      // are column reads for every lane (A: rows < U, address step s - 1;
      // B: rows >= U, step -s), partners from w + 32 on are row reads (D,
      // step 1), and only the 32 partners in between (C) need per-lane code.
      const int w = j - (tid & 31);
      const int eA = min(w, U);
      {
        const float2 *p = tri + (j - 1);
        const int st = s - 1;
        int m = 0;
#pragma unroll 8
        for (; m < eA; ++m, p += st) {
          const float2 v = *p;
          ax = __fsub_rn(ax, v.x);
          ay = __fsub_rn(ay, v.y);
        }
      }
      {
        const float2 *p = tri + ((n - 2 - U) * s + j);
#pragma unroll 8
        for (int m = U; m < w; ++m, p -= s) {
          const float2 v = *p;
          ax = __fsub_rn(ax, v.x);
          ay = __fsub_rn(ay, v.y);
        }
      }
      const int rowbase = j < U ? j * s - j - 1 : (n - 2 - j) * s;
      const int eC = min(w + 32, n);
      for (int m = w; m < eC; m += kMidUnroll) {  // loads ahead, exact sign flips
        float2 v[kMidUnroll];
        unsigned int neg[kMidUnroll];
        bool use[kMidUnroll];
#pragma unroll
        for (int k = 0; k < kMidUnroll; ++k) {
          const int mm = m + k;
          use[k] = mm < eC && mm != j;
          const int ca = mm < U ? mm * (s - 1) + j - 1 : (n - 2 - mm) * s + j;
          neg[k] = mm < j ? 0x80000000u : 0u;
          v[k] = tri[use[k] ? (mm < j ? ca : rowbase + mm) : 0];
        }
#pragma unroll
        for (int k = 0; k < kMidUnroll; ++k)
          if (use[k]) {
            ax = __fadd_rn(ax, __uint_as_float(__float_as_uint(v[k].x) ^ neg[k]));
            ay = __fadd_rn(ay, __uint_as_float(__float_as_uint(v[k].y) ^ neg[k]));
          }
      }
      {
        const float2 *p = tri + rowbase;
#pragma unroll 8
        for (int m = eC; m < n; ++m) {
          const float2 v = p[m];
          ax = __fadd_rn(ax, v.x);
          ay = __fadd_rn(ay, v.y);
        }
      }
      if (b.trace && it == 0) b.trace[g0 + j] = make_float2(ax, ay);
      const float2 v0 = sv[j];
      const float vx = __fmul_rn(__fadd_rn(v0.x, __fmul_rn(ax, b.dt)), b.damping);
      const float vy = __fmul_rn(__fadd_rn(v0.y, __fmul_rn(ay, b.dt)), b.damping);
      sv[j] = make_float2(vx, vy);
      nxy[j] = make_float2(rclamp(__fadd_rn(pj.x, __fmul_rn(vx, b.dt)), min_x, max_x),
                           rclamp(__fadd_rn(pj.y, __fmul_rn(vy, b.dt)), min_y, max_y));
    }
    pair_sync<T, kBar>();
  }
  const float2 *fxy = xy + (b.iters & 1) * nmax;
  for (int i = tid; i < n; i += T) {
    const int g = b.gate[g0 + i];  // ~gate: a later slot of the batch writes this gate
    if (g >= 0) {
      const float2 f = fxy[i];
      b.out_x[g] = f.x;
      b.out_y[g] = f.y;
    }
  }
}

// One half of a block: leaves order[split..) from counter[1], named barrier kBar.
template <int H, int kBar, bool Fast>
__device__ __forceinline__ void half_loop(const LeafBatch &b, int split, int nhalf, float2 *tri,
                                          float *pos, int ht, int *next) {
  while (true) {
    if (ht == 0) {
      const unsigned int w = atomicAdd(&b.counter[1], 1u);
      *next = (unsigned)split + w < (unsigned)b.n_leaves ? b.order[split + w] : -1;
    }
    pair_sync<H, kBar>();
    const int leaf = *next;
    pair_sync<H, kBar>();
    if (leaf < 0) break;
    place_leaf_pairs<H, kBar, Fast>(b, leaf, nhalf, tri, pos, ht);
  }
}

// T-thread blocks pull leaves largest-first from counter[0] while they are
// larger than nhalf; then each half of the block (T/2 threads, its own named
// barrier and half of the shared memory) pulls the remaining leaves from
// counter[1]. Two leaves of at most nhalf gates fit where one of nmax does,
// so the smaller leaves run twice as many to an SM.
template <int T, bool Fast>
__global__ void __launch_bounds__(T, 3)
leaf_pairs_kernel(LeafBatch b, int nmax, int split, int nhalf) {
  extern __shared__ float4 lpair[];
  __shared__ int next[2];
  {
    float2 *tri = reinterpret_cast<float2 *>(lpair);
    float *pos = reinterpret_cast<float *>(tri + (size_t)pair_rows(nmax) * pair_stride(nmax));
    while (true) {
      if (threadIdx.x == 0) {
        const unsigned int w = atomicAdd(&b.counter[0], 1u);
        next[0] = w < (unsigned)split ? b.order[w] : -1;
      }
      __syncthreads();
      const int leaf = next[0];
      __syncthreads();
      if (leaf < 0) break;
      place_leaf_pairs<T, 0, Fast>(b, leaf, nmax, tri, pos, threadIdx.x);
    }
  }
  if (split >= b.n_leaves) return;
  constexpr int H = T / 2;
  const int h = threadIdx.x / H, ht = threadIdx.x % H;
  float2 *tri = reinterpret_cast<float2 *>(reinterpret_cast<char *>(lpair) +
                                           h * pair_smem_bytes(nhalf));
  float *pos = reinterpret_cast<float *>(tri + (size_t)pair_rows(nhalf) * pair_stride(nhalf));
  if (h == 0)
    half_loop<H, 1, Fast>(b, split, nhalf, tri, pos, ht, next);
  else
    half_loop<H, 2, Fast>(b, split, nhalf, tri, pos, ht, next + 1);
}

// The batch's split for leaf_pairs_kernel: the largest nhalf whose two slots
// fit in one nmax slot, and the number of leaves (largest first) above it.
struct PairPlan {
  int nmax, nhalf, split;
};

static PairPlan pair_plan(int n_leaves, const int32_t *leaf_ptr, const std::vector<int32_t> &order) {
  PairPlan p;
  p.nmax = 1;
  for (int l = 0; l < n_leaves; ++l) p.nmax = std::max(p.nmax, leaf_ptr[l + 1] - leaf_ptr[l]);
  const size_t whole = pair_smem_bytes(p.nmax);
  p.nhalf = p.nmax;
  while (p.nhalf > 0 && 2 * pair_smem_bytes(p.nhalf) > whole) --p.nhalf;
  p.split = 0;
  while (p.split < n_leaves &&
         leaf_ptr[order[p.split] + 1] - leaf_ptr[order[p.split]] > p.nhalf)
    ++p.split;
  if (p.nhalf < 1) p.split = n_leaves;
  return p;
}

template <int T, bool Fast>
static int launch_pairs(fx_ctx *ctx, const LeafBatch &b, const PairPlan &plan, cudaStream_t s) {
  if (plan.nmax > kPairMax) {
    set_error("pair schedules take leaves of at most %d gates (largest: %d)", kPairMax,
              plan.nmax);
    return FX_EINVAL;
  }
  const size_t smem = pair_smem_bytes(plan.nmax);
  FX_TRY(raise_smem_limit(reinterpret_cast<const void *>(leaf_pairs_kernel<T, Fast>),
                          (int)smem));
  int per_sm = 0;
  FX_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, leaf_pairs_kernel<T, Fast>, T, smem));
  if (per_sm < 1) per_sm = 1;
  int grid = (ctx->persistent_sms > 0 ? ctx->persistent_sms : ctx->num_sms) * per_sm;
  if (grid > b.n_leaves) grid = b.n_leaves;
  if (grid < 1) grid = 1;
  FX_CHECK_CUDA(cudaMemsetAsync(b.counter, 0, 8, s));
  leaf_pairs_kernel<T, Fast><<<grid, T, smem, s>>>(b, plan.nmax, plan.split, plan.nhalf);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

// Host-side leaf structures: in-leaf adjacency in the reference's order and
// a largest-first processing order.
struct LeafHost {
  std::vector<int32_t> aptr;
  std::vector<int16_t> aidx;
  std::vector<int32_t> order;
};

// In-leaf adjacency of leaves [l0, l1) into aptr (counts relative to the
// range's first entry) and out; local: a -1-filled gate map of d->n entries,
// left -1-filled.
static void leaf_adjacency(const fx_design *d, int l0, int l1, const int32_t *leaf_ptr,
                           const int32_t *leaf_gate, std::vector<int32_t> &local,
                           int32_t *aptr, std::vector<int16_t> &out) {
  for (int l = l0; l < l1; ++l) {
    const int32_t b = leaf_ptr[l], e = leaf_ptr[l + 1];
    bool repeats = false;
    for (int32_t i = b; i < e; ++i) {
      const int32_t g = leaf_gate[i];
      repeats |= local[g] >= 0;
      local[g] = i - b;  // HashMap insert: a repeated gate keeps the last slot
    }
    for (int32_t i = b; i < e; ++i) {
      const int32_t g = leaf_gate[i];
      // The reference adds every listing's springs to the gate's mapped
      // (last) slot, in slot order: that slot's row is the neighbour list
      // once per listing, the gate's other slots have none.
      int32_t reps = 1;
      if (repeats) {
        reps = 0;
        if (local[g] == i - b)
          for (int32_t k = b; k <= i; ++k) reps += leaf_gate[k] == g;
      }
      for (int32_t r = 0; r < reps; ++r)
        for (int32_t q = d->h_adj_ptr[g]; q < d->h_adj_ptr[g + 1]; ++q) {
          const int32_t j = d->h_adj_idx[q];
          if (local[j] >= 0) out.push_back((int16_t)local[j]);
        }
      aptr[(size_t)i + 1] = (int32_t)out.size();
    }
    for (int32_t i = b; i < e; ++i) local[leaf_gate[i]] = -1;
  }
}

static int build_leaf_host(const fx_design *d, int L, const int32_t *leaf_ptr,
                           const int32_t *leaf_gate, LeafHost &h) {
  const int32_t G = leaf_ptr[L];
  for (int l = 0; l < L; ++l)
    if (leaf_ptr[l + 1] - leaf_ptr[l] > kLeafMax) {
      set_error("leaf %d has %d gates (limit %d)", l, leaf_ptr[l + 1] - leaf_ptr[l], kLeafMax);
      return FX_EINVAL;
    }
  for (int32_t i = 0; i < G; ++i)
    if (leaf_gate[i] < 0 || leaf_gate[i] >= d->n) {
      set_error("leaf gate %d out of range", leaf_gate[i]);
      return FX_EINVAL;
    }
  h.aptr.assign((size_t)G + 1, 0);
  h.aidx.clear();
  // Leaves are independent: large batches split them over host threads in
  // ranges of about equal gate counts, then join the ranges in leaf order.
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = G >= 65536 ? (int)std::min<unsigned>(std::min(hw, 16u), (unsigned)L) : 1;
  if (nt <= 1) {
    std::vector<int32_t> local((size_t)d->n, -1);
    leaf_adjacency(d, 0, L, leaf_ptr, leaf_gate, local, h.aptr.data(), h.aidx);
  } else {
    std::vector<int> cut(nt + 1, L);
    cut[0] = 0;
    for (int t = 1, l = 0; t < nt; ++t) {
      const int64_t target = (int64_t)G * t / nt;
      while (l < L && leaf_ptr[l] < target) ++l;
      cut[t] = l;
    }
    std::vector<std::vector<int16_t>> part(nt);
    auto range = [&](int t) {
      std::vector<int32_t> local((size_t)d->n, -1);
      leaf_adjacency(d, cut[t], cut[t + 1], leaf_ptr, leaf_gate, local, h.aptr.data(), part[t]);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) {
      try {
        pool.emplace_back(range, t);
      } catch (const std::system_error &) {
        range(t);  // no thread to be had: do this range here
      }
    }
    range(0);
    for (auto &th : pool) th.join();
    size_t off = 0;
    for (int t = 0; t < nt; ++t) {
      for (int32_t i = leaf_ptr[cut[t]]; i < leaf_ptr[cut[t + 1]]; ++i)
        h.aptr[(size_t)i + 1] += (int32_t)off;
      off += part[t].size();
    }
    h.aidx.reserve(off);
    for (auto &p : part) h.aidx.insert(h.aidx.end(), p.begin(), p.end());
  }
  h.order.resize(L);
  std::iota(h.order.begin(), h.order.end(), 0);
  std::stable_sort(h.order.begin(), h.order.end(), [&](int a, int c) {
    return leaf_ptr[a + 1] - leaf_ptr[a] > leaf_ptr[c + 1] - leaf_ptr[c];
  });
  return FX_OK;
}

template <int T, bool Fast>
static int launch_leaf(fx_ctx *ctx, const LeafBatch &b, bool per_cluster,
                       cudaStream_t s) {
  constexpr int kGroups = 256 / T;
  const size_t smem = (size_t)kGroups * kLeafArrays * kLeafMax * sizeof(float);
  FX_TRY(raise_smem_limit(reinterpret_cast<const void *>(leaf_batch_kernel<T, Fast>),
                          (int)smem));
  if (per_cluster) {
    for (int l = 0; l < b.n_leaves; ++l)
      leaf_batch_kernel<T, Fast><<<1, 256, smem, s>>>(b, l);
    FX_CHECK_LAUNCH();
    ctx->launches += b.n_leaves;
    return FX_OK;
  }
  int per_sm = 0;
  FX_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, leaf_batch_kernel<T, Fast>, 256, smem));
  if (per_sm < 1) per_sm = 1;
  int grid = (ctx->persistent_sms > 0 ? ctx->persistent_sms : ctx->num_sms) * per_sm;
  const int need = (b.n_leaves + kGroups - 1) / kGroups;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  FX_CHECK_CUDA(cudaMemsetAsync(b.counter, 0, 4, s));
  leaf_batch_kernel<T, Fast><<<grid, 256, smem, s>>>(b, -1);
  FX_CHECK_LAUNCH();
  ctx->launches += 1;
  return FX_OK;
}

template <bool Fast>
static int run_schedule_p(fx_ctx *ctx, const LeafBatch &b, int schedule, const PairPlan &plan,
                          cudaStream_t s) {
  switch (schedule) {
    case FX_LEAF_PAIR64: return launch_pairs<64, Fast>(ctx, b, plan, s);
    case FX_LEAF_PAIR128: return launch_pairs<128, Fast>(ctx, b, plan, s);
    case FX_LEAF_PAIR256: return launch_pairs<256, Fast>(ctx, b, plan, s);
    case FX_LEAF_WARP: return launch_leaf<32, Fast>(ctx, b, false, s);
    case FX_LEAF_CTA64: return launch_leaf<64, Fast>(ctx, b, false, s);
    case FX_LEAF_CTA128: return launch_leaf<128, Fast>(ctx, b, false, s);
    case FX_LEAF_CTA256: return launch_leaf<256, Fast>(ctx, b, false, s);
    case FX_LEAF_PER_CLUSTER: return launch_leaf<128, Fast>(ctx, b, true, s);
  }
  set_error("unknown leaf schedule %d", schedule);
  return FX_EINVAL;
}

static int run_schedule(fx_ctx *ctx, const LeafBatch &b, int schedule, const PairPlan &plan,
                        bool fast, cudaStream_t s) {
  return fast ? run_schedule_p<true>(ctx, b, schedule, plan, s)
              : run_schedule_p<false>(ctx, b, schedule, plan, s);
}

}  // namespace fx

using namespace fx;

extern "C" int fx_leaf_cfg_default(fx_leaf_cfg *c) {
  if (!c) return FX_EINVAL;
  c->force_iterations = 50;
  c->attract_weight = 1.0f;
  c->repel_weight = 0.5f;
  c->damping = 0.9f;
  c->dt = 0.1f;
  c->schedule = FX_LEAF_AUTO;
  c->precision = FX_LEAF_IEEE;
  c->reserved1 = 0;
  return FX_OK;
}

extern "C" int fx_hapr_place_leaves(fx_ctx *ctx, fx_design *d, int32_t n_leaves,
                                    const int32_t *leaf_ptr, const int32_t *leaf_gate,
                                    const float *region, const fx_leaf_cfg *cfg,
                                    float *out_x, float *out_y, int32_t *out_schedule) {
  if (!ctx || !d || n_leaves < 0 || (n_leaves > 0 && (!leaf_ptr || !leaf_gate || !region)) ||
      !cfg || !out_x || !out_y || cfg->force_iterations < 0 ||
      (cfg->precision != FX_LEAF_IEEE && cfg->precision != FX_LEAF_FAST)) {
    set_error("fx_hapr_place_leaves: invalid arguments");
    return FX_EINVAL;
  }
  const bool fast = cfg->precision == FX_LEAF_FAST;
  if (n_leaves == 0) return FX_OK;
  if (leaf_ptr[0] != 0) {
    set_error("fx_hapr_place_leaves: leaf_ptr[0] must be 0");
    return FX_EINVAL;
  }
  for (int l = 0; l < n_leaves; ++l)
    if (leaf_ptr[l + 1] < leaf_ptr[l]) {
      set_error("fx_hapr_place_leaves: leaf_ptr decreases at %d", l);
      return FX_EINVAL;
    }
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream;
  LeafHost h;
  FX_TRY(build_leaf_host(d, n_leaves, leaf_ptr, leaf_gate, h));
  const int32_t G = leaf_ptr[n_leaves];
  const PairPlan plan = pair_plan(n_leaves, leaf_ptr, h.order);
  DevBuf<int32_t> gptr, gate, aptr, order;
  DevBuf<int16_t> aidx;
  DevBuf<float4> reg;
  DevBuf<float> ox, oy;
  DevBuf<unsigned int> counter;
  FX_TRY(gptr.alloc((size_t)n_leaves + 1));
  FX_TRY(gate.alloc(G > 0 ? (size_t)G : 1));
  FX_TRY(aptr.alloc((size_t)G + 1));
  FX_TRY(aidx.alloc(h.aidx.empty() ? 1 : h.aidx.size()));
  FX_TRY(order.alloc((size_t)n_leaves));
  FX_TRY(reg.alloc((size_t)n_leaves));
  FX_TRY(ox.alloc((size_t)d->n));
  FX_TRY(oy.alloc((size_t)d->n));
  FX_TRY(counter.alloc(2));
  auto up = [&](void *dst, const void *src, size_t bytes) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
  };
  FX_CHECK_CUDA(up(gptr.p, leaf_ptr, ((size_t)n_leaves + 1) * 4));
  // The reference writes the positions slot by slot, leaf by leaf, so a gate
  // listed more than once keeps its last slot's position. The kernels write
  // concurrently: every slot but a gate's last goes up as ~gate and skips
  // the write. Batches without repeats go up unchanged.
  std::vector<int32_t> gate_last;
  {
    std::vector<uint8_t> seen((size_t)d->n, 0);
    for (int32_t i = G - 1; i >= 0; --i) {
      const int32_t g = leaf_gate[i];
      if (seen[g]) {
        if (gate_last.empty()) gate_last.assign(leaf_gate, leaf_gate + G);
        gate_last[i] = ~g;
      }
      seen[g] = 1;
    }
  }
  FX_CHECK_CUDA(up(gate.p, gate_last.empty() ? leaf_gate : gate_last.data(), (size_t)G * 4));
  FX_CHECK_CUDA(up(aptr.p, h.aptr.data(), h.aptr.size() * 4));
  FX_CHECK_CUDA(up(aidx.p, h.aidx.data(), h.aidx.size() * 2));
  FX_CHECK_CUDA(up(order.p, h.order.data(), h.order.size() * 4));
  FX_CHECK_CUDA(up(reg.p, region, (size_t)n_leaves * 16));
  FX_CHECK_CUDA(up(ox.p, out_x, (size_t)d->n * 4));
  FX_CHECK_CUDA(up(oy.p, out_y, (size_t)d->n * 4));
  if (d->trace_on) {
    FX_TRY(d->leaf_trace.alloc(G > 0 ? (size_t)G : 1));
    FX_CHECK_CUDA(cudaMemsetAsync(d->leaf_trace.p, 0, (size_t)std::max(G, 1) * 8, s));
    d->leaf_trace_n = G;
  }
  LeafBatch b{gptr.p, gate.p, aptr.p, aidx.p, reg.p, order.p, n_leaves,
              cfg->force_iterations, cfg->attract_weight, cfg->repel_weight,
              cfg->damping, cfg->dt, ox.p, oy.p, counter.p,
              d->trace_on ? d->leaf_trace.p : nullptr};
  int schedule = cfg->schedule;
  bool done = false;
  auto lg2 = [](int64_t v) {
    int b = 0;
    while (v > 1) {
      v >>= 1;
      ++b;
    }
    return b;
  };
  const uint32_t shape = (uint32_t)lg2(n_leaves) | ((uint32_t)lg2(G / std::max(1, n_leaves)) << 8) |
                         ((uint32_t)lg2(cfg->force_iterations) << 16) |
                         ((uint32_t)fast << 24);
  if (schedule == FX_LEAF_AUTO) {
    auto it = ctx->leaf_tuned.find(shape);
    if (it != ctx->leaf_tuned.end()) schedule = it->second;
  }
  if (schedule == FX_LEAF_AUTO) {
    // Autotune: time each schedule once on this batch (results are identical,
    // so the last run's output stands) and keep the fastest for batches of
    // this shape on this context.
    float best = 1e30f;
    int best_s = FX_LEAF_CTA128;
    cudaEvent_t e0, e1;
    FX_CHECK_CUDA(cudaEventCreate(&e0));
    FX_CHECK_CUDA(cudaEventCreate(&e1));
    for (int sc : {FX_LEAF_WARP, FX_LEAF_CTA64, FX_LEAF_CTA128, FX_LEAF_CTA256,
                   FX_LEAF_PAIR64, FX_LEAF_PAIR128, FX_LEAF_PAIR256}) {
      if (sc >= FX_LEAF_PAIR64 && plan.nmax > kPairMax) continue;
      FX_CHECK_CUDA(cudaEventRecord(e0, s));
      int rc = run_schedule(ctx, b, sc, plan, fast, s);
      if (rc != FX_OK) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
      }
      FX_CHECK_CUDA(cudaEventRecord(e1, s));
      FX_CHECK_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      FX_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) {
        best = ms;
        best_s = sc;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->leaf_tuned[shape] = best_s;
    schedule = best_s;
    done = true;
  }
  ctx->leaf_schedule = schedule;
  if (!done) {
    cudaEvent_t ev;
    timer_begin(ctx, FX_STAGE_LEAF, s, &ev);
    FX_TRY(run_schedule(ctx, b, schedule, plan, fast, s));
    timer_end(ctx, FX_STAGE_LEAF, s, ev);
  }
  FX_CHECK_CUDA(cudaMemcpyAsync(out_x, ox.p, (size_t)d->n * 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(out_y, oy.p, (size_t)d->n * 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (out_schedule) *out_schedule = schedule;
  for (auto *p : {&gptr, &gate, &aptr, &order}) p->release();
  aidx.release();
  reg.release();
  ox.release();
  oy.release();
  counter.release();
  return FX_OK;
}

extern "C" int fx_design_leaf_trace_get(fx_design *d, float *out_fx, float *out_fy) {
  if (!d || !d->ctx) return FX_EINVAL;
  if (!d->leaf_trace.p || d->leaf_trace_n <= 0) {
    set_error("fx_design_leaf_trace_get: no traced leaf batch (enable fx_design_trace, "
              "then run fx_hapr_place_leaves)");
    return FX_EINVAL;
  }
  fx_ctx *ctx = d->ctx;
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  std::vector<float2> t((size_t)d->leaf_trace_n);
  FX_CHECK_CUDA(cudaMemcpyAsync(t.data(), d->leaf_trace.p, t.size() * 8,
                                cudaMemcpyDeviceToHost, ctx->stream));
  FX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  for (size_t i = 0; i < t.size(); ++i) {
    if (out_fx) out_fx[i] = t[i].x;
    if (out_fy) out_fy[i] = t[i].y;
  }
  return FX_OK;
}
