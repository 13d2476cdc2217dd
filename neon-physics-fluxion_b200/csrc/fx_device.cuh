// fx_device.cuh -- small device helpers shared by the kernels.
#pragma once
#include <cfloat>
#include <cstdint>

namespace fx {

__device__ __forceinline__ int lin_tid() {
  return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
__device__ __forceinline__ int block_threads() {
  return blockDim.x * blockDim.y * blockDim.z;
}

// Rust's `(v / cell) as usize` followed by `.min(n - 1)` (grid.rs:58-62):
// IEEE f32 division, truncation toward zero, NaN and negatives saturate to 0,
// large values (and +inf) clamp to n - 1. `cell` is the f32 cell size.
__device__ __forceinline__ int cell_at(float v, float cell, int n) {
  const float q = __fdiv_rn(v, cell);
  if (!(q >= 1.0f)) return 0;
  if (q >= (float)n) return n - 1;
  const int c = (int)q;
  return c < n - 1 ? c : n - 1;
}

// Deterministic block reductions (fixed shuffle tree, fixed warp order).
// Every thread of the block must call them; the result is valid everywhere.
__device__ __forceinline__ double block_sum_double(double v) {
  __shared__ double ws[32];
  __shared__ double total;
  const int t = lin_tid(), lane = t & 31, w = t >> 5;
  const int nw = (block_threads() + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    double u = lane < nw ? ws[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) u += __shfl_down_sync(0xffffffffu, u, o);
    if (lane == 0) total = u;
  }
  __syncthreads();
  return total;
}

__device__ __forceinline__ float block_max_float(float v) {
  __shared__ float ws[32];
  __shared__ float total;
  const int t = lin_tid(), lane = t & 31, w = t >> 5;
  const int nw = (block_threads() + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    float u = lane < nw ? ws[lane] : -FLT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) u = fmaxf(u, __shfl_down_sync(0xffffffffu, u, o));
    if (lane == 0) total = u;
  }
  __syncthreads();
  return total;
}

// Cross-block FP64 sum in a fixed order: each block stores its partial, the
// last block to finish adds all partials (same order every run) into
// *result and re-arms the counter.
__device__ __forceinline__ void last_block_sum(double block_value,
                                               double *partial,
                                               unsigned int *done,
                                               double *result) {
  __shared__ bool last;
  const int t = lin_tid();
  if (t == 0) {
    partial[blockIdx.x] = block_value;
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double a = 0.0;
  for (int i = t; i < (int)gridDim.x; i += block_threads())
    a += ((volatile double *)partial)[i];
  a = block_sum_double(a);
  if (t == 0) {
    *result = a;
    *done = 0;
  }
}

// Global adds whose old value is not needed, issued as reductions: the warp
// does not wait for the L2 round trip of an atomic that returns a value.
__device__ __forceinline__ void red_add_global(int *p, int v) {
  asm volatile("red.relaxed.gpu.global.add.s32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)),
               "r"(v)
               : "memory");
}
__device__ __forceinline__ void red_add_global(unsigned long long *p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)),
               "l"(v)
               : "memory");
}

// Warp-aggregated atomic adds: lanes naming the same element (idx >= 0) are
// combined and one lane issues the atomic. Every lane of the warp must call
// these (idx < 0 = nothing to add); base is global memory. Sums of integers
// are exact, so the result does not depend on the grouping.
__device__ __forceinline__ void agg_add_u64(unsigned long long *base, long long idx,
                                            unsigned long long v) {
  const unsigned lane = threadIdx.x & 31u;
  // indexes fit 31 bits (density bins: G^2 <= 8192^2): a 32-bit match
  const unsigned peers = __match_any_sync(0xffffffffu, (int)idx);
  const bool alone = __all_sync(0xffffffffu, peers == (1u << lane));
  if (alone) {
    if (idx >= 0) red_add_global(base + idx, v);
    return;
  }
  unsigned long long sum = 0;
#pragma unroll
  for (int src = 0; src < 32; ++src) {
    const unsigned long long w = __shfl_sync(0xffffffffu, v, src);
    if ((peers >> src) & 1u) sum += w;
  }
  if (idx >= 0 && lane == (unsigned)(__ffs(peers) - 1)) red_add_global(base + idx, sum);
}

// Adds the same constant `v` from every lane naming idx (>= 0).
__device__ __forceinline__ void agg_add_const_i32(int *base, long long idx, int v) {
  const unsigned lane = threadIdx.x & 31u;
  // indexes fit 31 bits: a 32-bit match is the cheaper instruction
  const unsigned peers = __match_any_sync(0xffffffffu, (int)idx);
  if (idx >= 0 && lane == (unsigned)(__ffs(peers) - 1))
    red_add_global(base + idx, v * __popc(peers));
}

// Order-preserving float <-> uint mapping for atomicMin/atomicMax.
__device__ __forceinline__ unsigned int f2ord(float f) {
  const unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned int u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

}  // namespace fx
