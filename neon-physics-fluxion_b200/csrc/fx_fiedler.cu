// fx_fiedler.cu -- row G: batched power iteration on the induced Laplacians
// of many clusters at once (compute_fiedler_vector, H/src/algorithm/
// partitioner.rs:106-185).
//
// For every cluster (a gate subset, e.g. all clusters of one hierarchy
// level) the reference builds the induced subgraph Laplacian (degree = number
// of in-cluster adjacency entries, :124-137), starts from
// v_i = sin(i * 2.71828) normalised (:145-155) and repeats
//   lv = deg * v - A v ; lv -= mean(lv) ; lv /= |lv| if |lv| > 1e-10
// (:157-182). Here all clusters advance together:
//   * the SpMV keeps the reference's f32 order per row (deg*v, then minus
//     each in-cluster neighbour in adjacency order);
//   * one warp per chunk of <= 4096 rows accumulates, in FP64, sum(lv),
//     sum(lv^2) and v.lv (the Rayleigh quotient of the normalised v), then
//     one thread per cluster adds its chunks in order: the reductions are
//     deterministic. mean and |lv - mean|^2 = sum(lv^2) - n mean^2 come from
//     the same pass (1^T L v = 0, so there is no cancellation);
//   * the update subtracts the f32 mean and divides by the f32 norm.
// With tol > 0 a cluster stops once its Rayleigh quotient changes by at most
// tol (relative) between iterations; with tol = 0 it runs exactly max_iters
// iterations, as the reference's fixed 30 (H/src/main.rs:80).
#include <cmath>

#include "fx_internal.h"

namespace fx {

constexpr int kRowChunk = 4096;

struct FiedlerArgs {
  const int32_t *rptr, *ridx;  // in-cluster adjacency by position
  const float *deg;
  float *v, *lv;
  const int32_t *chunk_start;  // [K+1]
  const int32_t *chunk_cluster;
  const int32_t *cl_ptr;       // positions of cluster c: [cl_ptr[c], cl_ptr[c+1])
  const int32_t *cl_chunk;     // chunks of cluster c: [cl_chunk[c], cl_chunk[c+1])
  double *part;                // [3K]
  float *mean, *inv;           // per cluster: f32 mean and norm (0 = no divide)
  double *lambda;
  int32_t *active;             // per cluster
  int32_t *iters;
  int n_chunks, n_clusters;
  double tol;
};

__global__ void fiedler_spmv_kernel(FiedlerArgs a) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= a.n_chunks) return;
  const int c = a.chunk_cluster[warp];
  if (!a.active[c]) return;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int p = a.chunk_start[warp] + lane; p < a.chunk_start[warp + 1]; p += 32) {
    const float vp = a.v[p];
    float l = __fmul_rn(a.deg[p], vp);
    for (int e = a.rptr[p]; e < a.rptr[p + 1]; ++e) l = __fsub_rn(l, a.v[a.ridx[e]]);
    a.lv[p] = l;
    s1 += (double)l;
    s2 += (double)l * (double)l;
    s3 += (double)vp * (double)l;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
    s3 += __shfl_down_sync(0xffffffffu, s3, o);
  }
  if (lane == 0) {
    a.part[3 * warp] = s1;
    a.part[3 * warp + 1] = s2;
    a.part[3 * warp + 2] = s3;
  }
}

__global__ void fiedler_stats_kernel(FiedlerArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n_clusters || !a.active[c]) return;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int k = a.cl_chunk[c]; k < a.cl_chunk[c + 1]; ++k) {
    s1 += a.part[3 * k];
    s2 += a.part[3 * k + 1];
    s3 += a.part[3 * k + 2];
  }
  const double n = (double)(a.cl_ptr[c + 1] - a.cl_ptr[c]);
  const double mean = s1 / n;
  const double var = fmax(s2 - s1 * mean, 0.0);
  const double norm = sqrt(var);
  a.mean[c] = (float)mean;
  a.inv[c] = norm > 1e-10 ? (float)norm : 0.0f;
  const double prev = a.lambda[c];
  a.lambda[c] = s3;
  a.iters[c] += 1;
  if (a.tol > 0.0 && a.iters[c] > 1 && fabs(s3 - prev) <= a.tol * fabs(s3))
    a.active[c] = 2;  // converged: this update is the last
}

__global__ void fiedler_update_kernel(FiedlerArgs a, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  // position -> cluster by binary search over cl_ptr
  int lo = 0, hi = a.n_clusters - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.cl_ptr[mid] <= p) lo = mid; else hi = mid - 1;
  }
  if (!a.active[lo]) return;
  float x = __fsub_rn(a.lv[p], a.mean[lo]);
  const float nr = a.inv[lo];
  if (nr > 0.0f) x = __fdiv_rn(x, nr);
  a.v[p] = x;
}

// Exact mode (tol == 0): v = lv / norm, lv already deflated in place by
// part_seq_kernel (the reference's f32 folds), or lv when norm <= 1e-10.
__global__ void fiedler_div_kernel(FiedlerArgs a, const float *__restrict__ nrm, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int lo = 0, hi = a.n_clusters - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.cl_ptr[mid] <= p) lo = mid; else hi = mid - 1;
  }
  const float r = nrm[lo];
  a.v[p] = r > 0.0f ? __fdiv_rn(a.lv[p], r) : a.lv[p];
}

// v . L v (FP64, chunk partials of the last SpMV added in order) of the
// returned vectors; the host divides by v . v.
__global__ void fiedler_lambda_kernel(FiedlerArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n_clusters) return;
  double s3 = 0.0;
  for (int k = a.cl_chunk[c]; k < a.cl_chunk[c + 1]; ++k) s3 += a.part[3 * k + 2];
  a.lambda[c] = s3;
}

__global__ void fiedler_retire_kernel(int32_t *active, int n_clusters, int last) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_clusters) return;
  if (active[c] == 2 || last) active[c] = 0;
}

}  // namespace fx

using namespace fx;

extern "C" int fx_fiedler(fx_ctx *ctx, fx_design *d, int32_t n_clusters,
                          const int32_t *cluster_ptr, const int32_t *cluster_gate,
                          int32_t max_iters, double tol, float *out_v,
                          int32_t *out_iters, double *out_lambda) {
  if (!ctx || !d || n_clusters < 0 || max_iters < 0 || !(tol >= 0.0) ||
      (n_clusters > 0 && (!cluster_ptr || !cluster_gate || !out_v))) {
    set_error("fx_fiedler: invalid arguments");
    return FX_EINVAL;
  }
  if (n_clusters == 0) return FX_OK;
  if (cluster_ptr[0] != 0) {
    set_error("fx_fiedler: cluster_ptr[0] must be 0");
    return FX_EINVAL;
  }
  const int32_t G = cluster_ptr[n_clusters];
  // Host: positions, in-cluster adjacency (reference order), degrees, the
  // reference's start vector, and the chunking.
  std::vector<int32_t> cl_of((size_t)d->n, -1), pos_of((size_t)d->n, -1);
  for (int c = 0; c < n_clusters; ++c) {
    if (cluster_ptr[c + 1] < cluster_ptr[c]) {
      set_error("fx_fiedler: cluster_ptr decreases at %d", c);
      return FX_EINVAL;
    }
    for (int32_t p = cluster_ptr[c]; p < cluster_ptr[c + 1]; ++p) {
      const int32_t g = cluster_gate[p];
      if (g < 0 || g >= d->n || cl_of[g] >= 0) {
        set_error("fx_fiedler: gate %d out of range or in two clusters", g);
        return FX_EINVAL;
      }
      cl_of[g] = c;
      pos_of[g] = p;
    }
  }
  std::vector<int32_t> rptr((size_t)G + 1, 0), ridx;
  std::vector<float> deg((size_t)G), v((size_t)G);
  for (int c = 0; c < n_clusters; ++c) {
    const int32_t b = cluster_ptr[c], e = cluster_ptr[c + 1], n = e - b;
    for (int32_t p = b; p < e; ++p) {
      const int32_t g = cluster_gate[p];
      int32_t cnt = 0;
      for (int32_t q = d->h_adj_ptr[g]; q < d->h_adj_ptr[g + 1]; ++q) {
        const int32_t j = d->h_adj_idx[q];
        if (cl_of[j] == c) {
          ridx.push_back(pos_of[j]);
          ++cnt;
        }
      }
      rptr[(size_t)p + 1] = (int32_t)ridx.size();
      float dg = 0.0f;  // degree[local_g] += 1.0 per entry (partitioner.rs:133)
      for (int32_t k = 0; k < cnt; ++k) dg += 1.0f;
      deg[p] = dg;
    }
    // partitioner.rs:143-155: v_i = sin(i * 2.71828) in f32, normalised.
    for (int32_t i = 0; i < n; ++i) v[(size_t)b + i] = std::sin((float)i * 2.71828f);
    float norm = 0.0f;
    for (int32_t i = 0; i < n; ++i) norm += v[(size_t)b + i] * v[(size_t)b + i];
    norm = std::sqrt(norm);
    if (norm > 1e-10f)
      for (int32_t i = 0; i < n; ++i) v[(size_t)b + i] /= norm;
  }
  std::vector<int32_t> chunk_start, chunk_cluster, cl_chunk((size_t)n_clusters + 1, 0);
  for (int c = 0; c < n_clusters; ++c) {
    for (int32_t p = cluster_ptr[c]; p < cluster_ptr[c + 1]; p += kRowChunk) {
      chunk_start.push_back(p);
      chunk_cluster.push_back(c);
    }
    cl_chunk[(size_t)c + 1] = (int32_t)chunk_start.size();
  }
  chunk_start.push_back(G);
  const int K = (int)chunk_cluster.size();
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t s = ctx->stream;
  DevBuf<int32_t> d_rptr, d_ridx, d_cs, d_cc, d_clp, d_clc, d_act, d_it;
  DevBuf<float> d_deg, d_v, d_lv, d_mean, d_inv;
  DevBuf<double> d_part, d_lam;
  FX_TRY(d_rptr.alloc(rptr.size()));
  FX_TRY(d_ridx.alloc(ridx.empty() ? 1 : ridx.size()));
  FX_TRY(d_cs.alloc(chunk_start.size()));
  FX_TRY(d_cc.alloc(K > 0 ? (size_t)K : 1));
  FX_TRY(d_clp.alloc((size_t)n_clusters + 1));
  FX_TRY(d_clc.alloc((size_t)n_clusters + 1));
  FX_TRY(d_act.alloc((size_t)n_clusters));
  FX_TRY(d_it.alloc((size_t)n_clusters));
  FX_TRY(d_deg.alloc(G > 0 ? (size_t)G : 1));
  FX_TRY(d_v.alloc(G > 0 ? (size_t)G : 1));
  FX_TRY(d_lv.alloc(G > 0 ? (size_t)G : 1));
  FX_TRY(d_mean.alloc((size_t)n_clusters));
  FX_TRY(d_inv.alloc((size_t)n_clusters));
  FX_TRY(d_part.alloc(3 * (size_t)(K > 0 ? K : 1)));
  FX_TRY(d_lam.alloc((size_t)n_clusters));
  auto up = [&](void *dst, const void *src, size_t bytes) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
  };
  std::vector<int32_t> ones((size_t)n_clusters, 1);
  FX_CHECK_CUDA(up(d_rptr.p, rptr.data(), rptr.size() * 4));
  FX_CHECK_CUDA(up(d_ridx.p, ridx.data(), ridx.size() * 4));
  FX_CHECK_CUDA(up(d_cs.p, chunk_start.data(), chunk_start.size() * 4));
  FX_CHECK_CUDA(up(d_cc.p, chunk_cluster.data(), chunk_cluster.size() * 4));
  FX_CHECK_CUDA(up(d_clp.p, cluster_ptr, ((size_t)n_clusters + 1) * 4));
  FX_CHECK_CUDA(up(d_clc.p, cl_chunk.data(), cl_chunk.size() * 4));
  FX_CHECK_CUDA(up(d_act.p, ones.data(), ones.size() * 4));
  FX_CHECK_CUDA(cudaMemsetAsync(d_it.p, 0, (size_t)n_clusters * 4, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d_lam.p, 0, (size_t)n_clusters * 8, s));
  FX_CHECK_CUDA(up(d_deg.p, deg.data(), deg.size() * 4));
  FX_CHECK_CUDA(up(d_v.p, v.data(), v.size() * 4));
  FiedlerArgs a{d_rptr.p, d_ridx.p, d_deg.p, d_v.p, d_lv.p, d_cs.p, d_cc.p, d_clp.p,
                d_clc.p, d_part.p, d_mean.p, d_inv.p, d_lam.p, d_act.p, d_it.p,
                K, n_clusters, tol};
  cudaEvent_t ev;
  timer_begin(ctx, FX_STAGE_FIEDLER, s, &ev);
  const int kb = (K * 32 + 255) / 256, cb = (n_clusters + 255) / 256, gb = (G + 255) / 256;
  int ran = 0;
  // tol == 0: the reference's own f32 mean and norm (sequential folds), so
  // the vectors are bit-identical to compute_fiedler_vector's
  const bool exact = tol == 0.0;
  DevBuf<float> d_nrm;
  if (exact) FX_TRY(d_nrm.alloc((size_t)n_clusters));
  for (int it = 0; it < max_iters; ++it) {
    ++ran;
    fiedler_spmv_kernel<<<kb, 256, 0, s>>>(a);
    fiedler_stats_kernel<<<cb, 256, 0, s>>>(a);
    if (exact) {
      part_seq_kernel<<<n_clusters, 32, 0, s>>>(n_clusters, d_clp.p, d_clp.p + 1, d_lv.p, 1,
                                                d_nrm.p);
      fiedler_div_kernel<<<gb, 256, 0, s>>>(a, d_nrm.p, G);
    } else {
      fiedler_update_kernel<<<gb, 256, 0, s>>>(a, G);
    }
    fiedler_retire_kernel<<<cb, 256, 0, s>>>(d_act.p, n_clusters, it == max_iters - 1);
    // With a tolerance, stop as soon as every cluster has converged.
    if (tol > 0.0 && (it % 16) == 15) {
      std::vector<int32_t> act((size_t)n_clusters);
      FX_CHECK_CUDA(cudaMemcpyAsync(act.data(), d_act.p, act.size() * 4,
                                    cudaMemcpyDeviceToHost, s));
      FX_CHECK_CUDA(cudaStreamSynchronize(s));
      bool any = false;
      for (int32_t x : act) any |= x != 0;
      if (!any) break;
    }
  }
  // the Rayleigh quotient of the vectors returned: one more SpMV on them
  FX_CHECK_CUDA(up(d_act.p, ones.data(), ones.size() * 4));
  fiedler_spmv_kernel<<<kb, 256, 0, s>>>(a);
  fiedler_lambda_kernel<<<cb, 256, 0, s>>>(a);
  FX_CHECK_LAUNCH();
  ctx->launches += (exact ? 5 : 4) * (int64_t)ran + 2;
  timer_end(ctx, FX_STAGE_FIEDLER, s, ev);
  FX_CHECK_CUDA(cudaMemcpyAsync(out_v, d_v.p, (size_t)G * 4, cudaMemcpyDeviceToHost, s));
  if (out_iters)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_iters, d_it.p, (size_t)n_clusters * 4,
                                  cudaMemcpyDeviceToHost, s));
  if (out_lambda)
    FX_CHECK_CUDA(cudaMemcpyAsync(out_lambda, d_lam.p, (size_t)n_clusters * 8,
                                  cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  if (out_lambda)
    for (int c = 0; c < n_clusters; ++c) {
      double vv = 0.0;
      for (int32_t p = cluster_ptr[c]; p < cluster_ptr[c + 1]; ++p)
        vv += (double)out_v[p] * (double)out_v[p];
      out_lambda[c] = vv > 0.0 ? out_lambda[c] / vv : 0.0;
    }
  return FX_OK;
}
