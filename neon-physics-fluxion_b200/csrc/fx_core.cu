// fx_core.cu -- context, error reporting, stage timing and design upload.
#include <algorithm>
#include <cstdarg>
#include <cstring>
#include <new>

#include <algorithm>
#include <map>
#include <mutex>
#include <thread>
#include <utility>

#include "fx_internal.h"

namespace fx {

static thread_local char g_err[512] = "";
thread_local cudaStream_t g_alloc_stream = nullptr;

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

cudaEvent_t StageTimer::get_event() {
  if (!pool.empty()) {
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

void StageTimer::resolve() {
  for (auto &p : pending) {
    float t = 0.f;
    if (cudaEventSynchronize(p.b) == cudaSuccess &&
        cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) {
      ms[p.stage] += t;
      calls[p.stage] += 1;
    }
    pool.push_back(p.a);
    pool.push_back(p.b);
  }
  pending.clear();
}

void StageTimer::add_elapsed(const std::vector<Pending> &pairs) {
  for (auto &p : pairs) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) {
      ms[p.stage] += t;
      calls[p.stage] += 1;
    }
  }
}

void StageTimer::destroy() {
  resolve();
  for (auto &p : captured) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  captured.clear();
  for (auto e : pool) cudaEventDestroy(e);
  pool.clear();
}

// Under stream capture the events are recorded as event record nodes of the
// graph (cudaEventRecordExternal) and the pair is kept in `captured`.
static bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(s, &st) == cudaSuccess && st == cudaStreamCaptureStatusActive;
}

void timer_begin(fx_ctx *ctx, int stage, cudaStream_t s, cudaEvent_t *a) {
  *a = nullptr;
  if (!ctx->timer.enabled || !((ctx->timer.mask >> stage) & 1u)) return;
  *a = ctx->timer.get_event();
  if (!*a) return;
  if (capturing(s))
    cudaEventRecordWithFlags(*a, s, cudaEventRecordExternal);
  else
    cudaEventRecord(*a, s);
}

void timer_end(fx_ctx *ctx, int stage, cudaStream_t s, cudaEvent_t a) {
  if (!ctx->timer.enabled || !a) return;
  cudaEvent_t b = ctx->timer.get_event();
  if (!b) return;
  if (capturing(s)) {
    cudaEventRecordWithFlags(b, s, cudaEventRecordExternal);
    ctx->timer.captured.push_back({stage, a, b});
    return;
  }
  cudaEventRecord(b, s);
  ctx->timer.pending.push_back({stage, a, b});
  if (ctx->timer.pending.size() > 4096) ctx->timer.resolve();
}

int raise_smem_limit(const void *func, int bytes) {
  int dev = 0;
  FX_CHECK_CUDA(cudaGetDevice(&dev));
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> limit;  // (kernel, device)
  std::lock_guard<std::mutex> lock(mu);
  int &cur = limit[{func, dev}];
  if (bytes <= cur) return FX_OK;
  FX_CHECK_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  cur = bytes;
  return FX_OK;
}

// Deduplicated clique-expansion adjacency (H/src/data/circuit.rs:154-171),
// in the reference's insertion order. The reference walks the pairs (i < j)
// of every net in net order and appends each endpoint to the other's list
// unless present. For a gate a at pin position p of net e that yields the
// net's pins in pin order without position p; so each list is "incident
// nets in net order, pins in pin order, skipping a and duplicates". A net
// that names a twice also appends a itself; such nets replay the pair loop
// for a to keep the exact order. Built from the gate->net incidence in
// O(sum over nets of degree^2) with a marker array instead of Vec::contains.
static int build_adjacency(int32_t N, int32_t M, const int32_t *net_ptr,
                           const int32_t *net_gate, std::vector<int32_t> &ptr,
                           std::vector<int32_t> &idx) {
  const int64_t P = net_ptr[M];
  std::vector<int32_t> inc_ptr((size_t)N + 1, 0);
  for (int64_t q = 0; q < P; ++q) inc_ptr[(size_t)net_gate[q] + 1]++;
  for (int32_t g = 0; g < N; ++g) inc_ptr[g + 1] += inc_ptr[g];
  std::vector<int32_t> inc((size_t)P);
  {
    std::vector<int32_t> fill(inc_ptr.begin(), inc_ptr.end() - 1);
    for (int32_t e = 0; e < M; ++e)
      for (int32_t q = net_ptr[e]; q < net_ptr[e + 1]; ++q)
        inc[fill[net_gate[q]]++] = e;
  }
  // Each gate's list depends only on its own nets, so gate ranges are built
  // independently (a stamp array per range) and concatenated in gate order.
  auto build_range = [&](int32_t g0, int32_t g1, std::vector<int32_t> &cnt,
                         std::vector<int32_t> &out) {
    std::vector<int32_t> mark((size_t)N, -1);
    auto push = [&](int32_t a, int32_t b) {
      if (mark[b] != a) {
        mark[b] = a;
        out.push_back(b);
      }
    };
    for (int32_t a = g0; a < g1; ++a) {
      const size_t before = out.size();
      for (int32_t t = inc_ptr[a]; t < inc_ptr[a + 1]; ++t) {
        const int32_t e = inc[t];
        if (t > inc_ptr[a] && inc[t - 1] == e) continue;  // net already done
        const bool repeated = t + 1 < inc_ptr[a + 1] && inc[t + 1] == e;
        const int32_t b0 = net_ptr[e], b1 = net_ptr[e + 1];
        if (!repeated) {
          for (int32_t q = b0; q < b1; ++q)
            if (net_gate[q] != a) push(a, net_gate[q]);
        } else {  // replay circuit.rs:158-168 for the pairs that touch a
          for (int32_t i = b0; i < b1; ++i)
            for (int32_t j = i + 1; j < b1; ++j) {
              if (net_gate[i] == a) push(a, net_gate[j]);
              if (net_gate[j] == a) push(a, net_gate[i]);
            }
        }
      }
      cnt[(size_t)(a - g0)] = (int32_t)(out.size() - before);
    }
  };
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int T = N >= 200000 ? (int)std::min<unsigned>(8, hw) : 1;
  std::vector<std::vector<int32_t>> cnt((size_t)T), part((size_t)T);
  std::vector<int32_t> lo((size_t)T + 1);
  for (int t = 0; t <= T; ++t) lo[(size_t)t] = (int32_t)((int64_t)N * t / T);
  for (int t = 0; t < T; ++t) {
    cnt[(size_t)t].assign((size_t)(lo[t + 1] - lo[t]), 0);
    part[(size_t)t].reserve((size_t)((int64_t)P * 4 / T));
  }
  if (T == 1) {
    build_range(0, N, cnt[0], part[0]);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t)
      th.emplace_back(build_range, lo[t], lo[t + 1], std::ref(cnt[(size_t)t]),
                      std::ref(part[(size_t)t]));
    for (auto &x : th) x.join();
  }
  size_t total = 0;
  for (auto &v : part) total += v.size();
  if (total > (size_t)INT32_MAX) {
    set_error("adjacency exceeds 2^31 entries");
    return FX_EINVAL;
  }
  ptr.assign((size_t)N + 1, 0);
  idx.resize(total);
  size_t off = 0;
  for (int t = 0; t < T; ++t) {
    for (int32_t a = lo[t]; a < lo[t + 1]; ++a)
      ptr[(size_t)a + 1] = ptr[(size_t)a] + cnt[(size_t)t][(size_t)(a - lo[t])];
    std::copy(part[(size_t)t].begin(), part[(size_t)t].end(), idx.begin() + (int64_t)off);
    off += part[(size_t)t].size();
  }
  return FX_OK;
}

}  // namespace fx

using namespace fx;

extern "C" const char *fx_last_error(void) { return fx::g_err; }
extern "C" const char *fx_version(void) { return "fluxion_b200 0.1"; }

extern "C" int fx_ctx_create(fx_ctx **out_ctx, int device) {
  if (!out_ctx) return FX_EINVAL;
  *out_ctx = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    set_error("no CUDA device visible");
    return FX_ENODEV;
  }
  if (device < 0 || device >= count) {
    set_error("device %d out of range (%d devices)", device, count);
    return FX_EINVAL;
  }
  cudaDeviceProp prop;
  FX_CHECK_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_error("device %d is sm_%d%d; the library targets sm_100a", device,
              prop.major, prop.minor);
    return FX_ENODEV;
  }
  FX_CHECK_CUDA(cudaSetDevice(device));
  fx_ctx *c = new (std::nothrow) fx_ctx();
  if (!c) return FX_ENOMEM;
  c->device = device;
  c->num_sms = prop.multiProcessorCount;
  // The primary stream (the Barnes-Hut chain and everything serial) gets the
  // highest priority, the side stream (the density solve that overlaps it)
  // the lowest, so the short sort and tree kernels are not held back by GEMM
  // blocks.
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  if (cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->stream2, cudaStreamNonBlocking, prio_low) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming) != cudaSuccess) {
    set_error("stream/event creation failed");
    delete c;
    return FX_ECUDA;
  }
  // The word is zeroed on the primary stream and the creation waits for it,
  // so no GEMM of this context (on either stream) can see a stale value.
  if (cudaMallocHost((void **)&c->readback, sizeof(fx::IterReadback)) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&c->readback_dev, c->readback, 0) != cudaSuccess ||
      cudaMalloc((void **)&c->tc_err, sizeof(unsigned int)) != cudaSuccess ||
      cudaMemsetAsync(c->tc_err, 0, sizeof(unsigned int), c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error("error word allocation failed");
    if (c->tc_err) cudaFree(c->tc_err);
    if (c->readback) cudaFreeHost(c->readback);
    cudaEventDestroy(c->fork);
    cudaEventDestroy(c->join);
    cudaStreamDestroy(c->stream);
    cudaStreamDestroy(c->stream2);
    delete c;
    return FX_ECUDA;
  }
  // Freed stream-ordered allocations stay in the device's pool for reuse,
  // so a call's temporaries cost no driver allocation after the first.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  *out_ctx = c;
  return FX_OK;
}

namespace fx {
// Re-creates a fresh context's two streams at the given priorities (lower
// numbers run first; cudaDeviceGetStreamPriorityRange gives the range). The
// context must have no work in flight.
int ctx_set_priorities(fx_ctx *c, int primary, int side) {
  FX_CHECK_CUDA(cudaSetDevice(c->device));
  FX_CHECK_CUDA(cudaStreamSynchronize(c->stream));
  FX_CHECK_CUDA(cudaStreamSynchronize(c->stream2));
  cudaStream_t a = nullptr, b = nullptr;
  FX_CHECK_CUDA(cudaStreamCreateWithPriority(&a, cudaStreamNonBlocking, primary));
  if (cudaStreamCreateWithPriority(&b, cudaStreamNonBlocking, side) != cudaSuccess) {
    cudaStreamDestroy(a);
    set_error("stream creation failed");
    return FX_ECUDA;
  }
  cudaStreamDestroy(c->stream);
  cudaStreamDestroy(c->stream2);
  c->stream = a;
  c->stream2 = b;
  return FX_OK;
}
}  // namespace fx

extern "C" int fx_ctx_destroy(fx_ctx *ctx) {
  if (!ctx) return FX_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamSynchronize(ctx->stream2);
  ctx->timer.destroy();
  for (auto &e : ctx->marks)
    if (e) cudaEventDestroy(e);
  cudaEventDestroy(ctx->fork);
  cudaEventDestroy(ctx->join);
  if (ctx->tc_err) cudaFree(ctx->tc_err);
  if (ctx->readback) cudaFreeHost(ctx->readback);
  cudaStreamDestroy(ctx->stream);
  cudaStreamDestroy(ctx->stream2);
  delete ctx;
  return FX_OK;
}

extern "C" int fx_ctx_set_profiling(fx_ctx *ctx, int enable) {
  if (!ctx) return FX_EINVAL;
  ctx->timer.enabled = enable != 0;
  return FX_OK;
}

extern "C" int fx_ctx_set_profiling_stages(fx_ctx *ctx, uint32_t stage_mask) {
  if (!ctx) return FX_EINVAL;
  ctx->timer.mask = stage_mask;
  return FX_OK;
}

extern "C" int fx_ctx_stage_times(fx_ctx *ctx, double *out_ms,
                                  int64_t *out_calls, int n) {
  if (!ctx) return FX_EINVAL;
  cudaSetDevice(ctx->device);
  ctx->timer.resolve();
  for (int s = 0; s < n && s < FX_STAGE_COUNT; ++s) {
    if (out_ms) out_ms[s] = ctx->timer.ms[s];
    if (out_calls) out_calls[s] = ctx->timer.calls[s];
  }
  return FX_OK;
}

extern "C" int fx_ctx_reset_stage_times(fx_ctx *ctx) {
  if (!ctx) return FX_EINVAL;
  cudaSetDevice(ctx->device);
  ctx->timer.resolve();
  for (int s = 0; s < FX_STAGE_COUNT; ++s) {
    ctx->timer.ms[s] = 0.0;
    ctx->timer.calls[s] = 0;
  }
  return FX_OK;
}

extern "C" int64_t fx_ctx_kernel_launches(fx_ctx *ctx) {
  return ctx ? ctx->launches : -1;
}

extern "C" int fx_ctx_mark(fx_ctx *ctx, int slot) {
  if (!ctx || slot < 0 || slot >= 16) return FX_EINVAL;
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  if (!ctx->marks[slot]) FX_CHECK_CUDA(cudaEventCreate(&ctx->marks[slot]));
  FX_CHECK_CUDA(cudaEventRecord(ctx->marks[slot], ctx->stream));
  return FX_OK;
}

extern "C" int fx_ctx_elapsed(fx_ctx *ctx, int a, int b, float *out_ms) {
  if (!ctx || !out_ms || a < 0 || a >= 16 || b < 0 || b >= 16 ||
      !ctx->marks[a] || !ctx->marks[b])
    return FX_EINVAL;
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  FX_CHECK_CUDA(cudaEventSynchronize(ctx->marks[b]));
  FX_CHECK_CUDA(cudaEventElapsedTime(out_ms, ctx->marks[a], ctx->marks[b]));
  return FX_OK;
}

extern "C" int fx_ctx_synchronize(fx_ctx *ctx) {
  if (!ctx) return FX_EINVAL;
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  FX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  FX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream2));
  return FX_OK;
}

static int validate_netlist(int32_t n_gates, int32_t n_nets,
                            const int32_t *net_ptr, const int32_t *net_gate) {
  if (n_gates <= 0 || n_nets < 0 || !net_ptr || (n_nets > 0 && !net_gate)) {
    set_error("invalid netlist arguments");
    return FX_EINVAL;
  }
  if (net_ptr[0] != 0) {
    set_error("net_ptr[0] must be 0");
    return FX_EINVAL;
  }
  for (int32_t e = 0; e < n_nets; ++e)
    if (net_ptr[e + 1] < net_ptr[e]) {
      set_error("net_ptr decreases at net %d", e);
      return FX_EINVAL;
    }
  const int64_t P = net_ptr[n_nets];
  for (int64_t q = 0; q < P; ++q)
    if (net_gate[q] < 0 || net_gate[q] >= n_gates) {
      set_error("pin %lld names gate %d (n_gates=%d)", (long long)q, net_gate[q],
                n_gates);
      return FX_EINVAL;
    }
  return FX_OK;
}

extern "C" int64_t fx_adjacency_build(int32_t n_gates, int32_t n_nets,
                                      const int32_t *net_ptr,
                                      const int32_t *net_gate,
                                      int32_t *out_adj_ptr, int32_t *out_adj_idx,
                                      int64_t cap) {
  if (!out_adj_ptr) return FX_EINVAL;
  FX_TRY(validate_netlist(n_gates, n_nets, net_ptr, net_gate));
  std::vector<int32_t> ptr, idx;
  FX_TRY(build_adjacency(n_gates, n_nets, net_ptr, net_gate, ptr, idx));
  memcpy(out_adj_ptr, ptr.data(), ptr.size() * 4);
  if (out_adj_idx && cap > 0)
    memcpy(out_adj_idx, idx.data(),
           (size_t)std::min<int64_t>(cap, (int64_t)idx.size()) * 4);
  return (int64_t)idx.size();
}

extern "C" int fx_design_load(fx_ctx *ctx, int32_t n_gates, int32_t n_nets,
                              const int32_t *net_ptr, const int32_t *net_gate,
                              const float *gate_w, const float *gate_h,
                              float chip_w, float chip_h,
                              fx_design **out_design) {
  if (!ctx || !out_design) {
    set_error("fx_design_load: invalid arguments");
    return FX_EINVAL;
  }
  *out_design = nullptr;
  if (!(chip_w > 0.f) || !(chip_h > 0.f)) {
    set_error("fx_design_load: chip size must be positive");
    return FX_EINVAL;
  }
  FX_TRY(validate_netlist(n_gates, n_nets, net_ptr, net_gate));
  const int64_t P = net_ptr[n_nets];
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  AllocScope alloc_scope(ctx->stream);
  fx_design *d = new (std::nothrow) fx_design();
  if (!d) return FX_ENOMEM;
  d->ctx = ctx;
  d->n = n_gates;
  d->m = n_nets;
  d->p = P;
  d->chip_w = chip_w;
  d->chip_h = chip_h;
  int rc = build_adjacency(n_gates, n_nets, net_ptr, net_gate, d->h_adj_ptr,
                           d->h_adj_idx);
  if (rc != FX_OK) {
    delete d;
    return rc;
  }
  d->a = (int64_t)d->h_adj_idx.size();
  d->h_w.resize(n_gates);
  d->h_h.resize(n_gates);
  std::vector<float> area(n_gates);
  for (int32_t g = 0; g < n_gates; ++g) {
    d->h_w[g] = gate_w ? gate_w[g] : 2.0f;
    d->h_h[g] = gate_h ? gate_h[g] : 10.0f;
    area[g] = d->h_w[g] * d->h_h[g];
  }
  const size_t N = (size_t)n_gates;
  auto fail = [&](int code) {
    fx_design_free(d);
    return code;
  };
  if ((rc = d->net_ptr.alloc((size_t)n_nets + 1)) ||
      (rc = d->net_gate.alloc(P > 0 ? (size_t)P : 1)) ||
      (rc = d->adj_ptr.alloc(N + 1)) ||
      (rc = d->adj_idx.alloc(d->a > 0 ? (size_t)d->a : 1)) ||
      (rc = d->area.alloc(N)) || (rc = d->x[0].alloc(N)) ||
      (rc = d->y[0].alloc(N)) || (rc = d->x[1].alloc(N)) ||
      (rc = d->y[1].alloc(N)) || (rc = d->vx.alloc(N)) ||
      (rc = d->vy.alloc(N)) || (rc = d->fattr.alloc(N)) || (rc = d->box_flag.alloc(1)))
    return fail(rc);
  cudaStream_t s = ctx->stream;
  if (cudaMemcpyAsync(d->net_ptr.p, net_ptr, ((size_t)n_nets + 1) * 4,
                      cudaMemcpyHostToDevice, s) != cudaSuccess ||
      (P > 0 && cudaMemcpyAsync(d->net_gate.p, net_gate, (size_t)P * 4,
                                cudaMemcpyHostToDevice, s) != cudaSuccess) ||
      cudaMemcpyAsync(d->adj_ptr.p, d->h_adj_ptr.data(), (N + 1) * 4,
                      cudaMemcpyHostToDevice, s) != cudaSuccess ||
      (d->a > 0 && cudaMemcpyAsync(d->adj_idx.p, d->h_adj_idx.data(),
                                   (size_t)d->a * 4, cudaMemcpyHostToDevice,
                                   s) != cudaSuccess) ||
      cudaMemcpyAsync(d->area.p, area.data(), N * 4, cudaMemcpyHostToDevice,
                      s) != cudaSuccess ||
      cudaMemsetAsync(d->x[0].p, 0, N * 4, s) != cudaSuccess ||
      cudaMemsetAsync(d->y[0].p, 0, N * 4, s) != cudaSuccess ||
      cudaMemsetAsync(d->vx.p, 0, N * 4, s) != cudaSuccess ||
      cudaMemsetAsync(d->vy.p, 0, N * 4, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    set_error("fx_design_load: upload failed: %s",
              cudaGetErrorString(cudaGetLastError()));
    return fail(FX_ECUDA);
  }
  *out_design = d;
  return FX_OK;
}

extern "C" int fx_design_free(fx_design *d) {
  if (!d) return FX_OK;
  cudaSetDevice(d->ctx->device);
  cudaStreamSynchronize(d->ctx->stream);
  cudaStreamSynchronize(d->ctx->stream2);
  for (auto &g : d->g1) g.reset();
  d->net_ptr.release();
  d->net_gate.release();
  d->adj_ptr.release();
  d->adj_idx.release();
  d->area.release();
  for (int i = 0; i < 2; ++i) {
    d->x[i].release();
    d->y[i].release();
  }
  d->vx.release();
  d->vy.release();
  d->fattr.release();
  d->box_flag.release();
  for (auto &b : d->saved) b.release();
  auto rel = [](auto &buf) { buf.release(); };
  d->bh.for_each(rel);
  d->dens.for_each(rel);
  d->cong.for_each(rel);
  d->step.for_each(rel);
  delete d;
  return FX_OK;
}

extern "C" int fx_design_sizes(const fx_design *d, int64_t *out_n,
                               int64_t *out_m, int64_t *out_p,
                               int64_t *out_a) {
  if (!d) return FX_EINVAL;
  if (out_n) *out_n = d->n;
  if (out_m) *out_m = d->m;
  if (out_p) *out_p = d->p;
  if (out_a) *out_a = d->a;
  return FX_OK;
}

extern "C" int fx_design_adjacency(const fx_design *d, int32_t *out_adj_ptr,
                                   int32_t *out_adj_idx) {
  if (!d) return FX_EINVAL;
  if (out_adj_ptr)
    memcpy(out_adj_ptr, d->h_adj_ptr.data(), d->h_adj_ptr.size() * 4);
  if (out_adj_idx && !d->h_adj_idx.empty())
    memcpy(out_adj_idx, d->h_adj_idx.data(), d->h_adj_idx.size() * 4);
  return FX_OK;
}

// Clears *flag when a position lies outside [0, w] x [0, h] or is NaN.
__global__ void box_check_kernel(const float *__restrict__ x, const float *__restrict__ y,
                                 int n, float w, float h, unsigned int *__restrict__ flag) {
  bool out = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out |= !(x[i] >= 0.f && x[i] <= w && y[i] >= 0.f && y[i] <= h);
  if (__any_sync(0xffffffffu, out) && (threadIdx.x & 31) == 0) *flag = 0u;
}

extern "C" int fx_design_set_positions(fx_design *d, const float *x,
                                       const float *y) {
  if (!d || !x || !y) return FX_EINVAL;
  FX_CHECK_CUDA(cudaSetDevice(d->ctx->device));
  cudaStream_t s = d->ctx->stream;
  const size_t b = (size_t)d->n * 4;
  d->cur = 0;
  FX_CHECK_CUDA(cudaMemcpyAsync(d->x[0].p, x, b, cudaMemcpyHostToDevice, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(d->y[0].p, y, b, cudaMemcpyHostToDevice, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d->vx.p, 0, b, s));
  FX_CHECK_CUDA(cudaMemsetAsync(d->vy.p, 0, b, s));
  // whether the positions lie in the die (it lets Barnes-Hut skip its deep
  // key kernels when the die is small enough), read with the sync below
  unsigned int in_box = 0;
  FX_CHECK_CUDA(cudaMemsetAsync(d->box_flag.p, 0xFF, 4, s));
  if (d->n > 0) {
    const int nb = std::min((d->n + 255) / 256, 4 * d->ctx->num_sms);
    box_check_kernel<<<nb, 256, 0, s>>>(d->x[0].p, d->y[0].p, d->n, d->chip_w, d->chip_h,
                                        d->box_flag.p);
    FX_CHECK_CUDA(cudaGetLastError());
    d->ctx->launches += 1;
  }
  FX_CHECK_CUDA(cudaMemcpyAsync(&in_box, d->box_flag.p, 4, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  d->pos_in_box = in_box != 0u;
  return FX_OK;
}

extern "C" int fx_design_get_positions(fx_design *d, float *out_x,
                                       float *out_y) {
  if (!d || !out_x || !out_y) return FX_EINVAL;
  FX_CHECK_CUDA(cudaSetDevice(d->ctx->device));
  cudaStream_t s = d->ctx->stream;
  const size_t b = (size_t)d->n * 4;
  FX_CHECK_CUDA(cudaMemcpyAsync(out_x, d->x[d->cur].p, b, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaMemcpyAsync(out_y, d->y[d->cur].p, b, cudaMemcpyDeviceToHost, s));
  FX_CHECK_CUDA(cudaStreamSynchronize(s));
  return FX_OK;
}

namespace fx {
namespace {
// The four state arrays (x, y, vx, vy) in one launch: four floats of each
// per thread, 16-byte accesses where the array is long enough.
struct State4 {
  const float *src[4];
  float *dst[4];
};
__global__ void state_copy_kernel(int n, State4 a) {
  const int i = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n) return;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (i + 3 < n) {
      reinterpret_cast<float4 *>(a.dst[k])[i >> 2] =
          reinterpret_cast<const float4 *>(a.src[k])[i >> 2];
    } else {
      for (int j = i; j < n; ++j) a.dst[k][j] = a.src[k][j];
    }
  }
}

int state_copy(fx_design *d, const State4 &a, cudaStream_t s) {
  if (d->n <= 0) return FX_OK;
  const int threads = (d->n + 3) / 4;
  state_copy_kernel<<<(threads + 255) / 256, 256, 0, s>>>(d->n, a);
  FX_CHECK_LAUNCH();
  d->ctx->launches += 1;
  return FX_OK;
}
}  // namespace
}  // namespace fx

extern "C" int fx_design_save_state(fx_design *d) {
  if (!d) return FX_EINVAL;
  FX_CHECK_CUDA(cudaSetDevice(d->ctx->device));
  AllocScope alloc_scope(d->ctx->stream);
  cudaStream_t s = d->ctx->stream;
  fx::State4 a{{d->x[d->cur].p, d->y[d->cur].p, d->vx.p, d->vy.p}, {}};
  for (int i = 0; i < 4; ++i) {
    if (!d->saved[i].p) FX_TRY(d->saved[i].alloc(d->n));
    a.dst[i] = d->saved[i].p;
  }
  FX_TRY(fx::state_copy(d, a, s));
  d->saved_in_box = d->pos_in_box;
  return FX_OK;
}

extern "C" int fx_design_restore_state(fx_design *d) {
  if (!d) return FX_EINVAL;
  if (!d->saved[0].p) {
    set_error("fx_design_restore_state: no saved state");
    return FX_EINVAL;
  }
  FX_CHECK_CUDA(cudaSetDevice(d->ctx->device));
  cudaStream_t s = d->ctx->stream;
  fx::State4 a{{d->saved[0].p, d->saved[1].p, d->saved[2].p, d->saved[3].p},
               {d->x[d->cur].p, d->y[d->cur].p, d->vx.p, d->vy.p}};
  FX_TRY(fx::state_copy(d, a, s));
  d->pos_in_box = d->saved_in_box;
  return FX_OK;
}

extern "C" int64_t fx_design_device_bytes(const fx_design *d) {
  if (!d) return -1;
  int64_t t = 0;
  t += d->net_ptr.bytes() + d->net_gate.bytes() + d->adj_ptr.bytes() +
       d->adj_idx.bytes() + d->area.bytes();
  for (int i = 0; i < 2; ++i) t += d->x[i].bytes() + d->y[i].bytes();
  t += d->vx.bytes() + d->vy.bytes() + d->fattr.bytes();
  for (int i = 0; i < 4; ++i) t += d->saved[i].bytes();
  auto add = [&t](auto &buf) { t += (int64_t)buf.bytes(); };
  fx_design *m = const_cast<fx_design *>(d);
  m->bh.for_each(add);
  m->dens.for_each(add);
  m->cong.for_each(add);
  m->step.for_each(add);
  return t;
}
