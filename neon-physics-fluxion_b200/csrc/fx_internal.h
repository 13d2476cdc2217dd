// fx_internal.h -- shared declarations of libfluxion_b200 (not installed).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/fluxion_b200.h"

namespace fx {

// ---- error handling --------------------------------------------------------
void set_error(const char *fmt, ...);

struct Status {
  int code = FX_OK;
};

#define FX_CHECK_CUDA(expr)                                                   \
  do {                                                                        \
    cudaError_t _e = (expr);                                                  \
    if (_e != cudaSuccess) {                                                  \
      ::fx::set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr,              \
                      cudaGetErrorString(_e));                                \
      return FX_ECUDA;                                                        \
    }                                                                         \
  } while (0)

#define FX_TRY(expr)                                                          \
  do {                                                                        \
    int _rc = (expr);                                                         \
    if (_rc != FX_OK) return _rc;                                             \
  } while (0)

// Checks the launch that was just issued.
#define FX_CHECK_LAUNCH() FX_CHECK_CUDA(cudaGetLastError())

// ---- device buffers --------------------------------------------------------
// Allocation stream of the calling thread. Inside an API call it is the
// context's primary stream (set by AllocScope), and DevBufs are then
// stream-ordered (cudaMallocAsync / cudaFreeAsync from the device's pool,
// whose memory is retained): allocating or freeing does not wait for the
// whole device, so jobs on other contexts keep running. Memory allocated
// this way is used on that stream, or on another stream only after an
// event recorded on it later. Without a scope (library globals) DevBuf uses
// cudaMalloc / cudaFree.
extern thread_local cudaStream_t g_alloc_stream;

struct AllocScope {
  cudaStream_t prev;
  explicit AllocScope(cudaStream_t s) : prev(g_alloc_stream) { g_alloc_stream = s; }
  ~AllocScope() { g_alloc_stream = prev; }
  AllocScope(const AllocScope &) = delete;
  AllocScope &operator=(const AllocScope &) = delete;
};

// A typed device allocation owned by a design, a context or a call.
template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaStream_t owner = nullptr;  // stream of a pooled allocation
  bool pooled = false;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  int alloc(size_t count) {
    if (count <= n && p) return FX_OK;
    release();
    if (count == 0) return FX_OK;
    cudaError_t e;
    if (g_alloc_stream) {
      e = cudaMallocAsync((void **)&p, count * sizeof(T), g_alloc_stream);
      pooled = true;
      owner = g_alloc_stream;
    } else {
      e = cudaMalloc((void **)&p, count * sizeof(T));
      pooled = false;
      owner = nullptr;
    }
    if (e != cudaSuccess) {
      p = nullptr;
      set_error("device allocation of %zu bytes: %s", count * sizeof(T),
                cudaGetErrorString(e));
      return FX_ENOMEM;
    }
    n = count;
    return FX_OK;
  }
  void release() {
    if (p) {
      if (pooled) cudaFreeAsync(p, owner);
      else cudaFree(p);
    }
    p = nullptr;
    n = 0;
    pooled = false;
    owner = nullptr;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// ---- per-stage timing ------------------------------------------------------
struct StageTimer {
  bool enabled = false;
  uint32_t mask = ~0u;  // stages timed while enabled (bit per FX_STAGE_*)
  double ms[FX_STAGE_COUNT] = {};
  int64_t calls[FX_STAGE_COUNT] = {};
  // Pending (start, stop) pairs, resolved lazily on query.
  struct Pending {
    int stage;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> pool;
  // Pairs recorded while a stream was being captured into a CUDA graph (as
  // event record nodes): they belong to that graph and are read after each
  // of its replays (add_elapsed), not resolved here.
  std::vector<Pending> captured;
  cudaEvent_t get_event();
  void resolve();
  void add_elapsed(const std::vector<Pending> &pairs);
  void destroy();
};

// ---- Barnes-Hut workspace ----------------------------------------------------
struct BHWork {
  int n = 0;
  DevBuf<uint32_t> keys[2];     // radix sort ping-pong (keys[0] = sorted)
  DevBuf<int32_t> idx[2];       // gate index payload (idx[0] = sorted order)
  DevBuf<uint32_t> tile_hist;   // radix sort: digit x tile counts
  DevBuf<uint32_t> tile_scan;   // per-digit exclusive scan of tile_hist
  DevBuf<uint32_t> digit_total; // 256 digit totals
  DevBuf<float2> spos;          // positions in sorted order
  DevBuf<int32_t> child;        // internal nodes: 2 children (leaf s -> ~s)
  DevBuf<int32_t> range;        // internal nodes: first, last
  DevBuf<int32_t> dnode;        // internal nodes: prefix length
  DevBuf<int32_t> dparent;      // internal nodes: parent's prefix length
  DevBuf<int4> qchild;          // internal nodes: up to 4 quad children
  DevBuf<ulonglong4> tile_fix;  // per-tile exact (x, y) sums, then offsets
  DevBuf<ulonglong4> prefix;    // inclusive exact prefix sums of spos (2 x int128)
  DevBuf<float4> node;          // internal nodes: 2 x float4 walk records
  DevBuf<float> root;           // {x_min, y_min, size, deep (1) or not (0)}
  // deep keys (levels 16..27) when a level-15 cell could be opened:
  DevBuf<uint32_t> klo;         // 24-bit sub-cell key per gate (gate order)
  DevBuf<uint32_t> kl[2];       // its radix sort ping-pong
  DevBuf<int32_t> il[2];        // gate index payload of that sort
  DevBuf<uint32_t> slo;         // sub-cell key in sorted order
  DevBuf<unsigned int> bbox;    // [0..3] ordered-int box, [4] error flag
  DevBuf<float2> force;         // per gate (original order)
  DevBuf<uint32_t> os_ws;       // one-sweep key sort: digit counts, look-back words
  template <class F>
  void for_each(F &&f) {
    f(os_ws);
    for (auto &b : keys) f(b);
    for (auto &b : idx) f(b);
    f(tile_hist); f(tile_scan); f(digit_total); f(spos); f(child); f(range);
    f(dnode); f(dparent); f(qchild); f(klo); f(kl[0]); f(kl[1]); f(il[0]); f(il[1]); f(slo);
    f(tile_fix); f(prefix); f(node); f(root); f(bbox); f(force);
  }
};

// ---- density (DCT Poisson) workspace -----------------------------------------
struct DensityWork {
  int G = 0;
  int precision = -1;
  DevBuf<unsigned long long> area_fx;  // fixed-point area per bin (G*G)
  DevBuf<float> cmat;                  // DCT-II ortho matrix C (G*G)
  DevBuf<float> cmat_t;                // C^T
  DevBuf<float> cmat_lo;               // C - tf32(C) for the 3xTF32 split
  DevBuf<float> cmat_t_lo;
  DevBuf<uint16_t> cmat_bf, cmat_t_bf; // bf16 copies
  DevBuf<float> inv_eig;               // -1/lambda with DC = 0 (G*G)
  DevBuf<float> dxct, dyct;            // stencil x C^T (field operators)
  DevBuf<float> dxct_lo, dyct_lo;
  DevBuf<uint16_t> dxct_bf, dyct_bf;
  DevBuf<float> buf[5];                // rho, T1^T/T3^T, phi_hat, phi, T4^T
  DevBuf<float> lo[4];                 // low parts for 3xTF32 operands
  DevBuf<uint16_t> bf[3];              // bf16 operand staging
  DevBuf<float> ex, ey;                // field
  DevBuf<double> energy;               // FP64 partials
  DevBuf<float2> force;                // per gate
  DevBuf<float> split_ws;              // SIMT split-K partial tiles
  // even/odd path (G a multiple of 256): the half operators
  // [C even rows | C odd rows], [C^T even cols | odd cols], Dx C^T, Dy C^T
  // likewise, each (G/2) x (G/2) pair in one buffer of G*G/2; and three
  // folded or split data operands of G*G each
  bool halves = false;
  DevBuf<float> c_h, ct_h, dx_h, dy_h;
  DevBuf<float> c_h_lo, ct_h_lo, dx_h_lo, dy_h_lo;      // 3xTF32 residuals
  DevBuf<uint16_t> c_h_bf, ct_h_bf, dx_h_bf, dy_h_bf;   // bf16 copies
  DevBuf<float> hw[3], hw_lo[3];
  DevBuf<uint16_t> hw_bf[3];
  // FX_DCT_I8: 8-bit slices (G x 4G) and row scales of the operators C, C^T,
  // Dx C^T, Dy C^T, and of two data operands at a time
  DevBuf<int8_t> op8[4], d8[2];
  DevBuf<float> op_sc[4], d_sc[2];
  template <class F>
  void for_each(F &&f) {
    f(area_fx); f(cmat); f(cmat_t); f(cmat_lo); f(cmat_t_lo); f(cmat_bf);
    f(cmat_t_bf); f(inv_eig); f(dxct); f(dyct); f(dxct_lo); f(dyct_lo);
    f(dxct_bf); f(dyct_bf);
    for (auto &b : buf) f(b);
    for (auto &b : lo) f(b);
    for (auto &b : bf) f(b);
    f(ex); f(ey); f(energy); f(force); f(split_ws);
    f(c_h); f(ct_h); f(dx_h); f(dy_h);
    f(c_h_lo); f(ct_h_lo); f(dx_h_lo); f(dy_h_lo);
    f(c_h_bf); f(ct_h_bf); f(dx_h_bf); f(dy_h_bf);
    for (auto &b : hw) f(b);
    for (auto &b : hw_lo) f(b);
    for (auto &b : hw_bf) f(b);
    for (auto &b : op8) f(b);
    for (auto &b : d8) f(b);
    for (auto &b : op_sc) f(b);
    for (auto &b : d_sc) f(b);
  }
};

// ---- congestion workspace ----------------------------------------------------
struct CongWork {
  int cols = 0, rows = 0;
  DevBuf<int32_t> diff;        // (rows+1) x (cols+1) difference array
  DevBuf<uint32_t> counts;     // rows x cols
  DevBuf<double> partial;      // per-block FP64 partial sums
  DevBuf<float> partial_max;
  DevBuf<unsigned int> done;   // last-block counters
  DevBuf<double> result;       // {hpwl, total_overflow}
  DevBuf<float> result_max;
  template <class F>
  void for_each(F &&f) {
    f(diff); f(counts); f(partial); f(partial_max); f(done); f(result);
    f(result_max);
  }
};

// ---- fused attraction/integrate step: cross-block reductions ------------------
struct StepWork {
  DevBuf<float4> bbox_part;     // per block {min x, min y, max x, max y}
  DevBuf<double> e_part;        // per block density energy
  DevBuf<unsigned int> done;    // last-block counter
  DevBuf<double> energy;        // result
  template <class F>
  void for_each(F &&f) {
    f(bbox_part); f(e_part); f(done); f(energy);
  }
};

// Statistics of fx_force_iterate, read back into pinned host memory.
struct IterReadback {
  double res[2];        // HPWL, total overflow
  double energy;        // density energy
  float max_overflow;
  unsigned int err;     // Barnes-Hut error word
  unsigned int tc_err;  // tensor-core GEMM error word
};

}  // namespace fx

struct fx_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;   // main stream
  cudaStream_t stream2 = nullptr;  // side stream (density || Barnes-Hut)
  cudaEvent_t fork = nullptr, join = nullptr;
  int num_sms = 0;
  // SMs the persistent leaf kernels spread over (0: all); a server's
  // placement contexts leave the rest to other jobs' kernels, whose blocks
  // could not start while a persistent grid holds every SM
  int persistent_sms = 0;
  // Error word of this context's tensor-core GEMMs (bit 1: a bounded wait
  // expired); zeroed at creation, cleared again after it is reported.
  unsigned int *tc_err = nullptr;
  fx::IterReadback *readback = nullptr;  // pinned host memory
  fx::IterReadback *readback_dev = nullptr;  // the same block, as the device addresses it
  fx::StageTimer timer;
  int64_t launches = 0;
  cudaEvent_t marks[16] = {};
  int leaf_schedule = 0;           // last autotuned leaf schedule
  // FX_LEAF_AUTO decisions by batch shape (leaf count, mean leaf size and
  // iteration count, each as a power-of-two bucket)
  std::unordered_map<uint32_t, int> leaf_tuned;
};

struct fx_design {
  fx_ctx *ctx = nullptr;
  int32_t n = 0, m = 0;
  int64_t p = 0, a = 0;
  float chip_w = 0.f, chip_h = 0.f;
  // netlist
  fx::DevBuf<int32_t> net_ptr, net_gate;
  fx::DevBuf<int32_t> adj_ptr, adj_idx;
  fx::DevBuf<float> area;        // w*h per gate
  std::vector<int32_t> h_adj_ptr, h_adj_idx;
  std::vector<float> h_w, h_h;
  // state: ping-pong positions, velocities
  fx::DevBuf<float> x[2], y[2];
  int cur = 0;
  fx::DevBuf<float> vx, vy;
  fx::DevBuf<float> saved[4];    // checkpoint: x, y, vx, vy
  // The positions are known to lie in [0, chip_w] x [0, chip_h] (set by the
  // box check of fx_design_set_positions and by every integration step, which
  // clamps to the die); with the saved copy's flag.
  bool pos_in_box = false, saved_in_box = false;
  fx::DevBuf<unsigned int> box_flag;
  fx::DevBuf<float2> fattr;      // attraction-only force output (stage API)
  // force trace (fx_design_trace): each plain iteration stores its total
  // force, start positions and start velocities (6 x n floats)
  bool trace_on = false;
  fx::DevBuf<float> trace;
  // and of fx_hapr_place_leaves: each slot's force in the first iteration
  fx::DevBuf<float2> leaf_trace;
  int32_t leaf_trace_n = 0;
  // workspaces
  fx::BHWork bh;
  fx::DensityWork dens;
  fx::CongWork cong;
  fx::StepWork step;
  // Single-iteration calls of fx_force_iterate on resident positions, as a
  // CUDA graph per ping-pong parity. `key` fingerprints what the graph was
  // captured with (configuration, context, the state flag the tree build
  // reads, and the address and size of every buffer it touches); `seen` is
  // the key an eager call left behind, so a second call with the same key
  // captures and later ones replay.
  // With stage timing on, the graph records its stages' events itself
  // (`timing`), read after every replay.
  struct IterGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> key, seen, failed;  // failed: a key whose capture failed
    int64_t launches = 0;
    std::vector<fx::StageTimer::Pending> timing;
    void reset() {
      if (exec) cudaGraphExecDestroy(exec);
      exec = nullptr;
      for (auto &t : timing) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
      }
      timing.clear();
    }
  } g1[2];
};

namespace fx {
// stage launchers (return FX_* codes), all on ctx->stream unless noted.
// Sizes the congestion scratch for a cols x rows grid (zeroed on s); a no-op
// when it already fits. congestion_run calls it; callers that capture the
// run into a CUDA graph call it first, outside the capture.
int congestion_alloc(fx_design *d, int cols, int rows, cudaStream_t s);
int congestion_run(fx_ctx *ctx, fx_design *d, const float *dx, const float *dy,
                   int cols, int rows, cudaStream_t s);
int attraction_run(fx_ctx *ctx, fx_design *d, float k, float2 *out, cudaStream_t s);
int bh_run(fx_ctx *ctx, fx_design *d, float k, float theta, float min_dist, int walk,
           cudaStream_t s, int32_t *term_count = nullptr);
int density_run(fx_ctx *ctx, fx_design *d, int G, float target, float weight,
                int precision, bool need_phi, cudaStream_t s);
int fused_step(fx_ctx *ctx, fx_design *d, const fx_iter_cfg &cfg,
               cudaStream_t s);
// Stable LSD radix sort of (key, value) pairs (fx_bh.cu).
int radix_sort_pairs(uint32_t *k[2], int32_t *v[2], int n, int passes,
                     uint32_t *tile_hist, uint32_t *tile_scan, uint32_t *digit_total,
                     cudaStream_t s);
int radix_sort_tiles(int n);
// The same sort in 1 + passes launches (decoupled look-back; fx_bh.cu): ws
// holds os_sort_words(n, passes) words; an expired look-back sets bit 4 of
// *err.
size_t os_sort_words(int n, int passes);
int radix_sort_onesweep(uint32_t *k[2], int32_t *v[2], int n, int passes, uint32_t *ws,
                        unsigned int *err, cudaStream_t s, const float *px = nullptr,
                        const float *py = nullptr, float2 *spos = nullptr);
// The Barnes-Hut error word (walk stack overflow, sort look-back) as a status.
int bh_error(unsigned int err);
// The reference's f32 Iterator::sum folds of the power iteration, one warp
// per cluster [beg[c], end[c]) (fx_partition.cu): with `deflate`, the mean
// of x is subtracted in place; nrm[c] = |x| when > 1e-10, else 0.
__global__ void part_seq_kernel(int C, const int32_t *__restrict__ beg,
                                const int32_t *__restrict__ end, float *__restrict__ x,
                                int deflate, float *__restrict__ nrm);
void timer_begin(fx_ctx *ctx, int stage, cudaStream_t s, cudaEvent_t *a);
void timer_end(fx_ctx *ctx, int stage, cudaStream_t s, cudaEvent_t a);
// Raises kernel `func`'s dynamic shared-memory limit on the current device to
// at least `bytes`. Under a lock and never downwards, so host threads that
// launch the kernel with different sizes cannot undo each other's setting.
int raise_smem_limit(const void *func, int bytes);
// Re-creates an idle context's streams at the given priorities (fx_core.cu).
int ctx_set_priorities(fx_ctx *c, int primary, int side);
}  // namespace fx
