// fx_serve.cu -- the request server: admission by device footprint,
// continuous batching of placement and ECO jobs over worker slots, resident
// designs.
//
// Each slot is a host thread with two fx_ctx (two non-blocking streams
// each): ECO jobs run on the slot's foreground context, PLACE jobs on its
// background one, whose streams have the lowest priority and whose
// persistent leaf kernels spread over half the SMs, so an ECO job's short
// kernels pass the queued kernels of running placements.
// A worker takes the first queued job that (a) fits in what the HBM budget
// has left and (b) does not wait on a design that is busy or not yet placed,
// runs it to completion on its context, and posts the result. Jobs therefore
// join the device as soon as a slot and memory free up, and the kernels of
// up to `slots` jobs overlap. Device buffers are stream-ordered allocations
// (DevBuf), so one job's allocations and frees do not stall the others.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fx_internal.h"

namespace fx {
namespace {

struct Job {
  int64_t id = 0;
  fx_job_desc desc{};  // pointers cleared; data below
  std::vector<int32_t> net_ptr, net_gate, move_gate;
  std::vector<float> w, h, move_dx, move_dy;
  fx_part_cfg part{};
  fx_leaf_cfg leaf{};
  fx_refine_cfg refine{};
  fx_iter_cfg iter{};
  bool has_iter = false;
  int64_t est = 0;
  fx_job_result res{};
};

struct Resident {
  fx_design *d = nullptr;
  int64_t bytes = 0;
  bool busy = false;
};

// ECO: move the listed gates, clamped to the die (the plain iteration's box).
__global__ void serve_move_kernel(int n, const int32_t *__restrict__ gate,
                                  const float *__restrict__ dx, const float *__restrict__ dy,
                                  float *__restrict__ x, float *__restrict__ y, float w,
                                  float h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = gate[i];
  x[g] = fminf(fmaxf(__fadd_rn(x[g], dx[i]), 0.f), w);
  y[g] = fminf(fmaxf(__fadd_rn(y[g], dy[i]), 0.f), h);
}

int32_t eco_bins(int32_t n) {
  int32_t g = (int32_t)std::lround(std::sqrt((double)n) / 128.0) * 128;
  return std::min(1024, std::max(128, g));
}

// Upper bound of the clique adjacency entries (sum of d(d-1) over nets).
int64_t adjacency_bound(int32_t m, const int32_t *net_ptr) {
  int64_t a = 0;
  for (int32_t e = 0; e < m; ++e) {
    const int64_t d = net_ptr[e + 1] - net_ptr[e];
    a += d * (d - 1);
  }
  return a;
}

int64_t estimate_place(int64_t n, int64_t m, int64_t p, int64_t a, const fx_refine_cfg &rc) {
  const int64_t cells = (int64_t)(rc.grid_cols + 1) * (rc.grid_rows + 1);
  return 4 * (m + 1) + 4 * p          // netlist
         + 4 * (n + 1) + 4 * a        // adjacency
         + 60 * n                     // area, positions (2 buffers), velocities, forces
         + 64 * n + 16 * (n / 2048 + 1) * 256  // partition work + sort tiles
         + 40 * n + 2 * a             // leaf batch (gate lists, in-leaf adjacency, outputs)
         + 8 * cells + 4 * 65536      // congestion grid and partials
         + ((int64_t)4 << 20);
}

int64_t estimate_eco(int64_t n, const fx_iter_cfg &it, int64_t moves) {
  const int64_t G = it.density_bins;
  const int64_t cells = (int64_t)(it.cong_cols + 1) * (it.cong_rows + 1);
  return 224 * n                      // Barnes-Hut work (keys, sub-keys, sort, tree, forces)
         + 120 * G * G                // density grids, operators, split copies
         + 8 * cells + 4 * 65536 + 16 * n  // congestion, step partials
         + 12 * moves + ((int64_t)4 << 20);
}

}  // namespace
}  // namespace fx

struct fx_server {
  fx_serve_cfg cfg{};
  std::vector<fx_ctx *> ctxs;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<fx::Job *> queue;
  std::deque<fx_job_result> done;
  std::unordered_map<int64_t, fx::Resident> designs;
  std::unordered_map<int64_t, int> pending_place;  // PLACE jobs queued or running
  int64_t reserved = 0;
  int64_t next_id = 1;
  int running = 0;
  bool stop = false;
  std::chrono::steady_clock::time_point t0;
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

using namespace fx;

namespace {

// Fills the job's defaults and admission estimate.
int prepare_job(Job &j, int64_t eco_n) {
  const fx_job_desc &in = j.desc;
  if (in.part) j.part = *in.part; else fx_part_cfg_default(&j.part);
  if (in.leaf) {
    j.leaf = *in.leaf;
  } else {
    // The leaf batch is most of a placement's device work; the server
    // places with the tolerance-mode forces (within 1e-5 of FP64, final HPWL
    // within 0.5 % of the reference's), a quarter of the IEEE schedule's time.
    fx_leaf_cfg_default(&j.leaf);
    j.leaf.precision = FX_LEAF_FAST;
  }
  if (in.refine) j.refine = *in.refine; else fx_refine_cfg_default(&j.refine);
  if (in.kind == FX_JOB_PLACE) {
    j.est = estimate_place(in.n_gates, in.n_nets, in.net_ptr[in.n_nets],
                           adjacency_bound(in.n_nets, in.net_ptr), j.refine);
  } else {
    if (in.iter) {
      j.iter = *in.iter;
    } else {
      fx_iter_cfg_default(&j.iter);
      j.iter.density_bins = eco_bins((int32_t)eco_n);
      // Below 1024 bins the FP32 CUDA-core products finish sooner than the
      // int8-slice ones (short K, few tiles); both are FP32-accurate.
      if (j.iter.density_bins < 1024) j.iter.dct_precision = FX_DCT_SIMT;
      j.iter.cong_cols = 256;
      j.iter.cong_rows = 256;
    }
    j.has_iter = true;
    j.est = estimate_eco(eco_n, j.iter, in.n_moves);
  }
  return FX_OK;
}

int validate_desc(const fx_job_desc *jd) {
  if (!jd || (jd->kind != FX_JOB_PLACE && jd->kind != FX_JOB_ECO)) return FX_EINVAL;
  if (jd->kind == FX_JOB_PLACE) {
    if (jd->n_gates <= 0 || jd->n_nets < 0 || !jd->net_ptr || (!jd->net_gate && jd->n_nets) ||
        !jd->gate_w || !jd->gate_h || !(jd->chip_w > 0.f) || !(jd->chip_h > 0.f))
      return FX_EINVAL;
  } else {
    if (jd->n_moves < 0 || jd->iterations < 0 ||
        (jd->n_moves > 0 && (!jd->move_gate || !jd->move_dx || !jd->move_dy)))
      return FX_EINVAL;
  }
  return FX_OK;
}

// PLACE: the main.rs flow on a new design.
int run_place(fx_ctx *ctx, Job &j, fx_design **out_d) {
  const fx_job_desc &in = j.desc;
  fx_design *d = nullptr;
  FX_TRY(fx_design_load(ctx, in.n_gates, in.n_nets, j.net_ptr.data(), j.net_gate.data(),
                        j.w.data(), j.h.data(), in.chip_w, in.chip_h, &d));
  const int32_t n = in.n_gates;
  std::vector<int32_t> lp((size_t)n + 2), lg((size_t)n), ld((size_t)n + 1);
  std::vector<float> rg(4 * ((size_t)n + 1));
  fx_part_stats ps{};
  int rc = fx_partition(ctx, d, &j.part, n + 1, lp.data(), lg.data(), rg.data(), ld.data(),
                        &ps);
  std::vector<float> x((size_t)n, 0.f), y((size_t)n, 0.f);
  if (rc == FX_OK)
    rc = fx_hapr_place_leaves(ctx, d, ps.n_leaves, lp.data(), lg.data(), rg.data(), &j.leaf,
                              x.data(), y.data(), nullptr);
  fx_refine_stats rs{};
  if (rc == FX_OK) rc = fx_refine(ctx, d, &j.refine, x.data(), y.data(), &rs, nullptr);
  if (rc != FX_OK) {
    fx_design_free(d);
    return rc;
  }
  j.res.n_leaves = ps.n_leaves;
  j.res.iterations = (int32_t)rs.iterations;
  j.res.hpwl = rs.hpwl;
  j.res.total_overflow = rs.total_overflow;
  j.res.max_overflow = rs.max_overflow;
  *out_d = d;
  return FX_OK;
}

// ECO: moves on the resident positions, then plain iterations.
int run_eco(fx_ctx *ctx, Job &j, fx_design *d) {
  d->ctx = ctx;  // the previous job on this design has finished and synchronised
  FX_CHECK_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const int32_t nm = j.desc.n_moves;
  if (nm > 0) {
    // the moves apply in parallel, so each gate may be listed once
    std::vector<uint8_t> listed((size_t)d->n, 0);
    for (int32_t i = 0; i < nm; ++i) {
      const int32_t g = j.move_gate[i];
      if (g < 0 || g >= d->n) {
        set_error("ECO move of gate %d outside the design", g);
        return FX_EINVAL;
      }
      if (listed[g]) {
        set_error("ECO moves list gate %d twice", g);
        return FX_EINVAL;
      }
      listed[g] = 1;
    }
    AllocScope as(s);
    DevBuf<int32_t> g;
    DevBuf<float> dx, dy;
    FX_TRY(g.alloc(nm));
    FX_TRY(dx.alloc(nm));
    FX_TRY(dy.alloc(nm));
    FX_CHECK_CUDA(cudaMemcpyAsync(g.p, j.move_gate.data(), (size_t)nm * 4,
                                  cudaMemcpyHostToDevice, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(dx.p, j.move_dx.data(), (size_t)nm * 4,
                                  cudaMemcpyHostToDevice, s));
    FX_CHECK_CUDA(cudaMemcpyAsync(dy.p, j.move_dy.data(), (size_t)nm * 4,
                                  cudaMemcpyHostToDevice, s));
    serve_move_kernel<<<(nm + 255) / 256, 256, 0, s>>>(nm, g.p, dx.p, dy.p, d->x[d->cur].p,
                                                       d->y[d->cur].p, d->chip_w, d->chip_h);
    FX_CHECK_LAUNCH();
    ctx->launches += 1;
  }
  fx_iter_stats st{};
  FX_TRY(fx_force_iterate(ctx, d, &j.iter, j.desc.iterations, nullptr, nullptr, &st));
  j.res.iterations = j.desc.iterations;
  j.res.hpwl = st.hpwl;
  j.res.total_overflow = st.total_overflow;
  j.res.max_overflow = st.max_overflow;
  return FX_OK;
}

// Under the lock: the first queued job that can start now.
Job *pick(fx_server *sv) {
  const int64_t budget = sv->cfg.hbm_budget_bytes;
  std::vector<int64_t> blocked;  // designs with an earlier job still waiting
  for (auto it = sv->queue.begin(); it != sv->queue.end(); ++it) {
    Job *j = *it;
    if (j->desc.kind == FX_JOB_ECO) {
      const int64_t did = j->desc.design_id;
      if (std::find(blocked.begin(), blocked.end(), did) != blocked.end()) continue;
      auto r = sv->designs.find(did);
      if (r == sv->designs.end()) {
        if (sv->pending_place.count(did)) {  // not placed yet
          blocked.push_back(did);
          continue;
        }
        sv->queue.erase(it);  // unknown design: fails at once
        return j;
      }
      if (r->second.busy || sv->reserved + j->est > budget) {
        blocked.push_back(did);
        continue;
      }
      r->second.busy = true;
    } else if (sv->reserved + j->est > budget) {
      continue;
    }
    sv->reserved += j->est;
    sv->queue.erase(it);
    return j;
  }
  return nullptr;
}

void worker(fx_server *sv, int slot) {
  fx_ctx *fg = sv->ctxs[2 * slot], *bg = sv->ctxs[2 * slot + 1];
  cudaSetDevice(fg->device);
  for (;;) {
    Job *j = nullptr;
    fx_design *eco_d = nullptr;
    {
      std::unique_lock<std::mutex> lock(sv->mu);
      sv->cv_work.wait(lock, [&] { return sv->stop || (j = pick(sv)) != nullptr; });
      if (!j) return;  // stopping
      ++sv->running;
      if (j->desc.kind == FX_JOB_ECO) {
        auto r = sv->designs.find(j->desc.design_id);
        if (r != sv->designs.end()) eco_d = r->second.d;
      }
    }
    j->res.start_s = sv->now();
    fx_ctx *ctx = j->desc.kind == FX_JOB_PLACE ? bg : fg;
    int rc = FX_OK;
    fx_design *placed = nullptr;
    if (j->desc.kind == FX_JOB_PLACE) {
      rc = run_place(ctx, *j, &placed);
    } else if (!eco_d) {
      set_error("ECO job for design %lld, which is not resident",
                (long long)j->desc.design_id);
      rc = FX_EINVAL;
    } else {
      rc = run_eco(ctx, *j, eco_d);
    }
    if (rc != FX_OK) std::snprintf(j->res.error, sizeof j->res.error, "%s", fx_last_error());
    j->res.status = rc;
    j->res.end_s = sv->now();
    int64_t placed_bytes = 0;
    if (placed) {
      if (j->desc.keep_resident) {
        placed_bytes = fx_design_device_bytes(placed);
      } else {
        fx_design_free(placed);
        placed = nullptr;
      }
    }
    int64_t eco_bytes = eco_d ? fx_design_device_bytes(eco_d) : 0;
    {
      std::lock_guard<std::mutex> lock(sv->mu);
      sv->reserved -= j->est;
      if (j->desc.kind == FX_JOB_PLACE) {
        sv->pending_place.erase(j->id);
        if (placed) {
          Resident r;
          r.d = placed;
          r.bytes = placed_bytes;
          sv->designs[j->id] = r;
          sv->reserved += placed_bytes;
        }
      } else if (eco_d) {
        Resident &r = sv->designs[j->desc.design_id];
        sv->reserved += eco_bytes - r.bytes;  // workspaces the iteration added
        r.bytes = eco_bytes;
        r.busy = false;
      }
      --sv->running;
      sv->done.push_back(j->res);
    }
    delete j;
    sv->cv_done.notify_all();
    sv->cv_work.notify_all();
  }
}

}  // namespace

extern "C" int fx_serve_cfg_default(fx_serve_cfg *c) {
  if (!c) return FX_EINVAL;
  c->device = 0;
  c->slots = 8;
  c->queue_capacity = 65536;
  c->reserved0 = 0;
  c->hbm_budget_bytes = 0;
  return FX_OK;
}

extern "C" int fx_serve_estimate(const fx_job_desc *jd, int64_t *out) {
  if (validate_desc(jd) != FX_OK || !out) {
    set_error("fx_serve_estimate: invalid job");
    return FX_EINVAL;
  }
  Job j;
  j.desc = *jd;
  FX_TRY(prepare_job(j, jd->n_gates));
  *out = j.est;
  return FX_OK;
}

extern "C" int fx_serve_create(const fx_serve_cfg *cfg, fx_server **out) {
  if (!cfg || !out || cfg->slots < 1 || cfg->slots > 256 || cfg->queue_capacity < 1 ||
      cfg->hbm_budget_bytes < 0) {
    set_error("fx_serve_create: invalid configuration");
    return FX_EINVAL;
  }
  *out = nullptr;
  fx_server *sv = new (std::nothrow) fx_server();
  if (!sv) return FX_ENOMEM;
  sv->cfg = *cfg;
  sv->t0 = std::chrono::steady_clock::now();
  int prio_low = 0, prio_high = 0;
  cudaSetDevice(cfg->device);
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  for (int i = 0; i < 2 * cfg->slots; ++i) {
    fx_ctx *c = nullptr;
    int rc = fx_ctx_create(&c, cfg->device);
    // odd contexts serve PLACE jobs: both streams at the lowest priority; the
    // foreground ones keep the highest for the Barnes-Hut chain and one step
    // above the lowest for the density stream
    if (rc == FX_OK)
      rc = (i & 1) ? ctx_set_priorities(c, prio_low, prio_low)
                   : ctx_set_priorities(c, prio_high, prio_low > prio_high ? prio_low - 1
                                                                           : prio_low);
    // and their persistent leaf kernels take half the SMs
    if (rc == FX_OK && (i & 1)) c->persistent_sms = std::max(1, c->num_sms / 2);
    if (rc != FX_OK) {
      if (c) fx_ctx_destroy(c);
      for (fx_ctx *x : sv->ctxs) fx_ctx_destroy(x);
      delete sv;
      return rc;
    }
    sv->ctxs.push_back(c);
  }
  if (sv->cfg.hbm_budget_bytes == 0) {
    size_t free_b = 0, total_b = 0;
    FX_CHECK_CUDA(cudaSetDevice(cfg->device));
    FX_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
    sv->cfg.hbm_budget_bytes = (int64_t)(0.8 * (double)free_b);
  }
  for (int i = 0; i < cfg->slots; ++i) sv->workers.emplace_back(worker, sv, i);
  *out = sv;
  return FX_OK;
}

extern "C" int fx_serve_destroy(fx_server *sv) {
  if (!sv) return FX_EINVAL;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
    for (Job *j : sv->queue) delete j;
    sv->queue.clear();
  }
  sv->cv_work.notify_all();
  for (auto &t : sv->workers) t.join();
  for (auto &kv : sv->designs) fx_design_free(kv.second.d);
  sv->designs.clear();
  for (fx_ctx *c : sv->ctxs) fx_ctx_destroy(c);
  delete sv;
  return FX_OK;
}

extern "C" int fx_serve_submit(fx_server *sv, const fx_job_desc *jd, int64_t *out_id) {
  if (!sv || validate_desc(jd) != FX_OK) {
    set_error("fx_serve_submit: invalid job");
    return FX_EINVAL;
  }
  Job *j = new (std::nothrow) Job();
  if (!j) return FX_ENOMEM;
  j->desc = *jd;
  if (jd->kind == FX_JOB_PLACE) {
    const int32_t n = jd->n_gates, m = jd->n_nets;
    j->net_ptr.assign(jd->net_ptr, jd->net_ptr + m + 1);
    if (m > 0) j->net_gate.assign(jd->net_gate, jd->net_gate + jd->net_ptr[m]);
    j->w.assign(jd->gate_w, jd->gate_w + n);
    j->h.assign(jd->gate_h, jd->gate_h + n);
  } else if (jd->n_moves > 0) {
    j->move_gate.assign(jd->move_gate, jd->move_gate + jd->n_moves);
    j->move_dx.assign(jd->move_dx, jd->move_dx + jd->n_moves);
    j->move_dy.assign(jd->move_dy, jd->move_dy + jd->n_moves);
  }
  j->desc.net_ptr = j->desc.net_gate = nullptr;
  j->desc.gate_w = j->desc.gate_h = nullptr;
  j->desc.move_gate = nullptr;
  j->desc.move_dx = j->desc.move_dy = nullptr;
  j->desc.part = nullptr;
  j->desc.leaf = nullptr;
  j->desc.refine = nullptr;
  j->desc.iter = nullptr;
  std::unique_lock<std::mutex> lock(sv->mu);
  int64_t eco_n = 0;
  if (jd->kind == FX_JOB_ECO) {
    auto r = sv->designs.find(jd->design_id);
    if (r != sv->designs.end()) {
      eco_n = r->second.d->n;
    } else if (sv->pending_place.count(jd->design_id)) {
      eco_n = sv->pending_place[jd->design_id];
    } else {
      delete j;
      set_error("fx_serve_submit: design %lld is not resident", (long long)jd->design_id);
      return FX_EINVAL;
    }
  }
  // the caller's configurations, read now
  {
    fx_job_desc tmp = *jd;
    Job probe;
    probe.desc = tmp;
    if (jd->kind == FX_JOB_PLACE) {
      probe.desc.net_ptr = j->net_ptr.data();
    }
    prepare_job(probe, eco_n);
    j->part = probe.part;
    j->leaf = probe.leaf;
    j->refine = probe.refine;
    j->iter = probe.iter;
    j->has_iter = probe.has_iter;
    j->est = probe.est;
  }
  if (j->est > sv->cfg.hbm_budget_bytes) {
    const long long e = (long long)j->est, b = (long long)sv->cfg.hbm_budget_bytes;
    delete j;
    set_error("fx_serve_submit: job needs about %lld bytes, the budget is %lld", e, b);
    return FX_EADMIT;
  }
  if ((int)sv->queue.size() >= sv->cfg.queue_capacity) {
    delete j;
    set_error("fx_serve_submit: queue full (%d jobs)", sv->cfg.queue_capacity);
    return FX_EADMIT;
  }
  j->id = sv->next_id++;
  j->res.job_id = j->id;
  j->res.kind = jd->kind;
  j->res.design_id = jd->kind == FX_JOB_PLACE ? j->id : jd->design_id;
  j->res.n_gates = jd->kind == FX_JOB_PLACE ? jd->n_gates : (int32_t)eco_n;
  j->res.est_bytes = j->est;
  j->res.submit_s = sv->now();
  if (jd->kind == FX_JOB_PLACE) sv->pending_place[j->id] = jd->n_gates;
  sv->queue.push_back(j);
  if (out_id) *out_id = j->id;
  lock.unlock();
  sv->cv_work.notify_one();
  return FX_OK;
}

extern "C" int fx_serve_poll(fx_server *sv, int32_t wait_ms, fx_job_result *out) {
  if (!sv || !out) return FX_EINVAL;
  std::unique_lock<std::mutex> lock(sv->mu);
  auto ready = [&] {
    return !sv->done.empty() || (wait_ms < 0 && sv->queue.empty() && sv->running == 0);
  };
  if (wait_ms < 0) {
    sv->cv_done.wait(lock, ready);
  } else if (wait_ms > 0) {
    sv->cv_done.wait_for(lock, std::chrono::milliseconds(wait_ms), ready);
  }
  if (sv->done.empty()) return 0;
  *out = sv->done.front();
  sv->done.pop_front();
  return 1;
}

extern "C" int fx_serve_positions(fx_server *sv, int64_t design_id, float *x, float *y) {
  if (!sv || !x || !y) return FX_EINVAL;
  std::unique_lock<std::mutex> lock(sv->mu);
  for (;;) {
    auto r = sv->designs.find(design_id);
    if (r == sv->designs.end()) {
      set_error("fx_serve_positions: design %lld is not resident", (long long)design_id);
      return FX_EINVAL;
    }
    if (!r->second.busy) {
      r->second.busy = true;
      fx_design *d = r->second.d;
      lock.unlock();
      const int rc = fx_design_get_positions(d, x, y);
      lock.lock();
      sv->designs[design_id].busy = false;
      lock.unlock();
      sv->cv_work.notify_all();
      return rc;
    }
    sv->cv_done.wait(lock);
  }
}

extern "C" int fx_serve_release(fx_server *sv, int64_t design_id) {
  if (!sv) return FX_EINVAL;
  std::unique_lock<std::mutex> lock(sv->mu);
  for (;;) {
    auto r = sv->designs.find(design_id);
    if (r == sv->designs.end()) {
      set_error("fx_serve_release: design %lld is not resident", (long long)design_id);
      return FX_EINVAL;
    }
    if (!r->second.busy) {
      fx_design *d = r->second.d;
      sv->reserved -= r->second.bytes;
      sv->designs.erase(r);
      lock.unlock();
      const int rc = fx_design_free(d);
      sv->cv_work.notify_all();
      return rc;
    }
    sv->cv_done.wait(lock);
  }
}

extern "C" int fx_serve_stats(fx_server *sv, int64_t *reserved, int32_t *queued,
                              int32_t *running, int32_t *resident, int64_t *launches) {
  if (!sv) return FX_EINVAL;
  std::lock_guard<std::mutex> lock(sv->mu);
  if (launches) {  // kernels launched by all worker contexts so far
    int64_t l = 0;
    for (fx_ctx *c : sv->ctxs) l += c->launches;
    *launches = l;
  }
  if (reserved) *reserved = sv->reserved;
  if (queued) *queued = (int32_t)sv->queue.size();
  if (running) *running = sv->running;
  if (resident) *resident = (int32_t)sv->designs.size();
  return FX_OK;
}
