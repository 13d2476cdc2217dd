// fx_oracle.cpp -- CPU oracle for the HAPR placement hot path.
//
// TEST INFRASTRUCTURE ONLY. This file restates the reference's Rust CPU path
// (HAPR_fluxion_v4/src, written H/ below) in plain C++ so the CUDA product
// can be checked against it. Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load it; the product never does.
//
// Build: g++ -O2 -std=c++17 -ffp-contract=off (no FMA contraction, no
// fast-math), which keeps Rust's IEEE f32 semantics: Rust never contracts
// a*b+c into an FMA. Every function cites the reference lines it follows.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <chrono>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <thread>

// Static-chunked parallel loop over [0, n) on `threads` std::threads (1 = run
// inline). Used only to make the CPU baseline use the host's cores.
template <typename F>
static void par_for(int32_t n, int32_t threads, F f) {
  if (threads <= 1 || n < 1024) {
    for (int32_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> pool;
  for (int32_t t = 0; t < threads; ++t)
    pool.emplace_back([=, &f] {
      for (int32_t i = t; i < n; i += threads) f(i);
    });
  for (auto &th : pool) th.join();
}

// Rust f32::clamp (NaN passes through).
static inline float rust_clamp(float v, float lo, float hi) {
  if (v < lo) v = lo;
  if (v > hi) v = hi;
  return v;
}

extern "C" {

// ---------------------------------------------------------------------------
// H/src/data/grid.rs:58-62  cell_at: `((x / self.cell_width) as usize)
// .min(self.cols - 1)`. Rust's float->usize cast saturates: NaN and values
// <= -1 .. 0 give 0, values >= 2^64 give usize::MAX; otherwise truncation.
static uint64_t rust_f32_as_usize(float q) {
  if (q != q) return 0;
  if (q <= 0.0f) return 0;  // (-1, 0] truncates to 0; below saturates to 0
  if (q >= 18446744073709551616.0f) return UINT64_MAX;
  return (uint64_t)q;
}

int64_t or_cell_at(float v, float cell, int64_t n) {
  uint64_t c = rust_f32_as_usize(v / cell);
  uint64_t m = (uint64_t)(n - 1);
  return (int64_t)(c < m ? c : m);
}

// H/src/data/grid.rs:25-32  RoutingGrid::new geometry.
void or_grid_geometry(float chip_w, float chip_h, int64_t cols, int64_t rows,
                      float *cell_w, float *cell_h, float *capacity) {
  const float cw = chip_w / (float)cols;
  const float ch = chip_h / (float)rows;
  *cell_w = cw;
  *cell_h = ch;
  *capacity = (cw + ch) * 0.5f;
}

// H/src/algorithm/congestion.rs:11-62  compute_congestion_cpu, literally:
// two f32 grids, +1.0 per covered cell, h loop row-major, v loop col-major.
void or_congestion(int32_t m, const int32_t *net_ptr, const int32_t *net_gate,
                   const float *x, const float *y, float chip_w, float chip_h,
                   int64_t cols, int64_t rows, float *h, float *v) {
  float cw, ch, cap;
  or_grid_geometry(chip_w, chip_h, cols, rows, &cw, &ch, &cap);
  const size_t cells = (size_t)(cols * rows);
  std::fill(h, h + cells, 0.0f);  // grid.clear() (grid.rs:44-47)
  std::fill(v, v + cells, 0.0f);
  for (int32_t e = 0; e < m; ++e) {
    const int32_t b = net_ptr[e], t = net_ptr[e + 1];
    if (t - b < 2) continue;
    float min_x = 3.40282347e+38f, max_x = -3.40282347e+38f;
    float min_y = 3.40282347e+38f, max_y = -3.40282347e+38f;
    for (int32_t q = b; q < t; ++q) {
      const float px = x[net_gate[q]], py = y[net_gate[q]];
      min_x = std::fmin(min_x, px);
      max_x = std::fmax(max_x, px);
      min_y = std::fmin(min_y, py);
      max_y = std::fmax(max_y, py);
    }
    const int64_t min_col = or_cell_at(min_x, cw, cols);
    const int64_t min_row = or_cell_at(min_y, ch, rows);
    const int64_t max_col = or_cell_at(max_x, cw, cols);
    const int64_t max_row = or_cell_at(max_y, ch, rows);
    for (int64_t r = min_row; r <= max_row; ++r)
      for (int64_t c = min_col; c <= max_col; ++c) {
        const size_t idx = (size_t)(r * cols + c);
        if (idx < cells) h[idx] += 1.0f;
      }
    for (int64_t c = min_col; c <= max_col; ++c)
      for (int64_t r = min_row; r <= max_row; ++r) {
        const size_t idx = (size_t)(r * cols + c);
        if (idx < cells) v[idx] += 1.0f;
      }
  }
}

// The counts of compute_congestion_cpu (h == v) for large netlists: the same
// bounding boxes and cell_at, with each covered rectangle added through a
// 2-D difference array and prefix sums (O(nets + cells) instead of
// O(sum of rectangle areas)); checked against or_congestion by the tests.
void or_congestion_counts(int32_t m, const int32_t *net_ptr, const int32_t *net_gate,
                          const float *x, const float *y, float chip_w, float chip_h,
                          int64_t cols, int64_t rows, uint32_t *counts) {
  float cw, ch, cap;
  or_grid_geometry(chip_w, chip_h, cols, rows, &cw, &ch, &cap);
  const int64_t ld = cols + 1;
  std::vector<int64_t> diff((size_t)(ld * (rows + 1)), 0);
  for (int32_t e = 0; e < m; ++e) {
    const int32_t b = net_ptr[e], t = net_ptr[e + 1];
    if (t - b < 2) continue;
    float min_x = 3.40282347e+38f, max_x = -3.40282347e+38f;
    float min_y = 3.40282347e+38f, max_y = -3.40282347e+38f;
    for (int32_t q = b; q < t; ++q) {
      const float px = x[net_gate[q]], py = y[net_gate[q]];
      min_x = std::fmin(min_x, px);
      max_x = std::fmax(max_x, px);
      min_y = std::fmin(min_y, py);
      max_y = std::fmax(max_y, py);
    }
    const int64_t c0 = or_cell_at(min_x, cw, cols), r0 = or_cell_at(min_y, ch, rows);
    const int64_t c1 = or_cell_at(max_x, cw, cols), r1 = or_cell_at(max_y, ch, rows);
    if (c0 > c1 || r0 > r1) continue;
    diff[(size_t)(r0 * ld + c0)] += 1;
    diff[(size_t)(r0 * ld + c1 + 1)] -= 1;
    diff[(size_t)((r1 + 1) * ld + c0)] -= 1;
    diff[(size_t)((r1 + 1) * ld + c1 + 1)] += 1;
  }
  for (int64_t r = 0; r <= rows; ++r)
    for (int64_t c = 1; c <= cols; ++c) diff[(size_t)(r * ld + c)] += diff[(size_t)(r * ld + c - 1)];
  for (int64_t r = 1; r <= rows; ++r)
    for (int64_t c = 0; c <= cols; ++c) diff[(size_t)(r * ld + c)] += diff[(size_t)((r - 1) * ld + c)];
  for (int64_t r = 0; r < rows; ++r)
    for (int64_t c = 0; c < cols; ++c) counts[(size_t)(r * cols + c)] = (uint32_t)diff[(size_t)(r * ld + c)];
}

// compute_congestion_cpu restricted to nets e with e % stride == 0 (the grids
// are cleared first). Used to time a bounded sample of the reference's
// congestion loop; the full call is stride 1.
void or_congestion_sample(int32_t m, const int32_t *net_ptr,
                          const int32_t *net_gate, const float *x,
                          const float *y, float chip_w, float chip_h,
                          int64_t cols, int64_t rows, int32_t stride, float *h,
                          float *v) {
  float cw, ch, cap;
  or_grid_geometry(chip_w, chip_h, cols, rows, &cw, &ch, &cap);
  const size_t cells = (size_t)(cols * rows);
  std::fill(h, h + cells, 0.0f);
  std::fill(v, v + cells, 0.0f);
  for (int32_t e = 0; e < m; e += stride) {
    const int32_t b = net_ptr[e], t = net_ptr[e + 1];
    if (t - b < 2) continue;
    float min_x = 3.40282347e+38f, max_x = -3.40282347e+38f;
    float min_y = 3.40282347e+38f, max_y = -3.40282347e+38f;
    for (int32_t q = b; q < t; ++q) {
      const float px = x[net_gate[q]], py = y[net_gate[q]];
      min_x = std::fmin(min_x, px);
      max_x = std::fmax(max_x, px);
      min_y = std::fmin(min_y, py);
      max_y = std::fmax(max_y, py);
    }
    const int64_t c0 = or_cell_at(min_x, cw, cols), r0 = or_cell_at(min_y, ch, rows);
    const int64_t c1 = or_cell_at(max_x, cw, cols), r1 = or_cell_at(max_y, ch, rows);
    for (int64_t r = r0; r <= r1; ++r)
      for (int64_t c = c0; c <= c1; ++c) {
        const size_t idx = (size_t)(r * cols + c);
        if (idx < cells) h[idx] += 1.0f;
      }
    for (int64_t c = c0; c <= c1; ++c)
      for (int64_t r = r0; r <= r1; ++r) {
        const size_t idx = (size_t)(r * cols + c);
        if (idx < cells) v[idx] += 1.0f;
      }
  }
}

// H/src/data/grid.rs:71-91  overflow_at / max_overflow / total_overflow.
void or_overflow(const float *h, const float *v, int64_t cols, int64_t rows,
                 float capacity, float *total, float *maxv) {
  float t = 0.0f, mx = 0.0f;
  for (int64_t r = 0; r < rows; ++r)
    for (int64_t c = 0; c < cols; ++c) {
      const size_t idx = (size_t)(r * cols + c);
      const float tot = h[idx] + v[idx];
      float ov = tot - capacity;
      ov = std::fmax(ov, 0.0f);  // f32::max(0.0)
      t += ov;
      mx = std::fmax(mx, ov);
    }
  *total = t;
  *maxv = mx;
}

// H/src/data/placement.rs:48-74  compute_hpwl, literally (f32 running sum).
float or_hpwl_f32(int32_t m, const int32_t *net_ptr, const int32_t *net_gate,
                  const float *x, const float *y) {
  float total = 0.0f;
  for (int32_t e = 0; e < m; ++e) {
    const int32_t b = net_ptr[e], t = net_ptr[e + 1];
    if (t - b < 2) continue;
    float min_x = 3.40282347e+38f, max_x = -3.40282347e+38f;
    float min_y = 3.40282347e+38f, max_y = -3.40282347e+38f;
    for (int32_t q = b; q < t; ++q) {
      const float px = x[net_gate[q]], py = y[net_gate[q]];
      min_x = std::fmin(min_x, px);
      max_x = std::fmax(max_x, px);
      min_y = std::fmin(min_y, py);
      max_y = std::fmax(max_y, py);
    }
    total += (max_x - min_x) + (max_y - min_y);
  }
  return total;
}

// FP64 twin of compute_hpwl: same per-net f32 extremes, FP64 sum.
double or_hpwl_f64(int32_t m, const int32_t *net_ptr, const int32_t *net_gate,
                   const float *x, const float *y) {
  double total = 0.0;
  for (int32_t e = 0; e < m; ++e) {
    const int32_t b = net_ptr[e], t = net_ptr[e + 1];
    if (t - b < 2) continue;
    float min_x = 3.40282347e+38f, max_x = -3.40282347e+38f;
    float min_y = 3.40282347e+38f, max_y = -3.40282347e+38f;
    for (int32_t q = b; q < t; ++q) {
      const float px = x[net_gate[q]], py = y[net_gate[q]];
      min_x = std::fmin(min_x, px);
      max_x = std::fmax(max_x, px);
      min_y = std::fmin(min_y, py);
      max_y = std::fmax(max_y, py);
    }
    total += ((double)max_x - (double)min_x) + ((double)max_y - (double)min_y);
  }
  return total;
}

// H/src/algorithm/refiner.rs:34-126  refine_placement, literally: congestion,
// f32 total overflow, stop / stall rules, then every gate in a hot cell
// (gates_in_hot_cells, congestion.rs:77-93) moves toward the first
// least-congested cell within radius 3 (move_gate_from_hot_cell), against
// the grid of that iteration. x/y are updated in place. Returns the
// iterations that moved gates; out[0..2] = final total overflow, max
// overflow, f32 HPWL (placement.rs:48-74).
int32_t or_refine(int32_t n, int32_t m, const int32_t *net_ptr,
                  const int32_t *net_gate, float *x, float *y, float chip_w,
                  float chip_h, int32_t max_iters, float move_distance,
                  float threshold, int64_t cols, int64_t rows, float *out) {
  float cw, ch, cap;
  or_grid_geometry(chip_w, chip_h, cols, rows, &cw, &ch, &cap);
  const size_t cells = (size_t)(cols * rows);
  std::vector<float> h(cells), v(cells);
  std::vector<char> hot(cells);
  float prev = 3.40282347e+38f;
  int32_t stall = 0, moved_iters = 0;
  for (int32_t it = 0; it < max_iters; ++it) {
    or_congestion(m, net_ptr, net_gate, x, y, chip_w, chip_h, cols, rows, h.data(),
                  v.data());
    float total, mx;
    or_overflow(h.data(), v.data(), cols, rows, cap, &total, &mx);
    if (total <= threshold) break;
    if (std::fabs(prev - total) < 0.01f * std::fmax(prev, 1.0f)) {
      if (++stall >= 10) break;
    } else {
      stall = 0;
    }
    prev = total;
    for (size_t i = 0; i < cells; ++i) {
      float ov = (h[i] + v[i]) - cap;
      ov = std::fmax(ov, 0.0f);
      hot[i] = ov > threshold;
    }
    for (int32_t g = 0; g < n; ++g) {
      const float gx = x[g], gy = y[g];
      const int64_t col = or_cell_at(gx, cw, cols), row = or_cell_at(gy, ch, rows);
      if (!hot[(size_t)(row * cols + col)]) continue;
      bool found = false;
      int64_t bc = 0, br = 0;
      float best = 0.0f;
      for (int64_t dr = -3; dr <= 3; ++dr)
        for (int64_t dc = -3; dc <= 3; ++dc) {
          if (dr == 0 && dc == 0) continue;
          const int64_t nc = col + dc, nr = row + dr;
          if (nc < 0 || nc >= cols || nr < 0 || nr >= rows) continue;
          const size_t idx = (size_t)(nr * cols + nc);
          const float tot = h[idx] + v[idx];
          if (!found || tot < best) {  // min_by keeps the first minimum
            found = true;
            best = tot;
            bc = nc;
            br = nr;
          }
        }
      if (!found) continue;
      const float tx = ((float)bc + 0.5f) * cw, ty = ((float)br + 0.5f) * ch;
      const float dx = rust_clamp(tx - gx, -move_distance, move_distance);
      const float dy = rust_clamp(ty - gy, -move_distance, move_distance);
      x[g] = rust_clamp(gx + dx, 0.0f, chip_w);
      y[g] = rust_clamp(gy + dy, 0.0f, chip_h);
    }
    ++moved_iters;
  }
  or_congestion(m, net_ptr, net_gate, x, y, chip_w, chip_h, cols, rows, h.data(),
                v.data());
  or_overflow(h.data(), v.data(), cols, rows, cap, &out[0], &out[1]);
  out[2] = or_hpwl_f32(m, net_ptr, net_gate, x, y);
  return moved_iters;
}

// H/src/data/circuit.rs:154-171  build_adjacency, literally: for every net,
// every pair i < j, push each endpoint into the other's list unless it is
// already there (Vec::contains). Returns the entry count; writes at most
// `cap` entries.
int64_t or_build_adjacency(int32_t n, int32_t m, const int32_t *net_ptr,
                           const int32_t *net_gate, int32_t *adj_ptr,
                           int32_t *adj_idx, int64_t cap) {
  std::vector<std::vector<int32_t>> adj((size_t)n);
  for (int32_t e = 0; e < m; ++e) {
    const int32_t b = net_ptr[e], t = net_ptr[e + 1];
    for (int32_t i = b; i < t; ++i)
      for (int32_t j = i + 1; j < t; ++j) {
        const int32_t a = net_gate[i], c = net_gate[j];
        auto &la = adj[(size_t)a];
        if (std::find(la.begin(), la.end(), c) == la.end()) la.push_back(c);
        auto &lc = adj[(size_t)c];
        if (std::find(lc.begin(), lc.end(), a) == lc.end()) lc.push_back(a);
      }
  }
  int64_t total = 0;
  adj_ptr[0] = 0;
  for (int32_t g = 0; g < n; ++g) {
    for (int32_t j : adj[(size_t)g]) {
      if (total < cap) adj_idx[total] = j;
      ++total;
    }
    adj_ptr[g + 1] = (int32_t)total;
  }
  return total;
}

// H/src/algorithm/placer.rs:243-255 over the full adjacency, f32 in the
// reference's order: fx[i] += k * (x[j] - x[i]) per neighbour.
void or_attraction_f32(int32_t n, const int32_t *adj_ptr, const int32_t *adj_idx,
                       const float *x, const float *y, float k, float *fx,
                       float *fy) {
  for (int32_t i = 0; i < n; ++i) {
    float ax = 0.0f, ay = 0.0f;
    for (int32_t q = adj_ptr[i]; q < adj_ptr[i + 1]; ++q) {
      const int32_t j = adj_idx[q];
      const float dx = x[j] - x[i];
      const float dy = y[j] - y[i];
      ax += k * dx;
      ay += k * dy;
    }
    fx[i] = ax;
    fy[i] = ay;
  }
}

// FP64 recomputation of the same sum.
void or_attraction_f64(int32_t n, const int32_t *adj_ptr, const int32_t *adj_idx,
                       const float *x, const float *y, double k, double *fx,
                       double *fy) {
  for (int32_t i = 0; i < n; ++i) {
    double ax = 0.0, ay = 0.0;
    for (int32_t q = adj_ptr[i]; q < adj_ptr[i + 1]; ++q) {
      const int32_t j = adj_idx[q];
      ax += (double)x[j] - (double)x[i];
      ay += (double)y[j] - (double)y[i];
    }
    fx[i] = k * ax;
    fy[i] = k * ay;
  }
}

// H/src/algorithm/placer.rs:275-280  damped Euler step with clamp to the
// box [xlo, xhi] x [ylo, yhi] (Rust clamp: NaN passes through).

void or_integrate(int32_t n, float *x, float *y, float *vx, float *vy,
                  const float *fx, const float *fy, float dt, float damping,
                  float xlo, float ylo, float xhi, float yhi) {
  for (int32_t i = 0; i < n; ++i) {
    vx[i] = (vx[i] + fx[i] * dt) * damping;
    vy[i] = (vy[i] + fy[i] * dt) * damping;
    x[i] = rust_clamp(x[i] + vx[i] * dt, xlo, xhi);
    y[i] = rust_clamp(y[i] + vy[i] * dt, ylo, yhi);
  }
}

// H/src/algorithm/placer.rs:210-287  place_gates_in_leaf, literally. Writes
// the leaf's final positions into the global arrays out_x/out_y.
void or_place_leaf(int32_t n, const int32_t *gates, const int32_t *adj_ptr,
                   const int32_t *adj_idx, float cx, float cy, float w, float h,
                   int32_t iters, float attract, float repel, float damping,
                   float dt, float *out_x, float *out_y) {
  if (n == 0) return;
  const float half_w = w / 2.0f, half_h = h / 2.0f;
  const float min_x = cx - half_w, min_y = cy - half_h;
  std::vector<float> px((size_t)n), py((size_t)n), vx((size_t)n, 0.0f),
      vy((size_t)n, 0.0f), fx((size_t)n), fy((size_t)n);
  for (int32_t i = 0; i < n; ++i) {
    px[i] = min_x + ((float)i / (float)n) * w;
    py[i] = min_y + ((float)((int64_t)i * 7 % n) / (float)n) * h;
  }
  std::unordered_map<int32_t, int32_t> g2l;
  for (int32_t i = 0; i < n; ++i) g2l[gates[i]] = i;
  for (int32_t it = 0; it < iters; ++it) {
    std::fill(fx.begin(), fx.end(), 0.0f);
    std::fill(fy.begin(), fy.end(), 0.0f);
    for (int32_t gi = 0; gi < n; ++gi) {
      const int32_t g = gates[gi];
      const int32_t li = g2l[g];
      for (int32_t q = adj_ptr[g]; q < adj_ptr[g + 1]; ++q) {
        auto f = g2l.find(adj_idx[q]);
        if (f == g2l.end()) continue;
        const int32_t lj = f->second;
        const float dx = px[lj] - px[li];
        const float dy = py[lj] - py[li];
        fx[li] += attract * dx;
        fy[li] += attract * dy;
      }
    }
    for (int32_t i = 0; i < n; ++i)
      for (int32_t j = i + 1; j < n; ++j) {
        const float dx = px[i] - px[j];
        const float dy = py[i] - py[j];
        const float dist_sq = dx * dx + dy * dy;
        const float dist = std::fmax(std::sqrt(dist_sq), 0.1f);
        const float force = repel / (dist * dist);
        const float fx_ij = force * dx / dist;
        const float fy_ij = force * dy / dist;
        fx[i] += fx_ij;
        fy[i] += fy_ij;
        fx[j] -= fx_ij;
        fy[j] -= fy_ij;
      }
    for (int32_t i = 0; i < n; ++i) {
      vx[i] = (vx[i] + fx[i] * dt) * damping;
      vy[i] = (vy[i] + fy[i] * dt) * damping;
      px[i] = rust_clamp(px[i] + vx[i] * dt, min_x, min_x + w);
      py[i] = rust_clamp(py[i] + vy[i] * dt, min_y, min_y + h);
    }
  }
  for (int32_t i = 0; i < n; ++i) {
    out_x[gates[i]] = px[i];
    out_y[gates[i]] = py[i];
  }
}

// One force evaluation of place_gates_in_leaf in FP64 from given local
// positions (attraction within the leaf + all-pairs repulsion), for the
// per-iteration force check of the batched leaf kernel.
void or_leaf_forces_f64(int32_t n, const int32_t *gates, const int32_t *adj_ptr,
                        const int32_t *adj_idx, const float *px,
                        const float *py, double attract, double repel,
                        double *fx, double *fy) {
  std::unordered_map<int32_t, int32_t> g2l;
  for (int32_t i = 0; i < n; ++i) g2l[gates[i]] = i;
  for (int32_t i = 0; i < n; ++i) fx[i] = fy[i] = 0.0;
  for (int32_t i = 0; i < n; ++i) {
    const int32_t g = gates[i];
    for (int32_t q = adj_ptr[g]; q < adj_ptr[g + 1]; ++q) {
      auto f = g2l.find(adj_idx[q]);
      if (f == g2l.end()) continue;
      fx[i] += attract * ((double)px[f->second] - (double)px[i]);
      fy[i] += attract * ((double)py[f->second] - (double)py[i]);
    }
  }
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = i + 1; j < n; ++j) {
      const double dx = (double)px[i] - px[j], dy = (double)py[i] - py[j];
      const double dist = std::max(std::sqrt(dx * dx + dy * dy), 0.1);
      const double f = repel / (dist * dist);
      fx[i] += f * dx / dist;
      fy[i] += f * dy / dist;
      fx[j] -= f * dx / dist;
      fy[j] -= f * dy / dist;
    }
}

// ---------------------------------------------------------------------------
// Hierarchy: H/src/algorithm/partitioner.rs:36-213 and the region assignment
// of H/src/algorithm/placer.rs:34-74,111-141, literally.
struct ONode {
  int32_t id, depth;
  std::vector<int32_t> gates;
  std::vector<ONode> children;
  float cx = 0.f, cy = 0.f, w = 0.f, h = 0.f;
};

// partitioner.rs:106-185 compute_fiedler_vector.
static std::vector<float> fiedler(const int32_t *adj_ptr, const int32_t *adj_idx,
                                  const std::vector<int32_t> &gi, int32_t iters) {
  const size_t n = gi.size();
  if (n <= 1) return std::vector<float>(n, 0.0f);
  std::unordered_map<int32_t, int32_t> g2l;
  for (size_t l = 0; l < n; ++l) g2l[gi[l]] = (int32_t)l;
  std::vector<float> degree(n, 0.0f);
  std::vector<std::pair<int32_t, int32_t>> pairs;
  for (int32_t g : gi)
    for (int32_t q = adj_ptr[g]; q < adj_ptr[g + 1]; ++q) {
      auto f = g2l.find(adj_idx[q]);
      if (f == g2l.end()) continue;
      const int32_t lg = g2l[g];
      pairs.push_back({lg, f->second});
      degree[(size_t)lg] += 1.0f;
    }
  std::vector<float> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = std::sin((float)i * 2.71828f);
  float norm = 0.0f;
  for (float a : v) norm += a * a;
  norm = std::sqrt(norm);
  if (norm > 1e-10f)
    for (float &a : v) a /= norm;
  std::vector<float> lv(n);
  for (int32_t it = 0; it < iters; ++it) {
    for (size_t i = 0; i < n; ++i) lv[i] = degree[i] * v[i];
    for (auto &p : pairs) lv[(size_t)p.first] -= v[(size_t)p.second];
    float sum = 0.0f;
    for (float a : lv) sum += a;
    const float mean = sum / (float)n;
    for (float &a : lv) a -= mean;
    float nn = 0.0f;
    for (float a : lv) nn += a * a;
    nn = std::sqrt(nn);
    if (nn > 1e-10f)
      for (float &a : lv) a /= nn;
    v.swap(lv);
  }
  return v;
}

static ONode bisect(const int32_t *adj_ptr, const int32_t *adj_idx,
                    const std::vector<int32_t> &gi, int32_t depth,
                    int32_t max_leaf, int32_t min_cluster, float balance,
                    int32_t iters, int32_t &next_id) {
  ONode node;
  node.id = next_id++;
  node.depth = depth;
  node.gates = gi;
  if ((int32_t)gi.size() <= max_leaf || (int32_t)gi.size() <= min_cluster)
    return node;
  std::vector<float> f = fiedler(adj_ptr, adj_idx, gi, iters);
  // partitioner.rs:189-213 split_by_fiedler (stable sort, balanced split).
  const size_t n = gi.size();
  std::vector<std::pair<int32_t, float>> idx(n);
  for (size_t i = 0; i < n; ++i) idx[i] = {gi[i], f[i]};
  std::stable_sort(idx.begin(), idx.end(),
                   [](const std::pair<int32_t, float> &a,
                      const std::pair<int32_t, float> &b) { return a.second < b.second; });
  const size_t min_size = (size_t)std::ceil((float)n * balance);
  size_t split = n / 2;
  split = std::max(split, min_size);
  split = std::min(split, n - min_size);
  std::vector<int32_t> left, right;
  for (size_t i = 0; i < split; ++i) left.push_back(idx[i].first);
  for (size_t i = split; i < n; ++i) right.push_back(idx[i].first);
  if (left.empty() || right.empty()) return node;
  node.children.push_back(bisect(adj_ptr, adj_idx, left, depth + 1, max_leaf,
                                 min_cluster, balance, iters, next_id));
  node.children.push_back(bisect(adj_ptr, adj_idx, right, depth + 1, max_leaf,
                                 min_cluster, balance, iters, next_id));
  return node;
}

static int32_t max_depth_of(const ONode &n) {
  if (n.children.empty()) return n.depth;
  int32_t m = n.depth;
  for (auto &c : n.children) m = std::max(m, max_depth_of(c));
  return m;
}

// placer.rs:111-141 place_level_recursive.
static void place_level(ONode &node, int32_t target) {
  if (node.depth + 1 == target && !node.children.empty()) {
    const size_t n = node.children.size();
    const float half_w = node.w / 2.0f, half_h = node.h / 2.0f;
    const float ox = node.cx - half_w, oy = node.cy - half_h;
    const size_t cols = (size_t)std::ceil(std::sqrt((float)n));
    const size_t rows = (n + cols - 1) / cols;
    for (size_t i = 0; i < n; ++i) {
      const size_t col = i % cols, row = i / cols;
      const float cw = node.w / (float)cols;
      const float ch = node.h / (float)rows;
      ONode &c = node.children[i];
      c.cx = ox + ((float)col + 0.5f) * cw;
      c.cy = oy + ((float)row + 0.5f) * ch;
      c.w = cw;
      c.h = ch;
    }
  } else {
    for (auto &c : node.children) place_level(c, target);
  }
}

static void collect_leaves(const ONode &n, std::vector<const ONode *> &out) {
  if (n.children.empty()) {
    out.push_back(&n);
    return;
  }
  for (auto &c : n.children) collect_leaves(c, out);
}

static int32_t count_nodes(const ONode &n) {
  int32_t c = 1;
  for (auto &ch : n.children) c += count_nodes(ch);
  return c;
}

// build_hierarchy (partitioner.rs:36-49) + the region pass of hapr_placement
// (placer.rs:40-63). Outputs leaves in HierarchyTree::leaves() order
// (hierarchy.rs:176-190): out_leaf_ptr[L+1], out_leaf_gate[N],
// out_region[4L] = (cx, cy, w, h), out_leaf_depth[L]. Returns L;
// *out_nodes / *out_max_depth receive num_nodes / max_depth.
int32_t or_build_hierarchy(int32_t n, const int32_t *adj_ptr,
                           const int32_t *adj_idx, int32_t max_leaf,
                           int32_t min_cluster, float balance, int32_t iters,
                           float chip_w, float chip_h, int32_t *out_leaf_ptr,
                           int32_t *out_leaf_gate, float *out_region,
                           int32_t *out_leaf_depth, int32_t *out_nodes,
                           int32_t *out_max_depth) {
  std::vector<int32_t> all((size_t)n);
  for (int32_t i = 0; i < n; ++i) all[i] = i;
  int32_t next_id = 0;
  ONode root = bisect(adj_ptr, adj_idx, all, 0, max_leaf, min_cluster, balance,
                      iters, next_id);
  root.cx = chip_w / 2.0f;
  root.cy = chip_h / 2.0f;
  root.w = chip_w;
  root.h = chip_h;
  const int32_t md = max_depth_of(root);
  for (int32_t depth = 1; depth <= md; ++depth) place_level(root, depth);
  std::vector<const ONode *> leaves;
  collect_leaves(root, leaves);
  int32_t off = 0;
  for (size_t l = 0; l < leaves.size(); ++l) {
    const ONode *lf = leaves[l];
    if (out_leaf_ptr) out_leaf_ptr[l] = off;
    for (int32_t g : lf->gates) {
      if (out_leaf_gate) out_leaf_gate[off] = g;
      ++off;
    }
    if (out_region) {
      out_region[4 * l + 0] = lf->cx;
      out_region[4 * l + 1] = lf->cy;
      out_region[4 * l + 2] = lf->w;
      out_region[4 * l + 3] = lf->h;
    }
    if (out_leaf_depth) out_leaf_depth[l] = lf->depth;
  }
  if (out_leaf_ptr) out_leaf_ptr[leaves.size()] = off;
  if (out_nodes) *out_nodes = count_nodes(root);
  if (out_max_depth) *out_max_depth = md;
  return (int32_t)leaves.size();
}

// partitioner.rs:106-185 on one gate subset (exposed for the power-iteration
// check): writes the f32 vector after `iters` iterations.
void or_fiedler_vector(const int32_t *adj_ptr, const int32_t *adj_idx,
                       int32_t n, const int32_t *gates, int32_t iters,
                       float *out_v) {
  std::vector<int32_t> gi(gates, gates + n);
  std::vector<float> v = fiedler(adj_ptr, adj_idx, gi, iters);
  std::copy(v.begin(), v.end(), out_v);
}

// ---------------------------------------------------------------------------
// Barnes-Hut with the tree rules of O/src/cpp/BarnesHutTree.cpp, restated on
// a Morton-key radix tree (the construction the device code uses), with
// FP64 force accumulation.
//
// Root square (BarnesHutTree.cpp:24-46) and keys in f32 without contraction;
// a point on a cell boundary belongs to the lower cell (`<=` rule of
// BarnesHutTree.cpp:107-123).
static uint32_t q15(float p, float o, float size) {
  const float t = ((p - o) / size) * 32768.0f;
  if (!(t > 0.0f)) return 0u;
  const float c = std::ceil(t);
  if (c >= 32768.0f) return 32767u;
  return (uint32_t)c - 1u;
}

// The sub-cell (0..4095) of p within its level-15 cell c15, in f64: the
// deep keys of levels 16..27, used when a level-15 cell is not accepted by
// every point (device: quantize_sub).
static uint32_t q_sub(float p, float o, float size, uint32_t c15) {
  const double w = (double)size / 32768.0;
  const double o15 = (double)o + (double)c15 * w;
  const double t = (((double)p - o15) / w) * 4096.0;
  if (!(t > 0.0)) return 0u;
  const double c = std::ceil(t);
  if (c >= 4096.0) return 4095u;
  return (uint32_t)c - 1u;
}

static uint32_t interleave15(uint32_t qx, uint32_t qy) {
  uint32_t k = 0;
  for (int b = 14; b >= 0; --b) {
    k = (k << 1) | ((qx >> b) & 1u);
    k = (k << 1) | ((qy >> b) & 1u);
  }
  return k;
}

void or_bh_root(int32_t n, const float *x, const float *y, float *root) {
  float mnx = x[0], mxx = x[0], mny = y[0], mxy = y[0];
  for (int32_t i = 1; i < n; ++i) {
    mnx = std::fmin(mnx, x[i]);
    mxx = std::fmax(mxx, x[i]);
    mny = std::fmin(mny, y[i]);
    mxy = std::fmax(mxy, y[i]);
  }
  mnx = mnx - 1.0f;
  mxx = mxx + 1.0f;
  mny = mny - 1.0f;
  mxy = mxy + 1.0f;
  const float size = std::fmax(mxx - mnx, mxy - mny);
  const float cx = (mnx + mxx) * 0.5f, cy = (mny + mxy) * 0.5f;
  const float half = size * 0.5f;
  root[0] = cx - half;
  root[1] = cy - half;
  root[2] = size;
}

void or_bh_keys(int32_t n, const float *x, const float *y, const float *root,
                uint32_t *keys) {
  for (int32_t i = 0; i < n; ++i)
    keys[i] = interleave15(q15(x[i], root[0], root[2]), q15(y[i], root[1], root[2]));
}

namespace {
// Exact prefix sums of the sorted positions, as the device computes them:
// each position becomes the 128-bit integer trunc(v * 2^64) (exact for
// |v| >= 2^-41, non-finite values count as 0), node sums are differences of
// integer prefixes, and a centre of mass is
// ((double)hi * 2^64 + (double)lo) * 2^-64 / count (hi/lo: the upper signed and
// lower unsigned 64 bits), each step rounded to nearest.
static __int128 fixed64(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  const int e = (int)((u >> 23) & 255u);
  if (e == 0 || e == 255) return 0;
  const unsigned long long m = (u & 0x7fffffu) | 0x800000u;
  const int sh = e - 86;
  unsigned __int128 r = 0;
  if (sh >= 0) r = (unsigned __int128)m << sh;
  else if (sh > -64) r = m >> (-sh);
  return (u >> 31) ? -(__int128)r : (__int128)r;
}

static double fixed_to_double(__int128 v) {
  const long long hi = (long long)(v >> 64);
  const unsigned long long lo = (unsigned long long)v;
  const double a = (double)hi * 18446744073709551616.0;
  const double b = a + (double)lo;
  return b * 5.42101086242752217003726400434970855712890625e-20;
}

// The radix tree over the sorted keys, built top-down: node [f, l] splits
// after the last position s with delta(f, s) > delta(f, l). Children are
// internal node ids or ~leaf (sorted position), as on the device.
struct BHTree {
  int32_t n;
  bool deep = false;              // 24-bit sub-keys below the 30-bit keys
  int kb = 30;                    // prefix length of a bucket (30 or 54)
  std::vector<uint32_t> key;      // sorted keys
  std::vector<uint32_t> lo;       // sorted sub-keys (deep)
  std::vector<int32_t> perm;      // sorted -> original
  std::vector<float> sx, sy;      // sorted positions
  std::vector<__int128> px, py;   // exact fixed-point prefix sums
  float rsize;
  struct Node {
    int32_t f, l, dn, dp, left, right;
    double cxd, cyd;                // FP64 centre of mass
    float hx, hy, lx, ly, s2;       // COM hi/lo, size^2 (<0: no quad level)
    bool bucket;
  };
  std::vector<Node> nodes;
  int delta(int32_t i, int32_t j) const {
    if (j < 0 || j >= n) return -1;
    if (key[i] != key[j]) return __builtin_clz(key[i] ^ key[j]) - 2;
    if (deep) {
      if (lo[i] != lo[j]) return 30 + __builtin_clz(lo[i] ^ lo[j]) - 8;
      return 54 + __builtin_clz((uint32_t)(i ^ j));
    }
    return 30 + __builtin_clz((uint32_t)(i ^ j));
  }
  int32_t split(int32_t f, int32_t l) const {
    const int dn = delta(f, l);
    int32_t lo = f, hi = l - 1;
    while (lo < hi) {
      const int32_t mid = lo + (hi - lo + 1) / 2;
      if (delta(f, mid) > dn) lo = mid; else hi = mid - 1;
    }
    return lo;
  }
  int32_t build(int32_t f, int32_t l, int dp) {
    const int32_t id = (int32_t)nodes.size();
    nodes.push_back(Node{});
    const int dn = delta(f, l);
    const int32_t g = split(f, l);
    const int32_t left = g == f ? ~f : build(f, g, dn);
    const int32_t right = g + 1 == l ? ~l : build(g + 1, l, dn);
    Node &nd = nodes[id];
    nd.f = f;
    nd.l = l;
    nd.dn = dn;
    nd.dp = dp;
    nd.left = left;
    nd.right = right;
    __int128 sxi = px[l], syi = py[l];
    if (f > 0) {
      sxi -= px[f - 1];
      syi -= py[f - 1];
    }
    const int32_t cnt = l - f + 1;
    nd.cxd = fixed_to_double(sxi) / (double)cnt;
    nd.cyd = fixed_to_double(syi) / (double)cnt;
    nd.hx = (float)nd.cxd;
    nd.hy = (float)nd.cyd;
    nd.lx = (float)(nd.cxd - (double)nd.hx);
    nd.ly = (float)(nd.cyd - (double)nd.hy);
    nd.bucket = dn >= kb;
    const int lmax = nd.bucket ? kb >> 1 : dn >> 1;
    const float sz = std::ldexp(rsize, -lmax);
    nd.s2 = (!nd.bucket && dp >= 0 && (dp >> 1) == lmax) ? -1.0f : sz * sz;
    return id;
  }
  // Up to four quad children of an internal node, in key order: a child that
  // stands for no quad level is replaced by its own two children.
  int quad_children(int32_t c, int32_t out[4]) const {
    int k = 0;
    const Node &nd = nodes[c];
    for (int32_t h : {nd.left, nd.right}) {
      if (h >= 0 && nodes[h].dn < kb && (nodes[h].dn >> 1) == (nd.dn >> 1)) {
        out[k++] = nodes[h].left;
        out[k++] = nodes[h].right;
      } else {
        out[k++] = h;
      }
    }
    return k;
  }
};

// The device's inverse square root: Lomont's bit-level estimate
// (0x5f375a86) and three Newton steps y * fma(-(h * y), y, 1.5), IEEE f32
// with the device's explicit fused multiply-adds and no other contraction.
static inline float rsqrt32(float x) {
  int32_t i;
  std::memcpy(&i, &x, 4);
  i = 0x5f375a86 - (i >> 1);
  float y;
  std::memcpy(&y, &i, 4);
  const float h = 0.5f * x;
  for (int k = 0; k < 3; ++k) y = y * std::fmaf(-(h * y), y, 1.5f);
  return y;
}

// f32 law, in the device's operation order.
static inline void term32(float dx, float dy, float r2c, float kq, float &fx,
                          float &fy) {
  const float inv = rsqrt32(r2c);
  const float f = ((kq * inv) * inv) * inv;
  fx = std::fmaf(f, dx, fx);
  fy = std::fmaf(f, dy, fy);
}

// Per-point walk with the device's rules and term order: for every opened
// cell, the terms of its children in key order (single points, accepted
// cells, opened buckets point by point), then the opened children in order.
struct Walker {
  const BHTree &t;
  double k, md;
  float kf, th2, md2;
  int32_t s;                 // sorted index of the target point
  float pxf, pyf;
  double fx = 0, fy = 0;     // FP64 recomputation of the same interactions
  float gx = 0.f, gy = 0.f;  // f32, device order
  int64_t inter = 0;
  void point(int32_t q) {
    const double dx = (double)pxf - (double)t.sx[q], dy = (double)pyf - (double)t.sy[q];
    const double d = std::max(std::sqrt(dx * dx + dy * dy), md);
    const double f = k / (d * d);
    fx += f * dx / d;
    fy += f * dy / d;
    const float ex = pxf - t.sx[q], ey = pyf - t.sy[q];
    const float r2 = std::fmaf(ex, ex, ey * ey);
    term32(ex, ey, std::fmax(r2, md2), kf, gx, gy);
    ++inter;
  }
  // Adds the terms child c contributes at this cell; true if c is a cell
  // this point must descend into.
  bool eval(int32_t c) {
    if (c < 0) {
      if (~c != s) point(~c);
      return false;
    }
    const BHTree::Node &nd = t.nodes[c];
    const float dx = (pxf - nd.hx) - nd.lx, dy = (pyf - nd.hy) - nd.ly;
    const float r2 = std::fmaf(dx, dx, dy * dy);
    const float r2c = std::fmax(r2, md2);
    if (nd.s2 >= 0.0f && nd.s2 < th2 * r2c) {
      const int32_t cnt = nd.l - nd.f + 1;
      const double ddx = (double)pxf - nd.cxd, ddy = (double)pyf - nd.cyd;
      const double d = std::max(std::sqrt(ddx * ddx + ddy * ddy), md);
      const double fm = k * cnt / (d * d);
      fx += fm * ddx / d;
      fy += fm * ddy / d;
      term32(dx, dy, r2c, kf * (float)cnt, gx, gy);
      ++inter;
      return false;
    }
    if (nd.bucket) {
      for (int32_t q = nd.f; q <= nd.l; ++q)
        if (q != s) point(q);
      return false;
    }
    return true;
  }
  void open(int32_t c) {
    int32_t ch[4];
    const int m = t.quad_children(c, ch);
    bool op[4] = {false, false, false, false};
    for (int h = 0; h < m; ++h) op[h] = eval(ch[h]);
    for (int h = 0; h < m; ++h)
      if (op[h]) open(ch[h]);
  }
};
}  // namespace

// Forces on every point (original order): FP64 recomputation (fx/fy) and the
// f32 values in the device's operation order (fx32/fy32, may be null), plus
// keys (gate order), sorted order, root square and interaction count per
// point (each may be null). The opening decisions use the f32 rounding of
// min_dist; the FP64 law uses min_dist as given.
void or_bh_forces(int32_t n, const float *x, const float *y, double k,
                  float theta, double min_dist, double *fx, double *fy,
                  uint32_t *out_keys, int32_t *out_perm, float *out_root,
                  int64_t *out_inter, int32_t threads, float *fx32,
                  float *fy32) {
  if (n <= 0) return;
  float root[3];
  or_bh_root(n, x, y, root);
  BHTree t;
  t.n = n;
  t.rsize = root[2];
  const float mdf = (float)min_dist;
  const float th2 = theta * theta, md2 = mdf * mdf, kf = (float)k;
  // deep keys when a level-15 cell is not accepted by every point
  const float s15 = std::ldexp(root[2], -15);
  t.deep = s15 * s15 >= th2 * md2;
  t.kb = t.deep ? 54 : 30;
  std::vector<uint32_t> keys((size_t)n), sub(t.deep ? (size_t)n : 0);
  or_bh_keys(n, x, y, root, keys.data());
  if (t.deep)
    for (int32_t i = 0; i < n; ++i)
      sub[i] = interleave15(q_sub(x[i], root[0], root[2], q15(x[i], root[0], root[2])),
                            q_sub(y[i], root[1], root[2], q15(y[i], root[1], root[2])));
  t.perm.resize((size_t)n);
  for (int32_t i = 0; i < n; ++i) t.perm[i] = i;
  std::stable_sort(t.perm.begin(), t.perm.end(), [&](int32_t a, int32_t b) {
    if (keys[a] != keys[b]) return keys[a] < keys[b];
    return t.deep && sub[a] < sub[b];
  });
  if (t.deep) {
    t.lo.resize((size_t)n);
    for (int32_t s = 0; s < n; ++s) t.lo[s] = sub[t.perm[s]];
  }
  t.key.resize((size_t)n);
  t.sx.resize((size_t)n);
  t.sy.resize((size_t)n);
  t.px.resize((size_t)n);
  t.py.resize((size_t)n);
  __int128 ax = 0, ay = 0;
  for (int32_t s = 0; s < n; ++s) {
    const int32_t g = t.perm[s];
    t.key[s] = keys[g];
    t.sx[s] = x[g];
    t.sy[s] = y[g];
    ax += fixed64(x[g]);
    ay += fixed64(y[g]);
    t.px[s] = ax;
    t.py[s] = ay;
  }
  t.nodes.reserve(n > 1 ? (size_t)n - 1 : 1);
  if (n >= 2) t.build(0, n - 1, -1);
  par_for(n, threads, [&](int32_t s) {
    Walker w{t, k, min_dist, kf, th2, md2, s, t.sx[s], t.sy[s]};
    if (n >= 2 && w.eval(0)) w.open(0);
    const int32_t g = t.perm[s];
    fx[g] = w.fx;
    fy[g] = w.fy;
    if (fx32) fx32[g] = w.gx;
    if (fy32) fy32[g] = w.gy;
    if (out_inter) out_inter[g] = w.inter;
  });
  if (out_keys) std::copy(keys.begin(), keys.end(), out_keys);
  if (out_perm) std::copy(t.perm.begin(), t.perm.end(), out_perm);
  if (out_root) std::copy(root, root + 3, out_root);
}

// Exact all-pairs repulsion k/max(d,min_dist)^2 along the unit vector in FP64
// (the law of placer.rs:258-272).
void or_repulsion_exact(int32_t n, const float *x, const float *y, double k,
                        double min_dist, double *fx, double *fy) {
  for (int32_t i = 0; i < n; ++i) {
    double ax = 0.0, ay = 0.0;
    for (int32_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double dx = (double)x[i] - x[j], dy = (double)y[i] - y[j];
      const double d = std::max(std::sqrt(dx * dx + dy * dy), min_dist);
      const double f = k / (d * d);
      ax += f * dx / d;
      ay += f * dy / d;
    }
    fx[i] = ax;
    fy[i] = ay;
  }
}

// compute_level_attention (H/src/algorithm/attention.rs:50-88) with its hash
// sets, for k sampled clusters of one level (all of them when k = n): the
// nets of each sampled cluster by nets_touching_gates (:90-99, a scan of every
// net), the k x k scores among them (HashSet intersection iterates the smaller
// set), and one top-k sort of an n-entry row per sample (:74-84, stable,
// descending). out_scores[k * k] (may be NULL) gets scores[rows[a]][rows[b]];
// t_out[3] the seconds of the three phases, for scaling to the whole level.
void or_attention_sample(int32_t m, const int32_t *net_ptr, const int32_t *net_gate,
                         int32_t n, const int32_t *cluster_ptr, const int32_t *cluster_gate,
                         int32_t k, const int32_t *rows, int32_t top_k, float *out_scores,
                         int32_t *out_topk, double *t_out) {
  using clk = std::chrono::steady_clock;
  auto secs = [](clk::time_point a, clk::time_point b) {
    return std::chrono::duration<double>(b - a).count();
  };
  const auto t0 = clk::now();
  std::vector<std::unordered_set<int64_t>> nets(k);
  for (int32_t a = 0; a < k; ++a) {
    const int32_t c = rows[a];
    std::unordered_set<int64_t> gates(cluster_gate + cluster_ptr[c],
                                      cluster_gate + cluster_ptr[c + 1]);
    for (int32_t e = 0; e < m; ++e)
      for (int32_t q = net_ptr[e]; q < net_ptr[e + 1]; ++q)
        if (gates.count(net_gate[q])) {
          nets[a].insert(e);
          break;
        }
  }
  const auto t1 = clk::now();
  std::vector<float> sc((size_t)k * k, 0.0f);
  for (int32_t a = 0; a < k; ++a) {
    const size_t total = nets[a].size();
    if (total == 0) continue;
    for (int32_t b = 0; b < k; ++b) {
      if (a == b) continue;
      const auto &x = nets[a].size() <= nets[b].size() ? nets[a] : nets[b];
      const auto &y = nets[a].size() <= nets[b].size() ? nets[b] : nets[a];
      size_t shared = 0;
      for (int64_t e : x) shared += y.count(e);
      sc[(size_t)a * k + b] = (float)shared / (float)total;
    }
  }
  const auto t2 = clk::now();
  // row a of the level: the sampled columns carry their scores, the rest 0
  std::vector<std::pair<int32_t, float>> row;
  for (int32_t a = 0; a < k; ++a) {
    std::vector<float> full((size_t)n, 0.0f);
    for (int32_t b = 0; b < k; ++b) full[rows[b]] = sc[(size_t)a * k + b];
    row.clear();
    for (int32_t j = 0; j < n; ++j)
      if (j != rows[a]) row.emplace_back(j, full[j]);
    std::stable_sort(row.begin(), row.end(),
                     [](const std::pair<int32_t, float> &u,
                        const std::pair<int32_t, float> &v) { return u.second > v.second; });
    int32_t w = 0;
    for (int32_t r = 0; r < top_k && r < (int32_t)row.size(); ++r)
      if (row[r].second > 0.0f && out_topk) out_topk[(size_t)a * top_k + w++] = row[r].first;
    if (out_topk)
      for (; w < top_k; ++w) out_topk[(size_t)a * top_k + w] = -1;
  }
  const auto t3 = clk::now();
  if (out_scores) std::copy(sc.begin(), sc.end(), out_scores);
  t_out[0] = secs(t0, t1);
  t_out[1] = secs(t1, t2);
  t_out[2] = secs(t2, t3);
}

}  // extern "C"
