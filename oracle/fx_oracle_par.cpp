// TEST INFRASTRUCTURE ONLY (the CPU reference arm of bench.py).
//
// compute_congestion_cpu (H/src/algorithm/congestion.rs:11-62) run on every
// host core: the reference's literal loops (per net: the f32 bounding box of
// its gates, cell_at of both corners, then +1.0 on every covered cell of the
// h grid row by row and of the v grid column by column), with the nets dealt
// out to threads in chunks and each thread adding into its own pair of
// grids; the grids are summed in thread order at the end. Every grid value is
// an integer below 2^24, so the f32 sums are exact and equal to the
// single-threaded loop's. Compiled at -O3, as the reference's release
// profile (Cargo.toml: opt-level = 3) compiles the Rust loop.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

extern "C" {
int64_t or_cell_at(float v, float cell, int64_t n);
void or_grid_geometry(float chip_w, float chip_h, int64_t cols, int64_t rows,
                      float *cell_w, float *cell_h, float *capacity);

void or_congestion_parallel(int32_t m, const int32_t *net_ptr, const int32_t *net_gate,
                            const float *x, const float *y, float chip_w, float chip_h,
                            int64_t cols, int64_t rows, int32_t threads, float *h, float *v) {
  float cw, ch, cap;
  or_grid_geometry(chip_w, chip_h, cols, rows, &cw, &ch, &cap);
  const size_t cells = (size_t)(cols * rows);
  const int T = threads > 0 ? threads : 1;
  std::vector<std::vector<float>> gh((size_t)T), gv((size_t)T);
  std::atomic<int32_t> next{0};
  constexpr int32_t kChunk = 2048;
  auto work = [&](int t) {
    std::vector<float> &hh = gh[(size_t)t], &vv = gv[(size_t)t];
    hh.assign(cells, 0.0f);
    vv.assign(cells, 0.0f);
    float *H = hh.data(), *V = vv.data();
    for (;;) {
      const int32_t e0 = next.fetch_add(kChunk);
      if (e0 >= m) break;
      const int32_t e1 = std::min(m, e0 + kChunk);
      for (int32_t e = e0; e < e1; ++e) {
        const int32_t b = net_ptr[e], t2 = net_ptr[e + 1];
        if (t2 - b < 2) continue;
        float min_x = 3.40282347e+38f, max_x = -3.40282347e+38f;
        float min_y = 3.40282347e+38f, max_y = -3.40282347e+38f;
        for (int32_t q = b; q < t2; ++q) {
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
            if (idx < cells) H[idx] += 1.0f;
          }
        for (int64_t c = min_col; c <= max_col; ++c)
          for (int64_t r = min_row; r <= max_row; ++r) {
            const size_t idx = (size_t)(r * cols + c);
            if (idx < cells) V[idx] += 1.0f;
          }
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < T; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto &th : pool) th.join();
  std::fill(h, h + cells, 0.0f);
  std::fill(v, v + cells, 0.0f);
  for (int t = 0; t < T; ++t) {
    const float *H = gh[(size_t)t].data(), *V = gv[(size_t)t].data();
    for (size_t i = 0; i < cells; ++i) {
      h[i] += H[i];
      v[i] += V[i];
    }
  }
}
}  // extern "C"
