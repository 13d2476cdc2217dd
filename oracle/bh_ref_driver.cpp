// bh_ref_driver.cpp -- TEST INFRASTRUCTURE ONLY: a C entry point around the
// reference's own Barnes-Hut tree (neon_old_codebase/src/cpp/
// BarnesHutTree.{h,cpp}), compiled from the reference sources where they lie.
// Calling convention of the reference's own caller (FluxionEngine.cpp:
// 149-178): build over all points, then computeForcesForParticle per point.
#include <vector>

#include "BarnesHutTree.h"

#include <thread>

// stride > 1 evaluates only points i with i % stride == 0 (the tree is
// always built over all points); used to time a bounded sample.
extern "C" void bh_ref_forces_sample(int n, const double *px, const double *py,
                                     const double *q, double theta, double k,
                                     double min_dist, double *fx, double *fy,
                                     int threads, int stride) {
  fluxion::BarnesHutTree tree(theta);
  tree.build(px, py, q, n);
  // The tree is read-only after build, so points can be split across
  // threads (threads <= 1 runs on the calling thread).
  if (stride < 1) stride = 1;
  auto work = [&](int t, int nthreads) {
    for (int i = t * stride; i < n; i += nthreads * stride) {
      double a = 0.0, b = 0.0;
      tree.computeForcesForParticle(i, px[i], py[i], q[i], k, min_dist, a, b);
      fx[i] = a;
      fy[i] = b;
    }
  };
  if (threads <= 1) {
    work(0, 1);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(work, t, threads);
    for (auto &th : pool) th.join();
  }
}

extern "C" void bh_ref_forces(int n, const double *px, const double *py,
                              const double *q, double theta, double k,
                              double min_dist, double *fx, double *fy,
                              int threads) {
  bh_ref_forces_sample(n, px, py, q, theta, k, min_dist, fx, fy, threads, 1);
}
