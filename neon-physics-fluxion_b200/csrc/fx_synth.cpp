// fx_synth.cpp -- seeded synthetic netlists with the shapes of the HAPR
// placement workloads (plain netlists and batches of independent leaves).
//
// The reference publishes no netlists for this path; its generators
// (O/examples/run_million_gates.py:25-79, O/benchmarks/run_benchmarks.py:
// 15-44) use Python's global RNG. This generator uses one SplitMix64 stream
// so the same seed gives the same bytes on any machine.
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "fx_internal.h"

#include "fx_netlist.h"

namespace {

struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  // uniform double in [0, 1)
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  // uniform float in [0, 1) with 24 random bits
  float uniform24() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }
  // uniform integer in [0, n)
  uint32_t below(uint32_t n) {
    return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32);
  }
};

// Discrete power law P(d) ~ d^-alpha on [lo, hi] by inverse CDF.
struct PowerLaw {
  std::vector<double> cdf;
  int lo;
  PowerLaw(int lo_, int hi, double alpha) : lo(lo_) {
    double acc = 0.0;
    for (int d = lo_; d <= hi; ++d) {
      acc += std::pow((double)d, -alpha);
      cdf.push_back(acc);
    }
    for (double &c : cdf) c /= acc;
  }
  int sample(double u) const {
    size_t k = 0;
    while (k + 1 < cdf.size() && u >= cdf[k]) ++k;
    return lo + (int)k;
  }
};

bool contains(const int32_t *b, const int32_t *e, int32_t g) {
  for (; b != e; ++b)
    if (*b == g) return true;
  return false;
}

}  // namespace

extern "C" int fx_synth_plain(uint64_t seed, int32_t n_gates, int32_t n_nets,
                              float die_w, float die_h, int32_t leaf_size,
                              fx_netlist **out) {
  if (!out || n_gates <= 0 || n_nets < 0 || leaf_size <= 0 || !(die_w > 0.f) ||
      !(die_h > 0.f)) {
    fx::set_error("fx_synth_plain: invalid arguments");
    return FX_EINVAL;
  }
  fx_netlist *nl = new (std::nothrow) fx_netlist();
  if (!nl) return FX_ENOMEM;
  SplitMix64 rng(seed);
  const int32_t N = n_gates;
  const int32_t L = (N + leaf_size - 1) / leaf_size;
  nl->n = N;
  nl->m = n_nets;
  nl->die_w = die_w;
  nl->die_h = die_h;
  nl->w.resize(N);
  nl->h.assign(N, 1.0f);
  for (int32_t g = 0; g < N; ++g) nl->w[g] = (float)(1 + rng.below(4));
  PowerLaw pl(2, 64, 2.5);
  nl->net_ptr.resize((size_t)n_nets + 1);
  nl->net_ptr[0] = 0;
  nl->net_gate.reserve((size_t)n_nets * 3);
  auto leaf_start = [&](int32_t l) { return l * leaf_size; };
  auto leaf_len = [&](int32_t l) {
    int32_t s = l * leaf_size;
    return (N - s < leaf_size) ? N - s : leaf_size;
  };
  for (int32_t e = 0; e < n_nets; ++e) {
    double r = rng.uniform();
    int d = r < 0.6 ? 2 : (r < 0.8 ? 3 : pl.sample(rng.uniform()));
    if (d > N) d = N;
    int32_t driver = (int32_t)rng.below((uint32_t)N);
    int32_t home = driver / leaf_size;
    int32_t sib = home ^ 1;
    if (sib >= L) sib = home;
    size_t base = nl->net_gate.size();
    nl->net_gate.push_back(driver);
    int tries = 0;
    while ((int)(nl->net_gate.size() - base) < d) {
      double q = rng.uniform();
      int32_t g;
      if (tries > 64 * d || q >= 0.9) {
        g = (int32_t)rng.below((uint32_t)N);
      } else {
        int32_t l = q < 0.7 ? home : sib;
        g = leaf_start(l) + (int32_t)rng.below((uint32_t)leaf_len(l));
      }
      ++tries;
      if (!contains(nl->net_gate.data() + base,
                    nl->net_gate.data() + nl->net_gate.size(), g))
        nl->net_gate.push_back(g);
    }
    nl->net_ptr[(size_t)e + 1] = (int32_t)nl->net_gate.size();
  }
  nl->x.resize(N);
  nl->y.resize(N);
  for (int32_t g = 0; g < N; ++g) {
    nl->x[g] = rng.uniform24() * die_w;
    nl->y[g] = rng.uniform24() * die_h;
  }
  nl->leaf_ptr.resize((size_t)L + 1);
  nl->region.resize((size_t)4 * L);
  for (int32_t l = 0; l <= L; ++l) nl->leaf_ptr[l] = l < L ? leaf_start(l) : N;
  for (int32_t l = 0; l < L; ++l) {
    nl->region[4 * l + 0] = die_w * 0.5f;
    nl->region[4 * l + 1] = die_h * 0.5f;
    nl->region[4 * l + 2] = die_w;
    nl->region[4 * l + 3] = die_h;
  }
  *out = nl;
  return FX_OK;
}

extern "C" int fx_synth_leaves(uint64_t seed, int32_t n_clusters,
                               int32_t min_size, int32_t max_size,
                               float nets_per_gate, fx_netlist **out) {
  if (!out || n_clusters <= 0 || min_size < 2 || max_size < min_size ||
      !(nets_per_gate >= 0.f)) {
    fx::set_error("fx_synth_leaves: invalid arguments");
    return FX_EINVAL;
  }
  fx_netlist *nl = new (std::nothrow) fx_netlist();
  if (!nl) return FX_ENOMEM;
  SplitMix64 rng(seed);
  const double llo = std::log((double)min_size);
  const double lhi = std::log((double)max_size + 1.0);
  nl->leaf_ptr.resize((size_t)n_clusters + 1);
  nl->leaf_ptr[0] = 0;
  for (int32_t c = 0; c < n_clusters; ++c) {
    int32_t s = (int32_t)std::floor(std::exp(llo + rng.uniform() * (lhi - llo)));
    if (s < min_size) s = min_size;
    if (s > max_size) s = max_size;
    nl->leaf_ptr[c + 1] = nl->leaf_ptr[c] + s;
  }
  const int32_t N = nl->leaf_ptr[n_clusters];
  nl->n = N;
  nl->w.resize(N);
  nl->h.assign(N, 1.0f);
  for (int32_t g = 0; g < N; ++g) nl->w[g] = (float)(1 + rng.below(4));
  nl->net_ptr.push_back(0);
  for (int32_t c = 0; c < n_clusters; ++c) {
    int32_t b = nl->leaf_ptr[c];
    int32_t s = nl->leaf_ptr[c + 1] - b;
    int32_t nets = (int32_t)std::lround((double)nets_per_gate * s);
    for (int32_t e = 0; e < nets; ++e) {
      int d = 2;
      while (d < 8 && rng.uniform() < 0.5) ++d;
      if (d > s) d = s;
      size_t base = nl->net_gate.size();
      while ((int)(nl->net_gate.size() - base) < d) {
        int32_t g = b + (int32_t)rng.below((uint32_t)s);
        if (!contains(nl->net_gate.data() + base,
                      nl->net_gate.data() + nl->net_gate.size(), g))
          nl->net_gate.push_back(g);
      }
      nl->net_ptr.push_back((int32_t)nl->net_gate.size());
    }
  }
  nl->m = (int32_t)nl->net_ptr.size() - 1;
  nl->x.assign(N, 0.f);
  nl->y.assign(N, 0.f);
  nl->die_w = 1.f;
  nl->die_h = 1.f;
  nl->region.resize((size_t)4 * n_clusters);
  for (int32_t c = 0; c < n_clusters; ++c) {
    nl->region[4 * c + 0] = 0.5f;
    nl->region[4 * c + 1] = 0.5f;
    nl->region[4 * c + 2] = 1.0f;
    nl->region[4 * c + 3] = 1.0f;
  }
  *out = nl;
  return FX_OK;
}

extern "C" int fx_netlist_sizes(const fx_netlist *nl, int64_t *out_n,
                                int64_t *out_m, int64_t *out_p,
                                int64_t *out_leaves) {
  if (!nl) return FX_EINVAL;
  if (out_n) *out_n = nl->n;
  if (out_m) *out_m = nl->m;
  if (out_p) *out_p = (int64_t)nl->net_gate.size();
  if (out_leaves) *out_leaves = (int64_t)nl->leaf_ptr.size() - 1;
  return FX_OK;
}

extern "C" int fx_netlist_copy(const fx_netlist *nl, int32_t *out_net_ptr,
                               int32_t *out_net_gate, float *out_w,
                               float *out_h, float *out_x, float *out_y,
                               float *out_die, int32_t *out_leaf_ptr,
                               float *out_region) {
  if (!nl) return FX_EINVAL;
  auto cp = [](void *dst, const void *src, size_t bytes) {
    if (dst && bytes) std::memcpy(dst, src, bytes);
  };
  cp(out_net_ptr, nl->net_ptr.data(), nl->net_ptr.size() * 4);
  cp(out_net_gate, nl->net_gate.data(), nl->net_gate.size() * 4);
  cp(out_w, nl->w.data(), nl->w.size() * 4);
  cp(out_h, nl->h.data(), nl->h.size() * 4);
  cp(out_x, nl->x.data(), nl->x.size() * 4);
  cp(out_y, nl->y.data(), nl->y.size() * 4);
  if (out_die) {
    out_die[0] = nl->die_w;
    out_die[1] = nl->die_h;
  }
  cp(out_leaf_ptr, nl->leaf_ptr.data(), nl->leaf_ptr.size() * 4);
  cp(out_region, nl->region.data(), nl->region.size() * 4);
  return FX_OK;
}

extern "C" int fx_netlist_free(fx_netlist *nl) {
  delete nl;
  return FX_OK;
}
