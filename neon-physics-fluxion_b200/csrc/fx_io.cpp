// fx_io.cpp -- (f.3) netlist ingestion (BLIF) and placement output (DEF),
// host-only: parser::blif::parse (H/src/parser/blif.rs:12-116) and
// parser::def::write_def (H/src/parser/def.rs:11-43).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <new>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "fx_internal.h"
#include "fx_netlist.h"

using fx::set_error;

namespace {

// Signal name -> list, remembering the order in which names first appear.
template <class V>
struct OrderedMap {
  std::unordered_map<std::string, size_t> index;
  std::vector<std::string> keys;
  std::vector<V> vals;
  V &operator[](const std::string &k) {
    auto it = index.find(k);
    if (it != index.end()) return vals[it->second];
    index.emplace(k, keys.size());
    keys.push_back(k);
    vals.emplace_back();
    return vals.back();
  }
  V *find(const std::string &k) {
    auto it = index.find(k);
    return it == index.end() ? nullptr : &vals[it->second];
  }
};

// Rust `(v as f32 * 1000.0) as i64`: f32 product, then truncation toward
// zero that saturates at the i64 range and maps NaN to 0.
long long def_coord(float v) {
  const float p = v * 1000.0f;
  if (std::isnan(p)) return 0;
  if (p >= 9.2233720368547758e18f) return std::numeric_limits<long long>::max();
  if (p <= -9.2233720368547758e18f) return std::numeric_limits<long long>::min();
  return (long long)p;
}

}  // namespace

extern "C" int fx_blif_read(const char *path, fx_netlist **out, char *design_name,
                            int32_t name_cap) {
  if (!path || !out) {
    set_error("fx_blif_read: invalid arguments");
    return FX_EINVAL;
  }
  *out = nullptr;
  std::ifstream f(path);
  if (!f) {
    set_error("Failed to open BLIF: %s", path);
    return FX_EINVAL;
  }
  int32_t gates = 0;
  OrderedMap<int32_t> driver;                 // signal -> driving gate
  std::vector<std::pair<int32_t, std::vector<std::string>>> gate_inputs;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    std::vector<std::string> tok;
    for (std::string t; ss >> t;) tok.push_back(t);
    if (tok.empty() || tok[0][0] == '#') continue;
    const std::string &kw = tok[0];
    if (kw != ".names" && kw != ".latch" && kw != ".gate") continue;
    const int32_t g = gates++;
    if (kw == ".names") {
      if (tok.size() >= 2) {
        driver[tok.back()] = g;
        gate_inputs.emplace_back(g, std::vector<std::string>(tok.begin() + 1, tok.end() - 1));
      }
    } else if (kw == ".latch") {
      if (tok.size() >= 3) {
        driver[tok[2]] = g;
        gate_inputs.emplace_back(g, std::vector<std::string>{tok[1]});
      }
    } else {  // .gate TYPE pin=signal ...
      std::vector<std::string> ins;
      for (size_t i = 2; i < tok.size(); ++i) {
        const size_t eq = tok[i].find('=');
        if (eq == std::string::npos) continue;
        const std::string sig = tok[i].substr(eq + 1);
        if (tok[i].rfind("O=", 0) == 0 || tok[i].rfind("Y=", 0) == 0) driver[sig] = g;
        else ins.push_back(sig);
      }
      gate_inputs.emplace_back(g, ins);
    }
  }
  OrderedMap<std::vector<int32_t>> readers;
  for (auto &gi : gate_inputs)
    for (auto &sig : gi.second) readers[sig].push_back(gi.first);
  fx_netlist *nl = new (std::nothrow) fx_netlist();
  if (!nl) return FX_ENOMEM;
  nl->n = gates;
  nl->net_ptr.push_back(0);
  std::vector<char> used(readers.keys.size(), 0);
  for (size_t k = 0; k < driver.keys.size(); ++k) {
    std::vector<int32_t> net{driver.vals[k]};
    auto it = readers.index.find(driver.keys[k]);
    if (it != readers.index.end()) {
      used[it->second] = 1;
      const auto &r = readers.vals[it->second];
      net.insert(net.end(), r.begin(), r.end());
    }
    if (net.size() > 1) {
      nl->net_gate.insert(nl->net_gate.end(), net.begin(), net.end());
      nl->net_ptr.push_back((int32_t)nl->net_gate.size());
    }
  }
  for (size_t k = 0; k < readers.keys.size(); ++k) {
    if (used[k] || readers.vals[k].size() < 2) continue;
    nl->net_gate.insert(nl->net_gate.end(), readers.vals[k].begin(), readers.vals[k].end());
    nl->net_ptr.push_back((int32_t)nl->net_gate.size());
  }
  nl->m = (int32_t)nl->net_ptr.size() - 1;
  nl->w.assign(gates, 2.0f);
  nl->h.assign(gates, 10.0f);
  nl->x.assign(gates, 0.0f);
  nl->y.assign(gates, 0.0f);
  nl->die_w = 1000.0f;
  nl->die_h = 1000.0f;
  nl->leaf_ptr.assign(1, 0);
  if (design_name && name_cap > 0) {
    std::string stem(path);
    const size_t slash = stem.find_last_of('/');
    if (slash != std::string::npos) stem = stem.substr(slash + 1);
    const size_t dot = stem.find_last_of('.');
    if (dot != std::string::npos && dot > 0) stem = stem.substr(0, dot);
    std::snprintf(design_name, (size_t)name_cap, "%s", stem.c_str());
  }
  *out = nl;
  return FX_OK;
}

extern "C" int fx_def_write(const char *path, const char *design_name, int32_t n,
                            const float *x, const float *y, float chip_w, float chip_h,
                            const char *names) {
  if (!path || n < 0 || (n > 0 && (!x || !y))) {
    set_error("fx_def_write: invalid arguments");
    return FX_EINVAL;
  }
  FILE *f = std::fopen(path, "w");
  if (!f) {
    set_error("Failed to create DEF: %s", path);
    return FX_EINVAL;
  }
  std::fprintf(f, "VERSION 5.8 ;\n");
  std::fprintf(f, "DIVIDERCHAR \"/\" ;\n");
  std::fprintf(f, "BUSBITCHARS \"[]\" ;\n");
  std::fprintf(f, "DESIGN %s ;\n", design_name ? design_name : "");
  std::fprintf(f, "UNITS DISTANCE MICRONS 1000 ;\n");
  std::fprintf(f, "\nDIEAREA ( 0 0 ) ( %lld %lld ) ;\n", def_coord(chip_w), def_coord(chip_h));
  std::fprintf(f, "\nCOMPONENTS %d ;\n", n);
  const char *nm = names;
  for (int32_t i = 0; i < n; ++i) {
    if (nm) {
      std::fprintf(f, "    - %s GATE_TYPE + PLACED ( %lld %lld ) N ;\n", nm, def_coord(x[i]),
                   def_coord(y[i]));
      nm += std::strlen(nm) + 1;
    } else {
      std::fprintf(f, "    - g%d GATE_TYPE + PLACED ( %lld %lld ) N ;\n", i, def_coord(x[i]),
                   def_coord(y[i]));
    }
  }
  std::fprintf(f, "END COMPONENTS ;\n");
  std::fprintf(f, "\nEND DESIGN\n");
  const bool bad = std::ferror(f) != 0;
  if (std::fclose(f) != 0 || bad) {
    set_error("Failed to write DEF: %s", path);
    return FX_EINVAL;
  }
  return FX_OK;
}
