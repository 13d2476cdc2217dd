// fluxion_cli.cpp -- the `fluxion` command: the reference CLI's flow
// (H/src/main.rs:1-120) on the B200, written against the public C ABI only.
//
//   fluxion [-c|--config FILE] [-i|--input FILE] [-o|--output FILE]
//
// Same flags, defaults (config/default.yaml), YAML keys (H/src/config.rs:7-84)
// and exit codes: 0 on success; 1 on a config error, a missing input, an
// unsupported format, a parse error, a circuit with no gates, or an export
// error (main.rs:33-119); 2 on bad arguments (clap's usage error). A GPU
// failure also exits 1. Log lines go to stderr as the reference's env_logger.
//
// Flow: BLIF -> build_hierarchy (fx_partition, the reference's f32 power
// iteration with 30 steps, main.rs:76-82) -> hapr_placement's leaf placement
// (fx_hapr_place_leaves with the placement keys) -> refine_placement
// (fx_refine with the congestion keys) -> write_def (fx_def_write). The
// attention phase (main.rs:84-89) is computed and never used by the
// reference placement, so it is not run.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "fluxion_b200.h"

namespace {

void log_info(const std::string &m) { std::fprintf(stderr, "[INFO  fluxion] %s\n", m.c_str()); }
void log_error(const std::string &m) { std::fprintf(stderr, "[ERROR fluxion] %s\n", m.c_str()); }

// ---- a YAML subset: nested mappings of scalars, '#' comments -------------
struct Yaml {
  std::map<std::string, std::string> kv;  // "section.key" or "key" -> scalar text
};

std::string trim(const std::string &s) {
  const size_t b = s.find_first_not_of(" \t\r");
  if (b == std::string::npos) return "";
  const size_t e = s.find_last_not_of(" \t\r");
  return s.substr(b, e - b + 1);
}

bool parse_yaml(const std::string &path, Yaml &y, std::string &err) {
  std::ifstream f(path);
  if (!f) {
    err = "Failed to open config: " + path;
    return false;
  }
  std::string line, section;
  int lineno = 0;
  while (std::getline(f, line)) {
    ++lineno;
    // drop a comment that is not inside quotes
    bool q = false;
    char qc = 0;
    for (size_t i = 0; i < line.size(); ++i) {
      const char c = line[i];
      if (q) {
        if (c == qc) q = false;
      } else if (c == '"' || c == '\'') {
        q = true;
        qc = c;
      } else if (c == '#' && (i == 0 || line[i - 1] == ' ' || line[i - 1] == '\t')) {
        line.resize(i);
        break;
      }
    }
    if (trim(line).empty()) continue;
    const size_t indent = line.find_first_not_of(' ');
    const std::string body = trim(line);
    const size_t colon = body.find(':');
    if (colon == std::string::npos) {
      err = "Failed to parse YAML: line " + std::to_string(lineno) + ": expected `key: value`";
      return false;
    }
    const std::string key = trim(body.substr(0, colon));
    std::string val = trim(body.substr(colon + 1));
    if (indent == 0) {
      if (val.empty()) {
        section = key;
        y.kv[key] = "\x01map";
        continue;
      }
      section.clear();
      y.kv[key] = val;
    } else {
      if (section.empty()) {
        err = "Failed to parse YAML: line " + std::to_string(lineno) + ": unexpected indentation";
        return false;
      }
      y.kv[section + "." + key] = val;
    }
  }
  return true;
}

struct Cfg {
  std::string input, output, format;
  long long max_leaf_size = 0, min_cluster_size = 0;
  float balance_factor = 0.f;
  long long force_iterations = 0;
  float attract_weight = 0.f, repel_weight = 0.f, damping = 0.f, dt = 0.f;
  long long grid_cols = 0, grid_rows = 0, refinement_iterations = 0;
  float overflow_threshold = 0.f, move_distance = 0.f;
};

std::string unquote(const std::string &v) {
  if (v.size() >= 2 && (v[0] == '"' || v[0] == '\'') && v.back() == v[0])
    return v.substr(1, v.size() - 2);
  return v;
}

// serde's field types: String, usize, f32, bool; every field is required.
bool get(const Yaml &y, const std::string &k, std::string &out, std::string &err) {
  auto it = y.kv.find(k);
  if (it == y.kv.end() || it->second == "\x01map") {
    err = "Failed to parse YAML: missing field `" + k + "`";
    return false;
  }
  out = unquote(it->second);
  return true;
}
bool get_usize(const Yaml &y, const std::string &k, long long &out, std::string &err) {
  std::string s;
  if (!get(y, k, s, err)) return false;
  char *end = nullptr;
  const long long v = std::strtoll(s.c_str(), &end, 10);
  if (s.empty() || *end || v < 0) {
    err = "Failed to parse YAML: " + k + ": invalid value `" + s + "`, expected usize";
    return false;
  }
  out = v;
  return true;
}
bool get_f32(const Yaml &y, const std::string &k, float &out, std::string &err) {
  std::string s;
  if (!get(y, k, s, err)) return false;
  char *end = nullptr;
  const float v = std::strtof(s.c_str(), &end);
  if (s.empty() || *end) {
    err = "Failed to parse YAML: " + k + ": invalid value `" + s + "`, expected f32";
    return false;
  }
  out = v;
  return true;
}
bool get_bool(const Yaml &y, const std::string &k, std::string &err) {
  std::string s;
  if (!get(y, k, s, err)) return false;
  if (s != "true" && s != "false") {
    err = "Failed to parse YAML: " + k + ": invalid value `" + s + "`, expected a boolean";
    return false;
  }
  return true;
}

bool load_config(const std::string &path, Cfg &c, std::string &err) {
  Yaml y;
  if (!parse_yaml(path, y, err)) return false;
  std::string s;
  long long u = 0;
  float f = 0.f;
  return get(y, "input", c.input, err) && get(y, "output", c.output, err) &&
         get(y, "format", c.format, err) &&
         get_usize(y, "partitioning.max_leaf_size", c.max_leaf_size, err) &&
         get_usize(y, "partitioning.min_cluster_size", c.min_cluster_size, err) &&
         get_f32(y, "partitioning.balance_factor", c.balance_factor, err) &&
         get(y, "partitioning.method", s, err) && get_usize(y, "attention.top_k", u, err) &&
         get_f32(y, "attention.decay", f, err) &&
         get_usize(y, "placement.force_iterations", c.force_iterations, err) &&
         get_f32(y, "placement.attract_weight", c.attract_weight, err) &&
         get_f32(y, "placement.repel_weight", c.repel_weight, err) &&
         get_f32(y, "placement.damping", c.damping, err) &&
         get_f32(y, "placement.dt", c.dt, err) && get(y, "placement.embed_method", s, err) &&
         get_usize(y, "congestion.grid_cols", c.grid_cols, err) &&
         get_usize(y, "congestion.grid_rows", c.grid_rows, err) &&
         get_f32(y, "congestion.overflow_threshold", c.overflow_threshold, err) &&
         get_usize(y, "congestion.refinement_iterations", c.refinement_iterations, err) &&
         get_f32(y, "congestion.move_distance", c.move_distance, err) &&
         get(y, "legalization.method", s, err) &&
         get_usize(y, "legalization.timeout_seconds", u, err) &&
         get_usize(y, "legalization.region_size", u, err) && get_bool(y, "gpu.enabled", err) &&
         get_usize(y, "gpu.workgroup_size", u, err) && get(y, "logging.level", s, err) &&
         get_bool(y, "logging.progress", err) && get_bool(y, "logging.metrics_per_level", err);
}

// Placement::update_wirelength (H/src/data/placement.rs:48-74) in f32.
float hpwl_f32(const std::vector<int32_t> &ptr, const std::vector<int32_t> &gate,
               const std::vector<float> &x, const std::vector<float> &y) {
  float total = 0.f;
  for (size_t e = 0; e + 1 < ptr.size(); ++e) {
    if (ptr[e + 1] - ptr[e] < 2) continue;
    float mnx = INFINITY, mxx = -INFINITY, mny = INFINITY, mxy = -INFINITY;
    for (int32_t q = ptr[e]; q < ptr[e + 1]; ++q) {
      mnx = std::fmin(mnx, x[gate[q]]);
      mxx = std::fmax(mxx, x[gate[q]]);
      mny = std::fmin(mny, y[gate[q]]);
      mxy = std::fmax(mxy, y[gate[q]]);
    }
    total += (mxx - mnx) + (mxy - mny);
  }
  return total;
}

int fail(const std::string &m) {
  log_error(m);
  return 1;
}

void usage(FILE *f) {
  std::fprintf(f,
               "FLUXION v4 — HAPR Placement Engine (B200)\n\n"
               "Usage: fluxion [OPTIONS]\n\n"
               "Options:\n"
               "  -c, --config <CONFIG>  Path to config YAML [default: config/default.yaml]\n"
               "  -i, --input <INPUT>    Override input circuit file\n"
               "  -o, --output <OUTPUT>  Override output DEF file\n"
               "  -h, --help             Print help\n"
               "  -V, --version          Print version\n");
}

}  // namespace

int main(int argc, char **argv) {
  std::string config = "config/default.yaml", input, output;
  bool have_in = false, have_out = false;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto value = [&](std::string &dst) {
      if (i + 1 >= argc) return false;
      dst = argv[++i];
      return true;
    };
    if (a == "-h" || a == "--help") {
      usage(stdout);
      return 0;
    } else if (a == "-V" || a == "--version") {
      std::printf("fluxion %s\n", fx_version());
      return 0;
    } else if (a == "-c" || a == "--config") {
      if (!value(config)) { usage(stderr); return 2; }
    } else if (a == "-i" || a == "--input") {
      if (!value(input)) { usage(stderr); return 2; }
      have_in = true;
    } else if (a == "-o" || a == "--output") {
      if (!value(output)) { usage(stderr); return 2; }
      have_out = true;
    } else if (a.rfind("--config=", 0) == 0) {
      config = a.substr(9);
    } else if (a.rfind("--input=", 0) == 0) {
      input = a.substr(8);
      have_in = true;
    } else if (a.rfind("--output=", 0) == 0) {
      output = a.substr(9);
      have_out = true;
    } else {
      std::fprintf(stderr, "error: unexpected argument '%s' found\n\n", a.c_str());
      usage(stderr);
      return 2;
    }
  }
  log_info("Starting FLUXION v4");
  Cfg cfg;
  std::string err;
  if (!load_config(config, cfg, err)) return fail("Config error: " + err);
  if (have_in) cfg.input = input;
  if (have_out) cfg.output = output;
  if (cfg.input.empty()) return fail("No input file specified in config or arguments");

  log_info("Parsing circuit: " + cfg.input);
  const size_t dot = cfg.input.find_last_of('.');
  const size_t slash = cfg.input.find_last_of('/');
  const std::string ext = (dot != std::string::npos && (slash == std::string::npos || dot > slash))
                              ? cfg.input.substr(dot + 1) : "";
  if (!(ext == "blif" || cfg.format == "blif"))
    return fail("Unsupported format (only BLIF supported in this demo)");
  fx_netlist *nl = nullptr;
  char name[256] = "";
  if (fx_blif_read(cfg.input.c_str(), &nl, name, sizeof name) != FX_OK)
    return fail(std::string("BLIF parse error: ") + fx_last_error());
  int64_t n64 = 0, m64 = 0, p64 = 0;
  fx_netlist_sizes(nl, &n64, &m64, &p64, nullptr);
  const int32_t n = (int32_t)n64, m = (int32_t)m64;
  std::vector<int32_t> net_ptr((size_t)m + 1), net_gate((size_t)std::max<int64_t>(p64, 1));
  std::vector<float> w((size_t)std::max(n, 1)), h((size_t)std::max(n, 1));
  float die[2] = {0.f, 0.f};
  fx_netlist_copy(nl, net_ptr.data(), net_gate.data(), w.data(), h.data(), nullptr, nullptr,
                  die, nullptr, nullptr);
  fx_netlist_free(nl);
  log_info("Parsed BLIF: " + std::to_string(n) + " gates, " + std::to_string(m) + " nets");
  if (n == 0) return fail("Circuit has 0 gates. Exiting.");

  fx_ctx *ctx = nullptr;
  fx_design *d = nullptr;
  auto gpu_fail = [&](const char *what) {
    const std::string msg = std::string(what) + ": " + fx_last_error();
    if (d) fx_design_free(d);
    if (ctx) fx_ctx_destroy(ctx);
    return fail(msg);
  };
  if (fx_ctx_create(&ctx, 0) != FX_OK) return gpu_fail("GPU context");
  if (fx_design_load(ctx, n, m, net_ptr.data(), net_gate.data(), w.data(), h.data(), die[0],
                     die[1], &d) != FX_OK)
    return gpu_fail("design upload");

  log_info("Phase 1: Hierarchical Partitioning");
  fx_part_cfg pc;
  fx_part_cfg_default(&pc);
  pc.max_leaf_size = (int32_t)std::min<long long>(cfg.max_leaf_size, 1 << 30);
  pc.min_cluster_size = (int32_t)std::min<long long>(cfg.min_cluster_size, 1 << 30);
  pc.balance_factor = cfg.balance_factor;
  pc.power_iterations = 30;
  pc.mode = FX_PART_EXACT;
  std::vector<int32_t> lp((size_t)n + 2), lg((size_t)n), ld((size_t)n + 1);
  std::vector<float> rg(4 * ((size_t)n + 1));
  fx_part_stats ps{};
  if (fx_partition(ctx, d, &pc, n + 1, lp.data(), lg.data(), rg.data(), ld.data(), &ps) != FX_OK)
    return gpu_fail("partitioning");
  log_info("Hierarchy built: " + std::to_string(ps.n_nodes) + " nodes, max_depth=" +
           std::to_string(ps.max_depth));

  log_info("Phase 3: Multi-level Placement");
  fx_leaf_cfg lc;
  fx_leaf_cfg_default(&lc);
  lc.force_iterations = (int32_t)std::min<long long>(cfg.force_iterations, 1 << 30);
  lc.attract_weight = cfg.attract_weight;
  lc.repel_weight = cfg.repel_weight;
  lc.damping = cfg.damping;
  lc.dt = cfg.dt;
  std::vector<float> x((size_t)n, 0.f), y((size_t)n, 0.f);
  if (fx_hapr_place_leaves(ctx, d, ps.n_leaves, lp.data(), lg.data(), rg.data(), &lc, x.data(),
                           y.data(), nullptr) != FX_OK)
    return gpu_fail("leaf placement");
  char buf[160];
  std::snprintf(buf, sizeof buf, "HAPR placement complete. HPWL = %.1f",
                hpwl_f32(net_ptr, net_gate, x, y));
  log_info(buf);

  log_info("Phase 4: Congestion Refinement");
  fx_refine_cfg rc;
  fx_refine_cfg_default(&rc);
  rc.max_iterations = (int32_t)std::min<long long>(cfg.refinement_iterations, 1 << 30);
  rc.move_distance = cfg.move_distance;
  rc.overflow_threshold = cfg.overflow_threshold;
  rc.grid_cols = (int32_t)std::min<long long>(cfg.grid_cols, 1 << 30);
  rc.grid_rows = (int32_t)std::min<long long>(cfg.grid_rows, 1 << 30);
  fx_refine_stats rs{};
  if (fx_refine(ctx, d, &rc, x.data(), y.data(), &rs, nullptr) != FX_OK)
    return gpu_fail("refinement");
  const float hp = hpwl_f32(net_ptr, net_gate, x, y);
  std::snprintf(buf, sizeof buf, "Refinement done. HPWL=%.1f, max_overflow=%.1f", hp,
                rs.max_overflow);
  log_info(buf);
  fx_design_free(d);
  fx_ctx_destroy(ctx);

  log_info("Phase 5: Export");
  if (fx_def_write(cfg.output.c_str(), name, n, x.data(), y.data(), die[0], die[1], nullptr) !=
      FX_OK)
    return fail(std::string("Export error: ") + fx_last_error());
  log_info("Wrote DEF to " + cfg.output);
  std::snprintf(buf, sizeof buf, "Done! HPWL: %.1f", hp);
  log_info(buf);
  return 0;
}
