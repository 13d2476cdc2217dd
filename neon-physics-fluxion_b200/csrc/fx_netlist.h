// fx_netlist.h -- the host-side netlist behind the fx_netlist handle (the
// synthetic generators and the BLIF reader fill it).
#pragma once
#include <cstdint>
#include <vector>

struct fx_netlist {
  int32_t n = 0, m = 0;
  std::vector<int32_t> net_ptr, net_gate;
  std::vector<float> w, h, x, y;
  float die_w = 0.f, die_h = 0.f;
  std::vector<int32_t> leaf_ptr;
  std::vector<float> region;
};
