// TEST INFRASTRUCTURE ONLY. Links the workload generator (the host-only
// fx_synth.cpp of the product sources) into oracle/_build/libsynth.so, so
// the CPU reference arm builds the same seeded netlists without loading the
// CUDA library. The generator reports errors through fx::set_error, which
// lives in the CUDA library; this is a plain stand-in for it.
#include <cstdarg>
#include <cstdio>

namespace fx {
thread_local char g_synth_err[512];
void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_synth_err, sizeof g_synth_err, fmt, ap);
  va_end(ap);
}
}  // namespace fx

extern "C" const char *or_synth_last_error(void) { return fx::g_synth_err; }
