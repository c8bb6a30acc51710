#include "abi_common.h"

#include "mvmc_b200.h"

namespace {
thread_local std::string g_last_error;
}

namespace mvmcb {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace mvmcb

extern "C" const char* mvmc_b200_last_error(void) { return g_last_error.c_str(); }

extern "C" void mvmc_b200_default_options(mvmc_b200_options* opt) {
  if (!opt) return;
  opt->walkers = 1;
  opt->precision = 64;
  opt->refresh_sweeps = 0;
  opt->saved_per_walker = 0;
  opt->seed = -1;
  opt->device = 0;
  opt->sr_precision = 0;
  opt->refresh_guard = 0.0;
  opt->c_order = 0;
  opt->sr_gram = 0;
  opt->measure_resident = 0;
}
