// pf_status.cu -- storage of the per-thread error message and the
// allocation-failure test hook.
#include <atomic>

#include "pf_status.h"

namespace pfb {
thread_local char g_last_error[512] = {0};
}

extern "C" const char* pf_last_error(void) { return pfb::g_last_error; }
extern "C" int pf_abi_version(void) { return PF_ABI_VERSION; }

namespace {
std::atomic<int> g_fail_alloc{0};  // > 0: the g_fail_alloc-th next allocation fails
}

bool pf_injected_alloc_failure() {
  int v = g_fail_alloc.load();
  while (v > 0) {
    if (g_fail_alloc.compare_exchange_weak(v, v - 1)) return v == 1;
  }
  return false;
}

extern "C" int pf_test_fail_alloc(int nth) {
  clear_err();
  if (nth < 0) return set_err(PF_EINVAL, "nth must be >= 0");
  g_fail_alloc.store(nth);
  return PF_OK;
}
