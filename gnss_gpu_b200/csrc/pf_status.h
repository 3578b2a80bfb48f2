// pf_status.h -- thread-local error message behind pf_last_error().
// The reference reports failures by throwing std::runtime_error from
// CUDA_CHECK (include/gnss_gpu/cuda_check.h:8-17); across a C ABI the same
// information travels as a status code plus this message.
#pragma once
#include <stdarg.h>
#include <stdio.h>

#include "../../include/gnss_pf_b200.h"

namespace pfb {
extern thread_local char g_last_error[512];
}

inline int set_err(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(pfb::g_last_error, sizeof(pfb::g_last_error), fmt, ap);
  va_end(ap);
  return status;
}

inline void clear_err() { pfb::g_last_error[0] = '\0'; }

// Test hook behind pf_test_fail_alloc: true when the library's allocation
// about to be made is the one chosen to fail (counts down over calls).
bool pf_injected_alloc_failure();
