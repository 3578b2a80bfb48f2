// pf_status.cu -- storage of the per-thread error message.
#include "pf_status.h"

namespace pfb {
thread_local char g_last_error[512] = {0};
}

extern "C" const char* pf_last_error(void) { return pfb::g_last_error; }
extern "C" int pf_abi_version(void) { return PF_ABI_VERSION; }
