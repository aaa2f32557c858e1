// Error reporting and version of the C ABI (include/homelbm.h).
#include <cstdarg>
#include <cstdio>

#include "hl_common.cuh"

namespace hl {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int cuda_status(cudaError_t e, const char* what) {
  set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
  return HL_ERR_CUDA;
}

}  // namespace hl

extern "C" const char* hl_last_error(void) { return hl::g_err; }
extern "C" const char* hl_version(void) { return "openhomelbm_b200 0.1 (sm_100a)"; }
