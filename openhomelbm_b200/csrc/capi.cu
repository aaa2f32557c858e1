// Error reporting and version of the C ABI (include/homelbm.h).
#include <cstdarg>
#include <cstdio>

#include "hl_common.cuh"

#include <cstring>

namespace hl {

static thread_local char g_err[512] = "";
int g_tune_d3_kernel = 0;
int g_tune_d3_chunks = 0;
int g_tune_d3_stages = 0;
int g_tune_d3_link_blocks = 0;

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

extern "C" int hl_set_tuning(const char* key, int value) {
  if (key == nullptr) {
    hl::set_error("hl_set_tuning: key is NULL");
    return HL_ERR_ARG;
  }
  if (!strcmp(key, "d3q27_kernel") && value >= 0 && value <= 2) {
    hl::g_tune_d3_kernel = value;
    return HL_OK;
  }
  if (!strcmp(key, "d3q27_chunks") && value >= 0 && value <= 64) {
    hl::g_tune_d3_chunks = value;
    return HL_OK;
  }
  if (!strcmp(key, "d3q27_link_blocks") && value >= 0 && value <= 4096) {
    hl::g_tune_d3_link_blocks = value;
    return HL_OK;
  }
  if (!strcmp(key, "d3q27_stages") && (value == 0 || (value >= 3 && value <= 5))) {
    hl::g_tune_d3_stages = value;
    return HL_OK;
  }
  hl::set_error("hl_set_tuning: unknown key or value (%s = %d)", key, value);
  return HL_ERR_ARG;
}
