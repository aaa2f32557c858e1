// Error reporting and version of the C ABI (include/homelbm.h).
#include <cstdarg>
#include <cstdio>

#include "hl_common.cuh"

#include <cstring>
#include <mutex>
#include <set>
#include <tuple>

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

int device_sms() {
  constexpr int kMaxDev = 128;
  static int cache[kMaxDev] = {};  // 0: not queried yet (written once per device, int-sized)
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
  if (dev < kMaxDev && __atomic_load_n(&cache[dev], __ATOMIC_ACQUIRE) > 0) return cache[dev];
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  if (dev < kMaxDev) __atomic_store_n(&cache[dev], n, __ATOMIC_RELEASE);
  return n;
}

int set_smem_attr(const void* kernel, int bytes, const char* what) {
  static std::mutex mu;
  static std::set<std::tuple<const void*, int, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, what);
  const auto key = std::make_tuple(kernel, dev, bytes);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(key)) return HL_OK;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return cuda_status(e, what);
  done.insert(key);
  return HL_OK;
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

namespace hl {
namespace {

// one thread per cell (per pair of cells when paired), every moment of it
template <class S>
__global__ void round_to_storage_kernel(const float* __restrict__ v, long long n, int nm, long long first, bool paired,
                                        typename S::T* __restrict__ out) {
  using T = typename S::T;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long c = paired ? 2 * t : t;
  if (c >= n) return;
  const unsigned cs0 = unsigned(first + c) * 0x9e3779b9u;
  if (paired && c + 1 < n) {
    const unsigned cs1 = unsigned(first + c + 1) * 0x9e3779b9u;
    for (int k = 0; k < nm; ++k) {
      T a, b;
      S::from_r_cell2(v[k * n + c], v[k * n + c + 1], cs0, cs1, unsigned(k), a, b);
      out[k * n + c] = a;
      out[k * n + c + 1] = b;
    }
  } else {
    for (int k = 0; k < nm; ++k) out[k * n + c] = S::from_r_cell(v[k * n + c], cs0, unsigned(k));
  }
}

template <class S>
int launch_round(const float* v, long long n, int nm, long long first, bool paired, void* out, cudaStream_t st) {
  const long long threads = paired ? (n + 1) / 2 : n;
  round_to_storage_kernel<S><<<unsigned((threads + 255) / 256), 256, 0, st>>>(v, n, nm, first, paired,
                                                                              static_cast<typename S::T*>(out));
  HL_LAUNCH_CHECK("round to storage");
  return HL_OK;
}

}  // namespace
}  // namespace hl

extern "C" int hl_round_to_storage(const float* values, long long n_cells, int n_moments, hl_dtype dtype,
                                   long long first_cell, int paired, void* out, hl_stream stream) {
  using namespace hl;
  HL_CHECK_ARG(n_cells >= 0 && n_cells < (1ll << 38) && n_moments >= 1 && n_moments <= 64,
               "round to storage: %lld cells of %d moments", n_cells, n_moments);
  HL_CHECK_ARG(n_cells == 0 || (values != nullptr && out != nullptr), "round to storage: values or out is NULL");
  HL_CHECK_ARG(first_cell >= 0, "round to storage: negative first cell");
  if (n_cells == 0) return HL_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool p = paired != 0;
  switch (dtype) {
    case HL_F32: return launch_round<StoreF32>(values, n_cells, n_moments, first_cell, p, out, st);
    case HL_F16: return launch_round<StoreF16>(values, n_cells, n_moments, first_cell, p, out, st);
    case HL_BF16: return launch_round<StoreBF16>(values, n_cells, n_moments, first_cell, p, out, st);
    case HL_F64: return launch_round<StoreF64>(values, n_cells, n_moments, first_cell, p, out, st);
  }
  set_error("round to storage: dtype %d", int(dtype));
  return HL_ERR_ARG;
}
