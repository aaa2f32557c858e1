// Masked world resets over device arrays of world descriptors (the reference's flows_wp):
// ResetSingleWorldFlow(3D), ResetSingleWorldSolidTransform(3D), ResetSingleWorldForces(3D)
// (envs/lbm/lbm_func.py:66-161, envs/lbm3d/lbm_func_3d.py:86-196), one launch for all worlds
// and all three parts. The mask is read on the device, as the reference's kernels read theirs,
// so a reset needs no host synchronisation and can sit in a CUDA graph.
//
// Values written. The reference rebuilds the rest state's populations (rho = 1, u = 0) and
// takes its moments: rho = 1, u = 0 and S = Pi / rho - cs2_local with cs2_local = Pi_xx
// ("Very Important!!!" quirk of the initial states), which is Pi_xx - Pi_xx = +0 in binary32 for
// every component since rho = 1. So a reset cell is rho = 1, u = 0, S = 0 in both buffers, with
// the body force zeroed; the encoded storages store rho - 1 = 0.
#include "hl_common.cuh"

namespace hl {
namespace rst {

template <class S>
__global__ void reset3d_kernel(const hl_flow3d* __restrict__ flows, const int32_t* __restrict__ mask, int what) {
  using R = typename S::R;
  using T = typename S::T;
  const int w = blockIdx.y;
  if (mask[w] == 0) return;
  const hl_flow3d f = flows[w];
  const long long N = (long long)f.nx * f.ny * f.nz;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if ((what & HL_RESET_FLOW) && i < N) {
    // stored rest state: rho (rho - 1 in the encoded storages), everything else 0
    R raw[10];
    for (int k = 0; k < 10; ++k) raw[k] = R(0);
    raw[0] = S::kEncoded ? R(0) : R(1);
    T* a = static_cast<T*>(f.m0);
    T* b = static_cast<T*>(f.m1);
    for (int k = 0; k < 10; ++k) {
      a[k * N + i] = S::from_r(raw[k]);
      b[k * N + i] = S::from_r(raw[k]);
    }
    if (f.force) f.force[i] = f.force[N + i] = f.force[2 * N + i] = 0.f;
  }
  // per-solid state: the first block of each world, a thread per solid
  if (blockIdx.x == 0 && int(threadIdx.x) < f.n_objects) {
    const int s = threadIdx.x;
    if (what & HL_RESET_SOLID_TRANSFORM) {  // identity transforms (p = 0, q = (0, 0, 0, 1)), not initialised
      for (int k = 0; k < 7; ++k) {
        const float v = k == 6 ? 1.f : 0.f;
        if (f.transforms) f.transforms[7 * s + k] = v;
        if (f.transforms_last) f.transforms_last[7 * s + k] = v;
      }
    }
    if ((what & (HL_RESET_SOLID_TRANSFORM | HL_RESET_INITIALIZED)) && f.initialized) f.initialized[s] = 0;
    if (what & HL_RESET_FORCES) {
      for (int k = 0; k < 3; ++k) {
        if (f.solid_force) f.solid_force[3 * s + k] = 0.f;
        if (f.solid_torque) f.solid_torque[3 * s + k] = 0.f;
      }
    }
  }
}

template <class S>
__global__ void reset2d_kernel(const hl_flow2d* __restrict__ flows, const int32_t* __restrict__ mask, int what) {
  using R = typename S::R;
  using T = typename S::T;
  const int w = blockIdx.y;
  if (mask[w] == 0) return;
  const hl_flow2d f = flows[w];
  const long long N = (long long)f.nx * f.ny;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if ((what & HL_RESET_FLOW) && i < N) {
    R raw[6];
    for (int k = 0; k < 6; ++k) raw[k] = R(0);
    raw[0] = S::kEncoded ? R(0) : R(1);
    T* a = static_cast<T*>(f.m0);
    T* b = static_cast<T*>(f.m1);
    for (int k = 0; k < 6; ++k) {
      a[k * N + i] = S::from_r(raw[k]);
      b[k * N + i] = S::from_r(raw[k]);
    }
    if (f.forcex) f.forcex[i] = 0.f;
    if (f.forcey) f.forcey[i] = 0.f;
  }
  // ResetSingleWorldSolidTransform: segments idx < solid_line_num[s] of every solid back to
  // (0, 0) in both transformed outlines; the segments past the count keep their values
  if ((what & HL_RESET_SOLID_TRANSFORM) && f.line_num && i < (long long)f.n_objects * f.max_segments) {
    const int s = int(i / f.max_segments), idx = int(i % f.max_segments);
    if (idx < f.line_num[s]) {
      const long long o = 2 * ((long long)s * f.max_segments + idx);
      if (f.line_tf) f.line_tf[o] = f.line_tf[o + 1] = 0.f;
      if (f.line_tf_last) f.line_tf_last[o] = f.line_tf_last[o + 1] = 0.f;
    }
  }
  if ((what & HL_RESET_FORCES) && blockIdx.x == 0 && int(threadIdx.x) < f.n_objects) {
    const int s = threadIdx.x;
    if (f.solid_forcex) f.solid_forcex[s] = 0.f;
    if (f.solid_forcey) f.solid_forcey[s] = 0.f;
    if (f.torque) f.torque[s] = 0.f;
  }
}

template <class S>
int launch3(const hl_flow3d* flows, int nworld, const int32_t* mask, int what, long long max_cells,
            cudaStream_t st) {
  const long long blocks = (max_cells + 255) / 256;
  reset3d_kernel<S><<<dim3(unsigned(blocks > 0 ? blocks : 1), unsigned(nworld)), 256, 0, st>>>(flows, mask, what);
  HL_LAUNCH_CHECK("ResetSingleWorldFlow3D");
  return HL_OK;
}

template <class S>
int launch2(const hl_flow2d* flows, int nworld, const int32_t* mask, int what, long long max_cells,
            cudaStream_t st) {
  const long long blocks = (max_cells + 255) / 256;
  reset2d_kernel<S><<<dim3(unsigned(blocks > 0 ? blocks : 1), unsigned(nworld)), 256, 0, st>>>(flows, mask, what);
  HL_LAUNCH_CHECK("ResetSingleWorldFlow");
  return HL_OK;
}

}  // namespace rst
}  // namespace hl

using namespace hl;

extern "C" int hl_d3q27_reset_worlds(const hl_flow3d* flows, int nworld, hl_dtype dtype, const int32_t* reset_mask,
                                     int what, long long max_cells, hl_stream stream) {
  HL_CHECK_ARG(flows != nullptr && reset_mask != nullptr, "reset_worlds_3d: flows or reset_mask is NULL");
  HL_CHECK_ARG(nworld >= 1 && nworld <= 65535, "reset_worlds_3d: %d worlds (1 .. 65535)", nworld);
  HL_CHECK_ARG((what & ~(HL_RESET_FLOW | HL_RESET_SOLID_TRANSFORM | HL_RESET_FORCES | HL_RESET_INITIALIZED)) == 0,
               "reset_worlds_3d: unknown parts %d", what);
  HL_CHECK_ARG(max_cells >= 0 && max_cells < (1ll << 40), "reset_worlds_3d: max_cells %lld", max_cells);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case HL_F32: return rst::launch3<StoreF32>(flows, nworld, reset_mask, what, max_cells, st);
    case HL_F64: return rst::launch3<StoreF64>(flows, nworld, reset_mask, what, max_cells, st);
    case HL_F16: return rst::launch3<StoreF16>(flows, nworld, reset_mask, what, max_cells, st);
    case HL_BF16: return rst::launch3<StoreBF16>(flows, nworld, reset_mask, what, max_cells, st);
  }
  set_error("reset_worlds_3d: bad dtype %d", int(dtype));
  return HL_ERR_ARG;
}

extern "C" int hl_d2q9_reset_worlds(const hl_flow2d* flows, int nworld, hl_dtype dtype, const int32_t* reset_mask,
                                    int what, long long max_cells, hl_stream stream) {
  HL_CHECK_ARG(flows != nullptr && reset_mask != nullptr, "reset_worlds_2d: flows or reset_mask is NULL");
  HL_CHECK_ARG(nworld >= 1 && nworld <= 65535, "reset_worlds_2d: %d worlds (1 .. 65535)", nworld);
  HL_CHECK_ARG((what & ~(HL_RESET_FLOW | HL_RESET_SOLID_TRANSFORM | HL_RESET_FORCES)) == 0,
               "reset_worlds_2d: unknown parts %d", what);
  HL_CHECK_ARG(max_cells >= 0 && max_cells < (1ll << 40), "reset_worlds_2d: max_cells %lld", max_cells);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case HL_F32: return rst::launch2<StoreF32>(flows, nworld, reset_mask, what, max_cells, st);
    case HL_F64: return rst::launch2<StoreF64>(flows, nworld, reset_mask, what, max_cells, st);
    case HL_F16: return rst::launch2<StoreF16>(flows, nworld, reset_mask, what, max_cells, st);
    case HL_BF16: return rst::launch2<StoreBF16>(flows, nworld, reset_mask, what, max_cells, st);
  }
  set_error("reset_worlds_2d: bad dtype %d", int(dtype));
  return HL_ERR_ARG;
}
