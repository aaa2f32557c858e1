// MuJoCo-Warp coupling kernels of the coupled environments (sm_100a): body poses into the
// solids of every world, solid loads out to MuJoCo's applied-force buffer. They replace the
// Warp kernels of envs/lbm/lbm_fluid_env_func.py and envs/lbm3d/lbm_fluid_env_3d_func.py with
// the same launch shape (nworld x selected solids) over batched per-world arrays
// [nworld][n_objects][...]. Each thread handles one (world, selected solid) pair; the work is
// a few hundred bytes per call, so these are launch-latency kernels meant to sit in the step's
// CUDA graph next to the stream-collide kernel rather than behind a host round trip.

#include <cmath>

#include "hl_common.cuh"

namespace hl {
namespace cpl {

constexpr int BLOCK = 128;

__device__ __forceinline__ bool pair_of(int nworld, int nsel, int& w, int& i) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nworld * nsel) return false;
  w = t / nsel;
  i = t % nsel;
  return true;
}

// extract_body_states(_3d), lbm_fluid_env_func.py:8-24 / lbm_fluid_env_3d_func.py:11-36
__global__ void body_states_kernel(int nworld, int nbody, int nsel, const float* xipos, const float* xquat,
                                   const int32_t* body_ids, float* pos_out, float* quat_out) {
  int w, i;
  if (!pair_of(nworld, nsel, w, i) || body_ids[i] < 0 || body_ids[i] >= nbody) return;
  const long long b = (long long)w * nbody + body_ids[i];
  const long long o = (long long)w * nsel + i;
  for (int k = 0; k < 3; ++k) pos_out[3 * o + k] = xipos[3 * b + k];
  for (int k = 0; k < 4; ++k) quat_out[4 * o + k] = xquat[4 * b + k];
}

// convert_and_update_solid_batch_3d, lbm_fluid_env_3d_func.py:42-100
__global__ void update3d_kernel(int nworld, int n, int nsel, const int32_t* solid_ids, const float* mj_pos,
                                const float* mj_quat, const float* mo, const float* lo, const float* scales, float* position,
                                float* quaternion, float* tf, float* tf_last, int32_t* init) {
  int w, i;
  if (!pair_of(nworld, nsel, w, i) || solid_ids[i] < 0 || solid_ids[i] >= n) return;
  const long long o = (long long)w * nsel + i;
  const long long s = (long long)w * n + solid_ids[i];
  const float sc = scales[i];
  float p[3];
  for (int k = 0; k < 3; ++k) {
    p[k] = (mj_pos[3 * o + k] - mo[3 * i + k]) * sc + lo[3 * i + k];
    position[3 * s + k] = p[k];
  }
  const float qw = mj_quat[4 * o], qx = mj_quat[4 * o + 1], qy = mj_quat[4 * o + 2], qz = mj_quat[4 * o + 3];
  quaternion[4 * s] = qw;
  quaternion[4 * s + 1] = qx;
  quaternion[4 * s + 2] = qy;
  quaternion[4 * s + 3] = qz;
  const bool initialized = init[s] > 0;
  if (initialized)
    for (int k = 0; k < 7; ++k) tf_last[7 * s + k] = tf[7 * s + k];
  const float t[7] = {p[0], p[1], p[2], qx, qy, qz, qw};  // wp.transform(p, wp.quat(x, y, z, w))
  for (int k = 0; k < 7; ++k) tf[7 * s + k] = t[k];
  if (!initialized) {
    for (int k = 0; k < 7; ++k) tf_last[7 * s + k] = t[k];
    init[s] = 1;
  }
}

// convert_and_update_solid_batch_2d, lbm_fluid_env_func.py:72-105
__global__ void update2d_kernel(int nworld, int n, int nsel, const int32_t* solid_ids, const float* mj_pos,
                                const float* mj_quat, const float* mo, const float* lo, const float* scales, float* position,
                                float* angle) {
  int w, i;
  if (!pair_of(nworld, nsel, w, i) || solid_ids[i] < 0 || solid_ids[i] >= n) return;
  const long long o = (long long)w * nsel + i;
  const long long s = (long long)w * n + solid_ids[i];
  const float sc = scales[i];
  position[2 * s] = (mj_pos[3 * o] - mo[2 * i]) * sc + lo[2 * i];
  position[2 * s + 1] = (mj_pos[3 * o + 1] - mo[2 * i + 1]) * sc + lo[2 * i + 1];
  const float qw = mj_quat[4 * o], qx = mj_quat[4 * o + 1], qy = mj_quat[4 * o + 2], qz = mj_quat[4 * o + 3];
  angle[s] = atan2f(2.f * (qw * qz + qx * qy), 1.f - 2.f * (qy * qy + qz * qz));
}

// extract_forces_torques_physical_3d (mode 0), extract_forces_torques_batch_3d (mode 1),
// extract_forces_torques_batch (mode 2, 2D loads)
__global__ void loads_kernel(int mode, int nworld, int n, int nsel, const int32_t* solid_ids, const float* force,
                             const float* torque, const float* scales, float fc, float tc, float* fo, float* to) {
  int w, i;
  if (!pair_of(nworld, nsel, w, i) || solid_ids[i] < 0 || solid_ids[i] >= n) return;
  const long long o = (long long)w * nsel + i;
  const long long s = (long long)w * n + solid_ids[i];
  if (mode == 2) {  // force = per world the planes solid_forcex, solid_forcey, torque of n solids
    const float sc = scales[i];
    const float* L = force + 3ll * n * w;
    const int k = solid_ids[i];
    fo[3 * o] = L[k] / sc;
    fo[3 * o + 1] = L[n + k] / sc;
    fo[3 * o + 2] = 0.f;
    to[3 * o] = 0.f;
    to[3 * o + 1] = 0.f;
    to[3 * o + 2] = L[2 * n + k] / sc;
    return;
  }
  for (int k = 0; k < 3; ++k) {
    if (mode == 0) {
      fo[3 * o + k] = force[3 * s + k] * fc;
      to[3 * o + k] = torque[3 * s + k] * tc;
    } else {
      const float sc = scales[i];
      fo[3 * o + k] = force[3 * s + k] / sc;
      to[3 * o + k] = torque[3 * s + k] / (sc * sc);
    }
  }
}

// fill_xfrc_kernel / fill_xfrc_3d_kernel, lbm_fluid_env_func.py:27-48 / lbm_fluid_env_3d_func.py:181-210
__global__ void xfrc_kernel(int nworld, int nbody, int nsel, const int32_t* body_ids, const float* forces,
                            const float* torques, float* xfrc) {
  int w, i;
  if (!pair_of(nworld, nsel, w, i) || body_ids[i] < 0 || body_ids[i] >= nbody) return;
  const long long o = (long long)w * nsel + i;
  const long long b = (long long)w * nbody + body_ids[i];
  for (int k = 0; k < 3; ++k) {
    xfrc[6 * b + k] = forces[3 * o + k];
    xfrc[6 * b + 3 + k] = torques[3 * o + k];
  }
}

inline unsigned blocks(int nworld, int nsel) { return unsigned((nworld * nsel + BLOCK - 1) / BLOCK); }

}  // namespace cpl
}  // namespace hl

using namespace hl;

#define HL_CPL_SIZES(nworld, nsel)                                                                          \
  HL_CHECK_ARG((nworld) >= 0 && (nsel) >= 0 && (long long)(nworld) * (nsel) < (1ll << 30),                \
               "coupling: bad sizes nworld=%d nsel=%d", int(nworld), int(nsel));                           \
  if ((nworld) == 0 || (nsel) == 0) return HL_OK

extern "C" int hl_couple_body_states(int nworld, int nbody, int nsel, const float* xipos, const float* xquat,
                                     const int32_t* body_ids, float* pos_out, float* quat_out, hl_stream stream) {
  HL_CPL_SIZES(nworld, nsel);
  HL_CHECK_ARG(nbody > 0 && xipos && xquat && body_ids && pos_out && quat_out, "extract_body_states: NULL buffer");
  cpl::body_states_kernel<<<cpl::blocks(nworld, nsel), cpl::BLOCK, 0, static_cast<cudaStream_t>(stream)>>>(
      nworld, nbody, nsel, xipos, xquat, body_ids, pos_out, quat_out);
  HL_LAUNCH_CHECK("extract_body_states");
  return HL_OK;
}

extern "C" int hl_couple3d_update_solids(int nworld, int n_objects, int nsel, const int32_t* solid_ids,
                                         const float* mj_pos, const float* mj_quat, const float* mujoco_origins,
                                         const float* lbm_origins, const float* scales, float* position,
                                         float* quaternion, float* transforms, float* transforms_last,
                                         int32_t* initialized, hl_stream stream) {
  HL_CPL_SIZES(nworld, nsel);
  HL_CHECK_ARG(n_objects > 0 && solid_ids && mj_pos && mj_quat && mujoco_origins && lbm_origins && scales && position &&
                   quaternion && transforms && transforms_last && initialized,
               "convert_and_update_solid_batch_3d: NULL buffer");
  cpl::update3d_kernel<<<cpl::blocks(nworld, nsel), cpl::BLOCK, 0, static_cast<cudaStream_t>(stream)>>>(
      nworld, n_objects, nsel, solid_ids, mj_pos, mj_quat, mujoco_origins, lbm_origins, scales, position, quaternion,
      transforms, transforms_last, initialized);
  HL_LAUNCH_CHECK("convert_and_update_solid_batch_3d");
  return HL_OK;
}

extern "C" int hl_couple2d_update_solids(int nworld, int n_objects, int nsel, const int32_t* solid_ids,
                                         const float* mj_pos, const float* mj_quat, const float* mujoco_origins,
                                         const float* lbm_origins, const float* scales, float* position, float* angle,
                                         hl_stream stream) {
  HL_CPL_SIZES(nworld, nsel);
  HL_CHECK_ARG(n_objects > 0 && solid_ids && mj_pos && mj_quat && mujoco_origins && lbm_origins && scales && position &&
                   angle,
               "convert_and_update_solid_batch_2d: NULL buffer");
  cpl::update2d_kernel<<<cpl::blocks(nworld, nsel), cpl::BLOCK, 0, static_cast<cudaStream_t>(stream)>>>(
      nworld, n_objects, nsel, solid_ids, mj_pos, mj_quat, mujoco_origins, lbm_origins, scales, position, angle);
  HL_LAUNCH_CHECK("convert_and_update_solid_batch_2d");
  return HL_OK;
}

extern "C" int hl_couple_loads(int mode, int nworld, int n_objects, int nsel, const int32_t* solid_ids,
                               const float* force, const float* torque, const float* scales, float force_conv,
                               float torque_conv, float* forces_out, float* torques_out, hl_stream stream) {
  HL_CHECK_ARG(mode >= 0 && mode <= 2, "extract_forces_torques: mode %d (0 physical, 1 / scale, 2 planar)", mode);
  HL_CPL_SIZES(nworld, nsel);
  HL_CHECK_ARG(n_objects > 0 && solid_ids && force && (torque || mode == 2) && forces_out && torques_out &&
                   (mode == 0 || scales),
               "extract_forces_torques: NULL buffer");
  cpl::loads_kernel<<<cpl::blocks(nworld, nsel), cpl::BLOCK, 0, static_cast<cudaStream_t>(stream)>>>(
      mode, nworld, n_objects, nsel, solid_ids, force, torque, scales, force_conv, torque_conv, forces_out, torques_out);
  HL_LAUNCH_CHECK("extract_forces_torques");
  return HL_OK;
}

extern "C" int hl_couple_fill_xfrc(int nworld, int nbody, int nsel, const int32_t* body_ids, const float* forces,
                                   const float* torques, float* xfrc, hl_stream stream) {
  HL_CPL_SIZES(nworld, nsel);
  HL_CHECK_ARG(nbody > 0 && body_ids && forces && torques && xfrc, "fill_xfrc: NULL buffer");
  cpl::xfrc_kernel<<<cpl::blocks(nworld, nsel), cpl::BLOCK, 0, static_cast<cudaStream_t>(stream)>>>(
      nworld, nbody, nsel, body_ids, forces, torques, xfrc);
  HL_LAUNCH_CHECK("fill_xfrc");
  return HL_OK;
}
