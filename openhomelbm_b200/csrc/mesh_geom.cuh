// Rigid-body transforms of the mesh solids (p + rotation by a unit quaternion x, y, z, w; the
// layout of the reference's wp.transform, envs/lbm3d/lbm_core_3d.py:91-119), shared by the cut
// links and the field diagnostics so both map world points into a body frame the same way.
#pragma once

namespace hl {
namespace geo {

template <class R> struct V3 {
  R x, y, z;
};
template <class R> struct Xf {
  V3<R> p;
  R qx, qy, qz, qw;
};

// Rotation by a unit quaternion: v (2 w^2 - 1) + 2 w (q_v x v) + 2 (q_v . v) q_v.
template <class R> __device__ __forceinline__ V3<R> qrot(R qx, R qy, R qz, R qw, V3<R> v) {
  const R c = R(2) * qw * qw - R(1);
  const R d = R(2) * (qx * v.x + qy * v.y + qz * v.z);
  const R e = R(2) * qw;
  const R cx = qy * v.z - qz * v.y, cy = qz * v.x - qx * v.z, cz = qx * v.y - qy * v.x;
  return {v.x * c + cx * e + qx * d, v.y * c + cy * e + qy * d, v.z * c + cz * e + qz * d};
}
template <class R> __device__ __forceinline__ Xf<R> load_xf(const float* t) {
  return {{R(t[0]), R(t[1]), R(t[2])}, R(t[3]), R(t[4]), R(t[5]), R(t[6])};
}
template <class R> __device__ __forceinline__ Xf<R> xinv(const Xf<R>& t) {
  const V3<R> p = qrot(-t.qx, -t.qy, -t.qz, t.qw, t.p);
  return {{-p.x, -p.y, -p.z}, -t.qx, -t.qy, -t.qz, t.qw};
}
template <class R> __device__ __forceinline__ V3<R> xpoint(const Xf<R>& t, V3<R> v) {
  const V3<R> r = qrot(t.qx, t.qy, t.qz, t.qw, v);
  return {r.x + t.p.x, r.y + t.p.y, r.z + t.p.z};
}

}  // namespace geo
}  // namespace hl
