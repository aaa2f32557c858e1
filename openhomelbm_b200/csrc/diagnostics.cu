// Field diagnostics (sm_100a): headless images of a world's current moments with the arithmetic
// of the reference's display kernels, written to caller-owned device buffers instead of a GL
// texture:
//   2D (envs/lbm/lbm_func.py): get_u_img 163-166, get_velocity_rgb 169-193, get_vorticity_img
//      196-233, get_vorticity_with_solid_img 236-319, get_solid_boundary_img 804-866 with
//      point_segment_dist 792-801;
//   3D (envs/lbm3d/lbm_func_3d.py): get_u_img_xy_3d / _yz_3d 753-776, get_vorticity_xy_3d /
//      _yz_3d 779-840, the _with_solid_3d variants 843-987, the projections 990-1313 with
//      any_mesh_hit_along_ray_3d 320-362.
//   live view (tools/lbm3d_realtime_control.py): _extract_live_vorticity_slices 68-148 with
//      its log-magnitude histogram, _live_vorticity_to_rgba 157-182 (into a device RGBA buffer
//      instead of the GL atlas); tools/lbm2d_realtime_control.py: lbm_uimg_to_rgba_kernel
//      417-464 (into a device buffer instead of the GL PBO), set_local_force_kernel 144-157.
// Velocities are the decoded u of the current buffer, in binary32 as the reference's fields.
//
// Third-party queries of the reference, restated: wp.mesh_query_ray (any hit with
// 0 <= t <= max_t) is a Moller-Trumbore test against every triangle of the solid in its body
// frame; wp.mesh_query_point_sign_normal (inside or outside, and the closest surface point,
// within max_dist = 100) is the closest point over the triangles (Ericson, "Real-Time
// Collision Detection", 5.1.5) and, for the sign, the parity of the crossings of a ray from the
// point (a closed mesh: odd = inside, which is what the signed query reports for one).

#include <cmath>

#include "hl_common.cuh"
#include "mesh_geom.cuh"

namespace hl {
namespace diag {

using namespace geo;

constexpr int BLOCK = 256;
constexpr float SOLID_MARK = 1000.f;  // the reference's sentinel for solid pixels

template <class S> __device__ __forceinline__ float vel(const void* cur, long long N, long long i, int comp, float us) {
  using T = typename S::T;
  const auto raw = S::to_r(static_cast<const T*>(cur)[(1 + comp) * N + i]);
  return S::kEncoded ? float(raw) * us : float(raw);
}

// --------------------------------------------------------------------------------------- 2D
struct W2 {
  int nx, ny;
  const void* cur;
  float us;
};

template <class S> __device__ __forceinline__ float u2(const W2& w, int x, int y, int comp) {
  return vel<S>(w.cur, (long long)w.nx * w.ny, (long long)x * w.ny + y, comp, w.us);
}

// dv/dx - du/dy, central inside, one-sided on the border rows (lbm_func.py:196-233)
template <class S> __device__ float vorticity2(const W2& w, int x, int y, float h) {
  float dvdx, dudy;
  if (x == 0)
    dvdx = (u2<S>(w, x + 1, y, 1) - u2<S>(w, x, y, 1)) / h;
  else if (x == w.nx - 1)
    dvdx = (u2<S>(w, x, y, 1) - u2<S>(w, x - 1, y, 1)) / h;
  else
    dvdx = (u2<S>(w, x + 1, y, 1) - u2<S>(w, x - 1, y, 1)) / (2.f * h);
  if (y == 0)
    dudy = (u2<S>(w, x, y + 1, 0) - u2<S>(w, x, y, 0)) / h;
  else if (y == w.ny - 1)
    dudy = (u2<S>(w, x, y, 0) - u2<S>(w, x, y - 1, 0)) / h;
  else
    dudy = (u2<S>(w, x, y + 1, 0) - u2<S>(w, x, y - 1, 0)) / (2.f * h);
  return dvdx - dudy;
}

// point_segment_dist (lbm_func.py:792-801)
__device__ __forceinline__ float point_segment_dist(float px, float py, float ax, float ay, float bx, float by) {
  const float abx = bx - ax, aby = by - ay, apx = px - ax, apy = py - ay;
  const float len_sq = abx * abx + aby * aby;
  if (len_sq == 0.f) return sqrtf(apx * apx + apy * apy);
  const float t = fminf(fmaxf((apx * abx + apy * aby) / len_sq, 0.f), 1.f);
  const float cx = ax + abx * t, cy = ay + aby * t;
  return sqrtf((px - cx) * (px - cx) + (py - cy) * (py - cy));
}

// Inside a polygon (even-odd rule with a +x ray) or within `thickness` of its outline, for any
// solid (get_vorticity_with_solid_img / get_solid_boundary_img, lbm_func.py:243-284, 810-862).
__device__ bool solid_pixel(const hl_solids2d& s, int nx, float px, float py, float thickness) {
  float min_d = 1.0e6f;
  bool inside = false;
  for (int o = 0; o < s.n_objects; ++o) {
    const float scale = s.scale[o] * float(nx);
    const float cx = s.position[2 * o], cy = s.position[2 * o + 1];
    const float max_r = s.max_radius[o] * scale * scale;
    if ((px - cx) * (px - cx) + (py - cy) * (py - cy) > max_r + thickness) continue;
    const int n = s.line_num[o];
    const float* tf = s.line_tf + size_t(o) * s.max_segments * 2;
    int crossings = 0;
    for (int k = 0; k < n; ++k) {
      const int k1 = k + 1 == n ? 0 : k + 1;
      const float x1 = tf[2 * k], y1 = tf[2 * k + 1], x2 = tf[2 * k1], y2 = tf[2 * k1 + 1];
      const float d = point_segment_dist(px, py, x1, y1, x2, y2);
      if (d < min_d) min_d = d;
      if ((y1 > py) != (y2 > py)) {
        const float ix = x1 + (py - y1) * (x2 - x1) / (y2 - y1);
        if (px < ix) ++crossings;
      }
    }
    if (crossings & 1) inside = true;
  }
  return inside || min_d < thickness;
}

struct Args2 {
  W2 w;
  hl_solids2d s;
  bool solids;
  int kind;  // 0 |u|, 1 velocity rgb, 2 vorticity, 3 solid image
  float param, h, thickness;
  float* out;
};

template <class S> __global__ void __launch_bounds__(BLOCK) image2d_kernel(const __grid_constant__ Args2 a) {
  const long long i = (long long)blockIdx.x * BLOCK + threadIdx.x;
  if (i >= (long long)a.w.nx * a.w.ny) return;
  const int x = int(i / a.w.ny), y = int(i % a.w.ny);
  if (a.kind == 0) {
    const float ux = u2<S>(a.w, x, y, 0), uy = u2<S>(a.w, x, y, 1);
    a.out[i] = sqrtf(ux * ux + uy * uy);
  } else if (a.kind == 1) {  // get_velocity_rgb: magnitude, x and y velocity mapped to [0, 1]
    const float ux = u2<S>(a.w, x, y, 0), uy = u2<S>(a.w, x, y, 1), m = a.param;
    const float mag = sqrtf(ux * ux + uy * uy);
    a.out[3 * i] = fminf(fmaxf(mag / m, 0.f), 1.f);
    a.out[3 * i + 1] = fminf(fmaxf((ux + m) / (2.f * m), 0.f), 1.f);
    a.out[3 * i + 2] = fminf(fmaxf((uy + m) / (2.f * m), 0.f), 1.f);
  } else if (a.kind == 2) {
    if (a.solids && solid_pixel(a.s, a.w.nx, float(x), float(y), a.thickness)) {
      a.out[i] = SOLID_MARK;
      return;
    }
    a.out[i] = vorticity2<S>(a.w, x, y, a.h);
  } else {
    a.out[i] = solid_pixel(a.s, a.w.nx, float(x), float(y), a.thickness) ? 1.f : 0.f;
  }
}

// --------------------------------------------------------------------------------------- 3D
struct W3 {
  int n[3];
  const void* cur;
  const int32_t* flag;
  float us;
};

template <class S> __device__ __forceinline__ float u3(const W3& w, const int c[3], int comp) {
  const long long N = (long long)w.n[0] * w.n[1] * w.n[2];
  return vel<S>(w.cur, N, ((long long)c[0] * w.n[1] + c[1]) * w.n[2] + c[2], comp, w.us);
}
__device__ __forceinline__ int flag_of(const W3& w, const int c[3]) {
  if (w.flag) return w.flag[((long long)c[0] * w.n[1] + c[1]) * w.n[2] + c[2]];
  // no flag array: the border cells are walls (InitBoundary3D)
  for (int a = 0; a < 3; ++a)
    if (c[a] == 0 || c[a] == w.n[a] - 1) return ML_WALL;
  return ML_FLUID;
}

// d u[comp] / d x[axis] at c: central inside, one-sided on the border (lbm_func_3d.py:779-840)
template <class S> __device__ float deriv(const W3& w, const int c[3], int comp, int axis, float h) {
  int p[3] = {c[0], c[1], c[2]}, m[3] = {c[0], c[1], c[2]};
  if (c[axis] == 0) {
    p[axis] = c[axis] + 1;
    return (u3<S>(w, p, comp) - u3<S>(w, c, comp)) / h;
  }
  if (c[axis] == w.n[axis] - 1) {
    m[axis] = c[axis] - 1;
    return (u3<S>(w, c, comp) - u3<S>(w, m, comp)) / h;
  }
  p[axis] = c[axis] + 1;
  m[axis] = c[axis] - 1;
  return (u3<S>(w, p, comp) - u3<S>(w, m, comp)) / (2.f * h);
}
// vorticity component along axis a: z: dv/dx - du/dy; x: dw/dy - dv/dz; y: du/dz - dw/dx
template <class S> __device__ float vorticity3(const W3& w, const int c[3], int a, float h) {
  if (a == 2) return deriv<S>(w, c, 1, 0, h) - deriv<S>(w, c, 0, 1, h);
  if (a == 0) return deriv<S>(w, c, 2, 1, h) - deriv<S>(w, c, 1, 2, h);
  return deriv<S>(w, c, 0, 2, h) - deriv<S>(w, c, 2, 0, h);
}

// Any double-sided hit 0 <= t <= max_t of o + t d with the triangles tri[0..ntri), boxes of the
// triangle and of the segment [o, o + max_t d] tested first.
__device__ bool ray_any(const float* tri, int ntri, V3<float> o, V3<float> d, float max_t) {
  const float ex = o.x + d.x * max_t, ey = o.y + d.y * max_t, ez = o.z + d.z * max_t;
  const float sx0 = fminf(o.x, ex) - 1e-3f, sx1 = fmaxf(o.x, ex) + 1e-3f;
  const float sy0 = fminf(o.y, ey) - 1e-3f, sy1 = fmaxf(o.y, ey) + 1e-3f;
  const float sz0 = fminf(o.z, ez) - 1e-3f, sz1 = fmaxf(o.z, ez) + 1e-3f;
  for (int k = 0; k < ntri; ++k) {
    const float* v = tri + 9 * k;
    if (fmaxf(fmaxf(v[0], v[3]), v[6]) < sx0 || fminf(fminf(v[0], v[3]), v[6]) > sx1 ||
        fmaxf(fmaxf(v[1], v[4]), v[7]) < sy0 || fminf(fminf(v[1], v[4]), v[7]) > sy1 ||
        fmaxf(fmaxf(v[2], v[5]), v[8]) < sz0 || fminf(fminf(v[2], v[5]), v[8]) > sz1)
      continue;
    const float e1x = v[3] - v[0], e1y = v[4] - v[1], e1z = v[5] - v[2];
    const float e2x = v[6] - v[0], e2y = v[7] - v[1], e2z = v[8] - v[2];
    const float px = d.y * e2z - d.z * e2y, py = d.z * e2x - d.x * e2z, pz = d.x * e2y - d.y * e2x;
    const float det = e1x * px + e1y * py + e1z * pz;
    if (det == 0.f) continue;
    const float inv = 1.f / det;
    const float sx = o.x - v[0], sy = o.y - v[1], sz = o.z - v[2];
    const float u = (sx * px + sy * py + sz * pz) * inv;
    if (u < 0.f || u > 1.f) continue;
    const float qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
    const float w = (d.x * qx + d.y * qy + d.z * qz) * inv;
    if (w < 0.f || u + w > 1.f) continue;
    const float t = (e2x * qx + e2y * qy + e2z * qz) * inv;
    if (t >= 0.f && t <= max_t) return true;
  }
  return false;
}

// Crossings with t > 0 of the ray from o along a fixed direction that no axis-aligned feature
// lines up with: odd for a point inside a closed mesh.
__device__ int crossings(const float* tri, int ntri, V3<float> o) {
  const V3<float> d{0.5773503f, 0.5773491f, 0.5773515f};
  int n = 0;
  for (int k = 0; k < ntri; ++k) {
    const float* v = tri + 9 * k;
    const float e1x = v[3] - v[0], e1y = v[4] - v[1], e1z = v[5] - v[2];
    const float e2x = v[6] - v[0], e2y = v[7] - v[1], e2z = v[8] - v[2];
    const float px = d.y * e2z - d.z * e2y, py = d.z * e2x - d.x * e2z, pz = d.x * e2y - d.y * e2x;
    const float det = e1x * px + e1y * py + e1z * pz;
    if (det == 0.f) continue;
    const float inv = 1.f / det;
    const float sx = o.x - v[0], sy = o.y - v[1], sz = o.z - v[2];
    const float u = (sx * px + sy * py + sz * pz) * inv;
    if (u < 0.f || u > 1.f) continue;
    const float qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
    const float w = (d.x * qx + d.y * qy + d.z * qz) * inv;
    if (w < 0.f || u + w > 1.f) continue;
    if ((e2x * qx + e2y * qy + e2z * qz) * inv > 0.f) ++n;
  }
  return n;
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return ax * bx + ay * by + az * bz;
}
// Squared distance from p to triangle abc: the closest point by Voronoi region (Ericson 5.1.5).
__device__ float tri_dist2(const float* v, V3<float> p) {
  const float ax = v[0], ay = v[1], az = v[2];
  const float abx = v[3] - ax, aby = v[4] - ay, abz = v[5] - az;
  const float acx = v[6] - ax, acy = v[7] - ay, acz = v[8] - az;
  const float apx = p.x - ax, apy = p.y - ay, apz = p.z - az;
  float cx, cy, cz;  // closest point
  const float d1 = dot3(abx, aby, abz, apx, apy, apz), d2 = dot3(acx, acy, acz, apx, apy, apz);
  const float bpx = p.x - v[3], bpy = p.y - v[4], bpz = p.z - v[5];
  const float d3 = dot3(abx, aby, abz, bpx, bpy, bpz), d4 = dot3(acx, acy, acz, bpx, bpy, bpz);
  const float cpx = p.x - v[6], cpy = p.y - v[7], cpz = p.z - v[8];
  const float d5 = dot3(abx, aby, abz, cpx, cpy, cpz), d6 = dot3(acx, acy, acz, cpx, cpy, cpz);
  const float vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
  if (d1 <= 0.f && d2 <= 0.f) {  // vertex a
    cx = ax, cy = ay, cz = az;
  } else if (d3 >= 0.f && d4 <= d3) {  // vertex b
    cx = v[3], cy = v[4], cz = v[5];
  } else if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {  // edge ab
    const float t = d1 / (d1 - d3);
    cx = ax + t * abx, cy = ay + t * aby, cz = az + t * abz;
  } else if (d6 >= 0.f && d5 <= d6) {  // vertex c
    cx = v[6], cy = v[7], cz = v[8];
  } else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {  // edge ac
    const float t = d2 / (d2 - d6);
    cx = ax + t * acx, cy = ay + t * acy, cz = az + t * acz;
  } else if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {  // edge bc
    const float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    cx = v[3] + t * (v[6] - v[3]), cy = v[4] + t * (v[7] - v[4]), cz = v[5] + t * (v[8] - v[5]);
  } else {  // face interior
    const float den = 1.f / (va + vb + vc), sv = vb * den, sw = vc * den;
    cx = ax + abx * sv + acx * sw, cy = ay + aby * sv + acy * sw, cz = az + abz * sv + acz * sw;
  }
  return (p.x - cx) * (p.x - cx) + (p.y - cy) * (p.y - cy) + (p.z - cz) * (p.z - cz);
}

// The solid overlay of the *_with_solid_3d slices (lbm_func_3d.py:851-890): ML_SOLID flag, or
// inside a mesh, or within `thickness` of it (body frame, scaled), the query limited to 100.
__device__ bool solid_voxel(const W3& w, const hl_solids3d& s, const int c[3], float thickness) {
  if (w.flag && flag_of(w, c) == ML_SOLID) return true;
  const V3<float> pos{float(c[0]), float(c[1]), float(c[2])};
  for (int o = 0; o < s.n_objects; ++o) {
    const int t0 = s.tri_offset[o], ntri = s.tri_offset[o + 1] - t0;
    if (ntri == 0) continue;
    const Xf<float> inv = xinv(load_xf<float>(s.transforms + 7 * o));
    const V3<float> lp = xpoint(inv, pos);
    const V3<float> lo{lp.x / s.scale_sizes[3 * o], lp.y / s.scale_sizes[3 * o + 1], lp.z / s.scale_sizes[3 * o + 2]};
    const float* tri = s.tris + 9ll * t0;
    float best = 1.0e30f;
    for (int k = 0; k < ntri; ++k) best = fminf(best, tri_dist2(tri + 9 * k, lo));
    if (best > 100.f * 100.f) continue;  // no surface point within max_dist: the query fails
    if (crossings(tri, ntri, lo) & 1) return true;
    if (sqrtf(best) < thickness) return true;
  }
  return false;
}

// any_mesh_hit_along_ray_3d (lbm_func_3d.py:320-362)
__device__ bool any_mesh_hit(const hl_solids3d& s, V3<float> origin, V3<float> dir, float max_t) {
  for (int o = 0; o < s.n_objects; ++o) {
    const int t0 = s.tri_offset[o], ntri = s.tri_offset[o + 1] - t0;
    if (ntri == 0) continue;
    const Xf<float> inv = xinv(load_xf<float>(s.transforms + 7 * o));
    const V3<float> lp = xpoint(inv, origin);
    const V3<float> ld = qrot(inv.qx, inv.qy, inv.qz, inv.qw, dir);
    const float sx = s.scale_sizes[3 * o], sy = s.scale_sizes[3 * o + 1], sz = s.scale_sizes[3 * o + 2];
    if (ray_any(s.tris + 9ll * t0, ntri, {lp.x / sx, lp.y / sy, lp.z / sz}, {ld.x / sx, ld.y / sy, ld.z / sz}, max_t))
      return true;
  }
  return false;
}

struct Args3 {
  W3 w;
  hl_solids3d s;
  bool solids;
  int mode;   // 0 slice, 1 projection
  int axis;   // slice normal / view axis (0 x, 1 y, 2 z)
  int index;  // slice position
  int kind;   // slice: 0 |u|, 1 vorticity; projection: 0 max |u|, 1 first |u| from the viewer, 2 vorticity
  float h, thickness;
  float* out;
};

// Output pixel (i, j) of the plane normal to `axis`: the two other axes in increasing order
// (axis 2: (x, y); axis 0: (y, z); axis 1: (x, z)), j fastest.
__host__ __device__ __forceinline__ void plane_axes(int axis, int& a, int& b) {
  a = axis == 0 ? 1 : 0;
  b = axis == 2 ? 1 : 2;
}

template <class S> __global__ void __launch_bounds__(BLOCK) image3d_kernel(const __grid_constant__ Args3 a) {
  int pa, pb;
  plane_axes(a.axis, pa, pb);
  const int na = a.w.n[pa], nb = a.w.n[pb], nl = a.w.n[a.axis];
  const long long i = (long long)blockIdx.x * BLOCK + threadIdx.x;
  if (i >= (long long)na * nb) return;
  int c[3];
  c[pa] = int(i / nb);
  c[pb] = int(i % nb);
  if (a.mode == 0) {
    c[a.axis] = a.index;
    if (a.kind == 0) {
      const float ux = u3<S>(a.w, c, 0), uy = u3<S>(a.w, c, 1), uz = u3<S>(a.w, c, 2);
      a.out[i] = sqrtf(ux * ux + uy * uy + uz * uz);
      return;
    }
    if (a.solids && solid_voxel(a.w, a.s, c, a.thickness)) {
      a.out[i] = SOLID_MARK;
      return;
    }
    a.out[i] = vorticity3<S>(a.w, c, a.axis, a.h);
    return;
  }
  // projections: the viewer sits beyond the high end of the view axis, looking down it
  V3<float> origin{float(c[0]), float(c[1]), float(c[2])}, dir{0.f, 0.f, 0.f};
  (a.axis == 0 ? origin.x : a.axis == 1 ? origin.y : origin.z) = float(nl) + 1.f;
  (a.axis == 0 ? dir.x : a.axis == 1 ? dir.y : dir.z) = -1.f;
  const float max_t = float(nl) + 2.f;
  if (a.kind == 1) {  // get_u_projection_topdown_3d: silhouette first, then the first moving cell
    if (a.solids && any_mesh_hit(a.s, origin, dir, max_t)) {
      a.out[i] = SOLID_MARK;
      return;
    }
    float result = 0.f;
    for (int l = nl - 1; l >= 0; --l) {
      c[a.axis] = l;
      if (flag_of(a.w, c) == ML_WALL) continue;
      const float ux = u3<S>(a.w, c, 0), uy = u3<S>(a.w, c, 1), uz = u3<S>(a.w, c, 2);
      const float m = sqrtf(ux * ux + uy * uy + uz * uz);
      if (m > 1e-8f) {
        result = m;
        break;
      }
    }
    a.out[i] = result;
    return;
  }
  float best = 0.f;
  if (a.kind == 0) {  // maximum |u| along the column
    for (int l = nl - 1; l >= 0; --l) {
      c[a.axis] = l;
      if (flag_of(a.w, c) == ML_WALL) continue;
      const float ux = u3<S>(a.w, c, 0), uy = u3<S>(a.w, c, 1), uz = u3<S>(a.w, c, 2);
      const float m = sqrtf(ux * ux + uy * uy + uz * uz);
      if (m > best) best = m;
    }
  } else {  // the vorticity component along the view axis of largest magnitude, sign kept
    for (int l = 1; l < nl - 1; ++l) {
      c[a.axis] = l;
      if (flag_of(a.w, c) == ML_WALL) continue;
      const float v = vorticity3<S>(a.w, c, a.axis, a.h);
      if (fabsf(v) > fabsf(best)) best = v;
    }
  }
  a.out[i] = a.solids && any_mesh_hit(a.s, origin, dir, max_t) ? SOLID_MARK : best;
}

// ------------------------------------------------------------------------------- live view
constexpr int LIVE_BINS = 256;
constexpr float LIVE_LOG_MIN = -18.420680743952367f;  // log(1e-8)
constexpr float LIVE_LOG_MAX = 0.0f;                   // log(1)

struct ArgsLive {
  W3 w;
  const int32_t* slice_pos;
  int n_slices, width, height, stride, slice_axis, color_axis, margin, collect;
  float* values;
  int32_t* hist;
};

// One sample of a stack of planes (p, q, slice) sampled every `stride` cells: a vorticity
// component from central differences clamped at the border (divided by the clamped span),
// zero within `margin` of a face; |value| > 1e-8 counts in the bin of its log magnitude over
// [log 1e-8, log 1]. A slice position outside the grid gives zeros and no count.
template <class S> __global__ void __launch_bounds__(BLOCK) live_slices_kernel(const __grid_constant__ ArgsLive a) {
  const long long per = (long long)a.width * a.height;
  const long long i = (long long)blockIdx.x * BLOCK + threadIdx.x;
  if (i >= per * a.n_slices) return;
  const int slice = int(i / per);
  const int rem = int(i - (long long)slice * per);
  const int q = rem / a.width, p = rem - q * a.width;
  const int nx = a.w.n[0], ny = a.w.n[1], nz = a.w.n[2];
  const int pos = a.slice_pos[slice];
  const int along = a.slice_axis == 0 ? nx : a.slice_axis == 1 ? ny : nz;
  if (pos < 0 || pos >= along) {
    a.values[i] = 0.f;
    return;
  }
  int x, y, z;
  if (a.slice_axis == 0) {
    x = pos, y = min(p * a.stride, ny - 1), z = min(q * a.stride, nz - 1);
  } else if (a.slice_axis == 1) {
    x = min(p * a.stride, nx - 1), y = pos, z = min(q * a.stride, nz - 1);
  } else {
    x = min(p * a.stride, nx - 1), y = min(q * a.stride, ny - 1), z = pos;
  }
  const int xm = max(x - 1, 0), xp = min(x + 1, nx - 1);
  const int ym = max(y - 1, 0), yp = min(y + 1, ny - 1);
  const int zm = max(z - 1, 0), zp = min(z + 1, nz - 1);
  const float inv_dx = 1.f / float(max(xp - xm, 1));
  const float inv_dy = 1.f / float(max(yp - ym, 1));
  const float inv_dz = 1.f / float(max(zp - zm, 1));
  auto u = [&](int cx, int cy, int cz, int comp) {
    const int c[3] = {cx, cy, cz};
    return u3<S>(a.w, c, comp);
  };
  float value;
  if (a.color_axis == 0)
    value = (u(x, yp, z, 2) - u(x, ym, z, 2)) * inv_dy - (u(x, y, zp, 1) - u(x, y, zm, 1)) * inv_dz;
  else if (a.color_axis == 1)
    value = (u(x, y, zp, 0) - u(x, y, zm, 0)) * inv_dz - (u(xp, y, z, 2) - u(xm, y, z, 2)) * inv_dx;
  else
    value = (u(xp, y, z, 1) - u(xm, y, z, 1)) * inv_dx - (u(x, yp, z, 0) - u(x, ym, z, 0)) * inv_dy;
  if (x < a.margin || x >= nx - a.margin || y < a.margin || y >= ny - a.margin || z < a.margin ||
      z >= nz - a.margin)
    value = 0.f;
  a.values[i] = value;
  if (a.collect) {
    const float mag = fabsf(value);
    if (mag > 1.0e-8f) {
      const float normalized = (logf(mag) - LIVE_LOG_MIN) / (LIVE_LOG_MAX - LIVE_LOG_MIN);
      const int bin = int(fminf(fmaxf(normalized, 0.f), 0.999999f) * float(LIVE_BINS));
      atomicAdd(&a.hist[bin], 1);
    }
  }
}

// Blue-white-red map of value / vmax (clamped to [-1, 1]) to RGBA bytes, alpha the same for
// every pixel; a channel is the binary32 level truncated to an integer.
__global__ void __launch_bounds__(BLOCK) live_rgba_kernel(const float* values, uint8_t* rgba, long long n, float vmax,
                                                          float alpha) {
  const long long i = (long long)blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n) return;
  const float normalized = fminf(fmaxf(0.5f + 0.5f * values[i] / fmaxf(vmax, 1.0e-8f), 0.f), 1.f);
  float r, g, b;
  if (normalized < 0.5f) {
    const float t = normalized * 2.f;
    r = 255.f * t, g = 255.f * t, b = 255.f;
  } else {
    const float t = (normalized - 0.5f) * 2.f;
    r = 255.f, g = 255.f * (1.f - t), b = 255.f * (1.f - t);
  }
  uint8_t* px = rgba + 4 * i;
  px[0] = uint8_t(r), px[1] = uint8_t(g), px[2] = uint8_t(b);
  px[3] = uint8_t(255.f * fminf(fmaxf(alpha, 0.f), 1.f));
}

// ------------------------------------------------------------------- 2D realtime view
__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.f), 1.f); }

// u_img (nx, ny) to RGBA bytes laid out (ny, nx, 4): render_mode 0 |u| on a dark-red-yellow
// ramp, 1 vorticity blue-white-red (values >= 999, the solid mark, light grey), 2 solid
// boundary as ink on white; alpha 255.
__global__ void __launch_bounds__(BLOCK) uimg_rgba_kernel(const float* img, int nx, int ny, int mode, float vmax,
                                                          uint8_t* out) {
  const long long i = (long long)blockIdx.x * BLOCK + threadIdx.x;
  if (i >= (long long)nx * ny) return;
  const int x = int(i / ny), y = int(i - (long long)x * ny);
  const float val = img[i];
  float r, g, b;
  if (mode == 2) {
    const float c = (1.f - clamp01(val)) * 255.f;
    r = c, g = c, b = c;
  } else if (mode == 1) {
    if (val >= 999.f) {
      r = 200.f, g = 200.f, b = 200.f;
    } else {
      const float n = clamp01(0.5f + 0.5f * val / fmaxf(vmax, 1.0e-6f));
      if (n < 0.5f) {
        const float t = n * 2.f;
        r = 255.f * t, g = 255.f * t, b = 255.f;
      } else {
        const float t = (n - 0.5f) * 2.f;
        r = 255.f, g = 255.f * (1.f - t), b = 255.f * (1.f - t);
      }
    }
  } else {
    const float n = clamp01(val / fmaxf(vmax, 1.0e-6f));
    r = 255.f * n, g = 180.f * n * n, b = 60.f * (1.f - n);
  }
  uint8_t* px = out + ((long long)y * nx + x) * 4;
  px[0] = uint8_t(r), px[1] = uint8_t(g), px[2] = uint8_t(b), px[3] = 255;
}

// A force field that falls off over an ellipse: f (1 - r^2) inside, 0 outside.
__global__ void __launch_bounds__(BLOCK) local_force_kernel(float* fxo, float* fyo, int nx, int ny, float cx, float cy,
                                                            float rx, float ry, float fx, float fy) {
  const long long i = (long long)blockIdx.x * BLOCK + threadIdx.x;
  if (i >= (long long)nx * ny) return;
  const int x = int(i / ny), y = int(i - (long long)x * ny);
  const float dx = (float(x) - cx) / fmaxf(rx, 1.0e-6f);
  const float dy = (float(y) - cy) / fmaxf(ry, 1.0e-6f);
  const float w = fmaxf(0.f, 1.f - (dx * dx + dy * dy));
  fxo[i] = fx * w;
  fyo[i] = fy * w;
}

template <class S, class A, class K> int launch(K kern, const A& a, long long pixels, cudaStream_t st) {
  if (pixels == 0) return HL_OK;
  kern<<<unsigned((pixels + BLOCK - 1) / BLOCK), BLOCK, 0, st>>>(a);
  HL_LAUNCH_CHECK("field diagnostics");
  return HL_OK;
}

}  // namespace diag
}  // namespace hl

using namespace hl;

extern "C" int hl_d2q9_image(const hl_world2d* w, int kind, float param, float grid_length, const hl_solids2d* solids,
                             float thickness, float* out, hl_stream stream) {
  HL_CHECK_ARG(w != nullptr && out != nullptr && w->cur != nullptr, "image: world, cur or out is NULL");
  HL_CHECK_ARG(w->nx >= 2 && w->ny >= 2, "image: grid %d x %d too small", w->nx, w->ny);
  HL_CHECK_ARG(kind >= 0 && kind <= 3, "image: kind %d (0 |u|, 1 rgb, 2 vorticity, 3 solids)", kind);
  HL_CHECK_ARG(kind != 1 || param > 0.f, "image: max_velocity must be positive");
  HL_CHECK_ARG(kind != 3 || solids != nullptr, "image: the solid image needs solids");
  HL_CHECK_ARG(solids == nullptr || (solids->n_objects >= 0 && (solids->n_objects == 0 ||
                                     (solids->line_tf && solids->line_num && solids->position && solids->scale &&
                                      solids->max_radius && solids->max_segments > 0))),
               "image: incomplete solids");
  diag::Args2 a{};
  a.w = {w->nx, w->ny, w->cur, w->storage.u_scale > 0.f ? w->storage.u_scale : 1.f};
  a.solids = solids != nullptr && solids->n_objects > 0;
  if (solids) a.s = *solids;
  a.kind = kind;
  a.param = param;
  a.h = grid_length > 0.f ? grid_length : 1.f / float(w->nx);
  a.thickness = thickness;
  a.out = out;
  const long long pix = (long long)w->nx * w->ny;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (w->storage.dtype) {
    case HL_F32: return diag::launch<StoreF32>(diag::image2d_kernel<StoreF32>, a, pix, st);
    case HL_F16: return diag::launch<StoreF16>(diag::image2d_kernel<StoreF16>, a, pix, st);
    case HL_BF16: return diag::launch<StoreBF16>(diag::image2d_kernel<StoreBF16>, a, pix, st);
    case HL_F64: return diag::launch<StoreF64>(diag::image2d_kernel<StoreF64>, a, pix, st);
  }
  set_error("image: storage dtype %d not supported", int(w->storage.dtype));
  return HL_ERR_UNSUPPORTED;
}

extern "C" int hl_d3q27_image(const hl_world3d* w, int mode, int axis, int index, int kind, float grid_length,
                              const hl_solids3d* solids, float thickness, float* out, hl_stream stream) {
  HL_CHECK_ARG(w != nullptr && out != nullptr && w->cur != nullptr, "image: world, cur or out is NULL");
  HL_CHECK_ARG(w->nx >= 2 && w->ny >= 2 && w->nz >= 2, "image: grid too small");
  HL_CHECK_ARG(mode == 0 || mode == 1, "image: mode %d (0 slice, 1 projection)", mode);
  HL_CHECK_ARG(axis >= 0 && axis <= 2, "image: axis %d", axis);
  const int n[3] = {w->nx, w->ny, w->nz};
  HL_CHECK_ARG(mode == 1 || (index >= 0 && index < n[axis]), "image: slice %d outside 0..%d", index, n[axis] - 1);
  HL_CHECK_ARG((mode == 0 && (kind == 0 || kind == 1)) || (mode == 1 && kind >= 0 && kind <= 2),
               "image: kind %d not available for mode %d", kind, mode);
  HL_CHECK_ARG(solids == nullptr || solids->n_objects == 0 ||
                   (solids->tri_offset && solids->tris && solids->transforms && solids->scale_sizes),
               "image: incomplete solids");
  diag::Args3 a{};
  a.w = {{w->nx, w->ny, w->nz}, w->cur, w->flag, w->storage.u_scale > 0.f ? w->storage.u_scale : 1.f};
  a.solids = solids != nullptr && solids->n_objects > 0;
  if (solids) a.s = *solids;
  a.mode = mode;
  a.axis = axis;
  a.index = index;
  a.kind = kind;
  a.h = grid_length > 0.f ? grid_length : 1.f / float(w->nx);
  a.thickness = thickness;
  a.out = out;
  int pa, pb;
  diag::plane_axes(axis, pa, pb);
  const long long pix = (long long)n[pa] * n[pb];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (w->storage.dtype) {
    case HL_F32: return diag::launch<StoreF32>(diag::image3d_kernel<StoreF32>, a, pix, st);
    case HL_F16: return diag::launch<StoreF16>(diag::image3d_kernel<StoreF16>, a, pix, st);
    case HL_BF16: return diag::launch<StoreBF16>(diag::image3d_kernel<StoreBF16>, a, pix, st);
    case HL_F64: return diag::launch<StoreF64>(diag::image3d_kernel<StoreF64>, a, pix, st);
  }
  set_error("image: storage dtype %d not supported", int(w->storage.dtype));
  return HL_ERR_UNSUPPORTED;
}

extern "C" int hl_d3q27_live_slices(const hl_world3d* w, const int32_t* slice_positions, int n_slices, int plane_width,
                                    int plane_height, int stride, int slice_axis, int color_axis, int boundary_margin,
                                    int collect_histogram, float* values, int32_t* histogram, hl_stream stream) {
  HL_CHECK_ARG(w != nullptr && w->cur != nullptr && values != nullptr && slice_positions != nullptr,
               "live slices: world, cur, slice positions or values is NULL");
  HL_CHECK_ARG(w->nx >= 1 && w->ny >= 1 && w->nz >= 1, "live slices: bad grid");
  HL_CHECK_ARG(n_slices >= 1 && plane_width >= 1 && plane_height >= 1 && stride >= 1,
               "live slices: %d slices of %d x %d, stride %d", n_slices, plane_width, plane_height, stride);
  HL_CHECK_ARG((long long)n_slices * plane_width * plane_height < (1ll << 38), "live slices: too many samples");
  HL_CHECK_ARG(slice_axis >= 0 && slice_axis <= 2 && color_axis >= 0 && color_axis <= 2,
               "live slices: slice axis %d, colour axis %d", slice_axis, color_axis);
  HL_CHECK_ARG(boundary_margin >= 0, "live slices: negative margin");
  HL_CHECK_ARG(!collect_histogram || histogram != nullptr, "live slices: the histogram is NULL");
  diag::ArgsLive a{};
  a.w = {{w->nx, w->ny, w->nz}, w->cur, nullptr, w->storage.u_scale > 0.f ? w->storage.u_scale : 1.f};
  a.slice_pos = slice_positions;
  a.n_slices = n_slices;
  a.width = plane_width;
  a.height = plane_height;
  a.stride = stride;
  a.slice_axis = slice_axis;
  a.color_axis = color_axis;
  a.margin = boundary_margin;
  a.collect = collect_histogram != 0;
  a.values = values;
  a.hist = histogram;
  const long long n = (long long)n_slices * plane_width * plane_height;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (w->storage.dtype) {
    case HL_F32: return diag::launch<StoreF32>(diag::live_slices_kernel<StoreF32>, a, n, st);
    case HL_F16: return diag::launch<StoreF16>(diag::live_slices_kernel<StoreF16>, a, n, st);
    case HL_BF16: return diag::launch<StoreBF16>(diag::live_slices_kernel<StoreBF16>, a, n, st);
    case HL_F64: return diag::launch<StoreF64>(diag::live_slices_kernel<StoreF64>, a, n, st);
  }
  set_error("live slices: storage dtype %d not supported", int(w->storage.dtype));
  return HL_ERR_UNSUPPORTED;
}

extern "C" int hl_live_rgba(const float* values, long long n, float vmax, float alpha, uint8_t* rgba, hl_stream stream) {
  HL_CHECK_ARG(n >= 0 && (n == 0 || (values != nullptr && rgba != nullptr)), "live rgba: values or rgba is NULL");
  if (n == 0) return HL_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  diag::live_rgba_kernel<<<unsigned((n + diag::BLOCK - 1) / diag::BLOCK), diag::BLOCK, 0, st>>>(values, rgba, n, vmax,
                                                                                                 alpha);
  HL_LAUNCH_CHECK("live rgba");
  return HL_OK;
}

extern "C" int hl_d2q9_uimg_rgba(const float* u_img, int nx, int ny, int render_mode, float vmax, uint8_t* rgba,
                                 hl_stream stream) {
  HL_CHECK_ARG(u_img != nullptr && rgba != nullptr, "uimg rgba: image or rgba is NULL");
  HL_CHECK_ARG(nx >= 1 && ny >= 1, "uimg rgba: image %d x %d", nx, ny);
  HL_CHECK_ARG(render_mode >= 0 && render_mode <= 2, "uimg rgba: render mode %d (0, 1, 2)", render_mode);
  const long long n = (long long)nx * ny;
  diag::uimg_rgba_kernel<<<unsigned((n + diag::BLOCK - 1) / diag::BLOCK), diag::BLOCK, 0,
                           static_cast<cudaStream_t>(stream)>>>(u_img, nx, ny, render_mode, vmax, rgba);
  HL_LAUNCH_CHECK("uimg rgba");
  return HL_OK;
}

extern "C" int hl_d2q9_local_force(float* forcex, float* forcey, int nx, int ny, float cx, float cy, float rx,
                                   float ry, float fx, float fy, hl_stream stream) {
  HL_CHECK_ARG(forcex != nullptr && forcey != nullptr, "local force: force field is NULL");
  HL_CHECK_ARG(nx >= 1 && ny >= 1, "local force: grid %d x %d", nx, ny);
  const long long n = (long long)nx * ny;
  diag::local_force_kernel<<<unsigned((n + diag::BLOCK - 1) / diag::BLOCK), diag::BLOCK, 0,
                             static_cast<cudaStream_t>(stream)>>>(forcex, forcey, nx, ny, cx, cy, rx, ry, fx, fy);
  HL_LAUNCH_CHECK("local force");
  return HL_OK;
}
