// Immersed triangle-mesh solids of the D3Q27 step (sm_100a): the near-solid part of
// stream_and_collide_3d (envs/lbm3d/lbm_func_3d.py:364-604).
//
// The stream-collide kernels (d3q27.cu, d3q27_tma.cu) update every fluid cell as if no solid
// existed. This file then recomputes the narrow band, the fluid cells within
// bound_radius + 2 of a solid (387-393), with the reference's per-link logic:
//   * the link's backward ray cell -> cell - c_i is cast against every solid near the cell
//     (get_cutcell_multi_3d, 254-316) in the solid's body frame, scaled by mesh_scale_sizes;
//     the closest hit with 0 <= t <= 1 wins;
//   * a cut link takes the population rebuilt from the cell's own density and stress with the
//     wall velocity of the hit point (452-489, not clamped); the momentum exchange against
//     the cell's own opposite population and its torque about solid_position (490-511) go to
//     the solid's loads;
//   * every other link takes the neighbour's clamped population (525-526);
// followed by the regularised collision (564-604). The band overwrites the cells' post values
// written by the plain kernel; both read only the current buffer.
//
// Launch: one block row per solid (blockIdx.y), covering that solid's bounding box of the
// band; a cell near several solids is handled by the lowest-numbered one. Only cells that can
// have a cut link are recomputed: with the triangle bins a cell whose bin lists no triangle
// of any near solid has none (the rays are at most sqrt(3) long), and keeps the plain
// kernel's result, which is the reference's arithmetic on plain links up to rounding. Each
// remaining cell is computed by a whole warp, one lane per direction; its moments are warp
// shuffle sums, and its loads are warp sums per solid hit, added per block in shared memory
// and per solid in binary64 global memory.
//
// Geometry in binary32 in every storage build: the band membership, the rays in the body
// frame and the hits are computed in binary32, as the reference's mesh query computes them, so
// the binary64 build (the accuracy reference of the reduced storages) makes the same cut-link
// decisions as the binary32 one and differs from it only by the fluid arithmetic. (Grazing
// links flip between cut and uncut with the last bit of the ray geometry, which would make a
// binary64 geometry a different boundary, not a more accurate one.)
//
// Ray-triangle test: Moller & Trumbore, "Fast, minimum storage ray-triangle intersection"
// (1997), double-sided; a link is cut at the closest hit with 0 <= t <= 1 (the reference's
// mesh query returns the closest hit up to max_t = 2, lbm_func_3d.py:308, and keeps it when
// t <= 1). The triangles tested are those the solid's bin lists for the cell (all of them
// without bins), screened by the warp against the box the cell's links reach, then paired
// with the directions whose link segment box they meet; each pair is tested by one lane.
// The screens only drop triangles that cannot be hit with 0 <= t <= 1, so the hits are those
// of a test against every triangle.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "hl_common.cuh"
#include "mesh_geom.cuh"

namespace hl {
namespace d3s {

constexpr int MAX_SOLIDS = 64;
constexpr int BLOCK = 128;

// D3Q27 velocities in the reference's order (envs/lbm3d/lbm_core_3d.py:12-35).
__constant__ signed char c_cx[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
__constant__ signed char c_cy[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
__constant__ signed char c_cz[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};

template <class R> __device__ __forceinline__ R weight(int i) {
  const int n = (c_cx[i] != 0) + (c_cy[i] != 0) + (c_cz[i] != 0);
  return n == 0 ? R(8.0 / 27.0) : n == 1 ? R(2.0 / 27.0) : n == 2 ? R(1.0 / 54.0) : R(1.0 / 216.0);
}
__device__ __forceinline__ int inverse(int i) { return i == 0 ? 0 : (i & 1) ? i + 1 : i - 1; }

using namespace geo;

// Moller-Trumbore, double-sided: the ray o + t d meets the triangle v[0..8] at t with
// 0 <= t <= max_t. Binary32, every product and sum rounded on its own (the file is compiled
// without contraction), as the reference's mesh query computes it.
__device__ __forceinline__ bool mt_hit(const float* v, V3<float> o, V3<float> d, float max_t, float* t_out) {
  const float v0x = v[0], v0y = v[1], v0z = v[2];
  const float e1x = v[3] - v0x, e1y = v[4] - v0y, e1z = v[5] - v0z;
  const float e2x = v[6] - v0x, e2y = v[7] - v0y, e2z = v[8] - v0z;
  const float px = d.y * e2z - d.z * e2y, py = d.z * e2x - d.x * e2z, pz = d.x * e2y - d.y * e2x;
  const float det = e1x * px + e1y * py + e1z * pz;
  if (det == 0.f) return false;
  const float inv = 1.f / det;
  const float sx = o.x - v0x, sy = o.y - v0y, sz = o.z - v0z;
  const float u = (sx * px + sy * py + sz * pz) * inv;
  if (u < 0.f || u > 1.f) return false;
  const float qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
  const float w = (d.x * qx + d.y * qy + d.z * qz) * inv;
  if (w < 0.f || u + w > 1.f) return false;
  const float t = (e2x * qx + e2y * qy + e2z * qz) * inv;
  if (t < 0.f || t > max_t) return false;
  *t_out = t;
  return true;
}

template <class R> __device__ __forceinline__ R vlen(R x, R y, R z) { return sqrt(x * x + y * y + z * z); }
// v / scale, skipping the division for the usual unit scale (where it is exact anyway).
template <class R> __device__ __forceinline__ R unscale(R v, R scale) { return scale == R(1) ? v : v / scale; }

// mlCalEquilibrium3D_s (lbm_func_3d.py:224-251) for direction (dx, dy, dz) with weight wi.
template <class R>
__device__ __forceinline__ R feq(R rho, R ux, R uy, R uz, R Sxx, R Sxy, R Sxz, R Syy, R Syz, R Szz, R dx, R dy, R dz,
                                 R wi) {
  const R cu = dx * ux + dy * uy + dz * uz;
  const R usq = ux * ux + uy * uy + uz * uz;
  const R third = R(1.0 / 3.0);
  const R Qxx = dx * dx - third, Qyy = dy * dy - third, Qzz = dz * dz - third;
  const R f_neq = R(1.5) * (Qxx * Sxx + Qyy * Syy + Qzz * Szz + R(2) * (dx * dy * Sxy + dx * dz * Sxz + dy * dz * Syz));
  return wi * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq + f_neq);
}

struct Args {
  hl_world3d w;
  double vis_shear;
  hl_solids3d s;
  Scale sc;
  int box_side;  // cells per side of the largest band box the launch covers
};

template <class S> __device__ __forceinline__ Mom3<typename S::R> load_cell(const Args& a, long long N, long long c) {
  using R = typename S::R;
  using T = typename S::T;
  const T* cur = static_cast<const T*>(a.w.cur);
  R raw[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) raw[k] = S::to_r(cur[k * N + c]);
  return decode3<S>(raw, a.sc);
}

// Index of the first solid (with a mesh) within bound_radius + 2 of the cell, or -1.
template <class R> __device__ __forceinline__ int first_near(const hl_solids3d& s, R x, R y, R z) {
  for (int k = 0; k < s.n_objects; ++k) {
    if (s.tri_offset[k + 1] == s.tri_offset[k]) continue;
    const R d = vlen(x - R(s.position[3 * k]), y - R(s.position[3 * k + 1]), z - R(s.position[3 * k + 2]));
    if (d <= R(s.bound_radius[k]) + R(2)) return k;
  }
  return -1;
}

// Candidate triangles of solid k for rays starting at the body-frame point lo: the bin's list,
// or every triangle when the solid has no bins (or a non-unit mesh scale). Returns false when
// the bin is empty or lo lies outside the grid: no link from there can hit the solid.
template <class R>
__device__ __forceinline__ bool candidates(const hl_solids3d& s, int k, int ntri, V3<R> los, R sx, R sy, R sz,
                                           const int32_t** list, int* ncand) {
  *list = nullptr;
  *ncand = ntri;
  if (s.bin_box == nullptr || s.bin_dims[4 * k] <= 0 || sx != R(1) || sy != R(1) || sz != R(1)) return ntri > 0;
  const float* bb = s.bin_box + 4 * k;
  const int* bd = s.bin_dims + 4 * k;
  const R inv_h = R(1) / R(bb[3]);
  const R fx = (los.x - R(bb[0])) * inv_h, fy = (los.y - R(bb[1])) * inv_h, fz = (los.z - R(bb[2])) * inv_h;
  if (!(fx >= R(0) && fy >= R(0) && fz >= R(0) && fx < R(bd[0]) && fy < R(bd[1]) && fz < R(bd[2]))) return false;
  const int b = bd[3] + (int(fx) * bd[1] + int(fy)) * bd[2] + int(fz);
  *list = s.bin_tris + s.bin_start[b];
  *ncand = s.bin_start[b + 1] - s.bin_start[b];
  return *ncand > 0;
}

// The solids whose triangles a link of the cell could hit: within bound_radius + 2 and with
// candidate triangles for rays from the cell. Bit k for solid k < 32; solids from 32 on are
// not tracked and are always tested (bit 31 stands for them). Zero: no cut link possible.
template <class R> __device__ unsigned cut_mask(const hl_solids3d& s, V3<R> cell) {
  unsigned mask = 0u;
  for (int k = 0; k < s.n_objects; ++k) {
    const int ntri = s.tri_offset[k + 1] - s.tri_offset[k];
    if (ntri == 0) continue;
    if (vlen(cell.x - R(s.position[3 * k]), cell.y - R(s.position[3 * k + 1]), cell.z - R(s.position[3 * k + 2])) >
        R(s.bound_radius[k]) + R(2))
      continue;
    const Xf<R> inv = xinv(load_xf<R>(s.transforms + 7 * k));
    const V3<R> lo = xpoint(inv, cell);
    const R sx = R(s.scale_sizes[3 * k]), sy = R(s.scale_sizes[3 * k + 1]), sz = R(s.scale_sizes[3 * k + 2]);
    const int32_t* list;
    int ncand;
    if (candidates(s, k, ntri, V3<R>{unscale(lo.x, sx), unscale(lo.y, sy), unscale(lo.z, sz)}, sx, sy, sz, &list,
                   &ncand))
      mask |= k < 31 ? (1u << k) : (1u << 31);
  }
  return mask;
}
__device__ __forceinline__ bool in_mask(unsigned mask, int k) { return (mask >> (k < 31 ? k : 31)) & 1u; }

template <class R> __device__ __forceinline__ R warp_sum(R v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <class R> __device__ __forceinline__ R lane0(R v) { return __shfl_sync(0xffffffffu, v, 0); }
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// One near cell with a possible cut link, computed by a whole warp: lane i < 27 rebuilds the
// population of direction i (a wall population with its momentum exchange if the link is
// cut, the clamped neighbour population otherwise), the moments are warp sums, and the
// lanes collide and store the cell (lane k < 10 moment k).
constexpr unsigned FULL = 0xffffffffu;
constexpr unsigned NO_HIT = 0xffffffffu;

// Per-warp shared scratch of cut_cell, for the solid being tested: per direction its link's
// segment box in the body frame (min xyz, pad, max xyz, pad; empty for an inactive
// direction) and ray direction, the current chunk's triangles (slot = lane), the queue of
// (direction, slot) pairs to test exactly, and per direction the bits of its closest hit.
struct __align__(16) WarpScratch {
  float seg[27 * 8];  // read as float4: 16-byte aligned at offset 0 of a 16-byte aligned struct
  float dir[27 * 3];
  float tri[32 * 9];
  unsigned q[32 * 27];
  unsigned best[32];
};
static_assert(sizeof(WarpScratch) % 16 == 0 && alignof(WarpScratch) == 16, "float4 reads of WarpScratch::seg");

template <class S>
__device__ void cut_cell(const Args& a, double* acc, WarpScratch& ws, int x, int y, int z, unsigned mask) {
  using R = typename S::R;
  using T = typename S::T;
  const hl_solids3d& s = a.s;
  const int nx = a.w.nx, ny = a.w.ny, nz = a.w.nz;
  const long long N = (long long)nx * ny * nz;
  const long long c = ((long long)x * ny + y) * nz + z;
  const int i = threadIdx.x & 31;
  R pop = R(0);
  const int ix = i < 27 ? c_cx[i] : 0, iy = i < 27 ? c_cy[i] : 0, iz = i < 27 ? c_cz[i] : 0;
  const R dx = R(ix), dy = R(iy), dz = R(iz);
  int xn = x - ix, yn = y - iy, zn = z - iz;
  if (a.w.periodic) {
    xn = wrap(xn, nx);
    yn = wrap(yn, ny);
    zn = wrap(zn, nz);
  }
  const bool active = i < 27 && xn >= 0 && xn < nx && yn >= 0 && yn < ny && zn >= 0 && zn < nz;
  // get_cutcell_multi_3d: the closest hit in [0, 1] over the solids near the cell. Which
  // solids and which candidate triangles depend on the cell only, so the loop is uniform
  // across the warp. The warp screens the candidates 32 at a time (a lane per triangle)
  // against the box that every link of the cell stays in, the cell's body-frame point
  // +- the largest |component| of the lanes' ray directions, widened by 2e-3. That box holds
  // each lane's segment box (widened by 1e-3), so a triangle outside it fails every lane's
  // segment test: dropping it changes no hit. A survivor is tested exactly only for the
  // directions whose segment box its bounding box meets (about a tenth of them): those
  // (direction, triangle) pairs are queued and tested a pair per lane.
  float cut = -1.f;  // geometry in binary32 (see the file comment)
  int sid = -1;
  const V3<R> cell{R(x), R(y), R(z)};
  const V3<R> dir{-dx, -dy, -dz};
  const V3<float> gcell{float(x), float(y), float(z)};
  const V3<float> gdir{-float(ix), -float(iy), -float(iz)};
  for (int k = 0; k < s.n_objects; ++k) {
    if (!in_mask(mask, k)) continue;  // no candidate triangles for this cell's rays
    const int t0 = s.tri_offset[k], ntri = s.tri_offset[k + 1] - t0;
    if (ntri == 0) continue;
    if (vlen(gcell.x - s.position[3 * k], gcell.y - s.position[3 * k + 1], gcell.z - s.position[3 * k + 2]) >
        s.bound_radius[k] + 2.f)
      continue;
    const Xf<float> inv = xinv(load_xf<float>(s.transforms + 7 * k));
    const V3<float> lo = xpoint(inv, gcell);
    const V3<float> ld = qrot(inv.qx, inv.qy, inv.qz, inv.qw, gdir);
    const float sx = s.scale_sizes[3 * k], sy = s.scale_sizes[3 * k + 1], sz = s.scale_sizes[3 * k + 2];
    const V3<float> los{unscale(lo.x, sx), unscale(lo.y, sy), unscale(lo.z, sz)};
    const V3<float> lds{unscale(ld.x, sx), unscale(ld.y, sy), unscale(ld.z, sz)};
    const int32_t* list;
    int ncand;
    if (!candidates(s, k, ntri, los, sx, sy, sz, &list, &ncand)) continue;
    const float rx = warp_max(i < 27 ? float(fabs(lds.x)) : 0.f) + 2e-3f;
    const float ry = warp_max(i < 27 ? float(fabs(lds.y)) : 0.f) + 2e-3f;
    const float rz = warp_max(i < 27 ? float(fabs(lds.z)) : 0.f) + 2e-3f;
    const float bx0 = float(los.x) - rx, bx1 = float(los.x) + rx;
    const float by0 = float(los.y) - ry, by1 = float(los.y) + ry;
    const float bz0 = float(los.z) - rz, bz1 = float(los.z) + rz;
    const float* tk = s.tris + 9ll * t0;
    // this solid's segment boxes and ray directions, one direction per lane
    const float eps = 1e-3f, inf = __int_as_float(0x7f800000);
    if (i < 27) {
      float* sb = ws.seg + 8 * i;
      sb[0] = active ? fminf(los.x, los.x + lds.x) - eps : inf;
      sb[1] = active ? fminf(los.y, los.y + lds.y) - eps : inf;
      sb[2] = active ? fminf(los.z, los.z + lds.z) - eps : inf;
      sb[4] = active ? fmaxf(los.x, los.x + lds.x) + eps : -inf;
      sb[5] = active ? fmaxf(los.y, los.y + lds.y) + eps : -inf;
      sb[6] = active ? fmaxf(los.z, los.z + lds.z) + eps : -inf;
      ws.dir[3 * i] = lds.x, ws.dir[3 * i + 1] = lds.y, ws.dir[3 * i + 2] = lds.z;
    }
    ws.best[i] = NO_HIT;
    __syncwarp();
    // software pipeline over the chunks: the vertices of chunk q + 1 and the list entries of
    // chunk q + 2 are loaded while chunk q is screened
    auto tri_of = [&](int q) { return list ? __ldg(list + q) : q; };
    float vn[9];
    if (i < ncand) {
      const int t = tri_of(i);
#pragma unroll
      for (int j = 0; j < 9; ++j) vn[j] = __ldg(tk + 9 * t + j);
    }
    int tri_n = 32 + i < ncand ? tri_of(32 + i) : 0;
    for (int q0 = 0; q0 < ncand; q0 += 32) {
      float v[9];
#pragma unroll
      for (int j = 0; j < 9; ++j) v[j] = vn[j];
      const bool live = q0 + i < ncand;
      if (q0 + 32 + i < ncand) {
#pragma unroll
        for (int j = 0; j < 9; ++j) vn[j] = __ldg(tk + 9 * tri_n + j);
      }
      if (q0 + 64 + i < ncand) tri_n = tri_of(q0 + 64 + i);
      const float mnx = fminf(fminf(v[0], v[3]), v[6]), mxx = fmaxf(fmaxf(v[0], v[3]), v[6]);
      const float mny = fminf(fminf(v[1], v[4]), v[7]), mxy = fmaxf(fmaxf(v[1], v[4]), v[7]);
      const float mnz = fminf(fminf(v[2], v[5]), v[8]), mxz = fmaxf(fmaxf(v[2], v[5]), v[8]);
      const bool keep = live && !(mxx < bx0 || mnx > bx1 || mxy < by0 || mny > by1 || mxz < bz0 || mnz > bz1);
      if (__ballot_sync(FULL, keep) == 0u) continue;  // uniform
      // the directions whose segment box this lane's triangle meets (27 independent tests)
      unsigned dm = 0u;
      if (keep) {
#pragma unroll 9
        for (int d = 0; d < 27; ++d) {
          const float4 l4 = *reinterpret_cast<const float4*>(ws.seg + 8 * d);
          const float4 h4 = *reinterpret_cast<const float4*>(ws.seg + 8 * d + 4);
          if (!(mxx < l4.x || mnx > h4.x || mxy < l4.y || mny > h4.y || mxz < l4.z || mnz > h4.z)) dm |= 1u << d;
        }
        if (dm) {
#pragma unroll
          for (int j = 0; j < 9; ++j) ws.tri[9 * i + j] = v[j];
        }
      }
      // queue the (direction, slot) pairs: exclusive scan of the lanes' counts
      const int cnt = __popc(dm);
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, o);
        if (i >= o) incl += t;
      }
      const int total = __shfl_sync(FULL, incl, 31);
      int off = incl - cnt;
      for (unsigned b = dm; b; b &= b - 1u) ws.q[off++] = (unsigned(__ffs(b) - 1) << 5) | unsigned(i);
      __syncwarp();
      // the exact tests, a pair per lane; a hit with 0 <= t <= 1 lowers best[direction]
      for (int p0 = 0; p0 < total; p0 += 32) {
        if (p0 + i < total) {
          const unsigned e = ws.q[p0 + i];
          const int d = int(e >> 5);
          const V3<float> dd{ws.dir[3 * d], ws.dir[3 * d + 1], ws.dir[3 * d + 2]};
          float t;
          if (mt_hit(ws.tri + 9 * (e & 31u), los, dd, 1.f, &t))
            atomicMin(&ws.best[d], t == 0.f ? 0u : __float_as_uint(t));
        }
      }
      __syncwarp();
    }
    __syncwarp();
    // this solid's closest hit per direction; ties keep the lower solid
    const unsigned bt = ws.best[i];
    if (bt != NO_HIT) {
      const float t = __uint_as_float(bt);
      if (cut < 0.f || t < cut) {
        cut = t;
        sid = k;
      }
    }
  }
  // no cut link: the cell keeps the plain kernel's result (the same arithmetic on plain links)
  if (__ballot_sync(FULL, sid >= 0) == 0u) return;
  // the cell's own moments, loaded after the ray tests (they are not needed there and would
  // hold registers through them); an uncut lane's neighbour load below overlaps this one
  const Mom3<R> mc = load_cell<S>(a, N, c);
  double lf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // this link's momentum exchange and torque
  if (active) {
    const R wi = weight<R>(i);
    {
      if (sid >= 0) {
        const Xf<R> tc = load_xf<R>(s.transforms + 7 * sid);
        const Xf<R> tl = load_xf<R>(s.transforms_last + 7 * sid);
        const R rc = R(cut);
        const V3<R> hit{cell.x + dir.x * rc, cell.y + dir.y * rc, cell.z + dir.z * rc};
        const V3<R> hl = xpoint(xinv(tc), hit);
        V3<R> up;
        const R spx = R(s.position[3 * sid]), spy = R(s.position[3 * sid + 1]), spz = R(s.position[3 * sid + 2]);
        if (s.initialized[sid] > 0) {
          const V3<R> pc = xpoint(tc, hl), pl = xpoint(tl, hl);
          up = {pc.x - pl.x, pc.y - pl.y, pc.z - pl.z};
        } else {
          const R ax = R(s.angle_v[3 * sid]), ay = R(s.angle_v[3 * sid + 1]), az = R(s.angle_v[3 * sid + 2]);
          const R rx = hit.x - spx, ry = hit.y - spy, rz = hit.z - spz;
          up = {R(s.linear_v[3 * sid]) + (ay * rz - az * ry), R(s.linear_v[3 * sid + 1]) + (az * rx - ax * rz),
                R(s.linear_v[3 * sid + 2]) + (ax * ry - ay * rx)};
        }
        const R rx = hit.x - spx, ry = hit.y - spy, rz = hit.z - spz;
        const R Sxx_s = up.x * up.x + mc.sxx - mc.ux * mc.ux;
        const R Sxy_s = up.x * up.y + mc.sxy - mc.ux * mc.uy;
        const R Sxz_s = up.x * up.z + mc.sxz - mc.ux * mc.uz;
        const R Syy_s = up.y * up.y + mc.syy - mc.uy * mc.uy;
        const R Syz_s = up.y * up.z + mc.syz - mc.uy * mc.uz;
        const R Szz_s = up.z * up.z + mc.szz - mc.uz * mc.uz;
        pop = feq<R>(mc.rho, up.x, up.y, up.z, Sxx_s, Sxy_s, Sxz_s, Syy_s, Syz_s, Szz_s, dx, dy, dz, wi);
        const int ii = inverse(i);
        const R ex = R(c_cx[ii]), ey = R(c_cy[ii]), ez = R(c_cz[ii]);
        const R cur_f = feq<R>(mc.rho, mc.ux, mc.uy, mc.uz, mc.sxx, mc.sxy, mc.sxz, mc.syy, mc.syz, mc.szz, ex, ey, ez,
                               weight<R>(ii));
        const R fx = cur_f * (ex - up.x) - pop * (dx - up.x);
        const R fy = cur_f * (ey - up.y) - pop * (dy - up.y);
        const R fz = cur_f * (ez - up.z) - pop * (dz - up.z);
        lf[0] = double(fx);
        lf[1] = double(fy);
        lf[2] = double(fz);
        lf[3] = double(ry * fz - rz * fy);
        lf[4] = double(rz * fx - rx * fz);
        lf[5] = double(rx * fy - ry * fx);
      } else {
        const Mom3<R> m = load_cell<S>(a, N, ((long long)xn * ny + yn) * nz + zn);
        pop = feq<R>(m.rho, m.ux, m.uy, m.uz, m.sxx, m.sxy, m.sxz, m.syy, m.syz, m.szz, dx, dy, dz, wi);
        if (pop < R(0)) pop = R(0);
      }
    }
  }
  // the loads of the cell's cut links, summed over the warp per solid hit (lanes of other
  // solids add zero), then one shared-memory add per component
  int pend = sid;  // >= 0 only on active lanes with a cut link
  for (unsigned left = __ballot_sync(0xffffffffu, pend >= 0); left; left = __ballot_sync(0xffffffffu, pend >= 0)) {
    const int target = __shfl_sync(0xffffffffu, pend, __ffs(left) - 1);
    const bool mine = pend == target;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const double v = warp_sum(mine ? lf[j] : 0.0);
      if (i == 0) atomicAdd(&acc[6 * target + j], v);
    }
    if (mine) pend = -1;
  }
  // moments (lbm_func_3d.py:528-562) as warp sums: rho, the signed first moments and the
  // second moments (c_a^2 = |c_a|)
  // (the butterfly sums can differ between lanes in the last bit; every lane takes lane 0's)
  const R rho = lane0(warp_sum(pop));
  const R jx = lane0(warp_sum(R(ix) * pop)), jy = lane0(warp_sum(R(iy) * pop)), jz = lane0(warp_sum(R(iz) * pop));
  const R pxx = lane0(warp_sum(R(ix * ix) * pop)), pyy = lane0(warp_sum(R(iy * iy) * pop));
  const R pzz = lane0(warp_sum(R(iz * iz) * pop));
  R pixy = lane0(warp_sum(R(ix * iy) * pop)), pixz = lane0(warp_sum(R(ix * iz) * pop));
  R piyz = lane0(warp_sum(R(iy * iz) * pop));
  // regularised collision (564-604), the same in every lane; lane k < 10 encodes and stores
  // moment k
  const R Fx = a.w.force ? R(a.w.force[c]) : R(0);
  const R Fy = a.w.force ? R(a.w.force[N + c]) : R(0);
  const R Fz = a.w.force ? R(a.w.force[2 * N + c]) : R(0);
  const R invRho = R(1) / rho;
  const R ux = (jx + R(0.5) * Fx) * invRho;
  const R uy = (jy + R(0.5) * Fy) * invRho;
  const R uz = (jz + R(0.5) * Fz) * invRho;
  const R omega = R(1) / (R(a.vis_shear) * R(3) + R(0.5));
  const R pixx_part = (R(2) * pxx - pyy - pzz) / R(3);
  const R piyy_part = (R(2) * pyy - pxx - pzz) / R(3);
  const R pizz_part = (R(2) * pzz - pxx - pyy) / R(3);
  const R RU2 = rho * ux * ux, RV2 = rho * uy * uy, RW2 = rho * uz * uz;
  const R RUVW2 = (RU2 + RV2 + RW2) / R(3);
  const R o1 = R(1) - omega;
  const R qxx = rho / R(3) + pixx_part * o1 + RUVW2 + (R(2) * RU2 * omega) / R(3) - (RV2 * omega) / R(3) -
                (RW2 * omega) / R(3) + Fx * ux;
  const R qyy = rho / R(3) + piyy_part * o1 + RUVW2 - (RU2 * omega) / R(3) + (R(2) * RV2 * omega) / R(3) -
                (RW2 * omega) / R(3) + Fy * uy;
  const R qzz = rho / R(3) + pizz_part * o1 + RUVW2 - (RU2 * omega) / R(3) - (RV2 * omega) / R(3) +
                (R(2) * RW2 * omega) / R(3) + Fz * uz;
  pixy = pixy - pixy * omega + ux * uy * rho * omega + (Fy * ux + Fx * uy) / R(2);
  pixz = pixz - pixz * omega + ux * uz * rho * omega + (Fz * ux + Fx * uz) / R(2);
  piyz = piyz - piyz * omega + uy * uz * rho * omega + (Fz * uy + Fy * uz) / R(2);
  const R cs2 = R(1.0 / 3.0);
  Mom3<R> m;
  m.rho = rho;
  m.drho = rho - R(1);
  m.ux = ux + Fx * invRho / R(2);
  m.uy = uy + Fy * invRho / R(2);
  m.uz = uz + Fz * invRho / R(2);
  m.sxx = qxx * invRho - cs2;
  m.syy = qyy * invRho - cs2;
  m.szz = qzz * invRho - cs2;
  m.sxy = pixy * invRho;
  m.sxz = pixz * invRho;
  m.syz = piyz * invRho;
  R raw[10];
  encode3<S>(m, a.sc, raw);
  R mine = raw[0];
#pragma unroll
  for (int k = 1; k < 10; ++k)
    if (i == k) mine = raw[k];
  if (i < 10) static_cast<T*>(a.w.post)[i * N + c] = S::from_r(mine, unsigned(i * N + c));
}

template <class S> __global__ void __launch_bounds__(BLOCK) band_kernel(const __grid_constant__ Args a) {
  using R = typename S::R;
  __shared__ double acc[MAX_SOLIDS * 6];
  const hl_solids3d& s = a.s;
  const int n = s.n_objects;
  for (int k = threadIdx.x; k < 6 * n; k += blockDim.x) acc[k] = 0.0;
  __syncthreads();

  const int k0 = blockIdx.y;
  const int nx = a.w.nx, ny = a.w.ny, nz = a.w.nz;
  // bounding box of solid k0's band, clipped to the grid
  const float px = s.position[3 * k0], py = s.position[3 * k0 + 1], pz = s.position[3 * k0 + 2];
  const float r = s.bound_radius[k0] + 2.f;
  const int side = a.box_side;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  // 1. each lane classifies its cell: fluid, in solid k0's band (and in no lower solid's), and
  //    with candidate triangles for its rays
  int x = 0, y = 0, z = 0;
  unsigned solids = 0u;
  bool flagged = false;
  if (s.tri_offset[k0 + 1] > s.tri_offset[k0] && isfinite(px) && isfinite(py) && isfinite(pz) && isfinite(r) &&
      idx < (long long)side * side * side) {
    x = int(floorf(px - r)) + int(idx / ((long long)side * side));
    y = int(floorf(py - r)) + int((idx / side) % side);
    z = int(floorf(pz - r)) + int(idx % side);
    const bool inside = x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz;
    const long long c = ((long long)x * ny + y) * nz + z;
    const bool fluid = inside && (a.w.flag == nullptr || a.w.flag[c] == ML_FLUID) &&
                       (a.w.flag != nullptr || a.w.periodic || (x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < nz - 1));
    if (fluid && first_near<float>(s, float(x), float(y), float(z)) == k0)
      solids = cut_mask<float>(s, V3<float>{float(x), float(y), float(z)});
    flagged = solids != 0u;
  }
  // 2. the warp computes its flagged cells one after another, a lane per direction
  __shared__ WarpScratch scratch[BLOCK / 32];
  unsigned mask = __ballot_sync(0xffffffffu, flagged);
  const bool any = mask != 0;
  while (mask) {
    const int src = __ffs(mask) - 1;
    mask &= mask - 1;
    const int cx = __shfl_sync(0xffffffffu, x, src), cy = __shfl_sync(0xffffffffu, y, src),
              cz = __shfl_sync(0xffffffffu, z, src);
    const unsigned cm = __shfl_sync(0xffffffffu, solids, src);
    cut_cell<S>(a, acc, scratch[threadIdx.x >> 5], cx, cy, cz, cm);
    __syncwarp();
  }
  if (!__syncthreads_or(any)) return;
  for (int k = threadIdx.x; k < 6 * n; k += blockDim.x)
    if (acc[k] != 0.0) atomicAdd(&s.loads64[k], acc[k]);
}

// Work-list form. The int32 scratch holds a header of WORK_HEAD ints (listed cells, finished
// process blocks, next cell to take, unused), zeroed before each call, then (cell, solid
// mask) pairs. classify_kernel: one thread per box cell appends the cells that can have a cut
// link (one atomic per warp); process_kernel: a fixed grid of warps takes the listed cells
// one at a time from a shared counter, a cell per warp as in band_kernel, so that a warp held
// by an expensive cell (near a joint, hundreds of candidate triangles) takes no others.
constexpr int WORK_HEAD = 4;
// Cell idx of solid k0's band box: its index c in the world and the mask of the solids whose
// triangles a link of it could reach (0: not a candidate cut cell, or not this solid's to do).
__device__ __forceinline__ unsigned classify_cell(const Args& a, int k0, long long idx, int& c) {
  const hl_solids3d& s = a.s;
  const int nx = a.w.nx, ny = a.w.ny, nz = a.w.nz;
  const float px = s.position[3 * k0], py = s.position[3 * k0 + 1], pz = s.position[3 * k0 + 2];
  const float r = s.bound_radius[k0] + 2.f;
  const int side = a.box_side;
  c = 0;
  if (!(s.tri_offset[k0 + 1] > s.tri_offset[k0] && isfinite(px) && isfinite(py) && isfinite(pz) && isfinite(r) &&
        idx < (long long)side * side * side))
    return 0u;
  const int x = int(floorf(px - r)) + int(idx / ((long long)side * side));
  const int y = int(floorf(py - r)) + int((idx / side) % side);
  const int z = int(floorf(pz - r)) + int(idx % side);
  const bool inside = x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz;
  c = (x * ny + y) * nz + z;
  const bool fluid = inside && (a.w.flag == nullptr || a.w.flag[c] == ML_FLUID) &&
                     (a.w.flag != nullptr || a.w.periodic || (x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < nz - 1));
  if (fluid && first_near<float>(s, float(x), float(y), float(z)) == k0)
    return cut_mask<float>(s, V3<float>{float(x), float(y), float(z)});
  return 0u;
}

template <class S> __global__ void __launch_bounds__(BLOCK) classify_kernel(const __grid_constant__ Args a) {
  const hl_solids3d& s = a.s;
  int c;
  const unsigned solids = classify_cell(a, blockIdx.y, (long long)blockIdx.x * blockDim.x + threadIdx.x, c);
  const bool flagged = solids != 0u;
  const unsigned mask = __ballot_sync(0xffffffffu, flagged);
  if (mask == 0) return;
  const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(s.work, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (flagged) {
    const int slot = base + __popc(mask & ((1u << lane) - 1));
    s.work[WORK_HEAD + 2 * slot] = c;
    s.work[WORK_HEAD + 1 + 2 * slot] = int(solids);
  }
}

// solid_force / solid_torque <- binary32 copies of the binary64 sums of solid k (loaded
// through L2: other blocks wrote them).
__device__ __forceinline__ void loads_out(const hl_solids3d& s, int k) {
  for (int j = 0; j < 3; ++j) {
    if (s.force) s.force[3 * k + j] = float(__ldcg(&s.loads64[6 * k + j]));
    if (s.torque) s.torque[3 * k + j] = float(__ldcg(&s.loads64[6 * k + 3 + j]));
  }
}

// The block that finishes last (work[1] counts finished blocks) writes the binary32 loads.
// Blocks of 16 warps (one per SM at 104 registers), each warp's scratch in dynamic shared
// memory: a warp spends most of a cell waiting on dependent loads, so more warps per SM hide
// more of it than the same warps spread over more SMs.
constexpr int PBLOCK = 512;
constexpr int PBLOCK_SMEM = int(sizeof(WarpScratch)) * (PBLOCK / 32);
template <class S> __global__ void __launch_bounds__(PBLOCK) process_kernel(const __grid_constant__ Args a) {
  __shared__ double acc[MAX_SOLIDS * 6];
  __shared__ bool last;
  extern __shared__ __align__(16) unsigned char process_smem[];
  WarpScratch* scratch = reinterpret_cast<WarpScratch*>(process_smem);  // [PBLOCK / 32]
  const hl_solids3d& s = a.s;
  const int n = s.n_objects;
  for (int k = threadIdx.x; k < 6 * n; k += blockDim.x) acc[k] = 0.0;
  __syncthreads();
  const int count = s.work[0];
  const int ny = a.w.ny, nz = a.w.nz;
  bool any = false;
  for (;;) {
    int j = 0;
    if ((threadIdx.x & 31) == 0) j = atomicAdd(s.work + 2, 1);
    j = __shfl_sync(FULL, j, 0);
    if (j >= count) break;
    const int c = s.work[WORK_HEAD + 2 * j];
    const unsigned cm = unsigned(s.work[WORK_HEAD + 1 + 2 * j]);
    any = true;
    cut_cell<S>(a, acc, scratch[threadIdx.x >> 5], c / (ny * nz), (c / nz) % ny, c % nz, cm);
    __syncwarp();
  }
  if (__syncthreads_or(any)) {
    for (int k = threadIdx.x; k < 6 * n; k += blockDim.x)
      if (acc[k] != 0.0) atomicAdd(&s.loads64[k], acc[k]);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(reinterpret_cast<unsigned*>(s.work + 1), 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = threadIdx.x; k < n; k += blockDim.x) loads_out(s, k);
}

__global__ void loads_out_kernel(hl_solids3d s) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < s.n_objects) loads_out(s, k);
}

// ------------------------------------------------------------------ batched domains
// The cut links of many domains in one classify and one process launch. Descriptor layout
// in device memory: a BatchHead, the per-domain Args for parity 0 then for parity 1 (parity p
// reads buffer p), then the classify launch's block rows, one (domain, solid) pair each. The
// work list holds LB_HEAD counters (entries, finished process blocks, next entry, unused) and
// (domain, cell, solid mask) entries.
constexpr int LB_HEAD = 4;
struct BatchHead {
  int n_domains, n_rows, max_box, pad;
};
__host__ __device__ constexpr size_t align64(size_t b) { return (b + 63) / 64 * 64; }
constexpr size_t LB_ARGS_OFF = align64(sizeof(BatchHead));
__host__ __device__ inline size_t lb_rows_off(int n) { return LB_ARGS_OFF + align64(2 * size_t(n) * sizeof(Args)); }

template <class S>
__global__ void __launch_bounds__(BLOCK) classify_batch_kernel(const unsigned char* __restrict__ desc, int parity,
                                                               int32_t* work) {
  const BatchHead& h = *reinterpret_cast<const BatchHead*>(desc);
  const Args* args = reinterpret_cast<const Args*>(desc + LB_ARGS_OFF) + size_t(parity) * h.n_domains;
  const int2 row = reinterpret_cast<const int2*>(desc + lb_rows_off(h.n_domains))[blockIdx.y];
  const Args& a = args[row.x];
  if (blockIdx.x == 0 && threadIdx.x < 6) a.s.loads64[6 * row.y + threadIdx.x] = 0.0;  // once per solid
  int c;
  const unsigned solids = classify_cell(a, row.y, (long long)blockIdx.x * blockDim.x + threadIdx.x, c);
  const bool flagged = solids != 0u;
  const unsigned mask = __ballot_sync(FULL, flagged);
  if (mask == 0) return;
  const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(work, __popc(mask));
  base = __shfl_sync(FULL, base, leader);
  if (flagged) {
    int32_t* e = work + LB_HEAD + 3 * (base + __popc(mask & ((1u << lane) - 1)));
    e[0] = row.x, e[1] = c, e[2] = int(solids);
  }
}

// Warps take the listed cells in turn; a cell's loads go straight to its domain's binary64
// sums (zeroed by the classify launch); the last block writes every domain's binary32 loads.
template <class S>
__global__ void __launch_bounds__(BLOCK) process_batch_kernel(const unsigned char* __restrict__ desc, int parity,
                                                              int32_t* work) {
  __shared__ WarpScratch scratch[BLOCK / 32];
  __shared__ bool last;
  const BatchHead& h = *reinterpret_cast<const BatchHead*>(desc);
  const Args* args = reinterpret_cast<const Args*>(desc + LB_ARGS_OFF) + size_t(parity) * h.n_domains;
  const int count = work[0];
  for (;;) {
    int j = 0;
    if ((threadIdx.x & 31) == 0) j = atomicAdd(work + 2, 1);
    j = __shfl_sync(FULL, j, 0);
    if (j >= count) break;
    const int32_t* e = work + LB_HEAD + 3 * j;
    const Args& a = args[e[0]];
    const int c = e[1], ny = a.w.ny, nz = a.w.nz;
    cut_cell<S>(a, a.s.loads64, scratch[threadIdx.x >> 5], c / (ny * nz), (c / nz) % ny, c % nz, unsigned(e[2]));
    __syncwarp();
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(reinterpret_cast<unsigned*>(work + 1), 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int d = 0; d < h.n_domains; ++d)
    for (int k = threadIdx.x; k < args[d].s.n_objects; k += blockDim.x) loads_out(args[d].s, k);
}

// prepared descriptors: address -> (domains, rows, largest band box side, work ints, dtype)
struct BatchInfo {
  int n_domains, n_rows, max_box;
  size_t work_ints;
  hl_dtype dtype;
};
std::mutex g_lb_mu;
std::map<const void*, BatchInfo> g_lb;

template <class S> int launch_batch(const void* desc, const BatchInfo& b, int parity, int32_t* work, cudaStream_t st);

int num_sms_local() { return device_sms(); }

int box_side_of(float max_bound_radius) { return int(ceilf(2.f * (max_bound_radius + 2.f))) + 2; }

template <class S> int launch(const hl_world3d* w, double vis, const hl_solids3d* s, cudaStream_t st) {
  Args a;
  a.w = *w;
  a.vis_shear = vis;
  a.s = *s;
  a.sc = make_scale(w->storage);
  // cells within r = max_bound_radius + 2 of a point lie in floor(p - r) .. floor(p - r) + side - 1
  a.box_side = box_side_of(s->max_bound_radius);
  const long long cells = (long long)a.box_side * a.box_side * a.box_side;
  const dim3 grid(unsigned((cells + BLOCK - 1) / BLOCK), unsigned(s->n_objects));
  if (s->work != nullptr) {
    cudaError_t e = cudaMemsetAsync(s->work, 0, WORK_HEAD * sizeof(int32_t), st);
    if (e != cudaSuccess) return cuda_status(e, "d3q27 solid links: zero work count");
    classify_kernel<S><<<grid, BLOCK, 0, st>>>(a);
    HL_LAUNCH_CHECK("d3q27 solid links (classify)");
    // one 16-warp block per SM unless set; the last block to finish writes the binary32 loads
    const int blocks = g_tune_d3_link_blocks > 0 ? g_tune_d3_link_blocks : num_sms_local();
    const int ar = set_smem_attr(reinterpret_cast<const void*>(&process_kernel<S>), PBLOCK_SMEM,
                                 "d3q27 solid links (cut cells)");
    if (ar != HL_OK) return ar;
    process_kernel<S><<<unsigned(blocks), PBLOCK, size_t(PBLOCK_SMEM), st>>>(a);
    HL_LAUNCH_CHECK("d3q27 solid links (cut cells)");
  } else {
    band_kernel<S><<<grid, BLOCK, 0, st>>>(a);
    HL_LAUNCH_CHECK("d3q27 solid links (band)");
    loads_out_kernel<<<(s->n_objects + 63) / 64, 64, 0, st>>>(*s);
    HL_LAUNCH_CHECK("d3q27 solid links (loads)");
  }
  return HL_OK;
}

}  // namespace d3s
}  // namespace hl

using namespace hl;

extern "C" int hl_d3q27_solid_links(const hl_world3d* w, double vis_shear, const hl_solids3d* s, hl_stream stream) {
  HL_CHECK_ARG(w != nullptr && s != nullptr, "d3q27 solid links: world or solids is NULL");
  HL_CHECK_ARG(w->nx >= 1 && w->ny >= 1 && w->nz >= 1, "d3q27 solid links: bad dims %d x %d x %d", w->nx, w->ny, w->nz);
  HL_CHECK_ARG(w->cur != nullptr && w->post != nullptr && w->cur != w->post, "d3q27 solid links: cur/post must be distinct");
  HL_CHECK_ARG(vis_shear > 0.0, "d3q27 solid links: viscosity must be positive");
  HL_CHECK_ARG(s->n_objects >= 0 && s->n_objects <= d3s::MAX_SOLIDS, "d3q27 solid links: %d solids (at most %d)",
               s->n_objects, d3s::MAX_SOLIDS);
  if (s->n_objects == 0) return HL_OK;
  HL_CHECK_ARG(s->tri_offset && s->tris && s->transforms && s->transforms_last && s->initialized && s->scale_sizes &&
                   s->position && s->bound_radius && s->linear_v && s->angle_v && s->loads64,
               "d3q27 solid links: a solid field is NULL");
  HL_CHECK_ARG(std::isfinite(s->max_bound_radius) && s->max_bound_radius >= 0.f && s->max_bound_radius < 512.f,
               "d3q27 solid links: max_bound_radius %g out of range", double(s->max_bound_radius));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(s->loads64, 0, sizeof(double) * 6 * size_t(s->n_objects), st);
  if (e != cudaSuccess) return cuda_status(e, "d3q27 solid links: zero loads");
  switch (w->storage.dtype) {
    case HL_F32: return d3s::launch<StoreF32>(w, vis_shear, s, st);
    case HL_F16: return d3s::launch<StoreF16>(w, vis_shear, s, st);
    case HL_BF16: return d3s::launch<StoreBF16>(w, vis_shear, s, st);
    case HL_F64: return d3s::launch<StoreF64>(w, vis_shear, s, st);
  }
  set_error("d3q27 solid links: storage dtype %d not supported", int(w->storage.dtype));
  return HL_ERR_UNSUPPORTED;
}

extern "C" size_t hl_d3q27_solid_links_work_ints(int n_objects, float max_bound_radius) {
  if (n_objects <= 0 || !(max_bound_radius >= 0.f) || max_bound_radius >= 512.f) return 0;
  const size_t side = size_t(d3s::box_side_of(max_bound_radius));
  // header (listed cells, finished blocks, next cell, unused), then (cell, solid mask) pairs
  return d3s::WORK_HEAD + 2 * size_t(n_objects) * side * side * side;
}

namespace hl {
namespace d3s {
template <class S> int launch_batch(const void* desc, const BatchInfo& b, int parity, int32_t* work, cudaStream_t st) {
  const auto* d = static_cast<const unsigned char*>(desc);
  const long long cells = (long long)b.max_box * b.max_box * b.max_box;
  classify_batch_kernel<S><<<dim3(unsigned((cells + BLOCK - 1) / BLOCK), unsigned(b.n_rows)), BLOCK, 0, st>>>(d, parity,
                                                                                                          work);
  HL_LAUNCH_CHECK("d3q27 solid links batch (classify)");
  const int blocks = g_tune_d3_link_blocks > 0 ? g_tune_d3_link_blocks : 4 * num_sms_local();
  process_batch_kernel<S><<<unsigned(blocks), BLOCK, 0, st>>>(d, parity, work);
  HL_LAUNCH_CHECK("d3q27 solid links batch (cut cells)");
  return HL_OK;
}
}  // namespace d3s
}  // namespace hl

extern "C" size_t hl_d3q27_links_batch_bytes(int n_domains, int n_solids_total) {
  if (n_domains <= 0 || n_solids_total < 0) return 0;
  return d3s::lb_rows_off(n_domains) + size_t(n_solids_total) * sizeof(int2);
}

extern "C" int hl_d3q27_links_batch_prepare(const hl_world3d* worlds, const hl_solids3d* solids, int n_domains,
                                            double vis_shear, void* desc, size_t desc_bytes, size_t* work_ints,
                                            hl_stream stream) {
  HL_CHECK_ARG(worlds != nullptr && solids != nullptr && work_ints != nullptr, "links batch: NULL argument");
  HL_CHECK_ARG(n_domains >= 1 && n_domains <= 4096, "links batch: %d domains (1 .. 4096)", n_domains);
  HL_CHECK_ARG(vis_shear > 0.0, "links batch: viscosity must be positive");
  HL_CHECK_ARG(desc != nullptr && (reinterpret_cast<uintptr_t>(desc) & 63) == 0,
               "links batch: descriptor buffer NULL or not 64-byte aligned");
  std::vector<d3s::Args> args(2 * size_t(n_domains));
  std::vector<int2> rows;
  size_t capacity = 0;
  int max_box = 0;
  for (int k = 0; k < n_domains; ++k) {
    const hl_world3d& w = worlds[k];
    const hl_solids3d& s = solids[k];
    HL_CHECK_ARG(w.nx >= 1 && w.ny >= 1 && w.nz >= 1 && w.cur && w.post && w.cur != w.post,
                 "links batch: domain %d world", k);
    HL_CHECK_ARG(w.storage.dtype == worlds[0].storage.dtype, "links batch: domain %d has another storage type", k);
    HL_CHECK_ARG(s.n_objects >= 1 && s.n_objects <= d3s::MAX_SOLIDS, "links batch: domain %d has %d solids", k,
                 s.n_objects);
    HL_CHECK_ARG(s.tri_offset && s.tris && s.transforms && s.transforms_last && s.initialized && s.scale_sizes &&
                     s.position && s.bound_radius && s.linear_v && s.angle_v && s.loads64,
                 "links batch: domain %d: a solid field is NULL", k);
    HL_CHECK_ARG(std::isfinite(s.max_bound_radius) && s.max_bound_radius >= 0.f && s.max_bound_radius < 512.f,
                 "links batch: domain %d: max_bound_radius out of range", k);
    for (int p = 0; p < 2; ++p) {
      d3s::Args& a = args[size_t(p) * n_domains + k];
      a.w = w;
      if (p == 1) {
        a.w.cur = w.post;
        a.w.post = const_cast<void*>(w.cur);
      }
      a.vis_shear = vis_shear;
      a.s = s;
      a.s.work = nullptr;
      a.sc = make_scale(w.storage);
      a.box_side = d3s::box_side_of(s.max_bound_radius);
    }
    const int box = d3s::box_side_of(s.max_bound_radius);
    max_box = std::max(max_box, box);
    capacity += size_t(s.n_objects) * box * box * box;
    for (int j = 0; j < s.n_objects; ++j) rows.push_back(make_int2(k, j));
  }
  HL_CHECK_ARG(rows.size() <= 65535, "links batch: %zu solids in all (at most 65535)", rows.size());
  HL_CHECK_ARG(desc_bytes >= hl_d3q27_links_batch_bytes(n_domains, int(rows.size())),
               "links batch: descriptor buffer too small");
  std::vector<unsigned char> h(hl_d3q27_links_batch_bytes(n_domains, int(rows.size())), 0);
  d3s::BatchHead head{n_domains, int(rows.size()), max_box, 0};
  std::memcpy(h.data(), &head, sizeof(head));
  std::memcpy(h.data() + d3s::LB_ARGS_OFF, args.data(), args.size() * sizeof(d3s::Args));
  std::memcpy(h.data() + d3s::lb_rows_off(n_domains), rows.data(), rows.size() * sizeof(int2));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(desc, h.data(), h.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "links batch: descriptor upload");
  *work_ints = d3s::LB_HEAD + 3 * capacity;
  std::lock_guard<std::mutex> lk(d3s::g_lb_mu);
  d3s::g_lb[desc] = {n_domains, int(rows.size()), max_box, *work_ints, worlds[0].storage.dtype};
  return HL_OK;
}

extern "C" int hl_d3q27_solid_links_batch(const void* desc, int n_domains, int parity, int32_t* work, size_t work_ints,
                                          hl_stream stream) {
  HL_CHECK_ARG(desc != nullptr && work != nullptr, "links batch: descriptors or work list is NULL");
  HL_CHECK_ARG(parity == 0 || parity == 1, "links batch: parity %d", parity);
  d3s::BatchInfo b;
  {
    std::lock_guard<std::mutex> lk(d3s::g_lb_mu);
    auto it = d3s::g_lb.find(desc);
    HL_CHECK_ARG(it != d3s::g_lb.end() && it->second.n_domains == n_domains,
                 "links batch: descriptors not prepared for %d domains", n_domains);
    b = it->second;
  }
  HL_CHECK_ARG(work_ints >= b.work_ints, "links batch: work list of %zu ints (needs %zu)", work_ints, b.work_ints);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(work, 0, d3s::LB_HEAD * sizeof(int32_t), st);
  if (e != cudaSuccess) return cuda_status(e, "links batch: zero work counters");
  switch (b.dtype) {
    case HL_F32: return d3s::launch_batch<StoreF32>(desc, b, parity, work, st);
    case HL_F16: return d3s::launch_batch<StoreF16>(desc, b, parity, work, st);
    case HL_BF16: return d3s::launch_batch<StoreBF16>(desc, b, parity, work, st);
    case HL_F64: return d3s::launch_batch<StoreF64>(desc, b, parity, work, st);
  }
  set_error("links batch: storage dtype %d not supported", int(b.dtype));
  return HL_ERR_UNSUPPORTED;
}
