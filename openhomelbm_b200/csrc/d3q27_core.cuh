// Shared D3Q27 arithmetic of the stream-collide kernels (d3q27.cu, d3q27_tma.cu).
#pragma once

#include "hl_common.cuh"

namespace hl {
namespace d3 {

struct StepArgs {
  const void* cur;
  void* post;
  long long N;  // cells per field plane
  int nx, ny, nz;
  int tiles_y, tiles_z, n_tiles;
  int chunk_len, n_items;
  double vis_shear;
  const float* force;
  const int* flag;
  Scale sc;
  double* partials;        // [gridDim.x] mass partials
  int* bad_partials;       // [gridDim.x]
  unsigned* counter;       // completion counter (returns to 0 after each launch)
  double* mass;
  int* health;
  int* status;             // set to HL_ERR_TIMEOUT if a bounded wait gives up (or NULL)
};

// host helpers shared by the launchers (d3q27.cu)
int num_sms();
size_t diag_scratch_bytes();
void fill_diag(StepArgs& a, const hl_diag* diag);
// TMA-staged variant (d3q27_tma.cu): every tile full (ny % 16 == 0, nz % 32 == 0)
bool tma_eligible(const hl_world3d* w);
int launch_step_tma(const hl_world3d* w, double vis_shear, const hl_diag* diag, cudaStream_t st);

// Partial moments of one destination cell.
template <class R> struct Acc {
  R rho, jx, jy, jz, pxx, pyy, pzz, pxy, pxz, pyz;
  __device__ void zero() { rho = jx = jy = jz = pxx = pyy = pzz = pxy = pxz = pyz = R(0); }
};

// Weight of a direction by its number of non-zero components (lbm_core_3d.py:24-31).
template <class R> __device__ __forceinline__ R w3(int nnz) {
  return nnz == 0 ? R(8.0 / 27.0) : nnz == 1 ? R(2.0 / 27.0) : nnz == 2 ? R(1.0 / 54.0) : R(1.0 / 216.0);
}

__host__ __device__ constexpr int dir_index(int cx, int cy, int cz) { return ((cx + 1) * 3 + (cy + 1)) * 3 + (cz + 1); }

// The 27 clamped populations a source cell sends, as deviations f - w, f[dir_index(c)].
template <class R> __device__ __forceinline__ void rebuild_all(const Mom3<R>& m, R f[27]) {
  const R usq = m.ux * m.ux + m.uy * m.uy + m.uz * m.uz;
  const R trS = m.sxx + m.syy + m.szz;
  const R A = m.drho - m.rho * (R(1.5) * usq + R(0.5) * trS);  // g - 1 at c = 0
  const R r3 = R(3) * m.rho, r15 = R(1.5) * m.rho, r45 = R(4.5) * m.rho, r9 = R(9) * m.rho;
  const R Bx = r3 * m.ux, By = r3 * m.uy, Bz = r3 * m.uz;
  const R Cxx = r45 * m.ux * m.ux + r15 * m.sxx;
  const R Cyy = r45 * m.uy * m.uy + r15 * m.syy;
  const R Czz = r45 * m.uz * m.uz + r15 * m.szz;
  const R Dxy = r9 * m.ux * m.uy + r3 * m.sxy;
  const R Dxz = r9 * m.ux * m.uz + r3 * m.sxz;
  const R Dyz = r9 * m.uy * m.uz + r3 * m.syz;
  // P(cy, cz) = g restricted to c_x = 0; Q(cy, cz) = the c_x-linear part.
  R P[3][3], Q[3][3];
  const R aY = A + Cyy, aZ = A + Czz, aYZ = aY + Czz;
  P[1][1] = A;
  P[2][1] = aY + By;
  P[0][1] = aY - By;
  P[1][2] = aZ + Bz;
  P[1][0] = aZ - Bz;
  const R s1 = By + Bz, s2 = By - Bz, bp = aYZ + Dyz, bm = aYZ - Dyz;
  P[2][2] = bp + s1;
  P[0][0] = bp - s1;
  P[2][0] = bm + s2;
  P[0][2] = bm - s2;
  const R t1 = Dxy + Dxz, t2 = Dxy - Dxz;
  Q[1][1] = Bx;
  Q[2][1] = Bx + Dxy;
  Q[0][1] = Bx - Dxy;
  Q[1][2] = Bx + Dxz;
  Q[1][0] = Bx - Dxz;
  Q[2][2] = Bx + t1;
  Q[0][0] = Bx - t1;
  Q[2][0] = Bx + t2;
  Q[0][2] = Bx - t2;
#pragma unroll
  for (int yi = 0; yi < 3; ++yi)
#pragma unroll
    for (int zi = 0; zi < 3; ++zi) {
      const int nyz = (yi != 1) + (zi != 1);
      const R p = P[yi][zi], pc = p + Cxx, q = Q[yi][zi];
      f[(1 * 3 + yi) * 3 + zi] = w3<R>(nyz) * fmax(p, R(-1));
      f[(2 * 3 + yi) * 3 + zi] = w3<R>(nyz + 1) * fmax(pc + q, R(-1));
      f[(0 * 3 + yi) * 3 + zi] = w3<R>(nyz + 1) * fmax(pc - q, R(-1));
    }
}

// Populations of the 9 (or 3) directions a halo cell sends into the tile, as deviations
// f - w. sel_y / sel_z (0, 1, 2 = c_y / c_z of -1, 0, +1, or -1 for any) pick the slice;
// out(dir_index(c), value) receives each population.
template <class R, class Out>
__device__ __forceinline__ void rebuild_slice(const Mom3<R>& m, int sel_y, int sel_z, Out out) {
  const R usq = m.ux * m.ux + m.uy * m.uy + m.uz * m.uz;
  const R trS = m.sxx + m.syy + m.szz;
  const R A = m.drho - m.rho * (R(1.5) * usq + R(0.5) * trS);
  const R r3 = R(3) * m.rho, r15 = R(1.5) * m.rho, r45 = R(4.5) * m.rho, r9 = R(9) * m.rho;
  const R Bx = r3 * m.ux, By = r3 * m.uy, Bz = r3 * m.uz;
  const R Cxx = r45 * m.ux * m.ux + r15 * m.sxx;
  const R Cyy = r45 * m.uy * m.uy + r15 * m.syy;
  const R Czz = r45 * m.uz * m.uz + r15 * m.szz;
  const R Dxy = r9 * m.ux * m.uy + r3 * m.sxy;
  const R Dxz = r9 * m.ux * m.uz + r3 * m.sxz;
  const R Dyz = r9 * m.uy * m.uz + r3 * m.syz;
#pragma unroll
  for (int yi = 0; yi < 3; ++yi)
#pragma unroll
    for (int zi = 0; zi < 3; ++zi) {
      if ((sel_y >= 0 && yi != sel_y) || (sel_z >= 0 && zi != sel_z)) continue;
      const R cy = R(yi - 1), cz = R(zi - 1);
      const R p = A + cy * By + cy * cy * Cyy + cz * Bz + cz * cz * Czz + cy * cz * Dyz;
      const R q = Bx + cy * Dxy + cz * Dxz;
      const R pc = p + Cxx;
      const int nyz = (yi != 1) + (zi != 1);
      out((1 * 3 + yi) * 3 + zi, w3<R>(nyz) * fmax(p, R(-1)));
      out((2 * 3 + yi) * 3 + zi, w3<R>(nyz + 1) * fmax(pc + q, R(-1)));
      out((0 * 3 + yi) * 3 + zi, w3<R>(nyz + 1) * fmax(pc - q, R(-1)));
    }
}

// A cell outside the domain: zero populations (f - w = -w), the reference's out-of-range rule.
template <class R> __device__ __forceinline__ Mom3<R> zero_cell() {
  Mom3<R> m;
  m.rho = R(0);
  m.drho = R(-1);
  m.ux = m.uy = m.uz = m.sxx = m.syy = m.szz = m.sxy = m.sxz = m.syz = R(0);
  return m;
}

// Regularised collision of stream_and_collide_3d (envs/lbm3d/lbm_func_3d.py:564-604), from
// deviation sums: a.rho = rho - 1, a.j = sum c f, a.p_ab = Pi_ab - delta_ab / 3. With
// Pi_aa = rho/3 + X_aa the reference's S_aa = Pi_aa/rho - 1/3 is X_aa / rho exactly.
template <class R>
__device__ __forceinline__ Mom3<R> collide(const Acc<R>& a, R Fx, R Fy, R Fz, R omega) {
  const R third = R(1.0 / 3.0);
  const R rho = R(1) + a.rho;
  const R inv = R(1) / rho;
  const R ux = (a.jx + R(0.5) * Fx) * inv;
  const R uy = (a.jy + R(0.5) * Fy) * inv;
  const R uz = (a.jz + R(0.5) * Fz) * inv;
  const R pxx_part = (R(2) * a.pxx - a.pyy - a.pzz) * third;
  const R pyy_part = (R(2) * a.pyy - a.pxx - a.pzz) * third;
  const R pzz_part = (R(2) * a.pzz - a.pxx - a.pyy) * third;
  const R RU2 = rho * ux * ux, RV2 = rho * uy * uy, RW2 = rho * uz * uz;
  const R RUVW2 = (RU2 + RV2 + RW2) * third;
  const R o1 = R(1) - omega;
  const R ot = omega * third;
  const R xxx = pxx_part * o1 + RUVW2 + R(2) * RU2 * ot - RV2 * ot - RW2 * ot + Fx * ux;
  const R xyy = pyy_part * o1 + RUVW2 - RU2 * ot + R(2) * RV2 * ot - RW2 * ot + Fy * uy;
  const R xzz = pzz_part * o1 + RUVW2 - RU2 * ot - RV2 * ot + R(2) * RW2 * ot + Fz * uz;
  const R pxy = a.pxy * o1 + ux * uy * rho * omega + (Fy * ux + Fx * uy) * R(0.5);
  const R pxz = a.pxz * o1 + ux * uz * rho * omega + (Fz * ux + Fx * uz) * R(0.5);
  const R pyz = a.pyz * o1 + uy * uz * rho * omega + (Fz * uy + Fy * uz) * R(0.5);
  Mom3<R> m;
  m.rho = rho;
  m.drho = a.rho;
  m.ux = ux + Fx * inv * R(0.5);
  m.uy = uy + Fy * inv * R(0.5);
  m.uz = uz + Fz * inv * R(0.5);
  m.sxx = xxx * inv;
  m.syy = xyy * inv;
  m.szz = xzz * inv;
  m.sxy = pxy * inv;
  m.sxz = pxz * inv;
  m.syz = pyz * inv;
  return m;
}

// Adds the group of 9 populations with one c_x (sx = c_x) to a destination's sums.
template <class R> __device__ __forceinline__ void accumulate_group(Acc<R>& a, const R p[3][3], int sx) {
  R Ry[3], Cz[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    Ry[i] = p[i][0] + p[i][1] + p[i][2];
    Cz[i] = p[0][i] + p[1][i] + p[2][i];
  }
  const R M0 = Ry[0] + Ry[1] + Ry[2];
  const R My = Ry[2] - Ry[0], Myy = Ry[2] + Ry[0];
  const R Mz = Cz[2] - Cz[0], Mzz = Cz[2] + Cz[0];
  const R Myz = (p[2][2] + p[0][0]) - (p[2][0] + p[0][2]);
  a.rho += M0;
  a.jy += My;
  a.jz += Mz;
  a.pyy += Myy;
  a.pzz += Mzz;
  a.pyz += Myz;
  if (sx != 0) {
    a.pxx += M0;
    if (sx > 0) {
      a.jx += M0;
      a.pxy += My;
      a.pxz += Mz;
    } else {
      a.jx -= M0;
      a.pxy -= My;
      a.pxz -= Mz;
    }
  }
}

template <class R> __device__ __forceinline__ bool healthy(const Mom3<R>& m) {
  const R s = m.ux + m.uy + m.uz + m.sxx + m.syy + m.szz + m.sxy + m.sxz + m.syz;
  return isfinite(m.rho) && isfinite(s) && m.rho > R(0);
}

// Block-wide sum (deterministic order) of a per-thread value; result valid in thread 0.
template <class V> __device__ V block_sum(V v, V* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  V s = V(0);
  if (threadIdx.x == 0)
    for (int i = 0; i < int(blockDim.x + 31) / 32; ++i) s += red[i];
  return s;
}

}  // namespace d3
}  // namespace hl
