// D3Q27 arithmetic on cell pairs (P2 lanes = two consecutive x planes of one column), for
// the TMA kernel (d3q27_tma.cu). Same mathematics as d3q27_core.cuh (the reference's
// mlCalEquilibrium3D_s rebuild, envs/lbm3d/lbm_func_3d.py:224-251, and the regularised
// collision, 564-604), arranged so that constants enter through a few loop-invariant pairs
// and every other operation is one packed instruction for both cells. The rearrangements
// (shared products, 3 rho u^2 built from 1.5 rho u^2, the trace-free parts as X - tr X / 3)
// change results only by rounding.
#pragma once

#include "d3q27_core.cuh"
#include "f32x2.cuh"

namespace hl {
namespace d3 {

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Loop-invariant pairs: lattice weights by number of non-zero velocity components, and the
// relaxation factors.
struct PairConst {
  P2 w0, w1, w2, w3;  // 8/27, 2/27, 1/54, 1/216
  P2 omega, o1;       // omega, 1 - omega
  P2 third, half;
};

__device__ __forceinline__ PairConst make_pair_const(float omega) {
  PairConst k;
  k.w0 = P2(8.0 / 27.0);
  k.w1 = P2(2.0 / 27.0);
  k.w2 = P2(1.0 / 54.0);
  k.w3 = P2(1.0 / 216.0);
  k.omega = P2(omega, omega);
  k.o1 = P2(1.f - omega, 1.f - omega);
  k.third = P2(1.0 / 3.0);
  k.half = P2(0.5);
  return k;
}

// Coefficients of the rebuilt deviation g(c) - 1 = A + c.B + sum_a c_a^2 C_aa + sum_{a<b}
// c_a c_b D_ab of one cell pair (rebuild_all in d3q27_core.cuh).
struct Coef {
  P2 A, Bx, By, Bz, Cxx, Cyy, Czz, Dxy, Dxz, Dyz;
};

__device__ __forceinline__ Coef coefficients(const Mom3<P2>& m, const PairConst& k) {
  Coef c;
  const P2 usq = m.ux * m.ux + m.uy * m.uy + m.uz * m.uz;
  const P2 trS = (m.sxx + m.syy) + m.szz;
  const P2 r15 = m.rho * k.half + m.rho;  // 1.5 rho
  const P2 r3 = r15 + r15, r45 = r3 + r15, r9 = r45 + r45;
  // A = drho - rho (1.5 |u|^2 + 0.5 tr S)
  c.A = m.drho - (r15 * usq + (m.rho * k.half) * trS);
  c.Bx = r3 * m.ux;
  c.By = r3 * m.uy;
  c.Bz = r3 * m.uz;
  c.Cxx = (r45 * m.ux) * m.ux + r15 * m.sxx;
  c.Cyy = (r45 * m.uy) * m.uy + r15 * m.syy;
  c.Czz = (r45 * m.uz) * m.uz + r15 * m.szz;
  const P2 r9x = r9 * m.ux;
  c.Dxy = r9x * m.uy + r3 * m.sxy;
  c.Dxz = r9x * m.uz + r3 * m.sxz;
  c.Dyz = (r9 * m.uy) * m.uz + r3 * m.syz;
  return c;
}

// w max(g, -1) = max(w g, -w) for w > 0, lane-wise: the clamp takes -w as an immediate.
template <int NNZ> __device__ __forceinline__ P2 clamp_w(P2 wg) {
  constexpr float w = NNZ == 0 ? float(8.0 / 27.0) : NNZ == 1 ? float(2.0 / 27.0) : NNZ == 2 ? float(1.0 / 54.0) : float(1.0 / 216.0);
  return P2(fmaxf(wg.x(), -w), fmaxf(wg.y(), -w));
}

// The three populations of one (c_y, c_z) with c_x = 0, +1, -1 (deviations f - w) from the
// c_x = 0 value p and the c_x-linear part q: w_n max(p, -1) and w_{n+1} max(p + Cxx +- q, -1),
// the latter as w_{n+1} p + w_{n+1} Cxx +- w_{n+1} q (one FFMA2 each).
template <int N>
__device__ __forceinline__ void column3(P2 p, P2 q, P2 wn, P2 wn1, P2 wCxx1, P2& f0, P2& fp, P2& fm) {
  f0 = clamp_w<N>(P2(wn * p));
  const P2 wpc = wn1 * p + wCxx1;
  fp = clamp_w<N + 1>(wn1 * q + wpc);
  fm = clamp_w<N + 1>(wpc - wn1 * q);
}

// All 27 clamped populations (deviations f - w) of an interior cell pair, f[dir_index].
__device__ __forceinline__ void rebuild_pair(const Coef& c, const PairConst& k, P2 f[27]) {
  P2 P[3][3], Q[3][3];
  const P2 aY = c.A + c.Cyy, aZ = c.A + c.Czz, aYZ = aY + c.Czz;
  P[1][1] = c.A;
  P[2][1] = aY + c.By;
  P[0][1] = aY - c.By;
  P[1][2] = aZ + c.Bz;
  P[1][0] = aZ - c.Bz;
  const P2 s1 = c.By + c.Bz, s2 = c.By - c.Bz, bp = aYZ + c.Dyz, bm = aYZ - c.Dyz;
  P[2][2] = bp + s1;
  P[0][0] = bp - s1;
  P[2][0] = bm + s2;
  P[0][2] = bm - s2;
  const P2 t1 = c.Dxy + c.Dxz, t2 = c.Dxy - c.Dxz;
  Q[1][1] = c.Bx;
  Q[2][1] = c.Bx + c.Dxy;
  Q[0][1] = c.Bx - c.Dxy;
  Q[1][2] = c.Bx + c.Dxz;
  Q[1][0] = c.Bx - c.Dxz;
  Q[2][2] = c.Bx + t1;
  Q[0][0] = c.Bx - t1;
  Q[2][0] = c.Bx + t2;
  Q[0][2] = c.Bx - t2;
  const P2 wC1 = k.w1 * c.Cxx, wC2 = k.w2 * c.Cxx, wC3 = k.w3 * c.Cxx;
#define HL_COL3(yi, zi, N, WN, WN1, WC)                                                                \
  column3<N>(P[yi][zi], Q[yi][zi], WN, WN1, WC, f[(1 * 3 + yi) * 3 + zi], f[(2 * 3 + yi) * 3 + zi], \
             f[(0 * 3 + yi) * 3 + zi])
  HL_COL3(1, 1, 0, k.w0, k.w1, wC1);
  HL_COL3(0, 1, 1, k.w1, k.w2, wC2);
  HL_COL3(2, 1, 1, k.w1, k.w2, wC2);
  HL_COL3(1, 0, 1, k.w1, k.w2, wC2);
  HL_COL3(1, 2, 1, k.w1, k.w2, wC2);
  HL_COL3(0, 0, 2, k.w2, k.w3, wC3);
  HL_COL3(0, 2, 2, k.w2, k.w3, wC3);
  HL_COL3(2, 0, 2, k.w2, k.w3, wC3);
  HL_COL3(2, 2, 2, k.w2, k.w3, wC3);
#undef HL_COL3
}

// The 9 populations a halo cell sends across one face of the tile: the slice with c_u = s
// (u = y for a row of the halo ring, z for a column), indexed [i][x] by the other component
// c_v = i - 1 and c_x = x - 1. sgn is the pair (s, s).
__device__ __forceinline__ void rebuild_face(const Coef& c, const PairConst& k, bool row, P2 sgn, P2 f[3][3]) {
  // g restricted to c_u = s: base + c_v lin + c_v^2 Cvv at c_x = 0, and the c_x-linear part
  // qb + c_v Dxv
  const P2 Bu = row ? c.By : c.Bz, Bv = row ? c.Bz : c.By;
  const P2 Cuu = row ? c.Cyy : c.Czz, Cvv = row ? c.Czz : c.Cyy;
  const P2 Dxu = row ? c.Dxy : c.Dxz, Dxv = row ? c.Dxz : c.Dxy;
  const P2 base = sgn * Bu + (c.A + Cuu);
  const P2 lin = sgn * c.Dyz + Bv;
  const P2 qb = sgn * Dxu + c.Bx;
  const P2 bC = base + Cvv;
  const P2 p[3] = {bC - lin, base, bC + lin};
  const P2 q[3] = {qb - Dxv, qb, qb + Dxv};
  const P2 wC2 = k.w2 * c.Cxx, wC3 = k.w3 * c.Cxx;
  column3<2>(p[0], q[0], k.w2, k.w3, wC3, f[0][1], f[0][2], f[0][0]);
  column3<1>(p[1], q[1], k.w1, k.w2, wC2, f[1][1], f[1][2], f[1][0]);
  column3<2>(p[2], q[2], k.w2, k.w3, wC3, f[2][1], f[2][2], f[2][0]);
}

// Regularised collision of a destination pair from its deviation sums (collide in
// d3q27_core.cuh), with the relaxation terms gathered: with R_a = rho u_a^2 and
// Rbar = (R_x + R_y + R_z) / 3, the reference's
//   X_aa = (1-omega) P_aa' + Rbar + omega/3 (2 R_a - R_b - R_c) + F_a u_a
// equals (1-omega)(P_aa' + Rbar) + omega R_a + F_a u_a.
template <bool FORCE>
__device__ __forceinline__ Mom3<P2> collide_pair(const Acc<P2>& a, P2 Fx, P2 Fy, P2 Fz, const PairConst& k) {
  const P2 rho = a.rho + P2(1.f, 1.f);
  // 1 / rho: the rcp.approx estimate (relative error below 2^-22 by the PTX ISA), then one
  // Newton-Raphson step for f(r) = 1/r - rho, r <- r + r (1 - rho r), which squares the relative
  // error to the binary32 rounding level; the parity tests against the binary64 oracle bound it
  const P2 r0(rcp_approx(rho.x()), rcp_approx(rho.y()));
  const P2 inv = r0 * (P2(1.f, 1.f) - rho * r0) + r0;
  P2 ux, uy, uz;
  if (FORCE) {
    ux = (Fx * k.half + a.jx) * inv;
    uy = (Fy * k.half + a.jy) * inv;
    uz = (Fz * k.half + a.jz) * inv;
  } else {
    ux = a.jx * inv;
    uy = a.jy * inv;
    uz = a.jz * inv;
  }
  const P2 tr3 = ((a.pxx + a.pyy) + a.pzz) * k.third;
  const P2 rux = rho * ux, ruy = rho * uy, ruz = rho * uz;
  const P2 RU2 = rux * ux, RV2 = ruy * uy, RW2 = ruz * uz;
  const P2 Rbar = ((RU2 + RV2) + RW2) * k.third;
  const P2 base = Rbar - tr3;  // Rbar - tr(P')/3
  P2 xxx = k.omega * RU2 + k.o1 * (a.pxx + base);
  P2 xyy = k.omega * RV2 + k.o1 * (a.pyy + base);
  P2 xzz = k.omega * RW2 + k.o1 * (a.pzz + base);
  P2 pxy = (rux * uy) * k.omega + a.pxy * k.o1;
  P2 pxz = (rux * uz) * k.omega + a.pxz * k.o1;
  P2 pyz = (ruy * uz) * k.omega + a.pyz * k.o1;
  Mom3<P2> m;
  m.rho = rho;
  m.drho = a.rho;
  if (FORCE) {
    xxx = Fx * ux + xxx;
    xyy = Fy * uy + xyy;
    xzz = Fz * uz + xzz;
    pxy = (Fy * ux + Fx * uy) * k.half + pxy;
    pxz = (Fz * ux + Fx * uz) * k.half + pxz;
    pyz = (Fz * uy + Fy * uz) * k.half + pyz;
    const P2 hi = inv * k.half;
    m.ux = Fx * hi + ux;
    m.uy = Fy * hi + uy;
    m.uz = Fz * hi + uz;
  } else {
    m.ux = ux;
    m.uy = uy;
    m.uz = uz;
  }
  m.sxx = xxx * inv;
  m.syy = xyy * inv;
  m.szz = xzz * inv;
  m.sxy = pxy * inv;
  m.sxz = pxz * inv;
  m.syz = pyz * inv;
  return m;
}

}  // namespace d3
}  // namespace hl
