// D2Q9 HOME-LBM step for sm_100a (replaces envs/lbm/lbm_func.py's kernels).
//
// One step of one or more worlds is four launches, the order of LBM_Solver.step
// (envs/lbm/lbm_solver.py:104-141):
//   1. prologue   precompute_transformed_segments (509-542), zeroing of the per-solid loads
//                 (init_force, 503-506) and the bounding box of the cells near any solid;
//   2. stream     stream_and_collide (322-467) for every fluid cell as if no solid existed;
//   3. band       the cells near a solid (get_cutcell's own test, 567-576) are recomputed
//                 with their cut links: the wall-velocity reconstruction of the link, the
//                 momentum exchange and the torque (349-401); loads are summed in binary64;
//   4. boundary   apply_bc (610-682) in the reference's sequential thread order, and the
//                 binary32 copies of the loads (solid_forcex, solid_forcey, torque).
// Cells in the band are computed twice; the band is a small part of the domain.

#include <cmath>

#include "hl_common.cuh"

namespace hl {
namespace d2 {

// D2Q9 velocities and opposites in the reference's order (envs/lbm/lbm_core.py:128-130).
__host__ __device__ constexpr int cx_of(int i) { return (i == 1 || i == 5 || i == 8) ? 1 : (i == 2 || i == 6 || i == 7) ? -1 : 0; }
__host__ __device__ constexpr int cy_of(int i) { return (i == 3 || i == 5 || i == 6) ? 1 : (i == 4 || i == 7 || i == 8) ? -1 : 0; }
__host__ __device__ constexpr int inv_of(int i) {
  return i == 0 ? 0 : i == 1 ? 2 : i == 2 ? 1 : i == 3 ? 4 : i == 4 ? 3 : i == 5 ? 7 : i == 6 ? 8 : i == 7 ? 5 : 6;
}
constexpr int MAX_SOLIDS = 64;

// D2Q9 weight of direction i (lbm_core.py:127).
template <class R> __device__ __forceinline__ R w2(int i) { return i == 0 ? R(4.0 / 9.0) : i < 5 ? R(1.0 / 9.0) : R(1.0 / 36.0); }

// Explicitly rounded operations: the population arithmetic below is written with them, so
// that every kernel using it rounds the same way whatever the surrounding code (the compiler
// neither fuses nor splits them), and a population is the same number whichever kernel and
// thread computes it.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// Third-order Hermite terms of mlCalDistribution (envs/lbm/lbm_func.py:695-696):
// Axxy = Sxx uy + 2 Sxy ux - 2 ux^2 uy, Axyy = Syy ux + 2 Sxy uy - 2 ux uy^2.
template <class R> __device__ __forceinline__ R third_xxy(const Mom2<R>& m) {
  const R u2 = mul_rn(mul_rn(R(2) * m.ux, m.ux), m.uy);
  return fma_rn(m.sxx, m.uy, fma_rn(R(2) * m.sxy, m.ux, -u2));
}
template <class R> __device__ __forceinline__ R third_xyy(const Mom2<R>& m) {
  const R u2 = mul_rn(mul_rn(R(2) * m.ux, m.uy), m.uy);
  return fma_rn(m.syy, m.ux, fma_rn(R(2) * m.sxy, m.uy, -u2));
}

// mlCalDistribution (envs/lbm/lbm_func.py:685-788): population i rebuilt from (rho, u, S)
// with the third-order Hermite terms Axxy, Axyy (given), returned as the deviation f_i - w_i
// (the reference's bracket minus one: w_i (rho - 1 + rho (bracket_i - 1))). Products by 2 and
// by powers of two are exact.
template <class R> __device__ __forceinline__ R feq_dev_a(const Mom2<R>& m, R Axxy, R Axyy, int i) {
  const R h = R(1.5), s3 = R(3), q = R(4.5), n = R(9);
  R b;
  switch (i) {
    case 0: b = fma_rn(-h, m.syy, mul_rn(-h, m.sxx)); break;
    case 1: b = fma_rn(-q, Axyy, fma_rn(-h, m.syy, fma_rn(s3, m.sxx, mul_rn(s3, m.ux)))); break;
    case 2: b = fma_rn(q, Axyy, fma_rn(-h, m.syy, fma_rn(s3, m.sxx, mul_rn(-s3, m.ux)))); break;
    case 3: b = fma_rn(-q, Axxy, fma_rn(s3, m.syy, fma_rn(-h, m.sxx, mul_rn(s3, m.uy)))); break;
    case 4: b = fma_rn(q, Axxy, fma_rn(s3, m.syy, fma_rn(-h, m.sxx, mul_rn(-s3, m.uy)))); break;
    case 5:
      b = fma_rn(n, add_rn(Axyy, Axxy), fma_rn(s3, fma_rn(s3, m.sxy, add_rn(m.sxx, m.syy)), mul_rn(s3, add_rn(m.ux, m.uy))));
      break;
    case 6:
      b = fma_rn(n, add_rn(Axxy, -Axyy),
                 fma_rn(s3, fma_rn(-s3, m.sxy, add_rn(m.sxx, m.syy)), fma_rn(s3, m.uy, mul_rn(-s3, m.ux))));
      break;
    case 7:
      b = fma_rn(-n, add_rn(Axxy, Axyy),
                 fma_rn(s3, fma_rn(s3, m.sxy, add_rn(m.sxx, m.syy)), fma_rn(-s3, m.uy, mul_rn(-s3, m.ux))));
      break;
    default:
      b = fma_rn(-n, add_rn(Axxy, -Axyy),
                 fma_rn(s3, fma_rn(-s3, m.sxy, add_rn(m.sxx, m.syy)), fma_rn(-s3, m.uy, mul_rn(s3, m.ux))));
      break;
  }
  return mul_rn(w2<R>(i), fma_rn(m.rho, b, m.drho));
}
template <class R> __device__ __forceinline__ R feq_dev(const Mom2<R>& m, int i) {
  return feq_dev_a<R>(m, third_xxy<R>(m), third_xyy<R>(m), i);
}

// The clamped deviation: f_i >= 0 is f_i - w_i >= -w_i (lbm_func.py:411-412).
template <class R> __device__ __forceinline__ R feq_dev_clamped(const Mom2<R>& m, int i) {
  return fmax(feq_dev<R>(m, i), -w2<R>(i));
}
template <class R> __device__ __forceinline__ R feq_dev_clamped_a(const Mom2<R>& m, R Axxy, R Axyy, int i) {
  return fmax(feq_dev_a<R>(m, Axxy, Axyy, i), -w2<R>(i));
}

// Moment-space collision of stream_and_collide (envs/lbm/lbm_func.py:414-467) from deviation
// populations pop[i] = f_i - w_i: rho = 1 + sum pop, Pi_aa = 1/3 + (deviation sum), and the
// reference's S_aa = Pi_aa/rho - 1/3 equals X_aa / rho with no cancellation. Written with the
// explicitly rounded operations, like the population arithmetic: every D2Q9 kernel (gridded,
// tile, strip and band) then collides a cell to the same number, whatever the compiler would
// contract in its surroundings. Multiplications by 0.5 are exact.
template <class R> __device__ __forceinline__ Mom2<R> collide(const R pop[9], R Fx, R Fy, R omega) {
  R drho = add_rn(pop[0], pop[1]);
#pragma unroll
  for (int i = 2; i < 9; ++i) drho = add_rn(drho, pop[i]);
  const R rho = add_rn(R(1), drho);
  const R inv = R(1) / rho;
  const R half = R(0.5);
  const R jx = add_rn(add_rn(add_rn(add_rn(add_rn(add_rn(pop[1], -pop[2]), pop[5]), -pop[6]), -pop[7]), pop[8]),
                      mul_rn(half, Fx));
  const R jy = add_rn(add_rn(add_rn(add_rn(add_rn(add_rn(pop[3], -pop[4]), pop[5]), pop[6]), -pop[7]), -pop[8]),
                      mul_rn(half, Fy));
  const R ux = mul_rn(jx, inv), uy = mul_rn(jy, inv);
  const R pixx0 = add_rn(add_rn(add_rn(add_rn(add_rn(pop[1], pop[2]), pop[5]), pop[6]), pop[7]), pop[8]);
  const R piyy0 = add_rn(add_rn(add_rn(add_rn(add_rn(pop[3], pop[4]), pop[5]), pop[6]), pop[7]), pop[8]);
  const R pixy0 = add_rn(add_rn(add_rn(pop[5], pop[7]), -pop[6]), -pop[8]);
  const R Ru2 = mul_rn(mul_rn(rho, ux), ux), Rv2 = mul_rn(mul_rn(rho, uy), uy);
  const R pxx_part = mul_rn(add_rn(pixx0, -piyy0), half), pyy_part = mul_rn(add_rn(piyy0, -pixx0), half);
  const R o1 = add_rn(R(1), -omega), oh = mul_rn(add_rn(R(1), omega), half), om = mul_rn(o1, half);
  const R fu = mul_rn(Fx, ux), fv = mul_rn(Fy, uy);
  const R pixy = fma_rn(o1, pixy0,
                        add_rn(mul_rn(mul_rn(mul_rn(ux, uy), rho), omega),
                               mul_rn(add_rn(R(1), -mul_rn(half, omega)), fma_rn(Fy, ux, mul_rn(Fx, uy)))));
  const R xxx = fma_rn(om, add_rn(fu, -fv), add_rn(fma_rn(om, Rv2, fma_rn(pxx_part, o1, mul_rn(oh, Ru2))), fu));
  const R xyy = fma_rn(om, add_rn(fv, -fu), add_rn(fma_rn(om, Ru2, fma_rn(pyy_part, o1, mul_rn(oh, Rv2))), fv));
  Mom2<R> m;
  m.rho = rho;
  m.drho = drho;
  m.ux = fma_rn(mul_rn(Fx, inv), half, ux);
  m.uy = fma_rn(mul_rn(Fy, inv), half, uy);
  m.sxx = mul_rn(xxx, inv);
  m.syy = mul_rn(xyy, inv);
  m.sxy = mul_rn(pixy, inv);
  return m;
}

template <class R> __device__ __forceinline__ R omega_of(double vis) { return R(1) / (R(vis) * R(3) + R(0.5)); }

// One world of a (possibly batched) 2D launch.
struct World {
  void* buf[2];  // the two moment buffers; cur = buf[parity], post = buf[parity ^ 1]
  const int* flag;
  const float* fx;
  const float* fy;
  int nx, ny;
  int periodic;
  double vis_shear;
  float grid_length, time_step;
  Scale sc;
  int bc_type[4];
  float bc_value[4][2];
  // solids
  int n_objects, max_segments;
  const float* line;
  const int* line_num;
  float* tf;
  float* tf_last;
  const float* position;
  const float* angle;
  const float* scale;
  const float* mass_center;
  const float* max_radius;
  double* loads64;
  float* force_x;
  float* force_y;
  float* torque;
  int* box;  // [4] x0, x1, y0, y1 of the cells near a solid (inclusive), empty if x0 > x1
};

// Kernel argument: one world by value, or a device array of worlds (batched launches).
struct Launch {
  World one;
  const World* many;
  int parity;
};

__device__ __forceinline__ const World& world_of(const Launch& L, int k) { return L.many ? L.many[k] : L.one; }
__device__ __forceinline__ const void* cur_of(const Launch& L, const World& w) { return w.buf[L.parity]; }
__device__ __forceinline__ void* post_of(const Launch& L, const World& w) { return w.buf[L.parity ^ 1]; }

template <class S> __device__ __forceinline__ Mom2<typename S::R> load2(const World& w, long long N, long long i,
                                                                        const typename S::T* m) {
  typename S::R raw[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) raw[k] = S::to_r(m[k * N + i]);
  return decode2<S>(raw, w.sc);
}
template <class S> __device__ __forceinline__ void store2(const World& w, long long N, long long i, typename S::T* m,
                                                          const Mom2<typename S::R>& v) {
  typename S::R raw[6];
  encode2<S>(v, w.sc, raw);
  // stochastic rounding of the reduced storages: one hash term per cell (dither_cell), the
  // same in every D2Q9 kernel so that they store a cell identically
  const unsigned cs = unsigned(i) * 0x9e3779b9u;
#pragma unroll
  for (int k = 0; k < 6; ++k) m[k * N + i] = S::from_r_cell(raw[k], cs, unsigned(k));
}

__device__ __forceinline__ bool is_fluid(const World& w, int x, int y, long long i) {
  if (w.flag) return w.flag[i] == ML_FLUID;
  if (w.periodic) return true;
  return x > 0 && x < w.nx - 1 && y > 0 && y < w.ny - 1;
}

// -------------------------------------------------------------------------- 1. prologue
__global__ void prologue_kernel(const __grid_constant__ Launch L) {
  const World& w = world_of(L, blockIdx.x);
  // a world of the batch without solids has no solid buffers (box, loads64 NULL)
  if (w.n_objects == 0 || w.box == nullptr) return;
  __shared__ int box[4];
  if (threadIdx.x == 0) {
    box[0] = w.nx;
    box[1] = -1;
    box[2] = w.ny;
    box[3] = -1;
  }
  __syncthreads();
  const int total = w.n_objects * w.max_segments;
  for (int k = threadIdx.x; k < total; k += blockDim.x) {
    const int sid = k / w.max_segments, idx = k % w.max_segments;
    if (idx >= w.line_num[sid]) continue;
    // precompute_transformed_segments, envs/lbm/lbm_func.py:509-542
    const float scale = w.scale[sid] * float(w.nx);
    float sa, ca;
    sincosf(w.angle[sid], &sa, &ca);
    const float ppx = (w.line[2 * k] - w.mass_center[2 * sid]) * scale;
    const float ppy = (w.line[2 * k + 1] - w.mass_center[2 * sid + 1]) * scale;
    const float nx_ = ppx * ca - ppy * sa + w.position[2 * sid];
    const float ny_ = ppx * sa + ppy * ca + w.position[2 * sid + 1];
    const float ox = w.tf[2 * k], oy = w.tf[2 * k + 1];
    if (ox == 0.f && oy == 0.f) {
      w.tf_last[2 * k] = nx_;
      w.tf_last[2 * k + 1] = ny_;
    } else {
      w.tf_last[2 * k] = ox;
      w.tf_last[2 * k + 1] = oy;
    }
    w.tf[2 * k] = nx_;
    w.tf[2 * k + 1] = ny_;
  }
  for (int s = threadIdx.x; s < w.n_objects; s += blockDim.x) {
    w.loads64[3 * s] = w.loads64[3 * s + 1] = w.loads64[3 * s + 2] = 0.0;
    if (w.line_num[s] <= 0) continue;
    // cells with |cell - position|^2 <= max_radius * (scale nx)^2 (get_cutcell, 567-576)
    const float sc = w.scale[s] * float(w.nx);
    const float r = sqrtf(fmaxf(w.max_radius[s] * sc * sc, 0.f)) + 1.f;
    const float px = w.position[2 * s], py = w.position[2 * s + 1];
    if (!(isfinite(px) && isfinite(py) && isfinite(r))) continue;
    const int x0 = max(0, int(floorf(px - r))), x1 = min(w.nx - 1, int(ceilf(px + r)));
    const int y0 = max(0, int(floorf(py - r))), y1 = min(w.ny - 1, int(ceilf(py + r)));
    if (x0 > x1 || y0 > y1) continue;
    atomicMin(&box[0], x0);
    atomicMax(&box[1], x1);
    atomicMin(&box[2], y0);
    atomicMax(&box[3], y1);
  }
  __syncthreads();
  if (threadIdx.x < 4) w.box[threadIdx.x] = box[threadIdx.x];
}

// -------------------------------------------------------------------------- 2. stream
// Pull streaming for every fluid cell, ignoring solids. blockIdx.z = world.
template <class S> __global__ void __launch_bounds__(256) stream_kernel(const __grid_constant__ Launch L) {
  using R = typename S::R;
  using T = typename S::T;
  const World& w = world_of(L, blockIdx.z);
  const int y = blockIdx.x * 32 + (threadIdx.x & 31);
  const int x = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (x >= w.nx || y >= w.ny) return;
  const long long N = (long long)w.nx * w.ny;
  const long long c = (long long)x * w.ny + y;
  if (!is_fluid(w, x, y, c)) return;
  const T* cur = static_cast<const T*>(cur_of(L, w));
  R pop[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    int xn = x - cx_of(i), yn = y - cy_of(i);
    if (w.periodic) {
      xn = wrap(xn, w.nx);
      yn = wrap(yn, w.ny);
    }
    if (xn >= 0 && xn < w.nx && yn >= 0 && yn < w.ny) {
      pop[i] = feq_dev_clamped<R>(load2<S>(w, N, (long long)xn * w.ny + yn, cur), i);
    } else {
      pop[i] = -w2<R>(i);  // out of range: f = 0
    }
  }
  const R Fx = w.fx ? R(w.fx[c]) : R(0), Fy = w.fy ? R(w.fy[c]) : R(0);
  store2<S>(w, N, c, static_cast<T*>(post_of(L, w)), collide<R>(pop, Fx, Fy, omega_of<R>(w.vis_shear)));
}

// ------------------------------------------------------------- 2b. stream over a tile work-list
// The stream phase of batched worlds of different sizes as one persistent launch: the CTAs of
// a fixed grid take the tiles of a work list in turn (tile t = {world, x0, y0, 0}, TX x TY
// cells, clipped to the world). Source side: every source cell of the tile and its one-cell
// halo is read once (coalesced rows along y) and decoded in registers; it rebuilds its
// clamped populations and writes each one into the shared-memory mailbox of the destination
// it streams to. A source outside a walled world writes -w_i (f = 0, stream_kernel's
// out-of-range rule). After a barrier every fluid destination reads its nine populations,
// collides and stores. Every population is stream_kernel's value (the same decode, the same
// third-order terms, feq_dev_clamped and collide), so the results are identical to it.
constexpr int TILE_THREADS = 256;

// Mailbox of a TX x TY tile: [9][(TX + 2) x (TY + 2)] destination slots, padded by one cell
// so that a source inside the tile writes all nine populations without checks (those that
// land in the padding are never read).
template <int TX, int TY, class R> constexpr size_t tile_smem_bytes() {
  return size_t(9) * (TX + 2) * (TY + 2) * sizeof(R);
}

// Source cell at padded tile coordinates (hx, hy) (tile cell (hx - 1, hy - 1)): its
// populations into the mailbox; CHECK: only those landing on a tile cell (halo sources).
template <class S, int TX, int TY, bool CHECK>
__device__ __forceinline__ void send_source(typename S::R* mb, int hx, int hy, int x0, int y0, int nx, int ny,
                                            bool periodic, long long N, const typename S::T* __restrict__ cur,
                                            const Scale& sc) {
  using R = typename S::R;
  constexpr int HY = TY + 2, HC = (TX + 2) * HY;
  int gx = x0 - 1 + hx, gy = y0 - 1 + hy;
  if (periodic) {
    gx = wrap(gx, nx);
    gy = wrap(gy, ny);
  }
  const bool in = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
  Mom2<R> m{};
  R axxy = R(0), axyy = R(0);
  if (in) {
    const long long i = (long long)gx * ny + gy;
    R raw[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) raw[k] = S::to_r(cur[k * N + i]);
    m = decode2<S>(raw, sc);
    axxy = third_xxy<R>(m);
    axyy = third_xyy<R>(m);
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const int dx = hx + cx_of(i), dy = hy + cy_of(i);  // destination slot
    if (CHECK && (dx < 1 || dx > TX || dy < 1 || dy > TY)) continue;
    mb[i * HC + dx * HY + dy] = in ? feq_dev_clamped_a<R>(m, axxy, axyy, i) : -w2<R>(i);
  }
}

template <class S, int TX, int TY>
__global__ void __launch_bounds__(TILE_THREADS) stream_tiles_kernel(const __grid_constant__ Launch L,
                                                                    const int4* __restrict__ tiles, int n_tiles) {
  using R = typename S::R;
  using T = typename S::T;
  constexpr int HY = TY + 2, HC = (TX + 2) * HY, NC = TX * TY, NH = 2 * HY + 2 * TX;
  extern __shared__ __align__(16) unsigned char tile_smem[];
  R* mb = reinterpret_cast<R*>(tile_smem);
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int4 tile = tiles[t];
    // the world's fields in registers: reads through the descriptor could not be kept across
    // the stores to post
    const World& wd = world_of(L, tile.x);
    const int nx = wd.nx, ny = wd.ny;
    const bool periodic = wd.periodic != 0;
    const int* __restrict__ flag = wd.flag;
    const float* __restrict__ fxp = wd.fx;
    const float* __restrict__ fyp = wd.fy;
    const Scale sc = wd.sc;
    const T* __restrict__ cur = static_cast<const T*>(cur_of(L, wd));
    T* __restrict__ post = static_cast<T*>(post_of(L, wd));
    const R omega = omega_of<R>(wd.vis_shear);
    const int x0 = tile.y, y0 = tile.z;
    const long long N = (long long)nx * ny;
    __syncthreads();  // the previous tile's destinations are done with the mailbox
    for (int c = threadIdx.x; c < NC; c += TILE_THREADS)  // sources on the tile
      send_source<S, TX, TY, false>(mb, 1 + c / TY, 1 + c % TY, x0, y0, nx, ny, periodic, N, cur, sc);
    for (int k = threadIdx.x; k < NH; k += TILE_THREADS) {  // the ring of halo sources
      int hx, hy;
      if (k < 2 * HY) {
        hx = k < HY ? 0 : TX + 1;
        hy = k < HY ? k : k - HY;
      } else {
        const int j = k - 2 * HY;
        hx = 1 + (j >> 1);
        hy = (j & 1) ? TY + 1 : 0;
      }
      send_source<S, TX, TY, true>(mb, hx, hy, x0, y0, nx, ny, periodic, N, cur, sc);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < NC; c += TILE_THREADS) {
      const int lx = c / TY, ly = c % TY;
      const int x = x0 + lx, y = y0 + ly;
      if (x >= nx || y >= ny) continue;
      const long long ci = (long long)x * ny + y;
      if (flag ? flag[ci] != ML_FLUID : !periodic && !(x > 0 && x < nx - 1 && y > 0 && y < ny - 1)) continue;
      const int slot = (lx + 1) * HY + ly + 1;
      R pop[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) pop[i] = mb[i * HC + slot];
      const R Fx = fxp ? R(fxp[ci]) : R(0), Fy = fyp ? R(fyp[ci]) : R(0);
      R raw[6];
      encode2<S>(collide<R>(pop, Fx, Fy, omega), sc, raw);
      const unsigned cs = unsigned(ci) * 0x9e3779b9u;  // as store2
#pragma unroll
      for (int k = 0; k < 6; ++k) post[k * N + ci] = S::from_r_cell(raw[k], cs, unsigned(k));
    }
  }
}

// ------------------------------------------------------------- 2c. stream over strips (a warp each)
// Strip tiles of the work list: TX planes along x by STRIP_Y = 30 rows along y, one warp each.
// Lane l holds row y0 - 1 + l (lanes 0 and 31 are the strip's halo rows) and the warp marches its
// source planes x0 - 1 .. x0 + TX. Each lane rebuilds its source cell's nine clamped populations
// (feq_dev_clamped_a on its decoded moments, -w_i for a source outside a walled world: the same
// values as stream_kernel), the populations with c_y = +-1 move one lane by a warp shuffle, and
// those with c_x = 0, +1 wait in registers for the next source planes: once source plane x_s is
// read, destination plane x_s - 1 has all nine of its populations, and the lanes of rows
// y0 .. y0 + 29 collide and store it with stream_kernel's collide and store. No shared memory and
// no block barrier; a strip needs 32/30 of the source work of its cells. Results are identical to
// stream_kernel. The 32-plane strips with 2- or 4-byte storage are held to 64 registers (four
// blocks of 8 warps per SM instead of three), which is faster for them; the 64- and 128-plane
// strips run slower at that cap, and binary64 storage would spill heavily.
constexpr int STRIP_Y = 30;
template <class S, int TX>
constexpr int strip_min_blocks() { return TX == 32 && sizeof(typename S::T) <= 4 ? 4 : 1; }

template <class S, int TX>
__global__ void __launch_bounds__(256, strip_min_blocks<S, TX>()) stream_strips_kernel(const __grid_constant__ Launch L,
                                                            const int4* __restrict__ tiles, int n_tiles) {
  using R = typename S::R;
  using T = typename S::T;
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < n_tiles; t += warps) {
    const int4 tile = tiles[t];
    const World& wd = world_of(L, tile.x);
    const int nx = wd.nx, ny = wd.ny;
    const bool periodic = wd.periodic != 0;
    const float* __restrict__ fxp = wd.fx;
    const float* __restrict__ fyp = wd.fy;
    const Scale sc = wd.sc;
    const T* __restrict__ cur = static_cast<const T*>(cur_of(L, wd));
    T* __restrict__ post = static_cast<T*>(post_of(L, wd));
    const R omega = omega_of<R>(wd.vis_shear);
    const long long N = (long long)nx * ny;
    const int x0 = tile.y, y0 = tile.z;
    const int x1 = x0 + TX < nx ? x0 + TX : nx;  // destination planes x0 .. x1 - 1
    const int yr = y0 - 1 + lane;                // this lane's row, before wrapping
    const int y = periodic ? wrap(yr, ny) : yr;
    const bool y_in = periodic || (yr >= 0 && yr < ny);
    const bool dest_lane = lane >= 1 && lane <= STRIP_Y && yr < ny;
    // incoming populations of the last two source planes: c_x = 0 (i = 0, 3, 4) of the previous
    // plane, c_x = +1 (i = 1, 5, 8) of the previous two
    R z0 = R(0), z3 = R(0), z4 = R(0), p1 = R(0), p5 = R(0), p8 = R(0), q1 = R(0), q5 = R(0), q8 = R(0);
    // the next source plane's stored moments are loaded one plane ahead
    auto fetch = [&](int xs, T* t) {
      const int xw = periodic ? wrap(xs, nx) : xs;
      if (y_in && (periodic || (xs >= 0 && xs < nx))) {
        const long long c = (long long)xw * ny + y;
#pragma unroll
        for (int k = 0; k < 6; ++k) t[k] = cur[k * N + c];
      }
    };
    T tn[6];
    fetch(x0 - 1, tn);
    for (int xs = x0 - 1; xs <= x1; ++xs) {
      const bool in = y_in && (periodic || (xs >= 0 && xs < nx));
      T tc[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) tc[k] = tn[k];
      if (xs < x1) fetch(xs + 1, tn);
      R f[9];
      if (in) {
        R raw[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) raw[k] = S::to_r(tc[k]);
        const Mom2<R> m = decode2<S>(raw, sc);
        const R axxy = third_xxy<R>(m), axyy = third_xyy<R>(m);
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = feq_dev_clamped_a<R>(m, axxy, axyy, i);
      } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = -w2<R>(i);
      }
      // what arrives at this lane's row from source plane xs: c_y = +1 from the lane below,
      // c_y = -1 from the lane above (lanes 0 and 31 receive garbage; they store nothing)
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        if (cy_of(i) == 1) f[i] = __shfl_up_sync(FULL, f[i], 1);
        else if (cy_of(i) == -1) f[i] = __shfl_down_sync(FULL, f[i], 1);
      }
      const int d = xs - 1;  // the destination plane now complete
      if (dest_lane && d >= x0 && d < x1) {
        const long long ci = (long long)d * ny + yr;
        if (is_fluid(wd, d, yr, ci)) {
          R pop[9];
          pop[0] = z0;
          pop[3] = z3;
          pop[4] = z4;
          pop[1] = q1;
          pop[5] = q5;
          pop[8] = q8;
          pop[2] = f[2];
          pop[6] = f[6];
          pop[7] = f[7];
          const R Fx = fxp ? R(fxp[ci]) : R(0), Fy = fyp ? R(fyp[ci]) : R(0);
          R raw[6];
          encode2<S>(collide<R>(pop, Fx, Fy, omega), sc, raw);
          const unsigned cs = unsigned(ci) * 0x9e3779b9u;  // as store2
#pragma unroll
          for (int k = 0; k < 6; ++k) post[k * N + ci] = S::from_r_cell(raw[k], cs, unsigned(k));
        }
      }
      q1 = p1;
      q5 = p5;
      q8 = p8;
      p1 = f[1];
      p5 = f[5];
      p8 = f[8];
      z0 = f[0];
      z3 = f[3];
      z4 = f[4];
    }
  }
}

// -------------------------------------------------------------------------- 3. band
struct Cut {
  float t, ratio;
  int solid, seg;
};

// get_cutcell (envs/lbm/lbm_func.py:545-607)
__device__ Cut get_cutcell(const World& w, float x, float y, float dx, float dy) {
  Cut r{-1.f, -1.f, -1, -1};
  const float ax = x - dx, ay = y - dy, bx = x, by = y;
  for (int s = 0; s < w.n_objects; ++s) {
    const float px = x - w.position[2 * s], py = y - w.position[2 * s + 1];
    const float scale = w.scale[s] * float(w.nx);
    if (px * px + py * py > w.max_radius[s] * scale * scale) continue;
    const int nseg = w.line_num[s];
    const float* tf = w.tf + size_t(s) * w.max_segments * 2;
    for (int n = 0; n < nseg; ++n) {
      const int n1 = n + 1 == nseg ? 0 : n + 1;
      const float cx = tf[2 * n], cy = tf[2 * n + 1], ex = tf[2 * n1], ey = tf[2 * n1 + 1];
      const float abc = (ax - cx) * (by - cy) - (ay - cy) * (bx - cx);
      const float abd = (ax - ex) * (by - ey) - (ay - ey) * (bx - ex);
      if (abc * abd >= 0.f) continue;
      const float cda = (cx - ax) * (ey - ay) - (cy - ay) * (ex - ax);
      const float cdb = cda + abc - abd;
      if (cda * cdb > 0.f) continue;
      const float t = 1.f - cda / (abd - abc);
      if (r.t < 0.f || t < r.t) {
        r.t = t;
        r.solid = s;
        r.ratio = abc / (abc - abd);
        r.seg = n;
      }
    }
  }
  return r;
}

// get_cutcell over a candidate list: cand[k] = (solid << 16) | segment, in ascending
// (solid, segment) order, holding every segment of a near solid that can cross a link of the
// cell. The per-segment arithmetic and the tie rule (first nearest wins) are get_cutcell's, so
// the result is the same.
// tf_all / nseg_all: the world's transformed segments [n][max_segments][2] and segment counts
// (shared-memory copies or the world's own arrays).
__device__ Cut get_cutcell_list(const float* tf_all, const int* nseg_all, int max_segments, const int* cand, int nc,
                                float x, float y, float dx, float dy) {
  Cut r{-1.f, -1.f, -1, -1};
  const float ax = x - dx, ay = y - dy, bx = x, by = y;
  for (int k = 0; k < nc; ++k) {
    const int s = cand[k] >> 16, n = cand[k] & 0xffff;
    const int nseg = nseg_all[s];
    const float* tf = tf_all + size_t(s) * max_segments * 2;
    const int n1 = n + 1 == nseg ? 0 : n + 1;
    const float cx = tf[2 * n], cy = tf[2 * n + 1], ex = tf[2 * n1], ey = tf[2 * n1 + 1];
    const float abc = (ax - cx) * (by - cy) - (ay - cy) * (bx - cx);
    const float abd = (ax - ex) * (by - ey) - (ay - ey) * (bx - ex);
    if (abc * abd >= 0.f) continue;
    const float cda = (cx - ax) * (ey - ay) - (cy - ay) * (ex - ax);
    const float cdb = cda + abc - abd;
    if (cda * cdb > 0.f) continue;
    const float t = 1.f - cda / (abd - abc);
    if (r.t < 0.f || t < r.t) {
      r.t = t;
      r.solid = s;
      r.ratio = abc / (abc - abd);
      r.seg = n;
    }
  }
  return r;
}

constexpr int MAX_CAND = 24;  // candidate segments kept per cell; more: the full scan
constexpr int BAND_TF_FLOATS = 4096;  // transformed segment coordinates staged per block

template <class S> __global__ void __launch_bounds__(256) band_kernel(const __grid_constant__ Launch L) {
  using R = typename S::R;
  using T = typename S::T;
  const World& w = world_of(L, blockIdx.y);
  if (w.n_objects == 0 || w.box == nullptr) return;  // a world of the batch without solids
  const int x0 = w.box[0], x1 = w.box[1], y0 = w.box[2], y1 = w.box[3];
  // (block-uniform) a block past the end of the band has no cell
  if (x0 > x1 || y0 > y1 || (long long)blockIdx.x * blockDim.x >= (long long)(x1 - x0 + 1) * (y1 - y0 + 1)) return;
  __shared__ double acc[MAX_SOLIDS * 3];
  __shared__ int touched;
  // the world's per-solid band radii and segments, read by every cell's screening and ray
  // tests: staged in shared memory (the segments when they fit)
  __shared__ float s_tf[BAND_TF_FLOATS];
  __shared__ float s_px[MAX_SOLIDS], s_py[MAX_SOLIDS], s_r2[MAX_SOLIDS];
  __shared__ int s_nseg[MAX_SOLIDS];
  const int nsol = min(w.n_objects, MAX_SOLIDS);
  const int n_tf = w.n_objects * w.max_segments * 2;
  const bool staged = w.n_objects <= MAX_SOLIDS && n_tf <= BAND_TF_FLOATS;
  for (int k = threadIdx.x; k < nsol * 3; k += blockDim.x) acc[k] = 0.0;
  for (int s = threadIdx.x; s < nsol; s += blockDim.x) {
    const float scale = w.scale[s] * float(w.nx);
    s_px[s] = w.position[2 * s];
    s_py[s] = w.position[2 * s + 1];
    s_r2[s] = w.max_radius[s] * scale * scale;
    s_nseg[s] = w.line_num[s];
  }
  if (staged)
    for (int k = threadIdx.x; k < n_tf; k += blockDim.x) s_tf[k] = w.tf[k];
  if (threadIdx.x == 0) touched = 0;
  __syncthreads();
  const float* tfb = staged ? s_tf : w.tf;
  const long long N = (long long)w.nx * w.ny;
  const T* cur = static_cast<const T*>(cur_of(L, w));
  {
    const int bw = y1 - y0 + 1;
    const long long area = (long long)(x1 - x0 + 1) * bw;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < area;
         k += (long long)gridDim.x * blockDim.x) {
      const int x = x0 + int(k / bw), y = y0 + int(k % bw);
      const long long c = (long long)x * w.ny + y;
      if (!is_fluid(w, x, y, c)) continue;
      // The segments of the near solids (get_cutcell's radius test) that can cross a link of
      // this cell: every link lies in the square [x-1, x+1] x [y-1, y+1], so a segment whose
      // box misses that square widened by 1e-3 crosses none. No candidate: no cut link, and
      // the stream kernel's value is already the cell's update.
      int cand[MAX_CAND];
      int nc = 0;
      bool overflow = false;
      const float fxc = float(x), fyc = float(y);
      for (int s = 0; s < nsol; ++s) {
        const int nseg = s_nseg[s];
        if (nseg <= 0) continue;
        const float px = fxc - s_px[s], py = fyc - s_py[s];
        if (px * px + py * py > s_r2[s]) continue;
        const float* tf = tfb + size_t(s) * w.max_segments * 2;
        for (int n = 0; n < nseg; ++n) {
          const int n1 = n + 1 == nseg ? 0 : n + 1;
          const float cx = tf[2 * n], cy = tf[2 * n + 1], ex = tf[2 * n1], ey = tf[2 * n1 + 1];
          if (fmaxf(cx, ex) < fxc - 1.001f || fminf(cx, ex) > fxc + 1.001f || fmaxf(cy, ey) < fyc - 1.001f ||
              fminf(cy, ey) > fyc + 1.001f)
            continue;
          if (nc < MAX_CAND)
            cand[nc++] = (s << 16) | n;
          else
            overflow = true;
        }
      }
      if (nc == 0) continue;
      const Mom2<R> me = load2<S>(w, N, c, cur);
      R pop[9];
      bool any_cut = false;
#pragma unroll 1
      for (int i = 0; i < 9; ++i) {
        int xn = x - cx_of(i), yn = y - cy_of(i);
        if (w.periodic) {
          xn = wrap(xn, w.nx);
          yn = wrap(yn, w.ny);
        }
        pop[i] = -w2<R>(i);
        if (!(xn >= 0 && xn < w.nx && yn >= 0 && yn < w.ny)) continue;
        const Cut cc = overflow ? get_cutcell(w, fxc, fyc, float(cx_of(i)), float(cy_of(i)))
                                : get_cutcell_list(tfb, s_nseg, w.max_segments, cand, nc, fxc, fyc, float(cx_of(i)),
                                                   float(cy_of(i)));
        if (cc.t >= 0.f && cc.solid >= 0) {
          any_cut = true;
          const int s = cc.solid, nseg = w.line_num[s];
          const int n1 = cc.seg + 1 == nseg ? 0 : cc.seg + 1;
          const float* tf = w.tf + size_t(s) * w.max_segments * 2;
          const float* tl = w.tf_last + size_t(s) * w.max_segments * 2;
          const float pcx = tf[2 * cc.seg] + (tf[2 * n1] - tf[2 * cc.seg]) * cc.ratio;
          const float pcy = tf[2 * cc.seg + 1] + (tf[2 * n1 + 1] - tf[2 * cc.seg + 1]) * cc.ratio;
          const float plx = tl[2 * cc.seg] + (tl[2 * n1] - tl[2 * cc.seg]) * cc.ratio;
          const float ply = tl[2 * cc.seg + 1] + (tl[2 * n1 + 1] - tl[2 * cc.seg + 1]) * cc.ratio;
          const R upx = R((pcx - plx) / w.time_step), upy = R((pcy - ply) / w.time_step);
          const R rx = R(pcx - w.position[2 * s]), ry = R(pcy - w.position[2 * s + 1]);
          Mom2<R> ms = me;
          ms.ux = upx;
          ms.uy = upy;
          ms.sxx = upx * upx + me.sxx - me.ux * me.ux;
          ms.syy = upy * upy + me.syy - me.uy * me.uy;
          ms.sxy = upx * upy + me.sxy - me.ux * me.uy;
          pop[i] = feq_dev_clamped<R>(ms, i);
          const int ii = inv_of(i);
          // momentum exchange with the full populations f = w + (f - w)
          const R cur_f = w2<R>(ii) + feq_dev<R>(me, ii);
          const R pop_f = w2<R>(i) + pop[i];
          const R fx = cur_f * (R(cx_of(ii)) - upx) - pop_f * (R(cx_of(i)) - upx);
          const R fy = cur_f * (R(cy_of(ii)) - upy) - pop_f * (R(cy_of(i)) - upy);
          const R tq = (rx * fy - ry * fx) * R(w.grid_length);
          if (s < MAX_SOLIDS) {
            atomicAdd(&acc[3 * s], double(fx));
            atomicAdd(&acc[3 * s + 1], double(fy));
            atomicAdd(&acc[3 * s + 2], double(tq));
            touched = 1;
          }
        } else {
          pop[i] = feq_dev_clamped<R>(load2<S>(w, N, (long long)xn * w.ny + yn, cur), i);
        }
      }
      if (!any_cut) continue;  // the stream kernel's value is already this cell's update
      const R Fx = w.fx ? R(w.fx[c]) : R(0), Fy = w.fy ? R(w.fy[c]) : R(0);
      store2<S>(w, N, c, static_cast<T*>(post_of(L, w)), collide<R>(pop, Fx, Fy, omega_of<R>(w.vis_shear)));
    }
  }
  __syncthreads();
  if (touched)
    for (int k = threadIdx.x; k < nsol * 3; k += blockDim.x)
      if (acc[k] != 0.0) atomicAdd(&w.loads64[k], acc[k]);
}

// -------------------------------------------------------------------------- 4. boundary
// f_eq_home (envs/lbm/lbm_func.py:660-682): S of the clamped equilibrium populations, from
// deviations: S_aa = (sum of f - w over c_a != 0 - (rho - 1)/3) / rho.
template <class R> __device__ void feq_s(R rho, R drho, R ux, R uy, R out[3]) {
  const R usq = ux * ux + uy * uy;
  R p[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const R cu = R(cx_of(i)) * ux + R(cy_of(i)) * uy;
    p[i] = fmax(w2<R>(i) * (drho + rho * (R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq)), -w2<R>(i));
  }
  const R inv = R(1) / rho;
  const R d3 = drho * R(1.0 / 3.0);
  out[0] = ((p[1] + p[2] + p[5] + p[6] + p[7] + p[8]) - d3) * inv;
  out[1] = ((p[3] + p[4] + p[5] + p[6] + p[7] + p[8]) - d3) * inv;
  out[2] = (p[5] + p[7] - p[6] - p[8]) * inv;
}

// apply_bc_core (envs/lbm/lbm_func.py:634-657)
template <class R> __device__ Mom2<R> bc_core(const World& w, int dr, const Mom2<R>& t, const Mom2<R>& nb) {
  Mom2<R> r = t;
  if (w.bc_type[dr] == 0) {
    r.ux = R(w.bc_value[dr][0]);
    r.uy = R(w.bc_value[dr][1]);
  } else if (w.bc_type[dr] == 1) {
    r.ux = nb.ux;
    r.uy = nb.uy;
  }
  r.rho = nb.rho;
  r.drho = nb.drho;
  R sc[3], sb[3];
  feq_s<R>(r.rho, r.drho, r.ux, r.uy, sc);
  feq_s<R>(nb.rho, nb.drho, nb.ux, nb.uy, sb);
  r.sxx = sc[0] - sb[0] + nb.sxx;
  r.syy = sc[1] - sb[1] + nb.syy;
  r.sxy = sc[2] - sb[2] + nb.sxy;
  return r;
}

// One CTA per world. Threads of the reference run in launch order (x outer, y inner): a
// corner reads a neighbour on a low face (x = 0 or y = 0) before that neighbour's update
// and one on a high face after it. Phase 1 updates the non-corner border cells, saving the
// four cells corners read "before update"; phase 2 updates the corners.
template <class S> __global__ void __launch_bounds__(512) boundary_kernel(const __grid_constant__ Launch L) {
  using R = typename S::R;
  using T = typename S::T;
  const World& w = world_of(L, blockIdx.x);
  const long long N = (long long)w.nx * w.ny;
  T* post = static_cast<T*>(post_of(L, w));
  __shared__ R snap[4][7];  // (1,0) (0,1) (1,ny-1) (nx-1,1)
  if (!w.periodic) {
    const int ex = w.nx - 2, ey = w.ny - 2;  // border cells per side without corners
    const int total = 2 * ey + 2 * ex;
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
      int x, y, dr, xn, yn;
      if (k < ey) { x = 0; y = 1 + k; dr = 0; xn = 1; yn = y; }
      else if (k < 2 * ey) { x = w.nx - 1; y = 1 + k - ey; dr = 2; xn = w.nx - 2; yn = y; }
      else if (k < 2 * ey + ex) { x = 1 + k - 2 * ey; y = w.ny - 1; dr = 1; xn = x; yn = w.ny - 2; }
      else { x = 1 + k - 2 * ey - ex; y = 0; dr = 3; xn = x; yn = 1; }
      const long long c = (long long)x * w.ny + y;
      const Mom2<R> t = load2<S>(w, N, c, post);
      int slot = -1;
      if (x == 1 && y == 0) slot = 0;
      else if (x == 0 && y == 1) slot = 1;
      else if (x == 1 && y == w.ny - 1) slot = 2;
      else if (x == w.nx - 1 && y == 1) slot = 3;
      if (slot >= 0) {
        snap[slot][0] = t.rho; snap[slot][1] = t.ux; snap[slot][2] = t.uy;
        snap[slot][3] = t.sxx; snap[slot][4] = t.syy; snap[slot][5] = t.sxy; snap[slot][6] = t.drho;
      }
      store2<S>(w, N, c, post, bc_core<R>(w, dr, t, load2<S>(w, N, (long long)xn * w.ny + yn, post)));
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      const int k = threadIdx.x;
      const int x = (k & 2) ? w.nx - 1 : 0, y = (k & 1) ? w.ny - 1 : 0;
      const long long c = (long long)x * w.ny + y;
      Mom2<R> t = load2<S>(w, N, c, post);
      auto from_snap = [&](int s) {
        Mom2<R> m;
        m.rho = snap[s][0]; m.ux = snap[s][1]; m.uy = snap[s][2];
        m.sxx = snap[s][3]; m.syy = snap[s][4]; m.sxy = snap[s][5]; m.drho = snap[s][6];
        return m;
      };
      // x face first (left dr 0 / right dr 2), then y face (top dr 1 / bottom dr 3)
      if (x == 0) t = bc_core<R>(w, 0, t, from_snap(y == 0 ? 0 : 2));
      else t = bc_core<R>(w, 2, t, load2<S>(w, N, (long long)(w.nx - 2) * w.ny + y, post));
      if (y == w.ny - 1) t = bc_core<R>(w, 1, t, load2<S>(w, N, (long long)x * w.ny + w.ny - 2, post));
      else t = bc_core<R>(w, 3, t, x == 0 ? from_snap(1) : from_snap(3));
      store2<S>(w, N, c, post, t);
    }
  }
  for (int s = threadIdx.x; s < w.n_objects; s += blockDim.x) {
    if (w.force_x) w.force_x[s] = float(w.loads64[3 * s]);
    if (w.force_y) w.force_y[s] = float(w.loads64[3 * s + 1]);
    if (w.torque) w.torque[s] = float(w.loads64[3 * s + 2]);
  }
}

// -------------------------------------------------------------------------- init
template <class S>
__global__ void init_uniform_kernel(long long N, typename S::T* ma, typename S::T* mb, float* fx, float* fy, float ux,
                                    float uy, Scale sc) {
  using R = typename S::R;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  // InitFlow / set_uniform_flow_kernel (lbm_func.py:26-63, karman_lbm_env.py:15-53)
  R p[9];
  const R usq = R(ux) * R(ux) + R(uy) * R(uy);
  for (int k = 0; k < 9; ++k) {
    const R wk = k == 0 ? R(4.0 / 9.0) : k < 5 ? R(1.0 / 9.0) : R(1.0 / 36.0);
    const R cu = R(cx_of(k)) * R(ux) + R(cy_of(k)) * R(uy);
    p[k] = wk * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq);
  }
  const R pixx = p[1] + p[2] + p[5] + p[6] + p[7] + p[8];
  const R piyy = p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
  const R pixy = p[5] + p[7] - p[6] - p[8];
  Mom2<R> m;
  m.rho = R(1);
  m.drho = R(0);
  m.ux = R(ux);
  m.uy = R(uy);
  m.sxx = pixx - pixx;  // cs2_local = pixx ("Very Important!!!", lbm_func.py:46)
  m.syy = piyy - pixx;
  m.sxy = pixy;
  R raw[6];
  encode2<S>(m, sc, raw);
  for (int k = 0; k < 6; ++k) {
    ma[k * N + i] = S::from_r(raw[k]);
    mb[k * N + i] = S::from_r(raw[k]);
  }
  if (fx) fx[i] = 0.f;
  if (fy) fy[i] = 0.f;
}

__global__ void init_boundary_kernel(int nx, int ny, int32_t* flag) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nx * ny) return;
  const int x = int(i / ny), y = int(i % ny);
  // InitBoundary (envs/lbm/lbm_func.py:17-23)
  if (flag[i] != 1 && flag[i] != 6 && (x == 0 || x == nx - 1 || y == 0 || y == ny - 1)) flag[i] = ML_WALL;
}

}  // namespace d2
}  // namespace hl

// ============================================================================ C ABI
using namespace hl;

namespace {

int fill_world(const hl_world2d* w, const hl_step2d* p, const hl_bc2d* bc, const hl_solids2d* s, d2::World* out) {
  HL_CHECK_ARG(w != nullptr && p != nullptr, "d2q9: world or step parameters are NULL");
  HL_CHECK_ARG(w->nx >= 3 && w->ny >= 3, "d2q9: grid must be at least 3 x 3 (got %d x %d)", w->nx, w->ny);
  HL_CHECK_ARG(w->cur && w->post && w->cur != w->post, "d2q9: cur/post must be distinct device buffers");
  HL_CHECK_ARG(p->vis_shear > 0.0, "d2q9: viscosity must be positive");
  d2::World x{};
  x.buf[0] = const_cast<void*>(w->cur);
  x.buf[1] = w->post;
  x.flag = w->flag;
  x.fx = w->forcex;
  x.fy = w->forcey;
  x.nx = w->nx;
  x.ny = w->ny;
  x.periodic = w->periodic;
  x.vis_shear = p->vis_shear;
  x.grid_length = p->grid_length > 0.f ? p->grid_length : 1.0f / float(w->nx);
  x.time_step = p->time_step > 0.f ? p->time_step : 1.0f;
  x.sc = make_scale(w->storage);
  for (int f = 0; f < 4; ++f) {
    x.bc_type[f] = bc ? bc->bc_type[f] : 1;
    x.bc_value[f][0] = bc ? bc->bc_value[f][0] : 0.f;
    x.bc_value[f][1] = bc ? bc->bc_value[f][1] : 0.f;
  }
  if (s && s->n_objects > 0) {
    HL_CHECK_ARG(s->n_objects <= d2::MAX_SOLIDS, "d2q9: at most %d solids per world", d2::MAX_SOLIDS);
    HL_CHECK_ARG(s->max_segments > 0 && s->max_segments < 65536, "d2q9: max_segments %d out of range (1..65535)",
                 s->max_segments);
    HL_CHECK_ARG(s->line && s->line_num && s->line_tf && s->line_tf_last && s->position && s->angle && s->scale &&
                     s->mass_center && s->max_radius && s->loads64 && s->band_box,
                 "d2q9: incomplete solid description");
    x.n_objects = s->n_objects;
    x.max_segments = s->max_segments;
    x.line = s->line;
    x.line_num = s->line_num;
    x.tf = s->line_tf;
    x.tf_last = s->line_tf_last;
    x.position = s->position;
    x.angle = s->angle;
    x.scale = s->scale;
    x.mass_center = s->mass_center;
    x.max_radius = s->max_radius;
    x.loads64 = s->loads64;
    x.force_x = s->force_x;
    x.force_y = s->force_y;
    x.torque = s->torque;
    x.box = s->band_box;
  }
  *out = x;
  return HL_OK;
}

// The tile shapes of the persistent stream launch (cells along x, along y).
// Shapes with 30 rows (d2::STRIP_Y) are strips: a warp per tile (stream_strips_kernel).
constexpr int TILE_SHAPES[][2] = {{8, 32}, {16, 32}, {4, 64}, {8, 64}, {16, 64}, {8, 128}, {32, 30}, {64, 30}, {128, 30}};
constexpr int N_TILE_SHAPES = int(sizeof(TILE_SHAPES) / sizeof(TILE_SHAPES[0]));

// A tile work-list for the stream phase (NULL: the gridded stream_kernel).
struct TileWork {
  const int4* tiles;
  int n_tiles, tile_x, tile_y, ctas;
};

template <class S, int TX, int TY> int launch_tiles(const d2::Launch& L, const TileWork& tw, cudaStream_t st) {
  auto kern = d2::stream_tiles_kernel<S, TX, TY>;
  const size_t smem = d2::tile_smem_bytes<TX, TY, typename S::R>();
  if (smem > 48 * 1024) {
    const int rc = set_smem_attr(reinterpret_cast<const void*>(kern), int(smem), "d2q9 tiles: shared memory size");
    if (rc != HL_OK) return rc;
  }
  const int grid = tw.n_tiles < tw.ctas ? tw.n_tiles : tw.ctas;
  kern<<<grid, d2::TILE_THREADS, smem, st>>>(L, tw.tiles, tw.n_tiles);
  HL_LAUNCH_CHECK("d2q9 stream_and_collide (tile work-list)");
  return HL_OK;
}

template <class S, int TX> int launch_strips(const d2::Launch& L, const TileWork& tw, cudaStream_t st) {
  // ctas blocks of 8 warps, a warp per strip, no more blocks than the strips fill
  const int need = (tw.n_tiles + 7) / 8;
  const int grid = need < tw.ctas ? need : tw.ctas;
  d2::stream_strips_kernel<S, TX><<<grid, 256, 0, st>>>(L, tw.tiles, tw.n_tiles);
  HL_LAUNCH_CHECK("d2q9 stream_and_collide (strip work-list)");
  return HL_OK;
}

template <class S> int stream_tiles(const d2::Launch& L, const TileWork& tw, cudaStream_t st) {
  if (tw.n_tiles == 0) return HL_OK;
  const int x = tw.tile_x, y = tw.tile_y;
  if (y == d2::STRIP_Y) {
    if (x == 32) return launch_strips<S, 32>(L, tw, st);
    if (x == 64) return launch_strips<S, 64>(L, tw, st);
    if (x == 128) return launch_strips<S, 128>(L, tw, st);
  }
  if (x == 8 && y == 32) return launch_tiles<S, 8, 32>(L, tw, st);
  if (x == 16 && y == 32) return launch_tiles<S, 16, 32>(L, tw, st);
  if (x == 4 && y == 64) return launch_tiles<S, 4, 64>(L, tw, st);
  if (x == 8 && y == 64) return launch_tiles<S, 8, 64>(L, tw, st);
  if (x == 16 && y == 64) return launch_tiles<S, 16, 64>(L, tw, st);
  if (x == 8 && y == 128) return launch_tiles<S, 8, 128>(L, tw, st);
  set_error("d2q9 tiles: unsupported tile shape %d x %d", x, y);
  return HL_ERR_ARG;
}

template <class S> int run_phases(const d2::Launch& L, int n, int maxx, int maxy, bool any_solid, int phases,
                                  cudaStream_t st, const TileWork* tw = nullptr) {
  if ((phases & HL_PHASE_SEGMENTS) && any_solid) {
    d2::prologue_kernel<<<n, 256, 0, st>>>(L);
    HL_LAUNCH_CHECK("d2q9 precompute_transformed_segments");
  }
  if (phases & HL_PHASE_STREAM) {
    if (tw) {
      const int rc = stream_tiles<S>(L, *tw, st);
      if (rc != HL_OK) return rc;
    } else {
      dim3 grid((maxy + 31) / 32, (maxx + 7) / 8, n);
      d2::stream_kernel<S><<<grid, 256, 0, st>>>(L);
      HL_LAUNCH_CHECK("d2q9 stream_and_collide");
    }
    if (any_solid) {
      d2::band_kernel<S><<<dim3(64, n), 256, 0, st>>>(L);
      HL_LAUNCH_CHECK("d2q9 cut-cell band");
    }
  }
  if (phases & HL_PHASE_BC) {
    d2::boundary_kernel<S><<<n, 512, 0, st>>>(L);
    HL_LAUNCH_CHECK("d2q9 apply_bc");
  }
  return HL_OK;
}

int dispatch(hl_dtype dt, const d2::Launch& L, int n, int maxx, int maxy, bool any_solid, int phases, cudaStream_t st,
             const TileWork* tw = nullptr) {
  switch (dt) {
    case HL_F32: return run_phases<StoreF32>(L, n, maxx, maxy, any_solid, phases, st, tw);
    case HL_F64: return run_phases<StoreF64>(L, n, maxx, maxy, any_solid, phases, st, tw);
    case HL_F16: return run_phases<StoreF16>(L, n, maxx, maxy, any_solid, phases, st, tw);
    case HL_BF16: return run_phases<StoreBF16>(L, n, maxx, maxy, any_solid, phases, st, tw);
  }
  set_error("d2q9: bad dtype");
  return HL_ERR_ARG;
}

}  // namespace

extern "C" int hl_d2q9_step_phases(const hl_world2d* w, const hl_step2d* p, const hl_bc2d* bc,
                                   const hl_solids2d* solids, int phases, hl_stream stream) {
  d2::Launch L{};
  const int rc = fill_world(w, p, bc, solids, &L.one);
  if (rc != HL_OK) return rc;
  L.many = nullptr;
  L.parity = 0;
  return dispatch(w->storage.dtype, L, 1, w->nx, w->ny, L.one.n_objects > 0, phases, static_cast<cudaStream_t>(stream));
}

extern "C" int hl_d2q9_step(const hl_world2d* w, const hl_step2d* p, const hl_bc2d* bc, const hl_solids2d* solids,
                            hl_stream stream) {
  return hl_d2q9_step_phases(w, p, bc, solids, HL_PHASE_ALL, stream);
}

extern "C" size_t hl_d2q9_desc_bytes(void) { return sizeof(d2::World); }

extern "C" int hl_d2q9_pack(const hl_world2d* w, const hl_step2d* p, const hl_bc2d* bc, const hl_solids2d* solids,
                            void* desc_host) {
  HL_CHECK_ARG(desc_host != nullptr, "d2q9: descriptor buffer is NULL");
  return fill_world(w, p, bc, solids, static_cast<d2::World*>(desc_host));
}

extern "C" int hl_d2q9_step_batch(const void* desc_dev, int n_worlds, int parity, hl_dtype dtype, int max_nx,
                                  int max_ny, int any_solid, int phases, hl_stream stream) {
  HL_CHECK_ARG(desc_dev != nullptr && n_worlds > 0 && max_nx > 0 && max_ny > 0, "d2q9: bad batch arguments");
  HL_CHECK_ARG(parity == 0 || parity == 1, "d2q9: parity must be 0 or 1");
  d2::Launch L{};
  L.many = static_cast<const d2::World*>(desc_dev);
  L.parity = parity;
  return dispatch(dtype, L, n_worlds, max_nx, max_ny, any_solid != 0, phases, static_cast<cudaStream_t>(stream));
}

extern "C" int hl_d2q9_tile_shapes(int32_t* out, int cap) {
  for (int k = 0; k < N_TILE_SHAPES && k < cap && out; ++k) {
    out[2 * k] = TILE_SHAPES[k][0];
    out[2 * k + 1] = TILE_SHAPES[k][1];
  }
  return N_TILE_SHAPES;
}

extern "C" int hl_d2q9_tile_list(const int32_t* nx, const int32_t* ny, int n_worlds, int tile_x, int tile_y,
                                 int32_t* out, size_t cap_tiles, size_t* n_tiles) {
  HL_CHECK_ARG(nx != nullptr && ny != nullptr && n_tiles != nullptr && n_worlds > 0, "d2q9 tiles: bad arguments");
  bool shape_ok = false;
  for (int k = 0; k < N_TILE_SHAPES; ++k) shape_ok |= TILE_SHAPES[k][0] == tile_x && TILE_SHAPES[k][1] == tile_y;
  HL_CHECK_ARG(shape_ok, "d2q9 tiles: unsupported tile shape %d x %d", tile_x, tile_y);
  size_t count = 0;
  for (int w = 0; w < n_worlds; ++w) {
    HL_CHECK_ARG(nx[w] >= 3 && ny[w] >= 3 && nx[w] < (1 << 30) && ny[w] < (1 << 30), "d2q9 tiles: world %d is %d x %d",
                 w, nx[w], ny[w]);
    for (int x0 = 0; x0 < nx[w]; x0 += tile_x)
      for (int y0 = 0; y0 < ny[w]; y0 += tile_y) {
        if (out != nullptr && count < cap_tiles) {
          out[4 * count] = w;
          out[4 * count + 1] = x0;
          out[4 * count + 2] = y0;
          out[4 * count + 3] = 0;
        }
        ++count;
      }
  }
  *n_tiles = count;
  HL_CHECK_ARG(out == nullptr || count <= cap_tiles, "d2q9 tiles: %zu tiles do not fit in %zu", count, cap_tiles);
  return HL_OK;
}

extern "C" int hl_d2q9_step_tiles(const void* desc_dev, int n_worlds, int parity, hl_dtype dtype,
                                  const int32_t* tiles_dev, int n_tiles, int tile_x, int tile_y, int ctas,
                                  int any_solid, int phases, hl_stream stream) {
  HL_CHECK_ARG(desc_dev != nullptr && n_worlds > 0, "d2q9: bad batch arguments");
  HL_CHECK_ARG(parity == 0 || parity == 1, "d2q9: parity must be 0 or 1");
  HL_CHECK_ARG(n_tiles >= 0 && (n_tiles == 0 || tiles_dev != nullptr), "d2q9 tiles: tile list is NULL");
  HL_CHECK_ARG(reinterpret_cast<uintptr_t>(tiles_dev) % 16 == 0, "d2q9 tiles: tile list must be 16-byte aligned");
  HL_CHECK_ARG(ctas >= 1, "d2q9 tiles: grid must have at least one CTA");
  d2::Launch L{};
  L.many = static_cast<const d2::World*>(desc_dev);
  L.parity = parity;
  const TileWork tw{reinterpret_cast<const int4*>(tiles_dev), n_tiles, tile_x, tile_y, ctas};
  return dispatch(dtype, L, n_worlds, 1, 1, any_solid != 0, phases, static_cast<cudaStream_t>(stream), &tw);
}

template <class S>
static int init_uniform_2d_t(int nx, int ny, hl_storage sto, void* a, void* b, float* fx, float* fy, float ux, float uy,
                             cudaStream_t st) {
  const long long N = (long long)nx * ny;
  d2::init_uniform_kernel<S><<<unsigned((N + 255) / 256), 256, 0, st>>>(
      N, static_cast<typename S::T*>(a), static_cast<typename S::T*>(b), fx, fy, ux, uy, make_scale(sto));
  HL_LAUNCH_CHECK("d2q9 init_uniform");
  return HL_OK;
}

extern "C" int hl_d2q9_init_uniform(int nx, int ny, hl_storage sto, void* a, void* b, float* fx, float* fy, float ux,
                                    float uy, hl_stream stream) {
  HL_CHECK_ARG(nx > 0 && ny > 0 && a && b, "init_uniform_2d: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (sto.dtype) {
    case HL_F32: return init_uniform_2d_t<StoreF32>(nx, ny, sto, a, b, fx, fy, ux, uy, st);
    case HL_F64: return init_uniform_2d_t<StoreF64>(nx, ny, sto, a, b, fx, fy, ux, uy, st);
    case HL_F16: return init_uniform_2d_t<StoreF16>(nx, ny, sto, a, b, fx, fy, ux, uy, st);
    case HL_BF16: return init_uniform_2d_t<StoreBF16>(nx, ny, sto, a, b, fx, fy, ux, uy, st);
  }
  set_error("init_uniform_2d: bad dtype");
  return HL_ERR_ARG;
}

extern "C" int hl_d2q9_init_boundary(int nx, int ny, int32_t* flag, hl_stream stream) {
  HL_CHECK_ARG(nx > 0 && ny > 0 && flag, "init_boundary_2d: bad arguments");
  const long long N = (long long)nx * ny;
  d2::init_boundary_kernel<<<unsigned((N + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(nx, ny, flag);
  HL_LAUNCH_CHECK("d2q9 init_boundary");
  return HL_OK;
}
