// CPU restatement of the HOME-LBM stream-collide path of kuiwuchn/OpenHOMELBM.
//
// TEST INFRASTRUCTURE ONLY. This is the correctness (float) and accuracy (double) oracle
// for the CUDA kernels of openhomelbm_b200. Only tests, the smoke check and bench.py's CPU
// baseline may load it; the product library never does.
//
// Parity status: pinned. tests/golden/*.npz hold the outputs of the reference's own Warp
// kernel source executed by tests/golden/warp_emu.py (Warp's CPU launch order, binary32,
// no FMA); tests/test_oracle_golden.py requires this file's float build to reproduce them
// bit for bit. Two pieces have no source in the reference tree (they are Warp native code)
// and are restated from their mathematical definitions identically here and in the
// emulator: the quaternion rotation behind wp.transform_* and wp.mesh_query_ray
// (brute-force double-sided Moller-Trumbore, closest hit with 0 <= t <= max_t).
//
// Every function follows one reference function statement by statement, in the same
// evaluation order, so that the float instantiation rounds exactly as binary32 Warp code
// on the CPU does. Build with -ffp-contract=off (no fused multiply-add).
//
// Layout (shared with the CUDA library): moments are SoA planes, one allocation of
// nmom x N values, N = nx*ny (2D, y fastest) or nx*ny*nz (3D, z fastest), plane order
//   2D: rho, ux, uy, Sxx, Syy, Sxy
//   3D: rho, ux, uy, uz, Sxx, Syy, Szz, Sxy, Sxz, Syz
// which is the reference's (nx, ny[, nz]) C-order per field.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr int ML_FLUID = 0;
constexpr int ML_SOLID = 1;
constexpr int ML_WALL = 2;
constexpr int ML_INVALID = 6;

// ---------------------------------------------------------------- D2Q9 tables
// envs/lbm/lbm_core.py:127-130
const double W2[9] = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
const int CX2[9] = {0, 1, -1, 0, 0, 1, -1, -1, 1};
const int CY2[9] = {0, 0, 0, 1, -1, 1, 1, -1, -1};
const int INV2[9] = {0, 2, 1, 4, 3, 7, 8, 5, 6};

// ---------------------------------------------------------------- D3Q27 tables
// envs/lbm3d/lbm_core_3d.py:12-35
const int CX3[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
const int CY3[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
const int CZ3[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
const int INV3[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};
double w3d(int i) {
  if (i == 0) return 8.0 / 27.0;
  if (i <= 6) return 2.0 / 27.0;
  if (i <= 18) return 1.0 / 54.0;
  return 1.0 / 216.0;
}

template <class T> struct V2 { T x, y; };
template <class T> struct V3 { T x, y, z; };

// cs2 of envs/lbm/lbm_func.py:4 (a binary32 rounding of a double sum) and
// envs/lbm3d/lbm_core_3d.py:37.
template <class T> T cs2_2d() { return T(1.0 / 9 + 1.0 / 9 + 1.0 / 36 + 1.0 / 36 + 1.0 / 36 + 1.0 / 36); }
template <class T> T cs2_3d() { return T(1.0 / 3.0); }

// ============================================================================ 2D
template <class T> struct Solids2 {
  int n_objects, max_segments;
  const T* line;          // [n][max_seg][2] local polygon
  const int* line_num;    // [n]
  T* tf;                  // [n][max_seg][2] solid_line_transformed
  T* tf_last;             // [n][max_seg][2] solid_line_transformed_last
  const T* position;      // [n][2]
  const T* angle;         // [n]
  const T* scale;         // [n]
  const T* mass_center;   // [n][2]
  const T* max_radius;    // [n]
  T* loads;               // [n][3] solid_forcex, solid_forcey, torque
};

template <class T> struct Params2 {
  int nx, ny;
  T vis_shear, grid_length, time_step;
  const int* bc_type;   // [4] left, top, right, bottom
  const T* bc_value;    // [4][2]
  int periodic;
};

// mlCalDistribution, envs/lbm/lbm_func.py:685-788
template <class T>
T ml_cal_distribution(T rhoVar, T ux, T uy, T Sxx, T Syy, T Sxy, int i) {
  const T Axxy = Sxx * uy + T(2.0) * Sxy * ux - T(2.0) * ux * ux * uy;
  const T Axyy = Syy * ux + T(2.0) * Sxy * uy - T(2.0) * ux * uy * uy;
  const T n9 = T(1.0 / 9.0), n36 = T(1.0 / 36.0), h = T(0.5 * 3.0);
  switch (i) {
    case 0: return T(4.0 / 9.0) * rhoVar * (T(1.0) - h * Sxx - h * Syy);
    case 1: return n9 * rhoVar * (T(1.0) + T(3.0) * ux + T(3.0) * Sxx - h * Syy - T(4.5) * Axyy);
    case 2: return n9 * rhoVar * (T(1.0) - T(3.0) * ux + T(3.0) * Sxx - h * Syy + T(4.5) * Axyy);
    case 3: return n9 * rhoVar * (T(1.0) + T(3.0) * uy - h * Sxx + T(3.0) * Syy - T(4.5) * Axxy);
    case 4: return n9 * rhoVar * (T(1.0) - T(3.0) * uy - h * Sxx + T(3.0) * Syy + T(4.5) * Axxy);
    case 5:
      return n36 * rhoVar *
             (T(1.0) + T(3.0) * (ux + uy) + T(3.0) * (Sxx + Syy + T(3.0) * Sxy) + T(9.0) * (Axyy + Axxy));
    case 6:
      return n36 * rhoVar *
             (T(1.0) - T(3.0) * ux + T(3.0) * uy + T(3.0) * (Sxx + Syy - T(3.0) * Sxy) + T(9.0) * (Axxy - Axyy));
    case 7:
      return n36 * rhoVar *
             (T(1.0) - T(3.0) * ux - T(3.0) * uy + T(3.0) * (Sxx + Syy + T(3.0) * Sxy) - T(9.0) * (Axxy + Axyy));
    default:
      return n36 * rhoVar *
             (T(1.0) + T(3.0) * ux - T(3.0) * uy + T(3.0) * (Sxx + Syy - T(3.0) * Sxy) - T(9.0) * (Axxy - Axyy));
  }
}

template <class T> struct Cut2 { T t; int solid; T ratio; int seg; };

// get_cutcell, envs/lbm/lbm_func.py:545-607
template <class T>
Cut2<T> get_cutcell(const Params2<T>& p, const Solids2<T>& s, T x, T y, T dx, T dy) {
  Cut2<T> r{T(-1.0), -1, T(-1.0), -1};
  const V2<T> a{x - dx, y - dy};
  const V2<T> b{x, y};
  for (int sid = 0; sid < s.n_objects; ++sid) {
    const T px = x - s.position[2 * sid], py = y - s.position[2 * sid + 1];
    const T dist_sq = px * px + py * py;
    const T scale = s.scale[sid] * T(p.nx);
    const T rmax_sq = s.max_radius[sid] * scale * scale;
    if (dist_sq > rmax_sq) continue;
    const int nseg = s.line_num[sid];
    for (int n = 0; n < nseg; ++n) {
      const T* c = s.tf + (size_t(sid) * s.max_segments + n) * 2;
      const T* d = s.tf + (size_t(sid) * s.max_segments + (n + 1) % nseg) * 2;
      const T area_abc = (a.x - c[0]) * (b.y - c[1]) - (a.y - c[1]) * (b.x - c[0]);
      const T area_abd = (a.x - d[0]) * (b.y - d[1]) - (a.y - d[1]) * (b.x - d[0]);
      if (area_abc * area_abd >= T(0.0)) continue;
      const T area_cda = (c[0] - a.x) * (d[1] - a.y) - (c[1] - a.y) * (d[0] - a.x);
      const T area_cdb = area_cda + area_abc - area_abd;
      if (area_cda * area_cdb > T(0.0)) continue;
      const T t = T(1.0) - area_cda / (area_abd - area_abc);
      if (r.t < T(0.0) || t < r.t) {
        r.t = t;
        r.solid = sid;
        r.ratio = area_abc / (area_abc - area_abd);
        r.seg = n;
      }
    }
  }
  return r;
}

// precompute_transformed_segments, envs/lbm/lbm_func.py:509-542
template <class T> void precompute_segments(const Params2<T>& p, Solids2<T>& s) {
  for (int sid = 0; sid < s.n_objects; ++sid) {
    for (int idx = 0; idx < s.max_segments; ++idx) {
      if (idx >= s.line_num[sid]) continue;
      const T scale = s.scale[sid] * T(p.nx);
      const T ca = T(std::cos(double(s.angle[sid])));
      const T sa = T(std::sin(double(s.angle[sid])));
      const size_t k = (size_t(sid) * s.max_segments + idx) * 2;
      const T ppx = (s.line[k] - s.mass_center[2 * sid]) * scale;
      const T ppy = (s.line[k + 1] - s.mass_center[2 * sid + 1]) * scale;
      const T nx_ = ppx * ca - ppy * sa + s.position[2 * sid];
      const T ny_ = ppx * sa + ppy * ca + s.position[2 * sid + 1];
      const T ox = s.tf[k], oy = s.tf[k + 1];
      if (ox == T(0.0) && oy == T(0.0)) {
        s.tf_last[k] = nx_;
        s.tf_last[k + 1] = ny_;
      } else {
        s.tf_last[k] = ox;
        s.tf_last[k + 1] = oy;
      }
      s.tf[k] = nx_;
      s.tf[k + 1] = ny_;
    }
  }
}

// stream_and_collide, envs/lbm/lbm_func.py:322-467, for the cells of x-rows [x0, x1).
template <class T>
void stream_collide_2d_rows(const Params2<T>& p, const Solids2<T>& s, const T* cur, T* post, const int* flag,
                            const T* forcex, const T* forcey, int x0, int x1, T* loads) {
  const int nx = p.nx, ny = p.ny;
  const size_t N = size_t(nx) * ny;
  const T* rho = cur;
  const T* uxf = cur + N;
  const T* uyf = cur + 2 * N;
  const T* sxx = cur + 3 * N;
  const T* syy = cur + 4 * N;
  const T* sxy = cur + 5 * N;
  const T cs2 = cs2_2d<T>();
  for (int x = x0; x < x1; ++x)
    for (int y = 0; y < ny; ++y) {
      const size_t c = size_t(x) * ny + y;
      const int fl = flag ? flag[c] : ML_FLUID;
      if (fl != ML_FLUID) continue;
      T pop[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      const T rho_c = rho[c], ux_c = uxf[c], uy_c = uyf[c], Sxx_c = sxx[c], Syy_c = syy[c], Sxy_c = sxy[c];
      for (int i = 0; i < 9; ++i) {
        const T dx = T(CX2[i]), dy = T(CY2[i]);
        int x1n = x - CX2[i], y1n = y - CY2[i];
        if (p.periodic) {
          x1n = (x1n + nx) % nx;
          y1n = (y1n + ny) % ny;
        }
        if (!(x1n >= 0 && x1n < nx && y1n >= 0 && y1n < ny)) continue;
        Cut2<T> cc{T(-1.0), -1, T(-1.0), -1};
        if (s.n_objects > 0) cc = get_cutcell(p, s, T(x), T(y), dx, dy);
        if (cc.t >= T(0.0) && cc.solid >= 0) {
          const int sid = cc.solid, seg = cc.seg, nseg = s.line_num[sid];
          const T* cC = s.tf + (size_t(sid) * s.max_segments + seg) * 2;
          const T* dC = s.tf + (size_t(sid) * s.max_segments + (seg + 1) % nseg) * 2;
          const T pcx = cC[0] + (dC[0] - cC[0]) * cc.ratio;
          const T pcy = cC[1] + (dC[1] - cC[1]) * cc.ratio;
          const T* cL = s.tf_last + (size_t(sid) * s.max_segments + seg) * 2;
          const T* dL = s.tf_last + (size_t(sid) * s.max_segments + (seg + 1) % nseg) * 2;
          const T plx = cL[0] + (dL[0] - cL[0]) * cc.ratio;
          const T ply = cL[1] + (dL[1] - cL[1]) * cc.ratio;
          const T upx = (pcx - plx) / p.time_step;
          const T upy = (pcy - ply) / p.time_step;
          const T rx = pcx - s.position[2 * sid];
          const T ry = pcy - s.position[2 * sid + 1];
          const T Sxx_s = upx * upx + Sxx_c - ux_c * ux_c;
          const T Syy_s = upy * upy + Syy_c - uy_c * uy_c;
          const T Sxy_s = upx * upy + Sxy_c - ux_c * uy_c;
          pop[i] = ml_cal_distribution<T>(rho_c, upx, upy, Sxx_s, Syy_s, Sxy_s, i);
          if (pop[i] < T(0.0)) pop[i] = T(0.0);
          const int ii = INV2[i];
          const T cur_f = ml_cal_distribution<T>(rho_c, ux_c, uy_c, Sxx_c, Syy_c, Sxy_c, ii);
          const T fx = cur_f * (T(CX2[ii]) - upx) - pop[i] * (T(CX2[i]) - upx);
          const T fy = cur_f * (T(CY2[ii]) - upy) - pop[i] * (T(CY2[i]) - upy);
          const T tq = (rx * fy - ry * fx) * p.grid_length;
          loads[3 * sid] += fx;
          loads[3 * sid + 1] += fy;
          loads[3 * sid + 2] += tq;
        } else {
          const size_t n = size_t(x1n) * ny + y1n;
          pop[i] = ml_cal_distribution<T>(rho[n], uxf[n], uyf[n], sxx[n], syy[n], sxy[n], i);
          if (pop[i] < T(0.0)) pop[i] = T(0.0);
        }
      }
      const T Fx = forcex ? forcex[c] : T(0.0);
      const T Fy = forcey ? forcey[c] : T(0.0);
      const T rhoVar = pop[0] + pop[1] + pop[2] + pop[3] + pop[4] + pop[5] + pop[6] + pop[7] + pop[8];
      const T invRho = T(1.0) / rhoVar;
      const T ux = (pop[1] - pop[2] + pop[5] - pop[6] - pop[7] + pop[8] + T(0.5) * Fx) * invRho;
      const T uy = (pop[3] - pop[4] + pop[5] + pop[6] - pop[7] - pop[8] + T(0.5) * Fy) * invRho;
      T pixx = pop[1] + pop[2] + pop[5] + pop[6] + pop[7] + pop[8];
      T piyy = pop[3] + pop[4] + pop[5] + pop[6] + pop[7] + pop[8];
      T pixy = pop[5] + pop[7] - pop[6] - pop[8];
      const T Omega = T(1.0) / (p.vis_shear * T(3.0) + T(0.5));
      const T Ru2 = rhoVar * ux * ux;
      const T Rv2 = rhoVar * uy * uy;
      const T pixx_part = (pixx - piyy) / T(2.0);
      const T piyy_part = (piyy - pixx) / T(2.0);
      pixy = (T(1.0) - Omega) * pixy + ux * uy * rhoVar * Omega + (T(1.0) - T(0.5) * Omega) * (Fy * ux + Fx * uy);
      pixx = rhoVar / T(3.0) + pixx_part * (T(1.0) - Omega) + (T(1.0) + Omega) / T(2.0) * Ru2 +
             (T(1.0) - Omega) / T(2.0) * Rv2 + Fx * ux + (T(1.0) - Omega) / T(2.0) * (Fx * ux - Fy * uy);
      piyy = rhoVar / T(3.0) + piyy_part * (T(1.0) - Omega) + (T(1.0) + Omega) / T(2.0) * Rv2 +
             (T(1.0) - Omega) / T(2.0) * Ru2 + Fy * uy + (T(1.0) - Omega) / T(2.0) * (Fy * uy - Fx * ux);
      post[c] = rhoVar;
      post[N + c] = ux + Fx * invRho / T(2.0);
      post[2 * N + c] = uy + Fy * invRho / T(2.0);
      post[3 * N + c] = pixx * invRho - cs2;
      post[4 * N + c] = piyy * invRho - cs2;
      post[5 * N + c] = pixy * invRho;
    }
}

// f_eq_home, envs/lbm/lbm_func.py:660-682
template <class T> void f_eq_home_2d(const T* post, size_t N, size_t c, T out[3]) {
  T pop[9];
  const T rho = post[c], ux = post[N + c], uy = post[2 * N + c];
  const T U_sqr = ux * ux + uy * uy;
  for (int i = 0; i < 9; ++i) {
    const T cu = T(CX2[i]) * ux + T(CY2[i]) * uy;
    pop[i] = rho * T(W2[i]) * (T(1.0) + T(3.0) * cu + T(4.5) * cu * cu - T(1.5) * U_sqr);
    if (pop[i] < T(0.0)) pop[i] = T(0.0);
  }
  const T invRho = T(1.0) / rho;
  T pixx = pop[1] + pop[2] + pop[5] + pop[6] + pop[7] + pop[8];
  T piyy = pop[3] + pop[4] + pop[5] + pop[6] + pop[7] + pop[8];
  T pixy = pop[5] + pop[7] - pop[6] - pop[8];
  out[0] = pixx * invRho - cs2_2d<T>();
  out[1] = piyy * invRho - cs2_2d<T>();
  out[2] = pixy * invRho;
}

// apply_bc_core, envs/lbm/lbm_func.py:634-657
template <class T>
void apply_bc_core_2d(const Params2<T>& p, T* post, int dr, int ibc, int jbc, int inb, int jnb) {
  const size_t N = size_t(p.nx) * p.ny;
  const size_t b = size_t(ibc) * p.ny + jbc, n = size_t(inb) * p.ny + jnb;
  if (p.bc_type[dr] == 0) {
    post[N + b] = p.bc_value[2 * dr];
    post[2 * N + b] = p.bc_value[2 * dr + 1];
  } else if (p.bc_type[dr] == 1) {
    post[N + b] = post[N + n];
    post[2 * N + b] = post[2 * N + n];
  }
  post[b] = post[n];
  T cur[3], back[3];
  f_eq_home_2d(post, N, b, cur);
  f_eq_home_2d(post, N, n, back);
  post[3 * N + b] = cur[0] - back[0] + post[3 * N + n];
  post[4 * N + b] = cur[1] - back[1] + post[4 * N + n];
  post[5 * N + b] = cur[2] - back[2] + post[5 * N + n];
}

// apply_bc, envs/lbm/lbm_func.py:610-631, threads run in launch order (x outer, y inner)
template <class T> void apply_bc_2d(const Params2<T>& p, T* post) {
  const int nx = p.nx, ny = p.ny;
  for (int x = 0; x < nx; ++x) {
    const bool xb = (x == 0 || x == nx - 1);
    for (int y = 0; y < ny; ++y) {
      if (!xb && y != 0 && y != ny - 1) continue;
      if (x == 0) apply_bc_core_2d(p, post, 0, 0, y, 1, y);
      else if (x == nx - 1) apply_bc_core_2d(p, post, 2, nx - 1, y, nx - 2, y);
      if (y == ny - 1) apply_bc_core_2d(p, post, 1, x, ny - 1, x, ny - 2);
      else if (y == 0) apply_bc_core_2d(p, post, 3, x, 0, x, 1);
    }
  }
}

int num_threads(int requested) {
  if (requested > 0) return requested;
  const unsigned hw = std::thread::hardware_concurrency();
  return hw ? int(hw) : 1;
}

// Runs fn(t, n) on n host threads (t = 0..n-1) and joins them.
template <class F> void parallel_for_threads(int n, F fn) {
  std::vector<std::thread> pool;
  for (int t = 1; t < n; ++t) pool.emplace_back(fn, t, n);
  fn(0, n);
  for (auto& th : pool) th.join();
}

// LBM_Solver.step, envs/lbm/lbm_solver.py:104-141 (zero loads, segments, stream-collide,
// apply_bc). The caller swaps cur/post afterwards (Swap_Mom).
template <class T>
void step_2d(const Params2<T>& p, Solids2<T>& s, const T* cur, T* post, const int* flag, const T* fx, const T* fy,
             int nthreads) {
  for (int i = 0; i < 3 * s.n_objects; ++i) s.loads[i] = T(0.0);
  if (s.n_objects > 0) precompute_segments(p, s);
  const int nt = num_threads(nthreads);
  if (nt <= 1) {
    stream_collide_2d_rows(p, s, cur, post, flag, fx, fy, 0, p.nx, s.loads);
  } else {
    std::vector<T> part(size_t(nt) * 3 * s.n_objects + 1, T(0.0));
    parallel_for_threads(nt, [&](int t, int n) {
      const int x0 = int(int64_t(p.nx) * t / n), x1 = int(int64_t(p.nx) * (t + 1) / n);
      stream_collide_2d_rows(p, s, cur, post, flag, fx, fy, x0, x1, part.data() + size_t(t) * 3 * s.n_objects);
    });
    for (int t = 0; t < nt; ++t)
      for (int i = 0; i < 3 * s.n_objects; ++i) s.loads[i] += part[size_t(t) * 3 * s.n_objects + i];
  }
  if (!p.periodic) apply_bc_2d(p, post);
}

// ============================================================================ 3D
template <class T> struct Quat { T x, y, z, w; };
template <class T> struct Xform { V3<T> p; Quat<T> q; };

// Rotation of v by unit quaternion q: v(2w^2-1) + 2w (q_v x v) + 2 (q_v . v) q_v.
// Restated from its definition (wp.quat_rotate is Warp native code); the golden emulator
// uses the same expression.
template <class T> V3<T> qrot(const Quat<T>& q, const V3<T>& v) {
  const T c = T(2.0) * q.w * q.w - T(1.0);
  const T d = T(2.0) * (q.x * v.x + q.y * v.y + q.z * v.z);
  const T cx = q.y * v.z - q.z * v.y, cy = q.z * v.x - q.x * v.z, cz = q.x * v.y - q.y * v.x;
  const T e = T(2.0) * q.w;
  return {v.x * c + cx * e + q.x * d, v.y * c + cy * e + q.y * d, v.z * c + cz * e + q.z * d};
}
template <class T> Xform<T> xinv(const Xform<T>& t) {
  Quat<T> qi{-t.q.x, -t.q.y, -t.q.z, t.q.w};
  V3<T> p = qrot(qi, t.p);
  return {{-p.x, -p.y, -p.z}, qi};
}
template <class T> V3<T> xpoint(const Xform<T>& t, const V3<T>& v) {
  V3<T> r = qrot(t.q, v);
  return {r.x + t.p.x, r.y + t.p.y, r.z + t.p.z};
}
template <class T> V3<T> xvec(const Xform<T>& t, const V3<T>& v) { return qrot(t.q, v); }
template <class T> Xform<T> load_xform(const T* a) { return {{a[0], a[1], a[2]}, {a[3], a[4], a[5], a[6]}}; }
template <class T> T vlen(const V3<T>& v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

// Closest double-sided Moller-Trumbore hit with 0 <= t <= max_t over all triangles.
template <class T> bool ray_mesh(const T* tri, int ntri, const V3<T>& o, const V3<T>& d, T max_t, T* t_out) {
  bool hit = false;
  T best = T(0.0);
  for (int k = 0; k < ntri; ++k) {
    const T* v0 = tri + 9 * k;
    const T* v1 = v0 + 3;
    const T* v2 = v0 + 6;
    const T e1x = v1[0] - v0[0], e1y = v1[1] - v0[1], e1z = v1[2] - v0[2];
    const T e2x = v2[0] - v0[0], e2y = v2[1] - v0[1], e2z = v2[2] - v0[2];
    const T px = d.y * e2z - d.z * e2y, py = d.z * e2x - d.x * e2z, pz = d.x * e2y - d.y * e2x;
    const T det = e1x * px + e1y * py + e1z * pz;
    if (det == T(0.0)) continue;
    const T inv = T(1.0) / det;
    const T sx = o.x - v0[0], sy = o.y - v0[1], sz = o.z - v0[2];
    const T u = (sx * px + sy * py + sz * pz) * inv;
    if (u < T(0.0) || u > T(1.0)) continue;
    const T qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
    const T v = (d.x * qx + d.y * qy + d.z * qz) * inv;
    if (v < T(0.0) || u + v > T(1.0)) continue;
    const T t = (e2x * qx + e2y * qy + e2z * qz) * inv;
    if (t < T(0.0) || t > max_t) continue;
    if (!hit || t < best) {
      best = t;
      hit = true;
    }
  }
  *t_out = best;
  return hit;
}

template <class T> struct Solids3 {
  int n_objects;
  const int* tri_offset;    // [n+1]; a solid with no triangles is an empty mesh id (skipped)
  const T* tris;            // [total][3][3] body-local, already scaled by lbm_scale*nx
  const T* transforms;      // [n][7] p, q(xyzw)
  const T* transforms_last; // [n][7]
  const int* initialized;   // [n]
  const T* scale_sizes;     // [n][3]
  const T* position;        // [n][3]
  const T* bound_radius;    // [n]
  const T* linear_v;        // [n][3]
  const T* angle_v;         // [n][3]
  T* loads;                 // [n][6] force xyz, torque xyz
};

template <class T> struct Params3 {
  int nx, ny, nz;
  T vis_shear;
  const int* bc_type;   // [6] left, right, top, bottom, front, back
  const T* bc_value;    // [6][3]
  int periodic;
};

// mlCalEquilibrium3D_s, envs/lbm3d/lbm_func_3d.py:224-251
template <class T>
T feq3(T rhoVar, T ux, T uy, T uz, T Sxx, T Sxy, T Sxz, T Syy, T Syz, T Szz, T dx, T dy, T dz, T wi) {
  const T cu = dx * ux + dy * uy + dz * uz;
  const T U_sqr = ux * ux + uy * uy + uz * uz;
  const T third = T(1.0 / 3.0);
  const T Qxx = dx * dx - third, Qyy = dy * dy - third, Qzz = dz * dz - third;
  const T Qxy = dx * dy, Qxz = dx * dz, Qyz = dy * dz;
  const T f_neq = T(1.5) * (Qxx * Sxx + Qyy * Syy + Qzz * Szz + T(2.0) * (Qxy * Sxy + Qxz * Sxz + Qyz * Syz));
  return wi * rhoVar * (T(1.0) + T(3.0) * cu + T(4.5) * cu * cu - T(1.5) * U_sqr + f_neq);
}

// get_cutcell_multi_3d, envs/lbm3d/lbm_func_3d.py:254-316
template <class T> void get_cutcell_3d(const Solids3<T>& s, const V3<T>& o, const V3<T>& d, T* cut, int* solid) {
  *cut = T(-1.0);
  *solid = -1;
  for (int sid = 0; sid < s.n_objects; ++sid) {
    const int ntri = s.tri_offset[sid + 1] - s.tri_offset[sid];
    if (ntri == 0) continue;
    const V3<T> rel{o.x - s.position[3 * sid], o.y - s.position[3 * sid + 1], o.z - s.position[3 * sid + 2]};
    if (vlen(rel) > s.bound_radius[sid] + T(2.0)) continue;
    const Xform<T> inv = xinv(load_xform(s.transforms + 7 * sid));
    const V3<T> lo = xpoint(inv, o);
    const V3<T> ld = xvec(inv, d);
    const T* sc = s.scale_sizes + 3 * sid;
    const V3<T> los{lo.x / sc[0], lo.y / sc[1], lo.z / sc[2]};
    const V3<T> lds{ld.x / sc[0], ld.y / sc[1], ld.z / sc[2]};
    T t;
    if (ray_mesh(s.tris + size_t(9) * s.tri_offset[sid], ntri, los, lds, T(2.0), &t)) {
      if ((*cut < T(0.0) || t < *cut) && t >= T(0.0) && t <= T(1.0)) {
        *cut = t;
        *solid = sid;
      }
    }
  }
}

// stream_and_collide_3d, envs/lbm3d/lbm_func_3d.py:364-604, for x-planes [x0, x1).
template <class T>
void stream_collide_3d_rows(const Params3<T>& p, const Solids3<T>& s, const T* cur, T* post, const int* flag,
                            const T* force, int64_t r0, int64_t r1, T* loads) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const size_t N = size_t(nx) * ny * nz;
  const T cs2 = cs2_3d<T>();
  const T* M[10];
  for (int k = 0; k < 10; ++k) M[k] = cur + k * N;
  // rows r = x * ny + y in [r0, r1): threads split (x, y) rows, so a thin slab still
  // gives every thread work
  for (int64_t r = r0; r < r1; ++r) {
    const int x = int(r / ny), y = int(r % ny);
    {
      for (int z = 0; z < nz; ++z) {
        const size_t c = (size_t(x) * ny + y) * nz + z;
        const int fl = flag ? flag[c] : ML_FLUID;
        if (fl != ML_FLUID) continue;
        const T rho_c = M[0][c], ux_c = M[1][c], uy_c = M[2][c], uz_c = M[3][c];
        const T Sxx_c = M[4][c], Syy_c = M[5][c], Szz_c = M[6][c], Sxy_c = M[7][c], Sxz_c = M[8][c],
                Syz_c = M[9][c];
        const V3<T> cell{T(x), T(y), T(z)};
        int near = 0;
        for (int sid = 0; sid < s.n_objects; ++sid) {
          if (s.tri_offset[sid + 1] - s.tri_offset[sid] == 0) continue;
          const V3<T> rel{cell.x - s.position[3 * sid], cell.y - s.position[3 * sid + 1],
                          cell.z - s.position[3 * sid + 2]};
          if (vlen(rel) <= s.bound_radius[sid] + T(2.0)) near = 1;
        }
        T rho_acc = 0, uxp = 0, uxm = 0, uyp = 0, uym = 0, uzp = 0, uzm = 0, pixx = 0, piyy = 0, pizz = 0;
        T pixy_p = 0, pixy_m = 0, pixz_p = 0, pixz_m = 0, piyz_p = 0, piyz_m = 0;
        for (int i = 0; i < 27; ++i) {
          const T dx = T(CX3[i]), dy = T(CY3[i]), dz = T(CZ3[i]);
          const T wi = T(w3d(i));
          int xn = x - CX3[i], yn = y - CY3[i], zn = z - CZ3[i];
          if (p.periodic) {
            xn = (xn + nx) % nx;
            yn = (yn + ny) % ny;
            zn = (zn + nz) % nz;
          }
          T pop_i = T(0.0);
          if (xn >= 0 && xn < nx && yn >= 0 && yn < ny && zn >= 0 && zn < nz) {
            T cutcell = T(-1.0);
            int sid = -1;
            const V3<T> dir{-dx, -dy, -dz};
            if (near == 1) get_cutcell_3d(s, cell, dir, &cutcell, &sid);
            if (cutcell >= T(0.0) && cutcell <= T(1.0) && sid >= 0) {
              const Xform<T> tc = load_xform(s.transforms + 7 * sid);
              const Xform<T> tl = load_xform(s.transforms_last + 7 * sid);
              const V3<T> hit{cell.x + dir.x * cutcell, cell.y + dir.y * cutcell, cell.z + dir.z * cutcell};
              const V3<T> hl = xpoint(xinv(tc), hit);
              V3<T> up;
              if (s.initialized[sid] > 0) {
                const V3<T> pc = xpoint(tc, hl), pl = xpoint(tl, hl);
                up = {pc.x - pl.x, pc.y - pl.y, pc.z - pl.z};
              } else {
                const T* sp = s.position + 3 * sid;
                const T* lv = s.linear_v + 3 * sid;
                const T* av = s.angle_v + 3 * sid;
                const V3<T> dv{hit.x - sp[0], hit.y - sp[1], hit.z - sp[2]};
                const V3<T> va{av[1] * dv.z - av[2] * dv.y, av[2] * dv.x - av[0] * dv.z, av[0] * dv.y - av[1] * dv.x};
                up = {lv[0] + va.x, lv[1] + va.y, lv[2] + va.z};
              }
              const T* sp = s.position + 3 * sid;
              const V3<T> dv{hit.x - sp[0], hit.y - sp[1], hit.z - sp[2]};
              const T Sxx_s = up.x * up.x + Sxx_c - ux_c * ux_c;
              const T Sxy_s = up.x * up.y + Sxy_c - ux_c * uy_c;
              const T Sxz_s = up.x * up.z + Sxz_c - ux_c * uz_c;
              const T Syy_s = up.y * up.y + Syy_c - uy_c * uy_c;
              const T Syz_s = up.y * up.z + Syz_c - uy_c * uz_c;
              const T Szz_s = up.z * up.z + Szz_c - uz_c * uz_c;
              pop_i = feq3<T>(rho_c, up.x, up.y, up.z, Sxx_s, Sxy_s, Sxz_s, Syy_s, Syz_s, Szz_s, dx, dy, dz, wi);
              const int ii = INV3[i];
              const T ex = T(CX3[ii]), ey = T(CY3[ii]), ez = T(CZ3[ii]);
              const T cur_f =
                  feq3<T>(rho_c, ux_c, uy_c, uz_c, Sxx_c, Sxy_c, Sxz_c, Syy_c, Syz_c, Szz_c, ex, ey, ez, T(w3d(ii)));
              const T fx = cur_f * (ex - up.x) - pop_i * (dx - up.x);
              const T fy = cur_f * (ey - up.y) - pop_i * (dy - up.y);
              const T fz = cur_f * (ez - up.z) - pop_i * (dz - up.z);
              T* L = loads + 6 * sid;
              L[0] += fx;
              L[1] += fy;
              L[2] += fz;
              L[3] += dv.y * fz - dv.z * fy;
              L[4] += dv.z * fx - dv.x * fz;
              L[5] += dv.x * fy - dv.y * fx;
            } else {
              const size_t n = (size_t(xn) * ny + yn) * nz + zn;
              pop_i = feq3<T>(M[0][n], M[1][n], M[2][n], M[3][n], M[4][n], M[7][n], M[8][n], M[5][n], M[9][n],
                              M[6][n], dx, dy, dz, wi);
              if (pop_i < T(0.0)) pop_i = T(0.0);
            }
          }
          rho_acc = rho_acc + pop_i;
          if (dx > T(0.0)) { uxp = uxp + pop_i; pixx = pixx + pop_i; }
          else if (dx < T(0.0)) { uxm = uxm + pop_i; pixx = pixx + pop_i; }
          if (dy > T(0.0)) { uyp = uyp + pop_i; piyy = piyy + pop_i; }
          else if (dy < T(0.0)) { uym = uym + pop_i; piyy = piyy + pop_i; }
          if (dz > T(0.0)) { uzp = uzp + pop_i; pizz = pizz + pop_i; }
          else if (dz < T(0.0)) { uzm = uzm + pop_i; pizz = pizz + pop_i; }
          const T dxy = dx * dy, dxz = dx * dz, dyz = dy * dz;
          if (dxy > T(0.0)) pixy_p = pixy_p + pop_i;
          else if (dxy < T(0.0)) pixy_m = pixy_m + pop_i;
          if (dxz > T(0.0)) pixz_p = pixz_p + pop_i;
          else if (dxz < T(0.0)) pixz_m = pixz_m + pop_i;
          if (dyz > T(0.0)) piyz_p = piyz_p + pop_i;
          else if (dyz < T(0.0)) piyz_m = piyz_m + pop_i;
        }
        const T Fx = force ? force[c] : T(0.0);
        const T Fy = force ? force[N + c] : T(0.0);
        const T Fz = force ? force[2 * N + c] : T(0.0);
        const T rhoVar = rho_acc;
        const T invRho = T(1.0) / rhoVar;
        const T ux = (uxp - uxm + T(0.5) * Fx) * invRho;
        const T uy = (uyp - uym + T(0.5) * Fy) * invRho;
        const T uz = (uzp - uzm + T(0.5) * Fz) * invRho;
        T pixy = pixy_p - pixy_m, pixz = pixz_p - pixz_m, piyz = piyz_p - piyz_m;
        const T Omega = T(1.0) / (p.vis_shear * T(3.0) + T(0.5));
        const T pixx_part = (T(2.0) * pixx - piyy - pizz) / T(3.0);
        const T piyy_part = (T(2.0) * piyy - pixx - pizz) / T(3.0);
        const T pizz_part = (T(2.0) * pizz - pixx - piyy) / T(3.0);
        const T RU2 = rhoVar * ux * ux, RV2 = rhoVar * uy * uy, RW2 = rhoVar * uz * uz;
        const T RUVW2 = (RU2 + RV2 + RW2) / T(3.0);
        const T o1 = T(1.0) - Omega;
        pixx = rhoVar / T(3.0) + pixx_part * o1 + RUVW2 + (T(2.0) * RU2 * Omega) / T(3.0) - (RV2 * Omega) / T(3.0) -
               (RW2 * Omega) / T(3.0) + Fx * ux;
        piyy = rhoVar / T(3.0) + piyy_part * o1 + RUVW2 - (RU2 * Omega) / T(3.0) + (T(2.0) * RV2 * Omega) / T(3.0) -
               (RW2 * Omega) / T(3.0) + Fy * uy;
        pizz = rhoVar / T(3.0) + pizz_part * o1 + RUVW2 - (RU2 * Omega) / T(3.0) - (RV2 * Omega) / T(3.0) +
               (T(2.0) * RW2 * Omega) / T(3.0) + Fz * uz;
        pixy = pixy - pixy * Omega + ux * uy * rhoVar * Omega + (Fy * ux + Fx * uy) / T(2.0);
        pixz = pixz - pixz * Omega + ux * uz * rhoVar * Omega + (Fz * ux + Fx * uz) / T(2.0);
        piyz = piyz - piyz * Omega + uy * uz * rhoVar * Omega + (Fz * uy + Fy * uz) / T(2.0);
        post[c] = rhoVar;
        post[N + c] = ux + Fx * invRho / T(2.0);
        post[2 * N + c] = uy + Fy * invRho / T(2.0);
        post[3 * N + c] = uz + Fz * invRho / T(2.0);
        post[4 * N + c] = pixx * invRho - cs2;
        post[5 * N + c] = piyy * invRho - cs2;
        post[6 * N + c] = pizz * invRho - cs2;
        post[7 * N + c] = pixy * invRho;
        post[8 * N + c] = pixz * invRho;
        post[9 * N + c] = piyz * invRho;
      }
    }
  }
}

// f_eq_home_3d, envs/lbm3d/lbm_func_3d.py:651-686 (no clamp, unlike 2D)
template <class T> void f_eq_home_3d(const T* post, size_t N, size_t c, T out[6]) {
  T pop[27];
  const T rho = post[c], ux = post[N + c], uy = post[2 * N + c], uz = post[3 * N + c];
  const T U_sqr = ux * ux + uy * uy + uz * uz;
  for (int i = 0; i < 27; ++i) {
    const T cu = T(CX3[i]) * ux + T(CY3[i]) * uy + T(CZ3[i]) * uz;
    pop[i] = T(w3d(i)) * rho * (T(1.0) + T(3.0) * cu + T(4.5) * cu * cu - T(1.5) * U_sqr);
  }
  const T invRho = T(1.0) / rho;
  T pixx = pop[1] + pop[2] + pop[7] + pop[8] + pop[9] + pop[10] + pop[13] + pop[14] + pop[15] + pop[16] + pop[19] +
           pop[20] + pop[21] + pop[22] + pop[23] + pop[24] + pop[25] + pop[26];
  T pixy = (pop[7] + pop[8] + pop[19] + pop[20] + pop[21] + pop[22]) -
           (pop[13] + pop[14] + pop[23] + pop[24] + pop[25] + pop[26]);
  T pixz = (pop[9] + pop[10] + pop[19] + pop[20] + pop[23] + pop[24]) -
           (pop[15] + pop[16] + pop[21] + pop[22] + pop[25] + pop[26]);
  T piyy = pop[3] + pop[4] + pop[7] + pop[8] + pop[11] + pop[12] + pop[13] + pop[14] + pop[17] + pop[18] + pop[19] +
           pop[20] + pop[21] + pop[22] + pop[23] + pop[24] + pop[25] + pop[26];
  T piyz = (pop[11] + pop[12] + pop[19] + pop[20] + pop[25] + pop[26]) -
           (pop[17] + pop[18] + pop[21] + pop[22] + pop[23] + pop[24]);
  T pizz = pop[5] + pop[6] + pop[9] + pop[10] + pop[11] + pop[12] + pop[15] + pop[16] + pop[17] + pop[18] + pop[19] +
           pop[20] + pop[21] + pop[22] + pop[23] + pop[24] + pop[25] + pop[26];
  const T cs2 = cs2_3d<T>();
  out[0] = pixx * invRho - cs2;  // xx
  out[1] = pixy * invRho;        // xy
  out[2] = pixz * invRho;        // xz
  out[3] = piyy * invRho - cs2;  // yy
  out[4] = piyz * invRho;        // yz
  out[5] = pizz * invRho - cs2;  // zz
}

// apply_bc_core_3d, envs/lbm3d/lbm_func_3d.py:627-648
template <class T> void apply_bc_core_3d(const Params3<T>& p, T* post, int dr, size_t b, size_t n) {
  const size_t N = size_t(p.nx) * p.ny * p.nz;
  if (p.bc_type[dr] == 0) {
    for (int k = 0; k < 3; ++k) post[(1 + k) * N + b] = p.bc_value[3 * dr + k];
  } else if (p.bc_type[dr] == 1) {
    for (int k = 0; k < 3; ++k) post[(1 + k) * N + b] = post[(1 + k) * N + n];
  }
  post[b] = post[n];
  T cur[6], back[6];
  f_eq_home_3d(post, N, b, cur);
  f_eq_home_3d(post, N, n, back);
  // stored plane order: Sxx(4) Syy(5) Szz(6) Sxy(7) Sxz(8) Syz(9); cur[] is xx xy xz yy yz zz
  const int plane[6] = {4, 7, 8, 5, 9, 6};
  for (int k = 0; k < 6; ++k) post[plane[k] * N + b] = cur[k] - back[k] + post[plane[k] * N + n];
}

// apply_bc_3d, envs/lbm3d/lbm_func_3d.py:607-624, threads in launch order (x, y, z)
template <class T> void apply_bc_3d(const Params3<T>& p, T* post) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  auto idx = [&](int x, int y, int z) { return (size_t(x) * ny + y) * nz + z; };
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y) {
      const bool xyb = (x == 0 || x == nx - 1 || y == 0 || y == ny - 1);
      for (int z = 0; z < nz; ++z) {
        if (!xyb && z != 0 && z != nz - 1) continue;
        if (x == 0) apply_bc_core_3d(p, post, 0, idx(0, y, z), idx(1, y, z));
        else if (x == nx - 1) apply_bc_core_3d(p, post, 1, idx(nx - 1, y, z), idx(nx - 2, y, z));
        if (y == ny - 1) apply_bc_core_3d(p, post, 2, idx(x, ny - 1, z), idx(x, ny - 2, z));
        else if (y == 0) apply_bc_core_3d(p, post, 3, idx(x, 0, z), idx(x, 1, z));
        if (z == nz - 1) apply_bc_core_3d(p, post, 4, idx(x, y, nz - 1), idx(x, y, nz - 2));
        else if (z == 0) apply_bc_core_3d(p, post, 5, idx(x, y, 0), idx(x, y, 1));
      }
    }
}

// LBM_Solver3D.step, envs/lbm3d/lbm_solver_3d.py:95-127 (zero loads, stream-collide,
// apply_bc). The caller swaps cur/post afterwards (Swap_Mom_3D).
template <class T>
void step_3d(const Params3<T>& p, Solids3<T>& s, const T* cur, T* post, const int* flag, const T* force,
             int nthreads) {
  for (int i = 0; i < 6 * s.n_objects; ++i) s.loads[i] = T(0.0);
  const int nt = num_threads(nthreads);
  if (nt <= 1) {
    stream_collide_3d_rows(p, s, cur, post, flag, force, 0, int64_t(p.nx) * p.ny, s.loads);
  } else {
    std::vector<T> part(size_t(nt) * 6 * s.n_objects + 1, T(0.0));
    const int64_t rows = int64_t(p.nx) * p.ny;
    parallel_for_threads(nt, [&](int t, int n) {
      const int64_t r0 = rows * t / n, r1 = rows * (t + 1) / n;
      stream_collide_3d_rows(p, s, cur, post, flag, force, r0, r1, part.data() + size_t(t) * 6 * s.n_objects);
    });
    for (int t = 0; t < nt; ++t)
      for (int i = 0; i < 6 * s.n_objects; ++i) s.loads[i] += part[size_t(t) * 6 * s.n_objects + i];
  }
  if (!p.periodic) apply_bc_3d(p, post);
}

}  // namespace

// ============================================================================ C ABI
extern "C" {

#define OR_2D_ARGS(T)                                                                                          \
  int nx, int ny, T vis_shear, T grid_length, T time_step, const int *bc_type, const T *bc_value, int periodic, \
      const T *cur, T *post, const int *flag, const T *forcex, const T *forcey, int n_objects, int max_segments, \
      const T *line, const int *line_num, T *tf, T *tf_last, const T *position, const T *angle, const T *scale,  \
      const T *mass_center, const T *max_radius, T *loads, int nthreads

#define OR_2D_BODY(T)                                                                                      \
  Params2<T> p{nx, ny, vis_shear, grid_length, time_step, bc_type, bc_value, periodic};                    \
  Solids2<T> s{n_objects, max_segments, line, line_num, tf, tf_last, position, angle, scale, mass_center, \
               max_radius, loads};                                                                         \
  step_2d(p, s, cur, post, flag, forcex, forcey, nthreads);                                                \
  return 0;

// One LBM_Solver.step of one world: post <- step(cur); loads <- per-solid loads.
int oracle_step_2d_f32(OR_2D_ARGS(float)) { OR_2D_BODY(float) }
int oracle_step_2d_f64(OR_2D_ARGS(double)) { OR_2D_BODY(double) }

#define OR_3D_ARGS(T)                                                                                          \
  int nx, int ny, int nz, T vis_shear, const int *bc_type, const T *bc_value, int periodic, const T *cur,      \
      T *post, const int *flag, const T *force, int n_objects, const int *tri_offset, const T *tris,           \
      const T *transforms, const T *transforms_last, const int *initialized, const T *scale_sizes,             \
      const T *position, const T *bound_radius, const T *linear_v, const T *angle_v, T *loads, int nthreads

#define OR_3D_BODY(T)                                                                                              \
  Params3<T> p{nx, ny, nz, vis_shear, bc_type, bc_value, periodic};                                                \
  Solids3<T> s{n_objects, tri_offset, tris, transforms, transforms_last, initialized, scale_sizes, position,       \
               bound_radius, linear_v, angle_v, loads};                                                            \
  step_3d(p, s, cur, post, flag, force, nthreads);                                                                 \
  return 0;

// One LBM_Solver3D.step of one world: post <- step(cur); loads <- per-solid force, torque.
int oracle_step_3d_f32(OR_3D_ARGS(float)) { OR_3D_BODY(float) }
int oracle_step_3d_f64(OR_3D_ARGS(double)) { OR_3D_BODY(double) }

int oracle_max_threads(void) { return num_threads(0); }

}  // extern "C"
