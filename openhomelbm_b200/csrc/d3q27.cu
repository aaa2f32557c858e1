// D3Q27 HOME-LBM step for sm_100a: stream-collide, outer boundaries, initial states.
//
// Stream-collide (replaces stream_and_collide_3d, envs/lbm3d/lbm_func_3d.py:364-604).
// The reference pulls, for every cell and direction i, the population rebuilt from the
// upwind neighbour's moments,
//     f_i = w_i rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u.u + 1.5 sum_ab Q_ab S_ab),
//     Q = c c - I/3 (off-diagonal terms counted twice)      [mlCalEquilibrium3D_s, 224-251]
// clamps it at zero and collides in moment space. Expanded in the lattice velocity c
// (components in {-1, 0, 1}) the bracket is, per SOURCE cell,
//     g(c) = A + c.B + sum_a c_a^2 C_aa + sum_{a<b} c_a c_b D_ab,
//     A = rho (1 - 1.5 u.u - 0.5 tr S), B_a = 3 rho u_a, C_aa = rho (4.5 u_a^2 + 1.5 S_aa),
//     D_ab = rho (9 u_a u_b + 3 S_ab),
// so a source cell's 27 populations come out of one shared add-tree (about 50 adds), not
// 27 independent evaluations (about 1200 flops). The kernel therefore works source-side:
//
//  * a CTA owns a TY x 32 (y, z) column tile and marches through x planes;
//  * each source plane (tile plus a one-cell halo, zero-filled outside non-periodic
//    domains: a zero cell rebuilds to zero populations, which is the reference's
//    out-of-range rule) is staged in shared memory by asynchronous copies two planes ahead;
//  * every thread rebuilds the 27 clamped populations of one source cell and posts them to a
//    shared-memory mailbox indexed by (direction, source);
//  * every destination thread reads its 27 incoming populations, reduces each group of 9
//    (same c_x) to partial moments and keeps running sums for the planes x-1, x, x+1; a plane
//    is complete once the source plane after it has been posted, then it collides (the
//    regularised collision of lines 564-604, same formulas) and is written out.
// Populations are carried as deviations from the rest state, f - w (g - 1 in the bracket):
// sums then have no O(1) offset, the zero clamp f >= 0 becomes f - w >= -w, and S comes
// out of the collision without the Pi/rho - 1/3 cancellation. The arithmetic is the
// reference's, evaluated with less rounding.
// HBM traffic is one read and one write of the 10 moments per cell (80 B in binary32).
// Halo reloads come from L2 because all CTAs march the same x range in step.

#include <cstdio>
#include <cstdlib>

#include "d3q27_core.cuh"

namespace hl {
namespace d3 {

constexpr int TZ = 32;
constexpr int BZ = TZ + 2;
constexpr int NSTAGE = 3;

template <int TY> struct Tile {
  static constexpr int BY = TY + 2;
  static constexpr int NSRC = BY * BZ;
  static constexpr int NDST = TY * TZ;
  static constexpr int THREADS = ((NSRC + 31) / 32) * 32;
};

template <int TY, class S, bool PERIODIC, bool FORCE, bool FLAGS, bool DIAG>
__global__ void __launch_bounds__(Tile<TY>::THREADS, 1) step_kernel(const StepArgs a) {
  using T = typename S::T;
  using R = typename S::R;
  using TL = Tile<TY>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* stage = reinterpret_cast<T*>(smem_raw);  // [NSTAGE][10][NSRC]
  R* mb = reinterpret_cast<R*>(smem_raw + ((NSTAGE * 10 * TL::NSRC * sizeof(T) + 15) / 16) * 16);  // [27][NSRC]

  const int tid = threadIdx.x;
  const bool is_src = tid < TL::NSRC;
  const int sy = tid / BZ, sz = tid - (tid / BZ) * BZ;
  const bool is_dst = tid < TL::NDST;
  const int ty = tid / TZ, tz = tid & (TZ - 1);
  const int dsrc = (ty + 1) * BZ + tz + 1;
  const long long N = a.N;
  const long long plane = (long long)a.ny * a.nz;
  const T* cur = static_cast<const T*>(a.cur);
  T* post = static_cast<T*>(a.post);
  const R omega = R(1) / (R(a.vis_shear) * R(3) + R(0.5));

  double mass = 0.0;
  int bad = 0;

  for (int item = blockIdx.x; item < a.n_items; item += gridDim.x) {
    const int tile = item % a.n_tiles, chunk = item / a.n_tiles;
    const int y0 = (tile / a.tiles_z) * TY, z0 = (tile % a.tiles_z) * TZ;
    const int xb = chunk * a.chunk_len;
    const int xe = min(xb + a.chunk_len, a.nx);
    int gy = y0 - 1 + sy, gz = z0 - 1 + sz;
    bool src_in = is_src;
    if (PERIODIC) {
      gy = ((gy % a.ny) + a.ny) % a.ny;
      gz = ((gz % a.nz) + a.nz) % a.nz;
    } else {
      src_in = src_in && gy >= 0 && gy < a.ny && gz >= 0 && gz < a.nz;
    }
    const long long src_col = src_in ? (long long)gy * a.nz + gz : 0;
    const int dy = y0 + ty, dz = z0 + tz;
    const bool dst_in = is_dst && dy < a.ny && dz < a.nz;

    auto issue = [&](int xs, int slot) {
      if (is_src) {
        int gx = xs;
        bool in = src_in;
        if (PERIODIC) gx = ((gx % a.nx) + a.nx) % a.nx;
        else in = in && gx >= 0 && gx < a.nx;
        const T* g = cur + (in ? (long long)gx * plane + src_col : 0);
        T* s = stage + (slot * 10) * TL::NSRC + tid;
#pragma unroll
        for (int k = 0; k < 10; ++k) {
          if constexpr (sizeof(T) == 4) {
            cp_async4(s + k * TL::NSRC, g + k * N, in ? 4 : 0);
          } else {
            s[k * TL::NSRC] = in ? g[k * N] : T(0);
          }
        }
      }
      cp_async_commit();
    };

    Acc<R> acc_cur, acc_next;
    acc_cur.zero();
    acc_next.zero();
    issue(xb - 1, 0);
    issue(xb, 1);
    int it = 0;
    for (int xs = xb - 1; xs <= xe; ++xs, ++it) {
      if (xs + 2 <= xe) issue(xs + 2, (it + 2) % NSTAGE);
      else cp_async_commit();
      cp_async_wait<2>();
      __syncthreads();  // the mailbox is free again; this thread's staged plane has landed
      if (is_src) {
        bool in = src_in;
        if (!PERIODIC) in = in && xs >= 0 && xs < a.nx;
        R f[27];
        Mom3<R> m;
        if (in) {
          const T* s = stage + ((it % NSTAGE) * 10) * TL::NSRC + tid;
          R raw[10];
#pragma unroll
          for (int k = 0; k < 10; ++k) raw[k] = S::to_r(s[k * TL::NSRC]);
          m = decode3<S>(raw, a.sc);
        } else {
          // outside the domain: zero populations (f - w = -w), the reference's out-of-range rule
          m.rho = R(0);
          m.drho = R(-1);
          m.ux = m.uy = m.uz = m.sxx = m.syy = m.szz = m.sxy = m.sxz = m.syz = R(0);
        }
        rebuild_all<R>(m, f);
#pragma unroll
        for (int d = 0; d < 27; ++d) mb[d * TL::NSRC + tid] = f[d];
      }
      __syncthreads();
      if (is_dst) {
        Acc<R> acc_new;
        acc_new.zero();
#pragma unroll
        for (int xi = 0; xi < 3; ++xi) {
          R p[3][3];
#pragma unroll
          for (int yi = 0; yi < 3; ++yi)
#pragma unroll
            for (int zi = 0; zi < 3; ++zi)
              p[yi][zi] = mb[((xi * 3 + yi) * 3 + zi) * TL::NSRC + dsrc - (yi - 1) * BZ - (zi - 1)];
          // c_x = -1 completes plane xs-1, 0 feeds plane xs, +1 starts plane xs+1
          if (xi == 0) accumulate_group<R>(acc_cur, p, -1);
          else if (xi == 1) accumulate_group<R>(acc_next, p, 0);
          else accumulate_group<R>(acc_new, p, 1);
        }
        const int dx = xs - 1;
        if (dst_in && dx >= xb) {
          const long long c = (long long)dx * plane + (long long)dy * a.nz + dz;
          bool fluid;
          if (FLAGS) fluid = a.flag[c] == ML_FLUID;
          else if (PERIODIC) fluid = true;
          else fluid = dx > 0 && dx < a.nx - 1 && dy > 0 && dy < a.ny - 1 && dz > 0 && dz < a.nz - 1;
          if (fluid) {
            R Fx = R(0), Fy = R(0), Fz = R(0);
            if (FORCE) {
              Fx = R(a.force[c]);
              Fy = R(a.force[N + c]);
              Fz = R(a.force[2 * N + c]);
            }
            const Mom3<R> m = collide<R>(acc_cur, Fx, Fy, Fz, omega);
            R raw[10];
            encode3<S>(m, a.sc, raw);
#pragma unroll
            for (int k = 0; k < 10; ++k) post[k * N + c] = S::from_r(raw[k], unsigned(k * N + c));
            if (DIAG) {
              mass += double(m.rho);
              bad += healthy<R>(m) ? 0 : 1;
            }
          }
        }
        acc_cur = acc_next;
        acc_next = acc_new;
      }
    }
    __syncthreads();  // stage slots and mailbox are reused by the next item
  }

  if (DIAG) {
    __shared__ double red_d[32];
    __shared__ int red_i[32];
    const double ms = block_sum<double>(mass, red_d);
    const int bs = block_sum<int>(bad, red_i);
    __shared__ bool last;
    if (tid == 0) {
      a.partials[blockIdx.x] = ms;
      a.bad_partials[blockIdx.x] = bs;
      __threadfence();
      last = atomicAdd(a.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && tid == 0) {
      __threadfence();
      double tot = 0.0;
      int tb = 0;
      for (unsigned b = 0; b < gridDim.x; ++b) {
        tot += reinterpret_cast<volatile double*>(a.partials)[b];
        tb += reinterpret_cast<volatile int*>(a.bad_partials)[b];
      }
      if (a.mass) *a.mass = tot;
      if (a.health) *a.health = tb;
      *a.counter = 0u;
    }
  }
}

// ----------------------------------------------------------------------------- host side
template <int TY, class S> size_t smem_bytes() {
  using TL = Tile<TY>;
  const size_t st = ((NSTAGE * 10 * TL::NSRC * sizeof(typename S::T) + 15) / 16) * 16;
  return st + 27 * TL::NSRC * sizeof(typename S::R);
}

int num_sms() { return device_sms(); }

// Work split: tiles x x-chunks. All CTAs march whole x ranges in step so that halo reloads
// are L2 hits; x is split only when that fills the SMs with less waste.
struct Plan {
  int tiles_y, tiles_z, n_tiles, chunks, chunk_len, n_items, grid;
};

template <int TY> Plan make_plan(int nx, int ny, int nz) {
  Plan p;
  p.tiles_y = (ny + TY - 1) / TY;
  p.tiles_z = (nz + TZ - 1) / TZ;
  p.n_tiles = p.tiles_y * p.tiles_z;
  const int sms = num_sms();
  double best = -1.0;
  int best_c = 1;
  const int forced = g_tune_d3_chunks;
  for (int c = 1; c <= 64 && c <= nx; ++c) {
    if (forced > 0 && c != forced) continue;
    const int len = (nx + c - 1) / c;
    const int items = p.n_tiles * ((nx + len - 1) / len);
    const int waves = (items + sms - 1) / sms;
    const double eff = double(items) / (double(waves) * sms) * double(len) / double(len + 2);
    if (eff > best + 1e-9) {
      best = eff;
      best_c = c;
    }
  }
  p.chunk_len = (nx + best_c - 1) / best_c;
  p.chunks = (nx + p.chunk_len - 1) / p.chunk_len;
  p.n_items = p.n_tiles * p.chunks;
  p.grid = p.n_items < sms ? p.n_items : sms;
  return p;
}

size_t diag_scratch_bytes() { return size_t(num_sms()) * (sizeof(double) + sizeof(int)) + 64; }

void fill_diag(StepArgs& a, const hl_diag* diag) {
  char* s = static_cast<char*>(diag->scratch);
  a.counter = reinterpret_cast<unsigned*>(s);
  a.partials = reinterpret_cast<double*>(s + 16);
  a.bad_partials = reinterpret_cast<int*>(s + 16 + sizeof(double) * num_sms());
  a.mass = diag->mass;
  a.health = diag->health;
}

template <int TY, class S, bool PERIODIC, bool FORCE, bool FLAGS, bool DIAG>
int launch_step(const hl_world3d* w, double vis_shear, const hl_diag* diag, cudaStream_t st) {
  const Plan p = make_plan<TY>(w->nx, w->ny, w->nz);
  StepArgs a{};
  a.cur = w->cur;
  a.post = w->post;
  a.N = (long long)w->nx * w->ny * w->nz;
  a.nx = w->nx;
  a.ny = w->ny;
  a.nz = w->nz;
  a.tiles_y = p.tiles_y;
  a.tiles_z = p.tiles_z;
  a.n_tiles = p.n_tiles;
  a.chunk_len = p.chunk_len;
  a.n_items = p.n_items;
  a.vis_shear = vis_shear;
  a.force = w->force;
  a.flag = w->flag;
  a.sc = make_scale(w->storage);
  if (DIAG) fill_diag(a, diag);
  const size_t smem = smem_bytes<TY, S>();
  auto kern = step_kernel<TY, S, PERIODIC, FORCE, FLAGS, DIAG>;
  const int rc = set_smem_attr(reinterpret_cast<const void*>(kern), int(smem), "cudaFuncSetAttribute(d3q27 step)");
  if (rc != HL_OK) return rc;
  kern<<<p.grid, Tile<TY>::THREADS, smem, st>>>(a);
  HL_LAUNCH_CHECK("d3q27 stream_collide launch");
  return HL_OK;
}

template <int TY, class S>
int dispatch_step(const hl_world3d* w, double vis, const hl_diag* d, cudaStream_t st) {
  const bool P = w->periodic != 0, F = w->force != nullptr, G = w->flag != nullptr && !P,
             D = d != nullptr && d->scratch != nullptr;
#define HL_D3_CASE(p, f, g, dg) \
  if (P == p && F == f && G == g && D == dg) return launch_step<TY, S, p, f, g, dg>(w, vis, d, st);
  HL_D3_CASE(true, false, false, false)
  HL_D3_CASE(true, false, false, true)
  HL_D3_CASE(true, true, false, false)
  HL_D3_CASE(true, true, false, true)
  HL_D3_CASE(false, false, false, false)
  HL_D3_CASE(false, false, false, true)
  HL_D3_CASE(false, true, false, false)
  HL_D3_CASE(false, true, false, true)
  HL_D3_CASE(false, false, true, false)
  HL_D3_CASE(false, false, true, true)
  HL_D3_CASE(false, true, true, false)
  HL_D3_CASE(false, true, true, true)
#undef HL_D3_CASE
  set_error("d3q27: unsupported option combination");
  return HL_ERR_UNSUPPORTED;
}

}  // namespace d3
}  // namespace hl

using namespace hl;

extern "C" int hl_d3q27_stream_collide(const hl_world3d* w, double vis_shear, const hl_diag* diag,
                                       hl_stream stream) {
  HL_CHECK_ARG(w != nullptr, "d3q27: world is NULL");
  HL_CHECK_ARG(w->nx >= 1 && w->ny >= 1 && w->nz >= 1, "d3q27: bad dims %d x %d x %d", w->nx, w->ny, w->nz);
  HL_CHECK_ARG(w->cur != nullptr && w->post != nullptr && w->cur != w->post, "d3q27: cur/post must be distinct");
  HL_CHECK_ARG(vis_shear > 0.0f, "d3q27: viscosity must be positive");
  HL_CHECK_ARG(diag == nullptr || diag->scratch == nullptr || diag->scratch_bytes >= d3::diag_scratch_bytes(),
               "d3q27: diagnostics scratch too small (%zu < %zu)", diag ? diag->scratch_bytes : 0,
               d3::diag_scratch_bytes());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (g_tune_d3_kernel == 2 && !d3::tma_eligible(w)) {
    set_error("d3q27: the TMA kernel needs ny %% 16 == 0, nz %% 32 == 0 and a non-float64 storage");
    return HL_ERR_UNSUPPORTED;
  }
  if (g_tune_d3_kernel != 1 && d3::tma_eligible(w)) return d3::launch_step_tma(w, vis_shear, diag, st);
  switch (w->storage.dtype) {
    case HL_F32: return d3::dispatch_step<16, StoreF32>(w, vis_shear, diag, st);
    case HL_F64: return d3::dispatch_step<8, StoreF64>(w, vis_shear, diag, st);
    default:
      set_error("d3q27: storage dtype %d not supported by this build", int(w->storage.dtype));
      return HL_ERR_UNSUPPORTED;
  }
}

extern "C" size_t hl_d3q27_scratch_bytes(const hl_world3d*) { return d3::diag_scratch_bytes(); }

// ============================================================================ allocation-free
// hl_d3q27_stream_collide_noalloc: the diagnostics-enabled stream-collide for callers that
// cannot allocate device memory (see include/homelbm.h). Its scratch - the per-CTA partial
// sums and the completion counter - lives in a file-scope device array instead of a
// caller-provided buffer.
#include <mutex>

namespace hl {
namespace d3 {

constexpr size_t kNoAllocScratchBytes = 16384;  // 16 + 12 bytes per CTA: up to 1364 CTAs (one per SM)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch on the current device. The host-side symbol is only a
// stand-in, so the address is resolved once per device with that device current.
static int noalloc_scratch(void** out) {
  static std::mutex mu;
  static void* addr[128] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "hl_d3q27_stream_collide_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= 128) {
    set_error("hl_d3q27_stream_collide_noalloc: device ordinal %d out of range", dev);
    return HL_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (addr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return cuda_status(e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                         "hl_d3q27_stream_collide_noalloc: cudaGetSymbolAddress");
    addr[dev] = p;
  }
  *out = addr[dev];
  return HL_OK;
}

}  // namespace d3
}  // namespace hl

extern "C" int hl_d3q27_stream_collide_noalloc(const hl_world3d* w, double vis_shear, double* mass, int32_t* health,
                                               hl_stream stream) {
  HL_CHECK_ARG(w != nullptr, "d3q27 (no-alloc): world is NULL");
  HL_CHECK_ARG(w->nx >= 1 && w->ny >= 1 && w->nz >= 1, "d3q27 (no-alloc): bad dims %d x %d x %d", w->nx, w->ny, w->nz);
  HL_CHECK_ARG(w->cur != nullptr && w->post != nullptr && w->cur != w->post,
               "d3q27 (no-alloc): cur/post must be distinct");
  HL_CHECK_ARG(vis_shear > 0.0, "d3q27 (no-alloc): viscosity must be positive");
  HL_CHECK_ARG(w->storage.dtype == HL_F32 || w->storage.dtype == HL_F64,
               "d3q27 (no-alloc): storage must be float32 or float64");
  const d3::Plan plan =
      w->storage.dtype == HL_F32 ? d3::make_plan<16>(w->nx, w->ny, w->nz) : d3::make_plan<8>(w->nx, w->ny, w->nz);
  const size_t need = 16 + size_t(d3::num_sms()) * (sizeof(double) + sizeof(int));
  HL_CHECK_ARG(need <= d3::kNoAllocScratchBytes && size_t(plan.grid) <= size_t(d3::num_sms()),
               "d3q27 (no-alloc): needs %zu bytes of scratch for %d SMs; the static scratch holds %zu", need,
               d3::num_sms(), d3::kNoAllocScratchBytes);
  void* scratch = nullptr;
  int rc = d3::noalloc_scratch(&scratch);
  if (rc != HL_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the completion counter must start at zero (a previous launch leaves it at zero; clear it
  // anyway so that an interrupted launch cannot poison the next one)
  cudaError_t e = cudaMemsetAsync(scratch, 0, 16, st);
  if (e != cudaSuccess) return cuda_status(e, "hl_d3q27_stream_collide_noalloc: clear counter");
  hl_diag d{scratch, d3::kNoAllocScratchBytes, mass, health};
  return w->storage.dtype == HL_F32 ? d3::dispatch_step<16, StoreF32>(w, vis_shear, &d, st)
                                    : d3::dispatch_step<8, StoreF64>(w, vis_shear, &d, st);
}
