// D3Q27 stream-collide with TMA-staged source planes (sm_100a).
//
// Same arithmetic and mailbox exchange as the fallback kernel in d3q27.cu (source-side
// population rebuild, (direction, source) mailbox in shared memory, x-marching with three
// planes of partial moments). What differs is how each source plane reaches shared memory:
// one elected thread issues nine tensor-memory-access (TMA) box copies per plane,
//
//              z0-WZ..z0-1   z0..z0+31   z0+32..z0+32+WZ-1
//   y0-1       corner        y edge      corner
//   y0..y0+15  z edge        interior    z edge
//   y0+16      corner        y edge      corner
//
// each box spanning the 10 moment planes (WZ = 16 bytes of elements: the narrowest box TMA
// copies). Every box gets its own coordinates, so periodic wrap-around of the halo is just a
// coordinate, and boxes outside a walled domain are zero-filled by the TMA unit (a zero cell
// rebuilds to zero populations: the reference's out-of-range rule). Completion is tracked by
// one mbarrier per stage with bounded waits. No multicast: every CTA loads its own boxes.
//
// Per plane: every thread rebuilds the 27 populations of one interior source cell (threads
// 0..99 then the 9 or 3 populations a halo cell sends into the tile) into a shared-memory
// mailbox indexed by (direction, source); after a block barrier every thread reads the 27
// populations arriving at its destination cell, adds them to partial moments of the planes
// x-1, x, x+1 and collides the completed plane. NS stages keep NS-1 planes in flight.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "d3q27_core.cuh"

namespace hl {
namespace d3 {
namespace tma {

constexpr int TY = 16, TZ = 32;
constexpr int BZ = TZ + 2, BY = TY + 2;
constexpr int NSRC = BY * BZ;  // 612 mailbox slots (tile plus one-cell halo)
constexpr int NDST = TY * TZ;  // 512
constexpr int THREADS = 512;       // one interior cell per thread
constexpr int NHALO = NSRC - NDST;  // 100 halo cells, taken by threads 0..99
constexpr long long MAX_SPIN = 1ll << 21;  // bounded mbarrier waits (far above any real latency)

// Shared-memory geometry of one stage for element type T.
template <class T, int NSTAGE> struct Geo {
  static constexpr int WZ = 16 / int(sizeof(T));
  static constexpr int E_MID = TY * TZ, E_YE = TZ, E_ZE = TY * WZ, E_C = WZ;  // elements per moment plane
  static constexpr int round128(int b) { return (b + 127) / 128 * 128; }
  static constexpr int B_MID = round128(10 * E_MID * int(sizeof(T)));
  static constexpr int B_YE = round128(10 * E_YE * int(sizeof(T)));
  static constexpr int B_ZE = round128(10 * E_ZE * int(sizeof(T)));
  static constexpr int B_C = round128(10 * E_C * int(sizeof(T)));
  // piece order: mid, ylo, yhi, zlo, zhi, (ylo,zlo), (ylo,zhi), (yhi,zlo), (yhi,zhi)
  static constexpr int OFF_MID = 0;
  static constexpr int OFF_YLO = B_MID;
  static constexpr int OFF_YHI = OFF_YLO + B_YE;
  static constexpr int OFF_ZLO = OFF_YHI + B_YE;
  static constexpr int OFF_ZHI = OFF_ZLO + B_ZE;
  static constexpr int OFF_C = OFF_ZHI + B_ZE;
  static constexpr int STAGE_BYTES = OFF_C + 4 * B_C;
  static constexpr int TX_BYTES = 10 * int(sizeof(T)) * (E_MID + 2 * E_YE + 2 * E_ZE + 4 * E_C);
  static constexpr int MB_BYTES = 27 * NSRC * 4;                      // the mailbox
  static constexpr int MB_OFF = NSTAGE * STAGE_BYTES;
  static constexpr int BAR_OFF = MB_OFF + MB_BYTES;                   // mbarriers
  static constexpr int SMEM = BAR_OFF + NSTAGE * 8 + 16 + 128;  // + alignment slack
};

struct Maps {
  CUtensorMap mid, yedge, zedge, corner;  // over the current buffer
};



// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ unsigned saddr(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load4(unsigned dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                          unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

// ---------------------------------------------------------------- kernel
template <class S, int NSTAGE, bool PERIODIC, bool FORCE, bool FLAGS, bool DIAG>
__global__ void __launch_bounds__(THREADS, 1) step_kernel_tma(const StepArgs a, const __grid_constant__ Maps maps) {
  using T = typename S::T;
  using R = typename S::R;
  using G = Geo<T, NSTAGE>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + G::BAR_OFF);
  R* mb = reinterpret_cast<R*>(smem + G::MB_OFF);
  __shared__ int box_c[6];  // z lo, z mid, z hi, y lo, y mid, y hi of the current item

  const int tid = threadIdx.x;
  const int ty = tid / TZ, tz = tid % TZ;
  const int dsrc = (ty + 1) * BZ + tz + 1;  // mailbox slot of this thread's interior cell
  // halo cell of threads 0..99: rows y0-1 / y0+16 (34 cells each), columns z0-1 / z0+32
  const bool has_halo = tid < NHALO;
  int hsy = 0, hsz = 0, piece_off = 0, cell_off = 0, mstride = 1, sel_y = -1, sel_z = -1;
  if (tid < 2 * BZ) {
    const bool hi = tid >= BZ;
    hsy = hi ? BY - 1 : 0;
    hsz = hi ? tid - BZ : tid;
    sel_y = hi ? 0 : 2;  // the row below the tile sends c_y = +1, the row above c_y = -1
    if (hsz == 0 || hsz == BZ - 1) {
      piece_off = G::OFF_C + ((hi ? 2 : 0) + (hsz == 0 ? 0 : 1)) * G::B_C;
      cell_off = hsz == 0 ? G::WZ - 1 : 0;
      mstride = G::E_C;
      sel_z = hsz == 0 ? 2 : 0;
    } else {
      piece_off = hi ? G::OFF_YHI : G::OFF_YLO;
      cell_off = hsz - 1;
      mstride = G::E_YE;
    }
  } else if (has_halo) {
    const int j = tid - 2 * BZ;
    const bool hi = j >= TY;
    hsy = (hi ? j - TY : j) + 1;
    hsz = hi ? BZ - 1 : 0;
    piece_off = hi ? G::OFF_ZHI : G::OFF_ZLO;
    cell_off = (hsy - 1) * G::WZ + (hi ? 0 : G::WZ - 1);
    mstride = G::E_ZE;
    sel_z = hi ? 0 : 2;
  }
  const int h_idx = hsy * BZ + hsz;
  const long long N = a.N;
  const long long plane = (long long)a.ny * a.nz;
  T* post = static_cast<T*>(a.post);
  const R omega = R(1) / (R(a.vis_shear) * R(3) + R(0.5));

  if (tid == 0) {
    for (int k = 0; k < NSTAGE; ++k) mbar_init(saddr(&bars[k]), 1);
    fence_mbar_init();
  }
  __syncthreads();

  double mass = 0.0;
  int bad = 0;
  bool timed_out = false;
  // running plane counter: plane q is staged in slot q % NSTAGE and its mbarrier completes
  // for the (q / NSTAGE)-th time
  int slot = 0, phase = 0;

  auto issue = [&](int xs, int q_slot) {
    // thread 0: nine boxes of plane xs into stage q_slot
    unsigned char* st = smem + q_slot * G::STAGE_BYTES;
    const unsigned bar = saddr(&bars[q_slot]);
    int gx = xs;
    if (PERIODIC) gx = gx < 0 ? gx + a.nx : (gx >= a.nx ? gx - a.nx : gx);
    const int zl = box_c[0], z0 = box_c[1], zh = box_c[2], yl = box_c[3], y0 = box_c[4], yh = box_c[5];
    fence_proxy_async();
    mbar_expect_tx(bar, G::TX_BYTES);
    tma_load4(saddr(st + G::OFF_MID), &maps.mid, z0, y0, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_YLO), &maps.yedge, z0, yl, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_YHI), &maps.yedge, z0, yh, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_ZLO), &maps.zedge, zl, y0, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_ZHI), &maps.zedge, zh, y0, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_C + 0 * G::B_C), &maps.corner, zl, yl, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_C + 1 * G::B_C), &maps.corner, zh, yl, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_C + 2 * G::B_C), &maps.corner, zl, yh, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_C + 3 * G::B_C), &maps.corner, zh, yh, gx, 0, bar);
  };

  for (int item = blockIdx.x; item < a.n_items; item += gridDim.x) {
    const int tile = item % a.n_tiles, chunk = item / a.n_tiles;
    const int y0 = (tile / a.tiles_z) * TY, z0 = (tile % a.tiles_z) * TZ;
    const int xb = chunk * a.chunk_len;
    const int xe = min(xb + a.chunk_len, a.nx);
    const int hgy = y0 - 1 + hsy, hgz = z0 - 1 + hsz;
    const bool h_in = PERIODIC || (hgy >= 0 && hgy < a.ny && hgz >= 0 && hgz < a.nz);
    const int dy = y0 + ty, dz = z0 + tz;
    if (tid == 0) {
      int zl = z0 - G::WZ, zh = z0 + TZ, yl = y0 - 1, yh = y0 + TY;
      if (PERIODIC) {
        if (zl < 0) zl += a.nz;
        if (zh >= a.nz) zh -= a.nz;
        if (yl < 0) yl += a.ny;
        if (yh >= a.ny) yh -= a.ny;
      }
      box_c[0] = zl;
      box_c[1] = z0;
      box_c[2] = zh;
      box_c[3] = yl;
      box_c[4] = y0;
      box_c[5] = yh;
      // fill the pipeline: planes xb-1 .. xb+NSTAGE-3 into the next NSTAGE-1 slots
      int s = slot;
      for (int k = 0; k < NSTAGE - 1 && xb - 1 + k <= xe; ++k) {
        issue(xb - 1 + k, s);
        s = s + 1 == NSTAGE ? 0 : s + 1;
      }
    }
    Acc<R> acc_cur, acc_next;
    acc_cur.zero();
    acc_next.zero();
    for (int xs = xb - 1; xs <= xe; ++xs) {
      __syncthreads();  // the mailbox is free and the stage read last iteration can be refilled
      if (tid == 0 && xs + NSTAGE - 1 <= xe) issue(xs + NSTAGE - 1, slot == 0 ? NSTAGE - 1 : slot - 1);
      {
        const unsigned bar = saddr(&bars[slot]);
        long long spin = 0;
        while (!mbar_try_wait(bar, unsigned(phase))) {
          if (++spin > MAX_SPIN) {  // the copy never landed: report, keep the barriers matched
            timed_out = true;
            break;
          }
        }
      }
      const bool x_in = PERIODIC || (xs >= 0 && xs < a.nx);
      const unsigned char* stage = smem + slot * G::STAGE_BYTES;
      {  // interior source cell (tiles are full, so always inside the y/z range)
        Mom3<R> m;
        if (x_in) {
          const T* p = reinterpret_cast<const T*>(stage + G::OFF_MID) + tid;
          R raw[10];
#pragma unroll
          for (int k = 0; k < 10; ++k) raw[k] = S::to_r(p[k * G::E_MID]);
          m = decode3<S>(raw, a.sc);
        } else {
          m = zero_cell<R>();
        }
        R f[27];
        rebuild_all<R>(m, f);
#pragma unroll
        for (int d = 0; d < 27; ++d) mb[d * NSRC + dsrc] = f[d];
      }
      if (has_halo) {
        Mom3<R> m;
        if (x_in && h_in) {
          const T* p = reinterpret_cast<const T*>(stage + piece_off) + cell_off;
          R raw[10];
#pragma unroll
          for (int k = 0; k < 10; ++k) raw[k] = S::to_r(p[k * mstride]);
          m = decode3<S>(raw, a.sc);
        } else {
          m = zero_cell<R>();
        }
        rebuild_slice<R>(m, sel_y, sel_z, [&](int d, R v) { mb[d * NSRC + h_idx] = v; });
      }
      __syncthreads();  // mailbox complete
      Acc<R> acc_new;
      acc_new.zero();
#pragma unroll
      for (int xi = 0; xi < 3; ++xi) {
        R p[3][3];
#pragma unroll
        for (int yi = 0; yi < 3; ++yi)
#pragma unroll
          for (int zi = 0; zi < 3; ++zi)
            p[yi][zi] = mb[((xi * 3 + yi) * 3 + zi) * NSRC + dsrc - (yi - 1) * BZ - (zi - 1)];
        if (xi == 0) accumulate_group<R>(acc_cur, p, -1);
        else if (xi == 1) accumulate_group<R>(acc_next, p, 0);
        else accumulate_group<R>(acc_new, p, 1);
      }
      const int dx = xs - 1;
      if (dx >= xb) {
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
          for (int k = 0; k < 10; ++k) post[k * N + c] = S::from_r(raw[k]);
          if (DIAG) {
            mass += double(m.rho);
            bad += healthy<R>(m) ? 0 : 1;
          }
        }
      }
      acc_cur = acc_next;
      acc_next = acc_new;
      slot = slot + 1 == NSTAGE ? 0 : slot + 1;
      if (slot == 0) phase ^= 1;
    }
  }
  if (timed_out && a.status) atomicExch(a.status, HL_ERR_TIMEOUT);
  __syncthreads();

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

// ---------------------------------------------------------------- host side
CUtensorMapDataType tmap_dtype(hl_dtype d) {
  switch (d) {
    case HL_F32: return CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    case HL_F64: return CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    case HL_F16: return CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    default: return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  }
}

size_t esize(hl_dtype d) { return d == HL_F64 ? 8 : d == HL_F32 ? 4 : 2; }

// Tensor maps over the (nz, ny, nx, 10) moment array (innermost first); cached per buffer.
int encode_maps(const hl_world3d* w, Maps* out) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, const void*, int, int, int, int>, Maps> cache;
  const auto key = std::make_tuple(w->cur, static_cast<const void*>(w->post), w->nx, w->ny, w->nz, int(w->storage.dtype));
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      *out = it->second;
      return HL_OK;
    }
  }
  const size_t es = esize(w->storage.dtype);
  const int wz = int(16 / es);
  const cuuint64_t dims[4] = {cuuint64_t(w->nz), cuuint64_t(w->ny), cuuint64_t(w->nx), 10};
  const cuuint64_t strides[3] = {cuuint64_t(w->nz) * es, cuuint64_t(w->ny) * w->nz * es,
                                 cuuint64_t(w->nx) * w->ny * w->nz * es};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const cuuint32_t boxes[4][4] = {{TZ, TY, 1, 10}, {TZ, 1, 1, 10}, {cuuint32_t(wz), TY, 1, 10}, {cuuint32_t(wz), 1, 1, 10}};
  // the driver entry point is resolved at run time, so the library loads without a driver
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (encode == nullptr) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || fn == nullptr) {
      set_error("d3q27: cuTensorMapEncodeTiled is unavailable (%s)", cudaGetErrorString(e));
      return HL_ERR_CUDA;
    }
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  CUtensorMap* dst[4] = {&out->mid, &out->yedge, &out->zedge, &out->corner};
  for (int k = 0; k < 4; ++k) {
    void* base = const_cast<void*>(w->cur);
    const CUresult r = encode(dst[k], tmap_dtype(w->storage.dtype), 4, base, dims,
                                              strides, boxes[k], estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      set_error("d3q27: cuTensorMapEncodeTiled failed (%d)", int(r));
      return HL_ERR_CUDA;
    }
  }
  std::lock_guard<std::mutex> lk(mu);
  if (cache.size() > 64) cache.clear();
  cache[key] = *out;
  return HL_OK;
}

template <class S, int NSTAGE, bool PERIODIC, bool FORCE, bool FLAGS, bool DIAG>
int launch(const hl_world3d* w, double vis, const hl_diag* diag, cudaStream_t st) {
  using G = Geo<typename S::T, NSTAGE>;
  Maps maps;
  int rc = encode_maps(w, &maps);
  if (rc != HL_OK) return rc;
  StepArgs a{};
  a.cur = w->cur;
  a.post = w->post;
  a.N = (long long)w->nx * w->ny * w->nz;
  a.nx = w->nx;
  a.ny = w->ny;
  a.nz = w->nz;
  a.tiles_y = w->ny / TY;
  a.tiles_z = w->nz / TZ;
  a.n_tiles = a.tiles_y * a.tiles_z;
  // x split (tuning override HL_D3_CHUNKS): all CTAs march x in step for L2 reuse of halos
  const int sms = num_sms();
  const int forced = g_tune_d3_chunks;
  int best_c = 1;
  double best = -1;
  for (int c = 1; c <= 64 && c <= w->nx; ++c) {
    if (forced > 0 && c != forced) continue;
    const int len = (w->nx + c - 1) / c;
    const int items = a.n_tiles * ((w->nx + len - 1) / len);
    const int waves = (items + sms - 1) / sms;
    const double eff = double(items) / (double(waves) * sms) * double(len) / double(len + 2);
    if (eff > best + 1e-9) {
      best = eff;
      best_c = c;
    }
  }
  a.chunk_len = (w->nx + best_c - 1) / best_c;
  a.n_items = a.n_tiles * ((w->nx + a.chunk_len - 1) / a.chunk_len);
  a.vis_shear = vis;
  a.force = w->force;
  a.flag = w->flag;
  a.sc = make_scale(w->storage);
  if (DIAG) fill_diag(a, diag);
  auto kern = step_kernel_tma<S, NSTAGE, PERIODIC, FORCE, FLAGS, DIAG>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(d3q27 tma)");
    attr = true;
  }
  const int grid = a.n_items < sms ? a.n_items : sms;
  kern<<<grid, THREADS, G::SMEM, st>>>(a, maps);
  HL_LAUNCH_CHECK("d3q27 stream_collide (tma) launch");
  return HL_OK;
}

template <class S, int NS> int dispatch(const hl_world3d* w, double vis, const hl_diag* d, cudaStream_t st) {
  const bool P = w->periodic != 0, F = w->force != nullptr, G = w->flag != nullptr && !P,
             D = d != nullptr && d->scratch != nullptr;
#define HL_T_CASE(p, f, g, dg) \
  if (P == p && F == f && G == g && D == dg) return launch<S, NS, p, f, g, dg>(w, vis, d, st);
  HL_T_CASE(true, false, false, false)
  HL_T_CASE(true, false, false, true)
  HL_T_CASE(true, true, false, false)
  HL_T_CASE(true, true, false, true)
  HL_T_CASE(false, false, false, false)
  HL_T_CASE(false, false, false, true)
  HL_T_CASE(false, true, false, false)
  HL_T_CASE(false, true, false, true)
  HL_T_CASE(false, false, true, false)
  HL_T_CASE(false, false, true, true)
  HL_T_CASE(false, true, true, false)
  HL_T_CASE(false, true, true, true)
#undef HL_T_CASE
  set_error("d3q27 (tma): unsupported option combination");
  return HL_ERR_UNSUPPORTED;
}

}  // namespace tma

bool tma_eligible(const hl_world3d* w) {
  if (w->storage.dtype == HL_F64) return false;
  if (w->ny % tma::TY != 0 || w->nz % tma::TZ != 0) return false;
  const size_t es = tma::esize(w->storage.dtype);
  if ((reinterpret_cast<uintptr_t>(w->cur) & 15) != 0 || (reinterpret_cast<uintptr_t>(w->post) & 15) != 0) return false;
  return (size_t(w->nz) * es) % 16 == 0;
}

template <int NS> int launch_ns(const hl_world3d* w, double vis, const hl_diag* diag, cudaStream_t st) {
  switch (w->storage.dtype) {
    case HL_F32: return tma::dispatch<StoreF32, NS>(w, vis, diag, st);
    case HL_F16: return tma::dispatch<StoreF16, NS>(w, vis, diag, st);
    case HL_BF16: return tma::dispatch<StoreBF16, NS>(w, vis, diag, st);
    default: break;
  }
  set_error("d3q27 (tma): dtype not supported");
  return HL_ERR_UNSUPPORTED;
}

int launch_step_tma(const hl_world3d* w, double vis, const hl_diag* diag, cudaStream_t st) {
  // pipeline depth: 4 stages (three planes in flight) unless tuned
  switch (g_tune_d3_stages) {
    case 3: return launch_ns<3>(w, vis, diag, st);
    case 5: return launch_ns<5>(w, vis, diag, st);
    default: return launch_ns<4>(w, vis, diag, st);
  }
  set_error("d3q27 (tma): dtype not supported");
  return HL_ERR_UNSUPPORTED;
}

}  // namespace d3
}  // namespace hl
