// D3Q27 stream-collide with TMA-staged source planes and paired-plane arithmetic (sm_100a).
//
// Same algorithm as the fallback kernel in d3q27.cu (source-side population rebuild,
// exchange through a shared-memory mailbox, x-marching columns). Two things differ.
//
// Staging: one elected thread issues nine tensor-memory-access (TMA) box copies per plane,
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
// Pairs of planes: each thread owns one (y, z) column of the 16 x 32 tile and handles two
// consecutive source planes per iteration. Every quantity is a pair (lane 0 plane s0, lane 1
// plane s0 + 1), so each arithmetic instruction is a packed FADD2 / FMUL2 / FFMA2 serving two
// cells, and the mailbox entries are 8-byte pairs. A thread rebuilds the 27 populations of
// its cell pair, keeps the three with c_y = c_z = 0 in registers and writes the other 24 to
// the mailbox slots of the destination cell, the three c_x of one (c_y, c_z) direction as one
// 16-byte and one 8-byte entry (threads 0..99 add the 9 or 3 populations a halo cell sends into
// the tile). After a block barrier each thread reads its 24 incoming pairs,
// forms the sums of the c_x = -1, 0, +1 groups, and completes the destination planes s0 - 1
// and s0 from them and from the previous pair's sums. Four stages keep the next pair in
// flight while the current one is computed. One block barrier per pair (mailbox written); the
// mailbox's reuse by the next pair is a split arrive/wait on an mbarrier.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <algorithm>
#include <vector>

#include "d3q27_core.cuh"
#include "d3q27_pair.cuh"

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
  static constexpr int MB_BYTES = 24 * NDST * 8;  // mailbox: 24 directions x 512 cells x 2 planes
  static constexpr int MB_OFF = NSTAGE * STAGE_BYTES;
  static constexpr int BAR_OFF = MB_OFF + MB_BYTES;  // mbarriers
  static constexpr int SMEM = BAR_OFF + NSTAGE * 8 + 16 + 128;  // + alignment slack
};

struct Maps {
  CUtensorMap mid, yedge, zedge, corner;  // over the current buffer
};

// One domain of a batched launch (device memory, 64-byte aligned like the maps in it): the
// tensor maps over each of its two buffers (parity p reads buf[p] and writes buf[p ^ 1]), its
// sizes and x split, and the first of its items in the batch's item sequence.
struct BatchDomain {
  Maps maps[2];
  void* buf[2];
  long long N;
  int nx, ny, nz, tiles_z, n_tiles, chunk_len, n_items, item_base;
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
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
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
// Tensor maps read from global memory: make the copy written before the launch visible to the
// tensor-map proxy before the first copy through it.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(reinterpret_cast<unsigned long long>(m))
               : "memory");
}

// ---------------------------------------------------------------- kernel
// Mailbox slot of direction (xi, yi, zi) with (yi, zi) != (1, 1): the populations a
// destination receives from a y/z neighbour, indexed by (direction, destination cell).
__host__ __device__ constexpr int mb_dir(int xi, int yi, int zi) {
  return xi * 8 + ((yi * 3 + zi) < 4 ? (yi * 3 + zi) : (yi * 3 + zi - 1));
}

// Sums of one direction group (fixed c_x) over its 9 populations p[yi][zi], for the pair
// of source planes: the parts of rho, j_y, j_z, Pi_yy, Pi_zz, Pi_yz it contributes (and, for
// c_x = -1 / +1, of rho * c_x, Pi_xx, Pi_xy, Pi_xz through its sign).
struct GroupSums {
  P2 m0, my, myy, mz, mzz, myz;
};

__device__ __forceinline__ GroupSums group_sums(const P2 p[3][3]) {
  const P2 ry0 = p[0][0] + p[0][1] + p[0][2];
  const P2 ry1 = p[1][0] + p[1][1] + p[1][2];
  const P2 ry2 = p[2][0] + p[2][1] + p[2][2];
  const P2 cz0 = p[0][0] + p[1][0] + p[2][0];
  const P2 cz2 = p[0][2] + p[1][2] + p[2][2];
  GroupSums g;
  g.myy = ry2 + ry0;
  g.my = ry2 - ry0;
  g.m0 = g.myy + ry1;
  g.mzz = cz2 + cz0;
  g.mz = cz2 - cz0;
  g.myz = (p[2][2] + p[0][0]) - (p[2][0] + p[0][2]);
  return g;
}

// Raw stored planes of a cell pair -> physical moments (decode3 of hl_common.cuh, per lane).
template <class S> __device__ __forceinline__ Mom3<P2> decode_pair(const P2 raw[10], const Scale& sc) {
  Mom3<P2> m;
  if constexpr (S::kEncoded) {
    const P2 su(sc.u), ss(sc.s);
    m.drho = raw[0];
    m.rho = raw[0] + P2(1.0);
    m.ux = raw[1] * su;
    m.uy = raw[2] * su;
    m.uz = raw[3] * su;
    m.sxx = raw[4] * ss + m.ux * m.ux;
    m.syy = raw[5] * ss + m.uy * m.uy;
    m.szz = raw[6] * ss + m.uz * m.uz;
    m.sxy = raw[7] * ss + m.ux * m.uy;
    m.sxz = raw[8] * ss + m.ux * m.uz;
    m.syz = raw[9] * ss + m.uy * m.uz;
  } else {
    m.rho = raw[0];
    m.drho = raw[0] - P2(1.0);
    m.ux = raw[1];
    m.uy = raw[2];
    m.uz = raw[3];
    m.sxx = raw[4];
    m.syy = raw[5];
    m.szz = raw[6];
    m.sxy = raw[7];
    m.sxz = raw[8];
    m.syz = raw[9];
  }
  return m;
}

// Physical moments of a cell pair -> raw stored planes (encode3 of hl_common.cuh, per lane).
template <class S> __device__ __forceinline__ void encode_pair(const Mom3<P2>& m, const Scale& sc, P2 raw[10]) {
  if constexpr (S::kEncoded) {
    const P2 iu(sc.inv_u), is(sc.inv_s);
    raw[0] = m.drho;
    raw[1] = m.ux * iu;
    raw[2] = m.uy * iu;
    raw[3] = m.uz * iu;
    raw[4] = (m.sxx - m.ux * m.ux) * is;
    raw[5] = (m.syy - m.uy * m.uy) * is;
    raw[6] = (m.szz - m.uz * m.uz) * is;
    raw[7] = (m.sxy - m.ux * m.uy) * is;
    raw[8] = (m.sxz - m.ux * m.uz) * is;
    raw[9] = (m.syz - m.uy * m.uz) * is;
  } else {
    raw[0] = m.rho;
    raw[1] = m.ux;
    raw[2] = m.uy;
    raw[3] = m.uz;
    raw[4] = m.sxx;
    raw[5] = m.syy;
    raw[6] = m.szz;
    raw[7] = m.sxy;
    raw[8] = m.sxz;
    raw[9] = m.syz;
  }
}

// Raw planes of one cell of a staged plane (k-th moment plane at p[k * stride]). A cell
// outside a walled domain must read as the zero cell. The TMA unit zero-fills boxes outside
// the tensor, which IS the zero cell of float32 storage (rho = 0, drho = -1); the encoded
// storages store rho - 1 and need the select (SEL) where an outside cell can feed a stored
// one: with a flag array (a border cell may be fluid). Without one, only the interior cells
// are stored and all their neighbours lie inside, so what an outside cell sends reaches only
// border cells, which are never stored. A lane past the last source plane of an item holds
// stale data: its populations only reach destinations that are never stored.
template <class S, bool SEL>
__device__ __forceinline__ void load_raw(const typename S::T* p0, const typename S::T* p1, int stride, bool in0,
                                         bool in1, P2 raw[10]) {
  const float z0 = S::kEncoded ? -1.f : 0.f;  // raw rho plane of the zero cell
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    const float zk = k == 0 ? z0 : 0.f;
    const float v0 = S::to_r(p0[k * stride]), v1 = S::to_r(p1[k * stride]);
    raw[k] = SEL ? P2(in0 ? v0 : zk, in1 ? v1 : zk) : P2(v0, v1);
  }
}

// BATCH: the items belong to the domains of doms[0 .. n_doms) (their item ranges in order);
// a's sizes, buffers and item count are unused except n_items (the batch's total), and each
// item takes its domain's sizes, buffers and maps at parity `parity`. Walled domains only.
template <class S, int NSTAGE, bool PERIODIC, bool FORCE, bool FLAGS, bool DIAG, bool BATCH>
__global__ void __launch_bounds__(THREADS, 1)
    step_kernel_tma(const StepArgs a, const __grid_constant__ Maps maps, const BatchDomain* __restrict__ doms,
                    int n_doms, int parity) {
  static_assert(!BATCH || (!PERIODIC && !FORCE && !FLAGS && !DIAG), "batched launches: walled domains, no fields");
  using T = typename S::T;
  static_assert(sizeof(typename S::R) == 4, "the paired kernel computes in binary32");
  using G = Geo<T, NSTAGE>;
  constexpr bool SEL = S::kEncoded && !PERIODIC && FLAGS;  // see load_raw
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + G::BAR_OFF);
  // mailbox by (c_y, c_z) direction (8) and destination (512): the c_x = -1 and 0 populations as
  // one 16-byte entry, the c_x = +1 one as an 8-byte entry (one STS.128 + one STS.64 per
  // direction instead of three STS.64, and the same for the loads)
  float4* mbA = reinterpret_cast<float4*>(smem + G::MB_OFF);                // [8][512]
  P2* mbB = reinterpret_cast<P2*>(smem + G::MB_OFF + 8 * NDST * 16);       // [8][512]

  const int tid = threadIdx.x;
  const int ty = tid / TZ, tz = tid % TZ;
  // which y/z neighbours of this thread's cell lie inside the tile
  const bool yl_ok = ty > 0, yh_ok = ty < TY - 1, zl_ok = tz > 0, zh_ok = tz < TZ - 1;
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
  const int hy = hsy - 1, hz = hsz - 1;  // halo cell in tile coordinates
  // The halo cell sends one face slice into the tile: a row cell (y0-1 or y0+16) the
  // populations with c_y = hs, a column cell (z0-1 or z0+32) those with c_z = hs; entry i of
  // the slice has the other component i - 1. Its mailbox rows and destination slots:
  const bool h_row = tid < 2 * BZ;
  const int hs = h_row ? (hy < 0 ? 1 : -1) : (hz < 0 ? 1 : -1);
  int h_dir[3], h_dst[3];
  bool h_ok[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int yi = h_row ? hs + 1 : i, zi = h_row ? i : hs + 1;
    const int idx = yi * 3 + zi;
    h_dir[i] = idx < 4 ? idx : idx - 1;  // mb_dir(0, yi, zi)
    const int ddy = hy + yi - 1, ddz = hz + zi - 1;
    h_ok[i] = has_halo && ddy >= 0 && ddy < TY && ddz >= 0 && ddz < TZ;
    h_dst[i] = ddy * TZ + ddz;
  }
  // the current item's domain (fixed for a single-domain launch)
  long long N = a.N;
  long long plane = (long long)a.ny * a.nz;
  int nx = a.nx, ny = a.ny, nz = a.nz;
  T* post = static_cast<T*>(a.post);
  const PairConst kc = make_pair_const(1.f / (float(a.vis_shear) * 3.f + 0.5f));

  if (tid == 0) {
    for (int k = 0; k < NSTAGE; ++k) mbar_init(saddr(&bars[k]), 1);
    mbar_init(saddr(&bars[NSTAGE]), THREADS / 32);  // mailbox read by every warp
    fence_mbar_init();
  }
  __syncthreads();

  double mass = 0.0;
  int bad = 0;
  bool timed_out = false;
  // The CTA's source planes form one sequence over all its items (per item xb-1 .. xe).
  // Plane q of the sequence is staged in slot q % NSTAGE, whose mbarrier completes for the
  // (q / NSTAGE)-th time. Thread 0 produces the sequence NSTAGE planes ahead of the
  // consumers, across item boundaries, so a new item starts with its planes already staged.
  int slot = 0, phase = 0;                                  // consumer position
  int p_item = blockIdx.x, p_x = 0, p_xe = 0, p_slot = 0;  // producer position (thread 0)
  int p_y0 = 0, p_z0 = 0, p_dom = -1;
  const Maps* p_maps = &maps;
  // the domain of a batch item: the last one whose item range starts at or before it
  auto find_dom = [&](int item) {
    int lo = 0, hi = n_doms - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (doms[mid].item_base <= item) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  };
  auto item_range = [&](int item, int& y0, int& z0, int& xb, int& xe, int& dom) {
    if constexpr (BATCH) {
      dom = find_dom(item);
      const BatchDomain& D = doms[dom];
      const int local = item - D.item_base;
      const int tile = local % D.n_tiles, chunk = local / D.n_tiles;
      y0 = (tile / D.tiles_z) * TY;
      z0 = (tile % D.tiles_z) * TZ;
      xb = chunk * D.chunk_len;
      xe = min(xb + D.chunk_len, D.nx);
    } else {
      dom = 0;
      const int tile = item % a.n_tiles, chunk = item / a.n_tiles;
      y0 = (tile / a.tiles_z) * TY;
      z0 = (tile % a.tiles_z) * TZ;
      xb = chunk * a.chunk_len;
      xe = min(xb + a.chunk_len, a.nx);
    }
  };
  // thread 0: the maps of the producer's current item (batch: acquired once per domain change)
  auto producer_maps = [&](int dom) {
    if constexpr (BATCH) {
      if (dom != p_dom) {
        p_dom = dom;
        p_maps = &doms[dom].maps[parity];
        tensormap_acquire(&p_maps->mid);
        tensormap_acquire(&p_maps->yedge);
        tensormap_acquire(&p_maps->zedge);
        tensormap_acquire(&p_maps->corner);
      }
    }
  };
  auto issue = [&](int xs, int q_slot, int y0, int z0) {
    // nine boxes of plane xs of the tile at (y0, z0) into stage q_slot
    unsigned char* st = smem + q_slot * G::STAGE_BYTES;
    const unsigned bar = saddr(&bars[q_slot]);
    int gx = xs;
    if (PERIODIC) gx = gx < 0 ? gx + a.nx : (gx >= a.nx ? gx - a.nx : gx);
    int zl = z0 - G::WZ, zh = z0 + TZ, yl = y0 - 1, yh = y0 + TY;
    if (PERIODIC) {
      if (zl < 0) zl += a.nz;
      if (zh >= a.nz) zh -= a.nz;
      if (yl < 0) yl += a.ny;
      if (yh >= a.ny) yh -= a.ny;
    }
    fence_proxy_async();
    mbar_expect_tx(bar, G::TX_BYTES);
    const Maps& m = *p_maps;
    tma_load4(saddr(st + G::OFF_MID), &m.mid, z0, y0, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_YLO), &m.yedge, z0, yl, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_YHI), &m.yedge, z0, yh, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_ZLO), &m.zedge, zl, y0, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_ZHI), &m.zedge, zh, y0, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_C + 0 * G::B_C), &m.corner, zl, yl, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_C + 1 * G::B_C), &m.corner, zh, yl, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_C + 2 * G::B_C), &m.corner, zl, yh, gx, 0, bar);
    tma_load4(saddr(st + G::OFF_C + 3 * G::B_C), &m.corner, zh, yh, gx, 0, bar);
  };
  auto produce = [&](int n) {  // thread 0: the next n planes of the sequence
    for (int k = 0; k < n && p_item < a.n_items; ++k) {
      issue(p_x, p_slot, p_y0, p_z0);
      p_slot = p_slot + 1 == NSTAGE ? 0 : p_slot + 1;
      if (++p_x > p_xe) {
        p_item += gridDim.x;
        if (p_item < a.n_items) {
          int xb, dom;
          item_range(p_item, p_y0, p_z0, xb, p_xe, dom);
          producer_maps(dom);
          p_x = xb - 1;
        }
      }
    }
  };
  if (tid == 0 && p_item < a.n_items) {
    int xb, dom;
    item_range(p_item, p_y0, p_z0, xb, p_xe, dom);
    producer_maps(dom);
    p_x = xb - 1;
    produce(NSTAGE);
  }
  // The mailbox is written by every thread before barrier 1 and read after it. Instead of a
  // second block barrier before the next pair's writes, each warp arrives on bars[NSTAGE] once
  // it has read its entries, and a thread waits for the phase only before its next writes: a
  // warp that finished reading goes on to its collision, stores and next rebuild while the
  // others still read.
  const unsigned mb_empty = saddr(&bars[NSTAGE]);
  int mb_phase = 0;
  bool mb_written = false;
  auto wait_mailbox_empty = [&]() {
    if (mb_written) {
      long long spin = 0;
      while (!mbar_try_wait(mb_empty, unsigned(mb_phase))) {
        if (++spin > MAX_SPIN) {
          timed_out = true;
          break;
        }
      }
      mb_phase ^= 1;
    }
    mb_written = true;
  };
  auto wait_stage = [&](int q_slot, int q_phase) {
    const unsigned bar = saddr(&bars[q_slot]);
    long long spin = 0;
    while (!mbar_try_wait(bar, unsigned(q_phase))) {
      if (++spin > MAX_SPIN) {  // the copy never landed: report, keep the barriers matched
        timed_out = true;
        break;
      }
    }
  };

  for (int item = blockIdx.x; item < a.n_items; item += gridDim.x) {
    int y0, z0, xb, xe, dom;
    item_range(item, y0, z0, xb, xe, dom);
    if constexpr (BATCH) {
      const BatchDomain& D = doms[dom];
      N = D.N;
      nx = D.nx;
      ny = D.ny;
      nz = D.nz;
      plane = (long long)D.ny * D.nz;
      post = static_cast<T*>(D.buf[parity ^ 1]);
    }
    const int hgy = y0 - 1 + hsy, hgz = z0 - 1 + hsz;
    const bool h_in = PERIODIC || (hgy >= 0 && hgy < ny && hgz >= 0 && hgz < nz);
    const int dy = y0 + ty, dz = z0 + tz;
    const int cyz = dy * nz + dz;  // the thread's cell within an x plane
    // group sums of the previous pair that the next destinations still need: all of c_x = +1,
    // the second plane's of c_x = 0
    GroupSums gp_prev;
    gp_prev.m0 = gp_prev.my = gp_prev.myy = gp_prev.mz = gp_prev.mzz = gp_prev.myz = P2(0.f, 0.f);
    float z_m0 = 0.f, z_my = 0.f, z_myy = 0.f, z_mz = 0.f, z_mzz = 0.f, z_myz = 0.f;

    // Source planes in pairs (s0, s0 + 1); lane 0 of every P2 is plane s0, lane 1 plane s0 + 1.
    for (int s0 = xb - 1; s0 <= xe; s0 += 2) {
      const int s1 = s0 + 1;
      const bool has1 = s1 <= xe;  // false: lane 1 is past the last source plane
      const int slot0 = slot, ph0 = phase;
      slot = slot + 1 == NSTAGE ? 0 : slot + 1;
      if (slot == 0) phase ^= 1;
      const int slot1 = slot, ph1 = phase;
      if (has1) {
        slot = slot + 1 == NSTAGE ? 0 : slot + 1;
        if (slot == 0) phase ^= 1;
      }
      wait_stage(slot0, ph0);
      if (has1) wait_stage(slot1, ph1);
      const bool in0 = PERIODIC || (s0 >= 0 && s0 < nx);
      const bool in1 = has1 && (PERIODIC || (s1 >= 0 && s1 < nx));
      const unsigned char* st0 = smem + slot0 * G::STAGE_BYTES;
      const unsigned char* st1 = smem + slot1 * G::STAGE_BYTES;

      P2 fc[3];  // populations that stay in this column (c_y = c_z = 0)
      {          // interior source cells (tiles are full, so always inside the y/z range)
        P2 raw[10];
        load_raw<S, SEL>(reinterpret_cast<const T*>(st0 + G::OFF_MID) + tid, reinterpret_cast<const T*>(st1 + G::OFF_MID) + tid,
                    G::E_MID, in0, in1, raw);
        const Coef cf = coefficients(decode_pair<S>(raw, a.sc), kc);
        wait_mailbox_empty();
        P2 f[27];
        rebuild_pair(cf, kc, f);
#pragma unroll
        for (int xi = 0; xi < 3; ++xi) fc[xi] = f[dir_index(xi - 1, 0, 0)];
#pragma unroll
        for (int yi = 0; yi < 3; ++yi)
#pragma unroll
          for (int zi = 0; zi < 3; ++zi) {
            if (yi == 1 && zi == 1) continue;
            const bool ok = (yi == 0 ? yl_ok : yi == 2 ? yh_ok : true) && (zi == 0 ? zl_ok : zi == 2 ? zh_ok : true);
            if (ok) {
              const int e = mb_dir(0, yi, zi) * NDST + tid + (yi - 1) * TZ + (zi - 1);
              const P2 a0 = f[(0 * 3 + yi) * 3 + zi], a1 = f[(1 * 3 + yi) * 3 + zi];
              mbA[e] = make_float4(a0.x(), a0.y(), a1.x(), a1.y());
              mbB[e] = f[(2 * 3 + yi) * 3 + zi];
            }
          }
      }
      if (has_halo) {
        P2 raw[10];
        load_raw<S, SEL>(reinterpret_cast<const T*>(st0 + piece_off) + cell_off,
                    reinterpret_cast<const T*>(st1 + piece_off) + cell_off, mstride, in0 && h_in, in1 && h_in, raw);
        const Coef cf = coefficients(decode_pair<S>(raw, a.sc), kc);
        P2 f[3][3];
        rebuild_face(cf, kc, h_row, P2(float(hs), float(hs)), f);
#pragma unroll
        for (int i = 0; i < 3; ++i)
          if (h_ok[i]) {
            const int e = h_dir[i] * NDST + h_dst[i];
            mbA[e] = make_float4(f[i][0].x(), f[i][0].y(), f[i][1].x(), f[i][1].y());
            mbB[e] = f[i][2];
          }
      }
      __syncthreads();  // mailbox complete; every thread is done with both stages
      if (tid == 0) produce(has1 ? 2 : 1);

      GroupSums g[3];
      {
        P2 p[3][3][3];  // [xi][yi][zi]
#pragma unroll
        for (int yi = 0; yi < 3; ++yi)
#pragma unroll
          for (int zi = 0; zi < 3; ++zi) {
            if (yi == 1 && zi == 1) {
#pragma unroll
              for (int xi = 0; xi < 3; ++xi) p[xi][1][1] = fc[xi];
              continue;
            }
            const int e = mb_dir(0, yi, zi) * NDST + tid;
            const float4 a = mbA[e];
            p[0][yi][zi] = P2(a.x, a.y);
            p[1][yi][zi] = P2(a.z, a.w);
            p[2][yi][zi] = mbB[e];
          }
#pragma unroll
        for (int xi = 0; xi < 3; ++xi) g[xi] = group_sums(p[xi]);
      }
      __syncwarp();
      if ((tid & 31) == 0) mbar_arrive(mb_empty);  // this warp is done with the mailbox
      // destinations d0 = s0 - 1 and d1 = s0: c_x = -1 populations from (s0, s1), c_x = +1
      // from the previous pair (s0 - 2, s0 - 1), c_x = 0 from (s0 - 1, s0)
      const GroupSums& gm = g[0];
      Acc<P2> acc;
      const GroupSums& g0 = g[1];
      acc.pxx = gm.m0 + gp_prev.m0;
      acc.rho = acc.pxx + P2(z_m0, g0.m0.x());
      acc.jx = gp_prev.m0 - gm.m0;
      acc.jy = (gm.my + gp_prev.my) + P2(z_my, g0.my.x());
      acc.pxy = gp_prev.my - gm.my;
      acc.jz = (gm.mz + gp_prev.mz) + P2(z_mz, g0.mz.x());
      acc.pxz = gp_prev.mz - gm.mz;
      acc.pyy = (gm.myy + gp_prev.myy) + P2(z_myy, g0.myy.x());
      acc.pzz = (gm.mzz + gp_prev.mzz) + P2(z_mzz, g0.mzz.x());
      acc.pyz = (gm.myz + gp_prev.myz) + P2(z_myz, g0.myz.x());
      gp_prev = g[2];
      z_m0 = g0.m0.y();
      z_my = g0.my.y();
      z_myy = g0.myy.y();
      z_mz = g0.mz.y();
      z_mzz = g0.mzz.y();
      z_myz = g0.myz.y();

      const int d0 = s0 - 1;
      const bool v0 = d0 >= xb && d0 < xe, v1 = d0 + 1 >= xb && d0 + 1 < xe;
      if (v0 || v1) {
        const long long c0 = (long long)d0 * plane + cyz, c1 = c0 + plane;
        T* const q0 = post + c0;  // moment k of the two cells: q0[k * N], q1[k * N]
        T* const q1 = q0 + plane;
        bool f0 = v0, f1 = v1;
        if (FLAGS) {
          f0 = f0 && a.flag[c0] == ML_FLUID;
          f1 = f1 && a.flag[c1] == ML_FLUID;
        } else if (!PERIODIC) {
          const bool yz = dy > 0 && dy < ny - 1 && dz > 0 && dz < nz - 1;
          f0 = f0 && yz && d0 > 0 && d0 < nx - 1;
          f1 = f1 && yz && d0 + 1 > 0 && d0 + 1 < nx - 1;
        }
        if (f0 || f1) {
          P2 Fx(0.f, 0.f), Fy(0.f, 0.f), Fz(0.f, 0.f);
          if (FORCE) {
            Fx = P2(f0 ? a.force[c0] : 0.f, f1 ? a.force[c1] : 0.f);
            Fy = P2(f0 ? a.force[N + c0] : 0.f, f1 ? a.force[N + c1] : 0.f);
            Fz = P2(f0 ? a.force[2 * N + c0] : 0.f, f1 ? a.force[2 * N + c1] : 0.f);
          }
          const Mom3<P2> m = collide_pair<FORCE>(acc, Fx, Fy, Fz, kc);
          P2 raw[10];
          encode_pair<S>(m, a.sc, raw);
          // stochastic rounding of the reduced storages: one salt term per cell (dither_cell)
          const unsigned cs0 = unsigned(c0) * 0x9e3779b9u, cs1 = unsigned(c1) * 0x9e3779b9u;
          if constexpr (S::kEncoded) {  // both cells' moment k in one conversion, packed
            unsigned d[10];
#pragma unroll
            for (int k = 0; k < 10; ++k) d[k] = S::round2(raw[k].x(), raw[k].y(), cs0, cs1, unsigned(k));
            if (f0) {
#pragma unroll
              for (int k = 0; k < 10; ++k) q0[k * N] = S::hi(d[k]);
            }
            if (f1) {
#pragma unroll
              for (int k = 0; k < 10; ++k) q1[k * N] = S::lo(d[k]);
            }
          } else {
            if (f0) {
#pragma unroll
              for (int k = 0; k < 10; ++k) q0[k * N] = S::from_r_cell(raw[k].x(), cs0, unsigned(k));
            }
            if (f1) {
#pragma unroll
              for (int k = 0; k < 10; ++k) q1[k * N] = S::from_r_cell(raw[k].y(), cs1, unsigned(k));
            }
          }
          if (DIAG) {
            const P2 s = m.ux + m.uy + m.uz + m.sxx + m.syy + m.szz + m.sxy + m.sxz + m.syz;
            if (f0) {
              mass += double(m.rho.x());
              bad += (isfinite(m.rho.x()) && isfinite(s.x()) && m.rho.x() > 0.f) ? 0 : 1;
            }
            if (f1) {
              mass += double(m.rho.y());
              bad += (isfinite(m.rho.y()) && isfinite(s.y()) && m.rho.y() > 0.f) ? 0 : 1;
            }
          }
        }
      }
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
  auto kern = step_kernel_tma<S, NSTAGE, PERIODIC, FORCE, FLAGS, DIAG, false>;
  {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (optin > 0 && G::SMEM > optin) {
      set_error("d3q27 (tma): %d pipeline stages need %d bytes of shared memory (device limit %d)", NSTAGE, G::SMEM,
                optin);
      return HL_ERR_UNSUPPORTED;
    }
  }
  rc = set_smem_attr(reinterpret_cast<const void*>(kern), G::SMEM, "cudaFuncSetAttribute(d3q27 tma)");
  if (rc != HL_OK) return rc;
  const int grid = a.n_items < sms ? a.n_items : sms;
  kern<<<grid, THREADS, G::SMEM, st>>>(a, maps, nullptr, 0, 0);
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

// ---------------------------------------------------------------- batched domains
// Prepared descriptor arrays (device address -> domains, items), so that a launch can only
// use counts that match what was written there.
std::mutex g_batch_mu;
std::map<const void*, std::pair<int, int>> g_batches;

template <class S, int NSTAGE>
int launch_batch(const BatchDomain* doms, int n_doms, int n_items, double vis, const hl_storage& storage, int parity,
                 int* status, cudaStream_t st) {
  using G = Geo<typename S::T, NSTAGE>;
  StepArgs a{};
  a.n_items = n_items;
  a.vis_shear = vis;
  a.sc = make_scale(storage);
  a.status = status;
  Maps maps;
  std::memset(&maps, 0, sizeof(maps));
  auto kern = step_kernel_tma<S, NSTAGE, false, false, false, false, true>;
  const int rc = set_smem_attr(reinterpret_cast<const void*>(kern), G::SMEM, "cudaFuncSetAttribute(d3q27 tma batch)");
  if (rc != HL_OK) return rc;
  const int sms = num_sms();
  const int grid = n_items < sms ? n_items : sms;
  kern<<<grid, THREADS, G::SMEM, st>>>(a, maps, doms, n_doms, parity);
  HL_LAUNCH_CHECK("d3q27 stream_collide (tma batch) launch");
  return HL_OK;
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
  // pipeline depth: 4 staged planes (the pair being computed and the next pair) unless tuned
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

using namespace hl;

extern "C" size_t hl_d3q27_batch_bytes(int n_domains) {
  return n_domains > 0 ? size_t(n_domains) * sizeof(d3::tma::BatchDomain) : 0;
}

extern "C" int hl_d3q27_batch_prepare(const hl_world3d* worlds, int n_domains, void* desc, size_t desc_bytes,
                                      int* n_items, hl_stream stream) {
  using d3::tma::BatchDomain;
  HL_CHECK_ARG(worlds != nullptr && n_items != nullptr, "d3q27 batch: worlds or n_items is NULL");
  HL_CHECK_ARG(n_domains >= 1 && n_domains <= 4096, "d3q27 batch: %d domains (1 .. 4096)", n_domains);
  HL_CHECK_ARG(desc != nullptr && (reinterpret_cast<uintptr_t>(desc) & 63) == 0,
               "d3q27 batch: descriptor buffer NULL or not 64-byte aligned");
  HL_CHECK_ARG(desc_bytes >= hl_d3q27_batch_bytes(n_domains), "d3q27 batch: descriptor buffer too small (%zu < %zu)",
               desc_bytes, hl_d3q27_batch_bytes(n_domains));
  const hl_world3d& w0 = worlds[0];
  HL_CHECK_ARG(w0.storage.dtype == HL_F32 || w0.storage.dtype == HL_F16 || w0.storage.dtype == HL_BF16,
               "d3q27 batch: storage dtype %d (float32, float16 or bfloat16)", int(w0.storage.dtype));
  std::vector<BatchDomain> h;
  h.resize(size_t(n_domains));
  long long total = 0;
  for (int k = 0; k < n_domains; ++k) {
    const hl_world3d& w = worlds[k];
    HL_CHECK_ARG(w.nx >= 3 && w.ny >= 3 && w.nz >= 3, "d3q27 batch: domain %d has dims %d x %d x %d", k, w.nx, w.ny,
                 w.nz);
    HL_CHECK_ARG(w.cur != nullptr && w.post != nullptr && w.cur != w.post, "d3q27 batch: domain %d buffers", k);
    HL_CHECK_ARG(d3::tma_eligible(&w), "d3q27 batch: domain %d is not TMA-eligible (ny %% 16, nz %% 32, alignment)",
                 k);
    HL_CHECK_ARG(!w.periodic && w.force == nullptr && w.flag == nullptr,
                 "d3q27 batch: domain %d must be walled, without force or flag fields", k);
    HL_CHECK_ARG(w.storage.dtype == w0.storage.dtype && w.storage.u_scale == w0.storage.u_scale &&
                     w.storage.s_scale == w0.storage.s_scale,
                 "d3q27 batch: domain %d has another storage type or scale than domain 0", k);
    BatchDomain& d = h[size_t(k)];
    hl_world3d flip = w;
    flip.cur = w.post;
    flip.post = const_cast<void*>(w.cur);
    int rc = d3::tma::encode_maps(&w, &d.maps[0]);
    if (rc != HL_OK) return rc;
    rc = d3::tma::encode_maps(&flip, &d.maps[1]);
    if (rc != HL_OK) return rc;
    d.buf[0] = const_cast<void*>(w.cur);
    d.buf[1] = w.post;
    d.N = (long long)w.nx * w.ny * w.nz;
    d.nx = w.nx;
    d.ny = w.ny;
    d.nz = w.nz;
    d.tiles_z = w.nz / d3::tma::TZ;
    d.n_tiles = (w.ny / d3::tma::TY) * d.tiles_z;
    // x chunks of about 32 planes (or the "d3q27_chunks" override): with the items of every
    // domain to spread over the SMs, the chunks only need to be long against the two halo
    // planes each one reads
    const int chunks = g_tune_d3_chunks > 0 ? std::min(g_tune_d3_chunks, w.nx) : std::max(1, (w.nx + 16) / 32);
    d.chunk_len = (w.nx + chunks - 1) / chunks;
    d.n_items = d.n_tiles * ((w.nx + d.chunk_len - 1) / d.chunk_len);
    d.item_base = int(total);
    total += d.n_items;
    HL_CHECK_ARG(total < (1ll << 30), "d3q27 batch: too many items");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(desc, h.data(), h.size() * sizeof(BatchDomain), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "d3q27 batch: descriptor upload");
  {
    std::lock_guard<std::mutex> lk(d3::tma::g_batch_mu);
    d3::tma::g_batches[desc] = {n_domains, int(total)};
  }
  *n_items = int(total);
  return HL_OK;
}

extern "C" int hl_d3q27_stream_collide_batch(const void* desc, int n_domains, int n_items, double vis_shear,
                                             const hl_storage* storage, int parity, int* status, hl_stream stream) {
  HL_CHECK_ARG(desc != nullptr && storage != nullptr, "d3q27 batch: descriptors or storage is NULL");
  HL_CHECK_ARG(vis_shear > 0.0, "d3q27 batch: viscosity must be positive");
  HL_CHECK_ARG(parity == 0 || parity == 1, "d3q27 batch: parity %d", parity);
  {
    std::lock_guard<std::mutex> lk(d3::tma::g_batch_mu);
    auto it = d3::tma::g_batches.find(desc);
    HL_CHECK_ARG(it != d3::tma::g_batches.end() && it->second.first == n_domains && it->second.second == n_items,
                 "d3q27 batch: descriptors not prepared for %d domains and %d items", n_domains, n_items);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const auto* doms = static_cast<const d3::tma::BatchDomain*>(desc);
  switch (storage->dtype) {
    case HL_F32: return d3::tma::launch_batch<StoreF32, 4>(doms, n_domains, n_items, vis_shear, *storage, parity, status, st);
    case HL_F16: return d3::tma::launch_batch<StoreF16, 4>(doms, n_domains, n_items, vis_shear, *storage, parity, status, st);
    case HL_BF16: return d3::tma::launch_batch<StoreBF16, 4>(doms, n_domains, n_items, vis_shear, *storage, parity, status, st);
    default: break;
  }
  set_error("d3q27 batch: storage dtype %d not supported", int(storage->dtype));
  return HL_ERR_UNSUPPORTED;
}
