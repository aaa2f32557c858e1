// D3Q27 outer boundaries and initial states.
//
// apply_bc_3d (envs/lbm3d/lbm_func_3d.py:607-648) runs one thread per cell; a border cell
// applies its x face, then its y face, then its z face, each copying rho from the inward
// neighbour, setting or copying u, and extrapolating S (non-equilibrium part). On the
// reference's CPU backend threads run in launch order (x, y, z), so a cell on a low face
// (x = 0, y = 0, z = 0) reads its inward neighbour before that neighbour's own boundary
// update, and a cell on a high face reads it after. Only cells on two or three faces read
// other border cells, so the order is reproduced exactly by three parallel waves:
//   wave 1: cells on one face (they read interior cells only); cells that an edge cell will
//           read "before update" first save their old value to a snapshot slot;
//   wave 2: cells on two faces (edges), reading snapshots for low faces and wave-1 results
//           for high faces; the cell next to each low-end corner saves its old value;
//   wave 3: the 8 corners, likewise.
// Face numbering is the reference's: 0 x=0, 1 x=nx-1, 2 y=ny-1, 3 y=0, 4 z=nz-1, 5 z=0.

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "hl_common.cuh"

namespace hl {
namespace d3bc {

// reference face index of (axis, side): side 0 = low (coordinate 0), 1 = high (n-1)
__host__ __device__ constexpr int face_dr(int axis, int side) {
  return axis == 0 ? (side ? 1 : 0) : axis == 1 ? (side ? 2 : 3) : (side ? 4 : 5);
}

struct BcArgs {
  void* post;
  long long N;
  int n[3];
  int bc_type[6];
  float bc_value[6][3];
  Scale sc;
  void* snap;  // [6 faces][2][maxn][10] then [12 edges][10] raw elements
  int maxn;
};

template <class T> __device__ __forceinline__ T* face_slot(const BcArgs& a, int fid, int which, int pos) {
  return static_cast<T*>(a.snap) + ((size_t(fid) * 2 + which) * a.maxn + pos) * 10;
}
template <class T> __device__ __forceinline__ T* edge_slot(const BcArgs& a, int eid) {
  return static_cast<T*>(a.snap) + (size_t(12) * a.maxn + eid) * 10;
}

__device__ __forceinline__ long long lin(const BcArgs& a, const int c[3]) {
  return ((long long)c[0] * a.n[1] + c[1]) * a.n[2] + c[2];
}

template <class S> __device__ __forceinline__ Mom3<typename S::R> load_cell(const BcArgs& a, long long i) {
  const typename S::T* p = static_cast<const typename S::T*>(a.post);
  typename S::R raw[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) raw[k] = S::to_r(p[k * a.N + i]);
  return decode3<S>(raw, a.sc);
}
template <class S>
__device__ __forceinline__ Mom3<typename S::R> load_slot(const BcArgs& a, const typename S::T* p) {
  typename S::R raw[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) raw[k] = S::to_r(p[k]);
  return decode3<S>(raw, a.sc);
}
template <class S> __device__ __forceinline__ void copy_raw(const BcArgs& a, long long i, typename S::T* dst) {
  const typename S::T* p = static_cast<const typename S::T*>(a.post);
#pragma unroll
  for (int k = 0; k < 10; ++k) dst[k] = p[k * a.N + i];
}
template <class S> __device__ __forceinline__ void store_cell(const BcArgs& a, long long i, const Mom3<typename S::R>& m) {
  typename S::T* p = static_cast<typename S::T*>(a.post);
  typename S::R raw[10];
  encode3<S>(m, a.sc, raw);
#pragma unroll
  for (int k = 0; k < 10; ++k) p[k * a.N + i] = S::from_r(raw[k], unsigned(k * a.N + i));
}

// f_eq_home_3d (envs/lbm3d/lbm_func_3d.py:651-686): S of the unclamped second-order
// equilibrium populations f_i = w_i (rho - 1 + rho (3 c.u + 4.5 (c.u)^2 - 1.5 u^2)), from
// deviations f - w (S_aa = (P_aa - (rho-1)/3)/rho, S_ab = P_ab/rho). The D3Q27 weights give
// sum w c_a c_b = delta_ab / 3, odd moments 0 and sum w c_a c_b c_c c_d = (delta_ab delta_cd +
// delta_ac delta_bd + delta_ad delta_bc) / 9, so P_ab = (rho - 1) delta_ab / 3 + rho u_a u_b
// and S_ab = u_a u_b exactly: computed in that closed form, not as the reference's 27-term
// binary32 sums (which agree with it to their rounding). out = xx, yy, zz, xy, xz, yz.
template <class R> __device__ __forceinline__ void feq_s(R ux, R uy, R uz, R out[6]) {
  out[0] = ux * ux;
  out[1] = uy * uy;
  out[2] = uz * uz;
  out[3] = ux * uy;
  out[4] = ux * uz;
  out[5] = uy * uz;
}

// apply_bc_core_3d (envs/lbm3d/lbm_func_3d.py:627-648): new state of boundary cell t from
// its own old state and its inward neighbour nb.
template <class R> __device__ Mom3<R> bc_core(const BcArgs& a, int dr, const Mom3<R>& t, const Mom3<R>& nb) {
  Mom3<R> r = t;
  if (a.bc_type[dr] == 0) {
    r.ux = R(a.bc_value[dr][0]);
    r.uy = R(a.bc_value[dr][1]);
    r.uz = R(a.bc_value[dr][2]);
  } else if (a.bc_type[dr] == 1) {
    r.ux = nb.ux;
    r.uy = nb.uy;
    r.uz = nb.uz;
  }
  r.rho = nb.rho;
  r.drho = nb.drho;
  R sc[6], sb[6];
  feq_s<R>(r.ux, r.uy, r.uz, sc);
  feq_s<R>(nb.ux, nb.uy, nb.uz, sb);
  r.sxx = sc[0] - sb[0] + nb.sxx;
  r.syy = sc[1] - sb[1] + nb.syy;
  r.szz = sc[2] - sb[2] + nb.szz;
  r.sxy = sc[3] - sb[3] + nb.sxy;
  r.sxz = sc[4] - sb[4] + nb.sxz;
  r.syz = sc[5] - sb[5] + nb.syz;
  return r;
}

// Wave 1: cells on exactly one face, face fid = axis * 2 + side; this thread's cells are
// first, first + stride, ... of the face's interior.
template <class S> __device__ __forceinline__ void wave1_face(const BcArgs& a, int fid, long long first, long long stride) {
  using T = typename S::T;
  const int ax = fid >> 1, side = fid & 1;
  const int b = ax == 0 ? 1 : 0, c = ax == 2 ? 1 : 2;  // the other axes, increasing
  const int nb = a.n[b] - 2, nc = a.n[c] - 2;
  if (nb <= 0 || nc <= 0) return;
  const long long total = (long long)nb * nc;
  for (long long k = first; k < total; k += stride) {
    int cell[3], nbr[3];
    cell[ax] = side ? a.n[ax] - 1 : 0;
    cell[b] = 1 + int(k / nc);
    cell[c] = 1 + int(k % nc);
    nbr[0] = cell[0];
    nbr[1] = cell[1];
    nbr[2] = cell[2];
    nbr[ax] = side ? a.n[ax] - 2 : 1;
    const long long i = lin(a, cell);
    // an edge cell at (cell - e_b) or (cell - e_c) reads this cell before its update
    if (cell[b] == 1) copy_raw<S>(a, i, face_slot<T>(a, fid, 0, cell[c]));
    if (cell[c] == 1) copy_raw<S>(a, i, face_slot<T>(a, fid, 1, cell[b]));
    const auto t = load_cell<S>(a, i);
    const auto n = load_cell<S>(a, lin(a, nbr));
    store_cell<S>(a, i, bc_core(a, face_dr(ax, side), t, n));
  }
}

// Wave 2: cells on exactly two faces, edge eid = free axis * 4 + s1 * 2 + s2, (s1, s2) the
// sides on the two face axes in increasing order; cells first, first + stride, ... of the edge.
template <class S> __device__ __forceinline__ void wave2_edge(const BcArgs& a, int eid, int first, int stride) {
  using T = typename S::T;
  const int a3 = eid >> 2, s1 = (eid >> 1) & 1, s2 = eid & 1;
  const int a1 = a3 == 0 ? 1 : 0, a2 = a3 == 2 ? 1 : 2;
  const int len = a.n[a3] - 2;
  for (int k = first; k < len; k += stride) {
    int cell[3];
    cell[a1] = s1 ? a.n[a1] - 1 : 0;
    cell[a2] = s2 ? a.n[a2] - 1 : 0;
    cell[a3] = 1 + k;
    const long long i = lin(a, cell);
    if (cell[a3] == 1) copy_raw<S>(a, i, edge_slot<T>(a, eid));
    auto t = load_cell<S>(a, i);
    // faces in axis order a1 < a2; the neighbour through face a_k lies on the other face
    for (int f = 0; f < 2; ++f) {
      const int ak = f ? a2 : a1, sk = f ? s2 : s1;
      const int ao = f ? a1 : a2, so = f ? s1 : s2;
      int nbr[3] = {cell[0], cell[1], cell[2]};
      nbr[ak] = sk ? a.n[ak] - 2 : 1;
      Mom3<typename S::R> n;
      if (sk == 0) {  // low face: the neighbour had not been updated yet
        const int fo = ao * 2 + so;
        const int ob = ao == 0 ? 1 : 0;  // first non-face axis of the other face
        n = load_slot<S>(a, face_slot<T>(a, fo, ak == ob ? 0 : 1, cell[a3]));
      } else {
        n = load_cell<S>(a, lin(a, nbr));
      }
      t = bc_core(a, face_dr(ak, sk), t, n);
    }
    store_cell<S>(a, i, t);
  }
}

// Wave 3: corner k of the 8 (corner bits x, y, z sides).
template <class S> __device__ __forceinline__ void wave3_corner(const BcArgs& a, int k) {
  using T = typename S::T;
  if (k >= 8) return;
  const int sd[3] = {(k >> 2) & 1, (k >> 1) & 1, k & 1};
  int cell[3];
  for (int q = 0; q < 3; ++q) cell[q] = sd[q] ? a.n[q] - 1 : 0;
  const long long i = lin(a, cell);
  auto t = load_cell<S>(a, i);
  for (int ax = 0; ax < 3; ++ax) {
    int nbr[3] = {cell[0], cell[1], cell[2]};
    nbr[ax] = sd[ax] ? a.n[ax] - 2 : 1;
    Mom3<typename S::R> n;
    if (sd[ax] == 0) {
      // the neighbour is the edge cell with free axis ax next to this corner
      const int o1 = ax == 0 ? 1 : 0, o2 = ax == 2 ? 1 : 2;
      const int eid = ax * 4 + sd[o1] * 2 + sd[o2];
      n = load_slot<S>(a, edge_slot<T>(a, eid));
    } else {
      n = load_cell<S>(a, lin(a, nbr));
    }
    t = bc_core(a, face_dr(ax, sd[ax]), t, n);
  }
  store_cell<S>(a, i, t);
}

// One world: blockIdx.y = face / edge.
template <class S> __global__ void wave1_kernel(const BcArgs a) {
  wave1_face<S>(a, blockIdx.y, blockIdx.x * (long long)blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
}
template <class S> __global__ void wave2_kernel(const BcArgs a) {
  wave2_edge<S>(a, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}
template <class S> __global__ void wave3_kernel(const BcArgs a) { wave3_corner<S>(a, threadIdx.x); }

// Many worlds: args[2 * w + parity] are world w's arguments at that parity, blockIdx.z (waves
// 1 and 2) or blockIdx.x (wave 3) the world.
template <class S> __global__ void wave1_batch_kernel(const BcArgs* __restrict__ args, int parity) {
  wave1_face<S>(args[2 * blockIdx.z + parity], blockIdx.y, blockIdx.x * (long long)blockDim.x + threadIdx.x,
                (long long)gridDim.x * blockDim.x);
}
template <class S> __global__ void wave2_batch_kernel(const BcArgs* __restrict__ args, int parity) {
  wave2_edge<S>(args[2 * blockIdx.z + parity], blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x,
                gridDim.x * blockDim.x);
}
template <class S> __global__ void wave3_batch_kernel(const BcArgs* __restrict__ args, int parity) {
  wave3_corner<S>(args[2 * blockIdx.x + parity], threadIdx.x);
}

// The boundary pass's arguments for world w, writing w->post.
BcArgs make_bc_args(const hl_world3d* w, const hl_bc3d* bc, void* scratch) {
  BcArgs a{};
  a.post = w->post;
  a.N = (long long)w->nx * w->ny * w->nz;
  a.n[0] = w->nx;
  a.n[1] = w->ny;
  a.n[2] = w->nz;
  for (int f = 0; f < 6; ++f) {
    a.bc_type[f] = bc->bc_type[f];
    for (int k = 0; k < 3; ++k) a.bc_value[f][k] = bc->bc_value[f][k];
  }
  a.sc = make_scale(w->storage);
  a.snap = scratch;
  a.maxn = w->nx > w->ny ? (w->nx > w->nz ? w->nx : w->nz) : (w->ny > w->nz ? w->ny : w->nz);
  return a;
}

// wave 1 blocks per face for faces of up to maxn x maxn cells (grid-stride beyond 1024)
int wave1_blocks(int maxn) {
  const long long g = ((long long)maxn * maxn + 255) / 256;
  return int(g > 1024 ? 1024 : g);
}

template <class S> int launch_bc(const hl_world3d* w, const hl_bc3d* bc, void* scratch, cudaStream_t st) {
  const BcArgs a = make_bc_args(w, bc, scratch);
  wave1_kernel<S><<<dim3(wave1_blocks(a.maxn), 6), 256, 0, st>>>(a);
  HL_LAUNCH_CHECK("d3q27 apply_bc wave 1");
  wave2_kernel<S><<<dim3((a.maxn + 127) / 128, 12), 128, 0, st>>>(a);
  HL_LAUNCH_CHECK("d3q27 apply_bc wave 2");
  wave3_kernel<S><<<1, 32, 0, st>>>(a);
  HL_LAUNCH_CHECK("d3q27 apply_bc wave 3");
  return HL_OK;
}

// Prepared batch descriptors: address -> (worlds, storage type, largest side).
struct BcBatchInfo {
  int n;
  hl_dtype dtype;
  int maxn;
};
std::mutex g_bcb_mu;
std::map<const void*, BcBatchInfo> g_bcb;

template <class S> int launch_bc_batch(const BcArgs* args, const BcBatchInfo& b, int parity, cudaStream_t st) {
  wave1_batch_kernel<S><<<dim3(wave1_blocks(b.maxn), 6, b.n), 256, 0, st>>>(args, parity);
  HL_LAUNCH_CHECK("d3q27 apply_bc batch wave 1");
  wave2_batch_kernel<S><<<dim3((b.maxn + 127) / 128, 12, b.n), 128, 0, st>>>(args, parity);
  HL_LAUNCH_CHECK("d3q27 apply_bc batch wave 2");
  wave3_batch_kernel<S><<<b.n, 32, 0, st>>>(args, parity);
  HL_LAUNCH_CHECK("d3q27 apply_bc batch wave 3");
  return HL_OK;
}

size_t elem_size(hl_dtype d) { return d == HL_F64 ? 8 : d == HL_F32 ? 4 : 2; }

// ----------------------------------------------------------------------------- init
// InitFlow3D / set_uniform_flow_3d_kernel: rho = 1, u = u0, S from the equilibrium
// populations with cs2_local = pixx (lbm_func_3d.py:55-61), i.e. diagonal S = 0 at rho = 1.
template <class S>
__global__ void init_uniform_kernel(long long N, typename S::T* ma, typename S::T* mb, float* force, float ux,
                                    float uy, float uz, Scale sc) {
  using R = typename S::R;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const R rho = R(1);
  R pxx = 0, pyy = 0, pzz = 0, pxy = 0, pxz = 0, pyz = 0;
  const R usq = R(ux) * R(ux) + R(uy) * R(uy) + R(uz) * R(uz);
  for (int cx = -1; cx <= 1; ++cx)
    for (int cy = -1; cy <= 1; ++cy)
      for (int cz = -1; cz <= 1; ++cz) {
        const int nnz = (cx != 0) + (cy != 0) + (cz != 0);
        const R w = nnz == 0 ? R(8.0 / 27.0) : nnz == 1 ? R(2.0 / 27.0) : nnz == 2 ? R(1.0 / 54.0) : R(1.0 / 216.0);
        const R cu = R(cx) * R(ux) + R(cy) * R(uy) + R(cz) * R(uz);
        const R f = w * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq);
        if (cx) pxx += f;
        if (cy) pyy += f;
        if (cz) pzz += f;
        if (cx * cy) pxy += R(cx * cy) * f;
        if (cx * cz) pxz += R(cx * cz) * f;
        if (cy * cz) pyz += R(cy * cz) * f;
      }
  Mom3<R> m;
  m.rho = rho;
  m.drho = R(0);
  m.ux = R(ux);
  m.uy = R(uy);
  m.uz = R(uz);
  // cs2_local = pixx is subtracted from every diagonal (lbm_func_3d.py:55-61)
  m.sxx = pxx * (R(1) / rho) - pxx;
  m.syy = pyy * (R(1) / rho) - pxx;
  m.szz = pzz * (R(1) / rho) - pxx;
  m.sxy = pxy / rho;
  m.sxz = pxz / rho;
  m.syz = pyz / rho;
  R raw[10];
  encode3<S>(m, sc, raw);
  for (int k = 0; k < 10; ++k) {
    ma[k * N + i] = S::from_r(raw[k]);
    mb[k * N + i] = S::from_r(raw[k]);
  }
  if (force) force[i] = force[N + i] = force[2 * N + i] = 0.f;
}

template <class S>
__global__ void init_tgv_kernel(int nx, int ny, int nz, typename S::T* ma, typename S::T* mb, float u0, Scale sc) {
  using R = typename S::R;
  const long long N = (long long)nx * ny * nz;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int z = int(i % nz), y = int((i / nz) % ny), x = int(i / ((long long)ny * nz));
  const double tp = 6.283185307179586;
  const double X = tp * x / nx, Y = tp * y / ny, Z = tp * z / nz;
  const double ux = u0 * sin(X) * cos(Y) * cos(Z);
  const double uy = -u0 * cos(X) * sin(Y) * cos(Z);
  const double rho = 1.0 + 3.0 * (double(u0) * u0 / 16.0) * (cos(2 * X) + cos(2 * Y)) * (cos(2 * Z) + 2.0);
  Mom3<R> m;
  m.rho = R(rho);
  m.drho = R(rho - 1.0);
  m.ux = R(ux);
  m.uy = R(uy);
  m.uz = R(0);
  m.sxx = R(ux * ux);
  m.syy = R(uy * uy);
  m.szz = R(0);
  m.sxy = R(ux * uy);
  m.sxz = R(0);
  m.syz = R(0);
  R raw[10];
  encode3<S>(m, sc, raw);
  for (int k = 0; k < 10; ++k) {
    ma[k * N + i] = S::from_r(raw[k]);
    mb[k * N + i] = S::from_r(raw[k]);
  }
}

// InitBoundary3D (envs/lbm3d/lbm_func_3d.py:13-19)
__global__ void init_boundary_kernel(int nx, int ny, int nz, int32_t* flag) {
  const long long N = (long long)nx * ny * nz;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int z = int(i % nz), y = int((i / nz) % ny), x = int(i / ((long long)ny * nz));
  if (x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1) flag[i] = ML_WALL;
}

}  // namespace d3bc
}  // namespace hl

using namespace hl;

extern "C" size_t hl_d3q27_bc_scratch_bytes(const hl_world3d* w) {
  if (!w) return 0;
  const int maxn = w->nx > w->ny ? (w->nx > w->nz ? w->nx : w->nz) : (w->ny > w->nz ? w->ny : w->nz);
  return (size_t(12) * maxn + 12) * 10 * d3bc::elem_size(w->storage.dtype);
}

extern "C" int hl_d3q27_apply_bc(const hl_world3d* w, const hl_bc3d* bc, void* scratch, hl_stream stream) {
  HL_CHECK_ARG(w != nullptr && bc != nullptr, "apply_bc_3d: NULL argument");
  if (w->periodic) return HL_OK;
  HL_CHECK_ARG(w->nx >= 3 && w->ny >= 3 && w->nz >= 3, "apply_bc_3d: walled worlds need every side >= 3");
  HL_CHECK_ARG(scratch != nullptr, "apply_bc_3d: scratch is NULL");
  HL_CHECK_ARG(w->post != nullptr, "apply_bc_3d: post is NULL");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (w->storage.dtype) {
    case HL_F32: return d3bc::launch_bc<StoreF32>(w, bc, scratch, st);
    case HL_F64: return d3bc::launch_bc<StoreF64>(w, bc, scratch, st);
    case HL_F16: return d3bc::launch_bc<StoreF16>(w, bc, scratch, st);
    case HL_BF16: return d3bc::launch_bc<StoreBF16>(w, bc, scratch, st);
  }
  set_error("apply_bc_3d: bad dtype");
  return HL_ERR_ARG;
}

extern "C" size_t hl_d3q27_bc_batch_bytes(int n_domains) {
  return n_domains > 0 ? size_t(2) * size_t(n_domains) * sizeof(d3bc::BcArgs) : 0;
}

extern "C" int hl_d3q27_bc_batch_prepare(const hl_world3d* worlds, const hl_bc3d* bcs, void* const* scratch,
                                         int n_domains, void* desc, size_t desc_bytes, hl_stream stream) {
  HL_CHECK_ARG(worlds != nullptr && bcs != nullptr && scratch != nullptr && desc != nullptr,
               "apply_bc_3d batch: NULL argument");
  HL_CHECK_ARG(n_domains > 0 && n_domains <= 65535, "apply_bc_3d batch: n_domains must be in 1..65535");
  const size_t bytes = hl_d3q27_bc_batch_bytes(n_domains);
  HL_CHECK_ARG(desc_bytes >= bytes, "apply_bc_3d batch: desc_bytes below hl_d3q27_bc_batch_bytes");
  HL_CHECK_ARG(reinterpret_cast<uintptr_t>(desc) % 16 == 0, "apply_bc_3d batch: desc not 16-byte aligned");
  const hl_dtype dtype = worlds[0].storage.dtype;
  std::vector<d3bc::BcArgs> host(size_t(2) * n_domains);
  int maxn = 0;
  for (int i = 0; i < n_domains; ++i) {
    const hl_world3d& w = worlds[i];
    HL_CHECK_ARG(!w.periodic, "apply_bc_3d batch: world %d is periodic (no boundary pass)", i);
    HL_CHECK_ARG(w.nx >= 3 && w.ny >= 3 && w.nz >= 3, "apply_bc_3d batch: world %d needs every side >= 3", i);
    HL_CHECK_ARG(w.storage.dtype == dtype, "apply_bc_3d batch: world %d has another storage type", i);
    HL_CHECK_ARG(w.cur != nullptr && w.post != nullptr && scratch[i] != nullptr,
                 "apply_bc_3d batch: world %d has a NULL buffer or scratch", i);
    // parity 0 writes post, parity 1 the other buffer (the step then reads post)
    d3bc::BcArgs a = d3bc::make_bc_args(&w, &bcs[i], scratch[i]);
    host[2 * i] = a;
    a.post = const_cast<void*>(w.cur);
    host[2 * i + 1] = a;
    maxn = std::max(maxn, a.maxn);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(desc, host.data(), bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host staging buffer ends here
  if (e != cudaSuccess) return cuda_status(e, "apply_bc_3d batch: descriptor upload");
  std::lock_guard<std::mutex> lock(d3bc::g_bcb_mu);
  d3bc::g_bcb[desc] = d3bc::BcBatchInfo{n_domains, dtype, maxn};
  return HL_OK;
}

extern "C" int hl_d3q27_apply_bc_batch(const void* desc, int n_domains, int parity, hl_stream stream) {
  HL_CHECK_ARG(desc != nullptr, "apply_bc_3d batch: desc is NULL");
  HL_CHECK_ARG(parity == 0 || parity == 1, "apply_bc_3d batch: parity must be 0 or 1");
  d3bc::BcBatchInfo b;
  {
    std::lock_guard<std::mutex> lock(d3bc::g_bcb_mu);
    auto it = d3bc::g_bcb.find(desc);
    HL_CHECK_ARG(it != d3bc::g_bcb.end(), "apply_bc_3d batch: desc was not prepared");
    b = it->second;
  }
  HL_CHECK_ARG(n_domains == b.n, "apply_bc_3d batch: n_domains %d differs from the prepared %d", n_domains, b.n);
  const auto* args = static_cast<const d3bc::BcArgs*>(desc);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (b.dtype) {
    case HL_F32: return d3bc::launch_bc_batch<StoreF32>(args, b, parity, st);
    case HL_F64: return d3bc::launch_bc_batch<StoreF64>(args, b, parity, st);
    case HL_F16: return d3bc::launch_bc_batch<StoreF16>(args, b, parity, st);
    case HL_BF16: return d3bc::launch_bc_batch<StoreBF16>(args, b, parity, st);
  }
  set_error("apply_bc_3d batch: bad dtype");
  return HL_ERR_ARG;
}

template <class S>
static int init_uniform_t(int nx, int ny, int nz, hl_storage sto, void* a, void* b, float* f, float ux, float uy,
                          float uz, cudaStream_t st) {
  const long long N = (long long)nx * ny * nz;
  d3bc::init_uniform_kernel<S><<<unsigned((N + 255) / 256), 256, 0, st>>>(
      N, static_cast<typename S::T*>(a), static_cast<typename S::T*>(b), f, ux, uy, uz, make_scale(sto));
  HL_LAUNCH_CHECK("d3q27 init_uniform");
  return HL_OK;
}

extern "C" int hl_d3q27_init_uniform(int nx, int ny, int nz, hl_storage sto, void* a, void* b, float* force, float ux,
                                     float uy, float uz, hl_stream stream) {
  HL_CHECK_ARG(nx > 0 && ny > 0 && nz > 0 && a && b, "init_uniform_3d: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (sto.dtype) {
    case HL_F32: return init_uniform_t<StoreF32>(nx, ny, nz, sto, a, b, force, ux, uy, uz, st);
    case HL_F64: return init_uniform_t<StoreF64>(nx, ny, nz, sto, a, b, force, ux, uy, uz, st);
    case HL_F16: return init_uniform_t<StoreF16>(nx, ny, nz, sto, a, b, force, ux, uy, uz, st);
    case HL_BF16: return init_uniform_t<StoreBF16>(nx, ny, nz, sto, a, b, force, ux, uy, uz, st);
  }
  set_error("init_uniform_3d: bad dtype");
  return HL_ERR_ARG;
}

template <class S>
static int init_tgv_t(int nx, int ny, int nz, hl_storage sto, void* a, void* b, float u0, cudaStream_t st) {
  const long long N = (long long)nx * ny * nz;
  d3bc::init_tgv_kernel<S><<<unsigned((N + 255) / 256), 256, 0, st>>>(nx, ny, nz, static_cast<typename S::T*>(a),
                                                                        static_cast<typename S::T*>(b), u0,
                                                                        make_scale(sto));
  HL_LAUNCH_CHECK("d3q27 init_tgv");
  return HL_OK;
}

extern "C" int hl_d3q27_init_tgv(int nx, int ny, int nz, hl_storage sto, void* a, void* b, float u0,
                                 hl_stream stream) {
  HL_CHECK_ARG(nx > 0 && ny > 0 && nz > 0 && a && b, "init_tgv: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (sto.dtype) {
    case HL_F32: return init_tgv_t<StoreF32>(nx, ny, nz, sto, a, b, u0, st);
    case HL_F64: return init_tgv_t<StoreF64>(nx, ny, nz, sto, a, b, u0, st);
    case HL_F16: return init_tgv_t<StoreF16>(nx, ny, nz, sto, a, b, u0, st);
    case HL_BF16: return init_tgv_t<StoreBF16>(nx, ny, nz, sto, a, b, u0, st);
  }
  set_error("init_tgv: bad dtype");
  return HL_ERR_ARG;
}

extern "C" int hl_d3q27_init_boundary(int nx, int ny, int nz, int32_t* flag, hl_stream stream) {
  HL_CHECK_ARG(nx > 0 && ny > 0 && nz > 0 && flag, "init_boundary_3d: bad arguments");
  const long long N = (long long)nx * ny * nz;
  d3bc::init_boundary_kernel<<<unsigned((N + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(nx, ny, nz,
                                                                                                      flag);
  HL_LAUNCH_CHECK("d3q27 init_boundary");
  return HL_OK;
}
