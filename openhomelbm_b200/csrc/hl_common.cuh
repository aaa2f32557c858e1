// Shared device helpers of libhomelbm: error reporting, moment storage codecs, async copies.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/homelbm.h"

namespace hl {

// ----------------------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
extern int g_tune_d3_kernel;  // hl_set_tuning("d3q27_kernel")
extern int g_tune_d3_chunks;  // hl_set_tuning("d3q27_chunks")
extern int g_tune_d3_stages;  // hl_set_tuning("d3q27_stages")
extern int g_tune_d3_link_blocks;  // hl_set_tuning("d3q27_link_blocks")

// Per-device host state (a process may drive several GPUs): the current device's SM count,
// and the dynamic shared-memory opt-in of a kernel, set once per (kernel, device, size).
int device_sms();
int set_smem_attr(const void* kernel, int bytes, const char* what);

#define HL_CHECK_ARG(cond, ...)       \
  do {                                \
    if (!(cond)) {                    \
      ::hl::set_error(__VA_ARGS__);   \
      return HL_ERR_ARG;              \
    }                                 \
  } while (0)

#define HL_LAUNCH_CHECK(what)                                        \
  do {                                                               \
    cudaError_t e_ = cudaGetLastError();                             \
    if (e_ != cudaSuccess) return ::hl::cuda_status(e_, what);       \
  } while (0)

// ----------------------------------------------------------------------------- lattice
constexpr int ML_FLUID = 0;
constexpr int ML_SOLID = 1;
constexpr int ML_WALL = 2;
constexpr float CS2 = 1.0f / 3.0f;

// ----------------------------------------------------------------------------- storage
// Decoded moments of one cell, binary32 (binary64 for the accuracy build). drho = rho - 1
// is carried beside rho: kernels work with deviations from the rest state (populations as
// f - w), which removes the O(1) offset from every sum.
template <class R> struct Mom3 {
  R rho, drho, ux, uy, uz, sxx, syy, szz, sxy, sxz, syz;
};
template <class R> struct Mom2 {
  R rho, drho, ux, uy, sxx, syy, sxy;
};

struct Scale {
  float u, inv_u, s, inv_s;
};

inline Scale make_scale(const hl_storage& st) {
  Scale s;
  s.u = st.u_scale > 0.f ? st.u_scale : 1.f;
  s.s = st.s_scale > 0.f ? st.s_scale : 1.f;
  s.inv_u = 1.f / s.u;
  s.inv_s = 1.f / s.s;
  return s;
}

// Storage codecs: StoreF32 / StoreF64 keep the moments as they are; StoreF16 / StoreBF16
// hold rho - 1, u / u_scale and (S - u u) / s_scale.
//
// The reduced storages round stochastically: a value between two representable neighbours
// goes to the upper one with probability equal to its distance from the lower one, in units
// of their spacing (unbiased in expectation). Round-to-nearest stores of a slowly varying
// field round the same way step after step and its error drifts; stochastic rounding makes
// the per-step errors independent. The random bits are bits of a multiplicative hash
// (Knuth's multiplicative hashing, golden-ratio and MurmurHash3-finaliser constants) of the
// value's own bit pattern and a salt (the element's index in its buffer): a store is a
// deterministic function of the value and its place, so a field gives the same result in
// every run, alone or batched, while equal values in different cells round independently.
// Bits 16 and up of the product depend on every input bit below them, the dropped low bits of
// the value included, and are uniform over the values and places a field holds, which is what
// unbiasedness needs.
__device__ __forceinline__ unsigned dither_bits(unsigned b, unsigned salt) {
  return (b ^ (salt * 0x9e3779b9u)) * 0x85ebca6bu;
}
// The same kind of hash for the moments of one cell stored together: the value's bits, the
// cell's term cell_salt = cell index * 0x9e3779b9 (taken once per cell) and moment k's own
// constant (folded at compile time) -- one three-way xor and one multiply per element.
__device__ __forceinline__ unsigned dither_cell(unsigned b, unsigned cell_salt, unsigned k) {
  return (b ^ cell_salt ^ (k * 0x632be5abu)) * 0x85ebca6bu;
}
// The rounding itself is the sm_100a conversion with caller-supplied random bits
// (cvt.rs.{f16x2,bf16x2}.f32): a goes to the upper half of the result and b to the lower one.
// binary16: a draws its 13 random bits from rbits[28:16], b from rbits[12:0]; they are added
// below the unit of the last place and the sum is truncated, the subnormal range (spacing
// 2^-24) included, where the fraction is first cut to 13 bits (a bias toward zero under
// 2^-37). bfloat16: 16 random bits each, a from rbits[31:16], b from rbits[15:0]. Finite
// values above the largest finite one round to it or to an infinity; infinities and NaNs
// stay non-finite. The probability and the bit fields are checked on the GPU by the rounding test
// of the storage codecs (hl_round_to_storage).
__device__ __forceinline__ unsigned cvt_rs_f16x2(float a, float b, unsigned rbits) {
  unsigned d;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(rbits));
  return d;
}
__device__ __forceinline__ unsigned cvt_rs_bf16x2(float a, float b, unsigned rbits) {
  unsigned d;
  asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(rbits));
  return d;
}
// rbits for a pair whose hashes are ha (value a) and hb (value b): bits 31..16 of ha in the
// upper half, bits 31..16 of hb in the lower half, so that a and b round exactly as they
// would alone (the single forms put a value in the a slot with its hash as rbits).
__device__ __forceinline__ unsigned pair_rbits(unsigned ha, unsigned hb) { return __byte_perm(ha, hb, 0x3276u); }
__device__ __forceinline__ __half half_hi(unsigned d) { return __ushort_as_half((unsigned short)(d >> 16)); }
__device__ __forceinline__ __half half_lo(unsigned d) { return __ushort_as_half((unsigned short)(d & 0xffffu)); }
__device__ __forceinline__ __nv_bfloat16 bf16_hi(unsigned d) {
  return __ushort_as_bfloat16((unsigned short)(d >> 16));
}
__device__ __forceinline__ __nv_bfloat16 bf16_lo(unsigned d) {
  return __ushort_as_bfloat16((unsigned short)(d & 0xffffu));
}
// binary32 -> binary16 / bfloat16, stochastic, with the element-index salt
__device__ __forceinline__ __half half_sr(float v, unsigned salt) {
  return half_hi(cvt_rs_f16x2(v, 0.f, dither_bits(__float_as_uint(v), salt)));
}
__device__ __forceinline__ __nv_bfloat16 bf16_sr(float v, unsigned salt) {
  return bf16_hi(cvt_rs_bf16x2(v, 0.f, dither_bits(__float_as_uint(v), salt)));
}

struct StoreF32 {
  using T = float;
  using R = float;
  static constexpr bool kEncoded = false;
  __device__ static float to_r(T v) { return v; }
  __device__ static T from_r(float v, unsigned = 0u) { return v; }
  __device__ static T from_r_cell(float v, unsigned, unsigned) { return v; }
  __device__ static void from_r_cell2(float a, float b, unsigned, unsigned, unsigned, T& oa, T& ob) {
    oa = a;
    ob = b;
  }
};
struct StoreF64 {
  using T = double;
  using R = double;
  static constexpr bool kEncoded = false;
  __device__ static double to_r(T v) { return v; }
  __device__ static T from_r(double v, unsigned = 0u) { return v; }
  __device__ static T from_r_cell(double v, unsigned, unsigned) { return v; }
  __device__ static void from_r_cell2(double a, double b, unsigned, unsigned, unsigned, T& oa, T& ob) {
    oa = a;
    ob = b;
  }
};
struct StoreF16 {
  using T = __half;
  using R = float;
  static constexpr bool kEncoded = true;
  __device__ static float to_r(T v) { return __half2float(v); }
  // salt: the element's index in its buffer
  __device__ static T from_r(float v, unsigned salt = 0u) { return half_sr(v, salt); }
  // moment k of the cell whose cell_salt is given (dither_cell)
  __device__ static T from_r_cell(float v, unsigned cell_salt, unsigned k) {
    return half_hi(cvt_rs_f16x2(v, 0.f, dither_cell(__float_as_uint(v), cell_salt, k)));
  }
  // moment k of two cells at once, packed (a in the upper half): the same results as two
  // from_r_cell calls, one conversion
  __device__ static unsigned round2(float a, float b, unsigned cs_a, unsigned cs_b, unsigned k) {
    return cvt_rs_f16x2(a, b, pair_rbits(dither_cell(__float_as_uint(a), cs_a, k),
                                         dither_cell(__float_as_uint(b), cs_b, k)));
  }
  __device__ static T hi(unsigned d) { return half_hi(d); }
  __device__ static T lo(unsigned d) { return half_lo(d); }
  __device__ static void from_r_cell2(float a, float b, unsigned cs_a, unsigned cs_b, unsigned k, T& oa, T& ob) {
    const unsigned d = round2(a, b, cs_a, cs_b, k);
    oa = hi(d);
    ob = lo(d);
  }
};
struct StoreBF16 {
  using T = __nv_bfloat16;
  using R = float;
  static constexpr bool kEncoded = true;
  __device__ static float to_r(T v) { return __bfloat162float(v); }
  __device__ static T from_r(float v, unsigned salt = 0u) { return bf16_sr(v, salt); }
  __device__ static T from_r_cell(float v, unsigned cell_salt, unsigned k) {
    return bf16_hi(cvt_rs_bf16x2(v, 0.f, dither_cell(__float_as_uint(v), cell_salt, k)));
  }
  __device__ static unsigned round2(float a, float b, unsigned cs_a, unsigned cs_b, unsigned k) {
    return cvt_rs_bf16x2(a, b, pair_rbits(dither_cell(__float_as_uint(a), cs_a, k),
                                          dither_cell(__float_as_uint(b), cs_b, k)));
  }
  __device__ static T hi(unsigned d) { return bf16_hi(d); }
  __device__ static T lo(unsigned d) { return bf16_lo(d); }
  __device__ static void from_r_cell2(float a, float b, unsigned cs_a, unsigned cs_b, unsigned k, T& oa, T& ob) {
    const unsigned d = round2(a, b, cs_a, cs_b, k);
    oa = hi(d);
    ob = lo(d);
  }
};

// raw[10] in plane order -> physical moments
template <class S>
__device__ __forceinline__ Mom3<typename S::R> decode3(const typename S::R raw[10], const Scale& sc) {
  using R = typename S::R;
  Mom3<R> m;
  if constexpr (S::kEncoded) {
    m.drho = raw[0];
    m.rho = raw[0] + R(1);
    m.ux = raw[1] * sc.u;
    m.uy = raw[2] * sc.u;
    m.uz = raw[3] * sc.u;
    m.sxx = fmaf(raw[4], sc.s, m.ux * m.ux);
    m.syy = fmaf(raw[5], sc.s, m.uy * m.uy);
    m.szz = fmaf(raw[6], sc.s, m.uz * m.uz);
    m.sxy = fmaf(raw[7], sc.s, m.ux * m.uy);
    m.sxz = fmaf(raw[8], sc.s, m.ux * m.uz);
    m.syz = fmaf(raw[9], sc.s, m.uy * m.uz);
  } else {
    m.rho = raw[0];
    m.drho = raw[0] - R(1);  // exact for rho in [0.5, 2] (Sterbenz)
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

template <class S>
__device__ __forceinline__ void encode3(const Mom3<typename S::R>& m, const Scale& sc, typename S::R raw[10]) {
  using R = typename S::R;
  if constexpr (S::kEncoded) {
    raw[0] = m.drho;
    raw[1] = m.ux * sc.inv_u;
    raw[2] = m.uy * sc.inv_u;
    raw[3] = m.uz * sc.inv_u;
    raw[4] = (m.sxx - m.ux * m.ux) * sc.inv_s;
    raw[5] = (m.syy - m.uy * m.uy) * sc.inv_s;
    raw[6] = (m.szz - m.uz * m.uz) * sc.inv_s;
    raw[7] = (m.sxy - m.ux * m.uy) * sc.inv_s;
    raw[8] = (m.sxz - m.ux * m.uz) * sc.inv_s;
    raw[9] = (m.syz - m.uy * m.uz) * sc.inv_s;
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

template <class S>
__device__ __forceinline__ Mom2<typename S::R> decode2(const typename S::R raw[6], const Scale& sc) {
  using R = typename S::R;
  Mom2<R> m;
  if constexpr (S::kEncoded) {
    m.drho = raw[0];
    m.rho = raw[0] + R(1);
    m.ux = raw[1] * sc.u;
    m.uy = raw[2] * sc.u;
    m.sxx = fmaf(raw[3], sc.s, m.ux * m.ux);
    m.syy = fmaf(raw[4], sc.s, m.uy * m.uy);
    m.sxy = fmaf(raw[5], sc.s, m.ux * m.uy);
  } else {
    m.rho = raw[0];
    m.drho = raw[0] - R(1);
    m.ux = raw[1];
    m.uy = raw[2];
    m.sxx = raw[3];
    m.syy = raw[4];
    m.sxy = raw[5];
  }
  return m;
}

template <class S>
__device__ __forceinline__ void encode2(const Mom2<typename S::R>& m, const Scale& sc, typename S::R raw[6]) {
  using R = typename S::R;
  if constexpr (S::kEncoded) {
    raw[0] = m.drho;
    raw[1] = m.ux * sc.inv_u;
    raw[2] = m.uy * sc.inv_u;
    // S - u u as one fused multiply-add, written out so that no kernel's surroundings change it
    raw[3] = fmaf(-m.ux, m.ux, m.sxx) * sc.inv_s;
    raw[4] = fmaf(-m.uy, m.uy, m.syy) * sc.inv_s;
    raw[5] = fmaf(-m.ux, m.uy, m.sxy) * sc.inv_s;
  } else {
    raw[0] = m.rho;
    raw[1] = m.ux;
    raw[2] = m.uy;
    raw[3] = m.sxx;
    raw[4] = m.syy;
    raw[5] = m.sxy;
  }
}

// ----------------------------------------------------------------------------- async copy
// 4-byte global -> shared asynchronous copy; src_bytes = 0 zero-fills the destination.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

}  // namespace hl
