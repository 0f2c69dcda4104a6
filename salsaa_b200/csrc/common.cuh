// common.cuh — shared device arithmetic for the SALSAA sm_100a kernels.
//
// All arithmetic is exact modulo q (q < 2^62, odd).  Three multiplication
// forms are used:
//   * Barrett (HAC 14.42, base 2) for two variable operands;
//   * Shoup's precomputed-quotient form for a fixed operand (NTT twiddles,
//     challenges), w' = floor(w * 2^64 / q);
//   * lazy 25-bit-limb accumulation for long dot products when q < 2^50:
//     a = a1*2^25 + a0, products of limbs are < 2^50 and add up in 64-bit
//     registers without reduction for 2^11 terms.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

typedef uint64_t u64;
typedef uint32_t u32;

namespace salsaa {

struct ModQ {
  u64 q;
  u64 mu;     // floor(2^(2s) / q)
  u32 s;      // bit length of q
  u64 r64;    // 2^64 mod q
};

__host__ inline ModQ make_modq(u64 q) {
  ModQ M;
  M.q = q;
  M.s = 64u - (u32)__builtin_clzll(q);
  M.mu = (u64)(((unsigned __int128)1 << (2 * M.s)) / q);
  M.r64 = (u64)((((unsigned __int128)1) << 64) % q);
  return M;
}

__host__ inline u64 shoup_pre(u64 w, u64 q) { return (u64)((((unsigned __int128)w) << 64) / q); }

__device__ __forceinline__ u64 add_mod(u64 a, u64 b, u64 q) {
  u64 r = a + b;
  return r >= q ? r - q : r;
}
__device__ __forceinline__ u64 sub_mod(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + (q - b); }

// Barrett reduction of the 128-bit value hi:lo < 2^(2s).
__device__ __forceinline__ u64 barrett128(const ModQ& M, u64 hi, u64 lo) {
  const u32 s = M.s;
  u64 q1 = (hi << (65 - s)) | (lo >> (s - 1));
  u64 q2lo = q1 * M.mu, q2hi = __umul64hi(q1, M.mu);
  u64 q3 = (q2hi << (63 - s)) | (q2lo >> (s + 1));
  u64 r = lo - q3 * M.q;
  if (r >= M.q) r -= M.q;
  if (r >= M.q) r -= M.q;
  return r;
}
__device__ __forceinline__ u64 mul_mod(const ModQ& M, u64 a, u64 b) {
  return barrett128(M, __umul64hi(a, b), a * b);
}
// x mod q for any 64-bit x: Barrett applies directly when 2^64 <= 2^(2s),
// i.e. q >= 2^31; smaller moduli use the hardware-less division.
__device__ __forceinline__ u64 reduce64(const ModQ& M, u64 x) {
  return M.s >= 32 ? barrett128(M, 0, x) : x % M.q;
}
// Reduction of an arbitrary 128-bit value: hi*2^64 + lo = (hi mod q)*(2^64 mod q) + lo.
__device__ __forceinline__ u64 reduce128_any(const ModQ& M, u64 hi, u64 lo) {
  u64 h = reduce64(M, hi);
  u64 t = mul_mod(M, h, M.r64);
  u64 l = reduce64(M, lo);
  return add_mod(t, l, M.q);
}
// Shoup: x * w mod q for any x < 2^64, w < q, wp = floor(w 2^64 / q).
__device__ __forceinline__ u64 mul_shoup(u64 x, u64 w, u64 wp, u64 q) {
  u64 h = __umul64hi(x, wp);
  u64 r = x * w - h * q;
  return r >= q ? r - q : r;
}

// Accumulate a reduced value into a global sum kept mod q.  With q < 2^50
// and fewer than 2^13 contributions a plain 64-bit add cannot overflow and
// the consumer reduces at the end; otherwise add modulo q with a CAS loop.
__device__ __forceinline__ void atomic_add_mod(u64* addr, u64 v, u64 q, bool plain) {
  if (plain) {
    atomicAdd((unsigned long long*)addr, (unsigned long long)v);
    return;
  }
  unsigned long long old = *(volatile unsigned long long*)addr, assumed;
  do {
    assumed = old;
    u64 nv = add_mod((u64)assumed % q, v, q);
    old = atomicCAS((unsigned long long*)addr, assumed, (unsigned long long)nv);
  } while (old != assumed);
}

// Shoup without the final correction: x * w mod q in [0, 2q) for any 64-bit x.
__device__ __forceinline__ u64 mul_shoup_lazy(u64 x, u64 w, u64 wp, u64 q) { return x * w - __umul64hi(x, wp) * q; }

// ---- lazy limb accumulator (q < 2^50) -------------------------------------
struct Acc3 {
  u64 lo, mid, hi;
};
__device__ __forceinline__ void acc_zero(Acc3& a) { a.lo = a.mid = a.hi = 0; }
// a += x * y with x = (x1, x0), y = (y1, y0) as 25-bit limbs (32-bit registers).
__device__ __forceinline__ void acc_mac(Acc3& a, u32 x1, u32 x0, u32 y1, u32 y0) {
  a.lo += (u64)x0 * y0;
  a.mid += (u64)x0 * y1 + (u64)x1 * y0;
  a.hi += (u64)x1 * y1;
}
__device__ __forceinline__ void split25(u64 v, u32& v1, u32& v0) {
  v0 = (u32)v & 0x1FFFFFFu;
  v1 = (u32)(v >> 25);
}
// value = lo + mid*2^25 + hi*2^50 reduced mod q.
__device__ __forceinline__ u64 acc_reduce(const ModQ& M, const Acc3& a) {
  // 128-bit sum: lo + (mid << 25) + (hi << 50)
  u64 l = a.lo, h = 0;
  u64 t = a.mid << 25;
  u64 th = a.mid >> 39;
  l += t;
  h += th + (l < t);
  t = a.hi << 50;
  th = a.hi >> 14;
  u64 l2 = l + t;
  h += th + (l2 < t);
  return reduce128_any(M, h, l2);
}

// ---- counter-based PRF (identical to the CPU oracle's so_prf) --------------
__host__ __device__ __forceinline__ u64 mix64(u64 z) {
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return z;
}
constexpr u64 PRF_GOLDEN = 0x9e3779b97f4a7c15ULL;
__host__ __device__ __forceinline__ u64 prf_key(u64 seed, u64 domain) { return mix64(seed ^ mix64(domain + PRF_GOLDEN)); }
__host__ __device__ __forceinline__ u64 prf_at(u64 key, u64 index) { return mix64(key + index * PRF_GOLDEN); }
__device__ __forceinline__ u64 uni_mod(u64 r, u64 q) { return __umul64hi(r, q); }

enum Domain : u64 { DOM_CRS = 1, DOM_WIT = 2, DOM_NC = 3, DOM_PROJ = 4, DOM_FOLD = 5 };
__host__ __device__ __forceinline__ u64 domain_id(u64 kind, u64 a, u64 b) { return (kind << 56) | (a << 24) | b; }

}  // namespace salsaa

#define SALSAA_CUDA_TRY(expr)                                      \
  do {                                                             \
    cudaError_t _e = (expr);                                       \
    if (_e != cudaSuccess) return salsaa_set_cuda_error(_e, #expr); \
  } while (0)

int salsaa_set_cuda_error(cudaError_t e, const char* what);
int salsaa_set_error(int code, const char* msg);
// Counts kernel launches issued by this library (reported by the benchmark).
void salsaa_count_launch();
// Optional device-time trace of named kernels (off unless enabled through the
// C ABI): an event pair on the launching stream around each traced launch.
// `work` is the launch's algorithmic work (bytes or operations, per kernel).
int salsaa_trace_begin(const char* name, cudaStream_t st, double work);
// Another measure of the launch that `token` brackets, read under `name`.
void salsaa_trace_alias(int token, const char* name, double work);
void salsaa_trace_end(int token, cudaStream_t st);
