// ntt.cuh — batched negacyclic NTT over Z_q[Y]/(Y^n + 1), HEXL conventions:
// forward output in bit-reversed order, a[i] = A(psi^(2*bitrev(i)+1)) with psi
// the minimal primitive 2n-th root; inverse takes bit-reversed input and
// returns natural order scaled by 1/n (hexl-bindings/hexl_wrapper.cpp:213-229).
//
// "incomplete" mode transforms ring elements of R_q = Z_q[X]/(X^d+1), d = 2n,
// between the coefficient layout and the incomplete-NTT ("slot") layout
// [NTT_n(even coefficients) | NTT_n(odd coefficients)]
// (src/cyclotomic_ring.rs:484-556).
#pragma once
#include "common.cuh"

namespace salsaa {

struct NttDev {
  u64 q;
  u32 n, logn;
  const u64* fwd;   // bit-reversed psi^i
  const u64* fwdp;  // Shoup companions
  const u64* inv;   // bit-reversed psi^-i
  const u64* invp;
  u64 ninv, ninvp;  // 1/n mod q and its Shoup companion
  u64 onep;         // Shoup companion of 1: floor(2^64 / q), for reductions
  const u64* zeta;  // shift factors NTT_n(Y) (slot order), for ring products
  const u64* zetap;
  // FP64 form of the tables for q < 2^50 (the FP64 butterflies in ntt.cu):
  // each twiddle w as a double and fl(w / 2q); q, 2q and fl(1/q).
  const double* fwd_d;
  const double* fwd_h;
  const double* inv_d;
  const double* inv_h;
  double qd, q2d, qinv, ninv_d, ninv_h;
};

// Tables for (n, q) on the current device, built once and kept for the
// process lifetime (thread-safe).  Returns nullptr when q has no 2n-th root.
const NttDev* ntt_tables(u32 n, u64 q);

// Kernel schedule of the register-path transform (see ntt.cu): variant 0 =
// one tile per CTA, 2..4 = persistent CTAs with that many bulk-copy stages;
// ctas_per_sm caps resident CTAs per SM (0 = no cap).
struct NttChoice {
  uint8_t variant, ctas_per_sm;
  // the schedule's arithmetic: FP64 butterflies (variants 1 and 5..7)
  __host__ __device__ bool fp64() const { return variant == 1 || variant >= 5; }
};
constexpr u64 NTT_LARGE_COEFFS = 1ULL << 22;  // batch class "large": at least this many coefficients per launch
NttChoice ntt_choice(u32 logn, bool incomplete, bool inverse, bool wide, bool large);
int ntt_tune_set(u32 logn, bool incomplete, bool inverse, bool wide, bool large, int variant, int ctas_per_sm);
int ntt_tune_load(const char* path);  // number of entries read, or < 0
void ntt_tune_reset();
// Fold products (launch_fold): 0 = integer Shoup products, 1 = FP64 (q < 2^50).
int fold_choice();
// Changes whenever the schedule table changes (see g_sched_gen).
unsigned long long schedule_generation();
int fold_tune_set(int variant);
int ntt_error_check();  // a bounded wait of the pipelined transform gave up

// count units of n (full) or ring elements of 2n (incomplete); in may equal out.
// With mag_or (register path only, ntt_mag_ok), the bitwise OR of the centred
// magnitudes min(v, q - v) of the coefficient-form side (the input of a
// forward, the output of an inverse transform) is OR-ed into *mag_or.
int ntt_launch(const u64* in, u64* out, u64 count, const NttDev& T, bool incomplete, bool inverse,
               cudaStream_t st, u64* mag_or = nullptr);
bool ntt_mag_ok(const u64* in, const u64* out, const NttDev& T, bool incomplete);

// Up to NTT_MULTI_MAX batches (count[i] units of n, or ring elements of 2n in
// incomplete mode) of one (n, q) transformed in one launch; every buffer
// 16-byte aligned and 16 <= n <= 4096 (2048 incomplete).  in[i] may equal out[i].
constexpr int NTT_MULTI_MAX = 64;
int ntt_multi_launch(const u64* const* in, u64* const* out, const u64* count, u32 ninst, const NttDev& T,
                     bool incomplete, bool inverse, cudaStream_t st);

// Digit decomposition fused with the forward incomplete transform: for rows
// source rows of width ring elements (2n coefficients, canonical), radix
// 2^ceil(bw / parts) from the OR of centred magnitudes *bw_or (its log2 goes
// to *rlog_out, the radix to *radix_out when not null), digit c of row k is
// written to row k * parts + c of dc (coefficients) and of ds (slot form).
// Needs 16 <= n <= 2048, rows <= 16 and 16-byte aligned dc and ds.
struct NttSrcRows {
  const u64* p[16];
};
bool ntt_digits_ok(const u64* dc, const u64* ds, u32 rows, const NttDev& T);
// narrow: the coefficient-form digits as centred int32 values (parts >= 2).
int ntt_digits_launch(const NttSrcRows& src, u32 rows, u64 width, u32 parts, const u64* bw_or, u64* rlog_out,
                      u64* radix_out, u64* dc, u64* ds, const NttDev& T, cudaStream_t st, bool narrow = false);

// Fused batched negacyclic product r = a * b mod (Y^n + 1), count polynomials
// of n words each (r may alias a or b).  Needs 16 <= n <= 4096 and 16-byte
// aligned buffers (ntt_mul_fused_ok); the C ABI falls back to three passes.
bool ntt_mul_fused_ok(const u64* a, const u64* b, const u64* r, const NttDev& T);
int ntt_mul_launch(const u64* a, const u64* b, u64* r, u64 count, const NttDev& T, cudaStream_t st);

// ---- FP64 modular arithmetic for q < 2^50 (exactness argument in ntt.cu) ----
constexpr double FP_MAGIC = 6755399441055744.0;  // 1.5 * 2^52: fl(t + M) - M rounds |t| < 2^51 to an integer
constexpr double FP_TWO52 = 4503599627370496.0;  // 2^52

__device__ __forceinline__ double fp_mulmod(double x, double w, double wh, double q2d) {
  const double h = __dmul_rn(x, w);
  const double l = __fma_rn(x, w, -h);
  const double c = __dsub_rn(__fma_rn(x, wh, FP_MAGIC), FP_MAGIC);
  return __dadd_rn(__fma_rn(-c, q2d, h), l);
}
__device__ __forceinline__ double fp_reduce(double v, double qinv, double qd) {
  const double c = __dsub_rn(__fma_rn(v, qinv, FP_MAGIC), FP_MAGIC);
  return __fma_rn(-c, qd, v);
}
// canonical word (< 2^52) -> double, and a reduced-range double -> canonical word
__device__ __forceinline__ double fp_from_word(u64 v) {
  return __dsub_rn(__longlong_as_double((long long)(v | 0x4330000000000000ULL)), FP_TWO52);
}
__device__ __forceinline__ u64 fp_to_word(double v, double qinv, double qd) {
  v = fp_reduce(v, qinv, qd);
  v = v < 0.0 ? __dadd_rn(v, qd) : v;
  return (u64)__double_as_longlong(__dadd_rn(v, FP_TWO52)) & 0x000FFFFFFFFFFFFFULL;
}


// ---- ring helpers in slot form, used by several kernels ----
// (a_e + X a_o)(b_e + X b_o) = a_e b_e + zeta a_o b_o + X (a_o b_e + a_e b_o)
// Inputs are taken by value, so outputs may alias them.
__device__ __forceinline__ void slot_mul(const ModQ& M, u64 ae, u64 ao, u64 be, u64 bo, u64 z, u64& re,
                                         u64& ro) {
  const u64 ee = mul_mod(M, ae, be);
  const u64 oo = mul_mod(M, mul_mod(M, ao, bo), z);
  const u64 x = add_mod(mul_mod(M, ao, be), mul_mod(M, ae, bo), M.q);
  re = add_mod(ee, oo, M.q);
  ro = x;
}

}  // namespace salsaa
