// kernels.cuh — launchers of the SALSAA prover kernels (sm_100a).
//
// Layouts in HBM (u64 words, canonical residues mod q):
//   coefficient form  row k of a witness: width x d, element-contiguous
//   slot form         same shape; element = [NTT_n(even coeffs) | NTT_n(odd)]
// Witness rows are passed as a RowSet of base pointers, so the split step
// (src/subroutines/split.rs:45-76) is a re-view of the decomposed rows and
// never copies.
#pragma once
#include "common.cuh"
#include "ntt.cuh"

namespace salsaa {

constexpr int MAX_WROWS = 16;  // witness rows in one call
constexpr u32 CK_BLOCK = 2048; // block of the scalar-row tables, column sums and projection chunks
// Two-level split of the commitment-key powers m^(i+1) = thi[i / B] tlo[i % B]:
// a commitment CTA accumulates up to B elements before its epilogue.
constexpr u32 CK_KEY_BLOCK = 8192;

struct RowSet {
  const u64* p[MAX_WROWS];
  // bit k set: row k holds centred int32 values (decomposition digits, whose
  // magnitudes stay below the radix <= 2^25) instead of canonical u64 words;
  // p[k] then points at int32 data and element offsets count int32 values
  u32 narrow;
};

// Row pointer advanced by `elems` elements of the row's type.
__host__ __device__ inline const u64* row_advance(const u64* p, bool narrow, u64 elems) {
  return narrow ? (const u64*)((const int*)p + elems) : p + elems;
}
// True when rows 0 .. rows-1 start on word_bytes boundaries (u64 rows) or
// narrow_bytes boundaries (narrow rows): the tensor-core passes load several
// neighbouring elements of a row at a time.
inline bool rowset_aligned(const RowSet& rs, u32 rows, u32 word_bytes, u32 narrow_bytes) {
  for (u32 k = 0; k < rows && k < MAX_WROWS; k++) {
    const uintptr_t a = (uintptr_t)rs.p[k];
    if (a % (((rs.narrow >> k) & 1) ? narrow_bytes : word_bytes)) return false;
  }
  return true;
}
// Element i of a coefficient-form row as a canonical residue mod q.
__device__ __forceinline__ u64 wres(const u64* p, bool narrow, u64 i, u64 q) {
  if (narrow) {
    const long long v = __ldg((const int*)p + i);
    return v < 0 ? (u64)(v + (long long)q) : (u64)v;
  }
  return __ldg(p + i);
}

// Per-proof device state that data-dependent steps write and later kernels read.
struct DevState {
  u64 seed;
  u64 bw_or[16];   // decomposition: OR of centred magnitudes, per decomposition index
  u64 rlog[16];    // decomposition: radix log2, per decomposition index
  u64 proj_flag;   // projection: set when a witness value does not fit int8
};

// Indices of the scalar rows one commitment pass covers (passed by value).
constexpr u32 SC_MAX_ROWS = 64;
struct ScRowList {
  u32 n;
  unsigned char idx[SC_MAX_ROWS];
};

// ---- statement rows -------------------------------------------------------
enum RowType : int { ROW_CK = 0, ROW_TENSOR = 1, ROW_PERIODIC = 2, ROW_ONES = 3 };

// Scalar-structured row: value(i) = s_hi[i / B'] * s_lo[i % B'] (times a ring
// base for TENSOR rows).  Tables are produced per commit call.
struct ScalarRowDesc {
  int type;
  u32 round, rep;  // TENSOR: which challenge stream
  u32 K;           // TENSOR: number of element-index challenges of the row
  u32 cw;          // PERIODIC: period
  const u64* cj;   // PERIODIC: cw scalars
};

// ---- launchers (all asynchronous on `st`; return 0 or a negative code) ----
int launch_gen_crs(u64* m_coef, u32 rows, u32 d, u64 q, u64 crs_seed, cudaStream_t st);
int launch_ck_tables(const u64* m_slot, u32 rows, const NttDev& T, const ModQ& M, u64 L, u64* tlo, u64* thi,
                     cudaStream_t st);
// Byte planes of the key tables for the tensor-core commitment (q < 2^56):
// tl8[s][mt][m][lo], m = (r_local * 3 + comp) * 7 + byte for the 6 key rows
// of M tile mt, comp = (even, odd, zeta * odd); rows m >= 126 are zero.
constexpr u32 CKM_ROWS = 6, CKM_BM = 128;
inline u64 ck_tl8_bytes(u32 nck, u32 n, u32 bt) { return (u64)n * ((nck + CKM_ROWS - 1) / CKM_ROWS) * CKM_BM * bt; }
int launch_ck_tl8(const u64* tlo, u32 nck, u32 n, u32 bt, bool packed, uint8_t* tl8, cudaStream_t st);
// tcgen05 key table: for each 128-element chunk position cc and slot s, the
// byte image of the B operand (rows (key row, comp c|d, byte), padded to nkp)
// in the canonical K-major shared-memory layout; q < 2^56, nck <= 18.
constexpr u32 CKU_MAX_KEYS = 18, CKU_MAX_WROWS = 9;
constexpr u32 CKU_MULTI_MAX = 8;  // witnesses per launch of the multi-witness key-row product
inline u32 ck_tk8_nkp(u32 nck) { return ((nck * 14 + 15) / 16) * 16; }
inline u64 ck_tk8_bytes(u32 nck, u32 n, u32 bt) { return (u64)bt * n * ck_tk8_nkp(nck); }
int launch_ck_tk8(const u64* tlo, u32 nck, u32 n, u32 bt, bool packed, uint8_t* tk8, cudaStream_t st);
// TENSOR rows on tcgen05 over the coefficient-form witness (see ck_umma.cu).
constexpr u64 SC_IMG_BYTES = (u64)CK_BLOCK * 128;
constexpr u32 SC_UMMA_MAX_ROWS = 18;
int launch_sc_umma(const RowSet& wc, u32 rows, u64 width, u32 d, u32 Bw, u32 nhi, const ScRowList& tl,
                   const u64* s_lo, const u64* s_hi, const ModQ& M, u64* acc, bool plain, uint8_t* img, u32* flags,
                   u64 flag_cap, cudaStream_t st);
// First sumcheck pass (rounds 0..3 of both repetitions) on tcgen05 through the
// Gram matrices of 16-element groups (see ck_umma.cu): launch_nc_gram writes
// the folded vectors and the Gram matrices, or raises the flag word after them
// when a value does not fit four signed byte limbs; launch_nc_gram_sums adds
// the round sums unless the flag is raised.
bool nc_gram_ok(const RowSet& w, u32 rows, u64 nlen, u64 q);
int launch_nc_gram(const RowSet& w, u32 rows, u64 nlen, const ModQ& M, const DevState* ds, u32 round, u64* out,
                   u64 sout, u64* gram, bool plain, cudaStream_t st);
int launch_nc_gram_sums(const u64* gram, u32 rows, const ModQ& M, const DevState* ds, u32 round, u64* sums, u32 nr,
                        bool plain, cudaStream_t st);
// Nonzero (and the last error set) when a tensor-core kernel's bounded wait gave up.
int tc_error_check();
int launch_gen_witness(u64* w, u32 rows, u64 width, u32 d, u64 q, const DevState* ds, cudaStream_t st);
int launch_expand_i8(const int8_t* in, u64 n, u64 q, u64* out, cudaStream_t st);
int launch_fill(u64* p, u64 n, u64 v, cudaStream_t st);
// r[i] = r[i] * b[i] mod q (canonical inputs)
int launch_pointwise_mul(u64* r, const u64* b, u64 n, u64 q, cudaStream_t st);

// sumcheck of `rows` witness rows (coefficient form, length nlen each), both
// amplification repetitions at once; see sumcheck implementation for buffers.
struct SumcheckBufs {
  u64* a;     // 2 * rows * nlen/2
  u64* b;     // 2 * rows * nlen/4
  u64* sums;  // 2 * nr * rows * 3 (zeroed by the launcher)
  u64* cap;   // 2 * rows * d: vector after log2(width) rounds
  u64* gram;  // rows * 256 + 1 (Gram matrices and a flag word) or null: first pass on tcgen05
};
int launch_sumcheck(RowSet w, u32 rows, u64 nlen, u32 d, const ModQ& M, const DevState* ds, u32 round,
                    SumcheckBufs B, u64* proof_claims, u64* proof_rep0, u64* proof_rep1, cudaStream_t st);
// Independent sumchecks of `count` <= 64 vectors of power-of-two lengths (one
// repetition each; instance i uses the norm-check challenges of (round, i)):
// claims[i] and the round polynomials of instance i at polys + 3 * sum_{i'<i} log2 len.
// The sumcheck over F_{q^2} = F_q[X]/(X^2 - shift) for count <= 64 vectors of
// uneven power-of-two lengths; scratch holds count * max_rounds * 6 +
// 1.5 * sum(lens) words.  polys: per instance log2(len) x 3 x (re, im).
int launch_sumcheck_fq2_batch(const u64* const* vecs, const u64* lens, u32 count, const ModQ& M, u64 shift,
                              u64 seed, u32 round, u64* claims, u64* polys, u64* scratch, cudaStream_t st);
int launch_sumcheck_batch(const u64* const* vecs, const u64* lens, u32 count, const ModQ& M, u64 seed, u32 round,
                          u64* claims, u64* polys, cudaStream_t st);
// norm_check_3 outputs: rhs (coef, into proof) and each repetition's ring base (slot).
int launch_norm3(const u64* cap, u32 rows, u32 nr, const NttDev& T, const ModQ& M, const DevState* ds,
                 u32 round, u64* proof_rep0, u64* proof_rep1, u64* base0, u64* base1, cudaStream_t st);

// mag_ready: ds->bw_or[didx] already holds the OR of the inputs' centred
// magnitudes (accumulated by the transforms that produced or read them).
int launch_decompose(RowSet in, u32 rows, u64 width, u32 d, u64 q, u32 parts, u32 didx, DevState* ds,
                     u64* out, u64* proof_radix, cudaStream_t st, bool mag_ready = false);
// The same, also writing the digits' slot form to out_slot (one fused pass
// with the forward transform when the shapes allow, else decomposition then
// transform).  With narrow_out given, the fused pass with parts >= 2 writes
// the coefficient-form digits as centred int32 values and sets *narrow_out.
int launch_decompose_ntt(RowSet in, u32 rows, u64 width, u32 d, u64 q, u32 parts, u32 didx, DevState* ds,
                         u64* out, u64* out_slot, u64* proof_radix, const NttDev& T, cudaStream_t st,
                         bool mag_ready = false, bool* narrow_out = nullptr);

// J as bit masks (CUDA-core path), as an int8 matrix 256 x cw (tensor-core
// path, optional) and cj[l] = sum_k J[k][l] (optional).
// Jc (optional): J again, as the tcgen05 A-operand image: for each 128-element
// chunk, both 128-row halves in the canonical K-major layout (256 x cw bytes).
int launch_proj_tables(const DevState* ds, u32 round, u32 cw, u32* pos_mask, u32* neg_mask, int8_t* J, u64* cj,
                       u64 q, cudaStream_t st, int8_t* Jc = nullptr);
// Tensor-core path when d is a multiple of 128 and J is given; exact CUDA-core
// recomputation (chosen on the device) whenever a value does not fit int8.
int launch_project(RowSet in, u32 rows, u64 width, u32 d, u64 q, const u32* pos_mask, const u32* neg_mask,
                   const int8_t* J, DevState* ds, u64* out, cudaStream_t st, const int8_t* Jc = nullptr);
// tcgen05 projection over chunks (see ck_umma.cu); Jc from launch_proj_tables.
int launch_project_umma(RowSet in, u32 rows, u64 nch, u32 d, u64 q, u32 cw, const int8_t* Jc, u64* out, u64* flag,
                        cudaStream_t st);

int launch_fold_challenge(const DevState* ds, u32 round, u32 rows, u32 d, u64 q, u64* c_coef, cudaStream_t st);
// pre: scratch of rows x n x 6 words (Shoup constants of the challenges)
int launch_fold(RowSet w_slot, u32 rows, u64 width, const NttDev& T, const ModQ& M, const u64* c_slot, u64* pre,
                u64* out_slot, cudaStream_t st);

// <statement rows, witness rows> in slot form.  acc: (nck + nsc) x rows x d
// scratch; out_slot: results in statement order given by `order`.
struct CommitArgs {
  RowSet w;          // slot-form witness rows
  RowSet wc;         // the same rows in coefficient form (used when coef_sc)
  bool coef_sc;      // scalar rows over wc, their sums moved to slot form after
  u32 rows;
  u64 width;
  u32 nck;           // commitment-key rows (statement rows 0..nck-1)
  const u64* tlo;    // nck x ck_bt x 3n
  const u64* thi;    // nck x ck_nhi x d
  u32 ck_bt;         // table block: min(L, CK_KEY_BLOCK)
  u32 ck_nhi;        // L / ck_bt
  u32 nsc;           // scalar rows
  const ScalarRowDesc* sc_desc_dev;  // nsc descriptors in device memory
  const int* sc_types_host;          // their types, on the host (required when nsc > 0)
  uint8_t* sc_img;   // scratch for the tcgen05 TENSOR-row pass (SC_IMG_BYTES), or null
  u32* sc_flags;     // scratch: one word per CTA of that pass
  u64 sc_flag_cap;   // words of sc_flags
  cudaStream_t st2;  // optional: statement rows on this stream beside the key rows
  cudaEvent_t ev_fork, ev_join;
  const u64* const* sc_base_dev;     // nsc ring bases (slot form) or null (= 1)
  u64* sc_lo;        // scratch nsc x CK_BLOCK
  u64* sc_hi;        // scratch nsc x max(width / CK_BLOCK, 1)
  const uint8_t* tl8;  // tensor-core key table (see launch_ck_tl8) or null
  const uint8_t* tk8;  // tcgen05 key table (see launch_ck_tk8) or null
  u64* colsum;       // scratch colsum_rows x min(width, CK_BLOCK) x d (scalar rows only)
  u32 colsum_rows;   // capacity of colsum in witness rows
  u64* acc;          // scratch (nck + nsc) x rows x d
  u64* out_slot;     // (nck + nsc) x rows x d, statement order = CK rows then scalar rows
};
int launch_commit(const CommitArgs& a, const NttDev& T, const ModQ& M, const DevState* ds, cudaStream_t st);
// Key rows of launch_commit on tcgen05 when ck_umma_ok (see ck_umma.cu).
bool ck_umma_ok(const CommitArgs& a, u32 n);
// Bw elements per block, G blocks (one key block apart) per CTA.
int launch_ck_umma(const CommitArgs& a, u32 n, u32 Bw, u32 G, const ModQ& M, const u64* zeta, bool plain,
                   cudaStream_t st);
// The block width and grouping launch_commit uses for a witness of this shape.
void ck_umma_shape(u64 width, u32 rows, u32 n, u32 ck_bt, u32* Bk, u32* G);
// Key rows of several witnesses (a[i].w, a[i].rows, a[i].width; the same
// context tables) in one launch; witness i's sums go to a[i].acc (nck x
// a[i].rows ring elements, zeroed by the caller).
int launch_ck_umma_multi(const CommitArgs* a, u32 ninst, u32 n, const ModQ& M, const u64* zeta, cudaStream_t st);
// The finalisation of launch_commit (key rows only): acc -> slot-form outputs.
int launch_commit_finalize(const u64* acc, u32 nck, u32 rows, const NttDev& T, const ModQ& M, u64* out,
                           cudaStream_t st);

// Commitment of a witness of width w from the commitment of its split halves
// (slot form): out[j][k] = t0_j * R[j][k] + t1_j * R[j][K + k] for statement
// rows j < nck + nsc, where (t0_j, t1_j) is row j's tensor factor of the
// layer of length w (verifier_split's relation, src/subroutines/split.rs:171-221).
// R has `ncols` witness columns per row; out has K.
struct DeriveArgs {
  const u64* R;
  u32 ncols, K, nck, nsc;
  u64 w;
  const u64* tlo;
  const u64* thi;
  u32 ck_bt, ck_nhi;
  bool packed;  // tlo stored as 25-bit limbs
  const ScalarRowDesc* sc_desc_dev;
  u64* out;
};
int launch_derive(const DeriveArgs& a, const NttDev& T, const ModQ& M, const DevState* ds, cudaStream_t st);

}  // namespace salsaa
