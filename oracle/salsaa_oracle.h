/*
 * salsaa_oracle.h — CPU restatement of the SALSAA prover hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path
 * (tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg).  The
 * product library (libsalsaa_gpu.so) never links, loads or calls it.
 *
 * It restates, in plain C with exact 64/128-bit integer arithmetic:
 *   - HEXL-convention negacyclic NTT        hexl-bindings/hexl_wrapper.cpp:213-229
 *   - incomplete-NTT ring R_q = Z_q[X]/(X^d+1) src/cyclotomic_ring.rs:484-564,700-791
 *   - power-series statement rows            src/arithmetic.rs:147-176, src/subroutines/crs.rs:43-72
 *   - every prover subroutine and protocol.rs control flow (src/protocol.rs:125-483)
 *   - the verifier checks the reference asserts inline (src/subroutines/)
 * with the reference's OS-seeded RNG replaced by a counter-based PRF (so_prf).
 */
#ifndef SALSAA_ORACLE_H
#define SALSAA_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Parameter set; field meaning follows src/protocol.rs:22-123.  The same
 * layout is used by the product header include/salsaa_gpu.h. */
typedef struct so_params {
  uint64_t d;               /* ring degree N */
  uint64_t q;               /* modulus MOD_Q */
  uint64_t module_size;     /* MODULE_SIZE: commitment-key rows */
  uint64_t wit_len;         /* WIT_LEN: witness width (ring elements per row) */
  uint64_t init_wit_rep;    /* INIT_WIT_REP: initial witness rows */
  uint64_t nof_rounds;      /* NOF_ROUNDS */
  uint64_t folding;         /* FOLDING_SCHEME (0 = SNARK) */
  uint64_t decomp_parts[12];/* DECOMP_PARTS */
} so_params;

/* --- scalar arithmetic (hexl_wrapper.cpp:34-70 semantics) --- */
uint64_t so_mul_mod(uint64_t a, uint64_t b, uint64_t q);
uint64_t so_add_mod(uint64_t a, uint64_t b, uint64_t q);
uint64_t so_sub_mod(uint64_t a, uint64_t b, uint64_t q);
uint64_t so_pow_mod(uint64_t a, uint64_t e, uint64_t q);
uint64_t so_inv_mod(uint64_t a, uint64_t q);
uint64_t so_minimal_root(uint64_t order, uint64_t q);

/* --- counter-based PRF: the deterministic challenge stream --- */
uint64_t so_prf(uint64_t seed, uint64_t domain, uint64_t index);

/* --- NTT, HEXL conventions (bit-reversed forward output, scaled inverse) --- */
int so_ntt_forward(uint64_t* a, uint64_t n, uint64_t q);
int so_ntt_inverse(uint64_t* a, uint64_t n, uint64_t q);
int so_get_roots(uint64_t n, uint64_t q, uint64_t* out);      /* bit-reversed psi^i */
int so_get_inv_roots(uint64_t n, uint64_t q, uint64_t* out);  /* bit-reversed psi^-i */
int so_multiply_poly(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q);

/* --- element-wise (hexl_wrapper.cpp:65-70,119-126,188-207,231-268) --- */
void so_eltwise_mult_mod(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q);
void so_eltwise_add_mod(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q);
void so_eltwise_sub_mod(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q);
void so_eltwise_fma_mod(uint64_t* r, const uint64_t* a, uint64_t s, const uint64_t* b, uint64_t n, uint64_t q);
void so_eltwise_reduce_mod(uint64_t* r, const uint64_t* a, uint64_t n, uint64_t q);
uint64_t so_sum(const uint64_t* a, uint64_t n, uint64_t q);
uint64_t so_sum_sq(const uint64_t* a, uint64_t n, uint64_t q);

/* --- ring R_q, incomplete-NTT ("slot") representation --- */
int so_ring_to_slot(uint64_t* out, const uint64_t* coef, uint64_t d, uint64_t q);
int so_ring_from_slot(uint64_t* out, const uint64_t* slot, uint64_t d, uint64_t q);
int so_ring_mul(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t d, uint64_t q);
int so_dense_commit(uint64_t* C, const uint64_t* A, const uint64_t* W, uint64_t n, uint64_t m, uint64_t r,
                    uint64_t d, uint64_t q);
void so_conjugate(uint64_t* r, const uint64_t* a, uint64_t d, uint64_t q);
int so_shift_factors(uint64_t* out, uint64_t d, uint64_t q);
void so_tensor(uint64_t* out, const uint64_t* cs, uint64_t k, uint64_t q);

/* --- subroutine-level entry points (parity checkers for the CUDA kernels) --- */
/* flattened witness row -> sum of squares and sumcheck transcript. */
int so_sumcheck(const uint64_t* w, uint64_t n, uint64_t q, const uint64_t* cs,
                uint64_t* claim, uint64_t* polys /* log2(n) x 3 */, uint64_t* final_v);
/* smallest quadratic non-residue mod q (the F_{q^2} shift below) */
uint64_t so_qnr(uint64_t q);
/* the same sumcheck over F_{q^2} = F_q[X]/(X^2 - shift): cs holds log2(n)
 * challenges as (re, im) pairs, polys log2(n) x 3 extension elements (re, im),
 * final_v the last folded value (re, im); the input has F_q entries. */
int so_sumcheck_fq2(const uint64_t* w, uint64_t n, uint64_t q, uint64_t shift, const uint64_t* cs,
                    uint64_t* claim, uint64_t* polys, uint64_t* final_v);
/* decompose_matrix_by_chunks: rows x width x d coef -> (rows*parts) x width x d */
int so_decompose(const uint64_t* w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q,
                 uint64_t parts, uint64_t* out, uint64_t* radix);
/* project: rows x width x d coef with J given as is_zero/sign bytes (256 x 256*rows) */
int so_project(const uint64_t* w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q,
               const uint8_t* is_zero, const uint8_t* sign, uint64_t* out);
/* commit with the CK rows of a CRS: module_size x rows ring elements (coef out) */
int so_commit_ck(const so_params* p, uint64_t crs_seed, const uint64_t* w, uint64_t rows,
                 uint64_t width, uint64_t* out);
/* fold: rows x width coef witness, ternary ring challenges c (rows x d coef) */
int so_fold(const uint64_t* w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q,
            const uint64_t* c, uint64_t* out);

/* --- sampling exactly as the prover does --- */
void so_sample_crs(const so_params* p, uint64_t crs_seed, uint64_t* m /* module_size x d */);
void so_sample_witness(const so_params* p, uint64_t seed, uint64_t* w /* rep x len x d */);

/* --- full protocol --- */
typedef struct so_timing {
  double commit, norm1, norm2, norm3, split, projection, fold, decomp, total;
} so_timing;

/* Proof size in bytes for a parameter set. */
uint64_t so_proof_size(const so_params* p);
/* One full prove.  witness may be NULL (then sampled from seed).
 * Returns 0 on success; the inline verifier's failure returns a negative code. */
int so_prove(const so_params* p, uint64_t crs_seed, uint64_t seed, const uint64_t* witness,
             uint8_t* proof, uint64_t proof_len, so_timing* t, int nthreads);
/* Stand-alone verifier over proof bytes; 0 = accept, negative = first failing check. */
int so_verify(const so_params* p, uint64_t crs_seed, uint64_t seed, const uint8_t* proof,
              uint64_t proof_len);

#ifdef __cplusplus
}
#endif
#endif
