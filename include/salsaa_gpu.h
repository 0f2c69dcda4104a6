/*
 * salsaa_gpu.h — C ABI of libsalsaa_gpu.so, the B200 (sm_100a) SALSAA prover.
 *
 * Two tiers, both plain C (pointers, sizes, integer status codes):
 *
 *  1. HEXL-compatible tier.  The twenty symbols that the reference's Rust
 *     crate binds from libhexl_wrapper.so (src/hexl/bindings.rs:1-74), with
 *     the signatures of hexl-bindings/hexl_wrapper.cpp.  Buffers are
 *     caller-owned HOST memory; array operations run on the GPU (one CUDA
 *     stream and staging buffer per calling thread), scalar ones on the host.
 *     They are thread-safe, and their tables are built once under a lock
 *     (the reference's NTTCache, hexl_wrapper.cpp:11-32, is not).
 *
 *  2. Device tier.  Subroutine-granularity entry points that keep witnesses,
 *     commitment-key tables and all intermediate state resident in HBM:
 *     one call per prover step (src/subroutines/) or per whole proof
 *     (src/protocol.rs:125-483).  Status 0 = success, negative = error
 *     (salsaa_last_error() gives the message); no C++ exception crosses the ABI.
 *
 * All arithmetic is exact modulo q (q < 2^62; the protocol moduli are 50-bit).
 * Randomness (CRS, witness, challenges) comes from a counter-based PRF keyed by
 * the caller's seeds, one domain per (kind, round, repetition).  A proof is the
 * prover's messages in protocol order as canonical little-endian u64 words in
 * coefficient form, after an 8-word header (magic "SALSAAP1", d, q,
 * module_size, wit_len, init_wit_rep, nof_rounds, folding).
 */
#ifndef SALSAA_GPU_H
#define SALSAA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ===================================================================== */
/* 1. HEXL-compatible tier (hexl-bindings/hexl_wrapper.cpp)               */
/* ===================================================================== */

/* hexl_wrapper.cpp:34-36 — a*b mod modulus */
uint64_t multiply_mod(uint64_t a, uint64_t b, uint64_t modulus);
/* hexl_wrapper.cpp:38-41 — (a+b) mod modulus */
uint64_t add_mod(uint64_t a, uint64_t b, uint64_t modulus);
/* hexl_wrapper.cpp:43-45 — (a-b) mod modulus */
uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t modulus);
/* hexl_wrapper.cpp:61-63 — a^b mod modulus */
uint64_t power_mod(uint64_t a, uint64_t b, uint64_t modulus);
/* hexl_wrapper.cpp:52-54 — a^-1 mod modulus (0 if not invertible) */
uint64_t inv_mod(uint64_t a, uint64_t modulus);
/* hexl_wrapper.cpp:47-50 — library-owned table of n roots, psi^i at bit-reversed i */
const uint64_t* get_roots(size_t n, uint64_t modulus);
/* hexl_wrapper.cpp:56-59 — library-owned table of n inverse roots, psi^-i at bit-reversed i */
const uint64_t* get_inv_roots(size_t n, uint64_t modulus);
/* hexl_wrapper.cpp:65-67 — result = operand1 * operand2 (element-wise) */
void eltwise_mult_mod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, uint64_t n,
                      uint64_t modulus);
/* hexl_wrapper.cpp:68-70 — result = operand1 * operand2 + operand3 */
void eltwise_fma_mod(uint64_t* result, const uint64_t* operand1, uint64_t operand2, const uint64_t* operand3,
                     uint64_t n, uint64_t modulus);
/* hexl_wrapper.cpp:188-196 */
void eltwise_add_mod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, size_t n,
                     uint64_t modulus);
/* hexl_wrapper.cpp:199-207 */
void eltwise_sub_mod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, size_t n,
                     uint64_t modulus);
/* hexl_wrapper.cpp:119-126 — any u64 input reduced mod modulus */
void eltwise_reduce_mod(uint64_t* result, const uint64_t* operand, size_t n, uint64_t modulus);
/* hexl_wrapper.cpp:158-186 — same result as eltwise_reduce_mod */
void eltwise_reduce_mod_naive(uint64_t* result, const uint64_t* operand, size_t n, uint64_t modulus);
/* hexl_wrapper.cpp:73-94 — negacyclic product in Z_q[X]/(X^n+1) */
void multiply_poly(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, uint64_t n,
                   uint64_t modulus);
/* hexl_wrapper.cpp:96-117 — kept for link compatibility; computes the
 * negacyclic product (the reference's body is unused and out of bounds) */
void polynomial_multiply_cyclotomic_mod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2,
                                        size_t phi, uint64_t mod_q);
/* hexl_wrapper.cpp:213-220 — forward negacyclic NTT in place (bit-reversed output) */
void ntt_forward_in_place(uint64_t* operand, size_t n, uint64_t modulus);
/* hexl_wrapper.cpp:222-229 — inverse NTT in place (bit-reversed input, scaled by 1/n) */
void ntt_inverse_in_place(uint64_t* operand, size_t n, uint64_t modulus);
/* hexl_wrapper.cpp:231-237 — sum mod modulus */
uint64_t sum(const uint64_t* operand1, uint64_t n, uint64_t modulus);
/* hexl_wrapper.cpp:239-260 — same value as sum() */
uint64_t sum_fast(const uint64_t* operand1, uint64_t n, uint64_t modulus);
/* hexl_wrapper.cpp:262-268 — sum of squares mod modulus */
uint64_t sum_sq(const uint64_t* operand1, uint64_t n, uint64_t modulus);
/* hexl_wrapper.cpp:271-276 — same value as sum_sq() */
uint64_t sum_sq_fast(const uint64_t* operand1, uint64_t n, uint64_t modulus);

/* ===================================================================== */
/* 2. Device tier                                                         */
/* ===================================================================== */

/* Parameter set (src/protocol.rs:22-123). */
typedef struct salsaa_params {
  uint64_t d;                /* ring degree N (power of two, 4..512) */
  uint64_t q;                /* modulus MOD_Q, q = 1 mod d, q < 2^62 */
  uint64_t module_size;      /* MODULE_SIZE: commitment-key rows */
  uint64_t wit_len;          /* WIT_LEN: witness width in ring elements (power of two) */
  uint64_t init_wit_rep;     /* INIT_WIT_REP */
  uint64_t nof_rounds;       /* NOF_ROUNDS */
  uint64_t folding;          /* FOLDING_SCHEME: 0 = SNARK, 1 = folding */
  uint64_t decomp_parts[12]; /* DECOMP_PARTS */
} salsaa_params;

typedef struct salsaa_ctx salsaa_ctx;       /* parameters + CRS tables on one GPU */
typedef struct salsaa_prover salsaa_prover; /* workspace + stream for one proof in flight */

/* Phase timings in milliseconds, named as the reference's t_* totals
 * (src/protocol.rs:474-482). */
typedef struct salsaa_timing {
  double commit, norm1, norm2, norm3, split, projection, fold, decomp, total;
} salsaa_timing;

/* Last error message of the calling thread. */
const char* salsaa_last_error(void);
/* Kernel launches this library has issued since it was loaded. */
uint64_t salsaa_kernel_launches(void);
/* 0 while no bounded wait inside a kernel (tensor-core and bulk-copy
 * mbarriers of the current device) has given up; -4 with a message once one
 * has, in which case the results of that launch are invalid.  Call it after
 * the launches in question have finished (after synchronizing their stream). */
int salsaa_device_status(void);
/* Device-time trace for measurement (off by default): enable/reset, then read
 * the summed device time (CUDA events on the launching stream), summed
 * algorithmic work and launch count of a traced kernel by name.  Traced:
 * "ck_umma_kernel" (work = algorithmic HBM bytes: the slot-form witness read
 * once and the accumulators written once), "ck_umma_kernel:int8" (the same
 * launches; work = int8 operations the tensor cores execute, 2 per byte-limb
 * product), "ck_umma_kernel:mac" (the same launches; work = exact mod-q
 * multiply-accumulates of the ring products), "ck_mma_kernel" (int8
 * operations), "nc_gram_kernel" (bytes), "ntt_kernel" (16 bytes per
 * coefficient) and "ntt_mul_kernel" (24 bytes per coefficient).  Reading
 * waits for the traced launches. */
void salsaa_trace_enable(int on);
int salsaa_trace_read(const char* name, double* total_ms, double* total_work, uint64_t* launches);
/* Fill *out with preset "A0".."C2", "F0".."F2" (src/protocol.rs:28-123). */
int salsaa_params_preset(const char* name, salsaa_params* out);
/* Proof length in bytes for a parameter set (0 if the set is invalid). */
uint64_t salsaa_proof_size(const salsaa_params* p);
/* Device bytes one in-flight proof needs (workspace), for admission control. */
uint64_t salsaa_workspace_bytes(const salsaa_params* p);

/* CRS::gen_crs + compute_commitment_keys (src/subroutines/crs.rs:23-72):
 * samples the module from crs_seed and builds the key tables on `device`. */
int salsaa_ctx_create(const salsaa_params* p, uint64_t crs_seed, int device, salsaa_ctx** out);
void salsaa_ctx_destroy(salsaa_ctx* ctx);

/* One proof slot: device workspace sized for the context's parameters and a
 * private CUDA stream.  Slots of one context may run concurrently. */
int salsaa_prover_create(salsaa_ctx* ctx, salsaa_prover** out);
void salsaa_prover_destroy(salsaa_prover* pr);
/* The slot's CUDA stream (cudaStream_t). */
void* salsaa_prover_stream(salsaa_prover* pr);

/* protocol() of src/protocol.rs:125-483, asynchronous on the slot's stream.
 * d_witness: device pointer to init_wit_rep x wit_len x d coefficients, or
 * NULL to sample the witness from `seed`; d_proof: device buffer of
 * salsaa_proof_size() bytes.  No host synchronisation inside. */
int salsaa_prover_enqueue(salsaa_prover* pr, uint64_t seed, const uint64_t* d_witness, uint8_t* d_proof);
/* Host-buffer variant of salsaa_prover_enqueue, still asynchronous: copies
 * h_witness (init_wit_rep x wit_len x d words; NULL = sample from seed) to
 * the slot's workspace, proves, and copies the proof to h_proof, all on the
 * slot's stream.  For overlap the host buffers should be page-locked; both
 * must then stay valid, and the witness unchanged, until salsaa_prover_query
 * reports the proof done (or salsaa_prover_sync returns). */
int salsaa_prover_enqueue_host(salsaa_prover* pr, uint64_t seed, const uint64_t* h_witness, uint8_t* h_proof);
/* Short-witness variant of salsaa_prover_enqueue_host: h_witness holds the
 * init_wit_rep x wit_len x d coefficients as centred signed bytes (value v
 * stands for v mod q), one byte each instead of eight, so the upload moves an
 * eighth of the bytes; the slot expands them on the device.  The witness of
 * the reference's relation is short (random_bounded, ternary in every
 * parameter set), so it always fits.  Proof bytes equal those of
 * salsaa_prover_enqueue_host for the same residues.  The upload runs on the
 * slot's own copy stream into one of two staging buffers (allocated on the
 * first call), so it may start while the slot's previous proof still runs;
 * the same buffer rules as salsaa_prover_enqueue_host apply. */
int salsaa_prover_enqueue_host_i8(salsaa_prover* pr, uint64_t seed, const int8_t* h_witness, uint8_t* h_proof);
/* No reference counterpart.  With on != 0 the slot's later proofs run each
 * round's projection on a second stream beside the norm-check sumcheck
 * (results unchanged): lower latency for a proof alone on the GPU, slightly
 * lower throughput when many slots already fill it.  Off by default. */
int salsaa_prover_set_overlap(salsaa_prover* pr, int on);
/* No reference counterpart.  With on != 0 the slot captures a proof's launch
 * sequence as a CUDA graph on its first enqueue for a (witness, proof) buffer
 * pair and replays it for later proofs into the same buffers, changing only
 * the seed (fewer launch gaps; results unchanged).  A new buffer pair is
 * captured again; if a capture fails the slot launches directly.  Per-phase
 * times (salsaa_prover_timing) are not kept for replayed proofs, and replay
 * is skipped while salsaa_trace_enable is on.  Off by default. */
int salsaa_prover_set_graph(salsaa_prover* pr, int on);
/* 1 while the last enqueued proof runs, 0 when done, negative on error. */
int salsaa_prover_query(salsaa_prover* pr);
int salsaa_prover_sync(salsaa_prover* pr);
/* Per-phase device times of the last completed proof (after sync). */
int salsaa_prover_timing(salsaa_prover* pr, salsaa_timing* t);

/* Blocking whole proof through host buffers: copies h_witness (or samples
 * it when NULL) to the GPU, proves, copies the proof to h_proof. */
int salsaa_prove(salsaa_ctx* ctx, uint64_t seed, const uint64_t* h_witness, uint8_t* h_proof,
                 uint64_t proof_len);

/* Blocking verification of a proof made with this context's parameters and
 * CRS and the given seed: the verifier's inline checks of the reference
 * (verify_decomp src/subroutines/decomp.rs:69-112, verify_norm_check_2/3
 * src/subroutines/fast_norm_check.rs:352-462, verifier_split
 * src/subroutines/split.rs:171-221, verify_batching / verifier_fold /
 * verifier_join src/subroutines/project.rs:205-275, fold.rs:58-67, and the
 * final check src/protocol.rs:464-472, which the reference runs inside
 * protocol() with assert!s).  Returns 0 when the check ran, with *verdict 0
 * for accept or a negative code naming the failed check (-3 header, -5
 * length, -20/-21 decomposition, -30/-31 sumcheck, -32 norm3, -40/-41 split,
 * -50 batching, -60 final check); a negative return is an API or CUDA error.
 * Uses the context's blocking slot, like salsaa_prove. */
int salsaa_verify(salsaa_ctx* ctx, uint64_t seed, const uint8_t* h_proof, uint64_t proof_len, int* verdict);

/* ---- serving: continuous batching on one GPU ---- */
/* No reference counterpart (the reference proves one statement per process,
 * src/main.rs:1-11).  A service holds parameter sets, each with a fixed number
 * of proof slots allocated at registration inside an HBM budget; requests are
 * admitted onto free slots as earlier proofs finish, and admitted proofs run
 * concurrently.  Proof bytes equal those of salsaa_prove() for the same
 * (parameters, CRS seed, seed, witness). */
typedef struct salsaa_server salsaa_server;
int salsaa_server_create(int device, uint64_t hbm_budget_bytes, salsaa_server** out);
int salsaa_server_register(salsaa_server* s, const salsaa_params* p, uint64_t crs_seed, uint32_t slots,
                           int* set_id);
/* Queue one proof; d_witness may be NULL (sampled from seed); d_proof is a
 * device buffer of salsaa_proof_size() bytes that must stay valid until done. */
int salsaa_server_submit(salsaa_server* s, int set_id, uint64_t seed, const uint64_t* d_witness, uint8_t* d_proof,
                         uint64_t* ticket);
/* Cap the proofs running at once over all sets (0 = only the slots limit). */
int salsaa_server_limit(salsaa_server* s, uint32_t max_inflight);
/* Retire finished proofs and admit queued ones; returns requests in flight. */
int salsaa_server_progress(salsaa_server* s);
/* 1 pending, 0 done (latency from submit and from admission, ms), < 0 failed. */
int salsaa_server_poll(salsaa_server* s, uint64_t ticket, double* latency_ms, double* run_ms);
/* Withdraw a queued request: 0 = removed (the ticket is forgotten and d_proof
 * is free again), 1 = already admitted (it runs to completion; poll it as
 * usual), < 0 = unknown ticket.  Proofs in flight are never interrupted. */
int salsaa_server_cancel(salsaa_server* s, uint64_t ticket);
void salsaa_server_destroy(salsaa_server* s);

/* ---- kernel schedules chosen by the autotuner ---- */
/* No reference counterpart (the reference's HEXL NTT has a fixed schedule).
 * The register-path NTT (16 <= n <= 4096, 16-byte aligned buffers) runs one
 * of: variant 0 = one 4096-coefficient tile per CTA; 1 = the same with FP64
 * butterflies (q < 2^50); variant 2, 3 or 4 = persistent CTAs that stage their
 * tiles with bulk copies (cp.async.bulk) that many tiles ahead; 5, 6, 7 = the
 * same with FP64 butterflies (q < 2^50); ctas_per_sm caps the resident CTAs
 * per SM (0 = as many as fit).  The choice is kept per (log2 n, incomplete, inverse,
 * wide_modulus = q >= 2^50, large = at least 2^22 coefficients in the call);
 * every variant gives the same outputs.  Untuned default: variant 0.
 * salsaa_b200/tune.py times the candidates on the GPU and writes a table file
 * ("ntt <log_n> <incomplete> <inverse> <wide> <large> <variant> <ctas_per_sm>"
 * per line, and the "fold" line below); the library loads it the first time a
 * transform launches, from $SALSAA_TUNE_FILE or tune_table.txt beside the
 * library.  salsaa_tune_load(NULL) reloads that file, salsaa_tune_load(path)
 * another (returns the entries read, < 0 if unreadable), salsaa_tune_reset()
 * restores the untuned defaults.  Schedules are process-wide. */
int salsaa_tune_load(const char* path);
int salsaa_tune_reset(void);
int salsaa_ntt_tune_set(uint32_t log_n, int incomplete, int inverse, int wide_modulus, int large, int variant,
                        int ctas_per_sm);
int salsaa_ntt_tune_get(uint32_t log_n, int incomplete, int inverse, int wide_modulus, int large, int* variant,
                        int* ctas_per_sm);
/* The fold's ring products (salsaa_fold and the prover's fold): variant 0 =
 * integer Shoup products, 1 = FP64 products (used only when q < 2^50); the
 * same outputs.  Table line: "fold <variant>".  _get returns the variant. */
int salsaa_fold_tune_set(int variant);
int salsaa_fold_tune_get(void);

/* ---- subroutine-level entry points (device pointers, cudaStream_t) ---- */

/* Batched negacyclic NTT.  incomplete = 0: `count` polynomials of n
 * coefficients; incomplete = 1: `count` ring elements of degree d = n in the
 * reference's IncompleteNTT layout (two size-n/2 transforms per element,
 * src/cyclotomic_ring.rs:484-556).
 * d_in may equal d_out. */
int salsaa_ntt(const uint64_t* d_in, uint64_t* d_out, uint64_t n, uint64_t count, uint64_t q, int inverse,
               int incomplete, void* stream);

/* Many uneven batches of one transform in ONE launch: the batched form of
 * salsaa_ntt (ntt_forward_in_place / ntt_inverse_in_place,
 * hexl-bindings/hexl_wrapper.cpp:213-229, and the IncompleteNTT conversions,
 * src/cyclotomic_ring.rs:484-556) for `ninst` <= 64 batches, batch i being
 * counts[i] units at d_in[i] -> d_out[i] (host arrays of device pointers;
 * d_in[i] may equal d_out[i]).  n and incomplete mean what they mean for
 * salsaa_ntt; needs 16 <= n <= 4096 (register path) and 16-byte aligned
 * buffers.  Outputs equal salsaa_ntt on each batch. */
int salsaa_ntt_multi(const uint64_t* const* d_in, uint64_t* const* d_out, const uint64_t* counts, uint32_t ninst,
                     uint64_t n, uint64_t q, int inverse, int incomplete, void* stream);

/* Many independent norm-check sumchecks in a few launches: the batched form
 * of norm_check_1 + sum_check (src/subroutines/fast_norm_check.rs:135-320) for
 * `count` <= 64 vectors of uneven power-of-two lengths (2..2^30), one
 * repetition each.  Instance i draws its round challenges from the
 * norm-check stream of (seed, round, repetition i).  d_vecs and lens are
 * host arrays (device pointers, lengths); d_claims gets count sums of squares
 * and d_polys the round polynomials (f0, f1, f2) of instance 0, then 1, ...
 * (log2 len_i rounds each).  Each pass level over all instances is one
 * persistent launch over equal tiles; one launch finishes every instance. */
int salsaa_sumcheck_batch(const uint64_t* const* d_vecs, const uint64_t* lens, uint32_t count, uint64_t q,
                          uint64_t seed, uint64_t round, uint64_t* d_claims, uint64_t* d_polys, void* stream);

/* The same norm-check sumcheck over the quadratic extension F_{q^2} =
 * F_q[X]/(X^2 - s), with the QuadraticExtension product of
 * src/quadratic_extension.rs:30-58 and s = salsaa_fq2_shift(q), the smallest
 * quadratic non-residue mod q (so the extension is a field): challenges and
 * folded values in F_{q^2}, inputs in F_q.  Instance i draws challenge j as
 * two PRF words (indices 2j, 2j + 1) of the domain (6, round, i).  d_claims:
 * count sums of squares (F_q); d_polys: per instance log2(len) x 3 extension
 * elements (f0, f1, f2), each as (re, im) words.  One launch per round level
 * covers every instance that still has rounds. */
uint64_t salsaa_fq2_shift(uint64_t q);
int salsaa_sumcheck_fq2_batch(const uint64_t* const* d_vecs, const uint64_t* lens, uint32_t count, uint64_t q,
                              uint64_t seed, uint64_t round, uint64_t* d_claims, uint64_t* d_polys, void* stream);

/* Dense ring-matrix commitment C = A * W over R_q: parallel_dot_matrix_matrix
 * (src/arithmetic.rs:429-457) in the Ajtai shape, C[j][c] = sum_i A[j][i] W[c][i].
 * The key holds A (n x m ring elements of degree d, coefficient form, given
 * once) prepared for the tensor cores (q < 2^56, n <= 18) or CUDA cores.
 * m is a power of two >= 128, n <= 64, d in 4..512, q = 1 mod d. */
typedef struct salsaa_dense_key salsaa_dense_key;
int salsaa_dense_key_create(const uint64_t* d_a, uint64_t n, uint64_t m, uint64_t d, uint64_t q, void* stream,
                            salsaa_dense_key** out);
void salsaa_dense_key_destroy(salsaa_dense_key* key);
/* d_w: r columns of m ring elements each (r x m x d, coefficient form);
 * d_c: n x r ring elements (coefficient form, row j = key row j).  d_w_slot is
 * an optional r x m x d workspace for W's NTT (NULL: allocated on the stream).
 * Calls sharing one key must not overlap on the GPU (the key holds the
 * accumulators). */
int salsaa_dense_commit(salsaa_dense_key* key, const uint64_t* d_w, uint64_t r, uint64_t* d_c, uint64_t* d_w_slot,
                        void* stream);

/* Self-test of the int8 tensor-core building block used by the commitment
 * kernels (tcgen05.mma kind::i8, accumulator in tensor memory): d_out (128 x n,
 * int32, row-major) = A (128 x k bytes, row-major) * B (n x k bytes)^T, with
 * 16 <= n <= 256 a multiple of 16 and k a multiple of 32 up to 256.  No
 * reference counterpart; it exists so the operand and descriptor encoding can
 * be checked against an exact integer product. */
int salsaa_selftest_umma_i8(const uint8_t* d_a, const uint8_t* d_b, uint32_t n, uint32_t k, int32_t* d_out,
                            void* stream);

/* Batched negacyclic product r = a * b mod (Y^n + 1) of `count` polynomial
 * pairs: the device-resident, batched form of multiply_poly
 * (hexl-bindings/hexl_wrapper.cpp, called from src/hexl/bindings.rs:60-66).
 * Inputs canonical in [0, q).  For 16 <= n <= 4096 and 16-byte aligned
 * buffers one fused kernel does forward, product and inverse per tile;
 * otherwise three passes with a temporary buffer.  d_r may alias d_a/d_b. */
int salsaa_poly_mul(const uint64_t* d_a, const uint64_t* d_b, uint64_t* d_r, uint64_t n, uint64_t count, uint64_t q,
                    void* stream);

/* parallel_dot_series_matrix with the commitment-key rows of ctx
 * (src/arithmetic.rs:459-505): d_w is rows x width x d coefficient form;
 * d_out receives module_size x rows ring elements (coefficient form). */
int salsaa_commit(salsaa_ctx* ctx, const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t* d_out,
                  void* stream);

/* Several parallel_dot_series_matrix calls (src/arithmetic.rs:459-505) with
 * the commitment-key rows of ctx, for `ninst` <= 8 witnesses of uneven shapes,
 * in one launch of each step (one transform to slot form for all witnesses,
 * ONE tensor-core launch over all witnesses' element blocks, one
 * finalisation, one inverse transform): witness i is rows[i] (<= 9) x
 * widths[i] (a power of two, 128 .. WIT_LEN) x d coefficients at d_w[i], its
 * commitment (module_size x rows[i] ring elements, coefficient form) goes to
 * d_out[i]; 16-byte aligned buffers; q < 2^56 and module_size <= 18 (the
 * tensor-core path).  Outputs equal salsaa_commit on each witness. */
int salsaa_commit_multi(salsaa_ctx* ctx, const uint64_t* const* d_w, const uint64_t* rows, const uint64_t* widths,
                        uint32_t ninst, uint64_t* const* d_out, void* stream);

/* norm_check_1 + sum_check (src/subroutines/fast_norm_check.rs:135-199,282-320)
 * of each row of d_w (rows x n coefficients, n a power of two >= 4) with the
 * challenges of (seed, round, rep 0 and 1).  d_claims: rows words;
 * d_polys: 2 x log2(n) x rows x 3 words (rep-major). */
int salsaa_sumcheck(const uint64_t* d_w, uint64_t rows, uint64_t n, uint64_t d, uint64_t q, uint64_t seed,
                    uint64_t round, uint64_t* d_claims, uint64_t* d_polys, void* stream);

/* decompose_matrix_by_chunks (src/arithmetic.rs:1572-1593): d_w rows x width
 * x d coefficients -> d_out (rows*parts) x width x d; *d_radix = radix. */
int salsaa_decompose(const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q, uint64_t parts,
                     uint64_t* d_out, uint64_t* d_radix, void* stream);

/* project (src/subroutines/project.rs:50-103) with the challenge of
 * (seed, round): d_w rows x width x d -> d_out width x d. */
int salsaa_project(const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q, uint64_t seed,
                   uint64_t round, uint64_t* d_out, void* stream);

/* No counterpart in the reference: salsaa_project() for callers that must not
 * allocate device memory on the call path, such as a serving loop that has
 * already divided HBM among in-flight proofs, or a host runtime that owns all
 * device allocations.  All scratch lives in a fixed 641 KiB array inside this
 * library (one per GPU, kept until the process exits), so at most 8 rows
 * (chunk width rows*256 <= 2048); larger inputs return -3 with a message.
 * The first call on a device (and the first after a device reset, or from
 * another context of that device) looks up that array's address and should
 * come before any stream capture on that device.  Calls share the array: two calls
 * whose work overlaps on the GPU race; serialise them on one stream. */
int salsaa_project_noalloc(const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q,
                           uint64_t seed, uint64_t round, uint64_t* d_out, void* stream);

/* fold (src/subroutines/fold.rs:22-27): d_w rows x width x d coefficients,
 * d_c rows ring challenges (coefficients) -> d_out width x d coefficients. */
int salsaa_fold(const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q,
                const uint64_t* d_c, uint64_t* d_out, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
