/*
 * salsaa_oracle.c — CPU restatement of the SALSAA prover hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, and the timed CPU baseline).  The
 * product library never links or calls this file.  Every function follows a
 * reference location, cited in its comment (paths are relative to the
 * lattice-arguments/salsaa project root).
 *
 * Arithmetic is exact modulo q.  Ring products and sums are therefore
 * independent of evaluation order, so the reference's lazily accumulated
 * sums, per-step reductions and parallel reduction trees all give the values
 * computed here.  The only deliberate departures from the reference:
 *   - randomness: the reference draws every CRS element, witness coefficient
 *     and challenge from the OS-seeded `rand::rng()`; here each comes from a
 *     counter-based PRF so_prf(seed, domain, index) (SplitMix64 finaliser,
 *     Steele/Lea/Flood 2014) mapped to [0,q) by the multiply-high method;
 *   - values sent to the verifier are canonical mod q (the reference's
 *     round-polynomial sums are chunk sums left unreduced,
 *     src/subroutines/fast_norm_check.rs:120-126).
 */
#include "salsaa_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t u64;
typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------ */
/* Modular arithmetic.  Barrett reduction, HAC algorithm 14.42 with base 2:  */
/* q < 2^s, mu = floor(2^(2s) / q); valid for x < 2^(2s) and q < 2^62.        */
/* ------------------------------------------------------------------------ */
typedef struct {
  u64 q, mu;
  unsigned s;
} Mod;

static Mod mod_make(u64 q) {
  Mod M;
  M.q = q;
  M.s = 64u - (unsigned)__builtin_clzll(q);
  M.mu = (u64)(((u128)1 << (2 * M.s)) / q);
  return M;
}

static inline u64 mod_red(const Mod* M, u128 x) {
  u128 q1 = x >> (M->s - 1);
  u128 q3 = (q1 * M->mu) >> (M->s + 1);
  u64 r = (u64)x - (u64)q3 * M->q;
  while (r >= M->q) r -= M->q;
  return r;
}
static inline u64 mod_red_any(const Mod* M, u128 x) { return (u64)(x % M->q); }
static inline u64 mod_mul(const Mod* M, u64 a, u64 b) { return mod_red(M, (u128)a * b); }
static inline u64 mod_add(u64 a, u64 b, u64 q) {
  u64 r = a + b;
  return r >= q ? r - q : r;
}
static inline u64 mod_sub(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + (q - b); }
/* Shoup's multiplication by a fixed w < q (V. Shoup, NTL): wp = floor(w 2^64 / q),
 * x w - floor(x wp / 2^64) q lies in [0, 2q) for any x < 2^64 and q < 2^63. */
static inline u64 shoup_pre(u64 w, u64 q) { return (u64)(((u128)w << 64) / q); }
static inline u64 mul_shoup(u64 x, u64 w, u64 wp, u64 q) {
  const u64 hi = (u64)(((u128)x * wp) >> 64);
  const u64 r = x * w - hi * q;
  return r >= q ? r - q : r;
}

/* hexl_wrapper.cpp:34-36 (MultiplyMod) */
u64 so_mul_mod(u64 a, u64 b, u64 q) { return (u64)(((u128)a * b) % q); }
/* hexl_wrapper.cpp:38-41 (AddUIntMod) */
u64 so_add_mod(u64 a, u64 b, u64 q) { return (u64)(((u128)(a % q) + (b % q)) % q); }
/* hexl_wrapper.cpp:43-45 (SubUIntMod) */
u64 so_sub_mod(u64 a, u64 b, u64 q) {
  a %= q;
  b %= q;
  return a >= b ? a - b : a + (q - b);
}
/* hexl_wrapper.cpp:61-63 (PowMod) */
u64 so_pow_mod(u64 a, u64 e, u64 q) {
  u64 r = 1 % q, b = a % q;
  while (e) {
    if (e & 1) r = (u64)(((u128)r * b) % q);
    b = (u64)(((u128)b * b) % q);
    e >>= 1;
  }
  return r;
}
/* hexl_wrapper.cpp:52-54 (InverseMod): extended Euclid; 0 when no inverse. */
u64 so_inv_mod(u64 a, u64 q) {
  __int128 t = 0, nt = 1, r = q, nr = a % q;
  while (nr != 0) {
    __int128 qt = r / nr, tmp;
    tmp = t - qt * nt; t = nt; nt = tmp;
    tmp = r - qt * nr; r = nr; nr = tmp;
  }
  if (r != 1) return 0;
  if (t < 0) t += q;
  return (u64)t;
}

/* Minimal primitive `order`-th root of unity mod q (order a power of two),
 * the root HEXL's NTT(n, q) uses with order = 2n: the smallest of the odd
 * powers of any primitive root of that order. */
u64 so_minimal_root(u64 order, u64 q) {
  if (order < 2 || (order & (order - 1)) || (q - 1) % order) return 0;
  u64 g = 0;
  for (u64 x = 2; x < q && x < 100000; x++) {
    u64 c = so_pow_mod(x, (q - 1) / order, q);
    if (so_pow_mod(c, order / 2, q) == q - 1) {
      g = c;
      break;
    }
  }
  if (!g) return 0;
  u64 g2 = so_mul_mod(g, g, q), cur = g, best = g;
  for (u64 i = 0; i < order / 2; i++) {
    if (cur < best) best = cur;
    cur = so_mul_mod(cur, g2, q);
  }
  return best;
}

/* ------------------------------------------------------------------------ */
/* Deterministic challenge stream.                                           */
/* ------------------------------------------------------------------------ */
static inline u64 mix64(u64 z) {
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return z;
}
#define PRF_GOLDEN 0x9e3779b97f4a7c15ULL
static inline u64 prf_key(u64 seed, u64 domain) { return mix64(seed ^ mix64(domain + PRF_GOLDEN)); }
static inline u64 prf_at(u64 key, u64 index) { return mix64(key + index * PRF_GOLDEN); }
u64 so_prf(u64 seed, u64 domain, u64 index) { return prf_at(prf_key(seed, domain), index); }
static inline u64 uni_mod(u64 r, u64 q) { return (u64)(((u128)r * q) >> 64); }

enum { DOM_CRS = 1, DOM_WIT = 2, DOM_NC = 3, DOM_PROJ = 4, DOM_FOLD = 5 };
#define DOMAIN(kind, a, b) ((((u64)(kind)) << 56) | (((u64)(a)) << 24) | ((u64)(b)))

/* ------------------------------------------------------------------------ */
/* NTT tables (HEXL conventions).  fwd[bitrev(i)] = psi^i, inv[bitrev(i)] =   */
/* psi^-i, psi the minimal primitive 2n-th root.  Tables are built once per  */
/* (n, q) under a mutex and never freed (the HEXL wrapper's NTTCache,        */
/* hexl_wrapper.cpp:11-32, without its data race).                           */
/* ------------------------------------------------------------------------ */
typedef struct NttTab {
  u64 n, q, psi, n_inv;
  unsigned logn;
  Mod M;
  u64* fwd;
  u64* inv;
  u64* fwd_p; /* Shoup constants of fwd / inv / n_inv */
  u64* inv_p;
  u64 n_inv_p;
  struct NttTab* next;
} NttTab;

static pthread_mutex_t g_tab_mu = PTHREAD_MUTEX_INITIALIZER;
static NttTab* g_tabs = NULL;

static inline u64 bitrev(u64 x, unsigned bits) {
  u64 r = 0;
  for (unsigned i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

static const NttTab* ntt_tab(u64 n, u64 q) {
  if (n < 1 || (n & (n - 1)) || q < 2 || q >= (1ULL << 62)) return NULL;
  pthread_mutex_lock(&g_tab_mu);
  for (NttTab* t = g_tabs; t; t = t->next)
    if (t->n == n && t->q == q) {
      pthread_mutex_unlock(&g_tab_mu);
      return t;
    }
  NttTab* T = NULL;
  u64 psi = so_minimal_root(2 * n, q);
  if (psi) {
    T = (NttTab*)calloc(1, sizeof(NttTab));
    T->n = n;
    T->q = q;
    T->psi = psi;
    T->M = mod_make(q);
    T->logn = (unsigned)__builtin_ctzll(n);
    T->n_inv = so_inv_mod(n % q, q);
    T->fwd = (u64*)malloc(n * sizeof(u64));
    T->inv = (u64*)malloc(n * sizeof(u64));
    T->fwd_p = (u64*)malloc(n * sizeof(u64));
    T->inv_p = (u64*)malloc(n * sizeof(u64));
    T->n_inv_p = shoup_pre(T->n_inv, q);
    u64 psi_inv = so_inv_mod(psi, q), p = 1, pi = 1;
    for (u64 i = 0; i < n; i++) {
      u64 j = bitrev(i, T->logn);
      T->fwd[j] = p;
      T->inv[j] = pi;
      p = so_mul_mod(p, psi, q);
      pi = so_mul_mod(pi, psi_inv, q);
    }
    for (u64 i = 0; i < n; i++) {
      T->fwd_p[i] = shoup_pre(T->fwd[i], q);
      T->inv_p[i] = shoup_pre(T->inv[i], q);
    }
    T->next = g_tabs;
    g_tabs = T;
  }
  pthread_mutex_unlock(&g_tab_mu);
  return T;
}

/* Cooley-Tukey negacyclic forward NTT, bit-reversed output:
 * a[i] <- A(psi^(2*bitrev(i)+1)).  hexl_wrapper.cpp:213-220. */
static void ntt_fwd(const NttTab* T, u64* a) {
  const u64 n = T->n, q = T->q;
  u64 t = n;
  for (u64 m = 1; m < n; m <<= 1) {
    t >>= 1;
    for (u64 i = 0; i < m; i++) {
      const u64 j1 = 2 * i * t, W = T->fwd[m + i], Wp = T->fwd_p[m + i];
      for (u64 j = j1; j < j1 + t; j++) {
        u64 U = a[j], V = mul_shoup(a[j + t], W, Wp, q);
        a[j] = mod_add(U, V, q);
        a[j + t] = mod_sub(U, V, q);
      }
    }
  }
}

/* Gentleman-Sande inverse of ntt_fwd, natural-order output scaled by 1/n.
 * hexl_wrapper.cpp:222-229. */
static void ntt_inv(const NttTab* T, u64* a) {
  const u64 n = T->n, q = T->q;
  u64 t = 1;
  for (u64 m = n; m > 1; m >>= 1) {
    u64 j1 = 0;
    const u64 h = m >> 1;
    for (u64 i = 0; i < h; i++) {
      const u64 W = T->inv[h + i], Wp = T->inv_p[h + i];
      for (u64 j = j1; j < j1 + t; j++) {
        u64 U = a[j], V = a[j + t];
        a[j] = mod_add(U, V, q);
        a[j + t] = mul_shoup(mod_sub(U, V, q), W, Wp, q);
      }
      j1 += 2 * t;
    }
    t <<= 1;
  }
  for (u64 j = 0; j < n; j++) a[j] = mul_shoup(a[j], T->n_inv, T->n_inv_p, q);
}

int so_ntt_forward(u64* a, u64 n, u64 q) {
  const NttTab* T = ntt_tab(n, q);
  if (!T) return -1;
  ntt_fwd(T, a);
  return 0;
}
int so_ntt_inverse(u64* a, u64 n, u64 q) {
  const NttTab* T = ntt_tab(n, q);
  if (!T) return -1;
  ntt_inv(T, a);
  return 0;
}
int so_get_roots(u64 n, u64 q, u64* out) {
  const NttTab* T = ntt_tab(n, q);
  if (!T) return -1;
  memcpy(out, T->fwd, n * sizeof(u64));
  return 0;
}
int so_get_inv_roots(u64 n, u64 q, u64* out) {
  const NttTab* T = ntt_tab(n, q);
  if (!T) return -1;
  memcpy(out, T->inv, n * sizeof(u64));
  return 0;
}

/* hexl_wrapper.cpp:73-94: forward both, pointwise product, inverse. */
int so_multiply_poly(u64* r, const u64* a, const u64* b, u64 n, u64 q) {
  const NttTab* T = ntt_tab(n, q);
  if (!T) return -1;
  u64* x = (u64*)malloc(n * sizeof(u64));
  u64* y = (u64*)malloc(n * sizeof(u64));
  for (u64 i = 0; i < n; i++) {
    x[i] = a[i] % q;
    y[i] = b[i] % q;
  }
  ntt_fwd(T, x);
  ntt_fwd(T, y);
  for (u64 i = 0; i < n; i++) x[i] = mod_mul(&T->M, x[i], y[i]);
  ntt_inv(T, x);
  memcpy(r, x, n * sizeof(u64));
  free(x);
  free(y);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Element-wise operations (hexl_wrapper.cpp:65-70,119-126,188-207,231-268). */
/* ------------------------------------------------------------------------ */
void so_eltwise_mult_mod(u64* r, const u64* a, const u64* b, u64 n, u64 q) {
  for (u64 i = 0; i < n; i++) r[i] = so_mul_mod(a[i], b[i], q);
}
void so_eltwise_add_mod(u64* r, const u64* a, const u64* b, u64 n, u64 q) {
  for (u64 i = 0; i < n; i++) r[i] = so_add_mod(a[i], b[i], q);
}
void so_eltwise_sub_mod(u64* r, const u64* a, const u64* b, u64 n, u64 q) {
  for (u64 i = 0; i < n; i++) r[i] = so_sub_mod(a[i], b[i], q);
}
void so_eltwise_fma_mod(u64* r, const u64* a, u64 s, const u64* b, u64 n, u64 q) {
  for (u64 i = 0; i < n; i++) r[i] = so_add_mod(so_mul_mod(a[i], s, q), b[i], q);
}
void so_eltwise_reduce_mod(u64* r, const u64* a, u64 n, u64 q) {
  for (u64 i = 0; i < n; i++) r[i] = a[i] % q;
}
u64 so_sum(const u64* a, u64 n, u64 q) {
  u128 s = 0;
  for (u64 i = 0; i < n; i++) s += a[i] % q;
  return (u64)(s % q);
}
u64 so_sum_sq(const u64* a, u64 n, u64 q) {
  /* squares of reduced values are below 2^124; 2^3 of them fit a 128-bit sum */
  const u64 blk = 8;
  u64 s = 0;
#pragma omp parallel
  {
    u64 part = 0;
#pragma omp for schedule(static)
    for (long long b = 0; b < (long long)((n + blk - 1) / blk); b++) {
      const u64 i0 = (u64)b * blk, i1 = i0 + blk < n ? i0 + blk : n;
      u128 acc = 0;
      for (u64 i = i0; i < i1; i++) {
        const u64 x = a[i] % q;
        acc += (u128)x * x;
      }
      part = so_add_mod(part, (u64)(acc % q), q);
    }
#pragma omp critical
    s = so_add_mod(s, part, q);
  }
  return s;
}

/* tensor() of src/subroutines/fast_norm_check.rs:25-39: first c is the most
 * significant index bit; factors (1-c, c). */
void so_tensor(u64* out, const u64* cs, u64 k, u64 q) {
  out[0] = 1 % q;
  u64 len = 1;
  for (u64 j = 0; j < k; j++) {
    u64 c = cs[j] % q, omc = mod_sub(1 % q, c, q);
    for (u64 i = len; i-- > 0;) {
      u64 v = out[i];
      out[2 * i] = so_mul_mod(v, omc, q);
      out[2 * i + 1] = so_mul_mod(v, c, q);
    }
    len *= 2;
  }
}

/* ------------------------------------------------------------------------ */
/* Ring R_q = Z_q[X]/(X^d+1) in the incomplete-NTT ("slot") representation:   */
/* data[0..n) = NTT_n(even coefficients), data[n..2n) = NTT_n(odd), n = d/2.   */
/* src/cyclotomic_ring.rs:484-556.                                           */
/* ------------------------------------------------------------------------ */
typedef struct {
  u64 d, n, q;
  Mod M;
  const NttTab* T;
  u64* zeta; /* shift factors: NTT_n(Y), src/cyclotomic_ring.rs:559-564 */
} Ring;

static int ring_init(Ring* R, u64 d, u64 q) {
  memset(R, 0, sizeof(*R));
  /* ring buffers below are sized for d <= 2048 (the reference's sets use d <= 512) */
  if (d < 4 || d > 2048 || (d & (d - 1))) return -1;
  R->d = d;
  R->n = d / 2;
  R->q = q;
  R->M = mod_make(q);
  R->T = ntt_tab(R->n, q);
  if (!R->T) return -1;
  R->zeta = (u64*)calloc(R->n, sizeof(u64));
  R->zeta[1] = 1;
  ntt_fwd(R->T, R->zeta);
  return 0;
}
static void ring_free(Ring* R) { free(R->zeta); }

static void to_slot(const Ring* R, const u64* coef, u64* out) {
  u64 tmp[2048];
  const u64 n = R->n;
  for (u64 i = 0; i < n; i++) {
    tmp[i] = coef[2 * i];
    tmp[n + i] = coef[2 * i + 1];
  }
  ntt_fwd(R->T, tmp);
  ntt_fwd(R->T, tmp + n);
  memcpy(out, tmp, 2 * n * sizeof(u64));
}
static void from_slot(const Ring* R, const u64* slot, u64* out) {
  u64 tmp[2048];
  const u64 n = R->n;
  memcpy(tmp, slot, 2 * n * sizeof(u64));
  ntt_inv(R->T, tmp);
  ntt_inv(R->T, tmp + n);
  for (u64 i = 0; i < n; i++) {
    out[2 * i] = tmp[i];
    out[2 * i + 1] = tmp[n + i];
  }
}
/* incomplete_ntt_multiplication with use_shift_factors = true,
 * src/cyclotomic_ring.rs:700-791:
 * (a_e + X a_o)(b_e + X b_o) = a_e b_e + zeta a_o b_o + X (a_o b_e + a_e b_o). */
static void slot_mul(const Ring* R, const u64* a, const u64* b, u64* r) {
  const u64 n = R->n, q = R->q;
  for (u64 s = 0; s < n; s++) {
    u64 ee = mod_mul(&R->M, a[s], b[s]);
    u64 oo = mod_mul(&R->M, mod_mul(&R->M, a[n + s], b[n + s]), R->zeta[s]);
    u64 x = mod_add(mod_mul(&R->M, a[n + s], b[s]), mod_mul(&R->M, a[s], b[n + s]), q);
    r[s] = mod_add(ee, oo, q);
    r[n + s] = x;
  }
}
/* conjugate(), src/cyclotomic_ring.rs:455-469 (coefficient form). */
void so_conjugate(u64* r, const u64* a, u64 d, u64 q) {
  u64 tmp[4096];
  tmp[0] = a[0];
  for (u64 i = 1; i < d; i++) tmp[i] = a[d - i] == 0 ? 0 : q - a[d - i];
  memcpy(r, tmp, d * sizeof(u64));
}

int so_ring_to_slot(u64* out, const u64* coef, u64 d, u64 q) {
  Ring R;
  if (ring_init(&R, d, q)) return -1;
  to_slot(&R, coef, out);
  ring_free(&R);
  return 0;
}
int so_ring_from_slot(u64* out, const u64* slot, u64 d, u64 q) {
  Ring R;
  if (ring_init(&R, d, q)) return -1;
  from_slot(&R, slot, out);
  ring_free(&R);
  return 0;
}
int so_ring_mul(u64* r, const u64* a, const u64* b, u64 d, u64 q) {
  Ring R;
  if (ring_init(&R, d, q)) return -1;
  u64 x[4096], y[4096];
  to_slot(&R, a, x);
  to_slot(&R, b, y);
  slot_mul(&R, x, y, x);
  from_slot(&R, x, r);
  ring_free(&R);
  return 0;
}
/* parallel_dot_matrix_matrix (src/arithmetic.rs:429-457) in the Ajtai shape:
 * C[j][c] = sum_i A[j][i] * W[c][i] in R_q; A is n x m, W is r x m, C is
 * n x r ring elements (coefficient form).  Products in slot form. */
int so_dense_commit(u64* C, const u64* A, const u64* W, u64 n, u64 m, u64 r, u64 d, u64 q) {
  Ring R;
  if (ring_init(&R, d, q)) return -1;
  u64* as = (u64*)malloc(n * m * d * sizeof(u64));
  u64* ws = (u64*)malloc(r * m * d * sizeof(u64));
  if (!as || !ws) {
    free(as);
    free(ws);
    ring_free(&R);
    return -1;
  }
#pragma omp parallel for schedule(static)
  for (long long t = 0; t < (long long)(n * m); t++) to_slot(&R, A + (u64)t * d, as + (u64)t * d);
#pragma omp parallel for schedule(static)
  for (long long t = 0; t < (long long)(r * m); t++) to_slot(&R, W + (u64)t * d, ws + (u64)t * d);
#pragma omp parallel for schedule(dynamic, 1)
  for (long long jc = 0; jc < (long long)(n * r); jc++) {
    const u64 j = (u64)jc / r, c = (u64)jc % r;
    u64 acc[2048], prod[2048];
    memset(acc, 0, d * sizeof(u64));
    for (u64 i = 0; i < m; i++) {
      slot_mul(&R, as + (j * m + i) * d, ws + (c * m + i) * d, prod);
      for (u64 x = 0; x < d; x++) acc[x] = mod_add(acc[x], prod[x], q);
    }
    from_slot(&R, acc, C + (u64)jc * d);
  }
  free(as);
  free(ws);
  ring_free(&R);
  return 0;
}

int so_shift_factors(u64* out, u64 d, u64 q) {
  Ring R;
  if (ring_init(&R, d, q)) return -1;
  memcpy(out, R.zeta, R.n * sizeof(u64));
  ring_free(&R);
  return 0;
}

static void slot_const(const Ring* R, u64 v, u64* out) {
  for (u64 s = 0; s < R->n; s++) {
    out[s] = v % R->q;
    out[R->n + s] = 0;
  }
}

/* ------------------------------------------------------------------------ */
/* Statement rows: PowerSeries (src/arithmetic.rs:147-176) kept as the tensor */
/* factors plus the base layer.  Expanded layer k has length blen*2^(K-k) and */
/* equals kron(tens[k], ..., tens[K-1], base) (complete_power_series).        */
/* ------------------------------------------------------------------------ */
typedef struct {
  u64 K;
  u64* tens; /* K x 2 x d, slot form; tens[0] is the outermost factor */
  u64 blen;
  u64* base; /* blen x d, slot form */
} Row;

typedef struct {
  Row* r;
  u64 n, cap;
} Stmt;

static void stmt_push(Stmt* S, Row row) {
  if (S->n == S->cap) {
    S->cap = S->cap ? 2 * S->cap : 16;
    S->r = (Row*)realloc(S->r, S->cap * sizeof(Row));
  }
  S->r[S->n++] = row;
}
static void stmt_free(Stmt* S) {
  for (u64 i = 0; i < S->n; i++) {
    free(S->r[i].tens);
    free(S->r[i].base);
  }
  free(S->r);
  memset(S, 0, sizeof(*S));
}

/* A fixed ring element t (slot form) prepared for repeated products t * x:
 * per slot its even part, odd part and zeta * odd part with their Shoup
 * constants.  (t_e + X t_o)(x_e + X x_o) = t_e x_e + zeta t_o x_o + X (t_o x_e + t_e x_o),
 * the product of slot_mul. */
typedef struct {
  u64 e[1024], o[1024], z[1024], ep[1024], op[1024], zp[1024];
} SlotConst;
static void slot_const_make(const Ring* R, const u64* t, SlotConst* c) {
  const u64 n = R->n, q = R->q;
  for (u64 s = 0; s < n; s++) {
    c->e[s] = t[s];
    c->o[s] = t[n + s];
    c->z[s] = mod_mul(&R->M, t[n + s], R->zeta[s]);
    c->ep[s] = shoup_pre(c->e[s], q);
    c->op[s] = shoup_pre(c->o[s], q);
    c->zp[s] = shoup_pre(c->z[s], q);
  }
}
static void slot_mul_const(const Ring* R, const SlotConst* c, const u64* x, u64* r) {
  const u64 n = R->n, q = R->q;
  for (u64 s = 0; s < n; s++) {
    const u64 xe = x[s], xo = x[n + s];
    const u64 ev = mod_add(mul_shoup(xe, c->e[s], c->ep[s], q), mul_shoup(xo, c->z[s], c->zp[s], q), q);
    const u64 od = mod_add(mul_shoup(xe, c->o[s], c->op[s], q), mul_shoup(xo, c->e[s], c->ep[s], q), q);
    r[s] = ev;
    r[n + s] = od;
  }
}

/* The expanded layer whose length is len; -1 when the row has none (the
 * reference panics "No matching layer found", src/arithmetic.rs:474). */
static int row_layer_index(const Row* row, u64 len, u64* jj) {
  if (len % row->blen) return -1;
  u64 f = len / row->blen;
  if (f & (f - 1)) return -1;
  u64 j = (u64)__builtin_ctzll(f);
  if (j > row->K) return -1;
  *jj = j;
  return 0;
}

static int row_layer(const Ring* R, const Row* row, u64 len, u64* out) {
  u64 j;
  if (row_layer_index(row, len, &j)) return -1;
  const u64 d = R->d;
  memcpy(out, row->base, row->blen * d * sizeof(u64));
  u64 cur = row->blen;
  SlotConst c0, c1;
  for (u64 step = 0; step < j; step++) {
    const u64 k = row->K - 1 - step;
    slot_const_make(R, row->tens + (2 * k) * d, &c0);
    slot_const_make(R, row->tens + (2 * k + 1) * d, &c1);
#pragma omp parallel for schedule(static)
    for (long long idx = 0; idx < (long long)cur; idx++) {
      slot_mul_const(R, &c1, out + idx * d, out + (cur + idx) * d);
      slot_mul_const(R, &c0, out + idx * d, out + idx * d);
    }
    cur *= 2;
  }
  return 0;
}

/* out[k] = sum_i E[i] * W_k[i] over slot-form vectors of length len
 * (parallel_dot_series_matrix / parallel_dot_single_series_matrix,
 * src/arithmetic.rs:459-536).  Lazy 128-bit sums, reduced per chunk; each
 * chunk of E is read once for all witness rows, element by element, so the
 * scan is sequential and the chunk stays in cache across the rows. */
static void dot_layer(const Ring* R, const u64* E, const u64* Ws, u64 rows, u64 len, u64* out) {
  const u64 n = R->n, d = R->d, q = R->q;
  const u64 CH = (q < (1ULL << 52)) ? 512 : 4;
  const u64 nch = (len + CH - 1) / CH;
  u64* part = (u64*)calloc(nch * rows * 3 * n, sizeof(u64));
#pragma omp parallel
  {
    u128* acc = (u128*)malloc(3 * n * sizeof(u128));
#pragma omp for schedule(dynamic, 4)
    for (long long c = 0; c < (long long)nch; c++) {
      const u64 i0 = (u64)c * CH, i1 = i0 + CH < len ? i0 + CH : len;
      for (u64 k = 0; k < rows; k++) {
        const u64* W = Ws + k * len * d;
        memset(acc, 0, 3 * n * sizeof(u128));
        for (u64 i = i0; i < i1; i++) {
          const u64* e = E + i * d;
          const u64* w = W + i * d;
          for (u64 s = 0; s < n; s++) {
            const u64 es = e[s], eo = e[n + s], ws = w[s], wo = w[n + s];
            acc[s] += (u128)es * ws;
            acc[n + s] += (u128)eo * wo;
            acc[2 * n + s] += (u128)eo * ws + (u128)es * wo;
          }
        }
        u64* pc = part + ((u64)c * rows + k) * 3 * n;
        for (u64 t = 0; t < 3 * n; t++) pc[t] = mod_red_any(&R->M, acc[t]);
      }
    }
    free(acc);
  }
  for (u64 k = 0; k < rows; k++) {
    for (u64 s = 0; s < n; s++) {
      u64 ee = 0, oo = 0, x = 0;
      for (u64 c = 0; c < nch; c++) {
        const u64* pc = part + (c * rows + k) * 3 * n;
        ee = mod_add(ee, pc[s], q);
        oo = mod_add(oo, pc[n + s], q);
        x = mod_add(x, pc[2 * n + s], q);
      }
      out[k * d + s] = mod_add(ee, mod_mul(&R->M, oo, R->zeta[s]), q);
      out[k * d + n + s] = x;
    }
  }
  free(part);
}

/* Commitment-key row: the power row (m, m^2, ..., m^L) of
 * compute_commitment_keys (src/subroutines/crs.rs:43-72) in tensor form:
 * tens[k] = (1, m^(L/2^(k+1))), base = (m, ..., m^(L/2^K)). */
static Row make_ck_row(const Ring* R, const u64* m_coef, u64 L) {
  const u64 d = R->d;
  Row row;
  u64 K = 0, cur = L;
  while (cur % 2 == 0) {
    cur /= 2;
    K++;
  }
  row.K = K;
  row.blen = cur;
  row.tens = (u64*)malloc((K ? K : 1) * 2 * d * sizeof(u64));
  row.base = (u64*)malloc(cur * d * sizeof(u64));
  u64 ms[4096], pw[4096];
  to_slot(R, m_coef, ms);
  memcpy(pw, ms, d * sizeof(u64));
  memcpy(row.base, ms, d * sizeof(u64));
  for (u64 i = 1; i < cur; i++) {
    slot_mul(R, pw, ms, pw);
    memcpy(row.base + i * d, pw, d * sizeof(u64));
  }
  /* m^(cur * 2^j) for j = 0..K-1 by squaring the highest base power. */
  u64 p[4096];
  memcpy(p, pw, d * sizeof(u64)); /* m^cur */
  for (u64 j = 0; j < K; j++) {
    u64 k = K - 1 - j; /* tens[k] multiplies by m^(L/2^(k+1)) = m^(cur*2^j) */
    slot_const(R, 1, row.tens + (2 * k) * d);
    memcpy(row.tens + (2 * k + 1) * d, p, d * sizeof(u64));
    slot_mul(R, p, p, p);
  }
  return row;
}

/* Row of scalar tensor factors (const(1-c), const(c)) over a base layer:
 * the shape built by norm_check_3 and batch_projections
 * (src/subroutines/fast_norm_check.rs:401-441, src/subroutines/project.rs:131-203). */
static Row make_scalar_tensor_row(const Ring* R, const u64* t0, const u64* t1, u64 K,
                                  const u64* base_slot, u64 blen) {
  const u64 d = R->d;
  Row row;
  row.K = K;
  row.blen = blen;
  row.tens = (u64*)malloc((K ? K : 1) * 2 * d * sizeof(u64));
  row.base = (u64*)malloc(blen * d * sizeof(u64));
  for (u64 k = 0; k < K; k++) {
    slot_const(R, t0[k], row.tens + (2 * k) * d);
    slot_const(R, t1[k], row.tens + (2 * k + 1) * d);
  }
  memcpy(row.base, base_slot, blen * d * sizeof(u64));
  return row;
}

/* ------------------------------------------------------------------------ */
/* Sampling (src/cyclotomic_ring.rs:257-339, src/arithmetic.rs:1160-1175).    */
/* ------------------------------------------------------------------------ */
void so_sample_crs(const so_params* p, u64 crs_seed, u64* m) {
  for (u64 r = 0; r < p->module_size; r++) {
    u64 key = prf_key(crs_seed, DOMAIN(DOM_CRS, 0, r));
    for (u64 i = 0; i < p->d; i++) m[r * p->d + i] = uni_mod(prf_at(key, i), p->q);
  }
}
/* random_bounded(2): magnitude random_range(0..2), negated with probability 1/2. */
static inline u64 ternary_from(u64 r, u64 q) {
  u64 mag = r & 1, neg = (r >> 1) & 1;
  return mag ? (neg ? q - 1 : 1) : 0;
}
void so_sample_witness(const so_params* p, u64 seed, u64* w) {
  const u64 per_row = p->wit_len * p->d;
  for (u64 k = 0; k < p->init_wit_rep; k++) {
    u64 key = prf_key(seed, DOMAIN(DOM_WIT, 0, k));
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)per_row; i++) w[k * per_row + i] = ternary_from(prf_at(key, (u64)i), p->q);
  }
}
/* random_biased(): uniform over {q-1, 0, 1}. */
static inline u64 biased_from(u64 r, u64 q) {
  u64 t = (u64)(((u128)r * 3) >> 64);
  return t == 0 ? q - 1 : (t == 1 ? 0 : 1);
}

/* ------------------------------------------------------------------------ */
/* Subroutines.                                                              */
/* ------------------------------------------------------------------------ */

/* One sum_check (src/subroutines/fast_norm_check.rs:135-199) of one row with
 * the challenge sequence cs; polys[j] = (f0, f1, f2), canonical mod q. */
static void sumcheck_rows(const Mod* M, u64** v, u64 rows, u64 len, const u64* cs, u64* polys) {
  const u64 q = M->q;
  u64 cur = len, j = 0;
  while (cur > 1) {
    const u64 h = cur / 2, c = cs[j], cp = shoup_pre(cs[j], q);
    /* products of reduced values are below 2^(2s); this many fit a 128-bit sum */
    const u64 lazy = M->s <= 52 ? 4096 : 1;
    for (u64 k = 0; k < rows; k++) {
      u64* x = v[k];
      u64 f0 = 0, f1 = 0, f2 = 0;
#pragma omp parallel
      {
        u64 a0 = 0, a1 = 0, a2 = 0;
#pragma omp for schedule(static)
        for (long long b = 0; b < (long long)((h + lazy - 1) / lazy); b++) {
          const u64 i0 = (u64)b * lazy, i1 = i0 + lazy < h ? i0 + lazy : h;
          u128 s0 = 0, s1 = 0, s2 = 0;
          for (u64 i = i0; i < i1; i++) {
            const u64 w0 = x[i], w1 = x[h + i], df = mod_sub(w1, w0, q);
            s0 += (u128)w0 * w0;
            s1 += (u128)w0 * df;
            s2 += (u128)df * df;
            x[i] = mod_add(mul_shoup(df, c, cp, q), w0, q);
          }
          a0 = mod_add(a0, (u64)(s0 % q), q);
          a1 = mod_add(a1, (u64)(s1 % q), q);
          a2 = mod_add(a2, (u64)(s2 % q), q);
        }
#pragma omp critical
        {
          f0 = mod_add(f0, a0, q);
          f1 = mod_add(f1, a1, q);
          f2 = mod_add(f2, a2, q);
        }
      }
      polys[(j * rows + k) * 3 + 0] = f0;
      polys[(j * rows + k) * 3 + 1] = f1;
      polys[(j * rows + k) * 3 + 2] = f2;
    }
    cur = h;
    j++;
  }
}

int so_sumcheck(const u64* w, u64 n, u64 q, const u64* cs, u64* claim, u64* polys, u64* final_v) {
  if (n == 0 || (n & (n - 1))) return -1;
  Mod M = mod_make(q);
  u64* v = (u64*)malloc(n * sizeof(u64));
  memcpy(v, w, n * sizeof(u64));
  *claim = so_sum_sq(w, n, q);
  sumcheck_rows(&M, &v, 1, n, cs, polys);
  if (final_v) *final_v = v[0];
  free(v);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Norm-check sumcheck over F_{q^2} = F_q[X]/(X^2 - s), s the smallest        */
/* quadratic non-residue mod q: the QuadraticExtension of                    */
/* src/quadratic_extension.rs:30-58 ((a + bX)(c + dX) = ac + s bd + (ad + bc)X */
/* ) with a non-residue shift, so the extension is a field.  Same rounds as  */
/* sum_check (src/subroutines/fast_norm_check.rs:135-199) with the           */
/* challenges and the folded vector in F_{q^2}: round polynomial              */
/* (f0, f1, f2) = (sum v0^2, sum v0 (v1 - v0), sum (v1 - v0)^2), fold           */
/* v <- v0 + c (v1 - v0).  The input vector has F_q entries.                 */
/* ------------------------------------------------------------------------ */
u64 so_qnr(u64 q) {
  for (u64 s = 2; s < q; s++)
    if (so_pow_mod(s, (q - 1) / 2, q) == q - 1) return s;
  return 0;
}
static inline void qe_mul(const Mod* M, u64 s, u64 a0, u64 a1, u64 b0, u64 b1, u64* r0, u64* r1) {
  const u64 q = M->q;
  const u64 t0 = mod_add(mod_mul(M, a0, b0), mod_mul(M, s, mod_mul(M, a1, b1)), q);
  const u64 t1 = mod_add(mod_mul(M, a0, b1), mod_mul(M, a1, b0), q);
  *r0 = t0;
  *r1 = t1;
}
int so_sumcheck_fq2(const u64* w, u64 n, u64 q, u64 shift, const u64* cs, u64* claim, u64* polys,
                    u64* final_v) {
  if (n == 0 || (n & (n - 1))) return -1;
  Mod M = mod_make(q);
  u64* v = (u64*)malloc(2 * n * sizeof(u64));
  for (u64 i = 0; i < n; i++) {
    v[2 * i] = w[i] % q;
    v[2 * i + 1] = 0;
  }
  *claim = so_sum_sq(w, n, q);
  u64 cur = n, j = 0;
  while (cur > 1) {
    const u64 h = cur / 2, c0 = cs[2 * j], c1 = cs[2 * j + 1];
    u64 f[6] = {0, 0, 0, 0, 0, 0};
    for (u64 i = 0; i < h; i++) {
      const u64 a0 = v[2 * i], a1 = v[2 * i + 1];
      const u64 e0 = mod_sub(v[2 * (h + i)], a0, q), e1 = mod_sub(v[2 * (h + i) + 1], a1, q);
      u64 r0, r1;
      qe_mul(&M, shift, a0, a1, a0, a1, &r0, &r1);
      f[0] = mod_add(f[0], r0, q);
      f[1] = mod_add(f[1], r1, q);
      qe_mul(&M, shift, a0, a1, e0, e1, &r0, &r1);
      f[2] = mod_add(f[2], r0, q);
      f[3] = mod_add(f[3], r1, q);
      qe_mul(&M, shift, e0, e1, e0, e1, &r0, &r1);
      f[4] = mod_add(f[4], r0, q);
      f[5] = mod_add(f[5], r1, q);
      qe_mul(&M, shift, c0, c1, e0, e1, &r0, &r1);
      v[2 * i] = mod_add(a0, r0, q);
      v[2 * i + 1] = mod_add(a1, r1, q);
    }
    memcpy(polys + 6 * j, f, sizeof(f));
    cur = h;
    j++;
  }
  if (final_v) {
    final_v[0] = v[0];
    final_v[1] = v[1];
  }
  free(v);
  return 0;
}

/* decompose_matrix_by_chunks (src/arithmetic.rs:1461-1593): centre-lift into
 * positive/negative parts, global bit width, radix 2^ceil(bw/parts), digits
 * pos_k - neg_k; new row index = row*parts + k. */
static void decompose_impl(const u64* w, u64 rows, u64 width, u64 d, u64 q, u64 parts, u64* out,
                           u64* radix_out) {
  const u64 tot = rows * width * d;
  u64 acc = 0;
#pragma omp parallel for reduction(| : acc) schedule(static)
  for (long long i = 0; i < (long long)tot; i++) {
    u64 v = w[i];
    acc |= (v * 2 > q) ? q - v : v;
  }
  u64 bw = acc ? 64 - (u64)__builtin_clzll(acc) : 0;
  u64 rlog = (bw + parts - 1) / parts;
  u64 radix = 1ULL << rlog, mask = radix - 1;
  *radix_out = radix;
  for (u64 r = 0; r < rows; r++)
    for (u64 c = 0; c < parts; c++) {
      u64* o = out + (r * parts + c) * width * d;
      const u64* x = w + r * width * d;
#pragma omp parallel for schedule(static)
      for (long long i = 0; i < (long long)(width * d); i++) {
        u64 v = x[i], pos = 0, neg = 0;
        if (v * 2 > q) neg = q - v;
        else pos = v;
        for (u64 s = 0; s < c; s++) {
          pos >>= rlog;
          neg >>= rlog;
        }
        o[i] = mod_sub(pos & mask, neg & mask, q);
      }
    }
}
int so_decompose(const u64* w, u64 rows, u64 width, u64 d, u64 q, u64 parts, u64* out, u64* radix) {
  if (parts < 1) return -1;
  decompose_impl(w, rows, width, d, q, parts, out, radix);
  return 0;
}

/* project (src/subroutines/project.rs:50-103): for chunk (i, j) of width
 * cw = rows*256 and output k, sum of the +-1-selected ring elements. */
#define PROJ_H 256
static int project_impl(const u64* w, u64 rows, u64 width, u64 d, u64 q, const uint8_t* iz,
                        const uint8_t* sg, u64* out) {
  const u64 cw = rows * PROJ_H;
  if (cw > width) return -1;
  const u64 nch = width / cw;
  const long long total = (long long)(rows * nch * PROJ_H);
#pragma omp parallel for schedule(dynamic, 16)
  for (long long o = 0; o < total; o++) {
    u64 idx = (u64)o / PROJ_H, k = (u64)o % PROJ_H;
    u64 i = idx / nch, j = idx % nch;
    const u64* chunk = w + (i * width + j * cw) * d;
    u64* dst = out + (idx * PROJ_H + k) * d;
    if (q < (1ULL << 52) && cw <= (1ULL << 11)) {
      /* canonical inputs below 2^52, at most 2^11 of them: the sums stay below 2^63 */
      u64 pos[2048], neg[2048];
      memset(pos, 0, d * sizeof(u64));
      memset(neg, 0, d * sizeof(u64));
      for (u64 l = 0; l < cw; l++) {
        if (iz[k * cw + l]) continue;
        const u64* e = chunk + l * d;
        u64* acc = sg[k * cw + l] ? pos : neg;
        for (u64 t = 0; t < d; t++) acc[t] += e[t];
      }
      for (u64 t = 0; t < d; t++) dst[t] = mod_sub(pos[t] % q, neg[t] % q, q);
      continue;
    }
    u128 pos[4096], neg[4096];
    memset(pos, 0, d * sizeof(u128));
    memset(neg, 0, d * sizeof(u128));
    for (u64 l = 0; l < cw; l++) {
      if (iz[k * cw + l]) continue;
      const u64* e = chunk + l * d;
      if (sg[k * cw + l])
        for (u64 t = 0; t < d; t++) pos[t] += e[t];
      else
        for (u64 t = 0; t < d; t++) neg[t] += e[t];
    }
    for (u64 t = 0; t < d; t++) dst[t] = mod_sub((u64)(pos[t] % q), (u64)(neg[t] % q), q);
  }
  return 0;
}
int so_project(const u64* w, u64 rows, u64 width, u64 d, u64 q, const uint8_t* iz, const uint8_t* sg,
               u64* out) {
  return project_impl(w, rows, width, d, q, iz, sg, out);
}

/* Witness to slot form (per ring element). */
static void witness_to_slot(const Ring* R, const u64* coef, u64* slot, u64 count) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)count; i++) to_slot(R, coef + (u64)i * R->d, slot + (u64)i * R->d);
}
static void witness_from_slot(const Ring* R, const u64* slot, u64* coef, u64 count) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)count; i++) from_slot(R, slot + (u64)i * R->d, coef + (u64)i * R->d);
}

/* fold (src/subroutines/fold.rs:22-27 via parallel_dot_matrix_matrix,
 * src/arithmetic.rs:429-457): out[i] = sum_k W_k[i] * c_k (slot form). */
static void fold_slot(const Ring* R, const u64* Ws, u64 rows, u64 width, const u64* cslot, u64* out) {
  const u64 d = R->d;
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)width; i++) {
    u64 acc[4096], t[4096];
    memset(acc, 0, d * sizeof(u64));
    for (u64 k = 0; k < rows; k++) {
      slot_mul(R, Ws + (k * width + (u64)i) * d, cslot + k * d, t);
      for (u64 s = 0; s < d; s++) acc[s] = mod_add(acc[s], t[s], R->q);
    }
    memcpy(out + (u64)i * d, acc, d * sizeof(u64));
  }
}
int so_fold(const u64* w, u64 rows, u64 width, u64 d, u64 q, const u64* c, u64* out) {
  Ring R;
  if (ring_init(&R, d, q)) return -1;
  u64* ws = (u64*)malloc(rows * width * d * sizeof(u64));
  u64* cs = (u64*)malloc(rows * d * sizeof(u64));
  u64* fs = (u64*)malloc(width * d * sizeof(u64));
  witness_to_slot(&R, w, ws, rows * width);
  witness_to_slot(&R, c, cs, rows);
  fold_slot(&R, ws, rows, width, cs, fs);
  witness_from_slot(&R, fs, out, width);
  free(ws);
  free(cs);
  free(fs);
  ring_free(&R);
  return 0;
}

/* <every statement row, every witness row>: S.n x rows ring elements (slot). */
static int commit_all(const Ring* R, const Stmt* S, const u64* Ws, u64 rows, u64 width, u64* out) {
  u64* E = (u64*)malloc(width * R->d * sizeof(u64));
  int rc = 0;
  for (u64 j = 0; j < S->n && !rc; j++) {
    rc = row_layer(R, &S->r[j], width, E);
    if (!rc) dot_layer(R, E, Ws, rows, width, out + j * rows * R->d);
  }
  free(E);
  return rc;
}

int so_commit_ck(const so_params* p, u64 crs_seed, const u64* w, u64 rows, u64 width, u64* out) {
  Ring R;
  if (ring_init(&R, p->d, p->q)) return -1;
  const u64 d = p->d;
  u64* m = (u64*)malloc(p->module_size * d * sizeof(u64));
  so_sample_crs(p, crs_seed, m);
  Stmt S = {0};
  for (u64 r = 0; r < p->module_size; r++) stmt_push(&S, make_ck_row(&R, m + r * d, p->wit_len));
  u64* ws = (u64*)malloc(rows * width * d * sizeof(u64));
  witness_to_slot(&R, w, ws, rows * width);
  u64* o = (u64*)malloc(S.n * rows * d * sizeof(u64));
  int rc = commit_all(&R, &S, ws, rows, width, o);
  if (!rc) witness_from_slot(&R, o, out, S.n * rows);
  free(o);
  free(ws);
  free(m);
  stmt_free(&S);
  ring_free(&R);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Proof layout (little-endian u64 words, ring elements in coefficient form): */
/*   header[8]: magic, d, q, module_size, wit_len, init_wit_rep, nof_rounds,   */
/*              folding                                                        */
/*   commitment                          module_size x init_wit_rep           */
/*   per round i:                                                              */
/*     SNARK and DECOMP_PARTS[i] > 1:    radix, rhs S x (K*parts)             */
/*     claims                            K words                               */
/*     for rep in 0,1: round polys       nr x K x 3 words, then norm3 rhs K    */
/*     SNARK: split rhs                  S x 2K                                */
/*     projected commitment              S x 1                                 */
/*     witness_rhs K, projection_rhs 1, l0, l1                                 */
/*     FOLDING: radix, rhs S x 4, then stop                                    */
/*   SNARK: final witness                K x width x d words                   */
/* ------------------------------------------------------------------------ */
#define PROOF_MAGIC 0x31504141534C4153ULL /* bytes "SALSAAP1" */

typedef struct {
  u64* w;
  u64 pos, cap;
  int overflow;
} Wr;
static inline void put(Wr* W, u64 v) {
  if (W->pos < W->cap) W->w[W->pos] = v;
  else W->overflow = 1;
  W->pos++;
}

typedef struct {
  const u64* w;
  u64 pos, cap;
  int underflow;
} Rd;
static inline u64 get(Rd* R) {
  if (R->pos < R->cap) return R->w[R->pos++];
  R->underflow = 1;
  R->pos++;
  return 0;
}

static u64 ilog2u(u64 x) { return x ? 63 - (u64)__builtin_clzll(x) : 0; }

u64 so_proof_size(const so_params* p) {
  const u64 d = p->d;
  u64 words = 8, S = p->module_size, K = p->init_wit_rep, width = p->wit_len;
  words += S * K * d;
  for (u64 i = 0; i < p->nof_rounds; i++) {
    u64 parts = p->decomp_parts[i < 12 ? i : 11];
    if (!p->folding && parts > 1) {
      words += 1 + S * K * parts * d;
      K *= parts;
    }
    words += K;
    u64 nr = ilog2u(width * d);
    for (int rep = 0; rep < 2; rep++) {
      words += nr * K * 3 + K * d;
      S += 1;
    }
    if (!p->folding) {
      words += S * 2 * K * d;
      K *= 2;
      width /= 2;
    }
    words += S * d;       /* projected commitment */
    words += (K + 1) * d; /* witness_rhs, projection_rhs */
    S += 1;
    words += 2 * d; /* l0, l1 */
    S += 1;
    K = 2;
    if (p->folding) {
      words += 1 + S * K * 2 * d;
      K *= 2;
      break;
    }
  }
  if (!p->folding) words += K * width * d;
  return words * 8;
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void put_ring_slot(const Ring* R, Wr* W, const u64* slot, u64 count) {
  u64 c[4096];
  for (u64 e = 0; e < count; e++) {
    from_slot(R, slot + e * R->d, c);
    for (u64 i = 0; i < R->d; i++) put(W, c[i]);
  }
}

/* norm_check_3 row from the challenges of one sum_check:
 * base = conj(tensor(last log2 d challenges)), ring tensors (1-c, c). */
static Row make_norm_row(const Ring* R, const u64* cs, u64 nr) {
  const u64 d = R->d, q = R->q, split = ilog2u(d), K = nr - split;
  u64 ext[4096], conj[4096], bslot[4096];
  so_tensor(ext, cs + K, split, q);
  so_conjugate(conj, ext, d, q);
  to_slot(R, conj, bslot);
  u64* t0 = (u64*)malloc((K ? K : 1) * sizeof(u64));
  u64* t1 = (u64*)malloc((K ? K : 1) * sizeof(u64));
  for (u64 k = 0; k < K; k++) {
    t0[k] = mod_sub(1, cs[k] % q, q);
    t1[k] = cs[k] % q;
  }
  Row row = make_scalar_tensor_row(R, t0, t1, K, bslot, 1);
  free(t0);
  free(t1);
  return row;
}

/* Rows pushed by batch_projections / send_cross_terms_before_join
 * (src/subroutines/project.rs:131-245) with c0 = 1: witness_lhs has base cj,
 * projected_lhs has base 1^256, both with (1, 1) factors. */
static void make_batch_rows(const Ring* R, const uint8_t* iz, const uint8_t* sg, u64 K, u64 width,
                            Row* wlhs, Row* plhs) {
  const u64 d = R->d, q = R->q, cw = K * PROJ_H;
  u64* cj = (u64*)malloc(cw * d * sizeof(u64));
  for (u64 j = 0; j < cw; j++) {
    long long v = 0;
    for (u64 i = 0; i < PROJ_H; i++)
      if (!iz[i * cw + j]) v += sg[i * cw + j] ? 1 : -1;
    u64 vm = v >= 0 ? (u64)v % q : q - ((u64)(-v) % q);
    slot_const(R, vm % q, cj + j * d);
  }
  u64 nof = ilog2u(width / cw), nofp = nof + ilog2u(K);
  u64* ones_t = (u64*)malloc((nofp ? nofp : 1) * sizeof(u64));
  for (u64 k = 0; k < nofp; k++) ones_t[k] = 1;
  *wlhs = make_scalar_tensor_row(R, ones_t, ones_t, nof, cj, cw);
  u64* ones = (u64*)malloc(PROJ_H * d * sizeof(u64));
  for (u64 j = 0; j < PROJ_H; j++) slot_const(R, 1, ones + j * d);
  *plhs = make_scalar_tensor_row(R, ones_t, ones_t, nofp, ones, PROJ_H);
  free(ones);
  free(ones_t);
  free(cj);
}

static void proj_challenge(u64 seed, u64 round, u64 cw, uint8_t* iz, uint8_t* sg) {
  u64 key = prf_key(seed, DOMAIN(DOM_PROJ, round, 0));
  for (u64 i = 0; i < PROJ_H * cw; i++) {
    u64 r = prf_at(key, i);
    iz[i] = (uint8_t)(r & 1);
    sg[i] = (uint8_t)((r >> 1) & 1);
  }
}

static void fold_challenge(const Ring* R, u64 seed, u64 round, u64 K, u64* cslot) {
  u64 key = prf_key(seed, DOMAIN(DOM_FOLD, round, 0));
  u64 c[4096];
  for (u64 k = 0; k < K; k++) {
    for (u64 i = 0; i < R->d; i++) c[i] = biased_from(prf_at(key, k * R->d + i), R->q);
    to_slot(R, c, cslot + k * R->d);
  }
}

static void nc_challenges(u64 seed, u64 round, u64 rep, u64 nr, u64 q, u64* cs) {
  u64 key = prf_key(seed, DOMAIN(DOM_NC, round, rep));
  for (u64 j = 0; j < nr; j++) cs[j] = uni_mod(prf_at(key, j), q);
}

static int params_ok(const so_params* p) {
  if (p->d < 4 || (p->d & (p->d - 1)) || p->d > 2048) return 0;
  if (p->q < 3 || p->q >= (1ULL << 62) || (p->q - 1) % p->d) return 0;
  if (!p->module_size || !p->wit_len || !p->init_wit_rep) return 0;
  if (p->nof_rounds > 12) return 0;
  return 1;
}

int so_prove(const so_params* p, u64 crs_seed, u64 seed, const u64* witness, uint8_t* proof,
             u64 proof_len, so_timing* tm, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  if (!params_ok(p)) return -1;
  const u64 need = so_proof_size(p);
  if (proof_len < need) return -2;
  so_timing T;
  memset(&T, 0, sizeof(T));
  Ring R;
  if (ring_init(&R, p->d, p->q)) return -1;
  const u64 d = p->d, q = p->q;
  Wr W = {(u64*)proof, 0, proof_len / 8, 0};
  put(&W, PROOF_MAGIC);
  put(&W, d);
  put(&W, q);
  put(&W, p->module_size);
  put(&W, p->wit_len);
  put(&W, p->init_wit_rep);
  put(&W, p->nof_rounds);
  put(&W, p->folding);

  int rc = 0;
  Stmt S = {0};
  u64* m = (u64*)malloc(p->module_size * d * sizeof(u64));
  so_sample_crs(p, crs_seed, m);
  for (u64 r = 0; r < p->module_size; r++) stmt_push(&S, make_ck_row(&R, m + r * d, p->wit_len));
  free(m);

  u64 K = p->init_wit_rep, width = p->wit_len;
  u64* Wc = (u64*)malloc(K * width * d * sizeof(u64));
  if (witness) memcpy(Wc, witness, K * width * d * sizeof(u64));
  else so_sample_witness(p, seed, Wc);
  u64* Ws = (u64*)malloc(K * width * d * sizeof(u64));

  double t0 = now_s(), tall = t0;
  witness_to_slot(&R, Wc, Ws, K * width);
  u64* out = (u64*)malloc(S.n * K * d * sizeof(u64));
  rc = commit_all(&R, &S, Ws, K, width, out);
  put_ring_slot(&R, &W, out, S.n * K);
  free(out);
  T.commit = now_s() - t0;

  for (u64 rd = 0; rd < p->nof_rounds && !rc; rd++) {
    const u64 parts = p->decomp_parts[rd < 12 ? rd : 11];
    if (!p->folding && parts > 1) {
      t0 = now_s();
      u64* nw = (u64*)malloc(K * parts * width * d * sizeof(u64));
      u64 radix;
      decompose_impl(Wc, K, width, d, q, parts, nw, &radix);
      free(Wc);
      Wc = nw;
      K *= parts;
      free(Ws);
      Ws = (u64*)malloc(K * width * d * sizeof(u64));
      witness_to_slot(&R, Wc, Ws, K * width);
      put(&W, radix);
      out = (u64*)malloc(S.n * K * d * sizeof(u64));
      rc = commit_all(&R, &S, Ws, K, width, out);
      put_ring_slot(&R, &W, out, S.n * K);
      free(out);
      T.decomp += now_s() - t0;
      if (rc) break;
    }
    /* norm_check_1 */
    t0 = now_s();
    const u64 flat = width * d, nr = ilog2u(flat);
    for (u64 k = 0; k < K; k++) put(&W, so_sum_sq(Wc + k * flat, flat, q));
    T.norm1 += now_s() - t0;
    for (u64 rep = 0; rep < 2 && !rc; rep++) {
      t0 = now_s();
      u64* cs = (u64*)malloc((nr ? nr : 1) * sizeof(u64));
      nc_challenges(seed, rd, rep, nr, q, cs);
      u64** v = (u64**)malloc(K * sizeof(u64*));
      for (u64 k = 0; k < K; k++) {
        v[k] = (u64*)malloc(flat * sizeof(u64));
        memcpy(v[k], Wc + k * flat, flat * sizeof(u64));
      }
      u64* polys = (u64*)malloc((nr ? nr : 1) * K * 3 * sizeof(u64));
      sumcheck_rows(&R.M, v, K, flat, cs, polys);
      for (u64 i = 0; i < nr * K * 3; i++) put(&W, polys[i]);
      for (u64 k = 0; k < K; k++) free(v[k]);
      free(v);
      free(polys);
      T.norm2 += now_s() - t0;
      t0 = now_s();
      Row row = make_norm_row(&R, cs, nr);
      u64* E = (u64*)malloc(width * d * sizeof(u64));
      rc = row_layer(&R, &row, width, E);
      u64* rhs = (u64*)malloc(K * d * sizeof(u64));
      if (!rc) dot_layer(&R, E, Ws, K, width, rhs);
      put_ring_slot(&R, &W, rhs, K);
      stmt_push(&S, row);
      free(rhs);
      free(E);
      free(cs);
      T.norm3 += now_s() - t0;
    }
    if (rc) break;
    if (!p->folding) {
      /* split (src/subroutines/split.rs:45-76): rows L_0..L_{K-1}, R_0..R_{K-1} */
      t0 = now_s();
      const u64 hw = width / 2;
      u64* nc = (u64*)malloc(K * width * d * sizeof(u64));
      u64* ns = (u64*)malloc(K * width * d * sizeof(u64));
      for (u64 k = 0; k < K; k++)
        for (u64 half = 0; half < 2; half++) {
          memcpy(nc + ((half * K + k) * hw) * d, Wc + (k * width + half * hw) * d, hw * d * sizeof(u64));
          memcpy(ns + ((half * K + k) * hw) * d, Ws + (k * width + half * hw) * d, hw * d * sizeof(u64));
        }
      free(Wc);
      free(Ws);
      Wc = nc;
      Ws = ns;
      K *= 2;
      width = hw;
      out = (u64*)malloc(S.n * K * d * sizeof(u64));
      rc = commit_all(&R, &S, Ws, K, width, out);
      put_ring_slot(&R, &W, out, S.n * K);
      free(out);
      T.split += now_s() - t0;
      if (rc) break;
    }
    /* project */
    t0 = now_s();
    const u64 cw = K * PROJ_H;
    if (cw > width) {
      rc = -3;
      break;
    }
    uint8_t* iz = (uint8_t*)malloc(PROJ_H * cw);
    uint8_t* sg = (uint8_t*)malloc(PROJ_H * cw);
    proj_challenge(seed, rd, cw, iz, sg);
    u64* P = (u64*)malloc(width * d * sizeof(u64));
    u64* Ps = (u64*)malloc(width * d * sizeof(u64));
    project_impl(Wc, K, width, d, q, iz, sg, P);
    witness_to_slot(&R, P, Ps, width);
    out = (u64*)malloc(S.n * d * sizeof(u64));
    rc = commit_all(&R, &S, Ps, 1, width, out);
    put_ring_slot(&R, &W, out, S.n);
    free(out);
    /* batch_projections */
    Row wlhs, plhs;
    make_batch_rows(&R, iz, sg, K, width, &wlhs, &plhs);
    u64* E = (u64*)malloc(width * d * sizeof(u64));
    u64* wrhs = (u64*)malloc(K * d * sizeof(u64));
    u64 prhs[4096], l0[4096], l1[4096];
    rc |= row_layer(&R, &wlhs, width, E);
    dot_layer(&R, E, Ws, K, width, wrhs);
    dot_layer(&R, E, Ps, 1, width, l1);
    rc |= row_layer(&R, &plhs, width, E);
    dot_layer(&R, E, Ps, 1, width, prhs);
    put_ring_slot(&R, &W, wrhs, K);
    put_ring_slot(&R, &W, prhs, 1);
    {
      u64 sum[4096];
      memset(sum, 0, d * sizeof(u64));
      for (u64 k = 0; k < K; k++)
        for (u64 i = 0; i < d; i++) sum[i] = mod_add(sum[i], wrhs[k * d + i], q);
      if (memcmp(sum, prhs, d * sizeof(u64))) rc = -10; /* project.rs:196-198 */
    }
    stmt_push(&S, wlhs);
    T.projection += now_s() - t0;
    /* fold + cross terms + join */
    t0 = now_s();
    u64* cslot = (u64*)malloc(K * d * sizeof(u64));
    fold_challenge(&R, seed, rd, K, cslot);
    u64* Fs = (u64*)malloc(width * d * sizeof(u64));
    fold_slot(&R, Ws, K, width, cslot, Fs);
    dot_layer(&R, E, Fs, 1, width, l0); /* E still holds projected_lhs */
    put_ring_slot(&R, &W, l0, 1);
    put_ring_slot(&R, &W, l1, 1);
    stmt_push(&S, plhs);
    free(Wc);
    free(Ws);
    K = 2;
    Wc = (u64*)malloc(K * width * d * sizeof(u64));
    Ws = (u64*)malloc(K * width * d * sizeof(u64));
    witness_from_slot(&R, Fs, Wc, width);
    memcpy(Wc + width * d, P, width * d * sizeof(u64));
    memcpy(Ws, Fs, width * d * sizeof(u64));
    memcpy(Ws + width * d, Ps, width * d * sizeof(u64));
    free(Fs);
    free(cslot);
    free(E);
    free(wrhs);
    free(P);
    free(Ps);
    free(iz);
    free(sg);
    T.fold += now_s() - t0;
    if (p->folding) {
      t0 = now_s();
      u64* nw = (u64*)malloc(K * 2 * width * d * sizeof(u64));
      u64 radix;
      decompose_impl(Wc, K, width, d, q, 2, nw, &radix);
      free(Wc);
      Wc = nw;
      K *= 2;
      free(Ws);
      Ws = (u64*)malloc(K * width * d * sizeof(u64));
      witness_to_slot(&R, Wc, Ws, K * width);
      put(&W, radix);
      out = (u64*)malloc(S.n * K * d * sizeof(u64));
      rc = commit_all(&R, &S, Ws, K, width, out);
      put_ring_slot(&R, &W, out, S.n * K);
      free(out);
      T.decomp += now_s() - t0;
      break;
    }
  }
  if (!rc && !p->folding)
    for (u64 i = 0; i < K * width * d; i++) put(&W, Wc[i]);
  T.total = now_s() - tall;
  if (tm) *tm = T;
  if (!rc && (W.overflow || W.pos * 8 != need)) rc = -4;
  free(Wc);
  free(Ws);
  stmt_free(&S);
  ring_free(&R);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Verifier: the checks the reference runs inline (verify_decomp,             */
/* verify_norm_check_2/3, verifier_split, verify_batching, verifier_fold,     */
/* verifier_join and the final assert of src/protocol.rs:464-472).            */
/* Returns 0 on accept, else the negative code of the first failing check.   */
/* ------------------------------------------------------------------------ */
static void get_ring_slot(const Ring* R, Rd* D, u64* slot, u64 count) {
  u64 c[4096];
  for (u64 e = 0; e < count; e++) {
    for (u64 i = 0; i < R->d; i++) c[i] = get(D);
    to_slot(R, c, slot + e * R->d);
  }
}

/* compose_with_radix_mod (src/arithmetic.rs:1719-1755), slot form. */
static void compose(const Ring* R, const u64* D, u64 rows, u64 cols, u64 parts, u64 radix, u64* out) {
  const u64 d = R->d, q = R->q, shift = (u64)__builtin_ctzll(radix);
  for (u64 j = 0; j < rows; j++)
    for (u64 i = 0; i < cols; i++)
      for (u64 t = 0; t < d; t++) {
        u64 acc = 0;
        for (u64 c = 0; c < parts; c++) {
          u64 pw = (shift * c < 64) ? ((1ULL << (shift * c)) % q) : 0;
          acc = mod_add(acc, mod_mul(&R->M, D[((j * cols + i) * parts + c) * d + t], pw), q);
        }
        out[(j * cols + i) * d + t] = acc;
      }
}

int so_verify(const so_params* p, u64 crs_seed, u64 seed, const uint8_t* proof, u64 proof_len) {
  if (!params_ok(p)) return -1;
  if (proof_len != so_proof_size(p)) return -2;
  Ring R;
  if (ring_init(&R, p->d, p->q)) return -1;
  const u64 d = p->d, q = p->q;
  Rd D = {(const u64*)proof, 0, proof_len / 8, 0};
  u64 hdr[8];
  for (int i = 0; i < 8; i++) hdr[i] = get(&D);
  if (hdr[0] != PROOF_MAGIC || hdr[1] != d || hdr[2] != q || hdr[3] != p->module_size ||
      hdr[4] != p->wit_len || hdr[5] != p->init_wit_rep || hdr[6] != p->nof_rounds || hdr[7] != p->folding)
    return -3;
  int rc = 0;
  Stmt S = {0};
  u64* m = (u64*)malloc(p->module_size * d * sizeof(u64));
  so_sample_crs(p, crs_seed, m);
  for (u64 r = 0; r < p->module_size; r++) stmt_push(&S, make_ck_row(&R, m + r * d, p->wit_len));
  free(m);
  u64 K = p->init_wit_rep, width = p->wit_len;
  /* verifier rhs: V[j][k], S.n x K ring elements, slot form */
  u64* V = (u64*)malloc(S.n * K * d * sizeof(u64));
  get_ring_slot(&R, &D, V, S.n * K);
  u64 tmp[4096], tmp2[4096];

  for (u64 rd = 0; rd < p->nof_rounds && !rc; rd++) {
    const u64 parts = p->decomp_parts[rd < 12 ? rd : 11];
    if (!p->folding && parts > 1) {
      u64 radix = get(&D);
      if (!radix || (radix & (radix - 1))) {
        rc = -20;
        break;
      }
      u64* Dm = (u64*)malloc(S.n * K * parts * d * sizeof(u64));
      get_ring_slot(&R, &D, Dm, S.n * K * parts);
      u64* C = (u64*)malloc(S.n * K * d * sizeof(u64));
      /* compose is linear, so composing slot forms equals composing coefficients */
      compose(&R, Dm, S.n, K, parts, radix, C);
      if (memcmp(C, V, S.n * K * d * sizeof(u64))) rc = -21; /* decomp.rs:105 */
      free(C);
      free(V);
      V = Dm;
      K *= parts;
    }
    if (rc) break;
    const u64 flat = width * d, nr = ilog2u(flat);
    u64* claims = (u64*)malloc(K * sizeof(u64));
    for (u64 k = 0; k < K; k++) claims[k] = get(&D);
    for (u64 rep = 0; rep < 2 && !rc; rep++) {
      u64* cl = (u64*)malloc(K * sizeof(u64));
      memcpy(cl, claims, K * sizeof(u64));
      u64* cs = (u64*)malloc((nr ? nr : 1) * sizeof(u64));
      nc_challenges(seed, rd, rep, nr, q, cs);
      for (u64 j = 0; j < nr; j++)
        for (u64 k = 0; k < K; k++) {
          u64 f0 = get(&D), f1 = get(&D), f2 = get(&D);
          if (f0 >= q || f1 >= q || f2 >= q) rc = rc ? rc : -30;
          u64 lhs = mod_add(mod_add(mod_add(f0, f0, q), mod_add(f1, f1, q), q), f2, q);
          if (lhs != cl[k]) rc = rc ? rc : -31; /* fast_norm_check.rs:364-371 */
          u64 c = cs[j];
          cl[k] = mod_add(mod_add(f0, mod_mul(&R.M, mod_add(f1, f1, q), c), q),
                          mod_mul(&R.M, mod_mul(&R.M, f2, c), c), q);
        }
      /* verify_norm_check_3: constant coefficient squared equals the final claim */
      u64* rhs = (u64*)malloc(K * d * sizeof(u64));
      for (u64 k = 0; k < K; k++) {
        for (u64 i = 0; i < d; i++) tmp[i] = get(&D);
        if (mod_mul(&R.M, tmp[0], tmp[0]) != cl[k]) rc = rc ? rc : -32; /* fast_norm_check.rs:450-457 */
        to_slot(&R, tmp, rhs + k * d);
      }
      V = (u64*)realloc(V, (S.n + 1) * K * d * sizeof(u64));
      memcpy(V + S.n * K * d, rhs, K * d * sizeof(u64));
      stmt_push(&S, make_norm_row(&R, cs, nr));
      free(rhs);
      free(cs);
      free(cl);
    }
    free(claims);
    if (rc) break;
    if (!p->folding) {
      /* verifier_split (src/subroutines/split.rs:171-221) */
      u64* SR = (u64*)malloc(S.n * 2 * K * d * sizeof(u64));
      get_ring_slot(&R, &D, SR, S.n * 2 * K);
      for (u64 j = 0; j < S.n && !rc; j++) {
        u64 jj;
        const Row* row = &S.r[j];
        if (row_layer_index(row, width, &jj) || jj == 0) {
          rc = -40;
          break;
        }
        const u64 idx = row->K - jj;
        const u64* t0 = row->tens + (2 * idx) * d;
        const u64* t1 = row->tens + (2 * idx + 1) * d;
        for (u64 k = 0; k < K; k++) {
          slot_mul(&R, t0, SR + (j * 2 * K + k) * d, tmp);
          slot_mul(&R, t1, SR + (j * 2 * K + K + k) * d, tmp2);
          for (u64 i = 0; i < d; i++) tmp[i] = mod_add(tmp[i], tmp2[i], q);
          if (memcmp(tmp, V + (j * K + k) * d, d * sizeof(u64))) rc = -41; /* split.rs:211 */
        }
      }
      free(V);
      V = SR;
      K *= 2;
      width /= 2;
      if (rc) break;
    }
    const u64 cw = K * PROJ_H;
    if (cw > width) {
      rc = -3;
      break;
    }
    const u64 Sp = S.n;
    u64* PC = (u64*)malloc(Sp * d * sizeof(u64));
    get_ring_slot(&R, &D, PC, Sp);
    uint8_t* iz = (uint8_t*)malloc(PROJ_H * cw);
    uint8_t* sg = (uint8_t*)malloc(PROJ_H * cw);
    proj_challenge(seed, rd, cw, iz, sg);
    Row wlhs, plhs;
    make_batch_rows(&R, iz, sg, K, width, &wlhs, &plhs);
    u64* wrhs = (u64*)malloc(K * d * sizeof(u64));
    u64 prhs[4096], l0[4096], l1[4096];
    get_ring_slot(&R, &D, wrhs, K);
    get_ring_slot(&R, &D, prhs, 1);
    memset(tmp, 0, d * sizeof(u64));
    for (u64 k = 0; k < K; k++)
      for (u64 i = 0; i < d; i++) tmp[i] = mod_add(tmp[i], wrhs[k * d + i], q);
    if (memcmp(tmp, prhs, d * sizeof(u64))) rc = -50; /* project.rs:214 */
    V = (u64*)realloc(V, (S.n + 1) * K * d * sizeof(u64));
    memcpy(V + S.n * K * d, wrhs, K * d * sizeof(u64));
    stmt_push(&S, wlhs);
    /* verifier_fold (src/subroutines/fold.rs:58-67) */
    u64* cslot = (u64*)malloc(K * d * sizeof(u64));
    fold_challenge(&R, seed, rd, K, cslot);
    u64* VF = (u64*)calloc(S.n * d, sizeof(u64));
    for (u64 j = 0; j < S.n; j++)
      for (u64 k = 0; k < K; k++) {
        slot_mul(&R, cslot + k * d, V + (j * K + k) * d, tmp);
        for (u64 i = 0; i < d; i++) VF[j * d + i] = mod_add(VF[j * d + i], tmp[i], q);
      }
    get_ring_slot(&R, &D, l0, 1);
    get_ring_slot(&R, &D, l1, 1);
    /* verifier_join (src/subroutines/project.rs:247-275) */
    stmt_push(&S, plhs);
    u64* NV = (u64*)malloc(S.n * 2 * d * sizeof(u64));
    for (u64 i = 0; i < Sp; i++) {
      memcpy(NV + (i * 2) * d, VF + i * d, d * sizeof(u64));
      memcpy(NV + (i * 2 + 1) * d, PC + i * d, d * sizeof(u64));
    }
    memcpy(NV + (Sp * 2) * d, VF + Sp * d, d * sizeof(u64));
    memcpy(NV + (Sp * 2 + 1) * d, l1, d * sizeof(u64));
    memcpy(NV + ((Sp + 1) * 2) * d, l0, d * sizeof(u64));
    memcpy(NV + ((Sp + 1) * 2 + 1) * d, prhs, d * sizeof(u64));
    free(V);
    V = NV;
    K = 2;
    free(VF);
    free(cslot);
    free(wrhs);
    free(iz);
    free(sg);
    free(PC);
    if (rc) break;
    if (p->folding) {
      u64 radix = get(&D);
      if (!radix || (radix & (radix - 1))) {
        rc = -20;
        break;
      }
      u64* Dm = (u64*)malloc(S.n * K * 2 * d * sizeof(u64));
      get_ring_slot(&R, &D, Dm, S.n * K * 2);
      u64* C = (u64*)malloc(S.n * K * d * sizeof(u64));
      compose(&R, Dm, S.n, K, 2, radix, C);
      if (memcmp(C, V, S.n * K * d * sizeof(u64))) rc = -21;
      free(C);
      free(V);
      V = Dm;
      K *= 2;
      break;
    }
  }
  if (!rc && !p->folding) {
    /* final check, src/protocol.rs:464-472 */
    u64* Wc = (u64*)malloc(K * width * d * sizeof(u64));
    for (u64 i = 0; i < K * width * d; i++) Wc[i] = get(&D);
    u64* Ws = (u64*)malloc(K * width * d * sizeof(u64));
    witness_to_slot(&R, Wc, Ws, K * width);
    u64* out = (u64*)malloc(S.n * K * d * sizeof(u64));
    rc = commit_all(&R, &S, Ws, K, width, out);
    if (!rc && memcmp(out, V, S.n * K * d * sizeof(u64))) rc = -60;
    free(out);
    free(Ws);
    free(Wc);
  }
  if (!rc && (D.underflow || D.pos != D.cap)) rc = -5;
  free(V);
  stmt_free(&S);
  ring_free(&R);
  return rc;
}
