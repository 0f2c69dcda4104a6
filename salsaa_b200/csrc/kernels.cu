// kernels.cu — the SALSAA prover kernels for sm_100a.
//
// Reference algorithms (paths relative to the lattice-arguments/salsaa root):
//   CRS / commitment keys    src/subroutines/crs.rs:23-72
//   witness sampling         src/cyclotomic_ring.rs:293-317, src/arithmetic.rs:1160-1175
//   norm-check sumcheck      src/subroutines/fast_norm_check.rs:135-199,282-441
//   decomposition            src/arithmetic.rs:1461-1593
//   projection               src/subroutines/project.rs:26-103
//   fold                     src/subroutines/fold.rs:22-27,70-75
//   structured dot products  src/arithmetic.rs:459-536
#include <vector>
#include "kernels.cuh"

namespace salsaa {

namespace {

inline int check_launch(const char* what) {
  salsaa_count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, what);
}

inline unsigned grid_1d(u64 work, unsigned threads, unsigned cap = 148 * 32) {
  u64 g = (work + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}


__device__ __forceinline__ u64 nc_challenge(const DevState* ds, u32 round, u32 rep, u64 j, u64 q) {
  return uni_mod(prf_at(prf_key(ds->seed, domain_id(DOM_NC, round, rep)), j), q);
}

}  // namespace

// ---------------------------------------------------------------------------
// CRS: MODULE_SIZE uniform ring elements (CyclotomicRing::random), and the
// two-level power tables of the commitment-key rows (m, m^2, ..., m^L):
//   tlo[r][lo] = m^(lo+1) as (even, odd, zeta*odd) planes,  lo < B
//   thi[r][hi] = m^(hi*B) in slot form,                     hi < L/B
// so that m^(i+1) = thi[i / B] * tlo[i % B].
// ---------------------------------------------------------------------------
__global__ void gen_crs_kernel(u64* m, u32 rows, u32 d, u64 q, u64 crs_seed) {
  u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (u64)rows * d) return;
  u32 r = (u32)(t / d), i = (u32)(t % d);
  m[t] = uni_mod(prf_at(prf_key(crs_seed, domain_id(DOM_CRS, 0, r)), i), q);
}

int launch_gen_crs(u64* m_coef, u32 rows, u32 d, u64 q, u64 crs_seed, cudaStream_t st) {
  u64 tot = (u64)rows * d;
  gen_crs_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(m_coef, rows, d, q, crs_seed);
  return check_launch("gen_crs");
}

// (be + X bo)^e in F_q[X]/(X^2 - z).
__device__ void slot_pow(const ModQ& M, u64 z, u64 be, u64 bo, u64 e, u64& re, u64& ro) {
  u64 ae = 1 % M.q, ao = 0, xe = be, xo = bo;
  while (e) {
    if (e & 1) slot_mul(M, ae, ao, xe, xo, z, ae, ao);
    e >>= 1;
    if (e) slot_mul(M, xe, xo, xe, xo, z, xe, xo);
  }
  re = ae;
  ro = ao;
}

__device__ __forceinline__ u64 pack25(u64 v) { return ((v >> 25) << 32) | (v & 0x1FFFFFFull); }

__global__ void ck_tlo_kernel(const u64* ms, u32 rows, u32 n, u32 B, ModQ M, const u64* zeta, u64* tlo) {
  u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (u64)rows * B * n) return;
  u32 s = (u32)(t % n);
  u64 rl = t / n;
  u32 lo = (u32)(rl % B), r = (u32)(rl / B);
  const u64* m = ms + (u64)r * 2 * n;
  u64 e, o;
  slot_pow(M, zeta[s], m[s], m[n + s], (u64)lo + 1, e, o);
  u64* dst = tlo + ((u64)r * B + lo) * 3 * n;
  const u64 z = mul_mod(M, zeta[s], o);
  if (M.q < (1ULL << 50)) {  // stored as 25-bit limbs in the two 32-bit halves
    dst[s] = pack25(e);
    dst[n + s] = pack25(o);
    dst[2 * n + s] = pack25(z);
  } else {
    dst[s] = e;
    dst[n + s] = o;
    dst[2 * n + s] = z;
  }
}

__global__ void ck_thi_kernel(const u64* ms, u32 rows, u32 n, u32 B, u32 nhi, ModQ M, const u64* zeta,
                              u64* thi) {
  u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (u64)rows * nhi * n) return;
  u32 s = (u32)(t % n);
  u64 rh = t / n;
  u32 hi = (u32)(rh % nhi), r = (u32)(rh / nhi);
  const u64* m = ms + (u64)r * 2 * n;
  u64 e, o;
  slot_pow(M, zeta[s], m[s], m[n + s], (u64)hi * B, e, o);
  u64* dst = thi + ((u64)r * nhi + hi) * 2 * n;
  dst[s] = e;
  dst[n + s] = o;
}

int launch_ck_tables(const u64* m_slot, u32 rows, const NttDev& T, const ModQ& M, u64 L, u64* tlo, u64* thi,
                     cudaStream_t st) {
  const u32 n = T.n;
  const u32 B = (u32)(L < CK_KEY_BLOCK ? L : CK_KEY_BLOCK);
  const u32 nhi = (u32)(L / B);
  u64 tot = (u64)rows * B * n;
  ck_tlo_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(m_slot, rows, n, B, M, T.zeta, tlo);
  int rc = check_launch("ck_tlo");
  if (rc) return rc;
  tot = (u64)rows * nhi * n;
  ck_thi_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(m_slot, rows, n, B, nhi, M, T.zeta, thi);
  return check_launch("ck_thi");
}

// ---------------------------------------------------------------------------
// Witness: random_bounded(2) coefficients (0 w.p. 1/2, +-1 w.p. 1/4 each).
// ---------------------------------------------------------------------------
__global__ void gen_witness_kernel(u64* w, u32 rows, u64 per_row, u64 q, const DevState* ds) {
  const u64 seed = ds->seed;
  for (u32 k = 0; k < rows; k++) {
    const u64 key = prf_key(seed, domain_id(DOM_WIT, 0, k));
    for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < per_row; t += (u64)gridDim.x * blockDim.x) {
      u64 r = prf_at(key, t);
      u64 mag = r & 1, neg = (r >> 1) & 1;
      w[k * per_row + t] = mag ? (neg ? q - 1 : 1) : 0;
    }
  }
}

int launch_gen_witness(u64* w, u32 rows, u64 width, u32 d, u64 q, const DevState* ds, cudaStream_t st) {
  const u64 per_row = width * d;
  gen_witness_kernel<<<grid_1d(per_row, 256), 256, 0, st>>>(w, rows, per_row, q, ds);
  return check_launch("gen_witness");
}

// Short witness sent as centred int8 coefficients: out[i] = in[i] mod q.
// Four coefficients per thread step (one 4-byte load, two 16-byte stores).
__global__ void expand_i8_kernel(const int8_t* __restrict__ in, u64 n, u64 q, u64* __restrict__ out) {
  const u64 stride = (u64)gridDim.x * blockDim.x, n4 = n / 4;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < n4; t += stride) {
    const u32 w = __ldg((const u32*)in + t);
    u64 e[4];
#pragma unroll
    for (u32 b = 0; b < 4; b++) {
      const int s = (int8_t)(w >> (8 * b));
      e[b] = s < 0 ? q - (u64)(-s) : (u64)s;
    }
    ulonglong2* o = (ulonglong2*)(out + 4 * t);
    o[0] = make_ulonglong2(e[0], e[1]);
    o[1] = make_ulonglong2(e[2], e[3]);
  }
  for (u64 i = 4 * n4 + (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int s = in[i];
    out[i] = s < 0 ? q - (u64)(-s) : (u64)s;
  }
}
int launch_expand_i8(const int8_t* in, u64 n, u64 q, u64* out, cudaStream_t st) {
  if (!n) return 0;
  if ((uintptr_t)in % 4 || (uintptr_t)out % 16) return salsaa_set_error(-2, "expand_i8: misaligned buffers");
  expand_i8_kernel<<<grid_1d((n + 3) / 4, 256), 256, 0, st>>>(in, n, q, out);
  return check_launch("expand_i8");
}

__global__ void fill_kernel(u64* p, u64 n, u64 v) {
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (u64)gridDim.x * blockDim.x) p[t] = v;
}
int launch_fill(u64* p, u64 n, u64 v, cudaStream_t st) {
  if (!n) return 0;
  fill_kernel<<<grid_1d(n, 256), 256, 0, st>>>(p, n, v);
  return check_launch("fill");
}

__global__ void pointwise_mul_kernel(u64* r, const u64* b, u64 n, ModQ M) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    r[i] = mul_mod(M, r[i], b[i]);
}

int launch_pointwise_mul(u64* r, const u64* b, u64 n, u64 q, cudaStream_t st) {
  if (!n) return 0;
  pointwise_mul_kernel<<<grid_1d(n, 256), 256, 0, st>>>(r, b, n, make_modq(q));
  return check_launch("pointwise_mul");
}

// ---------------------------------------------------------------------------
// Norm-check sumcheck (sum_check, src/subroutines/fast_norm_check.rs:135-199)
// for all witness rows and both amplification repetitions at once.
//
// Round j folds v_j (length L) into v_{j+1} = v_j[:L/2] + c_j (v_j[L/2:] -
// v_j[:L/2]); its polynomial is (f0, f1, f2) = (S00, S01 - S00,
// S11 - 2 S01 + S00) with S00 = sum v0^2, S01 = sum v0 v1, S11 = sum v1^2 over
// the halves.  The challenges are a PRF stream, known before the data, so
// one pass can run T rounds: a thread owns the 2^T elements
// v_j[g + m L/2^T] (m < 2^T), which are closed under the next T foldings,
// sums all T rounds' polynomials and writes v_{j+T}[g].  The first pass reads
// the witness once for both repetitions (round 0 is shared).
// sums[((rep * nr + j) * rows + k) * 3 + {0,1,2}] hold S00, S01, S11.
// ---------------------------------------------------------------------------
constexpr u32 SC_T = 4;          // rounds per streaming pass
constexpr u32 SC_TAIL = 16384;   // vectors this short finish in one CTA (batched sumchecks)
// A single sumcheck streams four-round passes over many CTAs while the vector
// is longer than this and the pass leaves at least d values (norm_check_3's
// vector is captured at length d by the tail); the tail then finishes in one
// CTA per (repetition, row).
constexpr u32 SC_TAIL_ONE = 2048;

// Lazy sums: with q < 2^50 each product is < 2^100 and a thread's sum of
// far fewer than 2^27 products fits in 128 bits.
struct Sum128 {
  u64 lo, hi;
};
__device__ __forceinline__ void s128_add_prod(Sum128& s, u64 a, u64 b) {
  const u64 pl = a * b, ph = __umul64hi(a, b);
  s.lo += pl;
  s.hi += ph + (s.lo < pl);
}
__device__ __forceinline__ void s128_add(Sum128& s, const Sum128& t) {
  s.lo += t.lo;
  s.hi += t.hi + (s.lo < t.lo);
}
// one accumulator slot: lazy 128-bit sum, or a residue when q >= 2^50
template <bool LAZY>
struct ScAcc {
  Sum128 s;
  u64 g;
  __device__ __forceinline__ void zero() {
    s.lo = s.hi = 0;
    g = 0;
  }
  __device__ __forceinline__ void mac(const ModQ& M, u64 a, u64 b) {
    if (LAZY) s128_add_prod(s, a, b);
    else g = add_mod(g, mul_mod(M, a, b), M.q);
  }
};
// Block totals of NV accumulator slots at once (one barrier for all of them,
// one more so the shared buffer can be reused); thread i < NV gets total i.
// red: NV x 32 slots of shared memory.
template <bool LAZY, int NV>
__device__ __forceinline__ u64 block_totals(const ModQ& M, ScAcc<LAZY> (&v)[NV], Sum128* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++) {
    if (LAZY) {
      Sum128 t = v[i].s;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        Sum128 u;
        u.lo = __shfl_down_sync(0xffffffffu, t.lo, o);
        u.hi = __shfl_down_sync(0xffffffffu, t.hi, o);
        s128_add(t, u);
      }
      if (lane == 0) red[i * 32 + wid] = t;
    } else {
      u64 t = v[i].g;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t = add_mod(t, __shfl_down_sync(0xffffffffu, t, o), M.q);
      if (lane == 0) red[i * 32 + wid].lo = t;
    }
  }
  __syncthreads();
  u64 r = 0;
  if (threadIdx.x < NV) {
    const int i = threadIdx.x;
    if (LAZY) {
      Sum128 a = red[i * 32];
      for (int w = 1; w < nw; w++) s128_add(a, red[i * 32 + w]);
      r = reduce128_any(M, a.hi, a.lo);
    } else {
      for (int w = 0; w < nw; w++) r = add_mod(r, red[i * 32 + w].lo, M.q);
    }
  }
  __syncthreads();
  return r;
}

// Round challenges t < T (chal(t)) and their Shoup companions, computed by
// threads 0 .. T-1 into shared memory sch[2T] and read by every thread: the
// companion is a 128-bit division, far too costly to repeat in every thread.
// Every thread of the CTA calls it; sch must not be read by a previous use
// after this call starts (the callers' block reductions in between order it).
template <u32 T, typename F>
__device__ __forceinline__ void shared_challenges(u64* sch, F chal, u64 q, u64 (&c)[T], u64 (&cp)[T]) {
  if (threadIdx.x < T) {
    const u64 v = chal(threadIdx.x);
    sch[threadIdx.x] = v;
    sch[T + threadIdx.x] = (u64)((((unsigned __int128)v) << 64) / q);
  }
  __syncthreads();
#pragma unroll
  for (u32 t = 0; t < T; t++) {
    c[t] = sch[t];
    cp[t] = sch[T + t];
  }
}

__device__ __forceinline__ u64 fold1(u64 a, u64 b, u64 c, u64 cp, u64 q) {
  return add_mod(a, mul_shoup(sub_mod(b, a, q), c, cp, q), q);
}
__device__ __forceinline__ u64 shoup_dev(u64 c, u64 q) { return (u64)((((unsigned __int128)c) << 64) / q); }

// T rounds on a group x[0 .. 2^T): sums of round t go to acc[t][0..2].
template <bool LAZY, u32 T>
__device__ __forceinline__ void group_rounds(const ModQ& M, u64 (&x)[1 << T], const u64* c, const u64* cp,
                                             ScAcc<LAZY> (&acc)[T][3], u32 t0) {
#pragma unroll
  for (u32 t = 0; t < T; t++) {
    const u32 h = (1u << T) >> (t + 1);
    if (t >= t0) {
#pragma unroll
      for (u32 m = 0; m < h; m++) {
        acc[t][0].mac(M, x[m], x[m]);
        acc[t][1].mac(M, x[m], x[m + h]);
        acc[t][2].mac(M, x[m + h], x[m + h]);
      }
    }
#pragma unroll
    for (u32 m = 0; m < h; m++) x[m] = fold1(x[m], x[m + h], c[t], cp[t], M.q);
  }
}

// First pass: v_0 rows (shared) -> v_T for each repetition.  The two
// repetitions run in neighbouring CTAs (blockIdx.x = 2 * block + rep) over
// the same witness range, so the second read of each range hits L2; this
// halves the per-thread accumulators (two CTAs per SM).  Round 0 is the same
// for both repetitions: the rep-0 CTA adds its sums to both.
template <bool LAZY>
__global__ void __launch_bounds__(256, 2) sc_first_kernel(RowSet w, u32 rows, u64 nlen, ModQ M, const DevState* ds,
                                                          u32 round, u64* out, u64 sout, u64* sums, u32 nr,
                                                          bool plain, const u32* only_if) {
  constexpr u32 T = SC_T, G = 1u << T;
  __shared__ Sum128 red[SC_T * 3 * 32];
  if (only_if && *only_if == 0) return;  // the tensor-core pass covered this launch
  const u32 k = blockIdx.y, rep = blockIdx.x & 1, bx = blockIdx.x >> 1, nbx = gridDim.x >> 1;
  const u64* x = w.p[k];
  const bool nar = (w.narrow >> k) & 1;
  const u64 q = M.q, ng = nlen / G;
  __shared__ u64 sch[2 * T];
  u64 c[T], cp[T];
  shared_challenges<T>(sch, [&](u32 t) { return nc_challenge(ds, round, rep, t, q); }, q, c, cp);
  ScAcc<LAZY> acc[T][3];  // acc[0] = round 0, only kept by the rep-0 CTAs
#pragma unroll
  for (u32 t = 0; t < T; t++)
#pragma unroll
    for (u32 a = 0; a < 3; a++) acc[t][a].zero();
  for (u64 g = (u64)bx * blockDim.x + threadIdx.x; g < ng; g += (u64)nbx * blockDim.x) {
    u64 v[G];
#pragma unroll
    for (u32 m = 0; m < G; m++) v[m] = wres(x, nar, g + m * ng, q);
    group_rounds<LAZY, T>(M, v, c, cp, acc, rep == 0 ? 0 : 1);
    out[((u64)rep * rows + k) * sout + g] = v[0];
  }
  ScAcc<LAZY> flat[T * 3];
#pragma unroll
  for (u32 t = 0; t < T; t++)
#pragma unroll
    for (u32 a = 0; a < 3; a++) flat[t * 3 + a] = acc[t][a];
  const u64 r = block_totals<LAZY, T * 3>(M, flat, red);
  if (threadIdx.x < T * 3) {
    const u32 t = threadIdx.x / 3, a = threadIdx.x % 3;
    if (t > 0 || rep == 0) atomic_add_mod(&sums[((rep * (u64)nr + t) * rows + k) * 3 + a], r, q, plain);
    if (t == 0 && rep == 0) atomic_add_mod(&sums[((1 * (u64)nr + 0) * rows + k) * 3 + a], r, q, plain);
  }
}

// Later passes: v_j (per (rep,row), stride sin) -> v_{j+T} (stride sout).
template <bool LAZY>
__global__ void __launch_bounds__(256) sc_round_kernel(const u64* in, u64 sin, u64* out, u64 sout, u64 L, u32 rows,
                                                       ModQ M, const DevState* ds, u32 round, u32 j, u64* sums,
                                                       u32 nr, bool plain) {
  constexpr u32 T = SC_T, G = 1u << T;
  __shared__ Sum128 red[SC_T * 3 * 32];
  const u32 pair = blockIdx.y, rep = pair / rows, k = pair % rows;
  const u64 q = M.q, ng = L / G;
  const u64* x = in + (u64)pair * sin;
  u64* y = out + (u64)pair * sout;
  __shared__ u64 sch[2 * T];
  u64 c[T], cp[T];
  shared_challenges<T>(sch, [&](u32 t) { return nc_challenge(ds, round, rep, j + t, q); }, q, c, cp);
  ScAcc<LAZY> acc[T][3];
#pragma unroll
  for (u32 t = 0; t < T; t++)
#pragma unroll
    for (u32 a = 0; a < 3; a++) acc[t][a].zero();
  for (u64 g = (u64)blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += (u64)gridDim.x * blockDim.x) {
    u64 v[G];
#pragma unroll
    for (u32 m = 0; m < G; m++) v[m] = __ldg(x + g + m * ng);
    group_rounds<LAZY, T>(M, v, c, cp, acc, 0);
    y[g] = v[0];
  }
  ScAcc<LAZY> flat[T * 3];
#pragma unroll
  for (u32 t = 0; t < T; t++)
#pragma unroll
    for (u32 a = 0; a < 3; a++) flat[t * 3 + a] = acc[t][a];
  const u64 r = block_totals<LAZY, T * 3>(M, flat, red);
  if (threadIdx.x < T * 3) {
    const u32 t = threadIdx.x / 3, a = threadIdx.x % 3;
    atomic_add_mod(&sums[((rep * (u64)nr + j + t) * rows + k) * 3 + a], r, q, plain);
  }
}

// One CTA per (rep,row) finishes rounds j0.. from v_{j0} (length L: at most
// SC_TAIL_ONE, or 16 d when norm_check_3's vector is longer),
// reading either a per-pair buffer or (j0 = 0) the witness row itself.
// T rounds of the tail on the vector v (length cur, shared memory): groups of
// 2^T values v[g + m ng] per thread, sums of all T rounds in one block
// reduction, folded values back to v[g] (only thread g touches v[g]).
template <bool LAZY, u32 T>
__device__ __forceinline__ void tail_step(u64* v, u64 cur, const ModQ& M, const DevState* ds, u32 round, u32 rep,
                                          u32 j, u64* sums, u32 nr, u32 rows, u32 k, Sum128* red, u64* sch) {
  constexpr u32 G = 1u << T;
  const u64 q = M.q, ng = cur >> T;
  u64 c[T], cp[T];
  shared_challenges<T>(sch, [&](u32 t) { return nc_challenge(ds, round, rep, j + t, q); }, q, c, cp);
  ScAcc<LAZY> acc[T][3];
#pragma unroll
  for (u32 t = 0; t < T; t++)
#pragma unroll
    for (u32 a = 0; a < 3; a++) acc[t][a].zero();
  for (u64 g = threadIdx.x; g < ng; g += blockDim.x) {
    u64 x[G];
#pragma unroll
    for (u32 m = 0; m < G; m++) x[m] = v[g + m * ng];
    group_rounds<LAZY, T>(M, x, c, cp, acc, 0);
    v[g] = x[0];
  }
  ScAcc<LAZY> flat[T * 3];
#pragma unroll
  for (u32 t = 0; t < T; t++)
#pragma unroll
    for (u32 a = 0; a < 3; a++) flat[t * 3 + a] = acc[t][a];
  const u64 r = block_totals<LAZY, T * 3>(M, flat, red);  // its barriers also publish v
  if (threadIdx.x < T * 3) sums[((rep * (u64)nr + j + threadIdx.x / 3) * rows + k) * 3 + threadIdx.x % 3] = r;
}

template <bool LAZY>
__global__ void __launch_bounds__(512) sc_tail_kernel(const u64* in, u64 sin, RowSet w0, u64 L, u32 rows, ModQ M,
                                                       const DevState* ds, u32 round, u32 j0, u64* sums, u32 nr,
                                                       u32 d, u64* cap) {
  extern __shared__ u64 v[];
  __shared__ Sum128 red[SC_T * 3 * 32];
  __shared__ u64 sch[2 * SC_T];
  const u32 pair = blockIdx.x, rep = pair / rows, k = pair % rows;
  const u64* x = (j0 == 0) ? w0.p[k] : in + (u64)pair * sin;
  const bool nar = j0 == 0 && ((w0.narrow >> k) & 1);
  for (u32 i = threadIdx.x; i < L; i += blockDim.x) v[i] = wres(x, nar, i, M.q);
  __syncthreads();
  u64 cur = L;
  u32 j = j0;
  while (cur > 1) {
    if (cur == d) {
      for (u32 i = threadIdx.x; i < d; i += blockDim.x) cap[(u64)pair * d + i] = v[i];
      __syncthreads();
    }
    // up to four rounds per step, stopping at length d (norm_check_3's vector)
    u32 T = 63u - (u32)__clzll((long long)cur);
    if (cur > d) {
      const u32 td = 63u - (u32)__clzll((long long)(cur / d));
      T = td < T ? td : T;
    }
    T = T < SC_T ? T : SC_T;
    switch (T) {
      case 4: tail_step<LAZY, 4>(v, cur, M, ds, round, rep, j, sums, nr, rows, k, red, sch); break;
      case 3: tail_step<LAZY, 3>(v, cur, M, ds, round, rep, j, sums, nr, rows, k, red, sch); break;
      case 2: tail_step<LAZY, 2>(v, cur, M, ds, round, rep, j, sums, nr, rows, k, red, sch); break;
      default: tail_step<LAZY, 1>(v, cur, M, ds, round, rep, j, sums, nr, rows, k, red, sch); break;
    }
    cur >>= T;
    j += T;
  }
}

// ---------------------------------------------------------------------------
// Batched uneven sumchecks: many independent vectors (one repetition each),
// instance i drawing its challenges from the norm-check stream of
// (round, repetition = i).  Every pass level is one persistent launch over
// equal tiles of all instances still longer than SC_TAIL (a tile = 1024
// groups of 16 elements; the tile -> instance map is a prefix table in shared
// memory), four rounds per pass; a final launch finishes every instance in
// shared memory (one CTA each).
// ---------------------------------------------------------------------------
struct SbInst {
  const u64* in;
  u64* out;
  u64 L;     // current length
  u64 tile0; // first tile of this instance in the level's tile space
  u32 j;     // index of the next round
  u32 id;    // instance index: its challenge stream and its rows of sums
};
constexpr u32 SB_MAX_INST = 64, SB_GPT = 4, SB_TILE_GROUPS = 256 * SB_GPT;

__device__ __forceinline__ u64 sb_challenge(u64 seed, u32 round, u32 inst, u64 j, u64 q) {
  return uni_mod(prf_at(prf_key(seed, domain_id(DOM_NC, round, inst)), j), q);
}

template <bool LAZY>
__global__ void __launch_bounds__(256, 2) sb_pass_kernel(const SbInst* inst, u32 ninst, u64 ntiles, ModQ M,
                                                         u64 seed, u32 round, u64* sums, u32 nrmax, bool plain) {
  constexpr u32 T = SC_T, G = 1u << T;
  __shared__ Sum128 red[SC_T * 3 * 32];
  __shared__ u64 t0s[SB_MAX_INST + 1];
  __shared__ u64 sch[2 * T];
  for (u32 i = threadIdx.x; i <= ninst; i += blockDim.x) t0s[i] = i < ninst ? inst[i].tile0 : ntiles;
  __syncthreads();
  const u64 q = M.q;
  for (u64 tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    u32 lo = 0, hi = ninst;  // t0s[lo] <= tile < t0s[hi]
    while (hi - lo > 1) {
      const u32 mid = (lo + hi) / 2;
      if (t0s[mid] <= tile) lo = mid;
      else hi = mid;
    }
    const SbInst I = inst[lo];
    const u64 ng = I.L / G, gbase = (tile - t0s[lo]) * SB_TILE_GROUPS;
    u64 c[T], cp[T];
    shared_challenges<T>(sch, [&](u32 t) { return sb_challenge(seed, round, I.id, I.j + t, q); }, q, c, cp);
    ScAcc<LAZY> acc[T][3];
#pragma unroll
    for (u32 t = 0; t < T; t++)
#pragma unroll
      for (u32 a = 0; a < 3; a++) acc[t][a].zero();
#pragma unroll 1
    for (u32 x = 0; x < SB_GPT; x++) {
      const u64 g = gbase + x * 256 + threadIdx.x;
      u64 v[G];
#pragma unroll
      for (u32 m = 0; m < G; m++) v[m] = __ldg(I.in + g + m * ng);
      group_rounds<LAZY, T>(M, v, c, cp, acc, 0);
      I.out[g] = v[0];
    }
    ScAcc<LAZY> flat[T * 3];
#pragma unroll
    for (u32 t = 0; t < T; t++)
#pragma unroll
      for (u32 a = 0; a < 3; a++) flat[t * 3 + a] = acc[t][a];
    const u64 r = block_totals<LAZY, T * 3>(M, flat, red);
    if (threadIdx.x < T * 3)
      atomic_add_mod(&sums[((u64)I.id * nrmax + I.j + threadIdx.x / 3) * 3 + threadIdx.x % 3], r, q, plain);
  }
}

template <bool LAZY>
__global__ void __launch_bounds__(1024) sb_tail_kernel(const SbInst* inst, ModQ M, u64 seed, u32 round, u64* sums,
                                                       u32 nrmax) {
  extern __shared__ u64 v[];
  __shared__ Sum128 red[3 * 32];
  __shared__ u64 sch[2];
  const u32 i = blockIdx.x;
  const SbInst I = inst[i];
  const u64 q = M.q;
  for (u64 e = threadIdx.x; e < I.L; e += blockDim.x) v[e] = I.in[e];
  __syncthreads();
  u64 cur = I.L;
  u32 j = I.j;
  while (cur > 1) {
    const u64 h = cur / 2;
    ScAcc<LAZY> a0, a1, a2;
    a0.zero();
    a1.zero();
    a2.zero();
    for (u64 e = threadIdx.x; e < h; e += blockDim.x) {
      const u64 p0 = v[e], p1 = v[e + h];
      a0.mac(M, p0, p0);
      a1.mac(M, p0, p1);
      a2.mac(M, p1, p1);
    }
    ScAcc<LAZY> tri[3] = {a0, a1, a2};
    const u64 r = block_totals<LAZY, 3>(M, tri, red);
    if (threadIdx.x < 3) sums[((u64)i * nrmax + j) * 3 + threadIdx.x] = r;
    if (threadIdx.x == 0) {
      const u64 cv = sb_challenge(seed, round, i, j, q);
      sch[0] = cv;
      sch[1] = shoup_dev(cv, q);
    }
    __syncthreads();
    const u64 c = sch[0], cp = sch[1];
    for (u64 e = threadIdx.x; e < h; e += blockDim.x) v[e] = fold1(v[e], v[e + h], c, cp, q);
    __syncthreads();
    cur = h;
    j++;
  }
}

// polys: instance i's nr_i x 3 block starts at offs[i] * 3
__global__ void sb_finalize_kernel(const u64* sums, const u32* nrs, const u64* offs, u32 ninst, u32 nrmax, u64 q,
                                   u64* claims, u64* polys) {
  const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (u64)ninst * nrmax) return;
  const u32 i = (u32)(t / nrmax), j = (u32)(t % nrmax);
  if (j >= nrs[i]) return;
  const u64* s = sums + t * 3;
  const u64 s00 = s[0] % q, s01 = s[1] % q, s11 = s[2] % q;
  u64* o = polys + (offs[i] + j) * 3;
  o[0] = s00;
  o[1] = sub_mod(s01, s00, q);
  o[2] = add_mod(sub_mod(sub_mod(s11, s01, q), s01, q), s00, q);
  if (j == 0) claims[i] = add_mod(s00, s11, q);
}

// ---------------------------------------------------------------------------
// Norm-check sumcheck over F_{q^2} = F_q[X]/(X^2 - s) (s a quadratic
// non-residue; the QuadraticExtension product of
// src/quadratic_extension.rs:30-58), batched over uneven instances: one
// launch per round level covers every instance that still has rounds, each
// thread folding pairs (v0, v1) -> v0 + c (v1 - v0) with the level's
// challenge while it accumulates the round sums (v0^2, v0 (v1 - v0),
// (v1 - v0)^2); warp shuffles and a shared-memory pass reduce the six words
// per block, which are added to the instance's sums in global memory.
// Round 0 reads the instance's F_q vector; later rounds the pairs written by
// the previous level.  Challenge j of instance i: two PRF words of the
// domain (6, round, i), indices 2j and 2j + 1.
// ---------------------------------------------------------------------------
constexpr u64 DOM_NC2 = 6;

struct Fq2Level {
  const u64* in[SB_MAX_INST];  // level input: F_q words (round 0) or (re, im) pairs
  u64* out[SB_MAX_INST];       // folded (re, im) pairs, half the length
  u64 half[SB_MAX_INST];       // pairs of this level
  u64 start[SB_MAX_INST + 1];  // prefix sums of half
  u32 id[SB_MAX_INST], j[SB_MAX_INST];
  u32 first[SB_MAX_INST];      // 1: input is F_q words
  u32 count;
};

__device__ __forceinline__ void qe_mul_dev(const ModQ& M, u64 s, u64 a0, u64 a1, u64 b0, u64 b1, u64& r0, u64& r1) {
  const u64 t0 = add_mod(mul_mod(M, a0, b0), mul_mod(M, s, mul_mod(M, a1, b1)), M.q);
  const u64 t1 = add_mod(mul_mod(M, a0, b1), mul_mod(M, a1, b0), M.q);
  r0 = t0;
  r1 = t1;
}

__global__ void __launch_bounds__(256) fq2_level_kernel(Fq2Level L, ModQ M, u64 shift, u64 seed, u32 round,
                                                        u64* sums, u32 nrmax) {
  __shared__ u64 red[6][8];
  const u64 q = M.q;
  const u64 total = L.start[L.count];
  // each block works on one instance's contiguous range of pairs
  for (u64 base = (u64)blockIdx.x * blockDim.x; base < total; base += (u64)gridDim.x * blockDim.x) {
    u32 lo = 0, hi = L.count;  // start[lo] <= base < start[hi]
    while (hi - lo > 1) {
      const u32 mid = (lo + hi) / 2;
      if (L.start[mid] <= base) lo = mid;
      else hi = mid;
    }
    const u32 inst = lo;
    const u64 h = L.half[inst];
    const u64 key = prf_key(seed, domain_id(DOM_NC2, round, L.id[inst]));
    const u64 c0 = uni_mod(prf_at(key, 2 * (u64)L.j[inst]), q), c1 = uni_mod(prf_at(key, 2 * (u64)L.j[inst] + 1), q);
    const u64 i = base - L.start[inst] + threadIdx.x;
    u64 f[6] = {0, 0, 0, 0, 0, 0};
    // the block's threads past its instance's end (a block never spans two
    // instances: start[] is a multiple of the block size) add nothing
    if (base - L.start[inst] + threadIdx.x < h) {
      u64 a0, a1, b0, b1;
      if (L.first[inst]) {
        a0 = L.in[inst][i] % q;
        a1 = 0;
        b0 = L.in[inst][h + i] % q;
        b1 = 0;
      } else {
        a0 = L.in[inst][2 * i];
        a1 = L.in[inst][2 * i + 1];
        b0 = L.in[inst][2 * (h + i)];
        b1 = L.in[inst][2 * (h + i) + 1];
      }
      const u64 e0 = sub_mod(b0, a0, q), e1 = sub_mod(b1, a1, q);
      qe_mul_dev(M, shift, a0, a1, a0, a1, f[0], f[1]);
      qe_mul_dev(M, shift, a0, a1, e0, e1, f[2], f[3]);
      qe_mul_dev(M, shift, e0, e1, e0, e1, f[4], f[5]);
      u64 r0, r1;
      qe_mul_dev(M, shift, c0, c1, e0, e1, r0, r1);
      L.out[inst][2 * i] = add_mod(a0, r0, q);
      L.out[inst][2 * i + 1] = add_mod(a1, r1, q);
    }
#pragma unroll
    for (u32 t = 0; t < 6; t++)
      for (int o = 16; o > 0; o >>= 1) f[t] = add_mod(f[t], __shfl_xor_sync(0xffffffffu, f[t], o), q);
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
      for (u32 t = 0; t < 6; t++) red[t][warp] = f[t];
    __syncthreads();
    if (threadIdx.x < 6) {
      u64 acc = 0;
      for (u32 w = 0; w < blockDim.x / 32; w++) acc = add_mod(acc, red[threadIdx.x][w], q);
      if (acc) atomic_add_mod(&sums[((u64)L.id[inst] * nrmax + L.j[inst]) * 6 + threadIdx.x], acc, q, false);
    }
    __syncthreads();
  }
}

__global__ void fq2_claims_kernel(const u64* sums, u32 count, u32 nrmax, u64 q, u64* claims) {
  const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const u64* f = sums + (u64)i * nrmax * 6;  // round 0: real parts f0, f1, f2 at 0, 2, 4
  u64 c = add_mod(f[0], f[0], q);
  c = add_mod(c, add_mod(f[2], f[2], q), q);
  claims[i] = add_mod(c, f[4], q);
}

int launch_sumcheck_fq2_batch(const u64* const* vecs, const u64* lens, u32 count, const ModQ& M, u64 shift,
                              u64 seed, u32 round, u64* claims, u64* polys, u64* scratch, cudaStream_t st) {
  if (count == 0 || count > SB_MAX_INST) return salsaa_set_error(-2, "sumcheck_fq2: 1..64 instances");
  u32 nrmax = 0;
  u64 scr = 0;
  for (u32 i = 0; i < count; i++) {
    if (lens[i] < 2 || (lens[i] & (lens[i] - 1)) || lens[i] > (1ULL << 30) || !vecs[i])
      return salsaa_set_error(-2, "sumcheck_fq2: lengths must be powers of two in 2..2^30");
    const u32 nr = 63u - (u32)__builtin_clzll(lens[i]);
    if (nr > nrmax) nrmax = nr;
    scr += lens[i];  // ping (n/2 pairs) + pong (n/4 pairs): n + n/2 words <= 2n
  }
  (void)scr;
  // sums[(i, j)] : 6 words each, zeroed; polys are written per instance at the end
  u64* sums = scratch;
  cudaError_t e = cudaMemsetAsync(sums, 0, (u64)count * nrmax * 6 * sizeof(u64), st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "sumcheck_fq2: memset");
  u64* pool = sums + (u64)count * nrmax * 6;
  // per instance: buffer A (len pairs / 2 = len words) and buffer B (len / 2 words)
  std::vector<u64*> bufA(count), bufB(count);
  {
    u64 off = 0;
    for (u32 i = 0; i < count; i++) {
      bufA[i] = pool + off;
      off += lens[i];
      bufB[i] = pool + off;
      off += lens[i] / 2;
    }
  }
  const u32 BS = 256;
  for (u32 j = 0; j < nrmax; j++) {
    Fq2Level L{};
    u64 start = 0;
    u32 k = 0;
    for (u32 i = 0; i < count; i++) {
      const u32 nr = 63u - (u32)__builtin_clzll(lens[i]);
      if (j >= nr) continue;
      const u64 half = lens[i] >> (j + 1);
      L.in[k] = j == 0 ? vecs[i] : ((j & 1) ? bufA[i] : bufB[i]);
      L.out[k] = (j & 1) ? bufB[i] : bufA[i];
      L.half[k] = half;
      L.start[k] = start;
      L.id[k] = i;
      L.j[k] = j;
      L.first[k] = j == 0;
      start += (half + BS - 1) / BS * BS;  // block-aligned ranges
      k++;
    }
    L.start[k] = start;
    L.count = k;
    u64 blocks = start / BS;
    if (blocks > 148ULL * 16) blocks = 148ULL * 16;
    fq2_level_kernel<<<(unsigned)blocks, BS, 0, st>>>(L, M, shift, seed, round, sums, nrmax);
    int rc = check_launch("sumcheck_fq2 level");
    if (rc) return rc;
  }
  // claims (2 f0 + 2 f1 + f2 of round 0, real) and the polynomials in order
  u64 po = 0;
  for (u32 i = 0; i < count; i++) {
    const u32 nr = 63u - (u32)__builtin_clzll(lens[i]);
    e = cudaMemcpyAsync(polys + po, sums + (u64)i * nrmax * 6, (u64)nr * 6 * sizeof(u64), cudaMemcpyDeviceToDevice,
                        st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "sumcheck_fq2: polys");
    po += (u64)nr * 6;
  }
  fq2_claims_kernel<<<(count + 63) / 64, 64, 0, st>>>(sums, count, nrmax, M.q, claims);
  return check_launch("sumcheck_fq2 claims");
}

int launch_sumcheck_batch(const u64* const* vecs, const u64* lens, u32 count, const ModQ& M, u64 seed, u32 round,
                          u64* claims, u64* polys, cudaStream_t st) {
  if (count == 0) return 0;
  if (count > SB_MAX_INST) return salsaa_set_error(-2, "sumcheck_batch: at most 64 instances");
  u32 nrmax = 0;
  std::vector<u32> nrs(count);
  std::vector<u64> offs(count);
  u64 tot_a = 0, tot_b = 0, off = 0, max_tiles = 0;
  for (u32 i = 0; i < count; i++) {
    const u64 L = lens[i];
    if (!vecs[i] || L < 2 || (L & (L - 1)) || L > (1ULL << 30))
      return salsaa_set_error(-2, "sumcheck_batch: lengths must be powers of two in 2..2^30");
    nrs[i] = 63u - (u32)__builtin_clzll(L);
    nrmax = nrs[i] > nrmax ? nrs[i] : nrmax;
    offs[i] = off;
    off += nrs[i];
    if (L > SC_TAIL) {
      tot_a += L / 16;
      tot_b += L / 256;
      const u64 tiles = L / 16 / SB_TILE_GROUPS;
      max_tiles = tiles > max_tiles ? tiles : max_tiles;
    }
  }
  const bool lazy = M.q < (1ULL << 50);
  const bool plain = lazy && max_tiles < (1ULL << 13);
  // device scratch: sums, two ping-pong areas, descriptors, nrs / offs
  const u32 maxlev = 8;  // 16^8 > 2^30
  const u64 desc_bytes = (u64)(maxlev + 1) * SB_MAX_INST * sizeof(SbInst);
  u64 *sums = nullptr, *bufa = nullptr, *bufb = nullptr, *doffs = nullptr;
  SbInst* ddesc = nullptr;
  u32* dnrs = nullptr;
  auto alloc = [&](void** p, u64 bytes) {
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, st);
    return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "sumcheck_batch: workspace");
  };
  struct Guard {
    std::vector<void*> v;
    cudaStream_t s;
    ~Guard() {
      for (void* p : v) cudaFreeAsync(p, s);
    }
  } guard{{}, st};
  int rc = 0;
  if ((rc = alloc((void**)&sums, (u64)count * nrmax * 3 * 8))) return rc;
  guard.v.push_back(sums);
  if ((rc = alloc((void**)&bufa, tot_a * 8))) return rc;
  guard.v.push_back(bufa);
  if ((rc = alloc((void**)&bufb, tot_b * 8))) return rc;
  guard.v.push_back(bufb);
  if ((rc = alloc((void**)&ddesc, desc_bytes))) return rc;
  guard.v.push_back(ddesc);
  if ((rc = alloc((void**)&dnrs, count * 4))) return rc;
  guard.v.push_back(dnrs);
  if ((rc = alloc((void**)&doffs, count * 8))) return rc;
  guard.v.push_back(doffs);
  cudaError_t e = cudaMemsetAsync(sums, 0, (u64)count * nrmax * 3 * 8, st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "sumcheck_batch: memset");
  // host plan: per level, the instances still longer than SC_TAIL, then the tail
  std::vector<SbInst> plan((maxlev + 1) * SB_MAX_INST);
  std::vector<u32> lev_n;
  std::vector<u64> lev_tiles;
  std::vector<const u64*> cur_in(vecs, vecs + count);
  std::vector<u64> cur_L(lens, lens + count);
  std::vector<u32> cur_j(count, 0);
  std::vector<u64> oa(count), ob(count);
  {
    u64 ta = 0, tb = 0;
    for (u32 i = 0; i < count; i++) {
      oa[i] = ta;
      ob[i] = tb;
      if (lens[i] > SC_TAIL) {
        ta += lens[i] / 16;
        tb += lens[i] / 256;
      }
    }
  }
  for (u32 lev = 0; lev < maxlev; lev++) {
    u64 tiles = 0;
    u32 n = 0;
    for (u32 i = 0; i < count; i++) {
      if (cur_L[i] <= SC_TAIL) continue;
      SbInst I{};
      I.in = cur_in[i];
      I.out = (lev % 2 == 0) ? bufa + oa[i] : bufb + ob[i];
      I.L = cur_L[i];
      I.tile0 = tiles;
      I.j = cur_j[i];
      I.id = i;
      plan[lev * SB_MAX_INST + n++] = I;
      tiles += cur_L[i] / 16 / SB_TILE_GROUPS;
      cur_in[i] = I.out;
      cur_L[i] /= 16;
      cur_j[i] += SC_T;
    }
    if (!n) break;
    lev_n.push_back(n);
    lev_tiles.push_back(tiles);
  }
  const u32 nlev = (u32)lev_n.size();
  u64 tail_max = 0;
  for (u32 i = 0; i < count; i++) {
    SbInst I{};
    I.in = cur_in[i];
    I.L = cur_L[i];
    I.j = cur_j[i];
    I.id = i;
    plan[maxlev * SB_MAX_INST + i] = I;
    tail_max = cur_L[i] > tail_max ? cur_L[i] : tail_max;
  }
  e = cudaMemcpyAsync(ddesc, plan.data(), desc_bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dnrs, nrs.data(), count * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(doffs, offs.data(), count * 8, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "sumcheck_batch: plan");
  // (from pageable memory the copies are staged before cudaMemcpyAsync returns)
  for (u32 lev = 0; lev < nlev; lev++) {
    const u64 grid = lev_tiles[lev] < 296 ? lev_tiles[lev] : 296;
    if (lazy)
      sb_pass_kernel<true><<<(unsigned)grid, 256, 0, st>>>(ddesc + lev * SB_MAX_INST, lev_n[lev], lev_tiles[lev],
                                                            M, seed, round, sums, nrmax, plain);
    else
      sb_pass_kernel<false><<<(unsigned)grid, 256, 0, st>>>(ddesc + lev * SB_MAX_INST, lev_n[lev],
                                                             lev_tiles[lev], M, seed, round, sums, nrmax, plain);
    if ((rc = check_launch("sb_pass"))) return rc;
  }
  const size_t smem = tail_max * sizeof(u64);
  auto tail = lazy ? sb_tail_kernel<true> : sb_tail_kernel<false>;
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "sumcheck_batch: tail smem");
  }
  tail<<<count, 1024, smem, st>>>(ddesc + maxlev * SB_MAX_INST, M, seed, round, sums, nrmax);
  if ((rc = check_launch("sb_tail"))) return rc;
  const u64 tot = (u64)count * nrmax;
  sb_finalize_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(sums, dnrs, doffs, count, nrmax, M.q, claims,
                                                                   polys);
  return check_launch("sb_finalize");
}

// Round polynomials and claims from the raw sums, canonical mod q.// Round polynomials and claims from the raw sums, canonical mod q.
__global__ void sc_finalize_kernel(const u64* sums, u32 rows, u32 nr, u64 q, u64* claims, u64* polys0,
                                   u64* polys1) {
  u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2ULL * nr * rows) return;
  const u32 rep = (u32)(t / ((u64)nr * rows));
  const u64 jk = t % ((u64)nr * rows);
  const u64* s = sums + t * 3;
  const u64 s00 = s[0] % q, s01 = s[1] % q, s11 = s[2] % q;
  const u64 f0 = s00, f1 = sub_mod(s01, s00, q);
  const u64 f2 = add_mod(sub_mod(sub_mod(s11, s01, q), s01, q), s00, q);
  u64* o = (rep ? polys1 : polys0) + jk * 3;
  o[0] = f0;
  o[1] = f1;
  o[2] = f2;
  if (rep == 0 && jk < rows) claims[jk] = add_mod(s00, s11, q);  // round 0: sum of squares
}

template <bool LAZY>
static int sumcheck_passes(RowSet w, u32 rows, u64 nlen, u32 d, const ModQ& M, const DevState* ds, u32 round,
                           SumcheckBufs B, u32 nr, bool plain, cudaStream_t st) {
  const u64 sa = nlen / 2, sb = nlen / 4;  // strides of the two ping-pong buffers
  u64 L = nlen;
  u32 j = 0;
  const u64* in = nullptr;
  u64 sin = 0;
  bool to_a = true;
  auto grid_for = [](u64 groups, u32 pairs) {
    // one resident wave in total (two CTAs per SM): few CTAs, each streaming
    // many groups, so the per-CTA reductions stay a small share
    u64 want = (148ULL * 2 + pairs - 1) / pairs;
    u64 g = (groups + 255) / 256;
    return (unsigned)(g < want ? (g ? g : 1) : want);
  };
  auto pass_ok = [d](u64 len) { return len > SC_TAIL_ONE && (len >> SC_T) >= d; };
  if (pass_ok(L)) {
    // rounds 0..3 on the tensor cores when the shapes allow; the CUDA-core
    // pass then runs only if a witness value did not fit the byte limbs
    const bool tc = B.gram && nc_gram_ok(w, rows, L, M.q);
    const u32* flag = tc ? (const u32*)(B.gram + (u64)rows * 256) : nullptr;
    int rc = 0;
    if (tc && (rc = launch_nc_gram(w, rows, L, M, ds, round, B.a, sa, B.gram, plain, st))) return rc;
    dim3 g(2 * grid_for(L / (1u << SC_T), 2 * rows), rows);
    sc_first_kernel<LAZY><<<g, 256, 0, st>>>(w, rows, L, M, ds, round, B.a, sa, B.sums, nr, plain, flag);
    rc = check_launch("sc_first");
    if (rc) return rc;
    if (tc && (rc = launch_nc_gram_sums(B.gram, rows, M, ds, round, B.sums, nr, plain, st))) return rc;
    in = B.a;
    sin = sa;
    to_a = false;
    L >>= SC_T;
    j = SC_T;
    while (pass_ok(L)) {
      u64* out = to_a ? B.a : B.b;
      const u64 so = to_a ? sa : sb;
      dim3 gr(grid_for(L / (1u << SC_T), 2 * rows), 2 * rows);
      sc_round_kernel<LAZY><<<gr, 256, 0, st>>>(in, sin, out, so, L, rows, M, ds, round, j, B.sums, nr, plain);
      rc = check_launch("sc_round");
      if (rc) return rc;
      in = out;
      sin = so;
      to_a = !to_a;
      L >>= SC_T;
      j += SC_T;
    }
  }
  const size_t smem = L * sizeof(u64);
  auto kern = sc_tail_kernel<LAZY>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "sc_tail smem attribute");
  }
  kern<<<2 * rows, 512, smem, st>>>(in, sin, w, L, rows, M, ds, round, j, B.sums, nr, d, B.cap);
  return check_launch("sc_tail");
}

int launch_sumcheck(RowSet w, u32 rows, u64 nlen, u32 d, const ModQ& M, const DevState* ds, u32 round,
                    SumcheckBufs B, u64* proof_claims, u64* proof_rep0, u64* proof_rep1, cudaStream_t st) {
  if (nlen < 4 || (nlen & (nlen - 1)) || rows == 0 || rows > MAX_WROWS || nlen < d)
    return salsaa_set_error(-2, "sumcheck: bad shape");
  const u32 nr = 63u - (u32)__builtin_clzll(nlen);
  const bool lazy = M.q < (1ULL << 50);
  // the lazy per-thread / per-block sums stay far below 2^128; with fewer than
  // 2^13 contributions per address the plain 64-bit atomics cannot overflow
  const bool plain = lazy;
  cudaError_t e = cudaMemsetAsync(B.sums, 0, 2ULL * nr * rows * 3 * sizeof(u64), st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "sumcheck memset");
  int rc = lazy ? sumcheck_passes<true>(w, rows, nlen, d, M, ds, round, B, nr, plain, st)
                : sumcheck_passes<false>(w, rows, nlen, d, M, ds, round, B, nr, plain, st);
  if (rc) return rc;
  u64 tot = 2ULL * nr * rows;
  sc_finalize_kernel<<<(unsigned)((tot + 127) / 128), 128, 0, st>>>(B.sums, rows, nr, M.q, proof_claims,
                                                                    proof_rep0, proof_rep1);
  return check_launch("sc_finalize");
}

// ---------------------------------------------------------------------------
// norm_check_3 (src/subroutines/fast_norm_check.rs:401-441).  The statement
// row is tensor(cs[0..K]) (x) base with base = conj(tensor(cs[K..nr])), so
// <row, w_k> = base * (the sumcheck vector after K = nr - log2 d rounds).
// One CTA per (rep, row) computes base, both NTTs and the product; the
// repetition's base (slot form) is kept for later commitments.
// ---------------------------------------------------------------------------
__device__ void blk_ntt(u64* a, u32 units, const NttDev& T, bool inverse) {
  const u32 n = T.n, logn = T.logn, half = n >> 1, loghalf = logn - 1;
  const u32 nbf = units << loghalf;
  const u64 q = T.q;
  if (!inverse) {
    u32 logt = logn;
    for (u32 m = 1; m < n; m <<= 1) {
      logt--;
      const u32 t = 1u << logt;
      for (u32 b = threadIdx.x; b < nbf; b += blockDim.x) {
        const u32 u = b >> loghalf, r = b & (half - 1), i = r >> logt, jj = r & (t - 1);
        const u32 j = (u << logn) + (i << (logt + 1)) + jj;
        const u64 U = a[j], V = mul_shoup(a[j + t], T.fwd[m + i], T.fwdp[m + i], q);
        a[j] = add_mod(U, V, q);
        a[j + t] = sub_mod(U, V, q);
      }
      __syncthreads();
    }
  } else {
    u32 logt = 0;
    for (u32 m = n; m > 1; m >>= 1) {
      const u32 h = m >> 1, t = 1u << logt;
      for (u32 b = threadIdx.x; b < nbf; b += blockDim.x) {
        const u32 u = b >> loghalf, r = b & (half - 1), i = r >> logt, jj = r & (t - 1);
        const u32 j = (u << logn) + (i << (logt + 1)) + jj;
        const u64 U = a[j], V = a[j + t];
        a[j] = add_mod(U, V, q);
        a[j + t] = mul_shoup(sub_mod(U, V, q), T.inv[h + i], T.invp[h + i], q);
      }
      logt++;
      __syncthreads();
    }
    for (u32 t = threadIdx.x; t < units * n; t += blockDim.x) a[t] = mul_shoup(a[t], T.ninv, T.ninvp, q);
    __syncthreads();
  }
}

__global__ void norm3_kernel(const u64* cap, u32 rows, u32 nr, NttDev T, ModQ M, const DevState* ds, u32 round,
                             u64* rhs0, u64* rhs1, u64* base0, u64* base1) {
  extern __shared__ u64 sm[];
  const u32 n = T.n, d = 2 * n, logd = T.logn + 1;
  const u32 pair = blockIdx.x, rep = pair / rows, k = pair % rows;
  const u64 q = M.q;
  const u32 K = nr - logd;
  u64* ext = sm;          // d
  u64* bs = sm + d;       // d: base, slot layout after NTT
  u64* vs = sm + 2 * d;   // d: vector, slot layout after NTT
  for (u32 i = threadIdx.x; i < d; i += blockDim.x) {
    u64 v = 1 % q;
    for (u32 b = 0; b < logd; b++) {
      const u64 c = nc_challenge(ds, round, rep, K + b, q);
      const u32 bit = (i >> (logd - 1 - b)) & 1;
      v = mul_mod(M, v, bit ? c : sub_mod(1 % q, c, q));
    }
    ext[i] = v;
  }
  __syncthreads();
  // conjugate, then de-interleave into [even | odd] for the incomplete NTT
  for (u32 i = threadIdx.x; i < d; i += blockDim.x) {
    u64 cv = (i == 0) ? ext[0] : (ext[d - i] == 0 ? 0 : q - ext[d - i]);
    bs[(i & 1) * n + (i >> 1)] = cv;
    vs[(i & 1) * n + (i >> 1)] = cap[(u64)pair * d + i];
  }
  __syncthreads();
  blk_ntt(bs, 2, T, false);
  blk_ntt(vs, 2, T, false);
  if (k == 0) {
    u64* bo = rep ? base1 : base0;
    for (u32 i = threadIdx.x; i < d; i += blockDim.x) bo[i] = bs[i];
  }
  for (u32 s = threadIdx.x; s < n; s += blockDim.x) {
    u64 e, o;
    slot_mul(M, bs[s], bs[n + s], vs[s], vs[n + s], T.zeta[s], e, o);
    ext[s] = e;
    ext[n + s] = o;
  }
  __syncthreads();
  blk_ntt(ext, 2, T, true);
  u64* out = (rep ? rhs1 : rhs0) + (u64)k * d;
  for (u32 i = threadIdx.x; i < d; i += blockDim.x) out[i] = ext[(i & 1) * n + (i >> 1)];
}

int launch_norm3(const u64* cap, u32 rows, u32 nr, const NttDev& T, const ModQ& M, const DevState* ds,
                 u32 round, u64* proof_rep0, u64* proof_rep1, u64* base0, u64* base1, cudaStream_t st) {
  const u32 d = 2 * T.n;
  const size_t smem = 3ULL * d * sizeof(u64);
  norm3_kernel<<<2 * rows, d < 256 ? d : 256, smem, st>>>(cap, rows, nr, T, M, ds, round, proof_rep0, proof_rep1,
                                                          base0, base1);
  return check_launch("norm3");
}

// ---------------------------------------------------------------------------
// Decomposition (decompose_matrix_by_chunks, src/arithmetic.rs:1572-1593):
// centre-lift, global bit width of the positive and negative parts, radix
// 2^ceil(bw/parts), digit_c = ((pos >> c*rlog) & mask) - ((neg >> c*rlog) & mask),
// output row index = row*parts + c.  The OR and the radix stay on the device.
// ---------------------------------------------------------------------------
__global__ void decomp_or_kernel(RowSet in, u32 rows, u64 per_row, u64 q, u64* bw_or) {
  u64 acc = 0;
  for (u32 k = 0; k < rows; k++) {
    const u64* x = in.p[k];
    for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < per_row; t += (u64)gridDim.x * blockDim.x) {
      const u64 v = x[t];
      acc |= (v * 2 > q) ? q - v : v;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc |= __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicOr((unsigned long long*)bw_or, (unsigned long long)acc);
}

__device__ __forceinline__ u32 radix_log_of(u64 orv, u32 parts) {
  const u32 bw = orv ? 64u - (u32)__clzll((long long)orv) : 0u;
  return (bw + parts - 1) / parts;
}

__global__ void decomp_digits_kernel(RowSet in, u32 rows, u64 per_row, u64 q, u32 parts, DevState* ds, u32 didx,
                                     u64* out, u64* proof_radix) {
  const u32 rlog = radix_log_of(ds->bw_or[didx], parts);
  const u64 mask = (rlog >= 64) ? ~0ULL : ((1ULL << rlog) - 1);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ds->rlog[didx] = rlog;
    if (proof_radix) *proof_radix = 1ULL << rlog;
  }
  for (u32 k = 0; k < rows; k++) {
    const u64* x = in.p[k];
    for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < per_row; t += (u64)gridDim.x * blockDim.x) {
      const u64 v = x[t];
      u64 pos = 0, neg = 0;
      if (v * 2 > q) neg = q - v;
      else pos = v;
      for (u32 c = 0; c < parts; c++) {
        const u32 sh = rlog * c;
        const u64 pd = (sh >= 64) ? 0 : ((pos >> sh) & mask);
        const u64 nd = (sh >= 64) ? 0 : ((neg >> sh) & mask);
        out[((u64)k * parts + c) * per_row + t] = sub_mod(pd, nd, q);
      }
    }
  }
}

int launch_decompose(RowSet in, u32 rows, u64 width, u32 d, u64 q, u32 parts, u32 didx, DevState* ds, u64* out,
                     u64* proof_radix, cudaStream_t st, bool mag_ready) {
  if (parts < 1 || didx >= 16) return salsaa_set_error(-2, "decompose: bad arguments");
  if (in.narrow) return salsaa_set_error(-2, "decompose: source rows must be canonical words");
  const u64 per_row = width * d;
  int rc = 0;
  if (!mag_ready) {
    cudaError_t e = cudaMemsetAsync(&ds->bw_or[didx], 0, sizeof(u64), st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "decompose memset");
    decomp_or_kernel<<<grid_1d(per_row, 256), 256, 0, st>>>(in, rows, per_row, q, &ds->bw_or[didx]);
    rc = check_launch("decomp_or");
    if (rc) return rc;
  }
  decomp_digits_kernel<<<grid_1d(per_row, 256), 256, 0, st>>>(in, rows, per_row, q, parts, ds, didx, out,
                                                                proof_radix);
  return check_launch("decomp_digits");
}

int launch_decompose_ntt(RowSet in, u32 rows, u64 width, u32 d, u64 q, u32 parts, u32 didx, DevState* ds,
                         u64* out, u64* out_slot, u64* proof_radix, const NttDev& T, cudaStream_t st,
                         bool mag_ready, bool* narrow_out) {
  if (parts < 1 || didx >= 16) return salsaa_set_error(-2, "decompose: bad arguments");
  if (in.narrow) return salsaa_set_error(-2, "decompose: source rows must be canonical words");
  if (narrow_out) *narrow_out = false;
  if (!ntt_digits_ok(out, out_slot, rows, T) || rows > MAX_WROWS || d != 2 * T.n) {
    const int rc = launch_decompose(in, rows, width, d, q, parts, didx, ds, out, proof_radix, st, mag_ready);
    if (rc) return rc;
    return ntt_launch(out, out_slot, (u64)rows * parts * width, T, true, false, st);
  }
  if (!mag_ready) {
    cudaError_t e = cudaMemsetAsync(&ds->bw_or[didx], 0, sizeof(u64), st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "decompose memset");
    decomp_or_kernel<<<grid_1d(width * d, 256), 256, 0, st>>>(in, rows, width * d, q, &ds->bw_or[didx]);
    int rc = check_launch("decomp_or");
    if (rc) return rc;
  }
  NttSrcRows src{};
  for (u32 k = 0; k < rows; k++) src.p[k] = in.p[k];
  // with two or more parts the digits are below 2^25: coefficient form as int32
  const bool narrow = narrow_out != nullptr && parts >= 2;
  const int rc = ntt_digits_launch(src, rows, width, parts, &ds->bw_or[didx], &ds->rlog[didx], proof_radix, out,
                                   out_slot, T, st, narrow);
  if (!rc && narrow_out) *narrow_out = narrow;
  return rc;
}

// ---------------------------------------------------------------------------
// Projection (src/subroutines/project.rs:26-103).  J is 256 x cw with
// entries 0 (is_zero), +1 (sign) or -1, drawn from the PRF.  Stored as two
// bit masks per output row; cj[l] = sum_k J[k][l] feeds batch_projections.
// ---------------------------------------------------------------------------
constexpr u32 PROJ_H = 256;

__global__ void proj_tables_kernel(const DevState* ds, u32 round, u32 cw, u32* pos_mask, u32* neg_mask,
                                   int8_t* J, int8_t* Jc) {
  const u32 words = cw / 32;
  u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (u64)PROJ_H * words) return;
  const u32 k = (u32)(t / words), w = (u32)(t % words);
  const u64 key = prf_key(ds->seed, domain_id(DOM_PROJ, round, 0));
  u32 pm = 0, nm = 0;
  for (u32 b = 0; b < 32; b++) {
    const u64 r = prf_at(key, (u64)k * cw + w * 32 + b);
    const u32 iz = r & 1, sg = (r >> 1) & 1;
    if (!iz) {
      if (sg) pm |= 1u << b;
      else nm |= 1u << b;
    }
    const int8_t v = iz ? 0 : (sg ? 1 : -1);
    if (J) J[(u64)k * cw + w * 32 + b] = v;
    if (Jc) {  // (chunk, half, 16-byte slice, row in half, byte)
      const u32 l = w * 32 + b, cc = l / 128, sl = (l % 128) / 16, h = k / 128, r = k % 128;
      Jc[((((u64)cc * 2 + h) * 8 + sl) * 128 + r) * 16 + (l % 16)] = v;
    }
  }
  pos_mask[t] = pm;
  neg_mask[t] = nm;
}

// cj[l] = sum_k J[k][l]: one CTA per 32 columns (one mask word), 32 x 32
// threads, thread (x, y) summing rows y, y + 32, ... of column x.
__global__ void __launch_bounds__(1024) proj_cj_kernel(u32 cw, const u32* pos_mask, const u32* neg_mask, u64* cj,
                                                       u64 q) {
  __shared__ int part[32][33];
  const u32 x = threadIdx.x & 31, y = threadIdx.x >> 5, wd = blockIdx.x, words = cw / 32;
  int v = 0;
  for (u32 k = y; k < PROJ_H; k += 32) {
    v += (pos_mask[(u64)k * words + wd] >> x) & 1;
    v -= (neg_mask[(u64)k * words + wd] >> x) & 1;
  }
  part[y][x] = v;
  __syncthreads();
  if (y == 0) {
    int t = 0;
    for (u32 r = 0; r < 32; r++) t += part[r][x];
    cj[wd * 32 + x] = t >= 0 ? (u64)t % q : q - ((u64)(-t) % q);
  }
}

int launch_proj_tables(const DevState* ds, u32 round, u32 cw, u32* pos_mask, u32* neg_mask, int8_t* J, u64* cj,
                       u64 q, cudaStream_t st, int8_t* Jc) {
  if (cw % 32) return salsaa_set_error(-2, "project: chunk width must be a multiple of 32");
  if (Jc && cw % 128) Jc = nullptr;
  u64 tot = (u64)PROJ_H * (cw / 32);
  proj_tables_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(ds, round, cw, pos_mask, neg_mask, J, Jc);
  int rc = check_launch("proj_tables");
  if (rc) return rc;
  if (cj) {
    proj_cj_kernel<<<cw / 32, 1024, 0, st>>>(cw, pos_mask, neg_mask, cj, q);
    rc = check_launch("proj_cj");
  }
  return rc;
}

// One CTA per (chunk, tile of KT outputs); one thread per coefficient.
// With q < 2^52 the +-1 sums (cw terms of value < q, negatives as q - w) fit
// in 64 bits and are reduced once.
template <int KT, bool LAZY>
__global__ void project_kernel(RowSet in, u64 width, u32 d, u64 q, u32 cw, u64 nch, const u32* pos_mask,
                               const u32* neg_mask, u64* out, const u64* gate) {
  extern __shared__ u32 msk[];  // KT x words (pos), then KT x words (neg)
  if (gate && *(volatile const u64*)gate == 0) return;  // the tensor-core pass was exact
  const u32 words = cw / 32;
  const u64 idx = blockIdx.x;
  const u32 i = (u32)(idx / nch);
  const u64 j = idx % nch;
  const u32 k0 = blockIdx.y * KT;
  for (u32 t = threadIdx.x; t < KT * words; t += blockDim.x) {
    const u32 kk = t / words, w = t % words;
    msk[t] = pos_mask[(u64)(k0 + kk) * words + w];
    msk[KT * words + t] = neg_mask[(u64)(k0 + kk) * words + w];
  }
  __syncthreads();
  const u32 pos = threadIdx.x;
  if (pos >= d) return;
  const bool nar = (in.narrow >> i) & 1;
  const u64* chunk = row_advance(in.p[i], nar, (j * cw) * d);
  u64 acc[KT];
#pragma unroll
  for (int kk = 0; kk < KT; kk++) acc[kk] = 0;
  for (u32 w = 0; w < words; w++) {
    u32 pm[KT], nm[KT];
#pragma unroll
    for (int kk = 0; kk < KT; kk++) {
      pm[kk] = msk[kk * words + w];
      nm[kk] = msk[KT * words + kk * words + w];
    }
    for (u32 b = 0; b < 32; b++) {
      const u64 x = wres(chunk, nar, (u64)(w * 32 + b) * d + pos, q);
      const u64 nx = x ? q - x : 0;
#pragma unroll
      for (int kk = 0; kk < KT; kk++) {
        u64 v = ((pm[kk] >> b) & 1) ? x : 0;
        v = ((nm[kk] >> b) & 1) ? nx : v;
        if (LAZY) acc[kk] += v;
        else acc[kk] = add_mod(acc[kk], v, q);
      }
    }
  }
#pragma unroll
  for (int kk = 0; kk < KT; kk++) out[((idx * PROJ_H) + k0 + kk) * d + pos] = LAZY ? acc[kk] % q : acc[kk];
}

// Tensor-core projection: per chunk, OUT (256 x d) = J (256 x cw) * W (cw x d)
// with W centre-lifted to int8, as mma.sync m16n8k32 s8 x s8 -> s32 tiles.
// A CTA owns 128 outputs x 128 coefficient positions of one chunk; 8 warps in
// a 4 x 2 grid of 32 x 64 warp tiles.  Shared-memory stages hold 128 columns
// of J (row-major, l contiguous) and the transposed witness tile (l
// contiguous per position), both with a 144-byte row stride so that the
// fragment loads of a warp hit 32 distinct banks.
constexpr u32 PJ_KS = 128, PJ_LD = 144, PJ_BM = 128, PJ_BN = 128;

__device__ __forceinline__ void mma_s8_16832(int (&c)[4], u32 a0, u32 a1, u32 a2, u32 a3, u32 b0, u32 b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__global__ void __launch_bounds__(256, 2) project_mma_kernel(RowSet in, u32 d, u64 q, u32 cw, u64 nch,
                                                             const int8_t* __restrict__ J, u64* __restrict__ out,
                                                             u64* flag) {
  __shared__ __align__(16) int8_t As[PJ_BM * PJ_LD];
  __shared__ __align__(16) int8_t Bs[PJ_BN * PJ_LD];
  const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32 g = lane >> 2, t4 = lane & 3;
  const u32 wm = warp & 3, wn = warp >> 2;
  const u32 mhalf = blockIdx.x & 1, nblk = blockIdx.x >> 1;
  const u64 idx = blockIdx.y;
  const u32 i = (u32)(idx / nch);
  const u64 j = idx % nch;
  const bool nar = (in.narrow >> i) & 1;
  const u64* chunk = row_advance(in.p[i], nar, (j * cw) * d + (u64)nblk * PJ_BN);
  const u32 k0 = mhalf * PJ_BM;
  const u64 half_q = q >> 1;
  int acc[2][8][4];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 8; b++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[a][b][c] = 0;
  bool bad = false;
  for (u32 l0 = 0; l0 < cw; l0 += PJ_KS) {
    for (u32 v = tid; v < PJ_BM * PJ_KS / 16; v += 256) {
      const u32 row = v >> 3, c16 = v & 7;
      *(int4*)&As[row * PJ_LD + c16 * 16] = *(const int4*)&J[(u64)(k0 + row) * cw + l0 + c16 * 16];
    }
    for (u32 t = tid; t < PJ_BN * (PJ_KS / 4); t += 256) {
      const u32 pos = t & (PJ_BN - 1), l4 = t >> 7;
      u32 packed = 0;
#pragma unroll
      for (u32 e = 0; e < 4; e++) {
        const u64 v = wres(chunk, nar, (u64)(l0 + l4 * 4 + e) * d + pos, q);
        long long c = v > half_q ? (long long)v - (long long)q : (long long)v;
        if (c < -128 || c > 127) {
          bad = true;
          c = 0;
        }
        packed |= ((u32)c & 0xffu) << (8 * e);
      }
      *(u32*)&Bs[pos * PJ_LD + l4 * 4] = packed;
    }
    __syncthreads();
#pragma unroll
    for (u32 kk = 0; kk < PJ_KS; kk += 32) {
      u32 a[2][4], b[8][2];
#pragma unroll
      for (int mt = 0; mt < 2; mt++) {
        const u32 r0 = wm * 32 + mt * 16 + g;
        a[mt][0] = *(const u32*)&As[r0 * PJ_LD + kk + t4 * 4];
        a[mt][1] = *(const u32*)&As[(r0 + 8) * PJ_LD + kk + t4 * 4];
        a[mt][2] = *(const u32*)&As[r0 * PJ_LD + kk + 16 + t4 * 4];
        a[mt][3] = *(const u32*)&As[(r0 + 8) * PJ_LD + kk + 16 + t4 * 4];
      }
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        const u32 c0 = wn * 64 + nt * 8 + g;
        b[nt][0] = *(const u32*)&Bs[c0 * PJ_LD + kk + t4 * 4];
        b[nt][1] = *(const u32*)&Bs[c0 * PJ_LD + kk + 16 + t4 * 4];
      }
#pragma unroll
      for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
          mma_s8_16832(acc[mt][nt], a[mt][0], a[mt][1], a[mt][2], a[mt][3], b[nt][0], b[nt][1]);
    }
    __syncthreads();
  }
  if (bad) atomicOr((unsigned long long*)flag, 1ULL);
#pragma unroll
  for (int mt = 0; mt < 2; mt++)
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const u32 row = k0 + wm * 32 + mt * 16 + g + 8 * h;
        const u32 col = nblk * PJ_BN + wn * 64 + nt * 8 + t4 * 2;
        u64* dst = out + ((idx * PROJ_H) + row) * d + col;
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int v = acc[mt][nt][h * 2 + e];
          dst[e] = v >= 0 ? (u64)v : q - (u64)(-(long long)v);
        }
      }
}

int launch_project(RowSet in, u32 rows, u64 width, u32 d, u64 q, const u32* pos_mask, const u32* neg_mask,
                   const int8_t* J, DevState* ds, u64* out, cudaStream_t st, const int8_t* Jc) {
  const u32 cw = rows * PROJ_H;
  if (rows == 0 || rows > MAX_WROWS || cw > width || width % cw)
    return salsaa_set_error(-3, "project: chunk width exceeds witness width");
  if (d > 1024) return salsaa_set_error(-2, "project: ring degree too large");
  const u64 nch = width / cw;
  if ((u64)rows * nch > 65535) return salsaa_set_error(-2, "project: too many chunks");
  const u64* gate = nullptr;
  if (Jc && ds && d % 128 == 0 && cw % 128 == 0 && rowset_aligned(in, rows, 16, 8)) {
    cudaError_t e = cudaMemsetAsync(&ds->proj_flag, 0, sizeof(u64), st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "project memset");
    int rc = launch_project_umma(in, rows, nch, d, q, cw, Jc, out, &ds->proj_flag, st);
    if (rc) return rc;
    gate = &ds->proj_flag;
  } else if (J && ds && d % PJ_BN == 0 && cw % PJ_KS == 0) {
    cudaError_t e = cudaMemsetAsync(&ds->proj_flag, 0, sizeof(u64), st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "project memset");
    dim3 gm(2 * (d / PJ_BN), (unsigned)(rows * nch));
    project_mma_kernel<<<gm, 256, 0, st>>>(in, d, q, cw, nch, J, out, &ds->proj_flag);
    int rc = check_launch("project_mma");
    if (rc) return rc;
    gate = &ds->proj_flag;
  }
  constexpr int KT = 16;
  dim3 g((unsigned)(rows * nch), PROJ_H / KT);
  const size_t smem = 2ULL * KT * (cw / 32) * sizeof(u32);
  const bool lazy = q < (1ULL << 52) && cw <= 4096;
  if (lazy) project_kernel<KT, true><<<g, d, smem, st>>>(in, width, d, q, cw, nch, pos_mask, neg_mask, out, gate);
  else project_kernel<KT, false><<<g, d, smem, st>>>(in, width, d, q, cw, nch, pos_mask, neg_mask, out, gate);
  return check_launch("project");
}

// ---------------------------------------------------------------------------
// Fold (src/subroutines/fold.rs:22-27,70-75): ternary ring challenges
// (random_biased: q-1, 0, 1 uniformly) and new_w[i] = sum_k w_k[i] * c_k.
// ---------------------------------------------------------------------------
__global__ void fold_chal_kernel(const DevState* ds, u32 round, u32 rows, u32 d, u64 q, u64* c) {
  u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (u64)rows * d) return;
  const u64 r = prf_at(prf_key(ds->seed, domain_id(DOM_FOLD, round, 0)), t);
  const u64 v = __umul64hi(r, 3);
  c[t] = v == 0 ? q - 1 : (v == 1 ? 0 : 1);
}

int launch_fold_challenge(const DevState* ds, u32 round, u32 rows, u32 d, u64 q, u64* c_coef, cudaStream_t st) {
  u64 tot = (u64)rows * d;
  fold_chal_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(ds, round, rows, d, q, c_coef);
  return check_launch("fold_challenge");
}

// Fold constants per (row k, slot s): c_e, c_o and zeta c_o with their Shoup
// companions, so each slot product is four Shoup multiplications:
// (c_e + X c_o)(w_e + X w_o) = c_e w_e + (zeta c_o) w_o + X (c_o w_e + c_e w_o).
// Per (row k, slot s): c_e, c_o, zeta_s c_o and their Shoup companions, as six
// planes pre[(j * rows + k) * n + s] so that neighbouring slots are adjacent.
// FP: the same six planes for the FP64 products (q < 2^50): each constant as
// a double and its quotient fl(c / 2q), stored as the doubles' bits.
__global__ void fold_pre_kernel(const u64* c, u32 rows, u32 n, ModQ M, const u64* zeta, u64* pre, bool fp) {
  const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= rows * n) return;
  const u32 k = t / n, s = t % n;
  const u64 ce = c[(u64)k * 2 * n + s], co = c[(u64)k * 2 * n + n + s], zco = mul_mod(M, zeta[s], co);
  const u64 plane = (u64)rows * n;
  if (fp) {
    const double q2d = 2.0 * (double)M.q;
    const u64 v[3] = {ce, co, zco};
    for (int j = 0; j < 3; j++) {
      pre[(2 * j) * plane + t] = (u64)__double_as_longlong((double)v[j]);
      pre[(2 * j + 1) * plane + t] = (u64)__double_as_longlong(__ddiv_rn((double)v[j], q2d));
    }
    return;
  }
  pre[0 * plane + t] = ce;
  pre[1 * plane + t] = shoup_dev(ce, M.q);
  pre[2 * plane + t] = co;
  pre[3 * plane + t] = shoup_dev(co, M.q);
  pre[4 * plane + t] = zco;
  pre[5 * plane + t] = shoup_dev(zco, M.q);
}

// fold_vec_kernel with FP64 products (q < 2^50, canonical slot-form rows):
// per row the two products of each output are at most 1.25 q each, and the
// running sum is reduced after every row, so every value stays below 4 q.
// A thread folds one slot pair of FOLD_EL consecutive elements, so each
// row's six constant planes are loaded once for FOLD_EL elements (the
// constants were three quarters of the load requests with one element per
// thread); a warp's loads of one element stay 512 contiguous bytes.
constexpr u32 FOLD_EL = 4;

__global__ void __launch_bounds__(256) fold_fp_kernel(RowSet w, u32 rows, u64 width, u32 logn, ModQ M,
                                                      const u64* __restrict__ pre, u64* out) {
  const u32 n = 1u << logn, hn = n >> 1;
  const u64 groups = (width + FOLD_EL - 1) / FOLD_EL;
  const u64 tot = groups << (logn - 1);
  const u64 plane = (u64)rows << logn;
  const double qd = (double)M.q, q2d = 2.0 * qd, qinv = 1.0 / qd;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u64 i0 = (t >> (logn - 1)) * FOLD_EL;
    const u32 s = 2 * ((u32)t & (hn - 1));
    const u32 nel = width - i0 < FOLD_EL ? (u32)(width - i0) : FOLD_EL;
    double ae[FOLD_EL][2], ao[FOLD_EL][2];
#pragma unroll
    for (u32 j = 0; j < FOLD_EL; j++) ae[j][0] = ae[j][1] = ao[j][0] = ao[j][1] = 0.0;
#pragma unroll 2
    for (u32 k = 0; k < rows; k++) {
      const u64* pk = pre + ((u64)k << logn) + s;
      ulonglong2 C[6], E[FOLD_EL], O[FOLD_EL];
#pragma unroll
      for (u32 g = 0; g < 6; g++) C[g] = __ldg((const ulonglong2*)(pk + g * plane));
      const u64* x = w.p[k] + (i0 << (logn + 1));
#pragma unroll
      for (u32 j = 0; j < FOLD_EL; j++)
        if (j < nel) {
          E[j] = __ldg((const ulonglong2*)(x + ((u64)j << (logn + 1)) + s));
          O[j] = __ldg((const ulonglong2*)(x + ((u64)j << (logn + 1)) + n + s));
        }
#pragma unroll
      for (u32 h = 0; h < 2; h++) {
        const double ce = __longlong_as_double((long long)(h ? C[0].y : C[0].x));
        const double ceh = __longlong_as_double((long long)(h ? C[1].y : C[1].x));
        const double co = __longlong_as_double((long long)(h ? C[2].y : C[2].x));
        const double coh = __longlong_as_double((long long)(h ? C[3].y : C[3].x));
        const double zc = __longlong_as_double((long long)(h ? C[4].y : C[4].x));
        const double zch = __longlong_as_double((long long)(h ? C[5].y : C[5].x));
#pragma unroll
        for (u32 j = 0; j < FOLD_EL; j++)
          if (j < nel) {
            const double we = fp_from_word(h ? E[j].y : E[j].x), wo = fp_from_word(h ? O[j].y : O[j].x);
            const double e = __dadd_rn(fp_mulmod(we, ce, ceh, q2d), fp_mulmod(wo, zc, zch, q2d));
            const double o = __dadd_rn(fp_mulmod(we, co, coh, q2d), fp_mulmod(wo, ce, ceh, q2d));
            ae[j][h] = fp_reduce(__dadd_rn(ae[j][h], e), qinv, qd);
            ao[j][h] = fp_reduce(__dadd_rn(ao[j][h], o), qinv, qd);
          }
      }
    }
#pragma unroll
    for (u32 j = 0; j < FOLD_EL; j++)
      if (j < nel) {
        u64* dst = out + ((i0 + j) << (logn + 1));
        *(ulonglong2*)(dst + s) = make_ulonglong2(fp_to_word(ae[j][0], qinv, qd), fp_to_word(ae[j][1], qinv, qd));
        *(ulonglong2*)(dst + n + s) =
            make_ulonglong2(fp_to_word(ao[j][0], qinv, qd), fp_to_word(ao[j][1], qinv, qd));
      }
  }
}

// out = sum_k c_k w_k in slot form.  LAZY (q < 2^57, at most 16 rows): the
// per-row terms (each below 4q) are summed without reduction and reduced once.
template <bool LAZY>
__global__ void fold_kernel(RowSet w, u32 rows, u64 width, u32 logn, ModQ M, const u64* __restrict__ pre,
                            u64* out) {
  const u32 n = 1u << logn;
  const u64 tot = width << logn, q = M.q, q2 = 2 * q;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u64 i = t >> logn;
    const u32 s = (u32)t & (n - 1);
    u64 ae = 0, ao = 0;
    for (u32 k = 0; k < rows; k++) {
      const u64* x = w.p[k] + (i << (logn + 1));
      const u64 we = x[s], wo = x[n + s];
      const u64 plane = (u64)rows << logn;
      const u64* p = pre + ((u64)(k << logn) + s);
      const u64 ce = __ldg(p), cep = __ldg(p + plane), co = __ldg(p + 2 * plane), cop = __ldg(p + 3 * plane);
      const u64 zc = __ldg(p + 4 * plane), zcp = __ldg(p + 5 * plane);
      u64 e = mul_shoup_lazy(we, ce, cep, q) + mul_shoup_lazy(wo, zc, zcp, q);
      u64 o = mul_shoup_lazy(we, co, cop, q) + mul_shoup_lazy(wo, ce, cep, q);
      if (LAZY) {
        ae += e;
        ao += o;
      } else {  // e, o < 4q < 2^64
        e = e >= q2 ? e - q2 : e;
        e = e >= q ? e - q : e;
        o = o >= q2 ? o - q2 : o;
        o = o >= q ? o - q : o;
        ae = add_mod(ae, e, q);
        ao = add_mod(ao, o, q);
      }
    }
    if (LAZY) {
      ae = reduce64(M, ae);
      ao = reduce64(M, ao);
    }
    out[(i << (logn + 1)) + s] = ae;
    out[(i << (logn + 1)) + n + s] = ao;
  }
}

// The same with two neighbouring slots per thread (16-byte accesses) and the
// loads of four witness rows issued before their products, so each thread
// keeps eight independent loads in flight (needs n >= 2 and 16-byte aligned
// rows and output).
template <bool LAZY>
__global__ void __launch_bounds__(256) fold_vec_kernel(RowSet w, u32 rows, u64 width, u32 logn, ModQ M,
                                                       const u64* __restrict__ pre, u64* out) {
  const u32 n = 1u << logn, hn = n >> 1;
  const u64 tot = width << (logn - 1), q = M.q, q2 = 2 * q;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u64 i = t >> (logn - 1);
    const u32 s = 2 * ((u32)t & (hn - 1));
    u64 ae[2] = {0, 0}, ao[2] = {0, 0};
    for (u32 k0 = 0; k0 < rows; k0 += 4) {
      ulonglong2 E[4], O[4];
#pragma unroll
      for (u32 j = 0; j < 4; j++)
        if (k0 + j < rows) {
          const u64* x = w.p[k0 + j] + (i << (logn + 1));
          E[j] = __ldg((const ulonglong2*)(x + s));
          O[j] = __ldg((const ulonglong2*)(x + n + s));
        }
#pragma unroll
      for (u32 j = 0; j < 4; j++)
        if (k0 + j < rows) {
          // both slots' constants: one 16-byte load per plane
          const u64 plane = (u64)rows << logn;
          const u64* pk = pre + ((u64)((k0 + j) << logn) + s);
          ulonglong2 C[6];
#pragma unroll
          for (u32 g = 0; g < 6; g++) C[g] = __ldg((const ulonglong2*)(pk + g * plane));
#pragma unroll
          for (u32 h = 0; h < 2; h++) {
            const u64 we = h ? E[j].y : E[j].x, wo = h ? O[j].y : O[j].x;
            const u64 ce = h ? C[0].y : C[0].x, cep = h ? C[1].y : C[1].x, co = h ? C[2].y : C[2].x;
            const u64 cop = h ? C[3].y : C[3].x, zc = h ? C[4].y : C[4].x, zcp = h ? C[5].y : C[5].x;
            u64 e = mul_shoup_lazy(we, ce, cep, q) + mul_shoup_lazy(wo, zc, zcp, q);
            u64 o = mul_shoup_lazy(we, co, cop, q) + mul_shoup_lazy(wo, ce, cep, q);
            if (LAZY) {
              ae[h] += e;
              ao[h] += o;
            } else {  // e, o < 4q < 2^64
              e = e >= q2 ? e - q2 : e;
              e = e >= q ? e - q : e;
              o = o >= q2 ? o - q2 : o;
              o = o >= q ? o - q : o;
              ae[h] = add_mod(ae[h], e, q);
              ao[h] = add_mod(ao[h], o, q);
            }
          }
        }
    }
    if (LAZY) {
#pragma unroll
      for (u32 h = 0; h < 2; h++) {
        ae[h] = reduce64(M, ae[h]);
        ao[h] = reduce64(M, ao[h]);
      }
    }
    *(ulonglong2*)(out + (i << (logn + 1)) + s) = make_ulonglong2(ae[0], ae[1]);
    *(ulonglong2*)(out + (i << (logn + 1)) + n + s) = make_ulonglong2(ao[0], ao[1]);
  }
}

int launch_fold(RowSet w_slot, u32 rows, u64 width, const NttDev& T, const ModQ& M, const u64* c_slot, u64* pre,
                u64* out_slot, cudaStream_t st) {
  if (rows == 0 || rows > MAX_WROWS) return salsaa_set_error(-2, "fold: bad row count");
  if (w_slot.narrow) return salsaa_set_error(-2, "fold: slot-form rows must be canonical words");
  const bool lazy = M.q < (1ULL << 57);
  bool vec = T.n >= 2 && (uintptr_t)out_slot % 16 == 0 && (uintptr_t)pre % 16 == 0 && ((u64)rows * T.n) % 2 == 0;
  for (u32 k = 0; k < rows; k++) vec = vec && (uintptr_t)w_slot.p[k] % 16 == 0;
  const bool fp = vec && M.q < (1ULL << 50) && fold_choice() == 1;
  fold_pre_kernel<<<(rows * T.n + 127) / 128, 128, 0, st>>>(c_slot, rows, T.n, M, T.zeta, pre, fp);
  int rc = check_launch("fold_pre");
  if (rc) return rc;
  if (fp) {
    fold_fp_kernel<<<grid_1d((width + FOLD_EL - 1) / FOLD_EL * T.n / 2, 256), 256, 0, st>>>(w_slot, rows, width,
                                                                                            T.logn, M, pre, out_slot);
    return check_launch("fold");
  }
  if (vec) {
    const unsigned g = grid_1d(width * T.n / 2, 256);
    if (lazy) fold_vec_kernel<true><<<g, 256, 0, st>>>(w_slot, rows, width, T.logn, M, pre, out_slot);
    else fold_vec_kernel<false><<<g, 256, 0, st>>>(w_slot, rows, width, T.logn, M, pre, out_slot);
    return check_launch("fold");
  }
  if (lazy)
    fold_kernel<true><<<grid_1d(width * T.n, 256), 256, 0, st>>>(w_slot, rows, width, T.logn, M, pre, out_slot);
  else
    fold_kernel<false><<<grid_1d(width * T.n, 256), 256, 0, st>>>(w_slot, rows, width, T.logn, M, pre, out_slot);
  return check_launch("fold");
}

// ---------------------------------------------------------------------------
// Structured commitment <statement row, witness row> (parallel_dot_series_matrix,
// src/arithmetic.rs:459-505), all rows in one pass over each witness chunk.
//
// Commitment-key rows: value(i) = m^(i+1) = thi[i/B] * tlo[i%B].  A CTA owns a
// chunk of CH elements inside one B-block; each thread owns one NTT slot and
// accumulates sum_lo tlo[lo] * w[i] lazily (25-bit limbs, no reduction), then
// multiplies the reduced sum by thi[hi] and adds it to the global total.
// ---------------------------------------------------------------------------
template <int RT, int KT, bool LIMB>
__global__ void __launch_bounds__(256) ck_commit_kernel(RowSet w, u32 rows, u32 nck, const u64* tlo,
                                                        const u64* thi, u32 Bt, u32 nhi_t, u32 CH, ModQ M,
                                                        const u64* zeta, u64* acc, bool plain) {
  // grid: x = row tile (fastest, so co-scheduled CTAs share the witness chunk in L2),
  //       y = element chunk, z = witness-row tile
  const u32 n = blockDim.x, s = threadIdx.x, d = 2 * n;
  const u64 i0 = (u64)blockIdx.y * CH;
  const u32 hi = (u32)(i0 / Bt), lo0 = (u32)(i0 % Bt);
  const u32 r0 = blockIdx.x * RT, k0 = blockIdx.z * KT;
  const u64 q = M.q;
  Acc3 re[RT][KT], im[RT][KT];
  u64 gre[RT][KT], gim[RT][KT];
#pragma unroll
  for (int a = 0; a < RT; a++)
#pragma unroll
    for (int b = 0; b < KT; b++) {
      acc_zero(re[a][b]);
      acc_zero(im[a][b]);
      gre[a][b] = gim[a][b] = 0;
    }
  const u64* wp[KT];
#pragma unroll
  for (int b = 0; b < KT; b++) wp[b] = ((k0 + b < rows) ? w.p[k0 + b] : w.p[k0]) + i0 * d + s;
  const u64* tp[RT];
#pragma unroll
  for (int a = 0; a < RT; a++) tp[a] = tlo + ((u64)((r0 + a < nck) ? r0 + a : r0) * Bt + lo0) * 3 * n + s;
  // operands of the current element, prefetched one element ahead
  u64 we[KT], wo[KT], tc[RT], td[RT], tz[RT];
#pragma unroll
  for (int b = 0; b < KT; b++) {
    we[b] = __ldg(wp[b]);
    wo[b] = __ldg(wp[b] + n);
  }
#pragma unroll
  for (int a = 0; a < RT; a++) {
    tc[a] = __ldg(tp[a]);
    td[a] = __ldg(tp[a] + n);
    tz[a] = __ldg(tp[a] + 2 * n);
  }
  for (u32 e = 0; e < CH; e++) {
    const u32 en = (e + 1 < CH) ? e + 1 : e;
    u64 nwe[KT], nwo[KT], ntc[RT], ntd[RT], ntz[RT];
#pragma unroll
    for (int b = 0; b < KT; b++) {
      nwe[b] = __ldg(wp[b] + (u64)en * d);
      nwo[b] = __ldg(wp[b] + (u64)en * d + n);
    }
#pragma unroll
    for (int a = 0; a < RT; a++) {
      const u64* t = tp[a] + (u64)en * 3 * n;
      ntc[a] = __ldg(t);
      ntd[a] = __ldg(t + n);
      ntz[a] = __ldg(t + 2 * n);
    }
    if (LIMB) {
      u32 e1[KT], e0[KT], o1[KT], o0[KT];
#pragma unroll
      for (int b = 0; b < KT; b++) {
        split25(we[b], e1[b], e0[b]);
        split25(wo[b], o1[b], o0[b]);
      }
#pragma unroll
      for (int a = 0; a < RT; a++) {
        const u32 c1 = (u32)(tc[a] >> 32), c0 = (u32)tc[a];
        const u32 d1 = (u32)(td[a] >> 32), d0 = (u32)td[a];
        const u32 z1 = (u32)(tz[a] >> 32), z0 = (u32)tz[a];
#pragma unroll
        for (int b = 0; b < KT; b++) {
          acc_mac(re[a][b], e1[b], e0[b], c1, c0);
          acc_mac(re[a][b], o1[b], o0[b], z1, z0);
          acc_mac(im[a][b], o1[b], o0[b], c1, c0);
          acc_mac(im[a][b], e1[b], e0[b], d1, d0);
        }
      }
    } else {
#pragma unroll
      for (int a = 0; a < RT; a++)
#pragma unroll
        for (int b = 0; b < KT; b++) {
          gre[a][b] = add_mod(gre[a][b], add_mod(mul_mod(M, we[b], tc[a]), mul_mod(M, wo[b], tz[a]), q), q);
          gim[a][b] = add_mod(gim[a][b], add_mod(mul_mod(M, wo[b], tc[a]), mul_mod(M, we[b], td[a]), q), q);
        }
    }
#pragma unroll
    for (int b = 0; b < KT; b++) {
      we[b] = nwe[b];
      wo[b] = nwo[b];
    }
#pragma unroll
    for (int a = 0; a < RT; a++) {
      tc[a] = ntc[a];
      td[a] = ntd[a];
      tz[a] = ntz[a];
    }
  }
  const u64 z = zeta[s];
#pragma unroll
  for (int a = 0; a < RT; a++) {
    if (r0 + a >= nck) break;
    const u64* th = thi + ((u64)(r0 + a) * nhi_t + hi) * d;
    const u64 he = th[s], ho = th[n + s];
#pragma unroll
    for (int b = 0; b < KT; b++) {
      if (k0 + b >= rows) break;
      u64 ev = LIMB ? acc_reduce(M, re[a][b]) : gre[a][b];
      u64 ov = LIMB ? acc_reduce(M, im[a][b]) : gim[a][b];
      slot_mul(M, ev, ov, he, ho, z, ev, ov);
      u64* dst = acc + ((u64)(r0 + a) * rows + k0 + b) * d;
      atomic_add_mod(dst + s, ev, q, plain);
      atomic_add_mod(dst + n + s, ov, q, plain);
    }
  }
}

// Scalar-structured rows: value(i) = s_hi[i/Bw] * s_lo[i%Bw]; one thread per
// coefficient position of the slot-form witness, operands prefetched one
// element ahead.  Row tiles are RT consecutive scalar rows; a launch handles
// either the TENSOR tiles (want_tensor = 1, over the witness) or the others
// (over the witness' column sums, since their s_hi is identically 1).
template <int RT, int KT, bool LIMB>
__global__ void __launch_bounds__(512) sc_commit_kernel(RowSet w, u32 rows, ScRowList list, const u64* s_lo,
                                                        const u64* s_hi, u32 Bw, u32 nhi, u32 CH, ModQ M, u64* acc,
                                                        bool plain) {
  const u32 d = blockDim.x, p = threadIdx.x;
  const u32 t0 = blockIdx.x * RT, k0 = blockIdx.z * KT;
  u32 row[RT];  // statement rows of this tile (the last one repeated past the list's end)
#pragma unroll
  for (int a = 0; a < RT; a++) row[a] = list.idx[(t0 + a < list.n) ? t0 + a : list.n - 1];
  const u64 i0 = (u64)blockIdx.y * CH;
  const u32 hi = (u32)(i0 / Bw), lo0 = (u32)(i0 % Bw);
  const u64 q = M.q, qh = q / 2;
  // LIMB (q < 2^50): the centred witness value c = wh 2^25 + wl (|wl| <= 2^24)
  // times the row value s = s1 2^25 + s0 accumulates as three signed sums
  // A0 = sum s0 wl, A1 = sum (s1 wl + s0 wh), A2 = sum s1 wh; each term is
  // below 2^51, so 2048 terms stay below 2^63.  When no value of the warp
  // needs wh (small witness, the common case in coefficient form) the two
  // wh products are skipped for the whole warp.
  long long A0[RT][KT], A1[RT][KT], A2[RT][KT];
  u64 g[RT][KT];
#pragma unroll
  for (int a = 0; a < RT; a++)
#pragma unroll
    for (int b = 0; b < KT; b++) {
      A0[a][b] = A1[a][b] = A2[a][b] = 0;
      g[a][b] = 0;
    }
  const u64* wp[KT];
  bool wn[KT];
  const u64 wo = i0 * d + p;
#pragma unroll
  for (int b = 0; b < KT; b++) {
    const u32 kk = (k0 + b < rows) ? k0 + b : k0;
    wp[b] = w.p[kk];
    wn[b] = (w.narrow >> kk) & 1;
  }
  const u64* sp[RT];
#pragma unroll
  for (int a = 0; a < RT; a++) sp[a] = s_lo + (u64)row[a] * Bw + lo0;
  u64 x[KT], sv[RT];
#pragma unroll
  for (int b = 0; b < KT; b++) x[b] = wres(wp[b], wn[b], wo, q);
#pragma unroll
  for (int a = 0; a < RT; a++) sv[a] = __ldg(sp[a]);
  for (u32 e = 0; e < CH; e++) {
    const u32 en = (e + 1 < CH) ? e + 1 : e;
    u64 nx[KT], ns[RT];
#pragma unroll
    for (int b = 0; b < KT; b++) nx[b] = wres(wp[b], wn[b], wo + (u64)en * d, q);
#pragma unroll
    for (int a = 0; a < RT; a++) ns[a] = __ldg(sp[a] + en);
    if (LIMB) {
      int wl[KT], wh[KT];
      bool big = false;
#pragma unroll
      for (int b = 0; b < KT; b++) {
        // small (|centred value| < 2^24): x < 2^24 or x > q - 2^24; then the
        // low 32 bits of x or x - q are the signed value itself
        const bool neg = x[b] > qh;
        wl[b] = (int)((u32)x[b] - (neg ? (u32)q : 0u));
        wh[b] = 0;
        big |= neg ? (x[b] <= q - (1ULL << 24)) : (x[b] >= (1ULL << 24));
      }
      big = __any_sync(0xffffffffu, big);
      if (big) {  // exact split of every value of this step
#pragma unroll
        for (int b = 0; b < KT; b++) {
          const long long c = x[b] > qh ? (long long)x[b] - (long long)q : (long long)x[b];
          const long long l = ((c + (1LL << 24)) & ((1LL << 25) - 1)) - (1LL << 24);
          wl[b] = (int)l;
          wh[b] = (int)((c - l) >> 25);
        }
      }
#pragma unroll
      for (int a = 0; a < RT; a++) {
        const int s0 = (int)(sv[a] & 0x1FFFFFFull), s1 = (int)(sv[a] >> 25);
#pragma unroll
        for (int b = 0; b < KT; b++) {
          A0[a][b] += (long long)s0 * wl[b];
          A1[a][b] += (long long)s1 * wl[b];
        }
        if (big) {
#pragma unroll
          for (int b = 0; b < KT; b++) {
            A1[a][b] += (long long)s0 * wh[b];
            A2[a][b] += (long long)s1 * wh[b];
          }
        }
      }
    } else {
#pragma unroll
      for (int a = 0; a < RT; a++)
#pragma unroll
        for (int b = 0; b < KT; b++) g[a][b] = add_mod(g[a][b], mul_mod(M, x[b], sv[a]), q);
    }
#pragma unroll
    for (int b = 0; b < KT; b++) x[b] = nx[b];
#pragma unroll
    for (int a = 0; a < RT; a++) sv[a] = ns[a];
  }
  // signed sums -> residues: add a multiple of q above 2^62 to negative ones
  const u64 cpos = LIMB ? ((((u64)1 << 62) / q) + 1) * q : 0;
  const u64 p25 = LIMB ? ((u64)1 << 25) % q : 0, p50 = LIMB ? ((u64)1 << 50) % q : 0;
  auto smod = [&](long long v) -> u64 { return reduce64(M, v < 0 ? (u64)(v + (long long)cpos) : (u64)v); };
#pragma unroll
  for (int a = 0; a < RT; a++) {
    if (t0 + a >= list.n) break;
    const u64 h = s_hi[(u64)row[a] * nhi + hi];
#pragma unroll
    for (int b = 0; b < KT; b++) {
      if (k0 + b >= rows) break;
      u64 v;
      if (LIMB) {
        v = add_mod(smod(A0[a][b]), mul_mod(M, smod(A1[a][b]), p25), q);
        v = add_mod(v, mul_mod(M, smod(A2[a][b]), p50), q);
      } else {
        v = g[a][b];
      }
      v = mul_mod(M, v, h);
      atomic_add_mod(acc + ((u64)row[a] * rows + k0 + b) * d + p, v, q, plain);
    }
  }
}

// Column sums U_k[lo] = sum_h W_k[h*Bw + lo] (mod q) for the rows whose
// weights repeat with a period dividing Bw (witness_lhs and projected_lhs).
__global__ void colsum_kernel(RowSet w, u32 rows, u64 width, u32 Bw, u32 d, ModQ M, u64* out) {
  const u64 per = (u64)Bw * d, tot = rows * per, nhi = width / Bw;
  const bool lazy = M.q < (1ULL << 50) && nhi <= 4096;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u64 k = t / per, r = t % per;
    const u64* x = w.p[k];
    const bool nar = (w.narrow >> k) & 1;
    u64 sacc = 0;
    if (lazy) {
      for (u64 h = 0; h < nhi; h++) sacc += wres(x, nar, r + h * per, M.q);
      sacc %= M.q;
    } else {
      for (u64 h = 0; h < nhi; h++) sacc = add_mod(sacc, wres(x, nar, r + h * per, M.q), M.q);
    }
    out[t] = sacc;
  }
}

// Per-call scalar tables.  TENSOR: the layer of length 2^j = width uses the
// last j of the row's K element-index challenges (MSB first):
// s(i) = prod_t (bit ? c : 1 - c); split at Bw into s_hi (high bits), s_lo.
__global__ void sc_tables_kernel(const ScalarRowDesc* desc, u32 nsc, u64 width, u32 Bw, u32 nhi, ModQ M,
                                 const DevState* ds, u64* s_lo, u64* s_hi) {
  const u32 r = blockIdx.y;
  const ScalarRowDesc D = desc[r];
  const u64 q = M.q;
  const u32 j = 63u - (u32)__clzll((long long)width);
  const u32 b = 31u - (u32)__clz((int)Bw);
  for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < Bw + nhi; t += gridDim.x * blockDim.x) {
    const bool is_lo = t < Bw;
    const u32 idx = is_lo ? t : t - Bw;
    u64 v = 1 % q;
    if (D.type == ROW_TENSOR) {
      // lo bits: challenges K-b .. K-1 ; hi bits: challenges K-j .. K-b-1
      const u32 nb = is_lo ? b : j - b;
      const u32 first = is_lo ? D.K - b : D.K - j;
      for (u32 u = 0; u < nb; u++) {
        const u64 c = nc_challenge(ds, D.round, D.rep, first + u, q);
        const u32 bit = (idx >> (nb - 1 - u)) & 1;
        v = mul_mod(M, v, bit ? c : sub_mod(1 % q, c, q));
      }
    } else if (D.type == ROW_PERIODIC) {
      v = is_lo ? D.cj[idx % D.cw] : 1 % q;
    }
    if (is_lo) s_lo[(u64)r * Bw + idx] = v;
    else s_hi[(u64)r * nhi + idx] = v;
  }
}

__global__ void commit_finalize_kernel(const u64* acc, u32 nck, u32 nsc, u32 rows, u32 n, ModQ M,
                                       const u64* zeta, const u64* const* bases, u64* out) {
  const u64 tot = (u64)(nck + nsc) * rows * n;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u32 s = (u32)(t % n);
    const u64 jk = t / n;
    const u32 j = (u32)(jk / rows);
    const u64* a = acc + jk * 2 * n;
    u64 e = reduce64(M, a[s]), o = reduce64(M, a[n + s]);
    if (j >= nck && bases) {
      const u64* bs = bases[j - nck];
      if (bs) slot_mul(M, e, o, bs[s], bs[n + s], zeta[s], e, o);
    }
    out[jk * 2 * n + s] = e;
    out[jk * 2 * n + n + s] = o;
  }
}

// ---------------------------------------------------------------------------
// Tensor-core commitment-key rows (q < 2^56).  Per NTT slot s the key rows'
// contribution is a matrix product over F_q: with T = m^(lo+1) = (c, d) and
// W = (a, b) in F_q[X]/(X^2 - zeta),
//   re = sum_lo c a + (zeta d) b,   im = sum_lo c b + d a.
// Every value is split into 7 bytes, so G = A * B^T is an exact u8 x u8 ->
// s32 product (sums of 2048 byte products stay below 2^31), with
//   A rows (r, comp, byte) from the key tables (comp = c, d, zeta d) and
//   B rows (k, part, byte) from the witness (part = a, b);
// then value = sum_{x,y} 2^(8(x+y)) G[(.., x), (.., y)] mod q.
// ---------------------------------------------------------------------------
constexpr u32 CKM_KS = 128, CKM_LD = 144;

__global__ void ck_tl8_kernel(const u64* tlo, u32 nck, u32 n, u32 bt, u32 nmt, bool packed, uint8_t* tl8) {
  const u64 tot = (u64)n * nmt * CKM_BM * bt;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u32 lo = (u32)(t % bt);
    u64 rest = t / bt;
    const u32 m = (u32)(rest % CKM_BM);
    rest /= CKM_BM;
    const u32 mt = (u32)(rest % nmt), s = (u32)(rest / nmt);
    uint8_t v = 0;
    if (m < CKM_ROWS * 21) {
      const u32 r = mt * CKM_ROWS + m / 21, comp = (m / 7) % 3, b = m % 7;
      if (r < nck) {
        u64 x = tlo[((u64)r * bt + lo) * 3 * n + comp * n + s];
        if (packed) x = ((x >> 32) << 25) | (x & 0x1FFFFFFull);
        v = (uint8_t)(x >> (8 * b));
      }
    }
    tl8[t] = v;
  }
}

int launch_ck_tl8(const u64* tlo, u32 nck, u32 n, u32 bt, bool packed, uint8_t* tl8, cudaStream_t st) {
  const u32 nmt = (nck + CKM_ROWS - 1) / CKM_ROWS;
  ck_tl8_kernel<<<grid_1d((u64)n * nmt * CKM_BM * bt, 256), 256, 0, st>>>(tlo, nck, n, bt, nmt, packed, tl8);
  return check_launch("ck_tl8");
}

__device__ __forceinline__ void mma_u8_16832(int (&c)[4], u32 a0, u32 a1, u32 a2, u32 a3, u32 b0, u32 b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldsm_x4(u32 (&r)[4], const void* p) {
  const u32 a = (u32)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
__device__ __forceinline__ void ldsm_x2(u32 (&r)[2], const void* p) {
  const u32 a = (u32)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(a));
}

// CTA = (slot s, M tile of 6 key rows, block of Bw elements), slot fastest in
// the grid so the 64 CTAs of one block share the witness rows in L2.  The
// witness is read in its slot-form u64 layout and split into bytes while it
// is staged; the next stage is prefetched into registers during the MMAs.
// 8 warps as 4 (M, 32 rows) x 2 (N, NTW n-tiles of 8).
template <int NTW>
__global__ void __launch_bounds__(256) ck_mma_kernel(const uint8_t* __restrict__ tl8, RowSet w, u32 rows, u64 width,
                                                     u32 nck, u32 nmt, u32 n, u32 bt, u32 Bw, const u64* thi,
                                                     u32 nhi_t, ModQ M, const u64* zeta, u64* acc, bool plain) {
  constexpr u32 NP = 2 * NTW * 8;
  constexpr u32 TPT = 3;  // witness staging tasks per thread (rows <= 12)
  extern __shared__ __align__(16) uint8_t smem[];
  uint8_t* As = smem;
  uint8_t* Bs = smem + CKM_BM * CKM_LD;
  const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32 g = lane >> 2, t4 = lane & 3, wm = warp & 3, wn = warp >> 2;
  const u32 s = blockIdx.x, mt = blockIdx.y, hb = blockIdx.z;
  const u32 d = 2 * n, NR = rows * 14;
  const u64 i0 = (u64)hb * Bw;
  const uint8_t* Ag = tl8 + ((u64)s * nmt + mt) * CKM_BM * bt + (i0 % bt);
  const u32 ntask = rows * 2 * (CKM_KS / 4);  // (k, part, 4 consecutive elements)
  // zero the padding rows of the witness tile once
  for (u32 v = tid; v < (NP - NR) * CKM_LD / 4; v += 256) ((u32*)(Bs + NR * CKM_LD))[v] = 0;
  uint4 ra[4];
  u64 rb[TPT][4];
  auto fetch = [&](u32 l0) {
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const u32 v = tid + x * 256, row = v >> 3, c16 = v & 7;
      ra[x] = *(const uint4*)&Ag[(u64)row * bt + l0 + c16 * 16];
    }
#pragma unroll
    for (int x = 0; x < TPT; x++) {
      const u32 task = tid + x * 256;
      if (task < ntask) {
        const u32 i4 = task % (CKM_KS / 4), kp = task / (CKM_KS / 4), k = kp >> 1, part = kp & 1;
        const u64* src = w.p[k] + (i0 + l0 + i4 * 4) * d + part * n + s;
#pragma unroll
        for (int e = 0; e < 4; e++) rb[x][e] = __ldg(src + (u64)e * d);
      }
    }
  };
  auto stash = [&]() {
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const u32 v = tid + x * 256, row = v >> 3, c16 = v & 7;
      *(uint4*)&As[row * CKM_LD + c16 * 16] = ra[x];
    }
#pragma unroll
    for (int x = 0; x < TPT; x++) {
      const u32 task = tid + x * 256;
      if (task < ntask) {
        const u32 i4 = task % (CKM_KS / 4), kp = task / (CKM_KS / 4);
#pragma unroll
        for (int b = 0; b < 7; b++) {
          u32 word = 0;
#pragma unroll
          for (int e = 0; e < 4; e++) word |= ((u32)(rb[x][e] >> (8 * b)) & 0xffu) << (8 * e);
          *(u32*)&Bs[(kp * 7 + b) * CKM_LD + i4 * 4] = word;
        }
      }
    }
  };
  int c[2][NTW][4];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < NTW; b++)
#pragma unroll
      for (int e = 0; e < 4; e++) c[a][b][e] = 0;
  fetch(0);
  stash();
  __syncthreads();
  for (u32 l0 = 0; l0 < Bw; l0 += CKM_KS) {
    const bool more = l0 + CKM_KS < Bw;
    if (more) fetch(l0 + CKM_KS);
#pragma unroll
    for (u32 kk = 0; kk < CKM_KS; kk += 32) {
      u32 a[2][4], b[NTW][2];
#pragma unroll
      for (int mi = 0; mi < 2; mi++) {
        const u32 r = wm * 32 + mi * 16 + (lane & 7) + ((lane >> 3) & 1) * 8;
        ldsm_x4(a[mi], &As[r * CKM_LD + kk + (lane >> 4) * 16]);
      }
#pragma unroll
      for (int ni = 0; ni < NTW; ni++) {
        const u32 r = wn * NTW * 8 + ni * 8 + (lane & 7);
        ldsm_x2(b[ni], &Bs[r * CKM_LD + kk + ((lane >> 3) & 1) * 16]);
      }
#pragma unroll
      for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < NTW; ni++)
          mma_u8_16832(c[mi][ni], a[mi][0], a[mi][1], a[mi][2], a[mi][3], b[ni][0], b[ni][1]);
    }
    __syncthreads();
    if (more) {
      stash();
      __syncthreads();
    }
  }
  // G[m][nn] in shared memory
  int* G = (int*)smem;
#pragma unroll
  for (int mi = 0; mi < 2; mi++)
#pragma unroll
    for (int ni = 0; ni < NTW; ni++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const u32 m = wm * 32 + mi * 16 + g + 8 * h;
        const u32 nn = wn * NTW * 8 + ni * 8 + t4 * 2;
        G[m * NP + nn] = c[mi][ni][h * 2];
        G[m * NP + nn + 1] = c[mi][ni][h * 2 + 1];
      }
  __syncthreads();
  // partial[rl][k][term][x] = (sum_y 2^(8y) G[(rl,comp,x)][(k,part,y)]) * 2^(8x) mod q
  // terms: 0 = (c, a), 1 = (zeta d, b)  [re];  2 = (c, b), 3 = (d, a)  [im]
  u64* part = (u64*)(smem + (u64)CKM_BM * NP * sizeof(int));
  const u32 ntk = CKM_ROWS * rows * 4 * 7;
  for (u32 t = tid; t < ntk; t += 256) {
    const u32 x = t % 7, term = (t / 7) % 4, k = (t / 28) % rows, rl = t / (28 * rows);
    const u32 comp = (term == 0 || term == 2) ? 0 : (term == 1 ? 2 : 1);
    const u32 pr = (term == 0 || term == 3) ? 0 : 1;
    const int* grow = G + ((rl * 3 + comp) * 7 + x) * NP + (k * 2 + pr) * 7;
    u64 lo = 0, hi = 0;
#pragma unroll
    for (u32 y = 0; y < 7; y++) {
      const u64 v = (u64)(u32)grow[y];
      const u64 sl = v << (8 * y), sh = (y == 0) ? 0 : (v >> (64 - 8 * y));
      lo += sl;
      hi += sh + (lo < sl);
    }
    u64 r = reduce128_any(M, hi, lo);
    r = mul_mod(M, r, ((1ULL << (8 * x)) % M.q));
    part[t] = r;
  }
  __syncthreads();
  for (u32 t = tid; t < CKM_ROWS * rows; t += 256) {
    const u32 k = t % rows, rl = t / rows, r = mt * CKM_ROWS + rl;
    if (r >= nck) continue;
    const u64* pp = part + (u64)(rl * rows + k) * 28;
    u64 re = 0, im = 0;
#pragma unroll
    for (u32 x = 0; x < 7; x++) {
      re = add_mod(re, add_mod(pp[0 * 7 + x], pp[1 * 7 + x], M.q), M.q);
      im = add_mod(im, add_mod(pp[2 * 7 + x], pp[3 * 7 + x], M.q), M.q);
    }
    const u32 hi_t = (u32)(i0 / bt);
    const u64* th = thi + ((u64)r * nhi_t + hi_t) * d;
    slot_mul(M, re, im, th[s], th[n + s], zeta[s], re, im);
    u64* dst = acc + ((u64)r * rows + k) * d;
    atomic_add_mod(dst + s, re, M.q, plain);
    atomic_add_mod(dst + n + s, im, M.q, plain);
  }
}

template <int NTW>
static int launch_ck_mma_t(const CommitArgs& a, u32 n, u32 Bw, const ModQ& M, const u64* zeta, bool plain,
                           cudaStream_t st) {
  constexpr u32 NP = 2 * NTW * 8;
  const u32 nmt = (a.nck + CKM_ROWS - 1) / CKM_ROWS;
  const size_t stage = (size_t)(CKM_BM + NP) * CKM_LD;
  const size_t epi = (size_t)CKM_BM * NP * sizeof(int) + (size_t)CKM_ROWS * a.rows * 28 * sizeof(u64);
  const size_t smem = stage > epi ? stage : epi;
  auto kern = ck_mma_kernel<NTW>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "ck_mma smem attribute");
  }
  dim3 g(n, nmt, (unsigned)(a.width / Bw));
  // algorithmic work: the exact byte-limb products, 3 key components x 7 bytes
  // against 2 witness parts x 7 bytes per (key row, witness row, element, slot)
  const int tr = salsaa_trace_begin("ck_mma_kernel", st, 2.0 * 294.0 * a.nck * a.rows * (double)a.width * n);
  kern<<<g, 256, smem, st>>>(a.tl8, a.w, a.rows, a.width, a.nck, nmt, n, a.ck_bt, Bw, a.thi, a.ck_nhi, M, zeta,
                             a.acc, plain);
  salsaa_trace_end(tr, st);
  return check_launch("ck_mma");
}

static int launch_ck_mma(const CommitArgs& a, u32 n, u32 Bw, const ModQ& M, const u64* zeta, bool plain,
                         cudaStream_t st) {
  switch ((a.rows * 14 + 15) / 16) {
    case 1: return launch_ck_mma_t<1>(a, n, Bw, M, zeta, plain, st);
    case 2: return launch_ck_mma_t<2>(a, n, Bw, M, zeta, plain, st);
    case 3: return launch_ck_mma_t<3>(a, n, Bw, M, zeta, plain, st);
    case 4: return launch_ck_mma_t<4>(a, n, Bw, M, zeta, plain, st);
    case 5: return launch_ck_mma_t<5>(a, n, Bw, M, zeta, plain, st);
    case 6: return launch_ck_mma_t<6>(a, n, Bw, M, zeta, plain, st);
    case 7: return launch_ck_mma_t<7>(a, n, Bw, M, zeta, plain, st);
    case 8: return launch_ck_mma_t<8>(a, n, Bw, M, zeta, plain, st);
    default: return salsaa_set_error(-2, "ck_mma: too many witness rows");
  }
}

template <int RT, int KT>
static void launch_ck_variant(const CommitArgs& a, u32 n, u32 Bt, u32 nhi_t, u32 CH, const ModQ& M,
                              const u64* zeta, bool plain, cudaStream_t st) {
  dim3 g((a.nck + RT - 1) / RT, (unsigned)(a.width / CH), (a.rows + KT - 1) / KT);
  if (M.q < (1ULL << 50))
    ck_commit_kernel<RT, KT, true><<<g, n, 0, st>>>(a.w, a.rows, a.nck, a.tlo, a.thi, Bt, nhi_t, CH, M, zeta, a.acc,
                                                   plain);
  else
    ck_commit_kernel<RT, KT, false><<<g, n, 0, st>>>(a.w, a.rows, a.nck, a.tlo, a.thi, Bt, nhi_t, CH, M, zeta,
                                                    a.acc, plain);
}

template <int RT, int KT>
static void launch_sc_variant(const CommitArgs& a, const RowSet& w, u64 width, const ScRowList& list, u32 d, u32 Bw,
                              u32 nhi, u32 CH, const ModQ& M, bool plain, u64* acc_sc, cudaStream_t st) {
  dim3 g((list.n + RT - 1) / RT, (unsigned)(width / CH), (a.rows + KT - 1) / KT);
  if (M.q < (1ULL << 50))
    sc_commit_kernel<RT, KT, true><<<g, d, 0, st>>>(w, a.rows, list, a.sc_lo, a.sc_hi, Bw, nhi, CH, M, acc_sc, plain);
  else
    sc_commit_kernel<RT, KT, false><<<g, d, 0, st>>>(w, a.rows, list, a.sc_lo, a.sc_hi, Bw, nhi, CH, M, acc_sc,
                                                    plain);
}

// One launch per row list (TENSOR rows over the witness; periodic / all-ones
// rows over its column sums), tiles of 2 rows x up to 4 witness rows.
static void launch_sc_pass(const CommitArgs& a, const RowSet& w, u64 width, const ScRowList& list, bool tensor, u32 d,
                           u32 Bw, u32 nhi, u32 CH, const ModQ& M, bool plain, u64* acc_sc, cudaStream_t st) {
  if (!list.n) return;
  (void)tensor;
  if (a.rows == 1) launch_sc_variant<2, 1>(a, w, width, list, d, Bw, nhi, CH, M, plain, acc_sc, st);
  else if (a.rows == 2) launch_sc_variant<2, 2>(a, w, width, list, d, Bw, nhi, CH, M, plain, acc_sc, st);
  else launch_sc_variant<2, 4>(a, w, width, list, d, Bw, nhi, CH, M, plain, acc_sc, st);
}

__global__ void reduce_inplace_kernel(u64* x, u64 n, ModQ M) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    x[i] = reduce64(M, x[i]);
}

int launch_commit(const CommitArgs& a, const NttDev& T, const ModQ& M, const DevState* ds, cudaStream_t st) {
  const u32 n = T.n, d = 2 * n;
  if (a.rows == 0 || a.rows > MAX_WROWS || a.width == 0 || (a.width & (a.width - 1)))
    return salsaa_set_error(-2, "commit: bad witness shape");
  if (d > 512) return salsaa_set_error(-2, "commit: ring degree above 512");
  if (a.w.narrow) return salsaa_set_error(-2, "commit: slot-form rows must be canonical words");
  const u32 Bw = (u32)(a.width < CK_BLOCK ? a.width : CK_BLOCK);
  const u32 nhi = (u32)(a.width / Bw);
  // chunk: >= 128 elements (each thread's lazy sums are reduced once per
  // chunk), at most 512 chunks, inside one block of either table
  u64 CH = a.width / 512;
  if (CH < 128) CH = 128;
  if (CH > Bw) CH = Bw;
  const bool plain = M.q < (1ULL << 50) && (a.width / CH) < (1ULL << 13);
  cudaError_t e =
      cudaMemsetAsync(a.acc, 0, (u64)(a.nck + a.nsc) * a.rows * d * sizeof(u64), st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "commit memset");
  // statement rows: on the side stream when given (they write their own
  // accumulator rows, after the memset), joined before the finalisation
  const bool side = a.st2 && a.nck && a.nsc;
  cudaStream_t ss = side ? a.st2 : st;
  if (side) {
    e = cudaEventRecord(a.ev_fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ss, a.ev_fork, 0);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "commit: fork");
  }
  if (a.nck && ck_umma_ok(a, n)) {
    u32 Bk, G;
    ck_umma_shape(a.width, a.rows, n, a.ck_bt, &Bk, &G);
    int rc = launch_ck_umma(a, n, Bk, G, M, T.zeta, plain, st);
    if (rc) return rc;
  } else if (a.nck && a.tl8 && M.q < (1ULL << 56) && a.width >= CKM_KS && a.rows <= 9 && n <= 512) {
    if (Bw > a.ck_bt) return salsaa_set_error(-2, "commit: witness wider than the key tables");
    int rc = launch_ck_mma(a, n, Bw, M, T.zeta, plain, st);
    if (rc) return rc;
  } else if (a.nck) {
    if (Bw > a.ck_bt || a.ck_bt % CH) return salsaa_set_error(-2, "commit: witness wider than the key tables");
    if (a.rows == 1) launch_ck_variant<4, 1>(a, n, a.ck_bt, a.ck_nhi, (u32)CH, M, T.zeta, plain, st);
    else if (a.rows == 2) launch_ck_variant<4, 2>(a, n, a.ck_bt, a.ck_nhi, (u32)CH, M, T.zeta, plain, st);
    else launch_ck_variant<2, 4>(a, n, a.ck_bt, a.ck_nhi, (u32)CH, M, T.zeta, plain, st);
    int rc = check_launch("ck_commit");
    if (rc) return rc;
  }
  if (a.nsc) {
    dim3 gt((Bw + nhi + 255) / 256, a.nsc);
    sc_tables_kernel<<<gt, 256, 0, ss>>>(a.sc_desc_dev, a.nsc, a.width, Bw, nhi, M, ds, a.sc_lo, a.sc_hi);
    int rc = check_launch("sc_tables");
    if (rc) return rc;
    u64* acc_sc = a.acc + (u64)a.nck * a.rows * d;
    // scalar rows are linear in the witness: with its coefficient form given,
    // sum there (small centred values) and move the sums to slot form after
    const RowSet& wsrc = a.coef_sc ? a.wc : a.w;
    if (!a.sc_types_host || a.nsc > SC_MAX_ROWS) return salsaa_set_error(-2, "commit: scalar row types missing");
    ScRowList tl{}, ol{};
    for (u32 j = 0; j < a.nsc; j++) {
      if (a.sc_types_host[j] == ROW_TENSOR) tl.idx[tl.n++] = (unsigned char)j;
      else ol.idx[ol.n++] = (unsigned char)j;
    }
    // TENSOR rows: one tensor-core pass over the coefficient-form witness when
    // the shapes fit, else CUDA cores.  Every scalar row weighs element i by
    // s_hi[i / Bw] s_lo[i % Bw], so when that pass runs anyway the periodic /
    // all-ones rows ride in it if they fit, and no column sums are needed.
    const bool tc_ok = a.coef_sc && a.sc_img && a.sc_flags && M.q < (1ULL << 56) && d % 128 == 0 &&
                       Bw % 128 == 0 && tl.n > 0 && tl.n <= SC_UMMA_MAX_ROWS && rowset_aligned(wsrc, a.rows, 16, 8);
    bool periodic_done = false;
    if (tc_ok) {
      ScRowList gl = tl;
      if (tl.n + ol.n <= SC_UMMA_MAX_ROWS) {
        for (u32 i = 0; i < ol.n; i++) gl.idx[gl.n++] = ol.idx[i];
        periodic_done = true;
      }
      rc = launch_sc_umma(wsrc, a.rows, a.width, d, Bw, nhi, gl, a.sc_lo, a.sc_hi, M, acc_sc, plain, a.sc_img,
                          a.sc_flags, a.sc_flag_cap, ss);
      if (rc) return rc;
      if (!periodic_done && ol.n <= SC_UMMA_MAX_ROWS) {
        // more rows than one pass holds: the periodic / all-ones rows in a second pass
        rc = launch_sc_umma(wsrc, a.rows, a.width, d, Bw, nhi, ol, a.sc_lo, a.sc_hi, M, acc_sc, plain, a.sc_img,
                            a.sc_flags, a.sc_flag_cap, ss);
        if (rc) return rc;
        periodic_done = true;
      }
    } else {
      launch_sc_pass(a, wsrc, a.width, tl, true, d, Bw, nhi, (u32)CH, M, plain, acc_sc, ss);
      rc = check_launch("sc_commit (tensor rows)");
      if (rc) return rc;
    }
    if (!periodic_done && ol.n) {
      // periodic and all-ones rows over the column sums
      RowSet u = wsrc;
      if (nhi > 1) {
        if (!a.colsum || a.rows > a.colsum_rows) return salsaa_set_error(-2, "commit: column-sum scratch too small");
        colsum_kernel<<<grid_1d((u64)a.rows * Bw * d, 256), 256, 0, ss>>>(wsrc, a.rows, a.width, Bw, d, M,
                                                                         a.colsum);
        rc = check_launch("colsum");
        if (rc) return rc;
        for (u32 k = 0; k < a.rows; k++) u.p[k] = a.colsum + (u64)k * Bw * d;
        u.narrow = 0;  // the column sums are canonical words
      }
      u64 CHu = Bw / 64;
      if (CHu < 16) CHu = 16;
      if (CHu > Bw) CHu = Bw;
      launch_sc_pass(a, u, Bw, ol, false, d, Bw, nhi, (u32)CHu, M, plain, acc_sc, ss);
      rc = check_launch("sc_commit (periodic rows)");
      if (rc) return rc;
    }
    if (a.coef_sc) {
      const u64 cnt = (u64)a.nsc * a.rows;
      reduce_inplace_kernel<<<grid_1d(cnt * d, 256), 256, 0, ss>>>(acc_sc, cnt * d, M);
      rc = check_launch("reduce");
      if (rc) return rc;
      rc = ntt_launch(acc_sc, acc_sc, cnt, T, true, false, ss);
      if (rc) return rc;
    }
  }
  if (side) {
    e = cudaEventRecord(a.ev_join, ss);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, a.ev_join, 0);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "commit: join");
  }
  const u64 tot = (u64)(a.nck + a.nsc) * a.rows * n;
  commit_finalize_kernel<<<grid_1d(tot, 256), 256, 0, st>>>(a.acc, a.nck, a.nsc, a.rows, n, M, T.zeta,
                                                          a.sc_base_dev, a.out_slot);
  return check_launch("commit_finalize");
}

int launch_commit_finalize(const u64* acc, u32 nck, u32 rows, const NttDev& T, const ModQ& M, u64* out,
                           cudaStream_t st) {
  const u64 tot = (u64)nck * rows * T.n;
  commit_finalize_kernel<<<grid_1d(tot, 256), 256, 0, st>>>(acc, nck, 0, rows, T.n, M, T.zeta, nullptr, out);
  return check_launch("commit_finalize");
}

// ---------------------------------------------------------------------------
// Derived commitments (see launch_derive in kernels.cuh).
// ---------------------------------------------------------------------------
__global__ void derive_kernel(DeriveArgs a, u32 n, ModQ M, const u64* zeta, const DevState* ds) {
  const u64 tot = (u64)(a.nck + a.nsc) * a.K * n;
  const u32 d = 2 * n;
  const u32 logw = 63u - (u32)__clzll((long long)a.w);
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u32 s = (u32)(t % n);
    const u64 jk = t / n;
    const u32 k = (u32)(jk % a.K), j = (u32)(jk / a.K);
    const u64* x = a.R + ((u64)j * a.ncols + k) * d;
    const u64* y = a.R + ((u64)j * a.ncols + a.K + k) * d;
    u64 re, ro;
    if (j < a.nck) {
      // t0 = 1, t1 = m^(w/2)
      const u64 e = a.w / 2;
      u64 te, to;
      if (e >= a.ck_bt) {
        const u64* th = a.thi + ((u64)j * a.ck_nhi + e / a.ck_bt) * d;
        te = th[s];
        to = th[n + s];
      } else {
        const u64* tl = a.tlo + ((u64)j * a.ck_bt + (e - 1)) * 3 * n;
        te = tl[s];
        to = tl[n + s];
        if (a.packed) {
          te = ((te >> 32) << 25) | (te & 0x1FFFFFFull);
          to = ((to >> 32) << 25) | (to & 0x1FFFFFFull);
        }
      }
      slot_mul(M, te, to, y[s], y[n + s], zeta[s], re, ro);
      re = add_mod(re, x[s], M.q);
      ro = add_mod(ro, x[n + s], M.q);
    } else {
      const ScalarRowDesc D = a.sc_desc_dev[j - a.nck];
      u64 t0 = 1 % M.q, t1 = 1 % M.q;
      if (D.type == ROW_TENSOR) {
        const u64 c = uni_mod(prf_at(prf_key(ds->seed, domain_id(DOM_NC, D.round, D.rep)), D.K - logw), M.q);
        t0 = sub_mod(1 % M.q, c, M.q);
        t1 = c;
      }
      re = add_mod(mul_mod(M, t0, x[s]), mul_mod(M, t1, y[s]), M.q);
      ro = add_mod(mul_mod(M, t0, x[n + s]), mul_mod(M, t1, y[n + s]), M.q);
    }
    a.out[jk * d + s] = re;
    a.out[jk * d + n + s] = ro;
  }
}

int launch_derive(const DeriveArgs& a, const NttDev& T, const ModQ& M, const DevState* ds, cudaStream_t st) {
  if (a.w < 2 || (a.w & (a.w - 1)) || a.ncols < 2 * a.K) return salsaa_set_error(-2, "derive: bad shape");
  const u64 tot = (u64)(a.nck + a.nsc) * a.K * T.n;
  derive_kernel<<<grid_1d(tot, 256), 256, 0, st>>>(a, T.n, M, T.zeta, ds);
  return check_launch("derive");
}

}  // namespace salsaa
