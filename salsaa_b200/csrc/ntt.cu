// ntt.cu — batched negacyclic NTT / INTT kernels and their twiddle tables.
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <map>
#include <atomic>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/salsaa_gpu.h"
#include "host_math.h"
#include "ntt.cuh"
#include "umma.cuh"

namespace salsaa {

namespace {
std::mutex g_tab_mu;
std::map<std::tuple<int, u32, u64>, NttDev*> g_tabs;
}  // namespace

const NttDev* ntt_tables(u32 n, u64 q) {
  if (n < 2 || (n & (n - 1)) || n > 8192 || q < 3 || q >= (1ULL << 62)) return nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(g_tab_mu);
  auto key = std::make_tuple(dev, n, q);
  auto it = g_tabs.find(key);
  if (it != g_tabs.end()) return it->second;
  const u64 psi = host::minimal_root(2ULL * n, q);
  if (!psi) return nullptr;
  const unsigned logn = host::ilog2(n);
  std::vector<u64> h(6 * (size_t)n + 2 * (size_t)n);
  u64 *fwd = h.data(), *fwdp = fwd + n, *inv = fwdp + n, *invp = inv + n, *zeta = invp + n, *zetap = zeta + n;
  const u64 psi_inv = host::invmod(psi, q);
  u64 p = 1, pi = 1;
  for (u64 i = 0; i < n; i++) {
    u32 j = host::bitrev(i, logn);
    fwd[j] = p;
    inv[j] = pi;
    p = host::mulmod(p, psi, q);
    pi = host::mulmod(pi, psi_inv, q);
  }
  for (u64 i = 0; i < n; i++) {
    fwdp[i] = shoup_pre(fwd[i], q);
    invp[i] = shoup_pre(inv[i], q);
  }
  // shift factors: forward NTT of Y, computed with the same tables on the host
  std::vector<u64> y(n, 0);
  y[1 % n] = (n > 1) ? 1 : 0;
  {
    u64 t = n;
    for (u64 m = 1; m < n; m <<= 1) {
      t >>= 1;
      for (u64 i = 0; i < m; i++)
        for (u64 j = 2 * i * t; j < 2 * i * t + t; j++) {
          u64 U = y[j], V = host::mulmod(y[j + t], fwd[m + i], q);
          y[j] = host::addmod(U, V, q);
          y[j + t] = host::submod(U, V, q);
        }
    }
  }
  for (u64 i = 0; i < n; i++) {
    zeta[i] = y[i];
    zetap[i] = shoup_pre(y[i], q);
  }
  u64* d = nullptr;
  if (cudaMalloc(&d, h.size() * sizeof(u64)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, h.data(), h.size() * sizeof(u64), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  // FP64 companions: exact doubles of the twiddles (w < q < 2^53) and the
  // correctly rounded quotients w / 2q
  std::vector<double> hd(4 * (size_t)n);
  const double q2d = 2.0 * (double)q;
  for (u64 i = 0; i < n; i++) {
    hd[i] = (double)fwd[i];
    hd[n + i] = (double)fwd[i] / q2d;
    hd[2 * n + i] = (double)inv[i];
    hd[3 * n + i] = (double)inv[i] / q2d;
  }
  double* dd = nullptr;
  if (cudaMalloc(&dd, hd.size() * sizeof(double)) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  if (cudaMemcpy(dd, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    cudaFree(dd);
    return nullptr;
  }
  NttDev* T = new NttDev;
  T->fwd_d = dd;
  T->fwd_h = dd + n;
  T->inv_d = dd + 2 * n;
  T->inv_h = dd + 3 * n;
  T->qd = (double)q;
  T->q2d = q2d;
  T->qinv = 1.0 / (double)q;
  T->q = q;
  T->n = n;
  T->logn = logn;
  T->fwd = d;
  T->fwdp = d + n;
  T->inv = d + 2 * n;
  T->invp = d + 3 * n;
  T->zeta = d + 4 * n;
  T->zetap = d + 5 * n;
  T->ninv = host::invmod(n % q, q);
  T->ninvp = shoup_pre(T->ninv, q);
  T->onep = shoup_pre(1, q);
  T->ninv_d = (double)T->ninv;
  T->ninv_h = (double)T->ninv / q2d;
  g_tabs[key] = T;
  return T;
}

// One CTA transforms `epb` elements staged in shared memory.  Element size is
// d = n (full) or d = 2n (incomplete, two interleaved halves).  Loads and
// stores are coalesced over the element-contiguous global layout; the
// even/odd de-interleave of the incomplete layout happens on the way into or
// out of shared memory.
template <bool INCOMPLETE, bool INVERSE>
__global__ void __launch_bounds__(256) ntt_kernel(const u64* in, u64* out, u64 count,
                                                  NttDev T, u32 epb) {
  extern __shared__ u64 sm[];
  const u32 n = T.n, logn = T.logn;
  const u32 logd = INCOMPLETE ? logn + 1 : logn;
  const u32 d = 1u << logd;
  const u64 q = T.q;
  const u64 e0 = (u64)blockIdx.x * epb;
  const u32 ne = (u32)min((u64)epb, count - e0);
  const u32 tot = ne << logd;
  const u64* src = in + (e0 << logd);
  for (u32 t = threadIdx.x; t < tot; t += blockDim.x) {
    u64 v = src[t];
    u32 dst = t;
    if (INCOMPLETE && !INVERSE) {
      u32 e = t >> logd, p = t & (d - 1);
      dst = (e << logd) + (p & 1) * n + (p >> 1);
    }
    sm[dst] = v;
  }
  __syncthreads();
  const u32 units = INCOMPLETE ? 2 * ne : ne;
  const u32 half = n >> 1, loghalf = logn - 1;
  const u32 nbf = units << loghalf;
  if (!INVERSE) {
    u32 logt = logn;
    for (u32 m = 1; m < n; m <<= 1) {
      logt--;
      const u32 t = 1u << logt;
      for (u32 b = threadIdx.x; b < nbf; b += blockDim.x) {
        const u32 u = b >> loghalf, r = b & (half - 1);
        const u32 i = r >> logt, jj = r & (t - 1);
        const u32 j = (u << logn) + (i << (logt + 1)) + jj;
        const u64 W = T.fwd[m + i], Wp = T.fwdp[m + i];
        const u64 U = sm[j], V = mul_shoup(sm[j + t], W, Wp, q);
        sm[j] = add_mod(U, V, q);
        sm[j + t] = sub_mod(U, V, q);
      }
      __syncthreads();
    }
  } else {
    u32 logt = 0;
    for (u32 m = n; m > 1; m >>= 1) {
      const u32 h = m >> 1, t = 1u << logt;
      for (u32 b = threadIdx.x; b < nbf; b += blockDim.x) {
        const u32 u = b >> loghalf, r = b & (half - 1);
        const u32 i = r >> logt, jj = r & (t - 1);
        const u32 j = (u << logn) + (i << (logt + 1)) + jj;
        const u64 W = T.inv[h + i], Wp = T.invp[h + i];
        const u64 U = sm[j], V = sm[j + t];
        sm[j] = add_mod(U, V, q);
        sm[j + t] = mul_shoup(sub_mod(U, V, q), W, Wp, q);
      }
      logt++;
      __syncthreads();
    }
    for (u32 t = threadIdx.x; t < tot; t += blockDim.x) sm[t] = mul_shoup(sm[t], T.ninv, T.ninvp, q);
    __syncthreads();
  }
  u64* dstp = out + (e0 << logd);
  for (u32 t = threadIdx.x; t < tot; t += blockDim.x) {
    u32 s = t;
    if (INCOMPLETE && INVERSE) {
      u32 e = t >> logd, p = t & (d - 1);
      s = (e << logd) + (p & 1) * n + (p >> 1);
    }
    dstp[t] = sm[s];
  }
}

// ---------------------------------------------------------------------------
// Kernel schedule of the register-path NTT per (log2 n, incomplete, inverse,
// q >= 2^50, batch class: large = at least 2^22 coefficients): variant 0 =
// one 4096-coefficient tile per CTA with integer butterflies
// (ntt_reg_kernel), 1 = the same with FP64 butterflies (ntt_fp_kernel; used
// only when q < 2^50, and also selecting the digit transform's arithmetic),
// 2..4 = persistent CTAs with that many bulk-copy stages (ntt_pipe_kernel),
// 5..7 = the same with FP64 butterflies (q < 2^50; else as 2..4);
// ctas_per_sm caps the resident CTAs per SM (0 = as many as fit).  The
// defaults are variant 0; a table written by the tuner (salsaa_b200/tune.py)
// replaces them: "ntt <log_n> <incomplete> <inverse> <wide> <large> <variant>
// <ctas_per_sm>" per line, loaded from SALSAA_TUNE_FILE or from
// tune_table.txt beside the library the first time a transform launches.
// ---------------------------------------------------------------------------
// Bumped by every change of the schedule table (loads, sets, resets), so a
// captured CUDA graph of a proof, which holds the kernels chosen at capture
// time, is captured again after a change.
std::atomic<unsigned long long> g_sched_gen{0};
unsigned long long schedule_generation() { return g_sched_gen.load(std::memory_order_acquire); }

namespace {
constexpr int TUNE_LOGN = 14;
std::mutex g_tune_mu;
NttChoice g_tune[TUNE_LOGN][2][2][2][2];
int g_fold_variant = 0;  // fold products: 0 = integer (Shoup), 1 = FP64 (q < 2^50)
bool g_tune_loaded = false;

int tune_index_ok(u32 logn) { return logn < (u32)TUNE_LOGN; }

int tune_load_locked(const char* path) {
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  g_sched_gen.fetch_add(1, std::memory_order_acq_rel);
  char line[256];
  int n = 0;
  while (fgets(line, sizeof line, f)) {
    unsigned fv;
    if (sscanf(line, "fold %u", &fv) == 1) {
      if (fv <= 1) {
        g_fold_variant = (int)fv;
        n++;
      }
      continue;
    }
    unsigned lg, inc, inv, wide, big, var, cps;
    if (sscanf(line, "ntt %u %u %u %u %u %u %u", &lg, &inc, &inv, &wide, &big, &var, &cps) != 7) continue;
    if (lg >= (unsigned)TUNE_LOGN || inc > 1 || inv > 1 || wide > 1 || big > 1 ||
        var > 7 || cps > 8)
      continue;
    g_tune[lg][inc][inv][wide][big] = NttChoice{(uint8_t)var, (uint8_t)cps};
    n++;
  }
  fclose(f);
  return n;
}

// The library's own directory (for the default table beside it).
std::string lib_dir() {
  Dl_info info;
  if (!dladdr((void*)&lib_dir, &info) || !info.dli_fname) return ".";
  std::string p = info.dli_fname;
  const size_t k = p.rfind('/');
  return k == std::string::npos ? std::string(".") : p.substr(0, k);
}

void tune_default_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char* env = getenv("SALSAA_TUNE_FILE");
  const std::string path = env && *env ? std::string(env) : lib_dir() + "/tune_table.txt";
  tune_load_locked(path.c_str());
}
}  // namespace

NttChoice ntt_choice(u32 logn, bool incomplete, bool inverse, bool wide, bool large) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_default_locked();
  if (!tune_index_ok(logn)) return NttChoice{0, 0};
  return g_tune[logn][incomplete][inverse][wide][large];
}

int ntt_tune_set(u32 logn, bool incomplete, bool inverse, bool wide, bool large, int variant, int ctas_per_sm) {
  if (!tune_index_ok(logn) || variant < 0 || variant > 7 || ctas_per_sm < 0 || ctas_per_sm > 8)
    return salsaa_set_error(-2, "ntt_tune_set: log_n < 14, variant 0..7, ctas_per_sm 0..8");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_default_locked();
  g_tune[logn][incomplete][inverse][wide][large] = NttChoice{(uint8_t)variant, (uint8_t)ctas_per_sm};
  g_sched_gen.fetch_add(1, std::memory_order_acq_rel);
  return 0;
}

int ntt_tune_load(const char* path) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_loaded = true;
  if (!path) {
    const char* env = getenv("SALSAA_TUNE_FILE");
    const std::string p = env && *env ? std::string(env) : lib_dir() + "/tune_table.txt";
    const int n = tune_load_locked(p.c_str());
    return n < 0 ? salsaa_set_error(-1, ("tune_load: cannot read " + p).c_str()) : n;
  }
  const int n = tune_load_locked(path);
  return n < 0 ? salsaa_set_error(-1, "tune_load: cannot read the table file") : n;
}

int fold_choice() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_default_locked();
  return g_fold_variant;
}

int fold_tune_set(int variant) {
  if (variant < 0 || variant > 1) return salsaa_set_error(-2, "fold_tune_set: variant 0 or 1");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_default_locked();
  g_fold_variant = variant;
  g_sched_gen.fetch_add(1, std::memory_order_acq_rel);
  return 0;
}

void ntt_tune_reset() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_loaded = true;  // defaults, and no automatic load afterwards
  g_sched_gen.fetch_add(1, std::memory_order_acq_rel);
  g_fold_variant = 0;
  for (auto& a : g_tune)
    for (auto& b : a)
      for (auto& c : b)
        for (auto& e : c)
          for (auto& f : e) f = NttChoice{0, 0};
}

// ---------------------------------------------------------------------------
// Register-resident NTT for 16 <= n <= 4096 (q < 2^62, which the tables
// guarantee).  Each thread holds 16 coefficients of one transform unit (a
// full polynomial, or one half of a ring element in incomplete mode) and runs
// up to 4 butterfly stages on them in registers between exchanges through
// shared memory, so a 1024-point transform takes 3 exchanges instead of 10.
// Butterflies are Harvey's lazy variants of the Cooley-Tukey (forward) and
// Gentleman-Sande (inverse) butterflies with Shoup multiplication: forward
// values stay in [0, 4q) and inverse values in [0, 2q), which needs 4q < 2^64;
// one correction at the end makes the outputs canonical, so they equal the
// fully reduced transform exactly.
//
// For q < 2^50 (the protocol's primes) the RELAX variants drop the per-
// butterfly corrections: forward values grow by at most 2q per stage, so stay
// below (2 log n + 1) q, and inverse sums at most double per stage, so stay
// below 2^(log n) q, with the difference offset by C = 2^(log n) q instead of
// 2q; both bounds are far below 2^63 for log n <= 12.  One Shoup reduction by
// 1 (x - floor(x floor(2^64/q) / 2^64) q, in [0, 2q)) and a subtraction make
// the outputs canonical.
//
// Stage numbering follows the generic kernel above: forward stage g pairs
// elements t = n >> (g+1) apart with twiddle fwd[2^g + j / 2t]; inverse stage
// g pairs elements t = 2^g apart with twiddle inv[(n >> (g+1)) + j / 2t].  A
// phase covering stages g0 .. g0+S-1 gives each thread "mini-blocks" of 2^S
// elements e = blk * (stride << S) + r + k * stride, k < 2^S, whose pairs in
// all S stages stay inside the mini-block (stride = n >> (g0+S) forward,
// 2^g0 inverse).
//
// The first phase reads global memory and the last writes it directly: the
// strided side (forward input, inverse output) is coalesced across lanes,
// including the even/odd interleave of incomplete mode (lanes alternate
// halves); the contiguous side (forward output, inverse input: 2^S
// consecutive coefficients per thread) uses 16-byte vector accesses, so it
// needs 16-byte aligned buffers.  Shared memory holds 4096 coefficients with
// one padding word every 16 to spread the strided phases over the banks.
// ---------------------------------------------------------------------------
namespace {

__host__ __device__ constexpr int ph_count(int L) { return (L + 3) / 4; }
__host__ __device__ constexpr int ph_size(int L, int p) { return L / ph_count(L) + (p < L % ph_count(L) ? 1 : 0); }
__host__ __device__ constexpr int ph_start(int L, int p) { return p == 0 ? 0 : ph_start(L, p - 1) + ph_size(L, p - 1); }

constexpr u32 NR_TILE = 4096;  // coefficients per CTA
constexpr u64 NR_RELAX_Q = 1ULL << 50;  // below this, butterflies skip their corrections
__device__ __forceinline__ u32 npad(u32 p) { return p + (p >> 4); }

// x * w mod q in [0, 2q) for any 64-bit x (Shoup, without the final correction)
__device__ __forceinline__ u64 shoup_lazy(u64 x, u64 w, u64 wp, u64 q) { return x * w - __umul64hi(x, wp) * q; }

struct NrCtx {
  const NttDev* T;
  u64 q, q2;
};

// Butterflies of phase P on one mini-block v[0 .. 2^S) with block index blk.
template <int LOGN, int P, bool INV, bool RELAX>
__device__ __forceinline__ void nr_block(u64* v, u32 blk, const NttDev& T, u64 q, u64 q2) {
  // inverse difference offset: 2q, or 2^LOGN q when sums are left unreduced
  const u64 cdiff = RELAX ? (q << LOGN) : q2;
  constexpr int S = ph_size(LOGN, P), G0 = ph_start(LOGN, P);
  constexpr u32 N = 1u << LOGN, K = 1u << S;
  // pairs p < 2^(S-1) of level l: k = (sb << (l'+1)) + kk, one twiddle per sb
#pragma unroll
  for (int l = 0; l < S; l++) {
    const u32 lt = INV ? l : S - 1 - l;  // log2 of the pair distance in k
    const u32 t = 1u << lt;
    u64 w = 0, wp = 0;
#pragma unroll
    for (u32 p = 0; p < K / 2; p++) {
      const u32 sb = p >> lt, kk = p & (t - 1), k = (sb << (lt + 1)) + kk;
      if (kk == 0) {
        const u32 idx = INV ? (N >> (G0 + l + 1)) + (blk << (S - l - 1)) + sb : (1u << (G0 + l)) + (blk << l) + sb;
        w = __ldg((INV ? T.inv : T.fwd) + idx);
        wp = __ldg((INV ? T.invp : T.fwdp) + idx);
      }
      if (!INV) {
        u64 a = v[k];
        if (!RELAX) a = a >= q2 ? a - q2 : a;
        const u64 b = shoup_lazy(v[k + t], w, wp, q);
        v[k] = a + b;
        v[k + t] = a - b + q2;
      } else {
        const u64 a = v[k], b = v[k + t];
        u64 s2 = a + b;
        if (!RELAX) s2 = s2 >= q2 ? s2 - q2 : s2;
        v[k] = s2;
        v[k + t] = shoup_lazy(a - b + cdiff, w, wp, q);
      }
    }
  }
}

template <int LOGN, int P, bool INV, bool RELAX>
__device__ __forceinline__ void nr_compute(u64 (&x)[16], u32 tu, const NttDev& T, u64 q, u64 q2) {
  constexpr int S = ph_size(LOGN, P), G0 = ph_start(LOGN, P);
  constexpr u32 N = 1u << LOGN, TPU = N / 16, MB = 16 >> S;
  constexpr u32 LSTR = INV ? G0 : LOGN - G0 - S;  // log2(stride)
#pragma unroll
  for (u32 j = 0; j < MB; j++) nr_block<LOGN, P, INV, RELAX>(x + j * (1u << S), (tu + j * TPU) >> LSTR, T, q, q2);
}

// element index (within its unit) of register (j, k) in phase P
template <int LOGN, int P, bool INV>
__device__ __forceinline__ u32 nr_elem(u32 tu, u32 j, u32 k) {
  constexpr int S = ph_size(LOGN, P), G0 = ph_start(LOGN, P);
  constexpr u32 N = 1u << LOGN, TPU = N / 16;
  constexpr u32 LSTR = INV ? G0 : LOGN - G0 - S;
  const u32 mb = tu + j * TPU, blk = mb >> LSTR, r = mb & ((1u << LSTR) - 1);
  return (blk << (LSTR + S)) + r + (k << LSTR);
}

// Shared-memory exchange: a thread reads and writes the same positions within
// a phase, so a phase can update the tile in place.
template <int LOGN, int P, bool INV, typename W>
__device__ __forceinline__ void nr_load_smem(W (&x)[16], const W* sm, u32 unit, u32 tu) {
  constexpr int S = ph_size(LOGN, P);
  constexpr u32 N = 1u << LOGN, MB = 16 >> S, K = 1u << S;
#pragma unroll
  for (u32 j = 0; j < MB; j++)
#pragma unroll
    for (u32 k = 0; k < K; k++) x[j * K + k] = sm[npad(unit * N + nr_elem<LOGN, P, INV>(tu, j, k))];
}
template <int LOGN, int P, bool INV, typename W>
__device__ __forceinline__ void nr_store_smem(const W (&x)[16], W* sm, u32 unit, u32 tu) {
  constexpr int S = ph_size(LOGN, P);
  constexpr u32 N = 1u << LOGN, MB = 16 >> S, K = 1u << S;
#pragma unroll
  for (u32 j = 0; j < MB; j++)
#pragma unroll
    for (u32 k = 0; k < K; k++) sm[npad(unit * N + nr_elem<LOGN, P, INV>(tu, j, k))] = x[j * K + k];
}

// Global side of the first phase (P = 0).
template <int LOGN, bool INC, bool INV>
__device__ __forceinline__ void nr_load_global(u64 (&x)[16], const u64* __restrict__ in, u64 ug, u32 tu) {
  constexpr int S = ph_size(LOGN, 0);
  constexpr u32 N = 1u << LOGN, MB = 16 >> S, K = 1u << S;
  if (!INV) {  // strided: e = r + k * stride (blk = 0), coalesced across lanes
#pragma unroll
    for (u32 j = 0; j < MB; j++)
#pragma unroll
      for (u32 k = 0; k < K; k++) {
        const u32 e = nr_elem<LOGN, 0, INV>(tu, j, k);
        const u64 g = INC ? (ug >> 1) * (2 * N) + 2 * e + (ug & 1) : ug * N + e;
        x[j * K + k] = __ldg(in + g);
      }
  } else {  // contiguous 2^S coefficients per mini-block
#pragma unroll
    for (u32 j = 0; j < MB; j++) {
      const ulonglong2* src = (const ulonglong2*)(in + ug * N + nr_elem<LOGN, 0, INV>(tu, j, 0));
#pragma unroll
      for (u32 k = 0; k < K / 2; k++) {
        const ulonglong2 v = __ldg(src + k);
        x[j * K + 2 * k] = v.x;
        x[j * K + 2 * k + 1] = v.y;
      }
    }
  }
}

__device__ __forceinline__ u64 nr_canon4(u64 a, u64 q, u64 q2) {  // [0, 4q) -> [0, q)
  a = a >= q2 ? a - q2 : a;
  return a >= q ? a - q : a;
}
// forward output -> [0, q): [0, 4q) normally, any value below 2^64 when relaxed
template <bool RELAX>
__device__ __forceinline__ u64 nr_canon(u64 a, u64 q, u64 q2, u64 onep) {
  if (!RELAX) return nr_canon4(a, q, q2);
  a = shoup_lazy(a, 1, onep, q);
  return a >= q ? a - q : a;
}

// Global side of the last phase: canonical forward output (contiguous), or
// the inverse output scaled by 1/n (strided).
__device__ __forceinline__ u64 nr_mag(u64 v, u64 q) { return 2 * v > q ? q - v : v; }

template <int LOGN, bool INC, bool INV, bool RELAX>
__device__ __forceinline__ void nr_store_global(const u64 (&x)[16], u64* __restrict__ out, u64 ug, u32 tu,
                                                const NttDev& T, u64 q, u64 q2, u64* mag = nullptr) {
  constexpr int P = ph_count(LOGN) - 1, S = ph_size(LOGN, P);
  constexpr u32 N = 1u << LOGN, MB = 16 >> S, K = 1u << S;
  if (!INV) {
#pragma unroll
    for (u32 j = 0; j < MB; j++) {
      ulonglong2* dst = (ulonglong2*)(out + ug * N + nr_elem<LOGN, P, INV>(tu, j, 0));
#pragma unroll
      for (u32 k = 0; k < K / 2; k++)
        dst[k] = make_ulonglong2(nr_canon<RELAX>(x[j * K + 2 * k], q, q2, T.onep),
                                 nr_canon<RELAX>(x[j * K + 2 * k + 1], q, q2, T.onep));
    }
  } else {
#pragma unroll
    for (u32 j = 0; j < MB; j++)
#pragma unroll
      for (u32 k = 0; k < K; k++) {
        const u32 e = nr_elem<LOGN, P, INV>(tu, j, k);
        u64 v = shoup_lazy(x[j * K + k], T.ninv, T.ninvp, q);
        v = v >= q ? v - q : v;
        const u64 g = INC ? (ug >> 1) * (2 * N) + 2 * e + (ug & 1) : ug * N + e;
        out[g] = v;
        if (mag) *mag |= nr_mag(v, q);
      }
  }
}

// Phases P .. PEND-1 entirely through shared memory.
template <int LOGN, int P, int PEND, bool INV, bool RELAX>
__device__ __forceinline__ void nr_mid(u64 (&x)[16], u64* sm, u32 unit, u32 tu, bool active, const NttDev& T,
                                       u64 q, u64 q2) {
  if constexpr (P < PEND) {
    if (active) {
      nr_load_smem<LOGN, P, INV>(x, sm, unit, tu);
      nr_compute<LOGN, P, INV, RELAX>(x, tu, T, q, q2);
      nr_store_smem<LOGN, P, INV>(x, sm, unit, tu);
    }
    __syncthreads();
    nr_mid<LOGN, P + 1, PEND, INV, RELAX>(x, sm, unit, tu, active, T, q, q2);
  }
}

// Thread -> (unit in tile, thread within unit); in incomplete mode lanes
// alternate the two halves of an element so the interleaved side coalesces.
template <int LOGN, bool INC>
__device__ __forceinline__ void nr_map(u32 tid, u32& unit, u32& tu) {
  constexpr u32 TPU = (1u << LOGN) / 16;
  if (INC) {
    unit = 2 * (tid / (2 * TPU)) + (tid & 1);
    tu = (tid % (2 * TPU)) >> 1;
  } else {
    unit = tid / TPU;
    tu = tid % TPU;
  }
}

// One 4096-coefficient tile (tile index blk) of a batch of `units` units;
// sm is the CTA's padded exchange tile.  Called by the single-batch kernel
// with blk = blockIdx.x and by the multi-batch kernel with its local tile.
template <int LOGN, bool INC, bool INV, bool RELAX>
__device__ __forceinline__ void nr_tile(const u64* in, u64* out, u64 units, u64 blk, const NttDev& T, u64* mag_or,
                                        u64* sm) {
  constexpr u32 N = 1u << LOGN, UPT = NR_TILE / N;
  constexpr int NPH = ph_count(LOGN);
  static_assert(!INC || UPT % 2 == 0, "incomplete mode keeps both halves of an element in one tile");
  u32 unit, tu;
  nr_map<LOGN, INC>(threadIdx.x, unit, tu);
  const u64 ug = blk * UPT + unit;
  const bool active = ug < units;
  const u64 q = T.q, q2 = 2 * T.q;
  u64 x[16], mag = 0;
  if (active) {
    nr_load_global<LOGN, INC, INV>(x, in, ug, tu);
    if (!INV && mag_or)
#pragma unroll
      for (u32 i = 0; i < 16; i++) mag |= nr_mag(x[i], q);
    nr_compute<LOGN, 0, INV, RELAX>(x, tu, T, q, q2);
  }
  if constexpr (NPH > 1) {
    if (active) nr_store_smem<LOGN, 0, INV>(x, sm, unit, tu);
    __syncthreads();
    nr_mid<LOGN, 1, NPH - 1, INV, RELAX>(x, sm, unit, tu, active, T, q, q2);
    if (active) {
      nr_load_smem<LOGN, NPH - 1, INV>(x, sm, unit, tu);
      nr_compute<LOGN, NPH - 1, INV, RELAX>(x, tu, T, q, q2);
    }
  }
  if (active) nr_store_global<LOGN, INC, INV, RELAX>(x, out, ug, tu, T, q, q2, INV && mag_or ? &mag : nullptr);
  if (mag_or) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mag |= __shfl_xor_sync(0xffffffffu, mag, o);
    if ((threadIdx.x & 31) == 0 && mag) atomicOr((unsigned long long*)mag_or, (unsigned long long)mag);
  }
}

template <int LOGN, bool INC, bool INV, bool RELAX>
__global__ void __launch_bounds__(256) ntt_reg_kernel(const u64* in, u64* out, u64 units, NttDev T, u64* mag_or) {
  __shared__ u64 sm[NR_TILE + NR_TILE / 16];
  nr_tile<LOGN, INC, INV, RELAX>(in, out, units, blockIdx.x, T, mag_or, sm);
}

// ---------------------------------------------------------------------------
// Bulk-copy staged ("pipe") variant of the register NTT.  The transform is
// memory-latency bound for short n: one tile per CTA leaves the loads of the
// next tile waiting behind the butterflies of this one.  Here each CTA is
// persistent over tiles blockIdx.x, blockIdx.x + gridDim.x, ...; a tile's
// input is contiguous in global memory (4096 coefficients = 32 KiB, whole
// units or ring elements), so one thread fetches it with one
// cp.async.bulk into a ring of STAGES shared-memory buffers, completing on
// that stage's mbarrier, STAGES tiles ahead of the tile being transformed.
// The first butterfly phase reads its registers from the staged copy (the
// same element indices as the global loads of ntt_reg_kernel); the exchange
// phases and the global stores are those of ntt_reg_kernel.
//
// Every mbarrier wait is bounded (umma::SPIN_LIMIT polls).  A CTA whose wait
// gives up records it in g_ntt_error (read by ntt_error_check), waits
// (bounded) for the copies it still has in flight and stops.
// ---------------------------------------------------------------------------
__device__ u32 g_ntt_error;

template <int LOGN, bool INC, bool INV>
__device__ __forceinline__ void nr_load_stage(u64 (&x)[16], const u64* stg, u32 unit, u32 tu) {
  constexpr int S = ph_size(LOGN, 0);
  constexpr u32 N = 1u << LOGN, MB = 16 >> S, K = 1u << S;
#pragma unroll
  for (u32 j = 0; j < MB; j++)
#pragma unroll
    for (u32 k = 0; k < K; k++) {
      const u32 e = nr_elem<LOGN, 0, INV>(tu, j, k);
      const u32 g = (INC && !INV) ? (unit >> 1) * (2 * N) + 2 * e + (unit & 1) : unit * N + e;
      x[j * K + k] = stg[g];
    }
}

constexpr u32 NP_ERR_WAIT = 0x4e54u;  // "NT": a stage's bulk copy did not complete in time

// ---------------------------------------------------------------------------
// FP64 butterflies for q < 2^50 (the protocol's primes).  On B200 the FP64
// pipe multiplies and adds 53-bit integers exactly at a far higher rate than
// the 32-bit integer multipliers assemble 64-bit Shoup products, so these
// kernels keep the coefficients as integer-valued doubles and reduce with
// error-free transformations (Dekker's exact product via FMA, as used for
// modular arithmetic in floating point by van der Hoeven, Lecerf and Quintin,
// "Modular SIMD arithmetic in Mathemagix", ACM TOMS 2016):
//
//   x * w mod q, |x| < 2^52, 0 <= w < q:  h = fl(x w), l = x w - h (one FMA,
//   exact), c = nearest integer to x fl(w / 2q) (one FMA against the
//   rounding constant 1.5 * 2^52 and one subtraction), r = (h - 2q c) + l.
//   Since |x w / 2q - c| <= 0.625 the integer x w - 2q c has magnitude at most
//   1.25 q < 2^51, so the FMA h - 2q c and the addition of l are exact: r is
//   x w mod q as an integer in [-1.25 q, 1.25 q].
//
//   v mod q, |v| < 2^52: c = nearest integer to v fl(1/q), r = v - c q
//   (exact, in [-q/2 - 1, q/2 + 1]).
//
// Forward (Cooley-Tukey): inputs in [0, q); each stage adds at most 1.25 q
// to a magnitude; all values are reduced after every odd-numbered stage, so
// magnitudes stay below 4 q < 2^52 and multiplicands below 2.5 q.  Inverse
// (Gentleman-Sande): the sum a + b is reduced in every stage (magnitudes of
// sums below 3 q, of differences below 3 q, of products below 1.25 q).  The
// outputs are reduced once more and shifted into [0, q), so they are the
// canonical residues, the same words as the integer kernels produce.
// Conversions between canonical words and doubles go through the exponent
// bits of 2^52 (v + 2^52 has v in its low 52 mantissa bits), one integer
// and one FP64 instruction each.
// ---------------------------------------------------------------------------
// Butterflies of phase P on one mini-block v[0 .. 2^S) with block index blk.
template <int LOGN, int P, bool INV>
__device__ __forceinline__ void nf_block(double* v, u32 blk, const NttDev& T) {
  constexpr int S = ph_size(LOGN, P), G0 = ph_start(LOGN, P);
  constexpr u32 N = 1u << LOGN, K = 1u << S;
  const double q2d = T.q2d, qd = T.qd, qinv = T.qinv;
#pragma unroll
  for (int l = 0; l < S; l++) {
    const u32 lt = INV ? l : S - 1 - l;
    const u32 t = 1u << lt;
    double w = 0, wh = 0;
#pragma unroll
    for (u32 p = 0; p < K / 2; p++) {
      const u32 sb = p >> lt, kk = p & (t - 1), k = (sb << (lt + 1)) + kk;
      if (kk == 0) {
        const u32 idx = INV ? (N >> (G0 + l + 1)) + (blk << (S - l - 1)) + sb : (1u << (G0 + l)) + (blk << l) + sb;
        w = __ldg((INV ? T.inv_d : T.fwd_d) + idx);
        wh = __ldg((INV ? T.inv_h : T.fwd_h) + idx);
      }
      const double a = v[k], b = v[k + t];
      if (!INV) {
        const double m = fp_mulmod(b, w, wh, q2d);
        v[k] = __dadd_rn(a, m);
        v[k + t] = __dsub_rn(a, m);
      } else {
        v[k] = fp_reduce(__dadd_rn(a, b), qinv, qd);
        v[k + t] = fp_mulmod(__dsub_rn(a, b), w, wh, q2d);
      }
    }
    if (!INV && ((G0 + l) & 1)) {
#pragma unroll
      for (u32 i = 0; i < K; i++) v[i] = fp_reduce(v[i], qinv, qd);
    }
  }
}

template <int LOGN, int P, bool INV>
__device__ __forceinline__ void nf_compute(double (&x)[16], u32 tu, const NttDev& T) {
  constexpr int S = ph_size(LOGN, P), G0 = ph_start(LOGN, P);
  constexpr u32 N = 1u << LOGN, TPU = N / 16, MB = 16 >> S;
  constexpr u32 LSTR = INV ? G0 : LOGN - G0 - S;
#pragma unroll
  for (u32 j = 0; j < MB; j++) nf_block<LOGN, P, INV>(x + j * (1u << S), (tu + j * TPU) >> LSTR, T);
}

// First-phase loads (as nr_load_global) converted to doubles; the OR of the
// centred magnitudes of the loaded words goes to *mag when mag is not null.
template <int LOGN, bool INC, bool INV>
__device__ __forceinline__ void nf_load_global(double (&x)[16], const u64* __restrict__ in, u64 ug, u32 tu,
                                               u64 q, u64* mag) {
  u64 w[16];
  nr_load_global<LOGN, INC, INV>(w, in, ug, tu);
#pragma unroll
  for (u32 i = 0; i < 16; i++) {
    if (mag) *mag |= nr_mag(w[i], q);
    x[i] = fp_from_word(w[i]);
  }
}

// Last-phase stores (as nr_store_global): canonical words, the inverse scaled by 1/n.
template <int LOGN, bool INC, bool INV>
__device__ __forceinline__ void nf_store_global(const double (&x)[16], u64* __restrict__ out, u64 ug, u32 tu,
                                                const NttDev& T, u64* mag) {
  constexpr int P = ph_count(LOGN) - 1, S = ph_size(LOGN, P);
  constexpr u32 N = 1u << LOGN, MB = 16 >> S, K = 1u << S;
  const double qd = T.qd, qinv = T.qinv;
  if (!INV) {
#pragma unroll
    for (u32 j = 0; j < MB; j++) {
      ulonglong2* dst = (ulonglong2*)(out + ug * N + nr_elem<LOGN, P, INV>(tu, j, 0));
#pragma unroll
      for (u32 k = 0; k < K / 2; k++)
        dst[k] = make_ulonglong2(fp_to_word(x[j * K + 2 * k], qinv, qd), fp_to_word(x[j * K + 2 * k + 1], qinv, qd));
    }
  } else {
#pragma unroll
    for (u32 j = 0; j < MB; j++)
#pragma unroll
      for (u32 k = 0; k < K; k++) {
        const u32 e = nr_elem<LOGN, P, INV>(tu, j, k);
        const u64 v = fp_to_word(fp_mulmod(x[j * K + k], T.ninv_d, T.ninv_h, T.q2d), qinv, qd);
        const u64 g = INC ? (ug >> 1) * (2 * N) + 2 * e + (ug & 1) : ug * N + e;
        out[g] = v;
        if (mag) *mag |= nr_mag(v, T.q);
      }
  }
}

template <int LOGN, int P, int PEND, bool INV>
__device__ __forceinline__ void nf_mid(double (&x)[16], double* sm, u32 unit, u32 tu, bool active, const NttDev& T) {
  if constexpr (P < PEND) {
    if (active) {
      nr_load_smem<LOGN, P, INV>(x, sm, unit, tu);
      nf_compute<LOGN, P, INV>(x, tu, T);
      nr_store_smem<LOGN, P, INV>(x, sm, unit, tu);
    }
    __syncthreads();
    nf_mid<LOGN, P + 1, PEND, INV>(x, sm, unit, tu, active, T);
  }
}

// The register NTT (ntt_reg_kernel's thread mapping, phases and exchanges)
// with FP64 butterflies; q < 2^50 and canonical inputs.
template <int LOGN, bool INC, bool INV>
__device__ __forceinline__ void nf_tile(const u64* in, u64* out, u64 units, u64 blk, const NttDev& T, u64* mag_or,
                                        double* sm) {
  constexpr u32 UPT = NR_TILE >> LOGN;
  constexpr int NPH = ph_count(LOGN);
  static_assert(!INC || UPT % 2 == 0, "incomplete mode keeps both halves of an element in one tile");
  u32 unit, tu;
  nr_map<LOGN, INC>(threadIdx.x, unit, tu);
  const u64 ug = blk * UPT + unit;
  const bool active = ug < units;
  double x[16];
  u64 mag = 0;
  if (active) {
    nf_load_global<LOGN, INC, INV>(x, in, ug, tu, T.q, !INV && mag_or ? &mag : nullptr);
    nf_compute<LOGN, 0, INV>(x, tu, T);
  }
  if constexpr (NPH > 1) {
    if (active) nr_store_smem<LOGN, 0, INV>(x, sm, unit, tu);
    __syncthreads();
    nf_mid<LOGN, 1, NPH - 1, INV>(x, sm, unit, tu, active, T);
    if (active) {
      nr_load_smem<LOGN, NPH - 1, INV>(x, sm, unit, tu);
      nf_compute<LOGN, NPH - 1, INV>(x, tu, T);
    }
  }
  if (active) nf_store_global<LOGN, INC, INV>(x, out, ug, tu, T, INV && mag_or ? &mag : nullptr);
  if (mag_or) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mag |= __shfl_xor_sync(0xffffffffu, mag, o);
    if ((threadIdx.x & 31) == 0 && mag) atomicOr((unsigned long long*)mag_or, (unsigned long long)mag);
  }
}

template <int LOGN, bool INC, bool INV>
__global__ void __launch_bounds__(256) ntt_fp_kernel(const u64* in, u64* out, u64 units, NttDev T, u64* mag_or) {
  __shared__ double sm[NR_TILE + NR_TILE / 16];
  nf_tile<LOGN, INC, INV>(in, out, units, blockIdx.x, T, mag_or, sm);
}

// ---------------------------------------------------------------------------
// Incomplete transforms of degree-128 ring elements (two 64-point halves)
// with FP64 butterflies, one thread per (element, column r < 8) holding
// both halves: 8 coefficients of each, e = r + 8k in the strided phase and
// e = 8r + k in the contiguous one.  The same butterflies and exchange as
// ntt_fp_kernel<6, true, INV> (identical words), with fewer L1 wavefronts
// per coefficient, the limit of that kernel: the interleaved side moves one
// 16-byte (half 0, half 1) pair per load or store, 8 lanes covering 128
// contiguous bytes of an element; the slot-form side moves 32 bytes per
// lane (256-bit loads and stores, rows 32-byte aligned); the exchange tile
// holds (half 0, half 1) pairs with 16 bytes of padding per 8 pairs, so
// both exchange patterns are free of bank conflicts.
// ---------------------------------------------------------------------------
constexpr u32 NP6_EL = 32;   // ring elements per CTA (4096 coefficients)
constexpr u32 NP6_ROW = 72;  // pairs per element in the exchange tile (64 + 8 padding)
__device__ __forceinline__ u32 np6_pos(u32 el, u32 e) { return el * NP6_ROW + e + (e >> 3); }

__device__ __forceinline__ void st_v4_u64(u64* p, u64 a, u64 b, u64 c, u64 d) {
  asm volatile("st.global.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(p), "l"(a), "l"(b), "l"(c), "l"(d) : "memory");
}
__device__ __forceinline__ void ld_v4_u64(const u64* p, u64& a, u64& b, u64& c, u64& d) {
  asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(p));
}

// Strided phase of the forward transform, exchange and contiguous phase;
// x0 / x1 hold half 0 / 1 at e = r + 8k on entry and at e = 8r + k on exit.
__device__ __forceinline__ void np6_forward(double (&x0)[8], double (&x1)[8], double2* sm, u32 el, u32 r,
                                            bool active, const NttDev& T) {
  if (active) {
    nf_block<6, 0, false>(x0, 0, T);
    nf_block<6, 0, false>(x1, 0, T);
#pragma unroll
    for (u32 k = 0; k < 8; k++) sm[np6_pos(el, r + 8 * k)] = make_double2(x0[k], x1[k]);
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (u32 k = 0; k < 8; k++) {
      const double2 v = sm[np6_pos(el, 8 * r + k)];
      x0[k] = v.x;
      x1[k] = v.y;
    }
    nf_block<6, 1, false>(x0, r, T);
    nf_block<6, 1, false>(x1, r, T);
  }
}

// Canonical words of the slot-form rows (2 e + h) of element e: 32 bytes per store.
__device__ __forceinline__ void np6_store_slots(const double (&x0)[8], const double (&x1)[8], u64* out, u64 eg,
                                                u32 r, const NttDev& T) {
  const double qd = T.qd, qinv = T.qinv;
  u64* d0 = out + 2 * eg * 64 + 8 * r;
#pragma unroll
  for (u32 h = 0; h < 2; h++) {
    const double* x = h ? x1 : x0;
#pragma unroll
    for (u32 c = 0; c < 2; c++)
      st_v4_u64(d0 + h * 64 + 4 * c, fp_to_word(x[4 * c], qinv, qd), fp_to_word(x[4 * c + 1], qinv, qd),
                fp_to_word(x[4 * c + 2], qinv, qd), fp_to_word(x[4 * c + 3], qinv, qd));
  }
}

template <bool INV>
__global__ void __launch_bounds__(256) ntt_fp6_kernel(const u64* in, u64* out, u64 count, NttDev T, u64* mag_or) {
  __shared__ double2 sm[NP6_EL * NP6_ROW];
  const u32 el = threadIdx.x >> 3, r = threadIdx.x & 7;
  const u64 eg = (u64)blockIdx.x * NP6_EL + el;
  const bool active = eg < count;
  const double qd = T.qd, qinv = T.qinv;
  double x0[8], x1[8];
  u64 mag = 0;
  if (!INV) {
    if (active) {
      const u64* src = in + eg * 128;
#pragma unroll
      for (u32 k = 0; k < 8; k++) {
        const ulonglong2 v = __ldg((const ulonglong2*)(src + 2 * (r + 8 * k)));
        if (mag_or) mag |= nr_mag(v.x, T.q) | nr_mag(v.y, T.q);
        x0[k] = fp_from_word(v.x);
        x1[k] = fp_from_word(v.y);
      }
    }
    np6_forward(x0, x1, sm, el, r, active, T);
    if (active) np6_store_slots(x0, x1, out, eg, r, T);
  } else {
    if (active) {
      const u64* s0 = in + 2 * eg * 64 + 8 * r;
#pragma unroll
      for (u32 h = 0; h < 2; h++) {
        double* x = h ? x1 : x0;
#pragma unroll
        for (u32 c = 0; c < 2; c++) {
          u64 a, b, cc, dd;
          ld_v4_u64(s0 + h * 64 + 4 * c, a, b, cc, dd);
          x[4 * c] = fp_from_word(a);
          x[4 * c + 1] = fp_from_word(b);
          x[4 * c + 2] = fp_from_word(cc);
          x[4 * c + 3] = fp_from_word(dd);
        }
      }
      nf_block<6, 0, true>(x0, r, T);
      nf_block<6, 0, true>(x1, r, T);
#pragma unroll
      for (u32 k = 0; k < 8; k++) sm[np6_pos(el, 8 * r + k)] = make_double2(x0[k], x1[k]);
    }
    __syncthreads();
    if (active) {
#pragma unroll
      for (u32 k = 0; k < 8; k++) {
        const double2 v = sm[np6_pos(el, r + 8 * k)];
        x0[k] = v.x;
        x1[k] = v.y;
      }
      nf_block<6, 1, true>(x0, 0, T);
      nf_block<6, 1, true>(x1, 0, T);
      u64* dst = out + eg * 128;
#pragma unroll
      for (u32 k = 0; k < 8; k++) {
        const u64 a = fp_to_word(fp_mulmod(x0[k], T.ninv_d, T.ninv_h, T.q2d), qinv, qd);
        const u64 b = fp_to_word(fp_mulmod(x1[k], T.ninv_d, T.ninv_h, T.q2d), qinv, qd);
        *(ulonglong2*)(dst + 2 * (r + 8 * k)) = make_ulonglong2(a, b);
        if (mag_or) mag |= nr_mag(a, T.q) | nr_mag(b, T.q);
      }
    }
  }
  if (mag_or) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mag |= __shfl_xor_sync(0xffffffffu, mag, o);
    if ((threadIdx.x & 31) == 0 && mag) atomicOr((unsigned long long*)mag_or, (unsigned long long)mag);
  }
}

// Full (not incomplete) 64-point transforms with integer butterflies in the
// same paired layout: a thread holds column r of two neighbouring
// polynomials (x0: polynomial 2 p, x1: 2 p + 1), the exchange tile holds
// (x0, x1) pairs, and the contiguous side (forward output, inverse input)
// moves 32 bytes per lane.  Same butterflies and words as
// ntt_reg_kernel<6, false, INV, RELAX>.
template <bool INV, bool RELAX>
__global__ void __launch_bounds__(256) ntt_int6_kernel(const u64* in, u64* out, u64 units, NttDev T, u64* mag_or) {
  __shared__ ulonglong2 sm[NP6_EL * NP6_ROW];
  const u32 el = threadIdx.x >> 3, r = threadIdx.x & 7;
  const u64 u0 = 2 * ((u64)blockIdx.x * NP6_EL + el);
  const bool a0 = u0 < units, a1 = u0 + 1 < units;
  const u64 q = T.q, q2 = 2 * T.q;
  u64 x0[8], x1[8];
  u64 mag = 0;
#pragma unroll
  for (u32 k = 0; k < 8; k++) x0[k] = x1[k] = 0;
  if (!INV) {
#pragma unroll
    for (u32 k = 0; k < 8; k++) {
      if (a0) x0[k] = __ldg(in + u0 * 64 + r + 8 * k);
      if (a1) x1[k] = __ldg(in + (u0 + 1) * 64 + r + 8 * k);
      if (mag_or) mag |= (a0 ? nr_mag(x0[k], q) : 0) | (a1 ? nr_mag(x1[k], q) : 0);
    }
    if (a0) {
      nr_block<6, 0, false, RELAX>(x0, 0, T, q, q2);
      nr_block<6, 0, false, RELAX>(x1, 0, T, q, q2);
#pragma unroll
      for (u32 k = 0; k < 8; k++) sm[np6_pos(el, r + 8 * k)] = make_ulonglong2(x0[k], x1[k]);
    }
    __syncthreads();
    if (a0) {
#pragma unroll
      for (u32 k = 0; k < 8; k++) {
        const ulonglong2 v = sm[np6_pos(el, 8 * r + k)];
        x0[k] = v.x;
        x1[k] = v.y;
      }
      nr_block<6, 1, false, RELAX>(x0, r, T, q, q2);
      nr_block<6, 1, false, RELAX>(x1, r, T, q, q2);
#pragma unroll
      for (u32 h = 0; h < 2; h++) {
        if (h && !a1) break;
        const u64* x = h ? x1 : x0;
        u64* dst = out + (u0 + h) * 64 + 8 * r;
#pragma unroll
        for (u32 c = 0; c < 2; c++)
          st_v4_u64(dst + 4 * c, nr_canon<RELAX>(x[4 * c], q, q2, T.onep), nr_canon<RELAX>(x[4 * c + 1], q, q2, T.onep),
                    nr_canon<RELAX>(x[4 * c + 2], q, q2, T.onep), nr_canon<RELAX>(x[4 * c + 3], q, q2, T.onep));
      }
    }
  } else {
    if (a0) {
#pragma unroll
      for (u32 h = 0; h < 2; h++) {
        if (h && !a1) break;
        u64* x = h ? x1 : x0;
        const u64* src = in + (u0 + h) * 64 + 8 * r;
#pragma unroll
        for (u32 c = 0; c < 2; c++) ld_v4_u64(src + 4 * c, x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]);
      }
      nr_block<6, 0, true, RELAX>(x0, r, T, q, q2);
      nr_block<6, 0, true, RELAX>(x1, r, T, q, q2);
#pragma unroll
      for (u32 k = 0; k < 8; k++) sm[np6_pos(el, 8 * r + k)] = make_ulonglong2(x0[k], x1[k]);
    }
    __syncthreads();
    if (a0) {
#pragma unroll
      for (u32 k = 0; k < 8; k++) {
        const ulonglong2 v = sm[np6_pos(el, r + 8 * k)];
        x0[k] = v.x;
        x1[k] = v.y;
      }
      nr_block<6, 1, true, RELAX>(x0, 0, T, q, q2);
      nr_block<6, 1, true, RELAX>(x1, 0, T, q, q2);
#pragma unroll
      for (u32 k = 0; k < 8; k++) {
        u64 v0 = shoup_lazy(x0[k], T.ninv, T.ninvp, q);
        v0 = v0 >= q ? v0 - q : v0;
        out[u0 * 64 + r + 8 * k] = v0;
        if (mag_or) mag |= nr_mag(v0, q);
        if (a1) {
          u64 v1 = shoup_lazy(x1[k], T.ninv, T.ninvp, q);
          v1 = v1 >= q ? v1 - q : v1;
          out[(u0 + 1) * 64 + r + 8 * k] = v1;
          if (mag_or) mag |= nr_mag(v1, q);
        }
      }
    }
  }
  if (mag_or) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mag |= __shfl_xor_sync(0xffffffffu, mag, o);
    if ((threadIdx.x & 31) == 0 && mag) atomicOr((unsigned long long*)mag_or, (unsigned long long)mag);
  }
}

// The paired kernel's alignment needs: 16-byte interleaved side, 32-byte slot side.
bool np6_aligned(const u64* in, const u64* out, bool inverse) {
  const uintptr_t il = (uintptr_t)(inverse ? out : in), sl = (uintptr_t)(inverse ? in : out);
  return il % 16 == 0 && sl % 32 == 0;
}

// FP: FP64 butterflies (q < 2^50, the nf_* code), else the integer ones.
template <int LOGN, bool INC, bool INV, bool RELAX, int STAGES, bool FP>
__global__ void __launch_bounds__(256) ntt_pipe_kernel(const u64* in, u64* out, u64 units, NttDev T, u64* mag_or) {
  using Wd = typename std::conditional<FP, double, u64>::type;
  constexpr u32 N = 1u << LOGN, UPT = NR_TILE / N;
  constexpr int NPH = ph_count(LOGN);
  static_assert(!INC || UPT % 2 == 0, "incomplete mode keeps both halves of an element in one tile");
  extern __shared__ __align__(128) unsigned char np_smem[];
  uint64_t* bar = (uint64_t*)np_smem;                                // STAGES mbarriers
  u64* stg = (u64*)(np_smem + 128);                                  // STAGES x NR_TILE words
  Wd* sm = (Wd*)(stg + (size_t)STAGES * NR_TILE);                    // padded exchange tile
  u32 unit, tu;
  nr_map<LOGN, INC>(threadIdx.x, unit, tu);
  const u64 q = T.q, q2 = 2 * T.q;
  const u64 ntiles = (units + UPT - 1) / UPT;
  const u64 t0 = blockIdx.x, tstep = gridDim.x;
  // bytes of tile t (a partial last tile holds whole units)
  auto tile_bytes = [&](u64 t) -> u32 {
    const u64 left = units - t * UPT;
    return (u32)((left < UPT ? left : UPT) * N * sizeof(u64));
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) umma::mbar_init(&bar[s], 1);
    umma::mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      const u64 t = t0 + (u64)s * tstep;
      if (t >= ntiles) break;
      const u32 b = tile_bytes(t);
      umma::mbar_expect_tx(&bar[s], b);
      umma::bulk_g2s(stg + (size_t)s * NR_TILE, in + t * NR_TILE, b, &bar[s]);
    }
  }
  u64 mag = 0;
  u64 i = 0;
  for (u64 t = t0; t < ntiles; t += tstep, i++) {
    const int s = (int)(i % STAGES);
    const u32 par = (u32)((i / STAGES) & 1);
    const bool ok = umma::mbar_wait(&bar[s], par, nullptr, 0);
    if (__syncthreads_or(!ok)) {
      // give up: record it, let the copies issued for later tiles land, stop
      if (threadIdx.x == 0) {
        atomicMax(&g_ntt_error, NP_ERR_WAIT);
        for (u64 j = 0; j < (u64)STAGES && t + j * tstep < ntiles; j++) {
          const int sj = (int)((i + j) % STAGES);
          umma::mbar_wait(&bar[sj], (u32)(((i + j) / STAGES) & 1), nullptr, 0);
        }
      }
      break;
    }
    const u64 ug = t * UPT + unit;
    const bool active = ug < units;
    Wd x[16];
    if (active) {
      u64 wv[16];
      nr_load_stage<LOGN, INC, INV>(wv, stg + (size_t)s * NR_TILE, unit, tu);
      if (!INV && mag_or)
#pragma unroll
        for (u32 k = 0; k < 16; k++) mag |= nr_mag(wv[k], q);
      if constexpr (FP) {
#pragma unroll
        for (u32 k = 0; k < 16; k++) x[k] = fp_from_word(wv[k]);
        nf_compute<LOGN, 0, INV>(x, tu, T);
      } else {
#pragma unroll
        for (u32 k = 0; k < 16; k++) x[k] = wv[k];
        nr_compute<LOGN, 0, INV, RELAX>(x, tu, T, q, q2);
      }
    }
    // Stage s is refilled with the tile STAGES ahead only after every thread
    // has consumed its values (the butterflies above use them) and ordered its
    // generic-proxy reads before the bulk copy's async-proxy writes.
    umma::fence_proxy_async();
    if constexpr (NPH > 1)
      if (active) nr_store_smem<LOGN, 0, INV>(x, sm, unit, tu);
    __syncthreads();
    if (threadIdx.x == 0) {
      const u64 tn = t + (u64)STAGES * tstep;
      if (tn < ntiles) {
        const u32 b = tile_bytes(tn);
        umma::mbar_expect_tx(&bar[s], b);
        umma::bulk_g2s(stg + (size_t)s * NR_TILE, in + tn * NR_TILE, b, &bar[s]);
      }
    }
    if constexpr (NPH > 1) {
      if constexpr (FP)
        nf_mid<LOGN, 1, NPH - 1, INV>(x, sm, unit, tu, active, T);
      else
        nr_mid<LOGN, 1, NPH - 1, INV, RELAX>(x, sm, unit, tu, active, T, q, q2);
      if (active) {
        nr_load_smem<LOGN, NPH - 1, INV>(x, sm, unit, tu);
        if constexpr (FP)
          nf_compute<LOGN, NPH - 1, INV>(x, tu, T);
        else
          nr_compute<LOGN, NPH - 1, INV, RELAX>(x, tu, T, q, q2);
      }
    }
    if (active) {
      if constexpr (FP)
        nf_store_global<LOGN, INC, INV>(x, out, ug, tu, T, INV && mag_or ? &mag : nullptr);
      else
        nr_store_global<LOGN, INC, INV, RELAX>(x, out, ug, tu, T, q, q2, INV && mag_or ? &mag : nullptr);
    }
  }
  if (mag_or) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mag |= __shfl_xor_sync(0xffffffffu, mag, o);
    if ((threadIdx.x & 31) == 0 && mag) atomicOr((unsigned long long*)mag_or, (unsigned long long)mag);
  }
}

// ---------------------------------------------------------------------------
// Many uneven batches of one transform shape in one launch (the batched form
// used by salsaa_ntt_multi): batch i owns the CTAs [bstart[i], bstart[i+1]),
// one 4096-coefficient tile each, found by a binary search over bstart.
// ---------------------------------------------------------------------------
struct NttMulti {
  const u64* in[NTT_MULTI_MAX];
  u64* out[NTT_MULTI_MAX];
  u64 units[NTT_MULTI_MAX];
  u64 bstart[NTT_MULTI_MAX + 1];
  u32 count;
};

template <int LOGN, bool INC, bool INV, bool RELAX, bool FP>
__global__ void __launch_bounds__(256) ntt_multi_kernel(NttMulti m, NttDev T) {
  __shared__ u64 sm[NR_TILE + NR_TILE / 16];
  const u64 b = blockIdx.x;
  u32 lo = 0, hi = m.count;  // invariant: bstart[lo] <= b < bstart[hi]
  while (hi - lo > 1) {
    const u32 mid = (lo + hi) / 2;
    if (m.bstart[mid] <= b) lo = mid;
    else hi = mid;
  }
  if constexpr (FP)
    nf_tile<LOGN, INC, INV>(m.in[lo], m.out[lo], m.units[lo], b - m.bstart[lo], T, nullptr, (double*)sm);
  else
    nr_tile<LOGN, INC, INV, RELAX>(m.in[lo], m.out[lo], m.units[lo], b - m.bstart[lo], T, nullptr, sm);
}

// Digit decomposition (decomp_ell, src/subroutines/decomp.rs:32-67) fused
// with the forward incomplete transform.  Ring element r of the digit space is
// (source element (k, i), digit c) with c fastest, so the warps that produce
// the digits of one source element load the same addresses and HBM sees the
// source once; digit c = ((pos >> c rlog) & mask) - ((neg >> c rlog) & mask)
// of the centre-lifted coefficient (pos or neg its magnitude) goes to row
// k * parts + c of dc, and its transform to the same row of ds.
template <int LOGN, bool RELAX, bool FP>
__global__ void __launch_bounds__(256)
    ntt_digits_kernel(NttSrcRows src, u64 width, u32 parts, const u64* bw_or, u64* rlog_out, u64* radix_out, u64* dc,
                      u64* ds, u64 units, NttDev T, bool narrow) {
  // FP: the FP64 butterflies (q < 2^50), else the integer ones.  narrow: the
  // coefficient-form digits go to dc as centred int32 values (parts >= 2, so
  // |digit| < radix <= 2^25), else as canonical words.
  using Wd = typename std::conditional<FP, double, u64>::type;
  constexpr u32 N = 1u << LOGN, UPT = NR_TILE / N, D = 2 * N;
  constexpr int NPH = ph_count(LOGN);
  constexpr int S0 = ph_size(LOGN, 0);
  constexpr u32 MB = 16 >> S0, KB = 1u << S0;
  __shared__ Wd sm[NR_TILE + NR_TILE / 16];
  u32 unit, tu;
  nr_map<LOGN, true>(threadIdx.x, unit, tu);
  const u64 ug = (u64)blockIdx.x * UPT + unit;
  const bool active = ug < units;
  const u64 q = T.q, q2 = 2 * T.q;
  const u64 orv = *bw_or;
  const u32 bw = orv ? 64u - (u32)__clzll((long long)orv) : 0u;
  const u32 rlog = (bw + parts - 1) / parts;
  const u64 mask = rlog >= 64 ? ~0ULL : ((1ULL << rlog) - 1);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *rlog_out = rlog;
    if (radix_out) *radix_out = 1ULL << rlog;
  }
  const u64 re = ug >> 1, h = ug & 1;
  const u32 c = (u32)(re % parts);
  const u64 se = re / parts;
  const u32 k = (u32)(se / width);
  const u64 i = se % width;
  const u64 dring = ((u64)k * parts + c) * width + i;  // output ring element
  const u32 sh = rlog * c;
  Wd x[16];
  if (active) {
    const u64* sp = src.p[k] + i * D + h;
    u64* dco = dc + dring * D + h;
    int* dcn = (int*)dc + dring * D + h;
#pragma unroll
    for (u32 j = 0; j < MB; j++)
#pragma unroll
      for (u32 kk = 0; kk < KB; kk++) {
        const u32 e = nr_elem<LOGN, 0, false>(tu, j, kk);
        const u64 v = __ldg(sp + 2 * e);
        const u64 pos = 2 * v > q ? 0 : v, neg = 2 * v > q ? q - v : 0;
        const u64 pd = sh >= 64 ? 0 : ((pos >> sh) & mask), nd = sh >= 64 ? 0 : ((neg >> sh) & mask);
        const u64 dv = pd >= nd ? pd - nd : pd + q - nd;
        if constexpr (FP)
          x[j * KB + kk] = fp_from_word(dv);
        else
          x[j * KB + kk] = dv;
        if (narrow)
          dcn[2 * e] = (int)((long long)pd - (long long)nd);
        else
          dco[2 * e] = dv;
      }
    if constexpr (FP)
      nf_compute<LOGN, 0, false>(x, tu, T);
    else
      nr_compute<LOGN, 0, false, RELAX>(x, tu, T, q, q2);
  }
  if constexpr (NPH > 1) {
    if (active) nr_store_smem<LOGN, 0, false>(x, sm, unit, tu);
    __syncthreads();
    if constexpr (FP)
      nf_mid<LOGN, 1, NPH - 1, false>(x, sm, unit, tu, active, T);
    else
      nr_mid<LOGN, 1, NPH - 1, false, RELAX>(x, sm, unit, tu, active, T, q, q2);
    if (active) {
      nr_load_smem<LOGN, NPH - 1, false>(x, sm, unit, tu);
      if constexpr (FP)
        nf_compute<LOGN, NPH - 1, false>(x, tu, T);
      else
        nr_compute<LOGN, NPH - 1, false, RELAX>(x, tu, T, q, q2);
    }
  }
  // forward output of unit (dring, half h) at ds + (2 dring + h) N
  if (active) {
    if constexpr (FP)
      nf_store_global<LOGN, true, false>(x, ds, 2 * dring + h, tu, T, nullptr);
    else
      nr_store_global<LOGN, true, false, RELAX>(x, ds, 2 * dring + h, tu, T, q, q2);
  }
}

// ntt_digits_kernel<6, true, true> in the paired layout of ntt_fp6_kernel:
// one thread per (digit ring element, column r) with both halves, so each
// source load and each coefficient-form digit store moves a (half 0,
// half 1) pair and the transform's output leaves in 32-byte stores.
__global__ void __launch_bounds__(256)
    ntt_digits6_kernel(NttSrcRows src, u64 width, u32 parts, const u64* bw_or, u64* rlog_out, u64* radix_out,
                       u64* dc, u64* ds, u64 count, NttDev T, bool narrow) {
  __shared__ double2 sm[NP6_EL * NP6_ROW];
  const u32 el = threadIdx.x >> 3, r = threadIdx.x & 7;
  const u64 re = (u64)blockIdx.x * NP6_EL + el;  // ring element of the digit space
  const bool active = re < count;
  const u64 q = T.q;
  const u64 orv = *bw_or;
  const u32 bw = orv ? 64u - (u32)__clzll((long long)orv) : 0u;
  const u32 rlog = (bw + parts - 1) / parts;
  const u64 mask = rlog >= 64 ? ~0ULL : ((1ULL << rlog) - 1);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *rlog_out = rlog;
    if (radix_out) *radix_out = 1ULL << rlog;
  }
  const u32 c = (u32)(re % parts);
  const u64 se = re / parts;
  const u32 k = active ? (u32)(se / width) : 0;
  const u64 i = se % width;
  const u64 dring = ((u64)k * parts + c) * width + i;  // output ring element
  const u32 sh = rlog * c;
  double x0[8], x1[8];
  if (active) {
    const u64* sp = src.p[k] + i * 128;
#pragma unroll
    for (u32 kk = 0; kk < 8; kk++) {
      const u32 e = r + 8 * kk;
      const ulonglong2 v2 = __ldg((const ulonglong2*)(sp + 2 * e));
      u64 dv[2];
      long long dn[2];
#pragma unroll
      for (u32 h = 0; h < 2; h++) {
        const u64 v = h ? v2.y : v2.x;
        const u64 pos = 2 * v > q ? 0 : v, neg = 2 * v > q ? q - v : 0;
        const u64 pd = sh >= 64 ? 0 : ((pos >> sh) & mask), nd = sh >= 64 ? 0 : ((neg >> sh) & mask);
        dv[h] = pd >= nd ? pd - nd : pd + q - nd;
        dn[h] = (long long)pd - (long long)nd;
      }
      x0[kk] = fp_from_word(dv[0]);
      x1[kk] = fp_from_word(dv[1]);
      if (narrow)
        *(int2*)((int*)dc + dring * 128 + 2 * e) = make_int2((int)dn[0], (int)dn[1]);
      else
        *(ulonglong2*)(dc + dring * 128 + 2 * e) = make_ulonglong2(dv[0], dv[1]);
    }
  }
  np6_forward(x0, x1, sm, el, r, active, T);
  if (active) np6_store_slots(x0, x1, ds, dring, r, T);
}

// Fused negacyclic product r = a * b mod (Y^n + 1) for a batch of polynomials:
// forward transforms of a and b, the pointwise product and the inverse
// transform in one pass over a tile, so HBM sees a and b read once and r
// written once (24 bytes per coefficient instead of 72 for three separate
// passes).  Same value as NTT^-1(NTT(a) . NTT(b)) with the generic kernels.
template <int LOGN, bool RELAX>
__global__ void __launch_bounds__(256) ntt_mul_kernel(const u64* a, const u64* b, u64* r, u64 units, NttDev T,
                                                      ModQ M) {
  constexpr u32 N = 1u << LOGN, UPT = NR_TILE / N;
  constexpr int NPH = ph_count(LOGN), PL = NPH - 1, SL = ph_size(LOGN, PL);
  constexpr u32 MBL = 16 >> SL, KL = 1u << SL;
  extern __shared__ u64 nm_smem[];  // two padded tiles
  u64* sa = nm_smem;
  u64* sb = nm_smem + NR_TILE + NR_TILE / 16;
  u32 unit, tu;
  nr_map<LOGN, false>(threadIdx.x, unit, tu);
  const u64 ug = (u64)blockIdx.x * UPT + unit;
  const bool active = ug < units;
  const u64 q = T.q, q2 = 2 * T.q;
  u64 x[16];
  // forward transform of a, left canonical in sa
  if (active) {
    nr_load_global<LOGN, false, false>(x, a, ug, tu);
    nr_compute<LOGN, 0, false, RELAX>(x, tu, T, q, q2);
  }
  if constexpr (NPH > 1) {
    if (active) nr_store_smem<LOGN, 0, false>(x, sa, unit, tu);
    __syncthreads();
    nr_mid<LOGN, 1, PL, false, RELAX>(x, sa, unit, tu, active, T, q, q2);
    if (active) {
      nr_load_smem<LOGN, PL, false>(x, sa, unit, tu);
      nr_compute<LOGN, PL, false, RELAX>(x, tu, T, q, q2);
    }
  }
  if (active) {
#pragma unroll
    for (u32 i = 0; i < 16; i++) x[i] = nr_canon<RELAX>(x[i], q, q2, T.onep);
    nr_store_smem<LOGN, PL, false>(x, sa, unit, tu);
  }
  // forward transform of b through sb, ending in registers
  if (active) {
    nr_load_global<LOGN, false, false>(x, b, ug, tu);
    nr_compute<LOGN, 0, false, RELAX>(x, tu, T, q, q2);
  }
  if constexpr (NPH > 1) {
    if (active) nr_store_smem<LOGN, 0, false>(x, sb, unit, tu);
    __syncthreads();
    nr_mid<LOGN, 1, PL, false, RELAX>(x, sb, unit, tu, active, T, q, q2);
    if (active) {
      nr_load_smem<LOGN, PL, false>(x, sb, unit, tu);
      nr_compute<LOGN, PL, false, RELAX>(x, tu, T, q, q2);
    }
  }
  // pointwise product into sa (each thread owns these positions of sa)
  if (active) {
#pragma unroll
    for (u32 j = 0; j < MBL; j++)
#pragma unroll
      for (u32 k = 0; k < KL; k++) {
        const u32 pos = npad(unit * N + nr_elem<LOGN, PL, false>(tu, j, k));
        sa[pos] = mul_mod(M, nr_canon<RELAX>(x[j * KL + k], q, q2, T.onep), sa[pos]);
      }
  }
  __syncthreads();
  // inverse transform from sa to r
  if (active) {
    nr_load_smem<LOGN, 0, true>(x, sa, unit, tu);
    nr_compute<LOGN, 0, true, RELAX>(x, tu, T, q, q2);
  }
  if constexpr (NPH > 1) {
    if (active) nr_store_smem<LOGN, 0, true>(x, sa, unit, tu);
    __syncthreads();
    nr_mid<LOGN, 1, PL, true, RELAX>(x, sa, unit, tu, active, T, q, q2);
    if (active) {
      nr_load_smem<LOGN, PL, true>(x, sa, unit, tu);
      nr_compute<LOGN, PL, true, RELAX>(x, tu, T, q, q2);
    }
  }
  if (active) nr_store_global<LOGN, false, true, RELAX>(x, r, ug, tu, T, q, q2);
}

template <int LOGN>
int nm_launch(const u64* a, const u64* b, u64* r, u64 count, const NttDev& T, cudaStream_t st) {
  constexpr u32 UPT = NR_TILE >> LOGN;
  const u64 blocks = (count + UPT - 1) / UPT;
  if (blocks > 0x7fffffffULL) return salsaa_set_error(-2, "ntt_mul: batch too large");
  const size_t smem = 2 * (NR_TILE + NR_TILE / 16) * sizeof(u64);
  auto go = [&](auto kern) -> int {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "ntt_mul smem attribute");
    kern<<<(unsigned)blocks, 256, smem, st>>>(a, b, r, count, T, make_modq(T.q));
    return 0;
  };
  return T.q < NR_RELAX_Q ? go(ntt_mul_kernel<LOGN, true>) : go(ntt_mul_kernel<LOGN, false>);
}

// Persistent bulk-copy pipeline: grid = min(tiles, SMs x resident CTAs),
// capped at ctas_per_sm CTAs per SM when that is > 0.
template <int LOGN, bool INC, bool INV, bool RELAX, int STAGES, bool FP>
int np_go(const u64* in, u64* out, u64 units, const NttDev& T, cudaStream_t st, u64* mag_or, int ctas_per_sm) {
  constexpr u32 UPT = NR_TILE >> LOGN;
  auto kern = ntt_pipe_kernel<LOGN, INC, INV, RELAX, STAGES, FP>;
  const size_t smem = 128 + ((size_t)STAGES * NR_TILE + NR_TILE + NR_TILE / 16) * sizeof(u64);
  static int resident_dev[64][2] = {};  // per instantiation and device: attribute set, resident CTAs per SM
  static std::mutex mu;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return salsaa_set_error(-1, "ntt pipe: device query");
  if (dev < 0 || dev >= 64) return salsaa_set_error(-1, "ntt pipe: device index out of range");
  int* resident = resident_dev[dev];
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!resident[0]) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return salsaa_set_cuda_error(e, "ntt pipe smem attribute");
      int r = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, kern, 256, smem);
      if (e != cudaSuccess || r < 1) return salsaa_set_error(-1, "ntt pipe: kernel does not fit an SM");
      resident[1] = r;
      resident[0] = 1;
    }
  }
  const int per_sm = (ctas_per_sm > 0 && ctas_per_sm < resident[1]) ? ctas_per_sm : resident[1];
  const u64 tiles = (units + UPT - 1) / UPT;
  const u64 cap = (u64)nsm * (u64)per_sm;
  const u64 blocks = tiles < cap ? tiles : cap;
  kern<<<(unsigned)blocks, 256, smem, st>>>(in, out, units, T, mag_or);
  return 0;
}

// variant 2..4: integer butterflies with that many stages; 5..7: FP64 ones
// (q < 2^50 only) with 2..4 stages.
template <int LOGN, bool INC, bool INV, bool RELAX>
int np_launch(const u64* in, u64* out, u64 units, const NttDev& T, cudaStream_t st, u64* mag_or, int variant,
              int ctas_per_sm) {
  if constexpr (RELAX) {
    switch (variant) {
      case 5: return np_go<LOGN, INC, INV, RELAX, 2, true>(in, out, units, T, st, mag_or, ctas_per_sm);
      case 6: return np_go<LOGN, INC, INV, RELAX, 3, true>(in, out, units, T, st, mag_or, ctas_per_sm);
      case 7: return np_go<LOGN, INC, INV, RELAX, 4, true>(in, out, units, T, st, mag_or, ctas_per_sm);
      default: break;
    }
  }
  switch (variant) {
    case 2: return np_go<LOGN, INC, INV, RELAX, 2, false>(in, out, units, T, st, mag_or, ctas_per_sm);
    case 3: return np_go<LOGN, INC, INV, RELAX, 3, false>(in, out, units, T, st, mag_or, ctas_per_sm);
    default: return np_go<LOGN, INC, INV, RELAX, 4, false>(in, out, units, T, st, mag_or, ctas_per_sm);
  }
}

template <int LOGN>
int nr_launch(const u64* in, u64* out, u64 units, const NttDev& T, bool incomplete, bool inverse, cudaStream_t st,
              u64* mag_or) {
  constexpr u32 UPT = NR_TILE >> LOGN;
  const u64 blocks = (units + UPT - 1) / UPT;
  if (blocks > 0x7fffffffULL) return salsaa_set_error(-2, "ntt: batch too large");
  const bool relax = T.q < NR_RELAX_Q;
  const NttChoice ch = ntt_choice(LOGN, incomplete, inverse, !relax, units * (1ULL << LOGN) >= NTT_LARGE_COEFFS);
  if (ch.variant == 1 && relax) {  // FP64 butterflies
    auto gof = [&](auto kern) -> int {
      kern<<<(unsigned)blocks, 256, 0, st>>>(in, out, units, T, mag_or);
      return 0;
    };
    if (LOGN == 6 && incomplete && np6_aligned(in, out, inverse)) {
      const u64 count = units / 2, g6 = (count + NP6_EL - 1) / NP6_EL;
      if (inverse) ntt_fp6_kernel<true><<<(unsigned)g6, 256, 0, st>>>(in, out, count, T, mag_or);
      else ntt_fp6_kernel<false><<<(unsigned)g6, 256, 0, st>>>(in, out, count, T, mag_or);
      return 0;
    }
    if (incomplete) {
      if constexpr (UPT >= 2)
        return inverse ? gof(ntt_fp_kernel<LOGN, true, true>) : gof(ntt_fp_kernel<LOGN, true, false>);
    } else {
      return inverse ? gof(ntt_fp_kernel<LOGN, false, true>) : gof(ntt_fp_kernel<LOGN, false, false>);
    }
  }
  if (ch.variant >= 2 && (!incomplete || UPT >= 2)) {
    if (incomplete) {
      if constexpr (UPT >= 2) {
        if (inverse)
          return relax ? np_launch<LOGN, true, true, true>(in, out, units, T, st, mag_or, ch.variant, ch.ctas_per_sm)
                       : np_launch<LOGN, true, true, false>(in, out, units, T, st, mag_or, ch.variant, ch.ctas_per_sm);
        return relax ? np_launch<LOGN, true, false, true>(in, out, units, T, st, mag_or, ch.variant, ch.ctas_per_sm)
                     : np_launch<LOGN, true, false, false>(in, out, units, T, st, mag_or, ch.variant, ch.ctas_per_sm);
      }
    } else {
      if (inverse)
        return relax ? np_launch<LOGN, false, true, true>(in, out, units, T, st, mag_or, ch.variant, ch.ctas_per_sm)
                     : np_launch<LOGN, false, true, false>(in, out, units, T, st, mag_or, ch.variant, ch.ctas_per_sm);
      return relax ? np_launch<LOGN, false, false, true>(in, out, units, T, st, mag_or, ch.variant, ch.ctas_per_sm)
                   : np_launch<LOGN, false, false, false>(in, out, units, T, st, mag_or, ch.variant, ch.ctas_per_sm);
    }
  }
  auto go = [&](auto kern) -> int {
    kern<<<(unsigned)blocks, 256, 0, st>>>(in, out, units, T, mag_or);
    return 0;
  };
  // full 64-point transforms: the paired layout when the contiguous side is 32-byte aligned
  if (LOGN == 6 && !incomplete && (uintptr_t)(inverse ? in : out) % 32 == 0) {
    const unsigned g6 = (unsigned)((units + 2 * NP6_EL - 1) / (2 * NP6_EL));
    if (inverse) {
      if (relax) ntt_int6_kernel<true, true><<<g6, 256, 0, st>>>(in, out, units, T, mag_or);
      else ntt_int6_kernel<true, false><<<g6, 256, 0, st>>>(in, out, units, T, mag_or);
    } else {
      if (relax) ntt_int6_kernel<false, true><<<g6, 256, 0, st>>>(in, out, units, T, mag_or);
      else ntt_int6_kernel<false, false><<<g6, 256, 0, st>>>(in, out, units, T, mag_or);
    }
    return 0;
  }
  if (incomplete) {
    if constexpr (UPT >= 2) {
      if (inverse)
        return relax ? go(ntt_reg_kernel<LOGN, true, true, true>) : go(ntt_reg_kernel<LOGN, true, true, false>);
      return relax ? go(ntt_reg_kernel<LOGN, true, false, true>) : go(ntt_reg_kernel<LOGN, true, false, false>);
    } else {
      return salsaa_set_error(-2, "ntt: incomplete register path needs two halves per tile");
    }
  }
  if (inverse)
    return relax ? go(ntt_reg_kernel<LOGN, false, true, true>) : go(ntt_reg_kernel<LOGN, false, true, false>);
  return relax ? go(ntt_reg_kernel<LOGN, false, false, true>) : go(ntt_reg_kernel<LOGN, false, false, false>);
}

}  // namespace

template <int LOGN>
int nm_multi_go(const NttMulti& m, u64 blocks, const NttDev& T, bool incomplete, bool inverse, cudaStream_t st,
                bool large) {
  const bool relax = T.q < NR_RELAX_Q;
  const bool fp = relax && ntt_choice(LOGN, incomplete, inverse, false, large).fp64();
  auto go = [&](auto kern) -> int {
    kern<<<(unsigned)blocks, 256, 0, st>>>(m, T);
    return 0;
  };
  if (incomplete) {
    if constexpr ((NR_TILE >> LOGN) >= 2) {
      if (inverse)
        return fp ? go(ntt_multi_kernel<LOGN, true, true, true, true>)
                  : relax ? go(ntt_multi_kernel<LOGN, true, true, true, false>)
                          : go(ntt_multi_kernel<LOGN, true, true, false, false>);
      return fp ? go(ntt_multi_kernel<LOGN, true, false, true, true>)
                : relax ? go(ntt_multi_kernel<LOGN, true, false, true, false>)
                        : go(ntt_multi_kernel<LOGN, true, false, false, false>);
    }
    return salsaa_set_error(-2, "ntt_multi: incomplete transforms need d <= 4096");
  }
  if (inverse)
    return fp ? go(ntt_multi_kernel<LOGN, false, true, true, true>)
              : relax ? go(ntt_multi_kernel<LOGN, false, true, true, false>)
                      : go(ntt_multi_kernel<LOGN, false, true, false, false>);
  return fp ? go(ntt_multi_kernel<LOGN, false, false, true, true>)
            : relax ? go(ntt_multi_kernel<LOGN, false, false, true, false>)
                    : go(ntt_multi_kernel<LOGN, false, false, false, false>);
}

bool ntt_mag_ok(const u64* in, const u64* out, const NttDev& T, bool incomplete) {
  const bool aligned = ((uintptr_t)in % 16 == 0) && ((uintptr_t)out % 16 == 0);
  return aligned && T.n >= 16 && T.n <= (incomplete ? 2048u : 4096u);
}

int ntt_launch(const u64* in, u64* out, u64 count, const NttDev& T, bool incomplete, bool inverse,
               cudaStream_t st, u64* mag_or) {
  if (count == 0) return 0;
  const u32 d = incomplete ? 2 * T.n : T.n;
  if (ntt_mag_ok(in, out, T, incomplete)) {
    const u64 units = incomplete ? 2 * count : count;
    const int tr = salsaa_trace_begin("ntt_kernel", st, 16.0 * (double)count * d);
    int rc = 0;
    switch (T.logn) {
      case 4: rc = nr_launch<4>(in, out, units, T, incomplete, inverse, st, mag_or); break;
      case 5: rc = nr_launch<5>(in, out, units, T, incomplete, inverse, st, mag_or); break;
      case 6: rc = nr_launch<6>(in, out, units, T, incomplete, inverse, st, mag_or); break;
      case 7: rc = nr_launch<7>(in, out, units, T, incomplete, inverse, st, mag_or); break;
      case 8: rc = nr_launch<8>(in, out, units, T, incomplete, inverse, st, mag_or); break;
      case 9: rc = nr_launch<9>(in, out, units, T, incomplete, inverse, st, mag_or); break;
      case 10: rc = nr_launch<10>(in, out, units, T, incomplete, inverse, st, mag_or); break;
      case 11: rc = nr_launch<11>(in, out, units, T, incomplete, inverse, st, mag_or); break;
      default: rc = nr_launch<12>(in, out, units, T, incomplete, inverse, st, mag_or); break;
    }
    salsaa_trace_end(tr, st);
    if (rc) return rc;
    salsaa_count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "ntt launch");
  }
  if (mag_or) return salsaa_set_error(-2, "ntt: magnitude OR needs the register path");
  // 32 KiB of elements per CTA (at least one element).
  u32 epb = 4096 / d;
  if (epb == 0) epb = 1;
  const size_t smem = (size_t)epb * d * sizeof(u64);
  const u64 blocks = (count + epb - 1) / epb;
  if (blocks > 0x7fffffffULL) return salsaa_set_error(-2, "ntt: batch too large");
  auto launch = [&](auto kern) -> int {
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return salsaa_set_cuda_error(e, "ntt smem attribute");
    }
    // algorithmic bytes: every coefficient read once and written once
    const int tr = salsaa_trace_begin("ntt_kernel", st, 16.0 * (double)count * d);
    kern<<<(unsigned)blocks, 256, smem, st>>>(in, out, count, T, epb);
    salsaa_trace_end(tr, st);
    salsaa_count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "ntt launch");
  };
  if (incomplete) return inverse ? launch(ntt_kernel<true, true>) : launch(ntt_kernel<true, false>);
  return inverse ? launch(ntt_kernel<false, true>) : launch(ntt_kernel<false, false>);
}

int ntt_multi_launch(const u64* const* in, u64* const* out, const u64* count, u32 ninst, const NttDev& T,
                     bool incomplete, bool inverse, cudaStream_t st) {
  if (ninst > (u32)NTT_MULTI_MAX) return salsaa_set_error(-2, "ntt_multi: at most 64 batches per launch");
  if (T.n < 16 || T.n > (incomplete ? 2048u : 4096u))
    return salsaa_set_error(-2, "ntt_multi: needs 16 <= n <= 4096 (2048 in incomplete mode)");
  NttMulti m{};
  const u32 upt = NR_TILE >> T.logn;
  u64 blocks = 0, coeffs = 0;
  u32 k = 0;
  for (u32 i = 0; i < ninst; i++) {
    if (!count[i]) continue;
    if (!in[i] || !out[i]) return salsaa_set_error(-1, "ntt_multi: null buffer");
    if ((uintptr_t)in[i] % 16 || (uintptr_t)out[i] % 16) return salsaa_set_error(-2, "ntt_multi: buffers must be 16-byte aligned");
    const u64 units = incomplete ? 2 * count[i] : count[i];
    m.in[k] = in[i];
    m.out[k] = out[i];
    m.units[k] = units;
    m.bstart[k] = blocks;
    blocks += (units + upt - 1) / upt;
    coeffs += units * T.n;
    k++;
  }
  if (k == 0) return 0;
  m.bstart[k] = blocks;
  m.count = k;
  if (blocks > 0x7fffffffULL) return salsaa_set_error(-2, "ntt_multi: batch too large");
  const bool large = coeffs >= NTT_LARGE_COEFFS;
  const int tr = salsaa_trace_begin("ntt_kernel", st, 16.0 * (double)coeffs);
  int rc = 0;
  switch (T.logn) {
    case 4: rc = nm_multi_go<4>(m, blocks, T, incomplete, inverse, st, large); break;
    case 5: rc = nm_multi_go<5>(m, blocks, T, incomplete, inverse, st, large); break;
    case 6: rc = nm_multi_go<6>(m, blocks, T, incomplete, inverse, st, large); break;
    case 7: rc = nm_multi_go<7>(m, blocks, T, incomplete, inverse, st, large); break;
    case 8: rc = nm_multi_go<8>(m, blocks, T, incomplete, inverse, st, large); break;
    case 9: rc = nm_multi_go<9>(m, blocks, T, incomplete, inverse, st, large); break;
    case 10: rc = nm_multi_go<10>(m, blocks, T, incomplete, inverse, st, large); break;
    case 11: rc = nm_multi_go<11>(m, blocks, T, incomplete, inverse, st, large); break;
    default: rc = nm_multi_go<12>(m, blocks, T, incomplete, inverse, st, large); break;
  }
  salsaa_trace_end(tr, st);
  if (rc) return rc;
  salsaa_count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "ntt_multi launch");
}

template <int LOGN>
int nd_launch(const NttSrcRows& src, u32 rows, u64 width, u32 parts, const u64* bw_or, u64* rlog_out,
              u64* radix_out, u64* dc, u64* ds, const NttDev& T, cudaStream_t st, bool narrow) {
  constexpr u32 UPT = NR_TILE >> LOGN;
  const u64 units = 2ULL * rows * parts * width;
  const u64 blocks = (units + UPT - 1) / UPT;
  if (blocks > 0x7fffffffULL) return salsaa_set_error(-2, "ntt_digits: batch too large");
  // the forward incomplete transform's schedule decides the arithmetic
  const bool relax = T.q < NR_RELAX_Q;
  const bool fp = relax && ntt_choice(LOGN, true, false, false, units * (1ULL << LOGN) >= NTT_LARGE_COEFFS).fp64();
  bool src16 = true;
  for (u32 k = 0; k < rows && k < 16; k++) src16 = src16 && (uintptr_t)src.p[k] % 16 == 0;
  if (fp && LOGN == 6 && (uintptr_t)ds % 32 == 0 && src16) {
    const u64 count = units / 2;
    ntt_digits6_kernel<<<(unsigned)((count + NP6_EL - 1) / NP6_EL), 256, 0, st>>>(src, width, parts, bw_or, rlog_out,
                                                                                   radix_out, dc, ds, count, T, narrow);
  } else if (fp)
    ntt_digits_kernel<LOGN, true, true><<<(unsigned)blocks, 256, 0, st>>>(src, width, parts, bw_or, rlog_out,
                                                                           radix_out, dc, ds, units, T, narrow);
  else if (relax)
    ntt_digits_kernel<LOGN, true, false><<<(unsigned)blocks, 256, 0, st>>>(src, width, parts, bw_or, rlog_out,
                                                                            radix_out, dc, ds, units, T, narrow);
  else
    ntt_digits_kernel<LOGN, false, false><<<(unsigned)blocks, 256, 0, st>>>(src, width, parts, bw_or, rlog_out,
                                                                             radix_out, dc, ds, units, T, narrow);
  return 0;
}

bool ntt_digits_ok(const u64* dc, const u64* ds, u32 rows, const NttDev& T) {
  return T.n >= 16 && T.n <= 2048 && rows >= 1 && rows <= 16 && (uintptr_t)dc % 16 == 0 && (uintptr_t)ds % 16 == 0;
}

int ntt_digits_launch(const NttSrcRows& src, u32 rows, u64 width, u32 parts, const u64* bw_or, u64* rlog_out,
                      u64* radix_out, u64* dc, u64* ds, const NttDev& T, cudaStream_t st, bool narrow) {
  if (!ntt_digits_ok(dc, ds, rows, T) || parts == 0 || width == 0 || (narrow && parts < 2))
    return salsaa_set_error(-2, "ntt_digits: shape or alignment not supported");
  const double bytes = 8.0 * rows * width * 2.0 * T.n * (1.0 + (narrow ? 1.5 : 2.0) * parts);
  const int tr = salsaa_trace_begin("ntt_digits_kernel", st, bytes);
  int rc = 0;
  switch (T.logn) {
    case 4: rc = nd_launch<4>(src, rows, width, parts, bw_or, rlog_out, radix_out, dc, ds, T, st, narrow); break;
    case 5: rc = nd_launch<5>(src, rows, width, parts, bw_or, rlog_out, radix_out, dc, ds, T, st, narrow); break;
    case 6: rc = nd_launch<6>(src, rows, width, parts, bw_or, rlog_out, radix_out, dc, ds, T, st, narrow); break;
    case 7: rc = nd_launch<7>(src, rows, width, parts, bw_or, rlog_out, radix_out, dc, ds, T, st, narrow); break;
    case 8: rc = nd_launch<8>(src, rows, width, parts, bw_or, rlog_out, radix_out, dc, ds, T, st, narrow); break;
    case 9: rc = nd_launch<9>(src, rows, width, parts, bw_or, rlog_out, radix_out, dc, ds, T, st, narrow); break;
    case 10: rc = nd_launch<10>(src, rows, width, parts, bw_or, rlog_out, radix_out, dc, ds, T, st, narrow); break;
    default: rc = nd_launch<11>(src, rows, width, parts, bw_or, rlog_out, radix_out, dc, ds, T, st, narrow); break;
  }
  salsaa_trace_end(tr, st);
  if (rc) return rc;
  salsaa_count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "ntt_digits launch");
}

bool ntt_mul_fused_ok(const u64* a, const u64* b, const u64* r, const NttDev& T) {
  return T.n >= 16 && T.n <= 4096 && (uintptr_t)a % 16 == 0 && (uintptr_t)b % 16 == 0 && (uintptr_t)r % 16 == 0;
}

int ntt_mul_launch(const u64* a, const u64* b, u64* r, u64 count, const NttDev& T, cudaStream_t st) {
  if (count == 0) return 0;
  if (!ntt_mul_fused_ok(a, b, r, T)) return salsaa_set_error(-2, "ntt_mul: size or alignment not supported");
  const int tr = salsaa_trace_begin("ntt_mul_kernel", st, 24.0 * (double)count * T.n);
  int rc = 0;
  switch (T.logn) {
    case 4: rc = nm_launch<4>(a, b, r, count, T, st); break;
    case 5: rc = nm_launch<5>(a, b, r, count, T, st); break;
    case 6: rc = nm_launch<6>(a, b, r, count, T, st); break;
    case 7: rc = nm_launch<7>(a, b, r, count, T, st); break;
    case 8: rc = nm_launch<8>(a, b, r, count, T, st); break;
    case 9: rc = nm_launch<9>(a, b, r, count, T, st); break;
    case 10: rc = nm_launch<10>(a, b, r, count, T, st); break;
    case 11: rc = nm_launch<11>(a, b, r, count, T, st); break;
    default: rc = nm_launch<12>(a, b, r, count, T, st); break;
  }
  salsaa_trace_end(tr, st);
  if (rc) return rc;
  salsaa_count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "ntt_mul launch");
}

}  // namespace salsaa

namespace salsaa {
int ntt_error_check() {
  u32 h = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&h, g_ntt_error, sizeof(u32));
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "ntt status");
  if (h) return salsaa_set_error(-4, "a bulk-copy wait of the NTT timed out; results of that launch are invalid");
  return 0;
}
}  // namespace salsaa

extern "C" int salsaa_tune_load(const char* path) { return salsaa::ntt_tune_load(path); }

extern "C" int salsaa_tune_reset(void) {
  salsaa::ntt_tune_reset();
  return 0;
}

extern "C" int salsaa_ntt_tune_set(uint32_t log_n, int incomplete, int inverse, int wide_modulus, int large,
                                   int variant, int ctas_per_sm) {
  return salsaa::ntt_tune_set(log_n, incomplete != 0, inverse != 0, wide_modulus != 0, large != 0, variant,
                              ctas_per_sm);
}

extern "C" int salsaa_fold_tune_set(int variant) { return salsaa::fold_tune_set(variant); }
extern "C" int salsaa_fold_tune_get(void) { return salsaa::fold_choice(); }

extern "C" int salsaa_ntt_tune_get(uint32_t log_n, int incomplete, int inverse, int wide_modulus, int large,
                                   int* variant, int* ctas_per_sm) {
  if (!variant || !ctas_per_sm) return salsaa_set_error(-1, "ntt_tune_get: null argument");
  const salsaa::NttChoice c =
      salsaa::ntt_choice(log_n, incomplete != 0, inverse != 0, wide_modulus != 0, large != 0);
  *variant = c.variant;
  *ctas_per_sm = c.ctas_per_sm;
  return 0;
}
