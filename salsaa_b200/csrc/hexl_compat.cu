// hexl_compat.cu — the twenty extern "C" symbols of hexl-bindings/hexl_wrapper.cpp
// with their signatures and host-memory semantics, so that the reference's
// Rust crate (src/hexl/bindings.rs:1-74, linked by build.rs:1-6) can link this
// library in place of libhexl_wrapper.so.
//
// Scalar functions are host arithmetic.  Array functions run on the GPU: each
// calling thread owns a CUDA stream and a growing device staging buffer, so
// concurrent callers (the reference calls from up to 64 rayon workers) never
// share state.  Invalid (n, modulus) pairs leave the output untouched and set
// salsaa_last_error() instead of aborting the process as HEXL does.
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/salsaa_gpu.h"
#include "host_math.h"
#include "ntt.cuh"

using namespace salsaa;

// ---- scalar tier -----------------------------------------------------------
extern "C" uint64_t multiply_mod(uint64_t a, uint64_t b, uint64_t modulus) { return host::mulmod(a, b, modulus); }
extern "C" uint64_t add_mod(uint64_t a, uint64_t b, uint64_t modulus) { return host::addmod(a, b, modulus); }
extern "C" uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t modulus) { return host::submod(a, b, modulus); }
extern "C" uint64_t power_mod(uint64_t a, uint64_t b, uint64_t modulus) { return host::powmod(a, b, modulus); }
extern "C" uint64_t inv_mod(uint64_t a, uint64_t modulus) { return host::invmod(a, modulus); }

// ---- root tables (library-owned, process lifetime) ------------------------
namespace {
std::mutex g_roots_mu;
std::map<std::pair<uint64_t, uint64_t>, std::pair<std::vector<uint64_t>, std::vector<uint64_t>>> g_roots;

const std::pair<std::vector<uint64_t>, std::vector<uint64_t>>* host_roots(size_t n, uint64_t q) {
  if (n < 1 || (n & (n - 1)) || q < 3 || q >= (1ULL << 62)) return nullptr;
  std::lock_guard<std::mutex> lk(g_roots_mu);
  auto key = std::make_pair((uint64_t)n, q);
  auto it = g_roots.find(key);
  if (it != g_roots.end()) return &it->second;
  const uint64_t psi = host::minimal_root(2 * (uint64_t)n, q);
  if (!psi) return nullptr;
  const unsigned logn = host::ilog2(n);
  std::vector<uint64_t> f(n), iv(n);
  const uint64_t pinv = host::invmod(psi, q);
  uint64_t p = 1, pi = 1;
  for (uint64_t i = 0; i < n; i++) {
    f[host::bitrev(i, logn)] = p;
    iv[host::bitrev(i, logn)] = pi;
    p = host::mulmod(p, psi, q);
    pi = host::mulmod(pi, pinv, q);
  }
  auto& slot = g_roots[key];
  slot.first = std::move(f);
  slot.second = std::move(iv);
  return &slot;
}

// ---- per-thread GPU staging --------------------------------------------------
struct Staging {
  int device = -1;
  cudaStream_t st = nullptr;
  uint64_t* buf = nullptr;
  size_t cap = 0;  // words
  ~Staging() {
    if (buf) cudaFree(buf);
    if (st) cudaStreamDestroy(st);
  }
  // three equal arrays of n words each
  uint64_t* get(size_t n3) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    if (dev != device) {
      if (buf) cudaFree(buf);
      if (st) cudaStreamDestroy(st);
      buf = nullptr;
      cap = 0;
      st = nullptr;
      device = dev;
      if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    }
    if (n3 > cap) {
      if (buf) cudaFree(buf);
      buf = nullptr;
      size_t c = n3 < 4096 ? 4096 : n3;
      if (cudaMalloc(&buf, c * sizeof(uint64_t)) != cudaSuccess) {
        cap = 0;
        return nullptr;
      }
      cap = c;
    }
    return buf;
  }
};
thread_local Staging g_stage;

enum EwOp { EW_MUL, EW_ADD, EW_SUB, EW_FMA, EW_RED };

__global__ void eltwise_kernel(int op, uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t s, uint64_t n,
                               ModQ M) {
  const uint64_t q = M.q;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t x = a[i] % q;
    uint64_t v;
    switch (op) {
      case EW_MUL: v = mul_mod(M, x, b[i] % q); break;
      case EW_ADD: v = salsaa::add_mod(x, b[i] % q, q); break;
      case EW_SUB: v = salsaa::sub_mod(x, b[i] % q, q); break;
      case EW_FMA: v = salsaa::add_mod(mul_mod(M, x, s % q), b[i] % q, q); break;
      default: v = x; break;
    }
    r[i] = v;
  }
}

__global__ void pointwise_mul_kernel(uint64_t* a, const uint64_t* b, uint64_t n, ModQ M) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    a[i] = mul_mod(M, a[i], b[i]);
}

__global__ void sum_kernel(const uint64_t* a, uint64_t n, ModQ M, int square, uint64_t* out) {
  __shared__ uint64_t sm[32];
  const uint64_t q = M.q;
  uint64_t acc = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t x = a[i] % q;
    acc = salsaa::add_mod(acc, square ? mul_mod(M, x, x) : x, q);
  }
  for (int o = 16; o > 0; o >>= 1) acc = salsaa::add_mod(acc, __shfl_down_sync(0xffffffffu, acc, o), q);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
    for (unsigned w = 0; w < (blockDim.x + 31) / 32; w++) t = salsaa::add_mod(t, sm[w], q);
    unsigned long long old = *(volatile unsigned long long*)out, assumed;
    do {
      assumed = old;
      old = atomicCAS((unsigned long long*)out, assumed, (unsigned long long)salsaa::add_mod((uint64_t)assumed, t, q));
    } while (old != assumed);
  }
}

bool modulus_ok(uint64_t q) {
  if (q < 2 || q >= (1ULL << 62)) {
    salsaa_set_error(-1, "modulus must be in [2, 2^62)");
    return false;
  }
  return true;
}

void run_eltwise(int op, uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t s, uint64_t n, uint64_t q) {
  if (!n || !modulus_ok(q)) return;
  uint64_t* d = g_stage.get(3 * n);
  if (!d) {
    salsaa_set_error(-1, "eltwise: staging allocation failed");
    return;
  }
  cudaStream_t st = g_stage.st;
  uint64_t *da = d, *db = d + n, *dr = d + 2 * n;
  cudaMemcpyAsync(da, a, n * 8, cudaMemcpyHostToDevice, st);
  if (b) cudaMemcpyAsync(db, b, n * 8, cudaMemcpyHostToDevice, st);
  unsigned g = (unsigned)((n + 255) / 256);
  if (g > 4096) g = 4096;
  eltwise_kernel<<<g, 256, 0, st>>>(op, dr, da, b ? db : da, s, n, make_modq(q));
  cudaMemcpyAsync(r, dr, n * 8, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) salsaa_set_cuda_error(e, "eltwise");
}

uint64_t run_sum(const uint64_t* a, uint64_t n, uint64_t q, int square) {
  if (!modulus_ok(q)) return 0;
  if (!n) return 0;
  uint64_t* d = g_stage.get(n + 1);
  if (!d) {
    salsaa_set_error(-1, "sum: staging allocation failed");
    return 0;
  }
  cudaStream_t st = g_stage.st;
  cudaMemcpyAsync(d, a, n * 8, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(d + n, 0, 8, st);
  unsigned g = (unsigned)((n + 255) / 256);
  if (g > 1024) g = 1024;
  sum_kernel<<<g, 256, 0, st>>>(d, n, make_modq(q), square, d + n);
  uint64_t out = 0;
  cudaMemcpyAsync(&out, d + n, 8, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) salsaa_set_cuda_error(e, "sum");
  return out;
}

void run_ntt(uint64_t* a, size_t n, uint64_t q, bool inverse) {
  const NttDev* T = ntt_tables((u32)n, q);
  if (!T) {
    salsaa_set_error(-1, "ntt: no negacyclic NTT for (n, modulus)");
    return;
  }
  uint64_t* d = g_stage.get(n);
  if (!d) {
    salsaa_set_error(-1, "ntt: staging allocation failed");
    return;
  }
  cudaStream_t st = g_stage.st;
  cudaMemcpyAsync(d, a, n * 8, cudaMemcpyHostToDevice, st);
  if (ntt_launch(d, d, 1, *T, false, inverse, st)) return;
  cudaMemcpyAsync(a, d, n * 8, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) salsaa_set_cuda_error(e, "ntt");
}

void run_poly_mul(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q) {
  const NttDev* T = ntt_tables((u32)n, q);
  if (!T) {
    salsaa_set_error(-1, "multiply_poly: no negacyclic NTT for (n, modulus)");
    return;
  }
  uint64_t* d = g_stage.get(3 * n);
  if (!d) {
    salsaa_set_error(-1, "multiply_poly: staging allocation failed");
    return;
  }
  cudaStream_t st = g_stage.st;
  const ModQ M = make_modq(q);
  uint64_t *da = d, *db = d + n;
  cudaMemcpyAsync(da, a, n * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(db, b, n * 8, cudaMemcpyHostToDevice, st);
  eltwise_kernel<<<1, 256, 0, st>>>(EW_RED, da, da, da, 0, n, M);
  eltwise_kernel<<<1, 256, 0, st>>>(EW_RED, db, db, db, 0, n, M);
  if (ntt_launch(da, da, 1, *T, false, false, st) || ntt_launch(db, db, 1, *T, false, false, st)) return;
  pointwise_mul_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(da, db, n, M);
  if (ntt_launch(da, da, 1, *T, false, true, st)) return;
  cudaMemcpyAsync(r, da, n * 8, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) salsaa_set_cuda_error(e, "multiply_poly");
}
}  // namespace

extern "C" const uint64_t* get_roots(size_t n, uint64_t modulus) {
  auto* t = host_roots(n, modulus);
  if (!t) {
    salsaa_set_error(-1, "get_roots: no negacyclic NTT for (n, modulus)");
    return nullptr;
  }
  return t->first.data();
}
extern "C" const uint64_t* get_inv_roots(size_t n, uint64_t modulus) {
  auto* t = host_roots(n, modulus);
  if (!t) {
    salsaa_set_error(-1, "get_inv_roots: no negacyclic NTT for (n, modulus)");
    return nullptr;
  }
  return t->second.data();
}

extern "C" void eltwise_mult_mod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, uint64_t n,
                                 uint64_t modulus) {
  run_eltwise(EW_MUL, result, operand1, operand2, 0, n, modulus);
}
extern "C" void eltwise_fma_mod(uint64_t* result, const uint64_t* operand1, uint64_t operand2,
                                const uint64_t* operand3, uint64_t n, uint64_t modulus) {
  run_eltwise(EW_FMA, result, operand1, operand3, operand2, n, modulus);
}
extern "C" void eltwise_add_mod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, size_t n,
                                uint64_t modulus) {
  run_eltwise(EW_ADD, result, operand1, operand2, 0, n, modulus);
}
extern "C" void eltwise_sub_mod(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, size_t n,
                                uint64_t modulus) {
  run_eltwise(EW_SUB, result, operand1, operand2, 0, n, modulus);
}
extern "C" void eltwise_reduce_mod(uint64_t* result, const uint64_t* operand, size_t n, uint64_t modulus) {
  run_eltwise(EW_RED, result, operand, nullptr, 0, n, modulus);
}
extern "C" void eltwise_reduce_mod_naive(uint64_t* result, const uint64_t* operand, size_t n, uint64_t modulus) {
  run_eltwise(EW_RED, result, operand, nullptr, 0, n, modulus);
}
extern "C" void multiply_poly(uint64_t* result, const uint64_t* operand1, const uint64_t* operand2, uint64_t n,
                              uint64_t modulus) {
  run_poly_mul(result, operand1, operand2, n, modulus);
}
extern "C" void polynomial_multiply_cyclotomic_mod(uint64_t* result, const uint64_t* operand1,
                                                   const uint64_t* operand2, size_t phi, uint64_t mod_q) {
  run_poly_mul(result, operand1, operand2, phi, mod_q);
}
extern "C" void ntt_forward_in_place(uint64_t* operand, size_t n, uint64_t modulus) {
  run_ntt(operand, n, modulus, false);
}
extern "C" void ntt_inverse_in_place(uint64_t* operand, size_t n, uint64_t modulus) {
  run_ntt(operand, n, modulus, true);
}
extern "C" uint64_t sum(const uint64_t* operand1, uint64_t n, uint64_t modulus) {
  return run_sum(operand1, n, modulus, 0);
}
extern "C" uint64_t sum_fast(const uint64_t* operand1, uint64_t n, uint64_t modulus) {
  return run_sum(operand1, n, modulus, 0);
}
extern "C" uint64_t sum_sq(const uint64_t* operand1, uint64_t n, uint64_t modulus) {
  return run_sum(operand1, n, modulus, 1);
}
extern "C" uint64_t sum_sq_fast(const uint64_t* operand1, uint64_t n, uint64_t modulus) {
  return run_sum(operand1, n, modulus, 1);
}
