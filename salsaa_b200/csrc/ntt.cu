// ntt.cu — batched negacyclic NTT / INTT kernels and their twiddle tables.
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "host_math.h"
#include "ntt.cuh"

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
  NttDev* T = new NttDev;
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

int ntt_launch(const u64* in, u64* out, u64 count, const NttDev& T, bool incomplete, bool inverse,
               cudaStream_t st) {
  if (count == 0) return 0;
  const u32 d = incomplete ? 2 * T.n : T.n;
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
    kern<<<(unsigned)blocks, 256, smem, st>>>(in, out, count, T, epb);
    salsaa_count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "ntt launch");
  };
  if (incomplete) return inverse ? launch(ntt_kernel<true, true>) : launch(ntt_kernel<true, false>);
  return inverse ? launch(ntt_kernel<false, true>) : launch(ntt_kernel<false, false>);
}

}  // namespace salsaa
