// dense.cu — dense ring-matrix commitment C = A * W over R_q
// (parallel_dot_matrix_matrix, src/arithmetic.rs:429-457, in the shape of an
// Ajtai commitment: A is n x m, W has r columns of m ring elements).
//
// A is prepared once into a key object: its slot form is stored as the same
// tables the commitment-key rows use (three components per slot and element,
// one "block" spanning all m elements, a high factor of 1) plus the tcgen05
// byte image.  A commitment then runs through launch_commit unchanged: the
// tensor-core kernel when q < 2^56 and n <= 18, the CUDA-core kernel
// otherwise, over groups of at most 9 columns of W.
#include <vector>

#include "../../include/salsaa_gpu.h"
#include "kernels.cuh"
#include "ntt.cuh"

using namespace salsaa;

struct salsaa_dense_key {
  u32 nrows = 0, d = 0, n = 0;
  u64 m = 0, q = 0;
  const NttDev* T = nullptr;
  ModQ M{};
  u64* tlo = nullptr;     // nrows x m x 3n (25-bit limb pairs when q < 2^50)
  u64* thi = nullptr;     // nrows x 1 x d: the slot form of 1
  uint8_t* tk8 = nullptr; // tcgen05 byte image, or null
  u64* scratch = nullptr; // acc + out for one group: 2 x nrows x 9 x d
  DevState* ds = nullptr;
};

namespace {

constexpr u32 DENSE_GROUP = CKU_MAX_WROWS;

__global__ void dense_tables_kernel(const u64* a_slot, u32 nrows, u64 m, u32 n, ModQ M, const u64* zeta,
                                    bool packed, u64* tlo, u64* thi) {
  const u64 tot = (u64)nrows * m * n;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u32 s = (u32)(t % n);
    const u64 ri = t / n;  // r * m + i
    const u64* x = a_slot + ri * 2 * n;
    const u64 e = x[s], o = x[n + s], z = mul_mod(M, zeta[s], o);
    u64* dst = tlo + ri * 3 * n;
    if (packed) {
      dst[s] = ((e >> 25) << 32) | (e & 0x1FFFFFFull);
      dst[n + s] = ((o >> 25) << 32) | (o & 0x1FFFFFFull);
      dst[2 * n + s] = ((z >> 25) << 32) | (z & 0x1FFFFFFull);
    } else {
      dst[s] = e;
      dst[n + s] = o;
      dst[2 * n + s] = z;
    }
    if (ri % m == 0) {  // one high factor per key row: 1 = (1, 0) in every slot
      thi[(ri / m) * 2 * n + s] = 1;
      thi[(ri / m) * 2 * n + n + s] = 0;
    }
  }
}

}  // namespace

extern "C" int salsaa_dense_key_create(const uint64_t* d_a, uint64_t nrows, uint64_t m, uint64_t d, uint64_t q,
                                       void* stream, salsaa_dense_key** out) {
  if (!d_a || !out) return salsaa_set_error(-1, "dense_key_create: null argument");
  *out = nullptr;
  if (nrows == 0 || nrows > 64 || m < 128 || (m & (m - 1)) || d < 4 || d > 512 || (d & (d - 1)))
    return salsaa_set_error(-1, "dense_key_create: needs 1 <= n <= 64, m a power of two >= 128, d in 4..512");
  const NttDev* T = ntt_tables((u32)(d / 2), q);
  if (!T) return salsaa_set_error(-1, "dense_key_create: no incomplete NTT for (d, q)");
  cudaStream_t st = (cudaStream_t)stream;
  salsaa_dense_key* k = new salsaa_dense_key;
  k->nrows = (u32)nrows;
  k->d = (u32)d;
  k->n = (u32)(d / 2);
  k->m = m;
  k->q = q;
  k->T = T;
  k->M = make_modq(q);
  u64* a_slot = nullptr;
  auto fail = [&](cudaError_t e, const char* what) {
    if (a_slot) cudaFree(a_slot);
    salsaa_dense_key_destroy(k);
    return salsaa_set_cuda_error(e, what);
  };
  cudaError_t e = cudaMalloc(&a_slot, nrows * m * d * sizeof(u64));
  if (e != cudaSuccess) return fail(e, "dense_key_create: alloc");
  if ((e = cudaMalloc(&k->tlo, nrows * m * 3 * (d / 2) * sizeof(u64))) != cudaSuccess) return fail(e, "alloc");
  if ((e = cudaMalloc(&k->thi, nrows * d * sizeof(u64))) != cudaSuccess) return fail(e, "alloc");
  if ((e = cudaMalloc(&k->scratch, 2 * nrows * DENSE_GROUP * d * sizeof(u64))) != cudaSuccess) return fail(e, "alloc");
  if ((e = cudaMalloc(&k->ds, sizeof(DevState))) != cudaSuccess) return fail(e, "alloc");
  cudaMemsetAsync(k->ds, 0, sizeof(DevState), st);
  int rc = ntt_launch(d_a, a_slot, nrows * m, *T, true, false, st);
  if (rc) {
    cudaFree(a_slot);
    a_slot = nullptr;
    salsaa_dense_key_destroy(k);
    return rc;
  }
  const bool packed = q < (1ULL << 50);
  u64 tot = nrows * m * (d / 2), g = (tot + 255) / 256;
  if (g > 65535ull * 16) g = 65535ull * 16;
  dense_tables_kernel<<<(unsigned)g, 256, 0, st>>>(a_slot, (u32)nrows, m, (u32)(d / 2), k->M, T->zeta, packed,
                                                    k->tlo, k->thi);
  salsaa_count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "dense_key_create: tables");
  if (q < (1ULL << 56) && nrows <= CKU_MAX_KEYS && (d / 2) % 2 == 0) {
    if ((e = cudaMalloc(&k->tk8, ck_tk8_bytes((u32)nrows, (u32)(d / 2), (u32)m))) != cudaSuccess)
      return fail(e, "dense_key_create: alloc");
    rc = launch_ck_tk8(k->tlo, (u32)nrows, (u32)(d / 2), (u32)m, packed, k->tk8, st);
    if (rc) {
      cudaFree(a_slot);
      a_slot = nullptr;
      salsaa_dense_key_destroy(k);
      return rc;
    }
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e, "dense_key_create");
  cudaFree(a_slot);
  *out = k;
  return 0;
}

extern "C" void salsaa_dense_key_destroy(salsaa_dense_key* k) {
  if (!k) return;
  cudaFree(k->tlo);
  cudaFree(k->thi);
  cudaFree(k->tk8);
  cudaFree(k->scratch);
  cudaFree(k->ds);
  delete k;
}

extern "C" int salsaa_dense_commit(salsaa_dense_key* k, const uint64_t* d_w, uint64_t r, uint64_t* d_c,
                                   uint64_t* d_w_slot, void* stream) {
  if (!k || !d_w || !d_c) return salsaa_set_error(-1, "dense_commit: null argument");
  if (r == 0 || r > 4096) return salsaa_set_error(-1, "dense_commit: r must be in 1..4096");
  cudaStream_t st = (cudaStream_t)stream;
  const u32 d = k->d, nr = k->nrows;
  const u64 m = k->m;
  u64* tmp = nullptr;
  if (!d_w_slot) {
    cudaError_t e = cudaMallocAsync(&tmp, r * m * d * sizeof(u64), st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "dense_commit: workspace");
    d_w_slot = tmp;
  }
  struct Free {
    u64* p;
    cudaStream_t s;
    ~Free() {
      if (p) cudaFreeAsync(p, s);
    }
  } free_tmp{tmp, st};
  int rc = ntt_launch(d_w, d_w_slot, r * m, *k->T, true, false, st);
  if (rc) return rc;
  u64* acc = k->scratch;
  u64* cout = k->scratch + (u64)nr * DENSE_GROUP * d;
  for (u64 g0 = 0; g0 < r; g0 += DENSE_GROUP) {
    const u32 G = (u32)((r - g0) < DENSE_GROUP ? (r - g0) : DENSE_GROUP);
    CommitArgs a{};
    for (u32 c = 0; c < G; c++) a.w.p[c] = d_w_slot + (g0 + c) * m * d;
    a.rows = G;
    a.width = m;
    a.nck = nr;
    a.tlo = k->tlo;
    a.thi = k->thi;
    a.ck_bt = (u32)m;
    a.ck_nhi = 1;
    a.tk8 = k->tk8;
    a.acc = acc;
    a.out_slot = cout;
    rc = launch_commit(a, *k->T, k->M, k->ds, st);
    if (rc) return rc;
    // cout is nr x G x d; column block g0 of C (slot form, nr x r x d) lives in d_c
    cudaError_t e = cudaMemcpy2DAsync(d_c + g0 * d, r * d * sizeof(u64), cout, (u64)G * d * sizeof(u64),
                                      (u64)G * d * sizeof(u64), nr, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "dense_commit: gather");
  }
  return ntt_launch(d_c, d_c, (u64)nr * r, *k->T, true, true, st);
}
