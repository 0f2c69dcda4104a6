// ck_umma.cu — tensor-core (tcgen05 / TMEM) paths for the commitment
// products, and a self-test of the int8 tensor-core building block.
#include <cuda_runtime.h>

#include "../../include/salsaa_gpu.h"
#include "kernels.cuh"
#include "umma.cuh"

using namespace salsaa;

namespace {

// D (128 x N, s32) = A (128 x K, u8) * B (N x K, u8)^T on one CTA: the
// operands are packed into the canonical K-major layout by the threads, the
// MMAs are issued by one thread, and the accumulator is read back from TMEM.
__global__ void __launch_bounds__(128) umma_selftest_kernel(const uint8_t* A, const uint8_t* B, u32 N, u32 K,
                                                            int32_t* out, u32* err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  uint8_t* sa = sm;
  uint8_t* sb = sm + 128 * K;
  const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (u32 t = tid; t < 128 * K; t += 128) {
    const u32 r = t / K, k = t % K;
    sa[(k / 16) * (128 * 16) + r * 16 + k % 16] = A[t];
  }
  for (u32 t = tid; t < N * K; t += 128) {
    const u32 r = t / K, k = t % K;
    sb[(k / 16) * (N * 16) + r * 16 + k % 16] = B[t];
  }
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    umma::mbar_fence_init();
  }
  if (warp == 0) umma::tmem_alloc(&tslot, 256);
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const u32 tmem = tslot;
  if (tid == 0) {
    const u32 idesc = umma::idesc_u8(128, N);
    for (u32 ks = 0; ks < K / 32; ks++) {
      const uint64_t ad = umma::desc_kmajor(umma::smem_u32(sa + ks * 2 * 128 * 16), 128 * 16, 128);
      const uint64_t bd = umma::desc_kmajor(umma::smem_u32(sb + ks * 2 * N * 16), N * 16, 128);
      umma::mma_i8(tmem, ad, bd, idesc, ks > 0);
    }
    umma::commit(&mbar);
  }
  __syncwarp();
  bool ok = umma::mbar_wait(&mbar, 0, err, 1);
  ok = __all_sync(0xffffffffu, ok);
  umma::fence_after_sync();
  if (ok) {
    for (u32 c = 0; c < N; c += 16) {
      uint32_t r[16];
      umma::tmem_ld16(tmem + ((warp * 32) << 16) + c, r);
      umma::tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 16; j++) out[(warp * 32 + lane) * N + c + j] = (int32_t)r[j];
    }
  } else {
    umma::mbar_wait(&mbar, 0, err, 2);  // give an MMA in flight more time before freeing TMEM
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 256);
}

}  // namespace

extern "C" int salsaa_selftest_umma_i8(const uint8_t* d_a, const uint8_t* d_b, uint32_t n, uint32_t k,
                                       int32_t* d_out, void* stream) {
  if (!d_a || !d_b || !d_out) return salsaa_set_error(-1, "selftest_umma_i8: null argument");
  if (n < 16 || n > 256 || n % 16 || k == 0 || k > 256 || k % 32)
    return salsaa_set_error(-1, "selftest_umma_i8: needs 16 <= n <= 256 (multiple of 16), k multiple of 32 <= 256");
  cudaStream_t st = (cudaStream_t)stream;
  u32* err = nullptr;
  cudaError_t e = cudaMallocAsync(&err, sizeof(u32), st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "selftest_umma_i8: alloc");
  cudaMemsetAsync(err, 0, sizeof(u32), st);
  const size_t smem = (size_t)(128 + n) * k;
  e = cudaFuncSetAttribute(umma_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    umma_selftest_kernel<<<1, 128, smem, st>>>(d_a, d_b, n, k, d_out, err);
    salsaa_count_launch();
    e = cudaGetLastError();
  }
  u32 h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(u32), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFreeAsync(err, st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "selftest_umma_i8");
  if (h) return salsaa_set_error(-4, "selftest_umma_i8: tensor-core wait timed out");
  return 0;
}
