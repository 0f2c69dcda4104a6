// no_alloc.cu — allocation-free variant of the projection entry point.
//
// Some callers of this library cannot allocate device memory on the call path:
// a serving loop that has already divided HBM among the proofs in flight (a
// hidden cudaMalloc could fail, or push a co-resident proof out of memory),
// and host runtimes that own all device allocations themselves and forbid
// libraries from adding their own.  salsaa_project_noalloc() gives them the
// projection of src/subroutines/project.rs:50-103 with every piece of scratch
// (the challenge masks, the int8 challenge matrix and the device state word)
// taken from a fixed array compiled into this library instead of from an
// allocator.  The caller still passes the input witness and the output buffer.
#include <cstring>
#include <mutex>

#include "../../include/salsaa_gpu.h"
#include "kernels.cuh"

using namespace salsaa;

namespace {

// Largest chunk width the scratch covers: rows * 256 <= 2048, i.e. rows <= 8.
constexpr u32 NOALLOC_MAX_CW = 2048;
constexpr size_t NOALLOC_OFF_DS = 0;
constexpr size_t NOALLOC_OFF_POS = 1024;  // after DevState (rounded up)
constexpr size_t NOALLOC_MASK_BYTES = 256ULL * (NOALLOC_MAX_CW / 32) * sizeof(u32);
constexpr size_t NOALLOC_OFF_NEG = NOALLOC_OFF_POS + NOALLOC_MASK_BYTES;
constexpr size_t NOALLOC_OFF_J = NOALLOC_OFF_NEG + NOALLOC_MASK_BYTES;
constexpr size_t NOALLOC_BYTES = NOALLOC_OFF_J + 256ULL * NOALLOC_MAX_CW;  // 640 KiB + 1 KiB
static_assert(sizeof(DevState) <= NOALLOC_OFF_POS, "device state must fit its slot");

// One scratch array per device that loads this library; it lives until the
// process exits.  Every call uses the same array.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
// Per device: the CUDA context the address was looked up in, and the address.
// A device reset (or a caller that switches to another context on the same
// device) loads this module again, possibly at another address, so the cached
// address is only reused while the same context is current.
void* g_noalloc_ctx[NOALLOC_MAX_DEVICES] = {};
unsigned char* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};

typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn g_ctx_get_current = nullptr;

__global__ void noalloc_seed_kernel(DevState* ds, u64 seed) { ds->seed = seed; }

// The current driver context, through the runtime's driver entry-point lookup
// (no link-time dependency on the driver library).
int noalloc_current_ctx(void** ctx) {
  if (!g_ctx_get_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult qr;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &qr);
    if (e != cudaSuccess || qr != cudaDriverEntryPointSuccess || !fn)
      return salsaa_set_error(-1, "project_noalloc: cuCtxGetCurrent is not available");
    g_ctx_get_current = (CtxGetCurrentFn)fn;
  }
  *ctx = nullptr;
  if (g_ctx_get_current(ctx) != 0) return salsaa_set_error(-1, "project_noalloc: cuCtxGetCurrent failed");
  return 0;
}

// Device address of this device's scratch array, looked up with that device
// current the first time a context of it calls here (host code cannot use the
// symbol itself: in host code its name only stands in for the device array).
int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "project_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return salsaa_set_error(-1, "project_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  void* ctx = nullptr;
  int rc = noalloc_current_ctx(&ctx);
  if (rc) return rc;
  if (!ctx || !g_noalloc_addr[dev] || g_noalloc_ctx[dev] != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // makes the primary context current if none was
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "project_noalloc: cudaGetSymbolAddress");
    rc = noalloc_current_ctx(&ctx);
    if (rc) return rc;
    if (!ctx) return salsaa_set_error(-1, "project_noalloc: no current CUDA context");
    g_noalloc_addr[dev] = (unsigned char*)p;
    g_noalloc_ctx[dev] = ctx;
  }
  *out = g_noalloc_addr[dev];
  return 0;
}

}  // namespace

extern "C" int salsaa_project_noalloc(const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q,
                                      uint64_t seed, uint64_t round, uint64_t* d_out, void* stream) {
  if (!d_w || !d_out) return salsaa_set_error(-1, "project_noalloc: null argument");
  // rows is bounded before it is multiplied, so the product cannot wrap.
  if (rows == 0 || rows > NOALLOC_MAX_CW / 256)
    return salsaa_set_error(-3, "project_noalloc: rows * 256 exceeds the 2048-column scratch (at most 8 rows)");
  const u64 cw = rows * 256;
  if (cw > width || width % cw) return salsaa_set_error(-3, "project_noalloc: chunk width exceeds the witness width");
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  DevState* ds = (DevState*)(base + NOALLOC_OFF_DS);
  u32* pm = (u32*)(base + NOALLOC_OFF_POS);
  u32* nm = (u32*)(base + NOALLOC_OFF_NEG);
  int8_t* J = (int8_t*)(base + NOALLOC_OFF_J);
  // The array keeps the previous call's contents: the seed is written here
  // and the projection clears its overflow flag itself before use; the masks
  // and J are fully rewritten for this call's chunk width.
  noalloc_seed_kernel<<<1, 1, 0, st>>>(ds, seed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "project_noalloc: seed");
  rc = launch_proj_tables(ds, (u32)round, (u32)cw, pm, nm, J, nullptr, q, st);
  if (rc) return rc;
  RowSet w{};
  for (u64 k = 0; k < rows; k++) w.p[k] = d_w + k * width * d;
  return launch_project(w, (u32)rows, width, (u32)d, q, pm, nm, J, ds, d_out, st);
}
