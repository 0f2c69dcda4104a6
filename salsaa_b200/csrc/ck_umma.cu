// ck_umma.cu — tensor-core (tcgen05 / TMEM) paths for the commitment
// products, and a self-test of the int8 tensor-core building block.
#include <cuda_runtime.h>

#include "../../include/salsaa_gpu.h"
#include "kernels.cuh"
#include "ntt.cuh"
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

// ---------------------------------------------------------------------------
// Commitment-key rows on tcgen05 (q < 2^56).  Per NTT slot s the key rows'
// contribution to the commitment is a matrix product over F_q[X]/(X^2 - zeta):
// with the key power T = (c, d) and the witness value W = (a, b),
//   re = sum c a + zeta sum d b,    im = sum c b + sum d a.
// Every value is split into 7 bytes, so one u8 x u8 -> s32 tensor-core
// product per slot gives all four sums exactly (2048 byte products per block
// stay below 2^27):
//   A (M = 128): witness rows (k, part a|b, byte y), y-th byte of W,
//   B (N = nkp): key rows (r, comp c|d, byte x), x-th byte of T,
//   D[(k,p,y)][(r,c,x)] = sum_i byte_y(W_k,p(i)) byte_x(T_r,c(i)),
// and value = sum_{x,y} 2^(8(x+y)) D mod q.  The key bytes are laid out once
// per context in the operand's shared-memory image (ck_tk8), so each
// 64-element chunk of both slots' key tiles is one bulk copy.
//
// CTA = (slot pair s0, s0 + 1; block of Bw elements), warp-specialised per
// 64-element chunk, with no CTA-wide barrier inside the loop: warps 0..13
// load the witness pairs (one 16-byte load covers both slots) and split them
// into byte planes in shared memory, then arrive on the stage's a_full
// mbarrier; one thread of warp 14 bulk-copies the two key tiles as soon as
// the MMAs that read the stage's previous keys complete (key_full); one
// thread of warp 15 issues 2 x 2 MMAs (K = 32) into two TMEM accumulators
// once both are full, and commits them to the stage's done mbarrier, which
// frees the stage for the next witness and key copies.  Two stages.  Every
// wait is bounded; a role that gives up stops its loop, and the others then
// give up on the arrivals it no longer makes.  Epilogue: each thread reads its TMEM lane (one
// witness byte row), folds the key bytes x, the block's 7 y-rows are folded
// through shared memory, and the result is multiplied by the block's high
// key factor and added into the accumulator as in the CUDA-core path.
// ---------------------------------------------------------------------------
constexpr u32 CKU_CHUNK = 64;  // elements per pipeline step (K of 2 MMAs per slot)
constexpr u32 CKU_THREADS = 512;
constexpr u32 CKU_CONV = 448;  // witness-converting threads (warps 0..13); warps 14, 15 copy keys and issue MMAs
constexpr u32 CKU_ATILE = 128 * CKU_CHUNK;  // witness byte tile of one slot

__global__ void ck_tk8_kernel(const u64* tlo, u32 nck, u32 n, u32 bt, u32 nkp, bool packed, uint8_t* tk8) {
  const u64 tot = (u64)bt * n * nkp;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u32 b = (u32)(t % 16);
    u64 rest = t / 16;
    const u32 row = (u32)(rest % nkp);
    rest /= nkp;
    const u32 j = (u32)(rest % (CKU_CHUNK / 16));
    rest /= CKU_CHUNK / 16;
    const u32 s = (u32)(rest % n), cc = (u32)(rest / n);
    uint8_t v = 0;
    if (row < nck * 14) {
      const u32 r = row / 14, comp = (row / 7) % 2, x = row % 7;
      const u32 lo = cc * CKU_CHUNK + j * 16 + b;
      u64 val = tlo[((u64)r * bt + lo) * 3 * n + (u64)comp * n + s];
      if (packed) val = ((val >> 32) << 25) | (val & 0x1FFFFFFull);
      v = (uint8_t)(val >> (8 * x));
    }
    tk8[t] = v;
  }
}

__device__ u32 g_tc_error;  // set when a tensor-core wait gave up

// o_i = byte i of a, b, c, d (in that order, a in the low byte)
__device__ __forceinline__ void transpose4x4(u32 a, u32 b, u32 c, u32 d, u32& o0, u32& o1, u32& o2, u32& o3) {
  const u32 t0 = __byte_perm(a, b, 0x5140), t1 = __byte_perm(a, b, 0x7362);
  const u32 t2 = __byte_perm(c, d, 0x5140), t3 = __byte_perm(c, d, 0x7362);
  o0 = __byte_perm(t0, t2, 0x5410);
  o1 = __byte_perm(t0, t2, 0x7632);
  o2 = __byte_perm(t1, t3, 0x5410);
  o3 = __byte_perm(t1, t3, 0x7632);
}

// One CTA of the key-row product: element-block group `by` of the witness w
// (rows x width, slot form); its sums go to acc rows (r * acc_rows + koff + k).
__device__ __forceinline__ void ck_umma_body(const uint8_t* __restrict__ tk8, const RowSet& w, u32 rows, u32 G,
                                             u32 nck, u32 nkp, u32 n, u32 bt, u32 Bw, const u64* thi, u32 nhi_t,
                                             const ModQ& M, const u64* zeta, u64* acc, u32 acc_rows, u32 koff,
                                             bool plain, u32 by) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t key_full[2], a_full[2], done_bar[2];
  __shared__ uint32_t tslot, last_commit;
  const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const u32 s0 = 2 * blockIdx.x, d = 2 * n;
  // element blocks g < G of this CTA start at i0 + g bt: the same offsets in
  // the key block, so they share every key tile; their witness rows stack as
  // the virtual rows g * rows + k of the MMA's M dimension
  const u32 lob = bt / Bw, lo_b = by % lob, hg = by / lob;
  const u64 i0 = (u64)hg * G * bt + (u64)lo_b * Bw;
  const u32 vrows = rows * G;
  const u32 btile = nkp * CKU_CHUNK;                  // one slot's key tile
  const u32 stage_bytes = 2 * CKU_ATILE + 2 * btile;  // A0 A1 B0 B1
  const u32 nchunks = Bw / CKU_CHUNK;
  const u32 cc0 = (u32)((i0 % bt) / CKU_CHUNK);
  u32* err = &g_tc_error;

  // zero both stages' witness tiles once: rows >= 14 * rows stay zero
  for (u32 v = tid; v < 2 * 2 * CKU_ATILE / 16; v += CKU_THREADS) {
    const u32 st = v / (2 * CKU_ATILE / 16), o = v % (2 * CKU_ATILE / 16);
    *(uint4*)(smem + st * stage_bytes + o * 16) = make_uint4(0, 0, 0, 0);
  }
  // converter tasks: TS task slots per chunk (kp in groups of 4, elements in
  // quads).  When two groups of TS threads fit, group g takes the chunks
  // c = g mod 2, so few witness rows still keep many loads in flight.  At
  // most two groups: then each stage (c & 1) and its two barriers belong to
  // one group, whose chunks pass them in order; with more groups a group
  // could wait on a stage barrier more than one phase ahead, where a parity
  // wait cannot tell the phases apart.
  const u32 nkpw = 2 * vrows, kpb = (nkpw + 3) / 4, TS = 32 * kpb * (CKU_CHUNK / 32);
  const u32 NG = CKU_CONV / TS >= 2 ? 2 : 1;
  if (tid == 0) {
    for (int i = 0; i < 2; i++) {
      umma::mbar_init(&key_full[i], 1);
      umma::mbar_init(&a_full[i], TS);
      umma::mbar_init(&done_bar[i], 1);
    }
    last_commit = 0xffffffffu;
    umma::mbar_fence_init();
  }
  // two accumulators of nkp columns: 2 x 128 columns when they fit, so two
  // CTAs with small key tables can share an SM's 512 TMEM columns
  const u32 cs = nkp <= 128 ? 128 : 256;
  if (warp == 0) umma::tmem_alloc(&tslot, 2 * cs);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const u32 tmem = tslot;
  bool ok = true;

  if (tid < NG * TS) {
    // witness task t of group gi: (i4lo, kp within a group of 4, i4mid, kp
    // group, i4hi); kp = (virtual row, part).  The same task in every chunk
    // of the group: its source (chunk 0) and shared-memory offset are
    // computed once.  Four register buffers hold the loads of the group's
    // next four chunks.
    const u32 gi = tid / TS, t = tid % TS;
    const u32 i4lo = t & 3, kpi = (t >> 2) & 3, i4mid = (t >> 4) & 1, rest = t >> 5;
    const u32 kp = kpi + 4 * (rest % kpb), i4hi = rest / kpb;
    const bool tval = kp < nkpw;
    const u32 v = kp >> 1, part = kp & 1, k = tval ? v % rows : 0, g = tval ? v / rows : 0;
    const u32 i4 = (i4hi * 2 + i4mid) * 4 + i4lo;  // elements 4 * i4 .. + 3 of the chunk
    const u64* tsrc = w.p[k] + (i0 + (u64)g * bt + i4 * 4) * d + part * n + s0;
    const u32 toff = (i4 >> 2) * (128 * 16) + (kp * 7) * 16 + (i4 & 3) * 4;
    uint4 wb[4][4];
    auto fetch = [&](u32 c, uint4 (&wv)[4]) {
      if (tval) {
        const u64* src = tsrc + (u64)c * CKU_CHUNK * d;
#pragma unroll
        for (u32 e = 0; e < 4; e++) wv[e] = __ldg((const uint4*)(src + (u64)e * d));
      }
    };
    auto stash = [&](u32 st, const uint4 (&wv)[4]) {
      if (!tval) return;
      uint8_t* A = smem + st * stage_bytes;
      // byte plane b of the four elements: a 4 x 4 byte transpose of their
      // low words (planes 0..3) and high words (planes 4..6)
#pragma unroll
      for (u32 sg = 0; sg < 2; sg++) {
        u32 lo[4], hi[4], p[8];
#pragma unroll
        for (u32 e = 0; e < 4; e++) {
          lo[e] = sg ? wv[e].z : wv[e].x;
          hi[e] = sg ? wv[e].w : wv[e].y;
        }
        transpose4x4(lo[0], lo[1], lo[2], lo[3], p[0], p[1], p[2], p[3]);
        transpose4x4(hi[0], hi[1], hi[2], hi[3], p[4], p[5], p[6], p[7]);
#pragma unroll
        for (u32 b = 0; b < 7; b++) *(u32*)(A + sg * CKU_ATILE + toff + b * 16) = p[b];
      }
    };
    // chunk c = gi + NG m: stage c & 1 (last read by the MMAs of chunk c - 2),
    // loads in buffer m & 3, refilled with chunk c + 4 NG once stashed
    auto step = [&](u32 c, uint4 (&wv)[4]) -> bool {
      const u32 st = c & 1;
      if (c >= 2 && !umma::mbar_wait(&done_bar[st], ((c - 2) >> 1) & 1, err, 1)) return false;
      stash(st, wv);
      if (c + 4 * NG < nchunks) fetch(c + 4 * NG, wv);
      umma::fence_proxy_async();
      umma::mbar_arrive(&a_full[st]);
      return true;
    };
#pragma unroll
    for (u32 b = 0; b < 4; b++)
      if (gi + b * NG < nchunks) fetch(gi + b * NG, wb[b]);
    for (u32 c = gi; c < nchunks; c += 4 * NG) {
      if (!(ok = step(c, wb[0]))) break;
      if (c + NG < nchunks && !(ok = step(c + NG, wb[1]))) break;
      if (c + 2 * NG < nchunks && !(ok = step(c + 2 * NG, wb[2]))) break;
      if (c + 3 * NG < nchunks && !(ok = step(c + 3 * NG, wb[3]))) break;
    }
  } else if (warp == CKU_CONV / 32 && lane == 0) {
    // key tiles of both slots, one bulk copy per chunk, into the stage freed
    // by the MMAs of chunk c - 2
    u32 issued = 0;
    for (u32 c = 0; c < nchunks; c++) {
      const u32 st = c & 1;
      if (c >= 2 && !(ok = umma::mbar_wait(&done_bar[st], ((c - 2) >> 1) & 1, err, 4))) break;
      umma::mbar_expect_tx(&key_full[st], 2 * btile);
      umma::bulk_g2s(smem + st * stage_bytes + 2 * CKU_ATILE, tk8 + ((u64)(cc0 + c) * n + s0) * btile, 2 * btile,
                     &key_full[st]);
      issued = c + 1;
    }
    // the copies still in flight (the last one of each stage) land before the CTA moves on
    for (u32 c = issued >= 2 ? issued - 2 : 0; c < issued; c++)
      umma::mbar_wait(&key_full[c & 1], (c >> 1) & 1, err, 5);
  } else if (warp == CKU_CONV / 32 + 1 && lane == 0) {
    const u32 idesc = umma::idesc_u8(128, nkp);
    for (u32 c = 0; c < nchunks; c++) {
      const u32 st = c & 1;
      uint8_t* stage = smem + st * stage_bytes;
      if (!(ok = umma::mbar_wait(&a_full[st], (c >> 1) & 1, err, 2))) break;
      if (!(ok = umma::mbar_wait(&key_full[st], (c >> 1) & 1, err, 2))) break;
      umma::fence_after_sync();
#pragma unroll
      for (u32 sg = 0; sg < 2; sg++)
#pragma unroll
        for (u32 ks = 0; ks < CKU_CHUNK / 32; ks++) {
          const uint64_t ad =
              umma::desc_kmajor(umma::smem_u32(stage + sg * CKU_ATILE + ks * 2 * 128 * 16), 128 * 16, 128);
          const uint64_t bd =
              umma::desc_kmajor(umma::smem_u32(stage + 2 * CKU_ATILE + sg * btile + ks * 2 * nkp * 16), nkp * 16, 128);
          umma::mma_i8(tmem + sg * cs, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
        }
      umma::commit(&done_bar[st]);
      last_commit = c;
    }
  }
  // all MMAs done (the last commit covers every earlier MMA of its thread)
  __syncthreads();
  const u32 lc = last_commit;
  if (lc != 0xffffffffu) ok &= umma::mbar_wait(&done_bar[lc & 1], (lc >> 1) & 1, err, 3);
  ok &= lc == nchunks - 1;
  ok = __syncthreads_and(ok);
  umma::fence_after_sync();

  // ---- epilogue ----
  u64* Pm = (u64*)smem;  // [slot][128 lanes][2 nck] partial sums over x
  const u32 ng = 2 * nck;
  // warp w: slot (w >> 2) & 1, TMEM lanes 32 (w & 3) .., and one half of the
  // 2 nck column groups (w >> 3), split at a group boundary
  const u32 sg = (warp >> 2) & 1, row = (warp & 3) * 32 + lane, ch = warp >> 3;
  if (ok) {
    const bool valid = row < vrows * 14;
    const u32 y = row % 7;
    const u64 pw = ((u64)1 << (8 * y)) % M.q;
    const u32 jb = 7 * (ch ? nck : 0), je = 7 * (ch ? 2 * nck : nck);
    u64 hi = 0, lo = 0;
    for (u32 cb = jb / 16; cb * 16 < je; cb++) {
      uint32_t r[16];
      umma::tmem_ld16(tmem + (((warp & 3) * 32) << 16) + sg * cs + cb * 16, r);
      umma::tmem_wait_ld();
#pragma unroll
      for (u32 i = 0; i < 16; i++) {
        const u32 j = cb * 16 + i;
        if (j >= jb && j < je) {
          const u32 x = j % 7;
          const u64 v = (u64)r[i];
          const u64 sl = v << (8 * x), sh = x ? (v >> (64 - 8 * x)) : 0;
          lo += sl;
          hi += sh + (lo < sl);
          if (x == 6) {
            u64 p = (M.s >= 39) ? barrett128(M, hi, lo) : reduce128_any(M, hi, lo);
            if (valid) Pm[((u64)sg * 128 + row) * ng + j / 7] = mul_mod(M, p, pw);
            hi = lo = 0;
          }
        }
      }
    }
  }
  __syncthreads();
  if (ok) {
    for (u32 t = tid; t < 2 * vrows * nck; t += CKU_THREADS) {
      const u32 r = t % nck, v = (t / nck) % vrows, g2 = t / (nck * vrows);
      const u32 k = v % rows, hi_t = (u32)(i0 / bt) + v / rows;
      const u32 s = s0 + g2;
      const u64* P = Pm + (u64)g2 * 128 * ng;
      u64 ca = 0, db = 0, cb = 0, da = 0;
#pragma unroll
      for (u32 y = 0; y < 7; y++) {
        const u64* pa = P + (u64)((2 * v) * 7 + y) * ng;      // part a rows
        const u64* pb = P + (u64)((2 * v + 1) * 7 + y) * ng;  // part b rows
        ca = salsaa::add_mod(ca, pa[2 * r], M.q);
        da = salsaa::add_mod(da, pa[2 * r + 1], M.q);
        cb = salsaa::add_mod(cb, pb[2 * r], M.q);
        db = salsaa::add_mod(db, pb[2 * r + 1], M.q);
      }
      u64 re = salsaa::add_mod(ca, mul_mod(M, zeta[s], db), M.q);
      u64 im = salsaa::add_mod(cb, da, M.q);
      const u64* th = thi + ((u64)r * nhi_t + hi_t) * d;
      slot_mul(M, re, im, th[s], th[n + s], zeta[s], re, im);
      u64* dst = acc + ((u64)r * acc_rows + koff + k) * d;
      atomic_add_mod(dst + s, re, M.q, plain);
      atomic_add_mod(dst + n + s, im, M.q, plain);
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 2 * cs);
}

__global__ void __launch_bounds__(CKU_THREADS, 1)
    ck_umma_kernel(const uint8_t* __restrict__ tk8, RowSet w, u32 rows, u32 G, u32 nck, u32 nkp, u32 n, u32 bt,
                   u32 Bw, const u64* thi, u32 nhi_t, ModQ M, const u64* zeta, u64* acc, bool plain) {
  ck_umma_body(tk8, w, rows, G, nck, nkp, n, bt, Bw, thi, nhi_t, M, zeta, acc, rows, 0, plain, blockIdx.y);
}

// Several witnesses (uneven widths and row counts) against the same key rows
// in one launch: witness i owns the grid rows [ystart[i], ystart[i+1]) and
// its own accumulator acc[i] (nck x rows[i] ring elements).
struct CkMulti {
  RowSet w[CKU_MULTI_MAX];
  u64* acc[CKU_MULTI_MAX];
  u32 rows[CKU_MULTI_MAX], G[CKU_MULTI_MAX], Bw[CKU_MULTI_MAX];
  u32 ystart[CKU_MULTI_MAX + 1];
  uint8_t plain[CKU_MULTI_MAX];
  u32 count;
};

__global__ void __launch_bounds__(CKU_THREADS, 1)
    ck_umma_multi_kernel(const uint8_t* __restrict__ tk8, CkMulti m, u32 nck, u32 nkp, u32 n, u32 bt,
                         const u64* thi, u32 nhi_t, ModQ M, const u64* zeta) {
  u32 i = 0;
  while (i + 1 < m.count && m.ystart[i + 1] <= blockIdx.y) i++;
  ck_umma_body(tk8, m.w[i], m.rows[i], m.G[i], nck, nkp, n, bt, m.Bw[i], thi, nhi_t, M, zeta, m.acc[i], m.rows[i],
               0, m.plain[i] != 0, blockIdx.y - m.ystart[i]);
}

}  // namespace

namespace salsaa {

int launch_ck_tk8(const u64* tlo, u32 nck, u32 n, u32 bt, bool packed, uint8_t* tk8, cudaStream_t st) {
  const u32 nkp = ck_tk8_nkp(nck);
  const u64 tot = (u64)bt * n * nkp;
  u64 g = (tot + 255) / 256;
  if (g > 65535 * 16) g = 65535 * 16;
  ck_tk8_kernel<<<(unsigned)g, 256, 0, st>>>(tlo, nck, n, bt, nkp, packed, tk8);
  salsaa_count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "ck_tk8");
}

// The smallest shared-memory carveout (percent of the SM's 228 KiB) that
// holds one CTA's stages plus its static barriers: the rest stays L1, which
// holds the witness loads in flight (one 16-byte load per 32-byte sector).
static int ck_carveout(size_t smem) {
  const size_t need = smem + 2048;
  const size_t pct = (need * 100 + 228 * 1024 - 1) / (228 * 1024);
  return pct > 100 ? 100 : (int)pct;
}

bool ck_umma_ok(const CommitArgs& a, u32 n) {
  if (!a.tk8 || a.rows == 0 || a.rows > CKU_MAX_WROWS || a.nck == 0 || a.nck > CKU_MAX_KEYS || (n & 1)) return false;
  if (a.width < CKU_CHUNK || a.ck_bt < CKU_CHUNK) return false;
  for (u32 k = 0; k < a.rows; k++)
    if ((uintptr_t)a.w.p[k] % 16) return false;
  return true;
}

void ck_umma_shape(u64 width, u32 rows, u32 n, u32 ck_bt, u32* Bk_out, u32* G_out) {
  // element block per CTA: a whole key-table block (one epilogue per block),
  // halved while the grid would not fill the GPU
  u32 Bk = (u32)(width < ck_bt ? width : ck_bt);
  while (Bk > CK_BLOCK && (u64)(n / 2) * (width / Bk) < 296) Bk /= 2;
  // few witness rows: G blocks one key block apart per CTA share the key
  // tiles (virtual rows g * rows + k), while the grid keeps a full wave
  u32 G = 1;
  while (width >= ck_bt && rows * G * 2 <= CKU_MAX_WROWS && (width / ck_bt) % (G * 2) == 0 &&
         (u64)(n / 2) * (width / Bk) / (G * 2) >= 148)
    G *= 2;
  *Bk_out = Bk;
  *G_out = G;
}

int launch_ck_umma_multi(const CommitArgs* a, u32 ninst, u32 n, const ModQ& M, const u64* zeta, cudaStream_t st) {
  if (ninst == 0 || ninst > CKU_MULTI_MAX) return salsaa_set_error(-2, "ck_umma_multi: 1..8 witnesses per launch");
  CkMulti m{};
  u32 y = 0;
  double wit_bytes = 0, out_bytes = 0, ops = 0, macs = 0;
  for (u32 i = 0; i < ninst; i++) {
    const CommitArgs& c = a[i];
    if (!ck_umma_ok(c, n) || c.nck != a[0].nck || c.tk8 != a[0].tk8)
      return salsaa_set_error(-2, "ck_umma_multi: a witness does not fit the tensor-core key-row product");
    u32 Bk, G;
    ck_umma_shape(c.width, c.rows, n, c.ck_bt, &Bk, &G);
    if (c.rows * G > CKU_MAX_WROWS || c.ck_bt % Bk || c.width % ((u64)Bk * G))
      return salsaa_set_error(-2, "ck_umma_multi: bad block grouping");
    u64 CH = c.width / 512;
    if (CH < 128) CH = 128;
    if (CH > Bk) CH = Bk;
    m.w[i] = c.w;
    m.rows[i] = c.rows;
    m.G[i] = G;
    m.Bw[i] = Bk;
    m.acc[i] = c.acc;
    m.plain[i] = (M.q < (1ULL << 50) && (c.width / CH) < (1ULL << 13)) ? 1 : 0;
    m.ystart[i] = y;
    y += (u32)(c.width / Bk / G);
    wit_bytes += 8.0 * c.rows * (double)c.width * 2 * n;
    out_bytes += 8.0 * c.nck * c.rows * 2 * n;
    ops += 2.0 * 196.0 * c.nck * c.rows * (double)c.width * n;
    macs += (double)c.nck * c.rows * (double)c.width * 2 * n;
  }
  m.ystart[ninst] = y;
  m.count = ninst;
  const u32 nck = a[0].nck, nkp = ck_tk8_nkp(nck);
  const size_t stage = 2 * (size_t)CKU_ATILE + 2 * (size_t)nkp * CKU_CHUNK;
  const size_t epi = 2 * 128 * (size_t)(2 * nck) * sizeof(u64);
  const size_t smem = 2 * stage > epi ? 2 * stage : epi;
  cudaError_t e =
      cudaFuncSetAttribute(ck_umma_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ck_umma_multi_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, ck_carveout(smem));
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "ck_umma_multi smem attribute");
  const int tr = salsaa_trace_begin("ck_umma_kernel", st, wit_bytes + out_bytes);
  salsaa_trace_alias(tr, "ck_umma_kernel:int8", ops);
  salsaa_trace_alias(tr, "ck_umma_kernel:mac", macs);
  ck_umma_multi_kernel<<<dim3(n / 2, y), CKU_THREADS, smem, st>>>(a[0].tk8, m, nck, nkp, n, a[0].ck_bt, a[0].thi,
                                                                   a[0].ck_nhi, M, zeta);
  salsaa_trace_end(tr, st);
  salsaa_count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "ck_umma_multi launch");
}

int launch_ck_umma(const CommitArgs& a, u32 n, u32 Bw, u32 G, const ModQ& M, const u64* zeta, bool plain,
                   cudaStream_t st) {
  if (G == 0 || a.rows * G > CKU_MAX_WROWS || (G > 1 && (a.width < a.ck_bt || (a.width / a.ck_bt) % G)) ||
      a.ck_bt % Bw || a.width % ((u64)Bw * G))
    return salsaa_set_error(-2, "ck_umma: bad block grouping");
  const u32 nkp = ck_tk8_nkp(a.nck);
  const size_t stage = 2 * (size_t)CKU_ATILE + 2 * (size_t)nkp * CKU_CHUNK;
  const size_t epi = 2 * 128 * (size_t)(2 * a.nck) * sizeof(u64);
  const size_t smem = 2 * stage > epi ? 2 * stage : epi;
  cudaError_t e = cudaFuncSetAttribute(ck_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ck_umma_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, ck_carveout(smem));
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "ck_umma smem attribute");
  dim3 g(n / 2, (unsigned)(a.width / Bw / G));
  // Traced measures of one launch: algorithmic HBM bytes (the slot-form
  // witness read once, the accumulators written once), the int8 operations
  // the tensor cores execute (2 x 14 x 14 byte products per key row, witness
  // row, element and slot pair half), and the exact mod-q multiply-accumulates
  // of the ring products (2d per key row, witness row and element).
  const double wit_bytes = 8.0 * a.rows * (double)a.width * 2 * n;
  const double out_bytes = 8.0 * a.nck * a.rows * 2 * n;
  const int tr = salsaa_trace_begin("ck_umma_kernel", st, wit_bytes + out_bytes);
  salsaa_trace_alias(tr, "ck_umma_kernel:int8", 2.0 * 196.0 * a.nck * a.rows * (double)a.width * n);
  salsaa_trace_alias(tr, "ck_umma_kernel:mac", (double)a.nck * a.rows * (double)a.width * 2 * n);
  ck_umma_kernel<<<g, CKU_THREADS, smem, st>>>(a.tk8, a.w, a.rows, G, a.nck, nkp, n, a.ck_bt, Bw, a.thi, a.ck_nhi,
                                               M, zeta, a.acc, plain);
  salsaa_trace_end(tr, st);
  salsaa_count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "ck_umma launch");
}

// ---------------------------------------------------------------------------
// Projection on tcgen05 (project, src/subroutines/project.rs:50-103): per
// chunk of cw witness elements, out[256 x d] = J (256 x cw, entries -1/0/1) x
// W (cw x d, centre-lifted, int8).  CTA = (chunk, block of 128 coefficient
// positions); per 128-element step thread 0 bulk-copies both 128-row halves
// of J from their canonical image (Jc, see launch_proj_tables) and issues
// 2 x 4 MMAs (kind::i8, signed x signed, M = 128 J rows, N = 128 positions,
// K = 32) into two TMEM accumulators; the threads convert the witness step to
// int8 in the canonical layout.  A value outside [-128, 127] sets the flag and
// the exact CUDA-core kernel recomputes every output (same as the mma.sync
// path).  Two stages: the witness of step c + 1 is staged while the MMAs of
// step c run.
// ---------------------------------------------------------------------------
constexpr u32 PU_POS = 128, PU_KS = 64;
constexpr u32 PU_IMG = 2 * 128 * 128;  // Jc: both J halves of one 128-element chunk (32 KiB)
constexpr u32 PU_A = 2 * 128 * PU_KS;  // both J halves of one step (16 KiB)
constexpr u32 PU_B = PU_POS * PU_KS;   // witness int8 tile (8 KiB)
constexpr u32 PU_STAGE = PU_A + PU_B;

__global__ void __launch_bounds__(256, 2)
    project_umma_kernel(RowSet in, u32 d, u64 q, u32 cw, u64 nch, const int8_t* __restrict__ Jc,
                        u64* __restrict__ out, u64* flag) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t full_bar[2], done_bar[2];
  __shared__ uint32_t tslot;
  const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const u32 nblk = blockIdx.x;
  const u64 idx = blockIdx.y;
  const u32 i = (u32)(idx / nch);
  const u64 j = idx % nch;
  const bool nar = (in.narrow >> i) & 1;
  const u64* chunk = row_advance(in.p[i], nar, (j * cw) * d + (u64)nblk * PU_POS);
  const u64 half_q = q >> 1;
  const u32 nsteps = cw / PU_KS;
  u32* err = &g_tc_error;
  if (tid == 0) {
    for (int b = 0; b < 2; b++) {
      umma::mbar_init(&full_bar[b], 1);
      umma::mbar_init(&done_bar[b], 1);
    }
    umma::mbar_fence_init();
  }
  if (warp == 0) umma::tmem_alloc(&tslot, 256);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const u32 tmem = tslot;
  // signed int8 x signed int8 -> s32, M = N = 128
  const u32 idesc = umma::idesc_u8(128, PU_POS) | (1u << 7) | (1u << 10);
  bool bad = false, ok = true;
  // task of this thread: 16 consecutive elements x 2 neighbouring positions,
  // one 16-byte load per element for word rows (two u64 values) and one
  // 8-byte load for narrow rows (two int32 values, kept in wv[e].x); a
  // step's values stay in registers from their loads (issued before the
  // previous step's barrier) to their conversion
  ulonglong2 wv[16];
  const u32 nkq = tid >> 6, np2 = tid & 63;
  auto load = [&](u32 c) {
    if (nar) {
      const int* src = (const int*)chunk + (u64)c * PU_KS * d;
#pragma unroll
      for (u32 e = 0; e < 16; e++)
        wv[e].x = (u64)__ldg((const long long*)(src + (u64)(16 * nkq + e) * d + 2 * np2));
    } else {
      const u64* src = chunk + (u64)c * PU_KS * d;
#pragma unroll
      for (u32 e = 0; e < 16; e++) wv[e] = __ldg((const ulonglong2*)(src + (u64)(16 * nkq + e) * d + 2 * np2));
    }
  };
  load(0);
  for (u32 c = 0; c < nsteps; c++) {
    const u32 st = c & 1;
    uint8_t* stage = smem + st * PU_STAGE;
    if (c >= 2) ok &= umma::mbar_wait(&done_bar[st], ((c - 2) >> 1) & 1, err, 1);
    if (tid == 0) {  // K slices of this step from the chunk's image, one copy per J half
      umma::mbar_expect_tx(&full_bar[st], PU_A);
      const int8_t* img = Jc + (u64)(c / 2) * PU_IMG + (c % 2) * (PU_A / 2);
      umma::bulk_g2s(stage, img, PU_A / 2, &full_bar[st]);
      umma::bulk_g2s(stage + PU_A / 2, img + PU_IMG / 2, PU_A / 2, &full_bar[st]);
    }
    // witness step: 128 positions x 64 elements as int8, (k / 16, pos, k % 16):
    // the 16 bytes of one position are one 16-byte store
    uint8_t* B = stage + PU_A;
#pragma unroll
    for (u32 p = 0; p < 2; p++) {
      u32 w4[4];
#pragma unroll
      for (u32 g = 0; g < 4; g++) {
        u32 tq[4];  // centred value + 128: below 256 iff it fits int8
#pragma unroll
        for (u32 e = 0; e < 4; e++) {
          const ulonglong2 v2 = wv[4 * g + e];
          if (nar) {
            const int cv = (int)(u32)(p ? (v2.x >> 32) : v2.x);
            bad |= (cv > 127) | (cv < -128);
            tq[e] = (u32)cv + 128u;
          } else {
            const u64 v = p ? v2.y : v2.x;
            const long long cv = v > half_q ? (long long)v - (long long)q : (long long)v;
            const unsigned long long tb = (unsigned long long)(cv + 128);
            bad |= tb > 255ULL;
            tq[e] = (u32)tb;
          }
        }
        // low bytes of the four values, e in byte e
        const u32 packed =
            __byte_perm(__byte_perm(tq[0], tq[1], 0x0040), __byte_perm(tq[2], tq[3], 0x0040), 0x5410);
        w4[g] = packed ^ 0x80808080u;
      }
      *(uint4*)(B + nkq * (PU_POS * 16) + (2 * np2 + p) * 16) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
    if (c + 1 < nsteps) load(c + 1);
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      ok &= umma::mbar_wait(&full_bar[st], (c >> 1) & 1, err, 2);
#pragma unroll
      for (u32 h = 0; h < 2; h++)
#pragma unroll
        for (u32 ks = 0; ks < PU_KS / 32; ks++) {
          const uint64_t ad =
              umma::desc_kmajor(umma::smem_u32(stage + h * (PU_A / 2) + ks * 2 * 128 * 16), 128 * 16, 128);
          const uint64_t bd = umma::desc_kmajor(umma::smem_u32(B + ks * 2 * PU_POS * 16), PU_POS * 16, 128);
          umma::mma_i8(tmem + h * 128, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
        }
      umma::commit(&done_bar[st]);
    }
  }
  ok &= umma::mbar_wait(&done_bar[(nsteps - 1) & 1], ((nsteps - 1) >> 1) & 1, err, 3);
  ok = __syncthreads_and(ok);
  if (bad) atomicOr((unsigned long long*)flag, 1ULL);
  umma::fence_after_sync();
  if (ok) {
    const u32 h = warp >> 2, row = (warp & 3) * 32 + lane;
    u64* dst = out + ((idx * 256) + h * 128 + row) * d + (u64)nblk * PU_POS;
    for (u32 cb = 0; cb < PU_POS; cb += 16) {
      uint32_t r[16];
      umma::tmem_ld16(tmem + (((warp & 3) * 32) << 16) + h * 128 + cb, r);
      umma::tmem_wait_ld();
#pragma unroll
      for (u32 e = 0; e < 16; e += 2) {
        const int v0 = (int)r[e], v1 = (int)r[e + 1];
        const u64 a = v0 >= 0 ? (u64)v0 : q - (u64)(-(long long)v0);
        const u64 b = v1 >= 0 ? (u64)v1 : q - (u64)(-(long long)v1);
        *(ulonglong2*)(dst + cb + e) = make_ulonglong2(a, b);
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 256);
}

int launch_project_umma(RowSet in, u32 rows, u64 nch, u32 d, u64 q, u32 cw, const int8_t* Jc, u64* out, u64* flag,
                        cudaStream_t st) {
  const size_t smem = 2 * (size_t)PU_STAGE;
  cudaError_t e = cudaFuncSetAttribute(project_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "project_umma smem attribute");
  dim3 g(d / PU_POS, (unsigned)(rows * nch));
  project_umma_kernel<<<g, 256, smem, st>>>(in, d, q, cw, nch, Jc, out, flag);
  salsaa_count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "project_umma launch");
}

// ---------------------------------------------------------------------------
// TENSOR statement rows on tcgen05 (the scalar rows of
// parallel_dot_series_matrix, src/arithmetic.rs:459-505, whose weights are
// s(i) = s_hi[i / Bw] s_lo[i % Bw]), over the coefficient-form witness.
// For one witness row k, one block of Bw elements (one s_hi factor) and 128
// coefficient positions, sum_i s_lo(i) w(i) is an integer matrix product:
//   A (M = 128): rows (tensor row r, byte x) of s_lo, unsigned bytes,
//   B (N = 128): coefficient positions, the centred witness split into three
//     signed byte limbs (exact for |w| < 2^23), one MMA chain per limb,
//   D_l[(r,x)][pos] = sum_i byte_x(s_lo(i)) limb_l(w(i, pos)),
// and the row sum is sum_{x,l} 2^(8(x+l)) D_l mod q.  A CTA that meets a
// larger value adds nothing and flags itself; sc_exact_kernel then redoes
// exactly the flagged CTAs on CUDA cores.  The sums land in the coefficient-
// form accumulators that launch_commit moves to slot form.
// ---------------------------------------------------------------------------
constexpr u32 SU_POS = 128, SU_KS = 128, SU_LIMBS = 3;
constexpr u32 SU_A = 128 * SU_KS;                   // scalar byte tile (16 KiB)
constexpr u32 SU_B = SU_POS * SU_KS;                // one limb tile (16 KiB)
constexpr u32 SU_STAGE = SU_A + SU_LIMBS * SU_B;    // 64 KiB

__global__ void sc_img_kernel(const u64* s_lo, u32 Bw, ScRowList tl, uint8_t* img) {
  const u64 tot = (u64)Bw * 128;  // (chunk, slice, row, byte) = Bw / 128 x 8 x 128 x 16
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (u64)gridDim.x * blockDim.x) {
    const u32 b = (u32)(t % 16), row = (u32)((t / 16) % 128), sl = (u32)((t / 2048) % 8), cc = (u32)(t / 16384);
    uint8_t v = 0;
    if (row < tl.n * 7) {
      const u32 r = row / 7, x = row % 7;
      v = (uint8_t)(s_lo[(u64)tl.idx[r] * Bw + cc * 128 + sl * 16 + b] >> (8 * x));
    }
    img[t] = v;
  }
}

__global__ void __launch_bounds__(512, 1)
    sc_umma_kernel(RowSet wc, u32 rows, u32 d, u32 Bw, u32 nhi, u32 split, ScRowList tl,
                   const uint8_t* __restrict__ img, const u64* s_hi, ModQ M, u64* acc, bool plain, u32* flags) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t full_bar[2], done_bar[2];
  __shared__ uint32_t tslot;
  const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // CTA: positions pb, element block hb (one s_hi factor), its part sub of split
  const u32 pb = blockIdx.x, hb = blockIdx.y / split, sub = blockIdx.y % split, k = blockIdx.z;
  const u64 q = M.q, half_q = q >> 1;
  const u32 nsteps = Bw / SU_KS / split, c0 = sub * nsteps;
  const bool nar = (wc.narrow >> k) & 1;
  const u64* src0 = row_advance(wc.p[k], nar, ((u64)hb * Bw + (u64)c0 * SU_KS) * d + (u64)pb * SU_POS);
  img += (u64)c0 * SU_A;
  u32* err = &g_tc_error;
  if (tid == 0) {
    for (int b = 0; b < 2; b++) {
      umma::mbar_init(&full_bar[b], 1);
      umma::mbar_init(&done_bar[b], 1);
    }
    umma::mbar_fence_init();
  }
  if (warp == 0) umma::tmem_alloc(&tslot, 512);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const u32 tmem = tslot;
  // unsigned bytes (A) x signed bytes (B) -> s32, M = N = 128
  const u32 idesc = umma::idesc_u8(128, SU_POS) | (1u << 10);
  bool bad = false, ok = true;
  // task of this thread: 16 consecutive elements x 2 neighbouring positions,
  // one 16-byte load per element for word rows (two u64 values) and one
  // 8-byte load for narrow rows (two int32 values, kept in wv[e].x); one
  // 16-byte store per limb plane and position
  ulonglong2 wv[16];
  const u32 nkq = tid >> 6, np2 = tid & 63;
  auto load = [&](u32 c) {
    if (nar) {
      const int* src = (const int*)src0 + (u64)c * SU_KS * d;
#pragma unroll
      for (u32 e = 0; e < 16; e++)
        wv[e].x = (u64)__ldg((const long long*)(src + (u64)(16 * nkq + e) * d + 2 * np2));
    } else {
      const u64* src = src0 + (u64)c * SU_KS * d;
#pragma unroll
      for (u32 e = 0; e < 16; e++) wv[e] = __ldg((const ulonglong2*)(src + (u64)(16 * nkq + e) * d + 2 * np2));
    }
  };
  load(0);
  for (u32 c = 0; c < nsteps; c++) {
    const u32 st = c & 1;
    uint8_t* stage = smem + st * SU_STAGE;
    if (c >= 2) ok &= umma::mbar_wait(&done_bar[st], ((c - 2) >> 1) & 1, err, 1);
    if (tid == 0) {
      umma::mbar_expect_tx(&full_bar[st], SU_A);
      umma::bulk_g2s(stage, img + (u64)c * SU_A, SU_A, &full_bar[st]);
    }
#pragma unroll
    for (u32 p = 0; p < 2; p++) {
      u32 l0[4], l1[4], l2[4];
#pragma unroll
      for (u32 g = 0; g < 4; g++) {
        u32 wq[4];
#pragma unroll
        for (u32 e = 0; e < 4; e++) {
          const ulonglong2 v2 = wv[4 * g + e];
          // centred value + 0x808080: its bytes are the signed limbs + 128 when
          // the value lies in [-0x808080, 0x7f7f7f] (three balanced base-256 digits)
          if (nar) {
            const int v = (int)(u32)(p ? (v2.x >> 32) : v2.x);
            bad |= (v > 0x7f7f7f) | (v < -0x808080);  // the value needs a fourth limb
            wq[e] = ((u32)v + 0x808080u) ^ 0x808080u;
          } else {
            const u64 v = p ? v2.y : v2.x;
            const u64 tb = v + 0x808080ULL - (v > half_q ? q : 0);
            bad |= (tb >> 24) != 0;
            wq[e] = (u32)tb ^ 0x808080u;
          }
        }
        // limb planes of the four values: byte l of wq[0..3]
        const u32 lo01 = __byte_perm(wq[0], wq[1], 0x5140), lo23 = __byte_perm(wq[2], wq[3], 0x5140);
        const u32 hi01 = __byte_perm(wq[0], wq[1], 0x0062), hi23 = __byte_perm(wq[2], wq[3], 0x0062);
        l0[g] = __byte_perm(lo01, lo23, 0x5410);
        l1[g] = __byte_perm(lo01, lo23, 0x7632);
        l2[g] = __byte_perm(hi01, hi23, 0x5410);
      }
      const u32 off = SU_A + nkq * (SU_POS * 16) + (2 * np2 + p) * 16;
      *(uint4*)(stage + off) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
      *(uint4*)(stage + off + SU_B) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
      *(uint4*)(stage + off + 2 * SU_B) = make_uint4(l2[0], l2[1], l2[2], l2[3]);
    }
    if (c + 1 < nsteps) load(c + 1);
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      ok &= umma::mbar_wait(&full_bar[st], (c >> 1) & 1, err, 2);
#pragma unroll
      for (u32 l = 0; l < SU_LIMBS; l++)
#pragma unroll
        for (u32 ks = 0; ks < SU_KS / 32; ks++) {
          const uint64_t ad = umma::desc_kmajor(umma::smem_u32(stage + ks * 2 * 128 * 16), 128 * 16, 128);
          const uint64_t bd =
              umma::desc_kmajor(umma::smem_u32(stage + SU_A + l * SU_B + ks * 2 * SU_POS * 16), SU_POS * 16, 128);
          umma::mma_i8(tmem + l * 128, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
        }
      umma::commit(&done_bar[st]);
    }
  }
  ok &= umma::mbar_wait(&done_bar[(nsteps - 1) & 1], ((nsteps - 1) >> 1) & 1, err, 3);
  ok = __syncthreads_and(ok);
  bad = __syncthreads_or(bad);
  umma::fence_after_sync();
  const u32 cta = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  if (bad && tid == 0) flags[cta] = 1;
  if (ok && !bad) {
    // per TMEM lane (row (r, x)), per position: sum_l 2^(8l) D_l, reduced, times 2^(8x)
    u64* Pm = (u64*)smem;  // 128 rows x 128 positions
    const u32 row = (warp & 3) * 32 + lane, quarter = warp >> 2;  // four groups of 32 positions
    const u32 x = row % 7;
    const u64 pw = ((u64)1 << (8 * x)) % q;
    const u64 cpos = ((((u64)1 << 62) / q) + 1) * q;
    for (u32 cb = quarter * 32; cb < quarter * 32 + 32; cb += 16) {
      uint32_t r0[16], r1[16], r2[16];
      const u32 base = tmem + (((warp & 3) * 32) << 16) + cb;
      umma::tmem_ld16(base, r0);
      umma::tmem_ld16(base + 128, r1);
      umma::tmem_ld16(base + 256, r2);
      umma::tmem_wait_ld();
#pragma unroll
      for (u32 e = 0; e < 16; e++) {
        const long long v = (long long)(int)r0[e] + ((long long)(int)r1[e] << 8) + ((long long)(int)r2[e] << 16);
        const u64 red = reduce64(M, v < 0 ? (u64)(v + (long long)cpos) : (u64)v);
        Pm[(u64)row * 128 + cb + e] = mul_mod(M, red, pw);
      }
    }
  }
  __syncthreads();
  if (ok && !bad) {
    const u64* Pm = (const u64*)smem;
    for (u32 t = tid; t < tl.n * SU_POS; t += 512) {
      const u32 r = t / SU_POS, pos = t % SU_POS;
      u64 v = 0;
#pragma unroll
      for (u32 x = 0; x < 7; x++) v = salsaa::add_mod(v, Pm[(u64)(r * 7 + x) * 128 + pos], q);
      const u32 j = tl.idx[r];
      v = mul_mod(M, v, s_hi[(u64)j * nhi + hb]);
      atomic_add_mod(acc + ((u64)j * rows + k) * d + (u64)pb * SU_POS + pos, v, q, plain);
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
}

// Exact CUDA-core sums for the CTAs sc_umma_kernel flagged (same grid).
__global__ void sc_exact_kernel(RowSet wc, u32 rows, u32 d, u32 Bw, u32 nhi, u32 split, ScRowList tl,
                                const u64* s_lo, const u64* s_hi, ModQ M, u64* acc, bool plain, const u32* flags) {
  const u32 cta = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  if (!flags[cta]) return;
  const u32 pb = blockIdx.x, hb = blockIdx.y / split, sub = blockIdx.y % split, k = blockIdx.z, pos = threadIdx.x;
  const u32 i0 = sub * (Bw / split), i1 = i0 + Bw / split;
  const bool nar = (wc.narrow >> k) & 1;
  const u64* src = row_advance(wc.p[k], nar, ((u64)hb * Bw) * d + (u64)pb * SU_POS + pos);
  for (u32 r = 0; r < tl.n; r++) {
    const u32 j = tl.idx[r];
    u64 v = 0;
    for (u32 i = i0; i < i1; i++)
      v = salsaa::add_mod(v, mul_mod(M, s_lo[(u64)j * Bw + i], wres(src, nar, (u64)i * d, M.q)), M.q);
    v = mul_mod(M, v, s_hi[(u64)j * nhi + hb]);
    atomic_add_mod(acc + ((u64)j * rows + k) * d + (u64)pb * SU_POS + pos, v, M.q, plain);
  }
}

int launch_sc_umma(const RowSet& wc, u32 rows, u64 width, u32 d, u32 Bw, u32 nhi, const ScRowList& tl,
                   const u64* s_lo, const u64* s_hi, const ModQ& M, u64* acc, bool plain, uint8_t* img, u32* flags,
                   u64 flag_cap, cudaStream_t st) {
  // short witnesses: split each element block over several CTAs (linear sums)
  // while the grid stays within one wave (one CTA per SM) and the flag scratch
  const u64 base = (u64)(d / SU_POS) * nhi * rows;
  u32 split = 1;
  while (split * 2 <= Bw / SU_KS && base * split * 2 <= 148 && base * split * 2 <= flag_cap) split *= 2;
  const u64 ctas = base * split;
  if (ctas > flag_cap) return salsaa_set_error(-2, "sc_umma: flag scratch too small");
  cudaError_t e = cudaMemsetAsync(flags, 0, ctas * sizeof(u32), st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "sc_umma flags");
  u64 g = ((u64)Bw * 128 + 255) / 256;
  sc_img_kernel<<<(unsigned)(g < 4096 ? g : 4096), 256, 0, st>>>(s_lo, Bw, tl, img);
  salsaa_count_launch();
  const size_t smem = 2 * (size_t)SU_STAGE;
  e = cudaFuncSetAttribute(sc_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "sc_umma smem attribute");
  dim3 grid(d / SU_POS, nhi * split, rows);
  sc_umma_kernel<<<grid, 512, smem, st>>>(wc, rows, d, Bw, nhi, split, tl, img, s_hi, M, acc, plain, flags);
  salsaa_count_launch();
  sc_exact_kernel<<<grid, SU_POS, 0, st>>>(wc, rows, d, Bw, nhi, split, tl, s_lo, s_hi, M, acc, plain, flags);
  salsaa_count_launch();
  e = cudaGetLastError();
  (void)width;
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "sc_umma launch");
}

// ---------------------------------------------------------------------------
// First streaming pass of the norm-check sumcheck on tcgen05
// (norm_check_1 + the first rounds of sum_check,
// src/subroutines/fast_norm_check.rs:135-320).  The pass reads groups
// v_g = (x[g + m ng])_{m < 16} of a witness row and needs, per repetition,
//   * the sums of rounds 0..3: every value of round t is a fixed linear
//     combination of v_g (the fold challenges are known up front), so each
//     sum is a quadratic form of v_g and all of them follow from the 16 x 16
//     Gram matrix C = sum_g v_g v_g^T (mod q);
//   * the folded vector v_4[g] = sum_m lambda[m] v_g[m] with
//     lambda[m] = prod_t (bit_{3-t}(m) ? c_t : 1 - c_t).
// The witness is small and centred (ternary, or decomposition digits), so
// each value splits exactly into four signed byte limbs, v = sum_x 2^(8x) l_x.
// A tile of 256 groups is stored once in shared memory as rows g of 64 bytes
// (m, x); with 8-group blocks of 8 x 16-byte slices that one image is
//   * the K-major A operand (M = g, K = (m, x)) of the fold product against
//     B = the bytes of mu[m, x] = 2^(8x) lambda[m] mod q (N = (rep, byte y)),
//   * the MN-major A and B operands (M, N = (m, x), K = g) of the Gram
//     product, accumulated in TMEM over all tiles of the CTA.
// The fold is sum_y 2^(8y) D[g][rep, y] mod q; C[m1][m2] is
// sum_{x1,x2} 2^(8(x1+x2)) D[(m1,x1)][(m2,x2)] mod q, added to a per-row
// accumulator; nc_gram_sums_kernel turns C into the round sums.  A value
// outside the limb range sets *flag; the CUDA-core pass then runs instead
// (sc_first_kernel gated on the flag) and the Gram sums are skipped.
// ---------------------------------------------------------------------------
constexpr u32 NG_T = 4;                          // rounds covered (groups of 16)
constexpr u32 NG_TILE = 256;                     // groups per tile (one per thread)
constexpr u32 NG_GBS = 1024;                     // one 8-group block: 8 slices x 128 B
constexpr u32 NG_STAGE = NG_TILE / 8 * NG_GBS;   // 32 KiB
constexpr u32 NG_MAX_TILES = 256;                // per CTA: Gram entries stay below 2^30
constexpr u32 NG_SMEM = 2 * NG_STAGE + 1024;     // two stages + the fold B table

__device__ __forceinline__ u64 ng_challenge(const DevState* ds, u32 round, u32 rep, u64 j, u64 q) {
  return uni_mod(prf_at(prf_key(ds->seed, domain_id(DOM_NC, round, rep)), j), q);
}

__global__ void __launch_bounds__(256, 2)
    nc_gram_kernel(RowSet w, u32 rows, u64 ng, u32 ntiles, ModQ M, const DevState* ds, u32 round, u64* out,
                   u64 sout, u64* gram, u32* flag, bool plain, u64 w32p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t done_bar[2];
  __shared__ uint32_t tslot;
  const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const u32 k = blockIdx.y;
  const u64 q = M.q, half_q = q >> 1;
  const u32 t0 = (u32)((u64)blockIdx.x * ntiles / gridDim.x), t1 = (u32)((u64)(blockIdx.x + 1) * ntiles / gridDim.x);
  const u64* x = w.p[k];
  const bool nar = (w.narrow >> k) & 1;
  u32* err = &g_tc_error;
  uint8_t* btab = smem + 2 * NG_STAGE;

  // slices 4..7 of every block stay zero: rows 64..127 of the Gram A operand
  for (u32 v = tid; v < 2 * (NG_TILE / 8) * 32; v += 256)
    *(uint4*)(smem + (v / 32) * NG_GBS + 512 + (v % 32) * 16) = make_uint4(0, 0, 0, 0);
  // fold B table (K-major, N = 16 rows (rep, y), K = 64 bytes (m, x)):
  // offset(n, kk) = (kk / 16) * 256 + (n / 8) * 128 + (n % 8) * 16 + kk % 16
  if (tid < 128) {
    const u32 rep = tid >> 6, m = (tid >> 2) & 15, xl = tid & 3;
    u64 lam = 1 % q;
#pragma unroll
    for (u32 t = 0; t < NG_T; t++) {
      const u64 c = ng_challenge(ds, round, rep, t, q);
      lam = mul_mod(M, lam, ((m >> (NG_T - 1 - t)) & 1) ? c : salsaa::sub_mod(1 % q, c, q));
    }
    const u64 mv = mul_mod(M, lam, ((u64)1 << (8 * xl)) % q);
    const u32 kk = m * 4 + xl;
#pragma unroll
    for (u32 y = 0; y < 8; y++) {
      const u32 n = rep * 8 + y;
      btab[(kk / 16) * 256 + (n / 8) * 128 + (n % 8) * 16 + kk % 16] = y < 7 ? (uint8_t)(mv >> (8 * y)) : 0;
    }
  }
  if (tid == 0) {
    umma::mbar_init(&done_bar[0], 1);
    umma::mbar_init(&done_bar[1], 1);
    umma::mbar_fence_init();
  }
  if (warp == 0) umma::tmem_alloc(&tslot, 128);
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const u32 tmem = tslot;  // columns 0..63 Gram, 64 + 32 s + 16 h fold of stage s, half h
  // s8 x s8, both MN-major, M = 128, N = 64
  const u32 id_gram = (2u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((64u >> 3) << 17) |
                      ((128u >> 4) << 24);
  // s8 (limbs) x u8 (mu bytes), both K-major, M = 128, N = 16
  const u32 id_fold = (2u << 4) | (1u << 7) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
  const u64 w32 = ((u64)1 << 32) % q;  // its Shoup companion w32p comes from the host (a 128-bit division)
  bool bad = false, ok = true;

  // loads of this thread: 4 consecutive groups g0 .. g0 + 3 (g0 = 4 (tid % 64))
  // x the 4 values m = 4 (tid / 64) .. + 3 of each, so one value index is
  // one 16-byte load for narrow rows (four int32 in wv[2 mm]) and two for
  // word rows (u64 pairs in wv[2 mm], wv[2 mm + 1]); the 16 limb bytes of
  // one group's four values are one 16-byte store to the tile
  ulonglong2 wv[8];
  const u32 g0 = 4 * (tid & 63), mq = tid >> 6;
  // stores of the four groups in the order rot, rot + 1, .. (mod 4): the 8
  // lanes of a store phase then hit 8 distinct 16-byte bank groups
  const u32 rot = (lane >> 1) & 3;
  auto load = [&](u32 tile) {
    const u64 o = (u64)tile * NG_TILE + g0;
    if (nar) {
      const int* xs = (const int*)x + o;
#pragma unroll
      for (u32 mm = 0; mm < 4; mm++) wv[2 * mm] = __ldg((const ulonglong2*)(xs + (u64)(4 * mq + mm) * ng));
    } else {
#pragma unroll
      for (u32 mm = 0; mm < 4; mm++)
#pragma unroll
        for (u32 h = 0; h < 2; h++)
          wv[2 * mm + h] = __ldg((const ulonglong2*)(x + o + (u64)(4 * mq + mm) * ng + 2 * h));
    }
  };
  auto epilogue = [&](u32 li, u32 tile) {
    const u32 se = li & 1;
    ok &= umma::mbar_wait(&done_bar[se], (li >> 1) & 1, err, 1);
    umma::fence_after_sync();
    uint32_t r[16];
    umma::tmem_ld16(tmem + (((warp & 3) * 32) << 16) + 64 + se * 32 + (warp >> 2) * 16, r);
    umma::tmem_wait_ld();
    const u64 g = (u64)tile * NG_TILE + tid;  // TMEM lane (warp & 3) * 32 + lane of half warp >> 2
#pragma unroll
    for (u32 rep = 0; rep < 2; rep++) {
      const int* D = (const int*)r + rep * 8;
      const long long lo = (long long)D[0] + ((long long)D[1] << 8) + ((long long)D[2] << 16) +
                           ((long long)D[3] << 24);
      const long long hi = (long long)D[4] + ((long long)D[5] << 8) + ((long long)D[6] << 16);
      const u64 loc = lo < 0 ? (u64)(lo + (long long)q) : (u64)lo;  // |lo| < 2^46 < q
      const u64 hic = hi < 0 ? (u64)(hi + (long long)q) : (u64)hi;  // |hi| < 2^38
      out[((u64)rep * rows + k) * sout + g] = salsaa::add_mod(mul_shoup(hic, w32, w32p, q), loc, q);
    }
  };

  if (t0 < t1) load(t0);
  for (u32 i = t0; i < t1; i++) {
    const u32 li = i - t0, s = li & 1;
    uint8_t* stage = smem + s * NG_STAGE;
    // stage s was last read by the MMAs of tile li - 2, whose completion the
    // epilogue of iteration li - 1 waited for
    uint32_t wd[4][4];  // [group][value]: the four signed limbs, byte x = limb x
#pragma unroll
    for (u32 gi = 0; gi < 4; gi++)
#pragma unroll
      for (u32 mm = 0; mm < 4; mm++) {
        if (nar) {
          const u64 pr = (gi & 2) ? wv[2 * mm].y : wv[2 * mm].x;
          const int cv = (int)(u32)((gi & 1) ? pr >> 32 : pr);  // centred value
          bad |= cv > 0x7f7f7f7f;  // below -0x80808080 is out of int32 range
          wd[gi][mm] = ((u32)cv + 0x80808080u) ^ 0x80808080u;
        } else {
          const ulonglong2 pr = wv[2 * mm + (gi >> 1)];
          const u64 v = (gi & 1) ? pr.y : pr.x;
          const u64 t = v + 0x80808080ULL - (v > half_q ? q : 0);  // centred value + limb bias
          bad |= (t >> 32) != 0;
          wd[gi][mm] = (uint32_t)t ^ 0x80808080u;
        }
      }
    // rotate the groups by rot (selects on a lane-uniform-per-pair value)
#pragma unroll
    for (u32 mm = 0; mm < 4; mm++) {
      if (rot & 1) {
        const u32 t0 = wd[0][mm];
        wd[0][mm] = wd[1][mm];
        wd[1][mm] = wd[2][mm];
        wd[2][mm] = wd[3][mm];
        wd[3][mm] = t0;
      }
      if (rot & 2) {
        u32 t0 = wd[0][mm];
        wd[0][mm] = wd[2][mm];
        wd[2][mm] = t0;
        t0 = wd[1][mm];
        wd[1][mm] = wd[3][mm];
        wd[3][mm] = t0;
      }
    }
#pragma unroll
    for (u32 sidx = 0; sidx < 4; sidx++) {
      const u32 g = g0 + ((sidx + rot) & 3);
      *(uint4*)(stage + (g >> 3) * NG_GBS + (g & 7) * 16 + mq * 128) =
          make_uint4(wd[sidx][0], wd[sidx][1], wd[sidx][2], wd[sidx][3]);
    }
    if (i + 1 < t1) load(i + 1);
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const u32 sa = umma::smem_u32(stage), sb = umma::smem_u32(btab);
#pragma unroll
      for (u32 kb = 0; kb < NG_TILE / 32; kb++) {
        // MN-major: LBO = stride of 8-group K blocks, SBO = stride of 16-byte MN slices
        const uint64_t dg = umma::desc_kmajor(sa + kb * 4 * NG_GBS, NG_GBS, 128);
        umma::mma_i8(tmem, dg, dg, id_gram, (li > 0 || kb > 0) ? 1u : 0u);
      }
#pragma unroll
      for (u32 h = 0; h < 2; h++)
#pragma unroll
        for (u32 j = 0; j < 2; j++) {
          const uint64_t ad = umma::desc_kmajor(sa + h * 16 * NG_GBS + j * 256, 128, NG_GBS);
          const uint64_t bd = umma::desc_kmajor(sb + j * 512, 256, 128);
          umma::mma_i8(tmem + 64 + s * 32 + h * 16, ad, bd, id_fold, j);
        }
      umma::commit(&done_bar[s]);
    }
    if (li > 0) epilogue(li - 1, i - 1);
  }
  if (t0 < t1) epilogue(t1 - 1 - t0, t1 - 1);

  // Gram epilogue: every MMA of this CTA has completed (the last wait covers them)
  ok = __syncthreads_and(ok);
  bad = __syncthreads_or(bad);
  if (bad && tid == 0) atomicOr(flag, 1u);
  umma::fence_after_sync();
  int* Dg = (int*)smem;  // 64 x 64 s32, over stage 0
  if (warp < 2 && t0 < t1) {
#pragma unroll
    for (u32 cb = 0; cb < 4; cb++) {
      uint32_t r[16];
      umma::tmem_ld16(tmem + ((warp * 32) << 16) + cb * 16, r);
      umma::tmem_wait_ld();
#pragma unroll
      for (u32 e = 0; e < 16; e++) Dg[(warp * 32 + lane) * 64 + cb * 16 + e] = (int)r[e];
    }
  }
  __syncthreads();
  if (ok && !bad && t0 < t1) {
    const u32 m1 = tid >> 4, m2 = tid & 15;
    u64 acc = 0;
#pragma unroll
    for (u32 x1 = 0; x1 < 4; x1++)
#pragma unroll
      for (u32 x2 = 0; x2 < 4; x2++) {
        const long long dv = Dg[(m1 * 4 + x1) * 64 + m2 * 4 + x2];
        long long rm = dv % (long long)q;
        if (rm < 0) rm += (long long)q;
        acc = salsaa::add_mod(acc, mul_mod(M, (u64)rm, ((u64)1 << (8 * (x1 + x2))) % q), q);
      }
    atomic_add_mod(gram + (u64)k * 256 + tid, acc, q, plain);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

// Round sums 0..3 of both repetitions from the Gram matrix of each row: with
// L_t the 2^(4-t) x 16 matrix giving the values of round t from v_g,
// (sum_g x_t[j] x_t[j']) = L_t[j]^T C L_t[j'].  One CTA per witness row.
__global__ void __launch_bounds__(256) nc_gram_sums_kernel(const u64* gram, const u32* flag, u32 rows, ModQ M,
                                                           const DevState* ds, u32 round, u64* sums, u32 nr,
                                                           bool plain) {
  if (*flag) return;
  __shared__ u64 C[256];
  __shared__ u64 L[2][30][16];  // rows 0..15 round 0, 16..23 round 1, 24..27 round 2, 28..29 round 3
  __shared__ u64 Y[2][30][16];  // C L
  __shared__ u64 ch[2][NG_T];
  const u32 k = blockIdx.x, tid = threadIdx.x;
  const u64 q = M.q;
  C[tid] = gram[(u64)k * 256 + tid] % q;
  if (tid < 2 * NG_T) ch[tid / NG_T][tid % NG_T] = ng_challenge(ds, round, tid / NG_T, tid % NG_T, q);
  for (u32 e = tid; e < 2 * 256; e += 256) {
    const u32 rep = e >> 8, j = (e >> 4) & 15, i = e & 15;
    L[rep][j][i] = (i == j) ? 1 % q : 0;
  }
  __syncthreads();
  u32 off = 0, len = 16;
  for (u32 t = 0; t + 1 < NG_T; t++) {
    const u32 h = len / 2;
    for (u32 e = tid; e < 2 * h * 16; e += 256) {
      const u32 rep = e / (h * 16), j = (e / 16) % h, i = e % 16;
      const u64 a = L[rep][off + j][i], b = L[rep][off + j + h][i];
      L[rep][off + len + j][i] = salsaa::add_mod(a, mul_mod(M, ch[rep][t], salsaa::sub_mod(b, a, q)), q);
    }
    __syncthreads();
    off += len;
    len = h;
  }
  // dot products as exact 128-bit sums (at most 128 products below 2^112),
  // one reduction each
  for (u32 e = tid; e < 2 * 30 * 16; e += 256) {
    const u32 rep = e / 480, r = (e / 16) % 30, i = e % 16;
    unsigned __int128 s = 0;
#pragma unroll
    for (u32 j = 0; j < 16; j++) s += (unsigned __int128)C[i * 16 + j] * L[rep][r][j];
    Y[rep][r][i] = reduce128_any(M, (u64)(s >> 64), (u64)s);
  }
  __syncthreads();
  if (tid < 2 * NG_T * 3) {
    const u32 rep = tid / (NG_T * 3), t = (tid / 3) % NG_T, a = tid % 3;
    const u32 o = 32 - (32 >> t), h = 8 >> t;  // first row and half length of round t
    unsigned __int128 s = 0;
    for (u32 j = 0; j < h; j++) {
      const u32 lrow = o + j + (a == 2 ? h : 0), rrow = o + j + (a == 0 ? 0 : h);
#pragma unroll
      for (u32 i = 0; i < 16; i++) s += (unsigned __int128)L[rep][lrow][i] * Y[rep][rrow][i];
    }
    atomic_add_mod(&sums[((rep * (u64)nr + t) * rows + k) * 3 + a], reduce128_any(M, (u64)(s >> 64), (u64)s), q,
                   plain);
  }
}

bool nc_gram_ok(const RowSet& w, u32 rows, u64 nlen, u64 q) {
  return q > (1ULL << 47) && q < (1ULL << 56) && nlen % (16ULL * NG_TILE) == 0 && nlen / 16 / NG_TILE >= 1 &&
         rowset_aligned(w, rows, 16, 16);
}

int launch_nc_gram(const RowSet& w, u32 rows, u64 nlen, const ModQ& M, const DevState* ds, u32 round, u64* out,
                   u64 sout, u64* gram, bool plain, cudaStream_t st) {
  const u64 ng = nlen / 16;
  const u32 ntiles = (u32)(ng / NG_TILE);
  cudaError_t e = cudaMemsetAsync(gram, 0, ((u64)rows * 256 + 1) * sizeof(u64), st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "nc_gram memset");
  e = cudaFuncSetAttribute(nc_gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)NG_SMEM);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "nc_gram smem attribute");
  u64 nb = (296 + rows - 1) / rows;
  const u64 need = (ntiles + NG_MAX_TILES - 1) / NG_MAX_TILES;
  if (nb < need) nb = need;
  if (nb > ntiles) nb = ntiles;
  u32* flag = (u32*)(gram + (u64)rows * 256);
  const bool gplain = plain && nb < (1u << 13);
  const int tr = salsaa_trace_begin("nc_gram_kernel", st, (double)rows * nlen * 8.0 * (1.0 + 2.0 / 16.0));
  const u64 w32p = (u64)(((unsigned __int128)(((u64)1 << 32) % M.q) << 64) / M.q);
  nc_gram_kernel<<<dim3((unsigned)nb, rows), 256, NG_SMEM, st>>>(w, rows, ng, ntiles, M, ds, round, out, sout, gram,
                                                                 flag, gplain, w32p);
  salsaa_trace_end(tr, st);
  salsaa_count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "nc_gram launch");
}

int launch_nc_gram_sums(const u64* gram, u32 rows, const ModQ& M, const DevState* ds, u32 round, u64* sums, u32 nr,
                        bool plain, cudaStream_t st) {
  const u32* flag = (const u32*)(gram + (u64)rows * 256);
  nc_gram_sums_kernel<<<rows, 256, 0, st>>>(gram, flag, rows, M, ds, round, sums, nr, plain);
  salsaa_count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : salsaa_set_cuda_error(e, "nc_gram_sums launch");
}

int tc_error_check() {
  u32 h = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&h, g_tc_error, sizeof(u32));
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "tensor-core status");
  if (h) return salsaa_set_error(-4, "a tensor-core wait timed out; results of that launch are invalid");
  return ntt_error_check();
}

}  // namespace salsaa

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
