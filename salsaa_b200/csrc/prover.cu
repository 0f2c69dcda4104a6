// prover.cu — device-resident SALSAA prover (src/protocol.rs:125-483) and the
// device tier of the C ABI (include/salsaa_gpu.h).
//
// A proof is enqueued on one CUDA stream with no host synchronisation: every
// challenge comes from the PRF on the device and data-dependent values (the
// decomposition radix) stay in device memory.  The host only walks the
// (data-independent) shapes of the protocol to place each prover message at
// its fixed offset of the proof buffer.
#include <atomic>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/salsaa_gpu.h"
#include "host_math.h"
#include "kernels.cuh"

using namespace salsaa;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
int salsaa_set_error(int code, const char* msg) {
  g_err = msg;
  return code;
}
int salsaa_set_cuda_error(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return -1000 - (int)e;
}
extern "C" const char* salsaa_last_error(void) { return g_err.c_str(); }

// ---- device-time trace ------------------------------------------------------
namespace {
constexpr int TRACE_MAX = 8192;
struct TraceRec {
  const char* name;
  cudaEvent_t a, b;
  double work;
  int done;
  int alias;  // shares the events of record `alias - 1` (another measure of the same launch)
};
std::mutex g_trace_mu;
std::atomic<int> g_trace_on{0};
std::vector<TraceRec> g_trace;
}  // namespace

int salsaa_trace_begin(const char* name, cudaStream_t st, double work) {
  if (!g_trace_on.load(std::memory_order_relaxed)) return -1;
  std::lock_guard<std::mutex> lk(g_trace_mu);
  if ((int)g_trace.size() >= TRACE_MAX) return -1;
  TraceRec r{name, nullptr, nullptr, work, 0, 0};
  if (cudaEventCreate(&r.a) != cudaSuccess || cudaEventCreate(&r.b) != cudaSuccess) return -1;
  cudaEventRecord(r.a, st);
  g_trace.push_back(r);
  return (int)g_trace.size() - 1;
}
void salsaa_trace_end(int token, cudaStream_t st) {
  if (token < 0) return;
  std::lock_guard<std::mutex> lk(g_trace_mu);
  if (token < (int)g_trace.size()) {
    cudaEventRecord(g_trace[token].b, st);
    g_trace[token].done = 1;
  }
}
void salsaa_trace_alias(int token, const char* name, double work) {
  if (token < 0) return;
  std::lock_guard<std::mutex> lk(g_trace_mu);
  if (token >= (int)g_trace.size() || (int)g_trace.size() >= TRACE_MAX) return;
  TraceRec r = g_trace[token];
  r.name = name;
  r.work = work;
  r.alias = token + 1;
  g_trace.push_back(r);
}
extern "C" void salsaa_trace_enable(int on) {
  std::lock_guard<std::mutex> lk(g_trace_mu);
  for (TraceRec& r : g_trace) {
    if (r.alias) continue;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  g_trace.clear();
  g_trace_on.store(on ? 1 : 0);
}
extern "C" int salsaa_trace_read(const char* name, double* total_ms, double* total_work, uint64_t* launches) {
  if (!name || !total_ms || !total_work || !launches) return salsaa_set_error(-1, "trace_read: null argument");
  std::lock_guard<std::mutex> lk(g_trace_mu);
  double t = 0, wk = 0;
  uint64_t n = 0;
  for (TraceRec& r : g_trace) {
    const int done = r.alias ? g_trace[r.alias - 1].done : r.done;
    if (!done || strcmp(r.name, name)) continue;
    cudaError_t e = cudaEventSynchronize(r.b);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "trace_read");
    float ms = 0;
    e = cudaEventElapsedTime(&ms, r.a, r.b);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "trace_read");
    t += ms;
    wk += r.work;
    n++;
  }
  *total_ms = t;
  *total_work = wk;
  *launches = n;
  return 0;
}

static bool salsaa_trace_active() { return g_trace_on.load(std::memory_order_relaxed) != 0; }

static std::atomic<uint64_t> g_launches{0};
void salsaa_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
extern "C" uint64_t salsaa_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }
extern "C" int salsaa_device_status(void) { return salsaa::tc_error_check(); }

#define TRY(x)            \
  do {                    \
    int _rc = (x);        \
    if (_rc) return _rc;  \
  } while (0)

// ---------------------------------------------------------------------------
// parameters and shapes
// ---------------------------------------------------------------------------
static const uint64_t Q0 = 1125899904679937ULL, Q1 = 1125899906840833ULL, Q2 = 1125899906822657ULL;

extern "C" int salsaa_params_preset(const char* name, salsaa_params* out) {
  struct Pre {
    const char* name;
    uint64_t d, q, ms, wl, nr, fold;
  } pre[] = {
      {"A0", 128, Q0, 12, 1u << 19, 8, 0},  {"A1", 256, Q1, 7, 1u << 18, 7, 0},  {"A2", 512, Q2, 4, 1u << 17, 6, 0},
      {"B0", 128, Q0, 12, 1u << 21, 10, 0}, {"B1", 256, Q1, 7, 1u << 20, 9, 0},  {"B2", 512, Q2, 4, 1u << 19, 8, 0},
      {"C0", 128, Q0, 12, 1u << 23, 12, 0}, {"C1", 256, Q1, 7, 1u << 22, 11, 0}, {"C2", 512, Q2, 4, 1u << 21, 10, 0},
      {"F0", 128, Q0, 12, 1u << 17, 1, 1},  {"F1", 128, Q0, 13, 1u << 19, 1, 1}, {"F2", 128, Q0, 13, 1u << 21, 1, 1},
  };
  if (!name || !out) return salsaa_set_error(-1, "params_preset: null argument");
  for (const Pre& p : pre)
    if (!strcmp(p.name, name)) {
      memset(out, 0, sizeof(*out));
      out->d = p.d;
      out->q = p.q;
      out->module_size = p.ms;
      out->wit_len = p.wl;
      out->nof_rounds = p.nr;
      out->folding = p.fold;
      out->init_wit_rep = p.fold ? 4 : 1;
      out->decomp_parts[0] = 1;
      for (int i = 1; i < 12; i++) out->decomp_parts[i] = 2;
      return 0;
    }
  return salsaa_set_error(-1, "params_preset: unknown name");
}

static u64 ilog2u(u64 x) { return x ? 63 - (u64)__builtin_clzll(x) : 0; }

// Walk of the protocol's shapes (identical in every proof of a parameter set).
struct Shapes {
  bool basic_ok = false;  // d, q, wit_len, module_size usable (enough for a context)
  bool ok = false;        // the whole protocol's shapes are valid (needed to prove)
  std::string why;
  u64 proof_words = 0;
  u64 max_d_rows_width = 0;  // decomposition output / initial witness, rows * width
  u64 max_nc_rows_width = 0; // norm check rows * width
  u64 max_fp_width = 0;      // width of projected / folded rows
  u32 max_rows = 0;          // witness rows in any call
  u32 max_stmt = 0;          // statement rows
  u32 nsc_total = 0;         // scalar rows pushed by the whole proof
};

static Shapes walk(const salsaa_params* p) {
  Shapes S;
  if (!p) {
    S.why = "null params";
    return S;
  }
  const u64 d = p->d, q = p->q;
  if (d < 4 || d > 512 || (d & (d - 1))) {
    S.why = "d must be a power of two in [4, 512]";
    return S;
  }
  if (q < 3 || q >= (1ULL << 62) || (q - 1) % d) {
    S.why = "q must satisfy q < 2^62 and q = 1 mod d";
    return S;
  }
  if (!host::minimal_root(d, q)) {
    S.why = "q has no primitive d-th root of unity";
    return S;
  }
  const u64 L = p->wit_len;
  if (L < 2 || (L & (L - 1))) {
    S.why = "wit_len must be a power of two >= 2";
    return S;
  }
  if (!p->module_size || p->module_size > 64 || !p->init_wit_rep || p->init_wit_rep > MAX_WROWS ||
      p->nof_rounds > 12) {
    S.why = "module_size, init_wit_rep or nof_rounds out of range";
    return S;
  }
  S.basic_ok = true;
  u64 w = 8, Sn = p->module_size, K = p->init_wit_rep, width = L;
  S.max_d_rows_width = K * width;
  S.max_rows = (u32)K;
  w += Sn * K * d;
  for (u64 i = 0; i < p->nof_rounds; i++) {
    const u64 parts = p->decomp_parts[i < 12 ? i : 11];
    if (!p->folding && parts > 1) {
      if (i == 0) {
        S.why = "decomposition in round 0 is not supported";
        return S;
      }
      w += 1 + Sn * K * parts * d;
      K *= parts;
      if (K * width > S.max_d_rows_width) S.max_d_rows_width = K * width;
    } else if (!p->folding && i > 0 && K * width > S.max_d_rows_width) {
      S.max_d_rows_width = K * width;  // the joined witness moves to the decomposition buffers
    }
    if (K > MAX_WROWS) {
      S.why = "too many witness rows";
      return S;
    }
    if (K * width > S.max_nc_rows_width) S.max_nc_rows_width = K * width;
    if (width * d < 4) {
      S.why = "witness too short for the sumcheck";
      return S;
    }
    w += K;
    const u64 nr = ilog2u(width * d);
    for (int rep = 0; rep < 2; rep++) {
      w += nr * K * 3 + K * d;
      Sn += 1;
      S.nsc_total++;
    }
    if (!p->folding) {
      w += Sn * 2 * K * d;
      K *= 2;
      width /= 2;
    }
    if (K > MAX_WROWS) {
      S.why = "too many witness rows";
      return S;
    }
    if (K > S.max_rows) S.max_rows = (u32)K;
    const u64 cw = K * 256;
    if (cw > width || width % cw) {
      S.why = "projection chunk width (rows*256) exceeds the witness width";
      return S;
    }
    if (cw > CK_BLOCK) {
      S.why = "projection chunk width (rows*256) above 2048: more than 8 witness rows after a split "
              "(decomposition into more than 2 parts) is not supported";
      return S;
    }
    if (width > S.max_fp_width) S.max_fp_width = width;
    w += Sn * d;
    w += (K + 1) * d;
    Sn += 1;
    w += 2 * d;
    Sn += 1;
    S.nsc_total += 2;
    K = 2;
    if (p->folding) {
      w += 1 + Sn * K * 2 * d;
      K *= 2;
      if (K * width > S.max_d_rows_width) S.max_d_rows_width = K * width;
      break;
    }
    if (Sn > S.max_stmt) S.max_stmt = (u32)Sn;
  }
  if (Sn > S.max_stmt) S.max_stmt = (u32)Sn;
  if (K > S.max_rows) S.max_rows = (u32)K;
  if (!p->folding) w += K * width * d;
  S.proof_words = w;
  S.ok = true;
  return S;
}

extern "C" uint64_t salsaa_proof_size(const salsaa_params* p) {
  Shapes S = walk(p);
  return S.ok ? S.proof_words * 8 : 0;
}

// ---------------------------------------------------------------------------
// context: parameters + commitment-key tables
// ---------------------------------------------------------------------------
struct salsaa_ctx {
  salsaa_params P;
  u64 crs_seed;
  int device;
  Shapes S;
  ModQ M;
  const NttDev* T;
  u32 d, n;
  u64 L;
  u32 ck_bt, ck_nhi;
  u64* m_slot = nullptr;
  u64* tlo = nullptr;
  u64* thi = nullptr;
  uint8_t* tl8 = nullptr;  // tensor-core key table (q < 2^56), else null
  uint8_t* tk8 = nullptr;  // tcgen05 key table (q < 2^56, <= 18 key rows, blocks of >= 128), else null
  std::mutex mu;
  salsaa_prover* blocking = nullptr;  // slot used by salsaa_prove()
};

struct DevBuf {
  std::vector<void*> ptrs;
  template <class T>
  int alloc(T** p, u64 count, const char* what) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, (count ? count : 1) * sizeof(T));
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, what);
    ptrs.push_back(v);
    *p = (T*)v;
    return 0;
  }
  void release() {
    for (void* v : ptrs) cudaFree(v);
    ptrs.clear();
  }
};

static int ctx_build(salsaa_ctx* c, DevBuf& mem) {
  const u32 d = c->d, n = c->n;
  const u32 ms = (u32)c->P.module_size;
  u64* m_coef = nullptr;
  TRY(mem.alloc(&m_coef, (u64)ms * d, "ctx: module"));
  TRY(mem.alloc(&c->m_slot, (u64)ms * d, "ctx: module slots"));
  TRY(mem.alloc(&c->tlo, (u64)ms * c->ck_bt * 3 * n, "ctx: key table lo"));
  TRY(mem.alloc(&c->thi, (u64)ms * c->ck_nhi * d, "ctx: key table hi"));
  TRY(launch_gen_crs(m_coef, ms, d, c->P.q, c->crs_seed, 0));
  TRY(ntt_launch(m_coef, c->m_slot, ms, *c->T, true, false, 0));
  TRY(launch_ck_tables(c->m_slot, ms, *c->T, c->M, c->L, c->tlo, c->thi, 0));
  if (c->P.q < (1ULL << 56)) {
    TRY(mem.alloc(&c->tl8, ck_tl8_bytes(ms, n, c->ck_bt), "ctx: key byte planes"));
    TRY(launch_ck_tl8(c->tlo, ms, n, c->ck_bt, c->P.q < (1ULL << 50), c->tl8, 0));
    if (ms <= CKU_MAX_KEYS && c->ck_bt >= 128 && n % 2 == 0) {
      TRY(mem.alloc(&c->tk8, ck_tk8_bytes(ms, n, c->ck_bt), "ctx: tcgen05 key tiles"));
      TRY(launch_ck_tk8(c->tlo, ms, n, c->ck_bt, c->P.q < (1ULL << 50), c->tk8, 0));
    }
  }
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "ctx: build");
  return 0;
}

static std::mutex g_ctx_bufs_mu;
static std::vector<std::pair<salsaa_ctx*, DevBuf>> g_ctx_bufs;

extern "C" int salsaa_ctx_create(const salsaa_params* p, uint64_t crs_seed, int device, salsaa_ctx** out) {
  if (!out) return salsaa_set_error(-1, "ctx_create: null output");
  *out = nullptr;
  Shapes S = walk(p);
  if (!S.basic_ok) return salsaa_set_error(-1, ("ctx_create: " + S.why).c_str());
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "ctx_create: cudaSetDevice");
  salsaa_ctx* c = new (std::nothrow) salsaa_ctx;
  if (!c) return salsaa_set_error(-1, "ctx_create: out of host memory");
  c->P = *p;
  c->crs_seed = crs_seed;
  c->device = device;
  c->S = S;
  c->M = make_modq(p->q);
  c->d = (u32)p->d;
  c->n = c->d / 2;
  c->L = p->wit_len;
  c->ck_bt = (u32)(c->L < CK_KEY_BLOCK ? c->L : CK_KEY_BLOCK);
  c->ck_nhi = (u32)(c->L / c->ck_bt);
  c->T = ntt_tables(c->n, p->q);
  if (!c->T) {
    delete c;
    return salsaa_set_error(-1, "ctx_create: NTT tables unavailable");
  }
  DevBuf mem;
  int rc = ctx_build(c, mem);
  if (rc) {
    mem.release();
    delete c;
    return rc;
  }
  {
    std::lock_guard<std::mutex> lk(g_ctx_bufs_mu);
    g_ctx_bufs.push_back({c, mem});
  }
  *out = c;
  return 0;
}

// ---------------------------------------------------------------------------
// one proof in flight
// ---------------------------------------------------------------------------
enum Phase { PH_COMMIT = 0, PH_NORM1, PH_NORM2, PH_NORM3, PH_SPLIT, PH_PROJ, PH_FOLD, PH_DECOMP, PH_N };
constexpr int MAX_EVENTS = 128;

struct salsaa_prover {
  salsaa_ctx* ctx;
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;  // side stream: the projection runs beside the sumcheck
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool overlap = false;        // use the side stream (salsaa_prover_set_overlap)
  DevBuf mem;
  DevState* ds = nullptr;
  u64 *Dc = nullptr, *Ds = nullptr, *Fc = nullptr, *Fs = nullptr, *Pc = nullptr, *Ps = nullptr;
  SumcheckBufs sc{};
  u64* row_base = nullptr;  // TENSOR row bases, nsc_total x d
  u64* row_cj = nullptr;    // PERIODIC row scalars, rounds x CK_BLOCK
  u32 *pmask = nullptr, *nmask = nullptr;
  int8_t* Jm = nullptr;  // projection challenge as int8, 256 x chunk width
  int8_t* Jc = nullptr;  // the same in the tcgen05 operand layout
  uint8_t* sc_img = nullptr;  // tcgen05 TENSOR-row pass: scalar byte image
  u32* sc_flags = nullptr;    // and its per-CTA fallback flags
  u64 sc_flag_words = 0;
  u64 *c_coef = nullptr, *c_slot = nullptr, *fold_pre = nullptr;
  ScalarRowDesc* sc_desc = nullptr;
  std::vector<int> sc_types;  // host copy of the scalar rows' types (launch tiling)
  const u64** sc_base = nullptr;
  u64 *sc_lo = nullptr, *sc_hi = nullptr, *acc = nullptr, *cout = nullptr, *colsum = nullptr;
  u64* cout2 = nullptr;  // coefficient-form staging of a merged commitment
  u64* header_pinned = nullptr;
  uint8_t* own_proof = nullptr;  // for the blocking API
  cudaEvent_t ev[MAX_EVENTS];
  int ev_phase[MAX_EVENTS];
  int nev = 0;
  int last_rc = 0;
  // CUDA-graph replay (salsaa_prover_set_graph): the proof's launch sequence
  // captured once for one (witness, proof) buffer pair; later proofs update
  // the seed kernel's argument and relaunch the executable graph.
  bool use_graph = false, capturing = false, graph_failed = false;
  cudaGraph_t graph = nullptr;  // kept with its executable: the seed node belongs to it
  cudaGraphExec_t gexec = nullptr;
  cudaGraphNode_t gseed = nullptr;
  cudaKernelNodeParams gseed_p{};
  const u64* g_witness = nullptr;
  u64* g_proof = nullptr;
  u64 g_kernels = 0;
  unsigned long long g_sched = 0;  // schedule table generation at capture
  bool g_overlap = false;          // overlap setting at capture
  // int8 witness uploads, double-buffered: the next proof's witness crosses
  // PCIe on cp_st into stage8[k % 2] while the current proof computes
  cudaStream_t cp_st = nullptr;
  int8_t* stage8[2] = {nullptr, nullptr};
  cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
  u64 n_i8 = 0;  // int8 uploads so far
};

static int mark(salsaa_prover* pr, int phase) {
  if (pr->capturing || pr->nev >= MAX_EVENTS) return 0;  // phase times are not kept for graph replays
  cudaError_t e = cudaEventRecord(pr->ev[pr->nev], pr->st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "event record");
  pr->ev_phase[pr->nev++] = phase;
  return 0;
}

extern "C" uint64_t salsaa_workspace_bytes(const salsaa_params* p) {
  Shapes S = walk(p);
  if (!S.ok) return 0;
  const u64 d = p->d, L = p->wit_len;
  u64 words = 0;
  words += 2 * S.max_d_rows_width * d;        // Dc, Ds
  words += 4 * S.max_fp_width * d;            // Fc, Fs, Pc, Ps
  words += S.max_nc_rows_width * d;           // sumcheck a
  words += S.max_nc_rows_width * d / 2;       // sumcheck b
  words += (u64)MAX_WROWS * 256 + 1;          // sumcheck Gram matrices
  words += (u64)S.nsc_total * d + p->nof_rounds * CK_BLOCK;
  const u64 stmt = S.max_stmt + 2;
  words += stmt * CK_BLOCK + stmt * (L / CK_BLOCK + 1);
  words += 3 * stmt * (MAX_WROWS + 1) * d;      // commitment accumulators and outputs
  words += (u64)(S.max_rows + 1) * (L < CK_BLOCK ? L : CK_BLOCK) * d;
  words += 2 * 256ULL * CK_BLOCK / 8;          // projection J and its tensor-core image (bytes)
  words += (u64)MAX_WROWS * (d / 2) * 6;       // fold constants
  words += SC_IMG_BYTES / 8 + (d / 128 + 1) * (L / CK_BLOCK + 1) * (S.max_rows + 2) / 2;  // scalar-row pass
  return words * 8 + (S.proof_words * 8);
}

extern "C" int salsaa_prover_create(salsaa_ctx* c, salsaa_prover** out) {
  if (!c || !out) return salsaa_set_error(-1, "prover_create: null argument");
  *out = nullptr;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_create: cudaSetDevice");
  if (!c->S.ok) return salsaa_set_error(-1, ("prover_create: " + c->S.why).c_str());
  salsaa_prover* pr = new (std::nothrow) salsaa_prover;
  if (!pr) return salsaa_set_error(-1, "prover_create: out of host memory");
  pr->ctx = c;
  const Shapes& S = c->S;
  const u64 d = c->d, L = c->L;
  auto fail = [&](int rc) {
    pr->mem.release();
    if (pr->ev_fork) cudaEventDestroy(pr->ev_fork);
    if (pr->ev_join) cudaEventDestroy(pr->ev_join);
    if (pr->st2) cudaStreamDestroy(pr->st2);
    if (pr->st) cudaStreamDestroy(pr->st);
    delete pr;
    return rc;
  };
  e = cudaStreamCreateWithFlags(&pr->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&pr->st2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pr->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pr->ev_join, cudaEventDisableTiming);
  if (e != cudaSuccess) return fail(salsaa_set_cuda_error(e, "prover_create: stream"));
  for (int i = 0; i < MAX_EVENTS; i++) {
    e = cudaEventCreate(&pr->ev[i]);
    if (e != cudaSuccess) return fail(salsaa_set_cuda_error(e, "prover_create: event"));
  }
  int rc = 0;
  DevBuf& m = pr->mem;
  const u64 stmt = S.max_stmt + 2;
  if ((rc = m.alloc(&pr->ds, 1, "ds")) || (rc = m.alloc(&pr->Dc, S.max_d_rows_width * d, "Dc")) ||
      (rc = m.alloc(&pr->Ds, S.max_d_rows_width * d, "Ds")) || (rc = m.alloc(&pr->Fc, S.max_fp_width * d, "Fc")) ||
      (rc = m.alloc(&pr->Fs, S.max_fp_width * d, "Fs")) || (rc = m.alloc(&pr->Pc, S.max_fp_width * d, "Pc")) ||
      (rc = m.alloc(&pr->Ps, S.max_fp_width * d, "Ps")) ||
      (rc = m.alloc(&pr->sc.a, S.max_nc_rows_width * d, "sumcheck a")) ||
      (rc = m.alloc(&pr->sc.b, S.max_nc_rows_width * d / 2 + 1, "sumcheck b")) ||
      (rc = m.alloc(&pr->sc.sums, 2ULL * 64 * MAX_WROWS * 3, "sumcheck sums")) ||
      (rc = m.alloc(&pr->sc.cap, 2ULL * MAX_WROWS * d, "sumcheck cap")) ||
      (rc = m.alloc(&pr->sc.gram, (u64)MAX_WROWS * 256 + 1, "sumcheck gram")) ||
      (rc = m.alloc(&pr->row_base, (u64)S.nsc_total * d + 1, "row bases")) ||
      (rc = m.alloc(&pr->row_cj, (c->P.nof_rounds + 1) * (u64)CK_BLOCK, "row cj")) ||
      (rc = m.alloc(&pr->pmask, 256ULL * CK_BLOCK / 32, "pos mask")) ||
      (rc = m.alloc(&pr->nmask, 256ULL * CK_BLOCK / 32, "neg mask")) ||
      (rc = m.alloc(&pr->Jm, 256ULL * CK_BLOCK, "projection J")) ||
      (rc = m.alloc(&pr->Jc, 256ULL * CK_BLOCK, "projection J (tensor-core layout)")) ||
      (rc = m.alloc(&pr->sc_img, SC_IMG_BYTES, "scalar-row byte image")) ||
      (rc = m.alloc(&pr->sc_flags, pr->sc_flag_words = (u64)(d / 128 + 1) * (L / CK_BLOCK + 1) * (S.max_rows + 2),
                    "scalar-row flags")) ||
      (rc = m.alloc(&pr->c_coef, (u64)MAX_WROWS * d, "fold c")) ||
      (rc = m.alloc(&pr->c_slot, (u64)MAX_WROWS * d, "fold c slot")) ||
      (rc = m.alloc(&pr->fold_pre, (u64)MAX_WROWS * (d / 2) * 6, "fold constants")) ||
      (rc = m.alloc(&pr->sc_desc, (u64)S.nsc_total + 1, "row descriptors")) ||
      (rc = m.alloc(&pr->sc_base, (u64)S.nsc_total + 1, "row base pointers")) ||
      (rc = m.alloc(&pr->sc_lo, stmt * CK_BLOCK, "commit s_lo")) ||
      (rc = m.alloc(&pr->sc_hi, stmt * (L / CK_BLOCK + 1), "commit s_hi")) ||
      (rc = m.alloc(&pr->acc, stmt * (MAX_WROWS + 1) * d, "commit acc")) ||
      (rc = m.alloc(&pr->colsum, (u64)(S.max_rows + 1) * (L < CK_BLOCK ? L : CK_BLOCK) * d, "commit column sums")) ||
      (rc = m.alloc(&pr->cout, stmt * (MAX_WROWS + 1) * d, "commit out")) ||
      (rc = m.alloc(&pr->cout2, stmt * (MAX_WROWS + 1) * d, "commit out (coefficients)")))
    return fail(rc);
  // Scalar statement rows of the whole proof, in push order: per round
  // TENSOR(rep 0), TENSOR(rep 1), PERIODIC (witness_lhs), ONES (projected_lhs).
  std::vector<ScalarRowDesc> desc;
  std::vector<const u64*> bases;
  {
    u64 K = c->P.init_wit_rep, width = L;
    for (u64 rd = 0; rd < c->P.nof_rounds; rd++) {
      const u64 parts = c->P.decomp_parts[rd < 12 ? rd : 11];
      if (!c->P.folding && parts > 1) K *= parts;
      for (u32 rep = 0; rep < 2; rep++) {
        ScalarRowDesc t{};
        t.type = ROW_TENSOR;
        t.round = (u32)rd;
        t.rep = rep;
        t.K = (u32)ilog2u(width);
        desc.push_back(t);
        bases.push_back(pr->row_base + (desc.size() - 1) * d);
      }
      if (!c->P.folding) {
        K *= 2;
        width /= 2;
      }
      ScalarRowDesc per{};
      per.type = ROW_PERIODIC;
      per.round = (u32)rd;
      per.cw = (u32)(K * 256);
      per.cj = pr->row_cj + rd * CK_BLOCK;
      desc.push_back(per);
      bases.push_back(nullptr);
      ScalarRowDesc ones{};
      ones.type = ROW_ONES;
      ones.round = (u32)rd;
      desc.push_back(ones);
      bases.push_back(nullptr);
      K = 2;
      if (c->P.folding) break;
    }
  }
  for (const ScalarRowDesc& sd : desc) pr->sc_types.push_back(sd.type);
  if (!desc.empty()) {
    e = cudaMemcpy(pr->sc_desc, desc.data(), desc.size() * sizeof(ScalarRowDesc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(pr->sc_base, bases.data(), bases.size() * sizeof(u64*), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(salsaa_set_cuda_error(e, "prover_create: descriptors"));
  }
  e = cudaMallocHost(&pr->header_pinned, 8 * sizeof(u64));
  if (e != cudaSuccess) return fail(salsaa_set_cuda_error(e, "prover_create: pinned header"));
  const salsaa_params& P = c->P;
  const u64 hdr[8] = {0x31504141534C4153ULL, P.d, P.q, P.module_size, P.wit_len, P.init_wit_rep, P.nof_rounds,
                      P.folding};
  memcpy(pr->header_pinned, hdr, sizeof(hdr));
  *out = pr;
  return 0;
}

static void drop_graph(salsaa_prover* pr);

extern "C" void salsaa_prover_destroy(salsaa_prover* pr) {
  if (!pr) return;
  cudaSetDevice(pr->ctx->device);
  if (pr->st) cudaStreamSynchronize(pr->st);
  if (pr->cp_st) cudaStreamSynchronize(pr->cp_st);
  drop_graph(pr);
  for (int i = 0; i < 2; i++) {
    if (pr->stage8[i]) cudaFree(pr->stage8[i]);
    if (pr->ev_copied[i]) cudaEventDestroy(pr->ev_copied[i]);
    if (pr->ev_free[i]) cudaEventDestroy(pr->ev_free[i]);
  }
  if (pr->cp_st) cudaStreamDestroy(pr->cp_st);
  pr->mem.release();
  if (pr->own_proof) cudaFree(pr->own_proof);
  if (pr->header_pinned) cudaFreeHost(pr->header_pinned);
  for (int i = 0; i < MAX_EVENTS; i++) cudaEventDestroy(pr->ev[i]);
  if (pr->ev_fork) cudaEventDestroy(pr->ev_fork);
  if (pr->ev_join) cudaEventDestroy(pr->ev_join);
  if (pr->st2) cudaStreamDestroy(pr->st2);
  if (pr->st) cudaStreamDestroy(pr->st);
  delete pr;
}

extern "C" void* salsaa_prover_stream(salsaa_prover* pr) { return pr ? (void*)pr->st : nullptr; }

extern "C" int salsaa_prover_set_overlap(salsaa_prover* pr, int on) {
  if (!pr) return salsaa_set_error(-1, "prover_set_overlap: null argument");
  pr->overlap = on != 0;
  return 0;
}

__global__ void set_seed_kernel(DevState* ds, u64 seed) { ds->seed = seed; }

// <statement rows [0, nck) ++ scalar rows [sc_first, sc_first + nsc), witness rows>
// -> slot-form ring elements in pr->cout, row-major (statement, witness).
// wc: the same witness rows in coefficient form (scalar rows are summed there), or null.
static int commit_rows_slot(salsaa_prover* pr, const RowSet& ws, const RowSet* wc, u32 rows, u64 width, u32 nck,
                            u32 sc_first, u32 nsc) {
  salsaa_ctx* c = pr->ctx;
  if ((u64)sc_first + nsc > c->S.nsc_total || nck > c->P.module_size)
    return salsaa_set_error(-9, "commit: statement row range outside the proof's rows");
  CommitArgs a{};
  a.w = ws;
  if (wc && nsc) {
    a.wc = *wc;
    a.coef_sc = true;
  }
  a.rows = rows;
  a.width = width;
  a.nck = nck;
  a.tlo = c->tlo;
  a.thi = c->thi;
  a.ck_bt = c->ck_bt;
  a.ck_nhi = c->ck_nhi;
  a.nsc = nsc;
  a.sc_desc_dev = pr->sc_desc + sc_first;
  a.sc_types_host = nsc ? pr->sc_types.data() + sc_first : nullptr;
  a.sc_base_dev = pr->sc_base + sc_first;
  a.sc_lo = pr->sc_lo;
  a.sc_hi = pr->sc_hi;
  a.acc = pr->acc;
  a.tl8 = c->tl8;
  a.tk8 = c->tk8;
  a.colsum = pr->colsum;
  a.colsum_rows = c->S.max_rows + 1;  // the merged split/projection pass has 2K + 1 rows
  if ((u64)(c->d / 128) * (width / CK_BLOCK > 0 ? width / CK_BLOCK : 1) * rows <= pr->sc_flag_words) {
    a.sc_img = pr->sc_img;
    a.sc_flags = pr->sc_flags;
    a.sc_flag_cap = pr->sc_flag_words;
  }
  if (pr->overlap) {
    a.st2 = pr->st2;
    a.ev_fork = pr->ev_fork;
    a.ev_join = pr->ev_join;
  }
  a.out_slot = pr->cout;
  return launch_commit(a, *c->T, c->M, pr->ds, pr->st);
}

// Same, in coefficient form at proof_out.
static int commit_rows(salsaa_prover* pr, const RowSet& ws, const RowSet* wc, u32 rows, u64 width, u32 nck,
                       u32 sc_first, u32 nsc, u64* proof_out) {
  TRY(commit_rows_slot(pr, ws, wc, rows, width, nck, sc_first, nsc));
  return ntt_launch(pr->cout, proof_out, (u64)(nck + nsc) * rows, *pr->ctx->T, true, true, pr->st);
}

static RowSet rows_of(const u64* base, u32 rows, u64 width, u32 d) {
  RowSet r{};
  for (u32 k = 0; k < rows; k++) r.p[k] = base + (u64)k * width * d;
  return r;
}
// The same rows stored as centred int32 values (decomposition digits).
static RowSet rows_of_narrow(const u64* base, u32 rows, u64 width, u32 d) {
  RowSet r{};
  for (u32 k = 0; k < rows; k++) r.p[k] = (const u64*)((const int*)base + (u64)k * width * d);
  r.narrow = rows >= 32 ? ~0u : ((1u << rows) - 1);
  return r;
}

static int enqueue_impl(salsaa_prover* pr, u64 seed, const u64* d_witness, u64* proof) {
  salsaa_ctx* c = pr->ctx;
  const salsaa_params& P = c->P;
  const u32 d = c->d, ms = (u32)P.module_size;
  const u64 q = P.q, L = c->L;
  const ModQ& M = c->M;
  const NttDev& T = *c->T;
  cudaStream_t st = pr->st;
  pr->nev = 0;
  u64 cur = 0;
  TRY(mark(pr, PH_COMMIT));
  cudaError_t e = cudaMemcpyAsync(proof, pr->header_pinned, 8 * sizeof(u64), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "enqueue: header");
  cur = 8;
  set_seed_kernel<<<1, 1, 0, st>>>(pr->ds, seed);
  salsaa_count_launch();
  u32 K = (u32)P.init_wit_rep;
  u64 width = L;
  RowSet Wc, Ws;
  const u64* wbase = d_witness;
  if (!wbase) {
    TRY(launch_gen_witness(pr->Dc, K, width, d, q, pr->ds, st));
    wbase = pr->Dc;
  }
  Wc = rows_of(wbase, K, width, d);
  TRY(ntt_launch(wbase, pr->Ds, (u64)K * width, T, true, false, st));
  Ws = rows_of(pr->Ds, K, width, d);
  // commitment: parallel_dot_series_matrix(crs.ck, witness), src/protocol.rs:138.
  // In the SNARK it is derived from round 0's split commitment through the
  // split relation (exact mod q), so the witness is not streamed twice.
  u64 pend_off = cur;             // pending derived commitment: proof offset,
  u32 pend_rows = ms, pend_K = K; // statement rows and witness rows
  bool pending = !P.folding && P.nof_rounds > 0;
  if (!pending) TRY(commit_rows(pr, Ws, &Wc, K, width, ms, 0, 0, proof + cur));
  cur += (u64)ms * K * d;
  u32 nsc = 0, didx = 0;
  bool mag_ready = false;  // bw_or[didx] filled by the transforms of the joined witness
  for (u32 rd = 0; rd < P.nof_rounds; rd++) {
    const u32 parts = (u32)P.decomp_parts[rd < 12 ? rd : 11];
    if (!P.folding && parts > 1) {
      // decomp_ell (src/subroutines/decomp.rs:32-67)
      TRY(mark(pr, PH_DECOMP));
      bool narrow = false;
      TRY(launch_decompose_ntt(Wc, K, width, d, q, parts, didx++, pr->ds, pr->Dc, pr->Ds, proof + cur, T, st,
                               mag_ready, &narrow));
      mag_ready = false;
      cur += 1;
      K *= parts;
      Wc = narrow ? rows_of_narrow(pr->Dc, K, width, d) : rows_of(pr->Dc, K, width, d);
      Ws = rows_of(pr->Ds, K, width, d);
      // decomp rhs: derived after this round's split (see below)
      pend_off = cur;
      pend_rows = ms + nsc;
      pend_K = K;
      pending = true;
      cur += (u64)(ms + nsc) * K * d;
    } else if (!P.folding && rd > 0) {
      // the witness is last round's joined [folded, projected] rows, whose
      // buffers this round's projection and fold overwrite: move it to the
      // decomposition buffers, which a round without decomposition leaves free
      for (u32 k = 0; k < K; k++) {
        e = cudaMemcpyAsync(pr->Dc + (u64)k * width * d, Wc.p[k], width * d * sizeof(u64), cudaMemcpyDeviceToDevice,
                            st);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(pr->Ds + (u64)k * width * d, Ws.p[k], width * d * sizeof(u64),
                              cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return salsaa_set_cuda_error(e, "enqueue: joined witness");
      }
      Wc = rows_of(pr->Dc, K, width, d);
      Ws = rows_of(pr->Ds, K, width, d);
    }
    // split (src/subroutines/split.rs:45-76): rows L_0..L_{K-1}, R_0..R_{K-1},
    // as views; the sumcheck below still reads the unsplit rows
    RowSet Wc2 = Wc, Ws2 = Ws;
    u32 K2 = K;
    u64 width2 = width;
    if (!P.folding) {
      const u64 hw = width / 2;
      for (u32 k = 0; k < K; k++) {
        Wc2.p[k] = Wc.p[k];
        Wc2.p[K + k] = row_advance(Wc.p[k], (Wc.narrow >> k) & 1, hw * d);
        Ws2.p[k] = Ws.p[k];
        Ws2.p[K + k] = Ws.p[k] + hw * d;
      }
      Wc2.narrow = Wc.narrow | (Wc.narrow << K);
      K2 = 2 * K;
      width2 = hw;
    }
    // project (src/subroutines/project.rs:50-103): it needs the split witness
    // and its own challenges only, so with overlap on it runs on the side
    // stream beside the norm check and joins before the merged commitment
    cudaStream_t ps = pr->overlap ? pr->st2 : st;
    if (pr->overlap) {
      e = cudaEventRecord(pr->ev_fork, st);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(pr->st2, pr->ev_fork, 0);
      if (e != cudaSuccess) return salsaa_set_cuda_error(e, "enqueue: fork");
    }
    {
      const u32 cw = K2 * 256;
      u64* cj = pr->row_cj + (u64)rd * CK_BLOCK;
      TRY(launch_proj_tables(pr->ds, rd, cw, pr->pmask, pr->nmask, pr->Jm, cj, q, ps, pr->Jc));
      TRY(launch_project(Wc2, K2, width2, d, q, pr->pmask, pr->nmask, pr->Jm, pr->ds, pr->Pc, ps, pr->Jc));
    }
    // the joined witness [folded, projected] is decomposed next: the two
    // transforms that read P and write the folded row collect the OR of its
    // centred magnitudes, so the decomposition needs no pass of its own
    const bool next_decomp =
        P.folding || (rd + 1 < P.nof_rounds && P.decomp_parts[rd + 1 < 12 ? rd + 1 : 11] > 1);
    u64* mag = nullptr;
    if (next_decomp && didx < 16 && ntt_mag_ok(pr->Pc, pr->Ps, T, true) && ntt_mag_ok(pr->Fs, pr->Fc, T, true)) {
      mag = &pr->ds->bw_or[didx];
      e = cudaMemsetAsync(mag, 0, sizeof(u64), ps);
      if (e != cudaSuccess) return salsaa_set_cuda_error(e, "enqueue: magnitude OR");
    }
    TRY(ntt_launch(pr->Pc, pr->Ps, width2, T, true, false, ps, mag));
    if (pr->overlap && (e = cudaEventRecord(pr->ev_join, ps)) != cudaSuccess)
      return salsaa_set_cuda_error(e, "enqueue: join");

    // norm_check_1 / norm_check_2 (x2) / norm_check_3 (x2), src/protocol.rs:206-259
    TRY(mark(pr, PH_NORM2));
    const u64 nr = ilog2u(width * d);
    u64* claims = proof + cur;
    cur += K;
    u64* polys0 = proof + cur;
    u64* rhs0 = polys0 + nr * K * 3;
    u64* polys1 = rhs0 + (u64)K * d;
    u64* rhs1 = polys1 + nr * K * 3;
    cur = (u64)(rhs1 + (u64)K * d - proof);
    TRY(launch_sumcheck(Wc, K, width * d, d, M, pr->ds, rd, pr->sc, claims, polys0, polys1, st));
    TRY(mark(pr, PH_NORM3));
    TRY(launch_norm3(pr->sc.cap, K, (u32)nr, T, M, pr->ds, rd, rhs0, rhs1, pr->row_base + (u64)nsc * d,
                     pr->row_base + (u64)(nsc + 1) * d, st));
    nsc += 2;
    Wc = Wc2;
    Ws = Ws2;
    K = K2;
    width = width2;
    TRY(mark(pr, P.folding ? PH_PROJ : PH_SPLIT));
    if (pr->overlap && (e = cudaStreamWaitEvent(st, pr->ev_join, 0)) != cudaSuccess)
      return salsaa_set_cuda_error(e, "enqueue: join");
    RowSet Pr = rows_of(pr->Ps, 1, width, d);
    RowSet Prc = rows_of(pr->Pc, 1, width, d);
    const u32 S = ms + nsc;
    if (!P.folding) {
      // split rhs and projected commitment in one pass over the statement
      // rows: witness columns L_0..L_{K/2-1}, R_0..R_{K/2-1}, P.  The
      // challenges are fixed in advance, so computing P first changes nothing.
      // The pass also takes this round's witness_lhs (PERIODIC) and
      // projected_lhs (ONES) rows, statement rows S and S + 1: their products
      // with the split witness and with P are witness_rhs, projection_rhs and
      // the cross term l1 of batch_projections / send_cross_terms_before_join.
      TRY(mark(pr, PH_SPLIT));
      RowSet both = Ws, bothc = Wc;
      both.p[K] = pr->Ps;
      bothc.p[K] = pr->Pc;
      TRY(commit_rows_slot(pr, both, &bothc, K + 1, width, ms, 0, nsc + 2));
      TRY(ntt_launch(pr->cout, pr->cout2, (u64)(S + 2) * (K + 1), T, true, true, st));
      const size_t row_bytes = (size_t)(K + 1) * d * sizeof(u64);
      e = cudaMemcpy2DAsync(proof + cur, (size_t)K * d * sizeof(u64), pr->cout2, row_bytes,
                            (size_t)K * d * sizeof(u64), S, cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return salsaa_set_cuda_error(e, "enqueue: split rhs");
      cur += (u64)S * K * d;
      e = cudaMemcpy2DAsync(proof + cur, (size_t)d * sizeof(u64), pr->cout2 + (u64)K * d, row_bytes,
                            (size_t)d * sizeof(u64), S, cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return salsaa_set_cuda_error(e, "enqueue: projected commitment");
      cur += (u64)S * d;
      if (pending) {
        // commitment of the unsplit witness (initial commitment or decomp rhs)
        DeriveArgs da{};
        da.R = pr->cout;
        da.ncols = K + 1;
        da.K = K / 2;
        da.nck = ms;
        da.nsc = pend_rows - ms;
        da.w = 2 * width;
        da.tlo = c->tlo;
        da.thi = c->thi;
        da.ck_bt = c->ck_bt;
        da.ck_nhi = c->ck_nhi;
        da.packed = q < (1ULL << 50);
        da.sc_desc_dev = pr->sc_desc;
        da.out = pr->acc;
        if (da.K != pend_K) return salsaa_set_error(-9, "enqueue: derived commitment shape mismatch");
        TRY(launch_derive(da, T, M, pr->ds, st));
        TRY(ntt_launch(pr->acc, proof + pend_off, (u64)pend_rows * pend_K, T, true, true, st));
        pending = false;
      }
    } else {
      TRY(commit_rows(pr, Pr, &Prc, 1, width, ms, 0, nsc, proof + cur));
      cur += (u64)S * d;
    }
    // batch_projections (src/subroutines/project.rs:131-203): witness_rhs, projection_rhs
    const u64* l1_src = nullptr;  // <witness_lhs, projected> when the merged pass made it
    if (!P.folding) {
      const u64* wl = pr->cout2 + (u64)S * (K + 1) * d;  // witness_lhs x [split witness, P]
      const u64* pl = wl + (u64)(K + 1) * d;             // projected_lhs x [split witness, P]
      e = cudaMemcpyAsync(proof + cur, wl, (size_t)K * d * sizeof(u64), cudaMemcpyDeviceToDevice, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(proof + cur + (u64)K * d, pl + (u64)K * d, (size_t)d * sizeof(u64),
                            cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return salsaa_set_cuda_error(e, "enqueue: batch projections");
      l1_src = wl + (u64)K * d;
    } else {
      TRY(commit_rows(pr, Ws, &Wc, K, width, 0, nsc, 1, proof + cur));
      TRY(commit_rows(pr, Pr, &Prc, 1, width, 0, nsc + 1, 1, proof + cur + (u64)K * d));
    }
    cur += (u64)K * d + d;
    nsc += 1;  // witness_lhs joins the statement
    // fold (src/subroutines/fold.rs:22-27)
    TRY(mark(pr, PH_FOLD));
    TRY(launch_fold_challenge(pr->ds, rd, K, d, q, pr->c_coef, st));
    TRY(ntt_launch(pr->c_coef, pr->c_slot, K, T, true, false, st));
    TRY(launch_fold(Ws, K, width, T, M, pr->c_slot, pr->fold_pre, pr->Fs, st));
    TRY(ntt_launch(pr->Fs, pr->Fc, width, T, true, true, st, mag));
    mag_ready = mag != nullptr;
    // send_cross_terms_before_join (src/subroutines/project.rs:229-245)
    RowSet Fr = rows_of(pr->Fs, 1, width, d), Frc = rows_of(pr->Fc, 1, width, d);
    TRY(commit_rows(pr, Fr, &Frc, 1, width, 0, nsc, 1, proof + cur));  // l0 = <projected_lhs, folded>
    cur += d;
    if (l1_src) {  // l1 = <witness_lhs, projected>
      e = cudaMemcpyAsync(proof + cur, l1_src, (size_t)d * sizeof(u64), cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return salsaa_set_cuda_error(e, "enqueue: cross term");
    } else {
      TRY(commit_rows(pr, Pr, &Prc, 1, width, 0, nsc - 1, 1, proof + cur));
    }
    cur += d;
    nsc += 1;  // projected_lhs joins the statement
    // join: witness = [folded, projected]
    K = 2;
    Wc = RowSet{};
    Wc.p[0] = pr->Fc;
    Wc.p[1] = pr->Pc;
    Ws = RowSet{};
    Ws.p[0] = pr->Fs;
    Ws.p[1] = pr->Ps;
    if (P.folding) {
      TRY(mark(pr, PH_DECOMP));
      bool narrow = false;
      TRY(launch_decompose_ntt(Wc, K, width, d, q, 2, didx++, pr->ds, pr->Dc, pr->Ds, proof + cur, T, st,
                               mag_ready, &narrow));
      mag_ready = false;
      cur += 1;
      K *= 2;
      Ws = rows_of(pr->Ds, K, width, d);
      const RowSet Dcr = narrow ? rows_of_narrow(pr->Dc, K, width, d) : rows_of(pr->Dc, K, width, d);
      TRY(commit_rows(pr, Ws, &Dcr, K, width, ms, 0, nsc, proof + cur));
      cur += (u64)(ms + nsc) * K * d;
      break;
    }
  }
  if (pending) return salsaa_set_error(-9, "enqueue: a derived commitment was never produced");
  if (!P.folding) {
    for (u32 k = 0; k < K; k++) {
      e = cudaMemcpyAsync(proof + cur, Wc.p[k], width * d * sizeof(u64), cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return salsaa_set_cuda_error(e, "enqueue: final witness");
      cur += width * d;
    }
  }
  TRY(mark(pr, PH_N));
  if (cur != c->S.proof_words) return salsaa_set_error(-9, "enqueue: proof layout mismatch");
  return 0;
}

extern "C" int salsaa_prover_set_graph(salsaa_prover* pr, int on) {
  if (!pr) return salsaa_set_error(-1, "prover_set_graph: null argument");
  pr->use_graph = on != 0;
  return 0;
}

static void drop_graph(salsaa_prover* pr) {
  if (pr->gexec) cudaGraphExecDestroy(pr->gexec);
  if (pr->graph) cudaGraphDestroy(pr->graph);
  pr->graph = nullptr;
  pr->gexec = nullptr;
  pr->gseed = nullptr;
  pr->g_witness = nullptr;
  pr->g_proof = nullptr;
  pr->g_kernels = 0;
}

// Captures the proof's launch sequence on the slot's stream (relaxed mode:
// the launchers' attribute calls are allowed), finds the seed kernel's node
// and instantiates the graph.  Nothing runs while capturing.  Returns 0, or
// nonzero when the capture could not be made (the caller then launches
// directly; the CUDA error state is cleared).
static int capture_graph(salsaa_prover* pr, u64 seed, const u64* d_witness, u64* proof) {
  drop_graph(pr);
  const uint64_t counted = g_launches.load(std::memory_order_relaxed);  // capturing launches nothing
  cudaError_t e = cudaStreamBeginCapture(pr->st, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  pr->capturing = true;
  const int rc = enqueue_impl(pr, seed, d_witness, proof);
  pr->capturing = false;
  g_launches.fetch_sub(g_launches.load(std::memory_order_relaxed) - counted, std::memory_order_relaxed);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(pr->st, &g);
  if (rc || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return -1;
  }
  size_t nn = 0;
  int out = -1;
  if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess) {
    std::vector<cudaGraphNode_t> nodes(nn);
    if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess) {
      u64 kernels = 0;
      for (cudaGraphNode_t n : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(n, &t) != cudaSuccess || t != cudaGraphNodeTypeKernel) continue;
        kernels++;
        cudaKernelNodeParams kp{};
        if (cudaGraphKernelNodeGetParams(n, &kp) == cudaSuccess && kp.func == (void*)set_seed_kernel) {
          pr->gseed = n;
          pr->gseed_p = kp;
        }
      }
      pr->g_kernels = kernels;
      if (pr->gseed && cudaGraphInstantiate(&pr->gexec, g, 0) == cudaSuccess) out = 0;
    }
  }
  pr->graph = g;
  if (out) {
    drop_graph(pr);
    cudaGetLastError();
    return -1;
  }
  pr->g_witness = d_witness;
  pr->g_proof = proof;
  pr->g_sched = schedule_generation();
  pr->g_overlap = pr->overlap;
  return 0;
}

// One proof, through the slot's graph when graph replay is on (captured on
// the first call for these buffers), else by direct launches.
static int enqueue_any(salsaa_prover* pr, u64 seed, const u64* d_witness, u64* proof) {
  const bool graph = pr->use_graph && !pr->graph_failed && !salsaa_trace_active();
  if (!graph) return enqueue_impl(pr, seed, d_witness, proof);
  if (!pr->gexec || pr->g_witness != d_witness || pr->g_proof != proof || pr->g_overlap != pr->overlap ||
      pr->g_sched != schedule_generation()) {
    if (capture_graph(pr, seed, d_witness, proof)) {
      pr->graph_failed = true;
      return enqueue_impl(pr, seed, d_witness, proof);
    }
  } else {
    DevState* ds = pr->ds;
    u64 sd = seed;
    void* args[2] = {&ds, &sd};
    cudaKernelNodeParams kp = pr->gseed_p;
    kp.kernelParams = args;
    kp.extra = nullptr;
    cudaError_t e = cudaGraphExecKernelNodeSetParams(pr->gexec, pr->gseed, &kp);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover graph: seed update");
  }
  pr->nev = 0;
  cudaError_t e = cudaGraphLaunch(pr->gexec, pr->st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover graph: launch");
  for (u64 i = 0; i < pr->g_kernels; i++) salsaa_count_launch();
  return 0;
}

extern "C" int salsaa_prover_enqueue(salsaa_prover* pr, uint64_t seed, const uint64_t* d_witness,
                                     uint8_t* d_proof) {
  if (!pr || !d_proof) return salsaa_set_error(-1, "prover_enqueue: null argument");
  if (((uintptr_t)d_proof) & 7) return salsaa_set_error(-1, "prover_enqueue: proof buffer not 8-byte aligned");
  cudaError_t e = cudaSetDevice(pr->ctx->device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue: cudaSetDevice");
  pr->last_rc = enqueue_any(pr, seed, d_witness, (u64*)d_proof);
  return pr->last_rc;
}

extern "C" int salsaa_prover_enqueue_host(salsaa_prover* pr, uint64_t seed, const uint64_t* h_witness,
                                          uint8_t* h_proof) {
  if (!pr || !h_proof) return salsaa_set_error(-1, "prover_enqueue_host: null argument");
  salsaa_ctx* c = pr->ctx;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host: cudaSetDevice");
  const u64 need = c->S.proof_words * 8;
  if (!pr->own_proof) {
    e = cudaMalloc(&pr->own_proof, need);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host: proof buffer");
  }
  const u64* dw = nullptr;
  if (h_witness) {
    const u64 bytes = c->P.init_wit_rep * c->L * c->d * sizeof(u64);
    e = cudaMemcpyAsync(pr->Dc, h_witness, bytes, cudaMemcpyHostToDevice, pr->st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host: witness upload");
    dw = pr->Dc;
  }
  pr->last_rc = enqueue_any(pr, seed, dw, (u64*)pr->own_proof);
  if (pr->last_rc) return pr->last_rc;
  e = cudaMemcpyAsync(h_proof, pr->own_proof, need, cudaMemcpyDeviceToHost, pr->st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host: proof download");
  return 0;
}

// The signed bytes cross PCIe on the slot's upload stream into one of two
// staging buffers (an eighth of the u64 witness each), so the next proof's
// witness uploads while the current proof runs; the slot's stream waits for
// its upload, expands it into the coefficient-form buffer and releases the
// staging buffer for the upload after next.
extern "C" int salsaa_prover_enqueue_host_i8(salsaa_prover* pr, uint64_t seed, const int8_t* h_witness,
                                             uint8_t* h_proof) {
  if (!pr || !h_proof || !h_witness) return salsaa_set_error(-1, "prover_enqueue_host_i8: null argument");
  salsaa_ctx* c = pr->ctx;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host_i8: cudaSetDevice");
  const u64 need = c->S.proof_words * 8;
  if (!pr->own_proof) {
    e = cudaMalloc(&pr->own_proof, need);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host_i8: proof buffer");
  }
  const u64 n = c->P.init_wit_rep * c->L * c->d;
  if (!pr->cp_st) {  // the upload stream, its two staging buffers and their events, on first use
    e = cudaStreamCreateWithFlags(&pr->cp_st, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; i++) {
      e = cudaMalloc(&pr->stage8[i], (n + 15) & ~(u64)15);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pr->ev_copied[i], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pr->ev_free[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host_i8: upload buffers");
  }
  // upload k into stage8[k % 2] once the expansion of upload k - 2 has read it
  const int b = (int)(pr->n_i8++ & 1);
  e = cudaStreamWaitEvent(pr->cp_st, pr->ev_free[b], 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(pr->stage8[b], h_witness, n, cudaMemcpyHostToDevice, pr->cp_st);
  if (e == cudaSuccess) e = cudaEventRecord(pr->ev_copied[b], pr->cp_st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(pr->st, pr->ev_copied[b], 0);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host_i8: witness upload");
  pr->last_rc = launch_expand_i8(pr->stage8[b], n, c->P.q, pr->Dc, pr->st);
  if (pr->last_rc) return pr->last_rc;
  e = cudaEventRecord(pr->ev_free[b], pr->st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host_i8: stage release");
  pr->last_rc = enqueue_any(pr, seed, pr->Dc, (u64*)pr->own_proof);
  if (pr->last_rc) return pr->last_rc;
  e = cudaMemcpyAsync(h_proof, pr->own_proof, need, cudaMemcpyDeviceToHost, pr->st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_enqueue_host_i8: proof download");
  return 0;
}

extern "C" int salsaa_prover_query(salsaa_prover* pr) {
  if (!pr) return salsaa_set_error(-1, "prover_query: null argument");
  if (pr->last_rc) return pr->last_rc;
  cudaError_t e = cudaStreamQuery(pr->st);
  if (e == cudaErrorNotReady) return 1;
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_query");
  return 0;
}

extern "C" int salsaa_prover_sync(salsaa_prover* pr) {
  if (!pr) return salsaa_set_error(-1, "prover_sync: null argument");
  cudaError_t e = cudaStreamSynchronize(pr->st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_sync");
  if (pr->last_rc) return pr->last_rc;
  return tc_error_check();
}

extern "C" int salsaa_prover_timing(salsaa_prover* pr, salsaa_timing* t) {
  if (!pr || !t) return salsaa_set_error(-1, "prover_timing: null argument");
  double ph[PH_N] = {0};
  double total = 0;
  for (int i = 0; i + 1 < pr->nev; i++) {
    float ms = 0;
    cudaError_t e = cudaEventElapsedTime(&ms, pr->ev[i], pr->ev[i + 1]);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prover_timing");
    if (pr->ev_phase[i] < PH_N) ph[pr->ev_phase[i]] += ms;
    total += ms;
  }
  t->commit = ph[PH_COMMIT];
  t->norm1 = ph[PH_NORM1];
  t->norm2 = ph[PH_NORM2];
  t->norm3 = ph[PH_NORM3];
  t->split = ph[PH_SPLIT];
  t->projection = ph[PH_PROJ];
  t->fold = ph[PH_FOLD];
  t->decomp = ph[PH_DECOMP];
  t->total = total;
  return 0;
}

extern "C" int salsaa_prove(salsaa_ctx* c, uint64_t seed, const uint64_t* h_witness, uint8_t* h_proof,
                            uint64_t proof_len) {
  if (!c || !h_proof) return salsaa_set_error(-1, "prove: null argument");
  if (!c->S.ok) return salsaa_set_error(-1, ("prove: " + c->S.why).c_str());
  const u64 need = c->S.proof_words * 8;
  if (proof_len < need) return salsaa_set_error(-2, "prove: proof buffer too small");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prove: cudaSetDevice");
  if (!c->blocking) {
    TRY(salsaa_prover_create(c, &c->blocking));
    e = cudaMalloc(&c->blocking->own_proof, need);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prove: proof buffer");
  }
  salsaa_prover* pr = c->blocking;
  const u64* dw = nullptr;
  if (h_witness) {
    const u64 bytes = c->P.init_wit_rep * c->L * c->d * sizeof(u64);
    e = cudaMemcpyAsync(pr->Dc, h_witness, bytes, cudaMemcpyHostToDevice, pr->st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prove: witness upload");
    dw = pr->Dc;
  }
  TRY(salsaa_prover_enqueue(pr, seed, dw, pr->own_proof));
  e = cudaMemcpyAsync(h_proof, pr->own_proof, need, cudaMemcpyDeviceToHost, pr->st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "prove: proof download");
  return salsaa_prover_sync(pr);
}

// ---------------------------------------------------------------------------
// Verifier.  The checks the reference's verifier makes inline
// (verify_decomp src/subroutines/decomp.rs:69-112, verify_norm_check_2/3
// src/subroutines/fast_norm_check.rs:352-462, verifier_split
// src/subroutines/split.rs:171-221, verify_batching / verifier_fold /
// verifier_join src/subroutines/project.rs:205-275 and fold.rs:58-67, and the
// final check src/protocol.rs:464-472) replayed on a proof.  The proof's ring
// elements move to slot form on the GPU; the scalar and per-element checks run
// on the host (a few thousand ring elements); the final check, the statement
// rows against the final witness, is a commitment over the witness and runs on
// the GPU through the prover's own commitment path.  Verdict codes: 0 accept,
// -3 header or shape, -5 length, -20 radix, -21 decomposition, -30/-31
// sumcheck, -32 norm3, -40/-41 split, -50 projection, -60 final check.
// ---------------------------------------------------------------------------
namespace {

struct HostSlots {
  u64 q;
  u32 n, d;
  std::vector<u64> zeta;
  // (a_e + a_o X)(b_e + b_o X) mod (X^2 - zeta_s), slot by slot
  void mul(const u64* a, const u64* b, u64* r) const {
    for (u32 s = 0; s < n; s++) {
      const u64 ae = a[s], ao = a[n + s], be = b[s], bo = b[n + s];
      const u64 e = host::addmod(host::mulmod(ae, be, q), host::mulmod(host::mulmod(ao, bo, q), zeta[s], q), q);
      const u64 o = host::addmod(host::mulmod(ae, bo, q), host::mulmod(ao, be, q), q);
      r[s] = e;
      r[n + s] = o;
    }
  }
};

// Statement rows as the verifier tracks them: PowerSeries shapes (a base
// layer of blen elements and K tensor factors).
struct VRow {
  int type;             // RowType
  u32 ck;               // commitment-key row
  u64 K, blen;
  std::vector<u64> c;   // TENSOR: the challenges of the K factors (1 - c, c)
};

u64 nc_chal_host(u64 seed, u64 round, u64 rep, u64 j, u64 q) {
  return (u64)(((unsigned __int128)prf_at(prf_key(seed, domain_id(DOM_NC, round, rep)), j) * q) >> 64);
}

// Ring-element segments (word offset, element count) of a proof, in order.
void proof_segments(const salsaa_params& P, std::vector<std::pair<u64, u64>>& seg) {
  const u64 d = P.d;
  u64 pos = 8, S = P.module_size, K = P.init_wit_rep, width = P.wit_len;
  auto ring = [&](u64 cnt) {
    seg.push_back({pos, cnt});
    pos += cnt * d;
  };
  ring(S * K);
  for (u64 rd = 0; rd < P.nof_rounds; rd++) {
    const u64 parts = P.decomp_parts[rd < 12 ? rd : 11];
    if (!P.folding && parts > 1) {
      pos += 1;
      ring(S * K * parts);
      K *= parts;
    }
    pos += K;
    const u64 nr = ilog2u(width * d);
    for (int rep = 0; rep < 2; rep++) {
      pos += nr * K * 3;
      ring(K);
      S += 1;
    }
    if (!P.folding) {
      ring(S * 2 * K);
      K *= 2;
      width /= 2;
    }
    ring(S);      // projected commitment
    ring(K);      // witness_rhs
    ring(1);      // projection_rhs
    S += 1;
    ring(2);      // l0, l1
    S += 1;
    K = 2;
    if (P.folding) {
      pos += 1;
      ring(S * K * 2);
      K *= 2;
      break;
    }
  }
  if (!P.folding) ring(K * width);
}

}  // namespace

static int verify_impl(salsaa_prover* pr, u64 seed, const u64* proof, int* verdict) {
  salsaa_ctx* c = pr->ctx;
  const salsaa_params& P = c->P;
  const NttDev& T = *c->T;
  const u64 d = c->d, n = c->n, q = P.q, ms = P.module_size, words = c->S.proof_words, L = c->L;
  cudaStream_t st = pr->st;
  *verdict = 0;
  const u64 hdr[8] = {0x31504141534C4153ULL, P.d, P.q, P.module_size, P.wit_len, P.init_wit_rep, P.nof_rounds,
                      P.folding};
  for (int i = 0; i < 8; i++)
    if (proof[i] != hdr[i]) {
      *verdict = -3;
      return 0;
    }
  if (words > c->S.max_d_rows_width * d) return salsaa_set_error(-9, "verify: proof larger than the slot's buffers");
  // the proof in coefficient form (own_proof) and its ring elements in slot form (Ds)
  cudaError_t e;
  if (!pr->own_proof && (e = cudaMalloc(&pr->own_proof, words * 8)) != cudaSuccess)
    return salsaa_set_cuda_error(e, "verify: proof buffer");
  u64* dcoef = (u64*)pr->own_proof;
  u64* dslot = pr->Ds;
  if ((e = cudaMemcpyAsync(dcoef, proof, words * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return salsaa_set_cuda_error(e, "verify: proof upload");
  set_seed_kernel<<<1, 1, 0, st>>>(pr->ds, seed);  // the challenges drawn on the device
  salsaa_count_launch();
  std::vector<std::pair<u64, u64>> seg;
  proof_segments(P, seg);
  for (const auto& s : seg) TRY(ntt_launch(dcoef + s.first, dslot + s.first, s.second, T, true, false, st));
  std::vector<u64> slot(words), mslot((u64)ms * d);
  HostSlots R{q, (u32)n, (u32)d, std::vector<u64>(n)};
  if ((e = cudaMemcpyAsync(slot.data(), dslot, words * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(R.zeta.data(), T.zeta, n * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(mslot.data(), c->m_slot, ms * d * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return salsaa_set_cuda_error(e, "verify: slot forms");
  // m_r^(2^j) for the split checks of the commitment-key rows
  const u32 logL = (u32)ilog2u(L);
  std::vector<u64> mpow((u64)ms * (logL + 1) * d);
  for (u64 r = 0; r < ms; r++) {
    u64* p = mpow.data() + r * (logL + 1) * d;
    memcpy(p, mslot.data() + r * d, d * 8);
    for (u32 j = 1; j <= logL; j++) R.mul(p + (j - 1) * d, p + (j - 1) * d, p + j * d);
  }

  u64 pos = 8;
  auto ring = [&](u64 cnt) {
    const u64* p = slot.data() + pos;
    pos += cnt * d;
    return p;
  };
  auto word = [&]() { return pos < words ? proof[pos++] : (pos++, 0ULL); };
  std::vector<VRow> rows;
  for (u64 r = 0; r < ms; r++) rows.push_back(VRow{ROW_CK, (u32)r, logL, 1, {}});
  u64 K = P.init_wit_rep, width = L;
  const u64* v0 = ring(ms * K);
  std::vector<u64> V(v0, v0 + ms * K * d), tmp(d), tmp2(d);
  struct RoundRows {
    u64 rd, nr, cw;
  };
  std::vector<RoundRows> rr;
  int rc = 0;
  auto compose_check = [&](u64 parts, u64 radix, const u64* Dm) {
    const u64 S = rows.size(), shift = (u64)__builtin_ctzll(radix);
    for (u64 j = 0; j < S; j++)
      for (u64 i = 0; i < K; i++)
        for (u64 t = 0; t < d; t++) {
          u64 acc = 0;
          for (u64 cc = 0; cc < parts; cc++) {
            const u64 pw = shift * cc < 64 ? ((1ULL << (shift * cc)) % q) : 0;
            acc = host::addmod(acc, host::mulmod(Dm[((j * K + i) * parts + cc) * d + t], pw, q), q);
          }
          if (acc != V[(j * K + i) * d + t]) return false;
        }
    return true;
  };

  for (u64 rd = 0; rd < P.nof_rounds && !rc; rd++) {
    const u64 parts = P.decomp_parts[rd < 12 ? rd : 11];
    if (!P.folding && parts > 1) {  // verify_decomp
      const u64 radix = word();
      if (!radix || (radix & (radix - 1))) {
        rc = -20;
        break;
      }
      const u64* Dm = ring(rows.size() * K * parts);
      if (!compose_check(parts, radix, Dm)) {
        rc = -21;
        break;
      }
      V.assign(Dm, Dm + rows.size() * K * parts * d);
      K *= parts;
    }
    const u64 nr = ilog2u(width * d);
    std::vector<u64> claims(K), cs(nr ? nr : 1);
    for (u64 k = 0; k < K; k++) claims[k] = word();
    for (u64 rep = 0; rep < 2; rep++) {  // verify_norm_check_2, verify_norm_check_3
      std::vector<u64> cl = claims;
      for (u64 j = 0; j < nr; j++) cs[j] = nc_chal_host(seed, rd, rep, j, q);
      for (u64 j = 0; j < nr; j++)
        for (u64 k = 0; k < K; k++) {
          const u64 f0 = word(), f1 = word(), f2 = word();
          if (f0 >= q || f1 >= q || f2 >= q) rc = rc ? rc : -30;
          const u64 lhs = host::addmod(host::addmod(host::addmod(f0, f0, q), host::addmod(f1, f1, q), q), f2, q);
          if (lhs != cl[k]) rc = rc ? rc : -31;
          const u64 cj = cs[j];
          cl[k] = host::addmod(host::addmod(f0, host::mulmod(host::addmod(f1, f1, q), cj, q), q),
                               host::mulmod(host::mulmod(f2, cj, q), cj, q), q);
        }
      for (u64 k = 0; k < K; k++) {
        const u64 c0 = proof[pos];
        if (host::mulmod(c0, c0, q) != cl[k]) rc = rc ? rc : -32;
        const u64* rhs = ring(1);
        V.insert(V.end(), rhs, rhs + d);
      }
      const u64 Kr = nr - ilog2u(d);
      rows.push_back(VRow{ROW_TENSOR, 0, Kr, 1, std::vector<u64>(cs.begin(), cs.begin() + Kr)});
    }
    rr.push_back(RoundRows{rd, nr, 0});
    if (rc) break;
    if (!P.folding) {  // verifier_split: t0 * L + t1 * R = the unsplit value, row by row
      const u64 S = rows.size();
      const u64* SR = ring(S * 2 * K);
      for (u64 j = 0; j < S && !rc; j++) {
        const VRow& w = rows[j];
        if (width % w.blen) {
          rc = -40;
          break;
        }
        const u64 f = width / w.blen;
        if (f & (f - 1)) {
          rc = -40;
          break;
        }
        const u64 jj = ilog2u(f);
        if (jj == 0 || jj > w.K) {
          rc = -40;
          break;
        }
        for (u64 k = 0; k < K && !rc; k++) {
          const u64* a = SR + (j * 2 * K + k) * d;
          const u64* b = SR + (j * 2 * K + K + k) * d;
          if (w.type == ROW_CK) {  // t0 = 1, t1 = m^(width / 2)
            R.mul(mpow.data() + ((u64)w.ck * (logL + 1) + jj - 1) * d, b, tmp.data());
            for (u64 t = 0; t < d; t++) tmp[t] = host::addmod(tmp[t], a[t], q);
          } else {  // scalar factors: (1 - c, c) for TENSOR rows, (1, 1) otherwise
            const u64 ci = w.type == ROW_TENSOR ? w.c[w.K - jj] : 0;
            const u64 t0 = w.type == ROW_TENSOR ? host::submod(1 % q, ci, q) : 1 % q;
            const u64 t1 = w.type == ROW_TENSOR ? ci : 1 % q;
            for (u64 t = 0; t < d; t++) tmp[t] = host::addmod(host::mulmod(a[t], t0, q), host::mulmod(b[t], t1, q), q);
          }
          if (memcmp(tmp.data(), V.data() + (j * K + k) * d, d * 8)) rc = -41;
        }
      }
      if (rc) break;
      V.assign(SR, SR + S * 2 * K * d);
      K *= 2;
      width /= 2;
    }
    const u64 cw = K * 256;
    if (cw > width) {
      rc = -3;
      break;
    }
    rr.back().cw = cw;
    const u64 Sp = rows.size();
    const u64* PC = ring(Sp);
    const u64* wrhs = ring(K);
    const u64* prhs = ring(1);
    std::fill(tmp.begin(), tmp.end(), 0);
    for (u64 k = 0; k < K; k++)
      for (u64 t = 0; t < d; t++) tmp[t] = host::addmod(tmp[t], wrhs[k * d + t], q);
    if (memcmp(tmp.data(), prhs, d * 8)) {  // verify_batching
      rc = -50;
      break;
    }
    V.insert(V.end(), wrhs, wrhs + K * d);
    rows.push_back(VRow{ROW_PERIODIC, 0, ilog2u(width / cw), cw, {}});
    // verifier_fold: VF_j = sum_k c_k V_jk with the fold challenges in slot form
    TRY(launch_fold_challenge(pr->ds, (u32)rd, (u32)K, (u32)d, q, pr->c_coef, st));
    TRY(ntt_launch(pr->c_coef, pr->c_slot, K, T, true, false, st));
    std::vector<u64> cslot(K * d);
    if ((e = cudaMemcpyAsync(cslot.data(), pr->c_slot, K * d * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return salsaa_set_cuda_error(e, "verify: fold challenge");
    const u64 S = rows.size();
    std::vector<u64> VF(S * d, 0);
    for (u64 j = 0; j < S; j++)
      for (u64 k = 0; k < K; k++) {
        R.mul(cslot.data() + k * d, V.data() + (j * K + k) * d, tmp.data());
        for (u64 t = 0; t < d; t++) VF[j * d + t] = host::addmod(VF[j * d + t], tmp[t], q);
      }
    const u64* l0 = ring(1);
    const u64* l1 = ring(1);
    rows.push_back(VRow{ROW_ONES, 0, ilog2u(width / cw) + ilog2u(K), 256, {}});
    // verifier_join: new rhs with witness columns [folded, projected]
    std::vector<u64> NV((Sp + 2) * 2 * d);
    for (u64 i = 0; i < Sp; i++) {
      memcpy(NV.data() + (i * 2) * d, VF.data() + i * d, d * 8);
      memcpy(NV.data() + (i * 2 + 1) * d, PC + i * d, d * 8);
    }
    memcpy(NV.data() + (Sp * 2) * d, VF.data() + Sp * d, d * 8);
    memcpy(NV.data() + (Sp * 2 + 1) * d, l1, d * 8);
    memcpy(NV.data() + ((Sp + 1) * 2) * d, l0, d * 8);
    memcpy(NV.data() + ((Sp + 1) * 2 + 1) * d, prhs, d * 8);
    V.swap(NV);
    K = 2;
    if (P.folding) {
      const u64 radix = word();
      if (!radix || (radix & (radix - 1))) {
        rc = -20;
        break;
      }
      const u64* Dm = ring(rows.size() * K * 2);
      if (!compose_check(2, radix, Dm)) {
        rc = -21;
        break;
      }
      V.assign(Dm, Dm + rows.size() * K * 2 * d);
      K *= 2;
      break;
    }
  }
  if (!rc && !P.folding) {
    // final check: every statement row against the final witness, on the GPU
    const u64 fw = K * width * d;
    if (pos + fw > words || 2 * fw > c->S.max_d_rows_width * d) {
      rc = -5;
    } else {
      u64* wc = pr->Dc;
      u64* ws = pr->Dc + fw;
      if ((e = cudaMemcpyAsync(wc, dcoef + pos, fw * 8, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return salsaa_set_cuda_error(e, "verify: final witness");
      pos += fw;
      TRY(ntt_launch(wc, ws, K * width, T, true, false, st));
      // the device-side statement rows: norm3 bases and projection sums per round
      if ((e = cudaMemsetAsync(pr->sc.cap, 0, 2 * d * 8, st)) != cudaSuccess)
        return salsaa_set_cuda_error(e, "verify: norm3 scratch");
      for (const RoundRows& x : rr) {
        TRY(launch_norm3(pr->sc.cap, 1, (u32)x.nr, T, c->M, pr->ds, (u32)x.rd, pr->cout2, pr->cout2 + d,
                         pr->row_base + (4 * x.rd) * d, pr->row_base + (4 * x.rd + 1) * d, st));
        TRY(launch_proj_tables(pr->ds, (u32)x.rd, (u32)x.cw, pr->pmask, pr->nmask, pr->Jm,
                               pr->row_cj + x.rd * CK_BLOCK, q, st, pr->Jc));
      }
      const u32 nsc = (u32)(rows.size() - ms);
      const RowSet fwc = rows_of(wc, (u32)K, width, (u32)d);
      TRY(commit_rows_slot(pr, rows_of(ws, (u32)K, width, (u32)d), &fwc, (u32)K, width, (u32)ms, 0, nsc));
      std::vector<u64> out(rows.size() * K * d);
      if ((e = cudaMemcpyAsync(out.data(), pr->cout, out.size() * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
          (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return salsaa_set_cuda_error(e, "verify: final check");
      TRY(tc_error_check());
      if (out != V) rc = -60;
    }
  }
  if (!rc && pos != words) rc = -5;
  *verdict = rc;
  return 0;
}

extern "C" int salsaa_verify(salsaa_ctx* c, uint64_t seed, const uint8_t* h_proof, uint64_t proof_len,
                             int* verdict) {
  if (!c || !h_proof || !verdict) return salsaa_set_error(-1, "verify: null argument");
  if (!c->S.ok) return salsaa_set_error(-1, ("verify: " + c->S.why).c_str());
  *verdict = -5;
  if (proof_len != c->S.proof_words * 8) return 0;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "verify: cudaSetDevice");
  if (!c->blocking) TRY(salsaa_prover_create(c, &c->blocking));
  std::vector<u64> words(c->S.proof_words);
  memcpy(words.data(), h_proof, proof_len);
  return verify_impl(c->blocking, seed, words.data(), verdict);
}

extern "C" void salsaa_ctx_destroy(salsaa_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->blocking) salsaa_prover_destroy(c->blocking);
  std::lock_guard<std::mutex> lk(g_ctx_bufs_mu);
  for (size_t i = 0; i < g_ctx_bufs.size(); i++)
    if (g_ctx_bufs[i].first == c) {
      g_ctx_bufs[i].second.release();
      g_ctx_bufs.erase(g_ctx_bufs.begin() + i);
      break;
    }
  delete c;
}

// ---------------------------------------------------------------------------
// subroutine-level entry points (stream-ordered temporary allocations)
// ---------------------------------------------------------------------------
namespace {
struct Tmp {
  cudaStream_t st;
  std::vector<void*> v;
  explicit Tmp(cudaStream_t s) : st(s) {}
  template <class T>
  int get(T** p, u64 count) {
    void* x = nullptr;
    cudaError_t e = cudaMallocAsync(&x, (count ? count : 1) * sizeof(T), st);
    if (e != cudaSuccess) return salsaa_set_cuda_error(e, "temporary allocation");
    v.push_back(x);
    *p = (T*)x;
    return 0;
  }
  ~Tmp() {
    for (void* x : v) cudaFreeAsync(x, st);
  }
};
}  // namespace

extern "C" int salsaa_ntt(const uint64_t* d_in, uint64_t* d_out, uint64_t n, uint64_t count, uint64_t q,
                          int inverse, int incomplete, void* stream) {
  if (!d_in || !d_out) return salsaa_set_error(-1, "ntt: null pointer");
  const u64 nn = incomplete ? n / 2 : n;
  if (incomplete && (n < 4 || n % 2)) return salsaa_set_error(-1, "ntt: incomplete mode needs even d >= 4");
  const NttDev* T = ntt_tables((u32)nn, q);
  if (!T || nn > 8192) return salsaa_set_error(-1, "ntt: no NTT for (n, q)");
  return ntt_launch(d_in, d_out, count, *T, incomplete != 0, inverse != 0, (cudaStream_t)stream);
}

extern "C" int salsaa_ntt_multi(const uint64_t* const* d_in, uint64_t* const* d_out, const uint64_t* counts,
                                uint32_t ninst, uint64_t n, uint64_t q, int inverse, int incomplete, void* stream) {
  if (!d_in || !d_out || !counts) return salsaa_set_error(-1, "ntt_multi: null argument");
  const u64 nn = incomplete ? n / 2 : n;
  if (incomplete && (n < 4 || n % 2)) return salsaa_set_error(-1, "ntt_multi: incomplete mode needs even d >= 4");
  const NttDev* T = ntt_tables((u32)nn, q);
  if (!T || nn > 8192) return salsaa_set_error(-1, "ntt_multi: no NTT for (n, q)");
  return ntt_multi_launch(d_in, d_out, counts, ninst, *T, incomplete != 0, inverse != 0, (cudaStream_t)stream);
}

extern "C" int salsaa_poly_mul(const uint64_t* d_a, const uint64_t* d_b, uint64_t* d_r, uint64_t n,
                               uint64_t count, uint64_t q, void* stream) {
  if (!d_a || !d_b || !d_r) return salsaa_set_error(-1, "poly_mul: null pointer");
  const NttDev* T = ntt_tables((u32)n, q);
  if (!T || n > 8192) return salsaa_set_error(-1, "poly_mul: no NTT for (n, q)");
  if (count == 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (ntt_mul_fused_ok(d_a, d_b, d_r, *T)) return ntt_mul_launch(d_a, d_b, d_r, count, *T, st);
  // three passes: NTT(a) -> r, NTT(b) -> tmp, r *= tmp, INTT(r)
  Tmp t(st);
  u64* tb;
  TRY(t.get(&tb, count * n));
  TRY(ntt_launch(d_b, tb, count, *T, false, false, st));
  TRY(ntt_launch(d_a, d_r, count, *T, false, false, st));
  TRY(launch_pointwise_mul(d_r, tb, count * n, q, st));
  return ntt_launch(d_r, d_r, count, *T, false, true, st);
}

extern "C" uint64_t salsaa_fq2_shift(uint64_t q) {
  if (q < 3 || q >= (1ULL << 62) || !(q & 1)) return 0;
  for (u64 s = 2; s < q && s < (1ULL << 20); s++)
    if (host::powmod(s, (q - 1) / 2, q) == q - 1) return s;
  return 0;
}

extern "C" int salsaa_sumcheck_fq2_batch(const uint64_t* const* d_vecs, const uint64_t* lens, uint32_t count,
                                         uint64_t q, uint64_t seed, uint64_t round, uint64_t* d_claims,
                                         uint64_t* d_polys, void* stream) {
  if (!d_vecs || !lens || !d_claims || !d_polys) return salsaa_set_error(-1, "sumcheck_fq2: null argument");
  if (q < 3 || q >= (1ULL << 62)) return salsaa_set_error(-1, "sumcheck_fq2: modulus must be in [3, 2^62)");
  const u64 shift = salsaa_fq2_shift(q);
  if (!shift) return salsaa_set_error(-1, "sumcheck_fq2: no quadratic non-residue found");
  if (count == 0 || count > 64) return salsaa_set_error(-2, "sumcheck_fq2: 1..64 instances");
  u64 words = 0, nrmax = 0;
  for (u32 i = 0; i < count; i++) {
    if (lens[i] < 2 || (lens[i] & (lens[i] - 1)) || lens[i] > (1ULL << 30))
      return salsaa_set_error(-2, "sumcheck_fq2: lengths must be powers of two in 2..2^30");
    words += lens[i] + lens[i] / 2;
    const u64 nr = ilog2u(lens[i]);
    if (nr > nrmax) nrmax = nr;
  }
  cudaStream_t st = (cudaStream_t)stream;
  Tmp t(st);
  u64* scratch;
  TRY(t.get(&scratch, words + (u64)count * nrmax * 6));
  return launch_sumcheck_fq2_batch(d_vecs, lens, count, make_modq(q), shift, seed, (u32)round, d_claims, d_polys,
                                   scratch, st);
}

extern "C" int salsaa_sumcheck_batch(const uint64_t* const* d_vecs, const uint64_t* lens, uint32_t count, uint64_t q,
                                     uint64_t seed, uint64_t round, uint64_t* d_claims, uint64_t* d_polys,
                                     void* stream) {
  if (!d_vecs || !lens || !d_claims || !d_polys) return salsaa_set_error(-1, "sumcheck_batch: null argument");
  if (q < 3 || q >= (1ULL << 62)) return salsaa_set_error(-1, "sumcheck_batch: modulus must be in [3, 2^62)");
  return launch_sumcheck_batch(d_vecs, lens, count, make_modq(q), seed, (u32)round, d_claims, d_polys,
                               (cudaStream_t)stream);
}

extern "C" int salsaa_commit(salsaa_ctx* c, const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t* d_out,
                             void* stream) {
  if (!c || !d_w || !d_out) return salsaa_set_error(-1, "commit: null argument");
  if (rows == 0 || rows > (u64)MAX_WROWS || width == 0 || width > c->L || (width & (width - 1)))
    return salsaa_set_error(-2, "commit: bad witness shape");
  cudaStream_t st = (cudaStream_t)stream;
  const u32 d = c->d, ms = (u32)c->P.module_size;
  Tmp t(st);
  u64 *ws, *acc, *cout;
  DevState* ds;
  TRY(t.get(&ws, rows * width * d));
  TRY(t.get(&acc, (u64)ms * rows * d));
  TRY(t.get(&cout, (u64)ms * rows * d));
  TRY(t.get(&ds, 1));
  TRY(ntt_launch(d_w, ws, rows * width, *c->T, true, false, st));
  CommitArgs a{};
  a.tl8 = c->tl8;
  a.tk8 = c->tk8;
  a.w = rows_of(ws, (u32)rows, width, d);
  a.rows = (u32)rows;
  a.width = width;
  a.nck = ms;
  a.tlo = c->tlo;
  a.thi = c->thi;
  a.ck_bt = c->ck_bt;
  a.ck_nhi = c->ck_nhi;
  a.acc = acc;
  a.out_slot = cout;
  TRY(launch_commit(a, *c->T, c->M, ds, st));
  return ntt_launch(cout, d_out, (u64)ms * rows, *c->T, true, true, st);
}

extern "C" int salsaa_commit_multi(salsaa_ctx* c, const uint64_t* const* d_w, const uint64_t* rows,
                                   const uint64_t* widths, uint32_t ninst, uint64_t* const* d_out, void* stream) {
  if (!c || !d_w || !rows || !widths || !d_out) return salsaa_set_error(-1, "commit_multi: null argument");
  if (ninst == 0 || ninst > CKU_MULTI_MAX) return salsaa_set_error(-2, "commit_multi: 1..8 witnesses per call");
  cudaStream_t st = (cudaStream_t)stream;
  const u32 d = c->d, ms = (u32)c->P.module_size;
  u64 wtot = 0, etot = 0;
  for (u32 i = 0; i < ninst; i++) {
    if (!d_w[i] || !d_out[i]) return salsaa_set_error(-1, "commit_multi: null buffer");
    if (rows[i] == 0 || rows[i] > CKU_MAX_WROWS || widths[i] < 128 || widths[i] > c->L ||
        (widths[i] & (widths[i] - 1)) || (uintptr_t)d_w[i] % 16 || (uintptr_t)d_out[i] % 16)
      return salsaa_set_error(-2, "commit_multi: witness shape or alignment outside the one-launch path");
    wtot += rows[i] * widths[i] * d;
    etot += (u64)ms * rows[i] * d;
  }
  Tmp t(st);
  u64 *ws, *acc, *cout;
  TRY(t.get(&ws, wtot));
  TRY(t.get(&acc, etot));
  TRY(t.get(&cout, etot));
  // every witness to slot form in one launch
  const u64* ins[CKU_MULTI_MAX];
  u64* outs[CKU_MULTI_MAX];
  u64 cnt[CKU_MULTI_MAX];
  CommitArgs a[CKU_MULTI_MAX];
  u64 wo = 0, eo = 0;
  for (u32 i = 0; i < ninst; i++) {
    ins[i] = d_w[i];
    outs[i] = ws + wo;
    cnt[i] = rows[i] * widths[i];
    a[i] = CommitArgs{};
    a[i].tl8 = c->tl8;
    a[i].tk8 = c->tk8;
    a[i].w = rows_of(ws + wo, (u32)rows[i], widths[i], d);
    a[i].rows = (u32)rows[i];
    a[i].width = widths[i];
    a[i].nck = ms;
    a[i].tlo = c->tlo;
    a[i].thi = c->thi;
    a[i].ck_bt = c->ck_bt;
    a[i].ck_nhi = c->ck_nhi;
    a[i].acc = acc + eo;
    wo += cnt[i] * d;
    eo += (u64)ms * rows[i] * d;
  }
  TRY(ntt_multi_launch(ins, outs, cnt, ninst, *c->T, true, false, st));
  cudaError_t e = cudaMemsetAsync(acc, 0, etot * sizeof(u64), st);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "commit_multi: memset");
  // the key rows of every witness in one launch, then one finalisation over
  // all accumulators and one inverse transform into the callers' buffers
  TRY(launch_ck_umma_multi(a, ninst, c->T->n, c->M, c->T->zeta, st));
  TRY(launch_commit_finalize(acc, 1, (u32)(etot / d), *c->T, c->M, cout, st));
  const u64* cin[CKU_MULTI_MAX];
  u64 ecnt[CKU_MULTI_MAX];
  eo = 0;
  for (u32 i = 0; i < ninst; i++) {
    cin[i] = cout + eo;
    ecnt[i] = (u64)ms * rows[i];
    eo += ecnt[i] * d;
  }
  return ntt_multi_launch(cin, d_out, ecnt, ninst, *c->T, true, true, st);
}

extern "C" int salsaa_sumcheck(const uint64_t* d_w, uint64_t rows, uint64_t n, uint64_t d, uint64_t q,
                               uint64_t seed, uint64_t round, uint64_t* d_claims, uint64_t* d_polys,
                               void* stream) {
  if (!d_w || !d_claims || !d_polys) return salsaa_set_error(-1, "sumcheck: null argument");
  if (rows == 0 || rows > (u64)MAX_WROWS || n < 4 || (n & (n - 1)) || d == 0 || n % d)
    return salsaa_set_error(-2, "sumcheck: bad shape");
  if (q < 3 || q >= (1ULL << 62)) return salsaa_set_error(-2, "sumcheck: bad modulus");
  cudaStream_t st = (cudaStream_t)stream;
  Tmp t(st);
  SumcheckBufs B{};
  DevState* ds;
  TRY(t.get(&B.a, rows * n));
  TRY(t.get(&B.b, rows * n / 2));
  TRY(t.get(&B.sums, 2ULL * 64 * rows * 3));
  TRY(t.get(&B.cap, 2ULL * rows * d));
  TRY(t.get(&B.gram, rows * 256 + 1));
  TRY(t.get(&ds, 1));
  set_seed_kernel<<<1, 1, 0, st>>>(ds, seed);
  const u64 nr = ilog2u(n);
  RowSet w = rows_of(d_w, (u32)rows, n / d, (u32)d);
  return launch_sumcheck(w, (u32)rows, n, (u32)d, make_modq(q), ds, (u32)round, B, d_claims, d_polys,
                         d_polys + nr * rows * 3, st);
}

extern "C" int salsaa_decompose(const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q,
                                uint64_t parts, uint64_t* d_out, uint64_t* d_radix, void* stream) {
  if (!d_w || !d_out || !d_radix) return salsaa_set_error(-1, "decompose: null argument");
  if (rows == 0 || rows > (u64)MAX_WROWS || parts == 0 || parts > 64) return salsaa_set_error(-2, "decompose: bad shape");
  cudaStream_t st = (cudaStream_t)stream;
  Tmp t(st);
  DevState* ds;
  TRY(t.get(&ds, 1));
  RowSet w = rows_of(d_w, (u32)rows, width, (u32)d);
  return launch_decompose(w, (u32)rows, width, (u32)d, q, (u32)parts, 0, ds, d_out, d_radix, st);
}

extern "C" int salsaa_project(const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q,
                              uint64_t seed, uint64_t round, uint64_t* d_out, void* stream) {
  if (!d_w || !d_out) return salsaa_set_error(-1, "project: null argument");
  const u64 cw = rows * 256;
  if (rows == 0 || rows > (u64)MAX_WROWS || cw > width || width % cw || cw > CK_BLOCK)
    return salsaa_set_error(-3, "project: chunk width (rows*256) exceeds the witness width");
  cudaStream_t st = (cudaStream_t)stream;
  Tmp t(st);
  DevState* ds;
  u32 *pm, *nm;
  int8_t* J;
  TRY(t.get(&ds, 1));
  TRY(t.get(&pm, 256 * cw / 32));
  TRY(t.get(&nm, 256 * cw / 32));
  TRY(t.get(&J, 256 * cw));
  set_seed_kernel<<<1, 1, 0, st>>>(ds, seed);
  TRY(launch_proj_tables(ds, (u32)round, (u32)cw, pm, nm, J, nullptr, q, st));
  RowSet w = rows_of(d_w, (u32)rows, width, (u32)d);
  return launch_project(w, (u32)rows, width, (u32)d, q, pm, nm, J, ds, d_out, st);
}

extern "C" int salsaa_fold(const uint64_t* d_w, uint64_t rows, uint64_t width, uint64_t d, uint64_t q,
                           const uint64_t* d_c, uint64_t* d_out, void* stream) {
  if (!d_w || !d_c || !d_out) return salsaa_set_error(-1, "fold: null argument");
  if (rows == 0 || rows > (u64)MAX_WROWS || d < 4 || (d & (d - 1))) return salsaa_set_error(-2, "fold: bad shape");
  const NttDev* T = ntt_tables((u32)(d / 2), q);
  if (!T) return salsaa_set_error(-1, "fold: no NTT for (d, q)");
  cudaStream_t st = (cudaStream_t)stream;
  Tmp t(st);
  u64 *ws, *cs, *fs, *pre;
  TRY(t.get(&ws, rows * width * d));
  TRY(t.get(&cs, rows * d));
  TRY(t.get(&fs, width * d));
  TRY(t.get(&pre, rows * (d / 2) * 6));
  TRY(ntt_launch(d_w, ws, rows * width, *T, true, false, st));
  TRY(ntt_launch(d_c, cs, rows, *T, true, false, st));
  TRY(launch_fold(rows_of(ws, (u32)rows, width, (u32)d), (u32)rows, width, *T, make_modq(q), cs, pre, fs, st));
  return ntt_launch(fs, d_out, width, *T, true, true, st);
}
