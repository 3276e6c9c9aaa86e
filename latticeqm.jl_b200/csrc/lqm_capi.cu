// C ABI of libkspace (declared in include/kspace.h).  Host side: argument
// validation, device buffers, the k-batch loop and kernel launches.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "kspace.h"
#include "lqm_kernels.cuh"
#include "lqm_large.cuh"
#include "lqm_hf.cuh"
#include "lqm_zgemm.cuh"
#include "lqm_plan.h"

using namespace lqm;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct PlanDev {
  int n = 0;
  int* d_buf = nullptr;
  DCPlan plan{};
};

struct LqmError {
  int code;
  std::string msg;
};

}  // namespace

struct lqm_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  double timeout_s = 600.0;
  int num_sms = 0;
  double last_ms = 0.0;
  std::map<int, PlanDev> plans;
  std::map<int, int> eigh_nt;  // one-CTA eigensolver block size per order n (autotuned or set), else the rule
  DevBuf ws[52];
  // per-kernel device-time statistics (CUDA events on the context stream)
  bool stats_on = false;
  bool phases_on = false;  // per-phase cycle counters inside the eigensolver (clock reads)
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pending, ev_pool;
  double eigh_ms = 0.0;
  int64_t eigh_launches = 0, launches = 0;
  // the blocked path's mat-vec kernel (the dominant kernel of a large-n pass), timed per launch
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> symv_pending;
  double symv_ms = 0.0, symv_bytes = 0.0;
  // the two-stage path's stage-2 back-transformation (its dominant kernel with vectors), timed per launch
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> q2_pending;
  double q2_ms = 0.0, q2_flops = 0.0;
  int64_t q2_launches = 0;
  int64_t symv_launches = 0;
  unsigned long long* d_phase = nullptr;  // per-phase cycle counters (profiling)
  bool scf_graph_used = false;            // the last SCF replayed a captured iteration
  int64_t blocked_min_n = 0;              // n >= this uses the blocked path (0: the default switch)
  int two_stage = -1;                     // blocked path reduction: 1 two-stage, 0 one-stage, -1 by order
  // autotuned reduction per (order, pass kind): key 2 n + (pass returns all eigenvectors)
  std::map<int, int> two_stage_tuned;
  int scf_anderson_depth = 0;             // SCF acceleration: 0 linear mixing, > 0 Anderson history depth
  int scf_residual = 0;                   // SCF residual: 0 relative density change, 1 commutator norm
  bool scf_hartree = true, scf_fock = true;  // HartreeFock(h, v; hartree, fock)
  // ExchangeKernel(j, siteof, flavorof) of the next SCF calls (ns == 0: none)
  int64_t ex_ns = 0, ex_nf = 0, ex_nJ = 0;
  int ex_d = 0;
  std::vector<int64_t> ex_keys;   // d x nJ
  std::vector<double> ex_blocks;  // ns x ns x nJ complex (interleaved)
  std::vector<int> ex_sf2idx;     // ns x nf, column-major: (site a, flavor f) -> orbital
  double scf_eJ = 0.0;            // exchange energy of the last SCF
  // device buffers of freed Hops kept for the next uploads (base pointer, bytes):
  // a caller that uploads H, runs one pass and frees it every call then makes no
  // cudaMalloc/cudaFree, whose device-wide synchronisation and driver work cost
  // from milliseconds to most of a second per call on B200
  std::vector<std::pair<void*, size_t>> hops_cache;
  size_t hops_cache_bytes = 0;
  // device error word set by kernels whose waits are bounded (the TMA mat-vec);
  // wait_stream reads it once such a kernel has been launched since the last check
  int* d_err = nullptr;
  bool err_armed = false;
  int64_t dev_wait_limit = 0;  // polls before a device-side wait of the bulge chase gives up (0: the default)
  // NCCL communicator of the k-point shards (lqm_ctx_set_comm; lqm_comm.inc)
  void* comm = nullptr;
  int comm_nranks = 1, comm_rank = 0;
};

struct lqm_hops {
  int64_t n = 0, nR = 0;
  int32_t d = 0;
  double2* blocks = nullptr;  // base of one device buffer: the blocks, then (256-byte aligned) the keys
  int64_t* keys = nullptr;
  std::vector<int64_t> hkeys;
  int device = -1;            // device of the buffer
  size_t buf_bytes = 0;       // its size
};

namespace {

[[noreturn]] void fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw LqmError{code, buf};
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation) fail(LQM_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
    fail(LQM_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  }
}

template <class F>
int guarded(lqm_ctx* ctx, F&& f) {
  if (!ctx) return LQM_EINVAL;
  try {
    ctx->err.clear();
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    f();
    return LQM_OK;
  } catch (const LqmError& e) {
    ctx->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    ctx->err = "host allocation failed";
    return LQM_ENOMEM;
  } catch (...) {
    ctx->err = "unknown error";
    return LQM_EINVAL;
  }
}

// A named NVTX range for the lifetime of a scope, so that the stages of a call
// (eigen pass, fold, DOS, SCF iteration) show on a profiler's timeline.  NVTX
// calls do nothing unless a profiling tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

void collect_stats(lqm_ctx* ctx) {
  for (auto& pr : ctx->ev_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) ctx->eigh_ms += ms;
    ctx->ev_pool.push_back(pr);
  }
  ctx->ev_pending.clear();
  for (auto& pr : ctx->symv_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) ctx->symv_ms += ms;
    ctx->ev_pool.push_back(pr);
  }
  ctx->symv_pending.clear();
  for (auto& pr : ctx->q2_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) ctx->q2_ms += ms;
    ctx->ev_pool.push_back(pr);
  }
  ctx->q2_pending.clear();
}

void wait_stream(lqm_ctx* ctx) {
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(ctx->stream);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) ck(e, "device execution");
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > ctx->timeout_s) fail(LQM_ETIMEOUT, "device work exceeded the %.1f s timeout", ctx->timeout_s);
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  ck(cudaGetLastError(), "kernel launch");
  collect_stats(ctx);
  if (ctx->err_armed && ctx->d_err) {
    ctx->err_armed = false;
    int e = 0;
    ck(cudaMemcpy(&e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost), "error word");
    if (e != 0) {
      ck(cudaMemset(ctx->d_err, 0, sizeof(int)), "error word");
      fail(LQM_EDEVICE, "a device-side wait gave up (a TMA copy or a bulge-chase dependency not complete within its limit)");
    }
  }
}

std::pair<cudaEvent_t, cudaEvent_t> stat_events(lqm_ctx* ctx) {
  if (!ctx->ev_pool.empty()) {
    auto pr = ctx->ev_pool.back();
    ctx->ev_pool.pop_back();
    return pr;
  }
  std::pair<cudaEvent_t, cudaEvent_t> pr;
  ck(cudaEventCreate(&pr.first), "event");
  ck(cudaEventCreate(&pr.second), "event");
  return pr;
}

void* ws_get(lqm_ctx* ctx, int slot, size_t bytes) {
  DevBuf& b = ctx->ws[slot];
  if (b.bytes < bytes) {
    if (b.p) { wait_stream(ctx); cudaFree(b.p); b.p = nullptr; b.bytes = 0; }
    size_t want = std::max(bytes, (size_t)256);
    ck(cudaMalloc(&b.p, want), "cudaMalloc(workspace)");
    b.bytes = want;
  }
  return b.p;
}

// Cache of freed Hops buffers (lqm_ctx::hops_cache): at most kHopsCacheCount
// buffers and kHopsCacheBytes in total.  A buffer serves a request of `need`
// bytes when it is at least that large and at most twice that plus 1 MiB, so a
// small H does not pin a large buffer.
constexpr size_t kHopsCacheBytes = size_t(1) << 30;
constexpr size_t kHopsCacheCount = 16;

void* hops_buffer_take(lqm_ctx* ctx, size_t need, size_t* got) {
  size_t best = ctx->hops_cache.size();
  for (size_t i = 0; i < ctx->hops_cache.size(); ++i) {
    const size_t b = ctx->hops_cache[i].second;
    if (b >= need && b <= 2 * need + (size_t(1) << 20) &&
        (best == ctx->hops_cache.size() || b < ctx->hops_cache[best].second))
      best = i;
  }
  if (best == ctx->hops_cache.size()) return nullptr;
  void* p = ctx->hops_cache[best].first;
  *got = ctx->hops_cache[best].second;
  ctx->hops_cache_bytes -= *got;
  ctx->hops_cache.erase(ctx->hops_cache.begin() + (std::ptrdiff_t)best);
  return p;
}

// Keeps a freed buffer if the cache has room (true), else the caller frees it.
bool hops_buffer_keep(lqm_ctx* ctx, void* p, size_t bytes) {
  if (!p || bytes == 0 || ctx->hops_cache.size() >= kHopsCacheCount ||
      ctx->hops_cache_bytes + bytes > kHopsCacheBytes)
    return false;
  ctx->hops_cache.emplace_back(p, bytes);
  ctx->hops_cache_bytes += bytes;
  return true;
}

enum WsSlot {
  WS_SCRATCH = 0, WS_KS, WS_BANDS, WS_U, WS_RHOK, WS_COEF, WS_EBK, WS_RHO, WS_W, WS_MISC, WS_PART,
  WS_OMEGA, WS_DOS, WS_LKEYS, WS_HF, WS_HF2, WS_MU, WS_BANDS2,
  WS_LA, WS_LU, WS_LAUX, WS_LDC, WS_VU, WS_VB, WS_VX, WS_VT, WS_VG, WS_ONES, WS_SCFY, WS_AND, WS_EXCH, WS_HFPART, WS_BDG, WS_BDGE, WS_BDGI, WS_BDGK, WS_BDGP, WS_BDGB, WS_CSC, WS_UNIW, WS_SPAN, WS_GRAD, WS_GRADE, WS_HFPART2, WS_GEMMSPLIT, WS_GRAM, WS_TSP, WS_TSB, WS_TSV2
};
static_assert(WS_TSV2 < 52, "workspace slots");

}  // namespace
#include "lqm_comm.inc"
namespace {

// ---- divide-and-conquer plan (lqm_plan.h), uploaded once per order n ----
const DCPlan& get_plan(lqm_ctx* ctx, int n) {
  auto it = ctx->plans.find(n);
  if (it != ctx->plans.end()) return it->second.plan;
  const DCPlanHost P = make_dc_plan_host(n);
  PlanDev pd;
  pd.n = n;
  ck(cudaMalloc(&pd.d_buf, P.buf.size() * sizeof(int)), "cudaMalloc(plan)");
  ck(cudaMemcpy(pd.d_buf, P.buf.data(), P.buf.size() * sizeof(int), cudaMemcpyHostToDevice), "plan upload");
  pd.plan.nnodes = P.nnodes;
  pd.plan.nheights = P.nheights;
  pd.plan.hstart = pd.d_buf + P.off_hstart;
  pd.plan.lo = pd.d_buf + P.off_lo;
  pd.plan.mid = pd.d_buf + P.off_mid;
  pd.plan.hi = pd.d_buf + P.off_hi;
  pd.plan.owner = pd.d_buf + P.off_own;
  return ctx->plans.emplace(n, pd).first->second.plan;
}

void check_finite(const double* x, int64_t m, const char* what) {
  for (int64_t i = 0; i < m; ++i)
    if (!std::isfinite(x[i])) fail(LQM_EINVAL, "%s contains a non-finite value at index %lld", what, (long long)i);
}

void check_hops(const lqm_hops* H) {
  if (!H || !H->blocks) fail(LQM_EINVAL, "null hops");
}

// Threads of the one-CTA eigensolver for n >= 64 (a compile-time choice; 384
// measured fastest at n = 96 on B200: 168 registers per thread instead of the
// 128 that 512 threads allow).
#ifndef LQM_EIGH_NT_LARGE
#define LQM_EIGH_NT_LARGE 384
#endif
int eigh_threads(int n) { return n <= 16 ? 32 : (n <= 32 ? 64 : (n < 64 ? 128 : LQM_EIGH_NT_LARGE)); }
// The block size of the one-CTA eigensolver for order n on this context: the value
// set by lqm_ctx_set_eigh_threads / lqm_autotune_eigh, else the rule above.
int eigh_threads_for(const lqm_ctx* ctx, int n) {
  const auto it = ctx->eigh_nt.find(n);
  return it != ctx->eigh_nt.end() ? it->second : eigh_threads(n);
}

// eigh_kernel instantiation for a block size.  Blocks of up to 128 threads
// (small n, where shared memory leaves room for many CTAs per SM) take
// instantiations whose launch bounds cap the registers per thread so that
// more CTAs share an SM than the 254 registers of the 256-thread
// instantiation allow.  Measured on B200 (rho pass, 65 536 k):
//   32 threads, 128 registers (16 CTAs/SM instead of 8): n = 8 10.7 -> 8.7 ms;
//   64 threads, 168 registers (6 instead of 4): n = 24 41.1 -> 37.0 ms
//     (128 registers, 8 CTAs, spilled: 41.7 ms);
//   128 threads, 128 registers (4 instead of 2): n = 24 53.6 -> 43.7 ms.
using EighFn = void (*)(EighArgs);
EighFn eigh_fn(int nt) {
  if (nt <= 32) return &eigh_kernel<32, 16>;
  if (nt <= 64) return &eigh_kernel<64, 6>;
  if (nt <= 128) return &eigh_kernel<128, 4>;
  return nt > 384 ? &eigh_kernel<512> : (nt > 256 ? &eigh_kernel<384> : &eigh_kernel<256>);
}

void timer_start(lqm_ctx* ctx) { ck(cudaEventRecord(ctx->ev0, ctx->stream), "event"); }
void timer_stop(lqm_ctx* ctx) {
  ck(cudaEventRecord(ctx->ev1, ctx->stream), "event");
}
void timer_collect(lqm_ctx* ctx) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->last_ms = ms;
}

// Fused density output of the eigen pass: rho_k = U f(eps - mu) U^H and w_k sum f eps.
struct RhoOut {
  double2* rhok;
  double* ebk;
  const double* w;
  double mu, T;
};

// ---- blocked large-n path (lqm_large.cuh) ----
// The library's batched GEMMs run on the context's stream (and its workspace).
lqm_ctx* blas_handle(lqm_ctx* ctx) { return ctx; }

template <int BM, int BN, int WM, int WN, int BK, int ST>
void launch_zgemm_dmma(cudaStream_t st, const GemmArgs& g, int batch) {
  constexpr int nt = (BM / WM) * (BN / WN) * 32;
  constexpr int smem = zgemm_smem_bytes<BM, BN, BK, ST>();
  static std::atomic<unsigned long long> attr_done{0};  // devices on which the smem limit is raised
  int dev = 0;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attr_done.load() & bit)) {
    ck(cudaFuncSetAttribute(zgemm_dmma_kernel<BM, BN, WM, WN, BK, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            smem),
       "smem attr");
    attr_done.fetch_or(bit);
  }
  const dim3 grid((unsigned)((g.m + BM - 1) / BM), (unsigned)((g.n + BN - 1) / BN), (unsigned)batch);
  zgemm_dmma_kernel<BM, BN, WM, WN, BK, ST><<<grid, nt, smem, st>>>(g);
}

// C_b = alpha op(A_b) op(B_b) + beta C_b for b < batch (column-major, strided):
// the library's DMMA kernel (lqm_zgemm.cuh), with the tile shape chosen by the
// product's shape (skinny n: the Fourier fold; small m: the back-transformation's
// panel products; short k: the rank-2nb updates).
void zgemm_sb(lqm_ctx* ctx, GemmOp ta, GemmOp tb, int m, int n, int k, double alpha_re, const double2* A, int lda,
              long long sA, const double2* B, int ldb, long long sB, double beta_re, double2* C, int ldc, long long sC,
              int batch) {
  if (m <= 0 || n <= 0 || batch <= 0) return;
  if (batch > 65535) fail(LQM_EINVAL, "GEMM batch %d exceeds the grid limit", batch);
  cudaStream_t h = ctx->stream;
  GemmArgs g{m, n, k, alpha_re, beta_re, A, lda, sA, B, ldb, sB, C, ldc, sC, (int)ta, (int)tb, 0, k};
  // a single product with few output tiles and a long k (the Fourier fold of small
  // orders): split k over the SMs, partial products in a workspace, then an ordered sum
  const int64_t tiles = (int64_t)((m + 127) / 128) * ((n + 15) / 16);
  if (batch == 1 && n <= 16 && k >= 1024 && ta != OP_HL && tiles < 2 * (int64_t)ctx->num_sms) {
    int nsplit = (int)std::min<int64_t>((2 * ctx->num_sms + tiles - 1) / tiles, k / 512);
    nsplit = std::max(2, std::min(nsplit, 64));
    const int kc = (k + nsplit - 1) / nsplit;
    nsplit = (k + kc - 1) / kc;
    double2* P = (double2*)ws_get(ctx, WS_GEMMSPLIT, (size_t)nsplit * m * n * sizeof(double2));
    GemmArgs gs = g;
    gs.beta = 0.0; gs.C = P; gs.ldc = m; gs.sC = (long long)m * n; gs.split = nsplit; gs.k = kc; gs.ktot = k;
    launch_zgemm_dmma<128, 16, 32, 16, 8, 3>(h, gs, nsplit);
    const int64_t mn = (int64_t)m * n;
    zgemm_split_reduce_kernel<<<(unsigned)std::min<int64_t>((mn + 255) / 256, 8 * ctx->num_sms), 256, 0, h>>>(
        m, n, nsplit, P, beta_re, C, ldc, 0, 1);
    ck(cudaGetLastError(), "zgemm split launch");
    return;
  }
  // batched products with a tiny output and a long k (V^H X of the two-stage panels):
  // k in chunks of 128 on 16 x 16 tiles of one warp, then the ordered sum per entry
  if (m <= 16 && n <= 16 && k >= 512 && ta != OP_HL) {
    const int kc = 128;
    const int nsplit = std::min((k + kc - 1) / kc, 65535 / batch);
    if (nsplit >= 2) {
      const int kcs = (k + nsplit - 1) / nsplit;
      const int ns = (k + kcs - 1) / kcs;
      double2* P = (double2*)ws_get(ctx, WS_GEMMSPLIT, (size_t)batch * ns * m * n * sizeof(double2));
      GemmArgs gs = g;
      gs.beta = 0.0; gs.C = P; gs.ldc = m; gs.sC = (long long)m * n; gs.split = ns; gs.k = kcs; gs.ktot = k;
      launch_zgemm_dmma<16, 16, 16, 16, 8, 3>(h, gs, batch * ns);
      const int64_t tot = (int64_t)m * n * batch;
      zgemm_split_reduce_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, 8 * ctx->num_sms), 256, 0, h>>>(
          m, n, ns, P, beta_re, C, ldc, sC, batch);
      ck(cudaGetLastError(), "zgemm split launch");
      return;
    }
  }
  if (n <= 16 && m >= 512)
    launch_zgemm_dmma<128, 16, 16, 16, 8, 3>(h, g, batch);  // eight warps per tile: tall skinny products
  else if (n <= 16)
    launch_zgemm_dmma<128, 16, 32, 16, 8, 3>(h, g, batch);
  else if (m <= 32)
    launch_zgemm_dmma<32, 64, 32, 16, 8, 3>(h, g, batch);
  else if (k <= 64)
    launch_zgemm_dmma<64, 64, 32, 16, 8, 3>(h, g, batch);
  else
    launch_zgemm_dmma<64, 64, 32, 32, 8, 3>(h, g, batch);
  ck(cudaGetLastError(), "zgemm launch");
}

// Hermitian rank-2k update of the lower triangle of a batch of m x m blocks:
//   C_b -= X_b Y_b^H + Y_b X_b^H  (X, Y: m x k, column-major, strided),
// one launch, both products summed in one k-loop (C read and written once), tiles
// entirely above the diagonal skipped.  The upper triangle's tiles that straddle the
// diagonal are written too (it is never read).
void zher2k_lower(lqm_ctx* ctx, int m, int k, const double2* X, int ldx, long long sX, const double2* Y, int ldy,
                  long long sY, double2* C, int ldc, long long sC, int batch) {
  if (m <= 0 || k <= 0 || batch <= 0) return;
  if (batch > 65535) fail(LQM_EINVAL, "GEMM batch %d exceeds the grid limit", batch);
  GemmArgs g{m, m, k, -1.0, 1.0, X, ldx, sX, Y, ldy, sY, C, ldc, sC, (int)OP_N, (int)OP_C, 0, k,
             Y, ldy, sY, X, ldx, sX, k, 1};
  launch_zgemm_dmma<64, 64, 32, 16, 8, 3>(ctx->stream, g, batch);
  ck(cudaGetLastError(), "zher2k launch");
}

struct RhoOut;
bool use_blocked(const lqm_ctx* ctx, int n, int nR);
bool use_two_stage(const lqm_ctx* ctx, int n, bool all_vectors);

// Eigen pass of the blocked path: same outputs as launch_eigh.  Reduction by
// zlatrd panels (column kernels + batched rank-2nb updates), divide and
// conquer per k, compact-WY back-transformation and rho_k = U f U^H as batched
// GEMMs.  k-points are processed in batches sized to ~24 GB of work buffers.
// TMA descriptors of a batch of B matrices (n x n complex, column-major, contiguous):
// 3-D (2n doubles, n columns, B k-points), zero fill out of bounds; `map` boxes of 16
// doubles (8 complex rows) x 64 columns x 1 with 128-byte swizzle (the tiles),
// `vmap` boxes of 128 doubles x 1 column x 1 (the reflector segments).  cuTensorMapEncodeTiled is
// taken from the driver through the runtime (no link-time libcuda dependency).
bool make_symv_map(CUtensorMap* map, CUtensorMap* vmap, const double2* A, int n, int64_t B) {
  static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    cudaGetLastError();
  });
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)(2 * n), (cuuint64_t)n, (cuuint64_t)B};
  const cuuint64_t strides[2] = {(cuuint64_t)n * 16, (cuuint64_t)n * n * 16};
  const cuuint32_t box[3] = {16, (cuuint32_t)kSymvTB, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  if (enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)A, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
      CUDA_SUCCESS)
    return false;
  // the reflector segments: 64 complex rows of one column, no swizzle
  const cuuint32_t vbox[3] = {2 * (cuuint32_t)kSymvTB, 1, 1};
  return enc(vmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)A, dims, strides, vbox, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void launch_eigh_large(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, double* d_bands,
                       double2* d_U, double2* rhok, double* ebk, const double* w, double mu, double T) {
  NvtxRange nvtx_("eigen pass (blocked)");
  const int n = (int)H->n;
  const int nb = kBlkNB;
  const int P = (n + nb - 1) / nb;
  const int nbt = kBlkNBT;                // back-transformation panels
  const int P2 = (n + nbt - 1) / nbt;
  const int wc = std::max(nb, nbt);       // columns of W / X and of Y per k-point
  const bool vec = d_U || rhok;
  // two-stage: dense -> band (kTsB) -> tridiagonal; reflector j of the first stage
  // starts at row j + off, n - off of them
  const bool ts = use_two_stage(ctx, n, d_U != nullptr);
  const int off = ts ? kTsB : 1;
  const int NR = n - off;
  const int64_t nn = (int64_t)n * n;
  const int64_t pstride = ts ? 0 : symv_part_stride(n), tstride = ts ? 0 : t12_part_stride(n, nb);
  const int64_t auxk = 2 * (int64_t)n * wc /*W, Y*/ + (int64_t)nbt * nbt * P2 /*Tm*/ + n /*tau*/ + 2 * nb /*t12*/ +
                       pstride /*mat-vec partials*/ + tstride /*panel-product partials*/;
  const int64_t tspk = ts ? 3 * (int64_t)n * kTsB + 3 * kTsB * kTsB : 0;   // Vb, Y, X; T, S, Z
  const int64_t tsbk = ts ? 2 * (int64_t)kTsB * n : 0;                        // the band
  const int64_t tsvk = (ts && vec) ? ts_v2_stride(n) + ts_tau2_stride(n) : 0; // stage-2 reflectors
  const double per_k = 16.0 * (double)nn * ((vec && !d_U) ? 2.0 : 1.0) + 16.0 * (double)(auxk + tspk + tsbk + tsvk) +
                       16.0 * n;
  int64_t B = std::max<int64_t>(1, std::min<int64_t>(nk, (int64_t)(64.0e9 / per_k)));
  B = std::min<int64_t>(B, 65535);
  {  // batches of equal size (no short tail batch)
    const int64_t nbat = (nk + B - 1) / B;
    B = (nk + nbat - 1) / nbat;
  }
  const int64_t slotd = dc_large_slot_doubles(n, vec);
  const bool dc_small = n < kDcTileMin;  // no tiled merges: 128-thread CTAs, four per SM
  const int64_t G = std::min<int64_t>(B, (int64_t)ctx->num_sms * (dc_small ? 4 : 1));
  double2* A = (double2*)ws_get(ctx, WS_LA, (size_t)B * nn * sizeof(double2));
  double2* Uw = (vec && !d_U) ? (double2*)ws_get(ctx, WS_LU, (size_t)B * nn * sizeof(double2)) : nullptr;
  double2* aux = (double2*)ws_get(ctx, WS_LAUX, (size_t)B * (auxk + n) * sizeof(double2));
  double2* W = aux;                                   // B x (n x nb); reused as X (nbt x n) in the back-transform
  double2* Yb = W + B * (int64_t)n * wc;              // B x (nbt x n)
  double2* Tm = Yb + B * (int64_t)n * wc;             // B x P2 x (nbt x nbt)
  double2* tau = Tm + B * (int64_t)nbt * nbt * P2;    // B x n
  double2* t12 = tau + B * (int64_t)n;                // B x 2nb
  double2* part = t12 + B * 2 * (int64_t)nb;          // B x pstride
  double2* tpart = part + B * pstride;                // B x tstride
  double* dd = (double*)(tpart + B * tstride);        // B x n
  double* ee = dd + B * (int64_t)n;                   // B x n
  double2* tsp = ts ? (double2*)ws_get(ctx, WS_TSP, (size_t)B * tspk * sizeof(double2)) : nullptr;
  double2* Bd = ts ? (double2*)ws_get(ctx, WS_TSB, (size_t)B * tsbk * sizeof(double2)) : nullptr;
  double2* V2 = (ts && vec) ? (double2*)ws_get(ctx, WS_TSV2, (size_t)B * tsvk * sizeof(double2)) : nullptr;
  double2* tau2 = V2 ? V2 + B * ts_v2_stride(n) : nullptr;
  double* slots = (double*)ws_get(ctx, WS_LDC, (size_t)G * slotd * sizeof(double));
  const DCPlan& plan = get_plan(ctx, n);
  lqm_ctx* h = blas_handle(ctx);
  CUtensorMap symv_map, symv_vmap;
  bool symv_tma = false;
  if (!ts) {
    ck(cudaFuncSetAttribute(blk_symv_pipe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSymvPipeSmem),
       "smem attr");
    ck(cudaFuncSetAttribute(blk_symv_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSymvTmaSmem),
       "smem attr");
    // the mat-vec moves its tiles by TMA from n = 64 on (the descriptor covers the batch)
    const char* pipe_env = std::getenv("LQM_SYMV_PIPE");
    symv_tma = n >= 64 && !(pipe_env && pipe_env[0] == '1') && make_symv_map(&symv_map, &symv_vmap, A, n, B);
  }
  if ((symv_tma || ts) && !ctx->d_err) {
    ck(cudaMalloc(&ctx->d_err, sizeof(int)), "cudaMalloc(error word)");
    ck(cudaMemset(ctx->d_err, 0, sizeof(int)), "memset(error word)");
  }
  ck(cudaFuncSetAttribute(dc_large_kernel<kDcThreads, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          dc_tile_smem(n)),
     "smem attr");
  std::pair<cudaEvent_t, cudaEvent_t> evs{};
  if (ctx->stats_on) { evs = stat_events(ctx); ck(cudaEventRecord(evs.first, ctx->stream), "event"); }
  for (int64_t k0 = 0; k0 < nk; k0 += B) {
    const int nbk = (int)std::min<int64_t>(B, nk - k0);
    const size_t bsm = (size_t)H->nR * sizeof(double2) + (size_t)H->d * sizeof(double) + 16;
    blk_bloch_kernel<<<nbk, kBlkThreads, bsm, ctx->stream>>>(n, (int)H->nR, H->d, H->blocks, H->keys, nbk,
                                                              d_ks + k0 * H->d, A);
    ctx->launches++;
    if (ts) {
      // stage 1: per panel the QR below the band, then A22 <- Q^H A22 Q by GEMMs
      double2* Vb = tsp;                              // nbk x (n x kTsB)
      double2* Yt = Vb + B * (int64_t)n * kTsB;
      double2* Xt = Yt + B * (int64_t)n * kTsB;
      double2* Tt = Xt + B * (int64_t)n * kTsB;       // nbk x (kTsB x kTsB): T, S, Z
      double2* St = Tt + B * (int64_t)kTsB * kTsB;
      double2* Zt = St + B * (int64_t)kTsB * kTsB;
      const long long sv = (long long)n * kTsB, s2 = (long long)kTsB * kTsB;
      for (int j0 = 0; j0 + kTsB < n; j0 += kTsB) {
        const int m = n - j0 - kTsB, nr = std::min(kTsB, m);
        ts_panel_kernel<<<nbk, kTsPanelThreads, 0, ctx->stream>>>(n, j0, A, tau, Vb, Tt);
        double2* A22 = A + (j0 + kTsB) + (int64_t)(j0 + kTsB) * n;
        zgemm_sb(h, OP_HL, OP_N, m, nr, m, 1.0, A22, n, nn, Vb, n, sv, 0.0, Yt, n, sv, nbk);           // Y = A22 V
        zgemm_sb(h, OP_N, OP_N, m, nr, nr, 1.0, Yt, n, sv, Tt, kTsB, s2, 0.0, Xt, n, sv, nbk);         // X = Y T
        zgemm_sb(h, OP_C, OP_N, nr, nr, m, 1.0, Vb, n, sv, Xt, n, sv, 0.0, St, kTsB, s2, nbk);         // S = V^H X
        zgemm_sb(h, OP_C, OP_N, nr, nr, nr, 0.5, Tt, kTsB, s2, St, kTsB, s2, 0.0, Zt, kTsB, s2, nbk);  // Z = T^H S / 2
        zgemm_sb(h, OP_N, OP_N, m, nr, nr, -1.0, Vb, n, sv, Zt, kTsB, s2, 1.0, Xt, n, sv, nbk);        // W = X - V Z
        zher2k_lower(h, m, nr, Vb, n, sv, Xt, n, sv, A22, n, nn, nbk);                                 // A22 -= V W^H + W V^H
        ctx->launches += 7;
      }
      // stage 2: the band, then the bulge chase to the real tridiagonal
      ts_band_kernel<<<nbk, kBlkThreads, 0, ctx->stream>>>(n, A, Bd);
      ck(cudaFuncSetAttribute(ts_chase_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTsChaseSmem),
         "smem attr");
      ts_chase_kernel<<<nbk, kTsChaseWarps * 32, kTsChaseSmem, ctx->stream>>>(
          n, Bd, V2, tau2, dd, ee, ctx->d_err, ctx->dev_wait_limit > 0 ? ctx->dev_wait_limit : kTsWaitPolls);
      ctx->err_armed = true;
      ctx->launches += 2;
    } else {
      const BlkArgs ba{n, nb, A, W, tau, dd, ee, t12, part, pstride, tpart, tstride};
      for (int p = 0; p < P; ++p) {
        const int j0 = p * nb;
        const int nbp = std::min(nb, n - j0);
        for (int i = 0; i < nbp; ++i) {
          const int j = j0 + i;
          blk_column_kernel<<<nbk, kColThreads, 0, ctx->stream>>>(ba, j0, i);
          ctx->launches++;
          if (j <= n - 2) {
            const int64_t nbl = (n - j - 1 + kSymvTB - 1) / kSymvTB;
            const int64_t nitems = nbl * (nbl + 1) / 2 * nbk;
            const int64_t grid = std::min<int64_t>(nitems, (int64_t)ctx->num_sms);
            std::pair<cudaEvent_t, cudaEvent_t> sev{};
            if (ctx->stats_on) { sev = stat_events(ctx); ck(cudaEventRecord(sev.first, ctx->stream), "event"); }
            if (symv_tma) {
              blk_symv_tma_kernel<<<(unsigned)grid, kSymvTmaThreads, kSymvTmaSmem, ctx->stream>>>(
                  symv_map, symv_vmap, ba, j, nitems, ctx->d_err);
              ctx->err_armed = true;
            } else {
              blk_symv_pipe_kernel<<<(unsigned)grid, kSymvThreads, kSymvPipeSmem, ctx->stream>>>(ba, j, nitems);
            }
            ctx->launches++;
            if (ctx->stats_on) {
              ck(cudaEventRecord(sev.second, ctx->stream), "event");
              ctx->symv_pending.push_back(sev);
              const double m = (double)(n - j - 1);
              ctx->symv_bytes += (double)nbk * m * (m + 1.0) / 2.0 * 16.0;  // lower triangle of A22, once
              ctx->symv_launches++;
            }
            if (i > 0) {
              const dim3 g2((unsigned)((n - j - 1 + 127) / 128), (unsigned)nbk);
              blk_t12_kernel<<<g2, kBlkThreads, 0, ctx->stream>>>(ba, j0, i);
              ctx->launches++;
            }
          }
        }
        if (j0 + nbp < n) {
          blk_finish_kernel<<<nbk, kColThreads, 0, ctx->stream>>>(ba, j0, nbp - 1);
          ctx->launches++;
          // A22 -= V W^H + W V^H on the lower triangle, one launch
          const int m2 = n - j0 - nbp;
          double2* Cb = A + (j0 + nbp) + (int64_t)(j0 + nbp) * n;
          const double2* Vr = A + (j0 + nbp) + (int64_t)j0 * n;
          const double2* Wr = W + (j0 + nbp);
          zher2k_lower(h, m2, nbp, Vr, n, nn, Wr, n, (long long)n * nb, Cb, n, nn, nbk);
          ctx->launches += 1;
        }
      }
    }
    ck(cudaGetLastError(), "blocked reduction launch");
    double2* Ucur = d_U ? d_U + k0 * nn : Uw;
    DCLargeArgs da;
    da.n = n; da.nk = nbk; da.plan = plan; da.d = dd; da.e = ee; da.bands = d_bands + k0 * n;
    da.U = vec ? Ucur : nullptr; da.slots = slots; da.slot_doubles = slotd;
    da.phase_cycles = ctx->phases_on ? ctx->d_phase : nullptr;
    if (dc_small)
      dc_large_kernel<128, 4><<<(unsigned)std::min<int64_t>(G, nbk), 128, 0, ctx->stream>>>(da);
    else
      dc_large_kernel<kDcThreads, 1><<<(unsigned)std::min<int64_t>(G, nbk), kDcThreads, dc_tile_smem(n), ctx->stream>>>(da);
    ctx->launches++;
    ck(cudaGetLastError(), "divide-and-conquer launch");
    if (!vec) continue;
    // When only rho_k is wanted, the back-transformation forms just the columns of U
    // that carry it: the states that are not exactly empty (rho_k = U_K f U_K^H) or,
    // when fewer, those that are not exactly filled (rho_k = I - U_K (1 - f) U_K^H),
    // K = the largest such count over the batch (a host read of two integers).
    int c0 = 0, K = n;
    bool complement = false;
    if (rhok && !d_U) {
      int* span = (int*)ws_get(ctx, WS_SPAN, 2 * sizeof(int));
      ck(cudaMemsetAsync(span, 0, 2 * sizeof(int), ctx->stream), "memset");
      blk_occ_span_kernel<<<nbk, kBlkThreads, 0, ctx->stream>>>(n, d_bands + k0 * n, mu, T, span);
      ctx->launches++;
      int hspan[2] = {n, n};
      ck(cudaMemcpyAsync(hspan, span, sizeof(hspan), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
      wait_stream(ctx);
      if (hspan[0] < hspan[1]) {
        complement = true;
        K = hspan[0];
        c0 = n - K;
      } else {
        K = hspan[1];
      }
    }
    if (K > 0 && ts) {
      // Z <- Q2 Z on the K columns: the stage-2 reflectors in groups of 16 sweeps,
      // a register window of each column per thread
      std::pair<cudaEvent_t, cudaEvent_t> qev{};
      if (ctx->stats_on) { qev = stat_events(ctx); ck(cudaEventRecord(qev.first, ctx->stream), "event"); }
      ts_q2g_kernel<<<dim3((unsigned)((K + kTsQ2gThreads - 1) / kTsQ2gThreads), (unsigned)nbk), kTsQ2gThreads, 0,
                      ctx->stream>>>(n, c0, K, V2, tau2, Ucur);
      ctx->launches++;
      if (ctx->stats_on) {
        ck(cudaEventRecord(qev.second, ctx->stream), "event");
        ctx->q2_pending.push_back(qev);
        // each reflector row meets each column twice (dot and update), 8 real flops each;
        // the reflectors of sweep s cover rows s+1 .. n-1 once: sum n(n-1)/2
        ctx->q2_flops += (double)nbk * 8.0 * (double)n * (double)(n - 1) * (double)K;
        ctx->q2_launches++;
      }
    }
    if (K > 0) {
      blk_prep_kernel<<<nbk, kBlkThreads, 0, ctx->stream>>>(n, A, off);
      ctx->launches++;
      // Gram matrices G_p = V_p^H V_p of the back-transformation's panels (V explicit
      // and zero above its unit diagonal after blk_prep_kernel), then Tm from them
      const long long g2 = (long long)nbt * nbt;
      double2* G = (double2*)ws_get(ctx, WS_GRAM, (size_t)nbk * P2 * g2 * sizeof(double2));
      for (int p = 0; p < P2; ++p) {
        const int j0 = p * nbt;
        const int nbr = std::min(nbt, NR - j0);
        if (nbr <= 0) continue;
        const double2* V = A + (j0 + off) + (int64_t)j0 * n;
        zgemm_sb(h, OP_C, OP_N, nbr, nbr, n - j0 - off, 1.0, V, n, nn, V, n, nn, 0.0, G + p * g2, nbt,
                 (long long)P2 * g2, nbk);
        ctx->launches++;
      }
      const size_t lsm = (size_t)g2 * sizeof(double2);
      ck(cudaFuncSetAttribute(blk_larft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsm), "smem attr");
      blk_larft_kernel<<<dim3((unsigned)P2, (unsigned)nbk), kBlkThreads, lsm, ctx->stream>>>(n, nbt, P2, A, tau,
                                                                                             Tm, G, off);
      ctx->launches++;
    }
    for (int p = P2 - 1; p >= 0 && K > 0; --p) {
      const int j0 = p * nbt;
      const int nbr = std::min(nbt, NR - j0);
      if (nbr <= 0) continue;
      const int m = n - j0 - off;
      const double2* V = A + (j0 + off) + (int64_t)j0 * n;
      double2* Us = Ucur + (j0 + off) + (int64_t)c0 * n;
      // X = V^H Us (nbr x K), Y = Tm X, Us -= V Y
      zgemm_sb(h, OP_C, OP_N, nbr, K, m, 1.0, V, n, nn, Us, n, nn, 0.0, W, nbt, (long long)n * nbt,
               nbk);
      zgemm_sb(h, OP_N, OP_N, nbr, K, nbr, 1.0, Tm + (int64_t)p * nbt * nbt, nbt,
               (long long)nbt * nbt * P2, W, nbt, (long long)n * nbt, 0.0, Yb, nbt, (long long)n * nbt, nbk);
      zgemm_sb(h, OP_N, OP_N, m, K, nbr, -1.0, V, n, nn, Yb, nbt, (long long)n * nbt, 1.0, Us, n, nn,
               nbk);
      ctx->launches += 3;
    }
    if (rhok && !d_U) {
      blk_scale_f_cols_kernel<<<nbk, kBlkThreads, n * sizeof(double), ctx->stream>>>(
          n, Ucur, d_bands + k0 * n, mu, T, w + k0, A, ebk + k0, c0, K, complement ? 1 : 0);
      ctx->launches++;
      if (K > 0) {
        // rho_k is Hermitian: the lower column blocks by GEMM, the upper part mirrored
        const int cb = 128;
        const double al = complement ? -1.0 : 1.0;
        for (int cs = 0; cs < n; cs += cb) {
          const int cw = std::min(cb, n - cs);
          zgemm_sb(h, OP_N, OP_C, n - cs, cw, K, al, A + cs, n, nn, Ucur + (int64_t)c0 * n + cs, n, nn, 0.0,
                   rhok + k0 * nn + cs + (int64_t)cs * n, n, nn, nbk);
          ctx->launches++;
        }
        const int nt32 = (n + 31) / 32;
        if (nt32 > 1) {
          blk_herm_mirror_kernel<<<dim3((unsigned)(nt32 * (nt32 - 1) / 2), (unsigned)nbk), 256, 0, ctx->stream>>>(
              n, rhok + k0 * nn);
          ctx->launches++;
        }
      } else {
        ck(cudaMemsetAsync(rhok + k0 * nn, 0, (size_t)(nbk * nn) * sizeof(double2), ctx->stream), "memset");
      }
      if (complement) {
        blk_add_identity_kernel<<<nbk, kBlkThreads, 0, ctx->stream>>>(n, rhok + k0 * nn);
        ctx->launches++;
      }
    } else if (rhok) {
      blk_scale_f_kernel<<<nbk, kBlkThreads, n * sizeof(double), ctx->stream>>>(
          n, nbk, Ucur, d_bands + k0 * n, mu, nullptr, T, w + k0, A, ebk + k0);
      zgemm_sb(h, OP_N, OP_C, n, n, n, 1.0, A, n, nn, Ucur, n, nn, 0.0, rhok + k0 * nn, n, nn, nbk);
      ctx->launches += 2;
    }
    ck(cudaGetLastError(), "back-transformation launch");
  }
  if (ctx->stats_on) { ck(cudaEventRecord(evs.second, ctx->stream), "event"); ctx->ev_pending.push_back(evs); }
  ctx->eigh_launches++;
}

// Eigen pass over nk device k-points: bands (n x nk), optionally U and/or rho_k.
void launch_eigh(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, double* d_bands, double2* d_U,
                 const RhoOut* ro = nullptr) {
  NvtxRange nvtx_("eigen pass");
  const int n = (int)H->n;
  if (use_blocked(ctx, n, (int)H->nR)) {
    launch_eigh_large(ctx, H, nk, d_ks, d_bands, d_U, ro ? ro->rhok : nullptr, ro ? ro->ebk : nullptr,
                      ro ? ro->w : nullptr, ro ? ro->mu : 0.0, ro ? ro->T : 0.0);
    return;
  }
  const DCPlan& plan = get_plan(ctx, n);
  const int nt = eigh_threads_for(ctx, n);
  EighSmemLayout Ls = eigh_smem_layout(n, (int)H->nR, nt, 1);
  const int a_in_smem = Ls.total <= 225 * 1024;
  if (!a_in_smem) Ls = eigh_smem_layout(n, (int)H->nR, nt, 0);
  if (Ls.total > 225 * 1024) fail(LQM_EINVAL, "n=%d, nR=%lld exceeds the shared-memory plan", n, (long long)H->nR);
  const EighFn kfn = eigh_fn(nt);
  ck(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Ls.total), "smem attr");
  int per_sm = 0;
  ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, nt, Ls.total), "occupancy");
  if (per_sm < 1) fail(LQM_EINVAL, "eigh kernel cannot be resident for n=%d", n);
  const bool need_uwork = ro && !d_U && !a_in_smem;
  const int64_t slot = eigh_slot_doubles(n, a_in_smem, need_uwork);
  int64_t grid = std::min<int64_t>(nk, (int64_t)per_sm * ctx->num_sms);
  // keep the scratch below ~16 GB
  const int64_t max_slots = std::max<int64_t>(1, (int64_t)(16.0e9 / (8.0 * (double)slot)));
  grid = std::max<int64_t>(1, std::min(grid, max_slots));
  double* scratch = (double*)ws_get(ctx, WS_SCRATCH, (size_t)grid * slot * sizeof(double));
  EighArgs a;
  a.n = n; a.nR = (int)H->nR; a.dim = H->d; a.blocks = H->blocks; a.keys = H->keys;
  a.nk = nk; a.ks = d_ks; a.plan = plan; a.scratch = scratch; a.slot_doubles = slot;
  a.a_in_smem = a_in_smem; a.bands = d_bands; a.U = d_U;
  a.rhok = ro ? ro->rhok : nullptr;
  a.eband_k = ro ? ro->ebk : nullptr;
  a.w = ro ? ro->w : nullptr;
  a.mu = ro ? ro->mu : 0.0;
  a.T = ro ? ro->T : 0.0;
  a.phase_cycles = ctx->phases_on ? ctx->d_phase : nullptr;
  std::pair<cudaEvent_t, cudaEvent_t> evs{};
  if (ctx->stats_on) { evs = stat_events(ctx); ck(cudaEventRecord(evs.first, ctx->stream), "event"); }
  kfn<<<(unsigned)grid, nt, Ls.total, ctx->stream>>>(a);
  ck(cudaGetLastError(), "eigh_kernel launch");
  if (ctx->stats_on) { ck(cudaEventRecord(evs.second, ctx->stream), "event"); ctx->ev_pending.push_back(evs); }
  ctx->eigh_launches++;
  ctx->launches++;
}

// Path choice: the blocked path from n = 224 on, or from ctx->blocked_min_n when
// set, and always beyond the one-CTA kernel's shared-memory plan.  Measured on
// B200 (disordered honeycomb supercells, 1024 k-points, bands / rho k-points per
// second, one-CTA kernel against the blocked path): n = 144: 76.6k / 53.1k against
// 37.1k / 32.9k; n = 196: 31.2k / 19.8k against 23.5k / 18.8k; n = 256: 13.4k /
// 9.6k against 16.3k / 12.1k; n = 400: 3.2k / 2.3k against 8.2k / 5.0k.
constexpr int kBlockedDefaultMinN = 224;
bool use_blocked(const lqm_ctx* ctx, int n, int nR) {
  const int64_t nmin = ctx->blocked_min_n > 0 ? ctx->blocked_min_n : kBlockedDefaultMinN;
  if (n >= nmin) return true;
  return eigh_smem_layout(n, nR, eigh_threads_for(ctx, n), 0).total > 225 * 1024;
}

// Reduction of the blocked path: two-stage (dense -> band -> tridiagonal) or the
// one-stage zlatrd panels; ctx->two_stage when set (lqm_ctx_set_two_stage), else the
// two-stage form from kTwoStageDefaultMinN on (every order the blocked path serves)
// for passes that return no eigenvectors: eigenvalue-only passes, and density passes,
// which back-transform only the columns that carry rho_k.  Passes that return all n
// eigenvectors keep the one-stage reduction: the stage-2 back-transformation of n
// columns costs 8 n^3 flops per k-point.  Measured on B200 (576 k-points of the
// 24 x 24 grid unless noted): eigenvalues only at n = 1324 (400-point path) 0.50 s
// against 0.92 s; rho passes of 1024 k-points: n = 256 70 ms against 78, n = 400 163
// against 187; n = 508 177 against 178, n = 868 674 against 693, n = 1324 1.90 s
// against 1.92 s, n = 2884 (144 k-points) 3.94 s against 4.07 s; all vectors (the
// Hartree-Fock iteration at n = 2884, 144 k-points): 6.5 s against 5.3 s.
// LQM_TWO_STAGE=0/1 in the environment overrides both (development switch for
// measurements).
constexpr int kTwoStageDefaultMinN = 128;
bool use_two_stage(const lqm_ctx* ctx, int n, bool all_vectors) {
  if (n <= kTsB + 1) return false;
  const char* env = std::getenv("LQM_TWO_STAGE");
  if (env && (env[0] == '0' || env[0] == '1')) return env[0] == '1';
  if (ctx->two_stage >= 0) return ctx->two_stage == 1;
  const auto tuned = ctx->two_stage_tuned.find(2 * n + (all_vectors ? 1 : 0));
  if (tuned != ctx->two_stage_tuned.end()) return tuned->second == 1;
  return !all_vectors && n >= kTwoStageDefaultMinN;
}

int64_t batch_size_for(int64_t n, int64_t nk, double budget_bytes) {
  const double per_k = 16.0 * (double)n * (double)n;
  int64_t b = (int64_t)(budget_bytes / per_k);
  return std::max<int64_t>(1, std::min(b, nk));
}

// Density matrix on device arrays; accumulates eband into d_eb[0].
// rho_L (+)= sum_k coef[k,L] rho_k over a batch, as one ZGEMM: with rho_k the
// columns of R (nn x nb) and coef the nL x nb matrix C, rho_L (nn x nL) =
// R C^T (+ rho_L).  A skinny product (nL ~ 9 outputs per element read) that
// streams the rho_k batch once (the library's GEMM with 128 x 16 tiles, a fixed
// summation order for a given batch size).
void launch_fold(lqm_ctx* ctx, int64_t nn, int64_t nb, const double2* rk, const double2* coef, int nL,
                 double2* d_rho, int accumulate) {
  NvtxRange nvtx_("rho fold");
  zgemm_sb(blas_handle(ctx), OP_N, OP_T, (int)nn, nL, (int)nb, 1.0, rk, (int)nn, 0, coef, nL, 0,
           accumulate ? 1.0 : 0.0, d_rho, (int)nn, 0, 1);
}

// bands_out (n x nk, device) receives every k's eigenvalues when non-null.
// With `shard` and a communicator on the context, this rank processes its share of
// the k list, rho_L and the band energy are summed over the ranks and bands_out is
// gathered (lqm_comm.inc).
void density_dev(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, const double* d_w, double mu,
                 double T, int64_t nL, const int64_t* d_Lkeys, double2* d_rho, double* d_eb,
                 double* bands_out = nullptr, bool shard = false) {
  NvtxRange nvtx_("density matrix");
  const int n = (int)H->n;
  const int64_t nn = (int64_t)n * n;
  if (shard && sharded(ctx)) {
    const KShard s = kshard(ctx, nk);
    if (s.count() > 0)
      density_dev(ctx, H, s.count(), d_ks + s.k0 * H->d, d_w + s.k0, mu, T, nL, d_Lkeys, d_rho, d_eb,
                  bands_out ? bands_out + s.k0 * n : nullptr, false);
    else {
      ck(cudaMemsetAsync(d_rho, 0, (size_t)(nL * nn) * sizeof(double2), ctx->stream), "memset");
      ck(cudaMemsetAsync(d_eb, 0, sizeof(double), ctx->stream), "memset");
    }
    comm_allreduce(ctx, (double*)d_rho, (size_t)(2 * nL * nn));
    comm_allreduce(ctx, d_eb, 1);
    if (bands_out) comm_gather_k(ctx, bands_out, n, nk);
    return;
  }
  // rho_k batch: 4 GB, or one k-point per SM for large n (the blocked path
  // runs one divide-and-conquer CTA per k-point)
  const double budget = std::max(4.0e9, 16.0 * (double)nn * (double)std::min<int64_t>(nk, ctx->num_sms));
  const int64_t B = batch_size_for(n, nk, budget);
  double2* rk = (double2*)ws_get(ctx, WS_RHOK, (size_t)B * nn * sizeof(double2));
  double* bandsb = bands_out ? nullptr : (double*)ws_get(ctx, WS_BANDS, (size_t)B * n * sizeof(double));
  double* ebk = (double*)ws_get(ctx, WS_EBK, (size_t)B * sizeof(double));
  double2* coef = (double2*)ws_get(ctx, WS_COEF, (size_t)B * nL * sizeof(double2));
  for (int64_t k0 = 0; k0 < nk; k0 += B) {
    const int64_t nb = std::min(B, nk - k0);
    double* bands = bands_out ? bands_out + k0 * n : bandsb;
    const RhoOut ro{rk, ebk, d_w + k0, mu, T};
    launch_eigh(ctx, H, nb, d_ks + k0 * H->d, bands, nullptr, &ro);
    ordered_sum_kernel<<<1, 256, 0, ctx->stream>>>(ebk, nb, d_eb, k0 > 0);
    fold_coef_kernel<<<(unsigned)std::min<int64_t>((nb * nL + 255) / 256, 4096), 256, 0, ctx->stream>>>(
        nb, H->d, d_ks + k0 * H->d, d_w + k0, (int)nL, d_Lkeys, coef);
    launch_fold(ctx, nn, nb, rk, coef, (int)nL, d_rho, k0 > 0);
    ctx->launches += 2;
  }
}

// Eigen pass over a k list split over the ranks of the context's communicator:
// each rank solves its share, then bands (and U) are gathered so that every rank
// holds all of them.  Without a communicator this is launch_eigh.
void eigh_sharded(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, double* d_bands,
                  double2* d_U) {
  if (!sharded(ctx)) {
    launch_eigh(ctx, H, nk, d_ks, d_bands, d_U);
    return;
  }
  const KShard s = kshard(ctx, nk);
  const int64_t n = H->n;
  if (s.count() > 0)
    launch_eigh(ctx, H, s.count(), d_ks + s.k0 * H->d, d_bands + s.k0 * n, d_U ? d_U + s.k0 * n * n : nullptr);
  comm_gather_k(ctx, d_bands, n, nk);
  if (d_U) comm_gather_k(ctx, (double*)d_U, 2 * n * n, nk);
}

// Chemical potential entirely on the device: mu_out (device double) receives
// mu and err_out (device double, cleared here) counts failed searches.  No host
// synchronisation, so the sequence can be captured in a CUDA graph.
// WS_MISC layout (64 doubles): [0,1] min/max, [4..13] MuState, [16] mu,
// [17,18] order statistics, [19] error count, [40..44] SCF scalars.
void chempot_enqueue(lqm_ctx* ctx, int64_t n, int64_t nk, const double* d_bands, const double* d_w, double filling,
                     double T, double* mu_out, double* err_out) {
  const int64_t nv = n * nk;
  double* mm = (double*)ws_get(ctx, WS_MISC, 64 * sizeof(double));
  MuState* st = (MuState*)(mm + 4);
  ck(cudaMemsetAsync(err_out, 0, sizeof(double), ctx->stream), "memset");
  minmax_kernel<<<1, 1024, 0, ctx->stream>>>(d_bands, nv, mm);
  ctx->launches += 1;
  const int64_t nbk = std::max<int64_t>(1, std::min<int64_t>((nv + 4095) / 4096, (int64_t)ctx->num_sms * 4));
  const int64_t chunk = (nv + nbk - 1) / nbk;
  if (T > 0) {
    double* part = (double*)ws_get(ctx, WS_MU, (size_t)nbk * sizeof(double));
    mu_init_kernel<<<1, 1, 0, ctx->stream>>>(st, mm);
    const double norm = d_w ? 1.0 / (double)n : 1.0 / (double)nv;
    for (int it = 0; it < 140; ++it) {
      filling_partial_kernel<<<(unsigned)nbk, 256, 0, ctx->stream>>>(d_bands, (int)n, nv, d_w, st, T, chunk, part);
      mu_update_kernel<<<1, 32, 0, ctx->stream>>>(part, (int)nbk, st, filling, norm);
    }
    mu_store_kernel<<<1, 32, 0, ctx->stream>>>(st, mu_out, err_out);
    ctx->launches += 2 + 2 * 140;
    ck(cudaGetLastError(), "chemical potential launch");
    return;
  }
  // T == 0: midpoint of order statistics i, i+1 (1-based), chemicalpotential.jl:9-23
  if (filling >= 1.0 || filling <= 0.0) {
    mu_special_kernel<<<1, 32, 0, ctx->stream>>>(mm, mu_out, filling >= 1.0);
    ctx->launches += 1;
    ck(cudaGetLastError(), "chemical potential launch");
    return;
  }
  const long long i1 = 1 + (long long)std::floor(filling * (double)(nv - 1));
  long long* part = (long long*)ws_get(ctx, WS_MU, (size_t)nbk * sizeof(long long));
  for (int s = 0; s < 2; ++s) {
    os_init_kernel<<<1, 1, 0, ctx->stream>>>(st, mm, i1 + s);
    for (int it = 0; it < 140; ++it) {
      count_partial_kernel<<<(unsigned)nbk, 256, 0, ctx->stream>>>(d_bands, nv, st, chunk, part);
      os_update_kernel<<<1, 32, 0, ctx->stream>>>(part, (int)nbk, st);
    }
    mu_store_kernel<<<1, 32, 0, ctx->stream>>>(st, mm + 17 + s, err_out);
    ctx->launches += 2 + 2 * 140;
  }
  mu_avg_kernel<<<1, 32, 0, ctx->stream>>>(mm + 17, mm + 18, mu_out);
  ctx->launches += 1;
  ck(cudaGetLastError(), "order statistic launch");
}

double chempot_dev(lqm_ctx* ctx, int64_t n, int64_t nk, const double* d_bands, const double* d_w, double filling,
                   double T) {
  double* mm = (double*)ws_get(ctx, WS_MISC, 64 * sizeof(double));
  chempot_enqueue(ctx, n, nk, d_bands, d_w, filling, T, mm + 16, mm + 19);
  double h[4];
  ck(cudaMemcpyAsync(h, mm + 16, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "mu readback");
  wait_stream(ctx);
  if (h[3] != 0.0)
    fail(LQM_EDEVICE, T > 0 ? "filling - target does not change sign on [min eps, max eps]"
                            : "order-statistic bisection did not terminate");
  return h[0];
}

void dos_dev(lqm_ctx* ctx, int64_t n, int64_t nk, const double* d_bands, const double* d_w, int64_t nw,
             const double* d_om, double gamma, double* d_dos) {
  NvtxRange nvtx_("dos");
  const int64_t nv = n * nk;
  const int64_t nbk = std::max<int64_t>(1, std::min<int64_t>((nv + 1023) / 1024, (int64_t)ctx->num_sms * 2));
  const int64_t chunk = (nv + nbk - 1) / nbk;
  double* part = (double*)ws_get(ctx, WS_PART, (size_t)nbk * nw * sizeof(double));
  const int nt = nw >= 256 ? 256 : (int)((nw + 31) / 32 * 32);
  dos_partial_kernel<<<(unsigned)nbk, nt, 0, ctx->stream>>>(d_bands, (int)n, nv, d_w, (int)nw, d_om, gamma, chunk,
                                                           part);
  dos_reduce_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, ctx->stream>>>(part, (int)nbk, (int)nw,
                                                                         d_w ? 1.0 : 1.0 / (double)nk, d_dos);
  ck(cudaGetLastError(), "dos launch");
  ctx->launches += 2;
}

template <class T>
T* upload(lqm_ctx* ctx, int slot, const T* h, size_t count) {
  T* d = (T*)ws_get(ctx, slot, count * sizeof(T));
  ck(cudaMemcpyAsync(d, h, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream), "H2D");
  return d;
}

double* uniform_weights(lqm_ctx* ctx, int64_t nk, int slot = WS_W) {
  std::vector<double> w((size_t)nk, 1.0 / (double)nk);
  double* d = upload(ctx, slot, w.data(), w.size());
  wait_stream(ctx);
  return d;
}

void check_ks(const double* ks, int64_t nk, int d) {
  if (nk < 1) fail(LQM_EINVAL, "nk must be >= 1");
  if (!ks) fail(LQM_EINVAL, "null k-point array");
  check_finite(ks, nk * d, "ks");
}

void check_precision(int precision) {
  if (precision != 0) fail(LQM_EINVAL, "precision=%d: only the FP64 path (0) is available", precision);
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================
namespace {

// One eigen pass over the k-points of several models of uneven order (the one-CTA
// eigensolver's orders) as ONE launch of eigh_multi_kernel: model m's k-points go to
// teams of its own block size, several teams per CTA on named barriers.  Writes
// each model's bands and rho_k batch (with the band energies per k).
void launch_eigh_multi(lqm_ctx* ctx, int nm, const lqm_hops* const* H, int64_t nk, const double* d_ks,
                       double* const* bands, double2* const* rhok, double* const* ebk, const double* d_w, double mu,
                       double T) {
  NvtxRange nvtx_("eigen pass (several models, one launch)");
  if (nm < 1 || nm > kMaxModels) fail(LQM_EINVAL, "between 1 and %d models per launch", kMaxModels);
  int tnt[kMaxModels];
  int NT = 0;
  for (int m = 0; m < nm; ++m) {
    const int n = (int)H[m]->n;
    if (use_blocked(ctx, n, (int)H[m]->nR))
      fail(LQM_EINVAL, "model %d (n=%d) is served by the blocked eigensolver, not the one-CTA one", m, n);
    tnt[m] = eigh_threads_for(ctx, n);
    NT = std::max(NT, tnt[m]);
  }
  NT = NT <= 384 ? 384 : 512;
  for (int m = 0; m < nm; ++m) {
    if (NT % tnt[m] != 0) tnt[m] = NT;            // a team size that does not tile the CTA runs CTA-wide
    while (NT / tnt[m] > 15) tnt[m] *= 2;         // at most 15 named barriers per CTA
  }
  EighMultiArgs ma{};
  ma.nmodels = nm;
  int64_t smem = 0, slot = 0, slots_per_cta = 1;
  for (int m = 0; m < nm; ++m) {
    const int n = (int)H[m]->n, nR = (int)H[m]->nR;
    const int teams = NT / tnt[m];
    EighSmemLayout Ls = eigh_smem_layout(n, nR, tnt[m], 1);
    int a_in_smem = (int64_t)teams * (int64_t)lqm_align16(Ls.total) <= 225 * 1024;
    if (!a_in_smem) Ls = eigh_smem_layout(n, nR, tnt[m], 0);
    const int64_t per_team = (int64_t)lqm_align16(Ls.total);
    if ((int64_t)teams * per_team > 225 * 1024) fail(LQM_EINVAL, "model %d (n=%d) exceeds the shared-memory plan", m, n);
    smem = std::max(smem, (int64_t)teams * per_team);
    slot = std::max(slot, eigh_slot_doubles(n, a_in_smem, !a_in_smem));
    slots_per_cta = std::max<int64_t>(slots_per_cta, teams);
    EighArgs& a = ma.m[m];
    a.n = n; a.nR = nR; a.dim = H[m]->d; a.blocks = H[m]->blocks; a.keys = H[m]->keys;
    a.nk = nk; a.ks = d_ks; a.plan = get_plan(ctx, n); a.a_in_smem = a_in_smem;
    a.bands = bands[m]; a.U = nullptr; a.rhok = rhok[m]; a.eband_k = ebk[m]; a.w = d_w; a.mu = mu; a.T = T;
    a.phase_cycles = nullptr;
    ma.team_nt[m] = tnt[m];
    ma.smem_team[m] = per_team;
  }
  // items: model after model, k-points in groups of one per team of a CTA
  ma.item_begin[0] = 0;
  for (int m = 0; m < nm; ++m) {
    const int teams = NT / tnt[m];
    ma.item_begin[m + 1] = ma.item_begin[m] + (nk + teams - 1) / teams;
  }
  ma.slots_per_cta = slots_per_cta;
  auto kfn = NT == 384 ? &eigh_multi_kernel<384> : &eigh_multi_kernel<512>;
  ck(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
  int per_sm = 0;
  ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, NT, (size_t)smem), "occupancy");
  if (per_sm < 1) fail(LQM_EINVAL, "the model-batched eigensolver cannot be resident");
  int64_t grid = std::min<int64_t>(ma.item_begin[nm], (int64_t)per_sm * ctx->num_sms);
  const int64_t max_cta = std::max<int64_t>(1, (int64_t)(16.0e9 / (8.0 * (double)slot * (double)slots_per_cta)));
  grid = std::max<int64_t>(1, std::min(grid, max_cta));
  double* scratch = (double*)ws_get(ctx, WS_SCRATCH, (size_t)(grid * slots_per_cta * slot) * sizeof(double));
  for (int m = 0; m < nm; ++m) {
    ma.m[m].scratch = scratch;
    ma.m[m].slot_doubles = slot;
  }
  std::pair<cudaEvent_t, cudaEvent_t> evs{};
  if (ctx->stats_on) { evs = stat_events(ctx); ck(cudaEventRecord(evs.first, ctx->stream), "event"); }
  kfn<<<(unsigned)grid, NT, (size_t)smem, ctx->stream>>>(ma);
  ck(cudaGetLastError(), "eigh_multi_kernel launch");
  if (ctx->stats_on) { ck(cudaEventRecord(evs.second, ctx->stream), "event"); ctx->ev_pending.push_back(evs); }
  ctx->eigh_launches++;
  ctx->launches++;
}

}  // namespace

extern "C" {

int lqm_ctx_create(int device, lqm_ctx** out) {
  if (!out) return LQM_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LQM_ECUDA;
  if (device < 0 || device >= ndev) return LQM_EINVAL;
  lqm_ctx* c = new (std::nothrow) lqm_ctx();
  if (!c) return LQM_ENOMEM;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    delete c;
    return LQM_ECUDA;
  }
  *out = c;
  return LQM_OK;
}

int lqm_ctx_destroy(lqm_ctx* ctx) {
  if (!ctx) return LQM_EINVAL;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  try {
    comm_release(ctx);
  } catch (const LqmError&) {
  }
  for (auto& b : ctx->ws)
    if (b.p) cudaFree(b.p);
  for (auto& kv : ctx->plans) cudaFree(kv.second.d_buf);
  for (auto& b : ctx->hops_cache) cudaFree(b.first);
  if (ctx->d_phase) cudaFree(ctx->d_phase);
  if (ctx->d_err) cudaFree(ctx->d_err);
  cudaEventDestroy(ctx->ev0);
  cudaEventDestroy(ctx->ev1);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return LQM_OK;
}

const char* lqm_last_error(const lqm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int lqm_ctx_set_timeout(lqm_ctx* ctx, double seconds) {
  if (!ctx || !(seconds > 0)) return LQM_EINVAL;
  ctx->timeout_s = seconds;
  return LQM_OK;
}

int lqm_ctx_set_scf_acceleration(lqm_ctx* ctx, int anderson_depth) {
  if (!ctx || anderson_depth < 0 || anderson_depth > 8) return LQM_EINVAL;  // kAndMaxDepth (lqm_anderson.inc)
  ctx->scf_anderson_depth = anderson_depth;
  return LQM_OK;
}

int lqm_ctx_set_scf_residual(lqm_ctx* ctx, int mode) {
  if (!ctx || mode < 0 || mode > 1) return LQM_EINVAL;
  ctx->scf_residual = mode;
  return LQM_OK;
}

int lqm_ctx_set_scf_terms(lqm_ctx* ctx, int hartree, int fock) {
  if (!ctx) return LQM_EINVAL;
  ctx->scf_hartree = hartree != 0;
  ctx->scf_fock = fock != 0;
  return LQM_OK;
}

int lqm_ctx_set_scf_exchange(lqm_ctx* ctx, int64_t ns, int64_t nJ, int32_t d, const int64_t* jkeys,
                             const double* jblocks, int64_t n, const int64_t* siteof, const int64_t* flavorof) {
  return guarded(ctx, [&] {
    if (ns == 0) {  // no exchange kernel
      ctx->ex_ns = ctx->ex_nf = ctx->ex_nJ = 0;
      ctx->ex_keys.clear();
      ctx->ex_blocks.clear();
      ctx->ex_sf2idx.clear();
      return;
    }
    if (ns < 1 || nJ < 1 || d < 1 || d > 3 || !jkeys || !jblocks || n < 1 || !siteof || !flavorof)
      fail(LQM_EINVAL, "invalid exchange kernel arguments");
    // ExchangeKernel(j, siteof, flavorof), hartreefock.jl:47-76 (0-based sites and flavors here)
    int64_t nf = 0;
    for (int64_t I = 0; I < n; ++I) {
      if (siteof[I] < 0 || siteof[I] >= ns) fail(LQM_EINVAL, "siteof[%lld] outside 0..%lld", (long long)I, (long long)(ns - 1));
      if (flavorof[I] < 0) fail(LQM_EINVAL, "flavorof[%lld] is negative", (long long)I);
      nf = std::max<int64_t>(nf, flavorof[I] + 1);
    }
    if (ns * nf != n) fail(LQM_EINVAL, "every (site, flavor) pair must appear once");
    std::vector<int> sf((size_t)(ns * nf), -1);
    for (int64_t I = 0; I < n; ++I) {
      int& slot = sf[(size_t)(siteof[I] + ns * flavorof[I])];
      if (slot >= 0) fail(LQM_EINVAL, "duplicate (site, flavor) = (%lld, %lld)", (long long)siteof[I], (long long)flavorof[I]);
      slot = (int)I;
    }
    check_finite(jblocks, 2 * ns * ns * nJ, "exchange kernel");
    int64_t z = -1;
    for (int64_t l = 0; l < nJ && z < 0; ++l) {
      bool zero = true;
      for (int c = 0; c < d; ++c) zero = zero && jkeys[l * d + c] == 0;
      if (zero) z = l;
    }
    if (z < 0) fail(LQM_EINVAL, "the exchange kernel needs the zero key");
    for (int64_t a = 0; a < ns; ++a) {
      const double* e = jblocks + 2 * (z * ns * ns + a + a * ns);
      if (e[0] != 0.0 || e[1] != 0.0)
        fail(LQM_EINVAL, "onsite self-exchange j[0][a,a] must be zero (it is part of the direct interaction)");
    }
    ctx->ex_ns = ns;
    ctx->ex_nf = nf;
    ctx->ex_nJ = nJ;
    ctx->ex_d = d;
    ctx->ex_keys.assign(jkeys, jkeys + nJ * d);
    ctx->ex_blocks.assign(jblocks, jblocks + 2 * ns * ns * nJ);
    ctx->ex_sf2idx = sf;
  });
}

int lqm_ctx_scf_exchange_energy(const lqm_ctx* ctx, double* eJ) {
  if (!ctx || !eJ) return LQM_EINVAL;
  *eJ = ctx->scf_eJ;
  return LQM_OK;
}

int lqm_ctx_set_eigh_threads(lqm_ctx* ctx, int64_t n, int nt) {
  if (!ctx || n < 1 || nt < 0 || nt > 512 || nt % 32 != 0) return LQM_EINVAL;
  if (nt == 0) ctx->eigh_nt.erase((int)n);
  else ctx->eigh_nt[(int)n] = nt;
  return LQM_OK;
}

int lqm_ctx_set_blocked_min_n(lqm_ctx* ctx, int64_t n_min) {
  if (!ctx || n_min < 0) return LQM_EINVAL;
  ctx->blocked_min_n = n_min;
  return LQM_OK;
}

int lqm_ctx_set_device_wait_limit(lqm_ctx* ctx, int64_t polls) {
  if (!ctx || polls < 0) return LQM_EINVAL;
  ctx->dev_wait_limit = polls;
  return LQM_OK;
}

int lqm_ctx_set_two_stage(lqm_ctx* ctx, int mode) {
  if (!ctx || mode < -1 || mode > 1) return LQM_EINVAL;
  ctx->two_stage = mode;
  return LQM_OK;
}

int lqm_ctx_last_kernel_ms(const lqm_ctx* ctx, double* ms) {
  if (!ctx || !ms) return LQM_EINVAL;
  *ms = ctx->last_ms;
  return LQM_OK;
}

int lqm_ctx_reset_stats(lqm_ctx* ctx, int enable_timing) {
  return guarded(ctx, [&] {
    wait_stream(ctx);
    if (!ctx->d_phase) ck(cudaMalloc(&ctx->d_phase, PH_COUNT * sizeof(unsigned long long)), "cudaMalloc(stats)");
    ck(cudaMemset(ctx->d_phase, 0, PH_COUNT * sizeof(unsigned long long)), "memset(stats)");
    ctx->stats_on = enable_timing != 0;
    ctx->phases_on = enable_timing >= 2;
    ctx->eigh_ms = 0.0;
    ctx->eigh_launches = 0;
    ctx->launches = 0;
    ctx->symv_ms = 0.0;
    ctx->q2_ms = 0.0;
    ctx->q2_flops = 0.0;
    ctx->q2_launches = 0;
    ctx->symv_bytes = 0.0;
    ctx->symv_launches = 0;
  });
}

int lqm_ctx_phase_cycles(lqm_ctx* ctx, double* cycles) {
  return guarded(ctx, [&] {
    if (!cycles) fail(LQM_EINVAL, "null output");
    unsigned long long h[PH_COUNT] = {0};
    if (ctx->d_phase) {
      wait_stream(ctx);
      ck(cudaMemcpy(h, ctx->d_phase, sizeof(h), cudaMemcpyDeviceToHost), "D2H");
    }
    for (int i = 0; i < 16; ++i) cycles[i] = (double)h[i];
  });
}

int lqm_ctx_kernel_stats(const lqm_ctx* ctx, int kernel_class, double* ms, int64_t* launches,
                         double* algorithmic_bytes) {
  if (!ctx || kernel_class < 0 || kernel_class > 2) return LQM_EINVAL;
  if (kernel_class == 0) {
    if (ms) *ms = ctx->eigh_ms;
    if (launches) *launches = ctx->eigh_launches;
    if (algorithmic_bytes) *algorithmic_bytes = 0.0;
  } else if (kernel_class == 2) {
    if (ms) *ms = ctx->q2_ms;
    if (launches) *launches = ctx->q2_launches;
    if (algorithmic_bytes) *algorithmic_bytes = ctx->q2_flops;  // algorithmic flops for this class
  } else {
    if (ms) *ms = ctx->symv_ms;
    if (launches) *launches = ctx->symv_launches;
    if (algorithmic_bytes) *algorithmic_bytes = ctx->symv_bytes;
  }
  return LQM_OK;
}

int lqm_ctx_stats(const lqm_ctx* ctx, double* eigh_ms, int64_t* eigh_launches, int64_t* launches) {
  if (!ctx) return LQM_EINVAL;
  if (eigh_ms) *eigh_ms = ctx->eigh_ms;
  if (eigh_launches) *eigh_launches = ctx->eigh_launches;
  if (launches) *launches = ctx->launches;
  return LQM_OK;
}

int lqm_hops_upload_dense(lqm_ctx* ctx, int64_t n, int64_t nR, int32_t d, const int64_t* keys,
                          const double* blocks, lqm_hops** out) {
  return guarded(ctx, [&] {
    if (!out) fail(LQM_EINVAL, "null output pointer");
    *out = nullptr;
    if (n < 1 || nR < 1 || d < 1 || d > 3) fail(LQM_EINVAL, "invalid sizes n=%lld nR=%lld d=%d", (long long)n, (long long)nR, d);
    if (n > 4096) fail(LQM_EINVAL, "n=%lld exceeds the supported maximum 4096", (long long)n);
    if (!keys || !blocks) fail(LQM_EINVAL, "null keys or blocks");
    check_finite(blocks, 2 * n * n * nR, "blocks");
    const size_t bb = (size_t)(n * n * nR) * sizeof(double2);
    const size_t koff = (bb + 255) / 256 * 256;
    const size_t need = koff + (size_t)(d * nR) * sizeof(int64_t);
    size_t got = 0;
    void* buf = hops_buffer_take(ctx, need, &got);
    if (!buf) {
      if (cudaMalloc(&buf, need) != cudaSuccess) {
        cudaGetLastError();
        fail(LQM_ENOMEM, "device allocation for hops failed");
      }
      got = need;
    }
    lqm_hops* h = new lqm_hops();
    h->n = n; h->nR = nR; h->d = d;
    h->hkeys.assign(keys, keys + d * nR);
    h->blocks = (double2*)buf;
    h->keys = (int64_t*)((char*)buf + koff);
    h->device = ctx->device;
    h->buf_bytes = got;
    try {
      ck(cudaMemcpyAsync(h->blocks, blocks, bb, cudaMemcpyHostToDevice, ctx->stream), "hops upload");
      ck(cudaMemcpyAsync(h->keys, keys, (size_t)(d * nR) * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream),
         "keys upload");
      wait_stream(ctx);
    } catch (const LqmError& e) {  // neither the buffer nor the handle outlives a failed upload
      if (e.code != LQM_ETIMEOUT) cudaFree(buf);  // (after a timeout the copy may still run: leave it)
      delete h;
      throw;
    }
    *out = h;
  });
}

int lqm_hops_upload_csc(lqm_ctx* ctx, int64_t n, int64_t nR, int32_t d, const int64_t* keys,
                        const int64_t* const* colptr, const int64_t* const* rowval, const double* const* nzval,
                        const int64_t* nnz, lqm_hops** out) {
  return guarded(ctx, [&] {
    if (!out) fail(LQM_EINVAL, "null output pointer");
    *out = nullptr;
    if (!colptr || !rowval || !nzval || !nnz || !keys) fail(LQM_EINVAL, "null argument");
    if (n < 1 || nR < 1 || d < 1 || d > 3) fail(LQM_EINVAL, "invalid sizes n=%lld nR=%lld d=%d", (long long)n, (long long)nR, d);
    if (n > 4096) fail(LQM_EINVAL, "n=%lld exceeds the supported maximum 4096", (long long)n);
    // Host validation of every block before anything reaches the device: colptr is
    // 1-based and non-decreasing, its last entry stays within the caller's nnz[r]
    // (the lengths of rowval[r] and nzval[r]/2), rows lie in 1..n, values are finite.
    std::vector<int64_t> used((size_t)nR);
    size_t stage = 0;
    for (int64_t r = 0; r < nR; ++r) {
      const int64_t* cp = colptr[r];
      if (!cp || nnz[r] < 0) fail(LQM_EINVAL, "invalid colptr or nnz in block %lld", (long long)r);
      if (cp[0] != 1) fail(LQM_EINVAL, "colptr of block %lld does not start at 1", (long long)r);
      for (int64_t j = 0; j < n; ++j)
        if (cp[j + 1] < cp[j]) fail(LQM_EINVAL, "colptr of block %lld decreases at column %lld", (long long)r, (long long)j);
      const int64_t m = cp[n] - 1;
      if (m > nnz[r])
        fail(LQM_EINVAL, "block %lld: colptr ends at %lld entries, beyond its nnz %lld", (long long)r, (long long)m,
             (long long)nnz[r]);
      if (m > 0 && (!rowval[r] || !nzval[r])) fail(LQM_EINVAL, "null rowval or nzval in block %lld", (long long)r);
      for (int64_t p = 0; p < m; ++p)
        if (rowval[r][p] < 1 || rowval[r][p] > n)
          fail(LQM_EINVAL, "row index out of range in block %lld", (long long)r);
      if (m > 0) check_finite(nzval[r], 2 * m, "nzval");
      used[(size_t)r] = m;
      stage += (size_t)(n + 1 + m) * sizeof(int64_t) + (size_t)m * sizeof(double2);
    }
    const size_t bb = (size_t)(n * n * nR) * sizeof(double2);
    const size_t koff = (bb + 255) / 256 * 256;
    const size_t need = koff + (size_t)(d * nR) * sizeof(int64_t);
    size_t got = 0;
    void* buf = hops_buffer_take(ctx, need, &got);
    if (!buf) {
      if (cudaMalloc(&buf, need) != cudaSuccess) {
        cudaGetLastError();
        fail(LQM_ENOMEM, "device allocation for hops failed");
      }
      got = need;
    }
    lqm_hops* h = new lqm_hops();
    h->n = n; h->nR = nR; h->d = d;
    h->hkeys.assign(keys, keys + d * nR);
    h->blocks = (double2*)buf;
    h->keys = (int64_t*)((char*)buf + koff);
    h->device = ctx->device;
    h->buf_bytes = got;
    try {
      // Only the stored entries cross PCIe (about a tenth of the dense bytes for the
      // twisted bilayers); the blocks are zeroed and filled on the device.
      char* st = (char*)ws_get(ctx, WS_CSC, stage + 256 * (size_t)(3 * nR + 1));
      ck(cudaMemsetAsync(h->blocks, 0, bb, ctx->stream), "hops memset");
      ck(cudaMemcpyAsync(h->keys, keys, (size_t)(d * nR) * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream),
         "keys upload");
      size_t off = 0;
      auto place = [&](size_t bytes) { char* p = st + off; off = (off + bytes + 255) / 256 * 256; return p; };
      for (int64_t r = 0; r < nR; ++r) {
        const int64_t m = used[(size_t)r];
        int64_t* dcp = (int64_t*)place((size_t)(n + 1) * sizeof(int64_t));
        int64_t* drv = (int64_t*)place((size_t)m * sizeof(int64_t));
        double2* dnz = (double2*)place((size_t)m * sizeof(double2));
        ck(cudaMemcpyAsync(dcp, colptr[r], (size_t)(n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream),
           "colptr upload");
        if (m > 0) {
          ck(cudaMemcpyAsync(drv, rowval[r], (size_t)m * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream),
             "rowval upload");
          ck(cudaMemcpyAsync(dnz, nzval[r], (size_t)m * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream),
             "nzval upload");
        }
        csc_scatter_kernel<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(n, dcp, drv, dnz,
                                                                               h->blocks + r * n * n);
        ctx->launches += 1;
      }
      ck(cudaGetLastError(), "csc scatter launch");
      wait_stream(ctx);
    } catch (const LqmError& e) {  // neither the buffer nor the handle outlives a failed upload
      if (e.code != LQM_ETIMEOUT) cudaFree(buf);
      delete h;
      throw;
    }
    *out = h;
  });
}

int lqm_hops_free(lqm_ctx* ctx, lqm_hops* h) {
  if (!h) return LQM_EINVAL;
  if (!ctx) {  // no context: cudaFree itself waits for the device's work
    if (h->device >= 0) cudaSetDevice(h->device);
    cudaFree(h->blocks);
    delete h;
    return LQM_OK;
  }
  return guarded(ctx, [&] {
    // Kernels queued on the context may still read the blocks: wait for them with the
    // context's limit.  On LQM_ETIMEOUT nothing is released and h stays valid.
    wait_stream(ctx);
    if (!(ctx->device == h->device && hops_buffer_keep(ctx, h->blocks, h->buf_bytes))) {
      if (h->device >= 0) cudaSetDevice(h->device);
      cudaFree(h->blocks);
      cudaSetDevice(ctx->device);
    }
    delete h;
  });
}

int lqm_hops_dims(const lqm_hops* h, int64_t* n, int64_t* nR, int32_t* d) {
  if (!h || !n || !nR || !d) return LQM_EINVAL;
  *n = h->n; *nR = h->nR; *d = h->d;
  return LQM_OK;
}

int lqm_bloch_dev(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, double* d_Hk) {
  return guarded(ctx, [&] {
    check_hops(H);
    if (nk < 1 || !d_ks || !d_Hk) fail(LQM_EINVAL, "invalid arguments");
    timer_start(ctx);
    const int64_t g = std::min<int64_t>(nk, (int64_t)ctx->num_sms * 8);
    bloch_kernel<<<(unsigned)g, 256, (size_t)H->nR * sizeof(double2), ctx->stream>>>(
        (int)H->n, (int)H->nR, H->d, H->blocks, H->keys, nk, d_ks, (double2*)d_Hk);
    ck(cudaGetLastError(), "bloch_kernel launch");
    ctx->launches += 1;
    timer_stop(ctx);
    wait_stream(ctx);
    timer_collect(ctx);
  });
}

int lqm_bloch(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, double* Hk) {
  return guarded(ctx, [&] {
    check_hops(H);
    check_ks(ks, nk, H->d);
    if (!Hk) fail(LQM_EINVAL, "null output");
    const double* dks = upload(ctx, WS_KS, ks, (size_t)(nk * H->d));
    const size_t ob = (size_t)(nk * H->n * H->n) * sizeof(double2);
    double* dH = (double*)ws_get(ctx, WS_U, ob);
    int st = lqm_bloch_dev(ctx, H, nk, dks, dH);
    if (st != LQM_OK) fail(st, "%s", ctx->err.c_str());
    ck(cudaMemcpyAsync(Hk, dH, ob, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    wait_stream(ctx);
  });
}

int lqm_bandmatrix_dev(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, int want_vectors,
                       int precision, double* d_bands, double* d_U) {
  return guarded(ctx, [&] {
    check_hops(H);
    check_precision(precision);
    if (nk < 1 || !d_ks || !d_bands || (want_vectors && !d_U)) fail(LQM_EINVAL, "invalid arguments");
    timer_start(ctx);
    eigh_sharded(ctx, H, nk, d_ks, d_bands, want_vectors ? (double2*)d_U : nullptr);
    timer_stop(ctx);
    wait_stream(ctx);
    timer_collect(ctx);
  });
}

int lqm_bandmatrix(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, int want_vectors, int precision,
                   double* bands, double* U) {
  return guarded(ctx, [&] {
    check_hops(H);
    check_precision(precision);
    check_ks(ks, nk, H->d);
    if (!bands || (want_vectors && !U)) fail(LQM_EINVAL, "null output");
    const int64_t n = H->n;
    const double* dks = upload(ctx, WS_KS, ks, (size_t)(nk * H->d));
    double* db = (double*)ws_get(ctx, WS_BANDS, (size_t)(n * nk) * sizeof(double));
    double* dU = want_vectors ? (double*)ws_get(ctx, WS_U, (size_t)(n * n * nk) * sizeof(double2)) : nullptr;
    timer_start(ctx);
    eigh_sharded(ctx, H, nk, dks, db, (double2*)dU);
    timer_stop(ctx);
    wait_stream(ctx);  // poll with the context's limit: a copy into pageable host memory would block unbounded
    ck(cudaMemcpyAsync(bands, db, (size_t)(n * nk) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    if (want_vectors)
      ck(cudaMemcpyAsync(U, dU, (size_t)(n * n * nk) * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    wait_stream(ctx);
    timer_collect(ctx);
  });
}

int lqm_densitymatrix_dev(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, const double* d_w,
                          double mu, double T, int64_t nL, const int64_t* Lkeys, double* d_rho, double* eband,
                          int precision) {
  return guarded(ctx, [&] {
    check_hops(H);
    check_precision(precision);
    if (nk < 1 || !d_ks || nL < 1 || !Lkeys || !d_rho) fail(LQM_EINVAL, "invalid arguments");
    if (!std::isfinite(mu) || !(T >= 0) || !std::isfinite(T)) fail(LQM_EINVAL, "invalid mu/T");
    const int64_t* dL = upload(ctx, WS_LKEYS, Lkeys, (size_t)(nL * H->d));
    const double* dw = d_w ? d_w : uniform_weights(ctx, nk);
    double* d_eb = (double*)ws_get(ctx, WS_MISC, 64 * sizeof(double)) + 40;
    timer_start(ctx);
    density_dev(ctx, H, nk, d_ks, dw, mu, T, nL, dL, (double2*)d_rho, d_eb, nullptr, true);
    timer_stop(ctx);
    double eb = 0.0;
    wait_stream(ctx);  // poll with the context's limit: a copy into pageable host memory would block unbounded
    ck(cudaMemcpyAsync(&eb, d_eb, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    wait_stream(ctx);
    timer_collect(ctx);
    if (eband) *eband = eb;
  });
}

int lqm_densitymatrix(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w, double mu,
                      double T, int64_t nL, const int64_t* Lkeys, double* rho, double* eband, int precision) {
  return guarded(ctx, [&] {
    check_hops(H);
    check_ks(ks, nk, H->d);
    if (!rho || !Lkeys || nL < 1) fail(LQM_EINVAL, "invalid arguments");
    if (w) check_finite(w, nk, "w");
    const double* dks = upload(ctx, WS_KS, ks, (size_t)(nk * H->d));
    const double* dw = w ? upload(ctx, WS_W, w, (size_t)nk) : nullptr;
    const size_t rb = (size_t)(nL * H->n * H->n) * sizeof(double2);
    double* drho = (double*)ws_get(ctx, WS_RHO, rb);
    int st = lqm_densitymatrix_dev(ctx, H, nk, dks, dw, mu, T, nL, Lkeys, drho, eband, precision);
    if (st != LQM_OK) fail(st, "%s", ctx->err.c_str());
    ck(cudaMemcpyAsync(rho, drho, rb, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    wait_stream(ctx);
  });
}

int lqm_chemicalpotential_bands_dev(lqm_ctx* ctx, int64_t n, int64_t nk, const double* d_bands, const double* d_w,
                                    double filling, double T, double* mu) {
  return guarded(ctx, [&] {
    if (n < 1 || nk < 1 || !d_bands || !mu) fail(LQM_EINVAL, "invalid arguments");
    if (!std::isfinite(filling) || !(T >= 0) || !std::isfinite(T)) fail(LQM_EINVAL, "invalid filling/T");
    *mu = chempot_dev(ctx, n, nk, d_bands, d_w, filling, T);
  });
}

int lqm_chemicalpotential(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w,
                          double filling, double T, double* mu) {
  return guarded(ctx, [&] {
    check_hops(H);
    check_ks(ks, nk, H->d);
    if (!mu) fail(LQM_EINVAL, "null output");
    if (w) check_finite(w, nk, "w");
    const double* dks = upload(ctx, WS_KS, ks, (size_t)(nk * H->d));
    const double* dw = w ? upload(ctx, WS_W, w, (size_t)nk) : nullptr;
    double* db = (double*)ws_get(ctx, WS_BANDS, (size_t)(H->n * nk) * sizeof(double));
    timer_start(ctx);
    eigh_sharded(ctx, H, nk, dks, db, nullptr);
    timer_stop(ctx);
    wait_stream(ctx);
    timer_collect(ctx);
    int st = lqm_chemicalpotential_bands_dev(ctx, H->n, nk, db, dw, filling, T, mu);
    if (st != LQM_OK) fail(st, "%s", ctx->err.c_str());
  });
}

int lqm_dos_bands_dev(lqm_ctx* ctx, int64_t n, int64_t nk, const double* d_bands, const double* d_w, int64_t nw,
                      const double* d_omegas, double gamma, double* d_dos) {
  return guarded(ctx, [&] {
    if (n < 1 || nk < 1 || nw < 1 || !d_bands || !d_omegas || !d_dos) fail(LQM_EINVAL, "invalid arguments");
    if (!std::isfinite(gamma)) fail(LQM_EINVAL, "invalid gamma");
    dos_dev(ctx, n, nk, d_bands, d_w, nw, d_omegas, gamma, d_dos);
    wait_stream(ctx);
  });
}

int lqm_dos(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w, int64_t nw,
            const double* omegas, double gamma, double* dos) {
  return guarded(ctx, [&] {
    check_hops(H);
    check_ks(ks, nk, H->d);
    if (nw < 1 || !omegas || !dos) fail(LQM_EINVAL, "invalid arguments");
    check_finite(omegas, nw, "omegas");
    if (w) check_finite(w, nk, "w");
    const double* dks = upload(ctx, WS_KS, ks, (size_t)(nk * H->d));
    const double* dw = w ? upload(ctx, WS_W, w, (size_t)nk) : nullptr;
    const double* dom = upload(ctx, WS_OMEGA, omegas, (size_t)nw);
    double* db = (double*)ws_get(ctx, WS_BANDS, (size_t)(H->n * nk) * sizeof(double));
    double* dd = (double*)ws_get(ctx, WS_DOS, (size_t)nw * sizeof(double));
    timer_start(ctx);
    eigh_sharded(ctx, H, nk, dks, db, nullptr);
    dos_dev(ctx, H->n, nk, db, dw, nw, dom, gamma, dd);
    timer_stop(ctx);
    ck(cudaMemcpyAsync(dos, dd, (size_t)nw * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    wait_stream(ctx);
    timer_collect(ctx);
  });
}

int lqm_bands_dos_rho_dev(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, const double* d_w,
                          double mu, double T, int64_t nL, const int64_t* Lkeys, double* d_rho, double* eband,
                          int64_t nw, const double* d_omegas, double gamma, double* d_dos, double* d_bands,
                          int precision) {
  return guarded(ctx, [&] {
    check_hops(H);
    check_precision(precision);
    if (nk < 1 || !d_ks || nL < 1 || !Lkeys || !d_rho || nw < 1 || !d_omegas || !d_dos || !d_bands)
      fail(LQM_EINVAL, "invalid arguments");
    if (!std::isfinite(mu) || !(T >= 0) || !std::isfinite(T) || !std::isfinite(gamma))
      fail(LQM_EINVAL, "invalid mu/T/gamma");
    const int64_t* dL = upload(ctx, WS_LKEYS, Lkeys, (size_t)(nL * H->d));
    const double* dw = d_w ? d_w : uniform_weights(ctx, nk);
    double* d_eb = (double*)ws_get(ctx, WS_MISC, 64 * sizeof(double)) + 40;
    timer_start(ctx);
    density_dev(ctx, H, nk, d_ks, dw, mu, T, nL, dL, (double2*)d_rho, d_eb, d_bands, true);
    dos_dev(ctx, H->n, nk, d_bands, d_w, nw, d_omegas, gamma, d_dos);
    timer_stop(ctx);
    double eb = 0.0;
    wait_stream(ctx);  // poll with the context's limit: a copy into pageable host memory would block unbounded
    ck(cudaMemcpyAsync(&eb, d_eb, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    wait_stream(ctx);
    timer_collect(ctx);
    if (eband) *eband = eb;
  });
}

int lqm_bands_dos_rho_multi_dev(lqm_ctx* ctx, int nmodels, const lqm_hops* const* H, int64_t nk,
                                const double* d_ks, const double* d_w, double mu, double T, const int64_t* nL,
                                const int64_t* const* Lkeys, double* const* d_rho, double* eband, int64_t nw,
                                const double* const* d_omegas, double gamma, double* const* d_dos,
                                double* const* d_bands) {
  return guarded(ctx, [&] {
    if (nmodels < 1 || nmodels > kMaxModels || !H || !nL || !Lkeys || !d_rho || !d_omegas || !d_dos || !d_bands ||
        nk < 1 || !d_ks || nw < 1)
      fail(LQM_EINVAL, "invalid arguments");
    if (!std::isfinite(mu) || !(T >= 0) || !std::isfinite(T) || !std::isfinite(gamma))
      fail(LQM_EINVAL, "invalid mu/T/gamma");
    const int d = H[0] ? H[0]->d : 0;
    int64_t per_k = 0;
    for (int m = 0; m < nmodels; ++m) {
      check_hops(H[m]);
      if (H[m]->d != d) fail(LQM_EINVAL, "models must share the key dimension");
      if (nL[m] < 1 || !Lkeys[m] || !d_rho[m] || !d_omegas[m] || !d_dos[m] || !d_bands[m])
        fail(LQM_EINVAL, "invalid arguments of model %d", m);
      per_k += 16 * H[m]->n * H[m]->n;
    }
    const double* dw = d_w ? d_w : uniform_weights(ctx, nk);
    // every model's rho_k of a chunk of k-points stays resident (24 GB per chunk)
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(nk, (int64_t)(24.0e9 / (double)per_k)));
    std::vector<double2*> rk(nmodels);
    std::vector<double*> bandsp(nmodels), ebk(nmodels);
    char* rbuf = (char*)ws_get(ctx, WS_RHOK, (size_t)(chunk * per_k) + 256 * (size_t)nmodels);
    double* ebuf = (double*)ws_get(ctx, WS_EBK, (size_t)(chunk * nmodels) * sizeof(double));
    double* sc = (double*)ws_get(ctx, WS_MISC, 64 * sizeof(double));  // [48 ..) band energy per model
    int64_t maxnl = 0;
    for (int m = 0; m < nmodels; ++m) maxnl = std::max(maxnl, nL[m]);
    double2* coef = (double2*)ws_get(ctx, WS_COEF, (size_t)(chunk * maxnl) * sizeof(double2));
    int64_t* dL = (int64_t*)ws_get(ctx, WS_LKEYS, (size_t)(nmodels * maxnl * d) * sizeof(int64_t));
    for (int m = 0; m < nmodels; ++m)
      ck(cudaMemcpyAsync(dL + m * maxnl * d, Lkeys[m], (size_t)(nL[m] * d) * sizeof(int64_t), cudaMemcpyHostToDevice,
                         ctx->stream),
         "H2D");
    size_t off = 0;
    for (int m = 0; m < nmodels; ++m) {
      rk[m] = (double2*)(rbuf + off);
      off += (size_t)(chunk * 16 * H[m]->n * H[m]->n + 255) / 256 * 256;
      ebk[m] = ebuf + m * chunk;
    }
    timer_start(ctx);
    for (int64_t k0 = 0; k0 < nk; k0 += chunk) {
      const int64_t nb = std::min(chunk, nk - k0);
      for (int m = 0; m < nmodels; ++m) bandsp[m] = d_bands[m] + k0 * H[m]->n;
      launch_eigh_multi(ctx, nmodels, H, nb, d_ks + k0 * d, bandsp.data(), rk.data(), ebk.data(), dw + k0, mu, T);
      for (int m = 0; m < nmodels; ++m) {
        const int64_t nn = H[m]->n * H[m]->n;
        ordered_sum_kernel<<<1, 256, 0, ctx->stream>>>(ebk[m], nb, sc + 48 + m, k0 > 0);
        fold_coef_kernel<<<(unsigned)std::min<int64_t>((nb * nL[m] + 255) / 256, 4096), 256, 0, ctx->stream>>>(
            nb, d, d_ks + k0 * d, dw + k0, (int)nL[m], dL + m * maxnl * d, coef);
        launch_fold(ctx, nn, nb, rk[m], coef, (int)nL[m], (double2*)d_rho[m], k0 > 0);
        ctx->launches += 2;
      }
    }
    for (int m = 0; m < nmodels; ++m) dos_dev(ctx, H[m]->n, nk, d_bands[m], d_w, nw, d_omegas[m], gamma, d_dos[m]);
    timer_stop(ctx);
    std::vector<double> eb((size_t)nmodels, 0.0);
    wait_stream(ctx);
    ck(cudaMemcpyAsync(eb.data(), sc + 48, (size_t)nmodels * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
       "D2H");
    wait_stream(ctx);
    timer_collect(ctx);
    if (eband)
      for (int m = 0; m < nmodels; ++m) eband[m] = eb[(size_t)m];
  });
}

int lqm_bands_dos_rho(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w, double mu,
                      double T, int64_t nL, const int64_t* Lkeys, double* rho, double* eband, int64_t nw,
                      const double* omegas, double gamma, double* dos, double* bands, int precision) {
  return guarded(ctx, [&] {
    check_hops(H);
    check_ks(ks, nk, H->d);
    if (!rho || !Lkeys || nL < 1 || nw < 1 || !omegas || !dos || !bands) fail(LQM_EINVAL, "invalid arguments");
    if (w) check_finite(w, nk, "w");
    check_finite(omegas, nw, "omegas");
    const int64_t n = H->n;
    const double* dks = upload(ctx, WS_KS, ks, (size_t)(nk * H->d));
    const double* dw = w ? upload(ctx, WS_W, w, (size_t)nk) : nullptr;
    const double* dom = upload(ctx, WS_OMEGA, omegas, (size_t)nw);
    const size_t rb = (size_t)(nL * n * n) * sizeof(double2);
    double* drho = (double*)ws_get(ctx, WS_RHO, rb);
    double* db = (double*)ws_get(ctx, WS_BANDS2, (size_t)(n * nk) * sizeof(double));
    double* dd = (double*)ws_get(ctx, WS_DOS, (size_t)nw * sizeof(double));
    int st = lqm_bands_dos_rho_dev(ctx, H, nk, dks, dw, mu, T, nL, Lkeys, drho, eband, nw, dom, gamma, dd, db,
                                   precision);
    if (st != LQM_OK) fail(st, "%s", ctx->err.c_str());
    ck(cudaMemcpyAsync(rho, drho, rb, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    ck(cudaMemcpyAsync(bands, db, (size_t)(n * nk) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    ck(cudaMemcpyAsync(dos, dd, (size_t)nw * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    wait_stream(ctx);
  });
}

}  // extern "C"

#include "lqm_commutator.inc"
#include "lqm_anderson.inc"
#include "lqm_scf.inc"
#include "lqm_adjoint.inc"
#include "lqm_scfgrad.inc"
#include "lqm_obs.inc"
#include "lqm_sitedos.inc"
#include "lqm_berry.inc"
#include "lqm_kubo.inc"
#include "lqm_partial.inc"
#include "lqm_bdg.inc"
#include "lqm_scf_bdg.inc"
#include "lqm_autotune.inc"

// ============================================================================
// Allocation-free eigen pass.
//
// For callers that cannot allocate device memory themselves or through this
// library: hosts whose device memory belongs to another allocator (a Julia
// CUDA.jl memory pool, a framework's caching allocator) and that must not see
// foreign cudaMalloc/cudaFree calls, or latency-sensitive loops that cannot
// afford the device-wide synchronisation cudaMalloc/cudaFree imply.  The
// caller passes every input and output as a device pointer and a stream; the
// eigensolver's scratch and its divide-and-conquer plan live in the two
// file-scope device arrays below, which every GPU that loads this library
// holds until the process exits.  No cudaMalloc, cudaFree or allocating
// library routine is called.
//
// Host code must not use the array names as addresses (on the host they are
// stand-ins, not device pointers): the first call on each device, with that
// device current, resolves their device addresses with cudaGetSymbolAddress
// and caches them; make that first call before any stream capture.  All calls
// share the arrays, so calls that overlap on the GPU race; serialise them
// (one stream, or events).  Each call writes every scratch entry it later
// reads and rebuilds the plan for its own n, so nothing has to start at zero.
// ============================================================================
namespace {

constexpr int64_t kNoAllocScratchBytes = (int64_t)64 << 20;  // 64 MiB of FP64 scratch per device
constexpr int64_t kNoAllocScratchDoubles = kNoAllocScratchBytes / 8;
constexpr int kNoAllocMaxN = 1024;                           // matrix order limit
constexpr int kNoAllocPlanInts = 16384;                      // >= dc_plan_ints(1024)

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];
static __device__ __align__(256) int g_noalloc_plan[kNoAllocPlanInts];

// Builds the divide-and-conquer plan for order n in place (device code may
// name the array directly).
__global__ void noalloc_plan_kernel(int n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) dc_plan_fill(n, g_noalloc_plan);
}

struct NoAllocDevice {
  bool ready = false;
  double* scratch = nullptr;
  int* plan = nullptr;
  int sms = 0;
};
std::mutex g_noalloc_mutex;
NoAllocDevice g_noalloc_dev[64];

}  // namespace

extern "C" int lqm_bandmatrix_noalloc(void* stream, int64_t n, int64_t nR, int32_t d, const int64_t* d_keys,
                                      const double* d_blocks, int64_t nk, const double* d_ks, double* d_bands,
                                      double* d_U) {
  if (n < 1 || n > kNoAllocMaxN || nR < 1 || nR > 4096 || d < 1 || d > 3 || nk < 1) return LQM_EINVAL;
  if (!d_keys || !d_blocks || !d_ks || !d_bands) return LQM_EINVAL;
  if (dc_plan_ints((int)n) > kNoAllocPlanInts) return LQM_EINVAL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return LQM_ECUDA;
  NoAllocDevice& D = g_noalloc_dev[dev];
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!D.ready) {  // once per device, with that device current
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return LQM_ECUDA;
      D.scratch = (double*)p;
      p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_plan) != cudaSuccess || !p) return LQM_ECUDA;
      D.plan = (int*)p;
      if (cudaDeviceGetAttribute(&D.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return LQM_ECUDA;
      D.ready = true;
    }
  }
  const int ni = (int)n;
  const int nt = eigh_threads(ni);
  EighSmemLayout Ls = eigh_smem_layout(ni, (int)nR, nt, 1);
  const int a_in_smem = Ls.total <= 225 * 1024;
  if (!a_in_smem) Ls = eigh_smem_layout(ni, (int)nR, nt, 0);
  if (Ls.total > 225 * 1024) return LQM_EINVAL;
  const int64_t slot = eigh_slot_doubles(ni, a_in_smem, false);
  const int64_t max_slots = kNoAllocScratchDoubles / slot;
  if (max_slots < 1) return LQM_EINVAL;  // one k-point's scratch exceeds the 64 MiB array
  const EighFn kfn = eigh_fn(nt);
  if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Ls.total) != cudaSuccess)
    return LQM_ECUDA;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, nt, Ls.total) != cudaSuccess ||
      per_sm < 1)
    return LQM_ECUDA;
  const int64_t grid = std::min<int64_t>(std::min<int64_t>(nk, (int64_t)per_sm * D.sms), max_slots);
  const int H = dc_plan_height(ni);
  const int nnodes = ni - 1;
  EighArgs a{};
  a.n = ni; a.nR = (int)nR; a.dim = d; a.blocks = (const double2*)d_blocks; a.keys = d_keys;
  a.nk = nk; a.ks = d_ks;
  a.plan.nnodes = nnodes;
  a.plan.nheights = H;
  a.plan.hstart = D.plan;
  a.plan.lo = D.plan + (H + 1);
  a.plan.mid = a.plan.lo + nnodes;
  a.plan.hi = a.plan.mid + nnodes;
  a.plan.owner = a.plan.hi + nnodes;
  a.scratch = D.scratch;
  a.slot_doubles = slot;
  a.a_in_smem = a_in_smem;
  a.bands = d_bands;
  a.U = (double2*)d_U;
  cudaStream_t st = (cudaStream_t)stream;
  noalloc_plan_kernel<<<1, 1, 0, st>>>(ni);
  kfn<<<(unsigned)grid, nt, Ls.total, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? LQM_OK : LQM_ECUDA;
}

