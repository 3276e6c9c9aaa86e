// CUDA kernels of the k-space hot path (sm_100a, FP64).
#pragma once
#include <cuda_runtime.h>
#include "lqm_eigh.cuh"

namespace lqm {

// Shared-memory layout of eigh_kernel for order n, nR hopping keys, nt threads.
// With a_in_smem the Hermitian matrix lives in shared memory (leading
// dimension n+1, so column-strided double2 accesses do not conflict); the same
// region later holds the divide-and-conquer Q/Qt pair and then U.
struct EighSmemLayout {
  size_t offA, offC, offD, offI, total;
  int a_in_smem, pbuf_len;
};

__host__ __device__ inline size_t lqm_align16(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline EighSmemLayout eigh_smem_layout(int n, int nR, int nt, int a_in_smem) {
  EighSmemLayout L;
  L.a_in_smem = a_in_smem;
  const int nw = nt / 32;
  L.pbuf_len = (nw * n > nt) ? nw * n : nt;
  if (L.pbuf_len < 8 * n + 128) L.pbuf_len = 8 * n + 128;  // blocked back-transformation: V (n x 8), T, G
  size_t off = 0;
  L.offA = off;
  if (a_in_smem) off += lqm_align16((size_t)n * (n + 1) * 16);
  L.offC = off;  // double2: tau, v, w, vn, pn (n each), bc (2), ph (nR), pbuf
  off += lqm_align16((size_t)(5 * n + 2 + nR + L.pbuf_len) * 16);
  L.offD = off;  // doubles: 13 n + 128 (red) + 4 (kpt)
  off += lqm_align16((size_t)(13 * n + 132) * 8);
  L.offI = off;  // ints: 10 n
  off += lqm_align16((size_t)(10 * n) * 4);
  L.total = off;
  return L;
}

// doubles of global scratch per CTA
__host__ __device__ inline int64_t eigh_slot_doubles(int n, int a_in_smem, bool need_uwork) {
  const int64_t nn = (int64_t)n * n;
  if (a_in_smem) return 3 * nn;                  // R (2nn) | Qs
  return 4 * nn + (need_uwork ? 2 * nn : 0);     // A (2nn) | Q | Qt | U work
}

struct EighArgs {
  int n, nR, dim;
  const double2* blocks;  // nR x n x n
  const int64_t* keys;    // dim x nR
  int64_t nk;             // k-points in this launch
  const double* ks;       // dim x nk
  DCPlan plan;
  double* scratch;        // gridDim.x slots
  int64_t slot_doubles;
  int a_in_smem;
  double* bands;          // n x nk
  double2* U;             // n x n x nk, or null
  double2* rhok;          // n x n x nk: U f(eps - mu) U^H, or null
  double* eband_k;        // nk: w_k sum_j f_j eps_j (with rhok)
  const double* w;        // nk weights (with rhok)
  double mu, T;
  unsigned long long* phase_cycles;  // [16] per-phase SM cycles summed over CTAs, or null
};

enum { PH_BLOCH = 0, PH_HETRD = 1, PH_DC = 2, PH_BACK = 3, PH_OUT = 4, PH_DCSUB = 5, PH_COUNT = 16 };

__device__ __forceinline__ double fermi(double x, double T) {
  if (T > 0.0) return 1.0 / (exp(x / T) + 1.0);
  return (-x < 0.0) ? 0.0 : ((-x > 0.0) ? 1.0 : 0.5);
}

__device__ __forceinline__ void carve_vectors(unsigned char* smem, const EighSmemLayout& L, int n, int nR,
                                              EighVec& S, double2** ph, double** kpt) {
  double2* cbuf = (double2*)(smem + L.offC);
  double* dbuf = (double*)(smem + L.offD);
  int* ibuf = (int*)(smem + L.offI);
  S.tau = cbuf; S.v = cbuf + n; S.w = cbuf + 2 * n; S.vn = cbuf + 3 * n; S.pn = cbuf + 4 * n;
  S.bc = cbuf + 5 * n;
  *ph = cbuf + 5 * n + 2;
  S.pbuf = cbuf + 5 * n + 2 + nR;
  S.d = dbuf; S.e = dbuf + n; S.D = dbuf + 2 * n; S.z = dbuf + 3 * n; S.dl = dbuf + 4 * n;
  S.zl = dbuf + 5 * n; S.troot = dbuf + 6 * n; S.zhat = dbuf + 7 * n; S.vals = dbuf + 8 * n;
  S.dval = dbuf + 9 * n; S.rc = dbuf + 10 * n; S.rs = dbuf + 11 * n; S.nrho = dbuf + 12 * n;
  S.red = dbuf + 13 * n;
  *kpt = dbuf + 13 * n + 128;
  S.perm = ibuf; S.colnd = ibuf + n; S.org = ibuf + 2 * n; S.dcol = ibuf + 3 * n; S.newpos = ibuf + 4 * n;
  S.ri = ibuf + 5 * n; S.rj = ibuf + 6 * n; S.nk = ibuf + 7 * n; S.nrot = ibuf + 8 * n; S.ndef = ibuf + 9 * n;
}

// Per-phase SM cycle accounting of the eigensolver (profiling mode only).
struct EighProf {
  bool on = false;
  unsigned long long acc[5] = {0, 0, 0, 0, 0};
  unsigned long long dsub[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long hsub[3] = {0, 0, 0};
  long long tc = 0;
  __device__ __forceinline__ void start() {
    if (on) tc = clock64();
  }
  __device__ __forceinline__ void tick(int ph) {
    if (on) {
      const long long t = clock64();
      acc[ph] += (unsigned long long)(t - tc);
      tc = t;
    }
  }
};

// The whole per-k computation of one team on its shared-memory region `smem` and
// global scratch slot: H(k), Householder, divide and conquer, bands, and (when
// asked) the eigenvectors and/or rho_k with the band energy.
template <class TeamT>
__device__ __forceinline__ void eigh_point(const TeamT& T, const EighArgs& a, int64_t k, unsigned char* smem,
                                           double* slot, EighProf& P) {
  const int n = a.n;
  const EighSmemLayout L = eigh_smem_layout(n, a.nR, T.nt, a.a_in_smem);
  EighVec S;
  double2* ph;
  double* kpt;
  carve_vectors(smem, L, n, a.nR, S, &ph, &kpt);
  const int64_t nn = (int64_t)n * n;
  const bool in_smem = a.a_in_smem != 0;
  const int lda = in_smem ? n + 1 : n;
  double2* A = in_smem ? (double2*)(smem + L.offA) : (double2*)slot;
  double2* R = in_smem ? (double2*)slot : A;          // reflectors, leading dimension ldr
  const int ldr = in_smem ? n : lda;
  double* Q = in_smem ? (double*)(smem + L.offA) : slot + 2 * nn;
  double* Qt = Q + nn;
  double* Qs = slot + 2 * nn;                         // smem path: saved Q
  const bool need_vec = (a.U != nullptr) || (a.rhok != nullptr);

  P.start();
  if (T.tid < a.dim) kpt[T.tid] = a.ks[k * a.dim + T.tid];
  team_sync(T);
  bloch_build(T, n, a.nR, a.dim, a.blocks, a.keys, kpt, ph, A, lda);
  P.tick(PH_BLOCH);
  hetrd_lower(T, n, A, lda, S, P.on ? P.hsub : nullptr);
  if (in_smem && need_vec) {
    for (int c = T.wid; c < n - 1; c += T.nw)
      for (int r = c + 1 + T.lane; r < n; r += T.nl) R[r + (int64_t)c * n] = A[r + (int64_t)c * lda];
    team_sync(T);
  }
  P.tick(PH_HETRD);
  dc_solve(T, n, a.plan, S, Q, Qt, P.on ? P.dsub : nullptr, need_vec);
  for (int i = T.tid; i < n; i += T.nt) a.bands[k * n + i] = S.D[i];
  P.tick(PH_DC);
  if (need_vec) {
    // Columns of U to form: all of them when U is an output; for rho_k alone only
    // the eigenvectors rho_from_U reads (its complement form skips the states with
    // f = 1, the direct form those with f = 0), a contiguous range since f falls
    // with the ascending eigenvalues.
    int cbeg = 0, cend = n;
    if (a.rhok) {
      double eb = 0.0;
      for (int j = T.tid; j < n; j += T.nt) {
        const double fj = fermi(S.D[j] - a.mu, a.T);
        S.vals[j] = fj;
        eb += S.D[j] * fj;
      }
      eb = team_sum(T, eb, S.red);  // (its barriers publish S.vals)
      if (T.tid == 0) a.eband_k[k] = a.w[k] * eb;
      if (!a.U) {
        int n0 = 0, n1 = 0;
        for (int j = 0; j < n; ++j) {
          n0 += (S.vals[j] == 0.0);
          n1 += (S.vals[j] == 1.0);
        }
        const double skip = (n1 > n0) ? 1.0 : 0.0;
        cbeg = n;
        cend = 0;
        for (int j = 0; j < n; ++j)
          if (S.vals[j] != skip) {
            cbeg = cbeg < j ? cbeg : j;
            cend = j + 1;
          }
        if (cend < cbeg) cend = cbeg;
      }
    }
    double2* U;
    int ldu;
    if (in_smem) {
      for (int c = cbeg + T.wid; c < cend; c += T.nw)
        for (int r = T.lane; r < n; r += T.nl) Qs[r + (int64_t)c * n] = Q[r + (int64_t)c * n];
      team_sync(T);
      U = (double2*)(smem + L.offA);
      ldu = n + 1;
      for (int c = cbeg + T.wid; c < cend; c += T.nw)
        for (int r = T.lane; r < n; r += T.nl) U[r + (int64_t)c * ldu] = cmk(Qs[r + (int64_t)c * n], 0.0);
    } else {
      U = a.U ? a.U + k * nn : (double2*)(slot + 4 * nn);
      ldu = n;
      for (int c = cbeg + T.wid; c < cend; c += T.nw)
        for (int r = T.lane; r < n; r += T.nl) U[r + (int64_t)c * ldu] = cmk(Q[r + (int64_t)c * n], 0.0);
    }
    team_sync(T);
    backtransform(T, n, R, ldr, S, U, ldu, cbeg, cend);
    P.tick(PH_BACK);
    if (in_smem && a.U) {
      double2* Uo = a.U + k * nn;
      for (int c = T.wid; c < n; c += T.nw)
        for (int r = T.lane; r < n; r += T.nl) Uo[r + (int64_t)c * n] = U[r + (int64_t)c * ldu];
    }
    if (a.rhok) rho_from_U(T, n, U, ldu, S.vals, a.rhok + k * nn, n);
  }
  team_sync(T);
  P.tick(PH_OUT);
}

template <int NT, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) eigh_kernel(EighArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Team T = make_team();
  double* slot = a.scratch + (int64_t)blockIdx.x * a.slot_doubles;
  EighProf P;
  P.on = a.phase_cycles != nullptr;
  for (int64_t k = blockIdx.x; k < a.nk; k += gridDim.x) eigh_point(T, a, k, smem, slot, P);
  if (P.on && T.tid == 0) {
    for (int i = 0; i < 5; ++i) atomicAdd(&a.phase_cycles[i], P.acc[i]);
    for (int i = 0; i < 8; ++i) atomicAdd(&a.phase_cycles[PH_DCSUB + i], P.dsub[i]);
    for (int i = 0; i < 3; ++i) atomicAdd(&a.phase_cycles[PH_DCSUB + 8 + i], P.hsub[i]);
  }
}

// Several models of uneven order in ONE launch.  Model m's k-points go to teams of
// team_nt[m] threads (its one-CTA block size), blockDim.x / team_nt[m] teams per CTA,
// each on its own shared-memory region (smem_team[m] bytes) and scratch slot; a work
// item is one k-point per team of a CTA.  Items are numbered model after model
// (item_begin[m] ..), and the CTAs take them round-robin, so the small orders fill
// the SMs as the large ones drain.  Teams synchronise on named barriers.
constexpr int kMaxModels = 4;
struct EighMultiArgs {
  int nmodels;
  EighArgs m[kMaxModels];
  int team_nt[kMaxModels];
  int64_t smem_team[kMaxModels];
  int64_t item_begin[kMaxModels + 1];
  int64_t slots_per_cta;  // scratch slots per CTA (the largest team count)
};

template <int NT>
__global__ void __launch_bounds__(NT, 1) eigh_multi_kernel(EighMultiArgs ma) {
  extern __shared__ __align__(16) unsigned char smem[];
  EighProf P;
  for (int64_t it = blockIdx.x; it < ma.item_begin[ma.nmodels]; it += gridDim.x) {
    int mdl = 0;
    while (it >= ma.item_begin[mdl + 1]) ++mdl;
    const EighArgs& a = ma.m[mdl];
    const int tnt = ma.team_nt[mdl];
    const int nteams = NT / tnt;
    const int team = threadIdx.x / tnt;
    const int64_t k = (it - ma.item_begin[mdl]) * nteams + team;
    double* slot = a.scratch + ((int64_t)blockIdx.x * ma.slots_per_cta + team) * a.slot_doubles;
    if (tnt == NT) {
      eigh_point(make_team(), a, k, smem, slot, P);
    } else if (k < a.nk) {
      eigh_point(make_subteam(tnt), a, k, smem + team * ma.smem_team[mdl], slot, P);
    }
    __syncthreads();  // every team is done with the CTA's shared memory before the next item
  }
}

// Batched Bloch sum to HBM: Hk[k] = sum_R H_R exp(i 2 pi k.R); one CTA per k.
__global__ void __launch_bounds__(256) bloch_kernel(int n, int nR, int dim, const double2* __restrict__ blocks,
                                                    const int64_t* __restrict__ keys, int64_t nk,
                                                    const double* __restrict__ ks, double2* __restrict__ Hk) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* ph = (double2*)smem;
  const int64_t nn = (int64_t)n * n;
  for (int64_t k = blockIdx.x; k < nk; k += gridDim.x) {
    for (int r = threadIdx.x; r < nR; r += blockDim.x) {
      double dot = 0.0;
      for (int c = 0; c < dim; ++c) dot += ks[k * dim + c] * (double)keys[(int64_t)r * dim + c];
      double s, co;
      sincospi(2.0 * dot, &s, &co);
      ph[r] = cmk(co, s);
    }
    __syncthreads();
    double2* out = Hk + k * nn;
    for (int64_t idx = threadIdx.x; idx < nn; idx += blockDim.x) {
      double2 acc = cmk(0.0, 0.0);
      for (int r = 0; r < nR; ++r) acc = cadd(acc, cmul(__ldg(&blocks[(int64_t)r * nn + idx]), ph[r]));
      out[idx] = acc;
    }
    __syncthreads();
  }
}

// rho_k = U diag(f) U^H per k from eigenvectors in HBM; eband_k = w_k sum_j f_j eps_j.
__global__ void __launch_bounds__(256) rhok_kernel(int n, int64_t nk, const double2* __restrict__ U,
                                                   const double* __restrict__ bands, double mu_val,
                                                   const double* mu_ptr, double T,
                                                   const double* __restrict__ w, double2* __restrict__ rhok,
                                                   double* __restrict__ eband_k) {
  extern __shared__ __align__(16) unsigned char smem[];
  const double mu = mu_ptr ? *mu_ptr : mu_val;  // device-resident mu (SCF) or a host value
  double* f = (double*)smem;
  double* red = f + n;
  const Team Tm = make_team();
  const int64_t nn = (int64_t)n * n;
  for (int64_t k = blockIdx.x; k < nk; k += gridDim.x) {
    double eb = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      const double e = bands[k * n + j];
      const double fj = fermi(e - mu, T);
      f[j] = fj;
      eb += e * fj;
    }
    eb = team_sum(Tm, eb, red);
    if (threadIdx.x == 0) eband_k[k] = w[k] * eb;
    rho_from_U(Tm, n, U + k * nn, n, f, rhok + k * nn, n);
  }
}

// coef[kb*nL + l] = w_k exp(-i 2 pi k.L_l)
__global__ void fold_coef_kernel(int64_t nb, int dim, const double* __restrict__ ks, const double* __restrict__ w,
                                 int nL, const int64_t* __restrict__ Lkeys, double2* __restrict__ coef) {
  const int64_t tot = nb * nL;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t kb = t / nL;
    const int l = (int)(t % nL);
    double dot = 0.0;
    for (int c = 0; c < dim; ++c) dot += ks[kb * dim + c] * (double)Lkeys[(int64_t)l * dim + c];
    double s, co;
    sincospi(2.0 * dot, &s, &co);
    coef[t] = cmk(w[kb] * co, -w[kb] * s);
  }
}

// SparseHops upload (SparseMatrixCSC blocks, 1-based, validated on the host): one
// thread per column adds its stored entries into the zeroed dense block in storage
// order, so repeated (row, column) entries sum in the same order as a host loop.
__global__ void __launch_bounds__(128) csc_scatter_kernel(int64_t n, const int64_t* __restrict__ colptr,
                                                          const int64_t* __restrict__ rowval,
                                                          const double2* __restrict__ nzval, double2* block) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  double2* col = block + j * n;
  for (int64_t p = colptr[j] - 1; p < colptr[j + 1] - 1; ++p) {
    const int64_t i = rowval[p] - 1;
    const double2 v = nzval[p];
    double2 c = col[i];
    c.x += v.x;
    c.y += v.y;
    col[i] = c;
  }
}

// Fixed-order sum of x[0..m) into out[0] (single CTA).
__global__ void ordered_sum_kernel(const double* __restrict__ x, int64_t m, double* out, int accumulate) {
  __shared__ double red[32];
  const Team Tm = make_team();
  // contiguous chunks per thread, then a deterministic team reduction
  const int64_t chunk = (m + blockDim.x - 1) / blockDim.x;
  double s = 0.0;
  const int64_t b = threadIdx.x * chunk, e = (b + chunk < m) ? b + chunk : m;
  for (int64_t i = b; i < e; ++i) s += x[i];
  s = team_sum(Tm, s, red);
  if (threadIdx.x == 0) out[0] = accumulate ? out[0] + s : s;
}

// DOS: partial[b*nw + i] = sum over this block's values of w * Gamma/((omega_i - eps)^2 + Gamma^2)
__global__ void __launch_bounds__(256) dos_partial_kernel(const double* __restrict__ bands, int n, int64_t nvals,
                                                          const double* __restrict__ w, int nw,
                                                          const double* __restrict__ omegas, double gamma,
                                                          int64_t chunk, double* __restrict__ partial) {
  __shared__ double ev[1024];
  __shared__ double ew[1024];
  const int64_t b0 = blockIdx.x * chunk;
  const int64_t b1 = (b0 + chunk < nvals) ? b0 + chunk : nvals;
  const double g2 = gamma * gamma;
  for (int i0 = 0; i0 < nw; i0 += blockDim.x) {
    const int i = i0 + threadIdx.x;
    const double om = (i < nw) ? omegas[i] : 0.0;
    double acc = 0.0;
    for (int64_t t0 = b0; t0 < b1; t0 += 1024) {
      const int cnt = (int)((t0 + 1024 < b1) ? 1024 : (b1 - t0));
      __syncthreads();
      for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        ev[t] = bands[t0 + t];
        ew[t] = w ? w[(t0 + t) / n] : 1.0;
      }
      __syncthreads();
      if (i < nw) {
        for (int t = 0; t < cnt; ++t) {
          const double x = om - ev[t];
          acc += ew[t] * gamma / (x * x + g2);
        }
      }
    }
    if (i < nw) partial[(int64_t)blockIdx.x * nw + i] = acc;
  }
}

__global__ void dos_reduce_kernel(const double* __restrict__ partial, int nb, int nw, double scale,
                                  double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += partial[(int64_t)b * nw + i];
    out[i] = s * scale;
  }
}

// ---------------------------------------------------------------------------
// Chemical potential: bisection over the float64 order (Roots.jl Bisection).
// ---------------------------------------------------------------------------
struct MuState {
  double a, b, fa, fb, x, result;
  long long target;  // order-statistic search: wanted count
  int phase, done, iters, err;
};

__device__ __forceinline__ double float_mid(double a, double b) {
  if ((a < 0.0 && b > 0.0) || (b < 0.0 && a > 0.0)) return 0.0;
  unsigned long long ua = (unsigned long long)__double_as_longlong(fabs(a));
  unsigned long long ub = (unsigned long long)__double_as_longlong(fabs(b));
  double m = __longlong_as_double((long long)((ua + ub) >> 1));
  return (a + b < 0.0) ? -m : m;
}

__global__ void minmax_kernel(const double* __restrict__ x, int64_t m, double* out /* min, max */) {
  __shared__ double rmin[32], rmax[32];
  double lo = INFINITY, hi = -INFINITY;
  for (int64_t i = threadIdx.x; i < m; i += blockDim.x) { lo = fmin(lo, x[i]); hi = fmax(hi, x[i]); }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) { rmin[threadIdx.x >> 5] = lo; rmax[threadIdx.x >> 5] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { lo = fmin(lo, rmin[w]); hi = fmax(hi, rmax[w]); }
    lo = fmin(lo, rmin[0]); hi = fmax(hi, rmax[0]);
    out[0] = lo; out[1] = hi;
  }
}

__global__ void mu_init_kernel(MuState* st, const double* mm) {
  st->a = mm[0]; st->b = mm[1]; st->fa = st->fb = 0.0; st->x = mm[0]; st->result = 0.0;
  st->phase = 0; st->done = 0; st->iters = 0; st->err = 0;
}

// partial[b] = sum over block b's chunk of weight * f(v - x)
__global__ void __launch_bounds__(256) filling_partial_kernel(const double* __restrict__ bands, int n,
                                                              int64_t nvals, const double* __restrict__ w,
                                                              const MuState* st, double T, int64_t chunk,
                                                              double* __restrict__ partial) {
  __shared__ double red[32];
  if (st->done) return;
  const Team Tm = make_team();
  const double x = st->x;
  const int64_t b0 = blockIdx.x * chunk;
  const int64_t b1 = (b0 + chunk < nvals) ? b0 + chunk : nvals;
  double s = 0.0;
  for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
    const double f = fermi(bands[i] - x, T);
    s += w ? w[i / n] * f : f;
  }
  s = team_sum(Tm, s, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__device__ __forceinline__ double sgn(double v) { return (v > 0.0) - (v < 0.0); }

__global__ void mu_update_kernel(const double* __restrict__ partial, int nb, MuState* st, double filling,
                                 double norm) {
  if (threadIdx.x != 0 || st->done) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += partial[b];
  const double g = s * norm - filling;
  st->iters++;
  if (st->phase == 0) {
    st->fa = g;
    if (g == 0.0) { st->result = st->a; st->done = 1; return; }
    st->phase = 1; st->x = st->b; return;
  }
  if (st->phase == 1) {
    st->fb = g;
    if (g == 0.0) { st->result = st->b; st->done = 1; return; }
    if (sgn(st->fa) == sgn(st->fb)) { st->err = 1; st->result = NAN; st->done = 1; return; }
    st->phase = 2;
  } else {
    if (g == 0.0) { st->result = st->x; st->done = 1; return; }
    if (sgn(g) == sgn(st->fa)) { st->a = st->x; st->fa = g; } else { st->b = st->x; st->fb = g; }
  }
  const double m = float_mid(st->a, st->b);
  if (m == st->a || m == st->b || st->iters > 200) {
    st->result = (fabs(st->fa) <= fabs(st->fb)) ? st->a : st->b;
    st->done = 1;
    return;
  }
  st->x = m;
}

// mu result of a finished bisection into out; err accumulates 1 (no sign
// change) or 2 (not terminated).
__global__ void mu_store_kernel(const MuState* st, double* out, double* err) {
  if (threadIdx.x != 0) return;
  *out = st->result;
  if (st->err) *err += 1.0;
  else if (!st->done) *err += 2.0;
}

// filling >= 1: mu = max eps; filling <= 0: mu = min eps - 1 (chemicalpotential.jl:12-17)
__global__ void mu_special_kernel(const double* mm, double* out, int upper) {
  if (threadIdx.x == 0) *out = upper ? mm[1] : mm[0] - 1.0;
}

__global__ void mu_avg_kernel(const double* a, const double* b, double* out) {
  if (threadIdx.x == 0) *out = (*a + *b) / 2;
}

// Order statistic (T = 0): smallest float x in [min,max] with #{v <= x} >= target.
__global__ void __launch_bounds__(256) count_partial_kernel(const double* __restrict__ v, int64_t m,
                                                            const MuState* st, int64_t chunk,
                                                            long long* __restrict__ partial) {
  __shared__ long long red[32];
  if (st->done) return;
  const double x = st->x;
  const int64_t b0 = blockIdx.x * chunk;
  const int64_t b1 = (b0 + chunk < m) ? b0 + chunk : m;
  long long c = 0;
  for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) c += (v[i] <= x);
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
}

__global__ void os_init_kernel(MuState* st, const double* mm, long long target) {
  st->a = mm[0]; st->b = mm[1]; st->x = mm[0]; st->target = target;
  st->phase = 0; st->done = 0; st->iters = 0; st->err = 0; st->result = 0.0;
}

__global__ void os_update_kernel(const long long* __restrict__ partial, int nb, MuState* st) {
  if (threadIdx.x != 0 || st->done) return;
  long long c = 0;
  for (int b = 0; b < nb; ++b) c += partial[b];
  const bool ge = c >= st->target;
  st->iters++;
  if (st->phase == 0) {  // evaluated at min
    if (ge) { st->result = st->a; st->done = 1; return; }
    st->phase = 1;
  } else {
    if (ge) st->b = st->x; else st->a = st->x;
  }
  const double m = float_mid(st->a, st->b);
  if (m == st->a || m == st->b || st->iters > 200) { st->result = st->b; st->done = 1; return; }
  st->x = m;
}

}  // namespace lqm
