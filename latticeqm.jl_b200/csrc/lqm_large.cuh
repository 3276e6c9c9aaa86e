// Batched blocked eigensolver kernels for orders beyond the one-CTA shared-
// memory plan (n up to a few thousand).  A batch of B k-points is reduced
// together, one launch per column step:
//
//   blk_bloch_kernel    H(k) (full Hermitian, from the upper triangle), CTA per k
//   blk_column_kernel   zlatrd column step (lqm_blocked.cuh), CTA per k
//   blk_gemv_kernel     w = tau (A22 v - corrections), 128-row slabs x k
//   blk_finish_kernel   last w of a panel, CTA per k
//   (host)              rank-2nb trailing update, batched ZGEMM
//   dc_large_kernel     divide and conquer per k (vectors in global memory,
//                       tiled merge updates), writes bands and Z (complex)
//   blk_prep_kernel / blk_larft_kernel   compact WY factors per panel
//   (host)              U = (I - V T V^H) U per panel, batched ZGEMMs
//   blk_scale_f_kernel  Y = U diag(f), band energy; (host) rho_k = Y U^H
#pragma once
#include "lqm_blocked.cuh"
#include "lqm_kernels.cuh"

namespace lqm {

constexpr int kBlkNB = 32;      // panel width (reflectors per panel)
constexpr int kBlkRows = 128;   // rows per mat-vec CTA (4 per lane)
constexpr int kBlkThreads = 256;
constexpr int kDcThreads = 512;
constexpr int kDcTileMin = 160; // merges with at least this many rows use the tiled update

struct BlkArgs {
  int n, nb;
  double2* A;    // B x (n x n)
  double2* W;    // B x (n x nb)
  double2* tau;  // B x n
  double* d;     // B x n
  double* e;     // B x n
  double2* t12;  // B x 2nb
};

__global__ void __launch_bounds__(kBlkThreads) blk_bloch_kernel(int n, int nR, int dim,
                                                                const double2* __restrict__ blocks,
                                                                const int64_t* __restrict__ keys, int64_t nk,
                                                                const double* __restrict__ ks, double2* A) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* ph = (double2*)smem;
  double* kpt = (double*)(ph + nR);
  const Team T = make_team();
  const int64_t k = blockIdx.x;
  if (T.tid < dim) kpt[T.tid] = ks[k * dim + T.tid];
  team_sync();
  bloch_build(T, n, nR, dim, blocks, keys, kpt, ph, A + k * (int64_t)n * n, n);
}

__global__ void __launch_bounds__(kBlkThreads) blk_column_kernel(BlkArgs a, int j0, int i) {
  __shared__ double red[128];
  const Team T = make_team();
  const int64_t b = blockIdx.x;
  const int n = a.n;
  blk_column(T, n, a.nb, j0, i, a.A + b * (int64_t)n * n, n, a.W + b * (int64_t)n * a.nb, n, a.tau + b * n,
             a.d + b * n, a.e + b * n, a.t12 + b * 2 * a.nb, red);
}

__global__ void __launch_bounds__(kBlkThreads) blk_finish_kernel(BlkArgs a, int jp, int ip) {
  __shared__ double red[128];
  const Team T = make_team();
  const int64_t b = blockIdx.x;
  const int n = a.n;
  blk_finish_w(T, n, jp, ip, a.A + b * (int64_t)n * n, n, a.W + b * (int64_t)n * a.nb, n, a.tau + b * n, red);
}

// grid (ceil((n-j-1)/kBlkRows), B); dynamic smem: vs (n-j-1) | part (nw x 128), double2
__global__ void __launch_bounds__(kBlkThreads) blk_gemv_kernel(BlkArgs a, int j0, int i) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Team T = make_team();
  const int n = a.n, j = j0 + i;
  const int m = n - j - 1;
  double2* vs = (double2*)smem;
  double2* part = vs + m;
  const int64_t b = blockIdx.y;
  const int r0 = j + 1 + blockIdx.x * kBlkRows;
  const int r1 = (r0 + kBlkRows < n) ? r0 + kBlkRows : n;
  blk_gemv_rows(T, n, a.nb, j0, i, r0, r1, a.A + b * (int64_t)n * n, n, a.W + b * (int64_t)n * a.nb, n,
                a.tau + b * n, a.t12 + b * 2 * a.nb, vs, part);
}

__global__ void __launch_bounds__(kBlkThreads) blk_prep_kernel(int n, double2* A) {
  const Team T = make_team();
  blk_prep_reflectors(T, n, A + (int64_t)blockIdx.x * n * n, n);
}

// grid (P, B); Tm: B x P x (nb x nb); dynamic smem: G (nb x nb double2)
__global__ void __launch_bounds__(kBlkThreads) blk_larft_kernel(int n, int nb, int P, const double2* A,
                                                                const double2* tau, double2* Tm) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Team T = make_team();
  const int p = blockIdx.x;
  const int64_t b = blockIdx.y;
  const int j0 = p * nb;
  int nbr = n - 1 - j0;
  if (nbr > nb) nbr = nb;
  double2* Tp = Tm + (b * P + p) * (int64_t)nb * nb;
  if (nbr <= 0) {
    for (int q = T.tid; q < nb * nb; q += T.nt) Tp[q] = cmk(0.0, 0.0);
    return;
  }
  blk_larft(T, n, nb, j0, nbr, A + b * (int64_t)n * n, n, tau + b * n, Tp, (double2*)smem);
}

struct DCLargeArgs {
  int n;
  int64_t nk;
  DCPlan plan;
  const double* d;   // nk x n (hetrd diagonal)
  const double* e;   // nk x n (subdiagonal, n-1 used)
  double* bands;     // nk x n
  double2* U;        // nk x (n x n): Z as complex, or null (eigenvalues only)
  double* slots;     // gridDim.x slots
  int64_t slot_doubles;
};

__host__ __device__ inline int64_t dc_large_slot_doubles(int n, bool vec) {
  const int64_t nn = (int64_t)n * n;
  const int64_t vecs = 13 * (int64_t)n + 8 + (10 * (int64_t)n + 1) / 2 + 1 + (int64_t)(kDcThreads / 32) * n + 2;
  return (vec ? 3 * nn : 4 * (int64_t)n + 4) + vecs;
}

__global__ void __launch_bounds__(kDcThreads) dc_large_kernel(DCLargeArgs a) {
  __shared__ double red[128];
  __shared__ __align__(16) double tile[2048];
  const Team T = make_team();
  const int n = a.n;
  const bool vec = a.U != nullptr;
  const int64_t nn = (int64_t)n * n;
  double* slot = a.slots + (int64_t)blockIdx.x * a.slot_doubles;
  double* Q = slot;
  double* Qt = vec ? Q + nn : nullptr;
  double* Ub = vec ? Q + 2 * nn : nullptr;
  double* db = slot + (vec ? 3 * nn : 4 * (int64_t)n + 4);
  EighVec S;
  S.d = db; S.e = db + n; S.D = db + 2 * n; S.z = db + 3 * n; S.dl = db + 4 * n; S.zl = db + 5 * n;
  S.troot = db + 6 * n; S.zhat = db + 7 * n; S.vals = db + 8 * n; S.dval = db + 9 * n; S.rc = db + 10 * n;
  S.rs = db + 11 * n; S.nrho = db + 12 * n;
  S.red = red;
  int* ib = (int*)(db + 13 * (int64_t)n + 8);
  S.perm = ib; S.colnd = ib + n; S.org = ib + 2 * n; S.dcol = ib + 3 * n; S.newpos = ib + 4 * n;
  S.ri = ib + 5 * n; S.rj = ib + 6 * n; S.nk = ib + 7 * n; S.nrot = ib + 8 * n; S.ndef = ib + 9 * n;
  double* pb = db + 13 * (int64_t)n + 8 + (10 * (int64_t)n + 1) / 2 + 1;
  S.pbuf = (double2*)(((uintptr_t)pb + 15) & ~(uintptr_t)15);
  S.tau = S.v = S.w = S.vn = S.pn = S.bc = nullptr;
  S.tile = tile;
  for (int64_t k = blockIdx.x; k < a.nk; k += gridDim.x) {
    for (int i = T.tid; i < n; i += T.nt) {
      S.d[i] = a.d[k * n + i];
      S.e[i] = (i < n - 1) ? a.e[k * n + i] : 0.0;
    }
    team_sync();
    dc_solve(T, n, a.plan, S, Q, Qt, nullptr, vec, Ub, kDcTileMin);
    for (int i = T.tid; i < n; i += T.nt) a.bands[k * n + i] = S.D[i];
    if (vec) {
      double2* Uk = a.U + k * nn;
      for (int c = T.wid; c < n; c += T.nw)
        for (int r = T.lane; r < n; r += T.nl) Uk[r + (int64_t)c * n] = cmk(Q[r + (int64_t)c * n], 0.0);
    }
    team_sync();
  }
}

// Y[k] = U[k] diag(f(eps - mu)) and eband_k = w_k sum_j f_j eps_j; CTA per k.
__global__ void __launch_bounds__(kBlkThreads) blk_scale_f_kernel(int n, int64_t nk, const double2* U,
                                                                  const double* bands, double mu_val,
                                                                  const double* mu_ptr, double T_,
                                                                  const double* w, double2* Y,
                                                                  double* eband_k) {
  __shared__ double red[128];
  extern __shared__ __align__(16) unsigned char smem[];
  double* f = (double*)smem;
  const Team T = make_team();
  const int64_t k = blockIdx.x;
  const double mu = mu_ptr ? *mu_ptr : mu_val;
  const int64_t nn = (int64_t)n * n;
  double eb = 0.0;
  for (int j = T.tid; j < n; j += T.nt) {
    const double ej = bands[k * n + j];
    const double fj = fermi(ej - mu, T_);
    f[j] = fj;
    eb += ej * fj;
  }
  eb = team_sum(T, eb, red);
  if (T.tid == 0 && eband_k) eband_k[k] = w[k] * eb;
  for (int c = T.wid; c < n; c += T.nw) {
    const double fc = f[c];
    for (int r = T.lane; r < n; r += T.nl) Y[k * nn + r + (int64_t)c * n] = cscale(fc, U[k * nn + r + (int64_t)c * n]);
  }
}

}  // namespace lqm
