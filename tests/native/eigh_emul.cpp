// Host build of the per-k eigensolver team code (one thread, one lane).
//
// Test infrastructure: lets the CPU suite exercise the exact index
// arithmetic of bloch_build / hetrd_lower / dc_solve / backtransform from
// latticeqm.jl_b200/csrc/lqm_eigh.cuh against LAPACK, without a GPU.
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <vector>
#include <atomic>
#include <chrono>
#include <random>
#include <thread>

#include "lqm_blocked.cuh"
#include "lqm_twostage.cuh"
#include "lqm_eigh.cuh"
#include "lqm_plan.h"

extern "C" int lqm_emul_eigh(int n, int nR, int dim, const double* blocks, const int64_t* keys, const double* kpt,
                             int want_vectors, double* evals, double* U, double* tri_d, double* tri_e) {
  const Team T = make_host_team();
  const lqm::DCPlanHost PH = lqm::make_dc_plan_host(n);
  DCPlan P;
  P.nnodes = PH.nnodes;
  P.nheights = PH.nheights;
  P.hstart = PH.buf.data() + PH.off_hstart;
  P.lo = PH.buf.data() + PH.off_lo;
  P.mid = PH.buf.data() + PH.off_mid;
  P.hi = PH.buf.data() + PH.off_hi;
  P.owner = PH.buf.data() + PH.off_own;

  const size_t nn = (size_t)n * n;
  const int lda = n + 1;  // padded leading dimension, as the shared-memory path
  std::vector<double2> A((size_t)n * lda), cbuf(5 * n + 2 + nR + 8 * n + 256 + 128);
  std::vector<double> dbuf(13 * (size_t)n + 132), Q(nn), Qt(nn);
  std::vector<int> ibuf(10 * (size_t)n);
  EighVec S;
  S.tau = cbuf.data(); S.v = S.tau + n; S.w = S.tau + 2 * n; S.vn = S.tau + 3 * n; S.pn = S.tau + 4 * n;
  S.bc = S.tau + 5 * n;
  double2* ph = S.tau + 5 * n + 2;
  S.pbuf = ph + nR;
  double* db = dbuf.data();
  S.d = db; S.e = db + n; S.D = db + 2 * n; S.z = db + 3 * n; S.dl = db + 4 * n; S.zl = db + 5 * n;
  S.troot = db + 6 * n; S.zhat = db + 7 * n; S.vals = db + 8 * n; S.dval = db + 9 * n; S.rc = db + 10 * n;
  S.rs = db + 11 * n; S.nrho = db + 12 * n; S.red = db + 13 * n;
  int* ib = ibuf.data();
  S.perm = ib; S.colnd = ib + n; S.org = ib + 2 * n; S.dcol = ib + 3 * n; S.newpos = ib + 4 * n;
  S.ri = ib + 5 * n; S.rj = ib + 6 * n; S.nk = ib + 7 * n; S.nrot = ib + 8 * n; S.ndef = ib + 9 * n;

  bloch_build(T, n, nR, dim, (const double2*)blocks, keys, kpt, ph, A.data(), lda);
  hetrd_lower(T, n, A.data(), lda, S);
  if (tri_d) std::memcpy(tri_d, S.d, sizeof(double) * n);
  if (tri_e && n > 1) std::memcpy(tri_e, S.e, sizeof(double) * (n - 1));
  dc_solve(T, n, P, S, Q.data(), Qt.data());
  std::memcpy(evals, S.D, sizeof(double) * n);
  if (want_vectors) {
    double2* Uc = (double2*)U;
    for (int c = 0; c < n; ++c)
      for (int r = 0; r < n; ++r) Uc[r + (size_t)c * n] = cmk(Q[r + (size_t)c * n], 0.0);
    backtransform(T, n, A.data(), lda, S, Uc, n);
  }
  return 0;
}

// The eigen pass with the back-transformation restricted to the columns
// [cbeg, cend) of U (the rho-only path of the kernel); other columns are left zero.
extern "C" int lqm_emul_eigh_cols(int n, int nR, int dim, const double* blocks, const int64_t* keys,
                                  const double* kpt, int cbeg, int cend, double* evals, double* U) {
  lqm_emul_eigh(n, nR, dim, blocks, keys, kpt, 0, evals, nullptr, nullptr, nullptr);
  const Team T = make_host_team();
  const lqm::DCPlanHost PH = lqm::make_dc_plan_host(n);
  DCPlan P;
  P.nnodes = PH.nnodes;
  P.nheights = PH.nheights;
  P.hstart = PH.buf.data() + PH.off_hstart;
  P.lo = PH.buf.data() + PH.off_lo;
  P.mid = PH.buf.data() + PH.off_mid;
  P.hi = PH.buf.data() + PH.off_hi;
  P.owner = PH.buf.data() + PH.off_own;
  const size_t nn = (size_t)n * n;
  const int lda = n + 1;
  std::vector<double2> A((size_t)n * lda), cbuf(5 * n + 2 + nR + 8 * n + 256 + 128);
  std::vector<double> dbuf(13 * (size_t)n + 132), Q(nn), Qt(nn);
  std::vector<int> ibuf(10 * (size_t)n);
  EighVec S;
  S.tau = cbuf.data(); S.v = S.tau + n; S.w = S.tau + 2 * n; S.vn = S.tau + 3 * n; S.pn = S.tau + 4 * n;
  S.bc = S.tau + 5 * n;
  double2* ph = S.tau + 5 * n + 2;
  S.pbuf = ph + nR;
  double* db = dbuf.data();
  S.d = db; S.e = db + n; S.D = db + 2 * n; S.z = db + 3 * n; S.dl = db + 4 * n; S.zl = db + 5 * n;
  S.troot = db + 6 * n; S.zhat = db + 7 * n; S.vals = db + 8 * n; S.dval = db + 9 * n; S.rc = db + 10 * n;
  S.rs = db + 11 * n; S.nrho = db + 12 * n; S.red = db + 13 * n;
  int* ib = ibuf.data();
  S.perm = ib; S.colnd = ib + n; S.org = ib + 2 * n; S.dcol = ib + 3 * n; S.newpos = ib + 4 * n;
  S.ri = ib + 5 * n; S.rj = ib + 6 * n; S.nk = ib + 7 * n; S.nrot = ib + 8 * n; S.ndef = ib + 9 * n;
  bloch_build(T, n, nR, dim, (const double2*)blocks, keys, kpt, ph, A.data(), lda);
  hetrd_lower(T, n, A.data(), lda, S);
  dc_solve(T, n, P, S, Q.data(), Qt.data());
  double2* Uc = (double2*)U;
  for (size_t e = 0; e < nn; ++e) Uc[e] = cmk(0.0, 0.0);
  for (int c = cbeg; c < cend; ++c)
    for (int r = 0; r < n; ++r) Uc[r + (size_t)c * n] = cmk(Q[r + (size_t)c * n], 0.0);
  backtransform(T, n, A.data(), lda, S, Uc, n, cbeg, cend);
  return 0;
}

// D&C alone on a given symmetric tridiagonal (d, e): eigenvalues and Z.
extern "C" int lqm_emul_tridiag(int n, const double* d, const double* e, double* evals, double* Z, int vec) {
  const Team T = make_host_team();
  const lqm::DCPlanHost PH = lqm::make_dc_plan_host(n);
  DCPlan P;
  P.nnodes = PH.nnodes;
  P.nheights = PH.nheights;
  P.hstart = PH.buf.data() + PH.off_hstart;
  P.lo = PH.buf.data() + PH.off_lo;
  P.mid = PH.buf.data() + PH.off_mid;
  P.hi = PH.buf.data() + PH.off_hi;
  P.owner = PH.buf.data() + PH.off_own;
  const size_t nn = (size_t)n * n;
  std::vector<double> dbuf(13 * (size_t)n + 132), Qt(nn);
  std::vector<int> ibuf(10 * (size_t)n);
  std::vector<double2> cbuf(5 * n + 2 + 8 * n + 256 + 128);
  EighVec S;
  S.tau = cbuf.data(); S.v = S.tau + n; S.w = S.tau + 2 * n; S.vn = S.tau + 3 * n; S.pn = S.tau + 4 * n;
  S.bc = S.tau + 5 * n; S.pbuf = S.bc + 2;
  double* db = dbuf.data();
  S.d = db; S.e = db + n; S.D = db + 2 * n; S.z = db + 3 * n; S.dl = db + 4 * n; S.zl = db + 5 * n;
  S.troot = db + 6 * n; S.zhat = db + 7 * n; S.vals = db + 8 * n; S.dval = db + 9 * n; S.rc = db + 10 * n;
  S.rs = db + 11 * n; S.nrho = db + 12 * n; S.red = db + 13 * n;
  int* ib = ibuf.data();
  S.perm = ib; S.colnd = ib + n; S.org = ib + 2 * n; S.dcol = ib + 3 * n; S.newpos = ib + 4 * n;
  S.ri = ib + 5 * n; S.rj = ib + 6 * n; S.nk = ib + 7 * n; S.nrot = ib + 8 * n; S.ndef = ib + 9 * n;
  std::memcpy(S.d, d, sizeof(double) * n);
  if (n > 1) std::memcpy(S.e, e, sizeof(double) * (n - 1));
  std::vector<double> rows(4 * (size_t)n + 4);
  dc_solve(T, n, P, S, vec ? Z : rows.data(), Qt.data(), nullptr, vec != 0);
  std::memcpy(evals, S.D, sizeof(double) * n);
  return 0;
}

static DCPlan plan_view(const lqm::DCPlanHost& PH) {
  DCPlan P;
  P.nnodes = PH.nnodes;
  P.nheights = PH.nheights;
  P.hstart = PH.buf.data() + PH.off_hstart;
  P.lo = PH.buf.data() + PH.off_lo;
  P.mid = PH.buf.data() + PH.off_mid;
  P.hi = PH.buf.data() + PH.off_hi;
  P.owner = PH.buf.data() + PH.off_own;
  return P;
}

// The blocked large-n path on one k-point: panel reduction (blk_column,
// blk_symv_tile, blk_t12_slab, blk_prev_w; the rank-2nb update done here as loops),
// divide and conquer with the tiled merge update from tile_min rows on, and
// the compact-WY back-transformation (blk_larft, products done here).
extern "C" int lqm_emul_eigh_blocked(int n, int nR, int dim, const double* blocks, const int64_t* keys,
                                     const double* kpt, int nb, int tile_min, int want_vectors, double* evals,
                                     double* U) {
  const Team T = make_host_team();
  const size_t nn = (size_t)n * n;
  const int nbk = std::max(1, symv_nblk(T, n - 1));
  std::vector<double2> A(nn), W((size_t)n * nb), tau(n), t12(2 * nb), ph(nR + 1);
  const int TB = symv_tb(T);
  std::vector<double2> part((size_t)nbk * nbk * TB), ts((size_t)TB * (TB + 1)), svs(2 * TB), sred(2 * TB);
  const int nsl_max = std::max(1, (n - 1 + t12_rows(T) - 1) / t12_rows(T));
  std::vector<double2> tpart((size_t)nsl_max * 2 * nb);
  std::vector<double> d(n), e(n), red(128);
  bloch_build(T, n, nR, dim, (const double2*)blocks, keys, kpt, ph.data(), A.data(), n);
  const int P = (n + nb - 1) / nb;
  for (int p = 0; p < P; ++p) {
    const int j0 = p * nb, nbp = std::min(nb, n - j0);
    for (int i = 0; i < nbp; ++i) {
      const int j = j0 + i;
      blk_column(T, n, nb, j0, i, A.data(), n, W.data(), n, tau.data(), d.data(), e.data(), t12.data(), red.data(),
                 part.data(), tpart.data());
      if (j <= n - 2) {
        const int nbl = symv_nblk(T, n - j - 1);
        for (int R = 0; R < nbl; ++R)
          for (int C = 0; C <= R; ++C)
            blk_symv_tile(T, n, j, R, C, A.data(), n, part.data(), ts.data(), svs.data(), sred.data());
        const int nsl = (n - j - 1 + t12_rows(T) - 1) / t12_rows(T);
        for (int sl = 0; i > 0 && sl < nsl; ++sl)
          blk_t12_slab(T, n, nb, j0, i, sl, A.data(), n, W.data(), n, tpart.data());
      }
    }
    if (j0 + nbp < n) {
      blk_prev_w(T, n, nb, j0, nbp - 1, A.data(), n, W.data(), n, tau.data(), t12.data(), red.data(), part.data(),
                 tpart.data(), nullptr);
      for (int c = j0 + nbp; c < n; ++c)
        for (int r = c; r < n; ++r) {
          double2 a = A[r + (size_t)c * n];
          for (int l = 0; l < nbp; ++l) {
            const double2 vr = A[r + (size_t)(j0 + l) * n], vc = A[c + (size_t)(j0 + l) * n];
            const double2 wr = W[r + (size_t)l * n], wc = W[c + (size_t)l * n];
            a = csub(a, cadd(cmul(vr, cconj(wc)), cmul(wr, cconj(vc))));
          }
          A[r + (size_t)c * n] = a;
        }
    }
  }
  const lqm::DCPlanHost PH = lqm::make_dc_plan_host(n);
  const DCPlan PV = plan_view(PH);
  std::vector<double> dbuf(13 * (size_t)n + 132), Q(nn + 4 * (size_t)n + 4), Qt(nn), Ub(nn);
  std::vector<int> ibuf(10 * (size_t)n);
  std::vector<double2> pb((size_t)n + 8);
  EighVec S;
  double* db = dbuf.data();
  S.d = db; S.e = db + n; S.D = db + 2 * n; S.z = db + 3 * n; S.dl = db + 4 * n; S.zl = db + 5 * n;
  S.troot = db + 6 * n; S.zhat = db + 7 * n; S.vals = db + 8 * n; S.dval = db + 9 * n; S.rc = db + 10 * n;
  S.rs = db + 11 * n; S.nrho = db + 12 * n; S.red = db + 13 * n;
  int* ib = ibuf.data();
  S.perm = ib; S.colnd = ib + n; S.org = ib + 2 * n; S.dcol = ib + 3 * n; S.newpos = ib + 4 * n;
  S.ri = ib + 5 * n; S.rj = ib + 6 * n; S.nk = ib + 7 * n; S.nrot = ib + 8 * n; S.ndef = ib + 9 * n;
  S.pbuf = pb.data();
  std::memcpy(S.d, d.data(), sizeof(double) * n);
  std::memcpy(S.e, e.data(), sizeof(double) * n);
  if (n > 0) S.e[n - 1] = 0.0;
  dc_solve(T, n, PV, S, Q.data(), Qt.data(), nullptr, want_vectors != 0, Ub.data(), tile_min);
  std::memcpy(evals, S.D, sizeof(double) * n);
  if (!want_vectors) return 0;
  double2* Uc = (double2*)U;
  for (size_t i = 0; i < nn; ++i) Uc[i] = cmk(Q[i], 0.0);
  blk_prep_reflectors(T, n, A.data(), n);
  std::vector<double2> Tm((size_t)nb * nb), G((size_t)nb * nb), X((size_t)nb * n);
  for (int p = P - 1; p >= 0; --p) {
    const int j0 = p * nb, nbr = std::min(nb, n - 1 - j0);
    if (nbr <= 0) continue;
    const int m = n - j0 - 1;
    blk_larft(T, n, nb, j0, nbr, A.data(), n, tau.data(), Tm.data(), G.data());
    const double2* V = A.data() + (j0 + 1) + (size_t)j0 * n;
    double2* Us = Uc + (j0 + 1);
    for (int c = 0; c < n; ++c)
      for (int l = 0; l < nbr; ++l) {
        double2 acc = cmk(0.0, 0.0);
        for (int r = 0; r < m; ++r) acc = cadd(acc, cmulc(V[r + (size_t)l * n], Us[r + (size_t)c * n]));
        X[l + (size_t)c * nb] = acc;
      }
    for (int c = 0; c < n; ++c) {
      double2 y[64];
      for (int l = 0; l < nbr; ++l) {
        double2 acc = cmk(0.0, 0.0);
        for (int q = 0; q < nbr; ++q) acc = cadd(acc, cmul(Tm[l + (size_t)q * nb], X[q + (size_t)c * nb]));
        y[l] = acc;
      }
      for (int r = 0; r < m; ++r) {
        double2 u = Us[r + (size_t)c * n];
        for (int l = 0; l < nbr; ++l) u = csub(u, cmul(V[r + (size_t)l * n], y[l]));
        Us[r + (size_t)c * n] = u;
      }
    }
  }
  return 0;
}

// The two-stage large-n path on one k-point: stage 1 (ts_panel_qr, the GEMM
// chain of the trailing update done here as loops), band extraction, the bulge
// chase (ts_chase_sweep, sweeps in order), divide and conquer, then U = Q1 Q2 Z
// (ts_q2_apply_host, the compact-WY products of blk_larft with the rows offset
// by the half-bandwidth).
template <int B>
static int emul_twostage(int n, int nR, int dim, const double* blocks, const int64_t* keys, const double* kpt,
                         int want_vectors, double* evals, double* U, double* tri, bool q2_grouped) {
  const Team T = make_host_team();
  const size_t nn = (size_t)n * n;
  std::vector<double2> A(nn), ph(nR + 1), tau(n + 1), Vb(nn + 1), Tm(B * B), sm((T.nw + 2) * B + B * B + 8);
  std::vector<double2> Y(nn + 1), X(nn + 1), S(B * B), Z(B * B);
  bloch_build(T, n, nR, dim, (const double2*)blocks, keys, kpt, ph.data(), A.data(), n);
  for (int j0 = 0; j0 + B < n; j0 += B) {
    const int m = n - j0 - B, nr = std::min(B, m);
    ts_panel_qr<B>(T, n, j0, A.data(), n, tau.data(), Vb.data(), n, Tm.data(), sm.data());
    auto a22 = [&](int r, int c) -> double2 {
      return r >= c ? A[(j0 + B + r) + (size_t)(j0 + B + c) * n] : cconj(A[(j0 + B + c) + (size_t)(j0 + B + r) * n]);
    };
    for (int r = 0; r < m; ++r)
      for (int l = 0; l < nr; ++l) {
        double2 acc = cmk(0.0, 0.0);
        for (int q = 0; q < m; ++q) acc = cadd(acc, cmul(a22(r, q), Vb[q + (size_t)l * n]));
        Y[r + (size_t)l * n] = acc;
      }
    for (int r = 0; r < m; ++r)
      for (int l = 0; l < nr; ++l) {
        double2 acc = cmk(0.0, 0.0);
        for (int q = 0; q < nr; ++q) acc = cadd(acc, cmul(Y[r + (size_t)q * n], Tm[q + l * B]));
        X[r + (size_t)l * n] = acc;
      }
    for (int q = 0; q < nr; ++q)
      for (int l = 0; l < nr; ++l) {
        double2 acc = cmk(0.0, 0.0);
        for (int r = 0; r < m; ++r) acc = cadd(acc, cmulc(Vb[r + (size_t)q * n], X[r + (size_t)l * n]));
        S[q + l * B] = acc;
      }
    for (int q = 0; q < nr; ++q)
      for (int l = 0; l < nr; ++l) {
        double2 acc = cmk(0.0, 0.0);
        for (int p = 0; p < nr; ++p) acc = cadd(acc, cmulc(Tm[p + q * B], S[p + l * B]));
        Z[q + l * B] = cscale(0.5, acc);
      }
    for (int r = 0; r < m; ++r)
      for (int l = 0; l < nr; ++l) {
        double2 acc = X[r + (size_t)l * n];
        for (int q = 0; q < nr; ++q) acc = csub(acc, cmul(Vb[r + (size_t)q * n], Z[q + l * B]));
        Y[r + (size_t)l * n] = acc;  // W
      }
    for (int c = 0; c < m; ++c)
      for (int r = c; r < m; ++r) {
        double2& a = A[(j0 + B + r) + (size_t)(j0 + B + c) * n];
        for (int l = 0; l < nr; ++l) {
          const double2 vr = Vb[r + (size_t)l * n], vc = Vb[c + (size_t)l * n];
          const double2 wr = Y[r + (size_t)l * n], wc = Y[c + (size_t)l * n];
          a = csub(a, cadd(cmul(vr, cconj(wc)), cmul(wr, cconj(vc))));
        }
      }
  }
  const int ldb = 2 * B, tmax = ts_tmax(n, B);
  std::vector<double2> Bd((size_t)ldb * n), V2((size_t)std::max(n - 1, 1) * tmax * B), tau2((size_t)std::max(n - 1, 1) * tmax),
      sv(2 * B + 2);
  ts_band_extract<B>(T, n, A.data(), n, Bd.data());
  std::vector<double2> win(3 * B * (B + 1) + 2 * B);
  for (int s = 0; s <= n - 2; ++s)
    ts_chase_sweep<B>(T, n, s, Bd.data(), V2.data() + (size_t)s * tmax * B, tau2.data() + (size_t)s * tmax, win.data(),
                      [](int) { return true; }, [](int) {});
  std::vector<double> d(n), e(n, 0.0);
  double offmax = 0.0;  // entries outside the tridiagonal after the chase (should be zero)
  for (int j = 0; j < n; ++j) {
    d[j] = Bd[(size_t)j * ldb].x;
    if (j + 1 < n) e[j] = Bd[1 + (size_t)j * ldb].x;
    if (j + 1 < n) offmax = std::max(offmax, std::fabs(Bd[1 + (size_t)j * ldb].y));
    for (int o = 2; o < ldb && j + o < n; ++o) {
      const double2 x = Bd[o + (size_t)j * ldb];
      offmax = std::max(offmax, std::fabs(x.x) + std::fabs(x.y));
    }
  }
  if (tri) { std::memcpy(tri, d.data(), sizeof(double) * n); std::memcpy(tri + n, e.data(), sizeof(double) * n); tri[2 * n] = offmax; }
  const lqm::DCPlanHost PH = lqm::make_dc_plan_host(n);
  const DCPlan PV = plan_view(PH);
  std::vector<double> dbuf(13 * (size_t)n + 132), Q(nn + 4 * (size_t)n + 4), Qt(nn), Ub(nn);
  std::vector<int> ibuf(10 * (size_t)n);
  std::vector<double2> pb((size_t)n + 8);
  EighVec SV;
  double* db = dbuf.data();
  SV.d = db; SV.e = db + n; SV.D = db + 2 * n; SV.z = db + 3 * n; SV.dl = db + 4 * n; SV.zl = db + 5 * n;
  SV.troot = db + 6 * n; SV.zhat = db + 7 * n; SV.vals = db + 8 * n; SV.dval = db + 9 * n; SV.rc = db + 10 * n;
  SV.rs = db + 11 * n; SV.nrho = db + 12 * n; SV.red = db + 13 * n;
  int* ib = ibuf.data();
  SV.perm = ib; SV.colnd = ib + n; SV.org = ib + 2 * n; SV.dcol = ib + 3 * n; SV.newpos = ib + 4 * n;
  SV.ri = ib + 5 * n; SV.rj = ib + 6 * n; SV.nk = ib + 7 * n; SV.nrot = ib + 8 * n; SV.ndef = ib + 9 * n;
  SV.pbuf = pb.data();
  std::memcpy(SV.d, d.data(), sizeof(double) * n);
  std::memcpy(SV.e, e.data(), sizeof(double) * n);
  if (n > 0) SV.e[n - 1] = 0.0;
  dc_solve(T, n, PV, SV, Q.data(), Qt.data(), nullptr, want_vectors != 0, Ub.data(), 1 << 30);
  std::memcpy(evals, SV.D, sizeof(double) * n);
  if (!want_vectors) return 0;
  double2* Uc = (double2*)U;
  for (size_t i = 0; i < nn; ++i) Uc[i] = cmk(Q[i], 0.0);
  if (q2_grouped)
    ts_q2_apply_grouped_host<B>(n, V2.data(), tau2.data(), Uc, n, n);
  else
    ts_q2_apply_host<B>(n, V2.data(), tau2.data(), Uc, n, n);
  const int NR = n - B;
  blk_prep_reflectors(T, n, A.data(), n, B);
  const int nb = 2 * B;  // back-transformation panels of two stage-1 panels
  std::vector<double2> Tb((size_t)nb * nb), G((size_t)nb * nb), Xb((size_t)nb * n);
  for (int p = (NR + nb - 1) / nb - 1; p >= 0; --p) {
    const int j0 = p * nb, nbr = std::min(nb, NR - j0);
    if (nbr <= 0) continue;
    const int m = n - j0 - B;
    blk_larft(T, n, nb, j0, nbr, A.data(), n, tau.data(), Tb.data(), G.data(), nullptr, B);
    const double2* V = A.data() + (j0 + B) + (size_t)j0 * n;
    double2* Us = Uc + (j0 + B);
    for (int c = 0; c < n; ++c)
      for (int l = 0; l < nbr; ++l) {
        double2 acc = cmk(0.0, 0.0);
        for (int r = 0; r < m; ++r) acc = cadd(acc, cmulc(V[r + (size_t)l * n], Us[r + (size_t)c * n]));
        Xb[l + (size_t)c * nb] = acc;
      }
    for (int c = 0; c < n; ++c) {
      double2 y[64];
      for (int l = 0; l < nbr; ++l) {
        double2 acc = cmk(0.0, 0.0);
        for (int q = 0; q < nbr; ++q) acc = cadd(acc, cmul(Tb[l + (size_t)q * nb], Xb[q + (size_t)c * nb]));
        y[l] = acc;
      }
      for (int r = 0; r < m; ++r) {
        double2 u = Us[r + (size_t)c * n];
        for (int l = 0; l < nbr; ++l) u = csub(u, cmul(V[r + (size_t)l * n], y[l]));
        Us[r + (size_t)c * n] = u;
      }
    }
  }
  return 0;
}

// b: the half-bandwidth (4 or 16; negative: the grouped Q2 order); tri (or null): d, e and the largest entry
// left outside the tridiagonal (3n doubles... 2n + 1 used).
extern "C" int lqm_emul_eigh_twostage(int n, int nR, int dim, const double* blocks, const int64_t* keys,
                                      const double* kpt, int b, int want_vectors, double* evals, double* U,
                                      double* tri) {
  // b < 0: the Q2 back-transformation in the grouped order of the device kernel
  const bool grouped = b < 0;
  if (grouped) b = -b;
  if (b == 4) return emul_twostage<4>(n, nR, dim, blocks, keys, kpt, want_vectors, evals, U, tri, grouped);
  if (b == 16) return emul_twostage<16>(n, nR, dim, blocks, keys, kpt, want_vectors, evals, U, tri, grouped);
  return -1;
}

// The bulge chase of a band (ldb = 2B, n x ldb complex, lower band storage) run
// twice: sweep after sweep, and on `workers` threads with the device kernel's
// protocol (worker w takes sweeps w, w + workers, ...; before task t of sweep s it
// waits until sweep s - 1 has finished its tasks 0 .. t + 2, read from the previous
// worker's progress word with acquire / release ordering), with random pauses after
// tasks to vary the interleaving.  Returns 1 when the band, the reflectors and the
// taus of the two runs are bitwise equal, 0 when they differ.
template <int B>
static int emul_chase_schedules(int n, const double* band, int workers, unsigned seed) {
  const Team T = make_host_team();
  const int ldb = 2 * B, tmax = ts_tmax(n, B);
  const size_t nb = (size_t)ldb * n, nv = (size_t)std::max(n - 1, 1) * tmax;
  std::vector<double2> B1(nb), B2(nb), V1(nv * B), V2(nv * B), t1(nv), t2(nv);
  std::memcpy(B1.data(), band, nb * sizeof(double2));
  std::memcpy(B2.data(), band, nb * sizeof(double2));
  std::vector<double2> win(3 * B * (B + 1) + 2 * B);
  for (int s = 0; s <= n - 2; ++s)
    ts_chase_sweep<B>(T, n, s, B1.data(), V1.data() + (size_t)s * tmax * B, t1.data() + (size_t)s * tmax, win.data(),
                      [](int) { return true; }, [](int) {});
  const long long unit = tmax + 1;
  std::vector<std::atomic<long long>> prog(workers);
  for (auto& p : prog) p.store(-1);
  std::vector<std::thread> th;
  for (int w = 0; w < workers; ++w)
    th.emplace_back([&, w] {
      std::mt19937 rng(seed * 7919u + (unsigned)w);
      std::vector<double2> wwin(3 * B * (B + 1) + 2 * B);
      const int wp = (w + workers - 1) % workers;
      for (int s = w; s <= n - 2; s += workers) {
        const int ntp = (s > 0) ? ts_tasks(n, B, s - 1) : 0;
        auto wait = [&](int t) {
          if (s == 0) return true;
          const long long need = (long long)(s - 1) * unit + (t + 3 < ntp ? t + 3 : ntp);
          while (prog[wp].load(std::memory_order_acquire) < need) std::this_thread::yield();
          return true;
        };
        auto done = [&](int t) {
          prog[w].store((long long)s * unit + t + 1, std::memory_order_release);
          if (rng() % 16 == 0) std::this_thread::sleep_for(std::chrono::microseconds(rng() % 50));
        };
        ts_chase_sweep<B>(T, n, s, B2.data(), V2.data() + (size_t)s * tmax * B, t2.data() + (size_t)s * tmax,
                          wwin.data(), wait, done);
      }
    });
  for (auto& t : th) t.join();
  // slots of tasks that do not exist are never written by either run: compare the written ones
  bool same = std::memcmp(B1.data(), B2.data(), nb * sizeof(double2)) == 0;
  for (int s = 0; s <= n - 2 && same; ++s)
    for (int t = 0; t < ts_tasks(n, B, s) && same; ++t) {
      const size_t q = (size_t)s * tmax + t;
      same = std::memcmp(&V1[q * B], &V2[q * B], B * sizeof(double2)) == 0 &&
             std::memcmp(&t1[q], &t2[q], sizeof(double2)) == 0;
    }
  return same ? 1 : 0;
}

extern "C" int lqm_emul_chase_schedules(int n, int b, const double* band, int workers, unsigned seed) {
  if (b == 4) return emul_chase_schedules<4>(n, band, workers, seed);
  if (b == 16) return emul_chase_schedules<16>(n, band, workers, seed);
  return -1;
}

// rho_from_U on a given U (n x n, ld n) and occupations f.
extern "C" int lqm_emul_rho(int n, const double* U, const double* f, double* out) {
  const Team T = make_host_team();
  rho_from_U(T, n, (const double2*)U, n, f, (double2*)out, n);
  return 0;
}
