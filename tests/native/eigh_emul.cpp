// Host build of the per-k eigensolver team code (one thread, one lane).
//
// Test infrastructure: lets the CPU suite exercise the exact index
// arithmetic of bloch_build / hetrd_lower / dc_solve / backtransform from
// latticeqm.jl_b200/csrc/lqm_eigh.cuh against LAPACK, without a GPU.
#include <cstdint>
#include <cstring>
#include <vector>

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

// rho_from_U on a given U (n x n, ld n) and occupations f.
extern "C" int lqm_emul_rho(int n, const double* U, const double* f, double* out) {
  const Team T = make_host_team();
  rho_from_U(T, n, (const double2*)U, n, f, (double2*)out, n);
  return 0;
}
