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
  std::vector<double2> A(nn), cbuf(3 * n + 2 + nR);
  std::vector<double> dbuf(13 * (size_t)n + 36), Q(nn), Qt(nn), Us(nn);
  std::vector<int> ibuf(10 * (size_t)n);
  EighVec S;
  S.tau = cbuf.data(); S.v = S.tau + n; S.w = S.tau + 2 * n; S.bc = S.tau + 3 * n;
  double2* ph = S.tau + 3 * n + 2;
  double* db = dbuf.data();
  S.d = db; S.e = db + n; S.D = db + 2 * n; S.z = db + 3 * n; S.dl = db + 4 * n; S.zl = db + 5 * n;
  S.troot = db + 6 * n; S.zhat = db + 7 * n; S.vals = db + 8 * n; S.dval = db + 9 * n; S.rc = db + 10 * n;
  S.rs = db + 11 * n; S.nrho = db + 12 * n; S.red = db + 13 * n;
  int* ib = ibuf.data();
  S.perm = ib; S.colnd = ib + n; S.org = ib + 2 * n; S.dcol = ib + 3 * n; S.newpos = ib + 4 * n;
  S.ri = ib + 5 * n; S.rj = ib + 6 * n; S.nk = ib + 7 * n; S.nrot = ib + 8 * n; S.ndef = ib + 9 * n;

  bloch_build(T, n, nR, dim, (const double2*)blocks, keys, kpt, ph, A.data(), n);
  hetrd_lower(T, n, A.data(), n, S);
  if (tri_d) std::memcpy(tri_d, S.d, sizeof(double) * n);
  if (tri_e && n > 1) std::memcpy(tri_e, S.e, sizeof(double) * (n - 1));
  dc_solve(T, n, P, S, Q.data(), Qt.data(), Us.data());
  std::memcpy(evals, S.D, sizeof(double) * n);
  if (want_vectors) backtransform(T, n, A.data(), n, S, Q.data(), (double2*)U, n);
  return 0;
}

// D&C alone on a given symmetric tridiagonal (d, e): eigenvalues and Z.
extern "C" int lqm_emul_tridiag(int n, const double* d, const double* e, double* evals, double* Z) {
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
  std::vector<double> dbuf(13 * (size_t)n + 36), Qt(nn), Us(nn);
  std::vector<int> ibuf(10 * (size_t)n);
  std::vector<double2> cbuf(3 * n + 2);
  EighVec S;
  S.tau = cbuf.data(); S.v = S.tau + n; S.w = S.tau + 2 * n; S.bc = S.tau + 3 * n;
  double* db = dbuf.data();
  S.d = db; S.e = db + n; S.D = db + 2 * n; S.z = db + 3 * n; S.dl = db + 4 * n; S.zl = db + 5 * n;
  S.troot = db + 6 * n; S.zhat = db + 7 * n; S.vals = db + 8 * n; S.dval = db + 9 * n; S.rc = db + 10 * n;
  S.rs = db + 11 * n; S.nrho = db + 12 * n; S.red = db + 13 * n;
  int* ib = ibuf.data();
  S.perm = ib; S.colnd = ib + n; S.org = ib + 2 * n; S.dcol = ib + 3 * n; S.newpos = ib + 4 * n;
  S.ri = ib + 5 * n; S.rj = ib + 6 * n; S.nk = ib + 7 * n; S.nrot = ib + 8 * n; S.ndef = ib + 9 * n;
  std::memcpy(S.d, d, sizeof(double) * n);
  if (n > 1) std::memcpy(S.e, e, sizeof(double) * (n - 1));
  dc_solve(T, n, P, S, Z, Qt.data(), Us.data());
  std::memcpy(evals, S.D, sizeof(double) * n);
  return 0;
}
