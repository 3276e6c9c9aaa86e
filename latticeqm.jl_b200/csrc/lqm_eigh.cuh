// Per-k dense Hermitian eigensolver, one team (CTA) per k-point, FP64.
//
//   1. bloch_build:   H(k) = sum_R H_R exp(+i 2 pi k.R) into A (upper triangle is
//                     the source, mirrored to the lower one — the reference hands
//                     LAPACK `Hermitian(M)`, i.e. the upper triangle).
//   2. hetrd_lower:   Householder reduction to a real symmetric tridiagonal T
//                     (LAPACK zhetd2/zlarfg conventions, reflectors kept in A).
//   3. dc_solve:      Cuppen divide and conquer on T: tearing, bottom-up merges
//                     with dlaed2-style deflation, secular equations solved per
//                     root by a safeguarded two-pole rational iteration, and
//                     Gu-Eisenstat recomputed z for orthogonal eigenvectors.
//   4. backtransform: U = H_0 H_1 ... H_{n-2} Z.
//
// Every function is a team phase sequence (see lqm_team.cuh).
#pragma once
#include "lqm_team.cuh"

#ifndef LQM_DEPS
#define LQM_DEPS 1.1102230246251565e-16  /* relative machine precision, LAPACK dlamch('E') */
#endif

// Divide-and-conquer merge plan for one matrix order n (built on the host).
struct DCPlan {
  int nnodes;        // internal (merge) nodes, ordered by height
  int nheights;      // number of merge heights
  const int* hstart; // [nheights+1] node ranges per height
  const int* lo;     // [nnodes]
  const int* mid;    // [nnodes]
  const int* hi;     // [nnodes]
  const int* owner;  // [nheights*n] node id covering row i at that height, or -1
};

// Shared-memory vectors for one k-point (all length >= n unless noted).
struct EighVec {
  double *d, *e, *D, *z, *dl, *zl, *troot, *zhat, *vals, *dval, *rc, *rs, *nrho, *red;  // red: 128
  int *perm, *colnd, *org, *dcol, *newpos, *ri, *rj, *nk, *nrot, *ndef;
  double2 *tau, *v, *w, *vn, *pn, *bc, *pbuf;
  double* tile = nullptr;  // team scratch for the tiled merge update (large n): kDcTileRing doubles + n ints, or null
};

// ---------------------------------------------------------------------------
// 1. Bloch sum.  blocks: nR x (n x n) column-major complex; keys: d x nR int64.
// Column j by warp, rows i <= j by lane; the lower triangle is the mirror.
// ---------------------------------------------------------------------------
template <class TeamT>
LQM_FN void bloch_build(const TeamT& T, int n, int nR, int dim, const double2* __restrict__ blocks,
                        const int64_t* __restrict__ keys, const double* kpt, double2* ph,
                        double2* A, int lda) {
  for (int r = T.tid; r < nR; r += T.nt) {
    double dot = 0.0;
    for (int c = 0; c < dim; ++c) dot += kpt[c] * (double)keys[(int64_t)r * dim + c];
    double s, co;
    lqm_sincospi(2.0 * dot, &s, &co);
    ph[r] = cmk(co, s);
  }
  team_sync(T);
  const int64_t nn = (int64_t)n * n;
  for (int j = T.wid; j < n; j += T.nw) {
    for (int i = T.lane; i <= j; i += T.nl) {
      const int64_t idx = i + (int64_t)j * n;
      double2 acc = cmk(0.0, 0.0);
      for (int r = 0; r < nR; ++r) acc = cadd(acc, cmul(blocks[(int64_t)r * nn + idx], ph[r]));
      if (i == j) {
        A[i + (int64_t)j * lda] = cmk(acc.x, 0.0);
      } else {
        A[i + (int64_t)j * lda] = acc;
        A[j + (int64_t)i * lda] = cconj(acc);
      }
    }
  }
  team_sync(T);
}

// ---------------------------------------------------------------------------
// 2. Householder tridiagonalisation (lower storage, LAPACK zhetd2/zlarfg
// conventions).  The rank-2 update of step j and the mat-vec of step j+1 are
// one pass over the trailing block, so each element is read and written once
// per step.  Out: d[n], e[n-1] (real), tau[n-1]; reflector j is A[j+1.., j]
// with v0 = 1.
// ---------------------------------------------------------------------------

// zlarfg on (alpha, ||x||^2): tau, beta and the scale 1/(alpha - beta) of x.
// Every thread evaluates it on the same inputs (no serial section).
LQM_FN void zlarfg_scalars(double2 alpha, double xnorm2, double2* tau, double* beta, double2* scal) {
  if (xnorm2 == 0.0 && alpha.y == 0.0) {
    *tau = cmk(0.0, 0.0); *scal = cmk(0.0, 0.0); *beta = alpha.x;
    return;
  }
  const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
  const double b = (alpha.x >= 0.0) ? -nrm : nrm;
  // 1/b and 1/(alpha - b) = conj(alpha - b)/|alpha - b|^2 are independent
  // divisions (|alpha - b| >= |b| > 0 by the sign choice)
  const double dr = alpha.x - b, di = alpha.y;
  const double ib = 1.0 / b;
  const double idn = 1.0 / (dr * dr + di * di);
  *beta = b;
  *tau = cmk((b - alpha.x) * ib, -alpha.y * ib);
  *scal = cmk(dr * idn, -di * idn);
}

// One pass over the trailing block B = A[o:, o:] (order mb, o >= 1):
//   upd:  B[r,c] -= v[r+1] conj(w[c+1]) + w[r+1] conj(v[c+1])  (reflector o-2,
//         whose vectors start one row above B)
//   x[c] = (c == 0) ? 1 : scal * A[o+c, o-1]  (next reflector, formed on the fly
//         by the warp owning column c, stored to xs[] and back into A)
//   pbuf[warp][r] = sum over the warp's columns of B_new[r,c] x[c]
// Rows across lanes (up to 4 per lane and pass), columns across warps.
template <class TeamT>
LQM_FN void trailing_pass(const TeamT& T, int mb, double2* A, int lda, int o, const double2* v, const double2* w,
                          bool upd, double2 scal, double2* xs, double2* pbuf, int pstride) {
  double2* B = A + o + (int64_t)o * lda;
  double2* xcol = A + o + (int64_t)(o - 1) * lda;
  for (int r0 = 0; r0 < mb; r0 += 4 * T.nl) {
    double2 acc[4], vr[4], wr[4];
    int rr[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      rr[q] = r0 + q * T.nl + T.lane;
      acc[q] = cmk(0.0, 0.0);
      vr[q] = cmk(0.0, 0.0);
      wr[q] = cmk(0.0, 0.0);
      if (upd && rr[q] < mb) { vr[q] = v[rr[q] + 1]; wr[q] = w[rr[q] + 1]; }
    }
#pragma unroll 2
    for (int c = T.wid; c < mb; c += T.nw) {
      const double2 xc = (c == 0) ? cmk(1.0, 0.0) : cmul(scal, xcol[c]);
      double2 cw = cmk(0.0, 0.0), cv = cmk(0.0, 0.0);
      if (upd) { cw = cconj(w[c + 1]); cv = cconj(v[c + 1]); }
      double2* Bc = B + (int64_t)c * lda;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = rr[q];
        if (r < mb) {
          double2 a = Bc[r];
          if (upd) {
            a = cfms(cfms(a, vr[q], cw), wr[q], cv);
            if (r == c) a.y = 0.0;
            Bc[r] = a;
          }
          acc[q] = cfma(acc[q], a, xc);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (rr[q] < mb) pbuf[T.wid * pstride + rr[q]] = acc[q];
  }
}

// Stores the next reflector x (formed from column o-1 rows o..) into xs[] and
// back into A.  Called after trailing_pass and a barrier.
template <class TeamT>
LQM_FN void store_reflector(const TeamT& T, int mb, double2* A, int lda, int o, double2 scal, double2* xs) {
  double2* xcol = A + o + (int64_t)(o - 1) * lda;
  for (int c = T.tid; c < mb; c += T.nt) {
    const double2 x = (c == 0) ? cmk(1.0, 0.0) : cmul(scal, xcol[c]);
    xs[c] = x;
    xcol[c] = x;
  }
}

// Householder tridiagonalisation with 3 barriers per step:
//   pass (update j, mat-vec with reflector j+1) | p, p^H v -> alpha |
//   w, update of the next column, its norm -> next reflector scalars.
template <class TeamT>
LQM_FN_NOINLINE void hetrd_lower(const TeamT& T, int n, double2* A, int lda, EighVec& S,
                                 unsigned long long* sub = nullptr) {
#if defined(__CUDA_ARCH__)
  long long tsub = clock64();
  if (T.tid != 0) sub = nullptr;
#define LQM_HTICK(i_)                                          \
  if (sub) {                                                   \
    const long long t_ = clock64();                            \
    sub[i_] += (unsigned long long)(t_ - tsub);                \
    tsub = t_;                                                 \
  }
#else
  (void)sub;
#define LQM_HTICK(i_)
#endif
  if (n == 1) {
    if (T.tid == 0) S.d[0] = A[0].x;
    team_sync(T);
    return;
  }
  double* redA = S.red;
  double* redB = S.red + 64;
  double2* pb = S.pbuf;
  double2* tau_out = S.tau;
  double* d_out = S.d;
  double* e_out = S.e;
  double2* vc = S.v;   // current reflector
  double2* vx = S.vn;  // next reflector
  double2* wc = S.w;   // w of the current reflector
  double2* p = S.pn;
  // reflector 0 from column 0
  double s0 = 0.0, dummy = 0.0;
  for (int r = 2 + T.tid; r < n; r += T.nt) { const double2 x = A[r]; s0 += x.x * x.x + x.y * x.y; }
  team_sum2_1b(T, s0, dummy, redA);
  double2 tnext, scal;
  double beta;
  zlarfg_scalars(A[1], s0, &tnext, &beta, &scal);
  if (T.tid == 0) { tau_out[0] = tnext; e_out[0] = beta; d_out[0] = A[0].x; }
  // step j = -1 .. n-3: pass over A[j+2:, j+2:] (update j if j >= 0) with reflector j+1
  for (int j = -1; j <= n - 3; ++j) {
    const int o = j + 2;
    const int mb = n - o;
    LQM_HTICK(2);
    trailing_pass(T, mb, A, lda, o, vc, wc, j >= 0, scal, vx, pb, n);
    team_sync(T);
    LQM_HTICK(0);
    store_reflector(T, mb, A, lda, o, scal, vx);
    // p = tau_{j+1} * row sums; alpha = -1/2 tau (p^H x)
    double pr = 0.0, pi = 0.0;
    for (int r = T.tid; r < mb; r += T.nt) {
      double2 s0 = cmk(0.0, 0.0), s1 = s0, s2 = s0, s3 = s0;
      int wv = 0;
      for (; wv + 4 <= T.nw; wv += 4) {
        s0 = cadd(s0, pb[wv * n + r]);
        s1 = cadd(s1, pb[(wv + 1) * n + r]);
        s2 = cadd(s2, pb[(wv + 2) * n + r]);
        s3 = cadd(s3, pb[(wv + 3) * n + r]);
      }
      for (; wv < T.nw; ++wv) s0 = cadd(s0, pb[wv * n + r]);
      const double2 sacc = cadd(cadd(s0, s1), cadd(s2, s3));
      const double2 pv = cmul(tnext, sacc);
      p[r] = pv;
      const double2 q = cmulc(pv, vx[r]);  // vx[r] was stored by this same thread above
      pr += q.x; pi += q.y;
    }
    team_sum2_1b(T, pr, pi, redA);
    LQM_HTICK(1);
    const double2 alpha = cmul(cmk(-0.5 * tnext.x, -0.5 * tnext.y), cmk(pr, pi));
    // w = p + alpha x; column o gets update j+1; norm of its rows o+2.. for reflector j+2
    const double2 w0 = cadd(p[0], alpha);  // x[0] = 1
    const double2 cw0 = cconj(w0);
    double2* col = A + o + (int64_t)o * lda;
    double sn = 0.0;
    for (int r = T.tid; r < mb; r += T.nt) {
      const double2 x = vx[r];
      const double2 wr = cadd(p[r], cmul(alpha, x));
      wc[r] = wr;  // the old w is no longer read (the pass ended at the barrier)
      double2 a = csub(col[r], cadd(cmul(x, cw0), wr));  // x conj(w0) + w conj(x0), x0 = 1
      if (r == 0) a.y = 0.0;
      col[r] = a;
      if (r >= 2) sn += a.x * a.x + a.y * a.y;
    }
    double dn = 0.0;
    team_sum2_1b(T, sn, dn, redB);
    // swap: x becomes the current reflector
    double2* t = vc; vc = vx; vx = t;
    if (o <= n - 2) {  // reflector j+2 = o exists
      zlarfg_scalars(col[1], sn, &tnext, &beta, &scal);
      if (T.tid == 0) { tau_out[o] = tnext; e_out[o] = beta; d_out[o] = col[0].x; }
    } else {
      if (T.tid == 0) d_out[n - 1] = col[0].x;
    }
  }
  team_sync(T);
  LQM_HTICK(2);
#undef LQM_HTICK
}

// ---------------------------------------------------------------------------
// 3. Divide and conquer on the symmetric tridiagonal (d, e).
// ---------------------------------------------------------------------------

// Lane-group width for the secular roots of a merge with k non-deflated
// values: about twelve terms per lane, at most a warp.  Narrow groups keep
// several roots per warp in flight and their sums need fewer shuffle levels;
// the per-lane terms are independent divisions that pipeline.
LQM_FN int secular_width(int k, int nl) {
  int w = 1;
  while (w < nl && 12 * w < k) w <<= 1;
  return w;
}

// One root of the secular equation 1 + rho sum_j zl_j^2 / (dl_j - lambda) = 0,
// dl ascending, rho > 0, solved by a group of `gw` lanes (g = lane within the
// group): the lanes split the k terms of every sum and all lanes of the group
// then hold identical scalars.  `active` is false for lanes without a root;
// they still take part in every shuffle of their warp.  lambda = dl[org] + tau;
// interior roots take the nearer pole as origin.  Safeguarded two-pole
// rational steps (each step fits the poles left and right of the root
// separately to value and slope), bisection when a step leaves the bracket.
LQM_FN void secular_root_group(bool active, int gw, int g, int k, const double* dl, const double* zl, double rho,
                               int i, int* org_out, double* tau_out) {
  int org = 0;
  double lo = 0.0, hi = 0.0, f0 = 0.0, zs = 0.0;
  const bool last = active && (i >= k - 1);
  double gap = 0.0, mid = 0.0;
  if (active && !last) {
    gap = dl[i + 1] - dl[i];
    mid = 0.5 * gap;
    for (int j = g; j < k; j += gw) f0 += rho * zl[j] * zl[j] / ((dl[j] - dl[i]) - mid);
  }
  if (last)
    for (int j = g; j < k; j += gw) zs += zl[j] * zl[j];
  f0 = group_sum_bcast(f0, gw);
  zs = group_sum_bcast(zs, gw);
  if (active) {
    if (k == 1) {
      org = 0; lo = hi = rho * zl[0] * zl[0];
    } else if (!last) {
      if (1.0 + f0 >= 0.0) { org = i; lo = 0.0; hi = mid; }
      else { org = i + 1; lo = -(gap - mid); hi = 0.0; }
    } else {
      org = k - 1; lo = 0.0; hi = rho * zs * (1.0 + 4.0 * LQM_DEPS) + 1e-300;
    }
  }
  bool done = !active || k == 1;
  const double dorg = active ? dl[org] : 0.0;
  double tau = (k == 1 && active) ? lo : 0.5 * (lo + hi);
  for (int it = 0; it < 80; ++it) {
#if defined(__CUDA_ARCH__)
    if (__all_sync(0xffffffffu, done)) break;
#else
    if (done) break;
#endif
    double psi1 = 0.0, dpsi1 = 0.0, psi2 = 0.0, dpsi2 = 0.0, abss = 0.0;
    if (!done) {
      for (int j = g; j < k; j += gw) {
        const double del = (dl[j] - dorg) - tau;
        const double t = zl[j] / del;
        const double term = rho * zl[j] * t;
        const double dterm = rho * t * t;
        if (j <= i) { psi1 += term; dpsi1 += dterm; } else { psi2 += term; dpsi2 += dterm; }
        abss += fabs(term);
      }
    }
    psi1 = group_sum_bcast(psi1, gw);
    dpsi1 = group_sum_bcast(dpsi1, gw);
    psi2 = group_sum_bcast(psi2, gw);
    dpsi2 = group_sum_bcast(dpsi2, gw);
    abss = group_sum_bcast(abss, gw);
    if (done) continue;
    const double f = 1.0 + psi1 + psi2;
    if (f == 0.0) { done = true; continue; }
    if (f < 0.0) lo = tau; else hi = tau;
    if (fabs(f) <= 8.0 * LQM_DEPS * (1.0 + abss) * 2.0) { done = true; continue; }
    const double a = (dl[i] - dorg) - tau;
    double x = 0.0;
    bool ok = true;
    if (!last) {
      const double b = (dl[i + 1] - dorg) - tau;
      const double s1 = a * a * dpsi1, s2 = b * b * dpsi2;
      const double c = 1.0 + (psi1 - a * dpsi1) + (psi2 - b * dpsi2);
      const double B = c * (a + b) + s1 + s2;
      const double C = a * b * f;
      double disc = B * B - 4.0 * c * C;
      if (disc < 0.0) disc = 0.0;
      const double sq = sqrt(disc);
      if (c == 0.0) { if (B != 0.0) x = C / B; else ok = false; }
      else if (B > 0.0) x = 2.0 * C / (B + sq);
      else x = (B - sq) / (2.0 * c);
    } else {
      const double s1 = a * a * dpsi1;
      const double c = 1.0 + psi1 - a * dpsi1;
      if (c > 0.0) x = a + s1 / c; else ok = false;
    }
    double tn = ok ? tau + x : 0.5 * (lo + hi);
    if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
    const double chg = fabs(tn - tau);
    tau = tn;
    if (chg <= 2.0 * LQM_DEPS * fabs(tn)) done = true;
    else if (hi - lo <= 2.0 * LQM_DEPS * fmax(fabs(lo), fabs(hi))) done = true;
  }
  *org_out = org;
  *tau_out = tau;
}

// dlaed2-style deflation for one merge node (single thread), on the values in
// merged order: zs/ds[lo+p] = z/D of the p-th smallest (gathered in parallel
// before the scan, so the scan's loads do not wait on each other).
LQM_FN void deflate_node(int node, const DCPlan& P, EighVec& S, double eabs_beta, double* zs, double* ds) {
  const int lo = P.lo[node], hi = P.hi[node];
  const double rho = 2.0 * eabs_beta;
  double zmax = 0.0, dmax = 0.0;
  for (int p = lo; p < hi; ++p) { zmax = fmax(zmax, fabs(zs[p])); dmax = fmax(dmax, fabs(ds[p])); }
  const double tol = 8.0 * LQM_DEPS * fmax(dmax, zmax);
  int k = 0, nd = 0, nr = 0;
  if (rho * zmax <= tol) {
    for (int p = lo; p < hi; ++p) { S.dval[lo + nd] = ds[p]; S.dcol[lo + nd] = S.perm[p]; ++nd; }
  } else {
    int jp = -1;
    double zp = 0.0, dp = 0.0;
    for (int p = lo; p < hi; ++p) {
      const int j = S.perm[p];
      const double zj = zs[p], dj = ds[p];
      if (rho * fabs(zj) <= tol) { S.dval[lo + nd] = dj; S.dcol[lo + nd] = j; ++nd; continue; }
      if (jp < 0) { jp = j; zp = zj; dp = dj; continue; }
      const double t = dj - dp;
      // |t c s| <= tol with c = zj/tau, s = -zp/tau, tau^2 = zj^2 + zp^2 (no division)
      if (fabs(t * zj * zp) <= tol * (zj * zj + zp * zp)) {
        const double tau = hypot(zj, zp);
        const double cv = zj / tau, sv = -zp / tau;
        S.ri[lo + nr] = jp; S.rj[lo + nr] = j; S.rc[lo + nr] = cv; S.rs[lo + nr] = sv; ++nr;
        const double t2 = dp * cv * cv + dj * sv * sv;
        const double dnew = dp * sv * sv + dj * cv * cv;
        S.dval[lo + nd] = t2; S.dcol[lo + nd] = jp; ++nd;
        jp = j; zp = tau; dp = dnew;
      } else {
        S.dl[lo + k] = dp; S.zl[lo + k] = zp; S.colnd[lo + k] = jp; ++k;
        jp = j; zp = zj; dp = dj;
      }
    }
    if (jp >= 0) { S.dl[lo + k] = dp; S.zl[lo + k] = zp; S.colnd[lo + k] = jp; ++k; }
  }
  S.nk[node] = k; S.nrot[node] = nr; S.ndef[node] = nd; S.nrho[node] = rho;
}

// Optional per-step cycle accounting (device only): sub[0..7] += cycles of
// merge steps A (z, sort), B (deflation), C (secular), D (zhat), E-G (vectors,
// rotations, values), ranks, H (update), I (copy back).
#if defined(__CUDA_ARCH__)
#define LQM_SUBTICK(i_)                                                     \
  if (sub) {                                                                \
    const long long t_ = clock64();                                         \
    sub[i_] += (unsigned long long)(t_ - tsub);                             \
    tsub = t_;                                                              \
  }
#else
#define LQM_SUBTICK(i_)
#endif

// Merge update of one node as a tiled GEMM (large merges):
//   Qt[lo + r, newpos[it]] = sum_p Q[lo + r, colnd[p]] * Ubn[it + p*k],
// r < hi - lo, it < k (Ubn holds the secular vectors as rows).  A 512-thread
// team computes 128 x 128 output tiles on the FP64 tensor path (DMMA
// m8n8k4): 16 warps of 32 x 32, each a 4 x 4 grid of 8 x 8 accumulators.  The
// p range moves in 16-deep stages by cp.async through a 3-stage ring in `tile`
// (per stage 16 rows of 128 + 4 doubles for Q and for Ubn, p-major; the pitch of
// 132 == 4 mod 16 puts the 16 fragment reads of a half-warp on distinct bank
// pairs), followed by room for k column indices; two stages are in flight while
// one is summed.  p is summed in ascending 4-deep steps.  Other team sizes (the
// host emulation) take the plain loop.
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ void lqm_cp_async8(void* sdst, const void* gsrc, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  const int nbytes = valid ? 8 : 0;  // 0: zero-filled, nothing is read
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(nbytes) : "memory");
}
#endif
constexpr int kDcTileP = 132;                            // staged row pitch (doubles)
constexpr int kDcTileBK = 16;                            // p depth of a stage
constexpr int kDcTileStage = kDcTileBK * 2 * kDcTileP;   // doubles per stage (Q and Ubn slices)
constexpr int kDcTileRing = 3 * kDcTileStage;            // doubles of the ring
template <class TeamT>
LQM_FN void dc_tile_gemm(const TeamT& T, int n, int lo, int hi, int k, const int* colnd, const int* newpos,
                         const double* Q, double* Qt, const double* Ubn, double* tile) {
  const int s = hi - lo;
#if defined(__CUDA_ARCH__)
  if (T.nt == 512 && tile != nullptr) {
    constexpr int BM = 128, BN = 128, BK = kDcTileBK, PT = kDcTileP, STG = kDcTileStage, NS = 3;
    const int lane = T.tid & 31, warp = T.tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wr = (warp & 3) * 32, wc = (warp >> 2) * 32;  // the warp's 32 x 32 sub-tile
    int* cidx = (int*)(tile + kDcTileRing);                  // the node's column indices, staged once
    for (int p = T.tid; p < k; p += T.nt) cidx[p] = colnd[p];
    team_sync(T);
    for (int r0 = 0; r0 < s; r0 += BM) {
      for (int c0 = 0; c0 < k; c0 += BN) {
        double acc[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
        // element e = tid + 512 h of a stage: pp = e / 128, row / column e % 128
        auto issue = [&](int p0, int st) {
          double* As = tile + st * STG;
          double* Bs = As + BK * PT;
#pragma unroll
          for (int h = 0; h < BK * 128 / 512; ++h) {
            const int e = T.tid + 512 * h;
            const int pp = e >> 7, x = e & 127;
            const int p = p0 + pp, r = r0 + x, cc = c0 + x;
            const bool oka = p < k && r < s, okb = p < k && cc < k;
            lqm_cp_async8(As + pp * PT + x, oka ? (const void*)(Q + (lo + r) + (int64_t)cidx[p] * n) : (const void*)Q,
                          oka);
            lqm_cp_async8(Bs + pp * PT + x, okb ? (const void*)(Ubn + cc + (int64_t)p * k) : (const void*)Ubn, okb);
          }
        };
        const int nst = (k + BK - 1) / BK;
        issue(0, 0);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        if (nst > 1) issue(BK, 1);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        for (int it = 0; it < nst; ++it) {
          asm volatile("cp.async.wait_group 1;\n" ::: "memory");
          team_sync(T);
          if (it + 2 < nst) issue((it + 2) * BK, (it + 2) % NS);
          asm volatile("cp.async.commit_group;\n" ::: "memory");
          const double* As = tile + (it % NS) * STG;
          const double* Bs = As + BK * PT;
#pragma unroll
          for (int kk = 0; kk < BK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[(kk + t) * PT + wr + 8 * i + g];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[(kk + t) * PT + wc + 8 * j + g];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
              for (int j = 0; j < 4; ++j) dmma_884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
          }
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        team_sync(T);  // the ring is free before the next tile's prologue
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = r0 + wr + 8 * i + g;
#pragma unroll
          for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int cc = c0 + wc + 8 * j + 2 * t + h;
              if (r < s && cc < k) Qt[(lo + r) + (int64_t)newpos[cc] * n] = acc[i][j][h];
            }
        }
      }
    }
    return;
  }
#else
  (void)tile;
#endif
  for (int it = T.wid; it < k; it += T.nw) {
    double* dst = Qt + (int64_t)newpos[it] * n;
    for (int r = T.lane; r < s; r += T.nl) {
      double acc = 0.0;
      for (int p = 0; p < k; ++p) acc += Q[(lo + r) + (int64_t)colnd[p] * n] * Ubn[it + (int64_t)p * k];
      dst[lo + r] = acc;
    }
  }
}

// vec == false: eigenvalues only.  The merges then need just the first and
// last rows of each node's eigenvector matrix (they form z), so Q (>= 4n
// doubles) holds QF/QL (those rows, indexed by column) and FT/LT (the rows of
// the node being merged), and every merge is O(size^2).
// Ub (n*n doubles, or null) enables the tiled update for heights whose largest
// merge has >= tile_min rows: node [lo, hi) keeps its normalised secular
// vectors at Ub + lo*n as the rows of a k x k block (vector it at it + p*k).
template <class TeamT>
LQM_FN_NOINLINE void dc_solve(const TeamT& T, int n, const DCPlan& P, EighVec& S, double* Q, double* Qt,
                              unsigned long long* sub = nullptr, bool vec = true, double* Ub = nullptr,
                              int tile_min = 1 << 30) {
  double* ubuf = (double*)S.pbuf;  // per-warp secular eigenvectors (2n doubles each)
  double* QF = Q;
  double* QL = Q + n;
  double* FT = Q + 2 * n;
  double* LT = Q + 3 * n;
#if defined(__CUDA_ARCH__)
  long long tsub = clock64();
  if (T.tid != 0) sub = nullptr;
#else
  (void)sub;
#endif
  double mx = 0.0;
  for (int i = T.tid; i < n; i += T.nt) {
    mx = fmax(mx, fabs(S.d[i]));
    if (i < n - 1) mx = fmax(mx, fabs(S.e[i]));
  }
  mx = team_max(T, mx, S.red);
  double scale = 1.0;
  if (mx > 0.0) { int ex; frexp(mx, &ex); scale = ldexp(1.0, ex); }
  const double inv = 1.0 / scale;
  // Tearing: the leaves are single rows, so every boundary (i, i+1) is the
  // split point of exactly one merge node and row i loses |e[i-1]| + |e[i]|.
  // Each row is written by its own thread (no shared read-modify-write).
  for (int i = T.tid; i < n; i += T.nt) {
    const double el = (i > 0) ? fabs(S.e[i - 1] * inv) : 0.0;
    const double er = (i < n - 1) ? fabs(S.e[i] * inv) : 0.0;
    S.D[i] = (S.d[i] * inv - el) - er;
  }
  team_sync(T);
  for (int i = T.tid; i < n - 1; i += T.nt) S.e[i] *= inv;
  if (vec) {
    for (int c = T.wid; c < n; c += T.nw)
      for (int r = T.lane; r < n; r += T.nl) Q[r + (int64_t)c * n] = (r == c) ? 1.0 : 0.0;
  } else {
    for (int i = T.tid; i < n; i += T.nt) { QF[i] = 1.0; QL[i] = 1.0; }
  }
  team_sync(T);
  for (int h = 0; h < P.nheights; ++h) {
    const int h0 = P.hstart[h], h1 = P.hstart[h + 1];
    const int* own = P.owner + (int64_t)h * n;
    // A: merge vector z (scaled by 1/sqrt 2) and the merged sort order
    for (int i = T.tid; i < n; i += T.nt) {
      const int nd = own[i];
      if (nd < 0) continue;
      const int lo = P.lo[nd], m = P.mid[nd], hi = P.hi[nd];
      const double beta = S.e[m - 1];
      double zi;
      if (vec) {
        zi = (i < m) ? Q[(m - 1) + (int64_t)i * n] : ((beta < 0.0) ? -1.0 : 1.0) * Q[m + (int64_t)i * n];
      } else {
        zi = (i < m) ? QL[i] : ((beta < 0.0) ? -1.0 : 1.0) * QF[i];
        FT[i] = (i < m) ? QF[i] : 0.0;
        LT[i] = (i < m) ? 0.0 : QL[i];
      }
      S.z[i] = zi * 0.70710678118654752440;
      const double di = S.D[i];
      int cnt = 0;
      if (i < m) {
        int a = m, b = hi;  // first index in [m,hi) with D >= di
        while (a < b) { int c = (a + b) >> 1; if (S.D[c] < di) a = c + 1; else b = c; }
        cnt = a - m;
        S.perm[lo + (i - lo) + cnt] = i;
      } else {
        int a = lo, b = m;  // first index in [lo,m) with D > di
        while (a < b) { int c = (a + b) >> 1; if (S.D[c] <= di) a = c + 1; else b = c; }
        cnt = a - lo;
        S.perm[lo + (i - m) + cnt] = i;
      }
    }
    team_sync(T);
    LQM_SUBTICK(0);
    // B: gather z and D in merged order, then deflation, one thread per node
    for (int i = T.tid; i < n; i += T.nt) {
      if (own[i] < 0) continue;
      const int j = S.perm[i];
      S.zhat[i] = S.z[j];
      S.vals[i] = S.D[j];
    }
    team_sync(T);
    for (int nd = h0 + T.tid; nd < h1; nd += T.nt)
      deflate_node(nd, P, S, fabs(S.e[P.mid[nd] - 1]), S.zhat, S.vals);
    team_sync(T);
    LQM_SUBTICK(1);
    // C: secular roots
    {
      // lane-group width from the largest merge of this height (uniform)
      int kmax = 1;
      for (int nd = h0; nd < h1; ++nd) kmax = (S.nk[nd] > kmax) ? S.nk[nd] : kmax;
      const int gw = secular_width(kmax, T.nl);
      const int gpw = T.nl / gw;               // root groups per warp
      const int g = T.lane % gw;
      for (int base = T.wid * gpw; base < n; base += T.nw * gpw) {  // warp-uniform loop
        const int i = base + T.lane / gw;
        bool active = false;
        int lo = 0, q = 0, k = 0, nd = -1;
        if (i < n) {
          nd = own[i];
          if (nd >= 0) {
            lo = P.lo[nd]; q = i - lo; k = S.nk[nd];
            active = q < k;
          }
        }
        int org = 0; double tr = 0.0;
        secular_root_group(active, gw, g, active ? k : 1, active ? S.dl + lo : S.dl,
                           active ? S.zl + lo : S.zl, active ? S.nrho[nd] : 1.0, q, &org, &tr);
        if (active && g == 0) { S.org[lo + q] = org; S.troot[lo + q] = tr; }
      }
    }
    team_sync(T);
    LQM_SUBTICK(2);
    // D: Gu-Eisenstat z
    for (int i = T.tid; i < n; i += T.nt) {
      const int nd = own[i];
      if (nd < 0) continue;
      const int lo = P.lo[nd], q = i - lo, k = S.nk[nd];
      if (q >= k) continue;
      const double* dl = S.dl + lo;
      const double rho = S.nrho[nd];
      double prod = 1.0;
      for (int j = 0; j < k; ++j) {
        const double dij = (dl[q] - dl[S.org[lo + j]]) - S.troot[lo + j];
        if (j == q) prod *= -dij / rho; else prod *= -dij / (dl[j] - dl[q]);
      }
      const double zh = sqrt(fabs(prod));
      S.zhat[lo + q] = (S.zl[lo + q] < 0.0) ? -zh : zh;
    }
    team_sync(T);
    LQM_SUBTICK(3);
    // F: deflation rotations on the rows of Q (or on the two boundary rows)
    if (!vec) {
      for (int t2 = T.tid; t2 < 2 * (h1 - h0); t2 += T.nt) {
        const int nd = h0 + t2 / 2;
        double* row = (t2 & 1) ? LT : FT;
        const int lo = P.lo[nd], nr = S.nrot[nd];
        for (int t = 0; t < nr; ++t) {
          const int a = S.ri[lo + t], b = S.rj[lo + t];
          const double c = S.rc[lo + t], s = S.rs[lo + t];
          const double x = row[a], y = row[b];
          row[a] = c * x + s * y;
          row[b] = c * y - s * x;
        }
      }
    }
    for (int r = T.tid; r < n && vec; r += T.nt) {
      const int nd = own[r];
      if (nd < 0) continue;
      const int lo = P.lo[nd], nr = S.nrot[nd];
      for (int t = 0; t < nr; ++t) {
        const int a = S.ri[lo + t], b = S.rj[lo + t];
        const double c = S.rc[lo + t], s = S.rs[lo + t];
        const double x = Q[r + (int64_t)a * n], y = Q[r + (int64_t)b * n];
        Q[r + (int64_t)a * n] = c * x + s * y;
        Q[r + (int64_t)b * n] = c * y - s * x;
      }
    }
    // G: merged eigenvalue list of each node
    for (int i = T.tid; i < n; i += T.nt) {
      const int nd = own[i];
      if (nd < 0) continue;
      const int lo = P.lo[nd], it = i - lo, k = S.nk[nd];
      S.vals[i] = (it < k) ? S.dl[lo + S.org[lo + it]] + S.troot[lo + it] : S.dval[lo + it - k];
    }
    team_sync(T);
    LQM_SUBTICK(4);
    for (int i = T.tid; i < n; i += T.nt) {
      const int nd = own[i];
      if (nd < 0) continue;
      const int lo = P.lo[nd], hi = P.hi[nd];
      const double v = S.vals[i];
      int cnt = 0;
      for (int j = lo; j < hi; ++j) { const double vj = S.vals[j]; cnt += (vj < v) || (vj == v && j < i); }
      S.newpos[i] = lo + cnt;
    }
    team_sync(T);
    LQM_SUBTICK(5);
    // H: eigenvector update into Qt.  Column c by warp: the warp first forms
    // the normalised secular eigenvector u_p = zhat_p / (d_p - lambda_it) in its
    // shared buffer, then rows of the node by lane (3 independent chains).
    // Eigenvalues only: the two boundary rows, lanes splitting p.
    if (!vec) {
      for (int c = T.wid; c < n; c += T.nw) {
        const int nd = own[c];
        if (nd < 0) continue;
        const int lo = P.lo[nd], it = c - lo, k = S.nk[nd];
        const int dstc = S.newpos[c];
        if (it < k) {
          const double* dl = S.dl + lo;
          const double lorg = dl[S.org[lo + it]], tq = S.troot[lo + it];
          double ss = 0.0, f = 0.0, l = 0.0;
          for (int p = T.lane; p < k; p += T.nl) {
            const double u = S.zhat[lo + p] / ((dl[p] - lorg) - tq);
            const int col = S.colnd[lo + p];
            ss += u * u;
            f += FT[col] * u;
            l += LT[col] * u;
          }
          ss = warp_sum_bcast(ss);
          f = warp_sum_bcast(f);
          l = warp_sum_bcast(l);
          if (T.lane == 0) {
            const double sc = 1.0 / sqrt(ss);
            QF[dstc] = f * sc;
            QL[dstc] = l * sc;
          }
        } else if (T.lane == 0) {
          const int src = S.dcol[lo + it - k];
          QF[dstc] = FT[src];
          QL[dstc] = LT[src];
        }
      }
    }
    bool tiled = false;
    if (vec && Ub != nullptr)
      for (int nd = h0; nd < h1; ++nd) tiled = tiled || (P.hi[nd] - P.lo[nd] >= tile_min);
    if (tiled) {
      // secular vectors into Ub (warp per column), deflated columns copied
      for (int c = T.wid; c < n; c += T.nw) {
        const int nd = own[c];
        if (nd < 0) continue;
        const int lo = P.lo[nd], hi = P.hi[nd], it = c - lo, k = S.nk[nd];
        if (it < k) {
          double* ub = Ub + (int64_t)lo * n + it;  // row it of the node's k x k block (stride k)
          const double* dl = S.dl + lo;
          const double lorg = dl[S.org[lo + it]], tq = S.troot[lo + it];
          double ss = 0.0;
          for (int p = T.lane; p < k; p += T.nl) {
            const double u = S.zhat[lo + p] / ((dl[p] - lorg) - tq);
            ub[(int64_t)p * k] = u;
            ss += u * u;
          }
          const double sc = 1.0 / sqrt(warp_sum_bcast(ss));
          for (int p = T.lane; p < k; p += T.nl) ub[(int64_t)p * k] *= sc;
        } else {
          double* dst = Qt + (int64_t)S.newpos[c] * n;
          const double* src = Q + (int64_t)S.dcol[lo + it - k] * n;
          for (int r = lo + T.lane; r < hi; r += T.nl) dst[r] = src[r];
        }
      }
      team_sync(T);
      for (int nd = h0; nd < h1; ++nd) {
        const int lo = P.lo[nd];
        dc_tile_gemm(T, n, lo, P.hi[nd], S.nk[nd], S.colnd + lo, S.newpos + lo, Q, Qt, Ub + (int64_t)lo * n,
                     S.tile);
      }
    }
    // Columns in pairs (2t, 2t+1) by warp: when both are non-deflated columns
    // of the same merge, every Q element loaded serves both (the sums over p
    // keep their order, so the values are those of the one-column form).
    auto form_u = [&](int c, int lo, int it, int k, double* ub) {
      const double* dl = S.dl + lo;
      const double lorg = dl[S.org[lo + it]], tq = S.troot[lo + it];
      double ss = 0.0;
      for (int p = T.lane; p < k; p += T.nl) {
        const double u = S.zhat[lo + p] / ((dl[p] - lorg) - tq);
        ub[p] = u;
        ss += u * u;
      }
      const double sc = 1.0 / sqrt(warp_sum_bcast(ss));
      for (int p = T.lane; p < k; p += T.nl) ub[p] *= sc;
    };
    auto one_col = [&](int c) {
      const int nd = own[c];
      if (nd < 0) return;
      const int lo = P.lo[nd], hi = P.hi[nd], it = c - lo, k = S.nk[nd];
      double* dst = Qt + (int64_t)S.newpos[c] * n;
      if (it < k) {
        double* ub = ubuf + (int64_t)T.wid * 2 * n;
        form_u(c, lo, it, k, ub);
        team_syncwarp();
        for (int r0 = lo + T.lane; r0 < hi; r0 += 3 * T.nl) {
          const int r1 = r0 + T.nl, r2 = r0 + 2 * T.nl;
          const bool h1 = r1 < hi, h2 = r2 < hi;
          double a0 = 0.0, a1 = 0.0, a2 = 0.0;
          for (int p = 0; p < k; ++p) {
            const double* qc = Q + (int64_t)S.colnd[lo + p] * n;
            const double u = ub[p];
            a0 += qc[r0] * u;
            if (h1) a1 += qc[r1] * u;
            if (h2) a2 += qc[r2] * u;
          }
          dst[r0] = a0;
          if (h1) dst[r1] = a1;
          if (h2) dst[r2] = a2;
        }
        team_syncwarp();
      } else {
        const double* src = Q + (int64_t)S.dcol[lo + it - k] * n;
        for (int r = lo + T.lane; r < hi; r += T.nl) dst[r] = src[r];
      }
    };
    for (int t = T.wid; 2 * t < n && vec && !tiled; t += T.nw) {
      const int ca = 2 * t, cb = 2 * t + 1;
      const int nda = own[ca], ndb = (cb < n) ? own[cb] : -1;
      bool pair = false;
      if (nda >= 0 && ndb == nda) {
        const int lo = P.lo[nda], k = S.nk[nda];
        pair = (cb - lo) < k;  // ca < cb, so both are non-deflated
      }
      if (!pair) {
        one_col(ca);
        if (cb < n) one_col(cb);
        continue;
      }
      const int lo = P.lo[nda], hi = P.hi[nda], k = S.nk[nda];
      double* ua = ubuf + (int64_t)T.wid * 2 * n;
      double* ubb = ua + n;
      form_u(ca, lo, ca - lo, k, ua);
      form_u(cb, lo, cb - lo, k, ubb);
      team_syncwarp();
      double* da = Qt + (int64_t)S.newpos[ca] * n;
      double* db = Qt + (int64_t)S.newpos[cb] * n;
      for (int r0 = lo + T.lane; r0 < hi; r0 += 3 * T.nl) {
        const int r1 = r0 + T.nl, r2 = r0 + 2 * T.nl;
        const bool h1 = r1 < hi, h2 = r2 < hi;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0;
        for (int p = 0; p < k; ++p) {
          const double* qc = Q + (int64_t)S.colnd[lo + p] * n;
          const double u = ua[p], v = ubb[p];
          const double q0 = qc[r0];
          a0 += q0 * u;
          b0 += q0 * v;
          if (h1) { const double q1 = qc[r1]; a1 += q1 * u; b1 += q1 * v; }
          if (h2) { const double q2 = qc[r2]; a2 += q2 * u; b2 += q2 * v; }
        }
        da[r0] = a0;
        db[r0] = b0;
        if (h1) { da[r1] = a1; db[r1] = b1; }
        if (h2) { da[r2] = a2; db[r2] = b2; }
      }
      team_syncwarp();
    }
    team_sync(T);
    LQM_SUBTICK(6);
    // I: write back
    for (int c = T.wid; c < n && vec; c += T.nw) {
      const int nd = own[c];
      if (nd < 0) continue;
      const int lo = P.lo[nd], hi = P.hi[nd];
      for (int r = lo + T.lane; r < hi; r += T.nl) Q[r + (int64_t)c * n] = Qt[r + (int64_t)c * n];
    }
    for (int i = T.tid; i < n; i += T.nt) {
      if (own[i] < 0) continue;
      S.D[S.newpos[i]] = S.vals[i];
    }
    team_sync(T);
    LQM_SUBTICK(7);
  }
  for (int i = T.tid; i < n; i += T.nt) S.D[i] *= scale;
  team_sync(T);
}

// ---------------------------------------------------------------------------
// 4. Back-transformation U = H_0 ... H_{n-2} U (U holds Q on entry; with a column
// range [cbeg, cend) only those columns are read and transformed), applied
// in blocks of 8 reflectors with the compact WY form (LAPACK zlarft, forward,
// column-wise):  H_{j0} ... H_{j0+7} = I - V T V^H,  U_sub -= V (T (V^H U_sub)).
// Reflector j is R[j+1.., j] with v0 = 1.  V (zero-padded, ld n), T and the
// Gram matrix G = V^H V live in S.pbuf.  Each column of U belongs to a group
// of G lanes (G = 4 for n = 96 on 512 threads) that split its rows: partial
// V^H u over the group's rows, a group sum, T (V^H u), and the update of the
// group's rows, with 8 independent accumulators per lane.
// ---------------------------------------------------------------------------
template <class TeamT>
LQM_FN_NOINLINE void backtransform(const TeamT& T, int n, const double2* R, int ldr, EighVec& S, double2* U,
                                   int ldu, int cbeg = 0, int cend = -1) {
  // only the columns [cbeg, cend) of U are transformed (and read)
  if (cend < 0) cend = n;
  const int ncol = cend - cbeg;
  if (ncol <= 0) return;
  constexpr int NB = 8;
  double2* Vs = S.pbuf;                  // m x NB, leading dimension n
  double2* Ts = S.pbuf + (int64_t)NB * n;  // NB x NB
  double2* Gs = Ts + NB * NB;            // NB x NB
  for (int j1 = n - 2; j1 >= 0; j1 -= NB) {
    const int j0 = (j1 - NB + 1 > 0) ? j1 - NB + 1 : 0;
    const int b = j1 - j0 + 1;
    const int m = n - j0 - 1;  // rows j0+1 .. n-1 of U
    for (int i = T.wid; i < NB; i += T.nw)
      for (int r = T.lane; r < m; r += T.nl) {
        double2 v = cmk(0.0, 0.0);
        if (i < b && r >= i) v = R[(j0 + 1 + r) + (int64_t)(j0 + i) * ldr];
        Vs[r + (int64_t)i * n] = v;
      }
    team_sync(T);
    for (int pidx = T.wid; pidx < NB * NB; pidx += T.nw) {
      const int q = pidx % NB, i = pidx / NB;
      if (!(q < i && i < b)) continue;
      double sr = 0.0, si = 0.0;
      for (int r = i + T.lane; r < m; r += T.nl) {
        const double2 x = cmulc(Vs[r + (int64_t)q * n], Vs[r + (int64_t)i * n]);
        sr += x.x; si += x.y;
      }
      sr = warp_sum(sr); si = warp_sum(si);
      if (T.lane == 0) Gs[q + i * NB] = cmk(sr, si);
    }
    team_sync(T);
    for (int l = T.tid; l < NB; l += T.nt) {  // row l of T: T[l,l] = tau_l, T[l,i] = -tau_i sum_{q=l}^{i-1} T[l,q] G[q,i]
      double2 trow[NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) trow[i] = cmk(0.0, 0.0);
      if (l < b) trow[l] = S.tau[j0 + l];
#pragma unroll
      for (int i = 1; i < NB; ++i) {
        if (i > l && i < b) {
          double2 acc = cmk(0.0, 0.0);
#pragma unroll
          for (int q = 0; q < NB - 1; ++q)
            if (q >= l && q < i) acc = cadd(acc, cmul(trow[q], Gs[q + i * NB]));
          const double2 ti = S.tau[j0 + i];
          trow[i] = cmul(cmk(-ti.x, -ti.y), acc);
        }
      }
#pragma unroll
      for (int i = 0; i < NB; ++i) Ts[l + i * NB] = trow[i];
    }
    team_sync(T);
    // lanes per column: the largest power of two <= 8 with ncol * G <= nt (within a warp)
    int G = 1;
    while (G < 8 && 2 * G <= T.nl && ncol * (2 * G) <= T.nt) G *= 2;
    const int ngr = T.nt / G;                    // column groups
    const int g = T.tid % G;
    const int rounds = (ncol + ngr - 1) / ngr;   // uniform trip count (every lane takes part in the sums)
    for (int rd = 0; rd < rounds; ++rd) {
      const int c = cbeg + rd * ngr + T.tid / G;
      const bool act = c < cend;
      double2* Uc = U + (j0 + 1) + (int64_t)(act ? c : 0) * ldu;
      double2 w[NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) w[i] = cmk(0.0, 0.0);
      if (act) {
        for (int r = g; r < m; r += G) {
          const double2 u = Uc[r];
#pragma unroll
          for (int i = 0; i < NB; ++i) w[i] = cfma_conj(w[i], Vs[r + (int64_t)i * n], u);
        }
      }
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        w[i].x = group_sum_bcast(w[i].x, G);
        w[i].y = group_sum_bcast(w[i].y, G);
      }
      double2 wp[NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        double2 acc = cmk(0.0, 0.0);
#pragma unroll
        for (int l = 0; l < NB; ++l)
          if (l >= i) acc = cfma(acc, Ts[i + l * NB], w[l]);
        wp[i] = acc;
      }
      if (act) {
        for (int r = g; r < m; r += G) {
          double2 u = Uc[r];
#pragma unroll
          for (int i = 0; i < NB; ++i) u = cfms(u, Vs[r + (int64_t)i * n], wp[i]);
          Uc[r] = u;
        }
      }
    }
    team_sync(T);
  }
}

// ---------------------------------------------------------------------------
// 5. rho_k = U diag(f) U^H into out (n x n, leading dimension ldo), U unitary.
// rho_k is Hermitian: only entries r <= c are accumulated (tiles of 4 rows per
// lane by 4 columns per warp step; row slices entirely below the tile's columns
// are skipped) and the lower triangle is written as their conjugates.  When
// more occupations are exactly 1 than exactly 0 the complement
// rho_k = I - sum_j (1 - f_j) u_j u_j^H skips the filled states, otherwise the
// sum skips the empty ones.  Every output entry accumulates over j in order.
// ---------------------------------------------------------------------------
template <class TeamT>
LQM_FN_NOINLINE void rho_from_U(const TeamT& T, int n, const double2* U, int ldu, const double* f, double2* out,
                                int64_t ldo) {
  int n0 = 0, n1 = 0;
  for (int j = 0; j < n; ++j) {
    n0 += (f[j] == 0.0);
    n1 += (f[j] == 1.0);
  }
  const bool comp = n1 > n0;
  for (int r0 = 0; r0 < n; r0 += 4 * T.nl) {
    for (int c0 = 4 * T.wid; c0 < n; c0 += 4 * T.nw) {
      // row slices q with a row <= c0 + 3 (uniform across the warp)
      const int qn = (c0 + 3 < r0) ? 0 : ((c0 + 3 - r0) / T.nl + 1 < 4 ? (c0 + 3 - r0) / T.nl + 1 : 4);
      if (qn == 0) continue;
      double2 acc[4][4];
      int rr[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        rr[q] = r0 + q * T.nl + T.lane;
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[q][b] = cmk(0.0, 0.0);
      }
      for (int j = 0; j < n; ++j) {
        const double gj = comp ? 1.0 - f[j] : f[j];
        if (gj == 0.0) continue;
        const double2* Uj = U + (int64_t)j * ldu;
        double2 cb[4], ua[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int c = c0 + b;
          cb[b] = (c < n) ? cscale(gj, cconj(Uj[c])) : cmk(0.0, 0.0);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) ua[q] = (q < qn && rr[q] < n) ? Uj[rr[q]] : cmk(0.0, 0.0);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (q < qn)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[q][b] = cfma(acc[q][b], ua[q], cb[b]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int r = rr[q], c = c0 + b;
          if (q < qn && r < n && c < n && r <= c) {
            double2 v = acc[q][b];
            if (comp) v = cmk(((r == c) ? 1.0 : 0.0) - v.x, -v.y);
            out[r + (int64_t)c * ldo] = v;
            if (r != c) out[c + (int64_t)r * ldo] = cconj(v);
          }
        }
    }
  }
  team_sync(T);
}
