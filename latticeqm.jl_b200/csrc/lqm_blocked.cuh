// Blocked Householder tridiagonalisation for large n (LAPACK zhetrd + zlatrd,
// lower), written as team phases so the batched kernels and the host
// emulation share the arithmetic.
//
// Storage per k-point: A (n x n, leading dimension lda) holds the FULL
// Hermitian matrix; panels of `nb` columns are reduced one column at a time:
//
//   blk_column(j):  finish w of column j-1 (alpha = -1/2 tau w^H v, w += alpha v),
//                   update column j with the panel's earlier reflectors
//                   (A(j:,j) -= V(j:,0:i) W(j,0:i)^H + W(j:,0:i) V(j,0:i)^H),
//                   zlarfg on A(j+1:, j) (v0 = 1 stored at A(j+1, j)), and the
//                   panel products t1 = W(j+1:,0:i)^H v, t2 = V(j+1:,0:i)^H v;
//   blk_gemv_rows:  w(r) = tau_j (A(r, j+1:) v - V(r,0:i) t1 - W(r,0:i) t2) for a
//                   slab of rows r (several teams per k-point share one column);
//
// and after the panel the trailing block gets the rank-2nb update
// A22 -= V W^H + W V^H (both triangles, batched GEMMs issued by the host).
// Every entry the mat-vec reads is either untouched since the panel began or
// already updated in the same way LAPACK's zhemv sees it, so the w vectors are
// those of zlatrd.  Outputs: d[n], e[n-1], tau[n-1]; reflector j is
// A(j+1:, j) with v0 = 1 — the same reflectors the unblocked hetrd_lower makes.
//
// Reference: LAPACK zhetrd/zlatrd (lower), the reduction inside zheevr, which
// LatticeQM's Eigen.jl:22-23 reaches through Julia's LinearAlgebra.
#pragma once
#include "lqm_eigh.cuh"

// Finish w for column jp = j0 + ip (rows jp+1..n-1): alpha = -1/2 tau (w^H v),
// w += alpha v.  Ends with a barrier.
LQM_FN void blk_finish_w(const Team& T, int n, int jp, int ip, const double2* A, int lda, double2* W, int ldw,
                         const double2* tau, double* red) {
  const double2* v = A + (int64_t)jp * lda;
  double2* w = W + (int64_t)ip * ldw;
  double pr = 0.0, pi = 0.0;
  for (int r = jp + 1 + T.tid; r < n; r += T.nt) {
    const double2 q = cmulc(w[r], v[r]);
    pr += q.x; pi += q.y;
  }
  team_sum2_1b(T, pr, pi, red);
  const double2 tj = tau[jp];
  const double2 alpha = cmul(cmk(-0.5 * tj.x, -0.5 * tj.y), cmk(pr, pi));
  for (int r = jp + 1 + T.tid; r < n; r += T.nt) w[r] = cadd(w[r], cmul(alpha, v[r]));
  team_sync();
}

// Column j = j0 + i of the panel.  red: >= 128 doubles of team scratch;
// t12: 2*nb complex (t1 at [0, nb), t2 at [nb, 2nb)).
LQM_FN void blk_column(const Team& T, int n, int nb, int j0, int i, double2* A, int lda, double2* W, int ldw,
                       double2* tau, double* d, double* e, double2* t12, double* red) {
  const int j = j0 + i;
  if (i > 0) blk_finish_w(T, n, j - 1, i - 1, A, lda, W, ldw, tau, red);
  // update column j (rows j..n-1) with reflectors j0 .. j-1
  double2* col = A + (int64_t)j * lda;
  for (int r = j + T.tid; r < n; r += T.nt) {
    double2 a = col[r];
    if (r == j) a.y = 0.0;
    for (int l = 0; l < i; ++l) {
      const double2* vl = A + (int64_t)(j0 + l) * lda;
      const double2* wl = W + (int64_t)l * ldw;
      a = csub(a, cadd(cmul(vl[r], cconj(wl[j])), cmul(wl[r], cconj(vl[j]))));
    }
    if (r == j) a.y = 0.0;
    col[r] = a;
  }
  team_sync();
  if (T.tid == 0) d[j] = col[j].x;
  if (j >= n - 1) { team_sync(); return; }
  // zlarfg on (A(j+1, j), A(j+2:, j))
  double s = 0.0, dummy = 0.0;
  for (int r = j + 2 + T.tid; r < n; r += T.nt) { const double2 x = col[r]; s += x.x * x.x + x.y * x.y; }
  team_sum2_1b(T, s, dummy, red + 64);
  const double2 alpha = col[j + 1];
  double2 tj, scal;
  double beta;
  zlarfg_scalars(alpha, s, &tj, &beta, &scal);
  team_sync();  // every thread has read alpha before it is overwritten
  for (int r = j + 2 + T.tid; r < n; r += T.nt) col[r] = cmul(scal, col[r]);
  if (T.tid == 0) { col[j + 1] = cmk(1.0, 0.0); tau[j] = tj; e[j] = beta; }
  team_sync();
  // t1 = W(j+1:, 0:i)^H v, t2 = V(j+1:, 0:i)^H v, one warp per product
  for (int q = T.wid; q < 2 * i; q += T.nw) {
    const double2* x = (q < i) ? W + (int64_t)q * ldw : A + (int64_t)(j0 + q - i) * lda;
    double sr = 0.0, si = 0.0;
    for (int r = j + 1 + T.lane; r < n; r += T.nl) {
      const double2 p = cmulc(x[r], col[r]);
      sr += p.x; si += p.y;
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if (T.lane == 0) t12[(q < i) ? q : nb + (q - i)] = cmk(sr, si);
  }
  team_sync();
}

// w rows [r0, r1) of column j = j0 + i (r0 >= j+1):
//   w(r) = tau_j (sum_c A(r, c) v_c - V(r, 0:i) t1 - W(r, 0:i) t2), c = j+1..n-1.
// vs: team scratch of n - j - 1 complex (v is staged there); part: nw * RB
// complex for the per-warp column partials (RB = r1 - r0 <= 4 * nl).
LQM_FN void blk_gemv_rows(const Team& T, int n, int nb, int j0, int i, int r0, int r1, const double2* A, int lda,
                          double2* W, int ldw, const double2* tau, const double2* t12, double2* vs, double2* part) {
  const int j = j0 + i;
  const int m = n - j - 1;
  const double2* v = A + (int64_t)j * lda + (j + 1);
  for (int c = T.tid; c < m; c += T.nt) vs[c] = v[c];
  team_sync();
  const int rb = r1 - r0;
  for (int q0 = 0; q0 < rb; q0 += 4 * T.nl) {
    double2 acc[4];
    int rr[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) { rr[q] = q0 + q * T.nl + T.lane; acc[q] = cmk(0.0, 0.0); }
    for (int c = T.wid; c < m; c += T.nw) {
      const double2* Ac = A + (int64_t)(j + 1 + c) * lda + r0;
      const double2 vc = vs[c];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (rr[q] < rb) acc[q] = cadd(acc[q], cmul(Ac[rr[q]], vc));
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (rr[q] < rb) part[(int64_t)T.wid * (4 * T.nl) + rr[q] - q0] = acc[q];
    team_sync();
    const double2 tj = tau[j];
    for (int t = T.tid; t < 4 * T.nl && q0 + t < rb; t += T.nt) {
      const int r = r0 + q0 + t;
      double2 y = cmk(0.0, 0.0);
      for (int wv = 0; wv < T.nw; ++wv) y = cadd(y, part[(int64_t)wv * (4 * T.nl) + t]);
      for (int l = 0; l < i; ++l) {
        y = csub(y, cmul(A[r + (int64_t)(j0 + l) * lda], t12[l]));
        y = csub(y, cmul(W[r + (int64_t)l * ldw], t12[nb + l]));
      }
      W[r + (int64_t)i * ldw] = cmul(tj, y);
    }
    team_sync();
  }
}

// After the reduction: make the reflector columns explicit for the blocked
// back-transformation — zeros on and above the diagonal of columns 0..n-2,
// v0 = 1 below it.  Column c by warp.
LQM_FN void blk_prep_reflectors(const Team& T, int n, double2* A, int lda) {
  for (int c = T.wid; c < n; c += T.nw) {
    double2* col = A + (int64_t)c * lda;
    for (int r = T.lane; r <= c && r < n; r += T.nl) col[r] = cmk(0.0, 0.0);
    if (T.lane == 0 && c + 1 < n) col[c + 1] = cmk(1.0, 0.0);
  }
}

// Compact WY factor of reflectors j0 .. j0+nbr-1 (LAPACK zlarft, forward,
// column-wise): H_{j0} ... H_{j0+nbr-1} = I - V Tm V^H, Tm upper triangular
// (nb x nb, leading dimension nb, zero-padded).  V(:, l) = A(j0+1:, j0+l) after
// blk_prep_reflectors.  G: nb*nb complex team scratch.
LQM_FN void blk_larft(const Team& T, int n, int nb, int j0, int nbr, const double2* A, int lda, const double2* tau,
                      double2* Tm, double2* G) {
  const int m = n - j0 - 1;
  const double2* V = A + (int64_t)j0 * lda + (j0 + 1);
  for (int p = T.wid; p < nb * nb; p += T.nw) {
    const int q = p % nb, l = p / nb;
    if (!(q < l && l < nbr)) continue;
    double sr = 0.0, si = 0.0;
    for (int r = l + T.lane; r < m; r += T.nl) {
      const double2 x = cmulc(V[r + (int64_t)q * lda], V[r + (int64_t)l * lda]);
      sr += x.x; si += x.y;
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if (T.lane == 0) G[q + l * nb] = cmk(sr, si);
  }
  for (int p = T.tid; p < nb * nb; p += T.nt) {
    const int q = p % nb, l = p / nb;
    Tm[p] = (q == l && l < nbr) ? tau[j0 + l] : cmk(0.0, 0.0);
  }
  team_sync();
  // column l: Tm(0:l, l) = -tau_l Tm(0:l, 0:l) G(0:l, l), row q by thread
  for (int l = 1; l < nbr; ++l) {
    const double2 tl = tau[j0 + l];
    for (int q = T.tid; q < l; q += T.nt) {
      double2 acc = cmk(0.0, 0.0);
      for (int s = q; s < l; ++s) acc = cadd(acc, cmul(Tm[q + s * nb], G[s + l * nb]));
      Tm[q + l * nb] = cmul(cmk(-tl.x, -tl.y), acc);
    }
    team_sync();
  }
}
