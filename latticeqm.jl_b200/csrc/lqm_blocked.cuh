// Blocked Householder tridiagonalisation for large n (LAPACK zhetrd + zlatrd,
// lower), written as team phases so the batched kernels and the host
// emulation share the arithmetic.
//
// Storage per k-point: A (n x n, leading dimension lda) holds the Hermitian
// matrix in its lower triangle; panels of `nb` columns are reduced one column
// at a time:
//
//   blk_column(j):  finish w of column j-1 from its partials
//                   (w = tau (y - V t1 - W t2), alpha = -1/2 tau w^H v, w += alpha v)
//                   fused with the update of column j by the panel's earlier
//                   reflectors (A(j:,j) -= V(j:,0:i) W(j,0:i)^H + W(j:,0:i) V(j,0:i)^H),
//                   then zlarfg on A(j+1:, j) (v0 = 1 stored at A(j+1, j));
//   blk_symv_tile:  y = A22 v from the LOWER triangle only, one 2nl x 2nl tile
//                   per team (many teams per k-point), ordered partial vectors;
//   blk_t12_slab:   partial panel products t1 = W(j+1:,0:i)^H v, t2 = V(j+1:,0:i)^H v
//                   over row slabs (issued with the tiles of the same column);
//
// and after the panel the trailing block gets the rank-2nb update
// A22 -= V W^H + W V^H (lower triangle, batched GEMMs issued by the host).
// Only the lower triangle of A is read or kept current; every entry the
// mat-vec reads is untouched since the panel began, as in LAPACK's zhemv, so
// the w vectors are those of zlatrd.  Outputs: d[n], e[n-1], tau[n-1]; reflector j is
// A(j+1:, j) with v0 = 1 — the same reflectors the unblocked hetrd_lower makes.
//
// Reference: LAPACK zhetrd/zlatrd (lower), the reduction inside zheevr, which
// LatticeQM's Eigen.jl:22-23 reaches through Julia's LinearAlgebra.
#pragma once
#include "lqm_eigh.cuh"

// Tile size of the Hermitian mat-vec: 2 rows per lane (64 for a CUDA team).
LQM_FN int symv_tb(const Team& T) { return 2 * T.nl; }
LQM_FN int symv_nblk(const Team& T, int m) { return (m + symv_tb(T) - 1) / symv_tb(T); }

// Row slab of the panel products for column j = j0 + i: rows
// j+1 + slab*4nl .. (+4nl), one warp per product q < 2i:
//   tp[slab*2nb + q]       = sum_r conj(W(r, q)) v_r        (t1, q < i)
//   tp[slab*2nb + nb + l]  = sum_r conj(V(r, l)) v_r        (t2, q = i + l)
LQM_FN int t12_rows(const Team& T) { return 4 * T.nl; }
LQM_FN void blk_t12_slab(const Team& T, int n, int nb, int j0, int i, int slab, const double2* A, int lda,
                         const double2* W, int ldw, double2* tp) {
  const int j = j0 + i;
  const int r0 = j + 1 + slab * t12_rows(T);
  const double2* v = A + (int64_t)j * lda;
  double2 vr[4];
  int rr[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    rr[q] = r0 + q * T.nl + T.lane;
    vr[q] = (rr[q] < n) ? v[rr[q]] : cmk(0.0, 0.0);
  }
  for (int q = T.wid; q < 2 * i; q += T.nw) {
    const double2* x = (q < i) ? W + (int64_t)q * ldw : A + (int64_t)(j0 + q - i) * lda;
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (rr[u] < n) {
        const double2 p = cmulc(x[rr[u]], vr[u]);
        sr += p.x; si += p.y;
      }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if (T.lane == 0) tp[(int64_t)slab * 2 * nb + ((q < i) ? q : nb + (q - i))] = cmk(sr, si);
  }
}

// Finishes w of column jp = j0 + ip (rows jp+1..) from the tile partials
// `part` and slab partials `tp` of its mat-vec:
//   t1, t2 = sum over slabs (in order);  w' = tau (sum_src part - V(r,0:ip) t1 - W(r,0:ip) t2),
//   alpha = -1/2 tau (w'^H v),  w = w' + alpha v.
// With col != null (column j = jp + 1 of the same panel) the same row pass
// also applies the reflectors 0..ip-1 to col, and the last pass the reflector
// ip, so the panel rows are read once.  t12: 2*nb complex scratch.  Ends with
// a barrier.
LQM_FN void blk_prev_w(const Team& T, int n, int nb, int j0, int ip, double2* A, int lda, double2* W, int ldw,
                       const double2* tau, double2* t12, double* red, const double2* part, const double2* tp,
                       double2* col) {
  const int jp = j0 + ip, j = jp + 1;
  const int m = n - jp - 1;
  const int TB = symv_tb(T), nbk = symv_nblk(T, m);
  const int nsl = (m + t12_rows(T) - 1) / t12_rows(T);
  for (int q = T.tid; q < 2 * ip; q += T.nt) {
    const int idx = (q < ip) ? q : nb + (q - ip);
    double2 acc = cmk(0.0, 0.0);
    for (int sl = 0; sl < nsl; ++sl) acc = cadd(acc, tp[(int64_t)sl * 2 * nb + idx]);
    t12[idx] = acc;
  }
  team_sync();
  const double2* v = A + (int64_t)jp * lda;
  double2* w = W + (int64_t)ip * ldw;
  const double2 tj = tau[jp];
  double pr = 0.0, pi = 0.0;
  for (int r = j + T.tid; r < n; r += T.nt) {
    const int x = r - j, rb = x / TB, xo = x - rb * TB;
    const double2* prt = part + (int64_t)rb * nbk * TB + xo;
    double2 y = cmk(0.0, 0.0);
#pragma unroll 8
    for (int src = 0; src < nbk; ++src) y = cadd(y, prt[(int64_t)src * TB]);
    double2 c0 = cmk(0.0, 0.0), c1 = cmk(0.0, 0.0), u0 = cmk(0.0, 0.0), u1 = cmk(0.0, 0.0);
#pragma unroll 8
    for (int l = 0; l < ip; ++l) {
      const double2 vl = A[r + (int64_t)(j0 + l) * lda];
      const double2 wl = W[r + (int64_t)l * ldw];
      c0 = cadd(c0, cmul(vl, t12[l]));
      c1 = cadd(c1, cmul(wl, t12[nb + l]));
      if (col) {
        u0 = cadd(u0, cmul(vl, cconj(W[j + (int64_t)l * ldw])));
        u1 = cadd(u1, cmul(wl, cconj(A[j + (int64_t)(j0 + l) * lda])));
      }
    }
    const double2 wr = cmul(tj, csub(y, cadd(c0, c1)));
    w[r] = wr;
    const double2 q = cmulc(wr, v[r]);
    pr += q.x; pi += q.y;
    if (col) {
      double2 a = col[r];
      if (r == j) a.y = 0.0;
      col[r] = csub(a, cadd(u0, u1));
    }
  }
  team_sum2_1b(T, pr, pi, red);
  const double2 alpha = cmul(cmk(-0.5 * tj.x, -0.5 * tj.y), cmk(pr, pi));
  if (col) {
    // row j of the finished w (computed by every thread; v[j] = 1)
    const double2 wj = cadd(w[j], cmul(alpha, v[j]));
    const double2 cwj = cconj(wj), cvj = cconj(v[j]);
    team_sync();  // w[j] has been read by every thread before it is rewritten
    for (int r = j + T.tid; r < n; r += T.nt) {
      const double2 wr = cadd(w[r], cmul(alpha, v[r]));
      w[r] = wr;
      double2 a = csub(col[r], cadd(cmul(v[r], cwj), cmul(wr, cvj)));
      if (r == j) a.y = 0.0;
      col[r] = a;
    }
  } else {
    for (int r = j + T.tid; r < n; r += T.nt) w[r] = cadd(w[r], cmul(alpha, v[r]));
  }
  team_sync();
}

// Column j = j0 + i of the panel.  red: >= 128 doubles of team scratch;
// t12: 2*nb complex scratch; part/tp: partials of column j-1's mat-vec.
LQM_FN void blk_column(const Team& T, int n, int nb, int j0, int i, double2* A, int lda, double2* W, int ldw,
                       double2* tau, double* d, double* e, double2* t12, double* red, const double2* part,
                       const double2* tp) {
  const int j = j0 + i;
  double2* col = A + (int64_t)j * lda;
  if (i > 0) {
    blk_prev_w(T, n, nb, j0, i - 1, A, lda, W, ldw, tau, t12, red, part, tp, col);
  } else {
    if (T.tid == 0) col[j].y = 0.0;
    team_sync();
  }
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
}

// One tile (R, C), R >= C, of y = A22 v for column j (A22 = A(j+1:, j+1:),
// lower triangle only, v = A(j+1:, j)), tile size TB = 2 nl.  The tile is
// staged in shared memory (ts: TB x (TB+1) complex, padded so that row- and
// column-wise reads are conflict-free) with all its loads in flight at once;
// then threads own rows (direct product) and columns (transposed product) in
// groups that split the other index.  Writes
//   part[(R*nbk + C)*TB + x]  = sum_c A(R x, C c) v_c          (direct),
//   part[(C*nbk + R)*TB + x]  = sum_r conj(A(R r, C x)) v_r    (transposed),
// and on a diagonal tile their sum (lower entries only, the diagonal once).
// vs: 2 TB complex; red: 2 * max(1, nt/TB) * TB complex.
LQM_FN void blk_symv_tile(const Team& T, int n, int j, int R, int C, const double2* A, int lda, double2* part,
                          double2* ts, double2* vs, double2* red) {
  const int m = n - j - 1;
  const int TB = symv_tb(T), nbk = symv_nblk(T, m), ld = TB + 1;
  const double2* B = A + (j + 1) + (int64_t)(j + 1) * lda;  // A22
  const double2* v = A + (j + 1) + (int64_t)j * lda;
  const bool diag = (R == C);
  const int x0 = R * TB, y0 = C * TB;
  constexpr int kStage = 16;  // loads per thread in flight when TB * TB == 16 * nt
  if (TB * TB == kStage * T.nt) {
    double2 rg[kStage];
#pragma unroll
    for (int h = 0; h < kStage; ++h) {
      const int idx = T.tid + h * T.nt, rr = idx % TB, cc = idx / TB;
      const int x = x0 + rr, y = y0 + cc;
      rg[h] = (x < m && y < m && (!diag || rr >= cc)) ? B[x + (int64_t)y * lda] : cmk(0.0, 0.0);
    }
#pragma unroll
    for (int h = 0; h < kStage; ++h) {
      const int idx = T.tid + h * T.nt, rr = idx % TB, cc = idx / TB;
      double2 a = rg[h];
      if (diag && rr == cc) a.y = 0.0;
      ts[rr + cc * ld] = a;
    }
  } else {
    for (int idx = T.tid; idx < TB * TB; idx += T.nt) {
      const int rr = idx % TB, cc = idx / TB;
      const int x = x0 + rr, y = y0 + cc;
      double2 a = cmk(0.0, 0.0);
      if (x < m && y < m && (!diag || rr >= cc)) a = B[x + (int64_t)y * lda];
      if (diag && rr == cc) a.y = 0.0;
      ts[rr + cc * ld] = a;
    }
  }
  for (int t = T.tid; t < 2 * TB; t += T.nt) {
    const int x = (t < TB) ? x0 + t : y0 + (t - TB);
    vs[t] = (x < m) ? v[x] : cmk(0.0, 0.0);
  }
  team_sync();
  const int ng = (T.nt / TB > 0) ? T.nt / TB : 1;
  double2* rd = red;                    // [ng][TB] direct
  double2* rt = red + (int64_t)ng * TB; // [ng][TB] transposed
  for (int t = T.tid; t < ng * TB; t += T.nt) {
    const int q = t % TB, g = t / TB;
    double2 ad = cmk(0.0, 0.0), at = cmk(0.0, 0.0);
    for (int u = g; u < TB; u += ng) {
      ad = cadd(ad, cmul(ts[q + u * ld], vs[TB + u]));                // row q, column u
      if (!(diag && u == q)) at = cadd(at, cmulc(ts[u + q * ld], vs[u]));  // row u, column q
    }
    rd[t] = ad;
    rt[t] = at;
  }
  team_sync();
  double2* pd = part + ((int64_t)R * nbk + C) * TB;
  double2* pt = part + ((int64_t)C * nbk + R) * TB;
  for (int x = T.tid; x < TB; x += T.nt) {
    double2 yd = cmk(0.0, 0.0), yt = cmk(0.0, 0.0);
    for (int g = 0; g < ng; ++g) {
      yd = cadd(yd, rd[(int64_t)g * TB + x]);
      yt = cadd(yt, rt[(int64_t)g * TB + x]);
    }
    if (diag) {
      pd[x] = cadd(yd, yt);
    } else {
      pd[x] = yd;
      pt[x] = yt;
    }
  }
}

// After the reduction: make the reflector columns explicit for the blocked
// back-transformation — reflector c starts at row c + off (off = 1 for the
// one-stage reduction, the half-bandwidth for the two-stage one): zeros above
// that row, v0 = 1 on it.  Column c by warp.
LQM_FN void blk_prep_reflectors(const Team& T, int n, double2* A, int lda, int off = 1) {
  for (int c = T.wid; c < n; c += T.nw) {
    double2* col = A + (int64_t)c * lda;
    for (int r = T.lane; r < c + off && r < n; r += T.nl) col[r] = cmk(0.0, 0.0);
    if (T.lane == 0 && c + off < n) col[c + off] = cmk(1.0, 0.0);
  }
}

// Compact WY factor of reflectors j0 .. j0+nbr-1 (LAPACK zlarft, forward,
// column-wise): H_{j0} ... H_{j0+nbr-1} = I - V Tm V^H, Tm upper triangular
// (nb x nb, leading dimension nb, zero-padded).  V(:, l) = A(j0+off:, j0+l) after
// blk_prep_reflectors.  G: nb*nb complex team scratch for the Gram matrix V^H V,
// formed here from V or, with Gg != null, copied from Gg (nb x nb, leading
// dimension nb, formed beforehand by a GEMM).
LQM_FN void blk_larft(const Team& T, int n, int nb, int j0, int nbr, const double2* A, int lda, const double2* tau,
                      double2* Tm, double2* G, const double2* Gg = nullptr, int off = 1) {
  const int m = n - j0 - off;
  const double2* V = A + (int64_t)j0 * lda + (j0 + off);
  if (Gg) {
    for (int p = T.tid; p < nb * nb; p += T.nt) G[p] = Gg[p];
  } else {
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
