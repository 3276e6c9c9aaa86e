// Two-stage Hermitian tridiagonalisation for the batched large-n path, written
// as team phases so the CUDA kernels and the host emulation share the arithmetic.
//
//   stage 1, dense -> band of half-bandwidth b (LAPACK zhetrd_he2hb, lower): per
//     panel of b columns a QR of the m x b block below the band (ts_panel_qr),
//     then A22 <- Q^H A22 Q by GEMMs issued by the host:
//       Y = A22 V (A22 Hermitian, lower storage),  X = Y T,
//       W = X - 1/2 V (T^H (V^H X)),  A22 -= V W^H + W V^H  (lower triangle);
//     reflector j (j < n - b) is A(j+b:, j) with v0 = 1 implicit, A(j+b, j) = beta.
//   stage 2, band -> real tridiagonal (LAPACK zhetrd_hb2st): bulge chasing.
//     Sweep s annihilates column s below its subdiagonal; task t of the sweep
//     (ts_chase_sweep) makes one reflector from the first column of the block the
//     previous task filled, applies it from the left to the rest of that block,
//     two-sided to its diagonal block and from the right to the block below,
//     which becomes the next task's block.  Only the first column of each bulge
//     is removed; the rest lies in the columns the next sweep annihilates, so the
//     band never grows beyond 2b - 1 subdiagonals.  Successive sweeps can run
//     concurrently when sweep s+1 stays three tasks behind sweep s.
//   back-transformation U = Q1 Q2 Z: the stage-2 reflectors in the reverse order of
//     the chase (ts_q2_apply_host) or, as the device applies them, grouped by 16
//     sweeps and task index (ts_q2_apply_grouped_host: the same product, since the
//     reorder only exchanges reflectors on disjoint rows), then Q1 as compact-WY
//     products (blk_larft and the GEMMs of the one-stage path, rows offset by b).
//
// The reference reaches the same factorisation through Julia's LinearAlgebra
// (LAPACK zheevr on Hermitian(M), Eigen.jl:22-23); LAPACK's own two-stage driver
// (zheevr_2stage) reduces in these two steps.
#pragma once
#include "lqm_blocked.cuh"

// Band storage of stage 2: element (i, j), 0 <= i - j < ldb (ldb = 2b), at
// Bd[(i - j) + j * ldb]; the upper triangle is implied by Hermitian symmetry.
LQM_FN double2 ts_bget(const double2* Bd, int ldb, int i, int j) { return Bd[(i - j) + (int64_t)j * ldb]; }
LQM_FN double2* ts_bptr(double2* Bd, int ldb, int i, int j) { return Bd + (i - j) + (int64_t)j * ldb; }

#if defined(__CUDACC__)
#define LQM_HD __host__ __device__ inline
#else
#define LQM_HD static inline
#endif
// Tasks of sweep s: the row blocks [s+1+t b, s+1+(t+1) b) that start inside the matrix.
LQM_HD int ts_tasks(int n, int b, int s) { return (n - 1 - s + b - 1) / b; }
// Reflector slots per sweep in the stage-2 reflector store (the first sweep's count).
LQM_HD int ts_tmax(int n, int b) { return n > 1 ? (n - 1 + b - 1) / b : 1; }

// QR of the panel below the band (LAPACK zgeqr2 on rows j0+b..n-1 of columns
// j0..j0+pw-1, pw = min(b, n - j0), m = n - j0 - b rows, nr = min(b, m) reflectors),
// then the explicit reflectors Vb (m x nr, leading dimension ldv: zero above the
// unit diagonal) and the compact-WY factor Tm (b x b, leading dimension b, zlarft
// forward, upper triangular, zero-padded).  Per column c: zlarfg on A(j+b:, j),
// j = j0 + c; then H^H = I - conj(tau) v v^H on the panel columns right of it.
// sm: team scratch of >= (nw + 2) * B + B * B complex (nw = warps of the team).
template <int B, class TeamT>
LQM_FN void ts_panel_qr(const TeamT& T, int n, int j0, double2* A, int lda, double2* tau, double2* Vb, int ldv,
                        double2* Tm, double2* sm) {
  const int m = n - j0 - B;
  const int pw = (n - j0 < B) ? n - j0 : B;
  const int nr = (m < B) ? m : B;
  double2* part = sm;               // nw x B warp partials
  double2* wv = sm + T.nw * B;      // B: the reduced w_l
  double2* G = wv + 2 * B;          // B x B Gram matrix V^H V
  double* red = (double*)(wv + B);  // 2B doubles
  for (int c = 0; c < nr; ++c) {
    const int j = j0 + c;
    double2* col = A + (int64_t)j * lda;
    const int r0 = j + B;  // the reflector's first row
    double s = 0.0;
    for (int r = r0 + 1 + T.tid; r < n; r += T.nt) { const double2 x = col[r]; s += x.x * x.x + x.y * x.y; }
#if defined(__CUDACC__)
    s = warp_sum(s);
    if (T.lane == 0) red[T.wid] = s;
    team_sync(T);
    s = 0.0;
    for (int w = 0; w < T.nw; ++w) s += red[w];
#endif
    const double2 alpha = col[r0];
    double2 tj, scal;
    double beta;
    zlarfg_scalars(alpha, s, &tj, &beta, &scal);
    team_sync(T);  // alpha (and red) read by every thread
    for (int r = r0 + 1 + T.tid; r < n; r += T.nt) col[r] = cmul(scal, col[r]);
    if (T.tid == 0) { col[r0] = cmk(beta, 0.0); tau[j] = tj; }
    team_sync(T);
    if (c + 1 >= pw) continue;
    // w_l = sum_r conj(v_r) A(r, j0 + l), l = c+1 .. pw-1 (v_{r0} = 1)
    double2 acc[B];
#pragma unroll
    for (int l = 0; l < B; ++l) acc[l] = cmk(0.0, 0.0);
    for (int r = r0 + T.tid; r < n; r += T.nt) {
      const double2 vr = (r == r0) ? cmk(1.0, 0.0) : col[r];
#pragma unroll
      for (int l = 0; l < B; ++l)
        if (l > c && l < pw) acc[l] = cadd(acc[l], cmulc(vr, A[r + (int64_t)(j0 + l) * lda]));
    }
#pragma unroll
    for (int l = 0; l < B; ++l) {
      if (!(l > c && l < pw)) continue;
      const double ar = warp_sum(acc[l].x), ai = warp_sum(acc[l].y);
      if (T.lane == 0) part[T.wid * B + l] = cmk(ar, ai);
    }
    team_sync(T);
    for (int l = c + 1 + T.tid; l < pw; l += T.nt) {
      double2 w = cmk(0.0, 0.0);
      for (int q = 0; q < T.nw; ++q) w = cadd(w, part[q * B + l]);
      wv[l] = cmul(cconj(tj), w);  // conj(tau) w_l
    }
    team_sync(T);
    for (int r = r0 + T.tid; r < n; r += T.nt) {
      const double2 vr = (r == r0) ? cmk(1.0, 0.0) : col[r];
      for (int l = c + 1; l < pw; ++l) {
        double2* a = A + r + (int64_t)(j0 + l) * lda;
        *a = csub(*a, cmul(vr, wv[l]));
      }
    }
    team_sync(T);
  }
  if (nr <= 0) return;
  // explicit reflectors: Vb(r, c) = 0 (r < c), 1 (r == c), A(j0+B+r, j0+c) (r > c)
  for (int64_t idx = T.tid; idx < (int64_t)m * nr; idx += T.nt) {
    const int r = (int)(idx % m), c = (int)(idx / m);
    Vb[r + (int64_t)c * ldv] =
        (r < c) ? cmk(0.0, 0.0) : (r == c) ? cmk(1.0, 0.0) : A[(j0 + B + r) + (int64_t)(j0 + c) * lda];
  }
  team_sync(T);
  // Gram matrix G(q, l) = sum_r conj(V(r, q)) V(r, l), q < l (rows r >= l), warp per pair
  for (int p = T.wid; p < B * B; p += T.nw) {
    const int q = p % B, l = p / B;
    if (!(q < l && l < nr)) continue;
    double sr = 0.0, si = 0.0;
    for (int r = l + T.lane; r < m; r += T.nl) {
      const double2 x = cmulc(Vb[r + (int64_t)q * ldv], Vb[r + (int64_t)l * ldv]);
      sr += x.x; si += x.y;
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if (T.lane == 0) G[q + l * B] = cmk(sr, si);
  }
  for (int p = T.tid; p < B * B; p += T.nt) {
    const int q = p % B, l = p / B;
    Tm[p] = (q == l && l < nr) ? tau[j0 + l] : cmk(0.0, 0.0);
  }
  team_sync(T);
  // zlarft forward: Tm(0:l, l) = -tau_l Tm(0:l, 0:l) G(0:l, l)
  for (int l = 1; l < nr; ++l) {
    const double2 tl = tau[j0 + l];
    for (int q = T.tid; q < l; q += T.nt) {
      double2 acc = cmk(0.0, 0.0);
      for (int s2 = q; s2 < l; ++s2) acc = cadd(acc, cmul(Tm[q + s2 * B], G[s2 + l * B]));
      Tm[q + l * B] = cmul(cmk(-tl.x, -tl.y), acc);
    }
    team_sync(T);
  }
}

// Band of half-bandwidth B out of the stage-1 result (lower triangle of A): the
// diagonal blocks and the R factors; the fill diagonals B+1 .. 2B-1 start at zero.
template <int B, class TeamT>
LQM_FN void ts_band_extract(const TeamT& T, int n, const double2* A, int lda, double2* Bd) {
  const int ldb = 2 * B;
  for (int64_t idx = T.tid; idx < (int64_t)ldb * n; idx += T.nt) {
    const int o = (int)(idx % ldb), j = (int)(idx / ldb);
    const int i = j + o;
    double2 v = cmk(0.0, 0.0);
    if (i < n && o <= B) v = A[i + (int64_t)j * lda];
    if (o == 0) v.y = 0.0;
    Bd[idx] = v;
  }
}

// One sweep s of the bulge chase on the band Bd (ldb = 2B).  Task t makes the
// reflector H = I - tau v v^H (zlarfg: H^H x = beta e1, v0 = 1) from
//   t = 0:  x = column s, rows s+1 .. s+L
//   t > 0:  x = column c = s+1+(t-1)B, rows R0 .. R0+L-1 (R0 = s+1+tB)
// with L = min(B, n - R0); then
//   F <- H^H F   F = rows R0.., columns c+1 .. c+B-1 (t > 0: the rest of the bulge)
//   D <- H^H D H D = the diagonal block on rows R0 .. R0+L-1
//   E <- E H     E = rows R0+L .. R0+L+L'-1 (L' = min(B, n-R0-L)), columns of D
// The task's blocks live in the team's window `win` (3 B x (B+1) blocks + 2 B complex):
// D and E are loaded from the band together (one batch of independent loads), E
// stays in the window as the next task's x and F (the block it fills is the next
// task's), and F, x and D go back to the band once they are final.  wait(t) is
// called before task t's loads (false: give up, the sweep returns false) and done(t)
// after its stores.  vout / tauout (or null): task t's v (B complex, zero-padded)
// at vout + t B and tau at tauout[t].  The team is one warp on the device.
template <int B, class TeamT, class WaitF, class DoneF>
LQM_FN bool ts_chase_sweep(const TeamT& T, int n, int s, double2* Bd, double2* vout, double2* tauout,
                           double2* win, WaitF wait, DoneF done) {
  const int ldb = 2 * B;
  constexpr int LW = B + 1;        // window leading dimension (odd: row and column walks conflict-free)
  double2* EF = win;               // x (column 0) and F (columns 1 .. B-1): [r + l LW]
  double2* EN = win + B * LW;      // the next task's block E: [i + q LW]
  double2* D = win + 2 * B * LW;   // the diagonal block, lower triangle: [r + q LW], q <= r
  double2* v = win + 3 * B * LW;
  double2* w = v + B;
  const int nt = ts_tasks(n, B, s);
  for (int t = 0; t < nt; ++t) {
    if (!wait(t)) return false;
    const int R0 = (t == 0) ? s + 1 : s + 1 + t * B;
    const int c = (t == 0) ? s : s + 1 + (t - 1) * B;
    const int L = (n - R0 < B) ? n - R0 : B;
    const int R1 = R0 + L;
    const int L2 = (n - R1 < B) ? n - R1 : B;
    // loads: x (t = 0; later tasks find it in the window), D, E
    if (t == 0)
      for (int r = T.tid; r < L; r += T.nt) EF[r] = ts_bget(Bd, ldb, R0 + r, s);
    for (int idx = T.tid; idx < B * B; idx += T.nt) {
      const int r = idx % B, q = idx / B;
      if (q <= r && r < L) D[r + q * LW] = ts_bget(Bd, ldb, R0 + r, R0 + q);
      if (r < L2 && q < L) EN[r + q * LW] = ts_bget(Bd, ldb, R1 + r, R0 + q);
    }
    team_sync(T);
    // zlarfg on x
    double s2 = 0.0;
    for (int r = 1 + T.tid; r < L; r += T.nt) { const double2 x = EF[r]; s2 += x.x * x.x + x.y * x.y; }
    s2 = warp_sum_bcast(s2);
    const double2 alpha = EF[0];
    double2 tj, scal;
    double beta;
    zlarfg_scalars(alpha, s2, &tj, &beta, &scal);
    for (int r = T.tid; r < B; r += T.nt) {
      double2 vr = cmk(0.0, 0.0);
      if (r == 0) vr = cmk(1.0, 0.0);
      else if (r < L) vr = cmul(scal, EF[r]);
      v[r] = vr;
      if (vout) vout[(int64_t)t * B + r] = vr;
    }
    if (tauout && T.tid == 0) tauout[t] = tj;
    team_sync(T);
    for (int r = T.tid; r < L; r += T.nt) EF[r] = (r == 0) ? cmk(beta, 0.0) : cmk(0.0, 0.0);
    const double2 ctj = cconj(tj);
    // F <- H^H F, column l (1 .. B-1).  Device: lanes l and l + 16 take rows 0..7 and
    // 8..15 of column l, two partial sums each, added across the lane pair.
    if (t > 0) {
#if defined(__CUDACC__)
      const int l = T.lane & 15, hh = T.lane >> 4;
      double2* f = EF + l * LW;
      double2 a0 = cmk(0.0, 0.0), a1 = cmk(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 8; k += 2) {
        const int r0 = 8 * hh + k;
        if (r0 < L) a0 = cfma_conj(a0, v[r0], f[r0]);
        if (r0 + 1 < L) a1 = cfma_conj(a1, v[r0 + 1], f[r0 + 1]);
      }
      const double2 pp = cadd(a0, a1);
      const double2 fl = cmul(ctj, cadd(shfl_c(pp, l), shfl_c(pp, l + 16)));
      if (l >= 1) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int r = 8 * hh + k;
          if (r < L) f[r] = cfms(f[r], v[r], fl);
        }
      }
#else
      for (int l = 1 + T.tid; l < B; l += T.nt) {
        double2* f = EF + l * LW;
        double2 acc = cmk(0.0, 0.0);
        for (int r = 0; r < L; ++r) acc = cadd(acc, cmulc(v[r], f[r]));
        const double2 fl = cmul(ctj, acc);
        for (int r = 0; r < L; ++r) f[r] = csub(f[r], cmul(v[r], fl));
      }
#endif
    }
    team_sync(T);
    // x and F are final: back to the band (columns c .. c+B-1, rows R0 ..)
    const int ncol = (t > 0) ? B : 1;
    for (int idx = T.tid; idx < B * ncol; idx += T.nt) {
      const int r = idx % B, l = idx / B;
      if (r < L) *ts_bptr(Bd, ldb, R0 + r, c + l) = EF[r + l * LW];
    }
    // D <- H^H D H: y = D v, gamma = v^H y, w = tau y - 1/2 |tau|^2 gamma v; then
    // E <- E H: z_i = sum_q E(i, q) v_q, E(i, q) -= tau z_i conj(v_q).  Device: lanes
    // r and r + 16 take columns 0..7 and 8..15 of row r, two partial sums each.
#if defined(__CUDACC__)
    {
      const int r = T.lane & 15, hh = T.lane >> 4;
      double2 a0 = cmk(0.0, 0.0), a1 = cmk(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 8; k += 2) {
        const int q0 = 8 * hh + k, q1 = q0 + 1;
        if (r < L && q0 < L) a0 = cfma(a0, (q0 <= r) ? D[r + q0 * LW] : cconj(D[q0 + r * LW]), v[q0]);
        if (r < L && q1 < L) a1 = cfma(a1, (q1 <= r) ? D[r + q1 * LW] : cconj(D[q1 + r * LW]), v[q1]);
      }
      const double2 pp = cadd(a0, a1);
      const double2 yr = cadd(shfl_c(pp, r), shfl_c(pp, r + 16));
      const double g = warp_sum_bcast((hh == 0 && r < L) ? cmulc(v[r], yr).x : 0.0);
      const double h = -0.5 * (tj.x * tj.x + tj.y * tj.y) * g;
      if (hh == 0 && r < L) w[r] = cadd(cmul(tj, yr), cscale(h, v[r]));
      team_sync(T);  // w complete; every lane has read D
      if (r < L) {
        const double2 vr = v[r], wr = w[r];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int q = 8 * hh + k;
          if (q <= r) {
            double2 a = cfms(cfms(D[r + q * LW], wr, cconj(v[q])), vr, cconj(w[q]));
            if (q == r) a.y = 0.0;
            D[r + q * LW] = a;
          }
        }
      }
      double2 e0 = cmk(0.0, 0.0), e1 = cmk(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 8; k += 2) {
        const int q0 = 8 * hh + k, q1 = q0 + 1;
        if (r < L2 && q0 < L) e0 = cfma(e0, EN[r + q0 * LW], v[q0]);
        if (r < L2 && q1 < L) e1 = cfma(e1, EN[r + q1 * LW], v[q1]);
      }
      const double2 pe = cadd(e0, e1);
      const double2 z = cmul(tj, cadd(shfl_c(pe, r), shfl_c(pe, r + 16)));
      if (r < L2) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int q = 8 * hh + k;
          if (q < L) EN[r + q * LW] = cfms(EN[r + q * LW], z, cconj(v[q]));
        }
      }
    }
#else
    double2 yr = cmk(0.0, 0.0);
    double g = 0.0;
    for (int r = T.tid; r < L; r += T.nt) {
      double2 acc = cmk(0.0, 0.0);
      for (int q = 0; q < L; ++q) acc = cadd(acc, cmul((q <= r) ? D[r + q * LW] : cconj(D[q + r * LW]), v[q]));
      yr = acc;
      g += cmulc(v[r], acc).x;
#if !defined(__CUDACC__)
      w[r] = acc;  // one-thread team: y kept in w until gamma is complete
#endif
    }
    g = warp_sum_bcast(g);
    const double h = -0.5 * (tj.x * tj.x + tj.y * tj.y) * g;
#if defined(__CUDACC__)
    for (int r = T.tid; r < L; r += T.nt) w[r] = cadd(cmul(tj, yr), cscale(h, v[r]));
#else
    for (int r = 0; r < L; ++r) w[r] = cadd(cmul(tj, w[r]), cscale(h, v[r]));
#endif
    team_sync(T);  // every thread has read D before it is rewritten
    for (int r = T.tid; r < L; r += T.nt) {
      const double2 vr = v[r], wr = w[r];
      for (int q = 0; q <= r; ++q) {
        double2 a = csub(D[r + q * LW], cadd(cmul(wr, cconj(v[q])), cmul(vr, cconj(w[q]))));
        if (q == r) a.y = 0.0;
        D[r + q * LW] = a;
      }
    }
    // E <- E H: row i by thread, z_i = sum_q E(i, q) v_q, E(i, q) -= tau z_i conj(v_q)
    for (int i = T.tid; i < L2; i += T.nt) {
      double2 acc = cmk(0.0, 0.0);
      for (int q = 0; q < L; ++q) acc = cadd(acc, cmul(EN[i + q * LW], v[q]));
      const double2 z = cmul(tj, acc);
      for (int q = 0; q < L; ++q) EN[i + q * LW] = csub(EN[i + q * LW], cmul(z, cconj(v[q])));
    }
#endif
    team_sync(T);
    for (int idx = T.tid; idx < B * B; idx += T.nt) {
      const int r = idx % B, q = idx / B;
      if (q <= r && r < L) *ts_bptr(Bd, ldb, R0 + r, R0 + q) = D[r + q * LW];
    }
    // E becomes the next task's x and F
    double2* tmp = EF;
    EF = EN;
    EN = tmp;
    done(t);
  }
  return true;
}

// Applies H = I - tau v v^H of every stage-2 task to the rows of Z (n x nc, leading
// dimension ldz), in the reverse order of the chase (Z <- Q2 Z): the defining order,
// against which the emulation checks the grouped order of the device kernel.
// V2: reflectors of sweep s, task t at V2 + (s * tmax + t) * B; tau2 at s * tmax + t.
template <int B>
LQM_FN void ts_q2_apply_host(int n, const double2* V2, const double2* tau2, double2* Z, int ldz, int nc) {
  const int tmax = ts_tmax(n, B);
  for (int s = n - 2; s >= 0; --s) {
    const int nt = ts_tasks(n, B, s);
    for (int t = 0; t < nt; ++t) {
      const int R0 = (t == 0) ? s + 1 : s + 1 + t * B;
      const int L = (n - R0 < B) ? n - R0 : B;
      const double2* v = V2 + ((int64_t)s * tmax + t) * B;
      const double2 tj = tau2[(int64_t)s * tmax + t];
      for (int c = 0; c < nc; ++c) {
        double2* z = Z + (int64_t)c * ldz + R0;
        double2 acc = cmk(0.0, 0.0);
        for (int r = 0; r < L; ++r) acc = cadd(acc, cmulc(v[r], z[r]));
        const double2 f = cmul(tj, acc);
        for (int r = 0; r < L; ++r) z[r] = csub(z[r], cmul(v[r], f));
      }
    }
  }
}

// Q2 Z in the grouped order of the device kernel (ts_q2g_kernel): the sweeps in
// groups of B, the highest group first; within a group the task index t ascending,
// and for each t the group's reflectors of task t from the highest sweep down.  Two
// reflectors overlap only when they are of the same t, or of tasks t and t - 1 of
// sweeps less than 2B apart; this order applies every later-generated overlapping
// reflector first, as the reverse sweep order does, so the product is the same.  The
// reflectors of one (group, t) step act on a window of 2B - 1 rows that slides by B
// rows per step.
template <int B>
LQM_FN void ts_q2_apply_grouped_host(int n, const double2* V2, const double2* tau2, double2* Z, int ldz, int nc) {
  const int tmax = ts_tmax(n, B);
  const int ns = n - 1;  // sweeps 0 .. n-2
  if (ns <= 0) return;
  for (int s0 = ((ns - 1) / B) * B; s0 >= 0; s0 -= B) {
    const int nt = ts_tasks(n, B, s0);
    for (int t = 0; t < nt; ++t)
      for (int i = B - 1; i >= 0; --i) {
        const int s = s0 + i;
        if (s >= ns || t >= ts_tasks(n, B, s)) continue;
        const int R0 = s + 1 + t * B;
        const int L = (n - R0 < B) ? n - R0 : B;
        const double2* v = V2 + ((int64_t)s * tmax + t) * B;
        const double2 tj = tau2[(int64_t)s * tmax + t];
        for (int c = 0; c < nc; ++c) {
          double2* z = Z + (int64_t)c * ldz + R0;
          double2 acc = cmk(0.0, 0.0);
          for (int r = 0; r < L; ++r) acc = cadd(acc, cmulc(v[r], z[r]));
          const double2 f = cmul(tj, acc);
          for (int r = 0; r < L; ++r) z[r] = csub(z[r], cmul(v[r], f));
        }
      }
  }
}
