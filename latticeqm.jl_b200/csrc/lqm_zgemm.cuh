// Batched complex FP64 GEMM on the FP64 tensor path (DMMA, mma.sync m8n8k4 f64),
// the library's own replacement for a BLAS ZGEMM on every batched product of the
// eigen passes (blocked trailing updates, compact-WY back-transformation,
// rho_k = (U f) U^H, the Fourier fold, the adjoint and observable products):
//
//   C_b = alpha op(A_b) op(B_b) + beta C_b,  b < batch,  column-major, strided,
//   op in {N, T (transpose), C (conjugate transpose)}, alpha and beta real.
//
// A CTA computes a BM x BN tile of one batch entry, K in slices of BK staged in
// shared memory by an ST-deep cp.async ring (16-byte complex elements, zero fill past
// the matrix edges).  Both tiles are stored k-contiguous per row / column with a row
// pitch of BK + 4 elements, so the fragment reads of a quarter-warp fall on distinct
// 16-byte bank groups.  Each warp owns a WM x WN sub-tile: per 4-deep k-step it reads
// one complex A element per 8-row strip and one complex B element per 8-column strip
// and issues four real DMMAs per 8 x 8 output tile:
//   Cre += Are Bre - Aim Bim,  Cim += Are Bim + Aim Bre.
// The k-sum order is fixed, so results are deterministic.
//
// Fragment layout of mma.m8n8k4.f64 (PTX ISA): with g = lane / 4, t = lane % 4,
// A (8 x 4, row) holds A[g][t], B (4 x 8, col) holds B[t][g], C/D (8 x 8) holds
// C[g][2t] and C[g][2t + 1].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lqm_team.cuh"

namespace lqm {

// OP_HL (first operand only, no split and no second pair): the operand is a
// Hermitian matrix of which only the lower triangle is stored; element (r, k) is
// A(r, k) for r >= k and conj(A(k, r)) above, with the diagonal taken as real.
enum GemmOp { OP_N = 0, OP_T = 1, OP_C = 2, OP_HL = 3 };

// complex elements per staged row: BK + 4 (== 4 mod 8: conflict-free fragment reads)
__host__ __device__ constexpr int gemm_pitch(int BK) { return BK + 4; }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) { dmma_884(d0, d1, a, b); }

__device__ __forceinline__ void gemm_cp16(void* sdst, const void* gsrc, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  const int nbytes = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(nbytes) : "memory");
}

struct GemmArgs {
  int m, n, k;
  double alpha, beta;
  const double2* A;
  int lda;
  long long sA;
  const double2* B;
  int ldb;
  long long sB;
  double2* C;
  int ldc;
  long long sC;
  int opA, opB;
  // split-K: split > 0 chunks per batch entry; blockIdx.z = entry * split + chunk,
  // chunk covers [chunk k, chunk k + k) of ktot and writes its own C_z = C + z sC
  // with beta = 0; 0 = plain batched product
  int split, ktot;
  // optional second operand pair summed after the first (k2 > 0, same ops):
  //   C = alpha (op(A) op(B) + op(A2) op(B2)) + beta C,  the k-sum of A2 B2 after A B
  const double2* A2;
  int lda2;
  long long sA2;
  const double2* B2;
  int ldb2;
  long long sB2;
  int k2;
  // lower != 0: C starts on a diagonal of a Hermitian block; tiles entirely above
  // it (every row < every column) are skipped
  int lower;
};

// Stage one K-slice [k0, k0 + 8) of op(A) (BM rows) and op(B) (BN columns) into
// As[row][kk], Bs[col][kk].  op N of A / op T,C of B are contiguous along the
// row / column index, the other ops along k; threads follow the contiguous index.
template <int BM, int BN, int NT, int BK>
__device__ __forceinline__ void gemm_stage(const GemmArgs& g, const double2* A, int lda, const double2* B, int ldb,
                                           int m0, int n0, int k0, int kend, double2* As, double2* Bs) {
  constexpr int P = gemm_pitch(BK);
#pragma unroll
  for (int e = threadIdx.x; e < BM * BK; e += NT) {
    int r, kk;
    if (g.opA == OP_N || g.opA == OP_HL) { r = e % BM; kk = e / BM; } else { kk = e % BK; r = e / BK; }
    const int gm = m0 + r, gk = k0 + kk;
    const bool ok = gm < g.m && gk < kend;
    const bool lower = g.opA == OP_N || (g.opA == OP_HL && gm >= gk);
    const double2* src = lower ? A + gm + (int64_t)gk * lda : A + gk + (int64_t)gm * lda;
    gemm_cp16(As + r * P + kk, ok ? (const void*)src : (const void*)A, ok);
  }
#pragma unroll
  for (int e = threadIdx.x; e < BN * BK; e += NT) {
    int c, kk;
    if (g.opB == OP_N) { kk = e % BK; c = e / BK; } else { c = e % BN; kk = e / BN; }
    const int gn = n0 + c, gk = k0 + kk;
    const bool ok = gn < g.n && gk < kend;
    const double2* src = (g.opB == OP_N) ? B + gk + (int64_t)gn * ldb : B + gn + (int64_t)gk * ldb;
    gemm_cp16(Bs + c * P + kk, ok ? (const void*)src : (const void*)B, ok);
  }
}

// grid (ceil(m / BM), ceil(n / BN), batch); block (BM / WM) * (BN / WN) warps; K in
// slices of BK through an ST-deep ring.
template <int BM, int BN, int WM, int WN, int BK, int ST>
// eight-warp tiles keep two CTAs per SM (at most 128 registers per thread)
__global__ void __launch_bounds__((BM / WM) * (BN / WN) * 32, (BM / WM) * (BN / WN) >= 8 ? 2 : 1)
    zgemm_dmma_kernel(GemmArgs g) {
  constexpr int NT = (BM / WM) * (BN / WN) * 32;
  constexpr int MI = WM / 8, NJ = WN / 8;
  constexpr int P = gemm_pitch(BK);
  constexpr int STAGE = (BM + BN) * P;  // complex per stage
  extern __shared__ __align__(16) unsigned char gemm_smem[];
  double2* sm = (double2*)gemm_smem;
  const int64_t b = blockIdx.z;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  if (g.lower && m0 + BM <= n0) return;  // above the diagonal (uniform per block)
  const double2* A = g.A;
  const double2* B = g.B;
  const double2* A2 = g.A2 + b * g.sA2;
  const double2* B2 = g.B2 + b * g.sB2;
  double2* C = g.C + b * g.sC;
  int kend = g.k;  // k bound of this block's slice, relative to A and B
  if (g.split) {
    const int64_t e = b / g.split;                    // batch entry
    const int64_t kb = (b - e * g.split) * (int64_t)g.k;  // first k of the chunk
    A += e * g.sA + ((g.opA == OP_N) ? kb * g.lda : kb);
    B += e * g.sB + ((g.opB == OP_N) ? kb : kb * g.ldb);
    kend = (int)(g.ktot - kb < g.k ? g.ktot - kb : g.k);
  } else {
    A += b * g.sA;
    B += b * g.sB;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm0 = (warp % (BM / WM)) * WM, wn0 = (warp / (BM / WM)) * WN;
  const int gr = lane >> 2, gt = lane & 3;
  const double sa = (g.opA == OP_C) ? -1.0 : 1.0;  // conjugation of op(A) / op(B)
  const double sb = (g.opB == OP_C) ? -1.0 : 1.0;

  double re[MI][NJ][2], im[MI][NJ][2];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j) re[i][j][0] = re[i][j][1] = im[i][j][0] = im[i][j][1] = 0.0;

  // slices [0, nks1) from (A, B), then [nks1, nks) from (A2, B2)
  const int nks1 = (kend + BK - 1) / BK;
  const int nks = nks1 + (g.k2 > 0 ? (g.k2 + BK - 1) / BK : 0);
  auto stage = [&](int s, double2* dst) {
    if (s < nks1)
      gemm_stage<BM, BN, NT, BK>(g, A, g.lda, B, g.ldb, m0, n0, s * BK, kend, dst, dst + BM * P);
    else
      gemm_stage<BM, BN, NT, BK>(g, A2, g.lda2, B2, g.ldb2, m0, n0, (s - nks1) * BK, g.k2, dst, dst + BM * P);
  };
#pragma unroll
  for (int s = 0; s < ST - 1; ++s) {
    if (s < nks) stage(s, sm + s * STAGE);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  // beta != 0: the accumulators start at (beta / alpha) C, loaded while the first
  // slices are in flight (the epilogue then writes alpha acc without reading C)
  const bool cinit = g.beta != 0.0 && g.alpha != 0.0;
  if (cinit) {
    const double sc = g.beta / g.alpha;
#pragma unroll
    for (int i = 0; i < MI; ++i) {
      const int r = m0 + wm0 + 8 * i + gr;
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int c = n0 + wn0 + 8 * j + 2 * gt + h;
          if (r < g.m && c < g.n) {
            const double2 o = C[r + (int64_t)c * g.ldc];
            re[i][j][h] = sc * o.x;
            im[i][j][h] = sc * o.y;
          }
        }
    }
  }
  for (int ks = 0; ks < nks; ++ks) {
    if (ST > 1) {
      asm volatile("cp.async.wait_group %0;\n" ::"n"(ST > 1 ? ST - 2 : 0) : "memory");
      __syncthreads();
      const int nx = ks + ST - 1;
      const int st = nx % ST;
      if (nx < nks) stage(nx, sm + st * STAGE);
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    } else {  // one buffer: load, wait, compute, and fence the buffer before the next load
      __syncthreads();
      stage(ks, sm);
      asm volatile("cp.async.commit_group;\n" ::: "memory");
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
      __syncthreads();
    }
    const double2* As = sm + (ks % ST) * STAGE;
    const double2* Bs = As + BM * P;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double ar[MI], ai[MI], br[NJ], bi[NJ];
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const double2 a = As[(wm0 + 8 * i + gr) * P + kk + gt];
        ar[i] = a.x;
        ai[i] = sa * a.y;
      }
      if (g.opA == OP_HL) {  // entries above the diagonal were staged from their mirror
        const int kg = ks * BK + kk + gt;
#pragma unroll
        for (int i = 0; i < MI; ++i) {
          const int rg = m0 + wm0 + 8 * i + gr;
          ai[i] = (rg > kg) ? ai[i] : (rg < kg) ? -ai[i] : 0.0;
        }
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const double2 v = Bs[(wn0 + 8 * j + gr) * P + kk + gt];
        br[j] = v.x;
        bi[j] = sb * v.y;
      }
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const double nai = -ai[i];
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          dmma(re[i][j][0], re[i][j][1], ar[i], br[j]);
          dmma(re[i][j][0], re[i][j][1], nai, bi[j]);
          dmma(im[i][j][0], im[i][j][1], ar[i], bi[j]);
          dmma(im[i][j][0], im[i][j][1], ai[i], br[j]);
        }
      }
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  // epilogue: C = alpha acc (+ beta C when C was not folded into acc)
#pragma unroll
  for (int i = 0; i < MI; ++i) {
    const int r = m0 + wm0 + 8 * i + gr;
    if (r >= g.m) continue;
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = n0 + wn0 + 8 * j + 2 * gt + h;
        if (c >= g.n) continue;
        double2* p = C + r + (int64_t)c * g.ldc;
        double2 v = cmk(g.alpha * re[i][j][h], g.alpha * im[i][j][h]);
        if (!cinit && g.beta != 0.0) {
          const double2 o = *p;
          v.x += g.beta * o.x;
          v.y += g.beta * o.y;
        }
        *p = v;
      }
    }
  }
}

// Split-K finish: C_e = sum_z P_(e, z) + beta C_e in chunk order (P_(e, z) = C_z of
// entry e's chunks, m x n each, leading dimension m), for every batch entry e.
__global__ void __launch_bounds__(256) zgemm_split_reduce_kernel(int m, int n, int nsplit, const double2* P,
                                                                 double beta, double2* C, int ldc, long long sC,
                                                                 int batch) {
  const int64_t mn = (int64_t)m * n;
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < mn * batch;
       u += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = u / mn, t = u - e * mn;
    const double2* Pe = P + e * nsplit * mn;
    double2 acc = Pe[t];
    for (int z = 1; z < nsplit; ++z) acc = cadd(acc, Pe[z * mn + t]);
    const int64_t i = t % m, j = t / m;
    double2* c = C + e * sC + i + j * (int64_t)ldc;
    if (beta != 0.0) {
      const double2 o = *c;
      acc.x += beta * o.x;
      acc.y += beta * o.y;
    }
    *c = acc;
  }
}

template <int BM, int BN, int BK, int ST>
constexpr int zgemm_smem_bytes() {
  return ST * (BM + BN) * gemm_pitch(BK) * 16;
}

}  // namespace lqm
