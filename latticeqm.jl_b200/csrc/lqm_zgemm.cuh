// Batched complex FP64 GEMM on the FP64 tensor path (DMMA, mma.sync m8n8k4 f64),
// the library's own replacement for a BLAS ZGEMM on every batched product of the
// eigen passes (blocked trailing updates, compact-WY back-transformation,
// rho_k = (U f) U^H, the Fourier fold, the adjoint and observable products):
//
//   C_b = alpha op(A_b) op(B_b) + beta C_b,  b < batch,  column-major, strided,
//   op in {N, T (transpose), C (conjugate transpose)}, alpha and beta real.
//
// A CTA computes a BM x BN tile of one batch entry, K in steps of 8 staged in
// shared memory by a 3-deep cp.async ring (16-byte complex elements, zero fill past
// the matrix edges).  Both tiles are stored k-contiguous per row / column with a row
// pitch of 12 elements, so the fragment reads of a quarter-warp fall on distinct
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

enum GemmOp { OP_N = 0, OP_T = 1, OP_C = 2 };

constexpr int kGemmBK = 8;       // k per stage
constexpr int kGemmPitch = 12;   // complex elements per staged row (8 + 4: conflict-free fragment reads)
constexpr int kGemmStages = 3;

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

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
};

// Stage one K-slice [k0, k0 + 8) of op(A) (BM rows) and op(B) (BN columns) into
// As[row][kk], Bs[col][kk].  op N of A / op T,C of B are contiguous along the
// row / column index, the other ops along k; threads follow the contiguous index.
template <int BM, int BN, int NT>
__device__ __forceinline__ void gemm_stage(const GemmArgs& g, const double2* A, const double2* B, int m0, int n0,
                                           int k0, double2* As, double2* Bs) {
#pragma unroll
  for (int e = threadIdx.x; e < BM * kGemmBK; e += NT) {
    int r, kk;
    if (g.opA == OP_N) { r = e % BM; kk = e / BM; } else { kk = e % kGemmBK; r = e / kGemmBK; }
    const int gm = m0 + r, gk = k0 + kk;
    const bool ok = gm < g.m && gk < g.k;
    const double2* src = (g.opA == OP_N) ? A + gm + (int64_t)gk * g.lda : A + gk + (int64_t)gm * g.lda;
    gemm_cp16(As + r * kGemmPitch + kk, ok ? (const void*)src : (const void*)A, ok);
  }
#pragma unroll
  for (int e = threadIdx.x; e < BN * kGemmBK; e += NT) {
    int c, kk;
    if (g.opB == OP_N) { kk = e % kGemmBK; c = e / kGemmBK; } else { c = e % BN; kk = e / BN; }
    const int gn = n0 + c, gk = k0 + kk;
    const bool ok = gn < g.n && gk < g.k;
    const double2* src = (g.opB == OP_N) ? B + gk + (int64_t)gn * g.ldb : B + gn + (int64_t)gk * g.ldb;
    gemm_cp16(Bs + c * kGemmPitch + kk, ok ? (const void*)src : (const void*)B, ok);
  }
}

// grid (ceil(m / BM), ceil(n / BN), batch); block (BM / WM) * (BN / WN) warps.
template <int BM, int BN, int WM, int WN>
__global__ void __launch_bounds__((BM / WM) * (BN / WN) * 32) zgemm_dmma_kernel(GemmArgs g) {
  constexpr int NT = (BM / WM) * (BN / WN) * 32;
  constexpr int MI = WM / 8, NJ = WN / 8;
  constexpr int STAGE = (BM + BN) * kGemmPitch;  // complex per stage
  extern __shared__ __align__(16) unsigned char gemm_smem[];
  double2* sm = (double2*)gemm_smem;
  const int64_t b = blockIdx.z;
  const double2* A = g.A + b * g.sA;
  const double2* B = g.B + b * g.sB;
  double2* C = g.C + b * g.sC;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
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

  const int nks = (g.k + kGemmBK - 1) / kGemmBK;
#pragma unroll
  for (int s = 0; s < kGemmStages - 1; ++s) {
    if (s < nks) gemm_stage<BM, BN, NT>(g, A, B, m0, n0, s * kGemmBK, sm + s * STAGE, sm + s * STAGE + BM * kGemmPitch);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int ks = 0; ks < nks; ++ks) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kGemmStages - 2) : "memory");
    __syncthreads();
    {
      const int nx = ks + kGemmStages - 1;
      const int st = nx % kGemmStages;
      if (nx < nks)
        gemm_stage<BM, BN, NT>(g, A, B, m0, n0, nx * kGemmBK, sm + st * STAGE, sm + st * STAGE + BM * kGemmPitch);
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    const double2* As = sm + (ks % kGemmStages) * STAGE;
    const double2* Bs = As + BM * kGemmPitch;
#pragma unroll
    for (int kk = 0; kk < kGemmBK; kk += 4) {
      double ar[MI], ai[MI], br[NJ], bi[NJ];
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const double2 a = As[(wm0 + 8 * i + gr) * kGemmPitch + kk + gt];
        ar[i] = a.x;
        ai[i] = sa * a.y;
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const double2 v = Bs[(wn0 + 8 * j + gr) * kGemmPitch + kk + gt];
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
  // epilogue: C = alpha acc + beta C
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
        if (g.beta != 0.0) {
          const double2 o = *p;
          v.x += g.beta * o.x;
          v.y += g.beta * o.y;
        }
        *p = v;
      }
    }
  }
}

template <int BM, int BN, int WM, int WN>
constexpr int zgemm_smem_bytes() {
  return kGemmStages * (BM + BN) * kGemmPitch * 16;
}

}  // namespace lqm
