// Batched blocked eigensolver kernels for orders beyond the one-CTA shared-
// memory plan (n up to a few thousand).  A batch of B k-points is reduced
// together, one launch per column step:
//
//   blk_bloch_kernel    H(k) (full Hermitian, from the upper triangle), CTA per k
//   blk_column_kernel   zlatrd column step (lqm_blocked.cuh), CTA per k
//   blk_symv_kernel     y = A22 v from the lower triangle, 64 x 64 tiles x k,
//                       plus row slabs of the panel products t1, t2; ordered
//                       partials (summed by the next column step)
//   blk_finish_kernel   last w of a panel, CTA per k
//   (host)              rank-2nb trailing update, batched ZGEMM
//   dc_large_kernel     divide and conquer per k (vectors in global memory,
//                       tiled merge updates), writes bands and Z (complex)
//   blk_prep_kernel / blk_larft_kernel   compact WY factors per panel
//   (host)              U = (I - V T V^H) U per panel, batched ZGEMMs
//   blk_scale_f_kernel  Y = U diag(f), band energy; (host) rho_k = Y U^H
#pragma once
#include <cuda.h>

#include "lqm_blocked.cuh"
#include "lqm_kernels.cuh"
#include "lqm_twostage.cuh"

namespace lqm {

constexpr int kBlkNB = 32;      // panel width of the reduction (reflectors per panel)
constexpr int kBlkNBT = 64;     // panel width of the compact-WY back-transformation
constexpr int kBlkThreads = 256;
constexpr int kColThreads = 512;  // column step: latency-bound row passes, more rows in flight per k-point
constexpr int kSymvTB = 64;     // mat-vec tile (2 rows per lane of a 32-lane warp)
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
  double2* part; // B x part_stride: mat-vec tile partials
  int64_t part_stride;
  double2* tpart;  // B x tpart_stride: panel-product slab partials
  int64_t tpart_stride;
};

// complex per k-point for the panel-product partials: slabs of 128 rows x 2nb
__host__ __device__ inline int64_t t12_part_stride(int n, int nb) {
  const int64_t nsl = (n - 1 + 127) / 128;
  return (nsl < 1 ? 1 : nsl) * 2 * nb;
}

// complex per k-point for the mat-vec partials: nblk^2 tiles of kSymvTB
__host__ __device__ inline int64_t symv_part_stride(int n) {
  const int64_t nbk = (n - 1 + kSymvTB - 1) / kSymvTB;
  return (nbk < 1 ? 1 : nbk * nbk) * kSymvTB;
}

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

__global__ void __launch_bounds__(kColThreads) blk_column_kernel(BlkArgs a, int j0, int i) {
  __shared__ double red[128];
  __shared__ __align__(16) double2 t12[2 * kBlkNB];
  const Team T = make_team();
  const int64_t b = blockIdx.x;
  const int n = a.n;
  blk_column(T, n, a.nb, j0, i, a.A + b * (int64_t)n * n, n, a.W + b * (int64_t)n * a.nb, n, a.tau + b * n,
             a.d + b * n, a.e + b * n, t12, red, a.part + b * a.part_stride, a.tpart + b * a.tpart_stride);
}

// Last column of a panel: finish its w from the partials.
__global__ void __launch_bounds__(kColThreads) blk_finish_kernel(BlkArgs a, int j0, int ip) {
  __shared__ double red[128];
  __shared__ __align__(16) double2 t12[2 * kBlkNB];
  const Team T = make_team();
  const int64_t b = blockIdx.x;
  const int n = a.n;
  blk_prev_w(T, n, a.nb, j0, ip, a.A + b * (int64_t)n * n, n, a.W + b * (int64_t)n * a.nb, n, a.tau + b * n, t12,
             red, a.part + b * a.part_stride, a.tpart + b * a.tpart_stride, nullptr);
}

// grid (nslabs, B): row slabs of the panel products of column j = j0 + i.
__global__ void __launch_bounds__(kBlkThreads) blk_t12_kernel(BlkArgs a, int j0, int i) {
  const Team T = make_team();
  const int64_t b = blockIdx.y;
  blk_t12_slab(T, a.n, a.nb, j0, i, blockIdx.x, a.A + b * (int64_t)a.n * a.n, a.n, a.W + b * (int64_t)a.n * a.nb, a.n,
               a.tpart + b * a.tpart_stride);
}

// ---- Hermitian mat-vec of one column, persistent and pipelined ----
// The same arithmetic and partial layout as blk_symv_tile (64 x 64 lower
// tiles, direct + transposed partials), but each CTA walks a list of tiles
// (all k-points of the batch) with a kSymvStages-deep cp.async pipeline, so
// that two tiles are in flight from HBM while a third is summed.
constexpr int kSymvStages = 3;
constexpr int kSymvThreads = 512;
constexpr int kSymvLd = kSymvTB + 1;
constexpr int kSymvStageC = kSymvTB * kSymvLd + 2 * kSymvTB;  // complex per stage: tile + v_R, v_C
constexpr int kSymvPipeSmem = (kSymvStages * kSymvStageC + 2 * (kSymvThreads / kSymvTB) * kSymvTB) * 16;
static_assert(kSymvPipeSmem <= 227 * 1024, "mat-vec pipeline exceeds shared memory");

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  const int nbytes = valid ? 16 : 0;  // 0: the 16 bytes are zero-filled, nothing is read
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(nbytes) : "memory");
}
// a hint: the 128-byte line holding *p into L1 (and L2), no register written; callers
// pass only addresses inside their own buffers
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.L1 [%0];\n" ::"l"(p)); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_keep1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// tile t of the lower block triangle -> (R, C), R >= C, row-major
__device__ __forceinline__ void symv_tile_rc(int t, int* R, int* C) {
  int r = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((r + 1) * (r + 2) / 2 <= t) ++r;
  while (r * (r + 1) / 2 > t) --r;
  *R = r;
  *C = t - r * (r + 1) / 2;
}

// Issue the copies of work item `it` (k-point it / ntiles, tile it % ntiles)
// into stage buffer `st`; rows/columns beyond m are zero-filled.
__device__ __forceinline__ void symv_issue(const BlkArgs& a, int j, int m, int ntiles, int64_t it, double2* st) {
  const int64_t b = it / ntiles;
  int R, C;
  symv_tile_rc((int)(it - b * ntiles), &R, &C);
  const double2* A = a.A + b * (int64_t)a.n * a.n;
  const double2* B = A + (j + 1) + (int64_t)(j + 1) * a.n;
  const double2* v = A + (j + 1) + (int64_t)j * a.n;
  const int x0 = R * kSymvTB, y0 = C * kSymvTB;
#pragma unroll
  for (int h = 0; h < (kSymvTB * kSymvTB) / kSymvThreads; ++h) {
    const int idx = threadIdx.x + h * kSymvThreads, rr = idx % kSymvTB, cc = idx / kSymvTB;
    const int x = x0 + rr, y = y0 + cc;
    const bool ok = x < m && y < m;
    cp_async16(st + rr + cc * kSymvLd, ok ? (const void*)(B + x + (int64_t)y * a.n) : (const void*)B, ok);
  }
  if (threadIdx.x < 2 * kSymvTB) {
    const int t = threadIdx.x;
    const int x = (t < kSymvTB) ? x0 + t : y0 + (t - kSymvTB);
    cp_async16(st + kSymvTB * kSymvLd + t, x < m ? (const void*)(v + x) : (const void*)v, x < m);
  }
}

// grid: persistent (about one CTA per SM), kSymvPipeSmem dynamic smem.
__global__ void __launch_bounds__(kSymvThreads, 1) blk_symv_pipe_kernel(BlkArgs a, int j, int64_t nitems) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* stg = (double2*)smem;
  double2* rd = stg + kSymvStages * kSymvStageC;           // [ng][TB] direct
  constexpr int ng = kSymvThreads / kSymvTB;
  double2* rt = rd + ng * kSymvTB;                         // [ng][TB] transposed
  const int m = a.n - j - 1;
  const int nbk = (m + kSymvTB - 1) / kSymvTB;
  const int ntiles = nbk * (nbk + 1) / 2;
  const int64_t first = blockIdx.x, step = gridDim.x;
  // prologue: stages 0 .. kSymvStages-2
#pragma unroll
  for (int s = 0; s < kSymvStages - 1; ++s) {
    const int64_t it = first + s * step;
    if (it < nitems) symv_issue(a, j, m, ntiles, it, stg + s * kSymvStageC);
    cp_async_commit();
  }
  int stage = 0;
  for (int64_t it = first; it < nitems; it += step) {
    cp_async_wait_keep1();  // the group of item `it` has landed (kSymvStages == 3)
    __syncthreads();
    {
      const int64_t nx = it + (kSymvStages - 1) * step;
      const int ns = (stage + kSymvStages - 1) % kSymvStages;
      if (nx < nitems) symv_issue(a, j, m, ntiles, nx, stg + ns * kSymvStageC);
      cp_async_commit();
    }
    const double2* ts = stg + stage * kSymvStageC;
    const double2* vR = ts + kSymvTB * kSymvLd;
    const double2* vC = vR + kSymvTB;
    const int64_t b = it / ntiles;
    int R, C;
    symv_tile_rc((int)(it - b * ntiles), &R, &C);
    const bool diag = (R == C);
    {
      // thread (q, g): direct product of row q and transposed product of column q
      // over u = g, g + ng, ... (two interleaved accumulators each)
      const int q = threadIdx.x % kSymvTB, g = threadIdx.x / kSymvTB;
      double2 ad0 = cmk(0.0, 0.0), ad1 = ad0, at0 = ad0, at1 = ad0;
      if (!diag) {
#pragma unroll
        for (int h = 0; h < kSymvTB / ng; h += 2) {
          const int u0 = g + h * ng, u1 = u0 + ng;
          ad0 = cadd(ad0, cmul(ts[q + u0 * kSymvLd], vC[u0]));
          at0 = cadd(at0, cmulc(ts[u0 + q * kSymvLd], vR[u0]));
          ad1 = cadd(ad1, cmul(ts[q + u1 * kSymvLd], vC[u1]));
          at1 = cadd(at1, cmulc(ts[u1 + q * kSymvLd], vR[u1]));
        }
      } else {
        // lower part only: direct uses columns u <= q (diagonal real), transposed rows u > q
#pragma unroll
        for (int h = 0; h < kSymvTB / ng; ++h) {
          const int u = g + h * ng;
          double2 x = ts[q + u * kSymvLd];
          if (u > q) x = cmk(0.0, 0.0);
          else if (u == q) x.y = 0.0;
          double2 y = ts[u + q * kSymvLd];
          if (u <= q) y = cmk(0.0, 0.0);
          if (h & 1) {
            ad1 = cadd(ad1, cmul(x, vC[u]));
            at1 = cadd(at1, cmulc(y, vR[u]));
          } else {
            ad0 = cadd(ad0, cmul(x, vC[u]));
            at0 = cadd(at0, cmulc(y, vR[u]));
          }
        }
      }
      rd[threadIdx.x] = cadd(ad0, ad1);
      rt[threadIdx.x] = cadd(at0, at1);
    }
    __syncthreads();
    if (threadIdx.x < kSymvTB) {
      const int x = threadIdx.x;
      double2 yd = cmk(0.0, 0.0), yt = cmk(0.0, 0.0);
#pragma unroll
      for (int g = 0; g < ng; ++g) {
        yd = cadd(yd, rd[g * kSymvTB + x]);
        yt = cadd(yt, rt[g * kSymvTB + x]);
      }
      double2* part = a.part + b * a.part_stride;
      if (diag) {
        part[((int64_t)R * nbk + C) * kSymvTB + x] = cadd(yd, yt);
      } else {
        part[((int64_t)R * nbk + C) * kSymvTB + x] = yd;
        part[((int64_t)C * nbk + R) * kSymvTB + x] = yt;
      }
    }
    stage = (stage + 1) % kSymvStages;
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// ---- Hermitian mat-vec of one column, tiles moved by TMA ----
// The same partial layout as blk_symv_pipe_kernel, with each 64 x 64 lower tile
// brought into shared memory by eight 3-D tensor copies (cp.async.bulk.tensor:
// box = 8 complex rows x 64 columns x 1 k-point, 128-byte swizzle) that complete
// on one mbarrier per stage, issued by one thread; rows and columns beyond the
// matrix read as zeros (out-of-bounds fill), so the tensor map covers the whole
// batch for every column.
// Each tile element is read from shared memory once and used for both products:
// warp w owns the 16 x 16 sub-block (rows 16 (w % 4) .., columns 16 (w / 4) ..);
// lane (a = lane % 8, b = lane / 8) holds rows a, a + 8 and columns b + 4 i
// (i < 4) of it (with the swizzle, the eight lanes of each load phase hit eight
// distinct 16-byte bank groups).  The direct partials (row sums over the lane's
// columns) are reduced over b and the transposed ones (column sums over its rows)
// over a, by reduce-scatter shuffles (each step halves what a lane keeps), then
// written to a double-buffered slot per warp; after the next tile's barrier the
// four column- (row-) blocks of each row (column) are added in order and written
// out.  So there is one block barrier per tile.  Every mbarrier wait is bounded;
// on expiry the kernel sets *err and stops (the host reports LQM_EDEVICE).
constexpr int kSymvTmaThreads = 512;
constexpr int kSymvTmaStages = 3;
constexpr int kSymvTileBytes = kSymvTB * kSymvTB * 16;  // 64 KB
constexpr int kSymvVecBytes = 2 * kSymvTB * 16;               // v over the tile's rows, then over its columns
constexpr int kSymvRedBytes = 2 * 2 * 4 * kSymvTB * 16;  // [buffer][direct, transposed][block][64] complex
constexpr int kSymvTmaSmem = kSymvTmaStages * (kSymvTileBytes + kSymvVecBytes) + kSymvRedBytes +
                             1024 /* alignment */ + 64 /* mbarriers */;
static_assert(kSymvTmaSmem <= 227 * 1024, "TMA mat-vec pipeline exceeds shared memory");
constexpr long long kSymvWaitLimit = 1LL << 22;  // mbarrier polls before giving up (well under a second)

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
// bounded wait: false when the limit ran out
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity) {
  for (long long i = 0; i < kSymvWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(dst),
      "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

// byte offset of element (row r, column c) of a staged tile (eight swizzled boxes)
__device__ __forceinline__ int symv_sw(int r, int c) {
  return ((r >> 3) << 13) + (c << 7) + ((((r & 7) ^ (c & 7))) << 4);
}

// The tile of work item `it` (eight boxes) and the two 64-element segments of the
// reflector v = A(j+1:, j) it multiplies (rows of the tile's row block and of its
// column block; one box each from the vector map), all on the stage's mbarrier.
__device__ __forceinline__ void symv_tma_issue(const CUtensorMap* map, const CUtensorMap* vmap, int j, int ntiles,
                                               int64_t it, unsigned dst, unsigned vdst, unsigned bar) {
  const int64_t b = it / ntiles;
  int R, C;
  symv_tile_rc((int)(it - b * ntiles), &R, &C);
  mbar_arrive_expect_tx(bar, (unsigned)(kSymvTileBytes + kSymvVecBytes));
  const int row0 = j + 1 + R * kSymvTB, col0 = j + 1 + C * kSymvTB;
#pragma unroll
  for (int bx = 0; bx < kSymvTB / 8; ++bx)
    tma_load_3d(dst + (unsigned)(bx << 13), map, 2 * (row0 + 8 * bx), col0, (int)b, bar);
  tma_load_3d(vdst, vmap, 2 * row0, j, (int)b, bar);
  tma_load_3d(vdst + kSymvTB * 16, vmap, 2 * col0, j, (int)b, bar);
}

// Finish of one tile from its warp partials (red: [direct, transposed][block][64 rows]
// complex, as doubles): thread t < 256 adds the four blocks of output o = t / 2,
// component t % 2, in block order; outputs 0..63 are the direct rows, 64..127 the
// transposed columns (on a diagonal tile both go to the same row, summed).
__device__ __forceinline__ void symv_tma_finish(const double* red, double2* part, int nbk, int R, int C) {
  const int t = threadIdx.x;
  if (t >= 2 * 2 * kSymvTB) return;
  const int o = t >> 1, comp = t & 1;
  const bool diag = (R == C);
  if (diag && o >= kSymvTB) return;
  const int kind = o >= kSymvTB ? 1 : 0, x = o & (kSymvTB - 1);
  const double* src = red + kind * (4 * kSymvTB * 2) + x * 2 + comp;
  double v = src[0];
#pragma unroll
  for (int q = 1; q < 4; ++q) v += src[q * kSymvTB * 2];
  if (diag) {
    const double* s2 = red + 4 * kSymvTB * 2 + x * 2 + comp;
    double w = s2[0];
#pragma unroll
    for (int q = 1; q < 4; ++q) w += s2[q * kSymvTB * 2];
    v += w;
  }
  double* dst = (double*)(part + ((int64_t)(kind ? C : R) * nbk + (kind ? R : C)) * kSymvTB + x);
  dst[comp] = v;
}

__global__ void __launch_bounds__(kSymvTmaThreads, 1)
    blk_symv_tma_kernel(const __grid_constant__ CUtensorMap map, const __grid_constant__ CUtensorMap vmap, BlkArgs a,
                        int j, int64_t nitems, int* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const unsigned raw = smem_u32(smem_raw);
  const unsigned base = (raw + 1023u) & ~1023u;                // 1024-byte aligned tiles (128-byte swizzle)
  unsigned char* tiles = smem_raw + (base - raw);
  const unsigned vbase = base + kSymvTmaStages * kSymvTileBytes;  // v segments of each stage
  const unsigned char* vsm = tiles + kSymvTmaStages * kSymvTileBytes;
  double* redsm = (double*)(tiles + kSymvTmaStages * (kSymvTileBytes + kSymvVecBytes));  // 2 buffers
  const unsigned bars = vbase + kSymvTmaStages * kSymvVecBytes + kSymvRedBytes;  // one mbarrier per stage
  const int m = a.n - j - 1;
  const int nbk = (m + kSymvTB - 1) / kSymvTB;
  const int ntiles = nbk * (nbk + 1) / 2;
  const int64_t first = blockIdx.x, step = gridDim.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int la = lane & 7, lb = lane >> 3;
  const int rw = (warp & 3) * 16, cw = (warp >> 2) * 16;  // the warp's sub-block
  if (*(volatile int*)err != 0) return;  // an earlier launch gave up: the pass is void, end at once
  if (threadIdx.x == 0) {
    for (int s = 0; s < kSymvTmaStages; ++s) mbar_init(bars + 8 * s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < kSymvTmaStages - 1; ++s) {
      const int64_t it = first + s * step;
      if (it < nitems)
        symv_tma_issue(&map, &vmap, j, ntiles, it, base + s * kSymvTileBytes, vbase + s * kSymvVecBytes, bars + 8 * s);
    }
  }
  int stage = 0;
  unsigned parity = 0;
  int64_t pk = -1;               // k-point of the previous tile (finished after this tile's barrier), or -1
  int pR = 0, pC = 0;
  int rb = 0;                    // reduction buffer of this tile
  for (int64_t it = first; it < nitems; it += step) {
    const int64_t b = it / ntiles;
    int R, C;
    symv_tile_rc((int)(it - b * ntiles), &R, &C);
    // the stage's copies have landed, and every thread is past the previous tile (so
    // its stage may be refilled and its partials read); the outcome of the bounded
    // wait is the block's
    const int ok = __syncthreads_and(mbar_wait_bounded(bars + 8 * stage, parity) ? 1 : 0);
    if (!ok) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        // leave no copy in flight: the stage of this item and, if issued, the next one
        mbar_wait_bounded(bars + 8 * stage, parity);
        if (it + step < nitems) {
          const int s1 = (stage + 1) % kSymvTmaStages;
          mbar_wait_bounded(bars + 8 * s1, s1 == 0 ? parity ^ 1u : parity);
        }
      }
      return;
    }
    if (threadIdx.x == 0) {
      const int64_t nx = it + (kSymvTmaStages - 1) * step;
      const int ns = (stage + kSymvTmaStages - 1) % kSymvTmaStages;
      if (nx < nitems)
        symv_tma_issue(&map, &vmap, j, ntiles, nx, base + ns * kSymvTileBytes, vbase + ns * kSymvVecBytes,
                       bars + 8 * ns);
    }
    if (pk >= 0) symv_tma_finish(redsm + (rb ^ 1) * (2 * 4 * kSymvTB * 2), a.part + pk * a.part_stride, nbk, pR, pC);
    const unsigned char* ts = tiles + stage * kSymvTileBytes;
    const double2* vR = (const double2*)(vsm + stage * kSymvVecBytes);  // zeros past the matrix edge
    const double2* vC = vR + kSymvTB;
    const bool diag = (R == C);
    const int r0 = rw + la, r1 = r0 + 8;
    const double2 vr0 = vR[r0], vr1 = vR[r1];
    double2 yd0 = cmk(0.0, 0.0), yd1 = yd0, yt[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int u = cw + lb + 4 * i;
      const double2 vc = vC[u];
      double2 e0 = *(const double2*)(ts + symv_sw(r0, u));
      double2 e1 = *(const double2*)(ts + symv_sw(r1, u));
      double2 f0 = e0, f1 = e1;  // the transposed product's copies
      if (diag) {  // lower part only: direct uses u <= row (diagonal real), transposed u < row
        if (u > r0) e0 = cmk(0.0, 0.0); else if (u == r0) e0.y = 0.0;
        if (u > r1) e1 = cmk(0.0, 0.0); else if (u == r1) e1.y = 0.0;
        if (u >= r0) f0 = cmk(0.0, 0.0);
        if (u >= r1) f1 = cmk(0.0, 0.0);
      }
      yd0 = cadd(yd0, cmul(e0, vc));
      yd1 = cadd(yd1, cmul(e1, vc));
      yt[i] = cadd(cmulc(f0, vr0), cmulc(f1, vr1));
    }
    constexpr unsigned FULL = 0xffffffffu;
    // direct: reduce over lb (lane bits 3, 4); the lane keeps row r0 + 8 (lb & 1), component lb >> 1
    double dk;
    {
      const bool h = lb & 1;
      double k0 = h ? yd1.x : yd0.x, k1 = h ? yd1.y : yd0.y;
      const double s0 = h ? yd0.x : yd1.x, s1 = h ? yd0.y : yd1.y;
      k0 += __shfl_xor_sync(FULL, s0, 8);
      k1 += __shfl_xor_sync(FULL, s1, 8);
      const bool h2 = lb & 2;
      dk = h2 ? k1 : k0;
      dk += __shfl_xor_sync(FULL, h2 ? k0 : k1, 16);
    }
    // transposed: reduce over la (lane bits 0..2); the lane keeps column
    // cw + lb + 4 (2 (la & 1) + ((la >> 1) & 1)), component (la >> 2) & 1
    double tk;
    {
      const bool g0 = la & 1;
      double q0 = g0 ? yt[2].x : yt[0].x, q1 = g0 ? yt[2].y : yt[0].y;
      double q2 = g0 ? yt[3].x : yt[1].x, q3 = g0 ? yt[3].y : yt[1].y;
      const double s0 = g0 ? yt[0].x : yt[2].x, s1 = g0 ? yt[0].y : yt[2].y;
      const double s2 = g0 ? yt[1].x : yt[3].x, s3 = g0 ? yt[1].y : yt[3].y;
      q0 += __shfl_xor_sync(FULL, s0, 1);
      q1 += __shfl_xor_sync(FULL, s1, 1);
      q2 += __shfl_xor_sync(FULL, s2, 1);
      q3 += __shfl_xor_sync(FULL, s3, 1);
      const bool g1 = la & 2;
      double p0 = g1 ? q2 : q0, p1 = g1 ? q3 : q1;
      const double u0 = g1 ? q0 : q2, u1 = g1 ? q1 : q3;
      p0 += __shfl_xor_sync(FULL, u0, 2);
      p1 += __shfl_xor_sync(FULL, u1, 2);
      const bool g2 = la & 4;
      tk = g2 ? p1 : p0;
      tk += __shfl_xor_sync(FULL, g2 ? p0 : p1, 4);
    }
    {
      double* red = redsm + rb * (2 * 4 * kSymvTB * 2);
      const int xr = r0 + 8 * (lb & 1), cd = lb >> 1;
      red[((warp >> 2) * kSymvTB + xr) * 2 + cd] = dk;
      const int xc = cw + lb + 4 * (2 * (la & 1) + ((la >> 1) & 1)), ct = (la >> 2) & 1;
      red[((4 + (warp & 3)) * kSymvTB + xc) * 2 + ct] = tk;
    }
    pk = b; pR = R; pC = C;
    rb ^= 1;
    stage = (stage + 1) % kSymvTmaStages;
    if (stage == 0) parity ^= 1u;
  }
  __syncthreads();
  if (pk >= 0) symv_tma_finish(redsm + (rb ^ 1) * (2 * 4 * kSymvTB * 2), a.part + pk * a.part_stride, nbk, pR, pC);
}

// off: the row offset of the reflectors (1 one-stage, the half-bandwidth two-stage)
__global__ void __launch_bounds__(kBlkThreads) blk_prep_kernel(int n, double2* A, int off) {
  const Team T = make_team();
  blk_prep_reflectors(T, n, A + (int64_t)blockIdx.x * n * n, n, off);
}

// grid (P, B); Tm: B x P x (nb x nb); dynamic smem: G (nb x nb double2); Gg: the
// Gram matrices V_p^H V_p laid out as Tm, or null (formed in the kernel)
// off: the row offset of the reflectors; their count is n - off
__global__ void __launch_bounds__(kBlkThreads) blk_larft_kernel(int n, int nb, int P, const double2* A,
                                                                const double2* tau, double2* Tm,
                                                                const double2* Gg, int off) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Team T = make_team();
  const int p = blockIdx.x;
  const int64_t b = blockIdx.y;
  const int j0 = p * nb;
  int nbr = n - off - j0;
  if (nbr > nb) nbr = nb;
  double2* Tp = Tm + (b * P + p) * (int64_t)nb * nb;
  if (nbr <= 0) {
    for (int q = T.tid; q < nb * nb; q += T.nt) Tp[q] = cmk(0.0, 0.0);
    return;
  }
  blk_larft(T, n, nb, j0, nbr, A + b * (int64_t)n * n, n, tau + b * n, Tp, (double2*)smem,
            Gg ? Gg + (b * P + p) * (int64_t)nb * nb : nullptr, off);
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
  unsigned long long* phase_cycles;  // [16] as eigh_kernel's (d&c total and merge steps), or null
};

__host__ __device__ inline int64_t dc_large_slot_doubles(int n, bool vec) {
  const int64_t nn = (int64_t)n * n;
  const int64_t vecs = 13 * (int64_t)n + 8 + (10 * (int64_t)n + 1) / 2 + 1 + 2 * (int64_t)(kDcThreads / 32) * n + 2;
  return (vec ? 3 * nn : 4 * (int64_t)n + 4) + vecs;
}

// dynamic shared memory: the merge GEMM's cp.async ring and the column indices of one merge
__host__ __device__ inline int dc_tile_smem(int n) { return kDcTileRing * 8 + ((n + 3) / 4) * 16; }

// NT = 512 (one CTA per SM) for orders with tiled merges; below kDcTileMin the
// merges are small and latency-bound, and NT = 128 with four CTAs per SM keeps
// four k-points in flight per SM.
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) dc_large_kernel(DCLargeArgs a) {
  __shared__ double red[128];
  extern __shared__ __align__(16) double tile[];
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
  const bool prof = a.phase_cycles != nullptr;
  unsigned long long dsub[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long dtot = 0;
  for (int64_t k = blockIdx.x; k < a.nk; k += gridDim.x) {
    for (int i = T.tid; i < n; i += T.nt) {
      S.d[i] = a.d[k * n + i];
      S.e[i] = (i < n - 1) ? a.e[k * n + i] : 0.0;
    }
    team_sync();
    const long long t0 = prof ? clock64() : 0;
    dc_solve(T, n, a.plan, S, Q, Qt, prof ? dsub : nullptr, vec, Ub, kDcTileMin);
    if (prof) dtot += (unsigned long long)(clock64() - t0);
    for (int i = T.tid; i < n; i += T.nt) a.bands[k * n + i] = S.D[i];
    if (vec) {
      double2* Uk = a.U + k * nn;
      for (int c = T.wid; c < n; c += T.nw)
        for (int r = T.lane; r < n; r += T.nl) Uk[r + (int64_t)c * n] = cmk(Q[r + (int64_t)c * n], 0.0);
    }
    team_sync();
  }
  if (prof && T.tid == 0) {
    atomicAdd(&a.phase_cycles[PH_DC], dtot);
    for (int i = 0; i < 8; ++i) atomicAdd(&a.phase_cycles[PH_DCSUB + i], dsub[i]);
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

// Occupation span of each k-point's states (eigenvalues ascending, so the exactly
// filled states, f == 1, form a prefix and the exactly empty ones, f == 0, a suffix):
// span[0] = max over k of the states that are not exactly filled, span[1] = max over k
// of the states that are not exactly empty (integer maxima: order-independent).
__global__ void __launch_bounds__(kBlkThreads) blk_occ_span_kernel(int n, const double* bands, double mu,
                                                                   double T_, int* span) {
  __shared__ int cnt[2];
  const int64_t k = blockIdx.x;
  if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
  __syncthreads();
  int notfull = 0, notempty = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double fj = fermi(bands[k * n + j] - mu, T_);
    notfull += fj != 1.0;
    notempty += fj != 0.0;
  }
  atomicAdd(&cnt[0], notfull);
  atomicAdd(&cnt[1], notempty);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(&span[0], cnt[0]);
    atomicMax(&span[1], cnt[1]);
  }
}

// rho_k from the K columns [c0, c0 + K) of U that carry it: Y[:, c] = U[:, c0 + c] f
// (direct: the first K states hold every nonzero f) or U[:, c0 + c] (1 - f)
// (complement: the last K states hold every f < 1, rho_k = I - Y U_K^H); the band
// energy sum_j w f_j eps_j over all states as blk_scale_f_kernel computes it.
__global__ void __launch_bounds__(kBlkThreads) blk_scale_f_cols_kernel(int n, const double2* U, const double* bands,
                                                                       double mu, double T_, const double* w,
                                                                       double2* Y, double* eband_k, int c0, int K,
                                                                       int complement) {
  __shared__ double red[128];
  extern __shared__ __align__(16) unsigned char smem[];
  double* f = (double*)smem;
  const Team T = make_team();
  const int64_t k = blockIdx.x;
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
  for (int c = T.wid; c < K; c += T.nw) {
    const double fc = complement ? 1.0 - f[c0 + c] : f[c0 + c];
    const double2* Uc = U + k * nn + (int64_t)(c0 + c) * n;
    double2* Yc = Y + k * nn + (int64_t)c * n;
    for (int r = T.lane; r < n; r += T.nl) Yc[r] = cscale(fc, Uc[r]);
  }
}

// rho_k is Hermitian and only its lower column blocks are formed: the strictly upper
// part of each 32 x 32 tile pair (I < J) is the conjugate transpose of tile (J, I),
// moved through shared memory so both the reads and the writes are coalesced.
// grid (tiles above the diagonal (J > I) of the 32-tile grid, nk).
__global__ void __launch_bounds__(256) blk_herm_mirror_kernel(int n, double2* R) {
  __shared__ double2 t[32][33];
  const int nt = (n + 31) / 32;
  int p = blockIdx.x, I = 0;  // p-th pair (I, J), J > I, row-major over I
  while (p >= nt - 1 - I) { p -= nt - 1 - I; ++I; }
  const int J = I + 1 + p;
  double2* Rk = R + (int64_t)blockIdx.y * n * n;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  // read tile (J, I) of the lower part: rows 32J + tx, columns 32I + c
  for (int c = ty; c < 32; c += 8) {
    const int r = 32 * J + tx, col = 32 * I + c;
    if (r < n && col < n) t[c][tx] = Rk[r + (int64_t)col * n];
  }
  __syncthreads();
  // write tile (I, J): rows 32I + tx, columns 32J + c, value conj(R[32J + c, 32I + tx])
  for (int c = ty; c < 32; c += 8) {
    const int r = 32 * I + tx, col = 32 * J + c;
    if (r < n && col < n) Rk[r + (int64_t)col * n] = cconj(t[tx][c]);
  }
}

// rho_k = I - (Y U_K^H): the identity added to the diagonal (complement form).
__global__ void __launch_bounds__(kBlkThreads) blk_add_identity_kernel(int n, double2* R) {
  const int64_t nn = (int64_t)n * n;
  double2* Rk = R + blockIdx.x * nn;
  for (int i = threadIdx.x; i < n; i += blockDim.x) Rk[i + (int64_t)i * n].x += 1.0;
}


// ---- Two-stage reduction (lqm_twostage.cuh) ----
constexpr int kTsB = 16;              // half-bandwidth of the stage-1 band
constexpr int kTsPanelThreads = 512;  // panel QR: latency-bound row passes, CTA per k-point
constexpr int kTsChaseWarps = 8;      // bulge chase: sweeps in flight per k-point (one warp each)
constexpr int kTsWaitPolls = 1 << 26; // bound of one inter-warp wait of the chase (shared-memory polls, ~1 s)

// complex per k-point of the stage-2 reflector store (sweeps 0..n-2, tmax slots of kTsB each)
__host__ __device__ inline int64_t ts_v2_stride(int n) {
  return (int64_t)(n > 1 ? n - 1 : 1) * ts_tmax(n, kTsB) * kTsB;
}
__host__ __device__ inline int64_t ts_tau2_stride(int n) { return (int64_t)(n > 1 ? n - 1 : 1) * ts_tmax(n, kTsB); }

// grid (B): panel j0 of every k-point.  Vb: B x (n x kTsB), Tm: B x (kTsB x kTsB).
__global__ void __launch_bounds__(kTsPanelThreads) ts_panel_kernel(int n, int j0, double2* A, double2* tau,
                                                                   double2* Vb, double2* Tm) {
  __shared__ __align__(16) double2 sm[(kTsPanelThreads / 32 + 2) * kTsB + kTsB * kTsB];
  const Team T = make_team();
  const int64_t b = blockIdx.x;
  ts_panel_qr<kTsB>(T, n, j0, A + b * (int64_t)n * n, n, tau + b * n, Vb + b * (int64_t)n * kTsB, n,
                    Tm + b * kTsB * kTsB, sm);
}

// grid (B): the band (2 kTsB x n per k-point) out of the stage-1 result.
__global__ void __launch_bounds__(kBlkThreads) ts_band_kernel(int n, const double2* A, double2* Bd) {
  const Team T = make_team();
  const int64_t b = blockIdx.x;
  ts_band_extract<kTsB>(T, n, A + b * (int64_t)n * n, n, Bd + b * 2 * kTsB * (int64_t)n);
}

// grid (B), kTsChaseWarps warps: the bulge chase of one k-point.  Warp w takes the
// sweeps s = w, w + W, ... (ts_chase_sweep, its blocks in the warp's window of
// dynamic shared memory); before task t of sweep s it waits until sweep s - 1 has
// finished its tasks 0 .. t + 2 (the tasks whose rows and columns overlap task t's),
// read from a per-warp progress word in shared memory.  The band stays in global
// memory (L1/L2): a warp's stores are fenced at block scope before it publishes
// progress, and a waiting warp fences after it reads it.  Every wait is bounded
// (wait_polls polls of the progress word): on expiry the kernel records an error in
// *err, every warp stops at its next wait, and d / e are written as zeros.  V2 / tau2 (or null): the reflectors for the
// back-transformation.  Outputs: d (n) and e (n - 1) of the real tridiagonal.
constexpr int kTsWin = 3 * kTsB * (kTsB + 1) + 2 * kTsB;  // complex per warp window
constexpr int kTsChaseSmem = kTsChaseWarps * kTsWin * 16;
__global__ void __launch_bounds__(kTsChaseWarps * 32) ts_chase_kernel(int n, double2* Bd, double2* V2,
                                                                      double2* tau2, double* d, double* e,
                                                                      int* err, long long wait_polls) {
  extern __shared__ __align__(16) double2 tswin[];
  __shared__ long long prog[kTsChaseWarps];
  __shared__ int stop;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpTeam T = make_warpteam();
  const int64_t b = blockIdx.x;
  constexpr int ldb = 2 * kTsB;
  double2* Bk = Bd + b * ldb * (int64_t)n;
  const int tmax = ts_tmax(n, kTsB);
  const long long unit = tmax + 1;  // progress: s * unit + tasks done
  if (lane == 0) prog[w] = -1;
  if (threadIdx.x == 0) stop = (err && *(volatile int*)err) ? 1 : 0;
  __syncthreads();
  volatile long long* vprog = prog;
  volatile int* vstop = &stop;
  bool ok = *vstop == 0;
  const int wp = (w + kTsChaseWarps - 1) % kTsChaseWarps;  // the warp of sweep s - 1
  for (int s = w; ok && s <= n - 2; s += kTsChaseWarps) {
    const int ntp = (s > 0) ? ts_tasks(n, kTsB, s - 1) : 0;
    auto wait = [&](int t) -> bool {
      if (s == 0) return true;
      const long long need = (long long)(s - 1) * unit + (t + 3 < ntp ? t + 3 : ntp);
      bool good = true;
      if (lane == 0) {
        long long polls = 0;
        while (vprog[wp] < need) {
          if (*vstop) { good = false; break; }
          if (++polls > wait_polls) {
            *vstop = 1;
            if (err) atomicExch(err, 2);
            good = false;
            break;
          }
        }
      }
      good = __shfl_sync(0xffffffffu, good, 0);
      __syncwarp();
      __threadfence_block();
      return good;
    };
    auto done = [&](int t) {
      __threadfence_block();
      __syncwarp();
      if (lane == 0) vprog[w] = (long long)s * unit + t + 1;
    };
    double2* vo = V2 ? V2 + b * ts_v2_stride(n) + (int64_t)s * tmax * kTsB : nullptr;
    double2* to = tau2 ? tau2 + b * ts_tau2_stride(n) + (int64_t)s * tmax : nullptr;
    ok = ts_chase_sweep<kTsB>(T, n, s, Bk, vo, to, tswin + w * kTsWin, wait, done);
  }
  __syncthreads();
  const bool fin = *vstop == 0;  // after a failed wait: zeros, so the solver that follows stays bounded
  __threadfence_block();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[b * n + i] = fin ? Bk[(int64_t)i * ldb].x : 0.0;
    e[b * n + i] = (fin && i + 1 < n) ? Bk[1 + (int64_t)i * ldb].x : 0.0;
  }
}

// Q2 Z in the grouped order (ts_q2_apply_grouped_host): grid (ceil(K / 256), B),
// thread = one of the columns c0 .. c0+K-1 of U (n x n per k-point, in place).
// Each (group of 16 sweeps, task t) step applies 16 reflectors to a window of 31
// rows of the thread's column, held in registers (all indices compile-time); the
// window slides by 16 rows per step, so a group streams the column once.  The
// step's reflectors and taus (16 x 16 + 16 complex; zeros where a sweep has no
// task t) are copied into shared memory by cp.async one step ahead, and the 16 rows
// of the next slide are prefetched into L1.  A reflector's dot product runs in two
// partial sums: with four the prefetch addresses no longer fit the 255 registers
// (spills), and two with the prefetch measured 5% faster than four without it.
constexpr int kTsQ2gThreads = 256;
// rows r0 .. r0 + kTsB - 1 (those below n) of column c: 256 bytes, at most three lines,
// requested one step before the slide that loads them, so that they arrive while the
// step's reflectors are applied
__device__ __forceinline__ void prefetch_rows(const double2* c, int r0, int n) {
  if (r0 < n) prefetch_l1(c + r0);
  if (r0 + 8 < n) prefetch_l1(c + r0 + 8);
  if (r0 + kTsB - 1 < n) prefetch_l1(c + r0 + kTsB - 1);
}
constexpr int kTsQ2gStep = kTsB * kTsB + kTsB;  // complex per staged step
__global__ void __launch_bounds__(kTsQ2gThreads, 1) ts_q2g_kernel(int n, int c0, int K, const double2* V2,
                                                                  const double2* tau2, double2* U) {
  constexpr int B = kTsB, W = 2 * kTsB - 1;
  __shared__ __align__(16) double2 sv[2][kTsQ2gStep];
  const int64_t b = blockIdx.y;
  const int col = blockIdx.x * kTsQ2gThreads + threadIdx.x;
  const bool act = col < K;
  double2* Uc = U + b * (int64_t)n * n + (int64_t)(c0 + (act ? col : 0)) * n;
  const double2* Vk = V2 + b * ts_v2_stride(n);
  const double2* tk = tau2 + b * ts_tau2_stride(n);
  const int tmax = ts_tmax(n, B);
  const int ns = n - 1;
  if (ns <= 0) return;
  const int g0 = (ns - 1) / B;  // highest group
  // step (g, t) -> shared buffer: reflector i of the step = sweep g B + i, task t
  auto stage = [&](int g, int t, double2* dst) {
    for (int e = threadIdx.x; e < kTsQ2gStep; e += blockDim.x) {
      const int i = (e < B * B) ? e / B : e - B * B;
      const int s = g * B + i;
      const bool ok = s < ns && t < ts_tasks(n, B, s);
      const double2* src = (e < B * B) ? Vk + ((int64_t)s * tmax + t) * B + (e - i * B) : tk + (int64_t)s * tmax + t;
      cp_async16(dst + e, ok ? (const void*)src : (const void*)Vk, ok);
    }
  };
  int buf = 0;
  stage(g0, 0, sv[0]);
  cp_async_commit();
  for (int g = g0; g >= 0; --g) {
    const int s0 = g * B;
    const int nt = ts_tasks(n, B, s0);
    double2 z[W];
    const int w0 = s0 + 1;
#pragma unroll
    for (int j = 0; j < W; ++j) z[j] = (act && w0 + j < n) ? Uc[w0 + j] : cmk(0.0, 0.0);
    for (int t = 0; t < nt; ++t) {
      // next step: (g, t + 1), or the next group's first
      if (t + 1 < nt) stage(g, t + 1, sv[buf ^ 1]);
      else if (g > 0) stage(g - 1, 0, sv[buf ^ 1]);
      cp_async_commit();
      cp_async_wait_keep1();
      __syncthreads();
      const double2* vs = sv[buf];
#pragma unroll
      for (int i = B - 1; i >= 0; --i) {
        const double2 tj = vs[B * B + i];
        double2 a[2] = {cmk(0.0, 0.0), cmk(0.0, 0.0)};
#pragma unroll
        for (int r = 0; r < B; ++r) a[r & 1] = cfma_conj(a[r & 1], vs[i * B + r], z[i + r]);
        const double2 f = cmul(tj, cadd(a[0], a[1]));
#pragma unroll
        for (int r = 0; r < B; ++r) z[i + r] = cfms(z[i + r], vs[i * B + r], f);
      }
      __syncthreads();  // the buffer is refilled two steps on
      buf ^= 1;
      const int wt = w0 + t * B;  // first row of this step's window
      if (t + 1 < nt) {
#pragma unroll
        for (int j = 0; j < B; ++j)
          if (act && wt + j < n) Uc[wt + j] = z[j];
#pragma unroll
        for (int j = 0; j < W - B; ++j) z[j] = z[j + B];
#pragma unroll
        for (int j = W - B; j < W; ++j) z[j] = (act && wt + B + j < n) ? Uc[wt + B + j] : cmk(0.0, 0.0);
        if (act && t + 2 < nt) prefetch_rows(Uc, wt + B + W, n);  // the next step's slide
      } else {
#pragma unroll
        for (int j = 0; j < W; ++j)
          if (act && wt + j < n) Uc[wt + j] = z[j];
      }
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

}  // namespace lqm
