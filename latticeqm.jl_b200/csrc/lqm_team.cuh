// Thread-team abstraction shared by the CUDA kernels and their host emulation.
//
// Every per-k algorithm in this library is written as a sequence of "team
// phases": strided loops over work items (threads), warps (for column dot
// products) or a single thread, separated by team_sync().  Under nvcc the
// team is one CTA (tid = threadIdx.x, 32-lane warps).  Compiled by a host C++
// compiler the same code runs with a one-thread, one-lane team, where every
// loop visits all items in order and team_sync()/warp_sum() are identities.
// The host build exists only so the index arithmetic can be exercised on a
// CPU; the product path is the CUDA build.
#pragma once

#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define LQM_FN __device__ __forceinline__
#define LQM_FN_NOINLINE __device__ __noinline__
#else
#define LQM_FN static inline
#define LQM_FN_NOINLINE static
#ifndef LQM_HAVE_DOUBLE2
#define LQM_HAVE_DOUBLE2
struct double2 { double x, y; };
#endif
#endif

struct Team {
  int tid, nt;    // thread index / threads in team
  int lane, nl;   // lane index / lanes per warp
  int wid, nw;    // warp index / warps in team
};

#if defined(__CUDACC__)
LQM_FN Team make_team() {
  Team t;
  t.tid = threadIdx.x; t.nt = blockDim.x;
  t.lane = threadIdx.x & 31; t.nl = 32;
  t.wid = threadIdx.x >> 5; t.nw = blockDim.x >> 5;
  return t;
}
LQM_FN void team_sync() { __syncthreads(); }
LQM_FN void team_sync(const Team&) { __syncthreads(); }

// One FP64 tensor-core step D = A B + D of mma.sync.aligned.m8n8k4 (row-major A,
// column-major B): with g = lane / 4, t = lane % 4 the lane holds a = A[g][t],
// b = B[t][g] and d0, d1 = D[g][2t], D[g][2t + 1] (PTX ISA fragment layout).
LQM_FN void dmma_884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// One of the independent teams of `size` threads (a multiple of 32) that split a
// CTA: thread threadIdx.x belongs to team threadIdx.x / size, which synchronises on
// its own named barrier (1 + team index; at most 15 teams per CTA).  The per-k
// phases are templates on the team type, so the CTA-wide kernels keep
// __syncthreads and only the split kernels pay for named barriers.
struct SubTeam {
  int tid, nt;
  int lane, nl;
  int wid, nw;
  int bar;
};
LQM_FN SubTeam make_subteam(int size) {
  SubTeam t;
  t.tid = threadIdx.x % size; t.nt = size;
  t.lane = threadIdx.x & 31; t.nl = 32;
  t.wid = t.tid >> 5; t.nw = size >> 5;
  t.bar = 1 + threadIdx.x / size;
  return t;
}
LQM_FN void team_sync(const SubTeam& T) { asm volatile("bar.sync %0, %1;\n" ::"r"(T.bar), "r"(T.nt) : "memory"); }
// One warp as a team (warp-synchronous phases, e.g. one bulge-chasing sweep per warp).
struct WarpTeam {
  int tid, nt;
  int lane, nl;
  int wid, nw;
};
LQM_FN WarpTeam make_warpteam() {
  WarpTeam t;
  t.tid = threadIdx.x & 31; t.nt = 32;
  t.lane = t.tid; t.nl = 32;
  t.wid = 0; t.nw = 1;
  return t;
}
LQM_FN void team_sync(const WarpTeam&) { __syncwarp(); }
LQM_FN void team_syncwarp() { __syncwarp(); }
LQM_FN double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
LQM_FN double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// Butterfly sum whose result is then taken from lane 0, so every lane holds
// bit-identical values (uniform control flow may branch on it).
LQM_FN double warp_sum_bcast(double v) {
  v = warp_sum(v);
  return __shfl_sync(0xffffffffu, v, 0);
}
// Sum over aligned groups of `width` lanes (power of two); every lane of a
// group receives its group leader's value.  All 32 lanes must call it.
LQM_FN double group_sum_bcast(double v, int width) {
  for (int o = width >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, width);
  return __shfl_sync(0xffffffffu, v, 0, width);
}
#else
LQM_FN Team make_host_team() { Team t = {0, 1, 0, 1, 0, 1}; return t; }
LQM_FN void team_sync() {}
LQM_FN void team_sync(const Team&) {}
LQM_FN void team_syncwarp() {}
LQM_FN double warp_sum(double v) { return v; }
LQM_FN double warp_max(double v) { return v; }
LQM_FN double warp_sum_bcast(double v) { return v; }
LQM_FN double group_sum_bcast(double v, int width) { (void)width; return v; }
#endif

// Deterministic team reduction: warp trees, then every thread sums the warp
// partials in warp order.  `red` needs >= 32 doubles of shared memory.
template <class TeamT>
LQM_FN double team_sum(const TeamT& T, double v, double* red) {
#if defined(__CUDACC__)
  v = warp_sum(v);
  if (T.lane == 0) red[T.wid] = v;
  team_sync(T);
  double s = 0.0;
  for (int w = 0; w < T.nw; ++w) s += red[w];
  team_sync(T);
  return s;
#else
  (void)T; (void)red;
  return v;
#endif
}

template <class TeamT>
LQM_FN double team_max(const TeamT& T, double v, double* red) {
#if defined(__CUDACC__)
  v = warp_max(v);
  if (T.lane == 0) red[T.wid] = v;
  team_sync(T);
  double s = red[0];
  for (int w = 1; w < T.nw; ++w) s = fmax(s, red[w]);
  team_sync(T);
  return s;
#else
  (void)T; (void)red;
  return v;
#endif
}

// Two sums with ONE barrier: each caller alternates between two disjoint
// `red` halves (>= 64 doubles each) so that a half is only rewritten after
// another barrier has separated it from its last reads.
template <class TeamT>
LQM_FN void team_sum2_1b(const TeamT& T, double& a, double& b, double* red) {
#if defined(__CUDACC__)
  a = warp_sum(a);
  b = warp_sum(b);
  if (T.lane == 0) { red[2 * T.wid] = a; red[2 * T.wid + 1] = b; }
  team_sync(T);
  // four interleaved partial sums (in warp order within each) keep the
  // dependent-add chain short; the result is still fixed for a given team size
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0, b3 = 0.0;
  int w = 0;
  for (; w + 4 <= T.nw; w += 4) {
    a0 += red[2 * w]; b0 += red[2 * w + 1];
    a1 += red[2 * w + 2]; b1 += red[2 * w + 3];
    a2 += red[2 * w + 4]; b2 += red[2 * w + 5];
    a3 += red[2 * w + 6]; b3 += red[2 * w + 7];
  }
  for (; w < T.nw; ++w) { a0 += red[2 * w]; b0 += red[2 * w + 1]; }
  a = (a0 + a1) + (a2 + a3);
  b = (b0 + b1) + (b2 + b3);
#else
  (void)T; (void)red; (void)a; (void)b;
#endif
}

// ---- complex helpers (interleaved re/im, ABI-identical to Julia ComplexF64) ----
LQM_FN double2 cmk(double re, double im) { double2 z; z.x = re; z.y = im; return z; }
LQM_FN double2 cadd(double2 a, double2 b) { return cmk(a.x + b.x, a.y + b.y); }
LQM_FN double2 csub(double2 a, double2 b) { return cmk(a.x - b.x, a.y - b.y); }
LQM_FN double2 cmul(double2 a, double2 b) { return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// conj(a) * b
LQM_FN double2 cmulc(double2 a, double2 b) { return cmk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }
LQM_FN double2 cconj(double2 a) { return cmk(a.x, -a.y); }
LQM_FN double2 cscale(double s, double2 a) { return cmk(s * a.x, s * a.y); }
// a / b with Smith's scaling
// acc + conj(a) b, acc + a b and z - a b as four fused multiply-adds each (one rounding per
// real product-sum instead of a product, a sum and a second rounding)
LQM_FN double2 cfma_conj(double2 acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}
LQM_FN double2 cfma(double2 acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
LQM_FN double2 cfms(double2 z, double2 a, double2 b) {
  z.x = fma(-a.x, b.x, z.x);
  z.x = fma(a.y, b.y, z.x);
  z.y = fma(-a.x, b.y, z.y);
  z.y = fma(-a.y, b.x, z.y);
  return z;
}
#if defined(__CUDACC__)
// A complex value from lane `src` of the warp (all 32 lanes must call it).
LQM_FN double2 shfl_c(double2 v, int src) {
  return cmk(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
#endif
LQM_FN double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, den = b.x + b.y * r;
    return cmk((a.x + a.y * r) / den, (a.y - a.x * r) / den);
  } else {
    double r = b.x / b.y, den = b.y + b.x * r;
    return cmk((a.x * r + a.y) / den, (a.y * r - a.x) / den);
  }
}

// (cos(pi x), sin(pi x)) — CUDA's sincospi on the device; the host
// emulation uses the libm pair, which is only used for index checks.
LQM_FN void lqm_sincospi(double x, double* s, double* c) {
#if defined(__CUDACC__)
  sincospi(x, s, c);
#else
  *s = sin(M_PI * x);
  *c = cos(M_PI * x);
#endif
}
