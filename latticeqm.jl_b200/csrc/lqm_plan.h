// Divide-and-conquer merge plan for a tridiagonal of order n.
//
// The index range [0, n) is split recursively at mid = lo + (hi-lo)/2 down to
// single rows.  Every internal node is one merge; its height is
// 1 + max(child heights) = ceil(log2(size)).  Merges run height by height, so
// all children of a node are finished before it.  Flat int layout:
//   [ hstart (H+1) | lo (n-1) | mid (n-1) | hi (n-1) | owner (H*n) ]
// hstart[h-1] .. hstart[h] are the nodes of height h (in post-order), and
// owner[(h-1)*n + i] names the node of height h containing row i, or -1.
// dc_plan_fill() is shared by the host (uploaded plans) and the device
// (plans built in place by the allocation-free entry point).
#pragma once
#include <vector>

#if defined(__CUDACC__)
#define LQM_PLAN_FN __host__ __device__ inline
#else
#define LQM_PLAN_FN inline
#endif

namespace lqm {

LQM_PLAN_FN int dc_plan_height(int n) {
  int h = 0;
  while ((1 << h) < n) ++h;
  return h;
}

LQM_PLAN_FN int dc_plan_ints(int n) {
  const int H = dc_plan_height(n);
  const int nn = n > 1 ? n - 1 : 0;
  return (H + 1) + 3 * nn + H * n;
}

// Fills buf (dc_plan_ints(n) ints).  Single-threaded; the explicit stack bounds
// the depth at 64 (n < 2^63).
LQM_PLAN_FN void dc_plan_fill(int n, int* buf) {
  const int H = dc_plan_height(n);
  const int nnodes = n > 1 ? n - 1 : 0;
  int* hs = buf;
  int* lo = buf + (H + 1);
  int* mid = lo + nnodes;
  int* hi = mid + nnodes;
  int* own = hi + nnodes;
  // count nodes per height (height of a node of size s is ceil(log2 s))
  for (int h = 0; h <= H; ++h) hs[h] = 0;
  // iterative post-order traversal: stack of (lo, hi, visited)
  int slo[64], shi[64], svis[64];
  int top = 0;
  // pass 1: counts
  slo[0] = 0; shi[0] = n; svis[0] = 0; top = 1;
  while (top > 0) {
    const int a = slo[top - 1], b = shi[top - 1];
    if (b - a < 2) { --top; continue; }
    if (!svis[top - 1]) {
      svis[top - 1] = 1;
      const int m = a + (b - a) / 2;
      slo[top] = m; shi[top] = b; svis[top] = 0; ++top;   // right child (popped second)
      slo[top] = a; shi[top] = m; svis[top] = 0; ++top;   // left child (popped first)
    } else {
      hs[dc_plan_height(b - a)]++;
      --top;
    }
  }
  // prefix: hs[h-1] = first node of height h
  int run = 0;
  for (int h = 1; h <= H; ++h) { const int c = hs[h]; hs[h - 1] = run; run += c; }
  hs[H] = run;
  // pass 2: place nodes in post-order within their height
  int fill[64];
  for (int h = 1; h <= H; ++h) fill[h] = hs[h - 1];
  slo[0] = 0; shi[0] = n; svis[0] = 0; top = 1;
  while (top > 0) {
    const int a = slo[top - 1], b = shi[top - 1];
    if (b - a < 2) { --top; continue; }
    if (!svis[top - 1]) {
      svis[top - 1] = 1;
      const int m = a + (b - a) / 2;
      slo[top] = m; shi[top] = b; svis[top] = 0; ++top;
      slo[top] = a; shi[top] = m; svis[top] = 0; ++top;
    } else {
      const int h = dc_plan_height(b - a);
      const int id = fill[h]++;
      lo[id] = a; mid[id] = a + (b - a) / 2; hi[id] = b;
      --top;
    }
  }
  for (int i = 0; i < H * n; ++i) own[i] = -1;
  for (int id = 0; id < nnodes; ++id) {
    const int h = dc_plan_height(hi[id] - lo[id]);
    for (int i = lo[id]; i < hi[id]; ++i) own[(h - 1) * n + i] = id;
  }
}

struct DCPlanHost {
  std::vector<int> buf;
  int nnodes = 0, nheights = 0;
  size_t off_hstart = 0, off_lo = 0, off_mid = 0, off_hi = 0, off_own = 0;
};

inline DCPlanHost make_dc_plan_host(int n) {
  DCPlanHost P;
  P.nheights = dc_plan_height(n);
  P.nnodes = n > 1 ? n - 1 : 0;
  P.buf.assign((size_t)dc_plan_ints(n) + 1, 0);
  dc_plan_fill(n, P.buf.data());
  P.off_hstart = 0;
  P.off_lo = (size_t)P.nheights + 1;
  P.off_mid = P.off_lo + P.nnodes;
  P.off_hi = P.off_mid + P.nnodes;
  P.off_own = P.off_hi + P.nnodes;
  return P;
}

}  // namespace lqm
