// Divide-and-conquer merge plan for a tridiagonal of order n (host side).
//
// The index range [0, n) is split recursively at mid = lo + (hi-lo)/2 down to
// single rows.  Every internal node is one merge; its height is
// 1 + max(child heights).  Merges run height by height, so all children of a
// node are finished before it.  owner[(h-1)*n + i] names the node of height h
// that contains row i (or -1).  The flat int buffer is uploaded as is.
#pragma once
#include <algorithm>
#include <vector>

namespace lqm {

struct DCPlanHost {
  std::vector<int> buf;
  int nnodes = 0, nheights = 0;
  size_t off_hstart = 0, off_lo = 0, off_mid = 0, off_hi = 0, off_own = 0;
};

struct DCNodeH { int lo, mid, hi, h; };

inline int dc_build_tree(int lo, int hi, std::vector<DCNodeH>& nodes) {
  if (hi - lo < 2) return 0;
  const int mid = lo + (hi - lo) / 2;
  const int h1 = dc_build_tree(lo, mid, nodes);
  const int h2 = dc_build_tree(mid, hi, nodes);
  const int h = 1 + std::max(h1, h2);
  nodes.push_back({lo, mid, hi, h});
  return h;
}

inline DCPlanHost make_dc_plan_host(int n) {
  std::vector<DCNodeH> nodes;
  const int H = dc_build_tree(0, n, nodes);
  std::stable_sort(nodes.begin(), nodes.end(), [](const DCNodeH& a, const DCNodeH& b) { return a.h < b.h; });
  DCPlanHost P;
  P.nnodes = (int)nodes.size();
  P.nheights = H;
  std::vector<int> cnt(H + 1, 0), hs(H + 1, 0);
  for (const auto& nd : nodes) cnt[nd.h]++;
  for (int h = 1; h <= H; ++h) hs[h] = hs[h - 1] + cnt[h];
  P.off_hstart = 0;
  P.buf.insert(P.buf.end(), hs.begin(), hs.end());
  P.off_lo = P.buf.size();
  for (auto& nd : nodes) P.buf.push_back(nd.lo);
  P.off_mid = P.buf.size();
  for (auto& nd : nodes) P.buf.push_back(nd.mid);
  P.off_hi = P.buf.size();
  for (auto& nd : nodes) P.buf.push_back(nd.hi);
  P.off_own = P.buf.size();
  std::vector<int> owner((size_t)H * n, -1);
  for (int id = 0; id < P.nnodes; ++id)
    for (int i = nodes[id].lo; i < nodes[id].hi; ++i) owner[(size_t)(nodes[id].h - 1) * n + i] = id;
  P.buf.insert(P.buf.end(), owner.begin(), owner.end());
  if (P.buf.empty()) P.buf.push_back(0);
  return P;
}

}  // namespace lqm
