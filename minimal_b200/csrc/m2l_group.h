// Layout of the grouped M2L operators and the work plan of the GEMM kernels.
//
// Realified expansions: input x (scaled multipole) and output y (scaled
// local) are real vectors of length 2*NT (re, im of each m >= 0 coefficient,
// index 2*(n(n+1)/2+m) + {0,1}), padded to KP (a multiple of 16).  The
// operator of one group maps x to y; because the reference truncates M2L to
// j + n < P, the rows of output degree j only see the first 2*tri(P-j)
// inputs.  Rows are cut into blocks of 8 (the DMMA M); row block rb keeps
// only its K prefix kp4[rb] = 2*tri(P - j_min(rb)) rounded up to 4, stored
// k-major: W[woff[rb] + k*8 + r].
//
// The FP64 kernel runs 8 warps per tile of 32 targets; each warp owns up to
// GP_MAXP "pieces" (row block, k range), balanced by K length, with DMMA
// accumulators for all 4 column blocks of the tile held in registers.  A
// plan whose warps hold at most GP_MAXP_SMALL pieces (every order up to 10,
// and 12) is laid out with that stride and run by the kernel instantiated for
// it: fewer accumulator registers, so two CTAs share an SM.
#pragma once
#include <algorithm>
#include <vector>

namespace fmm {

constexpr int GP_WARPS = 8;
constexpr int GP_MAXP = 6;
constexpr int GP_MAXP_SMALL = 4;
constexpr int GP_TILE = 32;

struct GroupPlan {
  int P = 0, NT = 0, KP = 0, nrb = 0, wsize = 0;
  int maxp = 0;  // pieces per warp in the layout: GP_MAXP_SMALL or GP_MAXP
  std::vector<int> kp4, woff, jmin;
  // pieces[w*maxp + p] = rb | k0 << 8 | k1 << 20 (k1 exclusive), -1 none
  std::vector<int> pieces;
  // rank of the piece among the pieces of its row block (0 stores, >0 adds)
  std::vector<int> prank;
  int maxrank = 0;
};

inline int gp_tri(int n) { return n * (n + 1) / 2; }

inline GroupPlan make_group_plan(int P) {
  GroupPlan g;
  g.P = P;
  g.NT = gp_tri(P);
  g.KP = (2 * g.NT + 15) / 16 * 16;
  g.nrb = (2 * g.NT + 7) / 8;
  g.kp4.resize(g.nrb);
  g.woff.resize(g.nrb + 1);
  g.jmin.resize(g.nrb);
  g.woff[0] = 0;
  for (int rb = 0; rb < g.nrb; rb++) {
    const int o = (8 * rb) / 2;  // first output coefficient of the block
    int j = 0;
    while (gp_tri(j + 1) <= o) j++;
    g.jmin[rb] = j;
    const int klen = 2 * gp_tri(P - j);
    g.kp4[rb] = (klen + 3) / 4 * 4;
    g.woff[rb + 1] = g.woff[rb] + 8 * g.kp4[rb];
  }
  g.wsize = g.woff[g.nrb];
  // split row blocks into k pieces no longer than the per-warp share, then
  // assign longest first to the least loaded warp
  int total = 0;
  for (int rb = 0; rb < g.nrb; rb++) total += g.kp4[rb];
  if (g.nrb > GP_WARPS * GP_MAXP) return GroupPlan{};  // too many row blocks: P == 0 marks "no plan"
  for (int cap = (total + GP_WARPS - 1) / GP_WARPS; cap <= total + 4; cap += 4) {
    struct Pc { int rb, k0, k1; };
    std::vector<Pc> pcs;
    const int c4 = (cap + 3) / 4 * 4;
    for (int rb = 0; rb < g.nrb; rb++)
      for (int k0 = 0; k0 < g.kp4[rb]; k0 += c4) pcs.push_back({rb, k0, std::min(g.kp4[rb], k0 + c4)});
    std::sort(pcs.begin(), pcs.end(), [](const Pc &a, const Pc &b) { return a.k1 - a.k0 > b.k1 - b.k0; });
    std::vector<int> load(GP_WARPS, 0), cnt(GP_WARPS, 0);
    std::vector<std::vector<Pc>> wp(GP_WARPS);
    bool ok = true;
    for (const Pc &p : pcs) {
      int best = -1;
      for (int w = 0; w < GP_WARPS; w++)
        if (cnt[w] < GP_MAXP && (best < 0 || load[w] < load[best])) best = w;
      if (best < 0) { ok = false; break; }
      wp[best].push_back(p);
      load[best] += p.k1 - p.k0;
      cnt[best]++;
    }
    if (!ok) continue;
    g.maxp = *std::max_element(cnt.begin(), cnt.end()) <= GP_MAXP_SMALL ? GP_MAXP_SMALL : GP_MAXP;
    g.pieces.assign(GP_WARPS * g.maxp, -1);
    g.prank.assign(GP_WARPS * g.maxp, 0);
    std::vector<int> seen(g.nrb, 0);
    for (int w = 0; w < GP_WARPS; w++)
      for (size_t p = 0; p < wp[w].size(); p++) {
        const Pc &c = wp[w][p];
        g.pieces[w * g.maxp + p] = c.rb | (c.k0 << 8) | (c.k1 << 20);
        g.prank[w * g.maxp + p] = seen[c.rb]++;
        g.maxrank = std::max(g.maxrank, g.prank[w * g.maxp + p]);
      }
    return g;
  }
  return GroupPlan{};
}

}  // namespace fmm
