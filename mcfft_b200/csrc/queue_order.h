// Order of the batch queue's (pass, tile) items (host only, no CUDA).
//
// The batch kernel deals item i to CTA i % G and every CTA runs its items in
// order, all CTAs resident.  A tile of a pass at level > 0 waits until the
// previous pass of its transform group has completed the tile's key (its
// dependency counter).  If every dependency points to an earlier item, the
// earliest unfinished item never waits, so the queue always drains; within
// that rule the order decides how long CTAs sit idle on a dependency and how
// often a CTA switches pass (a switch reloads the pass's tables).
//
// The order built here:
//   - first passes in chunks of QC G tiles (QC consecutive tiles per CTA),
//     group after group, with no gap between groups;
//   - after each chunk, every dependent tile whose key was completed at
//     least QC G items earlier (so, per CTA, about QC items earlier), across
//     all groups: the tail of one group's dependent pass runs beside the
//     next group's first pass instead of waiting on the tiles just before it;
//   - once no first-pass tile is left and nothing meets the lag, the rest in
//     dependency order (the only place where a tile waits on a tile queued
//     just before it: the end of the queue).
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace mcfft {

struct QOrderPass {
  int64_t ntiles = 0;      // tiles of the pass
  int64_t col_blocks = 1;  // level > 0: tile t waits for key t / col_blocks
  int64_t sig_mul = 1;     // producer side: once tiles 0..t are done, the keys
  int64_t sig_div = 1;     //   k < (t + 1) sig_mul / sig_div of the next pass are complete
  int64_t keys = 0;        // level > 0: number of keys of the pass
  int grp = 0;             // transform group (a group's passes are consecutive)
};

struct QOrderItem {
  uint32_t pass;
  uint32_t tile;
};

// Returns the items in queue order, or an empty vector if the passes do not
// describe a consistent dependency chain (then the plan runs pass by pass).
// QLAG (0: QC) sets the lag, in tiles per CTA, between a key's completion
// and its dependent tiles separately from the chunk size.
inline std::vector<QOrderItem> queue_order(const std::vector<QOrderPass>& ps, int64_t G,
                                           int64_t QC, int64_t QLAG = 0) {
  struct Grp {
    size_t first = 0;
    int nl = 0;
    std::vector<int64_t> em;                   // tiles queued per level
    std::vector<std::vector<int64_t>> keypos;  // [l][k]: position completing key k of level l + 1
  };
  std::vector<Grp> grps;
  int64_t total = 0;
  for (size_t i = 0; i < ps.size();) {
    size_t j = i;
    while (j < ps.size() && ps[j].grp == ps[i].grp) ++j;
    Grp g;
    g.first = i;
    g.nl = (int)(j - i);
    g.em.assign(g.nl, 0);
    g.keypos.resize(g.nl);
    grps.push_back(g);
    for (size_t k = i; k < j; ++k) {
      if (ps[k].ntiles < 0 || ps[k].col_blocks < 1 || ps[k].sig_mul < 1 || ps[k].sig_div < 1)
        return {};
      if (k > i && ps[k].ntiles > 0 && ps[k].keys < 1) return {};
      total += ps[k].ntiles;
    }
    i = j;
  }
  const int64_t lag = std::max<int64_t>(1, (QLAG > 0 ? QLAG : QC) * G);
  std::vector<QOrderItem> out;
  out.reserve((size_t)total);
  auto emit = [&](Grp& g, int l) {
    const int64_t t = g.em[l]++;
    out.push_back({(uint32_t)(g.first + l), (uint32_t)t});
    if (l + 1 < g.nl) {
      const QOrderPass& P = ps[g.first + l];
      const QOrderPass& Q = ps[g.first + l + 1];
      const int64_t done = g.em[l] == P.ntiles
                               ? Q.keys
                               : std::min(Q.keys, (t + 1) * P.sig_mul / P.sig_div);
      while ((int64_t)g.keypos[l].size() < done) g.keypos[l].push_back((int64_t)out.size() - 1);
    }
  };
  size_t feed = 0;  // first group whose first pass has tiles left
  bool flush = false;
  while ((int64_t)out.size() < total) {
    bool any = false;
    for (int64_t c = 0; c < QC * G && feed < grps.size();) {
      Grp& g = grps[feed];
      if (g.em[0] == ps[g.first].ntiles) {
        ++feed;
        continue;
      }
      emit(g, 0);
      ++c;
      any = true;
    }
    const size_t started = std::min(feed + 1, grps.size());
    for (size_t gi = 0; gi < started; ++gi) {
      Grp& g = grps[gi];
      for (int l = 1; l < g.nl; ++l) {
        const QOrderPass& Q = ps[g.first + l];
        while (g.em[l] < Q.ntiles) {
          const int64_t key = g.em[l] / Q.col_blocks;
          if (key >= (int64_t)g.keypos[l - 1].size()) break;
          if (!flush && g.keypos[l - 1][key] + lag > (int64_t)out.size()) break;
          emit(g, l);
          any = true;
        }
      }
    }
    if (!any) {
      if (flush) return {};  // a key that no tile completes
      flush = true;
    }
  }
  return out;
}

}  // namespace mcfft
