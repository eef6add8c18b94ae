// Host checker of the batch queue's item order (mcfft_b200/csrc/queue_order.h)
// on synthetic plans: random mixes of single-pass groups, four-step 1D
// groups, 2D groups and 3D groups with the dependency data the plan builder
// gives them (mcfft_api.cu, link_group).  For every order it checks
//   - every (pass, tile) item appears exactly once;
//   - every later-pass tile comes after every producer tile that signals its
//     key (producer tile u signals keys [u m / d, ((u + 1) m - 1) / d]), so
//     the queue drains with all CTAs resident;
//   - a tile closer than QC G items to its last producer appears only after
//     the last first-pass tile of the plan (the final flush).
// Usage: queue_order_check <seed> <G> <QC>; prints "ok <items> <short>".
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../mcfft_b200/csrc/queue_order.h"

using mcfft::QOrderItem;
using mcfft::QOrderPass;

static int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

int main(int argc, char** argv) {
  if (argc < 4) return 2;
  const unsigned seed = (unsigned)std::atoi(argv[1]);
  const int64_t G = std::atoll(argv[2]), QC = std::atoll(argv[3]);
  std::mt19937 rng(seed);
  auto pick = [&](int lo, int hi) { return std::uniform_int_distribution<int>(lo, hi)(rng); };
  std::vector<QOrderPass> ps;
  const int ngroups = pick(1, 12);
  for (int g = 0; g < ngroups; ++g) {
    const int kind = pick(0, 3);
    const int64_t batch = 1 << pick(0, 6);
    if (kind == 0) {  // one pass, no dependency
      QOrderPass a;
      a.ntiles = batch * (1 << pick(0, 4));
      a.grp = g;
      ps.push_back(a);
    } else if (kind == 1) {  // four-step 1D: key = transform
      const int64_t cb0 = 1 << pick(0, 5), cb1 = 1 << pick(0, 5);
      QOrderPass a, b;
      a.ntiles = batch * cb0;
      a.sig_mul = 1;
      a.sig_div = cb0;
      b.ntiles = batch * cb1;
      b.col_blocks = cb1;
      b.keys = batch;
      a.grp = b.grp = g;
      ps.push_back(a);
      ps.push_back(b);
    } else if (kind == 2) {  // 2D rows (c per tile) then columns: key = 2D transform
      const int64_t nx = 1 << pick(4, 9), c = 1 << pick(2, 10), cb1 = 1 << pick(0, 4);
      QOrderPass a, b;
      a.ntiles = cdiv(nx * batch, c);
      a.sig_mul = c;
      a.sig_div = nx;
      b.ntiles = batch * cb1;
      b.col_blocks = cb1;
      b.keys = batch;
      a.grp = b.grp = g;
      ps.push_back(a);
      ps.push_back(b);
    } else {  // 3D: z rows, y columns (key = x slab), x columns (key = 3D transform)
      const int64_t nx = 1 << pick(4, 6), ny = 1 << pick(4, 6), c = 1 << pick(2, 8);
      const int64_t cb1 = 1 << pick(0, 3), cb2 = 1 << pick(0, 3);
      QOrderPass a, b, d;
      a.ntiles = cdiv(nx * ny * batch, c);
      a.sig_mul = c;
      a.sig_div = ny;
      b.ntiles = nx * batch * cb1;
      b.col_blocks = cb1;
      b.keys = nx * batch;
      b.sig_mul = 1;
      b.sig_div = cb1 * nx;
      d.ntiles = batch * cb2;
      d.col_blocks = cb2;
      d.keys = batch;
      a.grp = b.grp = d.grp = g;
      ps.push_back(a);
      ps.push_back(b);
      ps.push_back(d);
    }
  }
  const std::vector<QOrderItem> order = mcfft::queue_order(ps, G, QC);
  int64_t total = 0;
  for (const auto& p : ps) total += p.ntiles;
  if ((int64_t)order.size() != total) {
    std::printf("FAIL size %zu != %lld\n", order.size(), (long long)total);
    return 1;
  }
  std::vector<std::vector<int64_t>> pos(ps.size());
  for (size_t i = 0; i < ps.size(); ++i) pos[i].assign((size_t)ps[i].ntiles, -1);
  int64_t last_first = -1;
  for (size_t i = 0; i < order.size(); ++i) {
    const QOrderItem it = order[i];
    if (it.pass >= ps.size() || it.tile >= (uint64_t)ps[it.pass].ntiles || pos[it.pass][it.tile] >= 0) {
      std::printf("FAIL item %zu (pass %u tile %u) out of range or repeated\n", i, it.pass, it.tile);
      return 1;
    }
    pos[it.pass][it.tile] = (int64_t)i;
    if (it.pass == 0 || ps[it.pass - 1].grp != ps[it.pass].grp) last_first = (int64_t)i;
  }
  int64_t nshort = 0;
  for (size_t q = 1; q < ps.size(); ++q) {
    if (ps[q].grp != ps[q - 1].grp) continue;
    const QOrderPass& P = ps[q - 1];
    const QOrderPass& Q = ps[q];
    std::vector<int64_t> need((size_t)Q.keys, -1);  // latest producer position per key
    for (int64_t u = 0; u < P.ntiles; ++u) {
      const int64_t k0 = u * P.sig_mul / P.sig_div, k1 = ((u + 1) * P.sig_mul - 1) / P.sig_div;
      for (int64_t k = k0; k <= k1 && k < Q.keys; ++k) need[k] = std::max(need[k], pos[q - 1][u]);
    }
    for (int64_t t = 0; t < Q.ntiles; ++t) {
      const int64_t key = t / Q.col_blocks;
      if (key >= Q.keys || need[key] < 0) {
        std::printf("FAIL pass %zu tile %lld: key %lld has no producer\n", q, (long long)t,
                    (long long)key);
        return 1;
      }
      const int64_t at = pos[q][t];
      if (at <= need[key]) {
        std::printf("FAIL pass %zu tile %lld at %lld before its producer at %lld\n", q,
                    (long long)t, (long long)at, (long long)need[key]);
        return 1;
      }
      if (at - need[key] < QC * G) {
        ++nshort;
        if (at < last_first) {
          std::printf("FAIL pass %zu tile %lld at %lld only %lld after its producer, before the "
                      "last first-pass tile at %lld\n",
                      q, (long long)t, (long long)at, (long long)(at - need[key]),
                      (long long)last_first);
          return 1;
        }
      }
    }
  }
  std::printf("ok %zu %lld\n", order.size(), (long long)nshort);
  return 0;
}
