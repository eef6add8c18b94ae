// layout.cpp -- see layout.h.
#include "layout.h"

#include <algorithm>
#include <cstdlib>
#include <cstdio>
#include <functional>
#include <map>
#include <set>
#include <sstream>
#include <thread>

namespace mcfft {
namespace layout {

namespace {

int ilog2(int64_t x) {
  int r = 0;
  while ((int64_t(1) << r) < x) ++r;
  return r;
}

int swz_for(int row_bytes) {
  return row_bytes >= 128 ? 7 : row_bytes == 64 ? 3 : row_bytes == 32 ? 1 : 0;
}

// Bit ids: v bit j -> j, c bit j -> 64 + j.
constexpr int kC = 64;

struct RowMap {
  std::vector<int> src;  // r bit i <- source bit id src[i]
  std::vector<uint32_t> tv, tc;  // contributions of v and of c (disjoint bits)
  uint32_t apply(uint32_t v, uint32_t c) const { return tv[v] | tc[c]; }
};

RowMap make_rowmap(const std::vector<int>& low, int b, int g) {
  RowMap m;
  std::set<int> used(low.begin(), low.end());
  m.src = low;
  for (int j = 0; j < g; ++j)
    if (!used.count(kC + j)) m.src.push_back(kC + j);
  for (int j = 0; j < b; ++j)
    if (!used.count(j)) m.src.push_back(j);
  m.tv.assign((size_t)1 << b, 0);
  m.tc.assign((size_t)1 << g, 0);
  for (size_t i = 0; i < m.src.size(); ++i) {
    const int s = m.src[i];
    if (s >= kC) {
      for (uint32_t c = 0; c < m.tc.size(); ++c) m.tc[c] |= ((c >> (s - kC)) & 1u) << i;
    } else if (s < b) {
      for (uint32_t v = 0; v < m.tv.size(); ++v) m.tv[v] |= ((v >> s) & 1u) << i;
    }
  }
  return m;
}

// ---- bank-conflict model --------------------------------------------------
// Wavefronts of one warp-wide shared-memory access.  16-byte accesses are
// served per quarter-warp (8 lanes); within a group, lanes touching the same
// 16-byte bank group at different addresses serialise.  4-byte accesses:
// all 32 lanes; distinct words in one bank serialise.
double wavefronts(const std::vector<uint32_t>& addr, int bytes) {
  if (bytes == 16) {
    double w = 0;
    for (size_t p = 0; p < addr.size(); p += 8) {
      uint32_t seen[8][8];
      int cnt[8] = {0};
      int m = 0;
      for (size_t i = p; i < std::min(addr.size(), p + 8); ++i) {
        const int g = (addr[i] >> 4) & 7;
        const uint32_t a = addr[i] >> 4;
        bool dup = false;
        for (int k = 0; k < cnt[g]; ++k) dup |= seen[g][k] == a;
        if (!dup) seen[g][cnt[g]++] = a;
        m = std::max(m, cnt[g]);
      }
      w += m;
    }
    return w;
  }
  uint32_t seen[32][32];
  int cnt[32] = {0};
  int m = 0;
  for (uint32_t a : addr) {
    const int g = (a >> 2) & 31;
    const uint32_t wd = a >> 2;
    bool dup = false;
    for (int k = 0; k < cnt[g]; ++k) dup |= seen[g][k] == wd;
    if (!dup && cnt[g] < 32) seen[g][cnt[g]++] = wd;
    m = std::max(m, cnt[g]);
  }
  return m;
}
double ideal_wavefronts(size_t lanes, int bytes) {
  return bytes == 16 ? (double)((lanes + 7) / 8) : 1.0;
}

}  // namespace

uint32_t Staging::offset(uint32_t pos, uint32_t c) const {
  uint32_t raw;
  if (kind == ROW) {
    raw = ((pos / E) * C + c) * row_bytes + (pos % E) * elem;
  } else {
    uint32_t prow = pos;
    if (pmid >= 0) {
      const uint32_t lo = pos & ((1u << pmid) - 1u), mid = (pos >> pmid) & 7u;
      prow = mid | (lo << 3) | ((pos >> (pmid + 3)) << (pmid + 3));
    }
    raw = ((c / E) * L + prow) * row_bytes + (c % E) * elem;
  }
  return raw ^ (((raw >> 7) & swz) << 4);
}

namespace {
Staging make_staging_sw(Kind kind, int L, int C, int elem, int64_t sp, int64_t sc, int64_t so,
                        int64_t ncols, int64_t nouter, int pmid);
}  // namespace

Staging make_staging(Kind kind, int L, int C, int elem, int64_t sp, int64_t sc, int64_t so,
                     int64_t ncols, int64_t nouter, int pmid, bool noswz) {
  Staging s = make_staging_sw(kind, L, C, elem, sp, sc, so, ncols, nouter, pmid);
  if (noswz) s.swz = 0;
  return s;
}

namespace {
Staging make_staging_sw(Kind kind, int L, int C, int elem, int64_t sp, int64_t sc, int64_t so,
                        int64_t ncols, int64_t nouter, int pmid) {
  Staging s;
  s.kind = kind;
  s.L = L;
  s.C = C;
  s.elem = elem;
  const int per_row = 128 / elem;
  if (kind == COL && pmid >= 1 && C > per_row) {
    // Permuted point order with C / E > 1 column groups of E = 128 / elem
    // (t = lg L - 3, so that the point bits above t + 3 are empty and the
    // box fits five dims): column-low, point bits [t, t+3), [0, t),
    // column-high, outer.
    s.pmid = pmid;
    s.E = per_row;
    s.row_bytes = 128;
    s.swz = swz_for(s.row_bytes);
    const uint64_t nlo = uint64_t(1) << pmid;
    s.ndims = 5;
    s.gdim[0] = (uint64_t)s.E;             s.box[0] = (uint32_t)s.E;
    s.gdim[1] = 8;                         s.box[1] = 8;              s.gstride_bytes[1] = nlo * sp * elem;
    s.gdim[2] = nlo;                       s.box[2] = (uint32_t)nlo;  s.gstride_bytes[2] = (uint64_t)sp * elem;
    s.gdim[3] = (uint64_t)(ncols / s.E);   s.box[3] = (uint32_t)(C / s.E); s.gstride_bytes[3] = (uint64_t)s.E * elem;
    s.gdim[4] = (uint64_t)nouter;          s.box[4] = 1;              s.gstride_bytes[4] = (uint64_t)so * elem;
    s.cmul[3] = C / s.E;
    s.omul[4] = 1;
    if (nouter <= 1) s.ndims = 4;
    return s;
  }
  if (kind == COL && pmid >= 1) {
    // Permuted point order (see Staging::pmid): all C columns in one
    // shared-memory row; dims columns, point bits [t, t+3), [0, t), the
    // rest, outer.  The column block is the innermost coordinate (cb * C).
    s.pmid = pmid;
    s.E = C;
    s.row_bytes = C * elem;
    s.swz = swz_for(s.row_bytes);
    const uint64_t nlo = uint64_t(1) << pmid, nhi = (uint64_t)L >> (pmid + 3);
    s.ndims = 5;
    s.gdim[0] = (uint64_t)ncols;  s.box[0] = (uint32_t)C;
    s.gdim[1] = 8;                s.box[1] = 8;                 s.gstride_bytes[1] = nlo * sp * elem;
    s.gdim[2] = nlo;              s.box[2] = (uint32_t)nlo;     s.gstride_bytes[2] = (uint64_t)sp * elem;
    s.gdim[3] = nhi;              s.box[3] = (uint32_t)nhi;     s.gstride_bytes[3] = 8 * nlo * sp * elem;
    s.gdim[4] = (uint64_t)nouter; s.box[4] = 1;                 s.gstride_bytes[4] = (uint64_t)so * elem;
    s.cmul[0] = C;
    s.omul[4] = 1;
    if (nouter <= 1) s.ndims = 4;
    return s;
  }
  if (kind == ROW) {
    s.E = std::min(L, per_row);
    s.row_bytes = s.E * elem;
    s.swz = swz_for(s.row_bytes);
    // dims: point-low (E), column, point-high (L/E), outer
    s.ndims = 4;
    s.gdim[0] = (uint64_t)s.E;            s.box[0] = (uint32_t)s.E;
    s.gdim[1] = (uint64_t)ncols;          s.box[1] = (uint32_t)C;  s.gstride_bytes[1] = (uint64_t)sc * elem;
    s.gdim[2] = (uint64_t)(L / s.E);      s.box[2] = (uint32_t)(L / s.E); s.gstride_bytes[2] = (uint64_t)s.E * sp * elem;
    s.gdim[3] = (uint64_t)nouter;         s.box[3] = 1;            s.gstride_bytes[3] = (uint64_t)so * elem;
    s.cmul[1] = C;
    s.omul[3] = 1;
    if (nouter <= 1) s.ndims = 3;
  } else {
    s.E = std::min(C, per_row);
    s.row_bytes = s.E * elem;
    s.swz = swz_for(s.row_bytes);
    const int plo = std::min(L, 256), phi = L / plo;
    // dims: column-low (E), point-low, point-high, column-high, outer
    s.ndims = 5;
    s.gdim[0] = (uint64_t)s.E;             s.box[0] = (uint32_t)s.E;
    s.gdim[1] = (uint64_t)plo;             s.box[1] = (uint32_t)plo; s.gstride_bytes[1] = (uint64_t)sp * elem;
    s.gdim[2] = (uint64_t)phi;             s.box[2] = (uint32_t)phi; s.gstride_bytes[2] = (uint64_t)plo * sp * elem;
    s.gdim[3] = (uint64_t)(ncols / s.E);   s.box[3] = (uint32_t)(C / s.E); s.gstride_bytes[3] = (uint64_t)s.E * elem;
    s.gdim[4] = (uint64_t)nouter;          s.box[4] = 1;             s.gstride_bytes[4] = (uint64_t)so * elem;
    // A pass with fewer columns than C loads and stores only its own column
    // blocks (the outermost shared-memory dimension); the tile's other
    // columns hold stale data that is transformed but never stored.
    if ((int64_t)s.box[3] > (int64_t)s.gdim[3]) s.box[3] = (uint32_t)s.gdim[3];
    s.cmul[3] = C / s.E;
    s.omul[4] = 1;
    if (nouter <= 1) s.ndims = 4;
  }
  return s;
}
}  // namespace

namespace {

// Host threads for the layout search (MCFFT_LAYOUT_THREADS overrides; 1
// searches on the calling thread only).
size_t search_threads() {
  static const size_t n = [] {
    if (const char* e = std::getenv("MCFFT_LAYOUT_THREADS")) return (size_t)std::max(1, std::atoi(e));
    const unsigned h = std::thread::hardware_concurrency();
    return (size_t)std::min(16u, std::max(1u, h));
  }();
  return n;
}

// Runs fn(i) for i in [0, n) on the search threads.
template <class F>
void parallel_for(size_t n, F fn) {
  const size_t nthr = std::min(search_threads(), n);
  if (nthr <= 1) {
    for (size_t i = 0; i < n; ++i) fn(i);
    return;
  }
  auto work = [&](size_t t) {
    for (size_t i = t; i < n; i += nthr) fn(i);
  };
  std::vector<std::thread> pool;
  for (size_t t = 1; t < nthr; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
}

struct Ctx {
  PassLayout* pl;
  int b, g, rb;
};

// Epilogue of stage s with row maps m[s], m[s+1] (or the output staging for
// the last stage).  Fills tables if `fill`; returns excess wavefronts.
double eval_epilogue(const Ctx& x, const std::vector<RowMap>& m, int s, bool fill,
                     std::vector<uint32_t>* tab, std::vector<uint32_t>* kofs, bool* linear) {
  PassLayout& p = *x.pl;
  const uint32_t P = (uint32_t)p.R << (4 * s);
  const bool last = s == p.NST - 1;
  // row -> (v, c)
  std::vector<uint32_t> rv(p.NROWS), rc(p.NROWS);
  for (int v = 0; v < p.NV; ++v)
    for (int c = 0; c < p.C; ++c) {
      uint32_t r = m[s].apply(v, c);
      rv[r] = v;
      rc[r] = c;
    }
  std::vector<uint32_t> ofs(16);
  double w = 0, ideal = 0;
  std::vector<uint32_t> base(p.NROWS);
  for (int r = 0; r < p.NROWS; ++r) {
    const uint32_t v = rv[r], c = rc[r];
    for (int k = 0; k < 16; ++k) {
      uint32_t d;
      if (!last) {
        const uint32_t K = v % P, Rp = v / P;
        const uint32_t pos1 = K + P * (k + 16 * Rp);
        const uint32_t n1 = pos1 / p.NV, v1 = pos1 % p.NV;
        d = a_offset(m[s + 1].apply(v1, c), n1);
      } else {
        d = p.out.offset(v + p.NV * k, c);
      }
      if (k == 0) base[r] = d;
      const uint32_t o = d ^ base[r];
      if (r == 0) ofs[k] = o;
      else if (ofs[k] != o && linear) *linear = false;
    }
  }
  // conflicts: warps = 32 consecutive rows, one store per k
  const int bytes = last ? p.out.elem : 4;
  const int wstep = fill ? 32 : 32 * std::max(1, p.NROWS / 256);  // sample warps while searching
  for (int r0 = 0; r0 < p.NROWS; r0 += wstep) {
    for (int k = 0; k < 16; ++k) {
      std::vector<uint32_t> a;
      for (int l = 0; l < 32 && r0 + l < p.NROWS; ++l) a.push_back(base[r0 + l] ^ ofs[k]);
      if (bytes == 8) {
        // 64-bit stores: two half-warp phases
        std::vector<uint32_t> lo(a.begin(), a.begin() + std::min<size_t>(16, a.size()));
        std::vector<uint32_t> hi(a.begin() + std::min<size_t>(16, a.size()), a.end());
        auto w64 = [](const std::vector<uint32_t>& aa) {
          std::map<int, std::set<uint32_t>> gg;
          for (uint32_t q : aa) { gg[(q >> 2) & 31].insert(q >> 3); gg[((q >> 2) + 1) & 31].insert(q >> 3); }
          size_t mm = 0;
          for (auto& kv : gg) mm = std::max(mm, kv.second.size());
          return (double)mm;
        };
        w += w64(lo) + w64(hi);
        ideal += 2;
      } else {
        w += wavefronts(a, 4);
        ideal += 1;
      }
    }
  }
  if (fill) {
    for (int r = 0; r < p.NROWS; ++r) {
      const uint32_t v = rv[r], c = rc[r];
      uint32_t aux = last ? v * p.C + c : v / P;
      (*tab)[(size_t)s * p.NROWS + r] = (base[r] >> 2) | (aux << 16);
    }
    for (int k = 0; k < 16; ++k) (*kofs)[(size_t)s * 16 + k] = ofs[k];
  }
  return w / ideal - 1.0;
}

// Prologue: items and their lane order.  `lanebits` lists the item-index
// bits that vary fastest (the lanes of a warp), as ids into the item
// coordinate bits.  Returns excess wavefronts; fills tables if `fill`.
struct ItemSpace {
  // coordinate fields of an item: (name, nbits)
  std::vector<std::pair<char, int>> fields;
};

double eval_prologue(const Ctx& x, const RowMap& m0, const std::vector<int>& order, bool fill,
                     bool* linear) {
  PassLayout& p = *x.pl;
  // item coordinate bits: ROW R=1: c(g), w(b-2), q(2); COL R=1: v(b), cg(g-2), q(2)
  // ROW R>1: c(g), w(log2(NVR)-2); COL R>1: vr(log2 NVR), cg(g-2)
  const int NVR = p.L / p.R;
  const int lnvr = ilog2(NVR);
  std::vector<int> widths;  // field widths in order: f0, f1, f2
  if (p.R == 1) {
    if (p.in_kind == ROW) widths = {x.g, x.b - 2, 2};
    else widths = {x.b, x.g - 2, 2};
  } else {
    if (p.in_kind == ROW) widths = {x.g, lnvr - 2, 0};
    else widths = {lnvr, x.g - 2, 0};
  }
  int nbits = widths[0] + widths[1] + widths[2];
  const int nitems = 1 << nbits;
  // order: permutation of item-coordinate bit ids (0..nbits-1), giving item
  // index bit i <- coordinate bit order[i]
  auto coords = [&](uint32_t idx, uint32_t* f) {
    uint32_t cbits = 0;
    for (int i = 0; i < nbits; ++i) cbits |= ((idx >> i) & 1u) << order[i];
    f[0] = cbits & ((1u << widths[0]) - 1);
    f[1] = (cbits >> widths[0]) & ((1u << widths[1]) - 1);
    f[2] = (cbits >> (widths[0] + widths[1])) & ((1u << widths[2]) - 1);
  };
  // A 16-byte load covers 4 FP16 or 2 FP32 complex points: with FP32
  // staging each point group of an item takes two loads (halves h = 0, 1,
  // the second two points / columns), and load index j = group * nh + h.
  const int nh = p.in.elem == 8 ? 2 : 1;
  const int nl = (p.R == 1 ? 4 : p.R) * nh;     // loads per item
  const int ns = p.R == 1 ? 4 : 4 * p.R;        // stores per item
  const int sbytes = p.R == 1 ? 16 : 4;
  std::vector<uint32_t> lb(nitems), sb(nitems), tw(nitems);
  std::vector<uint32_t> lofs(nl), sofs(ns);
  std::vector<uint32_t> la((size_t)nitems * nl), sa((size_t)nitems * ns);
  const int istep = fill ? 32 : 32 * std::max(1, nitems / 256);  // sample warps while searching
  for (int it = 0; it < nitems; ++it) {
    if (!fill && (it % istep) >= 32) continue;
    uint32_t f[3];
    coords(it, f);
    for (int j = 0; j < nl; ++j) {
      const uint32_t jg = j / nh, h2 = 2 * (j % nh);
      uint32_t pos, c;
      if (p.R == 1) {
        if (p.in_kind == ROW) { c = f[0]; pos = (4 * f[2] + jg) * p.NV + 4 * f[1] + h2; }
        else { c = 4 * f[1] + h2; pos = (4 * f[2] + jg) * p.NV + f[0]; }
      } else {
        if (p.in_kind == ROW) { c = f[0]; pos = jg * NVR + 4 * f[1] + h2; }
        else { c = 4 * f[1] + h2; pos = jg * NVR + f[0]; }
      }
      la[(size_t)it * nl + j] = p.in.offset(pos, c);
    }
    for (int j = 0; j < ns; ++j) {
      uint32_t d;
      if (p.R == 1) {
        uint32_t v, c;
        if (p.in_kind == ROW) { c = f[0]; v = 4 * f[1] + j; }
        else { c = 4 * f[1] + j; v = f[0]; }
        d = a_offset(m0.apply(v, c), 4 * f[2]);
      } else {
        const int jj = j / p.R, k = j % p.R;
        uint32_t vr, c;
        if (p.in_kind == ROW) { c = f[0]; vr = 4 * f[1] + jj; }
        else { c = 4 * f[1] + jj; vr = f[0]; }
        const uint32_t pos1 = k + p.R * vr;
        d = a_offset(m0.apply(pos1 % p.NV, c), pos1 / p.NV);
      }
      sa[(size_t)it * ns + j] = d;
    }
    lb[it] = la[(size_t)it * nl];
    sb[it] = sa[(size_t)it * ns];
    tw[it] = p.R == 1 ? 0
             : p.in_kind == ROW ? 4 * f[1]
                                : (tail_row(f[0], std::max(p.in.pmid, 0)) | 0x80000000u);
    if (fill) {
      for (int j = 0; j < nl; ++j) {
        uint32_t o = la[(size_t)it * nl + j] ^ lb[it];
        if (it == 0) lofs[j] = o;
        else if (o != lofs[j] && linear) *linear = false;
      }
      for (int j = 0; j < ns; ++j) {
        uint32_t o = sa[(size_t)it * ns + j] ^ sb[it];
        if (it == 0) sofs[j] = o;
        else if (o != sofs[j] && linear) *linear = false;
      }
    }
  }
  double w = 0, ideal = 0;
  for (int i0 = 0; i0 < nitems; i0 += istep) {
    const int n = std::min(32, nitems - i0);
    for (int j = 0; j < nl; ++j) {
      std::vector<uint32_t> a;
      for (int l = 0; l < n; ++l) a.push_back(la[(size_t)(i0 + l) * nl + j]);
      w += wavefronts(a, 16);
      ideal += ideal_wavefronts(a.size(), 16);
    }
    for (int j = 0; j < ns; ++j) {
      std::vector<uint32_t> a;
      for (int l = 0; l < n; ++l) a.push_back(sa[(size_t)(i0 + l) * ns + j]);
      w += wavefronts(a, sbytes);
      ideal += ideal_wavefronts(a.size(), sbytes);
    }
  }
  if (fill) {
    p.items = nitems;
    p.item_loads = nl;
    p.item_stores = ns;
    p.item_tab.assign((size_t)nitems * 2, 0);
    for (int it = 0; it < nitems; ++it) {
      p.item_tab[2 * it] = (lb[it] >> 2) | ((sb[it] >> 2) << 16);
      p.item_tab[2 * it + 1] = tw[it];
    }
    p.lofs = lofs;
    p.sofs = sofs;
  }
  return w / ideal - 1.0;
}

}  // namespace

std::string PassLayout::describe() const {
  std::ostringstream o;
  o << "L=" << L << " R=" << R << " C=" << C << " NST=" << NST << " in=" << (in_kind == ROW ? "row" : "col")
    << " out=" << (out_kind == ROW ? "row" : "col") << " excess(prologue)=" << prologue_excess
    << " excess(epilogue)=" << epilogue_excess;
  return o.str();
}

bool build(PassLayout* pl, int L, int R, int C, Kind in_kind, Kind out_kind, int in_elem,
           int out_elem, int64_t in_sp, int64_t in_sc, int64_t in_so, int64_t out_sp,
           int64_t out_sc, int64_t out_so, int64_t ncols, int64_t nouter, std::string* err,
           int unsw) {
  PassLayout& p = *pl;
  p = PassLayout();
  p.L = L; p.R = R; p.C = C;
  p.NV = L / 16;
  p.NROWS = p.NV * C;
  p.in_kind = in_kind; p.out_kind = out_kind;
  int nst = 0;
  for (int t = L / R; t > 1; t >>= 4) ++nst;
  p.NST = nst;
  if ((1 << (4 * nst)) * R != L || nst < 1) { *err = "L is not 16^a * R"; return false; }
  // Column staging puts min(C, 128 / elem) columns innermost in its TMA box,
  // which must span 16 bytes: C >= 4 for FP16.  Row staging's innermost box
  // dimension is points (128 bytes), so a row-in / row-out pass also takes
  // two columns (L = 4096 in 8K-point tiles), and so does a row-in pass
  // whose column output is FP32 (two columns: 16 bytes).  Column input
  // keeps four columns.
  const int cmin = in_kind == ROW && (out_kind == ROW || 2 * out_elem >= 16) ? 2 : 4;
  if (C < cmin || (C & (C - 1))) {
    *err = "C must be a power of two >= 4 (>= 2 for row passes)";
    return false;
  }
  if (in_kind == COL && (ncols % std::min(C, 128 / in_elem))) { *err = "ncols"; return false; }
  if (out_kind == COL && (ncols % std::min(C, 128 / out_elem))) { *err = "ncols"; return false; }
  p.in = make_staging(in_kind, L, C, in_elem, in_sp, in_sc, in_so, ncols, nouter, -1,
                      (unsw & 1) != 0);
  p.out = make_staging(out_kind, L, C, out_elem, out_sp, out_sc, out_so, ncols, nouter, -1,
                       (unsw & 2) != 0);
  Ctx x{pl, ilog2(p.NV), ilog2(C), ilog2(R)};

  // Candidate bit ids for the low row bits.
  std::vector<int> cand;
  for (int j = 0; j < x.g; ++j) cand.push_back(kC + j);
  for (int j = 0; j < x.b; ++j) cand.push_back(j);
  const int top0 = x.b - 4, top1 = x.b - 3;

  // Non-last stage maps: [X0, X1, X2, T0, T1]; last: [Y0..Y4].
  std::vector<std::vector<int>> xs, ys;
  auto combos3 = [&](std::vector<std::vector<int>>* out, const std::vector<int>& pool) {
    for (size_t a = 0; a < pool.size(); ++a)
      for (size_t b = 0; b < pool.size(); ++b)
        for (size_t c = 0; c < pool.size(); ++c)
          if (a != b && b != c && a != c && b < c) out->push_back({pool[a], pool[b], pool[c]});
  };
  {
    std::vector<int> pool;
    for (int id : cand)
      if (x.b < 4 || (id != top0 && id != top1)) pool.push_back(id);
    if (pool.size() > 12) pool.resize(12);
    combos3(&xs, pool);
    if (xs.empty()) xs.push_back({});
  }
  {
    // last-stage low bits: 5 bits from a small pool (c bits and low v bits)
    std::vector<int> pool;
    for (int j = 0; j < std::min(x.g, 7); ++j) pool.push_back(kC + j);
    for (int j = 0; j < std::min(x.b, 5); ++j) pool.push_back(j);
    std::vector<std::vector<int>> cands;
    const int n = (int)pool.size();
    for (int m = 0; m < (1 << n); ++m) {
      if (__builtin_popcount(m) != 5) continue;
      std::vector<int> y;
      for (int i = 0; i < n; ++i)
        if (m >> i & 1) y.push_back(pool[i]);
      // the bit placed at r bit 0 matters for the bank: try each member first
      for (int f = 0; f < 5; ++f) {
        std::vector<int> yy = y;
        std::swap(yy[0], yy[f]);
        cands.push_back(yy);
      }
    }
    ys = cands;
    if (ys.empty()) ys.push_back({});
  }

  auto lowbits_nonlast = [&](const std::vector<int>& X) {
    std::vector<int> low = X;
    if (x.b >= 4) { low.push_back(top0); low.push_back(top1); }
    return low;
  };

  // Search.  The epilogue cost of stage s depends on maps[s] and maps[s+1];
  // non-last stages share one low-bit choice X, the last stage uses Y.
  // Rank X by the cost of stages 0..NST-3, Y by the last stage, then try
  // the best pairs on stage NST-2.
  auto maps_for = [&](const std::vector<int>& X, const std::vector<int>& Y,
                      std::vector<RowMap>* maps) {
    maps->assign(nst, RowMap());
    for (int s = 0; s < nst; ++s) {
      std::vector<int> low = (s == nst - 1) ? Y : lowbits_nonlast(X);
      std::set<int> u(low.begin(), low.end());
      if (u.size() != low.size()) return false;
      (*maps)[s] = make_rowmap(low, x.b, x.g);
      if ((int)(*maps)[s].src.size() != x.b + x.g) return false;
    }
    return true;
  };
  std::vector<std::pair<double, int>> xr, yr;
  const std::vector<int> ydef = ys[0];
  int xzero = 0, yzero = 0;
  // Column input that can use a permuted staging (below) needs more
  // choices for the bits of A row 0..2: the prologue's stores decide among
  // the epilogue-optimal maps.
  // (all C columns in one 128-byte row, or, for R = 1, groups of them with
  // t = lg L - 3)
  const bool permutable =
      in_kind == COL && ncols >= C && ilog2(L) >= 4 && (C * in_elem <= 128 || R == 1);
  const int xcap = permutable ? 64 : 12, ycap = permutable ? 8 : 24;
  for (int ix = 0; ix < (nst > 1 ? (int)xs.size() : 1) && xzero < xcap; ++ix) {
    std::vector<RowMap> maps;
    if (!maps_for(xs[ix], ydef, &maps)) { if (nst > 2) continue; }
    double c = 0;
    bool lin = true;
    if (nst > 2) {
      for (int s = 0; s < nst - 2; ++s) c += eval_epilogue(x, maps, s, false, nullptr, nullptr, &lin);
      if (!lin) continue;
    }
    xr.push_back({c, ix});
    if (c < 1e-9) ++xzero;
  }
  // last-stage candidates, evaluated in chunks in parallel and taken in
  // order until 24 conflict-free ones are found (as a sequential scan would)
  for (size_t c0 = 0; c0 < ys.size() && yzero < 24; c0 += 64) {
    const size_t cn = std::min<size_t>(64, ys.size() - c0);
    std::vector<double> cost(cn, 0.0);
    std::vector<char> ok(cn, 0);
    parallel_for(cn, [&](size_t k) {
      std::vector<RowMap> maps;
      if (!maps_for(xs.empty() ? std::vector<int>{} : xs[0], ys[c0 + k], &maps)) return;
      bool lin = true;
      cost[k] = eval_epilogue(x, maps, nst - 1, false, nullptr, nullptr, &lin);
      ok[k] = lin;
    });
    for (size_t k = 0; k < cn && yzero < 24; ++k) {
      if (!ok[k]) continue;
      yr.push_back({cost[k], (int)(c0 + k)});
      if (cost[k] < 1e-9) ++yzero;
    }
  }
  std::sort(xr.begin(), xr.end());
  std::sort(yr.begin(), yr.end());
  struct Cand { double cost; std::vector<RowMap> maps; };
  std::vector<Cand> cands;
  {
    const size_t ni = std::min<size_t>(xr.size(), xcap), nj = std::min<size_t>(yr.size(), ycap);
    std::vector<Cand> all(ni * nj);
    std::vector<char> ok(ni * nj, 0);
    parallel_for(ni * nj, [&](size_t k) {
      const size_t i = k / nj, j = k % nj;
      std::vector<RowMap> maps;
      if (!maps_for(xs[xr[i].second], ys[yr[j].second], &maps)) return;
      double c = xr[i].first + yr[j].first;
      bool lin = true;
      if (nst > 1) c += eval_epilogue(x, maps, nst - 2, false, nullptr, nullptr, &lin);
      if (!lin) return;
      all[k] = {c, maps};
      ok[k] = 1;
    });
    for (size_t k = 0; k < ni * nj; ++k)
      if (ok[k]) cands.push_back(std::move(all[k]));
  }
  if (cands.empty()) { *err = "no linear row map"; return false; }
  std::stable_sort(cands.begin(), cands.end(),
                   [](const Cand& a, const Cand& b) { return a.cost < b.cost; });
  if (permutable) {
    // among equally good maps, alternate the source of stage 0's row bit 0
    // (what the prologue's store banks depend on most)
    std::map<int, int> seen;
    std::vector<std::pair<std::pair<double, int>, size_t>> key;
    for (size_t i = 0; i < cands.size(); ++i)
      key.push_back({{cands[i].cost, seen[cands[i].maps[0].src[0]]++}, i});
    std::stable_sort(key.begin(), key.end(), [](const auto& a, const auto& b) {
      if (a.first.first < b.first.first - 1e-9) return true;
      if (b.first.first < a.first.first - 1e-9) return false;
      return a.first.second < b.first.second;
    });
    std::vector<Cand> re;
    for (auto& k : key) re.push_back(cands[k.second]);
    cands.swap(re);
  }

  // Prologue item order for the best few row-map candidates: 5 lane bits
  // among the item-coordinate bits (first three = one 8-lane phase).
  const int lnvr = ilog2(L / R);
  int nb;
  if (R == 1) nb = (in_kind == ROW) ? x.g + (x.b - 2) + 2 : x.b + (x.g - 2) + 2;
  else nb = (in_kind == ROW) ? x.g + (lnvr - 2) : lnvr + (x.g - 2);
  const int nl = std::min(5, nb);
  // Lane-bit pool: the low three and the top four bits of every item field
  // (low bits pick bank groups in staging, top bits pick K positions).
  std::vector<int> lane_pool;
  {
    std::vector<int> widths;
    if (R == 1) widths = (in_kind == ROW) ? std::vector<int>{x.g, x.b - 2, 2}
                                          : std::vector<int>{x.b, x.g - 2, 2};
    else widths = (in_kind == ROW) ? std::vector<int>{x.g, lnvr - 2} : std::vector<int>{lnvr, x.g - 2};
    int off = 0;
    for (int w : widths) {
      for (int i = 0; i < w; ++i)
        if (i < 3 || i >= w - 4) lane_pool.push_back(off + i);
      off += w;
    }
  }
  // Input staging candidates: for column input whose C columns fit one
  // shared-memory row (and a pass at least C columns wide) first the
  // permuted order that brings point bits [t, t+3) to the bank-selecting
  // row bits, t = lg(L/R) - 4 -- the A stores of an item are conflict-free
  // when the lanes differ in the stage-0 K position, point bits
  // [lg(L/R) - 4, lg(L/R)), which the natural order leaves out of the load
  // banks -- then, unless that layout is conflict-free, the natural order,
  // which wins ties.
  std::vector<int> pmids = {-1};
  const int tstar = C * in_elem <= 128 ? ilog2(L / R) - 4 : ilog2(L) - 3;
  if (permutable && tstar >= 1 && tstar <= ilog2(L) - 3) pmids.insert(pmids.begin(), tstar);
  double total_best = 1e30;
  std::vector<int> porder_best;
  std::vector<RowMap> maps_best;
  Staging in_best = p.in;
  const int epi_weight = 16 * nst;  // epilogue instructions per row-warp vs prologue per item-warp
  for (int pm : pmids) {
    if (total_best <= cands[0].cost * epi_weight / 16.0 + 1e-9) break;  // cannot do better
    p.in = make_staging(in_kind, L, C, in_elem, in_sp, in_sc, in_so, ncols, nouter, pm,
                        (unsw & 1) != 0);
    for (size_t ci = 0; ci < std::min<size_t>(cands.size(), permutable ? 32 : 4); ++ci) {
      if (ci > 0 && cands[ci].cost > cands[0].cost + 1e-9) break;
      if (total_best <= cands[0].cost * epi_weight / 16.0 + 1e-9) break;  // found the optimum
      // Candidate item orders: 5 lane bits from the pool (which 3 of them
      // form the 8-lane phase), the other bits after them; evaluated in
      // chunks on the host's threads and taken in enumeration order (the
      // first of the cheapest wins; a conflict-free order ends the search),
      // so the result does not depend on the thread count.
      std::vector<std::vector<int>> orders;
      {
        std::vector<int> comb(nl);
        std::function<void(int, int)> gen = [&](int start, int depth) {
          if (depth == nl) {
            for (int m = 0; m < (1 << nl); ++m) {
              if (__builtin_popcount(m) != std::min(3, nl)) continue;
              std::vector<int> order;
              for (int i = 0; i < nl; ++i) if (m >> i & 1) order.push_back(comb[i]);
              for (int i = 0; i < nl; ++i) if (!(m >> i & 1)) order.push_back(comb[i]);
              std::set<int> u(order.begin(), order.end());
              for (int i = 0; i < nb; ++i)
                if (!u.count(i)) order.push_back(i);
              orders.push_back(order);
            }
            return;
          }
          for (size_t i = start; i < lane_pool.size(); ++i) {
            comb[depth] = lane_pool[i];
            gen((int)i + 1, depth + 1);
          }
        };
        gen(0, 0);
      }
      double pbest = 1e30;
      std::vector<int> porder;
      const size_t nthr = search_threads();
      const size_t chunk = 32 * nthr;
      std::vector<double> cost(chunk);
      std::vector<char> lin(chunk);
      for (size_t c0 = 0; c0 < orders.size() && pbest > 1e-9; c0 += chunk) {
        const size_t cn = std::min(chunk, orders.size() - c0);
        auto work = [&](size_t t) {
          for (size_t i = t; i < cn; i += nthr) {
            bool l = true;
            cost[i] = eval_prologue(x, cands[ci].maps[0], orders[c0 + i], false, &l);
            lin[i] = l;
          }
        };
        std::vector<std::thread> pool;
        for (size_t t = 1; t < nthr; ++t) pool.emplace_back(work, t);
        work(0);
        for (auto& th : pool) th.join();
        for (size_t i = 0; i < cn && pbest > 1e-9; ++i)
          if (lin[i] && cost[i] < pbest - 1e-9) {
            pbest = cost[i];
            porder = orders[c0 + i];
          }
      }
      if (porder.empty()) continue;
      const double total = pbest + cands[ci].cost * epi_weight / 16.0;
      if (total < total_best - 1e-9 || (pm < 0 && total <= total_best + 1e-9)) {
        total_best = total;
        porder_best = porder;
        maps_best = cands[ci].maps;
        in_best = p.in;
      }
    }
  }
  p.in = in_best;
  p.tail_pm = (in_kind == COL && R > 1) ? std::max(p.in.pmid, 0) : -1;
  if (porder_best.empty()) { *err = "no linear prologue"; return false; }
  // Row items of R > 1: the bits above the lane bits only decide which warp
  // and which of its two items a thread gets (conflicts depend on the lane
  // bits alone).  Put a column bit on top, so that a thread's two items
  // (item indices i and i + half the items) differ only in their column and
  // read the same radix-R twiddle rows, which the kernel then loads once.
  bool paired = false;
  if (R > 1 && in_kind == ROW && nb > nl) {
    std::vector<int> high(porder_best.begin() + nl, porder_best.end());
    int pick = -1;
    for (int b : high)
      if (b < x.g) pick = b;  // field 0 = column bits
    if (pick >= 0) {
      high.erase(std::find(high.begin(), high.end(), pick));
      high.push_back(pick);
      std::copy(high.begin(), high.end(), porder_best.begin() + nl);
      paired = true;
    }
  }
  std::vector<RowMap> best_maps = maps_best;
  {
    bool lin = true;
    p.prologue_excess = eval_prologue(x, best_maps[0], porder_best, true, &lin);
    if (!lin) { *err = "prologue offsets are not XOR-linear"; return false; }
  }
  if (paired) p.tail_pm = kTailNaturalPaired;
  p.epi_tab.assign((size_t)nst * p.NROWS, 0);
  p.kofs.assign((size_t)nst * 16, 0);
  double e = 0;
  for (int s = 0; s < nst; ++s) {
    bool lin = true;
    e += eval_epilogue(x, best_maps, s, true, &p.epi_tab, &p.kofs, &lin);
    if (!lin) { *err = "epilogue offsets are not XOR-linear"; return false; }
  }
  p.epilogue_excess = e;
  p.row_v.assign(nst, std::vector<uint32_t>(p.NROWS));
  p.row_c.assign(nst, std::vector<uint32_t>(p.NROWS));
  p.row_of.assign(nst, std::vector<uint32_t>(p.NROWS));
  for (int s = 0; s < nst; ++s)
    for (int v = 0; v < p.NV; ++v)
      for (int c = 0; c < C; ++c) {
        uint32_t r = best_maps[s].apply(v, c);
        p.row_v[s][r] = v;
        p.row_c[s][r] = c;
        p.row_of[s][v * C + c] = r;
      }
  return true;
}

}  // namespace layout
}  // namespace mcfft
