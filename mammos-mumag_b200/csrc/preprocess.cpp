// Host preprocessing of a tetrahedral mesh for the device path:
//  * node graph, reverse Cuthill-McKee order (so a warp's SELL gathers hit nearby nodes),
//  * one SELL-32 pattern shared by every node-pair operator,
//  * greedy element colouring (so the assembly scatters need no atomics),
//  * the Poisson boundary branch of scripts/matrix.py:49-64 (airbox vs spherical shell)
//    with escript's whereZero tolerance, sqrt(eps) * Lsup(arg).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>

#include "mumag_internal.h"

namespace mumag {

namespace {

struct Graph {
  std::vector<int64_t> off;
  std::vector<int32_t> adj;
};

// Runs fn(begin, end, part) over `parts` contiguous chunks of [0, n) on their own threads
// (the calling thread takes chunk 0).  Every chunk writes only its own outputs, so the
// results do not depend on the number of parts.  An exception in any chunk is rethrown on
// the calling thread after all chunks have finished.
template <class F>
void parallel_chunks(int64_t n, int parts, F&& fn) {
  if (parts <= 1 || n < 2) {
    fn(int64_t(0), n, 0);
    return;
  }
  std::vector<std::exception_ptr> err(parts);
  auto run = [&](int p) {
    try {
      fn(n * p / parts, n * (p + 1) / parts, p);
    } catch (...) {
      err[p] = std::current_exception();
    }
  };
  std::vector<std::thread> th;
  for (int p = 1; p < parts; ++p) th.emplace_back(run, p);
  run(0);
  for (auto& t : th) t.join();
  for (auto& e : err)
    if (e) std::rethrow_exception(e);
}

// Host threads for a pass over n items: one below 2^17 items, at most 16, at most the
// hardware threads and at most MUMAG_HOST_THREADS when that is set to a positive number.
int host_parts(int64_t n) {
  int64_t hw = static_cast<int64_t>(std::max(1u, std::thread::hardware_concurrency()));
  if (const char* env = std::getenv("MUMAG_HOST_THREADS")) {
    const long cap = std::strtol(env, nullptr, 10);
    if (cap > 0) hw = std::min<int64_t>(hw, cap);
  }
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>({hw, int64_t(16), n >> 16})));
}

// Undirected node graph, CSR with sorted unique neighbours.  A node is its own neighbour
// only if an element lists it twice.  Built from the node -> element incidence with a
// per-node marker, so every node's list is gathered once and only its ~14 distinct
// neighbours are sorted.
Graph node_graph(int64_t N, const int32_t* T, int64_t E) {
  std::vector<int64_t> eoff(N + 1, 0);
  for (int64_t k = 0; k < 4 * E; ++k) eoff[T[k] + 1]++;
  for (int64_t i = 0; i < N; ++i) eoff[i + 1] += eoff[i];
  std::vector<int64_t> inc(4 * E);
  {
    std::vector<int64_t> pos(eoff.begin(), eoff.end() - 1);
    for (int64_t e = 0; e < E; ++e)
      for (int a = 0; a < 4; ++a) inc[pos[T[4 * e + a]]++] = e;
  }
  // each chunk of nodes gathers its lists into its own buffer; the buffers are then joined
  const int parts = host_parts(N);
  std::vector<std::vector<int32_t>> cadj(parts);
  std::vector<std::vector<int64_t>> clen(parts);
  parallel_chunks(N, parts, [&](int64_t b, int64_t e, int p) {
    std::vector<int32_t> mark(N, -1);  // node ids fit in 32 bits (validate)
    std::vector<int32_t> nb;
    auto& out = cadj[p];
    auto& len = clen[p];
    out.reserve(static_cast<size_t>(eoff[e] - eoff[b]) / 2);
    len.reserve(e - b);
    for (int64_t i = b; i < e; ++i) {
      nb.clear();
      mark[i] = static_cast<int32_t>(i);  // the node itself, unless an element repeats it
      for (int64_t k = eoff[i]; k < eoff[i + 1]; ++k) {
        const int32_t* t = T + 4 * inc[k];
        int self = 0;
        for (int a = 0; a < 4; ++a) {
          const int32_t j = t[a];
          if (j == i) {
            ++self;
          } else if (mark[j] != i) {
            mark[j] = static_cast<int32_t>(i);
            nb.push_back(j);
          }
        }
        if (self > 1 && mark[i] == i) {
          mark[i] = -2;  // listed twice: a self loop, once
          nb.push_back(static_cast<int32_t>(i));
        }
      }
      std::sort(nb.begin(), nb.end());
      out.insert(out.end(), nb.begin(), nb.end());
      len.push_back(static_cast<int64_t>(nb.size()));
    }
  });
  Graph g;
  g.off.assign(N + 1, 0);
  int64_t i = 0, total = 0;
  for (int p = 0; p < parts; ++p)
    for (int64_t l : clen[p]) g.off[++i] = (total += l);
  g.adj.resize(static_cast<size_t>(total));
  for (int p = 0, at = 0; p < parts; ++p) {
    std::copy(cadj[p].begin(), cadj[p].end(), g.adj.begin() + at);
    at += static_cast<int>(cadj[p].size());
  }
  return g;
}

void validate(int64_t N, const int32_t* T, int64_t E) {
  if (N <= 0 || E <= 0) throw std::runtime_error("mesh needs N > 0 nodes and E > 0 elements");
  if (N > std::numeric_limits<int32_t>::max() / 2)
    throw std::runtime_error("mesh too large for 32-bit node indices");
  for (int64_t k = 0; k < 4 * E; ++k)
    if (T[k] < 0 || T[k] >= N)
      throw std::runtime_error("element " + std::to_string(k / 4) + " references node " +
                               std::to_string(T[k]) + " outside [0, N)");
}

// BFS levels from r; returns the last level and the number of levels.
int bfs_levels(const Graph& g, int32_t r, std::vector<int32_t>& level, std::vector<int32_t>& last) {
  std::fill(level.begin(), level.end(), -1);
  std::vector<int32_t> cur{r}, next;
  level[r] = 0;
  int depth = 0;
  for (;;) {
    next.clear();
    for (int32_t v : cur)
      for (int64_t k = g.off[v]; k < g.off[v + 1]; ++k) {
        int32_t w = g.adj[k];
        if (level[w] < 0) {
          level[w] = depth + 1;
          next.push_back(w);
        }
      }
    if (next.empty()) break;
    cur.swap(next);
    ++depth;
  }
  last = cur;
  return depth;
}

// Reverse Cuthill-McKee order of graph g: order[new] = old.
std::vector<int32_t> rcm_of_graph(const Graph& g, int64_t N) {
  std::vector<int32_t> deg(N);
  for (int64_t i = 0; i < N; ++i) deg[i] = static_cast<int32_t>(g.off[i + 1] - g.off[i]);
  std::vector<char> seen(N, 0);
  std::vector<int32_t> order;
  order.reserve(N);
  std::vector<int32_t> level(N), last;
  std::vector<int32_t> nb;
  // nodes by increasing degree: start of each connected component
  std::vector<int32_t> bydeg(N);
  std::iota(bydeg.begin(), bydeg.end(), 0);
  std::stable_sort(bydeg.begin(), bydeg.end(), [&](int32_t a, int32_t b) { return deg[a] < deg[b]; });
  for (int32_t start : bydeg) {
    if (seen[start]) continue;
    // pseudo-peripheral node (George & Liu): walk to a min-degree node of the last level
    int32_t r = start;
    int ecc = bfs_levels(g, r, level, last);
    for (int it = 0; it < 8; ++it) {
      int32_t cand = *std::min_element(last.begin(), last.end(),
                                       [&](int32_t a, int32_t b) { return deg[a] < deg[b]; });
      int e2 = bfs_levels(g, cand, level, last);
      if (e2 <= ecc) break;
      r = cand;
      ecc = e2;
    }
    // Cuthill-McKee BFS, neighbours by increasing degree
    size_t head = order.size();
    order.push_back(r);
    seen[r] = 1;
    while (head < order.size()) {
      int32_t v = order[head++];
      nb.clear();
      for (int64_t k = g.off[v]; k < g.off[v + 1]; ++k)
        if (!seen[g.adj[k]]) nb.push_back(g.adj[k]);
      std::stable_sort(nb.begin(), nb.end(), [&](int32_t a, int32_t b) { return deg[a] < deg[b]; });
      for (int32_t w : nb) {
        seen[w] = 1;
        order.push_back(w);
      }
    }
  }
  std::reverse(order.begin(), order.end());
  return order;  // order[new] = old
}

}  // namespace

std::vector<int32_t> rcm_order(int64_t N, const int32_t* T, int64_t E) {
  validate(N, T, E);
  return rcm_of_graph(node_graph(N, T, E), N);
}

int32_t greedy_colour(int64_t N, const int32_t* T, int64_t E, const int64_t* order, int32_t* colour) {
  constexpr int kWords = 8;  // up to 512 colours
  std::vector<uint64_t> used(static_cast<size_t>(N) * kWords, 0);
  int32_t ncol = 0;
  for (int64_t q = 0; q < E; ++q) {
    int64_t e = order ? order[q] : q;
    uint64_t m[kWords] = {0};
    for (int a = 0; a < 4; ++a)
      for (int w = 0; w < kWords; ++w) m[w] |= used[static_cast<size_t>(T[4 * e + a]) * kWords + w];
    int c = -1;
    for (int w = 0; w < kWords && c < 0; ++w)
      if (~m[w]) c = 64 * w + __builtin_ctzll(~m[w]);
    if (c < 0) throw std::runtime_error("element colouring needs more than 512 colours");
    colour[e] = c;
    ncol = std::max(ncol, c + 1);
    for (int a = 0; a < 4; ++a) used[static_cast<size_t>(T[4 * e + a]) * kWords + c / 64] |= 1ull << (c % 64);
  }
  return ncol;
}

void preprocess(const double* X, int64_t N, const int32_t* T, const int32_t* tag, int64_t E,
                int32_t nmats, bool reorder, HostMesh& h) {
  validate(N, T, E);
  h.N = N;
  h.E = E;
  // ---- element tags -> material rows (scripts/materials.py:22-25)
  // sorted unique tags: a mesh has few, so a sorted insert beats sorting all E of them
  h.tags.clear();
  for (int64_t e = 0; e < E; ++e) {
    if (e > 0 && tag[e] == tag[e - 1]) continue;
    auto it = std::lower_bound(h.tags.begin(), h.tags.end(), tag[e]);
    if (it == h.tags.end() || *it != tag[e]) h.tags.insert(it, tag[e]);
  }
  if (static_cast<int32_t>(h.tags.size()) > nmats)
    throw std::runtime_error("materials file has " + std::to_string(nmats) + " rows for " +
                             std::to_string(h.tags.size()) + " element tags");
  // ---- node order
  const Graph g = node_graph(N, T, E);
  if (reorder) {
    h.perm = rcm_of_graph(g, N);
  } else {
    h.perm.resize(N);
    std::iota(h.perm.begin(), h.perm.end(), 0);
  }
  h.iperm.assign(N, 0);
  for (int64_t i = 0; i < N; ++i) h.iperm[h.perm[i]] = static_cast<int32_t>(i);
  // ---- node-pair pattern in device order: row inew = itself and its neighbours, sorted
  h.nslices = (N + kSlice - 1) / kSlice;
  h.Npad = h.nslices * kSlice;
  h.rowlen.assign(h.Npad, 0);
  std::vector<int64_t> roff(N + 1, 0);
  for (int64_t inew = 0; inew < N; ++inew) {
    const int32_t iold = h.perm[inew];
    roff[inew + 1] = roff[inew] + (g.off[iold + 1] - g.off[iold]) + 1;
  }
  std::vector<int32_t> rows(roff[N]);
  h.nnz = roff[N];
  const int parts = host_parts(N);
  std::vector<int64_t> bw0(parts, 0), bw1(parts, 0);
  parallel_chunks(N, parts, [&](int64_t b, int64_t e, int p) {
    int64_t m0 = 0, m1 = 0;
    for (int64_t inew = b; inew < e; ++inew) {
      const int32_t iold = h.perm[inew];
      int32_t* r = rows.data() + roff[inew];
      int32_t* w = r;
      *w++ = static_cast<int32_t>(inew);
      for (int64_t k = g.off[iold]; k < g.off[iold + 1]; ++k) {
        const int32_t jnew = h.iperm[g.adj[k]];
        *w++ = jnew;
        m0 = std::max<int64_t>(m0, std::llabs(int64_t(g.adj[k]) - iold));
        m1 = std::max<int64_t>(m1, std::llabs(int64_t(jnew) - inew));
      }
      std::sort(r, w);
      h.rowlen[inew] = static_cast<int32_t>(w - r);
    }
    bw0[p] = m0;
    bw1[p] = m1;
  });
  for (int p = 0; p < parts; ++p) {
    h.bandwidth_before = std::max(h.bandwidth_before, bw0[p]);
    h.bandwidth_after = std::max(h.bandwidth_after, bw1[p]);
  }
  h.sl_off.assign(h.nslices + 1, 0);
  h.sl_w.assign(h.nslices, 0);
  for (int64_t s = 0; s < h.nslices; ++s) {
    int32_t w = 0;
    for (int l = 0; l < kSlice; ++l) w = std::max(w, h.rowlen[s * kSlice + l]);
    h.sl_w[s] = w;
    h.sl_off[s + 1] = h.sl_off[s] + static_cast<int64_t>(w) * kSlice;
  }
  h.nent = h.sl_off[h.nslices];
  h.col.assign(h.nent, 0);
  parallel_chunks(h.nslices, host_parts(N), [&](int64_t b, int64_t e, int) {
    for (int64_t s = b; s < e; ++s)
      for (int l = 0; l < kSlice; ++l) {
        int64_t i = s * kSlice + l;
        for (int32_t k = 0; k < h.sl_w[s]; ++k) {
          int32_t c = static_cast<int32_t>(i);  // padding entries point at the row itself
          if (i < N && k < h.rowlen[i]) c = rows[roff[i] + k];
          h.col[h.sl_off[s] + static_cast<int64_t>(k) * kSlice + l] = c;
        }
      }
  });
  rows = std::vector<int32_t>();
  // ---- elements: device node ids, colour classes sorted by first node (locality)
  std::vector<int32_t> cn(4 * E);
  std::vector<int32_t> emin(E);
  parallel_chunks(E, host_parts(E), [&](int64_t b, int64_t e_end, int) {
    for (int64_t e = b; e < e_end; ++e) {
      for (int a = 0; a < 4; ++a) cn[4 * e + a] = h.iperm[T[4 * e + a]];
      emin[e] = std::min(std::min(cn[4 * e], cn[4 * e + 1]), std::min(cn[4 * e + 2], cn[4 * e + 3]));
    }
  });
  // elements by their smallest device node id, ties in input order (a stable counting sort)
  std::vector<int64_t> eorder(E);
  {
    std::vector<int64_t> cnt(N + 1, 0);
    for (int64_t e = 0; e < E; ++e) cnt[emin[e] + 1]++;
    for (int64_t i = 0; i < N; ++i) cnt[i + 1] += cnt[i];
    for (int64_t e = 0; e < E; ++e) eorder[cnt[emin[e]]++] = e;
  }
  std::vector<int32_t> colour(E);
  int32_t ncol = greedy_colour(N, cn.data(), E, eorder.data(), colour.data());
  std::vector<int64_t> byc(E);
  {
    std::vector<int64_t> cnt(ncol + 1, 0);
    for (int64_t e = 0; e < E; ++e) cnt[colour[e] + 1]++;
    for (int c = 0; c < ncol; ++c) cnt[c + 1] += cnt[c];
    h.colour_off = cnt;
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (int64_t q = 0; q < E; ++q) {
      int64_t e = eorder[q];
      byc[pos[colour[e]]++] = e;
    }
  }
  h.econn.resize(4 * E);
  h.etag.resize(E);
  {
    parallel_chunks(E, host_parts(E), [&](int64_t b, int64_t en, int) {
      for (int64_t q = b; q < en; ++q) {
        const int64_t e = byc[q];
        for (int a = 0; a < 4; ++a) h.econn[4 * q + a] = cn[4 * e + a];
        h.etag[q] = static_cast<int32_t>(std::lower_bound(h.tags.begin(), h.tags.end(), tag[e]) - h.tags.begin());
      }
    });
  }
  // ---- coordinates in device order
  h.Xd.assign(3 * h.Npad, 0.0);
  for (int64_t i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) h.Xd[3 * h.iperm[i] + c] = X[3 * i + c];
  // ---- boundary branch, scripts/matrix.py:49-64 and scripts/trafo.py:4-16
  const double rtol = std::sqrt(std::numeric_limits<double>::epsilon());
  std::vector<double> rn(N);
  double Rinf = 0.0;
  for (int64_t i = 0; i < N; ++i) {
    rn[i] = std::sqrt(X[3 * i] * X[3 * i] + X[3 * i + 1] * X[3 * i + 1] + X[3 * i + 2] * X[3 * i + 2]);
    Rinf = std::max(Rinf, rn[i]);
  }
  h.Rinf = Rinf;
  double lsup = 0.0;
  for (int64_t i = 0; i < N; ++i) lsup = std::max(lsup, std::fabs(rn[i] - Rinf));
  int64_t at_rinf = 0;
  for (int64_t i = 0; i < N; ++i) at_rinf += std::fabs(rn[i] - Rinf) <= rtol * lsup;
  h.airbox = (at_rinf == 8);
  std::vector<uint8_t> bold(N, 0);
  if (h.airbox) {
    for (int c = 0; c < 3; ++c) {
      double xe = -std::numeric_limits<double>::infinity();
      for (int64_t i = 0; i < N; ++i) xe = std::max(xe, X[3 * i + c]);
      for (int sgn = -1; sgn <= 1; sgn += 2) {
        double ls = 0.0;
        for (int64_t i = 0; i < N; ++i) ls = std::max(ls, std::fabs(X[3 * i + c] + sgn * xe));
        for (int64_t i = 0; i < N; ++i)
          if (std::fabs(X[3 * i + c] + sgn * xe) <= rtol * ls) bold[i] = 1;
      }
    }
  } else {
    if (h.tags.size() < 2)
      throw std::runtime_error("spherical-shell boundary needs at least two element tags");
    for (int64_t i = 0; i < N; ++i) bold[i] = std::fabs(rn[i] - Rinf) <= rtol * lsup;
    int32_t t2 = h.tags[h.tags.size() - 2];
    double R = 0.0;
    for (int64_t e = 0; e < E; ++e)
      if (tag[e] == t2)
        for (int a = 0; a < 4; ++a) R = std::max(R, rn[T[4 * e + a]]);
    h.R = R;
  }
  h.bnd.assign(h.Npad, 0);
  for (int64_t i = 0; i < N; ++i) h.bnd[h.iperm[i]] = bold[i];
}

}  // namespace mumag
