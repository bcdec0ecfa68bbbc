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

// The Poisson boundary branch, scripts/matrix.py:49-64 and scripts/trafo.py:4-16: airbox
// (exactly 8 nodes at the largest radius: Dirichlet nodes on the bounding-box faces) or
// spherical shell (Dirichlet nodes at the largest radius; R from the second-to-last tag).
// bold[i] = 1 for Dirichlet node i (mesh-file order).
void boundary_nodes(const double* X, int64_t N, const int32_t* T, const int32_t* tag, int64_t E, HostMesh& h,
                    std::vector<uint8_t>& bold) {
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
  bold.assign(N, 0);
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
}

// Spatial aggregates of the interior nodes for the two-level preconditioner: a grid of
// boxes over the interior nodes' bounding box, sized for about `target` nodes per box.
// Boxes with fewer than kMinBoxNodes nodes (interior and Dirichlet) are merged into the
// previous box in lexicographic order (the first ones into the next), so every box spans at
// least kMinBoxNodes consecutive device rows and a 32-row slice meets at most two boxes.
// key[i] = the (merged) box of node i, used for the node order; cbox[i] = the aggregate of
// interior node i (aggregates numbered in ascending key), -1 for a Dirichlet node.  The box
// size grows until there are at most kMaxCoarse aggregates.
void coarse_boxes(const double* X, int64_t N, const std::vector<uint8_t>& bold, int32_t target,
                  std::vector<int64_t>& key, std::vector<int32_t>& cbox, int32_t& nc) {
  key.assign(N, 0);
  cbox.assign(N, -1);
  nc = 0;
  double lo[3] = {std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                  std::numeric_limits<double>::infinity()};
  double hi[3] = {-lo[0], -lo[1], -lo[2]};
  int64_t nint = 0;
  for (int64_t i = 0; i < N; ++i) {
    if (bold[i]) continue;
    ++nint;
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], X[3 * i + d]);
      hi[d] = std::max(hi[d], X[3 * i + d]);
    }
  }
  if (nint == 0) return;
  double ext[3];
  int nd = 0;
  double vol = 1.0;
  for (int d = 0; d < 3; ++d) {
    ext[d] = hi[d] - lo[d];
    if (ext[d] > 0) {
      ++nd;
      vol *= ext[d];
    }
  }
  for (int64_t tgt = std::max<int64_t>(target, kMinBoxNodes);; tgt = tgt * 3 / 2 + 1) {
    const double want = std::max(1.0, static_cast<double>(nint) / static_cast<double>(tgt));
    const double b = nd > 0 ? std::pow(vol / want, 1.0 / nd) : 1.0;
    int64_t nb[3];
    for (int d = 0; d < 3; ++d)
      nb[d] = ext[d] > 0 ? std::max<int64_t>(1, std::llround(ext[d] / b)) : 1;
    const int64_t nkeys = nb[0] * nb[1] * nb[2];
    std::vector<int64_t> cnt(nkeys, 0), cint(nkeys, 0);
    for (int64_t i = 0; i < N; ++i) {
      int64_t k[3];
      for (int d = 0; d < 3; ++d) {
        const double t = ext[d] > 0 ? std::floor((X[3 * i + d] - lo[d]) / ext[d] * static_cast<double>(nb[d])) : 0.0;
        k[d] = std::min<int64_t>(nb[d] - 1, std::max<int64_t>(0, static_cast<int64_t>(t)));
      }
      key[i] = (k[2] * nb[1] + k[1]) * nb[0] + k[0];
      cnt[key[i]]++;
      cint[key[i]] += bold[i] ? 0 : 1;
    }
    // merge small boxes: into the last kept box before them, else into the first kept after
    std::vector<int64_t> map(nkeys, -1);
    int64_t last = -1;
    std::vector<int64_t> pending;
    for (int64_t k = 0; k < nkeys; ++k) {
      if (cnt[k] == 0) continue;
      if (cnt[k] >= kMinBoxNodes) {
        map[k] = k;
        last = k;
        for (int64_t q : pending) map[q] = k;
        pending.clear();
      } else if (last >= 0) {
        map[k] = last;
      } else {
        pending.push_back(k);
      }
    }
    for (int64_t q : pending) map[q] = pending.front();  // no box reached kMinBoxNodes
    if (!pending.empty()) map[pending.front()] = pending.front();
    std::vector<int64_t> mint(nkeys, 0);
    for (int64_t k = 0; k < nkeys; ++k)
      if (cnt[k]) mint[map[k]] += cint[k];
    std::vector<int32_t> cid(nkeys, -1);
    int32_t n = 0;
    for (int64_t k = 0; k < nkeys; ++k)
      if (map[k] == k && mint[k] > 0) cid[k] = n++;
    if (n > kMaxCoarse) continue;
    nc = n;
    for (int64_t i = 0; i < N; ++i) {
      key[i] = map[key[i]];
      cbox[i] = bold[i] ? -1 : cid[key[i]];
    }
    return;
  }
}
}  // namespace

void spd_inverse(int32_t n, int32_t bw, std::vector<double>& A) {
  if (n <= 0) return;
  if (A.size() != static_cast<size_t>(n) * n) throw std::logic_error("spd_inverse: matrix size");
  bw = std::max<int32_t>(0, std::min<int32_t>(bw, n - 1));
  const size_t N = static_cast<size_t>(n);
  // lower Cholesky factor L (row-major), and U = L^T row-major for the backward solves
  std::vector<double> L(N * N, 0.0);
  for (int32_t j = 0; j < n; ++j) {
    const double* Lj = L.data() + j * N;
    double d = A[j * N + j];
    for (int32_t k = std::max(0, j - bw); k < j; ++k) d -= Lj[k] * Lj[k];
    if (!(d > 0.0) || !std::isfinite(d))
      throw std::runtime_error("coarse Poisson matrix is not positive definite (aggregate " + std::to_string(j) + ")");
    const double djj = std::sqrt(d);
    L[j * N + j] = djj;
    const int32_t iend = std::min(n - 1, j + bw);
    for (int32_t i = j + 1; i <= iend; ++i) {
      double* Li = L.data() + i * N;
      double v = A[i * N + j];
      for (int32_t k = std::max(0, i - bw); k < j; ++k) v -= Li[k] * Lj[k];
      Li[j] = v / djj;
    }
  }
  std::vector<double> U(N * N, 0.0);
  for (size_t i = 0; i < N; ++i)
    for (size_t k = (i > static_cast<size_t>(bw) ? i - bw : 0); k <= i; ++k) U[k * N + i] = L[i * N + k];
  // column j of A^-1: L y = e_j (y is zero above j), then L^T x = y
  parallel_chunks(n, std::max(1, std::min(host_parts(int64_t(1) << 20), n)), [&](int64_t c0, int64_t c1, int) {
    std::vector<double> y(N);
    for (int64_t j = c0; j < c1; ++j) {
      std::fill(y.begin(), y.end(), 0.0);
      y[j] = 1.0 / L[j * N + j];
      for (int32_t i = static_cast<int32_t>(j) + 1; i < n; ++i) {
        const double* Li = L.data() + i * N;
        double v = 0.0;
        for (int32_t k = std::max<int32_t>(static_cast<int32_t>(j), i - bw); k < i; ++k) v += Li[k] * y[k];
        y[i] = -v / Li[i];
      }
      for (int32_t i = n - 1; i >= 0; --i) {
        const double* Ui = U.data() + i * N;
        double v = y[i];
        const int32_t kend = std::min(n - 1, i + bw);
        for (int32_t k = i + 1; k <= kend; ++k) v -= Ui[k] * y[k];
        y[i] = v / Ui[i];
      }
      for (int32_t i = 0; i < n; ++i) A[i * N + j] = y[i];
    }
  });
}

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
                int32_t nmats, bool reorder, int32_t coarse_nodes, HostMesh& h) {
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
  std::vector<uint8_t> bold;
  boundary_nodes(X, N, T, tag, E, h, bold);
  // ---- node order
  const Graph g = node_graph(N, T, E);
  if (reorder) {
    h.perm = rcm_of_graph(g, N);
  } else {
    h.perm.resize(N);
    std::iota(h.perm.begin(), h.perm.end(), 0);
  }
  std::vector<int32_t> cbox;
  h.nc = 0;
  if (coarse_nodes > 0) {  // box by box, the order above inside each box
    std::vector<int64_t> key;
    coarse_boxes(X, N, bold, coarse_nodes, key, cbox, h.nc);
    std::stable_sort(h.perm.begin(), h.perm.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
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
  h.bnd.assign(h.Npad, 0);
  for (int64_t i = 0; i < N; ++i) h.bnd[h.iperm[i]] = bold[i];
  h.rbox.assign(h.Npad, -1);
  if (h.nc > 0)
    for (int64_t i = 0; i < N; ++i) h.rbox[h.iperm[i]] = cbox[i];
}

}  // namespace mumag
