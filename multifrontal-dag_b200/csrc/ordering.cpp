// Fill-reducing ordering owned by the library: nested dissection of the
// matrix graph.  It stands where the reference calls METIS_NodeND
// (ordering_m.f90:11-36, use_metis = 1) and returns the same kind of
// permutation (new -> old, 1-based) that the analysis takes.
//
// Recursive bisection by BFS level structures: in each part, a
// pseudo-peripheral vertex (repeated BFS from the last level's
// lowest-degree vertex) roots a level structure; the smallest level near the
// middle (by vertex count) becomes the separator; separator vertices with
// no neighbour on one side move to the other side; both sides are ordered
// first (recursively), the separator last.  Disconnected parts are ordered
// one after another with no separator.  Parts of at most kLeaf vertices are
// ordered by increasing degree within the part (ties by index).  The graph is
// first compressed: vertices with identical closed neighbourhoods (the
// unknowns of one mesh node) become one vertex weighted by their count, and
// stay consecutive in the ordering.  Everything is deterministic (no
// randomness, ties broken by vertex index).
#include <algorithm>
#include <cstdint>
#include <vector>

#include "analysis.hpp"

namespace mfd {
namespace {

constexpr int kLeaf = 64;

struct Graph {
  int n = 0;
  std::vector<int64_t> ptr;
  std::vector<int32_t> adj;
  std::vector<int32_t> wt;      // vertex weight: original vertices a compressed vertex stands for
  int deg(int v) const { return (int)(ptr[v + 1] - ptr[v]); }
};

// symmetric adjacency (no diagonal) from the lower CCS, 1-based
bool build_graph(int32_t n, const int32_t* col, const int32_t* row, Graph& g) {
  g.n = n;
  std::vector<int64_t> cnt(n + 1, 0);
  for (int32_t j = 0; j < n; ++j)
    for (int32_t k = col[j] - 1; k < col[j + 1] - 1; ++k) {
      const int32_t i = row[k] - 1;
      if (i < 0 || i >= n) return false;
      if (i == j) continue;
      cnt[i + 1]++;
      cnt[j + 1]++;
    }
  for (int32_t v = 0; v < n; ++v) cnt[v + 1] += cnt[v];
  g.ptr = cnt;
  g.adj.assign(cnt[n], 0);
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (int32_t j = 0; j < n; ++j)
    for (int32_t k = col[j] - 1; k < col[j + 1] - 1; ++k) {
      const int32_t i = row[k] - 1;
      if (i == j) continue;
      g.adj[fill[i]++] = j;
      g.adj[fill[j]++] = i;
    }
  for (int32_t v = 0; v < n; ++v) std::sort(g.adj.begin() + g.ptr[v], g.adj.begin() + g.ptr[v + 1]);
  g.wt.assign(n, 1);
  return true;
}

// Compression: vertices with identical closed neighbourhoods (several
// unknowns of one mesh node) merge into one vertex of that weight; `members`
// lists each compressed vertex's original vertices in ascending order.
void compress(const Graph& g, Graph& c, std::vector<std::vector<int32_t>>& members) {
  const int n = g.n;
  std::vector<uint64_t> h(n);
  for (int32_t v = 0; v < n; ++v) {                     // order-independent hash of N[v] = {v} + adj(v)
    uint64_t a = 0x9e3779b97f4a7c15ull * (uint64_t)(v + 1), b = (uint64_t)(v + 1);
    for (int64_t k = g.ptr[v]; k < g.ptr[v + 1]; ++k) {
      a += 0x9e3779b97f4a7c15ull * (uint64_t)(g.adj[k] + 1);
      b ^= (uint64_t)(g.adj[k] + 1) * 0xc2b2ae3d27d4eb4full;
    }
    h[v] = a ^ (b << 1) ^ ((uint64_t)g.deg(v) << 56);
  }
  std::vector<int32_t> rep(n, -1), idx(n);
  for (int32_t v = 0; v < n; ++v) idx[v] = v;
  std::sort(idx.begin(), idx.end(), [&](int32_t x, int32_t y) { return h[x] != h[y] ? h[x] < h[y] : x < y; });
  auto same = [&](int32_t u, int32_t v) {               // N[u] == N[v] (u, v adjacent, equal degrees)
    if (g.deg(u) != g.deg(v)) return false;
    if (!std::binary_search(g.adj.begin() + g.ptr[u], g.adj.begin() + g.ptr[u + 1], v)) return false;
    int64_t i = g.ptr[u], j = g.ptr[v];
    while (i < g.ptr[u + 1] && j < g.ptr[v + 1]) {      // adj(u) - {v} == adj(v) - {u}
      if (g.adj[i] == v) { ++i; continue; }
      if (g.adj[j] == u) { ++j; continue; }
      if (g.adj[i] != g.adj[j]) return false;
      ++i; ++j;
    }
    while (i < g.ptr[u + 1] && g.adj[i] == v) ++i;
    while (j < g.ptr[v + 1] && g.adj[j] == u) ++j;
    return i == g.ptr[u + 1] && j == g.ptr[v + 1];
  };
  for (size_t a = 0; a < idx.size();) {
    size_t b = a;
    while (b < idx.size() && h[idx[b]] == h[idx[a]]) ++b;
    for (size_t i = a; i < b; ++i) {                    // within a hash bucket, ascending vertex index
      const int32_t u = idx[i];
      if (rep[u] >= 0) continue;
      rep[u] = u;
      for (size_t j = i + 1; j < b; ++j) {
        const int32_t v = idx[j];
        if (rep[v] < 0 && same(u, v)) rep[v] = u;
      }
    }
    a = b;
  }
  std::vector<int32_t> cid(n, -1);
  int nc = 0;
  members.clear();
  for (int32_t v = 0; v < n; ++v) {
    if (rep[v] == v) {
      cid[v] = nc++;
      members.push_back({});
    }
  }
  for (int32_t v = 0; v < n; ++v) {
    cid[v] = cid[rep[v]];
    members[cid[v]].push_back(v);
  }
  c.n = nc;
  c.ptr.assign(nc + 1, 0);
  c.adj.clear();
  c.wt.assign(nc, 0);
  for (int32_t x = 0; x < nc; ++x) {
    const int32_t v = members[x][0];
    c.wt[x] = (int32_t)members[x].size();
    const size_t start = c.adj.size();
    for (int64_t k = g.ptr[v]; k < g.ptr[v + 1]; ++k) {
      const int32_t y = cid[g.adj[k]];
      if (y != x) c.adj.push_back(y);
    }
    std::sort(c.adj.begin() + start, c.adj.end());
    c.adj.erase(std::unique(c.adj.begin() + start, c.adj.end()), c.adj.end());
    c.ptr[x + 1] = (int64_t)c.adj.size();
  }
}

struct Work {
  std::vector<int32_t> part;    // part id of every vertex (vertices of the current part share one id)
  std::vector<int32_t> level;   // BFS level scratch (-1: unvisited)
  int32_t next_id = 1;
};

// BFS inside part `pid` from root; fills `order` (visit order) and levels; returns the level count
int bfs(const Graph& g, Work& w, int32_t pid, int32_t root, std::vector<int32_t>& order) {
  order.clear();
  order.push_back(root);
  w.level[root] = 0;
  int nl = 1;
  for (size_t h = 0; h < order.size(); ++h) {
    const int32_t v = order[h];
    for (int64_t k = g.ptr[v]; k < g.ptr[v + 1]; ++k) {
      const int32_t u = g.adj[k];
      if (w.part[u] != pid || w.level[u] >= 0) continue;
      w.level[u] = w.level[v] + 1;
      nl = std::max(nl, w.level[u] + 1);
      order.push_back(u);
    }
  }
  return nl;
}

void clear_levels(Work& w, const std::vector<int32_t>& vs) {
  for (int32_t v : vs) w.level[v] = -1;
}

// order the vertices `vs` (one part) into out, appending
void dissect(const Graph& g, Work& w, std::vector<int32_t> vs, std::vector<int32_t>& out) {
  struct Task {
    std::vector<int32_t> vs;
    bool emit;                  // true: append vs as they are (a separator, already ordered)
  };
  std::vector<Task> stack;
  stack.push_back({std::move(vs), false});
  std::vector<int32_t> order, order2;
  while (!stack.empty()) {
    Task t = std::move(stack.back());
    stack.pop_back();
    if (t.emit) {
      out.insert(out.end(), t.vs.begin(), t.vs.end());
      continue;
    }
    std::vector<int32_t>& S = t.vs;
    const int32_t pid = w.next_id++;
    for (int32_t v : S) w.part[v] = pid;
    if ((int)S.size() <= kLeaf) {               // leaf: by degree inside the part, then index
      std::vector<std::pair<int, int32_t>> key;
      key.reserve(S.size());
      for (int32_t v : S) {
        int d = 0;
        for (int64_t k = g.ptr[v]; k < g.ptr[v + 1]; ++k) d += w.part[g.adj[k]] == pid;
        key.push_back({d, v});
      }
      std::sort(key.begin(), key.end());
      for (auto& kv : key) out.push_back(kv.second);
      continue;
    }
    // pseudo-peripheral root: start from the lowest-index vertex of minimum degree
    int32_t root = S[0];
    for (int32_t v : S)
      if (g.deg(v) < g.deg(root) || (g.deg(v) == g.deg(root) && v < root)) root = v;
    int nl = bfs(g, w, pid, root, order);
    for (int it = 0; it < 4; ++it) {
      int32_t cand = -1;
      for (size_t h = order.size(); h-- > 0;) {
        const int32_t v = order[h];
        if (w.level[v] != nl - 1) break;
        if (cand < 0 || g.deg(v) < g.deg(cand) || (g.deg(v) == g.deg(cand) && v < cand)) cand = v;
      }
      clear_levels(w, order);
      const int nl2 = bfs(g, w, pid, cand, order2);
      if (nl2 <= nl) {
        clear_levels(w, order2);
        nl = bfs(g, w, pid, root, order);
        break;
      }
      root = cand;
      nl = nl2;
      order.swap(order2);
    }
    if (order.size() < S.size()) {              // disconnected: this component, then the rest
      std::vector<int32_t> comp(order.begin(), order.end()), rest;
      rest.reserve(S.size() - comp.size());
      for (int32_t v : S)
        if (w.level[v] < 0) rest.push_back(v);
      clear_levels(w, order);
      std::sort(comp.begin(), comp.end());
      stack.push_back({std::move(rest), false});
      stack.push_back({std::move(comp), false});
      continue;
    }
    if (nl < 3) {                               // too shallow to split by levels: order as a leaf would
      clear_levels(w, order);
      std::vector<std::pair<int, int32_t>> key;
      for (int32_t v : S) key.push_back({g.deg(v), v});
      std::sort(key.begin(), key.end());
      for (auto& kv : key) out.push_back(kv.second);
      continue;
    }
    // level sizes; the separator: the smallest level among those whose
    // cumulative count lies within [0.3, 0.7] of the part (the middle one if none)
    std::vector<int64_t> lsz(nl, 0);
    int64_t total = 0;
    for (int32_t v : order) {
      lsz[w.level[v]] += g.wt[v];
      total += g.wt[v];
    }
    int best = -1;
    int64_t cum = 0, bestsz = INT64_MAX;
    for (int l = 0; l < nl; ++l) {
      const int64_t before = cum;
      cum += lsz[l];
      if (l == 0 || l == nl - 1) continue;
      if (before * 10 < total * 3 || before * 10 > total * 7) continue;
      if (lsz[l] < bestsz) {
        bestsz = lsz[l];
        best = l;
      }
    }
    if (best < 0) {
      cum = 0;
      for (int l = 1; l < nl - 1; ++l) {
        cum += lsz[l - 1];
        if (cum * 2 >= total) {
          best = l;
          break;
        }
      }
      if (best < 0) best = nl / 2;
    }
    std::vector<int32_t> A, B, Sep;
    for (int32_t v : order) {
      const int l = w.level[v];
      if (l < best) A.push_back(v);
      else if (l == best) Sep.push_back(v);
      else B.push_back(v);
    }
    // refinement: a separator vertex with no neighbour in B joins A, one with
    // none in A joins B (level membership marks the sides)
    std::vector<int32_t> Sep2;
    for (int32_t v : Sep) {
      bool na = false, nb = false;
      for (int64_t k = g.ptr[v]; k < g.ptr[v + 1]; ++k) {
        const int32_t u = g.adj[k];
        if (w.part[u] != pid) continue;
        const int lu = w.level[u];
        if (lu < best) na = true;
        else if (lu > best) nb = true;
      }
      if (!nb) {
        A.push_back(v);
        w.level[v] = best - 1;                  // now on side A for the later tests
      } else if (!na) {
        B.push_back(v);
        w.level[v] = best + 1;
      } else {
        Sep2.push_back(v);
      }
    }
    clear_levels(w, order);
    std::sort(A.begin(), A.end());
    std::sort(B.begin(), B.end());
    std::sort(Sep2.begin(), Sep2.end());
    // popped in reverse: A, B, then the separator
    stack.push_back({std::move(Sep2), true});
    stack.push_back({std::move(B), false});
    stack.push_back({std::move(A), false});
  }
}

}  // namespace

int nested_dissection(int32_t n, const int32_t* ccs_col, const int32_t* ccs_row, int32_t* order_perm) {
  if (n < 1 || !ccs_col || !ccs_row || !order_perm || ccs_col[0] != 1) return -1;
  Graph g0, g;
  if (!build_graph(n, ccs_col, ccs_row, g0)) return -1;
  std::vector<std::vector<int32_t>> members;
  compress(g0, g, members);
  Work w;
  w.part.assign(g.n, 0);
  w.level.assign(g.n, -1);
  std::vector<int32_t> all(g.n), out;
  for (int32_t v = 0; v < g.n; ++v) all[v] = v;
  out.reserve(g.n);
  dissect(g, w, std::move(all), out);
  if ((int32_t)out.size() != g.n) return -1;
  int32_t i = 0;
  for (int32_t x : out)
    for (int32_t v : members[x]) order_perm[i++] = v + 1;      // a compressed vertex's unknowns stay together
  return i == n ? 0 : -1;
}

}  // namespace mfd
