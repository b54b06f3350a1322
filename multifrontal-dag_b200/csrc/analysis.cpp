// Host symbolic analysis (see analysis.hpp).  Internally 0-based; the output
// arrays carry the reference's 1-based values.
#include "analysis.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <utility>

namespace mfd {
namespace {

using V = std::vector<int32_t>;

// Column- (or row-) compressed lists: entries of list i are v[off[i] .. off[i+1]).
struct Lists {
  V off, v;
  int32_t count() const { return (int32_t)off.size() - 1; }
  int32_t len(int32_t i) const { return off[i + 1] - off[i]; }
  const int32_t* at(int32_t i) const { return v.data() + off[i]; }
  int32_t* at(int32_t i) { return v.data() + off[i]; }
};

Lists lists_from_lengths(const V& len) {
  Lists L;
  L.off.assign(len.size() + 1, 0);
  for (size_t i = 0; i < len.size(); i++) L.off[i + 1] = L.off[i] + len[i];
  L.v.assign(L.off.back(), 0);
  return L;
}

// children of every node in ascending order (tree_m.f90:15-55)
Lists children_of(const V& parent) {
  int32_t n = (int32_t)parent.size();
  V cnt(n, 0);
  for (int32_t i = 0; i < n; i++)
    if (parent[i] >= 0) cnt[parent[i]]++;
  Lists c = lists_from_lengths(cnt);
  V fill(c.off.begin(), c.off.end() - 1);
  for (int32_t i = 0; i < n; i++)
    if (parent[i] >= 0) c.v[fill[parent[i]]++] = i;
  return c;
}

// parent array of a postordered tree given per-node child counts (tree_m.f90:57-76)
V parent_from_child_counts(const V& num_child) {
  int32_t n = (int32_t)num_child.size();
  V parent(n, -1), stack;
  stack.reserve(n);
  for (int32_t i = 0; i < n; i++) {
    for (int32_t j = 0; j < num_child[i]; j++) {
      parent[stack.back()] = i;
      stack.pop_back();
    }
    stack.push_back(i);
  }
  return parent;
}

// Reorder a lower CCS by a symmetric permutation; src records, per output
// entry, the index of the input entry (repostordering_ccs, reordering_m.f90:31-96).
Lists permute_columns(const Lists& a, const V& perm, const V& iperm, V* src) {
  int32_t n = a.count();
  V len(n);
  for (int32_t c = 0; c < n; c++) len[c] = a.len(perm[c]);
  Lists out = lists_from_lengths(len);
  if (src) src->assign(out.v.size(), 0);
  for (int32_t co = 0; co < n; co++) {
    int32_t cr = iperm[co];
    const int32_t* ro = a.at(co);
    int32_t* rr = out.at(cr);
    for (int32_t i = 0; i < a.len(co); i++) {
      rr[i] = iperm[ro[i]];
      if (src) (*src)[out.off[cr] + i] = a.off[co] + i;
    }
  }
  return out;
}

// Disjoint sets whose find() returns the label of the set (the tree node
// that currently represents the merged subtree).
struct LabeledSets {
  V up, size, label;
  explicit LabeledSets(int32_t n) : up(n), size(n, 1), label(n) {
    std::iota(up.begin(), up.end(), 0);
    std::iota(label.begin(), label.end(), 0);
  }
  int32_t root(int32_t x) {
    int32_t r = x;
    while (up[r] != r) r = up[r];
    while (up[x] != r) { int32_t nx = up[x]; up[x] = r; x = nx; }
    return r;
  }
  int32_t find(int32_t x) { return label[root(x)]; }
  void merge_into(int32_t child, int32_t parent_node) {  // set(child) joins set(parent_node), label parent_node
    int32_t a = root(child), b = root(parent_node);
    if (a == b) { label[a] = parent_node; return; }
    if (size[a] > size[b]) std::swap(a, b);
    up[a] = b;
    size[b] += size[a];
    label[b] = parent_node;
  }
};

// Linked lists over node ids with per-list head/tail (doubly_linked_lists_m.f90).
struct NodeLists {
  V head, tail, next, prev;
  explicit NodeLists(int32_t n) : head(n, -1), tail(n, -1), next(n, -1), prev(n, -1) {}
  void add(int32_t node, int32_t list) {
    if (head[list] < 0) { head[list] = tail[list] = node; }
    else { prev[node] = tail[list]; next[tail[list]] = node; tail[list] = node; }
  }
  void append(int32_t from, int32_t to) {       // move list `from` to the end of `to`
    if (head[from] < 0) return;
    if (head[to] < 0) { head[to] = head[from]; tail[to] = tail[from]; }
    else { next[tail[to]] = head[from]; tail[to] = tail[from]; }
    head[from] = tail[from] = -1;
  }
  void remove(int32_t node, int32_t list) {
    int32_t nx = next[node], pv = prev[node];
    if (node == head[list]) head[list] = nx; else next[pv] = nx;
    if (node == tail[list]) tail[list] = pv; else prev[nx] = pv;
    next[node] = prev[node] = -1;
  }
  int32_t length(int32_t list) const {
    int32_t c = 0;
    for (int32_t x = head[list]; x >= 0; x = next[x]) c++;
    return c;
  }
};

}  // namespace

int analyze(int32_t n, const int32_t* ccs_col, const int32_t* ccs_row, const int32_t* order_perm, int32_t max_zero,
            Symbolic& out) {
  if (n <= 0 || !ccs_col || !ccs_row) return -1;
  if (ccs_col[0] != 1) return -1;
  const int32_t nnz = ccs_col[n] - 1;
  // ---- input: lower CCS, diagonal first in every column --------------------
  Lists orig;
  orig.off.resize(n + 1);
  for (int32_t j = 0; j <= n; j++) orig.off[j] = ccs_col[j] - 1;
  orig.v.resize(nnz);
  for (int32_t j = 0; j < n; j++) {
    if (orig.off[j + 1] <= orig.off[j]) return -1;
    for (int32_t k = orig.off[j]; k < orig.off[j + 1]; k++) {
      int32_t r = ccs_row[k] - 1;
      if (r < j || r >= n) return -1;
      if ((k == orig.off[j]) != (r == j)) return -1;
      orig.v[k] = r;
    }
  }
  // ---- optional external ordering: the METIS branch (reordering_m.f90:98-148) ----
  Lists reo;
  V reo_src, reo_perm;
  if (order_perm) {
    reo_perm.resize(n);
    V ip(n, -1);
    for (int32_t i = 0; i < n; i++) {
      int32_t o = order_perm[i] - 1;
      if (o < 0 || o >= n || ip[o] >= 0) return -1;
      reo_perm[i] = o;
      ip[o] = i;
    }
    V len(n, 0);
    for (int32_t j = 0; j < n; j++)
      for (int32_t k = orig.off[j]; k < orig.off[j + 1]; k++) len[std::min(ip[j], ip[orig.v[k]])]++;
    reo = lists_from_lengths(len);
    reo_src.resize(nnz);
    V fill(reo.off.begin(), reo.off.end() - 1);
    for (int32_t j = 0; j < n; j++)
      for (int32_t k = orig.off[j]; k < orig.off[j + 1]; k++) {
        int32_t a = ip[j], b = ip[orig.v[k]];
        int32_t c = std::min(a, b), r = std::max(a, b);
        reo.v[fill[c]] = r;
        reo_src[fill[c]] = k;
        fill[c]++;
      }
    std::vector<std::pair<int32_t, int32_t>> tmp;
    for (int32_t c = 0; c < n; c++) {
      int32_t lo = reo.off[c], hi = reo.off[c + 1];
      tmp.clear();
      for (int32_t k = lo; k < hi; k++) tmp.emplace_back(reo.v[k], reo_src[k]);
      std::sort(tmp.begin(), tmp.end());
      for (int32_t k = lo; k < hi; k++) { reo.v[k] = tmp[k - lo].first; reo_src[k] = tmp[k - lo].second; }
    }
  } else {
    reo = orig;
  }

  // ---- elimination tree (compute_tree_m.f90:10-35) ----
  V etree(n, -1), anc(n, -1);
  {
    // row lists of the lower triangle, columns ascending
    V cnt(n, 0);
    for (int32_t j = 0; j < n; j++)
      for (int32_t k = reo.off[j]; k < reo.off[j + 1]; k++) cnt[reo.v[k]]++;
    Lists rows = lists_from_lengths(cnt);
    V fill(rows.off.begin(), rows.off.end() - 1);
    for (int32_t j = 0; j < n; j++)
      for (int32_t k = reo.off[j]; k < reo.off[j + 1]; k++) rows.v[fill[reo.v[k]]++] = j;
    for (int32_t i = 0; i < n; i++) {
      for (int32_t t = rows.off[i]; t < rows.off[i + 1] - 1; t++) {
        int32_t r = rows.v[t];
        while (anc[r] >= 0 && anc[r] != i) { int32_t nx = anc[r]; anc[r] = i; r = nx; }
        if (anc[r] < 0) { anc[r] = i; etree[r] = i; }
      }
    }
  }
  for (int32_t i = 0; i < n - 1; i++)
    if (etree[i] < 0) return -1;                  // the reference requires one tree rooted at n
  // ---- postorder (tree_m.f90:78-99) ----
  V post(n), ipost(n);
  {
    Lists ch = children_of(etree);
    V stack;
    stack.reserve(n);
    stack.push_back(n - 1);
    int32_t p = n - 1;
    while (!stack.empty()) {
      int32_t node = stack.back();
      stack.pop_back();
      post[p--] = node;
      for (int32_t k = ch.off[node]; k < ch.off[node + 1]; k++) stack.push_back(ch.v[k]);
    }
    for (int32_t i = 0; i < n; i++) ipost[post[i]] = i;
  }
  Lists pccs = permute_columns(reo, post, ipost, nullptr);
  V pparent(n, -1);
  for (int32_t i = 0; i < n - 1; i++) pparent[i] = ipost[etree[post[i]]];
  Lists ptc = children_of(pparent);

  // ---- column counts (column_count_m.f90:9-72) ----
  V cc(n, 0);
  {
    LabeledSets ds(n);
    V prev(n, -1), lca(pccs.v.size(), -1);
    for (int32_t j = 0; j < n - 1; j++) {
      for (int32_t k = pccs.off[j] + 1; k < pccs.off[j + 1]; k++) {
        int32_t r = pccs.v[k], pp = prev[r];
        lca[k] = pp >= 0 ? ds.find(pp) : -1;
        prev[r] = j;
      }
      ds.merge_into(j, pparent[j]);
    }
    for (int32_t i = 0; i < n; i++) cc[i] = ptc.len(i) == 0 ? 1 : 0;
    for (int32_t j = 0; j < n; j++) {
      if (j != n - 1) cc[pparent[j]]--;
      for (int32_t k = pccs.off[j] + 1; k < pccs.off[j + 1]; k++) {
        cc[j]++;
        if (lca[k] >= 0) cc[lca[k]]--;
      }
    }
    for (int32_t i = 0; i < n - 1; i++) cc[pparent[i]] += cc[i];
  }

  // ---- fundamental supernodes (analyse_phase_m.f90:73-89) ----
  V fsets;        // first column of every fundamental supernode, plus n
  V fcc;          // supernodal column counts
  V fnum_child;
  {
    V sub(n, 1), isleaf(n, 0), prev(n, -1);
    for (int32_t i = 0; i < n; i++)
      for (int32_t k = ptc.off[i]; k < ptc.off[i + 1]; k++) sub[i] += sub[ptc.v[k]];
    for (int32_t j = 0; j < n; j++) {
      int32_t first_desc = j - sub[j] + 1;
      for (int32_t k = pccs.off[j] + 1; k < pccs.off[j + 1]; k++) {
        int32_t r = pccs.v[k];
        if (prev[r] < first_desc) isleaf[j] = 1;
        prev[r] = j;
      }
    }
    for (int32_t i = 0; i < n; i++)
      if (isleaf[i] > 0 || ptc.len(i) > 1 || i == 0) fsets.push_back(i);
    fsets.push_back(n);
    int32_t nf = (int32_t)fsets.size() - 1;
    fcc.resize(nf);
    fnum_child.resize(nf);
    for (int32_t s = 0; s < nf; s++) {
      fcc[s] = cc[fsets[s + 1] - 1] - 1;
      fnum_child[s] = ptc.len(fsets[s]);
    }
  }
  const int32_t nfund = (int32_t)fsets.size() - 1;
  V fparent = parent_from_child_counts(fnum_child);
  Lists ftc = children_of(fparent);

  // ---- relaxed supernodes (relax_supernode_m.f90:13-90, relaxed_supernode_m.f90) ----
  NodeLists merge(nfund), sons(nfund);
  for (int32_t i = 0; i < nfund; i++) merge.add(i, i);
  {
    V ncol(nfund), nzero(nfund, 0), stack;
    for (int32_t i = 0; i < nfund; i++) ncol[i] = fsets[i + 1] - fsets[i];
    for (int32_t k = 0; k < nfund; k++) {
      if (ftc.len(k) == 0) continue;
      for (int32_t t = ftc.off[k]; t < ftc.off[k + 1]; t++) sons.add(ftc.v[t], k);
      for (;;) {
        int32_t best = -1, min_zero = max_zero;
        for (int32_t c = sons.head[k]; c >= 0; c = sons.next[c]) {
          int64_t add = (int64_t)(fcc[k] + ncol[k] - fcc[c]) * ncol[c] + nzero[k] + nzero[c];
          if (add <= min_zero && add <= max_zero) { best = c; min_zero = (int32_t)add; }
        }
        if (best >= 0) {
          merge.append(best, k);
          sons.remove(best, k);
          stack.push_back(best);
          nzero[k] = min_zero;
          ncol[k] += ncol[best];
        } else {
          while (!stack.empty()) { sons.append(stack.back(), k); stack.pop_back(); }
          break;
        }
      }
    }
  }
  V map;
  for (int32_t i = 0; i < nfund; i++)
    if (merge.head[i] >= 0) map.push_back(i);
  const int32_t nrel = (int32_t)map.size();
  V rsets(nrel + 1, 0), rperm(n), rnum_child(nrel), rcc(nrel);
  {
    int32_t p = 0;
    V stack;
    for (int32_t i = 0; i < nrel; i++) {
      int32_t cols = 0;
      for (int32_t x = merge.head[map[i]]; x >= 0; x = merge.next[x]) { stack.push_back(x); cols += fsets[x + 1] - fsets[x]; }
      rsets[i + 1] = rsets[i] + cols;
      while (!stack.empty()) {
        int32_t node = stack.back();
        stack.pop_back();
        for (int32_t j = fsets[node]; j < fsets[node + 1]; j++) rperm[p++] = j;
      }
      rnum_child[i] = sons.length(map[i]);
      rcc[i] = fcc[map[i]];
    }
  }
  V rparent = parent_from_child_counts(rnum_child);
  Lists rtc = children_of(rparent);
  V irperm(n);
  for (int32_t i = 0; i < n; i++) irperm[rperm[i]] = i;
  Lists rccs = permute_columns(pccs, rperm, irperm, nullptr);

  // ---- supernodal L structure (fundamental_supernode_m.f90:72-119, symbolic_factorize_m.f90:10-62) ----
  Lists L;
  {
    V len(rcc.begin(), rcc.end());
    L = lists_from_lengths(len);
    V mark(n, -1);
    for (int32_t k = 0; k < nrel; k++) {
      int32_t last = rsets[k + 1] - 1, p = 0;
      int32_t* out_rows = L.at(k);
      for (int32_t j = rsets[k]; j <= last; j++)
        for (int32_t t = rccs.off[j]; t < rccs.off[j + 1]; t++) {
          int32_t r = rccs.v[t];
          if (r <= last || mark[r] == k) continue;
          if (p >= L.len(k)) return -1;
          mark[r] = k;
          out_rows[p++] = r;
        }
      for (int32_t t = rtc.off[k]; t < rtc.off[k + 1]; t++) {
        int32_t c = rtc.v[t];
        for (int32_t q = L.off[c]; q < L.off[c + 1]; q++) {
          int32_t r = L.v[q];
          if (r <= last || mark[r] == k) continue;
          if (p >= L.len(k)) return -1;
          mark[r] = k;
          out_rows[p++] = r;
        }
      }
      if (p != L.len(k)) return -1;
      std::sort(out_rows, out_rows + p);
    }
  }

  // ---- compose permutations and the permuted A structure (hppllt.f90:56-71) ----
  V aperm(n), aiperm(n);
  for (int32_t i = 0; i < n; i++) aperm[i] = post[rperm[i]];
  for (int32_t i = 0; i < n; i++) aiperm[aperm[i]] = i;
  V asrc;
  Lists astr = permute_columns(reo, aperm, aiperm, &asrc);

  out.n = n;
  out.nnz = nnz;
  out.num_node = nrel;
  out.node_ptr.resize(nrel + 1);
  for (int32_t i = 0; i <= nrel; i++) out.node_ptr[i] = rsets[i] + 1;
  out.parent.resize(nrel);
  for (int32_t i = 0; i < nrel; i++) out.parent[i] = rparent[i] + 1;     // root -> 0
  out.lrow_ptr.resize(nrel + 1);
  for (int32_t i = 0; i <= nrel; i++) out.lrow_ptr[i] = L.off[i] + 1;
  out.lrow.resize(L.v.size());
  for (size_t i = 0; i < L.v.size(); i++) out.lrow[i] = L.v[i] + 1;
  out.acol_ptr.resize(n + 1);
  for (int32_t i = 0; i <= n; i++) out.acol_ptr[i] = astr.off[i] + 1;
  out.arow.resize(nnz);
  for (int32_t k = 0; k < nnz; k++) out.arow[k] = astr.v[k] + 1;
  out.ccs_perm.resize(nnz);
  for (int32_t k = 0; k < nnz; k++) out.ccs_perm[k] = (order_perm ? reo_src[asrc[k]] : asrc[k]) + 1;
  out.perm.resize(n);
  for (int32_t i = 0; i < n; i++) out.perm[i] = (order_perm ? reo_perm[aperm[i]] : aperm[i]) + 1;
  return 0;
}

}  // namespace mfd
