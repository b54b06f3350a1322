// Subtree partition of the supernodal elimination tree for p workers (GPUs):
// the reference's tree_pruning (src/main/algorithms/tree_pruning_m.f90:13-155),
// restated.  It is the mapping step of a multi-GPU factorization of one
// system: each returned subtree is factored by one GPU, the fronts above the
// subtrees by the GPU that receives the subtree roots' update matrices.
//
//   cost of node i     fcnt(i) = sum_{k=cc(i)+1}^{cc(i)+size(i)} k^2     (count_op_count, :75-88)
//   subtree weight     nodewt(i) = fcnt(i) + sum over children            (generate_tree_weights, :90-109)
//   start              the list holds the root (node n)
//   for ip = p, p+1, ...:
//     partition_tree   while the list has fewer than ip entries, replace the
//                      entry of largest weight (the first one met from the
//                      head, strict comparison) by its children, each added
//                      at the head in child order (:111-132, :134-151)
//     balance          the list's weights into ip bins, largest first into the
//                      lightest bin; stop when min bin / max bin > tol (:38-61)
//   result             the list from its head (:63-69)
// When no entry can be split (the weights are all zero) the reference
// restarts with tol = 0 and p = ip - 1 (:46-50); so does this.  Weights are
// 64-bit here (the reference's default integers overflow beyond fronts of
// about 1,300 rows).
#include <algorithm>
#include <cstdint>
#include <functional>
#include <queue>
#include <vector>

namespace mfd {

namespace {

// the reference's doubly linked list (doubly_linked_list_m.f90): add at the
// head, remove anywhere, iterate from the head
struct NodeList {
  std::vector<int32_t> next, prev;
  int32_t head = 0;
  explicit NodeList(int32_t n) : next(n + 1, 0), prev(n + 1, 0) {}
  void add(int32_t v) {
    if (head != 0) prev[head] = v;
    next[v] = head;
    head = v;
    prev[v] = 0;
  }
  void remove(int32_t v) {
    const int32_t nx = next[v], pv = prev[v];
    if (pv == 0) head = nx;
    else next[pv] = nx;
    if (nx != 0) prev[nx] = pv;
  }
  int32_t length() const {
    int32_t c = 0;
    for (int32_t v = head; v != 0; v = next[v]) ++c;
    return c;
  }
};

}  // namespace

// node_size, cc (nr), num_child: num_node entries; child: the children of
// node 1, then node 2, ... (1-based).  Returns the subtree roots (1-based) in
// list order; an empty result means bad input.
std::vector<int32_t> subtree_partition(int32_t num_node, const int32_t* node_size, const int32_t* cc,
                                       const int32_t* num_child, const int32_t* child, double tol, int32_t p) {
  std::vector<int32_t> out;
  if (num_node < 1 || p < 1) return out;
  std::vector<int64_t> cptr(num_node + 1, 0);
  for (int32_t i = 0; i < num_node; ++i) {
    if (num_child[i] < 0) return out;
    cptr[i + 1] = cptr[i] + num_child[i];
  }
  for (int64_t k = 0; k < cptr[num_node]; ++k)
    if (child[k] < 1 || child[k] > num_node) return out;
  std::vector<int64_t> fcnt(num_node), nodewt(num_node + 1, 0);
  for (int32_t i = 0; i < num_node; ++i) {
    const int64_t l = cc[i], k = node_size[i] + l;
    fcnt[i] = k * (k + 1) * (2 * k + 1) / 6 - l * (l + 1) * (2 * l + 1) / 6;
  }
  for (int32_t i = 1; i <= num_node; ++i) {              // children precede parents (postorder)
    nodewt[i] = fcnt[i - 1];
    for (int64_t k = cptr[i - 1]; k < cptr[i]; ++k) nodewt[i] += nodewt[child[k]];
  }
  for (;;) {
    NodeList list(num_node);
    list.add(num_node);
    double ratio = 0.0;
    int32_t ip = p - 1;
    bool stuck = false;
    while (ratio <= tol) {
      ++ip;
      while (list.length() < ip) {                        // partition_tree
        int32_t best = 0;
        int64_t bw = 0;
        for (int32_t v = list.head; v != 0; v = list.next[v])
          if (nodewt[v] > bw) {
            bw = nodewt[v];
            best = v;
          }
        if (best == 0) {
          stuck = true;
          break;
        }
        for (int64_t k = cptr[best - 1]; k < cptr[best]; ++k) list.add(child[k]);
        list.remove(best);
      }
      if (stuck) break;
      std::vector<int64_t> w;                             // LPT: heaviest first into the lightest bin
      for (int32_t v = list.head; v != 0; v = list.next[v]) w.push_back(nodewt[v]);
      std::sort(w.begin(), w.end(), std::greater<int64_t>());
      std::priority_queue<int64_t, std::vector<int64_t>, std::greater<int64_t>> bins;
      for (int32_t b = 0; b < ip; ++b) bins.push(0);
      for (int64_t x : w) {
        const int64_t top = bins.top();
        bins.pop();
        bins.push(top + x);
      }
      int64_t mn = bins.top(), mx = 0;
      while (!bins.empty()) {
        mx = std::max(mx, bins.top());
        bins.pop();
      }
      ratio = mx > 0 ? (double)mn / (double)mx : 0.0;
    }
    if (stuck) {                                          // the reference's restart (:46-50)
      if (ip - 1 < 1 || (tol == 0.0 && ip - 1 == p)) {
        for (int32_t v = list.head; v != 0; v = list.next[v]) out.push_back(v);
        return out;
      }
      tol = 0.0;
      p = ip - 1;
      continue;
    }
    for (int32_t v = list.head; v != 0; v = list.next[v]) out.push_back(v);
    return out;
  }
}

}  // namespace mfd
