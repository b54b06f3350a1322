/*
 * mfdag_oracle.c -- CPU restatement of the reference solver (to-mo-ki/multifrontal-DAG)
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke check
 * and the CPU-baseline leg of bench.py call it to produce the answers the GPU
 * path must reproduce.  Nothing in the product links or calls it.
 *
 * It restates, function by function, the reference's
 *   - symbolic analysis      (src/main/analyse_phase_m.f90, algorithms/*, data_structure_creators/*,
 *                             storage_converter/*, hppllt.f90:24-106)
 *   - index / layout layer   (node_data_m.f90, factors/*, right_hand/*, block_local_index_*_m.f90,
 *                             integer_function_m.f90)
 *   - sequential numeric path (zero_setter_m.f90, coefficient_setter_m.f90, seq_factorize/**,
 *                             seq_solve/**, perm_m.f90)
 * Every integer array holds the reference's 1-based values; C storage is 0-based,
 * so element k (1-based) of x is x[k-1].  Dense kernels restate the LAPACK/BLAS
 * routines the reference calls (DPOTRF "U", DTRSM "L,U,T,N", DSYRK "U,T",
 * DGEMM "T,N", DTRSV "U,T/N", DGEMV "T/N") as plain loops; optionally the
 * baseline leg swaps in a system BLAS (OpenBLAS) through orc_use_blas().
 *
 * Parity of this file is pinned by the reference's own unit tests (golden
 * vectors transcribed into tests/golden/reference_vectors.py).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <dlfcn.h>
#include <stdio.h>
#include <pthread.h>
#include <unistd.h>

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------- */
/* containers: contiguous_sets_m.f90 / jagged_array_m.f90                     */
/* ------------------------------------------------------------------------- */
typedef struct {
  int n;      /* number of arrays */
  int *ptr;   /* n+1 entries, ptr[0] = 1 (1-based, as contiguous_sets_c%ptr) */
  int *val;   /* ptr[n]-1 entries */
} jag_t;

static void *xmalloc(size_t n) { void *p = malloc(n ? n : 1); if (!p) abort(); return p; }
static void *xcalloc(size_t n, size_t s) { void *p = calloc(n ? n : 1, s ? s : 1); if (!p) abort(); return p; }

static int *ja(const jag_t *j, int i) { return j->val + (j->ptr[i - 1] - 1); } /* array i (1-based) */
static int jl(const jag_t *j, int i) { return j->ptr[i] - j->ptr[i - 1]; }
static int jtot(const jag_t *j) { return j->ptr[j->n] - 1; }

/* create_contiguous_sets (contiguous_sets_m.f90:18-31) */
static int *sets_from_lengths(int n, const int *len) {
  int *p = xmalloc(sizeof(int) * (n + 1));
  p[0] = 1;
  for (int i = 0; i < n; i++) p[i + 1] = p[i] + len[i];
  return p;
}
static jag_t jag_new(int n, const int *len) {
  jag_t j; j.n = n; j.ptr = sets_from_lengths(n, len);
  j.val = xcalloc(j.ptr[n] - 1, sizeof(int));
  return j;
}
static jag_t jag_same_shape(const jag_t *s) {
  jag_t j; j.n = s->n; j.ptr = xmalloc(sizeof(int) * (s->n + 1));
  memcpy(j.ptr, s->ptr, sizeof(int) * (s->n + 1));
  j.val = xcalloc(jtot(s), sizeof(int));
  return j;
}
static jag_t jag_copy(const jag_t *s) {
  jag_t j = jag_same_shape(s);
  memcpy(j.val, s->val, sizeof(int) * jtot(s));
  return j;
}
static void jag_free(jag_t *j) { free(j->ptr); free(j->val); j->ptr = NULL; j->val = NULL; }

/* ------------------------------------------------------------------------- */
/* integer_function_m.f90                                                     */
/* ------------------------------------------------------------------------- */
static int64_t psum1(int64_t e) { return e < 1 ? 0 : e * (e + 1) / 2; }          /* :199-206 */
static int64_t psum2(int64_t s, int64_t e) { return e < s ? 0 : psum1(e) - psum1(s - 1); } /* :208-215 */
static int64_t psqsum(int64_t s, int64_t e) {                                   /* :218-229 */
  int64_t r = 0; if (e < s) return 0;
  for (int64_t i = s; i <= e; i++) r += i * i;
  return r;
}
static int div_ceiling(int a, int p) { return (a - 1) / p + 1; }                 /* :231-234 */
static int mod2(int a, int p) { return (a - 1) % p + 1; }                        /* :236-239 */

/* ------------------------------------------------------------------------- */
/* disjoint_set_m.f90 (union by rank with separate "real root" bookkeeping)   */
/* ------------------------------------------------------------------------- */
typedef struct { int *parent, *realroot, *vroot, *rank; } dset_t;
static dset_t dset_new(int n) {
  dset_t d; d.parent = xmalloc(sizeof(int) * n); d.realroot = xmalloc(sizeof(int) * n);
  d.vroot = xmalloc(sizeof(int) * n); d.rank = xcalloc(n, sizeof(int));
  for (int i = 0; i < n; i++) { d.parent[i] = i + 1; d.realroot[i] = i + 1; d.vroot[i] = i + 1; }
  return d;
}
static void dset_free(dset_t *d) { free(d->parent); free(d->realroot); free(d->vroot); free(d->rank); }
static int dset_find2(dset_t *d, int idx) {                    /* :41-48, path compression */
  int r = idx;
  while (d->parent[r - 1] != r) r = d->parent[r - 1];
  while (d->parent[idx - 1] != r) { int nx = d->parent[idx - 1]; d->parent[idx - 1] = r; idx = nx; }
  return r;
}
static int dset_find(dset_t *d, int idx) { return d->realroot[dset_find2(d, idx) - 1]; } /* :32-39 */
static void dset_link(dset_t *d, int node, int parent) {       /* :50-69 */
  int nv = d->vroot[node - 1], pv = d->vroot[parent - 1];
  if (d->rank[parent - 1] > d->rank[node - 1]) {
    d->parent[nv - 1] = pv;
  } else if (d->rank[parent - 1] < d->rank[node - 1]) {
    d->parent[pv - 1] = nv;
    d->realroot[nv - 1] = d->realroot[pv - 1];
    d->vroot[parent - 1] = nv;
  } else {
    d->parent[nv - 1] = pv;
    d->rank[parent - 1] += 1;
  }
}

/* ------------------------------------------------------------------------- */
/* storage_converter/ccs_to_crs_m.f90:9-43                                   */
/* ------------------------------------------------------------------------- */
static jag_t ccs_to_crs(const jag_t *ccs) {
  int n = ccs->n;
  int *num = xcalloc(n, sizeof(int));
  for (int j = 1; j <= n; j++) { int *r = ja(ccs, j); for (int i = 0; i < jl(ccs, j); i++) num[r[i] - 1]++; }
  jag_t crs = jag_new(n, num);
  int *rp = xmalloc(sizeof(int) * n);
  for (int i = 0; i < n; i++) rp[i] = 1;
  for (int j = 1; j <= n; j++) {
    int *r = ja(ccs, j);
    for (int i = 0; i < jl(ccs, j); i++) { int row = r[i]; ja(&crs, row)[rp[row - 1] - 1] = j; rp[row - 1]++; }
  }
  free(num); free(rp);
  return crs;
}

/* ------------------------------------------------------------------------- */
/* algorithms/compute_tree_m.f90:10-35  (elimination tree)                    */
/* ------------------------------------------------------------------------- */
static int *compute_tree(const jag_t *crs) {
  int n = crs->n;
  int *parent = xcalloc(n, sizeof(int));
  dset_t d = dset_new(n);
  for (int i = 1; i <= n; i++) {
    parent[i - 1] = 0;
    int *cols = ja(crs, i);
    for (int k = 0; k < jl(crs, i) - 1; k++) {
      int t = dset_find(&d, cols[k]);
      if (parent[t - 1] == 0 && t != i) { parent[t - 1] = i; dset_link(&d, t, i); }
    }
  }
  dset_free(&d);
  return parent;
}

/* ------------------------------------------------------------------------- */
/* data_structure_creators/tree_m.f90                                         */
/* ------------------------------------------------------------------------- */
static jag_t tree_child_by_num_child_and_parent(int n, const int *num_child, const int *parent) { /* :15-37 */
  jag_t tc = jag_new(n, num_child);
  int *cp = xmalloc(sizeof(int) * n);
  for (int i = 0; i < n; i++) cp[i] = 1;
  for (int i = 1; i <= n; i++) {
    int p = parent[i - 1]; if (p == 0) continue;
    ja(&tc, p)[cp[p - 1] - 1] = i; cp[p - 1]++;
  }
  free(cp);
  return tc;
}
static jag_t tree_child_by_parent(int n, const int *parent) {                  /* :39-55 */
  int *nc = xcalloc(n, sizeof(int));
  for (int i = 1; i <= n - 1; i++) nc[parent[i - 1] - 1]++;
  jag_t tc = tree_child_by_num_child_and_parent(n, nc, parent);
  free(nc);
  return tc;
}
static int *parent_in_postordering_tree(int n, const int *num_child) {         /* :57-76 */
  int *parent = xcalloc(n, sizeof(int)), *stack = xmalloc(sizeof(int) * n), sp = 0;
  for (int i = 1; i <= n; i++) {
    for (int j = 0; j < num_child[i - 1]; j++) { int node = stack[--sp]; parent[node - 1] = i; }
    stack[sp++] = i;
  }
  free(stack);
  return parent;
}
static int *tree_traverse_postordering(const jag_t *tc) {                       /* :78-99 */
  int n = tc->n, ptr = n, sp = 0;
  int *perm = xmalloc(sizeof(int) * n), *stack = xmalloc(sizeof(int) * n);
  stack[sp++] = n;
  while (sp > 0) {
    int node = stack[--sp];
    perm[ptr - 1] = node; ptr--;
    int *ch = ja(tc, node);
    for (int i = 0; i < jl(tc, node); i++) stack[sp++] = ch[i];
  }
  free(stack);
  return perm;
}
static int *count_subtree_size(const jag_t *tc) {                               /* :101-116 */
  int n = tc->n; int *s = xmalloc(sizeof(int) * n);
  for (int i = 1; i <= n; i++) {
    s[i - 1] = 1; int *ch = ja(tc, i);
    for (int j = 0; j < jl(tc, i); j++) s[i - 1] += s[ch[j] - 1];
  }
  return s;
}
static int *create_parent(const jag_t *tc) {                                    /* :118-134 */
  int n = tc->n; int *p = xcalloc(n, sizeof(int));
  p[n - 1] = 0;
  for (int node = 1; node <= n; node++) { int *ch = ja(tc, node); for (int i = 0; i < jl(tc, node); i++) p[ch[i] - 1] = node; }
  return p;
}

/* ------------------------------------------------------------------------- */
/* data_structure_creators/perm_m.f90                                         */
/* ------------------------------------------------------------------------- */
static int *set_iperm(int n, const int *perm) {                                 /* :11-24 */
  int *ip = xmalloc(sizeof(int) * n);
  for (int i = 1; i <= n; i++) ip[perm[i - 1] - 1] = i;
  return ip;
}
static int *perm_product(int n, const int *first, const int *second) {         /* :26-37 */
  int *o = xmalloc(sizeof(int) * n);
  for (int i = 0; i < n; i++) o[i] = first[second[i] - 1];
  return o;
}

/* ------------------------------------------------------------------------- */
/* data_structure_creators/reordering_m.f90 + sort_m.f90                      */
/* ------------------------------------------------------------------------- */
static int *reordering_tree(int n, const int *parent, const int *perm, const int *iperm) { /* :17-29 */
  int *p = xmalloc(sizeof(int) * n);
  for (int i = 1; i <= n - 1; i++) p[i - 1] = iperm[parent[perm[i - 1] - 1] - 1];
  p[n - 1] = 0;
  return p;
}
/* repostordering_ccs1/2 (:31-96); ccs_perm may be NULL */
static jag_t repostordering_ccs(const jag_t *ccs, const int *perm, const int *iperm, int **ccs_perm) {
  int n = ccs->n;
  int *num = xmalloc(sizeof(int) * n);
  for (int c = 1; c <= n; c++) num[c - 1] = jl(ccs, perm[c - 1]);
  jag_t out = jag_new(n, num);
  int *pj = ccs_perm ? xmalloc(sizeof(int) * (jtot(&out) ? jtot(&out) : 1)) : NULL;
  int offset = 0;
  for (int co = 1; co <= n; co++) {
    int cr = iperm[co - 1];
    int *ro = ja(ccs, co), *rr = ja(&out, cr);
    int len = jl(&out, cr);
    for (int i = 0; i < len; i++) {
      rr[i] = iperm[ro[i] - 1];
      if (pj) pj[(out.ptr[cr - 1] - 1) + i] = offset + i + 1;
    }
    offset += len;
  }
  free(num);
  if (ccs_perm) *ccs_perm = pj;
  return out;
}
/* sort_with_perm (sort_m.f90:24-37): bubble sort, stable; restated as insertion
 * sort, which performs the same adjacent swaps and so yields the same result */
static void sort_with_perm(int *a, int *p, int n) {
  for (int i = 1; i < n; i++) {
    int j = i;
    while (j > 0 && a[j - 1] > a[j]) {
      int t = a[j - 1]; a[j - 1] = a[j]; a[j] = t;
      if (p) { t = p[j - 1]; p[j - 1] = p[j]; p[j] = t; }
      j--;
    }
  }
}
/* reordering_ccs (:98-148): apply an external symmetric ordering and map to lower triangle */
static jag_t reordering_ccs(const jag_t *ccs, const int *perm, const int *iperm, int **ccs_perm) {
  (void)perm;
  int n = ccs->n;
  int *num = xcalloc(n, sizeof(int));
  for (int j = 1; j <= n; j++) {
    int *r = ja(ccs, j);
    for (int i = 0; i < jl(ccs, j); i++) {
      int a = iperm[j - 1], b = iperm[r[i] - 1];
      num[(a < b ? a : b) - 1]++;
    }
  }
  jag_t out = jag_new(n, num);
  jag_t pj = jag_same_shape(&out);
  int *ptr = xmalloc(sizeof(int) * n);
  for (int i = 0; i < n; i++) ptr[i] = 1;
  int offset = 0;
  for (int j = 1; j <= n; j++) {
    int *r = ja(ccs, j);
    for (int i = 0; i < jl(ccs, j); i++) {
      int a = iperm[j - 1], b = iperm[r[i] - 1];
      int col = a < b ? a : b, row = a < b ? b : a;
      ja(&out, col)[ptr[col - 1] - 1] = row;
      ja(&pj, col)[ptr[col - 1] - 1] = offset + i + 1;
      ptr[col - 1]++;
    }
    offset += jl(ccs, j);
  }
  for (int j = 1; j <= n; j++) sort_with_perm(ja(&out, j), ja(&pj, j), jl(&out, j));
  free(num); free(ptr);
  *ccs_perm = pj.val; free(pj.ptr);
  return out;
}

/* ------------------------------------------------------------------------- */
/* algorithms/column_count_m.f90:9-72                                         */
/* ------------------------------------------------------------------------- */
static int *column_count(const jag_t *ccs, const jag_t *tc, const int *parent) {
  int n = ccs->n;
  dset_t d = dset_new(n);
  jag_t lca = jag_same_shape(ccs);
  int *prev_p = xcalloc(n, sizeof(int));
  for (int j = 1; j <= n - 1; j++) {
    int *rows = ja(ccs, j), *lr = ja(&lca, j);
    for (int i = 1; i < jl(ccs, j); i++) {
      int pp = prev_p[rows[i] - 1];
      lr[i] = pp != 0 ? dset_find(&d, pp) : 0;
      prev_p[rows[i] - 1] = j;
    }
    dset_link(&d, j, parent[j - 1]);
  }
  int *wt = xmalloc(sizeof(int) * n);
  for (int i = 1; i <= n; i++) wt[i - 1] = jl(tc, i) == 0 ? 1 : 0;
  for (int j = 1; j <= n; j++) {
    if (j != n) wt[parent[j - 1] - 1]--;
    int *lr = ja(&lca, j);
    for (int i = 1; i < jl(ccs, j); i++) {
      wt[j - 1]++;
      if (lr[i] != 0) wt[lr[i] - 1]--;
    }
  }
  for (int i = 1; i <= n - 1; i++) wt[parent[i - 1] - 1] += wt[i - 1];
  dset_free(&d); jag_free(&lca); free(prev_p);
  return wt;
}

/* ------------------------------------------------------------------------- */
/* algorithms/finding_leaves_m.f90:6-29                                       */
/* ------------------------------------------------------------------------- */
static int *finding_leaves(const int *subtree_size, const jag_t *ccs) {
  int n = ccs->n;
  int *isleaf = xcalloc(n, sizeof(int)), *prev = xcalloc(n, sizeof(int));
  for (int j = 1; j <= n; j++) {
    int *rows = ja(ccs, j);
    for (int i = 1; i < jl(ccs, j); i++) {
      if (prev[rows[i] - 1] < j - subtree_size[j - 1] + 1) isleaf[j - 1] = 1;
      prev[rows[i] - 1] = j;
    }
  }
  free(prev);
  return isleaf;
}

/* ------------------------------------------------------------------------- */
/* data_structure_creators/fundamental_supernode_m.f90                        */
/* ------------------------------------------------------------------------- */
static int *search_node_sets(const int *isleaf, const jag_t *tc, int *num_sets) { /* :11-40 -> sets ptr */
  int n = tc->n, count = 0;
  for (int i = 1; i <= n; i++) if (isleaf[i - 1] > 0 || jl(tc, i) > 1) count++;
  int *num = xcalloc(count, sizeof(int)), p = 0;
  for (int i = 1; i <= n; i++) {
    if (isleaf[i - 1] > 0 || jl(tc, i) > 1) p++;
    num[p - 1]++;   /* p == 0 here would be an out-of-bounds write in the reference too */
  }
  int *sets = sets_from_lengths(count, num);
  free(num);
  *num_sets = count;
  return sets;
}
static int *supernodal_column_count(int ns, const int *sets, const int *cc) {   /* :42-55 */
  int *o = xmalloc(sizeof(int) * ns);
  for (int i = 1; i <= ns; i++) o[i - 1] = cc[(sets[i] - 1) - 1] - 1;
  return o;
}
static int *supernodal_tree(int ns, const int *sets, const jag_t *tc) {         /* :57-69 */
  int *o = xmalloc(sizeof(int) * ns);
  for (int i = 1; i <= ns; i++) o[i - 1] = jl(tc, sets[i - 1]);
  return o;
}
static jag_t supernodal_ccs(int ns, const int *sets, const jag_t *ccs) {        /* :72-119 */
  int n = ccs->n;
  int *num = xcalloc(ns, sizeof(int)), *full = xcalloc(n, sizeof(int));
  for (int k = 1; k <= ns; k++) {
    int last = sets[k] - 1;
    for (int j = sets[k - 1]; j <= last; j++) {
      int *r = ja(ccs, j);
      for (int i = 0; i < jl(ccs, j); i++) {
        int row = r[i];
        if (row <= last || full[row - 1] == k) continue;
        full[row - 1] = k; num[k - 1]++;
      }
    }
  }
  jag_t out = jag_new(ns, num);
  memset(full, 0, sizeof(int) * n);
  for (int k = 1; k <= ns; k++) {
    int last = sets[k] - 1, p = 0; int *o = ja(&out, k);
    for (int j = sets[k - 1]; j <= last; j++) {
      int *r = ja(ccs, j);
      for (int i = 0; i < jl(ccs, j); i++) {
        int row = r[i];
        if (row <= last || full[row - 1] == k) continue;
        full[row - 1] = k; o[p++] = row;
      }
    }
  }
  free(num); free(full);
  return out;
}

/* ------------------------------------------------------------------------- */
/* doubly_linked_lists_m.f90 (head/tail per list, shared next/prev arrays)    */
/* ------------------------------------------------------------------------- */
typedef struct { int n; int *head, *tail, *next, *prev; } dll_t;
static dll_t dll_new(int n) {
  dll_t l; l.n = n; l.head = xcalloc(n, sizeof(int)); l.tail = xcalloc(n, sizeof(int));
  l.next = xcalloc(n, sizeof(int)); l.prev = xcalloc(n, sizeof(int));
  return l;
}
static void dll_free(dll_t *l) { free(l->head); free(l->tail); free(l->next); free(l->prev); }
static void dll_add(dll_t *l, int node, int idx) {                              /* :103-116 */
  if (l->head[idx - 1] == 0) { l->head[idx - 1] = node; l->tail[idx - 1] = node; }
  else { l->prev[node - 1] = l->tail[idx - 1]; l->next[l->tail[idx - 1] - 1] = node; l->tail[idx - 1] = node; }
}
static void dll_merge(dll_t *l, int from, int to) {                             /* :118-135 */
  if (l->head[from - 1] == 0) return;
  if (l->head[to - 1] == 0) { l->head[to - 1] = l->head[from - 1]; l->tail[to - 1] = l->tail[from - 1]; }
  else { l->next[l->tail[to - 1] - 1] = l->head[from - 1]; l->tail[to - 1] = l->tail[from - 1]; }
  l->head[from - 1] = 0; l->tail[from - 1] = 0;
}
static void dll_remove(dll_t *l, int node, int idx) {                           /* :137-160 */
  int nx = l->next[node - 1], pv = l->prev[node - 1];
  if (node == l->head[idx - 1]) l->head[idx - 1] = nx; else l->next[pv - 1] = nx;
  if (node == l->tail[idx - 1]) l->tail[idx - 1] = pv; else l->prev[nx - 1] = pv;
  l->next[node - 1] = 0; l->prev[node - 1] = 0;
}
static int dll_length(const dll_t *l, int idx) {                                /* :162-175 */
  int c = 0; for (int x = l->head[idx - 1]; x != 0; x = l->next[x - 1]) c++;
  return c;
}

/* ------------------------------------------------------------------------- */
/* algorithms/relax_supernode_m.f90:13-90                                     */
/* num_zeros is allocated but never initialised in the reference (:36); it is */
/* read as zero here, which is what a freshly mapped allocation holds.        */
/* ------------------------------------------------------------------------- */
static void compute_merge_lists(int n, const int *cc, const jag_t *tc, const int *sets, int max_zero,
                                dll_t *merge_lists, dll_t *son_lists) {
  *son_lists = dll_new(n); *merge_lists = dll_new(n);
  for (int i = 1; i <= n; i++) dll_add(merge_lists, i, i);
  int *ncol = xmalloc(sizeof(int) * n), *nzero = xcalloc(n, sizeof(int));
  for (int i = 1; i <= n; i++) ncol[i - 1] = sets[i] - sets[i - 1];
  int *stack = xmalloc(sizeof(int) * n), sp = 0;
  for (int k = 1; k <= n; k++) {
    if (jl(tc, k) == 0) continue;
    int *ch = ja(tc, k);
    for (int j = 0; j < jl(tc, k); j++) dll_add(son_lists, ch[j], k);
    for (;;) {
      /* choose_merge_node (:66-85) */
      int min_zero = max_zero, merge_node = 0;
      for (int c = son_lists->head[k - 1]; c != 0; c = son_lists->next[c - 1]) {
        int add = (cc[k - 1] + ncol[k - 1] - cc[c - 1]) * ncol[c - 1] + nzero[k - 1] + nzero[c - 1];
        if (add <= min_zero && add <= max_zero) { merge_node = c; min_zero = add; }
      }
      if (merge_node != 0) {
        dll_merge(merge_lists, merge_node, k);
        dll_remove(son_lists, merge_node, k);
        stack[sp++] = merge_node;
        nzero[k - 1] = min_zero;
        ncol[k - 1] += ncol[merge_node - 1];
      } else {
        while (sp > 0) { int m = stack[--sp]; dll_merge(son_lists, m, k); }
        break;
      }
    }
  }
  free(ncol); free(nzero); free(stack);
}

/* ------------------------------------------------------------------------- */
/* data_structure_creators/relaxed_supernode_m.f90                            */
/* ------------------------------------------------------------------------- */
static int *build_map(const dll_t *ml, int *num_lists) {                         /* :136-152 */
  int cnt = 0;
  for (int i = 1; i <= ml->n; i++) if (ml->head[i - 1] != 0) cnt++;
  int *map = xmalloc(sizeof(int) * (cnt ? cnt : 1)), p = 0;
  for (int i = 1; i <= ml->n; i++) if (dll_length(ml, i) > 0) map[p++] = i;
  *num_lists = cnt;
  return map;
}
static int *relaxed_node_sets(const int *fsets, int nmap, const int *map, const dll_t *ml) { /* :185-206 */
  int *num = xcalloc(nmap, sizeof(int));
  for (int i = 1; i <= nmap; i++)
    for (int x = ml->head[map[i - 1] - 1]; x != 0; x = ml->next[x - 1]) num[i - 1] += fsets[x] - fsets[x - 1];
  int *s = sets_from_lengths(nmap, num);
  free(num);
  return s;
}
static int *relaxed_perm(int nfund, const int *fsets, int nmap, const int *map, const dll_t *ml, int order) { /* :154-183 */
  int *perm = xmalloc(sizeof(int) * order), *stack = xmalloc(sizeof(int) * nfund), sp = 0, p = 1;
  for (int i = 1; i <= nmap; i++) {
    for (int x = ml->head[map[i - 1] - 1]; x != 0; x = ml->next[x - 1]) stack[sp++] = x;
    while (sp > 0) {
      int node = stack[--sp];
      for (int j = fsets[node - 1]; j <= fsets[node] - 1; j++) perm[(p++) - 1] = j;
    }
  }
  free(stack);
  return perm;
}
static int *count_num_child(const dll_t *sons, int nmap, const int *map) {      /* :208-220 */
  int *o = xmalloc(sizeof(int) * (nmap ? nmap : 1));
  for (int i = 1; i <= nmap; i++) o[i - 1] = dll_length(sons, map[i - 1]);
  return o;
}

/* ------------------------------------------------------------------------- */
/* algorithms/symbolic_factorize_m.f90:10-62                                  */
/* ------------------------------------------------------------------------- */
static jag_t symbolic_factorize(const jag_t *ccs_a, const int *sets, const int *cc, const jag_t *tc) {
  int n = ccs_a->n, order = sets[n] - 1;
  jag_t l = jag_new(n, cc);
  int *full = xcalloc(order, sizeof(int));
  for (int i = 1; i <= n; i++) {
    int *rl = ja(&l, i), p = 0, *ra = ja(ccs_a, i);
    for (int k = 0; k < jl(ccs_a, i); k++) { rl[p++] = ra[k]; full[ra[k] - 1] = i; }
    if (jl(tc, i) == 0) continue;
    int *ch = ja(tc, i), last = sets[i] - 1;
    for (int j = 0; j < jl(tc, i); j++) {
      int *rc = ja(&l, ch[j]);
      for (int k = 0; k < jl(&l, ch[j]); k++) {
        int row = rc[k];
        if (row <= last || full[row - 1] == i) continue;
        rl[p++] = row; full[row - 1] = i;
      }
    }
  }
  for (int node = 1; node <= n; node++) sort_with_perm(ja(&l, node), NULL, jl(&l, node));
  free(full);
  return l;
}

/* ------------------------------------------------------------------------- */
/* algorithms/create_supernodal_index_m.f90:10-40                             */
/* ------------------------------------------------------------------------- */
static jag_t create_supernodal_index(int ns, const int *sets, const jag_t *a, const jag_t *l) {
  int order = sets[ns] - 1;
  int *map = xcalloc(order, sizeof(int));
  jag_t si = jag_same_shape(a);
  for (int node = 1; node <= ns; node++) {
    int off = sets[node - 1] - 1, nc = sets[node] - sets[node - 1];
    for (int j = 1; j <= nc; j++) map[off + j - 1] = j;
    int *lr = ja(l, node);
    for (int i = 0; i < jl(l, node); i++) map[lr[i] - 1] = nc + i + 1;
    for (int j = sets[node - 1]; j <= sets[node] - 1; j++) {
      int *ar = ja(a, j), *sr = ja(&si, j);
      for (int i = 0; i < jl(a, j); i++) sr[i] = map[ar[i] - 1];
    }
  }
  free(map);
  return si;
}

/* ------------------------------------------------------------------------- */
/* algorithms/create_local_index_m.f90:10-45                                  */
/* ------------------------------------------------------------------------- */
static jag_t create_local_index(const jag_t *l, const int *sets, const jag_t *tc) {
  int ns = l->n, order = sets[ns] - 1;
  int *map = xcalloc(order, sizeof(int));
  jag_t li = jag_same_shape(l);
  for (int node = 1; node <= ns; node++) {
    if (jl(tc, node) == 0) continue;
    int nc = sets[node] - sets[node - 1], off = sets[node - 1] - 1;
    for (int i = 1; i <= nc; i++) map[off + i - 1] = i;
    int *r = ja(l, node);
    for (int i = 0; i < jl(l, node); i++) map[r[i] - 1] = nc + i + 1;
    int *ch = ja(tc, node);
    for (int j = 0; j < jl(tc, node); j++) {
      int c = ch[j]; int *loc = ja(&li, c), *rc = ja(l, c);
      for (int i = 0; i < jl(&li, c); i++) loc[i] = map[rc[i] - 1];
    }
  }
  free(map);
  return li;
}

/* ------------------------------------------------------------------------- */
/* node_data_m.f90 + block_size_calculator_m.f90                              */
/* ------------------------------------------------------------------------- */
enum { SUPERNODE_EX = 1, BORDER_EX = 2, WORK_EX = 3 };    /* extractor_types_m.f90 */
typedef struct { int nb, num_node; int *nc, *nr, *ss, *ws; } nd_t;

static nd_t nd_new(int num_node, const int *nc, const int *nr, int nb) {        /* :31-52 */
  nd_t d; d.nb = nb; d.num_node = num_node;
  d.nc = xmalloc(sizeof(int) * num_node); d.nr = xmalloc(sizeof(int) * num_node);
  d.ss = xmalloc(sizeof(int) * num_node); d.ws = xmalloc(sizeof(int) * num_node);
  memcpy(d.nc, nc, sizeof(int) * num_node); memcpy(d.nr, nr, sizeof(int) * num_node);
  for (int i = 0; i < num_node; i++) {
    d.ss[i] = nc[i] % nb;
    int t = nb - d.ss[i]; d.ws[i] = t < nr[i] ? t : nr[i];
  }
  return d;
}
static void nd_free(nd_t *d) { free(d->nc); free(d->nr); free(d->ss); free(d->ws); }
static int block_size(int idx, int nb, int n) { return (int64_t)idx * nb > n ? n % nb : nb; } /* block_size_calculator_m.f90:12-21 */
static int nd_divisible(const nd_t *d, int node) { return d->ss[node - 1] == 0; }
static int nd_matrix_num(const nd_t *d, int idx) { return (idx - 1) / d->nb + 1; }
static int nd_work_num(const nd_t *d, int idx, int node) { return nd_matrix_num(d, d->nc[node - 1] + idx); }
static int nd_num_matrix_block(const nd_t *d, int node) { return div_ceiling(d->nc[node - 1] + d->nr[node - 1], d->nb); }
static int nd_work_start(const nd_t *d, int node) {                              /* :102-115 */
  int nc = d->nc[node - 1], idx = nc / d->nb + 1;
  if (d->nr[node - 1] == 0) idx = div_ceiling(nc, d->nb) + 1;
  return idx;
}
static int nd_num_work_block(const nd_t *d, int node) { return nd_num_matrix_block(d, node) - nd_work_start(d, node) + 1; }
static int nd_msize(const nd_t *d, int idx, int node) { return block_size(idx, d->nb, d->nc[node - 1] + d->nr[node - 1]); }
static int nd_ssize(const nd_t *d, int idx, int node) { return block_size(idx, d->nb, d->nc[node - 1]); }
static int nd_wsize(const nd_t *d, int idx, int node) {                          /* :141-154 */
  if (idx == nd_work_start(d, node)) return d->ws[node - 1];
  return block_size(idx, d->nb, d->nc[node - 1] + d->nr[node - 1]);
}
static int nd_extractor(const nd_t *d, int idx, int node) {                      /* :156-178 */
  if (nd_divisible(d, node)) return idx <= nd_work_start(d, node) - 1 ? SUPERNODE_EX : WORK_EX;
  int w = nd_work_start(d, node);
  return idx < w ? SUPERNODE_EX : (idx > w ? WORK_EX : BORDER_EX);
}
static int nd_exist_border(const nd_t *d, int node) { return !nd_divisible(d, node) && d->nr[node - 1] != 0; }

/* ------------------------------------------------------------------------- */
/* factors/*_matrix_extractor_m.f90 : start positions (1-based), sizes, totals */
/* ------------------------------------------------------------------------- */
static int64_t sup_start(const nd_t *d, int node, int i, int j) {                /* supernode_matrix_extractor_m.f90:14-28 */
  int64_t n = d->nc[node - 1] + d->nr[node - 1], nb = d->nb;
  int64_t col = nd_ssize(d, j, node);
  int64_t left = psum2(n - (j - 1) * nb + 1, n) + psum1(nb - 1) * (j - 1);
  return left + (int64_t)(i - j) * nb * col + 1;
}
static int64_t sup_size(const nd_t *d, int node, int i, int j) { return (int64_t)nd_msize(d, i, node) * nd_ssize(d, j, node); }
static int64_t sup_estimate(const nd_t *d, int node) {                            /* :41-54 */
  int64_t nb = d->nb, nc = d->nc[node - 1], nr = d->nr[node - 1];
  return psum2(nr + 1, nc + nr) + psum1(nb - 1) * (nc / nb) + psum1(d->ss[node - 1] - 1);
}
static int64_t work_start_pos(const nd_t *d, int node, int i, int j) {          /* work_matrix_extractor_m.f90:14-38 */
  int64_t nb = d->nb, nc = d->nc[node - 1], nr = d->nr[node - 1], fw = d->ws[node - 1];
  int64_t col = nd_wsize(d, j, node), up_row, left;
  int w = nd_work_start(d, node);
  if (j == w) { up_row = nb * (i - 1) - nc; if (up_row < 0) up_row = 0; left = 0; }
  else {
    up_row = (int64_t)(i - j) * nb;
    int64_t wn = j - w - 1;
    left = psum2(nc + nr - (int64_t)(j - 1) * nb + 1, nr) + psum1(nb - 1) * wn + psum1(fw - 1);
  }
  return left + col * up_row + 1;
}
static int64_t work_size(const nd_t *d, int node, int i, int j) { return (int64_t)nd_wsize(d, j, node) * nd_wsize(d, i, node); }
static int64_t work_estimate(const nd_t *d, int node) {                          /* :51-74 */
  int64_t nb = d->nb, nr = d->nr[node - 1];
  int last = nd_num_matrix_block(d, node);
  int64_t lower_row = nd_msize(d, last, node), fw = d->ws[node - 1];
  int64_t wn = nd_num_work_block(d, node) - 2;
  return nr * fw + psum1(wn) * nb * nb + (nr - fw) * lower_row;
}
static int64_t border_start(const nd_t *d, int node, int i, int j) { (void)node; return (int64_t)(i - j) * d->nb * d->nb + 1; }
static int64_t border_size(const nd_t *d, int node, int i, int j) { return (int64_t)nd_msize(d, j, node) * nd_msize(d, i, node); }
static int64_t border_estimate(const nd_t *d, int node) {                         /* border_matrix_extractor_m.f90:28-47 */
  if (!nd_exist_border(d, node)) return 0;
  int nb = d->nb, nc = d->nc[node - 1], nr = d->nr[node - 1];
  int j = nd_work_start(d, node);
  return (int64_t)(nc + nr - (nc / nb) * nb) * nd_msize(d, j, node);
}

/* factors_m.f90: three FP64 buffers with per-node offsets (contiguous_sets_long) */
typedef struct {
  nd_t *nd;
  int64_t *off[3];   /* per node 0-based offset into buf */
  double *buf[3];
  int64_t total[3];
} factors_t;

static void factors_new(factors_t *f, nd_t *nd) {
  f->nd = nd;
  for (int t = 0; t < 3; t++) {
    f->off[t] = xmalloc(sizeof(int64_t) * (nd->num_node + 1));
    f->off[t][0] = 0;
    for (int node = 1; node <= nd->num_node; node++) {
      int64_t s = t == 0 ? sup_estimate(nd, node) : (t == 1 ? work_estimate(nd, node) : border_estimate(nd, node));
      f->off[t][node] = f->off[t][node - 1] + s;
    }
    f->total[t] = f->off[t][nd->num_node];
    f->buf[t] = NULL;          /* allocated on first factorize (factors_alloc) */
  }
}
static void factors_alloc(factors_t *f) {
  for (int t = 0; t < 3; t++)
    if (!f->buf[t]) f->buf[t] = xcalloc(f->total[t] ? f->total[t] : 1, sizeof(double));
}
static void factors_free(factors_t *f) { for (int t = 0; t < 3; t++) { free(f->off[t]); free(f->buf[t]); } }
static double *f_sup(factors_t *f, int node, int i, int j) { return f->buf[0] + f->off[0][node - 1] + sup_start(f->nd, node, i, j) - 1; }
static double *f_work(factors_t *f, int node, int i, int j) { return f->buf[1] + f->off[1][node - 1] + work_start_pos(f->nd, node, i, j) - 1; }
static double *f_border(factors_t *f, int node, int i, int j) { return f->buf[2] + f->off[2][node - 1] + border_start(f->nd, node, i, j) - 1; }
static double *f_matrix(factors_t *f, int node, int i, int j) {                  /* factors_m.f90:38-55 */
  switch (nd_extractor(f->nd, j, node)) {
    case SUPERNODE_EX: return f_sup(f, node, i, j);
    case BORDER_EX: return f_border(f, node, i, j);
    default: return f_work(f, node, i, j);
  }
}

/* right_hand/*: supernode part aliases the permuted RHS; work and border per node */
typedef struct {
  nd_t *nd;
  const int *sets;
  double *sup;        /* permuted b (aliased, length n) */
  double *work, *border;
  int64_t *woff, *boff;
} rh_t;
static void rh_new(rh_t *r, nd_t *nd, const int *sets) {
  r->nd = nd; r->sets = sets;
  r->woff = xmalloc(sizeof(int64_t) * (nd->num_node + 1)); r->boff = xmalloc(sizeof(int64_t) * (nd->num_node + 1));
  r->woff[0] = r->boff[0] = 0;
  for (int node = 1; node <= nd->num_node; node++) {
    r->woff[node] = r->woff[node - 1] + nd->nr[node - 1];
    r->boff[node] = r->boff[node - 1] + (nd_exist_border(nd, node) ? nd_msize(nd, nd_work_start(nd, node), node) : 0);
  }
  r->work = xcalloc(r->woff[nd->num_node] ? r->woff[nd->num_node] : 1, sizeof(double));
  r->border = xcalloc(r->boff[nd->num_node] ? r->boff[nd->num_node] : 1, sizeof(double));
  r->sup = NULL;
}
static void rh_free(rh_t *r) { free(r->woff); free(r->boff); free(r->work); free(r->border); }
static double *rh_sup(rh_t *r, int node, int idx) { return r->sup + (r->sets[node - 1] - 1) + (int64_t)(idx - 1) * r->nd->nb; } /* supernode_array_extractor_m.f90 */
static double *rh_work(rh_t *r, int node, int idx) {                            /* work_array_extractor_m.f90:14-28 */
  int w = nd_work_start(r->nd, node);
  int64_t pos = idx == w ? 1 : r->nd->ws[node - 1] + (int64_t)(idx - w - 1) * r->nd->nb + 1;
  return r->work + r->woff[node - 1] + pos - 1;
}
static double *rh_border(rh_t *r, int node, int idx) { (void)idx; return r->border + r->boff[node - 1]; }
static double *rh_arr(rh_t *r, int node, int idx) {                              /* right_hand_m.f90:47-64 */
  switch (nd_extractor(r->nd, idx, node)) {
    case SUPERNODE_EX: return rh_sup(r, node, idx);
    case BORDER_EX: return rh_border(r, node, idx);
    default: return rh_work(r, node, idx);
  }
}

/* ------------------------------------------------------------------------- */
/* block_local_index_info_m.f90 + block_local_index_creator_m.f90             */
/* ------------------------------------------------------------------------- */
typedef struct {
  int num_node;
  int *node_ptr;      /* num_node+1 : groups per node (contiguous sets) */
  int *block_ptr;     /* num_groups+1 : indices per group */
  int *parent_num, *child_num;   /* per group */
  int *val;           /* rebuilt local index values (mod2), length sum nr */
  int num_groups;
} bli_t;

static void bli_build(bli_t *b, const nd_t *nd, const jag_t *local) {
  int nn = nd->num_node;
  int *nblk = xcalloc(nn, sizeof(int));
  for (int node = 1; node <= nn - 1; node++) {                                  /* create_num_blocks :13-43 */
    int pp = 0, pc = 0, *loc = ja(local, node);
    for (int i = 1; i <= jl(local, node); i++) {
      int pn = nd_matrix_num(nd, loc[i - 1]), cn = nd_work_num(nd, i, node);
      if (pp != pn || pc != cn) { pp = pn; pc = cn; nblk[node - 1]++; }
    }
  }
  b->num_node = nn;
  b->node_ptr = sets_from_lengths(nn, nblk);
  int ng = b->node_ptr[nn] - 1;
  b->num_groups = ng;
  int *nidx = xcalloc(ng, sizeof(int));
  b->parent_num = xcalloc(ng, sizeof(int)); b->child_num = xcalloc(ng, sizeof(int));
  int ap = 0;
  for (int node = 1; node <= local->n - 1; node++) {                            /* create_num_indices :45-77 */
    int pp = 0, pc = 0, *loc = ja(local, node);
    for (int i = 1; i <= jl(local, node); i++) {
      int pn = nd_matrix_num(nd, loc[i - 1]), cn = nd_work_num(nd, i, node);
      if (pp != pn || pc != cn) { pp = pn; pc = cn; ap++; }
      nidx[ap - 1]++;
    }
  }
  b->block_ptr = sets_from_lengths(ng, nidx);
  for (int node = 1; node <= nn - 1; node++) {                                  /* create_block_nums :90-121 */
    int pp = 0, pc = 0, p = 1, *loc = ja(local, node), base = b->node_ptr[node - 1] - 1;
    for (int i = 1; i <= jl(local, node); i++) {
      int pn = nd_matrix_num(nd, loc[i - 1]), cn = nd_work_num(nd, i, node);
      if (pp != pn || pc != cn) {
        pp = pn; pc = cn;
        b->parent_num[base + p - 1] = pn; b->child_num[base + p - 1] = cn; p++;
      }
    }
  }
  int tot = jtot(local);
  b->val = xmalloc(sizeof(int) * (tot ? tot : 1));
  for (int i = 0; i < tot; i++) b->val[i] = mod2(local->val[i], nd->nb);        /* rebuild_val :79-89 */
  free(nblk); free(nidx);
}
static void bli_free(bli_t *b) { free(b->node_ptr); free(b->block_ptr); free(b->parent_num); free(b->child_num); free(b->val); }
static int bli_num_block(const bli_t *b, int node) { return b->node_ptr[node] - b->node_ptr[node - 1]; }
static int bli_gidx(const bli_t *b, int node, int idx) { return b->node_ptr[node - 1] - 1 + idx; } /* 1-based group */
static int *bli_arr(const bli_t *b, int node, int idx, int *len) {
  int g = bli_gidx(b, node, idx);
  *len = b->block_ptr[g] - b->block_ptr[g - 1];
  return b->val + (b->block_ptr[g - 1] - 1);
}
static int bli_start_row(const bli_t *b, int node, int idx) {                    /* get_start_row_num :58-69 */
  int fb = b->node_ptr[node - 1], bi = fb - 1 + idx;
  return b->block_ptr[bi - 1] - b->block_ptr[fb - 1] + 1;
}
static int bli_offset(const bli_t *b, const nd_t *nd, int node, int idx) {       /* get_block_offset :71-85 */
  int s = bli_start_row(b, node, idx);
  if (s <= nd->ws[node - 1]) return s - 1;
  return (nd->ss[node - 1] + s - 1) % nd->nb;
}

/* ------------------------------------------------------------------------- */
/* dense kernels: restatements of the LAPACK/BLAS calls in                    */
/* seq_factorize/kernel/factorize_kernel_m.f90 and seq_solve/kernlel/solve_kernel_m.f90 */
/* column-major, A(r,c) = a[r + c*lda], all 0-based here                      */
/* ------------------------------------------------------------------------- */
typedef void (*f_potrf)(const char*, const int*, double*, const int*, int*, size_t);
typedef void (*f_trsm)(const char*, const char*, const char*, const char*, const int*, const int*, const double*,
                       const double*, const int*, double*, const int*, size_t, size_t, size_t, size_t);
typedef void (*f_syrk)(const char*, const char*, const int*, const int*, const double*, const double*, const int*,
                       const double*, double*, const int*, size_t, size_t);
typedef void (*f_gemm)(const char*, const char*, const int*, const int*, const int*, const double*, const double*,
                       const int*, const double*, const int*, const double*, double*, const int*, size_t, size_t);
typedef void (*f_trsv)(const char*, const char*, const char*, const int*, const double*, const int*, double*, const int*,
                       size_t, size_t, size_t);
typedef void (*f_gemv)(const char*, const int*, const int*, const double*, const double*, const int*, const double*,
                       const int*, const double*, double*, const int*, size_t);
static struct { f_potrf potrf; f_trsm trsm; f_syrk syrk; f_gemm gemm; f_trsv trsv; f_gemv gemv; } g_blas;

static int k_potrf_u(int n, double *a, int lda) {               /* DPOTRF("U", n, a, lda) */
  if (n <= 0) return 0;
  if (g_blas.potrf) { int info = 0; g_blas.potrf("U", &n, a, &lda, &info, 1); return info; }
  for (int j = 0; j < n; j++) {
    double s = a[j + (int64_t)j * lda];
    for (int k = 0; k < j; k++) s -= a[k + (int64_t)j * lda] * a[k + (int64_t)j * lda];
    if (!(s > 0.0)) return j + 1;
    double u = sqrt(s);
    a[j + (int64_t)j * lda] = u;
    for (int i = j + 1; i < n; i++) {
      double t = a[j + (int64_t)i * lda];
      for (int k = 0; k < j; k++) t -= a[k + (int64_t)j * lda] * a[k + (int64_t)i * lda];
      a[j + (int64_t)i * lda] = t / u;
    }
  }
  return 0;
}
static void k_trsm_lutn(int m, int n, const double *a, int lda, double *b, int ldb) { /* DTRSM("L","U","T","N") */
  if (m <= 0 || n <= 0) return;
  if (g_blas.trsm) { double one = 1.0; g_blas.trsm("L", "U", "T", "N", &m, &n, &one, a, &lda, b, &ldb, 1, 1, 1, 1); return; }
  for (int c = 0; c < n; c++) {
    double *x = b + (int64_t)c * ldb;
    for (int i = 0; i < m; i++) {
      double t = x[i];
      for (int k = 0; k < i; k++) t -= a[k + (int64_t)i * lda] * x[k];
      x[i] = t / a[i + (int64_t)i * lda];
    }
  }
}
static void k_syrk_ut(int n, int k, const double *a, int lda, double *c, int ldc) { /* DSYRK("U","T",-1,..,1) */
  if (n <= 0 || k <= 0) return;
  if (g_blas.syrk) { double m1 = -1.0, one = 1.0; g_blas.syrk("U", "T", &n, &k, &m1, a, &lda, &one, c, &ldc, 1, 1); return; }
  for (int j = 0; j < n; j++)
    for (int i = 0; i <= j; i++) {
      double t = 0;
      for (int l = 0; l < k; l++) t += a[l + (int64_t)i * lda] * a[l + (int64_t)j * lda];
      c[i + (int64_t)j * ldc] -= t;
    }
}
static void k_gemm_tn(int m, int n, int k, const double *a, int lda, const double *b, int ldb, double *c, int ldc) { /* DGEMM("T","N",-1,..,1) */
  if (m <= 0 || n <= 0 || k <= 0) return;
  if (g_blas.gemm) { double m1 = -1.0, one = 1.0; g_blas.gemm("T", "N", &m, &n, &k, &m1, a, &lda, b, &ldb, &one, c, &ldc, 1, 1); return; }
  for (int j = 0; j < n; j++)
    for (int i = 0; i < m; i++) {
      double t = 0;
      for (int l = 0; l < k; l++) t += a[l + (int64_t)i * lda] * b[l + (int64_t)j * ldb];
      c[i + (int64_t)j * ldc] -= t;
    }
}
static void k_trsv_ut(int n, const double *a, int lda, double *x) {             /* DTRSV("U","T","N") */
  if (n <= 0) return;
  if (g_blas.trsv) { int one = 1; g_blas.trsv("U", "T", "N", &n, a, &lda, x, &one, 1, 1, 1); return; }
  for (int i = 0; i < n; i++) {
    double t = x[i];
    for (int k = 0; k < i; k++) t -= a[k + (int64_t)i * lda] * x[k];
    x[i] = t / a[i + (int64_t)i * lda];
  }
}
static void k_trsv_un(int n, const double *a, int lda, double *x) {             /* DTRSV("U","N","N") */
  if (n <= 0) return;
  if (g_blas.trsv) { int one = 1; g_blas.trsv("U", "N", "N", &n, a, &lda, x, &one, 1, 1, 1); return; }
  for (int i = n - 1; i >= 0; i--) {
    double t = x[i];
    for (int k = i + 1; k < n; k++) t -= a[i + (int64_t)k * lda] * x[k];
    x[i] = t / a[i + (int64_t)i * lda];
  }
}
static void k_gemv_t(const double *a, int m, int n, const double *x, double *y) { /* DGEMV("T",m,n,-1,a,m,x,1,1,y,1) */
  if (m <= 0 || n <= 0) return;
  if (g_blas.gemv) { double m1 = -1.0, one = 1.0; int inc = 1; g_blas.gemv("T", &m, &n, &m1, a, &m, x, &inc, &one, y, &inc, 1); return; }
  for (int j = 0; j < n; j++) { double t = 0; for (int i = 0; i < m; i++) t += a[i + (int64_t)j * m] * x[i]; y[j] -= t; }
}
static void k_gemv_n(const double *a, int m, int n, const double *x, double *y) { /* DGEMV("N",m,n,-1,a,m,x,1,1,y,1) */
  if (m <= 0 || n <= 0) return;
  if (g_blas.gemv) { double m1 = -1.0, one = 1.0; int inc = 1; g_blas.gemv("N", &m, &n, &m1, a, &m, x, &inc, &one, y, &inc, 1); return; }
  for (int i = 0; i < m; i++) { double t = 0; for (int j = 0; j < n; j++) t += a[i + (int64_t)j * m] * x[j]; y[i] -= t; }
}

/* Load a system BLAS/LAPACK (Fortran ABI) so the CPU baseline times the same
 * library calls the reference makes.  prefix is e.g. "scipy_" or "". */
EXPORT int orc_use_blas(const char *path, const char *prefix) {
  if (!path) { memset(&g_blas, 0, sizeof(g_blas)); return 0; }
  void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return -1;
  char name[128];
#define LOAD(field, sym) do { snprintf(name, sizeof(name), "%s%s", prefix ? prefix : "", sym); \
    *(void **)(&g_blas.field) = dlsym(h, name); if (!g_blas.field) { memset(&g_blas, 0, sizeof(g_blas)); return -2; } } while (0)
  LOAD(potrf, "dpotrf_"); LOAD(trsm, "dtrsm_"); LOAD(syrk, "dsyrk_"); LOAD(gemm, "dgemm_");
  LOAD(trsv, "dtrsv_"); LOAD(gemv, "dgemv_");
#undef LOAD
  return 0;
}

/* ------------------------------------------------------------------------- */
/* numeric phase: zero_setter_m.f90, coefficient_setter_m.f90, seq_factorize/** */
/* ------------------------------------------------------------------------- */
static void set_zero(factors_t *f) {                                             /* zero_setter_m.f90:12-31 */
  nd_t *d = f->nd;
  for (int node = 1; node <= d->num_node; node++) {
    int nbk = nd_num_matrix_block(d, node);
    for (int j = 1; j <= nbk; j++) {
      int ncol = nd_msize(d, j, node);
      double *a = f_matrix(f, node, j, j);
      for (int c = 0; c < ncol; c++) for (int r = 0; r <= c; r++) a[r + (int64_t)c * ncol] = 0.0;
      for (int i = j + 1; i <= nbk; i++) {
        int nrow = nd_msize(d, i, node);
        double *b = f_matrix(f, node, i, j);
        memset(b, 0, sizeof(double) * (size_t)ncol * nrow);
      }
    }
  }
}
static void set_coefficient(factors_t *f, const int *sets, const jag_t *si, const double *vals) { /* coefficient_setter_m.f90:15-50 */
  nd_t *d = f->nd; int nb = d->nb;
  for (int node = 1; node <= d->num_node; node++) {
    for (int j = sets[node - 1]; j <= sets[node] - 1; j++) {
      int *rows = ja(si, j); const double *v = vals + (si->ptr[j - 1] - 1);
      int col = j - sets[node - 1] + 1, bc = div_ceiling(col, nb), bj = mod2(col, nb);
      for (int i = 0; i < jl(si, j); i++) {
        int br = div_ceiling(rows[i], nb), bi = mod2(rows[i], nb);
        double *blk = f_matrix(f, node, br, bc);
        int ld = nd_msize(d, bc, node);
        blk[(bj - 1) + (int64_t)(bi - 1) * ld] = v[i];
      }
    }
  }
}
static int supernode_factorize(factors_t *f, int node) {                         /* seq_factorize_m.f90:31-52 */
  nd_t *d = f->nd; int nbk = nd_num_matrix_block(d, node), info = 0;
  for (int j = 1; j <= nd_work_start(d, node) - 1; j++) {
    int n = nd_msize(d, j, node);
    int r = k_potrf_u(n, f_matrix(f, node, j, j), n);                             /* factorize */
    if (r && !info) info = r + (j - 1) * d->nb;
    for (int i = j + 1; i <= nbk; i++)                                            /* solve */
      k_trsm_lutn(n, nd_msize(d, i, node), f_matrix(f, node, j, j), n, f_matrix(f, node, i, j), n);
    for (int i = j + 1; i <= nbk; i++) {
      int m = nd_msize(d, i, node);
      k_syrk_ut(m, n, f_matrix(f, node, i, j), n, f_matrix(f, node, i, i), m);     /* sym_update */
      for (int k = i + 1; k <= nbk; k++) {                                        /* update(i,k,j) */
        int un = nd_msize(d, i, node), ln = nd_msize(d, k, node);
        k_gemm_tn(un, ln, un, f_matrix(f, node, i, j), un, f_matrix(f, node, k, j), un, f_matrix(f, node, k, i), un);
      }
    }
  }
  return info;
}
static int border_factorize2(factors_t *f, int node) {                           /* seq_factorize_m.f90:54-79 */
  nd_t *d = f->nd;
  int j = nd_work_start(d, node), nbk = nd_num_matrix_block(d, node);
  int ss = d->ss[node - 1], ws = d->ws[node - 1], info = 0;
  { /* rearrange_diag -> split_tri_matrix (matrix_splitter_m.f90:5-28) */
    double *o = f_matrix(f, node, j, j), *l = f_sup(f, node, j, j), *r = f_work(f, node, j, j);
    int lo = ss + ws;
    for (int i = 1; i <= ss; i++) for (int jj = 1; jj <= i; jj++) l[(jj - 1) + (int64_t)(i - 1) * ss] = o[(jj - 1) + (int64_t)(i - 1) * lo];
    for (int i = ss + 1; i <= ss + ws; i++) for (int jj = 1; jj <= ss; jj++) l[(jj - 1) + (int64_t)(i - 1) * ss] = o[(jj - 1) + (int64_t)(i - 1) * lo];
    for (int i = 1; i <= ws; i++) for (int jj = 1; jj <= i; jj++) r[(jj - 1) + (int64_t)(i - 1) * ws] = o[(jj + ss - 1) + (int64_t)(i + ss - 1) * lo];
  }
  for (int i = j + 1; i <= nbk; i++) { /* rearrange_ndiag -> split_rect_matrix (:30-46) */
    double *o = f_matrix(f, node, i, j), *l = f_sup(f, node, i, j), *r = f_work(f, node, i, j);
    int nrow = nd_msize(d, i, node), lo = ss + ws;
    for (int ii = 0; ii < nrow; ii++) {
      for (int jj = 0; jj < ss; jj++) l[jj + (int64_t)ii * ss] = o[jj + (int64_t)ii * lo];
      for (int jj = 0; jj < ws; jj++) r[jj + (int64_t)ii * ws] = o[ss + jj + (int64_t)ii * lo];
    }
  }
  { /* border_factorize -> border_potrf (border_kernel_m.f90:9-19) */
    double *s = f_sup(f, node, j, j), *w = f_work(f, node, j, j);
    int r = k_potrf_u(ss, s, ss);
    if (r && !info) info = r + (j - 1) * d->nb;
    k_trsm_lutn(ss, ws, s, ss, s + (int64_t)ss * ss, ss);
    k_syrk_ut(ws, ss, s + (int64_t)ss * ss, ss, w, ws);
  }
  for (int i = j + 1; i <= nbk; i++) { /* border_solve -> border_trsm (:21-30) */
    int nrow = nd_msize(d, i, node);
    double *ds = f_sup(f, node, j, j), *ssp = f_sup(f, node, i, j), *sw = f_work(f, node, i, j);
    k_trsm_lutn(ss, nrow, ds, ss, ssp, ss);
    k_gemm_tn(ws, nrow, ss, ds + (int64_t)ss * ss, ss, ssp, ss, sw, ws);
  }
  for (int i = j + 1; i <= nbk; i++) {
    int nrow = nd_msize(d, i, node);
    k_syrk_ut(nrow, ss, f_sup(f, node, i, j), ss, f_matrix(f, node, i, i), nrow);   /* border_sym_update */
    for (int k = i + 1; k <= nbk; k++) {                                          /* border_update(i,k,j) */
      int un = nd_msize(d, i, node), ln = nd_msize(d, k, node);
      k_gemm_tn(un, ln, ss, f_sup(f, node, i, j), ss, f_sup(f, node, k, j), ss, f_matrix(f, node, k, i), un);
    }
  }
  return info;
}
static void extend_add(factors_t *f, const bli_t *b, int cn, int pn) {          /* seq_factorize_m.f90:81-98 */
  nd_t *d = f->nd;
  int nbk = bli_num_block(b, cn);
  for (int j = 1; j <= nbk; j++) {
    { /* extend_add_diag -> extend_add_tri (extend_add_kernel_m.f90:20-33) */
      int gj = bli_gidx(b, cn, j), cj = b->child_num[gj - 1], pj = b->parent_num[gj - 1], len;
      int off = bli_offset(b, d, cn, j); int *loc = bli_arr(b, cn, j, &len);
      double *from = f_work(f, cn, cj, cj), *to = f_matrix(f, pn, pj, pj);
      int ldp = nd_msize(d, pj, pn), ldc = nd_wsize(d, cj, cn);
      for (int i = 1; i <= len; i++) for (int jj = 1; jj <= i; jj++)
        to[(loc[jj - 1] - 1) + (int64_t)(loc[i - 1] - 1) * ldp] += from[(off + jj - 1) + (int64_t)(off + i - 1) * ldc];
    }
    for (int i = j + 1; i <= nbk; i++) { /* extend_add_ndiag -> extend_add_rect (:6-18) */
      int gi = bli_gidx(b, cn, i), gj = bli_gidx(b, cn, j);
      int ci = b->child_num[gi - 1], cj = b->child_num[gj - 1], pi = b->parent_num[gi - 1], pj = b->parent_num[gj - 1];
      int roff = bli_offset(b, d, cn, i), coff = bli_offset(b, d, cn, j), li, lj;
      int *il = bli_arr(b, cn, i, &li), *jlc = bli_arr(b, cn, j, &lj);
      double *from = f_work(f, cn, ci, cj), *to = f_matrix(f, pn, pi, pj);
      int ldp = nd_msize(d, pj, pn), ldc = nd_wsize(d, cj, cn);
      for (int ii = 1; ii <= li; ii++) for (int jj = 1; jj <= lj; jj++)
        to[(jlc[jj - 1] - 1) + (int64_t)(il[ii - 1] - 1) * ldp] += from[(coff + jj - 1) + (int64_t)(roff + ii - 1) * ldc];
    }
  }
}

/* seq_solve/** */
static void supernode_forward(factors_t *f, rh_t *r, int node) {                 /* seq_forward_m.f90:34-49 */
  nd_t *d = f->nd;
  for (int j = 1; j <= nd_work_start(d, node) - 1; j++) {
    int n = nd_msize(d, j, node);
    k_trsv_ut(n, f_sup(f, node, j, j), n, rh_arr(r, node, j));
    for (int i = j + 1; i <= nd_num_matrix_block(d, node); i++)
      k_gemv_t(f_sup(f, node, i, j), nd_ssize(d, j, node), nd_msize(d, i, node), rh_arr(r, node, j), rh_arr(r, node, i));
  }
}
static void border_forward2(factors_t *f, rh_t *r, int node) {                  /* seq_forward_m.f90:51-67 */
  nd_t *d = f->nd; int j = nd_work_start(d, node);
  double *bo = rh_border(r, node, j), *su = rh_sup(r, node, j), *wo = rh_work(r, node, j);
  int ls = nd_ssize(d, j, node), rs = nd_wsize(d, j, node);
  for (int i = 0; i < ls; i++) su[i] += bo[i];                                  /* split_array */
  for (int i = 0; i < rs; i++) wo[i] = bo[ls + i];
  int ncol = ls, nrow = nd_msize(d, j, node);
  double *a = f_sup(f, node, j, j);
  k_trsv_ut(ncol, a, ncol, su);                                                  /* border_dtrsv_l */
  k_gemv_t(a + (int64_t)ncol * ncol, ncol, nrow - ncol, su, wo);
  for (int i = j + 1; i <= nd_num_matrix_block(d, node); i++)
    k_gemv_t(f_sup(f, node, i, j), ncol, nd_msize(d, i, node), su, rh_arr(r, node, i));
}
static void supernode_backward(factors_t *f, rh_t *r, int node) {               /* seq_backward_m.f90:116-131 */
  nd_t *d = f->nd;
  for (int j = nd_work_start(d, node) - 1; j >= 1; j--) {
    for (int i = j + 1; i <= nd_num_matrix_block(d, node); i++)
      k_gemv_n(f_sup(f, node, i, j), nd_ssize(d, j, node), nd_msize(d, i, node), rh_arr(r, node, i), rh_arr(r, node, j));
    int n = nd_msize(d, j, node);
    k_trsv_un(n, f_sup(f, node, j, j), n, rh_arr(r, node, j));
  }
}
static void border_backward2(factors_t *f, rh_t *r, int node) {                 /* seq_backward_m.f90:133-149 */
  nd_t *d = f->nd; int j = nd_work_start(d, node);
  int ncol = nd_ssize(d, j, node), nrow = nd_msize(d, j, node);
  double *su = rh_sup(r, node, j), *wo = rh_work(r, node, j), *bo = rh_border(r, node, j);
  for (int i = j + 1; i <= nd_num_matrix_block(d, node); i++)
    k_gemv_n(f_sup(f, node, i, j), ncol, nd_msize(d, i, node), rh_arr(r, node, i), su);
  double *a = f_sup(f, node, j, j);
  k_gemv_n(a + (int64_t)ncol * ncol, ncol, nrow - ncol, wo, su);                 /* border_dtrsv_u */
  k_trsv_un(ncol, a, ncol, su);
  int rs = nd_wsize(d, j, node);
  for (int i = 0; i < ncol; i++) bo[i] = su[i];                                  /* join_array */
  for (int i = 0; i < rs; i++) bo[ncol + i] = wo[i];
}
static void solve_sparse_add(rh_t *r, const bli_t *b, int cn, int pn, int gather) { /* sparse_add_subroutines_m.f90 */
  for (int i = 1; i <= bli_num_block(b, cn); i++) {
    int g = bli_gidx(b, cn, i), cj = b->child_num[g - 1], pj = b->parent_num[g - 1], len;
    int off = bli_offset(b, r->nd, cn, i); int *loc = bli_arr(b, cn, i, &len);
    double *ca = rh_work(r, cn, cj) + off, *pa = rh_arr(r, pn, pj);
    if (gather) for (int k = 0; k < len; k++) ca[k] = pa[loc[k] - 1];
    else for (int k = 0; k < len; k++) pa[loc[k] - 1] += ca[k];
  }
}

/* ------------------------------------------------------------------------- */
/* the oracle handle: state after hppllt_analyze (hppllt_data_m.f90:14-29)    */
/* ------------------------------------------------------------------------- */
typedef struct {
  int n, nnz, nb, max_zero;
  int num_node;
  int *node_sets;      /* num_node+1 */
  int *parent;         /* num_node */
  jag_t tree_child;    /* supernodal */
  jag_t l_structure;
  jag_t a_structure;   /* permuted lower CCS (rows not sorted) */
  int *ccs_perm;       /* nnz */
  int *perm;           /* n */
  jag_t supernodal_index;
  jag_t local_index;   /* before rebuild_val */
  nd_t nd;
  bli_t bli;
  factors_t fac;
  rh_t rh;
  int info;
  int have_nd;
} orc_t;

static void orc_build_data(orc_t *h) {                                           /* hppllt.f90:83-106 */
  int nn = h->num_node;
  int *nc = xmalloc(sizeof(int) * nn), *nr = xmalloc(sizeof(int) * nn);
  for (int i = 1; i <= nn; i++) { nc[i - 1] = h->node_sets[i] - h->node_sets[i - 1]; nr[i - 1] = jl(&h->l_structure, i); }
  h->nd = nd_new(nn, nc, nr, h->nb);
  free(nc); free(nr);
  factors_new(&h->fac, &h->nd);
  rh_new(&h->rh, &h->nd, h->node_sets);
  h->supernodal_index = create_supernodal_index(nn, h->node_sets, &h->a_structure, &h->l_structure);
  h->local_index = create_local_index(&h->l_structure, h->node_sets, &h->tree_child);
  bli_build(&h->bli, &h->nd, &h->local_index);
  h->have_nd = 1;
}

/*
 * hppllt_analyze (hppllt.f90:24-81) with analyze_phase (analyse_phase_m.f90:22-108).
 * order_perm (new position -> original index, 1-based) plays the role of the
 * METIS ordering (options(USE_METIS)=1); NULL means use_metis = 0.
 */
EXPORT orc_t *orc_analyze(int n, const int *ccs_col, const int *ccs_row, int nb, int max_zero, const int *order_perm) {
  orc_t *h = xcalloc(1, sizeof(orc_t));
  h->n = n; h->nb = nb; h->max_zero = max_zero;
  h->nnz = ccs_col[n] - 1;
  jag_t origin; origin.n = n; origin.ptr = xmalloc(sizeof(int) * (n + 1)); memcpy(origin.ptr, ccs_col, sizeof(int) * (n + 1));
  origin.val = xmalloc(sizeof(int) * (h->nnz ? h->nnz : 1)); memcpy(origin.val, ccs_row, sizeof(int) * h->nnz);

  jag_t reordered; int *reo_perm = NULL, *reo_iperm = NULL, *reo_ccs_perm = NULL;
  if (order_perm) {
    reo_perm = xmalloc(sizeof(int) * n); memcpy(reo_perm, order_perm, sizeof(int) * n);
    reo_iperm = set_iperm(n, reo_perm);
    reordered = reordering_ccs(&origin, reo_perm, reo_iperm, &reo_ccs_perm);
  } else {
    reordered = jag_copy(&origin);
  }

  /* ---- analyze_phase ---- */
  jag_t crs = ccs_to_crs(&reordered);
  int *etree = compute_tree(&crs);
  jag_t tc0 = tree_child_by_parent(n, etree);
  int *post = tree_traverse_postordering(&tc0);
  int *ipost = set_iperm(n, post);
  jag_t pccs = repostordering_ccs(&reordered, post, ipost, NULL);
  int *pparent = reordering_tree(n, etree, post, ipost);
  jag_t tc = tree_child_by_parent(n, pparent);
  int *cc = column_count(&pccs, &tc, pparent);
  /* finding_supernode */
  int *subtree = count_subtree_size(&tc);
  int *isleaf = finding_leaves(subtree, &pccs);
  int nfs; int *fsets = search_node_sets(isleaf, &tc, &nfs);
  int *fnum_child = supernodal_tree(nfs, fsets, &tc);
  int *fparent = parent_in_postordering_tree(nfs, fnum_child);
  jag_t ftc = tree_child_by_num_child_and_parent(nfs, fnum_child, fparent);
  int *fcc = supernodal_column_count(nfs, fsets, cc);
  /* relax_supernode */
  dll_t ml, sons;
  compute_merge_lists(nfs, fcc, &ftc, fsets, max_zero, &ml, &sons);
  int nmap; int *map = build_map(&ml, &nmap);
  int *rsets = relaxed_node_sets(fsets, nmap, map, &ml);
  int *rperm = relaxed_perm(nfs, fsets, nmap, map, &ml, n);
  int *rnum_child = count_num_child(&sons, nmap, map);
  int *rparent = parent_in_postordering_tree(nmap, rnum_child);
  jag_t rtc = tree_child_by_num_child_and_parent(nmap, rnum_child, rparent);
  int *rcc = xmalloc(sizeof(int) * nmap);
  for (int i = 0; i < nmap; i++) rcc[i] = fcc[map[i] - 1];                         /* build_cc */
  int *irperm = set_iperm(n, rperm);
  jag_t rccs = repostordering_ccs(&pccs, rperm, irperm, NULL);
  jag_t ccs_sn = supernodal_ccs(nmap, rsets, &rccs);
  h->l_structure = symbolic_factorize(&ccs_sn, rsets, rcc, &rtc);
  int *analyze_perm = perm_product(n, post, rperm);
  h->num_node = nmap;
  h->node_sets = rsets;
  h->parent = create_parent(&rtc);
  h->tree_child = rtc;

  /* ---- back in hppllt_analyze ---- */
  h->perm = order_perm ? perm_product(n, reo_perm, analyze_perm) : analyze_perm;
  int *analyze_iperm = set_iperm(n, analyze_perm);
  int *a_ccs_perm = NULL;
  h->a_structure = repostordering_ccs(&reordered, analyze_perm, analyze_iperm, &a_ccs_perm);
  h->ccs_perm = order_perm ? perm_product(h->nnz, reo_ccs_perm, a_ccs_perm) : a_ccs_perm;
  orc_build_data(h);

  jag_free(&origin); jag_free(&reordered); jag_free(&crs); free(etree); jag_free(&tc0); free(post); free(ipost);
  jag_free(&pccs); free(pparent); jag_free(&tc); free(cc); free(subtree); free(isleaf); free(fsets);
  free(fnum_child); free(fparent); jag_free(&ftc); free(fcc); dll_free(&ml); dll_free(&sons); free(map);
  free(rperm); free(rnum_child); free(rparent); free(rcc); free(irperm); jag_free(&rccs); jag_free(&ccs_sn);
  free(analyze_iperm);
  if (order_perm) { free(reo_perm); free(reo_iperm); free(reo_ccs_perm); free(analyze_perm); free(a_ccs_perm); }
  return h;
}

/*
 * Build the handle directly from the reference's internal data (the form its
 * numeric unit tests start from, e.g. seq_factorize_test.f90:23-35): node sizes,
 * L row lists (global, permuted numbering), parent, A structure in supernodal-
 * index form, with ccs_perm = identity and perm = identity.
 */
EXPORT orc_t *orc_from_internal(int num_node, const int *node_size, const int *lptr, const int *lrow,
                                const int *parent, int n, const int *acol, const int *arow_global, int nb) {
  orc_t *h = xcalloc(1, sizeof(orc_t));
  h->n = n; h->nb = nb; h->num_node = num_node; h->nnz = acol[n] - 1;
  h->node_sets = sets_from_lengths(num_node, node_size);
  h->parent = xmalloc(sizeof(int) * num_node); memcpy(h->parent, parent, sizeof(int) * num_node);
  h->l_structure.n = num_node; h->l_structure.ptr = xmalloc(sizeof(int) * (num_node + 1));
  memcpy(h->l_structure.ptr, lptr, sizeof(int) * (num_node + 1));
  int lt = lptr[num_node] - 1;
  h->l_structure.val = xmalloc(sizeof(int) * (lt ? lt : 1)); memcpy(h->l_structure.val, lrow, sizeof(int) * lt);
  h->tree_child = tree_child_by_parent(num_node, parent);
  h->a_structure.n = n; h->a_structure.ptr = xmalloc(sizeof(int) * (n + 1)); memcpy(h->a_structure.ptr, acol, sizeof(int) * (n + 1));
  h->a_structure.val = xmalloc(sizeof(int) * (h->nnz ? h->nnz : 1)); memcpy(h->a_structure.val, arow_global, sizeof(int) * h->nnz);
  h->ccs_perm = xmalloc(sizeof(int) * (h->nnz ? h->nnz : 1)); for (int i = 0; i < h->nnz; i++) h->ccs_perm[i] = i + 1;
  h->perm = xmalloc(sizeof(int) * n); for (int i = 0; i < n; i++) h->perm[i] = i + 1;
  orc_build_data(h);
  return h;
}

EXPORT void orc_free(orc_t *h) {
  if (!h) return;
  free(h->node_sets); free(h->parent); jag_free(&h->tree_child); jag_free(&h->l_structure);
  jag_free(&h->a_structure); free(h->ccs_perm); free(h->perm); jag_free(&h->supernodal_index);
  jag_free(&h->local_index);
  if (h->have_nd) { bli_free(&h->bli); factors_free(&h->fac); rh_free(&h->rh); nd_free(&h->nd); }
  free(h);
}

/* hppllt_factorize (hppllt.f90:123-150), sequential branch.  Returns the first
 * failing pivot (1-based front-local column of the first node that failed,
 * offset by the node's first global column) or 0. */
EXPORT int orc_factorize(orc_t *h, const double *a) {
  factors_alloc(&h->fac);
  double *vals = xmalloc(sizeof(double) * (h->nnz ? h->nnz : 1));
  for (int k = 0; k < h->nnz; k++) vals[k] = a[h->ccs_perm[k] - 1];              /* permutate */
  set_zero(&h->fac);
  set_coefficient(&h->fac, h->node_sets, &h->supernodal_index, vals);
  free(vals);
  h->info = 0;
  for (int node = 1; node <= h->num_node; node++) {                             /* seq_factorize :13-29 */
    int r = supernode_factorize(&h->fac, node);
    if (nd_exist_border(&h->nd, node)) { int r2 = border_factorize2(&h->fac, node); if (!r) r = r2; }
    if (r && !h->info) h->info = h->node_sets[node - 1] - 1 + r;
    extend_add(&h->fac, &h->bli, node, h->parent[node - 1]);
  }
  return h->info;
}

/* hppllt_solve (hppllt.f90:152-173), single RHS in place, with the RHS work
 * and border arrays of r (h->rh, or a per-thread copy) */
static void solve_with(orc_t *h, rh_t *r, double *b) {
  int n = h->n;
  double *tmp = xmalloc(sizeof(double) * n);
  for (int i = 0; i < n; i++) tmp[i] = b[h->perm[i] - 1];                        /* permutate */
  memset(r->work, 0, sizeof(double) * (r->woff[h->num_node] ? r->woff[h->num_node] : 1));
  memset(r->border, 0, sizeof(double) * (r->boff[h->num_node] ? r->boff[h->num_node] : 1));
  r->sup = tmp;
  for (int node = 1; node <= h->num_node; node++) {                             /* seq_forward */
    supernode_forward(&h->fac, r, node);
    if (nd_exist_border(&h->nd, node)) border_forward2(&h->fac, r, node);
    solve_sparse_add(r, &h->bli, node, h->parent[node - 1], 0);
  }
  for (int node = h->num_node; node >= 1; node--) {                             /* seq_backward */
    solve_sparse_add(r, &h->bli, node, h->parent[node - 1], 1);
    if (nd_exist_border(&h->nd, node)) border_backward2(&h->fac, r, node);
    supernode_backward(&h->fac, r, node);
  }
  for (int i = 0; i < n; i++) b[h->perm[i] - 1] = tmp[i];                        /* inverse_permutate */
  r->sup = NULL;
  free(tmp);
}
EXPORT void orc_solve(orc_t *h, double *b) { solve_with(h, &h->rh, b); }

/* Several right-hand sides (column-major, leading dimension ldb), each solved
 * exactly as orc_solve does, the columns spread over nthreads host threads
 * with a private RHS work area per thread (the factor is only read). */
typedef struct { orc_t *h; double *b; int nrhs; int64_t ldb; int next; } many_ctx_t;
static void *many_worker(void *arg) {
  many_ctx_t *c = arg;
  rh_t r;
  rh_new(&r, &c->h->nd, c->h->node_sets);
  for (;;) {
    int k = __atomic_fetch_add(&c->next, 1, __ATOMIC_RELAXED);
    if (k >= c->nrhs) break;
    solve_with(c->h, &r, c->b + (int64_t)k * c->ldb);
  }
  rh_free(&r);
  return NULL;
}
EXPORT void orc_solve_many(orc_t *h, double *b, int nrhs, int64_t ldb, int nthreads) {
  many_ctx_t c = {h, b, nrhs, ldb, 0};
  int nt = nthreads < 1 ? 1 : nthreads > 256 ? 256 : nthreads;
  if (nt > nrhs) nt = nrhs;
  pthread_t th[256];
  for (int i = 1; i < nt; i++) pthread_create(&th[i], NULL, many_worker, &c);
  many_worker(&c);
  for (int i = 1; i < nt; i++) pthread_join(th[i], NULL);
}

/* ------------------------------------------------------------------------- */
/* accessors                                                                  */
/* ------------------------------------------------------------------------- */
enum {
  ORC_NODE_SETS = 1, ORC_PARENT, ORC_LPTR, ORC_LROW, ORC_APTR, ORC_AROW, ORC_CCS_PERM, ORC_PERM,
  ORC_SIDX, ORC_LOCAL, ORC_BLI_NODE_PTR, ORC_BLI_BLOCK_PTR, ORC_BLI_PARENT, ORC_BLI_CHILD, ORC_BLI_VAL,
  ORC_BLI_OFFSET, ORC_TREE_CHILD_PTR, ORC_TREE_CHILD
};
static int orc_array(orc_t *h, int which, const int **p) {
  switch (which) {
    case ORC_NODE_SETS: *p = h->node_sets; return h->num_node + 1;
    case ORC_PARENT: *p = h->parent; return h->num_node;
    case ORC_LPTR: *p = h->l_structure.ptr; return h->num_node + 1;
    case ORC_LROW: *p = h->l_structure.val; return jtot(&h->l_structure);
    case ORC_APTR: *p = h->a_structure.ptr; return h->n + 1;
    case ORC_AROW: *p = h->a_structure.val; return h->nnz;
    case ORC_CCS_PERM: *p = h->ccs_perm; return h->nnz;
    case ORC_PERM: *p = h->perm; return h->n;
    case ORC_SIDX: *p = h->supernodal_index.val; return h->nnz;
    case ORC_LOCAL: *p = h->local_index.val; return jtot(&h->local_index);
    case ORC_BLI_NODE_PTR: *p = h->bli.node_ptr; return h->num_node + 1;
    case ORC_BLI_BLOCK_PTR: *p = h->bli.block_ptr; return h->bli.num_groups + 1;
    case ORC_BLI_PARENT: *p = h->bli.parent_num; return h->bli.num_groups;
    case ORC_BLI_CHILD: *p = h->bli.child_num; return h->bli.num_groups;
    case ORC_BLI_VAL: *p = h->bli.val; return jtot(&h->local_index);
    case ORC_TREE_CHILD_PTR: *p = h->tree_child.ptr; return h->num_node + 1;
    case ORC_TREE_CHILD: *p = h->tree_child.val; return jtot(&h->tree_child);
    default: *p = NULL; return -1;
  }
}
EXPORT int orc_get_size(orc_t *h, int which) {
  if (which == ORC_BLI_OFFSET) return h->bli.num_groups;
  const int *p; return orc_array(h, which, &p);
}
EXPORT int orc_get(orc_t *h, int which, int *out) {
  if (which == ORC_BLI_OFFSET) { /* get_block_offset for every group, in group order */
    int k = 0;
    for (int node = 1; node <= h->num_node; node++)
      for (int i = 1; i <= bli_num_block(&h->bli, node); i++) out[k++] = bli_offset(&h->bli, &h->nd, node, i);
    return k;
  }
  const int *p; int s = orc_array(h, which, &p);
  if (s < 0) return s;
  memcpy(out, p, sizeof(int) * s);
  return s;
}
EXPORT int orc_num_node(orc_t *h) { return h->num_node; }
EXPORT int64_t orc_cost(orc_t *h) {                                              /* cost_calculator_m.f90:9-20 */
  int64_t c = 0;
  for (int i = 0; i < h->num_node; i++) c += psqsum(h->nd.nr[i] + 1, h->nd.nr[i] + h->nd.nc[i]);
  return c;
}
EXPORT int64_t orc_nonzero(orc_t *h) {                                           /* :22-33 (int64 here) */
  int64_t c = 0;
  for (int i = 0; i < h->num_node; i++) c += psum2(h->nd.nr[i] + 1, h->nd.nr[i] + h->nd.nc[i]);
  return c;
}
EXPORT int64_t orc_array_size(orc_t *h, int which) { return (which >= 1 && which <= 3) ? h->fac.total[which - 1] : -1; }

/* Copy a factor tile out: buffer 1=supernode 2=work 3=border / 0=get_matrix.
 * Returns its length (or -1). */
EXPORT int64_t orc_tile(orc_t *h, int buffer, int node, int i, int j, double *out) {
  double *p; int64_t len;
  nd_t *d = &h->nd;
  factors_alloc(&h->fac);
  int ex = buffer == 0 ? nd_extractor(d, j, node) : buffer;
  switch (ex) {
    case SUPERNODE_EX: p = f_sup(&h->fac, node, i, j); len = sup_size(d, node, i, j); break;
    case BORDER_EX: p = f_border(&h->fac, node, i, j); len = border_size(d, node, i, j); break;
    case WORK_EX: p = f_work(&h->fac, node, i, j); len = work_size(d, node, i, j); break;
    default: return -1;
  }
  if (out) memcpy(out, p, sizeof(double) * len);
  return len;
}
/* Write a supernode-buffer tile (used by the solve unit tests, which preset L). */
EXPORT void orc_set_tile(orc_t *h, int node, int i, int j, const double *in) {
  factors_alloc(&h->fac);
  memcpy(f_sup(&h->fac, node, i, j), in, sizeof(double) * sup_size(&h->nd, node, i, j));
}
/* Forward or backward sweep only on an already permuted RHS (the unit tests
 * seq_forward_test.f90 / seq_backward_test.f90 call them separately). */
EXPORT void orc_sweep(orc_t *h, double *tmp, int backward) {
  rh_t *r = &h->rh;
  memset(r->work, 0, sizeof(double) * (r->woff[h->num_node] ? r->woff[h->num_node] : 1));
  memset(r->border, 0, sizeof(double) * (r->boff[h->num_node] ? r->boff[h->num_node] : 1));
  r->sup = tmp;
  if (!backward) {
    for (int node = 1; node <= h->num_node; node++) {
      supernode_forward(&h->fac, r, node);
      if (nd_exist_border(&h->nd, node)) border_forward2(&h->fac, r, node);
      solve_sparse_add(r, &h->bli, node, h->parent[node - 1], 0);
    }
  } else {
    for (int node = h->num_node; node >= 1; node--) {
      solve_sparse_add(r, &h->bli, node, h->parent[node - 1], 1);
      if (nd_exist_border(&h->nd, node)) border_backward2(&h->fac, r, node);
      supernode_backward(&h->fac, r, node);
    }
  }
  r->sup = NULL;
}

/* ------------------------------------------------------------------------- */
/* tree_pruning (src/main/algorithms/tree_pruning_m.f90:13-155): subtree     */
/* roots for p workers; 64-bit weights.  roots needs num_node entries.       */
/* Returns the root count (0: bad input).                                    */
/* ------------------------------------------------------------------------- */
static int tp_len(const int *nx, int head) { int c = 0; for (int v = head; v; v = nx[v]) c++; return c; }
EXPORT int orc_tree_pruning(int nn, const int *node_size, const int *cc, const int *num_child, const int *child,
                            double tol, int p, int *roots) {
  if (nn < 1 || p < 1) return 0;
  int64_t *cptr = xcalloc(nn + 1, sizeof(int64_t)), *wt = xcalloc(nn + 1, sizeof(int64_t));
  for (int i = 0; i < nn; i++) cptr[i + 1] = cptr[i] + num_child[i];
  for (int i = 1; i <= nn; i++) {                        /* count_op_count + generate_tree_weights (:75-109) */
    int64_t l = cc[i - 1], k = node_size[i - 1] + l;
    wt[i] = k * (k + 1) * (2 * k + 1) / 6 - l * (l + 1) * (2 * l + 1) / 6;
    for (int64_t q = cptr[i - 1]; q < cptr[i]; q++) wt[i] += wt[child[q]];
  }
  int *nx = xcalloc(nn + 1, sizeof(int)), *pv = xcalloc(nn + 1, sizeof(int));
  int64_t *bins = xmalloc(sizeof(int64_t) * (nn + 2)), *w = xmalloc(sizeof(int64_t) * (nn + 1));
  int count = 0;
  for (;;) {
    memset(nx, 0, sizeof(int) * (nn + 1)); memset(pv, 0, sizeof(int) * (nn + 1));
    int head = nn;                                       /* call subtree_list%add(n) */
    double ratio = 0.0;
    int ip = p - 1, stuck = 0;
    while (ratio <= tol) {                               /* :38-61 */
      ip++;
      while (tp_len(nx, head) < ip) {                    /* partition_tree (:111-132) */
        int best = 0; int64_t bw = 0;
        for (int v = head; v; v = nx[v]) if (wt[v] > bw) { bw = wt[v]; best = v; }   /* find_node_with_max_op */
        if (!best) { stuck = 1; break; }
        for (int64_t q = cptr[best - 1]; q < cptr[best]; q++) {   /* add: at the head */
          int c = child[q];
          if (head) pv[head] = c;
          nx[c] = head; head = c; pv[c] = 0;
        }
        int a = nx[best], b = pv[best];                  /* remove */
        if (!b) head = a; else nx[b] = a;
        if (a) pv[a] = b;
      }
      if (stuck) break;
      int m = 0;                                         /* LPT over ip bins (op max-heap, bin min-heap) */
      for (int v = head; v; v = nx[v]) w[m++] = wt[v];
      for (int i = 0; i < ip; i++) bins[i] = 0;
      for (int t = 0; t < m; t++) {
        int imax = 0; for (int i = 1; i < m; i++) if (w[i] > w[imax]) imax = i;
        int imin = 0; for (int i = 1; i < ip; i++) if (bins[i] < bins[imin]) imin = i;
        bins[imin] += w[imax]; w[imax] = -1;
      }
      int64_t mn = bins[0], mx = bins[0];
      for (int i = 1; i < ip; i++) { if (bins[i] < mn) mn = bins[i]; if (bins[i] > mx) mx = bins[i]; }
      ratio = mx > 0 ? (double)mn / (double)mx : 0.0;
    }
    if (stuck && !(ip - 1 < 1 || (tol == 0.0 && ip - 1 == p))) { tol = 0.0; p = ip - 1; continue; }   /* :46-50 */
    for (int v = head; v; v = nx[v]) roots[count++] = v;
    break;
  }
  free(cptr); free(wt); free(nx); free(pv); free(bins); free(w);
  return count;
}

/* ------------------------------------------------------------------------- */
/* the driver's COO -> CCS conversion (example.f90:95-145), step by step:     */
/* counting sort by row (each row's entries placed from its segment's end,    */
/* so equal rows come out in reverse input order), then a counting sort by    */
/* column over that order taken backwards.  1-based in and out.               */
/* ------------------------------------------------------------------------- */
EXPORT void orc_coo_to_ccs(int n, int nnz, const int *coo_row, const int *coo_col, const double *coo_val,
                           int *ccs_col, int *ccs_row, double *ccs_val) {
  int *ncol = xcalloc(n + 1, sizeof(int)), *row_num = xcalloc(n + 1, sizeof(int));
  int *tmp_row = xmalloc(sizeof(int) * (nnz ? nnz : 1)), *tmp_col = xmalloc(sizeof(int) * (nnz ? nnz : 1));
  double *tmp_val = xmalloc(sizeof(double) * (nnz ? nnz : 1));
  for (int i = 0; i < nnz; i++) {                                   /* 1: key counting (:110-118) */
    if (coo_col[i] == 0) continue;
    ncol[coo_col[i] - 1]++;
    row_num[coo_row[i] - 1]++;
  }
  row_num[0] += 1;                                                  /* 2: locations (:120-127) */
  for (int i = 1; i < n; i++) row_num[i] += row_num[i - 1];
  ncol[0] += 1;
  for (int i = 1; i < n; i++) ncol[i] += ncol[i - 1];
  ccs_col[0] = 1;                                                   /* 3: set col (:129-132) */
  for (int i = 0; i < n; i++) ccs_col[i + 1] = ncol[i];
  for (int i = 0; i < nnz; i++) {                                   /* 4: sort by rows (:134-140) */
    int r = coo_row[i] - 1;
    row_num[r]--;
    tmp_row[row_num[r] - 1] = coo_row[i];
    tmp_col[row_num[r] - 1] = coo_col[i];
    tmp_val[row_num[r] - 1] = coo_val[i];
  }
  for (int i = nnz - 1; i >= 0; i--) {                              /* 5: set row (:142-146) */
    int c = tmp_col[i] - 1;
    ncol[c]--;
    ccs_row[ncol[c] - 1] = tmp_row[i];
    ccs_val[ncol[c] - 1] = tmp_val[i];
  }
  free(ncol); free(row_num); free(tmp_row); free(tmp_col); free(tmp_val);
}

/* ------------------------------------------------------------------------- */
/* unit-level entry points for the reference's algorithm tests                */
/* ------------------------------------------------------------------------- */
EXPORT void orc_t_compute_tree(int n, const int *crs_ptr, const int *crs_val, int *parent_out) {
  jag_t c; c.n = n; c.ptr = (int *)crs_ptr; c.val = (int *)crs_val;
  int *p = compute_tree(&c); memcpy(parent_out, p, sizeof(int) * n); free(p);
}
EXPORT void orc_t_column_count(int n, const int *ccs_ptr, const int *ccs_val, const int *parent, int *cc_out) {
  jag_t c; c.n = n; c.ptr = (int *)ccs_ptr; c.val = (int *)ccs_val;
  jag_t tc = tree_child_by_parent(n, parent);
  int *cc = column_count(&c, &tc, parent); memcpy(cc_out, cc, sizeof(int) * n); free(cc); jag_free(&tc);
}
EXPORT void orc_t_postorder(int n, const int *parent, int *perm_out, int *subtree_out) {
  jag_t tc = tree_child_by_parent(n, parent);
  int *p = tree_traverse_postordering(&tc); memcpy(perm_out, p, sizeof(int) * n); free(p);
  int *s = count_subtree_size(&tc); memcpy(subtree_out, s, sizeof(int) * n); free(s);
  jag_free(&tc);
}
EXPORT void orc_t_parent_in_postordering_tree(int n, const int *num_child, int *parent_out) {
  int *p = parent_in_postordering_tree(n, num_child); memcpy(parent_out, p, sizeof(int) * n); free(p);
}
EXPORT void orc_t_finding_leaves(int n, const int *subtree, const int *ccs_ptr, const int *ccs_val, int *out) {
  jag_t c; c.n = n; c.ptr = (int *)ccs_ptr; c.val = (int *)ccs_val;
  int *l = finding_leaves(subtree, &c); memcpy(out, l, sizeof(int) * n); free(l);
}
/* returns number of supernodes; writes sets ptr (ns+1) */
EXPORT int orc_t_search_node_sets(int n, const int *isleaf, const int *num_child, const int *child_val, int *sets_out) {
  jag_t tc; tc.n = n; tc.ptr = sets_from_lengths(n, num_child); tc.val = (int *)child_val;
  int ns; int *s = search_node_sets(isleaf, &tc, &ns); memcpy(sets_out, s, sizeof(int) * (ns + 1)); free(s); free(tc.ptr);
  return ns;
}
/* merge lists for compute_merge_lists; out holds, for each list i (1..n), its
 * members in list order, terminated by 0 */
EXPORT void orc_t_merge_lists(int n, const int *cc, const int *num_child, const int *child_val, const int *node_size,
                              int max_zero, int *out) {
  jag_t tc; tc.n = n; tc.ptr = sets_from_lengths(n, num_child); tc.val = (int *)child_val;
  int *sets = sets_from_lengths(n, node_size);
  dll_t ml, sons; compute_merge_lists(n, cc, &tc, sets, max_zero, &ml, &sons);
  int k = 0;
  for (int i = 1; i <= n; i++) { for (int x = ml.head[i - 1]; x != 0; x = ml.next[x - 1]) out[k++] = x; out[k++] = 0; }
  dll_free(&ml); dll_free(&sons); free(tc.ptr); free(sets);
}
/* symbolic_factorize_test.f90 */
EXPORT void orc_t_symbolic_factorize(int ns, const int *a_len, const int *a_val, const int *cc, const int *node_size,
                                     const int *num_child, const int *child_val, int *out) {
  jag_t a; a.n = ns; a.ptr = sets_from_lengths(ns, a_len); a.val = (int *)a_val;
  jag_t tc; tc.n = ns; tc.ptr = sets_from_lengths(ns, num_child); tc.val = (int *)child_val;
  int *sets = sets_from_lengths(ns, node_size);
  jag_t l = symbolic_factorize(&a, sets, cc, &tc);
  memcpy(out, l.val, sizeof(int) * jtot(&l));
  jag_free(&l); free(a.ptr); free(tc.ptr); free(sets);
}
/* supernodal ccs (fundamental_supernode_test.f90) */
EXPORT int orc_t_supernodal_ccs(int n, const int *ccs_ptr, const int *ccs_val, int ns, const int *sets, int *len_out, int *val_out) {
  jag_t c; c.n = n; c.ptr = (int *)ccs_ptr; c.val = (int *)ccs_val;
  jag_t s = supernodal_ccs(ns, sets, &c);
  for (int i = 1; i <= ns; i++) len_out[i - 1] = jl(&s, i);
  int t = jtot(&s); memcpy(val_out, s.val, sizeof(int) * t); jag_free(&s);
  return t;
}
/* create_supernodal_index_test.f90 */
EXPORT void orc_t_supernodal_index(int ns, const int *node_size, const int *l_len, const int *l_val, int n,
                                   const int *a_len, const int *a_val, int *out) {
  int *sets = sets_from_lengths(ns, node_size);
  jag_t l; l.n = ns; l.ptr = sets_from_lengths(ns, l_len); l.val = (int *)l_val;
  jag_t a; a.n = n; a.ptr = sets_from_lengths(n, a_len); a.val = (int *)a_val;
  jag_t si = create_supernodal_index(ns, sets, &a, &l);
  memcpy(out, si.val, sizeof(int) * jtot(&si));
  jag_free(&si); free(sets); free(l.ptr); free(a.ptr);
}
/* create_local_index_test.f90 */
EXPORT void orc_t_local_index(int ns, const int *node_size, const int *l_len, const int *l_val,
                              const int *num_child, const int *child_val, int *out) {
  int *sets = sets_from_lengths(ns, node_size);
  jag_t l; l.n = ns; l.ptr = sets_from_lengths(ns, l_len); l.val = (int *)l_val;
  jag_t tc; tc.n = ns; tc.ptr = sets_from_lengths(ns, num_child); tc.val = (int *)child_val;
  jag_t li = create_local_index(&l, sets, &tc);
  memcpy(out, li.val, sizeof(int) * jtot(&li));
  jag_free(&li); free(sets); free(l.ptr); free(tc.ptr);
}
/* block_local_index_info_test.f90: build from (node sizes, work sizes, local index).
 * Writes: node_ptr (nn+1), block_ptr (ng+1), parent/child/offset/start (ng), val (sum len). Returns ng. */
EXPORT int orc_t_block_local_index(int nn, const int *nc, const int *nr, int nb, const int *l_len, const int *l_val,
                                   int *node_ptr, int *block_ptr, int *pnum, int *cnum, int *offset, int *start, int *val) {
  nd_t d = nd_new(nn, nc, nr, nb);
  jag_t l; l.n = nn; l.ptr = sets_from_lengths(nn, l_len); l.val = (int *)l_val;
  bli_t b; bli_build(&b, &d, &l);
  int ng = b.num_groups;
  memcpy(node_ptr, b.node_ptr, sizeof(int) * (nn + 1));
  memcpy(block_ptr, b.block_ptr, sizeof(int) * (ng + 1));
  memcpy(pnum, b.parent_num, sizeof(int) * ng); memcpy(cnum, b.child_num, sizeof(int) * ng);
  int k = 0;
  for (int node = 1; node <= nn; node++)
    for (int i = 1; i <= bli_num_block(&b, node); i++) { offset[k] = bli_offset(&b, &d, node, i); start[k] = bli_start_row(&b, node, i); k++; }
  memcpy(val, b.val, sizeof(int) * jtot(&l));
  bli_free(&b); nd_free(&d); free(l.ptr);
  return ng;
}
/* node geometry: work start index, #blocks, border sizes, buffer totals (node_data_test / factors_test) */
EXPORT void orc_t_node_geometry(int nn, const int *nc, const int *nr, int nb, int *ws_out, int *nblk_out,
                                int *ssize_out, int *wsize_out, int64_t *totals_out) {
  nd_t d = nd_new(nn, nc, nr, nb);
  for (int i = 1; i <= nn; i++) {
    ws_out[i - 1] = nd_work_start(&d, i); nblk_out[i - 1] = nd_num_matrix_block(&d, i);
    ssize_out[i - 1] = d.ss[i - 1]; wsize_out[i - 1] = d.ws[i - 1];
  }
  int64_t t0 = 0, t1 = 0, t2 = 0;
  for (int i = 1; i <= nn; i++) { t0 += sup_estimate(&d, i); t1 += work_estimate(&d, i); t2 += border_estimate(&d, i); }
  totals_out[0] = t0; totals_out[1] = t1; totals_out[2] = t2;
  nd_free(&d);
}
/* start positions (1-based within the node's slab) of the three tile extractors */
EXPORT int64_t orc_t_tile_start(int nn, const int *nc, const int *nr, int nb, int kind, int node, int i, int j) {
  nd_t d = nd_new(nn, nc, nr, nb);
  int64_t r = kind == 1 ? sup_start(&d, node, i, j) : (kind == 2 ? work_start_pos(&d, node, i, j) : border_start(&d, node, i, j));
  nd_free(&d);
  return r;
}

typedef struct {
  orc_t *h; const int *order; const int *height; int *res; int level; int hi;
  int next; int mode;   /* 0 = factor nodes, 1 = extend-add per parent */
} par_ctx_t;
static void par_one(par_ctx_t *c, int t) {
  orc_t *h = c->h; int node = c->order[t];
  if (c->mode == 0) {
    int r = supernode_factorize(&h->fac, node);
    if (nd_exist_border(&h->nd, node)) { int r2 = border_factorize2(&h->fac, node); if (!r) r = r2; }
    c->res[node - 1] = r;
    return;
  }
  int p = h->parent[node - 1];
  if (!p) return;
  /* only the first child of p (tree_child order) found on this level does the work */
  int *ch = ja(&h->tree_child, p), first = 0;
  for (int k = 0; k < jl(&h->tree_child, p); k++) if (c->height[ch[k] - 1] == c->level) { first = ch[k]; break; }
  if (first != node) return;
  for (int k = 0; k < jl(&h->tree_child, p); k++)
    if (c->height[ch[k] - 1] == c->level) extend_add(&h->fac, &h->bli, ch[k], p);
}
static void *par_worker(void *arg) {
  par_ctx_t *c = arg;
  for (;;) {
    int t = __atomic_fetch_add(&c->next, 1, __ATOMIC_RELAXED);
    if (t >= c->hi) break;
    par_one(c, t);
  }
  return NULL;
}
static void par_run(par_ctx_t *c, int lo, int hi, int nthreads) {
  c->next = lo; c->hi = hi;
  int nt = nthreads; if (nt > hi - lo) nt = hi - lo; if (nt < 1) nt = 1;
  pthread_t th[256];
  if (nt > 256) nt = 256;
  for (int i = 1; i < nt; i++) pthread_create(&th[i], NULL, par_worker, c);
  par_worker(c);
  for (int i = 1; i < nt; i++) pthread_join(th[i], NULL);
}
/*
 * CPU baseline: the same numeric phase with etree-level parallelism over
 * nthreads host threads.  Nodes of one level are independent except for the
 * extend-add into a shared parent, which the reference's StarPU path marks
 * RW|COMMUTE; here it is serialised per parent in child order.
 */
EXPORT int orc_factorize_parallel(orc_t *h, const double *a, int nthreads) {
  int nn = h->num_node;
  factors_alloc(&h->fac);
  double *vals = xmalloc(sizeof(double) * (h->nnz ? h->nnz : 1));
  for (int k = 0; k < h->nnz; k++) vals[k] = a[h->ccs_perm[k] - 1];
  set_zero(&h->fac);
  set_coefficient(&h->fac, h->node_sets, &h->supernodal_index, vals);
  free(vals);
  int *height = xcalloc(nn, sizeof(int)), maxh = 0;
  for (int node = 1; node <= nn; node++) {
    int p = h->parent[node - 1];
    if (p) { int hh = height[node - 1] + 1; if (hh > height[p - 1]) height[p - 1] = hh; }
    if (height[node - 1] > maxh) maxh = height[node - 1];
  }
  int *cnt = xcalloc(maxh + 2, sizeof(int));
  for (int i = 0; i < nn; i++) cnt[height[i] + 1]++;
  for (int l = 0; l <= maxh; l++) cnt[l + 1] += cnt[l];
  int *order = xmalloc(sizeof(int) * nn), *fill = xmalloc(sizeof(int) * (maxh + 1));
  for (int l = 0; l <= maxh; l++) fill[l] = cnt[l];
  for (int i = 0; i < nn; i++) order[fill[height[i]]++] = i + 1;
  int *res = xcalloc(nn, sizeof(int));
  par_ctx_t c; c.h = h; c.order = order; c.height = height; c.res = res;
  for (int l = 0; l <= maxh; l++) {
    c.level = l;
    c.mode = 0; par_run(&c, cnt[l], cnt[l + 1], nthreads);
    c.mode = 1; par_run(&c, cnt[l], cnt[l + 1], nthreads);
  }
  h->info = 0;
  for (int node = 1; node <= nn; node++) if (res[node - 1] && !h->info) h->info = h->node_sets[node - 1] - 1 + res[node - 1];
  free(height); free(cnt); free(order); free(fill); free(res);
  return h->info;
}
EXPORT int orc_max_threads(void) { return (int)sysconf(_SC_NPROCESSORS_ONLN); }

/* ------------------------------------------------------------------------- */
/* CPU baseline with the reference's DAG schedule: starpu_factorize_m.f90     */
/* :13-101 submits one StarPU task per tile operation in the sequential loop  */
/* order and lets StarPU order them by each task's access modes on the tiles  */
/* (R, RW, RW|COMMUTE: factorize_tasks_m.f90:12-15, border_tasks_m.f90:12-13, */
/* rearrange_tasks_m.f90:12-13, extend_add_tasks_m.f90:12-13).  Here the same */
/* operations go out in the same order as OpenMP tasks whose depend clauses   */
/* restate those modes on the tiles' addresses: R -> in, RW -> inout,         */
/* RW|COMMUTE -> mutexinoutset (the children's extend-adds into one parent    */
/* tile, in any order, one at a time).  Each task calls the sequential BLAS   */
/* (the reference links -mkl=sequential).  Assembly is an OpenMP loop over    */
/* supernodes, as in zero_setter_m.f90:18 and coefficient_setter_m.f90:25.    */
/* ------------------------------------------------------------------------- */
static void dag_supernode(factors_t *f, int node, int *res);
static void dag_note(int *res, int node, int r) {
  if (!r) return;
  #pragma omp critical(orc_dag_info)
  { if (!res[node - 1] || r < res[node - 1]) res[node - 1] = r; }
}
static void dag_border(factors_t *f, int node, int *res) {                     /* seq_factorize_m.f90:54-79 as tasks */
  nd_t *d = f->nd;
  int j = nd_work_start(d, node), nbk = nd_num_matrix_block(d, node), nb = d->nb;
  int ss = d->ss[node - 1], ws = d->ws[node - 1];
  double *bjj = f_matrix(f, node, j, j), *sjj = f_sup(f, node, j, j), *wjj = f_work(f, node, j, j);
  #pragma omp task depend(in: bjj[0]) depend(inout: sjj[0], wjj[0]) firstprivate(bjj, sjj, wjj, ss, ws)
  { /* rearrange_diag -> split_tri_matrix (matrix_splitter_m.f90:5-28) */
    int lo = ss + ws;
    for (int i = 1; i <= ss; i++) for (int jj = 1; jj <= i; jj++) sjj[(jj - 1) + (int64_t)(i - 1) * ss] = bjj[(jj - 1) + (int64_t)(i - 1) * lo];
    for (int i = ss + 1; i <= ss + ws; i++) for (int jj = 1; jj <= ss; jj++) sjj[(jj - 1) + (int64_t)(i - 1) * ss] = bjj[(jj - 1) + (int64_t)(i - 1) * lo];
    for (int i = 1; i <= ws; i++) for (int jj = 1; jj <= i; jj++) wjj[(jj - 1) + (int64_t)(i - 1) * ws] = bjj[(jj + ss - 1) + (int64_t)(i + ss - 1) * lo];
  }
  for (int i = j + 1; i <= nbk; i++) { /* rearrange_ndiag -> split_rect_matrix (:30-46) */
    double *o = f_matrix(f, node, i, j), *l = f_sup(f, node, i, j), *r = f_work(f, node, i, j);
    int nrow = nd_msize(d, i, node);
    #pragma omp task depend(in: o[0]) depend(inout: l[0], r[0]) firstprivate(o, l, r, nrow, ss, ws)
    {
      int lo = ss + ws;
      for (int ii = 0; ii < nrow; ii++) {
        for (int jj = 0; jj < ss; jj++) l[jj + (int64_t)ii * ss] = o[jj + (int64_t)ii * lo];
        for (int jj = 0; jj < ws; jj++) r[jj + (int64_t)ii * ws] = o[ss + jj + (int64_t)ii * lo];
      }
    }
  }
  #pragma omp task depend(inout: sjj[0], wjj[0]) firstprivate(sjj, wjj, ss, ws, j, node, nb)
  { /* border_factorize -> border_potrf (border_kernel_m.f90:9-19) */
    int r = k_potrf_u(ss, sjj, ss);
    if (r) dag_note(res, node, r + (j - 1) * nb);
    k_trsm_lutn(ss, ws, sjj, ss, sjj + (int64_t)ss * ss, ss);
    k_syrk_ut(ws, ss, sjj + (int64_t)ss * ss, ss, wjj, ws);
  }
  for (int i = j + 1; i <= nbk; i++) { /* border_solve -> border_trsm (:21-30) */
    int nrow = nd_msize(d, i, node);
    double *ssp = f_sup(f, node, i, j), *sw = f_work(f, node, i, j);
    #pragma omp task depend(in: sjj[0]) depend(inout: ssp[0], sw[0]) firstprivate(sjj, ssp, sw, nrow, ss, ws)
    {
      k_trsm_lutn(ss, nrow, sjj, ss, ssp, ss);
      k_gemm_tn(ws, nrow, ss, sjj + (int64_t)ss * ss, ss, ssp, ss, sw, ws);
    }
  }
  for (int i = j + 1; i <= nbk; i++) {
    int nrow = nd_msize(d, i, node);
    double *si = f_sup(f, node, i, j), *tii = f_matrix(f, node, i, i);
    #pragma omp task depend(in: si[0]) depend(inout: tii[0]) firstprivate(si, tii, nrow, ss)
    k_syrk_ut(nrow, ss, si, ss, tii, nrow);                                      /* border_sym_update */
    for (int k = i + 1; k <= nbk; k++) {                                          /* border_update(i,k,j) */
      int un = nd_msize(d, i, node), ln = nd_msize(d, k, node);
      double *sk = f_sup(f, node, k, j), *tki = f_matrix(f, node, k, i);
      #pragma omp task depend(in: si[0], sk[0]) depend(inout: tki[0]) firstprivate(si, sk, tki, un, ln, ss)
      k_gemm_tn(un, ln, ss, si, ss, sk, ss, tki, un);
    }
  }
}
static void dag_extend_add(factors_t *f, const bli_t *b, int cn, int pn) {     /* seq_factorize_m.f90:81-98 as tasks */
  nd_t *d = f->nd;
  int nbk = bli_num_block(b, cn);
  for (int j = 1; j <= nbk; j++) {
    for (int i = j; i <= nbk; i++) {
      int gi = bli_gidx(b, cn, i), gj = bli_gidx(b, cn, j);
      int ci = b->child_num[gi - 1], cj = b->child_num[gj - 1], pi = b->parent_num[gi - 1], pj = b->parent_num[gj - 1];
      int roff = bli_offset(b, d, cn, i), coff = bli_offset(b, d, cn, j), li, lj;
      int *il = bli_arr(b, cn, i, &li), *jlc = bli_arr(b, cn, j, &lj);
      double *from = f_work(f, cn, ci, cj), *to = f_matrix(f, pn, pi, pj);
      int ldp = nd_msize(d, pj, pn), ldc = nd_wsize(d, cj, cn);
      if (i == j) {
        #pragma omp task depend(in: from[0]) depend(mutexinoutset: to[0]) firstprivate(from, to, il, li, coff, ldp, ldc)
        { /* extend_add_diag -> extend_add_tri (extend_add_kernel_m.f90:20-33) */
          for (int a = 1; a <= li; a++) for (int c = 1; c <= a; c++)
            to[(il[c - 1] - 1) + (int64_t)(il[a - 1] - 1) * ldp] += from[(coff + c - 1) + (int64_t)(coff + a - 1) * ldc];
        }
      } else {
        #pragma omp task depend(in: from[0]) depend(mutexinoutset: to[0]) firstprivate(from, to, il, li, jlc, lj, roff, coff, ldp, ldc)
        { /* extend_add_ndiag -> extend_add_rect (:6-18) */
          for (int a = 1; a <= li; a++) for (int c = 1; c <= lj; c++)
            to[(jlc[c - 1] - 1) + (int64_t)(il[a - 1] - 1) * ldp] += from[(coff + c - 1) + (int64_t)(roff + a - 1) * ldc];
        }
      }
    }
  }
}
EXPORT int orc_factorize_dag(orc_t *h, const double *a, int nthreads) {
  factors_alloc(&h->fac);
  double *vals = xmalloc(sizeof(double) * (h->nnz ? h->nnz : 1));
  for (int k = 0; k < h->nnz; k++) vals[k] = a[h->ccs_perm[k] - 1];              /* permutate */
  factors_t *f = &h->fac;
  nd_t *d = f->nd;
  int nn = h->num_node, nt = nthreads > 0 ? nthreads : 1;
  #pragma omp parallel for num_threads(nt) schedule(dynamic, 16)
  for (int node = 1; node <= nn; node++) {                                      /* set_zero, per supernode */
    int nbk = nd_num_matrix_block(d, node);
    for (int j = 1; j <= nbk; j++) {
      int ncol = nd_msize(d, j, node);
      double *t = f_matrix(f, node, j, j);
      for (int c = 0; c < ncol; c++) for (int r = 0; r <= c; r++) t[r + (int64_t)c * ncol] = 0.0;
      for (int i = j + 1; i <= nbk; i++) memset(f_matrix(f, node, i, j), 0, sizeof(double) * (size_t)ncol * nd_msize(d, i, node));
    }
  }
  const int *sets = h->node_sets; const jag_t *si = &h->supernodal_index; int nb = d->nb;
  #pragma omp parallel for num_threads(nt) schedule(dynamic, 16)
  for (int node = 1; node <= nn; node++) {                                      /* set_coefficient, per supernode */
    for (int j = sets[node - 1]; j <= sets[node] - 1; j++) {
      int *rows = ja(si, j); const double *v = vals + (si->ptr[j - 1] - 1);
      int col = j - sets[node - 1] + 1, bc = div_ceiling(col, nb), bj = mod2(col, nb);
      for (int i = 0; i < jl(si, j); i++) {
        int br = div_ceiling(rows[i], nb), bi = mod2(rows[i], nb);
        double *blk = f_matrix(f, node, br, bc);
        blk[(bj - 1) + (int64_t)(bi - 1) * nd_msize(d, bc, node)] = v[i];
      }
    }
  }
  free(vals);
  int *res = xcalloc(nn, sizeof(int));
  #pragma omp parallel num_threads(nt)
  #pragma omp single
  {
    for (int node = 1; node <= nn; node++) {                                    /* submission in postorder */
      dag_supernode(f, node, res);
      if (nd_exist_border(d, node)) dag_border(f, node, res);
      if (h->parent[node - 1]) dag_extend_add(f, &h->bli, node, h->parent[node - 1]);
    }
  }
  h->info = 0;
  for (int node = 1; node <= nn; node++) if (res[node - 1] && !h->info) h->info = h->node_sets[node - 1] - 1 + res[node - 1];
  free(res);
  return h->info;
}

static void dag_supernode(factors_t *f, int node, int *res) {                 /* seq_factorize_m.f90:31-52 as tasks */
  nd_t *d = f->nd; int nbk = nd_num_matrix_block(d, node), nb = d->nb;
  for (int j = 1; j <= nd_work_start(d, node) - 1; j++) {
    int n = nd_msize(d, j, node);
    double *tjj = f_matrix(f, node, j, j);
    #pragma omp task depend(inout: tjj[0]) firstprivate(n, tjj, j, node, nb)
    {
      int r = k_potrf_u(n, tjj, n);
      if (r) dag_note(res, node, r + (j - 1) * nb);
    }
    for (int i = j + 1; i <= nbk; i++) {
      int m = nd_msize(d, i, node);
      double *tij = f_matrix(f, node, i, j);
      #pragma omp task depend(in: tjj[0]) depend(inout: tij[0]) firstprivate(n, m, tjj, tij)
      k_trsm_lutn(n, m, tjj, n, tij, n);
    }
    for (int i = j + 1; i <= nbk; i++) {
      int m = nd_msize(d, i, node);
      double *tij = f_matrix(f, node, i, j), *tii = f_matrix(f, node, i, i);
      #pragma omp task depend(in: tij[0]) depend(inout: tii[0]) firstprivate(n, m, tij, tii)
      k_syrk_ut(m, n, tij, n, tii, m);
      for (int k = i + 1; k <= nbk; k++) {
        int un = nd_msize(d, i, node), ln = nd_msize(d, k, node);
        double *tkj = f_matrix(f, node, k, j), *tki = f_matrix(f, node, k, i);
        #pragma omp task depend(in: tij[0], tkj[0]) depend(inout: tki[0]) firstprivate(un, ln, tij, tkj, tki)
        k_gemm_tn(un, ln, un, tij, un, tkj, un, tki, un);
      }
    }
  }
}

