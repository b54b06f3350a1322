"""Multi-GPU partitions: a batch of independent systems, and the subtrees of
one system.

A batch shards naturally: every system is factored and solved on one GPU, with
no data-path collective (each rank owns its systems' fronts, values and
right-hand sides).  Systems are assigned by estimated factorization cost --
the reference's cost model, sum over supernodes of sum_{k=nr+1}^{nr+nc} k^2
(cost_calculator_m.f90:9-20) -- with the greedy longest-processing-time rule:
most expensive system first, each to the least loaded rank (ties to the lower
rank), so the assignment is deterministic.
"""
from __future__ import annotations

import numpy as np


def system_cost(n, ccs_col, ccs_row, order_perm=None, max_zero=10) -> int:
    """Factorization cost of one system from its symbolic analysis (host only)."""
    from . import hppllt as H
    sym = H.symbolic_analyze(n, ccs_col, ccs_row, order_perm, max_zero=max_zero)
    nc = np.diff(sym["node_ptr"]).astype(np.int64)
    nr = np.diff(sym["lptr"]).astype(np.int64)
    # sum_{k=nr+1}^{nr+nc} k^2 = S(nr+nc) - S(nr), S(m) = m (m+1) (2m+1) / 6
    s = lambda m: m * (m + 1) * (2 * m + 1) // 6
    return int((s(nr + nc) - s(nr)).sum())


def shard_lpt(costs, world: int) -> list[list[int]]:
    """Greedy LPT assignment of systems (by cost) to `world` ranks; returns the
    ascending system indices of every rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def subtree_weights(node_size, cc, num_child, child) -> list[int]:
    """Subtree weight of every supernode (1-based order): the sum over its
    subtree of sum_{k=nr+1}^{nr+nc} k^2 (tree_pruning_m.f90:75-109)."""
    ns = np.asarray(node_size, np.int64)
    nr = np.asarray(cc, np.int64)
    s = lambda m: m * (m + 1) * (2 * m + 1) // 6
    w = [int(x) for x in (s(ns + nr) - s(nr))]
    ptr = np.concatenate([[0], np.cumsum(num_child)])
    for i in range(len(w)):                      # children precede parents
        for k in range(ptr[i], ptr[i + 1]):
            w[i] += w[int(child[k]) - 1]
    return w


def assign_subtrees(weights, world: int) -> list[list[int]]:
    """Subtrees (by weight) to ranks: the LPT packing tree_pruning balances
    (heaviest first into the lightest rank, ties to the lower rank); returns
    the ascending subtree indices of every rank."""
    return shard_lpt(weights, world)
