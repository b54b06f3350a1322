"""Shared helpers for the parity tests: reading the oracle's factor in the
reference's tile layout as dense front panels, and building solvers."""
import numpy as np

from oracle import oracle as O


def oracle_front_panel(o: "O.Oracle", node: int, nc: int, nr: int, nb: int) -> np.ndarray:
    """The factor columns of one front (nf x nc, column-major, rows = front
    positions) read out of the oracle's supernode buffer tiles: tile (I, J)
    holds L(i, j) at (j mod nb) + (i - (I-1) nb) * ld with ld the tile column's
    supernode block size (supernode_matrix_extractor_m.f90, coefficient_setter_m.f90:45-50)."""
    nf = nc + nr
    out = np.zeros((nf, nc))
    tiles = {}
    for j in range(nc):
        J = j // nb + 1
        ld = nb if J * nb <= nc else nc % nb
        for i in range(j, nf):
            I = i // nb + 1
            key = (I, J)
            if key not in tiles:
                tiles[key] = o.tile(node, I, J, buffer=1)
            t = tiles[key]
            out[i, j] = t[(j % nb) + (i - (I - 1) * nb) * ld]
    return out


def lower_panel(flat: np.ndarray, nf: int, nc: int) -> np.ndarray:
    p = flat.reshape(nc, nf).T.copy()
    for j in range(nc):
        p[:j, j] = 0.0
    return p


def toy_symbolic():
    """The reference's 3-supernode fixture (seq_factorize_test.f90:23-35) as
    symbolic arrays: node sizes [4,5,4], L rows derived from the local index,
    A structure from the supernodal index, identity permutations."""
    from golden import reference_vectors as R
    sizes = R.TOY_NODE_SIZE
    first = np.concatenate([[1], 1 + np.cumsum(sizes)])
    loc = [R.TOY_LOCAL_VAL[0:5], R.TOY_LOCAL_VAL[5:8], []]
    lrows = [[], [], []]
    for node in (2, 1):
        p = R.TOY_PARENT[node - 1]
        for pos in loc[node - 1]:
            lrows[node - 1].append(int(first[p - 1] + pos - 1) if pos <= sizes[p - 1]
                                   else lrows[p - 1][pos - sizes[p - 1] - 1])
    arow, k = [], 0
    node_of_col = np.repeat(np.arange(1, 4), sizes)
    for col in range(13):
        node = node_of_col[col]
        nc = sizes[node - 1]
        for _ in range(R.TOY_SIDX_LEN[col]):
            pos = R.TOY_SIDX_VAL[k]
            arow.append(int(first[node - 1] + pos - 1) if pos <= nc else lrows[node - 1][pos - nc - 1])
            k += 1
    acol = O.sets_from_lengths(R.TOY_SIDX_LEN)
    nnz = len(arow)
    lens = [len(x) for x in lrows]
    return {
        "n": 13, "nnz": nnz, "num_node": 3, "node_ptr": O.sets_from_lengths(sizes), "parent": np.array(R.TOY_PARENT),
        "lptr": O.sets_from_lengths(lens), "lrow": np.array(sum(lrows, []), np.int32), "aptr": acol,
        "arow": np.array(arow, np.int32), "ccs_perm": np.arange(1, nnz + 1, dtype=np.int32),
        "perm": np.arange(1, 14, dtype=np.int32), "lrows": lrows,
    }
