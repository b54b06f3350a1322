"""Regenerate mtx_fixtures.json from the reference's test matrices.

The reference's end-to-end test (src/test/hppllt_test.f90:12-15) runs the whole
pipeline on test_matrix/bcsstk01.mtx and test_matrix/poisson_9_9.mtx.  This
script reads those two Matrix Market files from a checkout of the reference and
stores their coordinate lists (symmetric lower triangle, as written) so the
tests can use them without the reference tree.

usage: python tests/golden/make_mtx_fixtures.py /path/to/reference
"""
import json
import os
import sys


def read_mtx(path):
    rows, cols, vals = [], [], []
    with open(path) as f:
        lines = [ln for ln in f if not ln.startswith("%")]
    n, _, nnz = (int(t) for t in lines[0].split()[:3])
    for ln in lines[1 : 1 + nnz]:
        r, c, v = ln.split()[:3]
        rows.append(int(r)); cols.append(int(c)); vals.append(float(v))
    return {"n": n, "row": rows, "col": cols, "val": vals}


def main(ref_root):
    out = {}
    for name in ("bcsstk01.mtx", "poisson_9_9.mtx"):
        out[name] = read_mtx(os.path.join(ref_root, "test_matrix", name))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mtx_fixtures.json")
    with open(dst, "w") as f:
        json.dump(out, f)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
