"""The C-ABI library loads and exports every function include/mfdag.h declares
(no device work: runs without a GPU)."""
import os
import re
import subprocess

from mfdag import hppllt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mfdag.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:mfd|hppllt)_\w+)\s*\(", text)))


def test_library_loads_and_exports_header():
    L = hppllt.load()
    names = declared_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", hppllt.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    assert set(names) <= exported
    assert set(hppllt.EXPORTS) <= exported


def test_default_options():
    o = hppllt.default_options()
    assert (o.nb, o.max_zero, o.precision, o.use_graph) == (10, 10, 0, 1)
    assert o.ir_tol == 1e-12


def test_bad_input_rejected_before_device_work():
    import numpy as np
    # column 1 lacks its diagonal-first entry: the analysis rejects it (MFD_E_ARG)
    col = np.array([1, 2, 3], np.int32)
    row = np.array([2, 2], np.int32)
    try:
        hppllt.symbolic_analyze(2, col, row)
    except hppllt.MfdError as e:
        assert e.code == -1
    else:
        raise AssertionError("malformed input accepted")
