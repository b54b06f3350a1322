"""Confirm that the integer lists in reference_vectors.py appear verbatim in the
reference's Fortran test sources they cite.

Each constant in reference_vectors.py carries a comment naming a file; this
script rebuilds the Fortran array literal "[a, b, c]" (ignoring spaces) for
every list constant and searches the named file for it.  Run it against a
checkout of the reference:

    python tests/golden/check_transcription.py /path/to/reference
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def fortran_literals(path):
    text = open(path).read().replace(" ", "").replace("&\n", "")
    return set(re.findall(r"\[[-0-9,d.]*\]", text))


def resolve(ref_root, name):
    """Map a cited name (a project path or a bare file name) to a file."""
    full = os.path.join(ref_root, name)
    if os.path.exists(full):
        return full
    base = os.path.basename(name)
    for dirpath, _, files in os.walk(ref_root):
        if base in files:
            return os.path.join(dirpath, base)
    return None


def main(ref_root):
    src = open(os.path.join(HERE, "reference_vectors.py")).read()
    current_file = None
    checked = missing = 0
    for line in src.splitlines():
        m = re.search(r"#\s*([\w/]+\.f90)", line)
        if m:
            current_file = resolve(ref_root, m.group(1))
        m2 = re.match(r"\s*([A-Z0-9_]+)\s*=\s*(\[[-0-9, ]+\])", line)
        if m2 and current_file:
            lit = m2.group(2).replace(" ", "")
            lits = fortran_literals(current_file)
            ok = lit in lits
            checked += 1
            if not ok:
                missing += 1
                print("NOT FOUND:", m2.group(1), lit, "in", current_file)
    print(f"checked {checked} literals, {missing} not found verbatim")
    return missing


if __name__ == "__main__":
    sys.exit(1 if main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference") else 0)
