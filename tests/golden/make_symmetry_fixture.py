"""Generates tests/golden/sym_O.npz: the octahedral operators of the reference's interpolator.

testScripts/interpolator.m (check_symmetry, case 'O') lists the 24 operators as literal 3x3
matrices, each transposed after the literal.  This script reads those literals from the
reference source tree (the path is its argument) and stores them as golden data, so that the
CPU tests can check the generated set against the reference's own table:

    python tests/golden/make_symmetry_fixture.py <reference tree>
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    src = open(os.path.join(ref_root, "testScripts", "interpolator.m")).read()
    body = src[src.index("case 'O'"):src.index("case 'I'")]
    mats = []
    for m in re.finditer(r"\{\s*\d+\s*\+\s*1\}\s*=\s*\[([^\]]*)\]'", body):
        rows = [[float(v) for v in r.replace(",", " ").split()] for r in m.group(1).split(";")]
        mats.append(np.array(rows).T)  # the literal is transposed in the source
    mats = np.array(mats)
    assert mats.shape == (24, 3, 3), mats.shape
    np.savez_compressed(os.path.join(HERE, "sym_O.npz"), O=mats)
    print("wrote", mats.shape)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EMC_REFERENCE_DIR")
    if not root:
        sys.exit("usage: make_symmetry_fixture.py REFERENCE_ROOT (or set EMC_REFERENCE_DIR)")
    main(root)
