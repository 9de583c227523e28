"""Golden spherical Bessel / Hankel values of the reference's own tests (TEST
INFRASTRUCTURE).

The reference pins its spherical Bessel and Hankel routines (jfuns3d, h3dall of
pytential/qbx/target_specific/helmholtz_utils.c) with values it lists in
test/test_target_specific_qbx.py:44-119 (j_n and j_n' at z = 3i, h_n and h_n' at
z = 2 + 3i, n <= 9).  This script reads those arrays from the reference's test file
as text and stores them in bessel_reference.npz beside it.

  PYTENTIAL_REFERENCE=<reference checkout> python tests/golden/make_bessel_golden.py
"""

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def extract(text, name):
    m = re.search(name + r"\s*=\s*np\.array\(\[(.*?)\]\)", text, re.S)
    vals = []
    for re_, im_ in re.findall(r"([+-][\d.e+-]+)\s*\+\s*([+-][\d.e+-]+)j", m.group(1)):
        vals.append(complex(float(re_), float(im_)))
    return np.array(vals, np.complex128)


def main():
    ref = os.environ.get("PYTENTIAL_REFERENCE")
    if not ref:
        sys.exit("set PYTENTIAL_REFERENCE to the reference checkout")
    with open(os.path.join(ref, "test", "test_target_specific_qbx.py")) as f:
        text = f.read()
    out = {"j_z": np.complex128(3j), "h_z": np.complex128(2 + 3j)}
    for name in ["j_expected", "jder_expected", "h_expected", "hder_expected"]:
        out[name] = extract(text, name)
        assert len(out[name]) == 10, name
    np.savez(os.path.join(HERE, "bessel_reference.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
