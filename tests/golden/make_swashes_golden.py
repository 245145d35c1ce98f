"""Golden samples of the reference's SWASHES Stoker dam-break files.

Reads reference/swashes_1_nx={128,...,4096}.csv of a reference checkout (the
analytic wet dam break the reference's convergence notebooks compare
against: h = 0.005 / 0.001, L = 10, t = 6) and keeps 256 evenly spaced rows
of each resolution (all 128 of the smallest), columns x, h, u as printed.
The fixture lets tests/test_oracle.py pin the Stoker restatement without the
reference tree; with FVGPU_REFERENCE_ROOT set it also reads the full files.

    python tests/golden/make_swashes_golden.py [reference checkout]
"""

import os
import sys

import numpy as np

RESOLUTIONS = (128, 256, 512, 1024, 2048, 4096)
ROWS = 256


def load(ref_root, nx):
    path = os.path.join(ref_root, "reference", "swashes_1_nx=%d.csv" % nx)
    return np.genfromtxt(path, comments="#", delimiter="\t", usecols=(0, 1, 2))


if __name__ == "__main__":
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FVGPU_REFERENCE_ROOT", "")
    if not ref_root:
        sys.exit("usage: make_swashes_golden.py <reference checkout> (or set FVGPU_REFERENCE_ROOT)")
    out = {}
    for nx in RESOLUTIONS:
        d = load(ref_root, nx)
        idx = np.unique(np.linspace(0, len(d) - 1, min(ROWS, len(d))).round().astype(int))
        out["nx%d" % nx] = d[idx]
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "swashes_stoker.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, {k: v.shape for k, v in out.items()})
