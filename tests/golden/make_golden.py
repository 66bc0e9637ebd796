"""Pack the reference's golden vectors into tests/golden/golden_m100.npz.

The reference (ericwolter/rigidfibers_kth) keeps Fortran-written golden
vectors under tests/reference/100_{analytic,numeric}_{direct,gmres}/
{step}_{Quantity}.ref (F16.8 text, one value per line) and the M=100 layout
in fortran/XcT_init100.in (M, then 6 numbers per fiber: centre, orientation).
The run parameters are those of fortran/run100.in (direct) and
fortran/run100_iter.in (GMRES): N=5, eps=0.01, dt=0.1, NoQI=8,
GMRES restart 10, 100 iterations, tol 1e-5, ExtForce (0,0,-1).

This script reads those files from a checkout of the reference and writes one
compressed npz, so the tests never need the reference at run time.

    python tests/golden/make_golden.py PATH_TO_REFERENCE_CHECKOUT
"""
import os
import sys

import numpy as np

QUANTITIES = ["BVec", "XVec", "TRANSVel", "ROTVel", "POS", "ORIENT"]
CASES = ["100_analytic_direct", "100_analytic_gmres", "100_numeric_direct", "100_numeric_gmres"]


def read_column(path):
    with open(path) as f:
        return np.array([float(v) for v in f.read().split()], dtype=np.float64)


def main(ref_root):
    out = {}
    vals = open(os.path.join(ref_root, "fortran", "XcT_init100.in")).read().split()
    M = int(vals[0])
    nums = np.array([float(v) for v in vals[1 : 1 + 6 * M]], dtype=np.float64).reshape(M, 6)
    out["layout_pos"] = nums[:, 0:3].copy()
    out["layout_orient"] = nums[:, 3:6].copy()
    for case in CASES:
        for step in (0, 1):
            for q in QUANTITIES:
                p = os.path.join(ref_root, "tests", "reference", case, f"{step}_{q}.ref")
                out[f"{case}/{step}_{q}"] = read_column(p)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_m100.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst}: {len(out)} arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py PATH_TO_REFERENCE_CHECKOUT")
    main(sys.argv[1])
