"""Regenerates tests/golden/slab_meshes.npz from the reference's test meshes.

The reference's functional RBF test (tests/test_rbf-pum.py:113-122 of
messahelramzi/pacman) transfers the Franke 3D field between two slab point
clouds, tests/meshes/0.03.npz (438 points) and tests/meshes/0.003.npz
(38,112 points), and requires rel-L2 < 1.5e-2 against the analytic field.
This script copies those two point arrays (key "points", float64) into one
compressed fixture so the known-answer test runs where the reference tree is
absent.  Run it where the reference tree is mounted:

    python tests/golden/make_golden.py /path/to/pacman
"""
import os
import sys

import numpy as np


def main(ref_root):
    mesh = os.path.join(ref_root, "tests", "meshes")
    coarse = np.load(os.path.join(mesh, "0.03.npz"))["points"].astype(np.float64)
    fine = np.load(os.path.join(mesh, "0.003.npz"))["points"].astype(np.float64)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "slab_meshes.npz")
    np.savez_compressed(out, coarse=coarse, fine=fine)
    print(out, coarse.shape, fine.shape)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <root of the pacman source tree>")
    main(sys.argv[1])
