"""Record the collapsar model's shipped progenitor (model/collapsar/profile/
par.dat, hydro.dat, r_grid.dat, th_grid.dat, phi_grid.dat) as one small
fixture, so that the model builds and runs where the reference tree is not
present (the GPU tests):

    python tests/golden/make_collapsar_profile.py /root/reference

Writes tests/golden/collapsar_profile.npz: the arrays read_collapsar_profile
returns (par, rho, p, xF, yF, zF) and the SHA-256 of each source file.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cumc3d_b200 import models  # noqa: E402

FILES = ("par.dat", "hydro.dat", "r_grid.dat", "th_grid.dat", "phi_grid.dat")


def main(tree):
    d = os.path.join(tree, "model", "collapsar", "profile")
    prof = models.read_collapsar_profile(d)
    digests = {}
    for name in FILES:
        with open(os.path.join(d, name), "rb") as f:
            digests[name] = hashlib.sha256(f.read()).hexdigest()
    np.savez_compressed(os.path.join(HERE, "collapsar_profile.npz"),
                        sha256=np.array(["%s %s" % (k, v) for k, v in sorted(digests.items())]), **prof)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
