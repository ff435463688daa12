"""Record digests of the face-coordinate files the reference ships with its
torus models (model/torus-sph/grid/*.dat, model/torus-cyn/grid/*.dat), so
that tests/test_grids.py can check the restated generators against them
without the reference tree.

    python tests/golden/make_grid_digests.py /root/reference

For every file: the number of faces, the SHA-256 of the faces read as
float64 (little-endian) and the first and last face.  The files themselves
are not copied.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = {
    "torus-sph": ("r_grid.dat", "th_grid.dat", "phi_grid.dat"),
    "torus-cyn": ("r_grid.dat", "phi_grid.dat", "z_grid.dat"),
}


def digest(faces):
    a = np.ascontiguousarray(np.asarray(faces, dtype="<f8"))
    return hashlib.sha256(a.tobytes()).hexdigest()


def main(ref):
    out = {}
    for model, names in FILES.items():
        for nm in names:
            path = os.path.join(ref, "model", model, "grid", nm)
            with open(path) as f:
                faces = np.array([float(ln.split()[0]) for ln in f.read().splitlines()])
            out["%s/%s" % (model, nm)] = {"n_faces": int(faces.size), "sha256": digest(faces),
                                           "first": float(faces[0]), "last": float(faces[-1])}
    with open(os.path.join(HERE, "grid_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
