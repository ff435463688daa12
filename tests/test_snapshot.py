"""Snapshot files (CPU): the reference's output dataset names and shapes."""
import numpy as np

from cumc3d_b200 import models, snapshot


def test_snapshot_file_round_trip_with_the_reference_datasets(tmp_path):
    spec, _, _ = models.blast_3d(8, nx=8, ny=6, nz=4)
    prim, eps, bf = snapshot.buffers(spec)
    rng = np.random.default_rng(0)
    for a in (prim, eps, bf):
        a[...] = rng.random(a.shape)
    p = tmp_path / "rkiter-7-nm.npz"
    snapshot.write(p, spec, 1.25, prim, eps, bf)
    d = snapshot.read(p)
    assert sorted(d) == sorted(["time", "dimension", "coordinate", "x-interface", "y-interface", "z-interface",
                                "primitive", "epsilon", "bfield"])
    assert d["time"][0] == 1.25 and d["dimension"][0] == 3.0 and d["coordinate"][0] == 1.0
    assert d["x-interface"].shape == (8 + 3,) and d["x-interface"][1] == spec["xF"][3]  # xF(-1:nx+1)
    assert d["primitive"].shape == (6, 8, 10, 5) and d["bfield"].shape == (7, 9, 11, 3)
    assert np.array_equal(d["epsilon"], eps)
