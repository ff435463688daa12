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


def test_raw_snapshot_and_hdf5_converter(tmp_path, monkeypatch):
    """Raw binary snapshots (one file per dataset, the Fortran array's bytes,
    a JSON manifest of the shapes) round-trip bit for bit, and the HDF5
    converter writes every dataset of the reference's file under its name
    and shape (checked through a stand-in for h5py, which this image lacks)."""
    import sys
    import types
    spec, _, _ = models.blast_3d(8, nx=8, ny=6, nz=4)
    prim, eps, bf = snapshot.buffers(spec)
    rng = np.random.default_rng(1)
    for a in (prim, eps, bf):
        a[...] = rng.random(a.shape)
    prefix = str(tmp_path / "rkiter-3-nm")
    man = snapshot.write_raw(prefix, spec, 0.5, prim, eps, bf)
    assert man["primitive"]["fortran_shape"] == [5, 10, 8, 6] and man["bfield"]["fortran_shape"] == [3, 11, 9, 7]
    d = snapshot.read_raw(prefix)
    assert np.array_equal(d["primitive"], prim) and np.array_equal(d["bfield"], bf) and d["time"][0] == 0.5
    # the Fortran order of the bytes: element (v, j, k, l) at v + 5 (j + 10 (k + 8 l))
    raw = np.fromfile(prefix + ".primitive.bin", dtype="<f8")
    assert raw[2 + 5 * (3 + 10 * (4 + 8 * 1))] == prim[1, 4, 3, 2]
    written = {}

    class FakeFile:
        def __init__(self, path, mode):
            assert mode == "w"
        def __enter__(self):
            return self
        def __exit__(self, *a):
            return False
        def create_dataset(self, name, data):
            written[name] = np.array(data)
    monkeypatch.setitem(sys.modules, "h5py", types.SimpleNamespace(File=FakeFile))
    snapshot.to_hdf5(prefix, str(tmp_path / "rkiter-3-nm.hdf5"))
    assert sorted(written) == sorted(snapshot.DATASETS)
    assert written["primitive"].shape == (6, 8, 10, 5) and np.array_equal(written["epsilon"], eps)
    npz = tmp_path / "s.npz"
    snapshot.write(npz, spec, 0.5, prim, eps, bf)
    written.clear()
    snapshot.to_hdf5(str(npz), str(tmp_path / "s.hdf5"))
    assert np.array_equal(written["bfield"], bf)
