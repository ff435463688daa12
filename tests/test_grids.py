"""Non-uniform grid files and generators (CPU): the restated generators
against the grid files the reference ships (model/torus-*/grid/*.dat) --
through digests of those files recorded in tests/golden/grid_digests.json by
tests/golden/make_grid_digests.py, and against the files themselves when the
reference tree is present -- and the CUSTOM_GRID reader's checks."""
import json
import os

import numpy as np
import pytest

from cumc3d_b200 import grids

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference tree, when a user points CUMC_REFERENCE_TREE at it; without it
# the direct comparison is skipped and the digests above carry the check
_TREE = os.environ.get("CUMC_REFERENCE_TREE", "")
REF = os.path.join(_TREE, "model") if _TREE else ""


def _generated():
    nx, ny, nz, r, th, ph = grids.spherical_torus_grid()
    nr, nphi, nzc, rc, phc, zc = grids.cylindrical_torus_grid()
    return {"torus-sph/r_grid.dat": r, "torus-sph/th_grid.dat": th, "torus-sph/phi_grid.dat": ph,
            "torus-cyn/r_grid.dat": rc, "torus-cyn/phi_grid.dat": phc, "torus-cyn/z_grid.dat": zc}


def test_generators_match_the_digests_of_the_shipped_grid_files():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mgd", os.path.join(HERE, "golden", "make_grid_digests.py"))
    mgd = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mgd)
    with open(os.path.join(HERE, "golden", "grid_digests.json")) as f:
        want = json.load(f)
    got = _generated()
    assert sorted(got) == sorted(want)
    for name, faces in got.items():
        w = want[name]
        assert faces.size == w["n_faces"], name
        assert (faces[0], faces[-1]) == (w["first"], w["last"]), name
        assert mgd.digest(faces) == w["sha256"], name


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="CUMC_REFERENCE_TREE not set to the reference tree")
def test_generators_reproduce_the_shipped_grid_files_bitwise():
    nx, ny, nz, r, th, ph = grids.spherical_torus_grid()
    xF, yF, zF = grids.load_grid(os.path.join(REF, "torus-sph", "grid"), nx, ny, nz,
                                 names=("r_grid.dat", "th_grid.dat", "phi_grid.dat"))
    for a, b in ((r, xF), (th, yF), (ph, zF)):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    nr, nphi, nz, r, ph, z = grids.cylindrical_torus_grid()
    xF, yF, zF = grids.load_grid(os.path.join(REF, "torus-cyn", "grid"), nr, nphi, nz)
    for a, b in ((r, xF), (ph, yF), (z, zF)):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_generated_grids_have_the_expected_shape():
    nx, ny, nz, r, th, ph = grids.spherical_torus_grid()
    assert (nx, ny, nz) == (124, 44, 128)
    assert r[3] == 1.5 and abs(r[-4] - 31.5) < 1e-12 and th[3] == 0.0 and th[-4] == np.pi
    assert np.all(np.diff(r) > 0) and np.all(np.diff(th) > 0)
    # geometric stretching away from the equator, mirrored through it
    d = np.diff(th[3:-3])
    assert np.allclose(d, d[::-1]) and d[0] > d[len(d) // 2]
    nr, nphi, nz, r, ph, z = grids.cylindrical_torus_grid()
    assert (nr, nphi, nz) == (136, 128, 136)
    assert np.array_equal(z, -z[::-1])


def test_unsolvable_stretching_is_refused():
    with pytest.raises(ValueError, match="no theta stretching"):
        grids.spherical_torus_grid(nz=64)


def test_reader_checks_the_line_count_and_round_trips(tmp_path):
    nx, ny, nz, r, th, ph = grids.spherical_torus_grid(nz=96)
    p = tmp_path / "r_grid.dat"
    grids.write_faces(p, r)
    assert np.array_equal(grids.read_faces(p, nx), r)
    with pytest.raises(ValueError, match="inconsistent number of r-grid faces"):
        grids.read_faces(p, nx + 1, "r")
