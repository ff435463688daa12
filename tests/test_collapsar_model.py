"""The collapsar model from its shipped progenitor (CPU): GET_MODEL restated
from model/collapsar/src/model.f90:6-253 with the grids of CUSTOM_GRID
(custom.f90:78-150), built from the recorded copy of the profile files
(tests/golden/collapsar_profile.npz, made by make_collapsar_profile.py), and
the self-gravity iteration at the reference's over-relaxation factor 1.9 on
that grid."""
import math
import os

import numpy as np
import pytest

from cumc3d_b200 import models

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "collapsar_profile.npz")
_TREE = os.environ.get("CUMC_REFERENCE_TREE", "")


def test_model_from_the_shipped_profile(oracle_mod):
    spec, prim, eps = models.collapsar_model(FIXTURE)
    assert (spec["nx"], spec["ny"], spec["nz"]) == models.COLLAPSAR_GRID
    assert spec["coordinate_flag"] == 2 and spec["boundary_flag"] == [1, 1, 3, 3, 0, 0] and spec["fixpole"] == 1
    # the whole sphere, the hole inside the inner face
    assert spec["yF"][3] == 0.0 and abs(spec["yF"][-4] - math.pi) < 1e-15
    assert 2.0 * spec["m_bh"] / spec["c_code"] ** 2 < spec["xF"][3] < spec["s_core"]
    # the atmosphere is cell nx's state; the star rotates, the atmosphere does not
    nx = spec["nx"]
    rho = prim[3, 3, :, 0]
    assert spec["rho_atm"] == prim[3, 3, nx + 2, 0] == spec["model"]["rho_floor"]
    star = prim[3:-3, 3:-3, 3:-3, 0] > spec["rho_atm"]
    vphi = prim[3:-3, 3:-3, 3:-3, 3]
    assert np.all(vphi[~star] == 0.0) and np.all(vphi[star] >= 0.0) and vphi.max() > 0.0
    # the perturbation is a relative 1e-4 of the profile at most
    with np.load(FIXTURE) as z:
        profile_rho = z["rho"]
    assert np.array_equal(rho[:3], profile_rho[:3])  # ghost cells: the profile itself
    base = np.broadcast_to(profile_rho[3:-3][None, None], star.shape)
    assert np.all(np.abs(prim[3:-3, 3:-3, 3:-3, 0] / base - 1.0) <= 1e-4 + 1e-15)
    # a uniform field along the axis, divergence free on the discrete faces
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    bmax = float(np.abs(prim[..., 5:7]).max())
    dxmin = float(np.min(np.diff(spec["xF"][3:-3])))
    assert o.max_divb() <= 1e-12 * bmax / dxmin
    o.close()


@pytest.mark.skipif(not _TREE, reason="CUMC_REFERENCE_TREE not set to the reference tree")
def test_reader_reads_what_the_fixture_records():
    prof = models.read_collapsar_profile(os.path.join(_TREE, "model", "collapsar", "profile"))
    with np.load(FIXTURE) as z:
        for k in ("par", "rho", "p", "xF", "yF", "zF"):
            assert np.array_equal(prof[k], z[k]), k


def test_self_gravity_converges_at_1p9_on_the_shipped_grid(oracle_mod):
    """The reference runs omega = 1.9 on this grid; the oracle's iteration
    from phi = 0 contracts there (it diverges on coarse-phi grids that touch
    the poles, test_poisson_oracle)."""
    spec, prim, eps = models.collapsar_model(FIXTURE)
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    rho = prim[3:nz + 3, 3:ny + 3, 3:nx + 3, 0]
    phi, errs = None, []
    for _ in range(3):
        phi, it, err, conv = oracle_mod.poisson_solve(spec, rho, spec["rho_atm"], omega=1.9, tol=1e-10,
                                                      max_iter=200, phi=phi)
        errs.append(err)
    assert errs[0] > errs[1] > errs[2] and errs[2] < 1e-2
    assert np.all(np.isfinite(phi))
