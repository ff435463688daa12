"""The engine on non-uniform grids (the torus models' generated grids,
cumc3d_b200.grids) against the oracle, bit for bit: per-cell reconstruction
weights (no uniform-spacing shortcut), non-uniform metric terms."""
import math

import pytest

from cumc3d_b200 import grids, models
from parity_util import assert_bitwise, run_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("recon", ["weno", "ppm", "tvdmc"])
def test_spherical_stretched_grid_bitwise(recon, oracle_mod):
    nx, ny, nz, r, th, ph = grids.spherical_torus_grid(nz=96)
    spec, prim, eps = models.smooth_state(nx, ny, nz, 3, coordinate_flag=2, boundary_flag=(1, 1, 3, 3, 0, 0),
                                          faces=(r, th, ph), recon=recon, riemann="hlld", seed=11, fixpole=1)
    spec["model"]["source"] = "pm_sph"
    spec["model"]["bc"] = "torus_sph"
    g, o, dg, do = run_pair(spec, prim, eps, 2, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)


@pytest.mark.parametrize("recon", ["weno", "ppm"])
def test_cylindrical_log_grid_bitwise(recon, oracle_mod):
    nr, nphi, nz, r, ph, z = grids.cylindrical_torus_grid(nphi=16)
    spec, prim, eps = models.smooth_state(nr, nphi, nz, 3, coordinate_flag=1, boundary_flag=(1, 1, 0, 0, 1, 1),
                                          faces=(r, ph, z), recon=recon, riemann="hlld", seed=12)
    g, o, dg, do = run_pair(spec, prim, eps, 2, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)
