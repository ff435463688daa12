"""The spherical torus's initial model (CPU): GET_MODEL of
model/torus-sph/src/model.f90 restated in models.torus_sph -- its density
maximum at s_max on the equator, the atmosphere and floors, the field
normalised to the minimum plasma beta, and a face field whose discrete
divergence (the check at model.f90:228-241) is roundoff."""
import math

import numpy as np

from cumc3d_b200 import models
from cumc3d_b200.capi import IBX, IBY, IBZ, IRHO, ITAU, IVZ


def _metric(spec):
    xF, yF = spec["xF"], spec["yF"]
    nt = spec["ny"]
    x = models.centers(xF)
    dx = xF[1:] - xF[:-1]
    dy = yF[1:] - yF[:-1]
    sinf = np.sin(yF[1:])
    sinf[2], sinf[2 + nt] = 0.0, 0.0
    dcose = -(np.cos(yF[1:]) - np.cos(yF[:-1]))
    dx_cb = xF[1:] ** 3 - xF[:-1] ** 3
    return x, dx, dy, sinf, dcose, dx_cb, xF[1:]


def test_torus_on_the_shipped_grid():
    spec, prim, eps = models.torus_sph()
    assert (spec["nx"], spec["ny"], spec["nz"]) == (124, 44, 128)
    assert spec["coordinate_flag"] == 2 and spec["boundary_flag"] == [1, 1, 3, 3, 0, 0] and spec["fixpole"] == 1
    m = spec["model"]
    assert m["source"] == "pm_sph" and m["r_sh"] == 1.0 and m["bc"] == "torus_sph" and m["rho_floor"] == 1e-4
    rho = prim[3:-3, 3:-3, 3:-3, IRHO]
    # axisymmetric apart from the 1e-4 perturbation
    assert np.allclose(rho, rho[:1], rtol=2.01e-4, atol=0)
    x, y = models.centers(spec["xF"])[3:-3], models.centers(spec["yF"])[3:-3]
    l, k, j = np.unravel_index(np.argmax(rho), rho.shape)
    assert abs(x[j] * math.sin(y[k]) - 4.7) < 0.2 and abs(y[k] - math.pi / 2) < 0.1
    assert 0.99 < rho.max() <= 1.0001
    # outside the torus: the atmosphere rho_fac * rho_max, at rest
    atm = rho < 1.5e-4
    assert np.all(rho[atm] == 1e-4) and np.all(prim[3:-3, 3:-3, 3:-3, IVZ][atm] == 0.0)
    # inside: p = K rho^gamma before the density perturbation, eps = p/rho/(g-1) of the unperturbed rho
    g = 5.0 / 3.0
    p = prim[3:-3, 3:-3, 3:-3, ITAU]
    e = eps[3:-3, 3:-3, 3:-3]
    rho0 = p / e / (g - 1.0)
    assert np.allclose(rho, rho0, rtol=1.01e-4, atol=0)
    assert m["p_floor"] == p[atm][0] and abs(m["eps_floor"] - e[atm][0]) < 1e-15 * e[atm][0]


def test_field_has_minimum_beta_350_and_no_divergence():
    spec, prim, eps = models.torus_sph(40, 24, 8, r_range=(2.0, 10.0))
    nx, nt = spec["nx"], spec["ny"]
    x, dx, dy, sinf, dcose, dx_cb, xf = _metric(spec)
    bx = prim[0, :, :, IBX]
    by = prim[0, :, :, IBY]
    assert np.all(prim[..., IBZ] == 0.0) and np.abs(bx).max() > 0
    ki, ji = slice(3, 3 + nt), slice(3, 3 + nx)
    kim, jim = slice(2, 2 + nt), slice(2, 2 + nx)
    bxc = 1.5 * dx[None, ji] / dx_cb[None, ji] * (xf[None, ji] ** 2 * bx[ki, ji] + xf[None, jim] ** 2 * bx[ki, jim])
    byc = 0.5 * dy[ki, None] / dcose[ki, None] * (sinf[ki, None] * by[ki, ji] + sinf[kim, None] * by[kim, ji])
    b2 = bxc ** 2 + byc ** 2
    p = prim[0, ki, ji, ITAU]
    beta = 2.0 * p[b2 > 0] / b2[b2 > 0]
    assert abs(beta.min() / 350.0 - 1.0) < 1e-12
    div = ((xf[None, ji] ** 2 * bx[ki, ji] - xf[None, jim] ** 2 * bx[ki, jim]) / (dx_cb[None, ji] / 3.0)
           + (sinf[ki, None] * by[ki, ji] - sinf[kim, None] * by[kim, ji]) * (x[None, ji] * dx[None, ji])
           / (dx_cb[None, ji] * dcose[ki, None] / 3.0))
    scale = max(np.abs(bx).max(), np.abs(by).max()) / dx[3:3 + nx].min()
    assert np.abs(div).max() < 1e-12 * scale


def test_perturbation_is_seeded():
    a = models.torus_sph(24, 16, 8, r_range=(2.0, 10.0))[1]
    b = models.torus_sph(24, 16, 8, r_range=(2.0, 10.0))[1]
    c = models.torus_sph(24, 16, 8, r_range=(2.0, 10.0), seed=5)[1]
    assert np.array_equal(a, b) and not np.array_equal(a, c)
