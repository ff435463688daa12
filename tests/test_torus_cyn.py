"""The reference's own cylindrical torus (CPU): GET_MODEL of
model/torus-cyn/src/model.f90 restated in models.torus_cyn -- density
maximum at s_max on the mid-plane, the atmosphere, the field normalised to
minimum beta 350 over the radial face field alone (the reference's
cell-centred average), and a divergence-free face field."""
import numpy as np

from cumc3d_b200 import models
from cumc3d_b200.capi import IBX, IBY, IBZ, IRHO, ITAU, IVY


def test_torus_cyn_model():
    spec, prim, eps = models.torus_cyn(64, 8, 64, r_range=(1.5, 11.5), z_range=(-5.0, 5.0))
    assert spec["coordinate_flag"] == 1 and spec["boundary_flag"] == [1, 1, 0, 0, 1, 1]
    m = spec["model"]
    assert m["source"] == "pm_cyl" and m["r_sh"] == 1.0 and m["floor"] == "torus"
    nr, nz = spec["nx"], spec["nz"]
    rho = prim[3:-3, 3:-3, 3:-3, IRHO]
    x, z = models.centers(spec["xF"])[3:-3], models.centers(spec["zF"])[3:-3]
    l, k, j = np.unravel_index(np.argmax(rho), rho.shape)
    assert abs(x[j] - 4.7) < 0.2 and abs(z[l]) < 0.2 and 0.99 < rho.max() <= 1.0001
    atm = prim[3:-3, 3:-3, 3:-3, IVY] == 0.0        # at rest: the atmosphere, rho_fac * rho_max
    assert 0.5 < atm.mean() < 1.0 and np.all(rho[atm] == 1e-4) and np.all(rho[~atm] > 1e-4 * (1 - 1.01e-4))
    # minimum beta over the radial field alone
    xf = spec["xF"][1:]
    bx = prim[:, 0, :, IBX]
    li, ji, jim = slice(3, 3 + nz), slice(3, 3 + nr), slice(2, 2 + nr)
    bxc = (xf[None, ji] * bx[li, ji] + xf[None, jim] * bx[li, jim]) / (xf[None, ji] + xf[None, jim])
    p = prim[li, 0, ji, ITAU]
    b2 = bxc ** 2
    assert abs((2.0 * p[b2 > 0] / b2[b2 > 0]).min() / 350.0 - 1.0) < 1e-12
    assert np.all(prim[..., IBY] == 0.0)
    # cylindrical divergence (model.f90:229-238) at roundoff
    bz = prim[:, 0, :, IBZ]
    xc = models.centers(spec["xF"])
    dx = spec["xF"][1:] - spec["xF"][:-1]
    dz = spec["zF"][1:] - spec["zF"][:-1]
    lm = slice(2, 2 + nz)
    div = ((xf[None, ji] * bx[li, ji] - xf[None, jim] * bx[li, jim]) * dz[li, None]
           + (bz[li, ji] - bz[lm, ji]) * (xc[None, ji] * dx[None, ji]))
    scale = np.abs(bx).max() * xf.max() * dz.max()
    assert np.abs(div).max() < 1e-13 * scale
