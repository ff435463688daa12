"""The collapsar model's hooks in the oracle (CPU): its floors, the
self-gravity + black hole source and the black hole's growth from the
inner-face mass flux (model/collapsar/src/custom.f90:222-485)."""
import math

import numpy as np

from cumc3d_b200 import capi, models
from oracle import oracle as O
from parity_util import interior


def run(steps, m_bh=0.2, c_code=20.0, n=(16, 8, 8)):
    spec, prim, eps = models.collapsar_sph(*n, m_bh=m_bh, c_code=c_code)
    o = O.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    phi, it, _, conv = O.poisson_solve(spec, prim[3:-3, 3:-3, 3:-3, 0], spec["rho_atm"], tol=1e-10, max_iter=20000)
    assert conv
    o.set_phi(phi)
    o.collapsar_set(m_bh, c_code)
    hist = [o.collapsar_get()]
    for _ in range(steps):
        o.rk3_step(o.finddt())
        hist.append(o.collapsar_get())
    cons = o.get_array(capi.ARR_CONS)
    o.close()
    return spec, cons, hist


def test_black_hole_accretes_and_state_stays_finite():
    spec, cons, hist = run(4)
    m = [h[0] for h in hist]
    assert all(b > a for a, b in zip(m, m[1:]))            # inflow through the inner face
    assert all(abs(h[1] - 2 * h[0] / 20.0 ** 2) <= 1e-15 * h[1] for h in hist)   # r_sh = 2 m / c^2
    assert not any(h[2] for h in hist)
    assert np.isfinite(interior(cons, spec)).all()


def test_horizon_past_the_inner_face_is_flagged():
    # c chosen so that r_sh = 2 m / c^2 sits just inside xF(0) = 2: one step of accretion crosses it
    spec, _, hist = run(1, m_bh=0.2, c_code=math.sqrt(0.2 / 0.9999999))
    assert hist[0][1] < spec["xF"][3] <= hist[-1][1] and hist[-1][2]
