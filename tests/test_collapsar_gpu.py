"""The collapsar model on the GPU against the oracle: its floors, the
self-gravity + black hole source, the black hole's growth from the
inner-face mass flux after every stage, and the potential re-solved between
steps, as the reference's main loop does (model/collapsar/src/
custom.f90:222-620, solver/mhd/main.f90:98-112).  Every bit of the state, of
the potential and of the black hole's mass."""
import math
import os

import numpy as np
import pytest

from cumc3d_b200 import capi, engine, models
from oracle import oracle as O
from parity_util import interior

pytestmark = pytest.mark.gpu


def test_collapsar_steps_with_potential_resolves_bitwise():
    spec, prim, eps = models.collapsar_sph(20, 10, 8)
    m_bh, c = spec["m_bh"], spec["c_code"]
    ra = spec["rho_atm"]
    g = engine.Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    g.poisson_setup(ra, 1.9)
    g.poisson_solve(20000, 1e-10)  # the initial model's solve (p_in = 0)
    g.collapsar_set(m_bh, c)
    o = O.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    p0, _ = o.get_state()
    phi, _, _, _ = O.poisson_solve(spec, p0[3:-3, 3:-3, 3:-3, 0], ra, tol=1e-10, max_iter=20000)
    o.set_phi(phi)
    o.collapsar_set(m_bh, c)
    n_pot = 2
    for n_step in range(5):
        dg, do = g.finddt(), o.finddt()
        assert dg == do
        g.rungekutta(do)
        o.rk3_step(do)
        mg, rg = g.collapsar_get()
        mo, ro, hit = o.collapsar_get()
        assert (mg, rg) == (mo, ro) and not hit
        if n_step % n_pot == 0:  # CUSTOM_UPDATE at p_in = 3, MOD(n_step, n_pot) == 0
            itg, _, cg = g.poisson_solve(20000, 1e-10)
            po, _ = o.get_state()
            phi, ito, _, co = O.poisson_solve(spec, po[3:-3, 3:-3, 3:-3, 0], ra, tol=1e-10, max_iter=20000,
                                              phi=phi)
            o.set_phi(phi)
            assert cg and co and itg == ito
            assert np.array_equal(g.poisson_get().view(np.uint64), phi.view(np.uint64))
    cg_, co_ = interior(g.get_array(capi.ARR_CONS), spec), interior(o.get_array(capi.ARR_CONS), spec)
    assert np.array_equal(cg_.view(np.uint64), co_.view(np.uint64)), int((cg_ != co_).sum())
    pg, eg = g.get_state()
    po, eo = o.get_state()
    assert np.array_equal(interior(pg, spec).view(np.uint64), interior(po, spec).view(np.uint64))
    assert np.array_equal(interior(eg, spec).view(np.uint64), interior(eo, spec).view(np.uint64))
    assert mg > m_bh
    g.close()
    o.close()


def test_horizon_past_the_inner_face_ends_the_step():
    spec, prim, eps = models.collapsar_sph(16, 8, 8)
    g = engine.Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    g.poisson_setup(spec["rho_atm"], 1.9)
    g.poisson_solve(20000, 1e-10)
    with pytest.raises(engine.CumcError):
        g.collapsar_set(1.0, math.sqrt(1.0 / 1.0000001))  # r_sh already past xF(0) = 2
    g.collapsar_set(0.2, math.sqrt(0.2 / 0.9999999))       # r_sh just inside
    with pytest.raises(engine.CumcError, match="event horizon"):
        g.rungekutta(g.finddt())
    g.close()


def test_collapsar_source_needs_the_potential():
    spec, prim, eps = models.collapsar_sph(12, 8, 6)
    g = engine.Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    with pytest.raises(engine.CumcError):
        g.rungekutta(1e-3)
    g.close()


SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "collapsar_profile.npz")


def test_shipped_collapsar_model_bitwise():
    """The collapsar model from its shipped progenitor (156 x 44 x 128 on
    the shipped r, theta, phi faces, PPM + HLLD, CFL 0.8): the initial
    model's potential (300 red-black iterations at omega = 1.9 from phi = 0),
    then three steps with the floors, the self-gravity + black hole source,
    the radial clamps and FIXPOLE -- every bit equal to the oracle."""
    spec, prim, eps = models.collapsar_model(SHIPPED)
    m_bh, c, ra = spec["m_bh"], spec["c_code"], spec["rho_atm"]
    g = engine.Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    g.poisson_setup(ra, 1.9)
    itg, errg, _ = g.poisson_solve(300, 0.0)
    g.collapsar_set(m_bh, c)
    o = O.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    p0, _ = o.get_state()
    phi, ito, erro, _ = O.poisson_solve(spec, p0[3:-3, 3:-3, 3:-3, 0], ra, omega=1.9, tol=0.0, max_iter=300)
    assert itg == ito == 300 and errg == erro
    assert np.array_equal(g.poisson_get().view(np.uint64), phi.view(np.uint64))
    o.set_phi(phi)
    o.collapsar_set(m_bh, c)
    for _ in range(3):
        dg, do = g.finddt(), o.finddt()
        assert dg == do
        g.rungekutta(do)
        o.rk3_step(do)
        mg, rg = g.collapsar_get()
        mo, ro, hit = o.collapsar_get()
        assert (mg, rg) == (mo, ro) and not hit
    pg, eg = g.get_state()
    po, eo = o.get_state()
    assert np.array_equal(interior(pg, spec).view(np.uint64), interior(po, spec).view(np.uint64))
    assert np.array_equal(interior(eg, spec).view(np.uint64), interior(eo, spec).view(np.uint64))
    g.close()
    o.close()


def test_shipped_collapsar_potential_converges_at_1p9():
    """The initial model's full solve (phi = 0 to the reference's 1e-10) at
    omega = 1.9 on the shipped grid converges."""
    spec, prim, eps = models.collapsar_model(SHIPPED)
    g = engine.Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    g.poisson_setup(spec["rho_atm"], 1.9)
    it, err, conv = g.poisson_solve(100000, 1e-10)
    assert conv and err <= 1e-10 and it < 100000
    phi = g.poisson_get()
    assert np.all(np.isfinite(phi))
    g.close()
