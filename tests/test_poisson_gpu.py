"""Self-gravity potential of the collapsar model on the GPU (red-black SOR,
colour-split layout, poisson.cu) against the oracle's sequential
restatement of model/collapsar/src/custom.f90:511-620: every bit of phi,
the iteration count and the final error."""
import numpy as np
import pytest

from cumc3d_b200 import engine, models
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make(nr, nth, nph, **kw):
    spec, prim, eps = models.star_sph(nr, nth, nph, **kw)
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    return spec, prim, eps, s


@pytest.mark.parametrize("dims", [(24, 16, 12), (23, 15, 10)])
def test_converged_potential_is_bitwise_the_oracles(dims):
    spec, prim, eps, s = make(*dims)
    rho = prim[3:-3, 3:-3, 3:-3, 0]
    s.poisson_setup(spec["rho_atm"], 1.9)
    it, err, conv = s.poisson_solve(max_iter=20000, tol=1e-10)
    phi = s.poisson_get()
    po, ito, erro, convo = O.poisson_solve(spec, rho, spec["rho_atm"], omega=1.9, tol=1e-10, max_iter=20000)
    s.close()
    assert conv and convo and it == ito
    assert np.array_equal(np.float64(err).view(np.uint64), np.float64(erro).view(np.uint64))
    assert np.array_equal(phi.view(np.uint64), po.view(np.uint64)), int((phi != po).sum())


def test_iteration_limit_warm_start_and_new_density_bitwise():
    spec, prim, eps, s = make(24, 16, 12)
    rho = prim[3:-3, 3:-3, 3:-3, 0]
    ra = spec["rho_atm"]
    s.poisson_setup(ra, 1.9)
    # 7 iterations, then 7 more from there: the oracle's 14 from zero
    it1, _, c1 = s.poisson_solve(max_iter=7, tol=1e-10)
    it2, err2, c2 = s.poisson_solve(max_iter=7, tol=1e-10)
    p14, it14, err14, c14 = O.poisson_solve(spec, rho, ra, tol=1e-10, max_iter=14)
    assert (it1, c1, it2, c2, c14) == (7, False, 7, False, False)
    assert np.array_equal(s.poisson_get().view(np.uint64), p14.view(np.uint64))
    assert err2 == err14
    # a new density (as after 10 hydro steps) relaxes from the old potential
    prim2 = prim.copy()
    prim2[..., 0] *= 1.0 + 0.02 * np.sin(np.arange(prim.shape[2]))[None, None, :]
    s.set_state(prim2, eps)
    it3, err3, c3 = s.poisson_solve(max_iter=20000, tol=1e-9)
    po, ito, erro, co = O.poisson_solve(spec, prim2[3:-3, 3:-3, 3:-3, 0], ra, tol=1e-9, max_iter=20000, phi=p14)
    assert c3 and co and it3 == ito and err3 == erro
    assert np.array_equal(s.poisson_get().view(np.uint64), po.view(np.uint64))
    s.close()


def test_set_get_round_trip_and_restart():
    spec, prim, eps, s = make(23, 15, 10)
    s.poisson_setup(spec["rho_atm"], 1.9)
    rng = np.random.default_rng(3)
    guess = -1.0 - rng.random((spec["nz"] + 2, spec["ny"] + 2, spec["nx"] + 2))
    s.poisson_set(guess)
    assert np.array_equal(s.poisson_get(), guess)
    it, err, conv = s.poisson_solve(max_iter=20000, tol=1e-10)
    po, ito, erro, co = O.poisson_solve(spec, prim[3:-3, 3:-3, 3:-3, 0], spec["rho_atm"], tol=1e-10,
                                        max_iter=20000, phi=guess)
    assert conv and co and it == ito and err == erro
    assert np.array_equal(s.poisson_get().view(np.uint64), po.view(np.uint64))
    # setup again: phi back to zero, the first iteration from zero repeats
    s.poisson_setup(spec["rho_atm"], 1.9)
    assert not s.poisson_get().any()
    s.close()


def test_errors():
    spec, prim, eps = models.alfven_3d(8, recon="weno")
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    with pytest.raises(engine.CumcError):
        s.poisson_setup(1e-6, 1.9)  # Cartesian grid
    s.close()
    spec, prim, eps, s = make(12, 8, 6)
    with pytest.raises(engine.CumcError):
        s.poisson_solve()  # before setup
    with pytest.raises(engine.CumcError):
        s.poisson_setup(spec["rho_atm"], 2.0)  # omega outside (0, 2)
    s.poisson_setup(spec["rho_atm"], 1.9)
    with pytest.raises(engine.CumcError):
        s.poisson_solve(max_iter=0)
    s.close()
