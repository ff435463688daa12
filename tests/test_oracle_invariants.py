"""Pins of the CPU oracle (no GPU).

The reference ships no tests or golden vectors and cannot be built here, so
parity is unpinned; these are the invariants the reference's scheme
guarantees, checked on the restatement.
"""
import math

import numpy as np
import pytest

from cumc3d_b200 import capi, models
from parity_util import interior

RS = {"lf": 0, "hll": 1, "hllc": 2, "hlld": 3}
REC = capi.RECON


def run_oracle(O, spec, prim, eps, steps):
    o = O.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    for _ in range(steps):
        o.rk3_step(o.finddt())
    p, e = o.get_state()
    return o, p, e


@pytest.mark.parametrize("recon", ["tvdmm", "tvdvl", "tvdmc", "ppm", "weno"])
@pytest.mark.parametrize("riemann", ["lf", "hll", "hllc", "hlld"])
def test_uniform_state_stays_uniform(oracle_mod, recon, riemann):
    """A uniform moving magnetised state on a periodic box stays exactly
    uniform (every cell bit-identical) and unchanged up to the roundoff of the
    prim -> cons -> prim round trip (fromrvetou.f90:103, 210)."""
    spec, prim, eps = models.blast_3d(8, recon=recon, riemann=riemann, p_in=0.1)
    prim[..., capi.IVX] = 0.3
    prim[..., capi.IVY] = -0.2
    prim[..., capi.IVZ] = 0.1
    prim[..., capi.IBZ] = 0.4
    _, p, e = run_oracle(oracle_mod, spec, prim, eps, 3)
    P = interior(p, spec)
    E = interior(e, spec)
    assert np.all(P == P[0, 0, 0]) and np.all(E == E[0, 0, 0])
    idx = [0, 1, 2, 3, 5, 6, 7]
    assert np.array_equal(P[0, 0, 0, idx], prim[3, 3, 3, idx])
    assert abs(E[0, 0, 0] - eps[3, 3, 3]) <= 1e-14 * eps[3, 3, 3]


@pytest.mark.parametrize("riemann", ["lf", "hll", "hllc", "hlld"])
@pytest.mark.parametrize("direction", [1, 2, 3])
def test_riemann_flux_consistency(oracle_mod, riemann, direction):
    """F(U, U) = F(U) (rsolver_module.f90 solvers on identical states)."""
    rng = np.random.default_rng(5)
    for _ in range(50):
        p = np.array([rng.uniform(0.1, 3), *rng.uniform(-1, 1, 3), rng.uniform(0.05, 2), *rng.uniform(-1, 1, 3)])
        fo, fp = oracle_mod.riemann_face(direction, RS[riemann], 5.0 / 3.0, p, p)
        assert np.allclose(fo, fp, rtol=1e-13, atol=1e-14)


def test_riemann_flux_symmetry(oracle_mod):
    """Mirror states give mirrored HLLD fluxes (x -> -x flips vx, Bx)."""
    rng = np.random.default_rng(9)
    flip = np.array([1, -1, 1, 1, 1, -1, 1, 1.0])
    for _ in range(50):
        pl = np.array([rng.uniform(0.1, 3), *rng.uniform(-1, 1, 3), rng.uniform(0.05, 2), *rng.uniform(-1, 1, 3)])
        pr = np.array([rng.uniform(0.1, 3), *rng.uniform(-1, 1, 3), rng.uniform(0.05, 2), *rng.uniform(-1, 1, 3)])
        pr[5] = pl[5]
        f1, _ = oracle_mod.riemann_face(1, RS["hlld"], 5.0 / 3.0, pl, pr)
        f2, _ = oracle_mod.riemann_face(1, RS["hlld"], 5.0 / 3.0, pr * flip, pl * flip)
        # mass, energy and transverse momenta/field fluxes change sign; normal momentum flux does not
        sgn = np.array([-1, 1, -1, -1, -1, 0, -1, -1.0])
        assert np.allclose(f2[[0, 1, 2, 3, 4, 6, 7]], (sgn * f1)[[0, 1, 2, 3, 4, 6, 7]], rtol=1e-11, atol=1e-12)


@pytest.mark.parametrize("rec", ["ppm", "weno"])
def test_reconstruction_exact_on_low_degree_data(oracle_mod, rec):
    """Uniform grid: WENO-Z face values are exact for quadratic cell averages
    (every sub-stencil is exact, the weights sum to one); PPM for linear."""
    w = oracle_mod.weights(REC[rec], np.full(5, 0.1))
    x = np.arange(-2, 3) * 0.1
    # cell averages of f over [x-h/2, x+h/2]
    for coef in ([0.3, -1.2, 0.0], [1.0, 0.5, 2.0]) if rec == "weno" else ([0.3, -1.2, 0.0], [2.0, 0.7, 0.0]):
        a, b, c = coef
        avg = a + b * x + c * (x ** 2 + 0.1 ** 2 / 12.0)
        vm, vp = oracle_mod.recon_cell(REC[rec], w, avg)
        fm = a + b * (-0.05) + c * 0.05 ** 2
        fp = a + b * 0.05 + c * 0.05 ** 2
        assert abs(vm - fm) < 1e-12 and abs(vp - fp) < 1e-12


def test_ct_keeps_div_b_at_roundoff(oracle_mod):
    spec, prim, eps = models.blast_3d(20, recon="weno", riemann="hlld", radius=0.2, p_in=1.0)
    spec["fix_periodic_normal_faces"] = 1
    o, p, e = run_oracle(oracle_mod, spec, prim, eps, 6)
    bmax = np.abs(interior(p, spec)[..., 5:8]).max()
    assert o.max_divb() * (1.0 / 20) / bmax <= 1e-13


def test_periodic_conservation(oracle_mod):
    """Mass and total energy are conserved to roundoff while no wave has
    reached the periodic boundary (there the lower normal face lags a stage,
    fromrvetou.f90:201-207 vs boundary.f90:430-433, and FROMRVETOU's magnetic
    energy uses the lagged face)."""
    spec, prim, eps = models.blast_3d(24, recon="ppm", riemann="hlld", radius=0.12, p_in=1.0)
    spec["fix_periodic_normal_faces"] = 1
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    c0 = interior(o.get_array(capi.ARR_CONS), spec)
    for _ in range(3):
        o.rk3_step(o.finddt())
    c1 = interior(o.get_array(capi.ARR_CONS), spec)
    for v in (0, 4):
        assert abs(c1[..., v].sum() - c0[..., v].sum()) <= 1e-13 * abs(c0[..., v].sum())


def test_centred_blast_is_mirror_symmetric(oracle_mod):
    spec, prim, eps = models.blast_3d(16, recon="weno", riemann="hlld", radius=0.25, p_in=1.0)
    prim[..., capi.IBX] = 0.0
    prim[..., capi.IBY] = 0.0
    prim[..., capi.IBZ] = 0.5
    spec["fix_periodic_normal_faces"] = 1
    _, p, e = run_oracle(oracle_mod, spec, prim, eps, 4)
    rho = interior(p, spec)[..., 0]
    assert np.allclose(rho, rho[:, :, ::-1], rtol=1e-12, atol=1e-13)
    assert np.allclose(rho, rho[:, ::-1, :], rtol=1e-12, atol=1e-13)
    assert np.allclose(rho, np.transpose(rho, (0, 2, 1)), rtol=1e-12, atol=1e-13)


def test_reference_weno_hlld_breaks_on_the_headline_blast(oracle_mod):
    """Documents why the benchmark enables the positivity fallback: the
    reference's WENO-Z + HLLD turns the 100:1 blast non-finite within a few
    steps (negative reconstructed face pressure -> NaN sound speed)."""
    spec, prim, eps = models.blast_3d(32)
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    bad = False
    for _ in range(6):
        o.rk3_step(o.finddt())
        p, _ = o.get_state()
        if not np.isfinite(interior(p, spec)).all():
            bad = True
            break
    assert bad
    spec["positivity_fallback"] = 1
    _, p, _ = run_oracle(oracle_mod, spec, prim, eps, 6)
    assert np.isfinite(interior(p, spec)).all()


def test_brio_wu_structure(oracle_mod):
    """Brio-Wu at t = 0.1 (riemann1d.f90:229-250): the known wave pattern."""
    spec, prim, eps = models.brio_wu(400)
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    t, n = o.evolve(0.1, 100000)
    assert t == 0.1
    p, _ = o.get_state()
    rho = p[3, 3, 3:403, 0]
    # cell By (FROMRVETOU's average of the y faces); in 1D the lower y face
    # keeps its initial value, so the face array itself is not the field
    by = o.get_array(capi.ARR_BCELL)[3, 3, 3:403, 1]
    x = (np.arange(400) + 0.5) / 400
    assert abs(rho[x < 0.3].mean() - 1.0) < 1e-3 and abs(rho[x > 0.9].mean() - 0.125) < 1e-3
    assert 0.6 < rho[(x > 0.5) & (x < 0.54)].mean() < 0.75  # post compound-wave plateau
    assert by.min() > -1.05 and by.max() < 1.05  # small PPM overshoot at the fast rarefaction
    assert o.max_divb() >= 0.0


def _alfven_error(oracle_mod, n, recon):
    """Relative L1 of B_y after one period of the 3D CP Alfven wave, whose
    exact solution then equals the initial state."""
    from cumc3d_b200 import capi
    spec, prim, eps = models.alfven_3d(n, recon=recon)
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    c0 = o.get_array(capi.ARR_CONS)
    t, _ = o.evolve(spec["t_end"], 100000)
    c = o.get_array(capi.ARR_CONS)
    o.close()
    assert t == spec["t_end"]
    sl = (slice(3, n + 3),) * 3
    a, b = c[sl][..., 6], c0[sl][..., 6]
    return np.abs(a - b).sum() / np.abs(b).sum()


@pytest.mark.parametrize("recon", ["weno", "tvdmc"])
def test_alfven_wave_converges_at_second_order(oracle_mod, recon):
    """Known answer for smooth MHD: after one period the wave is back where
    it started, and the error falls at least at second order (the
    dimension-by-dimension flux and the CT average bound the order)."""
    e = [_alfven_error(oracle_mod, n, recon) for n in (8, 16, 32)]
    orders = np.log2(np.array(e[:-1]) / np.array(e[1:]))
    assert np.all(orders > 1.8), (e, orders)
    assert e[-1] < 3e-3


@pytest.mark.parametrize("riemann", ["hlld", "hllc", "hll", "lf"])
def test_stationary_contact_is_exact_for_the_contact_resolving_solvers(oracle_mod, riemann):
    """An isolated stationary contact (density jump at equal pressure, at
    rest, normal field only) is a fixed point of HLLD and HLLC -- their
    middle wave sits on it with zero mass flux (Miyoshi & Kusano 2005) --
    bit for bit; HLL and LF smear it."""
    left = dict(rho=1.0, p=1.0, vx=0.0, vy=0.0, vz=0.0, by=0.0, bz=0.0)
    right = dict(rho=0.3, p=1.0, vx=0.0, vy=0.0, vz=0.0, by=0.0, bz=0.0)
    for recon in ("ppm", "weno", "tvdmc"):
        spec, prim, eps = models.riemann_1d(100, left, right, 0.8, recon=recon, riemann=riemann)
        o = oracle_mod.Oracle(spec)
        o.set_state(prim, eps)
        o.initial_update()
        p0, _ = o.get_state()
        for _ in range(30):
            o.rk3_step(o.finddt())
        p, _ = o.get_state()
        o.close()
        d = np.abs(p[3, 3, 3:-3, 0] - p0[3, 3, 3:-3, 0]).max()
        if riemann in ("hlld", "hllc"):
            assert d == 0.0, (recon, d)
        else:
            assert d > 0.05, (recon, d)


def _entropy_wave_error(oracle_mod, n, recon):
    """Mean |rho - rho_exact| after one period of a density wave carried at
    v = 1, p = 1 through a periodic 1D tube (exact: the initial state)."""
    import math
    from cumc3d_b200.capi import IRHO, ITAU, IVX
    spec = models._base_spec(n, 1, 1, 1, (0, 0, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), (0.0, 1.0), cfl=0.4,
                             recon=recon, riemann="hlld", precision="fp64", model=dict(gamma=1.4, floor="eps"),
                             name="entropy_wave_%d" % n)
    prim, eps = models._alloc(n, 1, 1)
    x = models.centers(spec["xF"])
    prim[..., IRHO] = (1.0 + 0.2 * np.sin(2.0 * math.pi * x))[None, None, :]
    prim[..., IVX] = 1.0
    prim[..., ITAU] = 1.0
    eps[...] = prim[..., ITAU] / prim[..., IRHO] / 0.4
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    p0, _ = o.get_state()
    t, _ = o.evolve(1.0, 1000000)
    p, _ = o.get_state()
    o.close()
    assert t == 1.0
    return np.abs(p[3, 3, 3:-3, IRHO] - p0[3, 3, 3:-3, IRHO]).mean()


@pytest.mark.parametrize("recon,order", [("weno", 3.3), ("ppm", 1.8), ("tvdmc", 1.6), ("tvdvl", 1.7),
                                         ("tvdmm", 1.5)])
def test_1d_entropy_wave_converges_at_the_scheme_order(oracle_mod, recon, order):
    """Known answer for a smooth 1D flow: WENO-Z beyond third order at
    these resolutions (fifth in space, SSP-RK3 in time), PPM second, the TVD
    limiters between first and second (they clip the smooth extrema)."""
    e = [_entropy_wave_error(oracle_mod, n, recon) for n in (32, 64, 128)]
    orders = np.log2(np.array(e[:-1]) / np.array(e[1:]))
    assert np.all(orders > order), (e, orders)
