"""The riemann model's 1D set (CPU): the builders restated from
model/riemann/src/riemann1d.f90, and a known-answer pin of the oracle on its
hydrodynamic shock tubes -- the exact solution of the ideal-gas Riemann
problem (the pressure function solved by Newton's method and the fan
sampled at x/t, as in Toro, Riemann Solvers and Numerical Methods for Fluid
Dynamics, ch. 4), written here independently, against which the oracle's
PPM + HLLD density must converge as the grid is refined."""
import math

import numpy as np
import pytest

from cumc3d_b200 import models
from cumc3d_b200.capi import IRHO, ITAU, IVX
from oracle import oracle as O


def exact_riemann(g, left, right, xi):
    """Density, velocity, pressure of the exact solution at x/t = xi."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)

    def f(p, r, pk, ck):
        if p > pk:  # shock
            a, b = 2.0 / ((g + 1.0) * r), (g - 1.0) / (g + 1.0) * pk
            q = math.sqrt(a / (p + b))
            return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (p + b))
        e = (g - 1.0) / (2.0 * g)   # rarefaction
        return 2.0 * ck / (g - 1.0) * ((p / pk) ** e - 1.0), (p / pk) ** (-(g + 1.0) / (2.0 * g)) / (r * ck)

    p = max(1e-8, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = f(p, rl, pl, cl)
        fr, dr = f(p, rr, pr, cr)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(1e-12, p - dp)
        if abs(dp) < 1e-14 * p:
            break
    u = 0.5 * (ul + ur) + 0.5 * (f(p, rr, pr, cr)[0] - f(p, rl, pl, cl)[0])
    out = np.empty((len(xi), 3))
    for i, s in enumerate(xi):
        if s <= u:   # left of the contact
            r0, u0, p0, c0, sgn = rl, ul, pl, cl, 1.0
        else:
            r0, u0, p0, c0, sgn = rr, ur, pr, cr, -1.0
        if p > p0:   # shock
            ss = u0 - sgn * c0 * math.sqrt((g + 1.0) / (2.0 * g) * p / p0 + (g - 1.0) / (2.0 * g))
            behind = (s >= ss) if sgn > 0 else (s <= ss)
            rs = r0 * (p / p0 + (g - 1.0) / (g + 1.0)) / ((g - 1.0) / (g + 1.0) * p / p0 + 1.0)
            out[i] = (rs, u, p) if behind else (r0, u0, p0)
        else:        # rarefaction
            cs = c0 * (p / p0) ** ((g - 1.0) / (2.0 * g))
            head, tail = u0 - sgn * c0, u - sgn * cs
            if (s <= head) if sgn > 0 else (s >= head):
                out[i] = (r0, u0, p0)
            elif (s >= tail) if sgn > 0 else (s <= tail):
                out[i] = (r0 * (p / p0) ** (1.0 / g), u, p)
            else:    # inside the fan
                k = 2.0 / (g + 1.0) + sgn * (g - 1.0) / ((g + 1.0) * c0) * (u0 - s)
                uu = 2.0 / (g + 1.0) * (sgn * c0 + (g - 1.0) / 2.0 * u0 + s)
                out[i] = (r0 * k ** (2.0 / (g - 1.0)), uu, p0 * k ** (2.0 * g / (g - 1.0)))
    return out, p, u


@pytest.mark.parametrize("tm", [1, 3])
def test_exact_solution_conserves_mass_and_energy(tm):
    """The sampled exact solution of a tube at rest at both ends keeps the
    mass and total energy of the initial state while the waves stay inside
    [0, 1]; the momentum grows by (p_L - p_R) t."""
    _, g, _, t, left, right = models.RIEMANN_1D[tm]
    st = lambda s: (s.get(IRHO, 0.0), s.get(IVX, 0.0), s.get(ITAU, 0.0))  # noqa: E731
    L, R = st(left), st(right)
    x = (np.arange(200000) + 0.5) / 200000
    ex, p, u = exact_riemann(g, L, R, (x - 0.5) / t)
    rho, vel, pre = ex[:, 0], ex[:, 1], ex[:, 2]
    assert np.all(np.abs(ex[:10] - L) < 1e-12) and np.all(np.abs(ex[-10:] - R) < 1e-12)
    energy = lambda r, v, q: q / (g - 1.0) + 0.5 * r * v * v  # noqa: E731
    assert abs(rho.mean() - 0.5 * (L[0] + R[0])) < 2e-5 * L[0]
    e0 = 0.5 * (energy(*L) + energy(*R))
    assert abs(energy(rho, vel, pre).mean() - e0) < 2e-5 * e0
    assert abs((rho * vel).mean() - (L[2] - R[2]) * t) < 2e-5 * max(1.0, L[2] * t)


def test_brio_wu_builder_is_test_10():
    a, b = models.brio_wu(400), models.riemann_1d_test(10, 400)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2], equal_nan=True)


@pytest.mark.parametrize("tm", [1, 2, 3, 4, 5])
def test_oracle_converges_to_the_exact_solution(tm):
    name, g, _, t_end, left, right = models.RIEMANN_1D[tm]
    state = lambda s: (s.get(IRHO, 0.0), s.get(IVX, 0.0), s.get(ITAU, 0.0))  # noqa: E731
    errs = []
    for nx in (200, 400):
        spec, prim, eps = models.riemann_1d_test(tm, nx)
        o = O.Oracle(spec)
        o.set_state(prim, eps)
        o.initial_update()
        t, _ = o.evolve(t_end, 100000)
        p, _ = o.get_state()
        o.close()
        assert t == t_end
        x = models.centers(spec["xF"])[3:-3]
        ex, _, _ = exact_riemann(g, state(left), state(right), (x - 0.5) / t_end)
        rho = p[3, 3, 3:-3, IRHO]
        errs.append(np.mean(np.abs(rho - ex[:, 0])) / np.mean(ex[:, 0]))
    # first order at the discontinuities: the L1 error falls with the cell size
    assert errs[1] < 0.8 * errs[0], errs
    assert errs[1] < 0.05, errs


@pytest.mark.parametrize("tm", range(1, 14))
def test_every_1d_test_runs_to_its_end_time(tm):
    spec, prim, eps = models.riemann_1d_test(tm, 100)
    o = O.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    t, n = o.evolve(spec["t_end"], 100000)
    p, _ = o.get_state()
    o.close()
    assert t == spec["t_end"] and n > 10 and np.isfinite(p[3, 3, 3:-3]).all()
