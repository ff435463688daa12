"""Checkpoint/resume and failure detection through the C-ABI (GPU).

Failures are injected on the host (a bad state handed to cumc_set_state); no
kernel is made to fault, trap or hang.
"""
import numpy as np
import pytest

from cumc3d_b200 import capi, models
from cumc3d_b200.engine import CumcError, Solver
from parity_util import interior

pytestmark = pytest.mark.gpu


def test_checkpoint_resume_is_bitwise():
    """N steps straight == k steps -> get_state -> new handle -> N-k steps."""
    spec, prim, eps = models.blast_3d(24, radius=0.2)
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    a = Solver(spec)
    a.set_state(prim, eps)
    a.initial_update()
    a.evolve(1e30, 6)
    pa, ea = a.get_state()
    b = Solver(spec)
    b.set_state(prim, eps)
    b.initial_update()
    b.evolve(1e30, 3)
    pm, em = b.get_state()
    b.close()
    c = Solver(spec)
    c.set_state(pm, em)
    c.initial_update()
    c.evolve(1e30, 3)
    pc, ec = c.get_state()
    assert np.array_equal(interior(pa, spec), interior(pc, spec))
    assert np.array_equal(interior(ea, spec), interior(ec, spec))


def test_negative_density_is_reported_and_handle_survives():
    spec, prim, eps = models.blast_3d(16, radius=0.2, p_in=1.0)
    bad = prim.copy()
    bad[3 + 5, 3 + 6, 3 + 7, capi.IRHO] = -1.0  # cell (j,k,l) = (8,7,6)
    s = Solver(spec)
    s.set_state(bad, eps)
    with pytest.raises(CumcError) as e:
        s.initial_update()
    assert e.value.code == capi.CUMC_ESTATE
    assert "(8,7,6)" in str(e.value)
    # the handle stays usable once a good state is loaded
    s.set_state(prim, eps)
    s.initial_update()
    t, n = s.evolve(1e30, 2)
    assert n == 2


def test_nan_inside_a_step_is_reported():
    spec, prim, eps = models.blast_3d(16, radius=0.2, p_in=1.0)
    bad_eps = eps.copy()
    bad_eps[3 + 2, 3 + 2, 3 + 2] = np.nan
    s = Solver(spec)
    s.set_state(prim, bad_eps)
    with pytest.raises(CumcError) as e:
        s.initial_update()
    assert e.value.code == capi.CUMC_ESTATE


def test_evolve_respects_t_end_and_max_steps():
    spec, prim, eps = models.brio_wu(200)
    s = Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    t, n = s.evolve(0.1, 5)
    assert n == 5 and t < 0.1
    t, n2 = s.evolve(0.1)
    assert t == 0.1 and n2 > 0
    t3, n3 = s.evolve(0.1)
    assert n3 == 0 and t3 == 0.1
