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


def _resume(spec, prim, eps, n_total, n_first, make):
    a = make(spec)
    a.set_state(prim, eps)
    a.initial_update()
    a.evolve(1e30, n_total)
    straight = a.get_state()
    a.close()
    b = make(spec)
    b.set_state(prim, eps)
    b.initial_update()
    b.evolve(1e30, n_first)
    pm, em = b.get_state()
    b.close()
    c = make(spec)
    c.set_state(pm, em)
    c.initial_update()
    c.evolve(1e30, n_total - n_first)
    resumed = c.get_state()
    c.close()
    return straight, resumed


def test_checkpoint_resume_is_bitwise():
    """N steps straight == k steps -> get_state -> new handle -> N-k steps."""
    spec, prim, eps = models.blast_3d(24, radius=0.2)
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 0
    (pa, ea), (pc, ec) = _resume(spec, prim, eps, 6, 3, Solver)
    assert np.array_equal(interior(pa, spec), interior(pc, spec))
    assert np.array_equal(interior(ea, spec), interior(ec, spec))


def test_checkpoint_resume_with_frozen_faces_follows_the_reference(oracle_mod):
    """With fix_periodic_normal_faces = 1 (face 0 of a periodic direction
    follows face n; an option, the reference leaves face 0 frozen) the face is
    refilled after the recovery that used its previous value, so the cell
    field of cell 1 lags one stage behind the written faces and a restart
    from them is not bitwise (the CPU restatement behaves the same).  The
    engine must resume exactly as the restatement does."""
    spec, prim, eps = models.blast_3d(24, radius=0.2)
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    (_, _), (pg, eg) = _resume(spec, prim, eps, 6, 3, Solver)

    def oracle(sp):
        return oracle_mod.Oracle(sp)
    (_, _), (po, eo) = _resume(spec, prim, eps, 6, 3, oracle)
    assert np.array_equal(interior(pg, spec), interior(po, spec))
    assert np.array_equal(interior(eg, spec), interior(eo, spec))


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
