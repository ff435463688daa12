"""FP32 form against the FP64 plain form (its oracle for precision claims).

FP32 carries the reconstruction, face EOS and Riemann flux; FP64 keeps the
RK accumulation, the CT face-B update, the primitive recovery (including the
energy - kinetic - magnetic subtraction) and the CFL reduction.
"""
import math

import numpy as np
import pytest

from cumc3d_b200 import capi, models
from cumc3d_b200.engine import Solver
from parity_util import interior, rel_l1

pytestmark = pytest.mark.gpu


def run(spec, prim, eps, steps=None, t_end=None):
    s = Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    if t_end is not None:
        s.evolve(t_end)
    else:
        s.evolve(1e30, steps)
    cons = s.get_array(capi.ARR_CONS)
    divb = s.find_divb()
    s.close()
    return cons, divb


@pytest.mark.parametrize("recon", ["ppm", "weno"])
def test_alfven_fp32_l1_smooth(recon):
    """Config 3 (reduced to 32^3): CP Alfven wave, one period; the FP32 form
    must stay within 1e-5 relative L1 of the FP64 plain form."""
    spec, prim, eps = models.alfven_3d(32, recon=recon)
    c64, d64 = run(spec, prim, eps, t_end=spec["t_end"])
    spec32 = dict(spec, precision="fp32")
    c32, d32 = run(spec32, prim, eps, t_end=spec["t_end"])
    l1 = rel_l1(interior(c32, spec), interior(c64, spec))
    print("alfven", recon, "rel L1 fp32 vs fp64 per conserved variable:", l1)
    assert np.all(l1[[0, 1, 2, 3, 4]] <= 1e-5)
    bscale = 1.0 * 32
    assert d64 / bscale <= 1e-13 and d32 / bscale <= 1e-13  # CT keeps div B at roundoff in both forms


def test_blast_fp32_runs_and_keeps_divb():
    spec, prim, eps = models.blast_3d(32, recon="weno", riemann="hlld", radius=0.2)
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    c64, d64 = run(spec, prim, eps, steps=20)
    c32, d32 = run(dict(spec, precision="fp32"), prim, eps, steps=20)
    l1 = rel_l1(interior(c32, spec), interior(c64, spec))
    print("blast rel L1 fp32 vs fp64:", l1)
    assert np.all(np.isfinite(l1))
    assert np.all(l1 <= 1e-3)
    assert d32 / 32 <= 1e-13
