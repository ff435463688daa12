"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

CASES = sorted(make_golden.CASES)


def load(name):
    with np.load(os.path.join(HERE, "golden", name + ".npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden(oracle_mod, name):
    ref = load(name)
    out = make_golden.run_case(name, oracle_mod.Oracle)
    for k in ("prim", "eps", "bcell", "steps"):
        assert np.array_equal(out[k], ref[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_engine_reproduces_golden(name):
    from cumc3d_b200.engine import Solver
    ref = load(name)
    out = make_golden.run_case(name, Solver)
    for k in ("prim", "eps", "bcell", "steps"):
        assert np.array_equal(out[k], ref[k]), k


@pytest.mark.parametrize("name", sorted(make_golden.ORACLE_CASES))
def test_oracle_reproduces_golden_models(oracle_mod, name):
    ref = load(name)
    out = make_golden.run_case(name, oracle_mod.Oracle)
    for k in ("prim", "eps", "bcell", "steps"):
        assert np.array_equal(out[k], ref[k]), k
