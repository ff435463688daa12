"""cumc_batch_run1_noalloc: one 1D problem with no device allocation.

Collected last on purpose (file name): it must give the same answer whether
it runs alone in a fresh process or after every other test has used the
device.  The comparison is against the existing batched entry points
(cumc_batch_create / _set_state / _run / _get_state) on the same problem;
both launch the same kernel, so the tolerance is zero (bit-identical).
"""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from cumc3d_b200 import capi, models
from cumc3d_b200.engine import BatchSolver, CumcError, batch_run1_noalloc

pytestmark = pytest.mark.gpu

TOL = 0.0  # same kernel, same inputs: identical results


def problem(n, seed, precision="fp64", recon="ppm", riemann="hlld", t_end=0.05):
    prm = models.batch_problems(1, seed=seed, nmin=n, nmax=n)[0]
    return models.riemann_1d(n, prm["left"], prm["right"], prm["bx"], t_end=t_end, precision=precision,
                             recon=recon, riemann=riemann)


def existing_entry(spec, prim, eps, fallback=1):
    b = BatchSolver([spec], positivity_fallback=fallback)
    b.set_state(0, prim, eps)
    t, steps, status = b.run()
    p, e = b.get_state(0)
    b.close()
    return p, e, float(t[0]), int(steps[0])


def assert_same(a, b):
    pa, ea, ta, na = a
    pb, eb, tb, nb = b
    np.testing.assert_allclose(pa, pb, rtol=TOL, atol=TOL)
    np.testing.assert_allclose(ea, eb, rtol=TOL, atol=TOL)
    assert ta == tb and na == nb


def test_noalloc_two_calls_in_a_row_match_existing_entry():
    big = problem(2000, seed=21)    # > 1024 zones: shared by a CTA cluster
    small = problem(300, seed=22)   # one CTA
    ref_big = existing_entry(*big)
    ref_small = existing_entry(*small)
    first = batch_run1_noalloc(*big, positivity_fallback=1)
    second = batch_run1_noalloc(*small, positivity_fallback=1)
    assert_same(first, ref_big)
    assert_same(second, ref_small)
    # the scratch is cleared on every call: the big problem again gives the same
    assert_same(batch_run1_noalloc(*big, positivity_fallback=1), ref_big)


def test_noalloc_fp32_and_weno_match_existing_entry():
    for spec, prim, eps in (problem(700, seed=23, precision="fp32"), problem(1500, seed=24, recon="weno")):
        ref = existing_entry(spec, prim, eps)
        assert_same(batch_run1_noalloc(spec, prim, eps, positivity_fallback=1), ref)
        assert_same(batch_run1_noalloc(spec, prim, eps, positivity_fallback=1), ref)


def test_noalloc_tvd_weights_match_existing_entry():
    # TVD-MC (and minmod) reads the two TVD weights per cell, the branch of the
    # shared weight routine that PPM and WENO never take
    for recon, riemann in (("tvdmc", "hlld"), ("tvdmm", "hllc")):
        spec, prim, eps = problem(900, seed=27, recon=recon, riemann=riemann)
        ref = existing_entry(spec, prim, eps)
        assert_same(batch_run1_noalloc(spec, prim, eps, positivity_fallback=1), ref)
        assert_same(batch_run1_noalloc(spec, prim, eps, positivity_fallback=1), ref)


# run in a fresh interpreter so no other test's allocations move the numbers
_NO_GROWTH = textwrap.dedent("""
    import sys
    sys.path.insert(0, sys.argv[1])
    import torch
    from cumc3d_b200 import models
    from cumc3d_b200.engine import batch_run1_noalloc

    def problem(n, seed):
        prm = models.batch_problems(1, seed=seed, nmin=n, nmax=n)[0]
        return models.riemann_1d(n, prm["left"], prm["right"], prm["bx"], t_end=0.01)

    batch_run1_noalloc(*problem(200, 31), positivity_fallback=1)   # loads the module
    torch.cuda.init()
    free0, _ = torch.cuda.mem_get_info()
    for n, seed in ((4096, 32), (128, 33), (2500, 34), (700, 35)):
        batch_run1_noalloc(*problem(n, seed), positivity_fallback=1)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    print("FREE", free0, free1)
""")


def test_noalloc_calls_allocate_no_device_memory():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _NO_GROWTH, root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("FREE")][-1]
    free0, free1 = (int(x) for x in line.split()[1:])
    assert free1 == free0, "device free memory changed by %d bytes over four calls" % (free0 - free1)


def test_noalloc_rejects_more_than_4096_zones():
    spec, prim, eps = problem(4097, seed=25)
    with pytest.raises(CumcError) as ei:
        batch_run1_noalloc(spec, prim, eps)
    assert ei.value.code == capi.CUMC_EINVAL and "4096" in str(ei.value)
    # the limit itself is accepted
    spec, prim, eps = problem(4096, seed=26, t_end=0.002)
    assert_same(batch_run1_noalloc(spec, prim, eps, positivity_fallback=1), existing_entry(spec, prim, eps))
