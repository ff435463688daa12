"""What the trained smooth-face network gains over the method without it, on
the CP Alfven wave at 256^3 (WENO-Z + HLLD + CT, the bench's flag settings:
the network every 8 steps, logit threshold -4, a full-WENO-Z audit every 24
steps at 1e-5): the warps of the y and z sweeps that reconstruct with the
linear optimal weights instead of WENO-Z's nonlinear ones
(weno_module.f90:363-404), the step time with the flag against the same
form without it, and the accuracy against the plain FP64 form."""
import os

import numpy as np
import pytest
import torch

from cumc3d_b200 import capi, engine, models
from cumc3d_b200.accuracy import rel_l1

pytestmark = pytest.mark.gpu

N, WARM, STEPS = 256, 8, 24
PARAMS = os.path.join(os.path.dirname(engine.__file__), "data", "flag_mlp.npy")


def timed(spec, prim, eps, learned):
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    if learned:
        s.learn_set(np.load(PARAMS), threshold=-4.0, audit_interval=24, audit_tol=1e-5, flag_interval=8)
    s.autotune()
    s.evolve(1e30, WARM)
    s.sync()
    stream = torch.cuda.ExternalStream(s.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    s.evolve(1e30, STEPS)
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / STEPS
    linear = [float((s.learn_flags(d)[1] != 0).mean()) for d in range(3)] if learned else None
    cons = s.get_array(capi.ARR_CONS)[3:N + 3, 3:N + 3, 3:N + 3]
    s.close()
    return ms, linear, cons


def test_the_trained_flag_gains_over_the_method_without_it():
    spec, prim, eps = models.alfven_3d(N, recon="weno")
    ms64, _, ref = timed(dict(spec, precision="fp64"), prim, eps, False)
    ms64l, lin64, c64l = timed(dict(spec, precision="fp64", learned=1), prim, eps, True)
    ms32, _, c32 = timed(dict(spec, precision="fp32"), prim, eps, False)
    ms32l, lin32, c32l = timed(dict(spec, precision="fp32", learned=1), prim, eps, True)
    print("ms/step: fp64 %.2f, fp64+learned %.2f, fp32 %.2f, fp32+learned %.2f; linear warps %s %s" % (
        ms64, ms64l, ms32, ms32l, lin64, lin32))
    # most warps of the y and z sweeps run the linear weights (a warp of the x
    # sweep spans 32 cells along it, so fewer of those qualify)
    assert min(lin64[1:]) > 0.7 and min(lin32[1:]) > 0.6
    # the skipped nonlinear weights show in the step time of both forms
    assert ms64l < 0.9 * ms64
    assert ms32l < ms32
    # within relative L1 1e-5 of the plain FP64 form, the reduced forms' accuracy bar
    for c in (c64l, c32, c32l):
        assert rel_l1(c, ref).max() <= 1e-5
