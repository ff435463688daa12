"""Exact operation counts (CPU): the oracle on its counting scalar type
gives the same bits as on double, its phases add up to its total, and the
per-zone-update counts in profiles/op_counts.json (the flop side of the
benchmark's roofline, written by oracle/count_ops.py) are those of the
current oracle."""
import json
import os

import numpy as np

from cumc3d_b200 import capi, models
from oracle import count_ops
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_counting_type_changes_no_bit_and_phases_add_up():
    spec, prim, eps = models.blast_3d(10, radius=0.2)
    spec["positivity_fallback"] = 1
    out = []
    for counting in (False, True):
        o = O.Oracle(spec, counting=counting)
        o.set_state(prim, eps)
        o.initial_update()
        O.reset_counts()
        dt = o.finddt()
        o.rk3_step(dt)
        out.append((dt, o.get_array(capi.ARR_CONS)))
        o.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1].view(np.uint64), out[1][1].view(np.uint64))
    total = O.get_counts()
    parts = [O.get_counts(ph) for ph in O.PHASES]
    for k in total:
        assert total[k] == sum(p[k] for p in parts)
    assert all(O.get_counts(ph)["add"] > 0 for ph in ("recon", "riemann", "finddt", "other"))


def test_committed_counts_are_those_of_the_current_oracle():
    with open(os.path.join(ROOT, "profiles", "op_counts.json")) as f:
        got = json.load(f)
    for name in ("blast3d_weno_hlld", "briowu_ppm_hlld"):
        build, scales, ndir = count_ops.WORKLOADS[name]
        for s in scales:
            c, zones = count_ops.count_one(lambda s=s: build(s))
            want = got[name]["samples"][str(zones)]["flops_per_zone_update"]
            assert sum(sum(c[ph][k] for k in ("add", "mul", "div", "sqrt")) for ph in count_ops.PHASES) == want
    # WENO-Z reconstruction: the same integer count at every interior face
    r = got["blast3d_weno_hlld"]["per_zone_update"]["recon"]
    assert all(float(v).is_integer() for v in r.values())
