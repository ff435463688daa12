"""The timed CPU baseline (the oracle built with -march=native on the host
that runs it) computes the same bits as the parity build: a 3D blast step
sequence in a fresh process on the native build against this process's
generic build."""
import hashlib
import os
import subprocess
import sys
import textwrap

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_RUN = textwrap.dedent("""
    import hashlib, sys
    sys.path.insert(0, sys.argv[1])
    from oracle import oracle as O
    print("RECIPE", O.use_native())
    from cumc3d_b200 import models
    sp, p, e = models.blast_3d(24, nz=16, radius=0.2)
    sp["positivity_fallback"] = 1
    o = O.Oracle(sp)
    o.set_state(p, e)
    o.initial_update()
    for _ in range(3):
        o.rk3_step(o.finddt())
    pr, ep = o.get_state()
    print("DIGEST", hashlib.sha256(pr[3:-3, 3:-3, 3:-3].tobytes() + ep[3:-3, 3:-3, 3:-3].tobytes()).hexdigest())
""")


def test_native_build_gives_the_parity_builds_bits(oracle_mod):
    r = subprocess.run([sys.executable, "-c", _RUN, ROOT], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = dict(ln.split(" ", 1) for ln in r.stdout.splitlines() if ln.startswith(("RECIPE", "DIGEST")))
    assert "march=native" in lines["RECIPE"]
    from cumc3d_b200 import models
    sp, p, e = models.blast_3d(24, nz=16, radius=0.2)
    sp["positivity_fallback"] = 1
    o = oracle_mod.Oracle(sp)
    o.set_state(p, e)
    o.initial_update()
    for _ in range(3):
        o.rk3_step(o.finddt())
    pr, ep = o.get_state()
    o.close()
    want = hashlib.sha256(pr[3:-3, 3:-3, 3:-3].tobytes() + ep[3:-3, 3:-3, 3:-3].tobytes()).hexdigest()
    assert lines["DIGEST"] == want
    assert np.isfinite(pr[3:-3, 3:-3, 3:-3]).all()
