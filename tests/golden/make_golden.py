"""Regenerate the golden fixtures of tests/test_golden.py from the CPU oracle.

    python tests/golden/make_golden.py

The reference (Fortran, leon-astrophy/cumc3d) cannot be built or run in this
environment and ships no golden data, so these fixtures are outputs of the
oracle restatement (oracle/cumc_oracle.cpp); they pin it (and, through
tests/test_golden.py, the CUDA engine) against regressions.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cumc3d_b200 import capi, models  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    # config 1: Brio-Wu, PPM + HLLD, CFL 0.8, outflow, t_end = 0.1
    "brio_wu_800": dict(builder=lambda: models.brio_wu(800), t_end=0.1),
    # small 3D blast, WENO-Z + HLLD, 3 steps, with the benchmark's options
    "blast3d_12_weno_hlld": dict(builder=lambda: models.blast_3d(12, radius=0.2), steps=3,
                                 opts=dict(positivity_fallback=1, fix_periodic_normal_faces=1)),
    # cylindrical torus hooks (floors, point mass, clamps), 2 steps
    "torus_cyl_16x8x16": dict(builder=lambda: models.torus_cyl(16, 8, 16, r_range=(4.0, 16.0),
                                                              z_range=(-6.0, 6.0)), steps=2),
}


# pinned on the oracle only (their engine runs are compared with the oracle
# directly in the GPU parity suite)
ORACLE_CASES = {
    # the riemann model's Orszag-Tang vortex (riemann2d.f90 test 15), PPM + HLLD
    "orszag_tang_24": dict(builder=lambda: models.riemann_2d(15, 24), steps=6),
    # the spherical torus (torus-sph GET_MODEL), FIXPOLE, pseudo-Newtonian source
    "torus_sph_20x12x6": dict(builder=lambda: models.torus_sph(20, 12, 6, r_range=(2.0, 10.0)), steps=3),
}


def run_case(name, runner):
    c = CASES[name] if name in CASES else ORACLE_CASES[name]
    spec, prim, eps = c["builder"]()
    spec.update(c.get("opts", {}))
    s = runner(spec)
    s.set_state(prim, eps)
    s.initial_update()
    if "t_end" in c:
        t, n = s.evolve(c["t_end"], 100000)
    else:
        for _ in range(c["steps"]):
            dt = s.finddt()
            s.rk3_step(dt) if hasattr(s, "rk3_step") else s.rungekutta(dt)
        t, n = None, c["steps"]
    p, e = s.get_state()
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    sl = (slice(3, nz + 3), slice(3, ny + 3), slice(3, nx + 3))
    return dict(prim=p[sl], eps=e[sl], bcell=s.get_array(capi.ARR_BCELL)[sl], steps=np.int64(n))


def main():
    O.build()
    for name in list(CASES) + list(ORACLE_CASES):
        out = run_case(name, O.Oracle)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
