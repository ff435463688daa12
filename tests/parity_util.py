"""Shared helpers: run the same workload on the CUDA engine and on the oracle."""
import numpy as np

from cumc3d_b200 import capi


def interior(a, spec):
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    return a[3:nz + 3, 3:ny + 3, 3:nx + 3]


def rel_l1(a, b):
    """sum|a-b| / sum|b| per conserved/primitive variable (last axis)."""
    num = np.abs(a - b).reshape(-1, a.shape[-1]).sum(axis=0)
    den = np.abs(b).reshape(-1, b.shape[-1]).sum(axis=0)
    den = np.where(den == 0, 1.0, den)
    return num / den


def run_pair(spec, prim, eps, steps, oracle_mod, use_evolve=False, t_end=None):
    """Advance both implementations; return (gpu, oracle) dicts of arrays + per-step dt lists."""
    from cumc3d_b200.engine import Solver
    g = Solver(spec)
    o = oracle_mod.Oracle(spec)
    g.set_state(prim, eps)
    o.set_state(prim, eps)
    g.initial_update()
    o.initial_update()
    dts_g, dts_o = [], []
    if use_evolve:
        tg, ng = g.evolve(t_end, steps)
        to, no = o.evolve(t_end, steps)
        dts_g.append((tg, ng))
        dts_o.append((to, no))
    else:
        for _ in range(steps):
            dg = g.finddt()
            do = o.finddt()
            dts_g.append(dg)
            dts_o.append(do)
            g.rungekutta(do)
            o.rk3_step(do)
    out = []
    for s in (g, o):
        p, e = s.get_state()
        out.append(dict(prim=p, eps=e, cons=s.get_array(capi.ARR_CONS), bcell=s.get_array(capi.ARR_BCELL),
                        cs=s.get_array(capi.ARR_CS), divb=s.find_divb() if hasattr(s, "find_divb") else s.max_divb()))
    g.close()
    o.close()
    return out[0], out[1], dts_g, dts_o


def assert_bitwise(gpu, orc, spec, what=("prim", "eps", "bcell", "cs")):
    for key in what:
        a = interior(gpu[key], spec)
        b = interior(orc[key], spec)
        if not np.array_equal(a, b, equal_nan=True):
            diff = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))))
            raise AssertionError("%s differs at %d entries, first %s: gpu=%r oracle=%r" % (
                key, len(diff), diff[0].tolist(), a[tuple(diff[0])], b[tuple(diff[0])]))
