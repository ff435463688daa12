"""z-slab groups (cumc_group_*): one grid cut along z into slabs that swap
three ghost planes with their neighbours twice per RK stage.  Against the
undivided grid, bit for bit, step by step: the periodic blast (a ring of
slabs, even and uneven cuts, FP64 and FP32), outflow z, and the cylindrical
torus with its z velocity clamps."""
import numpy as np
import pytest

from cumc3d_b200 import capi, engine, models

pytestmark = pytest.mark.gpu


def compare(spec, prim, eps, sizes, steps):
    g = engine.SlabGroup(spec, sizes)
    s = engine.Solver(spec)
    g.set_state(prim, eps)
    s.set_state(prim, eps)
    g.initial_update()
    s.initial_update()
    for _ in range(steps):
        dg, ds = g.finddt(), s.finddt()
        assert dg == ds
        g.step(dg)
        s.rungekutta(ds)
    nz = spec["nz"]
    pg, eg = g.get_state()
    ps, es = s.get_state()
    for a, b in ((pg, ps[3:nz + 3]), (eg, es[3:nz + 3]),
                 (g.get_array(capi.ARR_CONS), s.get_array(capi.ARR_CONS)[3:nz + 3]),
                 (g.get_array(capi.ARR_BCELL), s.get_array(capi.ARR_BCELL)[3:nz + 3])):
        a, b = a[:, 3:-3, 3:-3], b[:, 3:-3, 3:-3]  # interior in x and y too
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), int((a != b).sum())
    g.close()
    s.close()


@pytest.mark.parametrize("sizes", [(12, 12), (8, 9, 7)])
def test_periodic_blast_ring_bitwise(sizes):
    spec, prim, eps = models.blast_3d(24, nx=24, ny=20, nz=24, radius=0.2, p_in=1.0)
    spec["fix_periodic_normal_faces"] = 1
    compare(spec, prim, eps, sizes, 4)


def test_periodic_blast_fp32_bitwise():
    spec, prim, eps = models.blast_3d(20, radius=0.2, p_in=1.0, precision="fp32")
    compare(spec, prim, eps, (10, 10), 3)


@pytest.mark.parametrize("recon", ["weno", "ppm"])
def test_outflow_z_bitwise(recon):
    spec, prim, eps = models.smooth_state(16, 12, 20, 3, boundary_flag=(0, 0, 1, 1, 1, 1), recon=recon, seed=5)
    compare(spec, prim, eps, (9, 11), 3)


def test_cylindrical_torus_with_z_clamps_bitwise():
    spec, prim, eps = models.torus_cyl(nr=24, nphi=12, nz=24)
    spec["positivity_fallback"] = 1
    compare(spec, prim, eps, (12, 12), 3)


def test_refused_configurations():
    import math
    spec, prim, eps = models.smooth_state(12, 12, 12, 3, coordinate_flag=2, boundary_flag=(1, 1, 3, 3, 0, 0),
                                          x_range=(1.0, 3.0), y_range=(0.0, math.pi), z_range=(0.0, 2 * math.pi),
                                          fixpole=1)
    g = engine.SlabGroup(spec, (6, 6))
    g.set_state(prim, eps)
    with pytest.raises(engine.CumcError, match="FIXPOLE"):
        g.initial_update()
    g.close()
    spec, prim, eps = models.blast_3d(12)
    with pytest.raises(ValueError):
        engine.SlabGroup(spec, (10, 2))
