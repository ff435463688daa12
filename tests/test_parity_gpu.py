"""FP64 plain form of the CUDA engine against the CPU oracle.

The plain form keeps the reference's floating-point operation order and is
compiled without FMA contraction, so the bar here is bitwise equality (which
implies relative L1 = 0 <= 1e-12 per variable) on the interior state, the
cell fields and the CFL step of every step.
"""
import numpy as np
import pytest

from cumc3d_b200 import models
from parity_util import assert_bitwise, interior, rel_l1, run_pair

pytestmark = pytest.mark.gpu


def test_brio_wu_full_run_bitwise(oracle_mod):
    """Config 1: 1D Brio-Wu, PPM + HLLD, CFL 0.8, outflow, t_end = 0.1."""
    spec, prim, eps = models.brio_wu(800)
    g, o, dg, do = run_pair(spec, prim, eps, 100000, oracle_mod, use_evolve=True, t_end=0.1)
    assert dg[0][1] == do[0][1]  # same number of steps
    assert dg[0][0] == do[0][0] == 0.1
    assert_bitwise(g, o, spec)
    l1 = rel_l1(interior(g["cons"], spec), interior(o["cons"], spec))
    assert np.all(l1 <= 1e-12)


@pytest.mark.parametrize("recon", ["tvdmm", "tvdvl", "tvdmc", "ppm", "weno"])
@pytest.mark.parametrize("riemann", ["lf", "hll", "hllc", "hlld"])
def test_blast3d_all_schemes_bitwise(oracle_mod, recon, riemann):
    # a 10:1 blast resolved by 8 zones across; the 100:1 blast of the bench
    # needs more zones before WENO keeps the face pressure positive
    spec, prim, eps = models.blast_3d(16, recon=recon, riemann=riemann, radius=0.25, p_in=1.0)
    g, o, dg, do = run_pair(spec, prim, eps, 3, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)
    assert_bitwise(g, o, spec, what=("cons",))


@pytest.mark.parametrize("fix", [0, 1])
def test_periodic_normal_faces_option(oracle_mod, fix):
    spec, prim, eps = models.blast_3d(16, recon="weno", riemann="hlld", radius=0.3, p_in=1.0)
    spec["fix_periodic_normal_faces"] = fix
    g, o, dg, do = run_pair(spec, prim, eps, 4, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)
    assert g["divb"] == o["divb"]


def test_smooth_2d_reflect_bitwise(oracle_mod):
    spec, prim, eps = models.smooth_state(20, 18, 1, 2, boundary_flag=(2, 1, 2, 2, 1, 1), recon="ppm",
                                          riemann="hlld", seed=3)
    g, o, dg, do = run_pair(spec, prim, eps, 4, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)


def test_smooth_3d_mixed_bc_bitwise(oracle_mod):
    spec, prim, eps = models.smooth_state(12, 10, 14, 3, boundary_flag=(1, 2, 0, 0, 2, 1), recon="weno",
                                          riemann="hllc", seed=5)
    g, o, dg, do = run_pair(spec, prim, eps, 3, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)


def test_cylindrical_torus_hooks_bitwise(oracle_mod):
    """Cylindrical geometry + torus floors, point-mass source and velocity clamps."""
    spec, prim, eps = models.torus_cyl(24, 16, 24, r_range=(4.0, 16.0), z_range=(-6.0, 6.0))
    g, o, dg, do = run_pair(spec, prim, eps, 3, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)


def test_spherical_fixpole_bitwise(oracle_mod):
    """Spherical (r, theta, phi) with axis boundaries and the FIXPOLE average."""
    import math
    spec, prim, eps = models.smooth_state(16, 12, 8, 3, coordinate_flag=2, boundary_flag=(1, 1, 3, 3, 0, 0),
                                          x_range=(1.0, 3.0), y_range=(0.0, math.pi), z_range=(0.0, 2 * math.pi),
                                          recon="ppm", riemann="hlld", seed=7, fixpole=1)
    spec["model"]["source"] = "pm_sph"
    spec["model"]["bc"] = "torus_sph"
    g, o, dg, do = run_pair(spec, prim, eps, 2, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)


@pytest.mark.parametrize("grid,recon", [("uniform", "ppm"), ("shipped_r_theta", "ppm"), ("uniform", "weno")])
def test_spherical_torus_model_bitwise(oracle_mod, grid, recon):
    """The spherical torus (model/torus-sph: pseudo-Newtonian point mass
    with r_sh = 1, torus floors, radial clamps, polar axis with FIXPOLE) from
    its own initial model, PPM + HLLD at CFL 0.8 as the reference ships it:
    on a uniform grid, and on the refined r and theta faces the model reads
    (with 8 phi cells); and WENO-Z with the positivity fallback."""
    import math
    from cumc3d_b200 import grids
    if grid == "uniform":
        spec, prim, eps = models.torus_sph(32, 20, 8, r_range=(2.0, 10.0), recon=recon)
    else:
        nx, ny, _, r, th, _ = grids.spherical_torus_grid()
        ph = models.faces(0.0, 2.0 * math.pi, 8)
        spec, prim, eps = models.torus_sph(nx, ny, 8, faces=(r, th, ph), recon=recon)
    spec["positivity_fallback"] = 1 if recon == "weno" else 0
    g, o, dg, do = run_pair(spec, prim, eps, 4, oracle_mod)
    assert np.isfinite(interior(g["prim"], spec)).all()
    assert dg == do
    assert_bitwise(g, o, spec)
    assert_bitwise(g, o, spec, what=("cons",))


def test_reference_cylindrical_torus_model_bitwise(oracle_mod):
    """The reference's own torus-cyn setup (pseudo-Newtonian r_sh = 1,
    PPM + HLLD at CFL 0.8), from its initial model."""
    spec, prim, eps = models.torus_cyn(40, 8, 40, r_range=(1.5, 9.5), z_range=(-4.0, 4.0))
    g, o, dg, do = run_pair(spec, prim, eps, 6, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)
    assert_bitwise(g, o, spec, what=("cons",))


@pytest.mark.parametrize("tm", range(1, 14))
def test_riemann_model_1d_set_to_end_time_bitwise(oracle_mod, tm):
    """The riemann model's 1D tests (riemann1d.f90: Toro 1-5, interacting
    blast waves, Shu-Osher, Sedov, Dai-Woodward, Brio-Wu, seven
    discontinuities, magnetosonic rarefactions, two fast shocks), PPM + HLLD
    at CFL 0.8, each to its end time in one device time loop."""
    spec, prim, eps = models.riemann_1d_test(tm, 200)
    g, o, dg, do = run_pair(spec, prim, eps, 100000, oracle_mod, use_evolve=True, t_end=spec["t_end"])
    assert dg == do and dg[0][0] == spec["t_end"]
    assert_bitwise(g, o, spec)
    assert_bitwise(g, o, spec, what=("cons",))


@pytest.mark.parametrize("tm", range(1, 13))
def test_riemann_model_2d_hydro_problems_bitwise(oracle_mod, tm):
    """The riemann model's 2D hydrodynamic tests (riemann2d.f90: Gresho,
    Toro's blast and explosion, implosion, Kelvin-Helmholtz,
    Rayleigh-Taylor with gravity, the four-quadrant problems); ten steps."""
    recon, riemann = ("weno", "hllc") if tm % 3 == 0 else ("ppm", "hlld")
    spec, prim, eps = models.riemann_2d(tm, 40, recon=recon, riemann=riemann)
    g, o, dg, do = run_pair(spec, prim, eps, 10, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)
    assert_bitwise(g, o, spec, what=("cons",))


@pytest.mark.parametrize("tm", [1, 2])
def test_riemann_model_3d_problems_bitwise(oracle_mod, tm):
    spec, prim, eps = models.riemann_3d(tm, 20)
    g, o, dg, do = run_pair(spec, prim, eps, 5, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)


@pytest.mark.parametrize("tm,recon,riemann", [(13, "ppm", "hlld"), (14, "weno", "hlld"), (15, "ppm", "hlld"),
                                              (15, "weno", "hllc"), (16, "ppm", "hlld"), (17, "weno", "hlld"),
                                              (18, "ppm", "hlld"), (19, "tvdmc", "hll")])
def test_riemann_model_2d_mhd_problems_bitwise(oracle_mod, tm, recon, riemann):
    """The riemann model's 2D MHD tests (riemann2d.f90:441-640): current
    sheet, rotor (outflow), Orszag-Tang, blast, Kelvin-Helmholtz,
    Rayleigh-Taylor (the model's constant-gravity source, reflecting y) and
    the advected current loop; ten steps, every bit."""
    spec, prim, eps = models.riemann_2d(tm, 40, 40 if tm != 19 else 20, recon=recon, riemann=riemann)
    g, o, dg, do = run_pair(spec, prim, eps, 10, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)
    assert_bitwise(g, o, spec, what=("cons",))
    assert g["divb"] == o["divb"]


def test_blast_100to1_with_positivity_fallback_bitwise(oracle_mod):
    """The headline blast (p 10 : 0.1, beta 0.2 outside) breaks the reference's
    WENO-Z + HLLD within a few steps (negative face pressure, see
    test_oracle_invariants); with the optional first-order fallback both
    implementations run it, bit for bit."""
    spec, prim, eps = models.blast_3d(24, recon="weno", riemann="hlld", radius=0.2)
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    g, o, dg, do = run_pair(spec, prim, eps, 8, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)
    assert np.isfinite(interior(g["prim"], spec)).all()


@pytest.mark.parametrize("tuning", [
    dict(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=4),
    dict(split=True, tpb_recon=128, tpb_riemann=64, riemann_min_blocks=1),
    dict(split=False, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=1),
    dict(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=1, recon_tile=1),
    dict(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=4, recon_tile=2),
    dict(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=6, recon_tile=1),
    dict(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=4, recon_tile=3),
    dict(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=5, recon_tile=4),
    dict(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=15, recon_tile=1),
    dict(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=14, recon_tile=4),
])
@pytest.mark.parametrize("recon", ["weno", "ppm", "tvdmc"])
def test_every_launch_shape_is_bitwise_identical(oracle_mod, tuning, recon):
    """The autotuner's candidates differ in blocking, staging and register
    budget only (grid extents not multiples of the tiles)."""
    from cumc3d_b200.engine import Solver
    spec, prim, eps = models.smooth_state(20, 12, 10, 3, boundary_flag=(1, 1, 0, 0, 2, 2), recon=recon,
                                          riemann="hlld", seed=11)
    g = Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    g.set_tuning(**tuning)
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    for _ in range(3):
        dt = o.finddt()
        assert g.finddt() == dt
        g.rungekutta(dt)
        o.rk3_step(dt)
    pg, eg = g.get_state()
    po, eo = o.get_state()
    assert np.array_equal(interior(pg, spec), interior(po, spec))
    assert np.array_equal(interior(eg, spec), interior(eo, spec))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_concurrent_sweeps_are_bitwise_identical(oracle_mod, precision):
    """The three flux sweeps as concurrent branches (their own streams and
    face-state buffers, joined before the EMFs): the same bits as the
    sequential sweeps, eager and in the captured step graph; FP64 also
    against the oracle."""
    from cumc3d_b200.engine import Solver
    spec, prim, eps = models.blast_3d(24, recon="weno", riemann="hlld", radius=0.25, p_in=1.0, precision=precision)
    runs = []
    for conc, graph in ((False, False), (True, False), (True, True)):
        g = Solver(spec)
        g.set_state(prim, eps)
        g.initial_update()
        g.set_tuning(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=4, recon_tile=1)
        g.set_concurrent_sweeps(conc)
        if graph:
            g.evolve(1e30, 4)
        else:
            for _ in range(4):
                g.rungekutta(g.finddt())
        p, e = g.get_state()
        runs.append((interior(p, spec), interior(e, spec)))
        g.close()
    for p, e in runs[1:]:
        assert np.array_equal(p.view(np.uint64), runs[0][0].view(np.uint64))
        assert np.array_equal(e.view(np.uint64), runs[0][1].view(np.uint64))
    if precision == "fp64":
        o = oracle_mod.Oracle(spec)
        o.set_state(prim, eps)
        o.initial_update()
        for _ in range(4):
            o.rk3_step(o.finddt())
        po, eo = o.get_state()
        o.close()
        assert np.array_equal(runs[2][0].view(np.uint64), interior(po, spec).view(np.uint64))


@pytest.mark.parametrize("n,nz", [(96, 96), (128, 40)])
def test_headline_blast_parameters_at_size_bitwise(oracle_mod, n, nz):
    """The bench's own blast (radius 0.1, p 10 : 0.1, B = (1, 1, 0)/sqrt 2,
    WENO-Z + HLLD + CT, CFL 0.4, positivity fallback and the periodic-face
    option) at 96^3 and on a 128 x 128 x 40 slab, through the captured step
    graph with the autotuned launch shapes, against the oracle bit for bit;
    the fallback counters of the two agree."""
    from cumc3d_b200.engine import Solver
    spec, prim, eps = models.blast_3d(n, nz=nz, recon="weno", riemann="hlld")
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    g = Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    g.autotune()
    g.fallback_count(1)
    tg, kg = g.evolve(1e30, 6)
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    to = 0.0
    for _ in range(6):
        dt = o.finddt()
        o.rk3_step(dt)
        to += dt
    assert kg == 6 and tg == to
    pg, eg = g.get_state()
    po, eo = o.get_state()
    assert np.array_equal(interior(pg, spec), interior(po, spec))
    assert np.array_equal(interior(eg, spec), interior(eo, spec))
    assert g.fallback_count() == o.fallback_count()
    g.close()
    o.close()


@pytest.mark.parametrize("recon", ["ppm", "weno"])
def test_alfven_benchmark_config_bitwise(oracle_mod, recon):
    """The circularly polarised Alfven wave workload (k = 2 pi (1, 1, 1),
    amplitude 0.1, face B from an edge vector potential, periodic, HLLD, CFL
    0.4) at 40^3 with the workload's PPM and WENO-Z, through the captured
    step graph with the autotuned launch shapes: 8 steps bit for bit, and
    div B equal."""
    from cumc3d_b200.engine import Solver
    spec, prim, eps = models.alfven_3d(40, recon=recon)
    g = Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    g.autotune()
    tg, kg = g.evolve(1e30, 8)
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    to = 0.0
    for _ in range(8):
        dt = o.finddt()
        o.rk3_step(dt)
        to += dt
    assert kg == 8 and tg == to
    pg, eg = g.get_state()
    po, eo = o.get_state()
    assert np.array_equal(interior(pg, spec).view(np.uint64), interior(po, spec).view(np.uint64))
    assert np.array_equal(interior(eg, spec).view(np.uint64), interior(eo, spec).view(np.uint64))
    assert g.find_divb() == o.max_divb()
    g.close()
    o.close()


def test_torus_benchmark_config_at_96x64x96_bitwise(oracle_mod):
    """The cylindrical torus workload (GM = 1 point mass, constant-l
    polytrope, A_phi field loops at min beta 100, 1% seeded pressure noise,
    r in [2, 42], z in [-20, 20], WENO-Z + HLLD + CT, positivity fallback and
    the periodic-face option) at 96 x 64 x 96, three steps, bit for bit."""
    spec, prim, eps = models.torus_cyl(nr=96, nphi=64, nz=96, recon="weno", riemann="hlld")
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    g, o, dg, do = run_pair(spec, prim, eps, 3, oracle_mod)
    assert dg == do
    assert_bitwise(g, o, spec)
    assert_bitwise(g, o, spec, what=("cons",))


def test_tma_staged_reconstruction_on_the_headline_blast(oracle_mod):
    """The TMA-staged, persistent reconstruction (recon_tile 3) on the bench's
    blast at 64^3 (tiles that wrap the persistent grid several times, boxes
    that reach past the padded grid): bit for bit the oracle's; and refused
    where the padded x extent is odd (its rows are not 16-byte multiples)."""
    from cumc3d_b200.engine import CumcError, Solver
    spec, prim, eps = models.blast_3d(64)
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    g = Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    g.set_tuning(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=4, recon_tile=3)
    tg, kg = g.evolve(1e30, 4)
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    to = 0.0
    for _ in range(4):
        dt = o.finddt()
        o.rk3_step(dt)
        to += dt
    assert tg == to
    pg, eg = g.get_state()
    po, eo = o.get_state()
    assert np.array_equal(interior(pg, spec), interior(po, spec))
    assert np.array_equal(interior(eg, spec), interior(eo, spec))
    g.close()
    o.close()
    spec, prim, eps = models.smooth_state(21, 12, 10, 3, recon="weno", riemann="hlld", seed=2)
    g = Solver(spec)
    g.set_state(prim, eps)
    g.initial_update()
    with pytest.raises(CumcError):
        g.set_tuning(split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=4, recon_tile=3)
    g.close()
