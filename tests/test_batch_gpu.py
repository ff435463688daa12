"""Batched 1D engine (many reference n_dim = 1 runs in one persistent launch).

Every batched problem must be bit-identical to the same problem run alone
through the 3D engine with ny = nz = 1 (which is itself bit-identical to the
oracle), for every reconstruction and Riemann solver, at uneven sizes; the
full seeded workload (512 problems, n log-uniform in [128, 4096]) is checked
through size-independent properties and a bitwise sample.
"""
import numpy as np
import pytest

from cumc3d_b200 import capi, models
from cumc3d_b200.engine import BatchSolver, CumcError, Solver

pytestmark = pytest.mark.gpu

VARS_CELL = [0, 1, 2, 3, 4, 6, 7]  # rho, v, p, the k = 1 / l = 1 faces of By, Bz


def problem_specs(params, t_end, **kw):
    out = []
    for prm in params:
        spec, prim, eps = models.riemann_1d(prm["n"], prm["left"], prm["right"], prm["bx"], t_end=t_end, **kw)
        out.append((spec, prim, eps))
    return out


def run_alone(spec, prim, eps):
    s = Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    t, n = s.evolve(spec["t_end"])
    p, e = s.get_state()
    s.close()
    return p[3, 3], e[3, 3], t, n  # the (k, l) = (1, 1) row


def run_batch(problems, positivity_fallback=0, max_steps=0, check=True):
    b = BatchSolver([sp for sp, _, _ in problems], positivity_fallback=positivity_fallback)
    for i, (_, prim, eps) in enumerate(problems):
        b.set_state(i, prim, eps)
    t, steps, status = b.run(max_steps, check=check)
    rows = [b.get_state(i) for i in range(len(problems))]
    b.close()
    return rows, t, steps, status


def assert_row_equal(pa, ea, pb, eb, n, label):
    for v in VARS_CELL:
        a, b = pa[3:n + 3, v], pb[3:n + 3, v]
        if not np.array_equal(a, b):
            j = int(np.argwhere(a != b)[0][0])
            raise AssertionError("%s var %d differs at j=%d: batch=%r alone=%r" % (label, v, j + 1, a[j], b[j]))
    assert np.array_equal(pa[2:n + 3, 5], pb[2:n + 3, 5]), label + " Bx faces 0..n"
    assert np.array_equal(ea[3:n + 3], eb[3:n + 3]), label + " eps"


def small_params(count, seed, nmin=8, nmax=160):
    return models.batch_problems(count, seed=seed, nmin=nmin, nmax=nmax)


@pytest.mark.parametrize("recon,riemann", [("ppm", "hlld"), ("weno", "hlld"), ("tvdmc", "hlld"),
                                           ("tvdmm", "hllc"), ("tvdvl", "hll"), ("ppm", "lf"),
                                           ("weno", "hllc"), ("ppm", "hll")])
def test_batch_bitwise_vs_3d_engine(recon, riemann):
    params = small_params(6, seed=11)
    probs = problem_specs(params, 0.05, recon=recon, riemann=riemann)
    rows, t, steps, status = run_batch(probs, check=False)
    for i, (spec, prim, eps) in enumerate(probs):
        if status[i] != 0:
            # the scheme itself breaks down on this problem (as the reference's
            # does): the lone run must report the same
            with pytest.raises(CumcError) as ei:
                run_alone(spec, prim, eps)
            assert ei.value.code == capi.CUMC_ESTATE
            continue
        pa, ea, ta, na = run_alone(spec, prim, eps)
        assert t[i] == ta and steps[i] == na, (i, t[i], ta, steps[i], na)
        assert_row_equal(rows[i][0], rows[i][1], pa, ea, spec["nx"], "problem %d (%s/%s)" % (i, recon, riemann))


def test_batch_matches_oracle_directly(oracle_mod):
    """Two tiny problems against the CPU restatement, no 3D engine between."""
    params = small_params(2, seed=5, nmin=16, nmax=40)
    probs = problem_specs(params, 0.03)
    rows, t, steps, status = run_batch(probs)
    for i, (spec, prim, eps) in enumerate(probs):
        o = oracle_mod.Oracle(spec)
        o.set_state(prim, eps)
        o.initial_update()
        to, no = o.evolve(spec["t_end"], 10 ** 6)
        po, eo = o.get_state()
        o.close()
        assert t[i] == to and steps[i] == no
        assert_row_equal(rows[i][0], rows[i][1], po[3, 3], eo[3, 3], spec["nx"], "problem %d" % i)


def test_batch_uneven_sizes_and_edges():
    """n = 1, 2, 3 (fewer cells than stencil width) and a large problem, one launch."""
    base = small_params(5, seed=3)
    for prm, n in zip(base, [1, 2, 3, 700, 5]):
        prm["n"] = n
    probs = problem_specs(base, 0.02)
    rows, t, steps, status = run_batch(probs)
    for i, (spec, prim, eps) in enumerate(probs):
        pa, ea, ta, na = run_alone(spec, prim, eps)
        assert t[i] == ta and steps[i] == na
        assert_row_equal(rows[i][0], rows[i][1], pa, ea, spec["nx"], "n=%d" % spec["nx"])


@pytest.mark.parametrize("cluster_size,coop_min_n", [(2, 40), (4, 64), (16, 100), (1, 1 << 30)])
def test_batch_cluster_shapes_are_bitwise_identical(cluster_size, coop_min_n):
    """The launch shape (CTAs per shared problem, the size above which a
    problem is shared) changes the split of the cells, not a bit of the
    results: against the default shape, uneven sizes around the thresholds."""
    base = small_params(7, seed=13, nmin=30, nmax=300)
    for prm, n in zip(base, [257, 41, 64, 65, 3, 101, 300]):
        prm["n"] = n
    probs = problem_specs(base, 0.03)
    ref, t0, s0, _ = run_batch(probs)
    b = BatchSolver([sp for sp, _, _ in probs])
    b.set_cluster(cluster_size, coop_min_n)
    for i, (_, prim, eps) in enumerate(probs):
        b.set_state(i, prim, eps)
    t, steps, _ = b.run()
    rows = [b.get_state(i) for i in range(len(probs))]
    b.close()
    assert np.array_equal(t, t0) and np.array_equal(steps, s0)
    for i, (spec, _, _) in enumerate(probs):
        assert_row_equal(rows[i][0], rows[i][1], ref[i][0], ref[i][1], spec["nx"], "cluster %d" % i)


def test_batch_cluster_shape_is_checked():
    probs = problem_specs(small_params(1, seed=2), 0.01)
    b = BatchSolver([sp for sp, _, _ in probs])
    for cs, mn in ((3, 100), (32, 100), (8, 0)):
        with pytest.raises(CumcError):
            b.set_cluster(cs, mn)
    b.close()


def test_batch_max_steps_and_rerun():
    params = small_params(3, seed=7, nmin=64, nmax=200)
    probs = problem_specs(params, 0.5)
    rows, t, steps, status = run_batch(probs, max_steps=4)
    assert list(steps) == [4, 4, 4] and np.all(t < 0.5)
    # a second run on the same handle restarts (INITIAL_UPDATE, t = 0) from
    # the state the first one left: 4 + 4 steps equal 8 steps bit for bit
    b = BatchSolver([sp for sp, _, _ in probs])
    for i, (_, prim, eps) in enumerate(probs):
        b.set_state(i, prim, eps)
    b.run(4)
    _, steps2, _ = b.run(4)
    split = [b.get_state(i) for i in range(len(probs))]
    b.close()
    rows8, _, steps8, _ = run_batch(probs, max_steps=8)
    assert list(steps2) == [4, 4, 4] and list(steps8) == [8, 8, 8]
    for i, (spec, _, _) in enumerate(probs):
        assert_row_equal(split[i][0], split[i][1], rows8[i][0], rows8[i][1], spec["nx"], "restart %d" % i)


def test_batch_full_workload_properties():
    """512 seeded problems, n log-uniform in [128, 4096], t_end 0.1, HLLD+PPM."""
    params = models.batch_problems(512)
    probs = problem_specs(params, 0.1)
    rows, t, steps, status = run_batch(probs, positivity_fallback=1)
    assert np.all(status == 0)
    assert np.all(t == 0.1)
    for i, (spec, prim, eps) in enumerate(probs):
        p, e = rows[i]
        n = spec["nx"]
        # the eps floor of the 1D models is eps >= 0 (custom.f90), so 0 is allowed
        assert np.all(np.isfinite(p[3:n + 3])) and np.all(p[3:n + 3, 0] > 0) and np.all(e[3:n + 3] >= 0)
    # bitwise against the 3D engine on the four smallest problems
    order = np.argsort([prm["n"] for prm in params])[:4]
    for i in order:
        spec, prim, eps = probs[i]
        spec = dict(spec, positivity_fallback=1)
        pa, ea, ta, na = run_alone(spec, prim, eps)
        assert t[i] == ta and steps[i] == na
        assert_row_equal(rows[i][0], rows[i][1], pa, ea, spec["nx"], "problem %d" % i)


def test_batch_fp32_close_to_fp64():
    params = small_params(8, seed=13, nmin=64, nmax=400)
    p64 = problem_specs(params, 0.05)
    p32 = problem_specs(params, 0.05, precision="fp32")
    r64, t64, _, s64 = run_batch(p64)
    r32, t32, _, s32 = run_batch(p32)
    assert np.all(s64 == 0) and np.all(s32 == 0)
    num = den = 0.0
    for i, (spec, _, _) in enumerate(p64):
        n = spec["nx"]
        a, b = r32[i][0][3:n + 3, :5], r64[i][0][3:n + 3, :5]
        num += np.abs(a - b).sum()
        den += np.abs(b).sum()
    # discontinuous data: shocks may move by a fraction of a cell
    assert num / den < 1e-3
