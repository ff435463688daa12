"""Learned smooth-face flag of the FP32 WENO form (GPU).

Checks, each against the CPU oracle or the form without the flag:
  * harvested samples (features + FP64 labels) bit-identical to the oracle;
  * the GPU trainer's loss and gradient against the oracle's FP64 ones;
  * tensor-core inference against an emulation of its BF16 arithmetic;
  * the fused reconstruction kernel with no cell flagged equals plain FP32;
  * the audit: every step audited reproduces plain FP32, no audit does not;
  * a trained network flags smooth cells, not shocks, and what it gains.
"""
import numpy as np
import pytest

from cumc3d_b200 import capi, engine, models
from parity_util import interior

pytestmark = pytest.mark.gpu

DELTA = 1e-4  # label: the linear weights change a face value by less than this (relative)


def stencil_rows(prim, bcell, spec, direction):
    """(n_cells, 7, 5) FP64 stencils in the harvest's cell order (x fastest)."""
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    tb1 = 1 if direction == 0 else 0
    tb2 = 1 if direction == 2 else 2
    fields = [prim[..., v] for v in range(5)] + [bcell[..., tb1], bcell[..., tb2]]
    out = np.empty((nz, ny, nx, 7, 5))
    for v, f in enumerate(fields):
        for m in range(5):
            o = m - 2
            sl = [slice(3, nz + 3), slice(3, ny + 3), slice(3, nx + 3)]
            ax = 2 - direction
            sl[ax] = slice(3 + o, (nz, ny, nx)[ax] + 3 + o)
            out[..., v, m] = f[tuple(sl)]
    return out.reshape(-1, 7, 5)


def run_fp64(spec, prim, eps, steps):
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    if steps:
        s.evolve(1e30, steps)
    return s


def harvest(spec, prim, eps, steps_list, stride=1):
    s = run_fp64(spec, prim, eps, 0)
    rows, done = [], 0
    for st in steps_list:
        if st > done:
            s.evolve(1e30, st - done)
            done = st
        for d in range(3):
            rows.append(s.learn_harvest(d, stride))
    s.close()
    return np.concatenate(rows)


def test_harvest_matches_oracle(oracle_mod):
    spec, prim, eps = models.blast_3d(12, radius=0.2, p_in=1.0)
    spec["fix_periodic_normal_faces"] = 1
    s = run_fp64(spec, prim, eps, 3)
    p, _ = s.get_state()
    bc = s.get_array(capi.ARR_BCELL)
    n = 12
    for d in range(3):
        got = s.learn_harvest(d, 1)
        st = stencil_rows(p, bc, spec, d)
        # the cell's own weights (face spacing can differ by an ulp between cells)
        dxa = np.diff(spec["xF" if d == 0 else "yF" if d == 1 else "zF"])
        wc = [oracle_mod.weights(capi.RECON["weno"], dxa[c:c + 5])[:10] for c in range(1, n + 1)]
        coord = np.indices((n, n, n))[2 - d].ravel()  # (z, y, x) order, x fastest; index along d
        ref = np.stack([oracle_mod.learn_sample(st[i], wc[coord[i]]) for i in range(st.shape[0])])
        assert got.shape == ref.shape
        assert np.array_equal(got, ref), "direction %d: %d rows differ" % (d, int((got != ref).any(1).sum()))
    s.close()


def test_gradient_matches_oracle(oracle_mod):
    spec, prim, eps = models.blast_3d(12, radius=0.2, p_in=1.0)
    samples = harvest(spec, prim, eps, [2])[:3000]
    P = engine.mlp_init(3)
    P[1536:1568] = np.linspace(-0.1, 0.1, 32)
    P[2656] = 0.2
    loss_g, g_g = engine.mlp_grad(P, samples, DELTA)
    loss_c, g_c = oracle_mod.mlp_loss_grad(P, samples, DELTA)
    assert abs(loss_g - loss_c) <= 1e-5 * max(1.0, abs(loss_c))
    scale = np.abs(g_c).max()
    assert np.abs(g_g - g_c).max() <= 1e-4 * scale + 1e-7
    # columns of the unused inputs carry no gradient
    assert np.all(g_g[0:1536].reshape(32, 48)[:, 35:] == 0)


def test_tensor_core_inference_matches_bf16_emulation(oracle_mod):
    spec, prim, eps = models.blast_3d(12, radius=0.2, p_in=1.0)
    X = harvest(spec, prim, eps, [2])[:1000, :35]  # 1000 rows: 7 full tiles and a partial one
    P = engine.mlp_init(5)
    P[1536:1568] = 0.05
    P[2592:2624] = 0.05
    z = engine.mlp_infer(P, X)
    zb = oracle_mod.mlp_forward_bf16(P, X)
    assert np.abs(z - zb).max() <= 2e-3 * (1.0 + np.abs(zb).max())
    z64 = oracle_mod.mlp_forward(P, X)
    assert np.abs(z - z64).max() <= 5e-2 * (1.0 + np.abs(z64).max())  # BF16 vs FP64: loose


def fp32_run(spec, prim, eps, steps, learned=None):
    sp = dict(spec, precision="fp32", learned=1 if learned is not None else 0)
    s = engine.Solver(sp)
    s.set_state(prim, eps)
    s.initial_update()
    if learned is not None:
        s.learn_set(**learned)
    s.evolve(1e30, steps)
    cons = s.get_array(capi.ARR_CONS)
    stats = s.learn_stats() if learned is not None else None
    s.close()
    return cons, stats


def flag_all_params(value=100.0):
    P = np.zeros(capi.LEARN_NP, dtype=np.float32)
    P[2656] = value
    return P


def test_fused_kernel_without_flags_equals_plain_fp32():
    spec, prim, eps = models.alfven_3d(32, recon="weno")
    plain, _ = fp32_run(spec, prim, eps, 8)
    off, st = fp32_run(spec, prim, eps, 8, dict(params=flag_all_params(-100.0), threshold=0.0,
                                                  audit_interval=4, audit_tol=1e-6))
    assert st["flagged"] == 0 and st["audits"] >= 2
    assert np.array_equal(interior(plain, spec), interior(off, spec))


def test_audit_every_step_reproduces_plain_fp32_and_no_audit_does_not():
    spec, prim, eps = models.alfven_3d(32, recon="weno")
    plain, _ = fp32_run(spec, prim, eps, 6)
    audited, st = fp32_run(spec, prim, eps, 6, dict(params=flag_all_params(), threshold=0.0, audit_interval=1,
                                                      audit_tol=0.0))
    # every cell but the two next to each end of a sweep is flagged
    assert st["audits"] >= 6 and st["flagged"] > 0.8 * st["audited"]
    assert np.array_equal(interior(plain, spec), interior(audited, spec))
    linear, st2 = fp32_run(spec, prim, eps, 6, dict(params=flag_all_params(), threshold=0.0, audit_interval=0,
                                                      audit_tol=0.0))
    assert st2["audits"] == 0
    a, b = interior(linear, spec), interior(plain, spec)
    assert not np.array_equal(a, b)
    # linear weights on a smooth wave stay close to WENO-Z
    assert np.abs(a - b).sum() / np.abs(b).sum() < 1e-3
    # an audit with zero tolerance sends every tile with a flagged cell back
    fb, st3 = fp32_run(spec, prim, eps, 4, dict(params=flag_all_params(), threshold=0.0, audit_interval=3,
                                                  audit_tol=0.0))
    assert st3["fallback_tiles"] > 0


def test_trained_flag_separates_smooth_from_shocked_cells():
    sa, pa, ea = models.alfven_3d(32, recon="weno")
    sb, pb, eb = models.blast_3d(32, radius=0.2, p_in=1.0)
    sb["positivity_fallback"] = 1
    smooth = harvest(sa, pa, ea, [0, 10, 20])
    shock = harvest(sb, pb, eb, [5, 15])
    data = np.concatenate([smooth, shock])
    rng = np.random.default_rng(0)
    rng.shuffle(data)
    n_tr = int(0.8 * len(data))
    P, losses = engine.mlp_train(data[:n_tr], engine.mlp_init(1), steps=1500, batch=4096, lr=2e-3, delta=DELTA)
    assert losses[-100:].mean() < 0.6 * losses[:20].mean()
    held = data[n_tr:]
    z = engine.mlp_infer(P, held[:, :35])
    y = held[:, 35] < DELTA
    acc = ((z > 0) == y).mean()
    assert acc > 0.9, acc
    # clearly non-smooth cells (change > 100 delta) are almost never flagged
    rough = held[:, 35] > 100 * DELTA
    assert rough.sum() > 100 and (z[rough] > 0).mean() < 0.02


@pytest.mark.parametrize("flag_interval", [1, 4])
def test_trained_flag_keeps_div_b_at_roundoff_on_a_periodic_box(flag_interval):
    """Face 0 and face n of a periodic axis are one face: the cells next to
    the ends of a sweep always use WENO-Z so both copies get the same flux
    and constrained transport keeps div B at roundoff."""
    import os
    P = np.load(os.path.join(os.path.dirname(engine.__file__), "data", "flag_mlp.npy"))
    spec, prim, eps = models.alfven_3d(48, recon="weno")
    sp = dict(spec, precision="fp32", learned=1)
    s = engine.Solver(sp)
    s.set_state(prim, eps)
    s.initial_update()
    s.learn_set(P, threshold=0.0, audit_interval=8, audit_tol=1e-5, flag_interval=flag_interval)
    s.evolve(1e30, 30)
    divb = s.find_divb()
    st = s.learn_stats()
    s.close()
    assert st["flagged"] > 0
    # |B| ~ 1, dx = 1/48: roundoff level is ~1e-13
    assert divb < 1e-11, divb


def fp64_learned_run(spec, prim, eps, steps, learned):
    sp = dict(spec, precision="fp64", learned=1)
    s = engine.Solver(sp)
    s.set_state(prim, eps)
    s.initial_update()
    s.learn_set(**learned)
    s.evolve(1e30, steps)
    cons = s.get_array(capi.ARR_CONS)
    divb = s.find_divb()
    stats = s.learn_stats()
    s.close()
    return cons, divb, stats


def plain_fp64(spec, prim, eps, steps):
    s = engine.Solver(dict(spec, precision="fp64"))
    s.set_state(prim, eps)
    s.initial_update()
    s.evolve(1e30, steps)
    cons = s.get_array(capi.ARR_CONS)
    s.close()
    return cons


def test_fp64_learned_without_flags_is_the_plain_form(oracle_mod):
    """The FP64 form with the flag network but no cell flagged runs the plain
    FP64 arithmetic: bit-identical to the plain form and to the oracle."""
    spec, prim, eps = models.alfven_3d(24, recon="weno")
    cons, _, st = fp64_learned_run(spec, prim, eps, 6, dict(params=flag_all_params(-100.0), threshold=0.0,
                                                               audit_interval=4, audit_tol=1e-6, flag_interval=2))
    assert st["flagged"] == 0 and st["audits"] >= 1
    ref = plain_fp64(spec, prim, eps, 6)
    assert np.array_equal(interior(cons, spec), interior(ref, spec))
    o = oracle_mod.Oracle(dict(spec, precision="fp64"))
    o.set_state(prim, eps)
    o.initial_update()
    o.evolve(1e30, 6)
    assert np.array_equal(interior(cons, spec), interior(o.get_array(capi.ARR_CONS), spec))
    o.close()


def test_fp64_learned_with_trained_flag_stays_close_to_plain():
    import os
    P = np.load(os.path.join(os.path.dirname(engine.__file__), "data", "flag_mlp.npy"))
    spec, prim, eps = models.alfven_3d(48, recon="weno")
    cons, divb, st = fp64_learned_run(spec, prim, eps, 30, dict(params=P, threshold=0.0, audit_interval=8,
                                                                  audit_tol=1e-5, flag_interval=4))
    ref = plain_fp64(spec, prim, eps, 30)
    a, b = interior(cons, spec).reshape(-1, 8), interior(ref, spec).reshape(-1, 8)
    l1 = np.abs(a - b).sum(0) / np.abs(b).sum(0)
    assert st["flagged"] > 0.5 * st["audited"]
    assert l1.max() < 1e-5, l1
    assert divb < 1e-11


def expected_warps(flags, tiles, spec, direction):
    """The linear decision of each warp of the staged reconstruction, restated
    from the stored per-cell flags: a warp (32 consecutive x-cells of one row)
    is linear when every one of its cells lies two or more cells inside the
    sweep, carries the flag together with its neighbours within two cells
    along the sweep, and sits in a 128-cell tile not marked to fall back."""
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    shape = [(nz, ny, nx + 2), (nz, ny + 2, nx), (nz + 2, ny, nx)][direction]
    sweep_axis = [2, 1, 0][direction]
    n = [nx, ny, nz][direction]
    g = np.moveaxis(flags.reshape(shape) != 0, sweep_axis, -1)
    tile_ok = np.moveaxis((tiles[np.arange(flags.size) >> 7] == 0).reshape(shape), sweep_axis, -1)
    ok = np.zeros_like(g)
    for c in range(2, n):
        ok[..., c] = g[..., c - 2:c + 3].all(-1) & tile_ok[..., c]
    ok = np.moveaxis(ok, -1, sweep_axis)
    nxc = (shape[2] + 31) // 32
    pad = np.zeros(shape[:2] + (nxc * 32,), dtype=bool)
    pad[..., :shape[2]] = ok
    return pad.reshape(shape[:2] + (nxc, 32)).all(-1).reshape(-1)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", ["all", "all_fallback", "trained"])
def test_warp_decisions_follow_the_dilated_flags(precision, case):
    """The per-warp decisions written after the network (k_learned_warps) equal
    the dilated per-cell rule restated in numpy, on a grid whose rows end in
    partial warps (72 cells: 74 along the x sweep).  Cases: every cell
    flagged (linear exactly where a warp lies two cells inside the sweep);
    the same with a zero-tolerance audit each step, which marks tiles to fall
    back; the trained network."""
    import os
    spec, prim, eps = models.alfven_3d(72, recon="weno")
    if case == "trained":
        P = np.load(os.path.join(os.path.dirname(engine.__file__), "data", "flag_mlp.npy"))
        learn = dict(params=P, threshold=0.0, audit_interval=0, audit_tol=1e-5)
    else:
        learn = dict(params=flag_all_params(), threshold=0.0, audit_interval=1 if case == "all_fallback" else 0,
                     audit_tol=0.0)
    s = engine.Solver(dict(spec, precision=precision, learned=1))
    s.set_state(prim, eps)
    s.initial_update()
    s.learn_set(flag_interval=1, **learn)
    s.evolve(1e30, 1)
    for d in range(3):
        flags, warps, tiles = s.learn_flags(d)
        exp = expected_warps(flags, tiles, spec, d)
        assert warps.shape == exp.shape
        assert np.array_equal(warps != 0, exp), (d, int((warps != 0).sum()), int(exp.sum()))
        if case == "all":
            assert 0 < exp.sum() < exp.size and not tiles.any()
        if case == "all_fallback":
            assert tiles.any()
    s.close()
