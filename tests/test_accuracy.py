"""The accuracy measures of the precision forms (CPU): relative L1 per
variable and the shock-position distance in zones."""
import numpy as np

from cumc3d_b200.accuracy import features, rel_l1, shock_offsets


def test_rel_l1_per_variable():
    b = np.ones((4, 5, 3))
    a = b.copy()
    a[0, 0, 1] = 1.5
    l1 = rel_l1(a, b)
    assert l1[0] == 0 and l1[2] == 0 and abs(l1[1] - 0.5 / 20) < 1e-15


def test_shock_offsets_measure_a_shift_in_zones():
    x = np.arange(400)
    ref = np.where(x < 200, 1.0, 0.125) + np.where(x < 300, 0.0, 0.5)
    same, m0 = shock_offsets(ref, ref)
    assert len(same) == 2 and m0 == 0.0
    moved = np.where(x < 201, 1.0, 0.125) + np.where(x < 300, 0.0, 0.5)
    offs, m1 = shock_offsets(ref, moved)
    assert abs(m1 - 1.0) < 1e-12
    # a jump smeared over two zones moves its centroid by half a zone
    smear = ref.copy()
    smear[200] = 0.5625
    _, m2 = shock_offsets(ref, smear)
    assert abs(m2 - 0.5) < 1e-12
    assert features(np.ones(50)) == []


def test_brio_wu_features_of_the_oracle_profile(oracle_mod):
    from cumc3d_b200 import models
    spec, prim, eps = models.brio_wu(400)
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    o.evolve(0.1, 10 ** 6)
    p, _ = o.get_state()
    rho = p[3, 3, 3:403, 0]
    f = features(rho)
    # compound wave, contact and slow shock at least
    assert len(f) >= 3
    _, m = shock_offsets(rho, rho)
    assert m == 0.0
    o.close()
