"""Every initial-model builder yields a spec that converts to a valid
cumc_config (CPU): face arrays of the right length, known option names,
model descriptor keys that exist -- a mistyped key is an error, not a
silently ignored default."""
import math

import numpy as np
import pytest

from cumc3d_b200 import capi, models

BUILDERS = [
    lambda: models.brio_wu(64),
    lambda: models.blast_3d(8),
    lambda: models.alfven_3d(8),
    lambda: models.torus_cyl(16, 8, 16),
    lambda: models.torus_cyn(16, 8, 16),
    lambda: models.torus_sph(16, 12, 8, r_range=(2.0, 10.0)),
    lambda: models.star_sph(16, 12, 8),
    lambda: models.collapsar_sph(16, 12, 8),
    lambda: models.smooth_state(8, 8, 8, 3, coordinate_flag=2, boundary_flag=(1, 1, 3, 3, 0, 0),
                                x_range=(1.0, 2.0), y_range=(0.0, math.pi), z_range=(0.0, 2 * math.pi)),
] + [lambda tm=tm: models.riemann_1d_test(tm, 32) for tm in range(1, 14)] \
  + [lambda tm=tm: models.riemann_2d(tm, 16) for tm in range(1, 20)] \
  + [lambda tm=tm: models.riemann_3d(tm, 8) for tm in (1, 2)]


@pytest.mark.parametrize("i", range(len(BUILDERS)))
def test_builder_spec_makes_a_config(i):
    spec, prim, eps = BUILDERS[i]()
    cfg, keep = capi.make_config(spec)
    assert (cfg.nx, cfg.ny, cfg.nz) == (spec["nx"], spec["ny"], spec["nz"])
    assert prim.shape == capi.padded_shape(spec) and eps.shape == prim.shape[:3]
    assert np.all(np.diff(spec["xF"]) > 0) and np.all(np.diff(spec["yF"]) > 0) and np.all(np.diff(spec["zF"]) > 0)
    assert cfg.model.gamma > 1.0


def test_a_mistyped_model_key_is_an_error():
    spec, _, _ = models.riemann_2d(18, 16)
    spec["model"]["g_cons"] = 0.2
    with pytest.raises(ValueError, match="g_cons"):
        capi.make_config(spec)
