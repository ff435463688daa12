"""z-slab cuts (CPU): the per-slab specs the group is built from."""
import numpy as np
import pytest

from cumc3d_b200 import capi, engine, models


def test_slab_specs_of_a_periodic_and_an_outflow_grid():
    spec, _, _ = models.blast_3d(12, nz=20)
    specs, offs = engine.slab_specs(spec, (7, 6, 7))
    assert offs == [0, 7, 13]
    zF = np.asarray(spec["zF"])
    for sp, o, m in zip(specs, offs, (7, 6, 7)):
        assert sp["nz"] == m and np.array_equal(sp["zF"], zF[o:o + m + 7])
        assert sp["zF"][3] == zF[o + 3] and sp["zF"][m + 3] == zF[o + m + 3]   # faces 0 and m
        assert sp["boundary_flag"][4:] == [capi.BOUNDARY_EXCHANGE] * 2          # periodic: a ring
        assert sp["boundary_flag"][:4] == spec["boundary_flag"][:4]
    spec, _, _ = models.smooth_state(8, 8, 12, 3, boundary_flag=(0, 0, 1, 1, 1, 2))
    specs, _ = engine.slab_specs(spec, (6, 6))
    assert specs[0]["boundary_flag"][4:] == [1, capi.BOUNDARY_EXCHANGE]
    assert specs[1]["boundary_flag"][4:] == [capi.BOUNDARY_EXCHANGE, 2]
    with pytest.raises(ValueError):
        engine.slab_specs(spec, (10, 2))
    with pytest.raises(ValueError):
        engine.slab_specs(spec, (6, 5))
