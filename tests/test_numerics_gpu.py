"""Device numerics the bitwise claims of the FP64 form rest on."""
import pytest

from cumc3d_b200 import engine

pytestmark = pytest.mark.gpu


def test_fma_corrected_div3_equals_ieee_division():
    """WENO-Z's /3 (weno_module.f90:363-365, 386-388) is evaluated as
    q = x*RN(1/3) plus one FMA correction; it must equal x/3.0 bit for bit."""
    total = 0
    for seed in (1, 2, 3, 4):
        bad, ex = engine.check_div3(seed * 0x1234567, 1 << 30)
        assert bad == 0, "div3 differs from x/3 for x=%r" % ex
        total += 1 << 30
    assert total == 1 << 32



def test_zero_numerator_division_equals_ieee_division():
    """The FP64 division of the flux and update kernels (a zero numerator
    returns the signed zero without the division's slow path) against x / y:
    2^28 pairs, a quarter of the numerators +-0, the denominators over every
    exponent with zeros, infinities, NaNs and subnormals among them."""
    for seed in (11, 12):
        bad, ex = engine.check_dv(seed * 0x9E3779B9, 1 << 27)
        assert bad == 0, "dv differs from x / y for (x, y) = %r" % (ex,)
