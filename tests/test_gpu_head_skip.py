"""The head transmission (headTransmission, IMRTClasses.cu:120-150) sums one
erf product per leaf pair.  The engine skips the pairs whose two y-edge erf
arguments lie beyond a bound on the same side: each of them contributes
0.5 * (erf(a2) - erf(a1)) = 0 exactly when the device's erff is exactly +-1
beyond that bound, and the sum of the remaining pairs is then bitwise the
sum over every pair.  This checks the bound against the compiled erff over
every float in [3, 4.5]."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def test_erf_saturated_beyond_skip_bound():
    from dosecuda_b200 import _lib

    lib = _lib.load()
    largest, bound = C.c_float(-1.0), C.c_float(-1.0)
    _lib.raise_for(lib.dc_photon_head_selftest(0, C.byref(largest), C.byref(bound)))
    # erff is not yet saturated at 3 (erfc(3) = 2.2e-5), so some float of the
    # scan is unsaturated; every argument past the bound must be
    assert 3.0 <= largest.value <= bound.value <= 4.5, (largest.value, bound.value)


def test_selftest_rejects_null_outputs():
    from dosecuda_b200 import _lib

    lib = _lib.load()
    v = C.c_float()
    assert lib.dc_photon_head_selftest(0, None, C.byref(v)) != 0
