"""The division-free nearest-voxel index of the WET smoothing
(``nearest_index`` in dosecuda_b200/csrc/dc_wet.cu), restated in float32
NumPy (IEEE round-to-nearest, no fused operations, as the kernel's explicit
``__fmul_rn``/``__fadd_rn``), against the reference's own expression
``(int)roundf(v / s)`` (CudaClasses.cuh:112-116) on random coordinates and on
coordinates at and next to every half-integer multiple of the spacing: the
fast path either declines (the kernel then evaluates the reference's
expression) or returns exactly the reference's index."""
import numpy as np
import pytest

F = np.float32
MAGIC = F(12582912.0)  # 1.5 * 2^23


def fast_path(v, s):
    r = F(1.0) / s
    qa = (v * r).astype(F)
    t = (qa + MAGIC).astype(F)
    d = np.abs((qa - (t - MAGIC).astype(F)).astype(F))
    aq = np.abs(qa)
    ok = (aq < F(2097152.0)) & ((F(0.5) - d).astype(F) > (aq * F(4.76837158203125e-07)).astype(F))
    return ok, t.view(np.int32).astype(np.int64) - 0x4B400000


def reference(v, s):
    q = (v / s).astype(F)  # IEEE float32 quotient
    return (np.sign(q) * np.floor(np.abs(q).astype(np.float64) + 0.5)).astype(np.int64)  # roundf: half away


@pytest.mark.parametrize("s", [1.0, 1.5, 2.0, 2.5, 3.0, 1.2, 0.977, 3.3, 1.9531])
def test_fast_nearest_index_is_the_reference_index(s):
    s = F(s)
    rng = np.random.default_rng(int(s * 1000))
    v = (rng.standard_normal(400_000) * 300.0).astype(F)
    k = rng.integers(-600, 600, 100_000).astype(F) + F(0.5)
    half = (k * s).astype(F)
    v = np.concatenate([v, half, np.nextafter(half, F(np.inf)), np.nextafter(half, F(-np.inf)),
                        (rng.integers(-600, 600, 50_000) * s).astype(F)])
    ok, n = fast_path(v, s)
    ref = reference(v, s)
    assert not np.any(ok & (n != ref))
    rand_ok = ok[:400_000].mean()
    assert rand_ok > 0.999  # the division is needed only next to half-integers
