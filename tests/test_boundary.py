"""dose_kernels drop-in: argument checking follows the reference extension
(dosemodule.cu:23-66, 110, 249, 383) — checked without a GPU, since every
check fires before the library touches a device."""
import numpy as np
import pytest

from dosecuda_b200 import dose_kernels as dk
from dosecuda_b200 import phantoms
from dosecuda_b200.plan import VolumeObject


def _proton(shape=(4, 5, 6)):
    grid, plan = phantoms.proton_small(shape=shape, spacing=2.0)
    rl = phantoms.volume_object(grid, grid.RLSPFromHU(plan.machine_name))
    return plan.beam_models[0], rl, plan.beam_list[0]


def test_wrong_dtype_is_value_error_with_reference_message():
    model, rl, beam = _proton()
    rl.voxel_data = rl.voxel_data.astype(np.float64)
    with pytest.raises(ValueError, match=r"^'voxel_data' must be 3-dimensional and of type float\.$"):
        dk.proton_raytrace_cuda(model, rl, beam, 0)


def test_wrong_rank_is_value_error():
    model, rl, beam = _proton()
    rl.spacing = np.array([[2.0, 2.0, 2.0]], np.float32)
    with pytest.raises(ValueError, match=r"'spacing' must be 1-dimensional"):
        dk.proton_raytrace_cuda(model, rl, beam, 0)


def test_non_array_attribute_is_value_error():
    model, rl, beam = _proton()
    beam.iso = [0.0, 0.0, 0.0]
    with pytest.raises(ValueError, match=r"'iso' must be 1-dimensional"):
        dk.proton_raytrace_cuda(model, rl, beam, 0)


def test_missing_attribute_propagates_attribute_error():
    model, rl, beam = _proton()

    class M:
        VSADX = 1340.0

    with pytest.raises(AttributeError):
        dk.proton_raytrace_cuda(M(), rl, beam, 0)


def test_gpu_id_must_be_integer():
    model, rl, beam = _proton()
    with pytest.raises(TypeError):
        dk.proton_raytrace_cuda(model, rl, beam, 0.0)


def test_spot_list_single_row_vector_is_rejected_like_reference():
    model, rl, beam = _proton()
    beam.spot_list = np.array([0, 0, 1, 40], np.float32)  # 1-D, as the reference's addSingleSpot makes
    with pytest.raises(ValueError, match=r"'spot_list' must be 2-dimensional"):
        dk.proton_spot_cuda(model, rl, rl, beam, 0)


def test_spot_list_needs_four_columns():
    model, rl, beam = _proton()
    beam.spot_list = np.zeros((3, 3), np.float32)
    with pytest.raises(ValueError, match="4 columns"):
        dk.proton_spot_cuda(model, rl, rl, beam, 0)


def test_invalid_energy_id_is_value_error():
    model, rl, beam = _proton()
    beam.spot_list = np.array([[0, 0, 1, 200]], np.float32)
    with pytest.raises(ValueError, match="energy id"):
        dk.proton_spot_cuda(model, rl, rl, beam, 0)


def test_photon_checks(imrt_plan):
    grid, plan = phantoms.photon_small(shape=(4, 4, 4), spacing=2.5)
    model = plan.beam_models[0]
    cp = plan.beam_list[0].cp_list[0]
    vol = phantoms.volume_object(grid, grid.DensityFromHU(plan.machine_name))
    bad = VolumeObject()
    bad.voxel_data = vol.voxel_data[0]
    bad.spacing, bad.origin = vol.spacing, vol.origin
    with pytest.raises(ValueError, match="'voxel_data' must be 3-dimensional"):
        dk.photon_dose_cuda(model, bad, cp, 0)

    class CP:
        iso = cp.iso
        mlc = np.zeros((60, 3), np.float32)
        mu, ga, ca, ta = 100.0, 0.0, 0.0, 0.0

    with pytest.raises(ValueError, match="4 columns"):
        dk.photon_dose_cuda(model, vol, CP(), 0)


def test_photon_views_read_logical_columns(imrt_plan):
    """The kernel and MLC arrays are read by logical column whatever their
    memory order; for the reference's own (Fortran-ordered) arrays that is the
    same as its raw-buffer read."""
    model = imrt_plan.beam_models[0]
    assert model.kernel.flags["F_CONTIGUOUS"] and not model.kernel.flags["C_CONTIGUOUS"]
    v1 = dk.PhotonModelView(model)
    raw = np.frombuffer(model.kernel.tobytes(order="A"), np.float32)  # the reference's raw view
    for c, key in enumerate(("k0", "k1", "k2", "k3", "k4", "k5")):
        np.testing.assert_array_equal(v1._keep[key], raw[6 * c:6 * c + 6])
    plan = imrt_plan
    plan.addSquareField("6", 10, 10)
    cp = plan.beam_list[-1].cp_list[0]
    raw = np.frombuffer(cp.mlc.tobytes(order="A"), np.float32)
    n = cp.mlc.shape[0]
    cv = dk.ControlPointView(cp)
    for c in range(4):
        np.testing.assert_array_equal(cv._cols[c], raw[c * n:(c + 1) * n])
