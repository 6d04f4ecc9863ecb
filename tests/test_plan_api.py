"""Plan API mirror: beam-model loading from the unchanged lookup tables, the
array layouts the engine boundary relies on, and the host-side helpers
(reference plan.py, plan_impt.py, plan_imrt.py)."""
import numpy as np
import pytest

import dosecuda_b200 as D
from dosecuda_b200.plan_imrt import IMRTControlPoint, _mlc_array


def test_public_names_match_reference_package():
    for n in ("IMPTDoseGrid", "IMPTPlan", "IMPTBeam", "IMRTDoseGrid", "IMRTPlan", "IMRTBeam", "IMRTControlPoint",
              "IMRTPhotonEnergy"):
        assert hasattr(D, n)


def test_proton_model_tables(impt_plan):
    assert list(impt_plan.dicom_rangeshifter_label.astype(str)) == ["0", "4"]
    m = impt_plan.beam_models[0]
    assert (m.VSADX, m.VSADY) == (1340.0, 1930.0)
    assert m.divergence_params.shape == (98, 5) and m.divergence_params.dtype == np.float32
    assert m.lut_depths.shape == (98, 400) and m.lut_idds.dtype == np.float32
    np.testing.assert_array_equal(m.divergence_params[34],
                                  np.array([101.3, 78.32, 1.377e-06, 6.485e-04, -1.140e-01], np.float32))
    np.testing.assert_array_equal(m.lut_depths[0, :3], np.array([0.0, 1.0, 2.0], np.float32))
    assert m.lut_depths[0, -1] == 399.0  # 400 rows, depth 400 mm dropped
    assert m.energyIDFromLabel(101.3) == 34
    with pytest.raises(Exception):
        m.energyIDFromLabel(1.0)


def test_photon_model_layouts(imrt_plan):
    m = imrt_plan.beam_models[0]
    m.validate_parameters()
    assert m.kernel.shape == (6, 6) and m.kernel.flags["F_CONTIGUOUS"]
    np.testing.assert_array_equal(m.kernel[:, 0], np.array([1.875, 20.625, 43.125, 61.875, 88.125, 106.875],
                                                           np.float32))
    assert m.n_mlc_pairs == 60
    assert m.primary_source_distance == 1000.0 and m.scatter_source_distance == 850.0
    assert m.mlc_distance == 491.0 and m.has_xjaws is True
    assert m.profile_radius.shape == (20,) and m.spectrum_attenuation_coefficients.shape == (12,)
    assert m.mu_calibration == pytest.approx(4.143232e-3)


def test_square_field_mlc_and_output_factor():
    plan = D.IMRTPlan()
    plan.addSquareField("6", 10, 10, mu=100)
    cp = plan.beam_list[0].cp_list[0]
    assert cp.mlc.shape == (60, 4) and cp.mlc.strides == (4, 240)  # transposed (4, 60) C array
    open_ = cp.mlc[:, 1] > cp.mlc[:, 0]
    assert open_.sum() == 20 and np.all(cp.mlc[open_, 0] == -50.0) and np.all(cp.mlc[open_, 1] == 50.0)
    # 10x10 cm: equivalent square 100 mm -> tabulated output factor
    assert plan.beam_models[0].outputFactor(cp) == pytest.approx(0.979229534, rel=1e-6)


def test_mlc_array_layout():
    x12 = np.array([[-1, -2], [1, 2]], np.float32)
    m = _mlc_array(x12, np.array([0.0, 5.0]), np.array([5.0, 5.0]))
    np.testing.assert_array_equal(m, [[-1, 1, 0, 5], [-2, 2, 5, 5]])
    cp = IMRTControlPoint(np.zeros(3, np.float32), 1.0, m, 0.0, 0.0, 0.0, None, None)
    assert cp.mlc is m


def test_hu_conversions():
    g = D.IMPTDoseGrid()
    g.HU = np.array([[[-1000.0, 0.0, 1369.0, 5000.0]]], np.float32)
    r = g.RLSPFromHU("HitachiProbeatJHU")
    np.testing.assert_allclose(r, [[[0.00113, 1.00653, 1.74967, 2.36825]]], rtol=1e-6)
    assert r.dtype == np.float32
    g2 = D.IMRTDoseGrid()
    g2.HU = g.HU
    np.testing.assert_allclose(g2.DensityFromHU("VarianTrueBeamHF"), r, rtol=1e-6)


def test_cube_phantom_and_couch():
    g = D.IMPTDoseGrid()
    g.createCubePhantom(size=[20, 20, 20], spacing=3.0)
    assert g.HU.shape == (20, 20, 20)
    assert g.HU[0, 0, 0] == -1000.0 and g.HU[10, 10, 10] == 0.0
    edge = round(10.0 / 3.0)
    assert g.HU[edge, edge, edge] == 0.0 and g.HU[edge - 1, 10, 10] == -1000.0
    g.applyCouchModel(couch_wet=8.0)
    n = int(50.0 / 3.0)
    np.testing.assert_allclose(g.HU[:, -n:, :], ((8.0 / (n * 3.0)) - 1.0) * 1000.0)


def test_single_spot_beam_is_two_dimensional():
    b = D.IMPTBeam()
    b.addSingleSpot(1.0, 2.0, 0.5, 40)
    assert b.spot_list.shape == (1, 4)
    b.addSingleSpot(3.0, 4.0, 0.5, 41)
    assert b.spot_list.shape == (2, 4) and b.n_spots == 2
    b.changeSpotEnergy(10)
    assert np.all(b.spot_list[:, 3] == 10)
    b.resetSpots()
    assert b.spot_list.shape == (0, 4) and b.n_spots == 0


def test_unknown_beam_model_is_value_error():
    g = D.IMPTDoseGrid()
    g.createCubePhantom(size=[8, 8, 8], spacing=3.0)
    plan = D.IMPTPlan()
    b = D.IMPTBeam()
    b.dicom_rangeshifter_label = "7"
    b.addSingleSpot(0, 0, 1, 10)
    plan.addBeam(b)
    with pytest.raises(ValueError, match="rangeshifter"):
        g.computeIMPTPlan(plan)


def test_anisotropic_grid_rejected_like_reference():
    g = D.IMPTDoseGrid()
    g.createCubePhantom(size=[8, 8, 8], spacing=3.0)
    g.spacing = np.array([3.0, 3.0, 2.0])
    with pytest.raises(Exception, match="isotropic"):
        g.computeIMPTPlan(D.IMPTPlan())


def test_io_methods_need_simpleitk():
    g = D.IMPTDoseGrid()
    try:
        import SimpleITK  # noqa: F401
        pytest.skip("SimpleITK present")
    except ImportError:
        pass
    with pytest.raises(ImportError, match="SimpleITK"):
        g.loadCTNRRD("x.nrrd")
