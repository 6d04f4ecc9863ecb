"""RT Ion Plan and RT Plan readers (readPlanDicom) against the reference's
own readers (plan_impt.py:610-643, plan_imrt.py:273-351) on the same
synthetic datasets.  pydicom is not installed here, so both readers get a
stand-in module whose dcmread returns an attribute tree with the DICOM
keywords the readers use; the reference package is the one installed from
the reference sources into baseline/_ref (skipped when absent).  CPU only."""
import os
import sys
import types
from types import SimpleNamespace as NS

import numpy as np
import pytest

from conftest import ROOT

REF_PKG = os.path.join(ROOT, "baseline", "_ref")


def _fake_pydicom(datasets):
    mod = types.ModuleType("pydicom")
    mod.dcmread = lambda path, force=False: datasets[path]
    ds = types.ModuleType("pydicom.dataset")
    for name in ("Dataset", "FileDataset", "FileMetaDataset"):
        setattr(ds, name, type(name, (), {}))
    uid = types.ModuleType("pydicom.uid")
    uid.generate_uid = lambda *a, **k: "1.2.3"
    uid.ExplicitVRLittleEndian = uid.RTIonPlanStorage = "1.2.3"
    mod.dataset, mod.uid = ds, uid
    return mod


def _ion_plan(labels, rng):
    beams = []
    for b, (ga, ta, rs) in enumerate([(0.0, 0.0, None), (90.0, 15.0, "4"), (235.0, 330.0, None)]):
        cps = []
        for layer, e in enumerate(labels[b::3][:4]):
            n = int(rng.integers(3, 9))
            pos = rng.uniform(-40, 40, size=(n, 2)).round(1).ravel().tolist()
            w = rng.uniform(0.1, 2.0, size=n).round(3).tolist()
            cp = NS(NominalBeamEnergy=float(e), ScanSpotPositionMap=pos, ScanSpotMetersetWeights=w,
                    GantryAngle=ga, PatientSupportAngle=ta, IsocenterPosition=[1.5, -2.0, 3.25])
            cps.append(cp)
            # the second control point of each layer pair (ignored by both readers)
            cps.append(NS(NominalBeamEnergy=float(e), ScanSpotPositionMap=pos, ScanSpotMetersetWeights=[0.0] * n))
        ibs = NS(NumberOfRangeShifters=0 if rs is None else 1, IonControlPointSequence=cps,
                 RangeShifterSequence=[NS(RangeShifterID=rs)] if rs else [])
        beams.append(ibs)
    return NS(FractionGroupSequence=[NS(NumberOfFractionsPlanned=5)], IonBeamSequence=beams)


def _rt_plan(n_pairs, rng):
    def devices(with_mlc):
        seq = [NS(RTBeamLimitingDeviceType="X", LeafJawPositions=[-50.0, 60.0]),
               NS(RTBeamLimitingDeviceType="Y", LeafJawPositions=[-40.0, 45.0])]
        if with_mlc:
            x1 = rng.uniform(-50, 0, n_pairs).round(1)
            x2 = x1 + rng.uniform(0, 60, n_pairs).round(1)
            seq.append(NS(RTBeamLimitingDeviceType="MLCX", LeafJawPositions=np.concatenate((x1, x2)).tolist()))
        return seq

    beams = []
    for b, (with_mlc, delivery) in enumerate([(True, "TREATMENT"), (False, "TREATMENT"), (True, "SETUP")]):
        cps = [NS(ControlPointIndex=0, NominalBeamEnergy="6", IsocenterPosition=[0.5, 1.0, -2.0],
                  BeamLimitingDeviceAngle=10.0 * b, PatientSupportAngle=5.0, GantryAngle=180.0,
                  BeamLimitingDevicePositionSequence=devices(with_mlc), CumulativeMetersetWeight=0.0)]
        cum = 0.0
        for c in range(1, 5):
            cum += float(rng.uniform(0.1, 0.4))
            cp = NS(ControlPointIndex=c, CumulativeMetersetWeight=min(cum, 1.0))
            if c < 4:
                cp.GantryAngle = 180.0 + 20.0 * c
                cp.BeamLimitingDevicePositionSequence = devices(with_mlc)
            cps.append(cp)
        beams.append(NS(TreatmentDeliveryType=delivery, ControlPointSequence=cps))
    return NS(FractionGroupSequence=[NS(NumberOfFractionsPlanned=2,
                                        ReferencedBeamSequence=[NS(BeamMeterset=123.0)])],
              BeamSequence=beams)


@pytest.fixture
def reference_package(monkeypatch):
    if not os.path.isdir(os.path.join(REF_PKG, "DoseCUDA")):
        pytest.skip("reference package not installed in baseline/_ref")
    saved = {k: sys.modules.get(k) for k in ("pydicom", "pydicom.dataset", "pydicom.uid", "SimpleITK",
                                             "dose_kernels")}
    fake = _fake_pydicom({})
    sys.modules.update({"pydicom": fake, "pydicom.dataset": fake.dataset, "pydicom.uid": fake.uid,
                        "SimpleITK": types.ModuleType("SimpleITK")})
    sys.path.insert(0, REF_PKG)
    try:
        import DoseCUDA.plan_impt as ref_impt
        import DoseCUDA.plan_imrt as ref_imrt
        yield ref_impt, ref_imrt
    finally:
        sys.path.remove(REF_PKG)
        for k in [k for k in sys.modules if k == "DoseCUDA" or k.startswith("DoseCUDA.")]:
            del sys.modules[k]
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v


def test_ion_plan_reader_matches_reference(reference_package, monkeypatch):
    ref_impt, _ = reference_package
    from dosecuda_b200 import plan_impt
    mine = plan_impt.IMPTPlan()
    labels = mine.beam_models[0].energy_table["energy_label"].to_numpy()[10:40]
    ds = _ion_plan(labels, np.random.default_rng(1))
    fake = _fake_pydicom({"plan.dcm": ds})
    monkeypatch.setattr(plan_impt, "_pydicom", lambda: fake)
    monkeypatch.setattr(ref_impt, "pyd", fake)
    theirs = ref_impt.IMPTPlan()
    mine.readPlanDicom("plan.dcm")
    theirs.readPlanDicom("plan.dcm")
    assert mine.n_fractions == theirs.n_fractions == 5.0
    assert mine.n_beams == theirs.n_beams == 3
    for a, b in zip(mine.beam_list, theirs.beam_list):
        assert a.dicom_rangeshifter_label == b.dicom_rangeshifter_label
        assert a.gantry_angle == b.gantry_angle and a.couch_angle == b.couch_angle
        np.testing.assert_array_equal(a.iso, b.iso)
        assert a.n_spots == b.n_spots
        np.testing.assert_array_equal(np.asarray(a.spot_list, np.float32), np.asarray(b.spot_list, np.float32))


def test_rt_plan_reader_matches_reference(reference_package, monkeypatch):
    _, ref_imrt = reference_package
    from dosecuda_b200 import plan_imrt
    mine = plan_imrt.IMRTPlan("VarianTrueBeamHF")
    ds = _rt_plan(mine.beam_models[0].n_mlc_pairs, np.random.default_rng(2))
    fake = _fake_pydicom({"rtplan.dcm": ds})
    monkeypatch.setattr(plan_imrt, "_pydicom", lambda: fake)
    monkeypatch.setattr(ref_imrt, "pyd", fake)
    theirs = ref_imrt.IMRTPlan("VarianTrueBeamHF")
    mine.readPlanDicom("rtplan.dcm")
    theirs.readPlanDicom("rtplan.dcm")
    assert mine.n_fractions == theirs.n_fractions == 2.0
    assert mine.n_beams == theirs.n_beams == 2  # the SETUP beam is skipped
    for a, b in zip(mine.beam_list, theirs.beam_list):
        assert a.dicom_energy_label == b.dicom_energy_label
        np.testing.assert_array_equal(a.iso, b.iso)
        assert len(a.cp_list) == len(b.cp_list) == 4
        for ca, cb in zip(a.cp_list, b.cp_list):
            assert ca.mu == pytest.approx(cb.mu, rel=1e-12)
            assert (ca.ga, ca.ca, ca.ta) == (cb.ga, cb.ca, cb.ta)
            np.testing.assert_array_equal(np.asarray(ca.mlc), np.asarray(cb.mlc))
            # the raw buffer the reference's extension reads column by column
            assert np.asarray(ca.mlc).flags["F_CONTIGUOUS"] == np.asarray(cb.mlc).flags["F_CONTIGUOUS"]
