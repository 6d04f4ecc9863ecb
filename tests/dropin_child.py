"""Child process of tests/test_gpu_dropin_reference_package.py (test
infrastructure).  Runs the reference's own plan package (DoseCUDA, installed
from the reference sources into baseline/_ref) through its public plan API:
IMPTDoseGrid.computeIMPTPlan (plan_impt.py:124-160) and
IMRTDoseGrid.computeIMRTPlan (plan_imrt.py:126-158).

    python tests/dropin_child.py engine|reference INPUTS.npz OUT.npz

``engine``: before the package is imported, ``sys.modules["dose_kernels"]``
is set to ``dosecuda_b200.dose_kernels``, so the reference's unmodified
``import dose_kernels`` (plan_impt.py:12, plan_imrt.py:9) binds this
engine.  ``reference``: the package's own compiled ``dose_kernels``.
pydicom and SimpleITK, imported at the top of the reference's modules but not
used on the dose path, are replaced by empty stand-in modules.
"""
import os
import sys
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _stub_modules():
    pyd = types.ModuleType("pydicom")
    ds = types.ModuleType("pydicom.dataset")
    uid = types.ModuleType("pydicom.uid")
    for name in ("Dataset", "FileDataset", "FileMetaDataset"):
        setattr(ds, name, type(name, (), {}))
    uid.generate_uid = lambda *a, **k: "1.2.3"
    uid.ExplicitVRLittleEndian = uid.RTIonPlanStorage = "1.2.3"
    pyd.dataset, pyd.uid = ds, uid
    sys.modules.update({"pydicom": pyd, "pydicom.dataset": ds, "pydicom.uid": uid,
                        "SimpleITK": types.ModuleType("SimpleITK")})


def main():
    mode, inp, out = sys.argv[1:4]
    _stub_modules()
    if mode == "engine":
        sys.path.insert(0, ROOT)
        from dosecuda_b200 import dose_kernels
        sys.modules["dose_kernels"] = dose_kernels
    sys.path.insert(0, os.path.join(ROOT, "baseline", "_ref"))
    import DoseCUDA as D
    import dose_kernels as bound
    z = np.load(inp)
    res = {"bound_file": np.array(str(getattr(bound, "__file__", "")))}

    g = D.IMPTDoseGrid()
    g.HU = z["p_hu"]
    g.origin, g.spacing, g.size = z["p_origin"], z["p_spacing"], np.array(z["p_hu"].shape)
    plan = D.IMPTPlan()
    beam = D.IMPTBeam()
    beam.spot_list = z["p_spots"]
    beam.n_spots = beam.spot_list.shape[0]
    beam.gantry_angle, beam.couch_angle = float(z["p_angles"][0]), float(z["p_angles"][1])
    beam.iso = z["p_iso"]
    beam.dicom_rangeshifter_label = "0"
    plan.addBeam(beam)
    plan.n_fractions = 2
    g.computeIMPTPlan(plan, gpu_id=0)
    res["proton"] = g.dose

    x = D.IMRTDoseGrid()
    x.HU = z["x_hu"]
    x.origin, x.spacing, x.size = z["x_origin"], z["x_spacing"], np.array(z["x_hu"].shape)
    xp = D.IMRTPlan("VarianTrueBeamHF")
    # every leaf pair open over the phantom, where the reference's TERMA is
    # sound on every voxel (test_gpu_reference_terma.py)
    xp.addSquareField("6", 40, 40, mu=100)
    xp.addSquareField("6", 40, 40, mu=50, gantry_angle=90.0)
    x.computeIMRTPlan(xp, gpu_id=0)
    res["photon"] = x.dose
    res["photon_beams"] = np.stack(x.beam_doses)
    np.savez(out, **res)


if __name__ == "__main__":
    main()
