"""The drop-in claim on the reference's own package: its unmodified plan
modules (installed from the reference sources into baseline/_ref) compute the
config-1 proton plan and a two-beam photon plan (40 x 40 cm fields over the
128^3 photon phantom, where the reference's TERMA is sound everywhere) through
their public API,
once with their own compiled ``dose_kernels`` and once with
``sys.modules["dose_kernels"] = dosecuda_b200.dose_kernels`` set before the
package is imported.  The doses must agree within the parity bar.  Each run is
a child process (tests/dropin_child.py) so that the two bindings never meet
in one interpreter."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT
from dosecheck import dose_diff, gamma_pass_rate

pytestmark = pytest.mark.gpu

REF_PKG = os.path.join(ROOT, "baseline", "_ref", "DoseCUDA")


def _run(mode, inp, out):
    env = dict(os.environ)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "dropin_child.py"), mode, inp, out],
                       env=env, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out)


def test_reference_package_binds_engine_and_matches(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.isdir(REF_PKG):
        pytest.skip("reference package not installed in baseline/_ref")
    from dosecuda_b200 import phantoms
    pg = phantoms.proton_phantom()
    pb = phantoms.proton_beam()
    xg = phantoms.photon_phantom()
    inp = str(tmp_path / "inputs.npz")
    np.savez(inp, p_hu=pg.HU, p_origin=np.asarray(pg.origin, np.float64), p_spacing=np.asarray(pg.spacing, np.float64),
             p_spots=pb.spot_list, p_angles=np.array([pb.gantry_angle, pb.couch_angle]), p_iso=pb.iso,
             x_hu=xg.HU, x_origin=np.asarray(xg.origin, np.float64), x_spacing=np.asarray(xg.spacing, np.float64))
    eng = _run("engine", inp, str(tmp_path / "engine.npz"))
    ref = _run("reference", inp, str(tmp_path / "reference.npz"))
    # which extension each run bound
    assert str(eng["bound_file"]).replace(os.sep, "/").endswith("dosecuda_b200/dose_kernels.py")
    assert "baseline/_ref/DoseCUDA/dose_kernels" in str(ref["bound_file"]).replace(os.sep, "/")
    dp = dose_diff(eng["proton"], ref["proton"])
    dx = dose_diff(eng["photon"], ref["photon"])
    gx = gamma_pass_rate(eng["photon"], ref["photon"], float(xg.spacing[0]))
    print("\n" + json.dumps({"proton_dD": dp, "photon_dD": dx, "photon_gamma": gx}))
    assert ref["proton"].max() > 0 and ref["photon"].max() > 0
    assert dp <= 1e-3
    assert gamma_pass_rate(eng["proton"], ref["proton"], float(pg.spacing[0])) >= 0.995
    assert dx <= 0.005
    assert gx >= 0.995
    for b in range(ref["photon_beams"].shape[0]):
        assert dose_diff(eng["photon_beams"][b], ref["photon_beams"][b]) <= 0.005
