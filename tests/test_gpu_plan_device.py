"""Device-resident plan loops: HU conversion on the GPU (fused into the ray
trace's texture), all beams / control points on the device, one copy back.

Each must reproduce the host path (np.interp conversion + one dose_kernels
call per beam or control point + numpy sums) bit for bit: the conversion
restates np.interp's arithmetic in explicitly rounded float64, and the sums
follow numpy's type promotion."""
import copy

import numpy as np
import pandas as pd
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_hu_conversion_equals_np_interp():
    from dosecuda_b200 import engine
    from dosecuda_b200.lookup import table_path
    rng = np.random.default_rng(0)
    for kind, name, col in (("protons", "HitachiProbeatJHU", "RLSP"), ("photons", "VarianTrueBeamHF", "Density")):
        df = pd.read_csv(table_path(kind, name, "HU_" + col + ".csv"))
        th, tv = df["HU"].to_numpy(), df[col].to_numpy()
        hu = rng.uniform(-1500.0, 4000.0, size=(6, 40, 50)).astype(np.float32)
        flat = hu.reshape(-1)
        flat[:len(th)] = th.astype(np.float32)          # on the breakpoints
        flat[len(th):2 * len(th)] = (th + 0.5).astype(np.float32)
        flat[-3:] = [-1e6, 1e6, float(th[-1])]          # beyond both ends, the last point
        ref = np.array(np.interp(hu, th, tv), dtype=np.single)
        got = engine.hu_convert(torch.as_tensor(hu).cuda(), (th, tv)).cpu().numpy()
        assert np.array_equal(got, ref), (kind, np.abs(got - ref).max())


def test_fused_hu_raytrace_equals_rlsp_raytrace():
    from dosecuda_b200 import engine, phantoms
    from dosecuda_b200.lookup import table_path
    grid, plan = phantoms.proton_small(shape=(48, 48, 48), spacing=3.0)
    model, beam = plan.beam_models[0], plan.beam_list[0]
    df = pd.read_csv(table_path("protons", plan.machine_name, "HU_RLSP.csv"))
    hu = torch.as_tensor(grid.HU).cuda()
    rlsp = torch.as_tensor(grid.RLSPFromHU(plan.machine_name)).cuda()
    a = engine.proton_wet_hu(hu, grid, beam, model, (df["HU"].to_numpy(), df["RLSP"].to_numpy()))
    b = engine.proton_wet(rlsp, grid, beam, model)
    assert torch.equal(a, b)


def test_impt_plan_on_device_equals_host_plan():
    from dosecuda_b200 import phantoms
    grid, plan = phantoms.proton_small(shape=(64, 64, 64), spacing=2.0)
    b2 = copy.deepcopy(plan.beam_list[0])
    b2.gantry_angle = 90.0
    plan.addBeam(b2)
    plan.n_fractions = 3
    grid.computeIMPTPlan(plan)
    host_dose, host_beams, host_rlsp = grid.dose.copy(), [b.copy() for b in grid.beam_doses], grid.RLSP.copy()
    grid.computeIMPTPlan(plan, device=True)
    assert np.array_equal(grid.RLSP, host_rlsp)
    assert len(grid.beam_doses) == 2
    for a, b in zip(grid.beam_doses, host_beams):
        assert np.array_equal(a, b)
    assert np.array_equal(grid.dose, host_dose)
    assert float(host_dose.max()) > 0


def test_imrt_plan_on_device_equals_host_plan():
    from dosecuda_b200 import phantoms
    from dosecuda_b200.plan_imrt import IMRTControlPoint
    grid, plan = phantoms.photon_small(shape=(64, 64, 64), spacing=2.5, field_cm=(8.0, 6.0), gantry=20.0)
    beam = plan.beam_list[0]
    cp0 = beam.cp_list[0]
    mlc = np.array(cp0.mlc, copy=True)
    mlc[:, 0] *= 0.5
    mlc[:, 1] *= 0.3
    beam.cp_list.append(IMRTControlPoint(cp0.iso, 60.0, mlc, 200.0, 10.0, 0.0, None, None))
    plan.addSquareField("6", 4.0, 5.0, mu=80.0, gantry_angle=90.0)
    plan.n_fractions = 2
    grid.computeIMRTPlan(plan)
    host_dose, host_beams, host_density = grid.dose.copy(), [b.copy() for b in grid.beam_doses], grid.Density.copy()
    grid.computeIMRTPlan(plan, device=True)
    assert np.array_equal(grid.Density, host_density)
    assert len(grid.beam_doses) == 2
    for a, b in zip(grid.beam_doses, host_beams):
        assert np.array_equal(a, b)
    assert np.array_equal(grid.dose, host_dose)
    assert float(host_dose.max()) > 0
