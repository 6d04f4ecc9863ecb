"""GPU parity of the sm_100a engines (through the C ABI) against
  * the golden fixtures produced by the reference's own CUDA build,
  * the reference build itself at the full small-workload sizes
    (oracle/_ref, when present), and
  * the FP64 CPU oracle.
Criteria: |dD| <= 0.5 % of Dmax in every voxel above 10 % Dmax and
gamma(2 %/2 mm) >= 99.5 %; the engine is held to tighter bounds where the
fixtures allow (noted per test)."""
import glob
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, golden_names, load_golden, proton_model
from dosecheck import dose_diff, gamma_pass_rate

pytestmark = pytest.mark.gpu

TOL = 0.005      # 0.5 % of Dmax above 10 % Dmax
GAMMA = 0.995


@pytest.fixture(scope="module")
def dk():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dosecuda_b200 import dose_kernels
    return dose_kernels


@pytest.fixture(scope="module")
def ref_dk():
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if not glob.glob(os.path.join(ref_dir, "dose_kernels*.so")):
        pytest.skip("reference build oracle/_ref not present")
    sys.path.insert(0, ref_dir)
    import dose_kernels as ref
    sys.path.remove(ref_dir)
    return ref


def _vol(data, spacing, origin):
    from dosecuda_b200.plan import VolumeObject
    v = VolumeObject()
    v.voxel_data = np.ascontiguousarray(data, dtype=np.float32)
    v.spacing = np.asarray(spacing, np.float32)
    v.origin = np.asarray(origin, np.float32)
    return v


class _Beam:
    def __init__(self, iso, gantry, couch, spots=None):
        self.iso = np.asarray(iso, np.float32)
        self.gantry_angle = gantry
        self.couch_angle = couch
        self.spot_list = spots


# ---------------------------------------------------------------- proton
@pytest.mark.parametrize("name", golden_names("proton"))
def test_proton_wet_matches_reference_golden(dk, impt_plan, name):
    meta, g = load_golden(name)
    model = proton_model(impt_plan, meta["rangeshifter"])
    wet = dk.proton_raytrace_cuda(model, _vol(g["rlsp"], g["spacing"], g["origin"]),
                                  _Beam(g["iso"], meta["gantry"], meta["couch"]), 0)
    # same sample positions and the same texture hardware: agreement to float rounding
    assert np.abs(wet - g["wet"]).max() <= 1e-4


@pytest.mark.parametrize("name", golden_names("proton"))
def test_proton_dose_matches_reference_golden(dk, impt_plan, name):
    meta, g = load_golden(name)
    model = proton_model(impt_plan, meta["rangeshifter"])
    v = _vol(g["rlsp"], g["spacing"], g["origin"])
    dose = dk.proton_spot_cuda(model, v, _vol(g["wet"], g["spacing"], g["origin"]),
                               _Beam(g["iso"], meta["gantry"], meta["couch"], g["spots"]), 0)
    assert dose_diff(dose, g["dose"]) <= 1e-3  # 0.1 % of Dmax
    assert gamma_pass_rate(dose, g["dose"], g["spacing"][0]) >= GAMMA


# ---------------------------------------------------------------- photon
class _CP:
    def __init__(self, g, meta):
        self.iso = g["iso"]
        self.mlc = g["mlc"]
        self.mu = meta["mu"]
        self.ga = meta["gantry"]
        self.ca = meta["collimator"]
        self.ta = meta["couch"]


def _clean_photon():
    return [n for n in golden_names("photon") if not n.endswith("_closed")]


@pytest.mark.parametrize("name", _clean_photon())
def test_photon_dose_matches_reference_golden(dk, imrt_plan, name):
    meta, g = load_golden(name)
    model = imrt_plan.beam_models[0]
    dose = dk.photon_dose_cuda(model, _vol(g["density"], g["spacing"], g["origin"]), _CP(g, meta), 0)
    assert dose_diff(dose, g["dose"]) <= TOL
    assert gamma_pass_rate(dose, g["dose"], g["spacing"][0]) >= GAMMA


def test_photon_closed_leaf_case_matches_oracle(dk, imrt_plan):
    """Closed leaf pairs over the phantom: the reference output carries its
    TERMA transmission-ratio artifact here; the engine must match the FP64
    restatement of the reference algorithm instead."""
    import oracle
    meta, g = load_golden("x_g0_closed")
    model = imrt_plan.beam_models[0]
    cp = _CP(g, meta)
    dose = dk.photon_dose_cuda(model, _vol(g["density"], g["spacing"], g["origin"]), cp, 0)
    o, _ = oracle.photon_dose(g["density"], g["spacing"][[0, 0, 0]], g["origin"], model, cp.iso, cp.mu, cp.ga, cp.ca,
                              cp.ta, cp.mlc)
    assert dose_diff(dose, o) <= TOL
    assert gamma_pass_rate(dose, o, g["spacing"][0]) >= GAMMA
    assert g["dose"].max() > 100 * o.max()  # the reference's artifact is present in the fixture


# ---------------------------------------------------------------- full-size workloads vs the reference build
def test_proton_small_workload_vs_reference_build(dk, ref_dk):
    from dosecuda_b200 import phantoms
    grid, plan = phantoms.proton_small()
    model, beam = plan.beam_models[0], plan.beam_list[0]
    rl = phantoms.volume_object(grid, grid.RLSPFromHU(plan.machine_name))
    w_ref = ref_dk.proton_raytrace_cuda(model, rl, beam, 0)
    w = dk.proton_raytrace_cuda(model, rl, beam, 0)
    assert np.abs(w - w_ref).max() <= 1e-4
    d_ref = ref_dk.proton_spot_cuda(model, rl, phantoms.volume_object(grid, w_ref), beam, 0)
    d = dk.proton_spot_cuda(model, rl, phantoms.volume_object(grid, w), beam, 0)
    assert dose_diff(d, d_ref) <= 1e-3
    assert gamma_pass_rate(d, d_ref, 2.0) >= GAMMA


def test_proton_small_workload_vs_oracle(dk):
    import oracle
    from dosecuda_b200 import phantoms
    grid, plan = phantoms.proton_small()
    model, beam = plan.beam_models[0], plan.beam_list[0]
    rl = phantoms.volume_object(grid, grid.RLSPFromHU(plan.machine_name))
    w = dk.proton_raytrace_cuda(model, rl, beam, 0)
    d = dk.proton_spot_cuda(model, rl, phantoms.volume_object(grid, w), beam, 0)
    sp = np.asarray(rl.spacing)[[0, 0, 0]]
    d_o, _ = oracle.proton_dose(w, sp, rl.origin, beam.iso, beam.gantry_angle, beam.couch_angle, model,
                                beam.spot_list)
    # float against FP64 on every voxel: the axis distance is computed without
    # the reference's cancellation (|ray x t|^2 / |t|^2)
    print("\nproton 96^3 vs FP64 oracle: %.2e of Dmax above 10 %%, %.2e on every voxel"
          % (dose_diff(d, d_o), dose_diff(d, d_o, thresh=0.0)))
    assert dose_diff(d, d_o) <= 1e-4
    assert dose_diff(d, d_o, thresh=0.0) <= 1e-4


def test_photon_small_workload_vs_oracle_and_reference(dk, imrt_plan):
    """128^3 CCCS: engine vs the FP64 oracle everywhere; vs the reference build
    on every voxel the reference's TERMA artifact does not reach."""
    import oracle
    from dosecuda_b200 import phantoms
    grid, plan = phantoms.photon_small()
    model, cp = plan.beam_models[0], plan.beam_list[0].cp_list[0]
    vol = phantoms.volume_object(grid, grid.DensityFromHU(plan.machine_name))
    d = dk.photon_dose_cuda(model, vol, cp, 0)
    o, _ = oracle.photon_dose(vol.voxel_data, np.asarray(vol.spacing)[[0, 0, 0]], vol.origin, model, cp.iso, cp.mu,
                              cp.ga, cp.ca, cp.ta, np.ascontiguousarray(cp.mlc))
    assert dose_diff(d, o) <= TOL
    assert gamma_pass_rate(d, o, 2.5) >= GAMMA
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if glob.glob(os.path.join(ref_dir, "dose_kernels*.so")):
        sys.path.insert(0, ref_dir)
        import dose_kernels as ref
        sys.path.remove(ref_dir)
        r = ref.photon_dose_cuda(model, vol, cp, 0)
        dmax = o.max()
        clean = np.abs(r - o) <= TOL * dmax  # voxels the artifact did not reach
        assert clean.mean() > 0.5
        assert np.abs(d - r)[clean & (o > 0.1 * dmax)].max() <= TOL * dmax


# ---------------------------------------------------------------- engine properties
def test_deterministic_bitwise(dk):
    from dosecuda_b200 import phantoms
    grid, plan = phantoms.proton_small(shape=(40, 40, 40), spacing=3.0, energy_ids=(5, 15, 25), field_mm=30.0)
    model, beam = plan.beam_models[0], plan.beam_list[0]
    rl = phantoms.volume_object(grid, grid.RLSPFromHU(plan.machine_name))
    w1 = dk.proton_raytrace_cuda(model, rl, beam, 0)
    w2 = dk.proton_raytrace_cuda(model, rl, beam, 0)
    d1 = dk.proton_spot_cuda(model, rl, phantoms.volume_object(grid, w1), beam, 0)
    d2 = dk.proton_spot_cuda(model, rl, phantoms.volume_object(grid, w1), beam, 0)
    assert np.array_equal(w1, w2) and np.array_equal(d1, d2)
    # spot order does not change the result beyond summation rounding (layers are sorted)
    beam.spot_list = beam.spot_list[::-1].copy()
    d3 = dk.proton_spot_cuda(model, rl, phantoms.volume_object(grid, w1), beam, 0)
    assert dose_diff(d3, d1) <= 1e-5


def test_device_api_matches_host_api(dk, imrt_plan):
    import torch
    from dosecuda_b200 import engine, phantoms
    grid, plan = phantoms.proton_small(shape=(32, 36, 40), spacing=3.0, energy_ids=(5, 15), field_mm=30.0)
    model, beam = plan.beam_models[0], plan.beam_list[0]
    rlsp = grid.RLSPFromHU(plan.machine_name)
    rl = phantoms.volume_object(grid, rlsp)
    w_h = dk.proton_raytrace_cuda(model, rl, beam, 0)
    d_h = dk.proton_spot_cuda(model, rl, phantoms.volume_object(grid, w_h), beam, 0)
    t = torch.from_numpy(rlsp).cuda()
    w_d = engine.proton_wet(t, grid, beam, model)
    d_d = engine.proton_dose(w_d, grid, beam, engine.ProtonModelDevice(model))
    torch.cuda.synchronize()
    assert np.array_equal(w_d.cpu().numpy(), w_h) and np.array_equal(d_d.cpu().numpy(), d_h)
    g2, p2 = phantoms.photon_small(shape=(32, 36, 40), spacing=3.0, field_cm=(6.0, 14.0))
    m2, cp2 = p2.beam_models[0], p2.beam_list[0].cp_list[0]
    dens = g2.DensityFromHU(p2.machine_name)
    x_h = dk.photon_dose_cuda(m2, phantoms.volume_object(g2, dens), cp2, 0)
    x_d = engine.photon_dose(torch.from_numpy(dens).cuda(), g2, m2, cp2)
    torch.cuda.synchronize()
    assert np.array_equal(x_d.cpu().numpy(), x_h)


def test_calls_on_two_streams_are_ordered(dk):
    """Device calls share the per-device scratch buffers; calls enqueued on
    different streams must still each see their own inputs."""
    import torch
    from dosecuda_b200 import engine, phantoms
    grid, plan = phantoms.proton_small(shape=(32, 32, 32), spacing=3.0, energy_ids=(5,), field_mm=20.0)
    model = plan.beam_models[0]
    b1 = plan.beam_list[0]
    from dosecuda_b200.plan_impt import IMPTBeam
    b2 = IMPTBeam(b1)
    b2.gantry_angle = 90.0
    rl = torch.from_numpy(grid.RLSPFromHU(plan.machine_name)).cuda()
    ref1 = engine.proton_wet(rl, grid, b1, model).cpu()
    ref2 = engine.proton_wet(rl, grid, b2, model).cpu()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    outs = []
    for _ in range(4):
        with torch.cuda.stream(s1):
            o1 = engine.proton_wet(rl, grid, b1, model)
        with torch.cuda.stream(s2):
            o2 = engine.proton_wet(rl, grid, b2, model)
        outs.append((o1, o2))
    torch.cuda.synchronize()
    for o1, o2 in outs:
        assert torch.equal(o1.cpu(), ref1) and torch.equal(o2.cpu(), ref2)


def test_invalid_device_is_runtime_error(dk):
    import torch
    from dosecuda_b200 import phantoms
    grid, plan = phantoms.proton_small(shape=(8, 8, 8))
    rl = phantoms.volume_object(grid, grid.RLSPFromHU(plan.machine_name))
    with pytest.raises(RuntimeError, match="^CUDA error: "):
        dk.proton_raytrace_cuda(plan.beam_models[0], rl, plan.beam_list[0], torch.cuda.device_count() + 3)


def test_plan_api_end_to_end(dk):
    """computeIMPTPlan / computeIMRTPlan through the mirrored plan classes."""
    import dosecuda_b200 as D
    g = D.IMPTDoseGrid()
    g.createCubePhantom(size=[40, 40, 40], spacing=3.0)
    plan = D.IMPTPlan()
    b = D.IMPTBeam()
    b.dicom_rangeshifter_label = "0"
    for e in range(10, 30, 4):
        for x in (-10.0, 0.0, 10.0):
            b.addSingleSpot(x, 0.0, 0.5, e)
    plan.addBeam(b)
    plan.n_fractions = 2
    g.computeIMPTPlan(plan)
    assert g.dose.shape == (40, 40, 40) and g.dose.max() > 0
    np.testing.assert_allclose(g.beam_doses[0], g.dose, rtol=1e-6)
    x = D.IMRTDoseGrid()
    x.createCubePhantom(size=[32, 32, 32], spacing=4.0)
    xp = D.IMRTPlan()
    xp.addSquareField("6", 8, 8, mu=100)
    xp.addSquareField("6", 6, 6, mu=50, gantry_angle=90.0, collimator_angle=20.0)
    x.computeIMRTPlan(xp)
    assert x.dose.max() > 0 and len(x.beam_doses) == 2


@pytest.mark.parametrize("machine,label", [("ElektaVersaSibAxesse", "6"), ("VarianTrueBeamHF", "10")])
def test_photon_other_machines_and_energies_vs_oracle(dk, machine, label):
    """The other photon beam models the reference ships through the same
    kernels: the Elekta machine (80-pair MLC of 5 mm leaves; its four energy
    folders hold identical tables in the reference, so one stands for all)
    and the Varian 10 MV spectrum and kernel.  Engine vs the FP64 oracle on a
    64^3 phantom, oblique gantry and collimator."""
    import oracle
    from dosecuda_b200 import phantoms
    from dosecuda_b200.plan_imrt import IMRTPlan
    grid = phantoms.photon_phantom((64, 64, 64), 4.0, seed=11)
    plan = IMRTPlan(machine)
    plan.addSquareField(label, 8, 6, mu=100, gantry_angle=30.0, collimator_angle=10.0)
    labels = list(plan.dicom_energy_label.astype(str))
    model = plan.beam_models[labels.index(label)]
    cp = plan.beam_list[0].cp_list[0]
    vol = phantoms.volume_object(grid, grid.DensityFromHU(machine))
    d = dk.photon_dose_cuda(model, vol, cp, 0)
    o, _ = oracle.photon_dose(vol.voxel_data, np.asarray(vol.spacing)[[0, 0, 0]], vol.origin, model, cp.iso, cp.mu,
                              cp.ga, cp.ca, cp.ta, np.ascontiguousarray(cp.mlc))
    assert d.max() > 0.1 * o.max() > 0
    assert dose_diff(d, o) <= TOL
    assert gamma_pass_rate(d, o, 4.0) >= GAMMA


def test_odd_sized_volumes_vs_oracle(dk):
    """Volume extents that are multiples of no tile (17 x 23 x 29 protons,
    19 x 21 x 25 photons), oblique couch / gantry: the partial tiles, warps
    and slices of every kernel against the FP64 oracle and, where it is
    built, the reference itself (bit for bit for the WET).  The WET is held
    to the oracle at gantry 0 only: at gantry 30 the smoothing's rotated
    sample points fall on the nearest-voxel rounding's knife edges often
    enough that the float64 oracle and the float32 reference disagree on
    some neighbours (up to 0.06 cm), while this engine still equals the
    reference exactly."""
    import oracle
    from dosecheck import wet_close
    from dosecuda_b200 import phantoms
    ref = _ref_module()
    for gantry, couch in ((0.0, 10.0), (30.0, 10.0)):
        grid, plan = phantoms.proton_small(shape=(17, 23, 29), spacing=3.0, energy_ids=(5, 15), field_mm=24.0,
                                           pitch_mm=4.0, gantry=gantry, couch=couch, seed=9)
        model, beam = plan.beam_models[0], plan.beam_list[0]
        rl = phantoms.volume_object(grid, grid.RLSPFromHU(plan.machine_name))
        w = dk.proton_raytrace_cuda(model, rl, beam, 0)
        assert w.shape == (17, 23, 29)
        sp = np.asarray(rl.spacing)[[0, 0, 0]]
        if gantry == 0.0:
            w_o, _ = oracle.proton_wet(rl.voxel_data, sp, rl.origin, beam.iso, beam.gantry_angle, beam.couch_angle,
                                       model.VSADX, model.VSADY)
            assert wet_close(w, w_o)
        if ref is not None:
            assert np.array_equal(w, ref.proton_raytrace_cuda(model, rl, beam, 0))
        d = dk.proton_spot_cuda(model, rl, phantoms.volume_object(grid, w), beam, 0)
        d_o, _ = oracle.proton_dose(w, sp, rl.origin, beam.iso, beam.gantry_angle, beam.couch_angle, model,
                                    beam.spot_list)
        assert d.max() > 0 and dose_diff(d, d_o) <= 1e-3
    g2, p2 = phantoms.photon_small(shape=(19, 21, 25), spacing=4.0, field_cm=(4.0, 6.0), gantry=45.0, seed=9)
    m2, cp2 = p2.beam_models[0], p2.beam_list[0].cp_list[0]
    vol = phantoms.volume_object(g2, g2.DensityFromHU(p2.machine_name))
    x = dk.photon_dose_cuda(m2, vol, cp2, 0)
    o, _ = oracle.photon_dose(vol.voxel_data, np.asarray(vol.spacing)[[0, 0, 0]], vol.origin, m2, cp2.iso, cp2.mu,
                              cp2.ga, cp2.ca, cp2.ta, np.ascontiguousarray(cp2.mlc))
    assert x.shape == (19, 21, 25) and x.max() > 0
    assert dose_diff(x, o) <= TOL and gamma_pass_rate(x, o, 4.0) >= GAMMA


def _ref_module():
    """The reference's own extension when oracle/_ref holds a build of it."""
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if not glob.glob(os.path.join(ref_dir, "dose_kernels*.so")):
        return None
    sys.path.insert(0, ref_dir)
    try:
        import dose_kernels as ref
    finally:
        sys.path.remove(ref_dir)
    return ref
