"""Batched IMPT: many plans (anisotropic grids, uneven beam and spot counts)
in one persistent launch.  Oracles: per-plan, per-beam calls of the existing
entry points, and the CPU oracle on one anisotropic plan; plus tile-shape
variants, the autotuner and CUDA-graph replay."""
import numpy as np
import pytest

from dosecheck import dose_diff

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dosecuda_b200 import engine, phantoms
    from dosecuda_b200.plan_impt import IMPTPlan
    model = IMPTPlan().beam_models[0]
    b = engine.ProtonBatch(model)
    plans = []
    for seed, shape, sp in ((1, (36, 44, 40), (3.0, 3.0, 4.0)), (2, (40, 40, 48), (3.0, 3.0, 3.0)),
                            (3, (32, 48, 44), (3.5, 3.0, 4.0))):
        grid, beams, _ = phantoms.batch_plan(seed, shape=shape, spacing=sp, model=model, pitch_range=(7.0, 9.0),
                                             max_spots=4000)
        rl = torch.from_numpy(grid.RLSPFromHU("HitachiProbeatJHU")).cuda()
        pid = b.add_plan(grid, rl)
        ids = [b.add_beam(pid, bm) for bm in beams]
        plans.append((grid, beams, rl, pid, ids))
    b.commit()
    b.wet()
    b.dose()
    torch.cuda.synchronize()
    return torch, engine, model, b, plans


def test_batch_matches_per_beam_calls(batch):
    torch, engine, model, b, plans = batch
    dm = engine.ProtonModelDevice(model)
    for grid, beams, rl, pid, ids in plans:
        ref = torch.zeros_like(rl)
        for bm, bid in zip(beams, ids):
            w = engine.proton_wet(rl, grid, bm, model)
            torch.cuda.synchronize()
            assert torch.equal(w, b.wets[bid])  # the batch's WET is the per-beam WET
            ref += engine.proton_dose(w, grid, bm, dm)
        torch.cuda.synchronize()
        assert dose_diff(b.doses[pid].cpu().numpy(), ref.cpu().numpy()) <= 1e-5


def test_batch_anisotropic_plan_matches_oracle(batch):
    import oracle
    torch, engine, model, b, plans = batch
    grid, beams, rl, pid, ids = plans[0]
    sp = np.asarray(grid.spacing, np.float32)
    ref = np.zeros(rl.shape)
    for bm, bid in zip(beams, ids):
        w = b.wets[bid].cpu().numpy()
        o, _ = oracle.proton_dose(w, sp, grid.origin, bm.iso, bm.gantry_angle, bm.couch_angle, model, bm.spot_list)
        ref += o
    d = b.doses[pid].cpu().numpy()
    # the distance to the spot axis is taken as |ray x t|^2 / |t|^2, free of
    # the cancellation in |ray|^2 - (t.ray)^2 / |t|^2, so float tracks FP64
    # closely on every voxel, not only above 10 % of the maximum
    print("\nbatch plan vs FP64 oracle: %.2e of Dmax above 10 %%, %.2e on every voxel"
          % (dose_diff(d, ref), dose_diff(d, ref, thresh=0.0)))
    assert dose_diff(d, ref) <= 1e-4
    assert dose_diff(d, ref, thresh=0.0) <= 1e-4


def test_batch_influence_matrix_equals_the_per_beam_matrix(batch):
    """Count-then-fill CSR of every beam of the batch against the single-beam
    entry point on the same WET (the same kernels: equal arrays), and the
    matrix-vector product of the plan's beams against the batch dose."""
    torch, engine, model, b, plans = batch
    for grid, beams, rl, pid, ids in plans[:2]:
        total = torch.zeros(rl.numel(), dtype=torch.float64, device="cuda")
        for bm, bid in zip(beams, ids):
            r, c, v = b.influence_csr(bid, cutoff=1e-4)
            r0, c0, v0 = engine.ProtonBeamPlan(grid, bm, model).influence_csr(b.wets[bid], cutoff=1e-4)
            torch.cuda.synchronize()
            assert int(r[-1]) == c.numel() > 0
            # the single-beam call zero-fills its arrays before the fill pass,
            # so an entry counted but never filled would show as a zero
            assert bool((v0 > 0).all())
            assert torch.equal(r, r0) and torch.equal(c, c0) and torch.equal(v, v0)
            a = torch.sparse_csr_tensor(r, c.long(), v.double(), size=(rl.numel(), bm.spot_list.shape[0]))
            mu = torch.as_tensor(np.asarray(bm.spot_list, np.float64)[:, 2], device="cuda")
            total += (a @ mu.unsqueeze(1)).squeeze(1)
        b.dose(b.mu0)
        torch.cuda.synchronize()
        d = b.doses[pid].reshape(-1).double()
        # entries below 1e-4 of their spot's maximum are dropped from the matrix
        assert float((total - d).abs().max()) <= 2e-3 * float(d.max())
    # host-side checks, before any launch: NULL buffers, and a fill for a beam
    # other than the one counted last
    lib = engine._lib.load()
    first = plans[0][4][0]
    with pytest.raises(ValueError):
        engine._lib.raise_for(lib.dc_proton_batch_influence_fill(b._h, first, None, None, None, 0, None))
    buf = torch.zeros(16, dtype=torch.int64, device="cuda")
    with pytest.raises(ValueError):
        engine._lib.raise_for(lib.dc_proton_batch_influence_fill(b._h, first, buf.data_ptr(), buf.data_ptr(),
                                                                 buf.data_ptr(), 16, None))


def test_tile_variants_agree_and_autotune(batch, tmp_path):
    torch, engine, model, b, plans = batch
    base = [d.clone() for d in b.dose(variant=0)]
    for v in range(1, b.n_variants):
        out = b.dose(variant=v)
        torch.cuda.synchronize()
        for d0, d in zip(base, out):
            assert dose_diff(d.cpu().numpy(), d0.cpu().numpy()) <= 1e-5
    cache = tmp_path / "tune.json"
    v = b.autotune(str(cache))
    assert 0 <= v < b.n_variants and cache.exists()
    assert b.autotune(str(cache)) == v  # served from the cache


def test_weights_and_cuda_graph_replay(batch):
    torch, engine, model, b, plans = batch
    mu = b.mu0.clone()
    b.dose(mu)
    torch.cuda.synchronize()
    d1 = [d.clone() for d in b.doses]
    mu2 = (2.0 * b.mu0).contiguous()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        b.dose(mu2)  # warm-up on the capture stream
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    with torch.cuda.graph(g):
        b.dose(mu2)
    for _ in range(2):
        for d in b.doses:
            d.zero_()
        g.replay()
        torch.cuda.synchronize()
        for d, r in zip(b.doses, d1):
            assert dose_diff(d.cpu().numpy(), 2.0 * r.cpu().numpy()) <= 1e-5
    del g


def test_dicom_plan_feeds_the_batch(monkeypatch):
    """An RT Ion plan read by IMPTPlan.readPlanDicom (synthetic dataset through
    a stand-in pydicom, as in test_dicom_readers.py) goes into the batched
    engine whole (ProtonBatch.add_impt_plan) and gives computeIMPTPlan's dose."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from types import SimpleNamespace as NS
    from dosecuda_b200 import engine, phantoms, plan_impt
    from test_dicom_readers import _fake_pydicom
    plan = plan_impt.IMPTPlan()
    labels = plan.beam_models[0].energy_table["energy_label"].to_numpy()
    rng = np.random.default_rng(7)
    beams = []
    for ga, ta in ((0.0, 0.0), (70.0, 10.0)):
        cps = []
        for e in labels[[12, 16, 20]]:
            pos = rng.uniform(-15, 15, size=(6, 2)).round(1).ravel().tolist()
            cp = NS(NominalBeamEnergy=float(e), ScanSpotPositionMap=pos,
                    ScanSpotMetersetWeights=rng.uniform(0.2, 1.5, 6).round(3).tolist(), GantryAngle=ga,
                    PatientSupportAngle=ta, IsocenterPosition=[2.0, -1.0, 0.5])
            cps += [cp, NS(NominalBeamEnergy=float(e), ScanSpotPositionMap=pos, ScanSpotMetersetWeights=[0.0] * 6)]
        beams.append(NS(NumberOfRangeShifters=0, IonControlPointSequence=cps, RangeShifterSequence=[]))
    ds = NS(FractionGroupSequence=[NS(NumberOfFractionsPlanned=3)], IonBeamSequence=beams)
    fake = _fake_pydicom({"ion.dcm": ds})
    monkeypatch.setattr(plan_impt, "_pydicom", lambda: fake)
    plan.readPlanDicom("ion.dcm")
    grid = phantoms.proton_phantom((40, 44, 36), 3.0, seed=3)
    b = engine.ProtonBatch(plan.beam_models[0])
    pid = b.add_impt_plan(grid, plan)
    b.commit()
    b.wet()
    b.dose()
    torch.cuda.synchronize()
    grid.computeIMPTPlan(plan)
    got = b.plan_dose(pid).cpu().numpy()
    assert grid.dose.max() > 0
    assert dose_diff(got, grid.dose) <= 1e-5
    b.close()
