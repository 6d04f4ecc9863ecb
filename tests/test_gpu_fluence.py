"""Photon dose in a beamlet fluence map (engine.PhotonFluenceBeam, C ABI
dc_photon_beam_fluence_*) and its hand-written adjoint, the transpose of the
collapsed-cone superposition.  Oracles: the unmodulated CCCS (an all-ones
map gives it bit for bit), an explicit beamlet-dose matrix assembled column
by column from unit maps (linearity, and the adjoint against its
transpose), and central finite differences of a nonlinear objective."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dosecuda_b200 import engine, phantoms
    grid, plan = phantoms.photon_small(shape=(28, 32, 30), spacing=5.0, field_cm=(6.0, 6.0), gantry=20.0,
                                       lung_mm=(40.0, 30.0, 30.0), bone_mm=15.0, seed=8)
    model, cp = plan.beam_models[0], plan.beam_list[0].cp_list[0]
    density = torch.from_numpy(grid.DensityFromHU(plan.machine_name)).cuda()
    fb = engine.PhotonFluenceBeam.field_map(density, grid, model, cp, pitch=15.0, margin=10.0)
    return torch, engine, grid, model, cp, density, fb


def test_all_ones_map_is_the_plain_cccs(setup):
    torch, engine, grid, model, cp, density, fb = setup
    ones = torch.ones((fb.nb, fb.na), dtype=torch.float32, device="cuda")
    d1 = fb.dose(ones).clone()
    d0 = fb.beam.dose()
    torch.cuda.synchronize()
    assert torch.equal(d1, d0)
    ref = engine.photon_dose(density, grid, model, cp)
    torch.cuda.synchronize()
    assert torch.equal(d1, ref)


def test_explicit_beamlet_matrix_linearity_and_transpose(setup):
    torch, engine, grid, model, cp, density, fb = setup
    nbm = fb.na * fb.nb
    cols = []
    for q in range(nbm):
        e = torch.zeros(nbm, dtype=torch.float32, device="cuda")
        e[q] = 1.0
        cols.append(fb.dose(e.reshape(fb.nb, fb.na)).double().reshape(-1).clone())
    A = torch.stack(cols, dim=1)  # voxels x beamlets
    g = torch.Generator(device="cpu").manual_seed(3)
    F = torch.rand(nbm, generator=g).cuda() * 1.5 + 0.25
    d = fb.dose(F.reshape(fb.nb, fb.na).float()).double().reshape(-1)
    ref = A @ F.double()
    assert float((d - ref).abs().max()) <= 1e-5 * float(ref.abs().max())
    gd = torch.randn(d.numel(), generator=g).cuda()
    adj = fb.adjoint(gd.reshape(fb.beam.shape).float()).reshape(-1)
    exp = A.t() @ gd.double()
    rel = float((adj - exp).abs().max() / exp.abs().max())
    print("\nbeamlets %d: adjoint vs explicit A^T g, max rel. error %.2e" % (nbm, rel))
    assert rel <= 1e-4


def test_central_differences_of_a_nonlinear_objective(setup):
    torch, engine, grid, model, cp, density, fb = setup
    g = torch.Generator(device="cpu").manual_seed(5)
    F0 = (torch.rand((fb.nb, fb.na), generator=g) * 0.5 + 0.75).cuda()
    target = fb.dose(torch.ones_like(F0)).double().clone() * 1.1

    def objective(F):
        d = engine.photon_fluence_dose_autograd(F, fb).double()
        return ((d - target) ** 2).sum()

    F = F0.clone().requires_grad_(True)
    f = objective(F)
    f.backward()
    grad = F.grad.double().reshape(-1)
    h = 1e-2
    picks = torch.randperm(F0.numel(), generator=g)[:12]
    for q in picks.tolist():
        fp = F0.clone().reshape(-1)
        fm = F0.clone().reshape(-1)
        fp[q] += h
        fm[q] -= h
        with torch.no_grad():
            num = (objective(fp.reshape(F0.shape)) - objective(fm.reshape(F0.shape))).item() / (2 * h)
        scale = max(abs(num), 1e-3 * float(grad.abs().max()))
        assert abs(float(grad[q]) - num) <= 2e-3 * scale, (q, float(grad[q]), num)


def test_fluence_optimizer_lowers_the_objective_and_resumes(setup, tmp_path):
    torch, engine, grid, model, cp, density, fb = setup
    from dosecuda_b200.optimize import DoseObjective, FluenceOptimizer
    d0 = fb.dose(torch.ones((fb.nb, fb.na), device="cuda")).clone()
    dmax = float(d0.max())
    # flatten the dose inside the field's high-dose region to 90 % of Dmax
    target = d0 > 0.5 * dmax
    obj = DoseObjective().uniform(target, 0.9 * dmax)
    opt = FluenceOptimizer([fb], obj, lr=0.05)
    f0 = opt.evaluate()
    opt.run(15)
    f1 = opt.evaluate()
    assert f1 < 0.7 * f0
    ck = str(tmp_path / "fl.pt")
    opt.save(ck)
    opt.run(5)
    after = opt.mu.detach().clone()
    opt2 = FluenceOptimizer([fb], obj, lr=0.05)
    opt2.load(ck)
    opt2.run(5)
    torch.cuda.synchronize()
    # float atomics in the adjoint reorder between runs
    assert float((opt2.mu.detach() - after).abs().max()) <= 1e-4 * float(after.abs().max())
