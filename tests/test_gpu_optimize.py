"""Spot-weight optimisation on the device (dosecuda_b200.optimize): two
beams, target sphere and an adjacent organ at risk; the objective falls,
weights stay non-negative, a resumed run continues the straight one, and the
influence-matrix cache reproduces the matrix and the dose."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    from dosecuda_b200 import engine, phantoms
    grid, plan = phantoms.proton_small(shape=(40, 44, 48), spacing=3.0, energy_ids=(8, 14, 20, 26), field_mm=36.0,
                                       pitch_mm=6.0, seed=5)
    model = plan.beam_models[0]
    beams = [plan.beam_list[0], phantoms.proton_beam(energy_ids=(8, 14, 20, 26), field_mm=36.0, pitch_mm=6.0,
                                                     gantry=90.0, seed=6)]
    rl = torch.from_numpy(grid.RLSPFromHU(plan.machine_name)).cuda()
    wets = [engine.proton_wet(rl, grid, b, model) for b in beams]
    nz, ny, nx = rl.shape
    sp = np.asarray(grid.spacing, np.float64)
    z, y, x = np.meshgrid(*(np.arange(n) * s + o for n, s, o in zip((nz, ny, nx), sp[[2, 1, 0]],
                                                                     np.asarray(grid.origin)[[2, 1, 0]])),
                          indexing="ij")
    target = torch.as_tensor(x ** 2 + y ** 2 + z ** 2 <= 15.0 ** 2).cuda()
    oar = torch.as_tensor((np.abs(x - 24.0) <= 6.0) & (np.abs(y) <= 12.0) & (np.abs(z) <= 12.0)).cuda()
    return torch, engine, grid, model, beams, wets, target, oar


def _optimizer(setup):
    torch, engine, grid, model, beams, wets, target, oar = setup
    from dosecuda_b200.optimize import DoseObjective, ImptOptimizer
    plans = [engine.ProtonBeamPlan(grid, b, model) for b in beams]
    obj = DoseObjective().uniform(target, 2.0).max_dose(oar, 1.0, 10.0)
    opt = ImptOptimizer(plans, wets, obj)
    opt.scale_to(target, 2.0)
    return opt


def test_optimisation_reduces_the_objective(setup):
    torch = setup[0]
    opt = _optimizer(setup)
    f0 = opt.evaluate()
    opt.run(40)
    torch.cuda.synchronize()
    f1 = opt.evaluate()
    assert f1 < 0.5 * f0, (f0, f1)
    assert float(opt.mu.detach().min()) >= 0.0 and opt.iteration == 40


def test_resumed_optimisation_continues_the_straight_run(setup, tmp_path):
    torch = setup[0]
    straight = _optimizer(setup)
    straight.run(16)
    first = _optimizer(setup)
    path = str(tmp_path / "opt.pt")
    first.run(8, checkpoint=path)
    resumed = _optimizer(setup)
    resumed.mu.data.fill_(3.0)  # everything must come from the checkpoint
    resumed.load(path)
    resumed.run(8)
    torch.cuda.synchronize()
    a, b = straight.mu.detach().double(), resumed.mu.detach().double()
    # the adjoint's float64 atomics are order-dependent: equal up to rounding
    assert (a - b).abs().max().item() <= 1e-5 * a.abs().max().item()
    assert resumed.iteration == 16


def test_influence_cache_reproduces_the_dose(setup, tmp_path):
    torch, engine, grid, model, beams, wets, target, oar = setup
    from dosecuda_b200.optimize import load_influence_csr, save_influence_csr
    bp = engine.ProtonBeamPlan(grid, beams[0], model)
    row_ptr, col, val = bp.influence_csr(wets[0], cutoff=0.0)
    path = str(tmp_path / "influence.npz")
    save_influence_csr(path, row_ptr, col, val, tuple(wets[0].shape), bp.n_spots)
    r2, c2, v2, shape, ns = load_influence_csr(path)
    assert torch.equal(r2, row_ptr) and torch.equal(c2, col) and torch.equal(v2, val)
    assert shape == tuple(wets[0].shape) and ns == bp.n_spots
    a = torch.sparse_csr_tensor(r2, c2.long(), v2.double(), size=(wets[0].numel(), ns))
    d = (a @ bp.mu.double().unsqueeze(1)).squeeze(1)
    ref = bp.dose(wets[0]).reshape(-1).double()
    torch.cuda.synchronize()
    assert (d - ref).abs().max().item() <= 1e-5 * ref.max().item()


def test_voxel_list_dose_and_adjoint_equal_the_volume_forms(setup):
    torch, engine, grid, model, beams, wets, target, oar = setup
    bp = engine.ProtonBeamPlan(grid, beams[0], model)
    wet = wets[0]
    vox = torch.nonzero((target | oar).reshape(-1)).squeeze(1)
    full = bp.dose(wet).reshape(-1)
    lst = bp.dose_list(wet, vox)
    ref = full[vox]
    scale = float(ref.abs().max())
    assert scale > 0 and float((lst - ref).abs().max()) <= 1e-6 * scale
    # entries outside the grid give 0, the others are unaffected
    bad = torch.tensor([-1, wet.numel(), int(vox[0])], device="cuda")
    out = bp.dose_list(wet, bad)
    assert float(out[0]) == 0.0 and float(out[1]) == 0.0 and float(out[2]) == float(lst[0])
    g = torch.randn(vox.numel(), device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    g_full = torch.zeros(wet.numel(), device="cuda")
    g_full[vox] = g
    a_full = bp.adjoint(wet, g_full.reshape(wet.shape))
    a_list = bp.adjoint_list(wet, vox, g)
    torch.cuda.synchronize()
    assert float((a_list - a_full).abs().max()) <= 1e-5 * float(a_full.abs().max())


def test_objective_voxel_optimiser_follows_the_volume_one(setup):
    torch = setup[0]
    from dosecuda_b200.optimize import ImptOptimizer
    vol = _optimizer(setup)
    f0 = vol.evaluate()
    vol.run(30)
    obj = vol.objective
    lst = ImptOptimizer(vol.plans, vol.wets, obj, voxels="objective")
    lst.scale_to(setup[6], 2.0)
    assert abs(lst.evaluate() - f0) <= 1e-5 * f0
    lst.run(30)
    torch.cuda.synchronize()
    with torch.no_grad():
        f_vol = float(obj(vol.dose()))
        f_lst = float(obj(lst.dose()))
    assert f_lst < 0.5 * f0
    assert abs(f_lst - f_vol) <= 1e-3 * f0
    a, b = vol.mu.detach().double(), lst.mu.detach().double()
    assert float((a - b).abs().max()) <= 1e-3 * float(a.abs().max())
