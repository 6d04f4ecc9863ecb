"""Segment-weight (fluence) gradients of a photon beam
(engine.PhotonPlanBasis, engine.photon_dose_autograd): the per-control-point
CCCS doses kept on the device as a linear basis, combined and adjointed by
hand-written kernels.  Oracles: the control-point plan loop (bit for bit at
unit weights), the explicit float64 gradient from the basis, and central
finite differences of a plan objective."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def arc():
    from dosecuda_b200 import engine, phantoms
    from dosecuda_b200.plan_imrt import IMRTControlPoint
    grid, plan = phantoms.photon_small(seed=2, shape=(64, 64, 64), spacing=4.0, field_cm=(6.0, 6.0))
    model = plan.beam_models[0]
    cp0 = plan.beam_list[0].cp_list[0]
    cps = [IMRTControlPoint(cp0.iso, 20.0, np.array(cp0.mlc, copy=True), g, 0.0, 0.0, None, None)
           for g in (0.0, 60.0, 120.0, 180.0, 240.0, 300.0)]
    density = torch.as_tensor(grid.DensityFromHU(plan.machine_name)).cuda()
    basis = engine.PhotonPlanBasis(density, grid, model, cps)
    return engine, grid, model, cps, density, basis


def test_unit_weights_equal_the_plan_loop(arc):
    engine, grid, model, cps, density, basis = arc
    of = [float(model.outputFactor(cp)) for cp in cps]
    ref = torch.zeros_like(density)
    engine.photon_plan_dose(density, grid, model, cps, of, ref)
    d = basis.dose()
    torch.cuda.synchronize()
    assert torch.equal(d, ref) and float(d.max()) > 0


def test_adjoint_equals_explicit_gradient(arc):
    engine, grid, model, cps, density, basis = arc
    g = torch.randn(density.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    adj = basis.adjoint(g)
    ref = basis.output_factors * (basis.basis.reshape(len(cps), -1).double() @ g.reshape(-1).double())
    torch.cuda.synchronize()
    assert torch.allclose(adj, ref, rtol=1e-10, atol=1e-12 * float(ref.abs().max()))


def test_autograd_matches_finite_differences_and_optimises(arc):
    engine, grid, model, cps, density, basis = arc
    d1 = basis.dose()
    target = d1 > 0.5 * float(d1.max())
    presc = float(d1[target].mean())
    outside = (d1 > 0.05 * float(d1.max())) & ~target

    def objective(dose):
        dd = dose.double()
        return ((dd[target] - presc) ** 2).sum() + 0.1 * (dd[outside] ** 2).sum()

    w = torch.linspace(0.5, 1.5, len(cps), device="cuda", dtype=torch.float64).requires_grad_(True)
    f = objective(engine.photon_dose_autograd(w, basis))
    f.backward()
    grad = w.grad.detach().clone()
    h = 1e-3
    for b in range(len(cps)):
        wp, wm = w.detach().clone(), w.detach().clone()
        wp[b] += h
        wm[b] -= h
        fd = (objective(basis.dose(wp)) - objective(basis.dose(wm))).item() / (2 * h)
        assert abs(fd - grad[b].item()) <= 2e-3 * grad.abs().max().item() + 1e-6, (b, fd, grad[b].item())
    # projected Adam on the segment weights lowers the objective
    w = torch.full((len(cps),), 1.5, device="cuda", dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([w], lr=0.02)
    f0 = objective(engine.photon_dose_autograd(w, basis)).item()
    for _ in range(60):
        opt.zero_grad()
        objective(engine.photon_dose_autograd(w, basis)).backward()
        opt.step()
        with torch.no_grad():
            w.clamp_(min=0.0)
    f1 = objective(engine.photon_dose_autograd(w, basis)).item()
    assert f1 < 0.5 * f0


def test_segment_weight_optimiser_and_resume(arc, tmp_path):
    engine, grid, model, cps, density, basis = arc
    from dosecuda_b200.optimize import DoseObjective, ImrtOptimizer
    d1 = basis.dose()
    target = d1 > 0.5 * float(d1.max())
    ring = (d1 > 0.1 * float(d1.max())) & ~target
    obj = DoseObjective().uniform(target, 1.2 * float(d1[target].mean())).max_dose(ring, 0.2 * float(d1.max()), 5.0)
    opt = ImrtOptimizer([basis], obj)
    assert torch.equal(opt.dose().detach(), d1)  # unit weights: the plan as delivered
    f0 = opt.evaluate()
    opt.run(40)
    assert opt.evaluate() < 0.7 * f0 and float(opt.mu.detach().min()) >= 0.0
    # checkpoint / resume continues the run
    a = ImrtOptimizer([basis], obj)
    a.run(20)
    path = str(tmp_path / "imrt.pt")
    b = ImrtOptimizer([basis], obj)
    b.run(10, checkpoint=path)
    c = ImrtOptimizer([basis], obj, weights=torch.full((len(cps),), 3.0, device="cuda"))
    c.load(path)
    c.run(10)
    assert c.iteration == 20
    assert float((c.mu.detach() - a.mu.detach()).abs().max()) <= 1e-5 * float(a.mu.detach().abs().max())
