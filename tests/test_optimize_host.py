"""Spot-weight optimiser (dosecuda_b200.optimize) on the CPU.

The device beams are replaced by a dense influence matrix with the same
``dose``/``adjoint`` interface as ``engine.ProtonBeamPlan`` (forward A mu,
backward A^T g in float64), so the objective, the projected Adam loop, the
gradient path through ``engine.proton_dose_autograd`` and checkpoint/resume
are checked exactly, without a GPU."""
import numpy as np
import pytest
import torch

from dosecuda_b200.optimize import DoseObjective, ImptOptimizer, load_influence_csr, save_influence_csr

SHAPE = (6, 7, 8)


class DensePlan:
    def __init__(self, a: torch.Tensor):
        self.A = a
        self.n_spots = a.shape[1]
        self.mu = torch.ones(self.n_spots)

    def dose(self, wet, mu=None, out=None, stream=None):
        m = self.mu if mu is None else mu
        return (self.A @ m.float()).reshape(wet.shape)

    def adjoint(self, wet, grad_dose, stream=None):
        return self.A.double().t() @ grad_dose.reshape(-1).double()


def _case(seed=0, spots=(9, 6)):
    g = torch.Generator().manual_seed(seed)
    n = int(np.prod(SHAPE))
    plans = [DensePlan(torch.rand((n, k), generator=g) * (torch.rand((n, 1), generator=g) < 0.6)) for k in spots]
    wets = [torch.zeros(SHAPE) for _ in spots]
    target = torch.zeros(SHAPE, dtype=torch.bool)
    target[2:5, 2:5, 2:6] = True
    oar = torch.zeros(SHAPE, dtype=torch.bool)
    oar[2:5, 5:7, 2:6] = True
    cold = torch.zeros(SHAPE, dtype=torch.bool)
    cold[0, :, :] = True
    obj = DoseObjective().uniform(target, 2.0).max_dose(oar, 1.0, 10.0).min_dose(cold, 0.5, 0.5)
    return plans, wets, obj, target, oar, cold


def test_objective_matches_its_definition():
    plans, wets, obj, target, oar, cold = _case()
    d = torch.rand(SHAPE, dtype=torch.float32) * 3
    dd = d.double()
    ref = ((dd[target] - 2) ** 2).sum() + 10 * (torch.clamp(dd[oar] - 1, min=0) ** 2).sum() + \
        0.5 * (torch.clamp(dd[cold] - 0.5, max=0) ** 2).sum()
    assert float(obj(d)) == pytest.approx(float(ref), rel=1e-14)
    with pytest.raises(ValueError):
        obj(torch.zeros((2, 2, 2)))
    with pytest.raises(ValueError):
        DoseObjective().add("mean", target, 1.0)
    with pytest.raises(ValueError):
        DoseObjective().uniform(target.float(), 1.0)


def test_gradient_is_the_adjoint_of_the_objective_gradient():
    plans, wets, obj, *_ = _case(1)
    opt = ImptOptimizer(plans, wets, obj)
    mu = opt.mu.detach().clone().requires_grad_(True)
    f = obj(opt.dose(mu))
    f.backward()
    # explicit: d f / d mu = A^T (d f / d D)
    a = torch.cat([p.A for p in plans], dim=1).double()
    d = (a @ mu.detach().double()).reshape(SHAPE).requires_grad_(True)
    obj(d).backward()
    ref = a.t() @ d.grad.reshape(-1)
    torch.testing.assert_close(mu.grad.double(), ref, rtol=1e-5, atol=1e-6 * float(ref.abs().max()))


def test_projected_adam_reduces_the_objective():
    plans, wets, obj, target, *_ = _case(2)
    opt = ImptOptimizer(plans, wets, obj)
    k = opt.scale_to(target, 2.0)
    assert k > 0 and float(opt.dose().detach()[target].double().mean()) == pytest.approx(2.0, rel=1e-5)
    f0 = opt.evaluate()
    opt.run(150)
    assert opt.iteration == 150 and float(opt.mu.detach().min()) >= 0.0
    assert opt.evaluate() < 0.5 * f0
    with pytest.raises(RuntimeError):
        opt.scale_to(target, 2.0)


def test_resume_continues_the_run_exactly(tmp_path):
    plans, wets, obj, target, *_ = _case(3)
    straight = ImptOptimizer(plans, wets, obj)
    straight.scale_to(target, 2.0)
    straight.run(12)

    first = ImptOptimizer(plans, wets, obj)
    first.scale_to(target, 2.0)
    path = str(tmp_path / "opt.pt")
    first.run(5, checkpoint=path)

    resumed = ImptOptimizer(plans, wets, obj, mu=torch.full((15,), 7.0))  # state comes from the file
    resumed.load(path)
    assert resumed.iteration == 5 and resumed.lr == first.lr
    resumed.run(7)
    assert torch.equal(resumed.mu.detach(), straight.mu.detach())
    assert resumed.iteration == 12

    other = ImptOptimizer(_case(3, spots=(8, 6))[0], wets, obj)
    with pytest.raises(ValueError):
        other.load(path)


def test_influence_cache_round_trip(tmp_path):
    g = torch.Generator().manual_seed(4)
    n_vox, n_spots = int(np.prod(SHAPE)), 11
    dense = torch.rand((n_vox, n_spots), generator=g) * (torch.rand((n_vox, n_spots), generator=g) < 0.2)
    nz = dense != 0
    row_ptr = torch.zeros(n_vox + 1, dtype=torch.int64)
    row_ptr[1:] = torch.cumsum(nz.sum(1), 0)
    col = torch.nonzero(nz)[:, 1].to(torch.int32)
    val = dense[nz].float()
    path = str(tmp_path / "influence.npz")
    save_influence_csr(path, row_ptr, col, val, SHAPE, n_spots)
    r2, c2, v2, shape, ns = load_influence_csr(path, device="cpu")
    assert torch.equal(r2, row_ptr) and torch.equal(c2, col) and torch.equal(v2, val)
    assert shape == SHAPE and ns == n_spots
    with pytest.raises(ValueError):
        save_influence_csr(path, row_ptr[:-1], col, val, SHAPE, n_spots)


def test_objective_on_voxel_list_equals_the_volume_form():
    plans, wets, obj, target, oar, cold = _case(5)
    d = torch.rand(SHAPE, dtype=torch.float32) * 3
    union = obj.voxel_union()
    assert bool((union[1:] > union[:-1]).all())  # sorted, unique
    expect = torch.nonzero((target | oar | cold).reshape(-1)).squeeze(1)
    assert torch.equal(union, expect)
    assert float(obj.on_list(d.reshape(-1)[union])) == float(obj(d))
    # a term added later extends the union
    extra = torch.zeros(SHAPE, dtype=torch.bool)
    extra[5, 6, 7] = True
    obj.max_dose(extra, 0.1)
    assert obj.voxel_union().numel() == union.numel() + 1


class DenseBasis:
    """CPU stand-in for engine.PhotonPlanBasis: per-control-point doses as
    rows of a dense matrix, output factors, same dose/adjoint interface."""

    def __init__(self, rows: torch.Tensor, of):
        self.basis = rows
        self.n = rows.shape[0]
        self.device = rows.device
        self.output_factors = torch.tensor(of, dtype=torch.float64)

    def dose(self, weights=None):
        w = torch.ones(self.n, dtype=torch.float64) if weights is None else weights.detach().double()
        return (self.basis.double().t() @ (w * self.output_factors)).float().reshape(SHAPE)

    def adjoint(self, grad):
        return self.output_factors * (self.basis.double() @ grad.reshape(-1).double())


def test_imrt_optimiser_and_resume_on_cpu(tmp_path):
    from dosecuda_b200.optimize import ImrtOptimizer
    g = torch.Generator().manual_seed(6)
    n = int(np.prod(SHAPE))
    bases = [DenseBasis(torch.rand((4, n), generator=g), [1.0, 0.98, 1.02, 1.01]),
             DenseBasis(torch.rand((3, n), generator=g), [0.97, 1.0, 1.03])]
    _, _, obj, target, *_ = _case(6)
    opt = ImrtOptimizer(bases, obj)
    assert torch.allclose(opt.dose().detach(), bases[0].dose() + bases[1].dose())
    f0 = opt.evaluate()
    opt.run(80)
    assert opt.evaluate() < 0.5 * f0 and float(opt.mu.detach().min()) >= 0.0
    straight = ImrtOptimizer(bases, obj)
    straight.run(12)
    path = str(tmp_path / "imrt.pt")
    first = ImrtOptimizer(bases, obj)
    first.run(5, checkpoint=path)
    resumed = ImrtOptimizer(bases, obj, weights=torch.full((7,), 2.0))
    resumed.load(path)
    resumed.run(7)
    assert torch.equal(resumed.mu.detach(), straight.mu.detach())
    with pytest.raises(ValueError):
        ImrtOptimizer(bases[:1], obj).load(path)


def test_build_cli_requires_an_output_for_the_checked_variant():
    import subprocess
    import sys
    r = subprocess.run([sys.executable, "-m", "dosecuda_b200.build", "--debug-bounds"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode != 0 and "--out" in r.stderr
