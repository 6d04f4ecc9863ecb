"""Proton beam handle: dose from device-side spot weights, the hand-written
adjoint D^T g behind torch.autograd, and the CSR dose-influence matrix.
Oracles: the existing spot-dose entry point, an explicit CSR gradient,
central finite differences, and the CPU oracle's single-spot doses."""
import numpy as np
import pytest

from dosecheck import dose_diff

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dosecuda_b200 import engine, phantoms
    grid, plan = phantoms.proton_small(shape=(40, 44, 48), spacing=3.0, energy_ids=(8, 16, 24), field_mm=36.0,
                                       pitch_mm=6.0, seed=3)
    model, beam = plan.beam_models[0], plan.beam_list[0]
    rl = torch.from_numpy(grid.RLSPFromHU(plan.machine_name)).cuda()
    wet = engine.proton_wet(rl, grid, beam, model)
    bp = engine.ProtonBeamPlan(grid, beam, model)
    return torch, engine, grid, plan, model, beam, wet, bp


def test_beam_dose_equals_spot_dose(setup):
    torch, engine, grid, plan, model, beam, wet, bp = setup
    d_ref = engine.proton_dose(wet, grid, beam, engine.ProtonModelDevice(model))
    d = bp.dose(wet)
    d_mu = bp.dose(wet, bp.mu.clone())
    torch.cuda.synchronize()
    assert torch.equal(d, d_ref) and torch.equal(d_mu, d_ref)


def test_dose_is_linear_in_weights(setup):
    torch, engine, grid, plan, model, beam, wet, bp = setup
    mu = bp.mu.clone()
    d1 = bp.dose(wet, mu)
    d2 = bp.dose(wet, 2.0 * mu)
    torch.cuda.synchronize()
    assert dose_diff(d2.cpu().numpy(), 2.0 * d1.cpu().numpy()) <= 1e-6


def _csr_dense_cols(torch, row_ptr, col, val, n_vox, cols):
    rows = torch.repeat_interleave(torch.arange(n_vox, device=row_ptr.device), row_ptr[1:] - row_ptr[:-1])
    out = {}
    for c in cols:
        m = col == c
        v = torch.zeros(n_vox, dtype=torch.float64, device=row_ptr.device)
        v[rows[m]] = val[m].double()
        out[c] = v
    return out


def test_adjoint_matches_explicit_csr_gradient(setup):
    torch, engine, grid, plan, model, beam, wet, bp = setup
    g = torch.randn(wet.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(7))
    adj = bp.adjoint(wet, g)
    row_ptr, col, val = bp.influence_csr(wet, cutoff=0.0)
    n_vox = wet.numel()
    rows = torch.repeat_interleave(torch.arange(n_vox, device="cuda"), row_ptr[1:] - row_ptr[:-1])
    grad_csr = torch.zeros(bp.n_spots, dtype=torch.float64, device="cuda")
    grad_csr.index_add_(0, col.long(), val.double() * g.reshape(-1)[rows].double())
    torch.cuda.synchronize()
    scale = grad_csr.abs().max().item()
    assert scale > 0
    assert (adj - grad_csr).abs().max().item() <= 1e-4 * scale


def test_csr_times_weights_is_the_dose(setup):
    torch, engine, grid, plan, model, beam, wet, bp = setup
    d = bp.dose(wet).reshape(-1).double()
    for cutoff, tol in ((0.0, 1e-5), (1e-4, 2e-3)):
        row_ptr, col, val = bp.influence_csr(wet, cutoff=cutoff)
        rows = torch.repeat_interleave(torch.arange(wet.numel(), device="cuda"), row_ptr[1:] - row_ptr[:-1])
        dd = torch.zeros_like(d)
        dd.index_add_(0, rows, val.double() * bp.mu.double()[col.long()])
        torch.cuda.synchronize()
        assert (dd - d).abs().max().item() <= tol * d.max().item(), cutoff
        assert col.dtype == torch.int32 and row_ptr.dtype == torch.int64 and val.dtype == torch.float32
        assert int(row_ptr[-1]) == col.numel()


def test_csr_is_deterministic_and_sorted_by_rows(setup):
    torch, engine, grid, plan, model, beam, wet, bp = setup
    a = bp.influence_csr(wet, cutoff=1e-4)
    b = bp.influence_csr(wet, cutoff=1e-4)
    torch.cuda.synchronize()
    assert all(torch.equal(x, y) for x, y in zip(a, b))
    assert bool((a[0][1:] >= a[0][:-1]).all())
    assert int(a[1].min()) >= 0 and int(a[1].max()) < bp.n_spots


def test_csr_columns_match_oracle_single_spot_doses(setup):
    import oracle
    torch, engine, grid, plan, model, beam, wet, bp = setup
    row_ptr, col, val = bp.influence_csr(wet, cutoff=0.0)
    cols = [0, bp.n_spots // 2, bp.n_spots - 1]
    dense = _csr_dense_cols(torch, row_ptr, col, val, wet.numel(), cols)
    w = wet.cpu().numpy()
    sp = np.asarray(grid.spacing, np.float32)[[0, 0, 0]]
    for c in cols:
        spot = beam.spot_list[c:c + 1].copy()
        spot[0, 2] = 1.0
        o, _ = oracle.proton_dose(w, sp, grid.origin, beam.iso, beam.gantry_angle, beam.couch_angle, model, spot)
        assert dose_diff(dense[c].cpu().numpy().reshape(w.shape), o) <= 1e-3


def test_autograd_gradient_matches_central_differences(setup):
    """Objective of the differentiable-optimisation workload: target voxels
    pulled to 2 Gy, an organ at risk penalised above 1 Gy (FP64 reduction);
    gradient by the adjoint kernel through torch.autograd, checked on 64
    seeded spots by central differences with h = 1e-3 MU."""
    torch, engine, grid, plan, model, beam, wet, bp = setup
    d0 = bp.dose(wet).double()
    scale = 2.0 / d0.max().item()
    target = d0 > 0.5 * d0.max()
    oar = (d0 > 0.1 * d0.max()) & ~target

    def objective(dose):
        d = dose.double() * scale
        return ((d[target] - 2.0) ** 2).sum() + 10.0 * (torch.clamp(d[oar] - 1.0, min=0.0) ** 2).sum()

    mu = bp.mu.clone().requires_grad_(True)
    f = objective(engine.proton_dose_autograd(mu, wet, bp))
    f.backward()
    grad = mu.grad.double()
    idx = torch.randperm(bp.n_spots, generator=torch.Generator().manual_seed(11))[:min(64, bp.n_spots)]
    h = 1e-3
    fd = []
    with torch.no_grad():
        for s in idx.tolist():
            mp = bp.mu.clone()
            mp[s] += h
            mm = bp.mu.clone()
            mm[s] -= h
            fd.append((objective(bp.dose(wet, mp)) - objective(bp.dose(wet, mm))).item() / (2 * h))
    fd = torch.tensor(fd, dtype=torch.float64)
    g = grad[idx].cpu()
    assert torch.allclose(g, fd, rtol=2e-2, atol=2e-3 * g.abs().max().item())
