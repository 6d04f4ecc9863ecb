"""Photon beam handle (dc_photon_beam_*) and the gamma kernel (dc_gamma).

The handle splits dc_photon_dose into its TERMA and CCCS passes: its full
dose must equal dc_photon_dose_dev bit for bit, and its sparse probe must
equal the full dose at the probe voxels bit for bit.  The gamma kernel is
checked against a NumPy evaluation of the same definition (global dose
criterion, trilinear evaluated dose on a dta/4 lattice inside the dta
sphere)."""
import numpy as np
import pytest
import torch
from scipy import ndimage

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    from dosecuda_b200 import engine, phantoms
    from dosecuda_b200.dose_kernels import ControlPointView, PhotonModelView
    grid, plan = phantoms.photon_small(seed=5, shape=(64, 64, 64), spacing=2.5, field_cm=(8.0, 6.0), gantry=30.0)
    density = torch.as_tensor(grid.DensityFromHU(plan.machine_name)).cuda()
    model = plan.beam_models[0]
    cp = plan.beam_list[0].cp_list[0]
    views = (PhotonModelView(model), ControlPointView(cp))
    ref = engine.photon_dose(density, grid, model, cp, views=views)
    torch.cuda.synchronize()
    return engine, grid, density, model, cp, views, ref


def test_beam_dose_equals_photon_dose(case):
    engine, grid, density, model, cp, views, ref = case
    beam = engine.PhotonBeam(grid, density.shape)
    beam.set_density(density)
    terma = beam.terma(model, cp, out=True, views=views)
    dose = beam.dose()
    assert torch.equal(dose, ref)
    assert float(terma.max()) > 0.1 and float(terma.min()) >= 0.0
    # a second control point on the same handle
    dose2 = beam.dose()
    assert torch.equal(dose2, ref)
    beam.close()


def test_probe_equals_full_dose_at_probe_voxels(case):
    engine, grid, density, model, cp, views, ref = case
    beam = engine.PhotonBeam(grid, density.shape)
    beam.set_density(density)
    beam.terma(model, cp, views=views)
    n = beam.select_probe()
    assert 200 < n < 0.05 * density.numel()
    _, n2, host = beam.probe_voxels()
    assert n2 == n and np.all(np.diff(host) > 0) and host.min() >= 0 and host.max() < density.numel()
    probe = beam.probe()
    assert torch.equal(probe, ref.view(-1)[torch.as_tensor(host, device="cuda").long()])
    # explicit voxel list (with an out-of-grid index, which gives 0)
    vox = torch.tensor([0, int(host[n // 2]), density.numel() + 5], dtype=torch.int32, device="cuda")
    p2 = beam.probe(vox)
    assert float(p2[0]) == float(ref.view(-1)[0]) and float(p2[1]) == float(ref.view(-1)[int(host[n // 2])])
    assert float(p2[2]) == 0.0
    # the probe covers the high-dose region
    assert float(probe.max()) >= 0.9 * float(ref.max())
    beam.close()


def _gamma_numpy(eval_vol, ref_vals, idx, spacing, norm, dta=2.0, dd=0.02, cutoff=0.1, steps=4):
    nz, ny, nx = eval_vol.shape
    k, rem = np.divmod(idx, nx * ny)
    j, i = np.divmod(rem, nx)
    h = dta / steps
    offs = [(a, b, c) for a in range(-steps, steps + 1) for b in range(-steps, steps + 1)
            for c in range(-steps, steps + 1) if (a * a + b * b + c * c) * h * h <= dta * dta * 1.0001]
    best = np.full(len(idx), np.inf)
    sx, sy, sz = spacing
    for ix, iy, iz in offs:
        x = i + ix * h / sx
        y = j + iy * h / sy
        z = k + iz * h / sz
        ok = (x >= 0) & (y >= 0) & (z >= 0) & (x <= nx - 1) & (y <= ny - 1) & (z <= nz - 1)
        E = ndimage.map_coordinates(eval_vol, [z, y, x], order=1, mode="nearest")
        g2 = (ix * ix + iy * iy + iz * iz) * h * h / dta ** 2 + ((E - ref_vals) / (dd * norm)) ** 2
        best = np.where(ok, np.minimum(best, g2), best)
    keep = ref_vals >= cutoff * norm
    return int(keep.sum()), int((best[keep] <= 1.0).sum())


def test_gamma_kernel_matches_numpy(case):
    engine, grid, density, model, cp, views, ref = case
    rng = np.random.default_rng(0)
    refn = ref.cpu().numpy().astype(np.float64)
    # evaluated dose: shifted by 1 mm along x and scaled by 1.5 %, plus noise
    ev = ndimage.shift(refn, (0.0, 0.0, 0.4), order=1, mode="nearest") * 1.015
    ev = ev * (1.0 + 0.01 * rng.standard_normal(ev.shape))
    ev = np.maximum(ev, 0.0).astype(np.float32)
    evt = torch.as_tensor(ev).cuda()
    idx = np.sort(rng.choice(refn.size, 4000, replace=False)).astype(np.int32)
    idx = np.concatenate([idx, np.flatnonzero(refn.reshape(-1) > 0.5 * refn.max())[:2000].astype(np.int32)])
    idx = np.unique(idx)
    ref_vals = refn.reshape(-1)[idx]
    norm = float(ev.max())
    counts = engine.gamma_counts(evt, grid.spacing, torch.as_tensor(ref_vals, dtype=torch.float32).cuda(),
                                 torch.as_tensor(idx).cuda())
    ev_gpu, ps_gpu = (int(v) for v in counts[:2].cpu())
    ev_np, ps_np = _gamma_numpy(ev.astype(np.float64), ref_vals.astype(np.float32).astype(np.float64), idx,
                                np.asarray(grid.spacing, np.float64), norm)
    assert ev_gpu == ev_np
    assert abs(ps_gpu - ps_np) <= max(2, int(0.002 * ev_np))  # fp32 vs fp64 at gamma == 1 knife edges
    assert 0.3 < ps_np / ev_np < 1.0
    # whole-volume mode and explicit normalisation
    c_all = engine.gamma_counts(evt, grid.spacing, ref, dose_norm=norm)
    e_all, p_all = (int(v) for v in c_all[:2].cpu())
    assert e_all == int((refn >= 0.1 * norm).sum())
    assert 0 < p_all <= e_all
    # identical volumes pass everywhere
    c_id = engine.gamma_counts(ref, grid.spacing, ref)
    e_id, p_id = (int(v) for v in c_id[:2].cpu())
    assert e_id > 0 and p_id == e_id
