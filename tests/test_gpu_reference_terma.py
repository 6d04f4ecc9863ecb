"""Parity on the 128^3 photon workload against the reference's own build,
pinned down where the reference departs from its own algorithm.

The reference's compiled termaKernel (IMRTClasses.cu:209-250) divides the
scatter by the primary head transmission, fminf(1, ts / tp).  Where the
algorithm's primary transmission vanishes (voxels under closed leaf pairs or
far outside the field), the compiled kernel can get a tiny negative tp
instead of 0, and its TERMA explodes as ts^2 / tp.  These tests
  * run the reference's own ray-trace and TERMA kernels through the checker
    harness (oracle/ref_terma.cu) and require that every voxel where its
    TERMA departs from the FP64 oracle is one where the oracle's primary
    transmission is zero to rounding, and that the artifact is there on the
    workload;
  * compare the engine with the reference build on every voxel the departing
    TERMA voxels cannot reach (the CCCS's longest window around them), and
    report how many dose voxels that leaves;
  * compare the engine with the reference build on the whole volume, with no
    mask, on the workload with every leaf pair open over the phantom (a
    40 x 40 cm field), where the reference's TERMA does not depart at all."""
import glob
import os
import sys

import numpy as np
import pytest

from conftest import ROOT
from dosecheck import dose_diff, gamma_pass_rate

pytestmark = pytest.mark.gpu

TOL = 0.005
GAMMA = 0.995
TP_ZERO = 1e-6       # primary transmission that is zero up to float rounding of the leaf edges
TERMA_DEPART = 1e-3  # a TERMA voxel departs when it is off the oracle by more than 0.1 % of max TERMA


@pytest.fixture(scope="module")
def ref_dk():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if not glob.glob(os.path.join(ref_dir, "dose_kernels*.so")):
        pytest.skip("reference build oracle/_ref not present")
    sys.path.insert(0, ref_dir)
    import dose_kernels as ref
    sys.path.remove(ref_dir)
    return ref


def _workload(variant):
    from dosecuda_b200 import phantoms
    grid, plan = phantoms.photon_small(field_cm=(40.0, 40.0) if variant == "open_field" else (10.0, 10.0))
    model, cp = plan.beam_models[0], plan.beam_list[0].cp_list[0]
    if variant == "half_voxel":
        cp.iso = np.array(cp.iso, np.float32) + np.float32([0.5 * grid.spacing[0], 0.0, 0.0])
    elif variant == "parked_leaves":
        mlc = np.array(cp.mlc, np.float32)
        closed = mlc[:, 0] == mlc[:, 1]
        mlc[closed, 0] = mlc[closed, 1] = 200.0  # beyond the 160 mm half-width at every depth
        # column-major, as the plan API builds it: the reference's extension
        # reads this array's raw buffer column by column (dosemodule.cu:228-240)
        cp.mlc = np.asfortranarray(mlc)
    vol = phantoms.volume_object(grid, grid.DensityFromHU(plan.machine_name))
    return grid, model, cp, vol


def _oracle(model, cp, vol):
    import oracle
    sp = np.asarray(vol.spacing)[[0, 0, 0]]
    mlc = np.ascontiguousarray(cp.mlc)
    dose, terma, _, _ = oracle.photon_dose(vol.voxel_data, sp, vol.origin, model, cp.iso, cp.mu, cp.ga, cp.ca, cp.ta,
                                           mlc, intermediates=True)
    tp, _ = oracle.photon_transmission(vol.voxel_data.shape, sp, vol.origin, model, cp.iso, cp.ga, cp.ca, cp.ta, mlc)
    return dose, terma, tp


def _departing(model, cp, vol, o_terma):
    import oracle
    if not oracle.reference_terma_available():
        pytest.skip("reference TERMA harness oracle/_ref/libref_terma.so not present")
    _, r_terma, _ = oracle.reference_photon_terma(vol.voxel_data, float(vol.spacing[0]), vol.origin, model, cp.iso,
                                                  cp.mu, cp.ga, cp.ca, cp.ta, np.ascontiguousarray(cp.mlc))
    r = r_terma.astype(np.float64)
    return ~(np.abs(r - o_terma) <= TERMA_DEPART * float(o_terma.max())), r  # NaN departs too


def _unreached(depart, model, spacing):
    """Voxels farther than the CCCS's longest window (plus one voxel for the
    trilinear sample) from every departing TERMA voxel."""
    from scipy import ndimage
    reach_mm = 10.0 * float(np.max(np.asarray(model.kernel, np.float32)[:, 5])) + spacing
    r = int(np.ceil(reach_mm / spacing))
    z, y, x = np.mgrid[-r:r + 1, -r:r + 1, -r:r + 1]
    ball = (x * x + y * y + z * z) * spacing * spacing <= reach_mm * reach_mm
    return ~ndimage.binary_dilation(depart, structure=ball)


def _masked_parity(ref_dk, model, cp, vol, o_dose, depart):
    from dosecuda_b200 import dose_kernels as dk
    d_ref = ref_dk.photon_dose_cuda(model, vol, cp, 0)
    d = dk.photon_dose_cuda(model, vol, cp, 0)
    clean = _unreached(depart, model, float(vol.spacing[0]))
    dmax = float(o_dose.max())
    hi = o_dose > 0.1 * dmax
    frac = float(clean[hi].mean())
    dd = dose_diff(d, d_ref, where=clean, dmax=dmax)
    g = gamma_pass_rate(d, d_ref, float(vol.spacing[0]), where=clean, dmax=dmax)
    return frac, dd, g


def test_reference_terma_departs_only_where_primary_transmission_vanishes(ref_dk):
    grid, model, cp, vol = _workload("as_is")
    o_dose, o_terma, tp = _oracle(model, cp, vol)
    depart, r_terma = _departing(model, cp, vol, o_terma)
    xs = np.arange(vol.voxel_data.shape[2]) * float(vol.spacing[0]) + float(vol.origin[0]) - float(cp.iso[0])
    on_plane = np.broadcast_to(np.abs(xs) < 1e-3, depart.shape)
    print("\nTERMA voxels departing from the oracle: %d of %d (%.1f %% on the central plane); max |TERMA_ref| %.3g"
          " vs oracle max %.3g" % (int(depart.sum()), depart.size, 100.0 * float(on_plane[depart].mean()),
                                   float(np.nanmax(np.abs(r_terma))), float(o_terma.max())))
    assert depart.any(), "the reference's TERMA artifact is expected on this workload"
    assert float(np.abs(tp[depart]).max()) <= TP_ZERO
    frac, dd, g = _masked_parity(ref_dk, model, cp, vol, o_dose, depart)
    print("dose voxels above 10 %% Dmax out of the artifact's reach: %.4f; engine vs reference there: |dD| %.5f"
          " Dmax, gamma %.5f" % (frac, dd, g))
    assert frac > 0.5
    assert dd <= TOL
    assert g >= GAMMA


@pytest.mark.parametrize("variant", ["half_voxel", "parked_leaves"])
def test_variants_vs_reference_out_of_the_artifacts_reach(ref_dk, variant):
    grid, model, cp, vol = _workload(variant)
    o_dose, o_terma, tp = _oracle(model, cp, vol)
    depart, _ = _departing(model, cp, vol, o_terma)
    assert float(np.abs(tp[depart]).max(initial=0.0)) <= TP_ZERO
    frac, dd, g = _masked_parity(ref_dk, model, cp, vol, o_dose, depart)
    print("\n%s: departing TERMA voxels %d; dose voxels above 10 %% Dmax out of their reach %.4f; |dD| %.5f Dmax,"
          " gamma %.5f" % (variant, int(depart.sum()), frac, dd, g))
    assert dd <= TOL
    assert g >= GAMMA


def test_open_field_vs_reference_whole_volume(ref_dk):
    """Every leaf pair open over the phantom: the reference's TERMA has no
    ts^2/tp artifact anywhere, and the engine equals the reference on every
    voxel.  A handful of voxels may still sit off the FP64 oracle by one
    boundary sample of the ray trace (a sample on the volume's face that the
    float position test counts and the FP64 one does not, or the reverse:
    0.05 cm of WET at the face's half-blended density, ~0.25 % of TERMA);
    those are bounded here, not masked."""
    from dosecuda_b200 import dose_kernels as dk
    grid, model, cp, vol = _workload("open_field")
    o_dose, o_terma, tp = _oracle(model, cp, vol)
    depart, r_terma = _departing(model, cp, vol, o_terma)
    off = np.abs(r_terma - o_terma)
    print("\nopen field: TERMA voxels off the oracle by more than %.1g of max: %d, worst %.5f of max"
          % (TERMA_DEPART, int(depart.sum()), float(np.nanmax(off)) / float(o_terma.max())))
    assert int(depart.sum()) <= 1e-5 * depart.size, "the reference is not sound on this variant"
    assert float(np.nanmax(off)) <= 0.005 * float(o_terma.max())
    d_ref = ref_dk.photon_dose_cuda(model, vol, cp, 0)
    d = dk.photon_dose_cuda(model, vol, cp, 0)
    dd = dose_diff(d, d_ref)
    g = gamma_pass_rate(d, d_ref, float(vol.spacing[0]))
    print("\nopen field: engine vs reference |dD| %.5f of Dmax, gamma %.5f; reference vs oracle |dD| %.5f"
          % (dd, g, dose_diff(d_ref, o_dose)))
    assert dd <= TOL
    assert g >= GAMMA
    assert dose_diff(d, o_dose) <= TOL
