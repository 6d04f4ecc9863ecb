"""Generate the golden fixtures of this directory by running the REFERENCE
DoseCUDA CUDA extension (built from the reference sources by
oracle/build_ref.sh into oracle/_ref/) on small seeded cases.

Needs a CUDA GPU.  Usage (from the repository root):

    python tests/golden/make_golden.py [--out tests/golden]

Each case is written to ``<name>.npz`` with the inputs the dose call saw
(RLSP or density volume, grid, beam geometry, spot list or MLC, beam-model
selection) and the reference's outputs (smoothed WET in cm and/or dose).
The fixtures pin the CPU oracle (tests/test_oracle_golden.py) and the GPU
engine (tests/test_gpu_parity.py).
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dosecuda_b200 import phantoms  # noqa: E402
from dosecuda_b200.plan import VolumeObject  # noqa: E402
from dosecuda_b200.plan_impt import IMPTBeam, IMPTPlan  # noqa: E402
from dosecuda_b200.plan_imrt import IMRTControlPoint, IMRTPlan, _mlc_array  # noqa: E402


def load_reference():
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if not glob.glob(os.path.join(ref_dir, "dose_kernels*.so")):
        raise SystemExit("reference extension missing: run oracle/build_ref.sh first")
    sys.path.insert(0, ref_dir)
    import dose_kernels  # the reference build
    return dose_kernels


def vol(data, spacing, origin):
    v = VolumeObject()
    v.voxel_data = np.ascontiguousarray(data, dtype=np.single)
    v.spacing = np.array(spacing, dtype=np.single)
    v.origin = np.array(origin, dtype=np.single)
    return v


PROTON_CASES = [
    # name, shape (nz,ny,nx), spacing, seed, rs label, energy ids, pitch, n per side, gantry, couch, iso
    ("p_g0", (32, 36, 40), 3.0, 11, "0", (5, 15, 25), 6.0, 4, 0.0, 0.0, (0.0, 0.0, 0.0)),
    ("p_g90", (32, 36, 40), 3.0, 12, "0", (10, 20), 5.0, 5, 90.0, 0.0, (5.0, -3.0, 2.0)),
    ("p_obl_rs4", (30, 34, 38), 3.0, 13, "4", (24, 40, 60), 7.0, 3, 235.0, 30.0, (-6.0, 4.0, 3.0)),
]

PHOTON_CASES = [
    # name, shape, spacing, seed, field (x,y) cm, mu, gantry, collimator, couch, irregular MLC seed, iso
    # Fields whose leaf pairs under the phantom are all open, isocentres off the voxel lattice.
    ("x_open_g0", (36, 40, 44), 3.0, 21, (6.0, 13.0), 100.0, 0.0, 0.0, 0.0, None, (1.3, 0.7, -1.1)),
    ("x_g90_c20", (36, 40, 44), 3.0, 22, (8.0, 16.0), 80.0, 90.0, 20.0, 0.0, None, (0.9, -1.3, 1.7)),
    ("x_obl_mlc", (34, 38, 42), 3.0, 23, (7.0, 16.0), 120.0, 300.0, 0.0, 15.0, 5, (-1.6, 0.4, 0.8)),
    # A 6x6 cm field with closed leaf pairs over the phantom and the isocentre on a
    # voxel centre: the reference's TERMA kernel produces its transmission-ratio
    # artifact here (kept as an exhibit, see tests/test_oracle_golden.py).
    ("x_g0_closed", (36, 40, 44), 3.0, 21, (6.0, 6.0), 100.0, 0.0, 0.0, 0.0, None, (0.0, 0.0, 0.0)),
]


def proton_case(dk, name, shape, spacing, seed, rs, eids, pitch, nside, gantry, couch, iso):
    grid = phantoms.proton_phantom(shape, spacing, seed)
    plan = IMPTPlan()
    labels = list(plan.dicom_rangeshifter_label.astype(str))
    model = plan.beam_models[labels.index(rs)]
    beam = phantoms.proton_beam(energy_ids=eids, field_mm=pitch * nside, pitch_mm=pitch, gantry=gantry,
                                couch=couch, iso=iso, seed=seed, rangeshifter=rs)
    rlsp = grid.RLSPFromHU(plan.machine_name)
    rv = vol(rlsp, grid.spacing, grid.origin)
    wet = dk.proton_raytrace_cuda(model, rv, beam, 0)
    dose = dk.proton_spot_cuda(model, rv, vol(wet, grid.spacing, grid.origin), beam, 0)
    meta = dict(kind="proton", machine=plan.machine_name, rangeshifter=rs, gantry=gantry, couch=couch)
    return meta, dict(rlsp=rlsp, spacing=rv.spacing, origin=rv.origin, iso=beam.iso, spots=beam.spot_list,
                      wet=wet, dose=dose)


def photon_case(dk, name, shape, spacing, seed, field, mu, gantry, coll, couch, mlc_seed, iso):
    grid = phantoms.photon_phantom(shape, spacing, seed, lung_mm=(30.0, 30.0, 24.0), bone_mm=12.0)
    plan = IMRTPlan("VarianTrueBeamHF")
    plan.addSquareField("6", field[0], field[1], mu=mu, gantry_angle=gantry, collimator_angle=coll,
                        table_angle=couch)
    cp = plan.beam_list[0].cp_list[0]
    model = plan.beam_models[0]
    mlc = cp.mlc
    if mlc_seed is not None:
        rng = np.random.default_rng(mlc_seed)
        x12 = np.zeros((2, model.n_mlc_pairs), dtype=np.single)
        half = field[1] * 10.0 / 2.0
        open_ = np.abs(model.mlc_offsets) < half
        x12[0, open_] = rng.uniform(-45.0, -5.0, size=open_.sum())
        x12[1, open_] = rng.uniform(5.0, 45.0, size=open_.sum())
        mlc = _mlc_array(x12, model.mlc_offsets, model.mlc_widths)
    cp = IMRTControlPoint(np.array(iso, dtype=np.single), mu, mlc, gantry, coll, couch, cp.xjaws, cp.yjaws)
    density = grid.DensityFromHU(plan.machine_name)
    dv = vol(density, grid.spacing, grid.origin)
    dose = dk.photon_dose_cuda(model, dv, cp, 0)
    meta = dict(kind="photon", machine=plan.machine_name, energy="6", mu=float(mu), gantry=gantry,
                collimator=coll, couch=couch)
    return meta, dict(density=density, spacing=dv.spacing, origin=dv.origin, iso=np.asarray(cp.iso, np.single),
                      mlc=np.ascontiguousarray(cp.mlc), dose=dose)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    dk = load_reference()
    os.makedirs(args.out, exist_ok=True)
    for c in PROTON_CASES:
        meta, arrs = proton_case(dk, *c)
        np.savez_compressed(os.path.join(args.out, c[0] + ".npz"), meta=json.dumps(meta), **arrs)
        print(c[0], "wet max %.4f dose max %.5g" % (arrs["wet"].max(), arrs["dose"].max()))
    for c in PHOTON_CASES:
        meta, arrs = photon_case(dk, *c)
        np.savez_compressed(os.path.join(args.out, c[0] + ".npz"), meta=json.dumps(meta), **arrs)
        print(c[0], "dose max %.5g" % arrs["dose"].max())


if __name__ == "__main__":
    main()
