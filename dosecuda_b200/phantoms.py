"""Seeded synthetic phantoms and plans for the benchmark and test workloads.

* ``proton_small``  — 96^3 voxels at 2.0 mm, water (0 HU) with a bone
  cylinder (1000 HU, r = 12 mm, axis along y) and a 20 mm lung slab
  (-700 HU) at seeded offsets; one beam at gantry 0 / couch 0 with 6 energy
  layers of the default range-shifter-free model (energy ids 34..59,
  101-139 MeV) and a 10x10 spot grid (5 mm pitch) per layer, MU ~ U(0.5, 1.5).
* ``photon_small``  — 128^3 voxels at 2.5 mm, water with a 60x60x40 mm lung
  block (-750 HU) and a 20 mm bone cube (1200 HU) at seeded positions; one
  10x10 cm 6 MV open MLC field, 100 MU, gantry 0, isocentre at the centre.
Both accept smaller shapes for tests.  No external data is used.
"""
from __future__ import annotations

import numpy as np

from .plan_impt import IMPTBeam, IMPTDoseGrid, IMPTPlan
from .plan_imrt import IMRTDoseGrid, IMRTPlan

PROTON_SMALL_ENERGY_IDS = (34, 39, 44, 49, 54, 59)


def _grid_coords(shape, spacing):
    nz, ny, nx = shape
    z = (np.arange(nz) - (nz - 1) / 2.0) * spacing
    y = (np.arange(ny) - (ny - 1) / 2.0) * spacing
    x = (np.arange(nx) - (nx - 1) / 2.0) * spacing
    return np.meshgrid(z, y, x, indexing="ij")


def proton_phantom(shape=(96, 96, 96), spacing=2.0, seed=0) -> IMPTDoseGrid:
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    grid = IMPTDoseGrid()
    grid.origin = np.array([-nx * spacing / 2.0, -ny * spacing / 2.0, -nz * spacing / 2.0])
    grid.spacing = np.array([spacing, spacing, spacing])
    grid.size = np.array(shape)
    hu = np.zeros(shape, dtype=np.single)
    Z, Y, X = _grid_coords(shape, spacing)
    ext = np.array([nz, ny, nx]) * spacing
    # bone cylinder, axis along y
    cx, cz = rng.uniform(-0.25, 0.25, size=2) * ext[[2, 0]]
    hu[(X - cx) ** 2 + (Z - cz) ** 2 < 12.0 ** 2] = 1000.0
    # lung slab, 20 mm thick along y
    y0 = rng.uniform(-0.3, 0.1) * ext[1]
    hu[(Y >= y0) & (Y < y0 + 20.0)] = -700.0
    grid.HU = hu
    return grid


def proton_beam(energy_ids=PROTON_SMALL_ENERGY_IDS, field_mm=50.0, pitch_mm=5.0, gantry=0.0, couch=0.0,
                iso=(0.0, 0.0, 0.0), seed=0, rangeshifter="0") -> IMPTBeam:
    rng = np.random.default_rng(seed + 1000)
    n = int(round(field_mm / pitch_mm))
    pos = (np.arange(n) - (n - 1) / 2.0) * pitch_mm
    xs, ys = np.meshgrid(pos, pos, indexing="xy")
    rows = []
    for e in energy_ids:
        mu = rng.uniform(0.5, 1.5, size=xs.size)
        rows.append(np.column_stack((xs.ravel(), ys.ravel(), mu, np.full(xs.size, e))))
    beam = IMPTBeam()
    beam.spot_list = np.array(np.vstack(rows), dtype=np.single)
    beam.n_spots = beam.spot_list.shape[0]
    beam.gantry_angle = float(gantry)
    beam.couch_angle = float(couch)
    beam.iso = np.array(iso, dtype=np.single)
    beam.dicom_rangeshifter_label = rangeshifter
    return beam


def proton_small(seed=0, shape=(96, 96, 96), spacing=2.0, **beam_kw):
    """(IMPTDoseGrid, IMPTPlan) of the small proton pencil-beam workload."""
    grid = proton_phantom(shape, spacing, seed)
    plan = IMPTPlan()
    plan.addBeam(proton_beam(seed=seed, **beam_kw))
    return grid, plan


def photon_phantom(shape=(128, 128, 128), spacing=2.5, seed=0, lung_mm=(60.0, 60.0, 40.0),
                   bone_mm=20.0) -> IMRTDoseGrid:
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    grid = IMRTDoseGrid()
    grid.origin = np.array([-nx * spacing / 2.0, -ny * spacing / 2.0, -nz * spacing / 2.0])
    grid.spacing = np.array([spacing, spacing, spacing])
    grid.size = np.array(shape)
    hu = np.zeros(shape, dtype=np.single)
    Z, Y, X = _grid_coords(shape, spacing)
    ext = np.array([nx, ny, nz]) * spacing
    lx, ly, lz = lung_mm
    c = rng.uniform(-0.2, 0.2, size=3) * ext
    hu[(np.abs(X - c[0]) < lx / 2) & (np.abs(Y - c[1]) < ly / 2) & (np.abs(Z - c[2]) < lz / 2)] = -750.0
    c = rng.uniform(-0.2, 0.2, size=3) * ext
    hu[(np.abs(X - c[0]) < bone_mm / 2) & (np.abs(Y - c[1]) < bone_mm / 2) & (np.abs(Z - c[2]) < bone_mm / 2)] = 1200.0
    grid.HU = hu
    return grid


def photon_small(seed=0, shape=(128, 128, 128), spacing=2.5, field_cm=(10.0, 10.0), mu=100.0, gantry=0.0,
                 collimator=0.0, couch=0.0, **phantom_kw):
    """(IMRTDoseGrid, IMRTPlan) of the small photon CCCS workload."""
    grid = photon_phantom(shape, spacing, seed, **phantom_kw)
    plan = IMRTPlan("VarianTrueBeamHF")
    plan.addSquareField("6", field_cm[0], field_cm[1], mu=mu, gantry_angle=gantry, collimator_angle=collimator,
                        table_angle=couch)
    return grid, plan


def volume_object(grid, data):
    from .plan import VolumeObject
    v = VolumeObject()
    v.voxel_data = np.array(data, dtype=np.single)
    v.origin = np.array(grid.origin, dtype=np.single)
    v.spacing = np.array(grid.spacing, dtype=np.single)
    return v
