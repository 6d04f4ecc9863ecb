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
                   bone_mm=20.0, body_mm=None) -> IMRTDoseGrid:
    """Water with a lung block and a bone cube at seeded offsets; with
    ``body_mm`` = (a, b, c) semi-axes (x, y, z), the water is an ellipsoidal
    body centred in the volume and everything outside it is air (-1000 HU)."""
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
    if body_mm is not None:
        a, b, cz = body_mm
        hu[(X / a) ** 2 + (Y / b) ** 2 + (Z / cz) ** 2 > 1.0] = -1000.0
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


# ---------------------------------------------------------------------------
# Batched IMPT workload: patient-like phantoms with a spherical target
# ---------------------------------------------------------------------------
def _axis_wet_profile(rlsp, spacing, origin, src, iso, step_mm=1.0):
    """WET (mm) along the line from the source through the isocentre, as a
    function of distance from the source (nearest-voxel samples)."""
    nz, ny, nx = rlsp.shape
    sp = np.asarray(spacing, np.float64)
    d = np.asarray(iso, np.float64) - np.asarray(src, np.float64)
    L = np.linalg.norm(d)
    u = d / L
    t = np.arange(0.0, L + 400.0, step_mm)
    pts = np.asarray(src, np.float64)[None, :] + t[:, None] * u[None, :]
    ijk = np.rint((pts - np.asarray(origin, np.float64)[None, :]) / sp[None, :]).astype(np.int64)
    inside = (ijk[:, 0] >= 0) & (ijk[:, 0] < nx) & (ijk[:, 1] >= 0) & (ijk[:, 1] < ny) & (ijk[:, 2] >= 0) & \
             (ijk[:, 2] < nz)
    rho = np.zeros(len(t))
    rho[inside] = rlsp[ijk[inside, 2], ijk[inside, 1], ijk[inside, 0]]
    return t, np.cumsum(np.maximum(rho, 0.0)) * step_mm


def batch_plan(seed=0, shape=(160, 256, 256), spacing=(1.5, 1.5, 2.0), model=None, pitch_range=(4.0, 6.0),
               max_beams=3, max_spots=12000, n_beams=None):
    """(IMPTDoseGrid, [IMPTBeam], target (centre, radius)) of one plan of the
    batched workload: a water-equivalent body ellipsoid (20 +- 40 HU) with 1-6
    random bone/lung/air ellipsoids (1000, -750, -1000 HU; semi-axes 5-40 mm)
    and a spherical target (r 20-45 mm); 1-3 beams at uniform gantry angles;
    energy layers covering the target at 3 mm R80 spacing; spots on a 4-6 mm
    grid over the target's projection; weights lognormal(0, 0.5)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    sx, sy, sz = spacing
    grid = IMPTDoseGrid()
    grid.origin = np.array([-nx * sx / 2.0, -ny * sy / 2.0, -nz * sz / 2.0])
    grid.spacing = np.array([sx, sy, sz])
    grid.size = np.array(shape)
    z = ((np.arange(nz) + 0.5) * sz + grid.origin[2]).astype(np.float32)
    y = ((np.arange(ny) + 0.5) * sy + grid.origin[1]).astype(np.float32)
    x = ((np.arange(nx) + 0.5) * sx + grid.origin[0]).astype(np.float32)
    ext = np.array([nx * sx, ny * sy, nz * sz]) / 2.0
    body_ax = ext * rng.uniform(0.78, 0.92, size=3)
    body = ((x / body_ax[0]) ** 2)[None, None, :] + ((y / body_ax[1]) ** 2)[None, :, None] + \
           ((z / body_ax[2]) ** 2)[:, None, None] <= 1.0
    hu = np.full(shape, -1000.0, np.float32)
    hu[body] = 20.0 + 40.0 * rng.standard_normal(int(body.sum()), dtype=np.float32)

    def ellipsoid(c, a):
        """(slices, mask) of an axis-aligned ellipsoid within its bounding box."""
        sl, axes = [], []
        for coords, cc, aa in ((z, c[2], a[2]), (y, c[1], a[1]), (x, c[0], a[0])):
            lo = int(np.searchsorted(coords, cc - aa))
            hi = int(np.searchsorted(coords, cc + aa, side="right"))
            sl.append(slice(lo, max(lo, hi)))
            axes.append(((coords[lo:max(lo, hi)] - cc) / aa) ** 2)
        m = axes[0][:, None, None] + axes[1][None, :, None] + axes[2][None, None, :] <= 1.0
        return tuple(sl), m

    for _ in range(int(rng.integers(1, 7))):
        c = rng.uniform(-0.5, 0.5, size=3) * body_ax
        a = rng.uniform(5.0, 40.0, size=3)
        val = float(rng.choice([1000.0, -750.0, -1000.0]))
        sl, m = ellipsoid(c, a)
        sub = hu[sl]
        sub[m & body[sl]] = val
    r_t = float(rng.uniform(20.0, 45.0))
    c_t = rng.uniform(-0.25, 0.25, size=3) * np.maximum(body_ax - r_t - 10.0, 0.0)
    sl, m = ellipsoid(c_t, np.array([r_t, r_t, r_t]))
    sub = hu[sl]
    sub[m] = 20.0 + 40.0 * rng.standard_normal(int(m.sum()), dtype=np.float32)
    grid.HU = hu

    if model is None:
        model = IMPTPlan().beam_models[0]
    rlsp = grid.RLSPFromHU("HitachiProbeatJHU")
    r80 = np.asarray(model.divergence_params[:, 1], np.float64)
    sad = (float(model.VSADX) + float(model.VSADY)) / 2.0
    beams = []
    total = 0
    nb = int(rng.integers(1, max_beams + 1)) if n_beams is None else int(n_beams)
    for _ in range(nb):
        ga = float(rng.uniform(0.0, 360.0))
        # source position for gantry ga (+180 inside the engine), couch 0
        g = np.deg2rad(np.float32((ga + 180.0) % 360.0))
        src = c_t + np.array([-sad * np.sin(g), sad * np.cos(g), 0.0])
        t, wet = _axis_wet_profile(rlsp, grid.spacing, grid.origin, src, c_t)
        dist = np.linalg.norm(c_t - src)
        w_prox = float(np.interp(dist - r_t, t, wet))
        w_dist = float(np.interp(dist + r_t, t, wet))
        ids = []
        for w in np.arange(w_prox, w_dist + 3.0, 3.0):
            e = int(np.argmin(np.abs(r80 - w)))
            if e not in ids:
                ids.append(e)
        pitch = float(rng.uniform(*pitch_range))
        n = int(np.ceil((r_t + 5.0) / pitch))
        pos = np.arange(-n, n + 1) * pitch
        gx, gy = np.meshgrid(pos, pos, indexing="xy")
        keep = gx ** 2 + gy ** 2 <= (r_t + 5.0) ** 2
        gx, gy = gx[keep], gy[keep]
        rows = []
        for e in ids:
            mu = rng.lognormal(0.0, 0.5, size=gx.size)
            rows.append(np.column_stack((gx, gy, mu, np.full(gx.size, e))))
        spots = np.array(np.vstack(rows), dtype=np.single)
        if beams and n_beams is None and total + spots.shape[0] > max_spots:
            break  # keep the plan within its spot budget
        total += spots.shape[0]
        beam = IMPTBeam()
        beam.spot_list = spots
        beam.n_spots = beam.spot_list.shape[0]
        beam.gantry_angle = ga
        beam.couch_angle = 0.0
        beam.iso = np.array(c_t, dtype=np.single)
        beam.dicom_rangeshifter_label = "0"
        beams.append(beam)
    return grid, beams, (c_t, r_t)
