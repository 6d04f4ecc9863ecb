"""Host-buffer entry points with page-locked buffers: the kernels read the
WET and write results in place in mapped host memory instead of copying
(dc_host_buffer_mapped).  Both routes must give the same bits, and the
mapping test must accept only a page-locked range inside one allocation."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _mapped(ptr, nbytes):
    from dosecuda_b200 import _lib
    flag = C.c_int(-1)
    _lib.raise_for(_lib.load().dc_host_buffer_mapped(0, C.c_void_p(ptr), nbytes, C.byref(flag)))
    return flag.value


def test_mapping_query():
    pinned = torch.empty(1 << 20, dtype=torch.float32, pin_memory=True)
    pageable = np.empty(1 << 20, dtype=np.float32)
    assert _mapped(pinned.data_ptr(), pinned.numel() * 4) == 1
    assert _mapped(pinned.data_ptr() + 4096, 4096) == 1
    assert _mapped(pinned.data_ptr(), 1 << 40) == 0  # beyond the allocation
    assert _mapped(pageable.ctypes.data, pageable.nbytes) == 0
    assert _mapped(0, 16) == 0


@pytest.fixture
def both_routes(monkeypatch):
    """Runs a dose_kernels call once with page-locked outputs (mapped route)
    and once with ordinary numpy outputs (copy route)."""
    from dosecuda_b200 import dose_kernels

    def run(fn):
        monkeypatch.setattr(dose_kernels, "_PINNED_OK", None)
        a = fn()
        monkeypatch.setattr(dose_kernels, "_PINNED_OK", False)
        b = fn()
        monkeypatch.setattr(dose_kernels, "_PINNED_OK", None)
        return a, b
    return run


def test_photon_mapped_output_equals_copy(both_routes):
    from dosecuda_b200 import dose_kernels, phantoms
    grid, plan = phantoms.photon_small(shape=(64, 64, 64), spacing=3.0, field_cm=(6.0, 8.0), gantry=20.0)
    model, cp = plan.beam_models[0], plan.beam_list[0].cp_list[0]
    vol = phantoms.volume_object(grid, grid.DensityFromHU(plan.machine_name))
    a, b = both_routes(lambda: dose_kernels.photon_dose_cuda(model, vol, cp, 0))
    assert _mapped(a.ctypes.data, a.nbytes) == 1 and _mapped(b.ctypes.data, b.nbytes) == 0
    assert np.array_equal(a, b) and a.max() > 0


def test_proton_mapped_io_equals_copy(both_routes):
    from dosecuda_b200 import dose_kernels, phantoms
    from dosecuda_b200.plan import VolumeObject
    grid, plan = phantoms.proton_small(shape=(48, 40, 56), spacing=2.5, seed=4)
    model, beam = plan.beam_models[0], plan.beam_list[0]
    vol = phantoms.volume_object(grid, grid.RLSPFromHU(plan.machine_name))
    wa, wb = both_routes(lambda: dose_kernels.proton_raytrace_cuda(model, vol, beam, 0))
    assert np.array_equal(wa, wb) and wa.max() > 0

    def spot(w):
        v = VolumeObject()
        v.voxel_data, v.origin, v.spacing = w, vol.origin, vol.spacing
        return lambda: dose_kernels.proton_spot_cuda(model, vol, v, beam, 0)
    # page-locked WET input (read in place) and pageable WET input (copied)
    da, db = both_routes(spot(wa))
    dc, dd = both_routes(spot(np.array(wa)))
    assert _mapped(wa.ctypes.data, wa.nbytes) == 1
    assert np.array_equal(da, db) and np.array_equal(da, dc) and np.array_equal(da, dd) and da.max() > 0


@pytest.mark.parametrize("shape", [(128, 128, 128), (37, 200, 190), (5, 9, 7)])
def test_pageable_input_pipelined_upload_equals_pinned(shape):
    """A pageable input volume goes through the pinned slab ring (host copy
    threads + DMA per slab; a 128^3 volume wraps the three-slab ring, a
    37 x 200 x 190 one ends on a partial slab); a page-locked one is copied
    directly.  The photon dose must be the same bits either way."""
    from dosecuda_b200 import dose_kernels, phantoms
    grid, plan = phantoms.photon_small(shape=shape, spacing=2.5, field_cm=(6.0, 6.0), lung_mm=(8.0, 8.0, 6.0),
                                       bone_mm=5.0, seed=2)
    model, cp = plan.beam_models[0], plan.beam_list[0].cp_list[0]
    dens = np.ascontiguousarray(grid.DensityFromHU(plan.machine_name))
    pinned = torch.from_numpy(dens).pin_memory()
    assert _mapped(dens.ctypes.data, dens.nbytes) == 0 and _mapped(pinned.data_ptr(), dens.nbytes) == 1
    a = dose_kernels.photon_dose_cuda(model, phantoms.volume_object(grid, dens), cp, 0)
    vol_p = phantoms.volume_object(grid, dens)
    vol_p.voxel_data = pinned.numpy()
    b = dose_kernels.photon_dose_cuda(model, vol_p, cp, 0)
    assert np.array_equal(a, b) and a.max() > 0
