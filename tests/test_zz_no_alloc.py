"""dc_proton_raytrace_noalloc: the WET ray trace for callers that cannot let
the library allocate device memory (host applications that own every device
buffer, fixed device-memory budgets, loops that cannot afford cudaMalloc's
implicit synchronisation).  It is called here through the C ABI on
caller-owned device buffers and checked against the existing entry point,
dc_proton_raytrace_dev, on two calls in a row.

This file sorts last so that a run stopping at its first failure has already
run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from dosecuda_b200 import _lib, phantoms

pytestmark = pytest.mark.gpu


def _texture_path_wet(lib, t, grid, beam, model, stream):
    import torch
    out = torch.empty_like(t)
    nz, ny, nx = t.shape
    rc = lib.dc_proton_raytrace_dev(0, C.c_void_p(t.data_ptr()), nz, ny, nx, _lib.f3(grid.spacing),
                                    _lib.f3(grid.origin), _lib.f3(beam.iso), float(beam.gantry_angle),
                                    float(beam.couch_angle), float(model.VSADX), float(model.VSADY),
                                    C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
    _lib.raise_for(rc)
    return out


def _noalloc_wet(lib, t, grid, beam, model, stream, out):
    nz, ny, nx = t.shape
    return lib.dc_proton_raytrace_noalloc(0, C.c_void_p(t.data_ptr()), nz, ny, nx, _lib.f3(grid.spacing),
                                          _lib.f3(grid.origin), _lib.f3(beam.iso), float(beam.gantry_angle),
                                          float(beam.couch_angle), float(model.VSADX), float(model.VSADY),
                                          C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))


def _close(a, b):
    # the WET tolerance the oracle is held to against the reference fixtures
    from dosecheck import wet_close
    return wet_close(a, b)


def test_noalloc_matches_existing_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib.load()
    grid, plan = phantoms.proton_small(shape=(40, 44, 48), spacing=3.0, energy_ids=(10,), field_mm=20.0)
    model = plan.beam_models[0]
    beam_a = plan.beam_list[0]
    from dosecuda_b200.plan_impt import IMPTBeam
    beam_b = IMPTBeam(beam_a)
    beam_b.gantry_angle, beam_b.couch_angle = 235.0, 20.0
    beam_b.iso = np.array([4.0, -3.0, 2.5], np.float32)
    t = torch.from_numpy(grid.RLSPFromHU(plan.machine_name)).cuda()
    stream = torch.cuda.current_stream()
    ref_a = _texture_path_wet(lib, t, grid, beam_a, model, stream)
    ref_b = _texture_path_wet(lib, t, grid, beam_b, model, stream)
    # caller-owned outputs; the entry point itself allocates nothing
    out_a = torch.full_like(t, -1.0)
    out_b = torch.full_like(t, -1.0)
    assert _noalloc_wet(lib, t, grid, beam_a, model, stream, out_a) == _lib.DC_OK
    assert _noalloc_wet(lib, t, grid, beam_b, model, stream, out_b) == _lib.DC_OK
    torch.cuda.synchronize()
    assert _close(out_a.cpu().numpy(), ref_a.cpu().numpy())
    assert _close(out_b.cpu().numpy(), ref_b.cpu().numpy())
    # the shared scratch keeps the previous call's contents; a repeat of the
    # first call must not see them
    out_a2 = torch.full_like(t, -1.0)
    # after the first call (which commits the scratch) further calls leave
    # the device's free memory and torch's pool untouched, and the calling
    # thread's current device as it was
    torch.cuda.synchronize()
    free0, reserved0, dev0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved(), torch.cuda.current_device()
    assert _noalloc_wet(lib, t, grid, beam_a, model, stream, out_a2) == _lib.DC_OK
    assert _noalloc_wet(lib, t, grid, beam_b, model, stream, out_b) == _lib.DC_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_reserved() == reserved0
    assert torch.cuda.current_device() == dev0
    assert torch.equal(out_a2, out_a)
    assert _close(out_b.cpu().numpy(), ref_b.cpu().numpy())


def test_noalloc_rejects_volumes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib.load()
    shape = (130, 180, 180)  # 4,212,000 voxels > 4,194,304
    t = torch.zeros(shape, dtype=torch.float32, device="cuda")
    out = torch.zeros_like(t)
    grid, plan = phantoms.proton_small(shape=(4, 4, 4))
    rc = _noalloc_wet(lib, t, grid, plan.beam_list[0], plan.beam_models[0], torch.cuda.current_stream(), out)
    assert rc == _lib.DC_ERR_VALUE
    assert "scratch limit" in lib.dc_last_error().decode()
