"""Device-resident interface of the dose engines.

Inputs and outputs are torch CUDA tensors (float32, C-contiguous, shape
(nz, ny, nx)); work is enqueued on the current torch stream of the tensor's
device (or the stream given) and the call returns without synchronising.
torch is used for device memory and streams only; the compute is
libdosecuda.so.

    wet  = engine.proton_wet(rlsp, grid, beam, model)
    dose = engine.proton_dose(wet, grid, beam, engine.ProtonModelDevice(model))
    dose = engine.photon_dose(density, grid, model, cp)

``grid`` is any object with ``spacing`` and ``origin`` (e.g. a DoseGrid).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .dose_kernels import ControlPointView, PhotonModelView


def _check_volume(t: torch.Tensor, name: str):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.dim() == 3):
        raise ValueError("'%s' must be a 3-dimensional float32 CUDA tensor." % name)
    if not t.is_contiguous():
        raise ValueError("'%s' must be C-contiguous." % name)


def _stream(t: torch.Tensor, stream):
    s = stream if stream is not None else torch.cuda.current_stream(t.device)
    return C.c_void_p(s.cuda_stream)


def _spacing(grid):
    sp = np.asarray(grid.spacing, dtype=np.float32)
    return _lib.f3((sp[0], sp[0], sp[0])) if sp.size == 1 else _lib.f3(sp)


def _out(like: torch.Tensor, out):
    if out is None:
        return torch.empty_like(like)
    _check_volume(out, "out")
    if out.shape != like.shape or out.device != like.device:
        raise ValueError("'out' must match the input volume's shape and device.")
    return out


def proton_wet(rlsp: torch.Tensor, grid, beam, model, out=None, stream=None) -> torch.Tensor:
    """Smoothed WET (cm) of every voxel for one proton beam."""
    _check_volume(rlsp, "rlsp")
    out = _out(rlsp, out)
    nz, ny, nx = rlsp.shape
    rc = _lib.load().dc_proton_raytrace_dev(
        rlsp.device.index, C.c_void_p(rlsp.data_ptr()), nz, ny, nx, _spacing(grid), _lib.f3(grid.origin),
        _lib.f3(beam.iso), float(beam.gantry_angle), float(beam.couch_angle), float(model.VSADX),
        float(model.VSADY), C.c_void_p(out.data_ptr()), _stream(rlsp, stream))
    _lib.raise_for(rc)
    return out


class ProtonModelDevice:
    """A proton beam model with its depth-dose tables resident on a device."""

    def __init__(self, model, device="cuda"):
        self.model = model
        self.VSADX = float(model.VSADX)
        self.VSADY = float(model.VSADY)
        self.divergence_params = np.ascontiguousarray(model.divergence_params, dtype=np.float32)
        self.lut_depths = torch.as_tensor(np.ascontiguousarray(model.lut_depths), device=device)
        self.lut_sigmas = torch.as_tensor(np.ascontiguousarray(model.lut_sigmas), device=device)
        self.lut_idds = torch.as_tensor(np.ascontiguousarray(model.lut_idds), device=device)
        self.n_energies, self.lut_len = self.lut_depths.shape


def proton_dose(wet: torch.Tensor, grid, beam, dmodel: ProtonModelDevice, out=None, stream=None,
                spots=None) -> torch.Tensor:
    """Pencil-beam dose of ``beam.spot_list`` (or ``spots``) from a smoothed WET."""
    _check_volume(wet, "wet")
    out = _out(wet, out)
    sp = np.ascontiguousarray(beam.spot_list if spots is None else spots, dtype=np.float32).reshape(-1, 4)
    nz, ny, nx = wet.shape
    rc = _lib.load().dc_proton_spot_dev(
        wet.device.index, C.c_void_p(wet.data_ptr()), nz, ny, nx, _spacing(grid), _lib.f3(grid.origin),
        _lib.f3(beam.iso), float(beam.gantry_angle), float(beam.couch_angle), dmodel.VSADX, dmodel.VSADY,
        dmodel.divergence_params.ctypes.data_as(C.c_void_p),
        dmodel.n_energies, dmodel.divergence_params.shape[1], C.c_void_p(dmodel.lut_depths.data_ptr()),
        C.c_void_p(dmodel.lut_sigmas.data_ptr()), C.c_void_p(dmodel.lut_idds.data_ptr()), dmodel.lut_len,
        sp.ctypes.data_as(C.c_void_p), sp.shape[0], C.c_void_p(out.data_ptr()), _stream(wet, stream))
    _lib.raise_for(rc)
    return out


def photon_dose(density: torch.Tensor, grid, model, cp, out=None, stream=None, views=None) -> torch.Tensor:
    """Collapsed-cone dose of one control point (before the output factor).
    ``views`` = (PhotonModelView, ControlPointView) may be passed to reuse the
    packed parameter blocks across calls."""
    _check_volume(density, "density")
    out = _out(density, out)
    mv, cv = views if views is not None else (PhotonModelView(model), ControlPointView(cp))
    nz, ny, nx = density.shape
    rc = _lib.load().dc_photon_dose_dev(
        density.device.index, C.c_void_p(density.data_ptr()), nz, ny, nx, _spacing(grid), _lib.f3(grid.origin),
        C.byref(mv.struct), C.byref(cv.struct), C.c_void_p(out.data_ptr()), _stream(density, stream))
    _lib.raise_for(rc)
    return out


def profile(gpu_id: int = 0, enable: bool | None = None, reset: bool = False):
    """Kernel timing control: enable/disable/reset, and read {kernel: (launches, ms)}."""
    lib = _lib.load()
    if enable is not None:
        _lib.raise_for(lib.dc_profile_enable(gpu_id, int(enable)))
    if reset:
        _lib.raise_for(lib.dc_profile_reset(gpu_id))
    return _lib.profile_read(gpu_id)
