"""Drop-in replacement of the reference's ``dose_kernels`` CPython extension.

Same three functions, same positional arguments, same attribute names read
from the duck-typed argument objects, same return value (a new float32
ndarray shaped like the input volume) and the same exception classes as
DoseCUDA/dose_kernels/dosemodule.cu:

* ``proton_raytrace_cuda(model, volume, beam, gpu_id)``      (dosemodule.cu:104-201)
* ``proton_spot_cuda(model, volume, wet, beam, gpu_id)``     (dosemodule.cu:243-374)
* ``photon_dose_cuda(model, volume, cp, gpu_id)``            (dosemodule.cu:377-557)

Argument checks follow ``pyobject_getarray`` (dosemodule.cu:50-66): an
attribute that is not an ndarray of the stated rank and dtype float32 raises
``ValueError("'<name>' must be <N>-dimensional and of type float.")``; a
missing attribute raises ``AttributeError``; ``gpu_id`` must be an integer.
Differences, all on inputs the reference mishandles:
* arrays are read by their logical layout (``np.ascontiguousarray``), where
  the reference reads the raw buffer; for the reference's own callers (the
  Fortran-ordered ``kernel`` and ``mlc`` arrays, dosemodule.cu:228-240,
  IMRTClasses.cu:292-297) both read the same numbers;
* ``spot_list`` must have 4 columns and every energy id must index the beam
  model (the reference silently drops or zeroes such spots);
* the LUT length is the arrays' second dimension (the reference hard-codes
  400, dosemodule.cu:349, which is what the shipped tables hold).

The compute runs in libdosecuda.so (hand-written sm_100a kernels); there is
no CPU path.
"""
from __future__ import annotations

import ctypes as C
import operator

import numpy as np

from . import _lib

_PINNED_OK = None


def _output(shape):
    """The new float32 array a call returns.  Backed by page-locked host
    memory when CUDA is usable (torch's caching pinned-host allocator), so the
    device-to-host copy of the result runs at full DMA speed instead of
    through the driver's staged pageable path; an ordinary numpy array to the
    caller either way."""
    global _PINNED_OK
    if _PINNED_OK is not False:
        try:
            import torch
            t = torch.empty(tuple(int(s) for s in shape), dtype=torch.float32, pin_memory=True)
            _PINNED_OK = True
            return t.numpy()
        except Exception:
            _PINNED_OK = False
    return np.empty(shape, dtype=np.float32)

__all__ = ["proton_raytrace_cuda", "proton_spot_cuda", "photon_dose_cuda"]


def _getarray(obj, attr: str, ndim: int) -> np.ndarray:
    a = getattr(obj, attr)
    if not (isinstance(a, np.ndarray) and a.ndim == ndim and a.dtype == np.float32):
        raise ValueError("'%s' must be %d-dimensional and of type float." % (attr, ndim))
    return a


def _getfloat(obj, attr: str) -> float:
    v = getattr(obj, attr)
    try:
        return float(v)
    except (TypeError, ValueError) as e:
        raise TypeError("must be real number, not %s" % type(v).__name__) from e


def _getbool(obj, attr: str) -> bool:
    return bool(getattr(obj, attr))


def _vec3(a: np.ndarray, attr: str, n: int = 3) -> np.ndarray:
    if a.shape[0] < n:
        raise ValueError("'%s' must hold at least %d values." % (attr, n))
    return np.ascontiguousarray(a[:n], dtype=np.float32)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _volume(volume):
    vox = _getarray(volume, "voxel_data", 3)
    spacing = _getarray(volume, "spacing", 1)
    origin = _getarray(volume, "origin", 1)
    return vox, spacing, origin


def proton_raytrace_cuda(model, volume, beam, gpu_id):
    """Smoothed water-equivalent thickness (cm) of every voxel along the ray to
    the proton source (reference: rayTraceKernel + smoothRayKernel)."""
    gpu_id = operator.index(gpu_id)
    vsadx = _getfloat(model, "VSADX")
    vsady = _getfloat(model, "VSADY")
    vox, spacing, origin = _volume(volume)
    iso = _getarray(beam, "iso", 1)
    ga = _getfloat(beam, "gantry_angle")
    ta = _getfloat(beam, "couch_angle")

    vox_c = np.ascontiguousarray(vox)
    sp = _vec3(spacing, "spacing", 1)
    out = _output(vox.shape)
    nz, ny, nx = vox.shape
    lib = _lib.load()
    rc = lib.dc_proton_raytrace(gpu_id, _ptr(vox_c), nz, ny, nx, _lib.f3((sp[0],) * 3),
                                _lib.f3(_vec3(origin, "origin")), _lib.f3(_vec3(iso, "iso")), ga, ta, vsadx,
                                vsady, _ptr(out))
    _lib.raise_for(rc)
    return out


def proton_spot_cuda(model, volume, wet, beam, gpu_id):
    """Double-Gaussian pencil-beam dose of every spot in ``beam.spot_list``
    given the smoothed WET (reference: pencilBeamKernel)."""
    gpu_id = operator.index(gpu_id)
    vsadx = _getfloat(model, "VSADX")
    vsady = _getfloat(model, "VSADY")
    dvp = _getarray(model, "divergence_params", 2)
    lut_d = _getarray(model, "lut_depths", 2)
    lut_s = _getarray(model, "lut_sigmas", 2)
    lut_i = _getarray(model, "lut_idds", 2)
    vox, spacing, origin = _volume(volume)
    wet_v = _getarray(wet, "voxel_data", 3)
    iso = _getarray(beam, "iso", 1)
    spots = _getarray(beam, "spot_list", 2)
    ga = _getfloat(beam, "gantry_angle")
    ta = _getfloat(beam, "couch_angle")

    if spots.shape[1] != 4:
        raise ValueError("'spot_list' must have 4 columns (x, y, MU, energy id).")
    n_e, lut_len = lut_d.shape
    if lut_s.shape != lut_d.shape or lut_i.shape != lut_d.shape:
        raise ValueError("'lut_depths', 'lut_sigmas' and 'lut_idds' must have the same shape.")
    if dvp.shape[0] < n_e:
        raise ValueError("'divergence_params' must have a row per LUT energy.")
    wet_c = np.ascontiguousarray(wet_v)
    spots_c = np.ascontiguousarray(spots)
    dvp_c = np.ascontiguousarray(dvp)
    lut_dc, lut_sc, lut_ic = (np.ascontiguousarray(a) for a in (lut_d, lut_s, lut_i))
    sp = _vec3(spacing, "spacing", 1)
    out = _output(wet_v.shape)
    nz, ny, nx = wet_v.shape
    lib = _lib.load()
    rc = lib.dc_proton_spot(gpu_id, _ptr(wet_c), nz, ny, nx, _lib.f3((sp[0],) * 3),
                            _lib.f3(_vec3(origin, "origin")), _lib.f3(_vec3(iso, "iso")), ga, ta, vsadx, vsady,
                            _ptr(dvp_c), n_e, dvp_c.shape[1], _ptr(lut_dc), _ptr(lut_sc), _ptr(lut_ic), lut_len,
                            _ptr(spots_c), spots_c.shape[0], _ptr(out))
    _lib.raise_for(rc)
    return out


_PHOTON_FLOATS = ("mu_calibration", "primary_source_distance", "scatter_source_distance", "primary_source_size",
                  "scatter_source_size", "mlc_distance", "scatter_source_weight", "electron_attenuation",
                  "electron_source_weight", "electron_fitted_dmax", "jaw_transmission", "mlc_transmission")
_PHOTON_ARRAYS = ("profile_radius", "profile_intensities", "profile_softening",
                  "spectrum_attenuation_coefficients", "spectrum_primary_weights", "spectrum_scatter_weights")


class PhotonModelView:
    """A beam model's arrays and scalars packed for the C ABI (keeps the numpy
    buffers alive for as long as the ctypes struct is used)."""

    def __init__(self, model):
        scal = {k: _getfloat(model, k) for k in _PHOTON_FLOATS}
        hx = _getbool(model, "has_xjaws")
        hy = _getbool(model, "has_yjaws")
        arrs = {k: _getarray(model, k, 1) for k in _PHOTON_ARRAYS}
        kernel = _getarray(model, "kernel", 2)
        if kernel.shape[1] != 6:
            raise ValueError("'kernel' must have 6 columns (theta, Am, am, Bm, bm, ray_length).")
        n_prof = arrs["profile_radius"].shape[0]
        if arrs["profile_intensities"].shape[0] != n_prof or arrs["profile_softening"].shape[0] != n_prof:
            raise ValueError("'profile_*' arrays must have the same length.")
        n_spec = arrs["spectrum_attenuation_coefficients"].shape[0]
        if (arrs["spectrum_primary_weights"].shape[0] != n_spec
                or arrs["spectrum_scatter_weights"].shape[0] != n_spec):
            raise ValueError("'spectrum_*' arrays must have the same length.")
        self._keep = {k: np.ascontiguousarray(v) for k, v in arrs.items()}
        cols = [np.ascontiguousarray(kernel[:, c], dtype=np.float32) for c in range(6)]
        self._keep.update({"k%d" % c: cols[c] for c in range(6)})
        m = _lib.PhotonModel()
        m.n_profile_points = n_prof
        m.profile_radius = _fptr(self._keep["profile_radius"])
        m.profile_intensities = _fptr(self._keep["profile_intensities"])
        m.profile_softening = _fptr(self._keep["profile_softening"])
        m.n_spectral_energies = n_spec
        m.spectrum_attenuation_coefficients = _fptr(self._keep["spectrum_attenuation_coefficients"])
        m.spectrum_primary_weights = _fptr(self._keep["spectrum_primary_weights"])
        m.spectrum_scatter_weights = _fptr(self._keep["spectrum_scatter_weights"])
        for k, v in scal.items():
            setattr(m, k, v)
        m.has_xjaws = int(hx)
        m.has_yjaws = int(hy)
        m.n_cones = kernel.shape[0]
        m.kernel_theta_deg, m.kernel_Am, m.kernel_am, m.kernel_Bm, m.kernel_bm, m.kernel_ray_length = (
            _fptr(c) for c in cols)
        self.struct = m


class ControlPointView:
    """A control point packed for the C ABI."""

    def __init__(self, cp):
        iso = _getarray(cp, "iso", 1)
        mlc = _getarray(cp, "mlc", 2)
        mu = _getfloat(cp, "mu")
        ga = _getfloat(cp, "ga")
        ca = _getfloat(cp, "ca")
        ta = _getfloat(cp, "ta")
        if mlc.shape[1] != 4:
            raise ValueError("'mlc' must have 4 columns (x1, x2, y_offset, y_width).")
        self._cols = [np.ascontiguousarray(mlc[:, c], dtype=np.float32) for c in range(4)]
        s = _lib.ControlPoint()
        v = _vec3(iso, "iso")
        s.iso[0], s.iso[1], s.iso[2] = float(v[0]), float(v[1]), float(v[2])
        s.mu = mu
        s.gantry_deg = ga
        s.collimator_deg = ca
        s.couch_deg = ta
        s.n_mlc_pairs = mlc.shape[0]
        s.mlc_x1, s.mlc_x2, s.mlc_y_offset, s.mlc_y_width = (_fptr(c) for c in self._cols)
        self.struct = s


def photon_dose_cuda(model, volume, cp, gpu_id):
    """Collapsed-cone dose of one control point (reference: rayTraceKernel +
    termaKernel + cccKernel), before the output factor."""
    gpu_id = operator.index(gpu_id)
    mv = PhotonModelView(model)
    vox, spacing, origin = _volume(volume)
    cv = ControlPointView(cp)
    vox_c = np.ascontiguousarray(vox)
    sp = _vec3(spacing, "spacing", 1)
    out = _output(vox.shape)
    nz, ny, nx = vox.shape
    lib = _lib.load()
    rc = lib.dc_photon_dose(gpu_id, _ptr(vox_c), nz, ny, nx, _lib.f3((sp[0],) * 3),
                            _lib.f3(_vec3(origin, "origin")), C.byref(mv.struct), C.byref(cv.struct), _ptr(out))
    _lib.raise_for(rc)
    return out
