"""ctypes binding of libdosecuda.so (the C ABI declared in include/dosecuda.h).

The library is built in-tree by ``dosecuda_b200.build``.  Loading fails loudly
when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdosecuda.so")

DC_OK = 0
DC_ERR_VALUE = 1
DC_ERR_MEMORY = 2
DC_ERR_CUDA = 3

_fp = C.POINTER(C.c_float)


class PhotonModel(C.Structure):
    """Mirror of ``dc_photon_model``."""
    _fields_ = [
        ("n_profile_points", C.c_int),
        ("profile_radius", _fp),
        ("profile_intensities", _fp),
        ("profile_softening", _fp),
        ("n_spectral_energies", C.c_int),
        ("spectrum_attenuation_coefficients", _fp),
        ("spectrum_primary_weights", _fp),
        ("spectrum_scatter_weights", _fp),
        ("mu_calibration", C.c_float),
        ("primary_source_distance", C.c_float),
        ("scatter_source_distance", C.c_float),
        ("primary_source_size", C.c_float),
        ("scatter_source_size", C.c_float),
        ("mlc_distance", C.c_float),
        ("scatter_source_weight", C.c_float),
        ("electron_attenuation", C.c_float),
        ("electron_source_weight", C.c_float),
        ("electron_fitted_dmax", C.c_float),
        ("jaw_transmission", C.c_float),
        ("mlc_transmission", C.c_float),
        ("has_xjaws", C.c_int),
        ("has_yjaws", C.c_int),
        ("n_cones", C.c_int),
        ("kernel_theta_deg", _fp),
        ("kernel_Am", _fp),
        ("kernel_am", _fp),
        ("kernel_Bm", _fp),
        ("kernel_bm", _fp),
        ("kernel_ray_length", _fp),
    ]


class FluenceMap(C.Structure):
    """dc_fluence_map: beamlet grid on the beam's-eye-view isocentre plane."""
    _fields_ = [("na", C.c_int), ("nb", C.c_int), ("a0", C.c_float), ("b0", C.c_float), ("pitch", C.c_float)]


class ControlPoint(C.Structure):
    """Mirror of ``dc_control_point``."""
    _fields_ = [
        ("iso", C.c_float * 3),
        ("mu", C.c_float),
        ("gantry_deg", C.c_double),
        ("collimator_deg", C.c_float),
        ("couch_deg", C.c_float),
        ("n_mlc_pairs", C.c_int),
        ("mlc_x1", _fp),
        ("mlc_x2", _fp),
        ("mlc_y_offset", _fp),
        ("mlc_y_width", _fp),
    ]


# Every symbol include/dosecuda.h declares, with its ctypes signature.
_F3 = C.c_float * 3
_VOL = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, _F3, _F3]
SIGNATURES = {
    "dc_last_error": (C.c_char_p, []),
    "dc_version": (C.c_int, []),
    "dc_device_count": (C.c_int, []),
    "dc_release_device": (C.c_int, [C.c_int]),
    "dc_photon_set_depth_mode": (C.c_int, [C.c_int, C.c_int]),
    "dc_photon_get_depth_mode": (C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    "dc_photon_head_selftest": (C.c_int, [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "dc_photon_depth_stats": (C.c_int, [C.c_int, C.POINTER(C.c_longlong)]),
    "dc_profile_enable": (C.c_int, [C.c_int, C.c_int]),
    "dc_profile_reset": (C.c_int, [C.c_int]),
    "dc_profile_read": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_int),
                                  C.POINTER(C.c_double)]),
    "dc_texture_fetch_rate": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "dc_proton_raytrace": (C.c_int, _VOL + [_F3, C.c_double, C.c_float, C.c_float, C.c_float, C.c_void_p]),
    "dc_proton_raytrace_dev": (C.c_int, _VOL + [_F3, C.c_double, C.c_float, C.c_float, C.c_float, C.c_void_p,
                                                C.c_void_p]),
    "dc_proton_raytrace_noalloc": (C.c_int, _VOL + [_F3, C.c_double, C.c_float, C.c_float, C.c_float,
                                                    C.c_void_p, C.c_void_p]),
    "dc_proton_spot": (C.c_int, _VOL + [_F3, C.c_double, C.c_float, C.c_float, C.c_float,
                                        C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                        C.c_void_p, C.c_int, C.c_void_p]),
    "dc_proton_spot_dev": (C.c_int, _VOL + [_F3, C.c_double, C.c_float, C.c_float, C.c_float,
                                            C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "dc_proton_beam_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _F3, _F3, _F3, C.c_double, C.c_float,
                                        C.c_float, C.c_float, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                        C.POINTER(C.c_void_p)]),
    "dc_proton_beam_destroy": (C.c_int, [C.c_void_p]),
    "dc_proton_beam_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_longlong)]),
    "dc_proton_beam_dose": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_proton_beam_adjoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_proton_beam_dose_list": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                           C.c_void_p]),
    "dc_proton_beam_adjoint_list": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                              C.c_void_p]),
    "dc_proton_beam_influence_nnz": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.POINTER(C.c_longlong),
                                               C.c_void_p]),
    "dc_proton_beam_influence_csr": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_longlong, C.c_void_p]),
    "dc_proton_batch_create": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_int, C.c_float, C.c_float, C.POINTER(C.c_void_p)]),
    "dc_proton_batch_add_plan": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, _F3, _F3, C.c_void_p,
                                           C.c_void_p, C.POINTER(C.c_int)]),
    "dc_proton_batch_add_beam": (C.c_int, [C.c_void_p, C.c_int, _F3, C.c_double, C.c_float, C.c_void_p, C.c_int,
                                           C.c_void_p, C.POINTER(C.c_int)]),
    "dc_proton_batch_commit": (C.c_int, [C.c_void_p]),
    "dc_proton_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int)]),
    "dc_proton_batch_beam_spot_offset": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "dc_proton_batch_wet": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dc_proton_batch_dose": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "dc_proton_batch_influence_count": (C.c_int, [C.c_void_p, C.c_int, C.c_float, C.c_void_p,
                                                  C.POINTER(C.c_longlong), C.c_void_p]),
    "dc_proton_batch_influence_fill": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_longlong, C.c_void_p]),
    "dc_proton_batch_destroy": (C.c_int, [C.c_void_p]),
    "dc_photon_dose": (C.c_int, _VOL + [C.POINTER(PhotonModel), C.POINTER(ControlPoint), C.c_void_p]),
    "dc_photon_dose_dev": (C.c_int, _VOL + [C.POINTER(PhotonModel), C.POINTER(ControlPoint), C.c_void_p,
                                            C.c_void_p]),
    "dc_hu_convert_dev": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_void_p]),
    "dc_proton_raytrace_hu_dev": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, _F3, _F3, C.c_void_p,
                                            C.c_void_p, C.c_int, _F3, C.c_double, C.c_float, C.c_float, C.c_float,
                                            C.c_void_p, C.c_void_p]),
    "dc_photon_plan_dose_dev": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                          C.c_int, C.c_int, _F3, _F3, C.POINTER(PhotonModel), C.c_void_p, C.c_int,
                                          C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_photon_beam_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _F3, _F3, C.POINTER(C.c_void_p)]),
    "dc_photon_beam_destroy": (C.c_int, [C.c_void_p]),
    "dc_photon_beam_set_density": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_photon_beam_terma": (C.c_int, [C.c_void_p, C.POINTER(PhotonModel), C.POINTER(ControlPoint), C.c_void_p,
                                       C.c_void_p]),
    "dc_photon_beam_dose": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_photon_beam_probe_config": (C.c_int, [C.c_void_p, C.c_int]),
    "dc_photon_beam_probe_select": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_void_p]),
    "dc_photon_beam_probe_list": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.c_void_p,
                                            C.c_int]),
    "dc_photon_beam_probe": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "dc_photon_beam_dose_sweep": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_photon_beam_fluence_dose": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_photon_beam_fluence_adjoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_gamma": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, _F3, C.c_void_p, C.c_void_p, C.c_longlong,
                           C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p, C.c_void_p]),
    "dc_net_packed_fragments": (C.c_longlong, [C.c_int, C.c_int, C.c_int]),
    "dc_net_packed_tc_bytes": (C.c_longlong, [C.c_int, C.c_int]),
    "dc_net_pack_weights_tc": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_void_p, C.c_void_p]),
    "dc_net_conv_tc": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                 C.c_longlong, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_net_tc_error": (C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    "dc_net_tc_selftest": (C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    "dc_host_buffer_mapped": (C.c_int, [C.c_int, C.c_void_p, C.c_ulonglong, C.POINTER(C.c_int)]),
    "dc_debug_bounds": (C.c_int, [C.c_int, C.POINTER(C.c_ulonglong), C.POINTER(C.c_int)]),
    "dc_basis_combine_dev": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "dc_basis_adjoint_dev": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "dc_net_pack_weights": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                      C.c_void_p]),
    "dc_net_conv": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                              C.c_longlong, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_net_conv_up": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                 C.c_longlong, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dc_net_wgrad": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                               C.c_int, C.c_void_p, C.c_void_p]),
    "dc_net_norm_finalize": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p,
                                       C.c_float, C.c_void_p, C.c_void_p]),
    "dc_net_norm_act": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_longlong, C.c_int, C.c_void_p, C.c_float,
                                  C.c_void_p, C.c_void_p]),
    "dc_net_norm_stats_act": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_longlong, C.c_int, C.c_void_p,
                                        C.c_longlong, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_void_p,
                                        C.c_void_p, C.c_void_p]),
    "dc_net_norm_act_bwd": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    "dc_net_pack_input": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_longlong, C.c_float, C.c_void_p,
                                    C.c_void_p]),
    "dc_net_head": (C.c_int, [C.c_int, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_float, C.c_float, C.c_void_p, C.c_void_p]),
    "dc_net_head_loss_bwd": (C.c_int, [C.c_int, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p]),
}

_lib = None
_lock = threading.Lock()


class DoseCudaError(RuntimeError):
    pass


def load(path: str | None = None):
    """Load (once) and return the ctypes handle of libdosecuda.so."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise ImportError(
                f"libdosecuda.so not found at {p}; build it with `python -m dosecuda_b200.build` "
                "(the dose engines have no CPU fallback)")
        lib = C.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def raise_for(rc: int):
    """Translate a C-ABI status code into the reference's Python exception class
    (dosemodule.cu:62,189-197)."""
    if rc == DC_OK:
        return
    msg = load().dc_last_error().decode("utf-8", "replace")
    if rc == DC_ERR_VALUE:
        raise ValueError(msg)
    if rc == DC_ERR_MEMORY:
        raise MemoryError(msg or "Not enough host memory")
    raise RuntimeError("CUDA error: " + msg)


def f3(v) -> C.Array:
    a = _F3()
    a[0], a[1], a[2] = float(v[0]), float(v[1]), float(v[2])
    return a


def profile_read(gpu_id: int = 0, max_kernels: int = 64):
    """{kernel: (launches, total_ms)} accumulated since the last reset."""
    lib = load()
    names = (C.c_char_p * max_kernels)()
    launches = (C.c_int * max_kernels)()
    totals = (C.c_double * max_kernels)()
    n = lib.dc_profile_read(gpu_id, max_kernels, names, launches, totals)
    if n < 0:
        raise_for(-n)
    return {names[i].decode(): (launches[i], totals[i]) for i in range(n)}
