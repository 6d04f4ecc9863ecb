"""ctypes wrapper of the CPU oracle (oracle/oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py, never by the product.  See the
header of oracle.c for what it restates and its arithmetic policy.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

_fp = C.POINTER(C.c_float)


class _PhotonModel(C.Structure):
    _fields_ = [("n_prof", C.c_int), ("prof_r", _fp), ("prof_i", _fp), ("prof_s", _fp),
                ("n_spec", C.c_int), ("spec_mu", _fp), ("spec_pw", _fp), ("spec_sw", _fp),
                ("mu_cal", C.c_float), ("psd", C.c_float), ("ssd", C.c_float), ("pss", C.c_float),
                ("sss", C.c_float), ("mlc_dist", C.c_float), ("ssw", C.c_float), ("ea", C.c_float),
                ("esw", C.c_float), ("efd", C.c_float), ("n_cones", C.c_int),
                ("k_theta", _fp), ("k_Am", _fp), ("k_am", _fp), ("k_Bm", _fp), ("k_bm", _fp), ("k_rl", _fp)]


class _Mlc(C.Structure):
    _fields_ = [("n_pairs", C.c_int), ("x1", _fp), ("x2", _fp), ("yoff", _fp), ("yw", _fp)]


def load():
    global _lib
    if _lib is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("_oracle_build", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        path = mod.build_oracle()
        lib = C.CDLL(path)
        F3 = C.c_float * 3
        vol = [C.c_void_p, C.c_int, C.c_int, C.c_int, F3, F3]
        lib.oracle_proton_wet.restype = C.c_long
        lib.oracle_proton_wet.argtypes = vol + [F3, C.c_double, C.c_float, C.c_float, C.c_float, C.c_int,
                                                C.c_void_p, C.c_void_p]
        lib.oracle_proton_dose.restype = C.c_long
        lib.oracle_proton_dose.argtypes = vol + [F3, C.c_double, C.c_float, C.c_float, C.c_float, C.c_void_p,
                                                 C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                                 C.c_void_p, C.c_int, C.c_void_p]
        lib.oracle_photon_dose.restype = C.c_long
        lib.oracle_photon_dose.argtypes = vol + [C.POINTER(_PhotonModel), F3, C.c_float, C.c_double, C.c_float,
                                                 C.c_float, C.POINTER(_Mlc), C.c_int, C.c_void_p, C.c_void_p,
                                                 C.c_void_p]
        lib.oracle_photon_transmission.restype = None
        lib.oracle_photon_transmission.argtypes = [C.c_int, C.c_int, C.c_int, F3, F3, C.POINTER(_PhotonModel), F3,
                                                   C.c_double, C.c_float, C.c_float, C.POINTER(_Mlc), C.c_void_p,
                                                   C.c_void_p]
        lib.oracle_last_near_pairs.restype = C.c_long
        lib.oracle_num_threads.restype = C.c_int
        _lib = lib
    return _lib


def num_threads() -> int:
    return load().oracle_num_threads()


def _f3(v):
    a = (C.c_float * 3)()
    a[0], a[1], a[2] = float(v[0]), float(v[1]), float(v[2])
    return a


def _c(a, dtype=np.float32):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def proton_wet(rlsp, spacing, origin, iso, gantry, couch, vsadx, vsady, tex_mode=0, raw=False):
    """Smoothed WET (cm) in float64; with raw=True also the unsmoothed WET.
    Also returns the number of texture samples of the march."""
    rl = _c(rlsp)
    nz, ny, nx = rl.shape
    wet = np.empty(rl.shape, np.float64)
    wraw = np.empty(rl.shape, np.float64)
    n = load().oracle_proton_wet(_p(rl), nz, ny, nx, _f3(spacing), _f3(origin), _f3(iso), float(gantry),
                                 float(couch), float(vsadx), float(vsady), int(tex_mode), _p(wraw), _p(wet))
    return (wet, wraw, n) if raw else (wet, n)


def proton_dose(wet, spacing, origin, iso, gantry, couch, model, spots, near_pairs=False):
    """Pencil-beam dose (float64) from a float32 smoothed WET; returns
    (dose, evaluated (voxel, spot) pairs), with near_pairs=True also the
    pairs within 6 halo sigmas of the spot axis."""
    w = _c(wet)
    nz, ny, nx = w.shape
    dvp = _c(model.divergence_params)
    ld, ls, li = _c(model.lut_depths), _c(model.lut_sigmas), _c(model.lut_idds)
    sp = _c(spots)
    if sp.ndim == 1:
        sp = sp.reshape(1, 4)
    dose = np.empty(w.shape, np.float64)
    n = load().oracle_proton_dose(_p(w), nz, ny, nx, _f3(spacing), _f3(origin), _f3(iso), float(gantry),
                                  float(couch), float(model.VSADX), float(model.VSADY), _p(dvp), ld.shape[0],
                                  dvp.shape[1], _p(ld), _p(ls), _p(li), ld.shape[1], _p(sp), sp.shape[0], _p(dose))
    if n < 0:
        raise ValueError("spot energy id outside the beam model")
    if near_pairs:
        return dose, n, load().oracle_last_near_pairs()
    return dose, n


def _photon_structs(model, mlc):
    keep = {}

    def fp(name, arr):
        keep[name] = _c(arr)
        return keep[name].ctypes.data_as(_fp)

    m = _PhotonModel()
    m.n_prof = len(model.profile_radius)
    m.prof_r = fp("pr", model.profile_radius)
    m.prof_i = fp("pi", model.profile_intensities)
    m.prof_s = fp("ps", model.profile_softening)
    m.n_spec = len(model.spectrum_attenuation_coefficients)
    m.spec_mu = fp("sm", model.spectrum_attenuation_coefficients)
    m.spec_pw = fp("sp", model.spectrum_primary_weights)
    m.spec_sw = fp("ss", model.spectrum_scatter_weights)
    for a, k in (("mu_cal", "mu_calibration"), ("psd", "primary_source_distance"),
                 ("ssd", "scatter_source_distance"), ("pss", "primary_source_size"),
                 ("sss", "scatter_source_size"), ("mlc_dist", "mlc_distance"), ("ssw", "scatter_source_weight"),
                 ("ea", "electron_attenuation"), ("esw", "electron_source_weight"), ("efd", "electron_fitted_dmax")):
        setattr(m, a, float(getattr(model, k)))
    kern = np.asarray(model.kernel, dtype=np.float32)
    m.n_cones = kern.shape[0]
    m.k_theta, m.k_Am, m.k_am, m.k_Bm, m.k_bm, m.k_rl = (fp("k%d" % c, kern[:, c]) for c in range(6))
    ml = np.asarray(mlc, dtype=np.float32)
    mm = _Mlc()
    mm.n_pairs = ml.shape[0]
    mm.x1, mm.x2, mm.yoff, mm.yw = (fp("m%d" % c, ml[:, c]) for c in range(4))
    return m, mm, keep


def photon_dose(density, spacing, origin, model, iso, mu, gantry, collimator, couch, mlc, tex_mode=0,
                intermediates=False):
    """CCCS dose (float64) of one control point; returns (dose, samples) or,
    with intermediates=True, (dose, terma, electron, samples)."""
    d = _c(density)
    nz, ny, nx = d.shape
    m, mm, keep = _photon_structs(model, mlc)
    dose = np.empty(d.shape, np.float64)
    terma = np.empty(d.shape, np.float64)
    elec = np.empty(d.shape, np.float64)
    n = load().oracle_photon_dose(_p(d), nz, ny, nx, _f3(spacing), _f3(origin), C.byref(m), _f3(iso), float(mu),
                                  float(gantry), float(collimator), float(couch), C.byref(mm), int(tex_mode),
                                  _p(terma), _p(elec), _p(dose))
    del keep
    return (dose, terma, elec, n) if intermediates else (dose, n)


def photon_transmission(shape, spacing, origin, model, iso, gantry, collimator, couch, mlc):
    """Primary and scatter head transmission (float64) at every voxel centre."""
    nz, ny, nx = shape
    m, mm, keep = _photon_structs(model, mlc)
    tp = np.empty(shape, np.float64)
    ts = np.empty(shape, np.float64)
    load().oracle_photon_transmission(nz, ny, nx, _f3(spacing), _f3(origin), C.byref(m), _f3(iso), float(gantry),
                                      float(collimator), float(couch), C.byref(mm), _p(tp), _p(ts))
    del keep
    return tp, ts


# ---------------------------------------------------------------------------
# The reference's own ray-trace + TERMA kernels (oracle/_ref/libref_terma.so,
# built from the reference sources by build_ref.sh; needs a GPU to run).
# ---------------------------------------------------------------------------
_ref_terma = None


def reference_terma_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_terma.so"))


def reference_photon_terma(density, spacing, origin, model, iso, mu, gantry, collimator, couch, mlc, gpu_id=0):
    """(WET, TERMA, electron) float32 volumes of one control point from the
    reference's rayTraceKernel and termaKernel (CudaClasses.cu:180-228,
    IMRTClasses.cu:209-250)."""
    global _ref_terma
    if _ref_terma is None:
        lib = C.CDLL(os.path.join(HERE, "_ref", "libref_terma.so"))
        F3 = C.c_float * 3
        lib.ref_photon_terma.restype = C.c_int
        lib.ref_photon_terma.argtypes = ([C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, F3, F3,
                                          C.c_float, C.c_float, C.c_float, C.c_void_p] +
                                         [C.c_int] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 3 +
                                         [C.c_int] + [C.c_void_p] * 4 + [C.c_float] + [C.c_void_p] * 3 +
                                         [C.c_char_p, C.c_int])
        _ref_terma = lib
    d = _c(density)
    nz, ny, nx = d.shape
    scal = _c([model.mu_calibration, model.primary_source_distance, model.scatter_source_distance,
               model.primary_source_size, model.scatter_source_size, model.mlc_distance,
               model.scatter_source_weight, model.electron_attenuation, model.electron_source_weight,
               model.electron_fitted_dmax])
    pr, pi, ps = (_c(getattr(model, k)) for k in ("profile_radius", "profile_intensities", "profile_softening"))
    sm, spw, ssw = (_c(getattr(model, k)) for k in ("spectrum_attenuation_coefficients", "spectrum_primary_weights",
                                                     "spectrum_scatter_weights"))
    ml = np.asarray(mlc, np.float32)
    cols = [_c(ml[:, c]) for c in range(4)]
    wet = np.empty(d.shape, np.float32)
    terma = np.empty(d.shape, np.float32)
    elec = np.empty(d.shape, np.float32)
    err = C.create_string_buffer(512)
    rc = _ref_terma.ref_photon_terma(int(gpu_id), _p(d), nz, ny, nx, float(spacing), _f3(origin), _f3(iso),
                                     float(gantry), float(collimator), float(couch), _p(scal), len(pr), _p(pr),
                                     _p(pi), _p(ps), len(sm), _p(sm), _p(spw), _p(ssw), ml.shape[0],
                                     *[_p(c) for c in cols], float(mu), _p(wet), _p(terma), _p(elec), err, 512)
    if rc != 0:
        raise RuntimeError("reference TERMA harness: " + err.value.decode())
    return wet, terma, elec
