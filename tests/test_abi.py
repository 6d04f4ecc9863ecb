"""The C ABI library: loads, exports every declared symbol, validates
arguments before touching a GPU (runs without one)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from dosecuda_b200 import _lib


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "dosecuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dc_[a-z0-9_]+)\s*\(", src)))


def test_library_builds_and_loads():
    lib = _lib.load()
    assert lib.dc_version() >= 100


def test_exports_every_declared_symbol():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(lib, s), s
    # the Python binding declares a signature for each of them
    assert set(syms) == set(_lib.SIGNATURES)


def test_device_count_without_gpu_is_not_an_error():
    n = _lib.load().dc_device_count()
    assert n >= 0 or n == -1


def _f3(v):
    return _lib.f3(v)


def test_value_errors_before_any_gpu_work():
    lib = _lib.load()
    out = np.zeros(8, np.float32)
    # zero-sized volume
    rc = lib.dc_proton_raytrace(0, out.ctypes.data_as(C.c_void_p), 0, 2, 2, _f3((1, 1, 1)), _f3((0, 0, 0)),
                                _f3((0, 0, 0)), 0.0, 0.0, 1340.0, 1930.0, out.ctypes.data_as(C.c_void_p))
    assert rc == _lib.DC_ERR_VALUE
    assert "dimensions" in lib.dc_last_error().decode()
    # non-positive spacing
    rc = lib.dc_proton_raytrace(0, out.ctypes.data_as(C.c_void_p), 2, 2, 2, _f3((0, 1, 1)), _f3((0, 0, 0)),
                                _f3((0, 0, 0)), 0.0, 0.0, 1340.0, 1930.0, out.ctypes.data_as(C.c_void_p))
    assert rc == _lib.DC_ERR_VALUE
    # zero VSAD
    rc = lib.dc_proton_raytrace(0, out.ctypes.data_as(C.c_void_p), 2, 2, 2, _f3((1, 1, 1)), _f3((0, 0, 0)),
                                _f3((0, 0, 0)), 0.0, 0.0, 0.0, 1930.0, out.ctypes.data_as(C.c_void_p))
    assert rc == _lib.DC_ERR_VALUE


def test_spot_table_errors_before_any_gpu_work(impt_plan):
    lib = _lib.load()
    m = impt_plan.beam_models[0]
    wet = np.zeros((2, 2, 2), np.float32)
    out = np.zeros_like(wet)
    dvp = np.ascontiguousarray(m.divergence_params)

    def call(spots):
        sp = np.ascontiguousarray(spots, np.float32)
        return lib.dc_proton_spot(0, wet.ctypes.data_as(C.c_void_p), 2, 2, 2, _f3((1, 1, 1)), _f3((0, 0, 0)),
                                  _f3((0, 0, 0)), 0.0, 0.0, 1340.0, 1930.0, dvp.ctypes.data_as(C.c_void_p),
                                  dvp.shape[0], 5, m.lut_depths.ctypes.data_as(C.c_void_p),
                                  m.lut_sigmas.ctypes.data_as(C.c_void_p), m.lut_idds.ctypes.data_as(C.c_void_p),
                                  400, sp.ctypes.data_as(C.c_void_p), sp.shape[0], out.ctypes.data_as(C.c_void_p))

    assert call(np.zeros((0, 4))) == _lib.DC_ERR_VALUE
    assert call([[0, 0, 1, 98]]) == _lib.DC_ERR_VALUE  # energy id out of the 98-entry table
    assert "energy id" in lib.dc_last_error().decode()
    assert call([[0, 0, 1, -1.5]]) == _lib.DC_ERR_VALUE
    assert call([[0, 0, 1, np.nan]]) == _lib.DC_ERR_VALUE


def test_no_device_maps_to_runtime_error(cuda_ok):
    if cuda_ok:
        pytest.skip("a GPU is present")
    from dosecuda_b200 import phantoms, dose_kernels
    grid, plan = phantoms.proton_small(shape=(4, 4, 4))
    rl = phantoms.volume_object(grid, grid.RLSPFromHU(plan.machine_name))
    with pytest.raises(RuntimeError, match="^CUDA error: "):
        dose_kernels.proton_raytrace_cuda(plan.beam_models[0], rl, plan.beam_list[0], 0)
