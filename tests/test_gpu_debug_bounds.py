"""Debug-build bounds checks (the compute-sanitizer substitute on this GPU
pool): the library built with -DDC_DEBUG_BOUNDS checks the index of every
instrumented global access of the dose kernels and records the first
violation instead of faulting.  Small cases of every dose path run through
that build must record none and give the release build's results (to
float32 rounding: the checks can change which multiply-adds the compiler
fuses)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import ctypes as C, json, sys
import numpy as np, torch
from dosecuda_b200 import _lib
lib = _lib.load(sys.argv[1])
from dosecuda_b200 import dose_kernels, engine, phantoms
out = {}
grid, plan = phantoms.photon_small(shape=(40, 44, 36), spacing=4.0, field_cm=(6.0, 8.0), gantry=30.0, seed=3)
model, cp = plan.beam_models[0], plan.beam_list[0].cp_list[0]
vol = phantoms.volume_object(grid, grid.DensityFromHU(plan.machine_name))
out["photon"] = dose_kernels.photon_dose_cuda(model, vol, cp, 0)
density = torch.as_tensor(vol.voxel_data).cuda()
basis = engine.PhotonPlanBasis(density, grid, model, [cp, cp])
out["basis"] = basis.dose().cpu().numpy()
out["basis_adj"] = basis.adjoint(torch.ones_like(density)).cpu().numpy()
pg, pp = phantoms.proton_small(shape=(17, 23, 29), spacing=3.0, energy_ids=(5, 15), field_mm=24.0, pitch_mm=4.0,
                               gantry=30.0, couch=10.0, seed=9)
pm, pb = pp.beam_models[0], pp.beam_list[0]
rl = phantoms.volume_object(pg, pg.RLSPFromHU(pp.machine_name))
w = dose_kernels.proton_raytrace_cuda(pm, rl, pb, 0)
out["wet"] = w
out["pdose"] = dose_kernels.proton_spot_cuda(pm, rl, phantoms.volume_object(pg, w), pb, 0)
wt = torch.as_tensor(np.array(w)).cuda()
bp = engine.ProtonBeamPlan(pg, pb, pm)
out["bdose"] = bp.dose(wt).cpu().numpy()
g = torch.linspace(-1, 1, wt.numel(), device="cuda").reshape(wt.shape)
out["adj"] = bp.adjoint(wt, g).cpu().numpy()
vox = torch.tensor([-5, 0, 7, wt.numel() - 1, wt.numel(), 123456789], dtype=torch.int32, device="cuda")
out["list"] = bp.dose_list(wt, vox).cpu().numpy()
out["list_adj"] = bp.adjoint_list(wt, vox, torch.ones(vox.numel(), device="cuda")).cpu().numpy()
nw = torch.empty_like(rlt := torch.as_tensor(rl.voxel_data).cuda())
_lib.raise_for(lib.dc_proton_raytrace_noalloc(0, C.c_void_p(rlt.data_ptr()), *rlt.shape, _lib.f3(pg.spacing),
                                              _lib.f3(pg.origin), _lib.f3(pb.iso), float(pb.gantry_angle),
                                              float(pb.couch_angle), float(pm.VSADX), float(pm.VSADY),
                                              C.c_void_p(nw.data_ptr()), C.c_void_p(0)))
out["noalloc_wet"] = nw.cpu().numpy()
r, c, v = bp.influence_csr(wt, cutoff=1e-4)
out["csr_r"], out["csr_c"], out["csr_v"] = r.cpu().numpy(), c.cpu().numpy(), v.cpu().numpy()
torch.cuda.synchronize()
viol, en = C.c_ulonglong(0), C.c_int(-1)
_lib.raise_for(lib.dc_debug_bounds(0, C.byref(viol), C.byref(en)))
np.savez(sys.argv[2], **out)
print(json.dumps({"enabled": en.value, "violation": viol.value}))
"""


def _run(lib, out):
    env = dict(os.environ)
    env["PYTHONPATH"] = ROOT + os.pathsep + env.get("PYTHONPATH", "")
    r = subprocess.run([sys.executable, "-c", _CHILD, lib, out], env=env, cwd=ROOT, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), np.load(out)


def test_bounds_checked_build_records_no_violation_and_matches_release(tmp_path):
    dbg = str(tmp_path / "libdosecuda_dbg.so")
    b = subprocess.run([sys.executable, "-m", "dosecuda_b200.build", "--debug-bounds", "--out", dbg], cwd=ROOT,
                       capture_output=True, text=True, timeout=1800)
    assert b.returncode == 0, b.stderr[-3000:]
    rel = os.path.join(ROOT, "dosecuda_b200", "libdosecuda.so")
    info_d, d = _run(dbg, str(tmp_path / "dbg.npz"))
    info_r, r = _run(rel, str(tmp_path / "rel.npz"))
    assert info_d == {"enabled": 1, "violation": 0}, info_d
    assert info_r == {"enabled": 0, "violation": 0}, info_r
    # The checks change the surrounding code, so the compiler may fuse a
    # multiply-add differently: results agree to float32 rounding, not bits.
    for k in d.files:
        if k in ("csr_r", "csr_c", "csr_v"):
            continue
        scale = float(np.abs(r[k]).max()) + 1e-30
        assert float(np.abs(d[k].astype(np.float64) - r[k]).max()) <= 1e-5 * scale, k
    # the influence matrix: same size up to entries at the cut-off's knife edge
    assert abs(int(d["csr_r"][-1]) - int(r["csr_r"][-1])) <= 1e-3 * int(r["csr_r"][-1])
    assert d["list"][0] == 0.0 and d["list"][4] == 0.0 and d["list"][5] == 0.0  # out-of-grid entries
