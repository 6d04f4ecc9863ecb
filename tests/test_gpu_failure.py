"""Failure detection without a GPU fault.

* Allocation failure (here): ``DC_INJECT_ALLOC_FAIL=N`` makes the N-th device /
  pinned / texture-array allocation of the process fail before the CUDA call,
  as an out-of-memory would.  Every public call must turn it into a Python
  error, leave no half-built state behind, and the next call must succeed
  with the exact result of a process that saw no failure.  Run in child
  processes (the counter is process-wide).
* Bounded tensor-core wait (test_gpu_net.py): the tcgen05 convolution's
  mbarrier wait is bounded; its self-test withholds the MMAs, so the wait
  must expire, be reported through the error flag, and leave the context
  usable."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import json, sys
import numpy as np
from dosecuda_b200 import dose_kernels, phantoms
grid, plan = phantoms.photon_small(shape=(48, 48, 48), spacing=4.0, field_cm=(6.0, 6.0))
model, cp = plan.beam_models[0], plan.beam_list[0].cp_list[0]
vol = phantoms.volume_object(grid, grid.DensityFromHU(plan.machine_name))
pgrid, pplan = phantoms.proton_small(shape=(48, 48, 48), spacing=3.0)
pbeam = pplan.beam_list[0]
pvol = phantoms.volume_object(pgrid, pgrid.RLSPFromHU(pplan.machine_name))
out = {"errors": []}
for attempt in range(3):
    try:
        d = dose_kernels.photon_dose_cuda(model, vol, cp, 0)
        w = dose_kernels.proton_raytrace_cuda(pplan.beam_models[0], pvol, pbeam, 0)
        np.save(sys.argv[1] + "_photon.npy", d)
        np.save(sys.argv[1] + "_wet.npy", w)
        break
    except Exception as e:
        out["errors"].append(type(e).__name__ + ": " + str(e))
print(json.dumps(out))
"""


def _run_child(tmp_path, tag, inject):
    env = dict(os.environ)
    env.pop("DC_INJECT_ALLOC_FAIL", None)
    if inject:
        env["DC_INJECT_ALLOC_FAIL"] = str(inject)
    env["PYTHONPATH"] = ROOT + os.pathsep + env.get("PYTHONPATH", "")
    base = str(tmp_path / tag)
    r = subprocess.run([sys.executable, "-c", _CHILD, base], env=env, cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    return out, np.load(base + "_photon.npy"), np.load(base + "_wet.npy")


def test_injected_allocation_failures_recover_exactly(tmp_path):
    clean, d0, w0 = _run_child(tmp_path, "clean", 0)
    assert clean["errors"] == [] and d0.max() > 0 and w0.max() > 0
    seen = 0
    for n in (1, 2, 3, 5, 8):
        out, d, w = _run_child(tmp_path, "inject%d" % n, n)
        # the injected allocation fails at most once; the retry succeeds exactly
        assert len(out["errors"]) <= 1, out["errors"]
        for e in out["errors"]:
            assert e.startswith("RuntimeError") and "injected failure of allocation %d" % n in e, e
        seen += len(out["errors"])
        assert np.array_equal(d, d0) and np.array_equal(w, w0)
    assert seen >= 3  # the first allocations of a call are reached by the injection
