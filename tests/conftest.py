import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    return meta, {k: z[k] for k in z.files if k != "meta"}


def golden_names(kind):
    out = []
    for f in sorted(os.listdir(GOLDEN)):
        if f.endswith(".npz"):
            meta, _ = load_golden(f[:-4])
            if meta["kind"] == kind:
                out.append(f[:-4])
    return out


@pytest.fixture(scope="session")
def impt_plan():
    from dosecuda_b200.plan_impt import IMPTPlan
    return IMPTPlan()


@pytest.fixture(scope="session")
def imrt_plan():
    from dosecuda_b200.plan_imrt import IMRTPlan
    return IMRTPlan("VarianTrueBeamHF")


def proton_model(plan, label):
    labels = list(plan.dicom_rangeshifter_label.astype(str))
    return plan.beam_models[labels.index(str(label))]


@pytest.fixture(scope="session")
def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
