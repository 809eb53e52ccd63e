import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "vx-rs_b200")
ORACLE = os.path.join(REPO, "oracle")
for p in (PKG, ORACLE, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    # Build (or confirm up to date) the library and the CPU checkers once per session.
    for d in (PKG, ORACLE):
        subprocess.run(["make", "-s", "-C", d], check=True)


@pytest.fixture(scope="session")
def gpu_ctx():
    import vx_sgm
    ctx = vx_sgm.Context(0)
    yield ctx
    ctx.close()


@pytest.fixture(params=["single", "pairs", "scan"])
def agg_form(request, monkeypatch):
    """Runs a test through each aggregation form: the single-scanline kernel, the
    scanline-pair kernel (large batches) and the across-lanes scan kernel (few
    units: single pairs, small batches)."""
    monkeypatch.setenv("VX_SGM_AGG_FORM", request.param)
    return request.param


@pytest.fixture(scope="session")
def sgm(gpu_ctx):
    import vx_sgm
    s = vx_sgm.SGMStereo(gpu_ctx)
    yield s
    s.close()


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np
    z = np.load(os.path.join(REPO, "tests", "golden", "reference_cases.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    cases = []
    for m in meta:
        c = dict(m)
        for k in ("left", "right", "census_l", "census_r", "disparity", "S_sum"):
            c[k] = z[f"{m['name']}/{k}"]
        c["S"] = z[f"{m['name']}/S"] if m["store_S"] else None
        cases.append(c)
    return cases
