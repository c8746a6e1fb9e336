"""The reference's own library and libsmoke_b200.so driven through the SAME C ABI calls with identical inputs.

The reference library is backend-cuda.cu compiled from its sources (oracle/_ref); this is the drop-in check:
every view after every step must agree. Both use the reference's solver semantics (fixed-count unpreconditioned
CG from x0 = 0), with enough iterations that both reach their FP32 floor, so the comparison is not dominated by
where each FP32 CG happens to stop.
"""
import json
import os

import numpy as np
import pytest
import torch

import scenes
import smoke_abi as abi
import smoke_b200

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIBRARY = os.path.join(ROOT, "oracle", "_ref", "libvisual-simulation-of-smoke.so")
REPORT = os.environ.get("SMOKE_PARITY_REPORT")

CASES = {
    "closed16_cubic": ((16, 16, 16), "closed", abi.MONOTONIC_CUBIC, False),
    "plume_cubic_solids": ((24, 20, 16), "plume", abi.MONOTONIC_CUBIC, True),
    "mixed_linear_solids": ((17, 13, 11), "mixed", abi.LINEAR, True),
    "slip_cubic_solids": ((12, 16, 20), "slip", abi.MONOTONIC_CUBIC, True),
    "zout_cubic_solids": ((37, 11, 13), "zout", abi.MONOTONIC_CUBIC, True),
}
STEPS = 4
# normwise max|b200 - reference| / max|reference| per field (measured on a B200: fields <= 3e-6, pressure <= 1.3e-5,
# divergence <= 4.6e-6 of its velocity scale)
TOL = {"default": 1e-5, "divergence": 2e-5, "pressure": 5e-5}


@pytest.fixture(scope="module")
def ref_lib():
    if not os.path.exists(REF_LIBRARY):
        pytest.fail(f"reference library missing: {REF_LIBRARY} (oracle/build_oracle.py builds it)")
    return smoke_b200.SmokeLibrary(REF_LIBRARY, extensions=False)


def _inputs(name):
    shape, boundary, mode, solids = CASES[name]
    cfg = scenes.make_config(*shape, boundary=boundary, mode=mode, pressure_iterations=400)
    inp = scenes.random_inputs(cfg, seed=5, solids=solids)
    for k in ("u", "v", "w"):
        inp.pop(k)
    for k in ("force_x", "force_y", "force_z"):
        inp[k] = (inp[k] * 40.0).astype(np.float32)
    return cfg, inp


@pytest.mark.parametrize("name", list(CASES))
def test_reference_and_b200_agree_through_the_abi(smoke_lib, ref_lib, cuda_stream, name):
    cfg, inp = _inputs(name)
    s_ref = torch.cuda.Stream()
    ref = smoke_b200.Simulation(ref_lib, cfg, s_ref)
    mine = smoke_b200.Simulation(smoke_lib, cfg, cuda_stream)
    k1 = scenes.load_gpu(ref, inp)
    k2 = scenes.load_gpu(mine, inp)
    worst = {}
    for _ in range(STEPS):
        with torch.cuda.stream(s_ref):
            ref.step()
        with torch.cuda.stream(cuda_stream):
            mine.step()
        a = ref.snapshot()
        b = mine.snapshot()
        for k in a:
            if k == "divergence":
                scale = max(np.abs(a[f"velocity_{ax}"]).max() for ax in "xyz") / cfg.cell_size
                e = float(np.abs(a[k] - b[k]).max() / scale) if scale > 0 else float(np.abs(a[k] - b[k]).max())
            else:
                e = scenes.rel_err(b[k], a[k])
            worst[k] = max(worst.get(k, 0.0), e)
    ref.close()
    mine.close()
    del k1, k2
    if REPORT:
        with open(REPORT, "a") as f:
            f.write(json.dumps({"check": f"reference/{name}", "value": worst}) + "\n")
    for k, e in worst.items():
        assert e < TOL.get(k, TOL["default"]), (k, e, worst)
