"""The oracle against the reference's own outputs (tests/golden/*.npz, made by tests/golden/make_golden.py from
the reference library run on a B200). CPU only.

The reference solves with fixed-count FP32 CG (cuBLAS dots); the oracle's FP32 mirror uses the same iteration
count with double-accumulated dots, so fields agree to FP32 rounding once both CG runs have reached their floor.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
import scenes
import smoke_abi as abi

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))

import importlib.util  # noqa: E402

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)

ORACLE_TO_VIEW = {"density": "density", "temperature": "temperature", "centered_x": "velocity_x", "centered_y": "velocity_y", "centered_z": "velocity_z",
                  "velocity_magnitude": "velocity_magnitude", "pressure": "pressure", "pressure_rhs": "pressure_rhs", "vorticity_x": "vorticity_x",
                  "vorticity_y": "vorticity_y", "vorticity_z": "vorticity_z", "vorticity_magnitude": "vorticity_magnitude"}
# Measured worst case over the four fixtures and both builds: 2.8e-6 (closed_linear_8, pressure).
TOL = 1e-5


def test_golden_fixtures_present():
    assert len(GOLDEN) == len(make_golden.CASES), GOLDEN


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_outputs(path, bits):
    name = os.path.basename(path)[:-4]
    data = np.load(path)
    cfg, generated = make_golden.case_inputs(name)
    inp = {k: data[f"input_{k}"] for k in generated}  # the exact inputs the reference saw
    st = O.OracleState(cfg, bits)
    scenes.load_oracle(st, inp)
    worst = {}
    for s in range(make_golden.STEPS):
        st.step(0, 5, mode=0)
        for o, vname in ORACLE_TO_VIEW.items():
            worst[vname] = max(worst.get(vname, 0.0), scenes.rel_err(st[o], data[f"step{s + 1}_{vname}"]))
        ref_div = data[f"step{s + 1}_divergence"]
        scale = max(np.abs(data[f"step{s + 1}_velocity_{a}"]).max() for a in "xyz") / cfg.cell_size
        worst["divergence"] = max(worst.get("divergence", 0.0), float(np.abs(st["divergence"] - ref_div).max() / scale))
        np.testing.assert_array_equal(data[f"step{s + 1}_occupancy"], inp["occupancy"].astype(np.float32))
    assert max(worst.values()) < TOL, worst
