"""Generates the golden fixtures of tests/golden/ by running the REFERENCE library (the reference's own
backend-cuda.cu, compiled from its sources into oracle/_ref by oracle/build_oracle.py) on a CUDA device.

Each case: a small grid with seeded inputs for every ABI field (no velocity: the ABI cannot set one, so motion
comes from the forces), stepped from rest through the reference's C ABI; every view is recorded after each step.
The fixtures pin the oracle (tests/test_oracle_golden.py) to the reference's own outputs.

python tests/golden/make_golden.py --out tests/golden   (needs a GPU and oracle/_ref/libvisual-simulation-of-smoke.so)
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "visual-simulation-of-smoke_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import scenes  # noqa: E402
import smoke_abi as abi  # noqa: E402

REF_LIBRARY = os.path.join(ROOT, "oracle", "_ref", "libvisual-simulation-of-smoke.so")

# name -> (shape, boundary, mode, solids, seed)
CASES = {
    "closed_linear_8": ((8, 8, 8), "closed", abi.LINEAR, False, 21),
    "plume_cubic_solids": ((10, 8, 6), "plume", abi.MONOTONIC_CUBIC, True, 22),
    "mixed_linear_solids": ((9, 7, 8), "mixed", abi.LINEAR, True, 23),
    "slip_cubic_solids": ((8, 6, 10), "slip", abi.MONOTONIC_CUBIC, True, 24),
}
STEPS = 2
PRESSURE_ITERATIONS = 200
FORCE_SCALE = 40.0


def case_inputs(name):
    shape, boundary, mode, solids, seed = CASES[name]
    cfg = scenes.make_config(*shape, boundary=boundary, mode=mode, pressure_iterations=PRESSURE_ITERATIONS)
    inp = scenes.random_inputs(cfg, seed=seed, solids=solids)
    for k in ("u", "v", "w"):
        inp.pop(k)
    for k in ("force_x", "force_y", "force_z"):
        inp[k] = (inp[k] * FORCE_SCALE).astype(np.float32)
    return cfg, inp


def run_case(lib, name, stream):
    import torch

    import smoke_b200

    cfg, inp = case_inputs(name)
    sim = smoke_b200.Simulation(lib, cfg, stream)
    keep = scenes.load_gpu(sim, inp)
    out = {f"input_{k}": v for k, v in inp.items()}
    for s in range(STEPS):
        with torch.cuda.stream(stream):
            sim.step()
        snap = sim.snapshot()
        for k, v in snap.items():
            out[f"step{s + 1}_{k}"] = v
    sim.close()
    del keep
    return out


def main():
    import smoke_b200

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    import torch

    lib = smoke_b200.SmokeLibrary(REF_LIBRARY, extensions=False)
    stream = torch.cuda.Stream()
    os.makedirs(args.out, exist_ok=True)
    for name in CASES:
        data = run_case(lib, name, stream)
        np.savez_compressed(os.path.join(args.out, f"{name}.npz"), **data)
        print(name, "ok", len(data), "arrays")


if __name__ == "__main__":
    main()
