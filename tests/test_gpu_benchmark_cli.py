"""The benchmark CLI on the GPU: the reference benchmark's two output lines, the same scene whichever library runs it
(`--library`: the reference's own build gives the same total and peak density as this library in the reference's
solver mode), and this library's solvers (`--solver`, `--json`)."""
import json
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "visual-simulation-of-smoke_b200", "smoke_b200_benchmark")
REF = os.path.join(ROOT, "oracle", "_ref", "libvisual-simulation-of-smoke.so")
SMALL = ["--nx", "32", "--ny", "40", "--nz", "32", "--warmup", "3", "--steps", "6"]


def run(*args):
    out = subprocess.run([CLI, *SMALL, *args], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    assert lines[0].startswith("benchmark grid=32x40x32 warmup=3 steps=6 ")
    timing = dict(kv.split("=") for kv in lines[1].split()[1:])
    return {k: float(v) for k, v in timing.items()}, lines


def test_output_lines():
    t, lines = run()
    assert set(t) == {"total_ms", "avg_step_ms", "mlups", "total_density", "peak_density"}
    assert t["avg_step_ms"] > 0 and t["total_density"] > 0 and t["peak_density"] > 0
    assert re.search(r"advection=monotonic_cubic$", lines[0])


@pytest.mark.skipif(not os.path.exists(REF), reason="the reference's library is not built")
@pytest.mark.parametrize("extra", [[], ["--linear-advection"]], ids=["cubic", "linear"])
def test_reference_library_gives_the_same_scene(extra):
    ours, _ = run(*extra)
    ref, _ = run("--library", REF, *extra)
    assert abs(ours["total_density"] - ref["total_density"]) <= 1e-4 * ref["total_density"]
    assert abs(ours["peak_density"] - ref["peak_density"]) <= 1e-4 * ref["peak_density"]


def test_solvers_and_json():
    _, lines = run("--solver", "multigrid", "--tolerance", "1e-6", "--autotune", "--json")
    rec = json.loads(lines[2])
    assert rec["solver"] == "multigrid" and rec["status"] == 0 and 0 < rec["true_relative_residual"] <= 1e-6
