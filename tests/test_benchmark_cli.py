"""The benchmark CLI (smoke_b200_benchmark) keeps the reference benchmark's interface (benchmark.cu:29-61): every
reference flag, --help, and exit code 1 on an unknown flag or a missing value. Argument handling needs no GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "visual-simulation-of-smoke_b200", "smoke_b200_benchmark")
REFERENCE_FLAGS = ["--nx", "--ny", "--nz", "--warmup", "--steps", "--pressure-iters", "--cell-size", "--dt", "--ambient-temperature", "--buoyancy-density", "--buoyancy-temperature", "--vorticity-confinement",
                   "--linear-advection"]


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        import build_smoke

        build_smoke.build()
    return CLI


def test_help_lists_the_reference_flags(cli):
    out = subprocess.run([cli, "--help"], capture_output=True, text=True)
    assert out.returncode == 0
    for flag in REFERENCE_FLAGS + ["--library", "--solver", "--autotune", "--json"]:
        assert flag in out.stdout, flag


@pytest.mark.parametrize("args,message", [(["--bogus"], "unknown argument: --bogus"), (["--nx"], "missing value for --nx"), (["--steps", "4", "--dt"], "missing value for --dt")])
def test_bad_arguments_fail(cli, args, message):
    out = subprocess.run([cli, *args], capture_output=True, text=True)
    assert out.returncode == 1 and message in out.stderr


def test_missing_library_fails(cli):
    out = subprocess.run([cli, "--library", "/nonexistent/libx.so"], capture_output=True, text=True)
    assert out.returncode == 1 and "cannot load" in out.stderr
