"""The FP64 modular arithmetic of the FP64 three-prime form (fp64mod.cuh),
restated in host C (tests/host/fp64mod_check.c) and checked against 128-bit
integer arithmetic on random and boundary inputs for the form's three primes:
results exact and within the ranges the transforms rely on.  The device code
itself is checked bit for bit by the GPU product and pi tests."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_fp64_modular_arithmetic_exact(tmp_path):
    exe = tmp_path / "fp64mod_check"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), os.path.join(HERE, "host", "fp64mod_check.c"),
                    "-lm"], check=True)
    out = subprocess.run([str(exe), "400000"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("bad=0")
    maxr = float(out.stdout.split("maxr=")[1])
    assert maxr <= 0.75
