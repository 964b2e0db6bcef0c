"""The raycaster's exact fast-forward of repeated float additions (csrc/kf_march.h), compiled
for the host and compared bit for bit with the plain additions on random and edge cases
(binade crossings, increments halfway between ulp multiples, step caps).  CPU only."""
import os
import shutil
import subprocess
import tempfile

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "native", "march_check.cpp")
INC = os.path.join(ROOT, "kinectfusion-cuda_b200", "csrc")


def test_advance_steps_equals_plain_additions():
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "march_check")
        # -ffp-contract=off: plain IEEE single additions, as the device's fadd.rn
        subprocess.run([cxx, "-O2", "-ffp-contract=off", "-std=c++17", "-I", INC, SRC, "-o", exe], check=True)
        out = subprocess.run([exe, "300000"], capture_output=True, text=True)
        assert out.returncode == 0, out.stdout
        assert "mismatches 0" in out.stdout
