"""The C++ host path: the reference-style driver calls CUDA only through the
C ABI (memphys_b200/host/memphys.hpp over include/memphys.h)."""
import os
import subprocess

import pytest

from memphys_b200 import build

pytestmark = pytest.mark.gpu


def test_cpp_cavity_driver_runs(mp_lib):
    exe = build.build_host_driver()
    r = subprocess.run([exe, "32", "6", "1e-4"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert len([ln for ln in lines if ln.startswith("step ")]) == 6
    last = lines[-1]
    assert last.startswith("OK")
    umax = float(last.split("max|u|=")[1].split()[0])
    assert 0.99 <= umax <= 1.0 + 1e-9  # the lid speed bounds the flow
