"""GPU: the multigrid host setup gives the same hierarchy for any host thread count.

The setup's row loops run in fixed chunks claimed by worker threads, with
partial sums combined in chunk order; with MP_VERBOSE the library prints an
FNV-1a checksum of every level's operator and prolongator.  One thread and
eight threads must print the same checksum for the same cloud.
"""
import os
import re
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROG = ("import sys; sys.path.insert(0, %r)\n"
        "from memphys_b200 import meshless\n"
        "meshless.cavity_setup(120, solver_type='cuda_bicgstab_amg')\n") % ROOT


def checksum(threads: int) -> str:
    env = dict(os.environ, MP_VERBOSE="1", MP_HOST_THREADS=str(threads))
    r = subprocess.run([sys.executable, "-c", PROG], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    sums = re.findall(r"hierarchy checksum ([0-9a-f]{16})", r.stderr)
    assert sums, r.stderr[-2000:]
    assert re.search(r"%d host threads" % threads, r.stderr)
    return sums[-1]


def test_hierarchy_independent_of_host_threads(mp_lib):
    assert checksum(1) == checksum(8)
