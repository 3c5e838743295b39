"""The drop-in boundary on CPU: the library builds for sm_100a, loads, and
exports every entry point that include/memphys.h declares (no kernel runs)."""
import os
import re
import subprocess

import numpy as np
import pytest

from memphys_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def built():
    return build.build()


def header_functions():
    src = open(os.path.join(ROOT, "include", "memphys.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(mp_\w+)\s*\(", src)))


def test_header_declares_the_api():
    names = header_functions()
    assert len(names) >= 40
    assert sorted(capi.EXPORTS) == names


def test_library_exports_every_declared_symbol(built):
    out = subprocess.run(["nm", "-D", "--defined-only", built], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\sT\s(mp_\w+)$", out, flags=re.M))
    missing = [n for n in header_functions() if n not in exported]
    assert not missing, missing
    L = capi.lib()
    for n in header_functions():
        assert hasattr(L, n)


def test_header_compiles_as_c(tmp_path):
    f = tmp_path / "t.c"
    f.write_text('#include "memphys.h"\nint main(void){mp_solver_cfg c; (void)c; return 0;}\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    "-c", str(f), "-o", str(tmp_path / "t.o")], check=True)


def test_host_parameter_functions_match_oracle(built):
    import oracle
    L = capi.lib()
    for dim in (2, 3):
        for p in range(2, 8):
            m = L.mp_num_poly_terms(dim, p)
            assert m == oracle.num_poly_terms(dim, p)
            e = np.zeros(m * dim, np.int32)
            assert L.mp_poly_exponents(dim, p, capi.ptr(e)) == capi.MP_OK
            assert np.array_equal(e.reshape(m, dim), oracle.poly_exponents(dim, p))
        assert L.mp_cloud_size(dim, 3, 2.0) == oracle.cloud_size(dim, 3, 2.0)


def test_solver_cfg_layout_matches_header(built):
    cfg = capi.solver_cfg()
    assert cfg.tol == 1e-8 and cfg.maxit == 1000 and cfg.precond == capi.MP_PRECOND_AMG


def test_last_error_is_thread_local_text(built):
    L = capi.lib()
    assert L.mp_poly_exponents(5, 3, None) == capi.MP_BAD_ARG
    assert "mp_poly_exponents" in capi.last_error()
