"""The C ABI library loads and exports exactly what include/phem.h declares
(no GPU needed; no compute calls)."""
import ctypes as C
import re
from pathlib import Path

import pytest

import phem_graph_b200 as P
from phem_graph_b200 import _lib
from tests.conftest import HAVE_GPU

HEADER = Path(__file__).resolve().parent.parent / "include" / "phem.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w \t\*]*?\b(phem_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for needed in ("phem_cc_solve", "phem_cc_stream", "phem_cc_merge", "phem_msf_solve", "phem_msf_solve_device",
                   "phem_msf_solve_csr", "phem_csr_to_coo", "phem_context_create"):
        assert needed in names


def test_library_exports_every_declared_symbol():
    lib = P.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_match_header():
    assert set(_lib.SIGNATURES) == set(declared_functions())


def test_status_strings():
    lib = P.lib()
    for code in range(8):
        assert lib.phem_status_string(code)
    assert lib.phem_version() == 100


def test_null_context_is_invalid():
    lib = P.lib()
    st = lib.phem_cc_solve(None, None, 0, 1, None, None, 0, None)
    assert st == _lib.PHEM_ERR_INVALID
    assert b"context" in lib.phem_last_error()
    for fn, args in (("phem_msf_solve", (None, None, 0, 1, None, None, None, None)),
                     ("phem_msf_stream", (None, None, 0, 1, 16, None, None, None, None))):
        assert getattr(lib, fn)(*args) == _lib.PHEM_ERR_INVALID, fn


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-device error path")
def test_no_device_fails_loudly():
    with pytest.raises(P.PhemError) as e:
        P.Context(0)
    assert e.value.status == _lib.PHEM_ERR_NO_DEVICE


def test_library_is_sm100a_only():
    """The build compiles for sm_100a and nothing else."""
    from phem_graph_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
