"""The C-ABI library loads and exports every function include/stmg.h declares;
argument errors come back as status codes. No GPU needed."""
import ctypes as C
import subprocess

import pytest

import stmg


def test_library_exports_every_header_symbol():
    L = stmg.lib()
    names = stmg.header_symbols()
    assert "stmg_op_vmult" in names and len(names) >= 10
    for name in names:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", stmg.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert set(names) <= exported
    # only the C ABI is exported (hidden visibility for everything else)
    assert all(s.startswith("stmg_") or s.startswith("_") or "@" in s for s in exported if " T " in s)


def test_bad_arguments_return_status_codes():
    L = stmg.lib()
    h = C.c_void_p()
    n = (C.c_int * 3)(4, 4, 4)
    lo = (C.c_double * 3)(0, 0, 0)
    hi = (C.c_double * 3)(1, 1, 1)
    assert L.stmg_mesh_create(4, n, 2, lo, hi, None, 0, None, C.byref(h)) == -1  # STMG_ERR_ARG
    assert b"dim" in L.stmg_last_error()
    assert L.stmg_mesh_create(3, n, 7, lo, hi, None, 0, None, C.byref(h)) == -8  # unsupported degree
    assert L.stmg_mesh_create(3, n, 5, lo, hi, None, 0, None, C.byref(h)) == -8  # 3-D degree 5
    assert L.stmg_mesh_create(3, n, 2, lo, hi, None, 1, None, C.byref(h)) == -1  # coefficient missing
    assert L.stmg_op_vmult(None, None, None, None) == -2  # null handle
    assert L.stmg_mesh_destroy(None) == -2
