"""The C++ drop-in classes (include/stmg_dealii.hpp: SystemMatrixGPU,
VankaGPU, STTransferGPU, DofPermutation) driven through the C ABI by a host
C++ program (tests/cpp/shim_test.cc, built by __graft_entry__.build())."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

EXE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp", "build", "shim_test")


def test_cpp_shims():
    if not os.path.exists(EXE):
        import sys
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(EXE)), "..", "..", "dealii-stfem_b200"))
        import build
        build.build_cpp_tests()
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ALL OK" in r.stdout, r.stdout + r.stderr
