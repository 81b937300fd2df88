"""The C++ drop-in API (include/hbdia/*.hpp) used the way the reference's own
programs use theirs (tests/cpp/test_dropin.cpp)."""
import subprocess

import pytest

pytestmark = pytest.mark.gpu


def test_cpp_dropin_program(lib):
    from hbdia_b200 import build
    exe = build.build_cpp_tests()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASSED" in r.stdout
