"""A non-Python caller of the C-ABI: tests/ccall_mirror/ccall_mirror.cpp calls
libefsi.so the way the Julia binding of INTEGRATION.md does (symbols by name, the
ccall argument lists, the 8-field StepReport as the Julia struct lays it out) and
checks three steps of the cavity against the oracle called the same way.  Building it
needs no GPU; running it does."""
import os
import subprocess

import pytest

from eulerianfsi_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "ccall_mirror", "ccall_mirror.cpp")


def _build(tmp_path):
    exe = os.path.join(str(tmp_path), "ccall_mirror")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", SRC, "-o", exe, "-ldl"], check=True)
    return exe


def test_ccall_mirror_builds(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_ccall_mirror_matches_oracle(tmp_path, oracle_lib):
    from oracle import oracle
    exe = _build(tmp_path)
    if not os.path.exists(_abi.LIBRARY_PATH):
        from eulerianfsi_b200 import build
        build.build()
    res = subprocess.run([exe, _abi.LIBRARY_PATH, oracle.LIB_PATH], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "ccall mirror ok" in res.stdout
