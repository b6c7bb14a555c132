"""CPU test: the header-only C++ drop-in (include/Helmholtz_CUDA.hpp) compiles
against the C ABI and links with libbaemm_cuda.so."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
@pytest.mark.parametrize("example", ["dropin_example.cpp", "dropin_farfield.cpp"])
def test_dropin_header_compiles_and_links(tmp_path, example):
    from baemm_b200 import _capi
    _capi.lib()   # the library exists
    exe = tmp_path / "dropin"
    cmd = ["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", example), "-L", os.path.join(ROOT, "baemm_b200"),
           "-lbaemm_cuda", f"-Wl,-rpath,{os.path.join(ROOT, 'baemm_b200')}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert exe.exists()
