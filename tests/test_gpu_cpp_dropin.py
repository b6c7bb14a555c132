"""GPU test of the C++ drop-in class (include/Helmholtz_CUDA.hpp) as a user
would run it: tests/cpp/dropin_farfield.cpp replays the reference's example
call sequence (Example_OpenCL/main.cpp:86-233: FarField, Derivative_FF with a
library-allocated du_dn, AdjointDerivative_FF of the derivative) on the
icosphere of level 2 written in the reference's mesh format; its F, DF and
DF^* DF outputs are compared with the CPU oracle within 1e-5."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from baemm_b200 import WaveType, meshes
from oracle import oracle as O
from tests.helpers import relerr

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KAPPA = 5.0 * np.pi     # (1 + 2 (i + 2)) pi for i = 0, Example_OpenCL/main.cpp:104-107
TOL = 1e-5


def _read_complex(path):
    a = np.loadtxt(path, ndmin=2)
    return a[:, 0::2] + 1j * a[:, 1::2]


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_cpp_dropin_example_sequence_matches_oracle(tmp_path):
    coords, tris = meshes.icosphere(2)
    inc = meshes.fibonacci_sphere(16)
    meas = meshes.fibonacci_sphere(64)
    meshes.write_mesh_txt(tmp_path / "mesh.txt", coords, tris)
    np.savetxt(tmp_path / "dirs.txt", inc, fmt="%.17g")
    np.savetxt(tmp_path / "meas.txt", meas, fmt="%.17g")
    exe = tmp_path / "dropin_farfield"
    lib_dir = os.path.join(ROOT, "baemm_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_farfield.cpp"), "-L", lib_dir, "-lbaemm_cuda",
           f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    tol = "1e-10"
    r = subprocess.run([str(exe), str(tmp_path / "mesh.txt"), str(tmp_path / "dirs.txt"), str(tmp_path / "meas.txt"),
                        repr(KAPPA), tol, tol, str(tmp_path / "out_")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    F = _read_complex(tmp_path / "out_F.txt")
    DF = _read_complex(tmp_path / "out_DF.txt")
    DFT = np.loadtxt(tmp_path / "out_DFT.txt", ndmin=2)

    # the same sequence on the FP32 oracle (the reference's arithmetic)
    coords_r, tris_r = meshes.read_mesh_txt(tmp_path / "mesh.txt")
    o = O.Oracle(coords_r, tris_r, meas, precision=32)
    k = np.array([KAPPA])
    Fo = np.zeros((64, 16), complex)
    o.FarField(k, inc, Fo, WaveType.Plane, 1e-10, 1e-10)
    du_o = np.zeros((coords.shape[0], 16), complex)
    o.Derivative_FF_Helper(k, inc, du_o, WaveType.Plane, 1e-10, 1e-10)
    DFo = np.zeros_like(Fo)
    o.Derivative_FF(k, inc, coords_r, DFo, du_o, False, WaveType.Plane, 1e-10, 1e-10)
    Wo = np.zeros((coords.shape[0], 3))
    o.AdjointDerivative_FF(k, inc, DFo, Wo, du_o, False, WaveType.Plane, 1e-10, 1e-10)
    e = (relerr(F, Fo), relerr(DF, DFo), relerr(DFT, Wo))
    print("C++ drop-in vs oracle: F %.2e, DF %.2e, DF^* DF %.2e" % e)
    assert max(e) < TOL
