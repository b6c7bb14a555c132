"""Generate tests/golden/refcl_small.npz from the reference's own kernels.

The dense kernels come from oracle/_ref/libbaemm_refcl.so: the reference's
BoundaryOperatorKernel.cl, FarFieldOperatorKernel.cl, HerglotzWaveKernel.cl and
NearFieldOperatorKernel.cl compiled as C++ by oracle/build_ref.sh (block_size 1).
The near-field cases evaluate at 45 seeded points inside, near and outside the
sphere (none on a midpoint).  Inputs are seeded and
small (icosphere level 2: 162 vertices / 320 triangles, 32 far-field
directions), so the fixture is a few hundred KB.  Geometry inputs are the
float32 midpoints/normals of the FP32 oracle restatement, which the CPU tests
separately pin against closed-form properties.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from baemm_b200 import meshes  # noqa: E402
from oracle import oracle as O  # noqa: E402

# (name, coeff per chunk [mass, SL, DL, adjDL], kappa list, wave_count, wave_chunk_size)
BOUNDARY_CASES = [
    ("sl", [0, 1, 0, 0], [2.0], 16, 16),
    ("dl", [0, 0, 1, 0], [2.0], 16, 16),
    ("adl", [0, 0, 0, 1], [2.0], 16, 16),
    ("bie_dl", [0.5, -2.0j, 1, 0], [2.0], 16, 16),
    ("mix_2k", [0, 1 + 0.5j, 1 - 2j, 0.3j], [3.0, 7.5], 32, 16),
    ("wcs4", [0, 0.25j, 1, 1], [1.0, 2.0, 4.0, 8.0], 16, 4),
]
NF_CASES = [
    ("nf_sl", [0, 1, 0, 0], [2.0], 16, 16),
    ("nf_dl", [0, 0, 1, 0], [2.0], 16, 16),
    ("nf_mix", [0.7, 1 + 0.5j, 1 - 2j, 0.3j], [3.0, 7.5], 32, 16),
    ("nf_wcs4", [0, 0.25j, 1, 1], [1.0, 2.0, 4.0, 8.0], 16, 4),
]
FF_CASES = [
    ("ff_sl", [0, 1, 0, 0], [2.0], 16, 16),
    ("ff_mix", [0, -4j, 1, 0], [4.0, 8.0], 32, 16),
]


def main(out_path: str | None = None) -> str:
    coords, tris = meshes.icosphere(2)
    meas = meshes.fibonacci_sphere(32)
    orc = O.Oracle(coords, tris, meas, precision=32)
    mid, nrm, area, diag = orc.geometry()
    mid32, nrm32 = mid.astype(np.float32), nrm.astype(np.float32)
    meas4 = np.zeros((meas.shape[0], 4), np.float32)
    meas4[:, :3] = meas
    rng = np.random.default_rng(1234)
    out = {"coords": coords, "tris": tris, "meas": meas, "mid4": mid32, "nrm4": nrm32,
           "area": area.astype(np.float32), "diag": diag.astype(np.float32)}
    n = tris.shape[0]
    for name, co, kap, wc, wcs in BOUNDARY_CASES:
        B = (rng.standard_normal((n, wc)) + 1j * rng.standard_normal((n, wc))).astype(np.complex64)
        coeff = np.array([co] * len(kap), np.complex128)
        C = O.ref_boundary(mid32, nrm32, B, np.array(kap), O.scaled_coefficients(coeff), wcs)
        out[f"bnd_{name}_B"] = B
        out[f"bnd_{name}_C"] = C
        out[f"bnd_{name}_coeff"] = coeff
        out[f"bnd_{name}_kappa"] = np.array(kap)
        out[f"bnd_{name}_wcs"] = np.array(wcs)
    for name, co, kap, wc, wcs in FF_CASES:
        B = (rng.standard_normal((n, wc)) + 1j * rng.standard_normal((n, wc))).astype(np.complex64)
        coeff = np.array([co] * len(kap), np.complex128)
        C = O.ref_farfield(mid32, nrm32, meas4, B, np.array(kap), O.scaled_coefficients(coeff), wcs)
        out[f"{name}_B"] = B
        out[f"{name}_C"] = C
        out[f"{name}_coeff"] = coeff
        out[f"{name}_kappa"] = np.array(kap)
        out[f"{name}_wcs"] = np.array(wcs)
    # Herglotz wave kernel, coefficients (0, -i k, 1, 0) scaled by 4 pi / m (CreateHerglotzWave.hpp:40)
    kap = np.array([2.0, 5.0])
    coeff = np.array([[0, -1j * k, 1, 0] for k in kap], np.complex128)
    G = (rng.standard_normal((meas.shape[0], 32)) + 1j * rng.standard_normal((meas.shape[0], 32))).astype(np.complex64)
    C = O.ref_herglotz(mid32, nrm32, meas4, G, kap, O.scaled_coefficients(coeff, 4 * np.pi / meas.shape[0]), 16)
    out.update({"hw_G": G, "hw_C": C, "hw_coeff": coeff, "hw_kappa": kap, "hw_wcs": np.array(16)})
    # near field (appended last: the cases above keep their random inputs)
    dirs = rng.standard_normal((45, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    radii = np.tile([0.3, 0.6, 0.9, 1.1, 1.5, 2.5, 4.0, 8.0, 0.05], 5)
    pts = dirs * radii[:, None]
    out["nf_points"] = pts
    for name, co, kap, wc, wcs in NF_CASES:
        B = (rng.standard_normal((n, wc)) + 1j * rng.standard_normal((n, wc))).astype(np.complex64)
        coeff = np.array([co] * len(kap), np.complex128)
        C = O.ref_nearfield(mid32, nrm32, B, pts, np.array(kap), O.scaled_coefficients(coeff), wcs)
        out[f"{name}_B"] = B
        out[f"{name}_C"] = C
        out[f"{name}_coeff"] = coeff
        out[f"{name}_kappa"] = np.array(kap)
        out[f"{name}_wcs"] = np.array(wcs)
    path = out_path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "refcl_small.npz")
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    print(main())
