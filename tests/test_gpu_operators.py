"""GPU parity of the operator applies against the oracle (through the C ABI).

Tolerances: the plain FP32 and the compensated tensor-core forms within 1e-5
relative (Frobenius) of the FP32 oracle and of the FP64 oracle; FP64 path
within 1e-11 of the FP64 oracle.  (Measured on the icosphere of level 3: at
most 1.6e-6 against the FP64 oracle for every operator combination.)
"""
import numpy as np
import pytest

from baemm_b200 import APPLY_FP32, APPLY_FP64, APPLY_TC, BaemmError, Helmholtz_CUDA, WaveType, _capi, meshes
from oracle import oracle as O
from tests.helpers import crandn, relerr, tiny_meshes

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5
FP32_VS64_TOL = 1e-5
FP64_TOL = 1e-11

COEFFS = {
    "mass": [1.5 - 0.5j, 0, 0, 0],
    "sl": [0, 1, 0, 0],
    "dl": [0, 0, 1, 0],
    "adl": [0, 0, 0, 1],
    "bie": [0.5, -1j, 1, 0],
    "dtn": [0.5, -1j, 0, 1],
    "all": [0.25 + 1j, 1 + 0.5j, 1 - 2j, 0.3j],
}
WAVES = {  # name: (wave_count, wave_chunk_size, kappa list)
    "w16": (16, 16, [2.0]),
    "w32": (32, 16, [4.0, 8.0]),
    "w8x4": (8, 4, [1.0, 3.0]),
    "w64": (64, 16, [2.0, 4.0, 8.0, 16.0]),
    "w64x32": (64, 32, [3.0, 6.0]),
}


@pytest.fixture(scope="module")
def env():
    coords, tris = meshes.icosphere(3)
    meas = meshes.fibonacci_sphere(48)
    H = Helmholtz_CUDA(coords, tris, meas)
    o32 = O.Oracle(coords, tris, meas, precision=32)
    o64 = O.Oracle(coords, tris, meas, precision=64)
    yield coords, tris, meas, H, o32, o64
    H.close()


def _coeff(name, kap):
    return np.array([COEFFS[name] if name != "bie" else [0.5, -1j * k, 1, 0] for k in kap], np.complex128)


def test_geometry_matches_oracle(env):
    coords, tris, meas, H, o32, o64 = env
    mid, nrm, area, diag = o32.geometry()
    assert relerr(H.Areas(), area) < 1e-6
    assert relerr(H.TriangleMidpoints(), mid) < 1e-6
    assert relerr(H.TriangleNormals(), nrm) < 1e-6
    assert relerr(H.SingleLayerDiagonal(), diag) < 1e-5
    assert H.VertexCount() == coords.shape[0] and H.SimplexCount() == tris.shape[0]
    assert H.GetMeasCount() == meas.shape[0]
    assert H.ClassName() == "Helmholtz_CUDA"
    assert "DEVICE_NAME" in H.DeviceInfo()


def test_mass_matrix_matches_oracle(env):
    coords, tris, meas, H, o32, o64 = env
    go, gi, gv = H.MassMatrix()
    oo, oi, ov = o32.mass_matrix()
    assert np.array_equal(go, oo) and np.array_equal(gi, oi)
    assert relerr(gv, ov) < 1e-6


@pytest.mark.parametrize("cname", list(COEFFS))
@pytest.mark.parametrize("wname", ["w16", "w32", "w8x4"])
def test_apply_boundary_fp32(env, cname, wname):
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES[wname]
    coeff = _coeff(cname, kap)
    rng = np.random.default_rng(hash((cname, wname)) % 2**32)
    nv = coords.shape[0]
    B = crandn(rng, nv, wc + 3)          # ld > wave_count
    C0 = crandn(rng, nv, wc + 1)
    alpha, beta = 0.7 - 0.2j, 0.3 + 0.1j
    Cg = C0.copy()
    H.SetApplyMode(APPLY_FP32)
    H.ApplyBoundaryOperators_PL(alpha, B, beta, Cg, kap, coeff, wc, wcs)
    C32 = C0.copy()
    o32.ApplyBoundaryOperators_PL(alpha, B, beta, C32, kap, coeff, wc, wcs)
    C64 = C0.copy()
    o64.ApplyBoundaryOperators_PL(alpha, B, beta, C64, kap, coeff, wc, wcs)
    assert relerr(Cg[:, :wc], C32[:, :wc]) < FP32_TOL
    assert relerr(Cg[:, :wc], C64[:, :wc]) < FP32_VS64_TOL
    assert np.array_equal(Cg[:, wc:], C0[:, wc:])   # columns beyond wave_count untouched


@pytest.mark.parametrize("cname", ["sl", "dl", "adl", "all"])
@pytest.mark.parametrize("wname", ["w16", "w64", "w64x32"])
def test_apply_boundary_fp64(env, cname, wname):
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES[wname]
    coeff = _coeff(cname, kap)
    rng = np.random.default_rng(17)
    B = crandn(rng, coords.shape[0], wc)
    Cg = np.zeros_like(B)
    H.SetApplyMode(APPLY_FP64)
    try:
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, Cg, kap, coeff, wc, wcs)
    finally:
        H.SetApplyMode(APPLY_FP32)
    C64 = np.zeros_like(B)
    o64.ApplyBoundaryOperators_PL(1.0, B, 0.0, C64, kap, coeff, wc, wcs)
    assert relerr(Cg, C64) < FP64_TOL


@pytest.mark.parametrize("cname", ["sl", "dl", "adl", "bie", "dtn", "all"])
@pytest.mark.parametrize("wname", ["w16", "w32", "w64"])
def test_apply_boundary_tensor_core(env, cname, wname):
    """Compensated tensor-core form (TF32 hi/lo, FP32 accumulation): within
    1e-5 of the FP64 oracle (the same bar as the FP32 path)."""
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES[wname]
    coeff = _coeff(cname, kap)
    rng = np.random.default_rng(41)
    B = crandn(rng, coords.shape[0], wc + 2)
    C0 = crandn(rng, coords.shape[0], wc)
    Cg = C0.copy()
    H.SetApplyMode(APPLY_TC)
    try:
        H.ApplyBoundaryOperators_PL(0.5 - 1j, B, 0.25, Cg, kap, coeff, wc, wcs)
    finally:
        H.SetApplyMode(APPLY_FP32)
    C64, C32 = C0.copy(), C0.copy()
    o64.ApplyBoundaryOperators_PL(0.5 - 1j, B, 0.25, C64, kap, coeff, wc, wcs)
    o32.ApplyBoundaryOperators_PL(0.5 - 1j, B, 0.25, C32, kap, coeff, wc, wcs)
    assert relerr(Cg, C64) < FP32_VS64_TOL
    assert relerr(Cg, C32) < FP32_VS64_TOL


@pytest.mark.parametrize("ctas", [1, 3, 7, 61, 148, 60000])
@pytest.mark.parametrize("wshape", [(64, [2.0, 4.0, 8.0, 16.0]), (48, [1.0, 5.0, 9.0]),
                                    (128, [1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0])])
def test_tensor_core_persistent_grid(env, ctas, wshape):
    """The persistent tensor-core grid splits target blocks between CTAs at any
    grid size (1 CTA, odd sizes, one 16-source tile per CTA); the split blocks
    are summed by the fix-up pass.  Same bar as the FP32 path against the FP64
    oracle, and repeated calls are bitwise identical at a fixed grid size."""
    coords, tris, meas, H, o32, o64 = env
    wc, kap = wshape
    coeff = _coeff("all", kap)
    rng = np.random.default_rng(1234 + wc)
    B = crandn(rng, coords.shape[0], wc)
    C64 = np.zeros_like(B)
    o64.ApplyBoundaryOperators_PL(1.0, B, 0.0, C64, kap, coeff, wc, 16)
    H.SetApplyMode(APPLY_TC)
    H.SetTuning(_capi.TUNE_TC_CTAS, ctas)
    try:
        assert H.GetTuning(_capi.TUNE_TC_CTAS) == ctas
        C1, C2 = np.zeros_like(B), np.zeros_like(B)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C1, kap, coeff, wc, 16)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C2, kap, coeff, wc, 16)
    finally:
        H.SetTuning(_capi.TUNE_TC_CTAS, 0)
        H.SetApplyMode(APPLY_FP32)
    assert relerr(C1, C64) < FP32_VS64_TOL
    assert np.array_equal(C1, C2)


@pytest.mark.parametrize("wc,wcs,kap", [(64, 32, [3.0, 6.0]), (128, 64, [2.0, 5.0]), (32, 32, [4.0])])
def test_tensor_core_wider_chunks(env, wc, wcs, kap):
    """wave_chunk_size a multiple of 16 (the Gauss-Newton configuration uses
    32): the tensor-core form runs each wavenumber over its 16-column groups."""
    coords, tris, meas, H, o32, o64 = env
    coeff = _coeff("all", kap)
    B = crandn(np.random.default_rng(5 + wc), coords.shape[0], wc)
    C64 = np.zeros_like(B)
    o64.ApplyBoundaryOperators_PL(1.0, B, 0.0, C64, kap, coeff, wc, wcs)
    H.SetApplyMode(APPLY_TC)
    try:
        C = np.zeros_like(B)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C, kap, coeff, wc, wcs)
    finally:
        H.SetApplyMode(APPLY_FP32)
    assert relerr(C, C64) < FP32_VS64_TOL


@pytest.mark.parametrize("stagger", [-1, 0, 3, 1000])
def test_tensor_core_sweep_stagger(env, stagger):
    """Rotating the source-tile order of whole-block pieces (the sweep
    stagger) changes only the summation order: same bar against FP64."""
    coords, tris, meas, H, o32, o64 = env
    kap = [2.0, 4.0, 8.0, 16.0]
    coeff = _coeff("all", kap)
    B = crandn(np.random.default_rng(99), coords.shape[0], 64)
    C64 = np.zeros_like(B)
    o64.ApplyBoundaryOperators_PL(1.0, B, 0.0, C64, kap, coeff, 64, 16)
    H.SetApplyMode(APPLY_TC)
    H.SetTuning(_capi.TUNE_TC_CTAS, 3)
    H.SetTuning(_capi.TUNE_TC_STAGGER, stagger)
    try:
        C = np.zeros_like(B)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C, kap, coeff, 64, 16)
    finally:
        H.SetTuning(_capi.TUNE_TC_STAGGER, 0)
        H.SetTuning(_capi.TUNE_TC_CTAS, 0)
        H.SetApplyMode(APPLY_FP32)
    assert relerr(C, C64) < FP32_VS64_TOL


@pytest.mark.parametrize("mode", [APPLY_TC, APPLY_FP32])
def test_autotune_keeps_results(env, mode):
    """The autotuner times its candidates (tensor-core form: generator warps x
    chunk groups per unit, then segment lengths), keeps the fastest in the
    context -- no slower than the setting in force before, up to timing noise
    -- and the apply with the chosen setting meets the same bar against FP64.
    A second call with the same problem key takes the cached choice."""
    coords, tris, meas, H, o32, o64 = env
    kap = [2.0, 4.0, 8.0, 16.0]
    coeff = _coeff("bie", kap)
    B = crandn(np.random.default_rng(3), coords.shape[0], 64)
    C64 = np.zeros_like(B)
    o64.ApplyBoundaryOperators_PL(1.0, B, 0.0, C64, kap, coeff, 64, 16)
    H.LoadBoundaryOperators_PL(kap, coeff, 64, 16)
    keys = (_capi.TUNE_TC_SEGMENT, _capi.TUNE_DENSE_VARIANT, _capi.TUNE_TC_GEN_WARPS, _capi.TUNE_TC_CHUNKS)
    saved = {k: H.GetTuning(k) for k in keys}
    H._lib.baemm_autotune_forget()
    try:
        r = H.Autotune(mode, repeats=2)
        assert r["apply_mode"] == mode and r["cached"] == 0
        assert 0 < r["best_ms"] <= r["before_ms"] * 1.05
        if mode == APPLY_TC:
            # 16 and 8 generator warps x 4, 2 and 1 chunk groups, then segments 8 and 32
            assert r["candidates"] == 8 and r["tc_segment"] in (8, 16, 32)
            assert r["tc_gen_warps"] in (8, 16) and r["tc_chunks"] in (1, 2, 4)
            assert H.GetTuning(_capi.TUNE_TC_SEGMENT) == r["tc_segment"]
            assert H.GetTuning(_capi.TUNE_TC_GEN_WARPS) == r["tc_gen_warps"]
        else:
            assert r["candidates"] == 3 and H.GetTuning(_capi.TUNE_DENSE_VARIANT) == r["dense_variant"]
        again = H.Autotune(mode, repeats=2)
        assert again["cached"] == 1 and again["best_ms"] == r["best_ms"]
        H.SetApplyMode(mode)
        C = np.zeros_like(B)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C)
    finally:
        H.SetApplyMode(APPLY_FP32)
        for k, v in saved.items():
            H.SetTuning(k, v)
        H.UnloadBoundaryOperators_PL()
        H._lib.baemm_autotune_forget()
    assert relerr(C, C64) < FP32_VS64_TOL


@pytest.mark.parametrize("gw", [8, 16])
@pytest.mark.parametrize("chunks", [1, 2, 4])
@pytest.mark.parametrize("cname", ["bie", "dtn", "all"])
def test_tensor_core_shapes_same_results(env, gw, chunks, cname):
    """Every generator-warp count and chunk grouping the tuner may pick gives
    the apply within the bar of the FP64 oracle (and the same result up to
    FP32 rounding)."""
    coords, tris, meas, H, o32, o64 = env
    kap = [2.0, 3.0, 5.0, 7.5]
    coeff = _coeff(cname, kap)
    B = crandn(np.random.default_rng(5), coords.shape[0], 64)
    C64 = np.zeros_like(B)
    o64.ApplyBoundaryOperators_PL(1.0, B, 0.0, C64, kap, coeff, 64, 16)
    H.SetApplyMode(APPLY_TC)
    H.SetTuning(_capi.TUNE_TC_GEN_WARPS, gw)
    H.SetTuning(_capi.TUNE_TC_CHUNKS, chunks)
    try:
        C = np.zeros_like(B)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C, kap, coeff, 64, 16)
    finally:
        H.SetTuning(_capi.TUNE_TC_GEN_WARPS, 16)
        H.SetTuning(_capi.TUNE_TC_CHUNKS, 0)
        H.SetApplyMode(APPLY_FP32)
    assert relerr(C, C64) < FP32_VS64_TOL


# (wave_count, wave_chunk_size, kappas, operator tuple, generator warps,
#  chunks setting, share setting, CTAs, groups per shared entry set)
SHARED_CASES = [
    (64, 64, [3.0], "bie", 16, 0, 4, 0, 4),
    (64, 16, [3.0] * 4, "bie", 16, 0, 4, 0, 4),     # equal wavenumbers in separate wave chunks
    (64, 32, [3.0, 5.0], "dtn", 16, 0, 4, 0, 2),
    (64, 64, [3.0], "bie3", 16, 0, 4, 0, 4),        # all three layers in the KI form
    (64, 64, [3.0], "bie", 8, 0, 4, 0, 4),
    (64, 64, [3.0], "bie", 16, 2, 4, 0, 2),
    (64, 64, [3.0], "bie", 16, 0, 2, 0, 2),
    (64, 64, [3.0], "bie", 16, 0, 1, 0, 1),
    (128, 64, [2.0, 5.0], "bie", 16, 0, 4, 3, 4),   # 3 CTAs: whole blocks, several segments each
    (128, 64, [2.0, 5.0], "dtn", 8, 0, 4, 7, 4),
    (32, 32, [4.0], "bie", 16, 0, 4, 0, 2),
    (48, 16, [4.0] * 3, "bie", 16, 0, 4, 0, 1),     # 3 groups of one wavenumber: one group per unit
    (64, 64, [3.0], "all", 16, 0, 4, 0, 1),         # not the KI form
]


@pytest.mark.parametrize("case", SHARED_CASES)
def test_tensor_core_shared_entries(env, case):
    """Groups of 16 columns with one wavenumber share one evaluation of the
    kernel entries (KI coefficient form): one MMA of N = 64 R per shared set.
    Within the bar of the FP64 oracle, and within 1e-6 of the same apply with
    every group evaluated on its own."""
    wc, wcs, kap, cname, gw, chunks, share, ctas, expect = case
    coords, tris, meas, H, o32, o64 = env
    # c1 = -i kappa with real common c2, c3: the KI form (not for "all")
    layers = {"bie": (1, 0), "dtn": (0, 1), "bie3": (1, 0.5)}
    if cname in layers:
        coeff = np.array([[0.5, -1j * k, *layers[cname]] for k in kap], np.complex128)
    else:
        coeff = _coeff(cname, kap)
    rng = np.random.default_rng(71 + wc + gw + share)
    B = crandn(rng, coords.shape[0], wc)
    C64 = np.zeros_like(B)
    o64.ApplyBoundaryOperators_PL(1.0, B, 0.0, C64, kap, coeff, wc, wcs)
    H.LoadBoundaryOperators_PL(kap, coeff, wc, wcs)
    H.SetApplyMode(APPLY_TC)
    try:
        H.SetTuning(_capi.TUNE_TC_GEN_WARPS, gw)
        H.SetTuning(_capi.TUNE_TC_CHUNKS, chunks)
        H.SetTuning(_capi.TUNE_TC_CTAS, ctas)
        H.SetTuning(_capi.TUNE_TC_SHARE, share)
        assert H.GetTuning(_capi.TUNE_TC_SHARE) == share
        assert H.TcEntrySharing() == expect
        C = np.zeros_like(B)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C)
        H.SetTuning(_capi.TUNE_TC_SHARE, 1)
        assert H.TcEntrySharing() == 1
        C1 = np.zeros_like(B)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C1)
        with pytest.raises(BaemmError):
            H.SetTuning(_capi.TUNE_TC_SHARE, 3)
    finally:
        H.SetTuning(_capi.TUNE_TC_GEN_WARPS, 16)
        H.SetTuning(_capi.TUNE_TC_CHUNKS, 0)
        H.SetTuning(_capi.TUNE_TC_CTAS, 0)
        H.SetTuning(_capi.TUNE_TC_SHARE, 4)
        H.SetApplyMode(APPLY_FP32)
        H.UnloadBoundaryOperators_PL()
    assert relerr(C, C64) < FP32_VS64_TOL
    assert relerr(C1, C64) < FP32_VS64_TOL
    assert relerr(C, C1) < 1e-6


@pytest.mark.parametrize("seg", [1, 2, 3, 5, 64])
@pytest.mark.parametrize("kap,share", [([3.0], 4), ([3.0], 1), ([2.0, 5.0], 4)])
@pytest.mark.parametrize("ctas", [0, 3])
def test_tensor_core_segment_lengths(env, seg, kap, share, ctas):
    """TMEM partial sums drained every `seg` tiles, including segments shorter
    than the ring of A stages (a segment's drain can then still be pending
    when the next one ends) and longer than a CTA's piece: same bar against
    the FP64 oracle."""
    coords, tris, meas, H, o32, o64 = env
    wc, wcs = 64, 64 // len(kap)
    coeff = np.array([[0.5, -1j * k, 1, 0] for k in kap], np.complex128)
    B = crandn(np.random.default_rng(900 + seg), coords.shape[0], wc)
    C64 = np.zeros_like(B)
    o64.ApplyBoundaryOperators_PL(1.0, B, 0.0, C64, kap, coeff, wc, wcs)
    H.LoadBoundaryOperators_PL(kap, coeff, wc, wcs)
    H.SetApplyMode(APPLY_TC)
    try:
        H.SetTuning(_capi.TUNE_TC_SEGMENT, seg)
        H.SetTuning(_capi.TUNE_TC_SHARE, share)
        H.SetTuning(_capi.TUNE_TC_CTAS, ctas)
        C = np.zeros_like(B)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C)
    finally:
        H.SetTuning(_capi.TUNE_TC_SEGMENT, 16)
        H.SetTuning(_capi.TUNE_TC_SHARE, 4)
        H.SetTuning(_capi.TUNE_TC_CTAS, 0)
        H.SetApplyMode(APPLY_FP32)
        H.UnloadBoundaryOperators_PL()
    assert relerr(C, C64) < FP32_VS64_TOL


def test_device_path_follows_torch_stream(env):
    """Without SetStream, torch CUDA tensors are processed on torch's current
    stream, so reading the result back through torch needs no extra sync."""
    import torch
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES["w64"]
    coeff = _coeff("bie", kap)
    B = crandn(np.random.default_rng(77), coords.shape[0], wc)
    ref = np.zeros_like(B)
    o32.ApplyBoundaryOperators_PL(1.0, B, 0.0, ref, kap, coeff, wc, wcs)
    H.LoadBoundaryOperators_PL(kap, coeff, wc, wcs)
    try:
        for mode in (APPLY_FP32, APPLY_TC):
            H.SetApplyMode(mode)
            for stream in (torch.cuda.current_stream(), torch.cuda.Stream()):
                with torch.cuda.stream(stream):
                    Bd = torch.from_numpy(B).to("cuda", non_blocking=True)
                    Cd = torch.full_like(Bd, float("nan"))
                    H.ApplyBoundaryOperators_PL(1.0, Bd, 0.0, Cd)
                    out = Cd.cpu().numpy()   # synchronises torch's stream only
                assert relerr(out, ref) < FP32_VS64_TOL
    finally:
        H.SetApplyMode(APPLY_FP32)
        H.UnloadBoundaryOperators_PL()
        H.SetStream(None)


def test_apply_complex64_and_device_paths(env):
    import torch
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES["w32"]
    coeff = _coeff("all", kap)
    rng = np.random.default_rng(5)
    B = crandn(rng, coords.shape[0], wc)
    ref = np.zeros_like(B)
    o32.ApplyBoundaryOperators_PL(1.0, B, 0.0, ref, kap, coeff, wc, wcs)
    # complex64 host blocks (the reference's Complex)
    C64h = np.zeros(B.shape, np.complex64)
    H.ApplyBoundaryOperators_PL(1.0, B.astype(np.complex64), 0.0, C64h, kap, coeff, wc, wcs)
    assert relerr(C64h, ref) < FP32_TOL
    # device-resident torch tensors, loaded operators (Load / Apply / Unload)
    H.LoadBoundaryOperators_PL(kap, coeff, wc, wcs)
    Bd = torch.from_numpy(B).cuda()
    Cd = torch.zeros_like(Bd)
    H.SetStream(torch.cuda.current_stream().cuda_stream)
    H.ApplyBoundaryOperators_PL(1.0, Bd, 0.0, Cd)
    torch.cuda.synchronize()
    H.SetStream(None)
    H.UnloadBoundaryOperators_PL()
    assert relerr(Cd.cpu().numpy(), ref) < FP32_TOL


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("cname", ["bie", "all"])
def test_dense_kernel_variants(env, variant, cname):
    """Every plain FP32 dense-kernel variant (scalar, packed x1, packed x2) matches the oracle."""
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES["w64x32"]
    coeff = _coeff(cname, kap)
    B = crandn(np.random.default_rng(31), coords.shape[0], wc)
    Cg, Co = np.zeros_like(B), np.zeros_like(B)
    H.SetKernelVariant(variant)
    try:
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, Cg, kap, coeff, wc, wcs)
    finally:
        H.SetKernelVariant(0)
    o32.ApplyBoundaryOperators_PL(1.0, B, 0.0, Co, kap, coeff, wc, wcs)
    assert relerr(Cg, Co) < FP32_TOL


def test_apply_is_deterministic(env):
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES["w32"]
    coeff = _coeff("bie", kap)
    B = crandn(np.random.default_rng(1), coords.shape[0], wc)
    C1, C2 = np.zeros_like(B), np.zeros_like(B)
    H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C1, kap, coeff, wc, wcs)
    H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C2, kap, coeff, wc, wcs)
    assert np.array_equal(C1, C2)


def test_use_diagonal_off(env):
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES["w16"]
    coeff = _coeff("sl", kap)
    B = crandn(np.random.default_rng(2), coords.shape[0], wc)
    Cg, Co = np.zeros_like(B), np.zeros_like(B)
    H.UseDiagonal(False)
    o32.UseDiagonal(False)
    try:
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, Cg, kap, coeff, wc, wcs)
        o32.ApplyBoundaryOperators_PL(1.0, B, 0.0, Co, kap, coeff, wc, wcs)
    finally:
        H.UseDiagonal(True)
        o32.UseDiagonal(True)
    assert relerr(Cg, Co) < FP32_TOL


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_FP64])
@pytest.mark.parametrize("cname", ["sl", "dl", "bie"])
def test_far_field(env, mode, cname):
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES["w32"]
    coeff = _coeff(cname, kap)
    rng = np.random.default_rng(9)
    B = crandn(rng, coords.shape[0], wc)
    F0 = crandn(rng, meas.shape[0], wc)
    Fg = F0.copy()
    H.SetApplyMode(mode)
    try:
        H.ApplyFarFieldOperators_PL(0.5 + 0.5j, B, -0.25, Fg, kap, coeff, wc, wcs)
    finally:
        H.SetApplyMode(APPLY_FP32)
    Fo = F0.copy()
    (o32 if mode == APPLY_FP32 else o64).ApplyFarFieldOperators_PL(0.5 + 0.5j, B, -0.25, Fo, kap, coeff, wc, wcs)
    assert relerr(Fg, Fo) < (FP32_TOL if mode == APPLY_FP32 else FP64_TOL)


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_FP64])
def test_herglotz_wave(env, mode):
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES["w32"]
    coeff = np.array([[0, -1j * k, 1, 0] for k in kap])
    rng = np.random.default_rng(10)
    g = crandn(rng, meas.shape[0], wc)
    Cg, Co = np.zeros((coords.shape[0], wc), complex), np.zeros((coords.shape[0], wc), complex)
    H.SetApplyMode(mode)
    try:
        H.CreateHerglotzWave_PL(1.0, g, 0.0, Cg, kap, coeff, wc, wcs)
    finally:
        H.SetApplyMode(APPLY_FP32)
    (o32 if mode == APPLY_FP32 else o64).CreateHerglotzWave_PL(1.0, g, 0.0, Co, kap, coeff, wc, wcs)
    assert relerr(Cg, Co) < (FP32_TOL if mode == APPLY_FP32 else FP64_TOL)


@pytest.mark.parametrize("wtype", [WaveType.Plane, WaveType.Radial])
@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_FP64])
def test_incident_wave(env, wtype, mode):
    coords, tris, meas, H, o32, o64 = env
    wc, wcs, kap = WAVES["w32"]
    coeff = np.array([[0, -1j * k, 1, 0] for k in kap])
    dirs = meshes.fibonacci_sphere(wcs) * (2.5 if wtype == WaveType.Radial else 1.0)
    C0 = crandn(np.random.default_rng(3), coords.shape[0], wc)
    Cg, Co = C0.copy(), C0.copy()
    H.SetApplyMode(mode)
    try:
        H.CreateIncidentWave_PL(1.0 - 1j, dirs, 0.5, Cg, kap, coeff, wc, wcs, wtype)
    finally:
        H.SetApplyMode(APPLY_FP32)
    (o32 if mode == APPLY_FP32 else o64).CreateIncidentWave_PL(1.0 - 1j, dirs, 0.5, Co, kap, coeff, wc, wcs, wtype)
    assert relerr(Cg, Co) < (FP32_TOL if mode == APPLY_FP32 else FP64_TOL)


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_FP64])
@pytest.mark.parametrize("wtype", [WaveType.Plane, WaveType.Radial])
def test_wave_overloads_with_loaded_parameters(env, mode, wtype):
    """The reference's second CreateIncidentWave_PL / CreateHerglotzWave_PL
    overloads (CreateIncidentWave.hpp:55-124, CreateHerglotzWave.hpp:51-95) use
    the loaded parameters; after LoadParameters with the factor the first
    overloads use (4 pi, 4 pi / meas_count) they give the same blocks bit for
    bit.  With nothing loaded they leave C_out untouched."""
    coords, tris, meas, H, o32, o64 = env
    nv = coords.shape[0]
    wc, wcs, kap = WAVES["w32"]
    coeff = np.array([[0, -1j * k, 1, 0] for k in kap])
    rng = np.random.default_rng(14)
    dirs = meshes.fibonacci_sphere(wcs) * (2.5 if wtype == WaveType.Radial else 1.0)
    g = crandn(rng, meas.shape[0], wc)
    C0 = crandn(rng, nv, wc)
    H.SetApplyMode(mode)
    try:
        I1, I2 = C0.copy(), C0.copy()
        H.CreateIncidentWave_PL(1.0 - 1j, dirs, 0.5, I1, kap, coeff, wc, wcs, wtype)
        H.LoadParameters(kap, coeff, wc, wcs, 4 * np.pi)
        H.CreateIncidentWave_PL(1.0 - 1j, dirs, 0.5, I2, wtype)
        G1, G2 = C0.copy(), C0.copy()
        H.CreateHerglotzWave_PL(0.5, g, -1.0, G1, kap, coeff, wc, wcs)
        H.LoadParameters(kap, coeff, wc, wcs, 4 * np.pi / meas.shape[0])
        H.CreateHerglotzWave_PL(0.5, g, -1.0, G2)
    finally:
        H.SetApplyMode(APPLY_FP32)
    assert np.array_equal(I1, I2) and np.array_equal(G1, G2)
    assert relerr(I1, C0) > 1e-3 and relerr(G1, C0) > 1e-3
    fresh = Helmholtz_CUDA(coords, tris, meas)
    try:
        C = C0.copy()
        fresh.CreateIncidentWave_PL(1.0, dirs, 0.0, C, wtype)
        fresh.CreateHerglotzWave_PL(1.0, g, 0.0, C)
        assert np.array_equal(C, C0)
    finally:
        fresh.close()


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_FP64])
def test_mass_inverse_and_lumped(env, mode):
    """CG mass inverse (20 iterations max).  The FP32 path uses the float mass
    values of the reference (Sparse_T<float>), which differ from the oracle's in
    the last bits, so the two M^-1 agree to ~1e-7; the FP64 path to 1e-11."""
    coords, tris, meas, H, o32, o64 = env
    orc, tol = (o32, 1e-6) if mode == APPLY_FP32 else (o64, 1e-11)
    rng = np.random.default_rng(4)
    nv = coords.shape[0]
    X = crandn(rng, nv, 8)
    Xr = rng.standard_normal((nv, 3))
    Yg, Yo = np.zeros_like(X), np.zeros_like(X)
    Yr, Yro = np.zeros_like(Xr), np.zeros_like(Xr)
    Lg, Lo = np.zeros_like(X), np.zeros_like(X)
    H.SetApplyMode(mode)
    try:
        H.ApplyMassInverse(X, Yg, 1e-10)
        H.ApplyMassInverse(Xr, Yr, 1e-10)
        H.ApplyLumpedMassInverse(X, Lg)
    finally:
        H.SetApplyMode(APPLY_FP32)
    orc.ApplyMassInverse(X, Yo, 1e-10)
    orc.ApplyMassInverse(Xr, Yro, 1e-10)
    orc.ApplyLumpedMassInverse(X, Lo)
    assert relerr(Yg, Yo) < tol
    assert relerr(Yr, Yro) < tol
    assert relerr(Lg, Lo) < (1e-6 if mode == APPLY_FP32 else 1e-14)


@pytest.mark.parametrize("ncols,cplx", [(1, False), (31, False), (33, False), (100, False), (1024, False),
                                        (512, True)])
def test_mass_inverse_column_counts(env, ncols, cplx):
    """FP64 CG on 1 ... 1024 real columns (512 complex = 1024 real) on the
    642-vertex mesh, which takes the one-launch path (one block per column,
    every iteration in one launch).  Column 0 is zero and converges at once
    while the others iterate."""
    coords, tris, meas, H, o32, o64 = env
    rng = np.random.default_rng(40 + ncols)
    nv = coords.shape[0]
    X = crandn(rng, nv, ncols) if cplx else rng.standard_normal((nv, ncols))
    X[:, 0] = 0
    Yg, Yo = np.zeros_like(X), np.zeros_like(X)
    H.SetApplyMode(APPLY_FP64)
    try:
        H.ApplyMassInverse(X, Yg, 1e-10)
    finally:
        H.SetApplyMode(APPLY_FP32)
    o64.ApplyMassInverse(X, Yo, 1e-10)
    assert np.all(Yg[:, 0] == 0)
    assert relerr(Yg, Yo) < 1e-11


def test_mass_inverse_small_mesh_takes_one_launch_path(env):
    """The 642-vertex test mesh's CG runs one block per column in one launch
    (the path the column-count tests above check against the oracle)."""
    coords, tris, meas, H, o32, o64 = env
    prof = H.ProfileKrylov(2, 2, 2)
    assert prof["cg_iteration"]["one_launch_path"]
    assert prof["cg_iteration"]["ms"] > 0


@pytest.mark.parametrize("ncols,cplx", [(3, False), (40, True)])
def test_mass_inverse_multi_block_path(ncols, cplx):
    """The CG mass inverse on a mesh above the one-launch path's 16384
    vertices (icosphere level 6, 40962): the three-launches-per-iteration
    kernels with two-level column sums, against the FP64 oracle; column 0 is
    zero and converges at once."""
    from oracle import oracle as O
    coords, tris = meshes.icosphere(6)
    rng = np.random.default_rng(60 + ncols)
    nv = coords.shape[0]
    X = crandn(rng, nv, ncols) if cplx else rng.standard_normal((nv, ncols))
    X[:, 0] = 0
    Yg, Yo = np.zeros_like(X), np.zeros_like(X)
    with Helmholtz_CUDA(coords, tris, np.eye(3)) as H:
        H.SetApplyMode(APPLY_FP64)
        H.ApplyMassInverse(X, Yg, 1e-10)
        prof = H.ProfileKrylov(4, 2, 2)
    O.Oracle(coords, tris, np.eye(3), precision=64).ApplyMassInverse(X, Yo, 1e-10)
    assert not prof["cg_iteration"]["one_launch_path"]
    assert np.all(Yg[:, 0] == 0)
    assert relerr(Yg, Yo) < 1e-11


def test_device_blocks_are_validated(env):
    """Torch blocks with too few rows or columns, another dtype or a column
    stride are refused by the Python mirror before any launch; a valid call
    afterwards still runs."""
    import torch
    coords, tris, meas, H, o32, o64 = env
    nv = coords.shape[0]
    B = torch.zeros((nv, 16), dtype=torch.complex64, device="cuda")
    H.LoadBoundaryOperators_PL([2.0], [[1, 1, 0, 0]], 16, 16)
    try:
        with pytest.raises(ValueError):
            H.ApplyBoundaryOperators_PL(1.0, B, 0.0, torch.zeros((nv - 1, 16), dtype=torch.complex64, device="cuda"))
        with pytest.raises(ValueError):
            H.ApplyBoundaryOperators_PL(1.0, B[:, :8], 0.0, B.clone())
        with pytest.raises(TypeError):
            H.ApplyBoundaryOperators_PL(1.0, B, 0.0, B.to(torch.complex128))
        with pytest.raises(ValueError):
            H.ApplyBoundaryOperators_PL(1.0, B, 0.0,
                                        torch.zeros((16, nv), dtype=torch.complex64, device="cuda").t())
        with pytest.raises(TypeError):
            H.ApplyFarFieldOperators_PL(1.0, B, 0.0,
                                        torch.zeros((meas.shape[0], 16), dtype=torch.complex64, device="cuda"))
        with pytest.raises(ValueError):
            H.ApplyBoundaryOperatorsRows(1.0, B, 0.0, B[:10], 0, 10)
        C = torch.zeros_like(B)
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C)
        torch.cuda.synchronize()
        assert torch.count_nonzero(C).item() == 0
    finally:
        H.UnloadBoundaryOperators_PL()


def test_two_contexts_from_one_thread_keep_the_callers_device(env):
    """Calls on two contexts interleaved from one thread give the results of
    each alone, and leave the caller's current device as it was."""
    import torch
    coords, tris, meas, H, o32, o64 = env
    before = torch.cuda.current_device()
    H2 = Helmholtz_CUDA(*meshes.icosphere(2), meas)
    try:
        rng = np.random.default_rng(9)
        nv2 = H2.VertexCount()
        X1, X2 = crandn(rng, coords.shape[0], 4), crandn(rng, nv2, 4)
        Y1, Y2 = np.zeros_like(X1), np.zeros_like(X2)
        Y1b, Y2b = np.zeros_like(X1), np.zeros_like(X2)
        H.ApplyMassInverse(X1, Y1, 1e-10)
        H2.ApplyMassInverse(X2, Y2, 1e-10)
        H.ApplyMassInverse(X1, Y1b, 1e-10)
        H2.ApplyMassInverse(X2, Y2b, 1e-10)
        assert np.array_equal(Y1, Y1b) and np.array_equal(Y2, Y2b)
        assert torch.cuda.current_device() == before
    finally:
        H2.close()


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_TC, APPLY_FP64])
def test_apply_at_the_maximum_wave_count(mode):
    """wave_count 512, the largest the API takes (8 wavenumbers x 64 columns):
    the tensor-core form runs its largest chunk count (32 groups of 16
    columns, 8 passes of 4).  One more chunk is refused with ERR_SIZE."""
    coords, tris = meshes.icosphere(2)
    nv = coords.shape[0]
    kap = np.linspace(1.0, 8.0, 8)
    coeff = np.array([[0.25 + 1j, 1 + 0.5j, 1 - 2j, 0.3j]] * 8)
    rng = np.random.default_rng(11)
    B, C0 = crandn(rng, nv, 512), crandn(rng, nv, 512)
    Cg = C0.copy()
    H = Helmholtz_CUDA(coords, tris, np.eye(3))
    try:
        H.SetApplyMode(mode)
        H.ApplyBoundaryOperators_PL(0.5 - 1j, B, 0.25, Cg, kap, coeff, 512, 64)
        with pytest.raises(BaemmError, match="ERR_SIZE"):
            Z = np.zeros((nv, 576), complex)
            H.ApplyBoundaryOperators_PL(1.0, Z, 0.0, Z.copy(), np.linspace(1.0, 9.0, 9),
                                        np.array([[0, 1, 0, 0]] * 9), 576, 64)
    finally:
        H.close()
    o = O.Oracle(coords, tris, np.eye(3), precision=64)
    Co = C0.copy()
    o.ApplyBoundaryOperators_PL(0.5 - 1j, B, 0.25, Co, kap, coeff, 512, 64)
    assert relerr(Cg, Co) < (1e-11 if mode == APPLY_FP64 else FP32_VS64_TOL)


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_TC, APPLY_FP64])
@pytest.mark.parametrize("name", ["tri1", "quad2", "tetra", "strip17"])
def test_apply_on_tiny_meshes(mode, name):
    """Meshes of 1, 2, 4 and 17 triangles: one partly filled source tile and
    target block, every row but a few past the end (masked), the self pair of
    each target inside the only tile."""
    coords, tris = tiny_meshes()[name]
    nv = coords.shape[0]
    coeff = np.array([[0.25 + 1j, 1 + 0.5j, 1 - 2j, 0.3j]])
    rng = np.random.default_rng(12)
    B, C0 = crandn(rng, nv, 16), crandn(rng, nv, 16)
    Cg = C0.copy()
    H = Helmholtz_CUDA(coords, tris, np.eye(3))
    try:
        H.SetApplyMode(mode)
        H.ApplyBoundaryOperators_PL(0.5 - 1j, B, 0.25, Cg, [3.0], coeff, 16, 16)
    finally:
        H.close()
    o = O.Oracle(coords, tris, np.eye(3), precision=64)
    Co = C0.copy()
    o.ApplyBoundaryOperators_PL(0.5 - 1j, B, 0.25, Co, [3.0], coeff, 16, 16)
    assert np.isfinite(Cg).all()
    assert relerr(Cg, Co) < (1e-11 if mode == APPLY_FP64 else FP32_VS64_TOL)


def test_error_statuses(env):
    coords, tris, meas, H, o32, o64 = env
    B = np.zeros((coords.shape[0], 16), complex)
    with pytest.raises(BaemmError, match="NOT_LOADED"):
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, B.copy())
    with pytest.raises(BaemmError, match="ERR_SIZE"):
        H.ApplyBoundaryOperators_PL(1.0, B, 0.0, B.copy(), [1.0], [[0, 1, 0, 0]], 16, 12)
    with pytest.raises(BaemmError, match="ERR_ARG"):
        H.ApplyBoundaryOperators_PL(1.0, B[:, :8], 0.0, B.copy(), [1.0], [[0, 1, 0, 0]], 16, 16)
    # the context stays usable after the errors
    C = np.zeros_like(B)
    H.ApplyBoundaryOperators_PL(1.0, B + 1, 0.0, C, [1.0], [[0, 1, 0, 0]], 16, 16)
    assert np.isfinite(C).all() and np.abs(C).max() > 0


def test_curl_operator_matches_oracle(env):
    """CurlOp (Initialize.hpp:146-211) built on the device: same CSR structure
    as the oracle, values within FP32 rounding, and area * nu x g on the vertex
    values of a linear field g . x."""
    coords, tris, meas, H, o32, o64 = env
    go, gi, gv = H.CurlOperator()
    oo, oi, ov = o32.curl_operator()
    assert np.array_equal(go, oo) and np.array_equal(gi, oi)
    assert relerr(gv, ov) < 1e-6
    _, nrm, area, _ = o64.geometry()
    g = np.array([-0.4, 0.9, 1.3])
    rows = np.add.reduceat(gv.astype(np.float64) * (coords @ g)[gi], go[:-1]).reshape(-1, 3)
    want = area[:, None] * np.cross(nrm[:, :3], g)
    assert np.max(np.abs(rows - want)) < 2e-5 * np.max(np.abs(want))
