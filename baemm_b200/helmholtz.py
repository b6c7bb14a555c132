"""Python mirror of the reference class BAEMM::Helmholtz_OpenCL over the C ABI.

Method names, argument order and meaning follow Helmholtz_OpenCL.hpp and the
member fragments it includes (ApplyBoundaryOperators.hpp, FarField.hpp, ...),
so code written against the reference reads the same.  Arrays are numpy
(host, copied through the device on every call, as the reference does) or
torch CUDA tensors (device-resident, no host round trip) for the operator
applies.  Complex blocks are row-major ``rows x ld`` with ``ld >= wave_count``.

Errors: every C call returns a status; a non-zero status raises BaemmError
with the library's message (the reference prints and continues).
"""
from __future__ import annotations

import contextlib
import ctypes as C

import numpy as np

from . import _capi
from ._capi import APPLY_FP32, APPLY_FP64, APPLY_TC, WAVE_PLANE, WAVE_RADIAL, BaemmError, SolveStats

_CUDA_STREAM_LEGACY = 0x1   # cudaStreamLegacy

__all__ = ["Helmholtz_CUDA", "WaveType", "BaemmError", "APPLY_FP32", "APPLY_TC", "APPLY_FP64"]


class WaveType:
    """BAEMM_Common.hpp:7-11."""
    Plane = WAVE_PLANE
    Radial = WAVE_RADIAL


def _dp(a):
    return a.ctypes.data_as(_capi.dp)


def _fp(a):
    return a.ctypes.data_as(_capi.fp)


def _cz(x) -> np.ndarray:
    return np.array([complex(x).real, complex(x).imag], dtype=np.float64)


def _cc(x) -> np.ndarray:
    return np.array([complex(x).real, complex(x).imag], dtype=np.float32)


def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _coeff(coeff) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(coeff, dtype=np.complex128).reshape(-1, 4))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _check_dev(t, dtype, rows, cols, device, name):
    """A torch CUDA block handed to a device-pointer entry point: the kernels
    read or write rows x cols entries at t.data_ptr() with leading dimension
    t.stride(0), on the context's device, so the tensor must hold them there."""
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise TypeError(f"{name} must be a torch CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if t.device.index != device:
        raise ValueError(f"{name} is on {t.device}, the context on cuda:{device}")
    if t.dim() != 2 or (t.shape[1] > 1 and t.stride(1) != 1):
        raise ValueError(f"{name} must be a 2-D tensor with unit column stride")
    if t.shape[0] < rows or t.shape[1] < cols or (rows > 1 and t.stride(0) < cols):
        raise ValueError(f"{name} must hold {rows} x {cols} entries (got shape {tuple(t.shape)}, "
                         f"row stride {t.stride(0)})")


def _check_host(a, dtype, rows, name, cols=None, exact_cols=False, allow_1d=False):
    """A host block the library writes in place (or reads without a copy): a
    C-contiguous numpy array of `dtype` with at least `rows` rows and `cols`
    columns, exactly `cols` where the entry point takes no leading dimension."""
    ok_dim = a.ndim == 2 or (allow_1d and a.ndim == 1) if isinstance(a, np.ndarray) else False
    if not (ok_dim and a.dtype == dtype and a.flags.c_contiguous):
        raise TypeError(f"{name} must be a C-contiguous numpy array of dtype {np.dtype(dtype).name}")
    c = a.shape[1] if a.ndim == 2 else 1
    if a.shape[0] < rows or (cols is not None and (c != cols if exact_cols else c < cols)):
        want = f"{rows} x {cols}" if cols is not None else f"{rows} rows of"
        raise ValueError(f"{name} must hold {want} entries (got shape {a.shape})")


def _need_rows(a, rows, name):
    if a.shape[0] < rows:
        raise ValueError(f"{name} must hold {rows} rows (got shape {a.shape})")


def _check_out(a, dtype, name):
    if not (isinstance(a, np.ndarray) and a.dtype == dtype and a.ndim == 2 and a.flags.c_contiguous):
        raise TypeError(f"{name} must be a C-contiguous 2-D numpy array of dtype {np.dtype(dtype).name}")


class Packer:
    """Packing of concurrent solves' tensor-core applies into one launch
    (baemm_packer_create; no reference counterpart).  Attach the contexts that
    serve concurrent solves (each driven by its own thread) with
    Helmholtz_CUDA.SetPacker; detach them before closing the packer."""

    def __init__(self, device: int = 0, max_wait_us: int = 2000):
        self._lib = _capi.lib()
        self._h = self._lib.baemm_packer_create(int(device), int(max_wait_us))
        if not self._h:
            raise BaemmError(2, self._lib.baemm_last_error(None).decode())

    def stats(self) -> dict:
        """Packed launches so far and the problems they carried."""
        a, b = C.c_int64(), C.c_int64()
        st = self._lib.baemm_packer_stats(self._h, C.byref(a), C.byref(b))
        if st != 0:
            raise BaemmError(st, "packer stats")
        return {"launches": int(a.value), "problems": int(b.value)}

    def close(self):
        if self._h:
            self._lib.baemm_packer_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Helmholtz_CUDA:
    """Drop-in for Helmholtz_OpenCL(coords, nv, tris, nt, meas, nm, device, threads)
    (Helmholtz_OpenCL.hpp:175-249)."""

    def __init__(self, vertex_coords, triangles, meas_directions, device: int = 0, cpu_threads: int = 1):
        L = _capi.lib()
        self._coords = _f64(vertex_coords).reshape(-1, 3)
        self._tris = np.ascontiguousarray(np.asarray(triangles, dtype=np.int64).reshape(-1, 3))
        self._meas = _f64(meas_directions).reshape(-1, 3)
        h = C.c_void_p()
        st = L.baemm_create(_dp(self._coords), self._coords.shape[0],
                            self._tris.ctypes.data_as(_capi.i64p), self._tris.shape[0],
                            _dp(self._meas), self._meas.shape[0], int(device), int(cpu_threads), C.byref(h))
        if st != 0:
            raise BaemmError(st, L.baemm_last_error(None).decode())
        self._h = h
        self._lib = L
        self._device = int(device)   # resolved on first use (an out-of-range number means device 0)
        self._user_stream = None   # set by SetStream; otherwise torch tensors join torch's current stream

    def _dev_index(self) -> int:
        import torch
        d = self._device
        return d if 0 <= d < torch.cuda.device_count() else 0

    def _check_pair(self, B, Cout, rows_c):
        """B (vertices x wave_count) and C (rows_c x wave_count) for a device call."""
        wc = self.GetWaveCount()
        dev = self._dev_index()
        _check_dev(B, B.dtype, self.VertexCount(), wc, dev, "B_in")
        _check_dev(Cout, B.dtype, rows_c, wc, dev, "C_out")

    # --- lifecycle ---------------------------------------------------------------
    def SetMesh(self, vertex_coords, triangles):
        """Replace the mesh, keeping device, stream, measurement directions and
        settings (baemm_set_mesh); the boundary operators must be loaded again."""
        coords = _f64(vertex_coords).reshape(-1, 3)
        tris = np.ascontiguousarray(np.asarray(triangles, dtype=np.int64).reshape(-1, 3))
        self._ck(self._lib.baemm_set_mesh(self._h, _dp(coords), coords.shape[0],
                                          tris.ctypes.data_as(_capi.i64p), tris.shape[0]))
        self._coords, self._tris = coords, tris

    def close(self):
        if getattr(self, "_h", None):
            self._lib.baemm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, st):
        if st != 0:
            raise BaemmError(st, self._lib.baemm_last_error(self._h).decode())

    # --- getters / setters (GetSetters.hpp) ----------------------------------------
    def ClassName(self) -> str:
        return self._lib.baemm_class_name().decode()

    def DeviceInfo(self) -> str:
        buf = C.create_string_buffer(4096)
        self._ck(self._lib.baemm_device_info(self._h, buf, 4096))
        return buf.value.decode()

    def VertexCount(self) -> int:
        return int(self._lib.baemm_vertex_count(self._h))

    def SimplexCount(self) -> int:
        return int(self._lib.baemm_simplex_count(self._h))

    def GetMeasCount(self) -> int:
        return int(self._lib.baemm_meas_count(self._h))

    def GetWaveCount(self) -> int:
        return int(self._lib.baemm_get_wave_count(self._h))

    def GetWaveChunkSize(self) -> int:
        return int(self._lib.baemm_get_wave_chunk_size(self._h))

    def SetWaveChunkSize(self, wcs: int):
        self._ck(self._lib.baemm_set_wave_chunk_size(self._h, int(wcs)))

    def GetBlockSize(self) -> int:
        return int(self._lib.baemm_get_block_size(self._h))

    def SetBlockSize(self, bs: int):
        self._ck(self._lib.baemm_set_block_size(self._h, int(bs)))

    def UseDiagonal(self, use_it: bool):
        self._ck(self._lib.baemm_use_diagonal(self._h, int(bool(use_it))))

    @property
    def gmres_max_iter(self) -> int:
        a, b = C.c_int(), C.c_int()
        self._ck(self._lib.baemm_get_gmres_params(self._h, C.byref(a), C.byref(b)))
        return a.value

    @gmres_max_iter.setter
    def gmres_max_iter(self, v: int):
        self._ck(self._lib.baemm_set_gmres_params(self._h, int(v), self.gmres_max_restarts))

    @property
    def gmres_max_restarts(self) -> int:
        a, b = C.c_int(), C.c_int()
        self._ck(self._lib.baemm_get_gmres_params(self._h, C.byref(a), C.byref(b)))
        return b.value

    @gmres_max_restarts.setter
    def gmres_max_restarts(self, v: int):
        self._ck(self._lib.baemm_set_gmres_params(self._h, self.gmres_max_iter, int(v)))

    def SetApplyMode(self, mode: int):
        self._ck(self._lib.baemm_set_apply_mode(self._h, int(mode)))

    def GetApplyMode(self) -> int:
        return int(self._lib.baemm_get_apply_mode(self._h))

    def SetTuning(self, key: int, value: int):
        self._ck(self._lib.baemm_set_tuning(self._h, int(key), int(value)))

    def GetTuning(self, key: int) -> int:
        return int(self._lib.baemm_get_tuning(self._h, int(key)))

    def TcEntrySharing(self) -> int:
        """Groups of 16 columns per shared kernel-entry evaluation of the
        tensor-core apply of the loaded operators (1, 2 or 4)."""
        r = int(self._lib.baemm_tc_entry_sharing(self._h))
        if r < 0:
            self._ck(r)
        return r

    def SetKernelVariant(self, variant: int):
        self.SetTuning(_capi.TUNE_DENSE_VARIANT, variant)

    def GetKernelVariant(self) -> int:
        return self.GetTuning(_capi.TUNE_DENSE_VARIANT)

    def SetRefinement(self, max_steps: int, inner_tol: float = 1e-4):
        self._ck(self._lib.baemm_set_refinement(self._h, int(max_steps), float(inner_tol)))

    def SetGraphs(self, on: bool = True):
        """Replay the solvers' inner operators as CUDA graphs (baemm_set_graphs)."""
        self._ck(self._lib.baemm_set_graphs(self._h, 1 if on else 0))

    def SetPacker(self, packer):
        """Submit the solves' dense stages to `packer` (a Packer; None detaches)."""
        self._ck(self._lib.baemm_set_packer(self._h, packer._h if packer is not None else None))

    def GraphStats(self) -> tuple:
        """(captures, replays) since the context was created."""
        a, b = C.c_int64(), C.c_int64()
        self._ck(self._lib.baemm_graph_stats(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def Autotune(self, mode=APPLY_TC, repeats: int = 2) -> dict:
        """Time the dense-kernel settings of `mode` on the loaded operators and
        keep the fastest (baemm_autotune); returns the chosen settings and times."""
        r = _capi.TuneResult()
        self._ck(self._lib.baemm_autotune(self._h, int(mode), int(repeats), C.byref(r)))
        return {f: getattr(r, f) for f, _ in _capi.TuneResult._fields_}

    def LastSolveStats(self) -> dict:
        s = SolveStats()
        self._ck(self._lib.baemm_last_solve_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in SolveStats._fields_}

    def _tri_field(self, fn, width):
        out = np.zeros((self.SimplexCount(), width) if width > 1 else self.SimplexCount(), dtype=np.float32)
        self._ck(fn(self._h, _fp(out)))
        return out

    def Areas(self) -> np.ndarray:
        return self._tri_field(self._lib.baemm_get_areas, 1)

    TriangleAreas = Areas

    def TriangleNormals(self) -> np.ndarray:
        return self._tri_field(self._lib.baemm_get_triangle_normals, 4)

    def TriangleMidpoints(self) -> np.ndarray:
        return self._tri_field(self._lib.baemm_get_triangle_midpoints, 4)

    def SingleLayerDiagonal(self) -> np.ndarray:
        return self._tri_field(self._lib.baemm_get_single_layer_diagonal, 1)

    def MassMatrix(self):
        """CSR (outer, inner, values) of the P1 mass matrix (GetSetters.hpp:113-116)."""
        nnz = C.c_int64()
        self._ck(self._lib.baemm_get_mass_matrix(self._h, None, None, None, C.byref(nnz)))
        outer = np.zeros(self.VertexCount() + 1, np.int64)
        inner = np.zeros(nnz.value, np.int32)
        vals = np.zeros(nnz.value, np.float32)
        self._ck(self._lib.baemm_get_mass_matrix(self._h, outer.ctypes.data_as(_capi.i64p),
                                                 inner.ctypes.data_as(_capi.i32p), _fp(vals), C.byref(nnz)))
        return outer, inner, vals

    def CurlOperator(self):
        """CSR (outer, inner, values) of CurlOp (Initialize.hpp:146-211): rows
        3 t + d, the triangle's vertex columns ascending, values (area nu x
        grad phi)[d] in FP32."""
        nnz = C.c_int64()
        self._ck(self._lib.baemm_get_curl_operator(self._h, None, None, None, C.byref(nnz)))
        outer = np.zeros(3 * self.SimplexCount() + 1, np.int64)
        inner = np.zeros(nnz.value, np.int32)
        vals = np.zeros(nnz.value, np.float32)
        self._ck(self._lib.baemm_get_curl_operator(self._h, outer.ctypes.data_as(_capi.i64p),
                                                   inner.ctypes.data_as(_capi.i32p), _fp(vals), C.byref(nnz)))
        return outer, inner, vals

    def SetProfiling(self, on: bool):
        self._ck(self._lib.baemm_set_profiling(self._h, int(bool(on))))

    def LastApplyTimes(self):
        """Device ms of the last boundary apply: (AvOp, dense kernel, epilogue)."""
        ms = np.zeros(3, np.float32)
        self._ck(self._lib.baemm_last_apply_times(self._h, _fp(ms)))
        return tuple(float(x) for x in ms)

    @staticmethod
    def KernelLaunchCount() -> int:
        return int(_capi.lib().baemm_kernel_launch_count())

    def stream(self) -> int:
        return int(self._lib.baemm_stream(self._h) or 0)

    def SetStream(self, stream_handle: int | None):
        """Enqueue on `stream_handle` (a cudaStream_t as int; the stream must
        outlive its use).  None or 0 returns to the default: the context's own
        stream for host arrays, and for torch CUDA tensors torch's current
        stream of the tensor's device, joined for the duration of each call."""
        self._ck(self._lib.baemm_set_stream(self._h, C.c_void_p(stream_handle or 0)))
        self._user_stream = stream_handle or None

    @contextlib.contextmanager
    def _on_torch_stream(self, t):
        # Device-pointer calls are asynchronous: they run on the stream that
        # produced their inputs and will consume their outputs, which for torch
        # tensors is torch's current stream.  The context is handed over to it
        # for the call and back afterwards (event ordering, no host sync), so it
        # never keeps a torch stream that may be destroyed later.
        if self._user_stream is not None:
            yield
            return
        import torch
        # torch's default stream is the legacy default stream (handle 0), which
        # the C ABI spells cudaStreamLegacy (0x1); a null handle there means the
        # context's own non-blocking stream.
        s = int(torch.cuda.current_stream(t.device).cuda_stream) or _CUDA_STREAM_LEGACY
        self._ck(self._lib.baemm_set_stream(self._h, C.c_void_p(s)))
        try:
            yield
        finally:
            self._ck(self._lib.baemm_set_stream(self._h, C.c_void_p(0)))

    def Synchronize(self):
        self._ck(self._lib.baemm_synchronize(self._h))

    # --- parameters / operators ----------------------------------------------------
    def LoadParameters(self, kappa, coeff, wave_count, wave_chunk_size, factor=1.0):
        k, c = _f64(kappa), _coeff(coeff)
        self._ck(self._lib.baemm_load_parameters(self._h, _dp(k), _dp(c.view(np.float64)), int(wave_count),
                                                 int(wave_chunk_size), float(factor)))

    def LoadBoundaryOperators_PL(self, kappa, coeff, wave_count, wave_chunk_size):
        k, c = _f64(kappa), _coeff(coeff)
        self._ck(self._lib.baemm_load_boundary_operators(self._h, _dp(k), _dp(c.view(np.float64)),
                                                         int(wave_count), int(wave_chunk_size)))

    def UnloadBoundaryOperators_PL(self):
        self._ck(self._lib.baemm_unload_boundary_operators(self._h))

    def ApplyBoundaryOperators_PL(self, alpha, B_in, beta, C_out, kappa=None, coeff=None, wave_count=None,
                                  wave_chunk_size=None):
        """C_out = alpha * A * B_in + beta * C_out (ApplyBoundaryOperators.hpp:238-391).

        With kappa/coeff/wave_count/wave_chunk_size given, loads, applies and
        unloads (the first overload); otherwise uses the loaded operators.
        numpy complex128 / complex64 host blocks or torch CUDA complex tensors.
        """
        full = kappa is not None
        if full:
            self.LoadBoundaryOperators_PL(kappa, coeff, wave_count, wave_chunk_size)
        try:
            if _is_torch_cuda(B_in):
                import torch
                if B_in.dtype == torch.complex128:
                    fn, cs, ptr = self._lib.baemm_apply_boundary_operators_dev_z, _cz, _dp
                elif B_in.dtype == torch.complex64:
                    fn, cs, ptr = self._lib.baemm_apply_boundary_operators_dev_c, _cc, _fp
                else:
                    raise TypeError("B_in must be complex64 or complex128")
                self._check_pair(B_in, C_out, self.VertexCount())
                with self._on_torch_stream(B_in):
                    self._ck(fn(self._h, ptr(cs(alpha)), C.c_void_p(B_in.data_ptr()), B_in.stride(0),
                                ptr(cs(beta)), C.c_void_p(C_out.data_ptr()), C_out.stride(0)))
            elif isinstance(B_in, np.ndarray) and B_in.dtype == np.complex64:
                _check_out(C_out, np.complex64, "C_out")
                B = np.ascontiguousarray(B_in)
                _need_rows(B, self.VertexCount(), "B_in")
                _need_rows(C_out, self.VertexCount(), "C_out")
                self._ck(self._lib.baemm_apply_boundary_operators_c(
                    self._h, _fp(_cc(alpha)), _fp(B.view(np.float32)), B.shape[1], _fp(_cc(beta)),
                    _fp(C_out.view(np.float32)), C_out.shape[1]))
            else:
                _check_out(C_out, np.complex128, "C_out")
                B = np.ascontiguousarray(B_in, dtype=np.complex128)
                _need_rows(B, self.VertexCount(), "B_in")
                _need_rows(C_out, self.VertexCount(), "C_out")
                self._ck(self._lib.baemm_apply_boundary_operators_z(
                    self._h, _dp(_cz(alpha)), _dp(B.view(np.float64)), B.shape[1], _dp(_cz(beta)),
                    _dp(C_out.view(np.float64)), C_out.shape[1]))
        finally:
            if full:
                self.UnloadBoundaryOperators_PL()
        return C_out

    def ApplyFarFieldOperators_PL(self, alpha, B_in, beta, C_out, kappa=None, coeff=None, wave_count=None,
                                  wave_chunk_size=None):
        """C_out (meas x wc) = alpha (c1 FF_SL + c2 FF_DL) B_in + beta C_out
        (ApplyFarFieldOperators.hpp:334-412)."""
        if _is_torch_cuda(B_in):
            import torch
            if kappa is not None:
                self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
            if B_in.dtype != torch.complex128:
                raise TypeError("the far field on torch tensors takes complex128")
            self._check_pair(B_in, C_out, self.GetMeasCount())
            with self._on_torch_stream(B_in):
                self._ck(self._lib.baemm_apply_far_field_operators_dev_z(
                    self._h, _dp(_cz(alpha)), C.c_void_p(B_in.data_ptr()), B_in.stride(0), _dp(_cz(beta)),
                    C.c_void_p(C_out.data_ptr()), C_out.stride(0)))
            return C_out
        _check_out(C_out, np.complex128, "C_out")
        B = np.ascontiguousarray(B_in, dtype=np.complex128)
        _need_rows(B, self.VertexCount(), "B_in")
        _need_rows(C_out, self.GetMeasCount(), "C_out")
        if kappa is not None:
            k, c = _f64(kappa), _coeff(coeff)
            self._ck(self._lib.baemm_apply_far_field_operators_z(
                self._h, _dp(_cz(alpha)), _dp(B.view(np.float64)), B.shape[1], _dp(_cz(beta)),
                _dp(C_out.view(np.float64)), C_out.shape[1], _dp(k), _dp(c.view(np.float64)), int(wave_count),
                int(wave_chunk_size)))
        else:
            self._ck(self._lib.baemm_apply_far_field_operators_loaded_z(
                self._h, _dp(_cz(alpha)), _dp(B.view(np.float64)), B.shape[1], _dp(_cz(beta)),
                _dp(C_out.view(np.float64)), C_out.shape[1]))
        return C_out

    def ApplyBoundaryOperatorsRows(self, alpha, B_in, beta, C_out, row_begin, row_end, with_mass=True):
        """One row shard of the loaded apply on torch CUDA tensors (no reference
        counterpart): C_out = alpha AvOp^T|rows (K[rows, :] + diag) AvOp B_in
        [+ alpha c0 M B_in if with_mass] + beta C_out, rows = triangles
        [row_begin, row_end).  See baemm_b200.sharded for the multi-GPU apply."""
        import torch
        if not _is_torch_cuda(B_in):
            raise TypeError("ApplyBoundaryOperatorsRows takes torch CUDA tensors")
        if B_in.dtype == torch.complex128:
            fn, cs, ptr = self._lib.baemm_apply_boundary_operators_rows_dev_z, _cz, _dp
        elif B_in.dtype == torch.complex64:
            fn, cs, ptr = self._lib.baemm_apply_boundary_operators_rows_dev_c, _cc, _fp
        else:
            raise TypeError("B_in must be complex64 or complex128")
        self._check_pair(B_in, C_out, self.VertexCount())
        with self._on_torch_stream(B_in):
            self._ck(fn(self._h, ptr(cs(alpha)), C.c_void_p(B_in.data_ptr()), B_in.stride(0), ptr(cs(beta)),
                        C.c_void_p(C_out.data_ptr()), C_out.stride(0), int(row_begin), int(row_end),
                        1 if with_mass else 0))
        return C_out

    def ProfileKrylov(self, columns=32, iterations=20, basis=12):
        """Device time of the Krylov-vector kernels on this mesh (no reference
        counterpart): the CG mass inverse on 2 * columns real columns and one
        Gram-Schmidt pass of a GMRES iteration on `columns` complex columns
        against `basis` vectors.  Per kernel: ms per launch, algorithmic bytes
        per launch and the rate (GB/s); `cg_iteration`: one whole CG iteration
        on the path this mesh's solves take."""
        out = np.zeros(10)
        self._ck(self._lib.baemm_profile_krylov(self._h, int(columns), int(iterations), int(basis), _dp(out)))
        names = ("cg_matvec", "cg_update", "cg_pupdate", "gs_dot", "gs_update")
        res = {n: {"ms": float(out[q]), "algorithmic_bytes": float(out[5 + q]),
                   "GB_s": float(out[5 + q] / (out[q] * 1e-3) / 1e9) if out[q] > 0 else None}
               for q, n in enumerate(names)}
        # one CG iteration on the path this mesh's solves take (baemm_profile_cg): on meshes of up to
        # 16384 vertices one block per column runs every iteration in one launch, so the three kernels
        # above are not what the solver runs there
        cg = np.zeros(3)
        self._ck(self._lib.baemm_profile_cg(self._h, int(columns), int(iterations), _dp(cg)))
        res["cg_iteration"] = {"ms": float(cg[0]), "algorithmic_bytes": float(cg[1]),
                               "GB_s": float(cg[1] / (cg[0] * 1e-3) / 1e9) if cg[0] > 0 else None,
                               "one_launch_path": bool(cg[2])}
        return res

    def BoundaryOperatorKernel(self, B_tri, C_tri, row_begin=0, row_end=None):
        """The dense stage alone on torch CUDA triangle blocks (simplex_count x
        wave_count): C_tri[i] = sum_{j != i} A_ij B_tri[j] for target triangles
        i in [row_begin, row_end), with the loaded operators and the current
        apply mode -- the reference's private BoundaryOperatorKernel()
        (BoundaryOperatorKernel.hpp:5-28).  complex64 blocks run the plain FP32
        or tensor-core form, complex128 blocks the FP64 form."""
        import torch
        if not (_is_torch_cuda(B_tri) and _is_torch_cuda(C_tri)):
            raise TypeError("BoundaryOperatorKernel takes torch CUDA tensors")
        if B_tri.dtype == torch.complex128:
            fn = self._lib.baemm_boundary_operator_kernel_dev_z
        elif B_tri.dtype == torch.complex64:
            fn = self._lib.baemm_boundary_operator_kernel_dev_c
        else:
            raise TypeError("B_tri must be complex64 or complex128")
        nt = self.SimplexCount()
        wc = self.GetWaveCount()
        for X in (B_tri, C_tri):
            if X.dtype != B_tri.dtype or tuple(X.shape) != (nt, wc) or not X.is_contiguous():
                raise ValueError(f"triangle blocks must be contiguous ({nt}, {wc}) tensors of one dtype")
        row_end = nt if row_end is None else int(row_end)
        with self._on_torch_stream(B_tri):
            self._ck(fn(self._h, C.c_void_p(B_tri.data_ptr()), C.c_void_p(C_tri.data_ptr()), int(row_begin), row_end))
        return C_tri

    def ApplyNearFieldOperators_PL(self, alpha, B_in, beta, C_out, *args):
        """C_out (points x wc) = alpha (c1 SL + c2 DL)(points) AvOp B_in + beta C_out
        (ApplyNearFieldOperators.hpp:27-122), the boundary potential at points
        off the surface.

        The reference's two overloads:
            ApplyNearFieldOperators_PL(alpha, B_in, beta, C_out, kappa, coeff, wave_count,
                                       wave_chunk_size, evaluation_points)
            ApplyNearFieldOperators_PL(alpha, B_in, beta, C_out, evaluation_points)
        (the second uses the loaded parameters).  evaluation_points: m x 3.
        numpy complex128 / complex64 host blocks or torch CUDA complex tensors
        (then the points may be a torch CUDA float64 tensor or host array).
        """
        if len(args) == 5:
            kappa, coeff, wave_count, wave_chunk_size, points = args
        elif len(args) == 1:
            kappa = coeff = wave_count = wave_chunk_size = None
            points = args[0]
        else:
            raise TypeError("ApplyNearFieldOperators_PL(alpha, B_in, beta, C_out, [kappa, coeff, wave_count, "
                            "wave_chunk_size,] evaluation_points)")
        if _is_torch_cuda(B_in):
            import torch
            if kappa is not None:
                self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
            if B_in.dtype == torch.complex128:
                fn, cs, ptr = self._lib.baemm_apply_near_field_operators_dev_z, _cz, _dp
            elif B_in.dtype == torch.complex64:
                fn, cs, ptr = self._lib.baemm_apply_near_field_operators_dev_c, _cc, _fp
            else:
                raise TypeError("B_in must be complex64 or complex128")
            if _is_torch_cuda(points):
                P = points.to(device=B_in.device, dtype=torch.float64).reshape(-1, 3).contiguous()
            else:
                P = torch.from_numpy(_f64(points).reshape(-1, 3)).to(B_in.device)
            self._check_pair(B_in, C_out, P.shape[0])
            with self._on_torch_stream(B_in):
                self._ck(fn(self._h, ptr(cs(alpha)), C.c_void_p(B_in.data_ptr()), B_in.stride(0), ptr(cs(beta)),
                            C.c_void_p(C_out.data_ptr()), C_out.stride(0), C.c_void_p(P.data_ptr()), P.shape[0]))
            return C_out
        if isinstance(B_in, np.ndarray) and B_in.dtype == np.complex64:
            if kappa is not None:
                self.LoadParameters(kappa, coeff, wave_count, wave_chunk_size)
            _check_out(C_out, np.complex64, "C_out")
            B = np.ascontiguousarray(B_in)
            P = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
            _need_rows(B, self.VertexCount(), "B_in")
            _need_rows(C_out, P.shape[0], "C_out")
            self._ck(self._lib.baemm_apply_near_field_operators_c(
                self._h, _fp(_cc(alpha)), _fp(B.view(np.float32)), B.shape[1], _fp(_cc(beta)),
                _fp(C_out.view(np.float32)), C_out.shape[1], _fp(P), P.shape[0]))
            return C_out
        _check_out(C_out, np.complex128, "C_out")
        B = np.ascontiguousarray(B_in, dtype=np.complex128)
        P = _f64(points).reshape(-1, 3)
        _need_rows(B, self.VertexCount(), "B_in")
        _need_rows(C_out, P.shape[0], "C_out")
        if kappa is not None:
            k, c = _f64(kappa), _coeff(coeff)
            self._ck(self._lib.baemm_apply_near_field_operators_full_z(
                self._h, _dp(_cz(alpha)), _dp(B.view(np.float64)), B.shape[1], _dp(_cz(beta)),
                _dp(C_out.view(np.float64)), C_out.shape[1], _dp(k), _dp(c.view(np.float64)), int(wave_count),
                int(wave_chunk_size), _dp(P), P.shape[0]))
        else:
            self._ck(self._lib.baemm_apply_near_field_operators_z(
                self._h, _dp(_cz(alpha)), _dp(B.view(np.float64)), B.shape[1], _dp(_cz(beta)),
                _dp(C_out.view(np.float64)), C_out.shape[1], _dp(P), P.shape[0]))
        return C_out

    def CreateIncidentWave_PL(self, alpha, incident_directions, beta, C_out, *args, wave_type=None):
        """C_out = alpha * wave + beta * C_out, the weak incident waves.  The
        reference's two overloads:
            CreateIncidentWave_PL(alpha, directions, beta, C_out, kappa, coeff, wave_count,
                                  wave_chunk_size[, wave_type])
                (CreateIncidentWave.hpp:21-50; loads the parameters with factor 4 pi)
            CreateIncidentWave_PL(alpha, directions, beta, C_out[, wave_type])
                (CreateIncidentWave.hpp:55-124; the loaded parameters, wave_chunk_size directions)
        wave_type defaults to WaveType.Plane."""
        _check_out(C_out, np.complex128, "C_out")
        if C_out.shape[0] < self.VertexCount():
            raise ValueError("C_out must hold vertex_count rows")
        d = _f64(incident_directions).reshape(-1, 3)
        if len(args) in (4, 5):
            kappa, coeff, wave_count, wave_chunk_size = args[:4]
            wt = args[4] if len(args) == 5 else (WaveType.Plane if wave_type is None else wave_type)
            k, c = _f64(kappa), _coeff(coeff)
            self._ck(self._lib.baemm_create_incident_wave_z(
                self._h, _dp(_cz(alpha)), _dp(d), d.shape[0], _dp(_cz(beta)), _dp(C_out.view(np.float64)),
                C_out.shape[1], _dp(k), _dp(c.view(np.float64)), int(wave_count), int(wave_chunk_size), int(wt)))
        elif len(args) in (0, 1):
            wt = args[0] if args else (WaveType.Plane if wave_type is None else wave_type)
            if d.shape[0] < self.GetWaveChunkSize():
                raise ValueError("the loaded-parameter overload reads wave_chunk_size incident directions")
            self._ck(self._lib.baemm_create_incident_wave_loaded_z(
                self._h, _dp(_cz(alpha)), _dp(d), _dp(_cz(beta)), _dp(C_out.view(np.float64)), C_out.shape[1],
                int(wt)))
        else:
            raise TypeError("CreateIncidentWave_PL(alpha, directions, beta, C_out, [kappa, coeff, wave_count, "
                            "wave_chunk_size,] [wave_type])")
        return C_out

    def CreateHerglotzWave_PL(self, alpha, g, beta, C_out, *args):
        """C_out = alpha * HerglotzWave(g) + beta * C_out, g meas_count x wave_count.
        The reference's two overloads:
            CreateHerglotzWave_PL(alpha, g, beta, C_out, kappa, coeff, wave_count, wave_chunk_size)
                (CreateHerglotzWave.hpp:25-44; loads with factor 4 pi / meas_count)
            CreateHerglotzWave_PL(alpha, g, beta, C_out)
                (CreateHerglotzWave.hpp:51-95; the loaded parameters)"""
        _check_out(C_out, np.complex128, "C_out")
        if C_out.shape[0] < self.VertexCount():
            raise ValueError("C_out must hold vertex_count rows")
        G = np.ascontiguousarray(g, dtype=np.complex128)
        if len(args) == 4:
            kappa, coeff, wave_count, wave_chunk_size = args
            k, c = _f64(kappa), _coeff(coeff)
            self._ck(self._lib.baemm_create_herglotz_wave_z(
                self._h, _dp(_cz(alpha)), _dp(G.view(np.float64)), G.shape[1], _dp(_cz(beta)),
                _dp(C_out.view(np.float64)), C_out.shape[1], _dp(k), _dp(c.view(np.float64)), int(wave_count),
                int(wave_chunk_size)))
        elif not args:
            if G.shape[0] < self.GetMeasCount():
                raise ValueError("g must hold meas_count rows")
            self._ck(self._lib.baemm_create_herglotz_wave_loaded_z(
                self._h, _dp(_cz(alpha)), _dp(G.view(np.float64)), G.shape[1], _dp(_cz(beta)),
                _dp(C_out.view(np.float64)), C_out.shape[1]))
        else:
            raise TypeError("CreateHerglotzWave_PL(alpha, g, beta, C_out[, kappa, coeff, wave_count, "
                            "wave_chunk_size])")
        return C_out

    def ApplyMassInverse(self, X, Y, cg_tol, nrhs=None):
        """Y = M^-1 X by CG (ApplyMassInverse.hpp:6-156); real or complex columns."""
        nv = self.VertexCount()
        if np.iscomplexobj(X):
            Xc = np.ascontiguousarray(X, dtype=np.complex128)
            n = Xc.shape[1] if nrhs is None else nrhs
            _need_rows(Xc, nv, "X")
            _check_host(Y, np.complex128, nv, "Y", n)
            self._ck(self._lib.baemm_apply_mass_inverse_z(self._h, _dp(Xc.view(np.float64)), Xc.shape[1],
                                                          _dp(Y.view(np.float64)), Y.shape[1], int(n),
                                                          float(cg_tol)))
        else:
            Xr = _f64(X)
            if Xr.ndim == 1:
                Xr = Xr[:, None]
            n = Xr.shape[1] if nrhs is None else nrhs
            _need_rows(Xr, nv, "X")
            _check_host(Y, np.float64, nv, "Y", n, allow_1d=True)
            Yv = Y if Y.ndim == 2 else Y.reshape(-1, 1)
            self._ck(self._lib.baemm_apply_mass_inverse_d(self._h, _dp(Xr), Xr.shape[1], _dp(Yv), Yv.shape[1],
                                                          int(n), float(cg_tol)))
        return Y

    def ApplyLumpedMassInverse(self, X, Y, nrhs=None):
        nv = self.VertexCount()
        if np.iscomplexobj(X):
            Xc = np.ascontiguousarray(X, dtype=np.complex128)
            n = Xc.shape[1] if nrhs is None else nrhs
            _need_rows(Xc, nv, "X")
            _check_host(Y, np.complex128, nv, "Y", n)
            self._ck(self._lib.baemm_apply_lumped_mass_inverse_z(self._h, _dp(Xc.view(np.float64)), Xc.shape[1],
                                                                 _dp(Y.view(np.float64)), Y.shape[1], int(n)))
        else:
            Xr = _f64(X)
            n = Xr.shape[1] if nrhs is None else nrhs
            _need_rows(Xr, nv, "X")
            _check_host(Y, np.float64, nv, "Y", n)
            self._ck(self._lib.baemm_apply_lumped_mass_inverse_d(self._h, _dp(Xr), Xr.shape[1], _dp(Y), Y.shape[1],
                                                                 int(n)))
        return Y

    def MassDot(self, alpha, X, beta, Y):
        """Y = alpha M X + beta Y on real columns (MassMatrix().Dot)."""
        Xr = _f64(X)
        _need_rows(Xr, self.VertexCount(), "X")
        _check_host(Y, np.float64, self.VertexCount(), "Y", Xr.shape[1])
        self._ck(self._lib.baemm_mass_dot_d(self._h, float(alpha), _dp(Xr), Xr.shape[1], float(beta), _dp(Y),
                                            Y.shape[1], Xr.shape[1]))
        return Y

    # --- solvers (FarField.hpp) -----------------------------------------------------
    def FarField(self, kappa, inc_directions, Y_out, wave_type=WaveType.Plane, cg_tol=1e-5, gmres_tol=1e-4):
        return self.FarField_parameters(kappa, inc_directions, Y_out, wave_type, None, cg_tol, gmres_tol)

    def FarField_parameters(self, kappa, inc_directions, Y_out, wave_type=WaveType.Plane, eta=None, cg_tol=1e-5,
                            gmres_tol=1e-4):
        k = _f64(kappa)
        d = _f64(inc_directions).reshape(-1, 3)
        _check_host(Y_out, np.complex128, self.GetMeasCount(), "Y_out", k.size * d.shape[0], exact_cols=True)
        e = _f64(eta) if eta is not None else None
        self._ck(self._lib.baemm_far_field_parameters(self._h, _dp(k), k.size, _dp(d), d.shape[0],
                                                      _dp(Y_out.view(np.float64)), int(wave_type),
                                                      _dp(e) if e is not None else None, float(cg_tol),
                                                      float(gmres_tol)))
        return Y_out

    def BoundaryPotential(self, kappa, coeff_out, wave, phi, wave_chunk_size, cg_tol, gmres_tol):
        k = _f64(kappa)
        W = np.ascontiguousarray(wave, dtype=np.complex128)
        wc, nv = k.size * int(wave_chunk_size), self.VertexCount()
        _check_host(W, np.complex128, nv, "wave", wc, exact_cols=True)
        _check_host(phi, np.complex128, nv, "phi", wc, exact_cols=True)
        _check_host(coeff_out, np.complex128, k.size, "coeff_out", 4, exact_cols=True)
        self._ck(self._lib.baemm_boundary_potential(self._h, _dp(k), _dp(coeff_out.view(np.float64)),
                                                    _dp(W.view(np.float64)), _dp(phi.view(np.float64)), k.size,
                                                    int(wave_chunk_size), float(cg_tol), float(gmres_tol)))
        return phi

    def DirichletToNeumann(self, kappa, wave, neumann_trace, wave_chunk_size, cg_tol, gmres_tol):
        k = _f64(kappa)
        W = np.ascontiguousarray(wave, dtype=np.complex128)
        wc, nv = k.size * int(wave_chunk_size), self.VertexCount()
        _check_host(W, np.complex128, nv, "wave", wc, exact_cols=True)
        _check_host(neumann_trace, np.complex128, nv, "neumann_trace", wc, exact_cols=True)
        self._ck(self._lib.baemm_dirichlet_to_neumann(self._h, _dp(k), _dp(W.view(np.float64)),
                                                      _dp(neumann_trace.view(np.float64)), k.size,
                                                      int(wave_chunk_size), float(cg_tol), float(gmres_tol)))
        return neumann_trace

    def Derivative_FF_Helper(self, kappa, inc_directions, du_dn, wave_type=WaveType.Plane, cg_tol=1e-5,
                             gmres_tol=1e-4):
        k = _f64(kappa)
        d = _f64(inc_directions).reshape(-1, 3)
        _check_host(du_dn, np.complex128, self.VertexCount(), "du_dn", k.size * d.shape[0], exact_cols=True)
        self._ck(self._lib.baemm_derivative_ff_helper(self._h, _dp(k), k.size, _dp(d), d.shape[0],
                                                      _dp(du_dn.view(np.float64)), int(wave_type), float(cg_tol),
                                                      float(gmres_tol)))
        return du_dn

    def _du_dn_ptr(self, du_dn, wc=None):
        if du_dn is None:
            return _capi.dp()   # NULL: the library callocs and fills it
        if wc is not None:
            _check_host(du_dn, np.complex128, self.VertexCount(), "du_dn", wc, exact_cols=True)
        return du_dn.view(np.float64).ctypes.data_as(_capi.dp)

    def _take_du_dn(self, ptr, du_dn, wc):
        if du_dn is not None:
            return du_dn
        n = self.VertexCount() * wc
        arr = np.ctypeslib.as_array(ptr, shape=(2 * n,)).copy().view(np.complex128).reshape(-1, wc)
        self._lib.baemm_free(C.cast(ptr, C.c_void_p))
        return arr

    def Derivative_FF(self, kappa, inc_directions, X_in, Y_out, du_dn=None, wave_type=WaveType.Plane, cg_tol=1e-5,
                      gmres_tol=1e-4):
        """Returns (Y_out, du_dn); du_dn=None lets the library compute it (FarField.hpp:273-283)."""
        k = _f64(kappa)
        d = _f64(inc_directions).reshape(-1, 3)
        X = _f64(X_in).reshape(-1, 3)
        wc = k.size * d.shape[0]
        _need_rows(X, self.VertexCount(), "X_in")
        _check_host(Y_out, np.complex128, self.GetMeasCount(), "Y_out", wc, exact_cols=True)
        ptr = self._du_dn_ptr(du_dn, wc)
        self._ck(self._lib.baemm_derivative_ff(self._h, _dp(k), k.size, _dp(d), d.shape[0], _dp(X),
                                               _dp(Y_out.view(np.float64)), C.byref(ptr), int(wave_type),
                                               float(cg_tol), float(gmres_tol)))
        return Y_out, self._take_du_dn(ptr, du_dn, k.size * d.shape[0])

    def AdjointDerivative_FF(self, kappa, inc_directions, g, Y_out, du_dn=None, wave_type=WaveType.Plane,
                             cg_tol=1e-5, gmres_tol=1e-4):
        k = _f64(kappa)
        d = _f64(inc_directions).reshape(-1, 3)
        G = np.ascontiguousarray(g, dtype=np.complex128)
        wc = k.size * d.shape[0]
        _check_host(G, np.complex128, self.GetMeasCount(), "g", wc, exact_cols=True)
        _check_host(Y_out, np.float64, self.VertexCount(), "Y_out", 3, exact_cols=True)
        ptr = self._du_dn_ptr(du_dn, wc)
        self._ck(self._lib.baemm_adjoint_derivative_ff(self._h, _dp(k), k.size, _dp(d), d.shape[0],
                                                       _dp(G.view(np.float64)), _dp(Y_out), C.byref(ptr),
                                                       int(wave_type), float(cg_tol), float(gmres_tol)))
        return Y_out, self._take_du_dn(ptr, du_dn, k.size * d.shape[0])

    def GaussNewtonSolve(self, kappa, inc_directions, M, P, alpha, B_in, beta, X_out, du_dn,
                         wave_type=WaveType.Plane, cg_tol=1e-5, gmres_tol_inner=5e-3, gmres_tol_outer=1e-2,
                         solver: int = 0) -> bool:
        """X = alpha (M + DF* DF)^-1 B + beta X (FarField.hpp:457-604).

        M, P: callables (x, y) on numpy (n, 3) float64 arrays, writing y in place.
        solver 0 = GMRES (the reference), 1 = CG.
        """
        k = _f64(kappa)
        d = _f64(inc_directions).reshape(-1, 3)
        n = self.VertexCount()
        B = _f64(B_in)
        _check_host(B, np.float64, n, "B_in", 3)
        _check_host(X_out, np.float64, n, "X_out", 3)

        def wrap(f):
            def cb(x, y, _user):
                xa = np.ctypeslib.as_array(x, shape=(n, 3))
                ya = np.ctypeslib.as_array(y, shape=(n, 3))
                f(xa, ya)
            return _capi.REAL_OP(cb)

        Mc, Pc = wrap(M), wrap(P)
        ptr = self._du_dn_ptr(du_dn, k.size * d.shape[0])
        ok = C.c_int(0)
        self._ck(self._lib.baemm_gauss_newton_solve(self._h, _dp(k), k.size, _dp(d), d.shape[0], Mc, None, Pc, None,
                                                    float(alpha), _dp(B), B.shape[1], float(beta), _dp(X_out),
                                                    X_out.shape[1], C.byref(ptr), int(wave_type), float(cg_tol),
                                                    float(gmres_tol_inner), float(gmres_tol_outer), int(solver),
                                                    C.byref(ok)))
        if du_dn is None:
            self._take_du_dn(ptr, None, k.size * d.shape[0])
        return bool(ok.value)
