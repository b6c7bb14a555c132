"""baemm_b200 -- BAEMM's boundary-element Helmholtz operator path on B200 (sm_100a).

The compute lives in libbaemm_cuda.so (hand-written CUDA kernels behind the C
ABI of include/baemm.h); this package is the Python mirror of the reference
class Helmholtz_OpenCL plus mesh utilities.  Importing it does not load the
shared library; the first Helmholtz_CUDA construction does, and fails loudly
when the library or a CUDA device is missing.
"""
from ._capi import APPLY_FP32, APPLY_FP64, APPLY_TC, WAVE_PLANE, WAVE_RADIAL, BaemmError, lib  # noqa: F401
from .helmholtz import Helmholtz_CUDA, Packer, WaveType  # noqa: F401
from . import meshes  # noqa: F401

__version__ = "0.1.0"
