"""ctypes binding of the reference's own GPU engine
(oracle/_ref/libeimp_refgpu.so: GPUEngine.cu and GPUKernels.cu -- crefTKernel,
pbwtPartedKernel -- compiled unmodified for sm_100a; oracle/Makefile target
``refgpu``).

TEST INFRASTRUCTURE ONLY: tests/ and bench.py's reference-baseline leg run it
beside the product's drop-in (eimp_gpu_run_cref_pbwt, the same interface) on
the same inputs, for parity and timing; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "_ref", "libeimp_refgpu.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIBPATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIBPATH)
        vp, sz = C.c_void_p, C.c_size_t
        L.refgpu_last_error.restype = C.c_char_p
        L.refgpu_create.restype = vp
        L.refgpu_create.argtypes = [C.c_int]
        L.refgpu_initialize.restype = C.c_int
        L.refgpu_initialize.argtypes = [vp, sz, sz, sz, sz, sz, sz, vp]
        L.refgpu_block_size.restype = sz
        L.refgpu_block_size.argtypes = [vp]
        L.refgpu_run.restype = C.c_int
        L.refgpu_run.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp]
        L.refgpu_destroy.argtypes = [vp]
        _lib = L
    return _lib


def _ptrs(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


class RefGPUEngine:
    """GPUEngine (GPUEngine.h:41-99) of the reference, same methods."""

    def __init__(self, index: int = 0):
        self.L = lib()
        self.h = self.L.refgpu_create(index)

    def _check(self, rc):
        if rc:
            raise RuntimeError("reference GPUEngine: " + self.L.refgpu_last_error().decode())

    def initialize(self, K, Kwords, M, Nrefhapscorr, NrefhapsAD, refTCapacity, refTData: np.ndarray):
        self._ref = np.ascontiguousarray(refTData)
        self._check(self.L.refgpu_initialize(self.h, K, Kwords, M, Nrefhapscorr, NrefhapsAD, refTCapacity,
                                             self._ref.ctypes.data))

    def getBlockSize(self) -> int:
        return int(self.L.refgpu_block_size(self.h))

    def runCrefPBWTKernel(self, tgtData, splitdata, besthapdata, crefTOffsets, cPBWT, count0s):
        off = np.ascontiguousarray(crefTOffsets, np.uint32)
        self._check(self.L.refgpu_run(self.h, len(tgtData), _ptrs(tgtData), _ptrs(splitdata), _ptrs(besthapdata),
                                      off.ctypes.data, _ptrs(cPBWT), _ptrs(count0s)))

    def free(self):
        if self.h:
            self.L.refgpu_destroy(self.h)
            self.h = None
