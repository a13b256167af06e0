"""ctypes binding of libeimp_b200.so (the C ABI in include/eimp_gpu.h).

The library is the product: every call runs CUDA kernels on the device.  If it
is missing or no GPU is present, the calls fail loudly -- there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libeimp_b200.so")

EIMP_OK, EIMP_E_CUDA, EIMP_E_ARG, EIMP_E_CAPACITY, EIMP_E_BEAM_EMPTY, EIMP_E_NOMEM = range(6)

_vp = C.c_void_p
_sz = C.c_size_t
_i32 = C.c_int


class EimpSiteStatsOpts(C.Structure):
    """eimp_site_stats_opts (include/eimp_gpu.h)"""
    _fields_ = [("overwriteCalls", C.c_int), ("improveCalls", C.c_int), ("r2filter", C.c_float),
                ("maffilter", C.c_float)]


class EimpPhaseParams(C.Structure):
    """eimp_phase_params (include/eimp_gpu.h)"""
    _fields_ = [("K", C.c_int), ("hsize", C.c_int), ("beamwidth", C.c_int), ("delta", C.c_int),
                ("hsize_fast", C.c_int), ("beamwidth_fast", C.c_int), ("delta_fast", C.c_int),
                ("cMmaxsplit", C.c_float), ("expectIBDcM", C.c_float), ("hist", C.c_float),
                ("pErr", C.c_float), ("pLimit", C.c_float), ("minfixsize", C.c_float),
                ("maxfixsize", C.c_float), ("minfixthr", C.c_float), ("maxfixthr", C.c_float),
                ("doPrePhasing", C.c_int), ("doRevPhasing", C.c_int)]


# (name, restype, argtypes) of every exported entry point
_PROTOS = [
    ("eimp_create", _i32, [_i32, C.POINTER(_vp)]),
    ("eimp_destroy", None, [_vp]),
    ("eimp_last_error", C.c_char_p, [_vp]),
    ("eimp_synchronize", _i32, [_vp]),
    ("eimp_kernel_launches", C.c_uint64, [_vp]),
    ("eimp_stream", _vp, [_vp]),
    ("eimp_set_timing", C.c_int, [_vp, C.c_int]),
    ("eimp_phase_stage_ms", C.c_int, [_vp, _vp, C.c_int]),
    ("eimp_capture_begin", C.c_int, [_vp]),
    ("eimp_capture_end", C.c_int, [_vp]),
    ("eimp_graph_launch", C.c_int, [_vp]),
    ("eimp_phase_reserve", C.c_int, [_vp, C.POINTER(EimpPhaseParams), _sz, _sz]),
    ("eimp_set_launch_shape", C.c_int, [_vp, C.c_int, C.c_int]),
    ("eimp_get_launch_shape", C.c_int, [_vp, C.c_int, C.POINTER(C.c_int)]),
    ("eimp_gpu_initialize", _i32, [_vp, _sz, _sz, _sz, _sz, _sz, _sz, _vp]),
    ("eimp_gpu_block_size", _sz, [_vp]),
    ("eimp_gpu_run_cref_pbwt", _i32, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("eimp_phase_set_reference", _i32, [_vp, _sz, _sz, _vp, _vp, _vp]),
    ("eimp_phase_set_reference_dev", _i32, [_vp, _sz, _sz, _vp, _sz, _vp, _vp]),
    ("eimp_phase_set_haploid_ref", _i32, [_vp, _sz, _vp]),
    ("eimp_phase_haploid_targets", _i32, [_vp, _sz, _vp]),
    ("eimp_imp_set_haploid_ref", _i32, [_vp, _sz, _vp]),
    ("eimp_imp_haploid_targets", _i32, [_vp, _sz, _vp]),
    ("eimp_phase_prep", _i32, [_vp, C.POINTER(EimpPhaseParams), _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("eimp_phase_cref_pbwt", _i32, [_vp, C.POINTER(EimpPhaseParams), _sz, _vp, C.POINTER(_sz), _vp, _vp, _vp, _vp]),
    ("eimp_phase_targets", _i32, [_vp, C.POINTER(EimpPhaseParams), _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("eimp_phase_targets_dev", _i32, [_vp, C.POINTER(EimpPhaseParams), _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("eimp_imp_set_reference", _i32, [_vp, _sz, _sz, _vp, _vp, _sz, _vp, _vp]),
    ("eimp_imp_set_reference_dev", _i32, [_vp, _sz, _sz, _vp, _vp, _sz, _vp, _vp]),
    ("eimp_imp_prepare", _i32, [_vp, _sz, _vp, _vp, _i32, _i32, _sz]),
    ("eimp_imp_prepare_dev", _i32, [_vp, _sz, _vp, _vp, _i32, _i32, _sz]),
    ("eimp_imp_bunch", _i32, [_vp, _sz, _sz, _vp, _vp]),
    ("eimp_imp_bunch_dev", _i32, [_vp, _sz, _sz, _vp, _sz, _vp, _sz]),
    ("eimp_imp_matches", _i32, [_vp, _sz, _vp, _sz, C.POINTER(_sz)]),
    ("eimp_imp_phased_dosages", _i32, [_vp, _vp, _vp]),
    ("eimp_phase_exclude_self", _i32, [_vp, C.c_int64]),
    ("eimp_phase_start_phases", _i32, [_vp, _sz, _vp]),
    ("eimp_qref_index", _i32, [_vp, _sz, _sz, _sz, _vp]),
    ("eimp_qref_decode", _i32, [_vp, _vp, _sz, _sz, _sz, _vp, _sz, _vp]),
    ("eimp_qref_decode_masked", _i32, [_vp, _vp, _sz, _sz, _sz, _sz, _vp, _vp, _sz, _vp, _vp, _sz, _vp]),
    ("eimp_qref_decode_dev", _i32, [_vp, _vp, _vp, _sz, _sz, _vp, _sz]),
    ("eimp_imp_bunch_stats", _i32, [_vp, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("eimp_imp_improve_stats", _i32, [_vp, _vp, _vp, _i32]),
    ("eimp_imp_site_stats_dev", _i32, [_vp, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _vp, _sz, _vp, _vp, _sz, _vp, _sz,
                                       _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("eimp_imp_refpbwt", _i32, [_vp, _vp, _vp]),
    ("eimp_imp_prefix_slice", _i32, [_vp, _sz, _sz, _sz, _vp]),
    ("eimp_transpose_bits_dev", _i32, [_vp, _vp, _sz, _sz, _vp, _sz, _sz]),
    ("eimp_besthaps_noalloc", _i32, [_vp, _sz, _sz, _vp, _vp, _sz, _sz, _vp, _vp]),
]

_lib = None


class EimpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"eimp error {code}: {msg}")
        self.code = code


def load():
    """Load libeimp_b200.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(f"{LIBPATH} is not built: run `python -m eimp_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(LIBPATH)
    for name, res, args in _PROTOS:
        f = getattr(L, name, None)
        if f is None:
            continue
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def exported_names():
    return [n for n, _, _ in _PROTOS]


def ptr(a) -> int | None:
    """Address of a C-contiguous numpy array / torch tensor (None passes NULL).

    The C ABI takes plain row-major buffers; a strided view would be read as
    if it were row-major, so non-contiguous inputs are rejected."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor passed to libeimp_b200 must be contiguous")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array passed to libeimp_b200 must be C-contiguous")
    return a.ctypes.data
