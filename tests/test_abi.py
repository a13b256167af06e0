"""The C-ABI library loads and exports every symbol include/*.h declares (no
device calls)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(eimp_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("eimp_create", "eimp_gpu_initialize", "eimp_gpu_run_cref_pbwt", "eimp_phase_targets",
              "eimp_imp_prepare", "eimp_imp_bunch"):
        assert n in names


def test_library_exports_all_declared_symbols():
    from eimp_b200 import build
    lib = build.build()
    L = ctypes.CDLL(lib)
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"


def test_python_binding_covers_header():
    from eimp_b200 import _lib
    assert set(_lib.exported_names()) == set(declared_symbols())


def test_no_device_means_loud_failure():
    """Without a device, context creation fails with an error (no CPU path)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    from eimp_b200.engine import Context
    with pytest.raises(Exception):
        Context(0)


def test_besthaps_noalloc_rejects_oversized_batches():
    """Batches beyond the fixed scratch array are refused on the host before
    any device work (the pointers are never dereferenced)."""
    from eimp_b200 import build
    L = ctypes.CDLL(build.build())
    f = L.eimp_besthaps_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    dummy = 0x1000
    # 5 targets x 2^20 haplotypes > 4 Mi entries -> EIMP_E_CAPACITY (3)
    assert f(None, 5, 10, dummy, dummy, 1 << 20, 4, dummy, dummy) == 3
    # missing buffers -> EIMP_E_ARG (2)
    assert f(None, 1, 10, None, dummy, 100, 4, dummy, dummy) == 2
