"""ctypes binding of the reference's own output writer numbers
(oracle/_ref/libeimp_refwriter.so: VCFData::writeVCFImputedBunch compiled from
the reference tree by ``make -C oracle refwriter``).

TEST INFRASTRUCTURE ONLY: the tests use it to pin the oracle restatement of the
output statistics and the GPU kernel to what the reference's writer puts into
its records.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "_ref", "libeimp_refwriter.so")

# htslib's bit patterns for a missing value and the end of a shorter vector
FLOAT_MISSING = np.uint32(0x7F800001).view(np.float32)
FLOAT_VECTOR_END = np.uint32(0x7F800002).view(np.float32)
INT32_VECTOR_END = np.int32(-2147483647)

_lib = None


def available() -> bool:
    return os.path.exists(LIBPATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIBPATH)
        p = C.c_void_p
        L.refw_write_bunch.restype = C.c_int
        L.refw_write_bunch.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, p, C.c_size_t, p, p,
                                       C.c_size_t, p, p, p, C.c_size_t, p, p, p, C.c_int, C.c_int, C.c_float,
                                       C.c_float, p, p, p, p, p, p, p, p, p, p]
        _lib = L
    return _lib


def write_bunch(mref_begin, bits, dos, phased, pdm, pdp, gt, typed, Mref, af_full, haploid=None,
                overwriteCalls=False, improveCalls=False, r2filter=0.0, maffilter=0.0, want_ds=True, want_gp=True,
                stale=np.float32(-7.0)):
    """Run the reference's writeVCFImputedBunch on one bunch and return what its
    records hold.  Inputs as for oracle.restate.site_stats; haploid: N bytes.
    DS/GP entries the writer leaves unset keep `stale`."""
    c = np.ascontiguousarray
    nh, nsites = dos.shape
    N, M = gt.shape
    typed = c(np.asarray(typed, np.int64))
    bits, dos, phased = c(bits, np.uint64), c(dos, np.float32), c(phased, np.uint64)
    pdm, pdp, gt, af_full = c(pdm, np.float32), c(pdp, np.float32), c(gt, np.uint8), c(af_full, np.float32)
    hap = c(np.asarray(haploid, np.uint8)) if haploid is not None else None
    written = np.zeros(nsites, np.uint8)
    ads = np.zeros((nh, nsites), np.float32)
    gtv = np.zeros((nh, nsites), np.int32)
    ds = np.full((N, nsites), stale, np.float32) if want_ds else None
    gp = np.full((3 * N, nsites), stale, np.float32) if want_gp else None
    info = np.zeros((nsites, 4), np.float32)
    acan = np.zeros((nsites, 2), np.int32)
    typedflag = np.zeros(nsites, np.uint8)
    counters = np.zeros(6, np.uint64)
    totals = np.zeros(5, np.float64)
    ptr = lambda a: a.ctypes.data if a is not None else None  # noqa: E731
    rc = lib().refw_write_bunch(N, Mref, mref_begin, nsites, ptr(bits), bits.shape[1], ptr(dos), ptr(phased),
                                phased.shape[1], ptr(pdm), ptr(pdp), ptr(gt), M, ptr(typed), ptr(af_full), ptr(hap),
                                int(overwriteCalls), int(improveCalls), r2filter, maffilter, ptr(written), ptr(ads),
                                ptr(gtv), ptr(ds), ptr(gp), ptr(info), ptr(acan), ptr(typedflag), ptr(counters),
                                ptr(totals))
    if rc:
        raise RuntimeError(f"reference writer harness failed ({rc})")
    return dict(written=written, ads=ads, gtv=gtv, ds=ds, gp=gp, refpanelaf=info[:, 0], af=info[:, 1],
                maf=info[:, 2], r2=info[:, 3], ac=acan[:, 0], an=acan[:, 1], typed=typedflag,
                conflicts=int(counters[0]), improve_counts=counters[1:].astype(np.int64), improve_totals=totals)
