"""ctypes binding of the reference-compiled oracle (oracle/_ref/libeimp_refcore.so).

TEST INFRASTRUCTURE ONLY.  The library is the reference's own hot-path C++
(Target, PBWT, Beam, TargetImp, PBWTImputer) built from the read-only reference
sources by ``make -C oracle ref``; this module lets tests, the golden-fixture
generator and bench.py's CPU-baseline leg call it.  The product never imports
it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from eimp_b200.bits import W

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "_ref", "libeimp_refcore.so")

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

_lib = None


def available() -> bool:
    return os.path.exists(LIBPATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIBPATH)
        L.refo_create.restype = C.c_void_p
        L.refo_create.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, _u64p, _u64p, _u64p, _i64p,
                                  _f32p, _f32p, _f32p, C.c_size_t, _u8p]
        L.refo_destroy.argtypes = [C.c_void_p]
        L.refo_set_iteration.argtypes = [C.c_void_p, C.c_size_t, C.c_int]
        L.refo_set_haploids.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.refo_imp_K.restype = C.c_size_t
        L.refo_imp_K.argtypes = [C.c_void_p]
        L.refo_imp_ntargethaps.restype = C.c_size_t
        L.refo_imp_ntargethaps.argtypes = [C.c_void_p]
        L.refo_set_start_phases.argtypes = [C.c_void_p, _u8p]
        L.refo_set_params.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int]
        L.refo_prep.restype = C.c_long
        L.refo_prep.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, _i64p, _u64p, _i64p, _i64p,
                                C.POINTER(C.c_size_t), _f32p]
        L.refo_cref_pbwt.restype = C.c_long
        L.refo_cref_pbwt.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
        L.refo_phase.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_float, C.c_float, C.c_float,
                                 C.c_float, C.c_int, C.c_int, _u64p, _u64p, _f32p, _f32p,
                                 C.POINTER(C.c_float), C.POINTER(C.c_size_t)]
        L.refo_phase_range.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_int, C.c_size_t, C.c_float,
                                       C.c_float, C.c_float, C.c_float, C.c_int, C.c_int,
                                       _u64p, _u64p, _f32p, _f32p]
        L.refo_imp_create.restype = C.c_void_p
        L.refo_imp_create.argtypes = [C.c_void_p, _u64p, C.c_uint, C.c_int, C.c_int]
        L.refo_imp_destroy.argtypes = [C.c_void_p]
        L.refo_imp_retarget.argtypes = [C.c_void_p, _u64p, C.c_uint]
        L.refo_imp_nmatches.restype = C.c_size_t
        L.refo_imp_nmatches.argtypes = [C.c_void_p, C.c_size_t]
        L.refo_imp_matches.argtypes = [C.c_void_p, C.c_size_t, _i64p]
        L.refo_imp_refpbwt.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.refo_imp_bunch.argtypes = [C.c_void_p, C.c_size_t, C.c_uint, _u64p, _f32p]
        L.refo_rle_encode.restype = C.c_long
        L.refo_rle_encode.argtypes = [_u64p, C.c_size_t, _u8p]
        L.refo_rle_decode.argtypes = [_u8p, C.c_size_t, _u64p, C.c_size_t]
        L.refo_rle_decode_masked.restype = C.c_size_t
        L.refo_rle_decode_masked.argtypes = [_u8p, C.c_size_t, _u64p, C.c_size_t, _u64p, C.c_size_t, _u8p]
        L.refo_qref_decode.restype = C.c_int
        L.refo_qref_decode.argtypes = [_u8p, C.c_size_t, C.c_size_t, C.c_size_t, _u64p]
        _lib = L
    return _lib


def rle_encode(words: np.ndarray):
    """The reference's runlengthEncode (utils.h:155-191): bytes, or None where
    it gives up (the encoding would not be shorter)."""
    w = np.ascontiguousarray(words, np.uint64)
    out = np.zeros(w.size * 8 + 3, np.uint8)
    n = lib().refo_rle_encode(w, w.size, out)
    return None if n < 0 else out[:n].copy()


def rle_decode(enc: np.ndarray, nwords: int) -> np.ndarray:
    """The reference's runlengthDecode (utils.h:194-), no masked samples; the
    sequence must be well-formed (the reference exits on a truncated one)."""
    e = np.ascontiguousarray(enc, np.uint8)
    out = np.zeros(nwords, np.uint64)
    lib().refo_rle_decode(e if e.size else np.zeros(1, np.uint8), e.size, out, nwords)
    return out


def rle_decode_masked(enc: np.ndarray, nwords: int, masked, masked_haploid):
    """The reference's runlengthDecode with masked samples (utils.h:194-):
    (the kept haplotypes in nwords words, the masked variant alleles it
    counts).  masked: ascending sample indices; the sequence must be
    well-formed."""
    e = np.ascontiguousarray(enc, np.uint8)
    out = np.zeros(nwords, np.uint64)
    m = np.ascontiguousarray(masked, np.uint64)
    mh = np.ascontiguousarray(masked_haploid, np.uint8)
    n = lib().refo_rle_decode_masked(e if e.size else np.zeros(1, np.uint8), e.size, out, nwords,
                                     m if m.size else np.zeros(1, np.uint64), m.size,
                                     mh if mh.size else np.zeros(1, np.uint8))
    return out, int(n)


def qref_decode(section: np.ndarray, Mref: int, nwords: int):
    """A Qref haplotype section decoded by the reference's own runlengthDecode
    (the decode part of VCFData::qRefLoadNextVariant): (rows, status)."""
    sec = np.ascontiguousarray(section, np.uint8)
    out = np.zeros((Mref, nwords), np.uint64)
    rc = lib().refo_qref_decode(sec, sec.size, Mref, nwords, out)
    return out, rc


class PhaseParams:
    """Phasing parameters with the reference's defaults (Args.cpp:274-299)."""

    def __init__(self, K=10000, hsize=100, beamwidth=128, delta=24, cMmaxsplit=0.125,
                 hsize_fast=30, beamwidth_fast=64, delta_fast=10, expectIBDcM=2.0,
                 hist=1.0, pErr=0.003, pLimit=None, doPrePhasing=False, doRevPhasing=True):
        self.K = K
        self.hsize = hsize
        self.beamwidth = beamwidth
        self.delta = delta
        self.cMmaxsplit = cMmaxsplit
        self.hsize_fast = hsize_fast
        self.beamwidth_fast = beamwidth_fast
        self.delta_fast = delta_fast
        self.expectIBDcM = expectIBDcM
        self.hist = hist
        self.pErr = pErr
        self.pLimit = pErr if pLimit is None else pLimit
        self.doPrePhasing = doPrePhasing
        self.doRevPhasing = doRevPhasing


class RefCore:
    """The reference's hot path over one panel + one target group."""

    def __init__(self, panel, targets, af_common=None):
        from eimp_b200.synth import typed_views
        L = lib()
        self.nhaps = panel.nhaps
        self.Mref = panel.nsites
        self.typed = np.ascontiguousarray(targets.typed, dtype=np.int64)
        self.M = len(self.typed)
        self.ntarget = targets.gt.shape[0]
        hm, sm, cm = typed_views(panel, self.typed)
        self.hapmajor_typed, self.sitemajor_typed, self.cm_typed = hm, sm, cm
        self.sitemajor_full = np.ascontiguousarray(panel.sitemajor)
        self.af_full = np.ascontiguousarray(panel.af, dtype=np.float32)
        if af_common is None:
            af_common = self.af_full[self.typed]
        self.af_common = np.ascontiguousarray(af_common, dtype=np.float32)
        self.gt = np.ascontiguousarray(targets.gt, dtype=np.uint8)
        self.h = L.refo_create(self.nhaps, self.M, self.Mref, hm, sm, self.sitemajor_full, self.typed,
                               cm, self.af_full, self.af_common, self.ntarget, self.gt)
        self.params = None

    @classmethod
    def typed_only(cls, hapmajor_typed, sitemajor_typed, cm_typed, gt, af_common):
        """A handle over a typed-site panel only (phasing; no imputation) --
        e.g. the panel of a phasing iteration after the first, the reference
        haplotypes followed by the phased targets."""
        self = cls.__new__(cls)
        L = lib()
        self.nhaps = hapmajor_typed.shape[0]
        self.M = sitemajor_typed.shape[0]
        self.Mref = self.M
        self.typed = np.arange(self.M, dtype=np.int64)
        self.ntarget = gt.shape[0]
        self.hapmajor_typed = np.ascontiguousarray(hapmajor_typed, np.uint64)
        self.sitemajor_typed = np.ascontiguousarray(sitemajor_typed, np.uint64)
        self.cm_typed = np.ascontiguousarray(cm_typed, np.float32)
        self.sitemajor_full = self.sitemajor_typed
        self.af_common = np.ascontiguousarray(af_common, np.float32)
        self.af_full = self.af_common
        self.gt = np.ascontiguousarray(gt, np.uint8)
        self.h = L.refo_create(self.nhaps, self.M, self.Mref, self.hapmajor_typed, self.sitemajor_typed,
                               self.sitemajor_full, self.typed, self.cm_typed, self.af_full, self.af_common,
                               self.ntarget, self.gt)
        self.params = None
        return self

    @property
    def ncorr(self) -> int:
        """Haplotypes a target chooses its K best from (PBWTPhaser.cpp:408-476):
        the panel less one per haploid sample, less the target's own two in
        iterations after the first."""
        n = self.nhaps - getattr(self, "nhaploid_ref", 0)
        return n - 2 if getattr(self, "nhaps_orig", 0) else n

    def set_haploids(self, ref=None, tgt=None):
        """Ploidy of the panel's samples (nhaps/2 flags) and of the targets
        (ntarget flags), 1 = haploid; None = all diploid.  Call after
        set_iteration in iterations after the first."""
        self._hr = None if ref is None else np.ascontiguousarray(ref, np.uint8)
        self._ht = None if tgt is None else np.ascontiguousarray(tgt, np.uint8)
        lib().refo_set_haploids(self.h, None if self._hr is None else self._hr.ctypes.data,
                                None if self._ht is None else self._ht.ctypes.data)
        self.nhaploid_ref = 0 if self._hr is None else int(self._hr.sum())

    def set_start_phases(self, phases):
        """VCFData::chunkStartPhase of every target (0 = Ref)."""
        lib().refo_set_start_phases(self.h, np.ascontiguousarray(phases, np.uint8))

    def set_iteration(self, nhaps_orig: int, last_iter: bool):
        """Phasing iteration after the first: the first nhaps_orig haplotypes
        are the reference, target t is sample nhaps_orig/2 + t of the panel."""
        lib().refo_set_iteration(self.h, nhaps_orig, int(last_iter))
        self.nhaps_orig = nhaps_orig

    def close(self):
        if self.h:
            lib().refo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p: PhaseParams):
        self.params = p
        lib().refo_set_params(p.hsize, p.beamwidth, p.delta, p.cMmaxsplit, p.hsize_fast,
                              p.beamwidth_fast, p.delta_fast)

    def prep(self, t: int):
        K = min(self.params.K, self.ncorr)
        bh = np.zeros(K, np.int64)
        monos = np.zeros(W(self.M), np.uint64)
        splits = np.zeros(self.M + 1, np.int64)
        calls = np.zeros(self.M + 1, np.int64)
        diffs = np.zeros(self.M + 2, np.float32)
        nc = C.c_size_t(0)
        S = lib().refo_prep(self.h, t, K, bh, monos, splits, calls, C.byref(nc), diffs)
        return dict(besthaps=bh, monos=monos, splits=splits[:S].copy(), calls=calls[:nc.value].copy(),
                    cmdiffs=diffs[:S + 1].copy() if nc.value else diffs[:0].copy())

    def cref_pbwt(self, t: int):
        K = min(self.params.K, self.ncorr)
        Mp = lib().refo_cref_pbwt(self.h, t, K, None, None, None)
        cref = np.zeros((Mp, W(K)), np.uint64)
        c0 = np.zeros(Mp, np.int32)
        kw = 2 * ((K + 31) // 32)
        pb = np.zeros((2 * Mp, kw), np.uint32)
        lib().refo_cref_pbwt(self.h, t, K, cref.ctypes.data, c0.ctypes.data, pb.ctypes.data)
        return cref, c0, pb

    def phase(self, t: int):
        p = self.params
        K = min(p.K, self.ncorr)
        mat = np.zeros(W(self.M), np.uint64)
        pat = np.zeros(W(self.M), np.uint64)
        dm = np.zeros(self.M, np.float32)
        dp = np.zeros(self.M, np.float32)
        tc = C.c_float(0)
        nc = C.c_size_t(0)
        lib().refo_phase(self.h, t, K, p.expectIBDcM, p.hist, p.pErr, p.pLimit, int(p.doPrePhasing),
                         int(p.doRevPhasing), mat, pat, dm, dp, C.byref(tc), C.byref(nc))
        return mat, pat, dm, dp, tc.value, nc.value

    def phase_range(self, t0: int, t1: int, nthreads: int):
        p = self.params
        K = min(p.K, self.ncorr)
        n = t1 - t0
        mats = np.zeros((n, W(self.M)), np.uint64)
        pats = np.zeros((n, W(self.M)), np.uint64)
        dm = np.zeros((n, self.M), np.float32)
        dp = np.zeros((n, self.M), np.float32)
        lib().refo_phase_range(self.h, t0, t1, nthreads, K, p.expectIBDcM, p.hist, p.pErr, p.pLimit,
                               int(p.doPrePhasing), int(p.doRevPhasing), mats, pats, dm, dp)
        return mats, pats, dm, dp

    def imputer(self, phased: np.ndarray, nthreads: int = 1, setmaxerrors: int = 0, imputeCalls: bool = False):
        return RefImputer(self, phased, nthreads, setmaxerrors, imputeCalls)


class RefImputer:
    def __init__(self, core: RefCore, phased: np.ndarray, nthreads: int, setmaxerrors: int, imputeCalls: bool):
        self.core = core
        phased = np.ascontiguousarray(phased, dtype=np.uint64)
        assert phased.shape == (2 * core.ntarget, W(core.M))
        self.h = lib().refo_imp_create(core.h, phased, nthreads, setmaxerrors, int(imputeCalls))

    def close(self):
        if self.h:
            lib().refo_imp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def retarget(self, phased: np.ndarray, nthreads: int = 1):
        """Matches of new phased haplotypes of the same targets against the
        PBWT already built (the match part of prepareImputation)."""
        phased = np.ascontiguousarray(phased, dtype=np.uint64)
        assert phased.shape == (2 * self.core.ntarget, W(self.core.M))
        lib().refo_imp_retarget(self.h, phased, nthreads)

    def matches(self, hap: int) -> np.ndarray:
        n = lib().refo_imp_nmatches(self.h, hap)
        out = np.zeros((n, 4), np.int64)
        if n:
            lib().refo_imp_matches(self.h, hap, out)
        return out

    @property
    def K(self) -> int:
        """haplotypes of the imputation PBWT (one per haploid panel sample)"""
        return int(lib().refo_imp_K(self.h))

    @property
    def ntargethaps(self) -> int:
        return int(lib().refo_imp_ntargethaps(self.h))

    def refpbwt(self):
        M, K = self.core.M, self.K
        kw = 2 * ((K + 31) // 32)
        compr = np.zeros((M, kw), np.uint32)
        absperm = np.zeros((M + 1, K), np.int32)
        lib().refo_imp_refpbwt(self.h, compr.ctypes.data, absperm.ctypes.data)
        return compr, absperm

    def bunch(self, bsize: int, nthreads: int = 1):
        nh = 2 * self.core.ntarget
        bits = np.zeros((nh, W(bsize)), np.uint64)
        dos = np.zeros((nh, bsize), np.float32)
        lib().refo_imp_bunch(self.h, bsize, nthreads, bits, dos)
        return bits, dos
