"""ctypes binding of the C restatement oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use this module as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from eimp_b200.bits import W, pack_genotypes

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "liboracle.so")

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


class PhaseParamsC(C.Structure):
    _fields_ = [("K", C.c_int), ("hsize", C.c_int), ("beamwidth", C.c_int), ("delta", C.c_int),
                ("hsize_fast", C.c_int), ("beamwidth_fast", C.c_int), ("delta_fast", C.c_int),
                ("cMmaxsplit", C.c_float), ("expectIBDcM", C.c_float), ("hist", C.c_float),
                ("pErr", C.c_float), ("pLimit", C.c_float), ("minfixsize", C.c_float),
                ("maxfixsize", C.c_float), ("minfixthr", C.c_float), ("maxfixthr", C.c_float),
                ("doPrePhasing", C.c_int), ("doRevPhasing", C.c_int)]


def params_c(K=10000, hsize=100, beamwidth=128, delta=24, hsize_fast=30, beamwidth_fast=64, delta_fast=10,
             cMmaxsplit=0.125, expectIBDcM=2.0, hist=1.0, pErr=0.003, pLimit=None, doPrePhasing=False,
             doRevPhasing=True) -> PhaseParamsC:
    return PhaseParamsC(K, hsize, beamwidth, delta, hsize_fast, beamwidth_fast, delta_fast, cMmaxsplit,
                        expectIBDcM, hist, pErr, pErr if pLimit is None else pLimit, 0.5, 0.9, 0.99, 1.0,
                        int(doPrePhasing), int(doRevPhasing))


_lib = None


def available() -> bool:
    return os.path.exists(LIBPATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIBPATH)
        L.eo_besthaps.argtypes = [_u64p, _u64p, C.c_size_t, C.c_size_t, C.c_size_t, _i64p, C.c_void_p]
        L.eo_monos.argtypes = [_u64p, C.c_size_t, C.c_size_t, _i64p, C.c_size_t, _u64p]
        L.eo_calllocs.restype = C.c_long
        L.eo_calllocs.argtypes = [_u8p, _u64p, _f32p, C.c_size_t, C.c_float, _i64p, _i64p,
                                  C.POINTER(C.c_size_t), _f32p]
        L.eo_cref.argtypes = [_u8p, _u64p, C.c_size_t, C.c_size_t, _i64p, C.c_size_t, _i64p, C.c_size_t,
                              _u64p, _i32p]
        L.eo_pbwt.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_int, _u32p, C.c_void_p, C.c_void_p]
        L.eo_rank.restype = C.c_int
        L.eo_rank.argtypes = [_u32p, C.c_int, C.c_int]
        L.eo_smmatches.restype = C.c_long
        L.eo_smmatches.argtypes = [_u32p, _i32p, C.c_size_t, C.c_size_t, _u64p, _i64p, C.c_size_t, C.c_int,
                                   _i64p, C.c_size_t]
        L.eo_impute.argtypes = [_i64p, C.c_size_t, _i32p, C.c_size_t, _u64p, C.c_size_t, C.c_size_t, _i64p,
                                C.c_size_t, _f32p, C.c_size_t, _i64p, C.c_size_t, C.c_int, _u64p, _u64p,
                                _f32p, _u8p, C.c_void_p]
        L.eo_site_stats.restype = C.c_long
        L.eo_site_stats.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, _u64p, C.c_size_t, _f32p, _u64p, C.c_size_t,
                                    _f32p, _f32p, _u8p, C.c_size_t, _i32p, _u8p, _f32p, C.c_void_p, C.c_int,
                                    C.c_int, C.c_float, C.c_float, _f32p, _u64p, C.c_void_p, C.c_void_p, _f32p,
                                    _f32p, _f32p, _i32p, _i32p, _u8p, _u64p, _f64p]
        L.eo_rle_encode.restype = C.c_long
        L.eo_rle_encode.argtypes = [_u64p, C.c_size_t, _u8p]
        L.eo_rle_decode.restype = C.c_int
        L.eo_rle_decode.argtypes = [_u8p, C.c_size_t, _u64p, C.c_size_t]
        L.eo_qref_decode.restype = C.c_int
        L.eo_qref_decode.argtypes = [_u8p, C.c_size_t, C.c_size_t, C.c_size_t, _u64p]
        L.eo_phase.restype = C.c_int
        L.eo_phase.argtypes = [_u8p, _u64p, _u64p, _f32p, C.c_size_t, C.c_size_t, C.POINTER(PhaseParamsC),
                               _u64p, _u64p, _f32p, _f32p, C.POINTER(C.c_float), C.POINTER(C.c_size_t)]
        L.eo_phase_many.restype = C.c_int
        L.eo_phase_many.argtypes = [_u8p, C.c_size_t, _u64p, _u64p, _f32p, C.c_size_t, C.c_size_t,
                                    C.POINTER(PhaseParamsC), C.c_int, _u64p, _u64p, _f32p, _f32p]
        _lib = L
    return _lib


def besthaps(gt_row: np.ndarray, hapmajor: np.ndarray, K: int):
    nh, wM = hapmajor.shape
    gtw = np.ascontiguousarray(pack_genotypes(gt_row))
    out = np.zeros(min(K, nh), np.int64)
    nerr = np.zeros(nh, np.uint32)
    lib().eo_besthaps(gtw, np.ascontiguousarray(hapmajor), nh, wM, K, out, nerr.ctypes.data)
    return out, nerr


def monos(hapmajor: np.ndarray, M: int, bh: np.ndarray):
    nh, wM = hapmajor.shape
    out = np.zeros(wM, np.uint64)
    lib().eo_monos(np.ascontiguousarray(hapmajor), wM, M, np.ascontiguousarray(bh, np.int64), len(bh), out)
    return out


def calllocs(gt_row, monos_w, cm, cMmaxsplit=0.125):
    M = len(gt_row)
    splits = np.zeros(M + 1, np.int64)
    calls = np.zeros(M + 1, np.int64)
    diffs = np.zeros(M + 2, np.float32)
    nc = C.c_size_t(0)
    S = lib().eo_calllocs(np.ascontiguousarray(gt_row, np.uint8), monos_w, np.ascontiguousarray(cm, np.float32),
                          M, cMmaxsplit, splits, calls, C.byref(nc), diffs)
    return splits[:S].copy(), calls[:nc.value].copy() if S else calls[:0].copy(), diffs[:S + 1].copy() if S else diffs[:0].copy()


def cref(gt_row, sitemajor, nhaps, bh, splits):
    M = len(gt_row)
    K = len(bh)
    Mp = 2 * len(splits) + 1
    out = np.zeros((Mp, W(K)), np.uint64)
    c0 = np.zeros(Mp, np.int32)
    lib().eo_cref(np.ascontiguousarray(gt_row, np.uint8), np.ascontiguousarray(sitemajor), M, nhaps,
                  np.ascontiguousarray(bh, np.int64), K, np.ascontiguousarray(splits, np.int64), len(splits), out, c0)
    return out, c0


def pbwt(rows: np.ndarray, K: int, reverse: bool = False, absperm: bool = False):
    Mp, rw = rows.shape
    kw = 2 * ((K + 31) // 32)
    out = np.zeros((Mp, kw), np.uint32)
    ap = np.zeros((Mp + 1, K), np.int32) if absperm else None
    c0 = np.zeros(Mp, np.int32)
    lib().eo_pbwt(np.ascontiguousarray(rows), rw, Mp, K, int(reverse), out,
                  ap.ctypes.data if ap is not None else None, c0.ctypes.data)
    return out, c0, ap


def smmatches(refpbwt, count0, M, K, hap_words, miss, setmaxerrors=0, maxmatches=None):
    if maxmatches is None:
        maxmatches = 4 * M + 64
    out = np.zeros((maxmatches, 4), np.int64)
    n = lib().eo_smmatches(np.ascontiguousarray(refpbwt), np.ascontiguousarray(count0, np.int32), M, K,
                           np.ascontiguousarray(hap_words, np.uint64), np.ascontiguousarray(miss, np.int64),
                           len(miss), setmaxerrors, out, maxmatches)
    if n < 0:
        raise RuntimeError("match buffer overflow")
    return out[:n].copy()


def impute(matches, absperm, sitemajor_full, typed, af_full, nrefhaps, miss, hap_words, imputeCalls=False,
           fp64=False):
    """TargetImp::imputeBunch of one haplotype over all panel sites: (bits,
    dosages, imputed-site flags), plus the FP64 dosage oracle (score/sum in
    double, not rounded to float) when fp64 is set."""
    Mref, wN = sitemajor_full.shape
    K = absperm.shape[1]
    bits = np.zeros(W(Mref), np.uint64)
    dos = np.zeros(Mref, np.float32)
    imp = np.zeros(Mref, np.uint8)
    d64 = np.zeros(Mref, np.float64) if fp64 else None
    m = np.ascontiguousarray(matches, np.int64).reshape(-1, 4)
    lib().eo_impute(m.reshape(-1) if len(m) else np.zeros(4, np.int64), len(m), np.ascontiguousarray(absperm, np.int32),
                    K, np.ascontiguousarray(sitemajor_full), wN, Mref, np.ascontiguousarray(typed, np.int64),
                    len(typed), np.ascontiguousarray(af_full, np.float32), nrefhaps,
                    np.ascontiguousarray(miss, np.int64) if len(miss) else np.zeros(1, np.int64), len(miss),
                    int(imputeCalls), np.ascontiguousarray(hap_words, np.uint64), bits, dos, imp,
                    d64.ctypes.data if fp64 else None)
    return (bits, dos, imp, d64) if fp64 else (bits, dos, imp)


def rle_encode(words: np.ndarray):
    """runlengthEncode (utils.h:155-191): bytes, or None (not shorter)."""
    w = np.ascontiguousarray(words, np.uint64)
    out = np.zeros(w.size * 8 + 3, np.uint8)
    n = lib().eo_rle_encode(w, w.size, out)
    return None if n < 0 else out[:n].copy()


def rle_decode(enc: np.ndarray, nwords: int):
    """runlengthDecode (utils.h:194-) without masked samples: (words, status)
    with status -1 for a truncated sequence."""
    e = np.ascontiguousarray(enc, np.uint8)
    out = np.zeros(nwords, np.uint64)
    rc = lib().eo_rle_decode(e if e.size else np.zeros(1, np.uint8), e.size, out, nwords)
    return out, rc


def qref_section(rows: np.ndarray) -> np.ndarray:
    """The haplotype section of a Qref file (qref_spec.md section I) for the
    site-major rows: each variant as <encsize u64><run-length bytes>, or
    <0><raw row> where the run-length code is not shorter."""
    parts = []
    for r in np.ascontiguousarray(rows, np.uint64):
        enc = rle_encode(r)
        if enc is None:
            parts += [np.zeros(8, np.uint8), r.view(np.uint8)]
        else:
            parts += [np.array([len(enc)], np.uint64).view(np.uint8), enc]
    return np.concatenate(parts) if parts else np.zeros(0, np.uint8)


def qref_decode(section: np.ndarray, Mref: int, nwords: int):
    """The Qref haplotype section decoded into Mref rows (VCFData::qRefLoadNextVariant):
    (rows, status) -- 0, -1 truncated run-length sequence, -2 short section."""
    s = np.ascontiguousarray(section, np.uint8)
    out = np.zeros((Mref, nwords), np.uint64)
    rc = lib().eo_qref_decode(s if s.size else np.zeros(1, np.uint8), s.size, Mref, nwords, out)
    return out, rc


def site_stats(mref_begin, bits, dos, phased, pdm, pdp, gt, typed, Mref, af_full, overwriteCalls=False,
               improveCalls=False, r2filter=0.0, maffilter=0.0, want_ds=False, want_gp=False, haploid=None):
    """VCFData::writeVCFImputedBunch's numbers for one bunch (eo_site_stats).
    bits: 2N x wb words, dos: 2N x nsites floats, phased: 2N x wM words,
    pdm/pdp: N x M phased dosages, gt: N x M, typed: ascending typed site
    indices into the Mref reference sites, haploid: N flags or None.
    improve_counts / improve_totals: the --improveCalls run statistics of the
    bunch (no change, het->het, hom->hom, het->hom, hom->het)."""
    nh, nsites = dos.shape
    N, M = gt.shape
    typed = np.asarray(typed, np.int64)
    cnt = np.searchsorted(typed, np.arange(Mref), side="right")
    typed_idx = np.maximum(cnt - 1, 0).astype(np.int32)
    is_typed = np.zeros(Mref, np.uint8)
    is_typed[typed] = 1
    wb = bits.shape[1]
    ads = np.zeros((nh, nsites), np.float32)
    gtbits = np.zeros((nh, wb), np.uint64)
    ds = np.zeros((N, nsites), np.float32) if want_ds else None
    gp = np.zeros((3 * N, nsites), np.float32) if want_gp else None
    r2 = np.zeros(nsites, np.float32)
    af = np.zeros(nsites, np.float32)
    maf = np.zeros(nsites, np.float32)
    ac = np.zeros(nsites, np.int32)
    an = np.zeros(nsites, np.int32)
    ps = np.zeros(nsites, np.uint8)
    icnt = np.zeros(5, np.uint64)
    itot = np.zeros(5, np.float64)
    hap = np.ascontiguousarray(np.asarray(haploid, np.uint8)) if haploid is not None else None
    conf = lib().eo_site_stats(N, mref_begin, nsites, np.ascontiguousarray(bits, np.uint64), wb,
                               np.ascontiguousarray(dos, np.float32), np.ascontiguousarray(phased, np.uint64),
                               phased.shape[1], np.ascontiguousarray(pdm, np.float32),
                               np.ascontiguousarray(pdp, np.float32), np.ascontiguousarray(gt, np.uint8), M,
                               typed_idx, is_typed, np.ascontiguousarray(af_full, np.float32),
                               hap.ctypes.data if hap is not None else None, int(overwriteCalls),
                               int(improveCalls), r2filter, maffilter, ads, gtbits,
                               ds.ctypes.data if ds is not None else None, gp.ctypes.data if gp is not None else None,
                               r2, af, maf, ac, an, ps, icnt, itot)
    return dict(ads=ads, gtbits=gtbits, ds=ds, gp=gp, r2=r2, af=af, maf=maf, ac=ac, an=an, passed=ps,
                conflicts=int(conf), improve_counts=icnt.astype(np.int64), improve_totals=itot)


def phase(gt_row, hapmajor, sitemajor, cm, params: PhaseParamsC):
    M = len(gt_row)
    nh = hapmajor.shape[0]
    mat = np.zeros(W(M), np.uint64)
    pat = np.zeros(W(M), np.uint64)
    dm = np.zeros(M, np.float32)
    dp = np.zeros(M, np.float32)
    tc = C.c_float(0)
    nc = C.c_size_t(0)
    rc = lib().eo_phase(np.ascontiguousarray(gt_row, np.uint8), np.ascontiguousarray(hapmajor),
                        np.ascontiguousarray(sitemajor), np.ascontiguousarray(cm, np.float32), M, nh,
                        C.byref(params), mat, pat, dm, dp, C.byref(tc), C.byref(nc))
    if rc:
        raise RuntimeError(f"oracle phasing failed ({rc})")
    return mat, pat, dm, dp, tc.value, nc.value


def phase_many(gt, hapmajor, sitemajor, cm, params: PhaseParamsC, nthreads=8):
    n, M = gt.shape
    nh = hapmajor.shape[0]
    mats = np.zeros((n, W(M)), np.uint64)
    pats = np.zeros((n, W(M)), np.uint64)
    dm = np.zeros((n, M), np.float32)
    dp = np.zeros((n, M), np.float32)
    rc = lib().eo_phase_many(np.ascontiguousarray(gt, np.uint8), n, np.ascontiguousarray(hapmajor),
                             np.ascontiguousarray(sitemajor), np.ascontiguousarray(cm, np.float32), M, nh,
                             C.byref(params), nthreads, mats, pats, dm, dp)
    if rc:
        raise RuntimeError(f"oracle phasing failed ({rc})")
    return mats, pats, dm, dp


def impute_fp64_sites(matches, sites, typed, af_full, nrefhaps_total, prefix_slice, site_bits):
    """FP64 dosage oracle on a sample of panel sites for one target haplotype:
    TargetImp::imputeBunch (TargetImp.cpp:474-558; eo_impute in
    eimp_oracle.c) with score and sum as exact integers and score/sum in
    double, without the reference's final rounding to float.

    matches: (n, 4) int [start, end, rs, re] in typed-site indices, in the
    order the match search emits them (ascending end); sites: ascending
    untyped panel sites; typed: the typed panel sites; af_full: float32 panel
    allele frequencies; prefix_slice(en, rs, re) -> gAbsPerm[en][rs..re];
    site_bits(j, refs) -> alleles (0/1) of reference haplotypes refs at
    sites[j].  Returns float64 (len(sites),), -1 where no match covers the
    site (DOSAGE_CONFLICT, :26)."""
    matches = np.asarray(matches, np.int64).reshape(-1, 4)
    starts, ends = matches[:, 0], matches[:, 1]
    n = len(matches)
    # the last typed site at or before each site (0 before the first)
    currm = np.searchsorted(np.asarray(typed), np.asarray(sites), side="right") - 1
    currm[currm < 0] = 0
    out = np.empty(len(sites), np.float64)
    n32 = np.float32(nrefhaps_total)
    for j, (s, c) in enumerate(zip(sites, currm)):
        i = int(np.searchsorted(ends, c, side="right"))     # first match with end > currm (:504-505)
        if i >= n or starts[i] > c:
            out[j] = -1.0
            continue
        af = np.float32(af_full[s])
        maf = np.float32(np.float32(1.0) - af) if af > np.float32(0.5) else af
        score = total = 0
        while i < n and starts[i] <= c:
            st, en, rs, re = (int(v) for v in matches[i])
            single = (int(c) - st + 1) * (en - int(c))
            height = re - rs + 1
            # :526: float maf * (float)size_t vs double 0.01 * size_t
            if float(np.float32(maf * n32)) < 0.01 * float(height):
                total += height * single
                if af > np.float32(0.5):
                    score += height * single
            else:
                ones = int(np.count_nonzero(site_bits(j, prefix_slice(en, rs, re))))
                total += height * single
                score += ones * single
            i += 1
        out[j] = float(score) / float(total)
    return out


def qref_mask_row(row, raw, masked, masked_haploid, nsamples, nwords_out):
    """A decoded Qref haplotype row (2 bits per sample, LSB first) with masked
    reference samples removed, as VCFData::qRefLoadNextVariant stores it for
    --excludeRefSamples (VCFData.cpp:2449-2523 for a raw vector,
    runlengthDecode utils.h:194- for a run-length code): the kept samples'
    bit pairs in order, then zeros; and the masked variant alleles it
    counts.  A raw vector counts a masked sample once if either bit is set and
    twice for a diploid 11; a run-length code counts each set bit of a
    diploid sample and, for a haploid one (stored as a homozygous pair), the
    second bit only after a set first bit."""
    row = np.asarray(row, np.uint64)
    s = np.arange(nsamples, dtype=np.int64)
    pairs = ((row[s >> 5] >> ((s & 31) * 2).astype(np.uint64)) & np.uint64(3)).astype(np.int64)
    mk = np.asarray(masked, np.int64)
    mh = np.asarray(masked_haploid, np.uint8).astype(bool)
    mp = pairs[mk]
    if raw:
        cnt = int(np.count_nonzero(mp) + np.count_nonzero((mp == 3) & ~mh))
    else:
        cnt = int(np.where(mh, mp == 3, (mp & 1) + (mp >> 1)).sum())
    keep = np.setdiff1d(s, mk)
    out = np.zeros(nwords_out * 64, np.uint8)
    kp = pairs[keep]
    out[0:2 * keep.size:2] = kp & 1
    out[1:2 * keep.size:2] = kp >> 1
    return np.packbits(out, bitorder="little").view(np.uint64), cnt


def qref_mask_af(af, an_before, an_after, masked_alleles):
    """The panel allele frequency after masking (VCFData.cpp:2429-2434,
    2517-2521): float(an_before) * af - masked, over float(an_after), in
    float arithmetic."""
    f = np.float32
    return f(f(f(an_before) * f(af)) - f(masked_alleles)) / f(an_after)
