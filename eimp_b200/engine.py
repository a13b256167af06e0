"""Host-side mirror of the reference's GPU and imputation interfaces.

* :class:`GPUEngine` -- GPUEngine (GPUEngine.h:41-99): initialize /
  getBlockSize / runCrefPBWTKernel / free, same argument meaning.
* :class:`Phaser` -- Target::prepPhase / Target::phase (Target.h:30-72) for a
  batch of targets on the device.
* :class:`PBWTImputer` -- PBWTImputer (PBWTImputer.h:30-64): prepareImputation /
  imputeBunch.

All work runs in libeimp_b200.so (CUDA, sm_100a); numpy arrays are host
buffers, torch CUDA tensors can be passed to the ``*_dev`` methods.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import _lib
from ._lib import EimpError, EimpPhaseParams, ptr
from .bits import W


class Context:
    """One eimp_ctx: a CUDA device, a stream and the device-resident state."""

    def __init__(self, device: int = 0):
        self.L = _lib.load()
        h = C.c_void_p()
        rc = self.L.eimp_create(device, C.byref(h))
        if rc != 0:
            raise EimpError(rc, f"eimp_create(device={device}) failed (no CUDA device?)")
        self.h = h.value
        self.device = device

    def check(self, rc: int):
        if rc != 0:
            raise EimpError(rc, self.L.eimp_last_error(self.h).decode())

    def synchronize(self):
        self.check(self.L.eimp_synchronize(self.h))

    @property
    def launches(self) -> int:
        return int(self.L.eimp_kernel_launches(self.h))

    @property
    def stream(self) -> int:
        return int(self.L.eimp_stream(self.h) or 0)

    def close(self):
        if getattr(self, "h", None):
            self.L.eimp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class PhaseParams:
    """Phasing parameters with the reference defaults (Args.cpp:274-299)."""
    K: int = 10000
    hsize: int = 100
    beamwidth: int = 128
    delta: int = 24
    hsize_fast: int = 30
    beamwidth_fast: int = 64
    delta_fast: int = 10
    cMmaxsplit: float = 0.125
    expectIBDcM: float = 2.0
    hist: float = 1.0
    pErr: float = 0.003
    pLimit: float | None = None
    minfixsize: float = 0.5
    maxfixsize: float = 0.9
    minfixthr: float = 0.99
    maxfixthr: float = 1.0
    doPrePhasing: bool = False
    doRevPhasing: bool = True

    def c(self) -> EimpPhaseParams:
        d = {f.name: getattr(self, f.name) for f in fields(self)}
        if d["pLimit"] is None:
            d["pLimit"] = d["pErr"]
        d["doPrePhasing"] = int(d["doPrePhasing"])
        d["doRevPhasing"] = int(d["doRevPhasing"])
        return EimpPhaseParams(**d)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class GPUEngine:
    """GPUEngine (GPUEngine.h:41-99) over libeimp_b200."""

    def __init__(self, index: int = 0, ctx: Context | None = None):
        self.ctx = ctx or Context(index)
        self.index = index

    def initialize(self, K, Kwords, M, Nrefhapscorr, NrefhapsAD, refTCapacity, refTData: np.ndarray):
        self._refT = _c(refTData, np.uint64)
        self.K, self.Kwords, self.M = K, Kwords, M
        self.ctx.check(self.ctx.L.eimp_gpu_initialize(self.ctx.h, K, Kwords, M, Nrefhapscorr, NrefhapsAD,
                                                      refTCapacity, ptr(self._refT)))

    def getBlockSize(self) -> int:
        return int(self.ctx.L.eimp_gpu_block_size(self.ctx.h))

    def runCrefPBWTKernel(self, tgtData, splitdata, besthapdata, crefTOffsets, cPBWT, count0s):
        n = len(tgtData)
        keep = [_c(a, np.uint64) for a in tgtData] + [_c(a, np.uint64) for a in splitdata] + \
               [_c(a, np.uint64) for a in besthapdata]
        P = C.c_void_p * n
        tg = P(*[ptr(a) for a in keep[:n]])
        sp = P(*[ptr(a) for a in keep[n:2 * n]])
        bh = P(*[ptr(a) for a in keep[2 * n:]])
        off = _c(crefTOffsets, np.uint32)
        for a in list(cPBWT) + list(count0s):
            if not a.flags["C_CONTIGUOUS"]:
                raise ValueError("output buffers must be contiguous")
        outp = P(*[ptr(a) for a in cPBWT])
        c0p = P(*[ptr(a) for a in count0s])
        self.ctx.check(self.ctx.L.eimp_gpu_run_cref_pbwt(self.ctx.h, n, tg, sp, bh, ptr(off), outp, c0p))

    def free(self):
        self.ctx.close()


class Phaser:
    """Target::prepPhase / Target::phase for batches of targets on the device."""

    def __init__(self, ctx: Context, hapmajor: np.ndarray, sitemajor: np.ndarray, cm: np.ndarray):
        self.ctx = ctx
        self.nhaps, self.wM = hapmajor.shape
        self.M = sitemajor.shape[0]
        self.self0 = -1
        ctx.check(ctx.L.eimp_phase_exclude_self(ctx.h, -1))
        ctx.check(ctx.L.eimp_phase_set_reference(ctx.h, self.M, self.nhaps, ptr(_c(hapmajor, np.uint64)),
                                                 ptr(_c(sitemajor, np.uint64)), ptr(_c(cm, np.float32))))
        self.nhaploid = 0

    def excludeSelf(self, first_sample: int):
        """Phasing iterations after the first: target t is sample
        first_sample + t of this reference and leaves its own haplotypes out
        of its best haplotypes (Target.cpp:791-811); -1 turns it off."""
        self.ctx.check(self.ctx.L.eimp_phase_exclude_self(self.ctx.h, int(first_sample)))
        self.self0 = int(first_sample)

    def setHaploidRef(self, haploid):
        """Haploid samples of this reference (nhaps/2 flags; None: all
        diploid): their second haplotype is never chosen and K is clamped to
        the haplotypes that exist (Target.cpp:798-838, PBWTPhaser.cpp:210)."""
        if haploid is None:
            self.ctx.check(self.ctx.L.eimp_phase_set_haploid_ref(self.ctx.h, 0, None))
            self.nhaploid = 0
            return
        f = _c(haploid, np.uint8)
        self.ctx.check(self.ctx.L.eimp_phase_set_haploid_ref(self.ctx.h, f.size, ptr(f)))
        self.nhaploid = int((f != 0).sum())

    def setHaploidTargets(self, haploid):
        """Haploid targets of the next phase() calls (one flag per target;
        None: all diploid): they are not phased (Target.cpp:166-203)."""
        if haploid is None:
            self.ctx.check(self.ctx.L.eimp_phase_haploid_targets(self.ctx.h, 0, None))
            return
        f = _c(haploid, np.uint8)
        self.ctx.check(self.ctx.L.eimp_phase_haploid_targets(self.ctx.h, f.size, ptr(f)))

    def setStartPhases(self, phases):
        """The maternal phase of every target's first heterozygous site carried
        over from the previous chunk (VCFData::getStartPhase; 0 = Ref) for the
        next phase() calls, which must then have len(phases) targets; None
        goes back to Ref for all."""
        if phases is None:
            self.ctx.check(self.ctx.L.eimp_phase_start_phases(self.ctx.h, 0, None))
            return
        ph = _c(phases, np.uint8)
        self.ctx.check(self.ctx.L.eimp_phase_start_phases(self.ctx.h, ph.size, ptr(ph)))

    def _K(self, params: PhaseParams) -> int:
        corr = self.nhaps - getattr(self, "nhaploid", 0)
        return min(params.K, corr - 2 if self.self0 >= 0 else corr)

    def prep(self, params: PhaseParams, gt: np.ndarray):
        gt = _c(gt, np.uint8)
        n, M = gt.shape
        K = self._K(params)
        out = dict(besthaps=np.zeros((n, K), np.int32), flags=np.zeros((n, W(self.nhaps)), np.uint64),
                   monos=np.zeros((n, W(M)), np.uint64), splits=np.zeros((n, M), np.int32),
                   calls=np.zeros((n, M), np.int32), cmdiffs=np.zeros((n, M + 1), np.float32),
                   nsplits=np.zeros(n, np.int32), ncalls=np.zeros(n, np.int32))
        p = params.c()
        self.ctx.check(self.ctx.L.eimp_phase_prep(self.ctx.h, C.byref(p), n, ptr(gt), *[ptr(out[k]) for k in (
            "besthaps", "flags", "monos", "splits", "calls", "cmdiffs", "nsplits", "ncalls")]))
        return out

    def cref_pbwt(self, params: PhaseParams, gt: np.ndarray):
        gt = _c(gt, np.uint8)
        n = gt.shape[0]
        K = self._K(params)
        p = params.c()
        rows = C.c_size_t(0)
        self.ctx.check(self.ctx.L.eimp_phase_cref_pbwt(self.ctx.h, C.byref(p), n, ptr(gt), C.byref(rows),
                                                       None, None, None, None))
        R = rows.value
        rowoff = np.zeros(n + 1, np.int64)
        cref = np.zeros((R, W(K)), np.uint64)
        c0 = np.zeros(R, np.int32)
        pb = np.zeros((2 * R, 2 * ((K + 31) // 32)), np.uint32)
        self.ctx.check(self.ctx.L.eimp_phase_cref_pbwt(self.ctx.h, C.byref(p), n, ptr(gt), C.byref(rows),
                                                       ptr(rowoff), ptr(cref), ptr(c0), ptr(pb)))
        return rowoff, cref, c0, pb

    def phase(self, params: PhaseParams, gt: np.ndarray):
        gt = _c(gt, np.uint8)
        n, M = gt.shape
        mats = np.zeros((n, W(M)), np.uint64)
        pats = np.zeros((n, W(M)), np.uint64)
        dm = np.zeros((n, M), np.float32)
        dp = np.zeros((n, M), np.float32)
        tc = np.zeros(n, np.float32)
        nc = np.zeros(n, np.int32)
        p = params.c()
        self.ctx.check(self.ctx.L.eimp_phase_targets(self.ctx.h, C.byref(p), n, ptr(gt), ptr(mats), ptr(pats),
                                                     ptr(dm), ptr(dp), ptr(tc), ptr(nc)))
        return mats, pats, dm, dp, tc, nc

    def phase_dev(self, params: PhaseParams, d_gt, d_mats, d_pats, d_dm, d_dp, d_tc, d_nc):
        p = params.c()
        n = d_gt.shape[0]
        self.ctx.check(self.ctx.L.eimp_phase_targets_dev(self.ctx.h, C.byref(p), n, ptr(d_gt), ptr(d_mats),
                                                         ptr(d_pats), ptr(d_dm), ptr(d_dp), ptr(d_tc), ptr(d_nc)))


def determine_start_phases(mats: np.ndarray, pats: np.ndarray, overlap_begin: int, M: int) -> np.ndarray:
    """VCFData::determineStartPhases (VCFData.cpp:2802-2816): for every target
    the maternal allele at its first heterozygous phased site from
    overlap_begin on (the start of the overlap with the next chunk), or at the
    last site when there is none -- the start phase of the next chunk."""
    from .bits import unpack_rows
    m = unpack_rows(_c(mats, np.uint64), M)
    p = unpack_rows(_c(pats, np.uint64), M)
    out = np.zeros(m.shape[0], np.uint8)
    for t in range(m.shape[0]):
        s = overlap_begin
        while True:
            mat, pat = m[t, s], p[t, s]
            s += 1
            if mat != pat or s >= M:
                break
        out[t] = mat
    return out


def _transpose_bits(rows: np.ndarray, ncols: int) -> np.ndarray:
    """Bit matrix rows x ncols (row words) -> ncols x rows (padded rows)."""
    from .bits import pack_rows, unpack_rows
    return pack_rows(np.ascontiguousarray(unpack_rows(rows, ncols).T), W(rows.shape[0]))


def phase_iterations(ctx: Context, hapmajor: np.ndarray, sitemajor: np.ndarray, cm: np.ndarray,
                     params: PhaseParams, gt: np.ndarray, iters: int, haploid_ref=None, haploid_tgt=None):
    """PBWTPhaser's phasing iterations (PBWTPhaser.cpp:406-476, --phaseIters):
    iteration 1 phases the targets against the reference; every further
    iteration phases them again against the reference followed by the phased
    targets of the previous iteration, each target leaving its own
    haplotypes out; reverse phasing and the call confidences only in the last
    iteration.  Haploid reference samples and targets (flags or None) stay
    haploid in the grown panel (VCFData.cpp:1926-1931).  Returns the last
    iteration's (mats, pats, dm, dp, tc, nc)."""
    import dataclasses
    gt = _c(gt, np.uint8)
    n, M = gt.shape
    nh = hapmajor.shape[0]
    hr = np.zeros(nh // 2, np.uint8) if haploid_ref is None else _c(haploid_ref, np.uint8)
    ht = np.zeros(n, np.uint8) if haploid_tgt is None else _c(haploid_tgt, np.uint8)
    ph = Phaser(ctx, hapmajor, sitemajor, cm)
    ph.setHaploidRef(hr if hr.any() else None)
    ph.setHaploidTargets(ht if ht.any() else None)
    out = None
    for it in range(1, iters + 1):
        p = dataclasses.replace(params, doRevPhasing=params.doRevPhasing and it == iters)
        if it > 1:
            mats, pats = out[0], out[1]
            tgt = np.empty((2 * n, mats.shape[1]), np.uint64)
            tgt[0::2], tgt[1::2] = mats, pats
            aug = np.concatenate([_c(hapmajor, np.uint64), tgt])
            ph = Phaser(ctx, aug, _transpose_bits(aug, M), cm)
            hf = np.concatenate([hr, ht])
            ph.setHaploidRef(hf if hf.any() else None)
            ph.setHaploidTargets(ht if ht.any() else None)
            ph.excludeSelf(nh // 2)
        out = ph.phase(p, gt)
    ph.excludeSelf(-1)
    ph.setHaploidTargets(None)
    return out


class PBWTImputer:
    """PBWTImputer (PBWTImputer.h:30-64) over libeimp_b200.

    The reference's per-block state machine (prepareBlocks / forwardBlock,
    TargetImp.cpp:250-304, 437-471) becomes a stateless site window: block b
    imputes ``[block_start[b], block_start[b] + bsize)`` per call and advances.
    """

    def __init__(self, ctx: Context, sitemajor_full: np.ndarray, af_full: np.ndarray, typed: np.ndarray,
                 sitemajor_typed: np.ndarray, nhaps: int, setmaxerrors: int = 0, imputeCalls: bool = False,
                 haploid_ref=None):
        self.ctx = ctx
        self.Mref = sitemajor_full.shape[0]
        self.M = len(typed)
        self.nhaps = nhaps
        self.setmaxerrors = setmaxerrors
        self.imputeCalls = imputeCalls
        # haploid panel samples: the PBWT without their placeholder columns
        hr = None if haploid_ref is None else _c(haploid_ref, np.uint8)
        self.K = nhaps - (0 if hr is None else int((hr != 0).sum()))
        ctx.check(ctx.L.eimp_imp_set_haploid_ref(ctx.h, 0 if hr is None else hr.size, None if hr is None else ptr(hr)))
        ctx.check(ctx.L.eimp_imp_set_reference(ctx.h, self.Mref, nhaps, ptr(_c(sitemajor_full, np.uint64)),
                                               ptr(_c(af_full, np.float32)), self.M, ptr(_c(typed, np.int64)),
                                               ptr(_c(sitemajor_typed, np.uint64))))
        self.ntargets = 0
        self.block_pos = {}

    def prepareImputation(self, phasedTargets: np.ndarray, gt: np.ndarray, num_sites_per_block=None,
                          match_cap: int = 0, haploid_targets=None):
        """haploid_targets: one flag per target (None: all diploid); only the
        first haplotype of a haploid target is imputed (PBWTImputer.cpp:130)."""
        phased = _c(phasedTargets, np.uint64)
        gt = _c(gt, np.uint8)
        self.ntargets = gt.shape[0]
        assert phased.shape == (2 * self.ntargets, W(self.M))
        ht = None if haploid_targets is None else _c(haploid_targets, np.uint8)
        self.ctx.check(self.ctx.L.eimp_imp_haploid_targets(self.ctx.h, 0 if ht is None else ht.size,
                                                           None if ht is None else ptr(ht)))
        self.ctx.check(self.ctx.L.eimp_imp_prepare(self.ctx.h, self.ntargets, ptr(phased), ptr(gt),
                                                   self.setmaxerrors, int(self.imputeCalls), match_cap))
        self.block_pos = {}
        if num_sites_per_block is not None:
            # first entry: sites of the left overlap to skip; block b starts
            # after the sites of the blocks before it (TargetImp.cpp:250-272)
            start = int(num_sites_per_block[0])
            for b in range(1, len(num_sites_per_block) - 1):
                self.block_pos[b - 1] = start
                start += int(num_sites_per_block[b])
        else:
            self.block_pos[0] = 0

    def imputeBunch(self, block: int, bsize: int):
        """Next ``bsize`` sites of ``block``: (bits 2N x W(bsize), dosages 2N x bsize)."""
        b0 = self.block_pos.get(block, 0)
        n = max(0, min(bsize, self.Mref - b0))
        bits, dos = self.impute_window(b0, n) if n else (np.zeros((2 * self.ntargets, W(bsize)), np.uint64),
                                                         np.zeros((2 * self.ntargets, bsize), np.float32))
        self.block_pos[block] = b0 + n
        return bits, dos

    def impute_window(self, mref_begin: int, nsites: int):
        nh = 2 * self.ntargets
        bits = np.zeros((nh, W(nsites)), np.uint64)
        dos = np.zeros((nh, nsites), np.float32)
        self.ctx.check(self.ctx.L.eimp_imp_bunch(self.ctx.h, mref_begin, nsites, ptr(bits), ptr(dos)))
        return bits, dos

    def setPhasedDosages(self, dos_mat: np.ndarray, dos_pat: np.ndarray):
        """phasedDosages of the prepared targets (N x M floats each, the mat and
        pat dosages phasing returned), kept on the device for the output
        statistics of writeVCFImputedBunch."""
        dm = np.ascontiguousarray(dos_mat, np.float32)
        dp = np.ascontiguousarray(dos_pat, np.float32)
        if dm.shape != (self.ntargets, self.M) or dp.shape != dm.shape:
            raise ValueError(f"phased dosages must be {self.ntargets} x {self.M}")
        self.ctx.check(self.ctx.L.eimp_imp_phased_dosages(self.ctx.h, ptr(dm), ptr(dp)))

    def writeImputedBunchStats(self, mref_begin: int, nsites: int, overwriteCalls: bool = False,
                               improveCalls: bool = False, r2filter: float = 0.0, maffilter: float = 0.0,
                               ds: bool = False, gp: bool = False) -> dict:
        """imputeBunch for the window plus the numbers VCFData::writeVCFImputedBunch
        (VCFData.cpp:3068-3446) writes for it: per haplotype and site the
        allele dosage (ads) and allele (gtbits); optionally DS and GP; per site
        r2, af, maf, ac, an and passed (the r2/MAF output filters); the number
        of imputation conflicts."""
        from ._lib import EimpSiteStatsOpts
        nh, N = 2 * self.ntargets, self.ntargets
        o = EimpSiteStatsOpts(int(overwriteCalls), int(improveCalls), float(r2filter), float(maffilter))
        out = dict(ads=np.zeros((nh, nsites), np.float32), gtbits=np.zeros((nh, W(nsites)), np.uint64),
                   ds=np.zeros((N, nsites), np.float32) if ds else None,
                   gp=np.zeros((3 * N, nsites), np.float32) if gp else None,
                   r2=np.zeros(nsites, np.float32), af=np.zeros(nsites, np.float32),
                   maf=np.zeros(nsites, np.float32), ac=np.zeros(nsites, np.int32), an=np.zeros(nsites, np.int32),
                   passed=np.zeros(nsites, np.uint8))
        conf = np.zeros(1, np.uint64)
        self.ctx.check(self.ctx.L.eimp_imp_bunch_stats(
            self.ctx.h, mref_begin, nsites, C.byref(o), ptr(out["ads"]), ptr(out["gtbits"]),
            ptr(out["ds"]) if ds else None, ptr(out["gp"]) if gp else None, ptr(out["r2"]), ptr(out["af"]),
            ptr(out["maf"]), ptr(out["ac"]), ptr(out["an"]), ptr(out["passed"]), ptr(conf)))
        out["conflicts"] = int(conf[0])
        return out

    def improveStats(self, reset: bool = False):
        """The --improveCalls run statistics (VCFData's improvecnt* /
        totalimprove* counters, VCFData.cpp:3306-3330) summed over the output
        statistics computed so far: counts and totals in the order no change,
        het->het, hom->hom, het->hom, hom->het."""
        counts = np.zeros(5, np.uint64)
        totals = np.zeros(5, np.float64)
        self.ctx.check(self.ctx.L.eimp_imp_improve_stats(self.ctx.h, ptr(counts), ptr(totals), int(reset)))
        return counts.astype(np.int64), totals

    def matches(self, hap: int) -> np.ndarray:
        n = C.c_size_t(0)
        self.ctx.check(self.ctx.L.eimp_imp_matches(self.ctx.h, hap, None, 0, C.byref(n)))
        out = np.zeros((n.value, 4), np.int32)
        if n.value:
            self.ctx.check(self.ctx.L.eimp_imp_matches(self.ctx.h, hap, ptr(out), n.value, C.byref(n)))
        return out

    def refpbwt(self):
        kw = 2 * ((self.K + 31) // 32)
        compr = np.zeros((self.M, kw), np.uint32)
        ap = np.zeros((self.M + 1, self.K), np.int32)
        self.ctx.check(self.ctx.L.eimp_imp_refpbwt(self.ctx.h, ptr(compr), ptr(ap)))
        return compr, ap


def decode_qref_haplotypes(ctx: Context, section: np.ndarray, Mref: int, Nref: int) -> np.ndarray:
    """The haplotype section of a Qref reference file (qref_spec.md section I:
    per variant <encsize u64> and a run-length code, or the raw vector) decoded
    on the device -- the decode of VCFData::qRefLoadNextVariant -- into Mref
    site-major rows of W(2*Nref) words (referenceFullT)."""
    sec = np.ascontiguousarray(section, np.uint8)
    out = np.zeros((Mref, W(2 * Nref)), np.uint64)
    ctx.check(ctx.L.eimp_qref_decode(ctx.h, ptr(sec) if sec.size else None, sec.size, Mref, Nref, None, 0,
                                     ptr(out)))
    return out

