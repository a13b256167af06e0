"""Seeded synthetic reference panels and targets (Li-Stephens mosaics).

The reference's headline configurations are quoted on real panels that are not
available here, so every run uses seeded synthetic data of the same shape:

* ``F`` founder haplotypes; per-site founder allele frequency ``f`` drawn from a
  1/x site-frequency spectrum on ``[maf_min, 0.5]`` (inverse CDF
  ``f = maf_min * (0.5/maf_min)**u``), a random half of the sites flipped to the
  alternative-major side; founder alleles ~ Bernoulli(f).
* site positions uniform-sorted over the segment, a linear genetic map of
  ``cm_per_mb`` cM/Mb.
* every reference and target haplotype is a mosaic of founders: it switches to a
  uniformly drawn founder with probability ``1 - exp(-lambda * d_cM)`` between
  consecutive sites (lambda = 1/``mean_segment_cm``), and each copied allele is
  flipped with the copying error probability.
* targets are held-out mosaics given as unphased genotypes 0/1/2 at a random
  subset of the panel sites ("typed" sites) with a per-target missing rate
  (genotype code 3).

The data of one configuration is cached as ``.npz`` under ``$EIMP_CACHE``
(default ``/tmp/eimp_cache``) keyed by all generator parameters.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os
from dataclasses import dataclass, field

import numpy as np

from .bits import W, gather_bits, pack_rows, transpose_bits


@dataclass(frozen=True)
class TargetGroup:
    ntargets: int
    typed_frac: float          # fraction of panel sites typed in this group
    miss_lo: float             # per-target missing rate drawn from U(miss_lo, miss_hi)
    miss_hi: float


@dataclass(frozen=True)
class SynthConfig:
    name: str
    nhaps: int                 # reference haplotypes (even: diploid samples)
    nsites: int                # reference sites (Mref)
    segment_mb: float
    founders: int
    groups: tuple = ()
    K: int = 1024
    beam: int = 64
    maf_min: float = 5e-4
    cm_per_mb: float = 1.0
    mean_segment_cm: float = 1.0
    copy_err: float = 1e-3
    seed: int = 1

    def key(self) -> str:
        d = dataclasses.asdict(self)
        return hashlib.sha1(json.dumps(d, sort_keys=True, default=str).encode()).hexdigest()[:16]


CONFIGS = {
    # unit-test sized
    "tiny": SynthConfig("tiny", nhaps=200, nsites=3000, segment_mb=1.0, founders=20,
                        groups=(TargetGroup(6, 0.2, 0.01, 0.01),), K=64, beam=16, seed=7),
    "small-test": SynthConfig("small-test", nhaps=600, nsites=8000, segment_mb=2.0, founders=40,
                              groups=(TargetGroup(8, 0.1, 0.01, 0.01),), K=200, beam=32, seed=11),
    # configs of the reference's headline workloads
    "cfg1": SynthConfig("cfg1", nhaps=5000, nsites=20000, segment_mb=5.0, founders=200,
                        groups=(TargetGroup(100, 0.10, 0.01, 0.01),), K=1024, beam=64, seed=1001),
    "cfg2": SynthConfig("cfg2", nhaps=10000, nsites=100000, segment_mb=20.0, founders=500,
                        groups=(TargetGroup(1000, 0.05, 0.02, 0.02),), K=4096, beam=128, seed=1002),
    "cfg3": SynthConfig("cfg3", nhaps=20000, nsites=400000, segment_mb=40.0, founders=1000,
                        groups=(TargetGroup(3334, 0.01, 0.0, 0.05), TargetGroup(3333, 0.03, 0.0, 0.05),
                                TargetGroup(3333, 0.08, 0.0, 0.05)), K=4096, beam=128, seed=1003),
    # generated on the device only (eimp_b200/synth_device.py): 25 GB bit-packed
    "cfg4": SynthConfig("cfg4", nhaps=200000, nsites=1000000, segment_mb=60.0, founders=5000,
                        groups=(TargetGroup(50000, 0.02, 0.01, 0.01),), K=8192, beam=128, maf_min=5e-6, seed=1004),
}


@dataclass
class Panel:
    """A reference panel in the reference's in-memory layouts."""
    nhaps: int
    nsites: int
    pos: np.ndarray            # int64 (Mref,) 0-based bp positions
    cm: np.ndarray             # float64 (Mref,) genetic positions
    af: np.ndarray             # float32 (Mref,) alt allele frequency in the panel
    hapmajor: np.ndarray       # uint64 (nhaps, W(Mref))  one row per haplotype
    sitemajor: np.ndarray      # uint64 (Mref, W(nhaps))  one row per site (referenceFullT)
    founders: np.ndarray | None = None   # uint64 (F, W(Mref)) the founders (for more targets)


@dataclass
class Targets:
    """One group of targets sharing a typed-site set."""
    typed: np.ndarray          # int64 (M,) indices into the panel sites, ascending
    gt: np.ndarray             # uint8 (ntargets, M) 0/1/2, 3 = missing
    truth: np.ndarray          # uint8 (2*ntargets, M) true haplotypes at typed sites


def _founders_words(rng, f, nfounders, nw, chunk=64):
    """Founder haplotypes as packed words (nfounders, nw): allele ~ Bernoulli(f)
    per site, drawn for ``chunk`` founders at a time."""
    n = f.size
    out = np.zeros((nfounders, nw), dtype=np.uint64)
    f32 = f.astype(np.float32)
    for a in range(0, nfounders, chunk):
        b = min(nfounders, a + chunk)
        alle = (rng.random((b - a, n), dtype=np.float32) < f32[None, :]).astype(np.uint8)
        out[a:b] = pack_rows(alle, nw)
    return out


def _mosaic_words(rng, Fw, cm, nhap, mean_seg, copy_err):
    """(nhap, nw) packed Li-Stephens mosaics of the packed founders Fw
    (F, nw): every haplotype switches to a uniformly drawn founder at
    Poisson(genetic length / mean_seg) uniform genetic positions (a switch at
    genetic position x takes effect from the first site at or after x), and
    each copied allele flips with probability copy_err.  Words are copied
    whole; the words a switch falls into are merged at the switch's bit."""
    F, nw = Fw.shape
    n = cm.size
    glen = float(cm[-1] - cm[0])
    counts = rng.poisson(glen / mean_seg, nhap)
    total = int(counts.sum())
    hid = np.repeat(np.arange(nhap), counts)
    x = rng.uniform(cm[0], cm[-1], total)
    order = np.lexsort((x, hid))
    x = x[order]
    brk = np.searchsorted(cm, x, side="left").astype(np.int64)          # first site of the new segment
    fid = rng.integers(0, F, total + nhap)                                # founder of every segment
    bp0 = np.concatenate(([0], np.cumsum(counts)))                        # first breakpoint of each hap
    seg0 = bp0[:-1] + np.arange(nhap)                                     # first segment of each hap
    # founder in effect at the first site of every word: segments started at or before it
    key = hid * (n + 1) + brk
    wkey = (np.arange(nhap, dtype=np.int64) * (n + 1))[:, None] + 64 * np.arange(nw, dtype=np.int64)[None, :]
    nbefore = np.searchsorted(key, wkey, side="right") - bp0[:-1, None]
    founder = fid[seg0[:, None] + nbefore]
    words = Fw[founder, np.arange(nw)[None, :]]
    # switches inside a word, in order along each haplotype
    rank = np.arange(total) - bp0[hid]
    inner = (brk % 64 != 0) & (brk < n)
    for r in range(int(counts.max()) if nhap else 0):
        s = np.flatnonzero(inner & (rank == r))
        if s.size == 0:
            continue
        h, b = hid[s], brk[s]
        w = b >> 6
        low = (np.uint64(1) << (b & 63).astype(np.uint64)) - np.uint64(1)
        fnew = fid[seg0[h] + r + 1]
        words[h, w] = (words[h, w] & low) | (Fw[fnew, w] & ~low)
    # copying errors
    nerr = rng.binomial(n, copy_err, nhap)
    eh = np.repeat(np.arange(nhap), nerr)
    ep = rng.integers(0, n, int(nerr.sum()))
    np.bitwise_xor.at(words, (eh, ep >> 6), np.uint64(1) << (ep & 63).astype(np.uint64))
    return words


def _cache_dir() -> str:
    d = os.environ.get("EIMP_CACHE", "/tmp/eimp_cache")
    os.makedirs(d, exist_ok=True)
    return d


# version of the generator's drawing order (part of the cache key)
GENERATOR = 3


def generate(cfg: SynthConfig | str, cache: bool = True):
    """Generate (or load from cache) ``(panel, [targets per group])``."""
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    path = os.path.join(_cache_dir(), f"{cfg.name}-g{GENERATOR}-{cfg.key()}.npz")
    if cache and os.path.exists(path):
        z = np.load(path)
        panel = Panel(cfg.nhaps, cfg.nsites, z["pos"], z["cm"], z["af"], z["hapmajor"], z["sitemajor"],
                      z["founders"])
        groups = [Targets(z[f"typed{g}"], np.ascontiguousarray(z[f"gt{g}"]), np.ascontiguousarray(z[f"truth{g}"]))
                  for g in range(len(cfg.groups))]
        return panel, groups

    rng = np.random.default_rng(cfg.seed)
    n = cfg.nsites
    L = int(cfg.segment_mb * 1e6)
    pos = np.sort(rng.integers(0, L - n, n)) + np.arange(n)
    cm = pos.astype(np.float64) * (cfg.cm_per_mb / 1e6)
    u = rng.uniform(0.0, 1.0, n)
    f = cfg.maf_min * (0.5 / cfg.maf_min) ** u
    flip = rng.uniform(0.0, 1.0, n) < 0.5
    f = np.where(flip, 1.0 - f, f)
    hap_w = W(n)
    Fw = _founders_words(rng, f, cfg.founders, hap_w)

    # reference haplotypes in blocks of 1024
    nh = cfg.nhaps
    hapmajor = np.zeros((nh, hap_w), dtype=np.uint64)
    blk = 1024
    for b0 in range(0, nh, blk):
        b1 = min(nh, b0 + blk)
        hapmajor[b0:b1] = _mosaic_words(rng, Fw, cm, b1 - b0, cfg.mean_segment_cm, cfg.copy_err)
    sitemajor = transpose_bits(hapmajor, nh, n)
    ac = np.bitwise_count(sitemajor).sum(axis=1, dtype=np.int64)
    af = (ac / float(nh)).astype(np.float32)
    panel = Panel(nh, n, pos.astype(np.int64), cm, af, hapmajor, sitemajor, Fw)

    groups = []
    for g in cfg.groups:
        m = max(2, int(round(g.typed_frac * n)))
        typed = np.sort(rng.choice(n, m, replace=False)).astype(np.int64)
        th = np.zeros((2 * g.ntargets, m), dtype=np.uint8)
        for a in range(0, 2 * g.ntargets, blk):
            b = min(2 * g.ntargets, a + blk)
            th[a:b] = gather_bits(_mosaic_words(rng, Fw, cm, b - a, cfg.mean_segment_cm, cfg.copy_err), typed)
        gt = (th[0::2].astype(np.uint8) + th[1::2]).astype(np.uint8)
        for t in range(g.ntargets):
            rate = rng.uniform(g.miss_lo, g.miss_hi) if g.miss_hi > g.miss_lo else g.miss_lo
            nmiss = int(round(rate * m))
            if nmiss:
                gt[t, rng.choice(m, nmiss, replace=False)] = 3
        groups.append(Targets(typed, np.ascontiguousarray(gt), np.ascontiguousarray(th)))

    if cache:
        kw = dict(pos=panel.pos, cm=panel.cm, af=panel.af, hapmajor=panel.hapmajor, sitemajor=panel.sitemajor,
                  founders=Fw)
        for i, t in enumerate(groups):
            kw[f"typed{i}"] = t.typed
            kw[f"gt{i}"] = t.gt
            kw[f"truth{i}"] = t.truth
        tmp = path + ".tmp.npz"
        np.savez(tmp, **kw)
        os.replace(tmp, path)
    return panel, groups


@dataclass
class WindowRequest:
    """A serving request: targets genotyped at their own typed sites inside a
    window [lo, hi) of the panel's sites.  typed holds window-relative site
    indices (ascending); gt is (n, len(typed)) with 3 = missing."""
    lo: int
    hi: int
    typed: np.ndarray
    gt: np.ndarray

    @property
    def n(self) -> int:
        return self.gt.shape[0]


def window_requests(cfg: SynthConfig, panel: Panel, nreq: int, seed: int, max_targets: int = 5000,
                    density=(0.01, 0.08), window_mb=(2.0, 10.0), miss=(0.0, 0.05)):
    """Seeded serving requests over a resident panel: log-uniform 1..max_targets
    targets, a typed density uniform in ``density``, a window of uniform length
    in ``window_mb`` Mb at a uniform position, per-target missingness uniform in
    ``miss``.  Targets are held-out mosaics of the panel's founders, like the
    configurations' targets."""
    if panel.founders is None:
        raise ValueError("the panel was generated without its founders")
    rng = np.random.default_rng(seed)
    span = float(panel.pos[-1] - panel.pos[0])
    out = []
    for _ in range(nreq):
        n = int(np.clip(np.exp(rng.uniform(0.0, np.log(max_targets))), 1, max_targets))
        d = rng.uniform(*density)
        wl = min(span, rng.uniform(*window_mb) * 1e6)
        start = panel.pos[0] + rng.uniform(0.0, span - wl)
        lo, hi = (int(x) for x in np.searchsorted(panel.pos, [start, start + wl]))
        m = max(2, int(round(d * (hi - lo))))
        typed = np.sort(rng.choice(hi - lo, m, replace=False)).astype(np.int64)
        th = np.zeros((2 * n, m), np.uint8)
        for a in range(0, 2 * n, 1024):
            b = min(2 * n, a + 1024)
            th[a:b] = gather_bits(_mosaic_words(rng, panel.founders, panel.cm, b - a, cfg.mean_segment_cm,
                                                cfg.copy_err), lo + typed)
        gt = (th[0::2] + th[1::2]).astype(np.uint8)
        rates = rng.uniform(*miss, n)
        gt[rng.random(gt.shape) < rates[:, None]] = 3
        out.append(WindowRequest(lo, hi, typed, np.ascontiguousarray(gt)))
    return out


def typed_views(panel: Panel, typed: np.ndarray):
    """Typed-site views of a panel, as the reference's VCFData keeps them.

    Returns ``(ref_hapmajor_typed (nhaps, W(M)), ref_sitemajor_typed (M, W(nhaps)),
    cm_typed float32 (M,))`` -- ``reference``, ``referenceT`` and ``cMs``
    (VCFData.h:199-205, 227).
    """
    M = len(typed)
    sitemajor_typed = np.ascontiguousarray(panel.sitemajor[typed])
    hapmajor_typed = transpose_bits(sitemajor_typed, M, panel.nhaps)
    cm_typed = panel.cm[typed].astype(np.float32)
    return hapmajor_typed, sitemajor_typed, cm_typed


# ---------------------------------------------------------------- Qref panels
_RLE_MAX = 32767


def _rle_row(row: np.ndarray):
    """The run-length code of one haplotype vector as the Qref writer stores
    it (runlengthEncode / addRunlength, utils.h:133-191): alternating run
    lengths starting with the 0-bit run, one byte below 128, two bytes (low 7
    bits with the high bit set, then the rest) below 32768, longer runs split
    into 32767-runs joined by empty runs.  None where the code would not be
    shorter than the vector."""
    nbytes_raw = row.size * 8
    bits = np.unpackbits(row.view(np.uint8), bitorder="little")
    change = np.flatnonzero(bits[1:] != bits[:-1]) + 1
    bounds = np.concatenate([[0], change, [bits.size]])
    runs = np.diff(bounds)
    if bits[0]:
        runs = np.concatenate([[0], runs])
    out = []
    for k, L in enumerate(runs.tolist()):
        while L > _RLE_MAX:
            out += [0xff, 0xff, 0x00]
            L -= _RLE_MAX
        if L >= 128:
            out += [(L & 0x7f) | 0x80, L >> 7]
        else:
            out.append(L)
        last = k == len(runs) - 1
        if not last and len(out) >= nbytes_raw:   # the writer gives up while it encodes
            return None
    if len(out) > nbytes_raw:
        return None
    return np.array(out, np.uint8)


def qref_section(rows: np.ndarray) -> np.ndarray:
    """The haplotype section of a Qref file (qref_spec.md section I) for
    site-major panel rows (one row of W(2*Nref) words per variant): per
    variant the uint64 size of its run-length code and the code, or size 0
    and the raw row where the code is not shorter."""
    rows = np.ascontiguousarray(rows, np.uint64)
    parts = []
    for r in rows:
        enc = _rle_row(r)
        if enc is None:
            parts += [np.zeros(8, np.uint8), r.view(np.uint8)]
        else:
            parts += [np.array([enc.size], np.uint64).view(np.uint8), enc]
    return np.concatenate(parts) if parts else np.zeros(0, np.uint8)
