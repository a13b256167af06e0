"""Generate the golden fixtures of tests/golden/ from the reference's OWN code.

Runs the reference's hot-path sources, compiled by ``make -C oracle ref`` into
oracle/_ref/libeimp_refcore.so, on a small seeded synthetic panel and stores
inputs and outputs as compressed .npz files:

  golden_tiny.npz  -- panel (200 haplotypes x 3000 sites), 8 targets (6 regular
                      targets, one without heterozygous sites, one with 60 %
                      missing genotypes), and per K in {64, 50, 200}:
                      best haplotypes, monos, split/call sites, cM differences,
                      condensed reference, count0, forward+backward compressed
                      PBWT, phased haplotypes, phasing dosages, confidences;
                      for K=64 also the imputation: reference PBWT + prefix
                      arrays, set-maximal matches and imputed bits/dosages.

  golden_haploid.npz -- the same panel with every fourth reference sample
                      haploid (stored as a homozygous diploid pair, its
                      second column a copy of the first) and 8 targets of
                      which 3 are haploid (genotypes 0/2/missing): for K in
                      {64, 200} (200 takes every existing haplotype, 175)
                      the best haplotypes, phased haplotypes, dosages and
                      confidences, and for K=64 the imputation over the
                      reduced reference (PBWTImputer.cpp:31-34, 67-114):
                      its PBWT and prefix arrays, the matches of the 13
                      target haplotypes and the imputed bits/dosages.

K=50 is not a multiple of 32, K=200 equals the number of haplotypes (the
reference's copy-all path, Target.cpp:969-974).  Usage:

    python tests/golden/make_golden.py            # both fixtures
    python tests/golden/make_golden.py haploid    # golden_haploid.npz only
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from eimp_b200 import synth  # noqa: E402
from eimp_b200.bits import W, unpack_rows  # noqa: E402
from oracle.refcore import PhaseParams, RefCore  # noqa: E402


def make_targets(groups):
    tg = groups[0]
    gt = tg.gt.copy()
    truth = tg.truth.copy()
    M = gt.shape[1]
    rng = np.random.default_rng(99)
    # a target without heterozygous sites
    h = truth[0]
    nohet = (2 * h).astype(np.uint8)
    # a target with 60 % missing genotypes (no set-maximal matches, TargetImp.cpp:79-80)
    hm = truth[2].astype(np.uint8) + truth[3]
    miss = rng.choice(M, int(0.6 * M), replace=False)
    hm = hm.astype(np.uint8)
    hm[miss] = 3
    gt = np.concatenate([gt, nohet[None], hm[None]])
    truth = np.concatenate([truth, np.stack([h, h]), truth[2:4]])
    return synth.Targets(tg.typed, gt, truth)


def main():
    panel, groups = synth.generate("tiny")
    tg = make_targets(groups)
    rc = RefCore(panel, tg)
    out = dict(nhaps=panel.nhaps, Mref=panel.nsites, M=len(tg.typed), typed=tg.typed, gt=tg.gt,
               sitemajor_full=panel.sitemajor, af_full=panel.af, hapmajor_typed=rc.hapmajor_typed,
               sitemajor_typed=rc.sitemajor_typed, cm_typed=rc.cm_typed)
    nt = tg.gt.shape[0]
    for K in (64, 50, 200):
        pp = PhaseParams(K=K, beamwidth=16)
        rc.set_params(pp)
        pre = f"K{K}_"
        Kc = min(K, panel.nhaps)
        bh = np.zeros((nt, Kc), np.int64)
        monos = np.zeros((nt, W(rc.M)), np.uint64)
        splits, calls, cmd = [], [], []
        crefs, c0s, pbs = [], [], []
        for t in range(nt):
            r = rc.prep(t)
            bh[t] = r["besthaps"]
            monos[t] = r["monos"]
            splits.append(r["splits"]); calls.append(r["calls"]); cmd.append(r["cmdiffs"])
            cr, c0, pb = rc.cref_pbwt(t)
            crefs.append(cr); c0s.append(c0); pbs.append(pb)
        out[pre + "besthaps"] = bh
        out[pre + "monos"] = monos
        out[pre + "nsplits"] = np.array([len(s) for s in splits], np.int64)
        out[pre + "ncalls"] = np.array([len(c) for c in calls], np.int64)
        out[pre + "splits"] = np.concatenate(splits) if splits else np.zeros(0, np.int64)
        out[pre + "calls"] = np.concatenate(calls)
        out[pre + "cmdiffs"] = np.concatenate(cmd)
        out[pre + "rows"] = np.array([c.shape[0] for c in crefs], np.int64)
        out[pre + "cref"] = np.concatenate(crefs)
        out[pre + "count0"] = np.concatenate(c0s)
        out[pre + "pbwt"] = np.concatenate(pbs)
        mats, pats, dm, dp, tcs, ncs = [], [], [], [], [], []
        for t in range(nt):
            a, b, c, d, tc, nc = rc.phase(t)
            mats.append(a); pats.append(b); dm.append(c); dp.append(d); tcs.append(tc); ncs.append(nc)
        out[pre + "mat"] = np.stack(mats)
        out[pre + "pat"] = np.stack(pats)
        out[pre + "dos_mat"] = np.stack(dm)
        out[pre + "dos_pat"] = np.stack(dp)
        out[pre + "totalconf"] = np.array(tcs, np.float32)
        out[pre + "ncallsites"] = np.array(ncs, np.int64)
        if K == 64:
            ph = np.zeros((2 * nt, W(rc.M)), np.uint64)
            ph[0::2] = out[pre + "mat"]
            ph[1::2] = out[pre + "pat"]
            imp = rc.imputer(ph, 1)
            compr, absperm = imp.refpbwt()
            out["imp_phased"] = ph
            out["imp_compr"] = compr
            out["imp_absperm"] = absperm
            ms = [imp.matches(h) for h in range(2 * nt)]
            out["imp_nmatches"] = np.array([len(m) for m in ms], np.int64)
            out["imp_matches"] = np.concatenate(ms) if ms else np.zeros((0, 4), np.int64)
            bits, dos = imp.bunch(rc.Mref, 1)
            out["imp_bits"] = bits
            out["imp_dos"] = dos
            imp.close()
    path = os.path.join(HERE, "golden_tiny.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


def haploid_case():
    """The tiny panel with every fourth reference sample haploid and targets
    1, 3 and 6 haploid (the inputs of golden_haploid.npz)."""
    from eimp_b200.bits import pack_rows, transpose_bits
    panel, groups = synth.generate("tiny")
    tg = make_targets(groups)
    nh, Mref = panel.nhaps, panel.nsites
    ref_hap = (np.arange(nh // 2) % 4 == 0).astype(np.uint8)
    dense = unpack_rows(panel.hapmajor, Mref)
    for s in np.flatnonzero(ref_hap):
        dense[2 * s + 1] = dense[2 * s]
    hm = pack_rows(dense, W(Mref))
    sm = transpose_bits(hm, nh, Mref)
    af = (dense.sum(axis=0) / nh).astype(np.float32)
    panel = synth.Panel(nh, Mref, panel.pos, panel.cm, af, hm, sm)
    tgt_hap = np.zeros(tg.gt.shape[0], np.uint8)
    tgt_hap[[1, 3, 6]] = 1
    gt = tg.gt.copy()
    truth = tg.truth.copy()
    for t in np.flatnonzero(tgt_hap):
        miss = gt[t] == 3
        gt[t] = 2 * truth[2 * t]
        gt[t][miss] = 3
        truth[2 * t + 1] = truth[2 * t]
    return panel, synth.Targets(tg.typed, gt, truth), ref_hap, tgt_hap


def main_haploid():
    panel, tg, ref_hap, tgt_hap = haploid_case()
    rc = RefCore(panel, tg)
    rc.set_haploids(ref_hap, tgt_hap)
    nt = tg.gt.shape[0]
    out = dict(nhaps=panel.nhaps, Mref=panel.nsites, M=len(tg.typed), typed=tg.typed, gt=tg.gt,
               sitemajor_full=panel.sitemajor, af_full=panel.af, hapmajor_typed=rc.hapmajor_typed,
               sitemajor_typed=rc.sitemajor_typed, cm_typed=rc.cm_typed, ref_haploid=ref_hap,
               tgt_haploid=tgt_hap)
    for K in (64, 200):
        rc.set_params(PhaseParams(K=K, beamwidth=16))
        pre = f"K{K}_"
        dip = np.flatnonzero(tgt_hap == 0)
        out[pre + "besthaps"] = np.stack([rc.prep(int(t))["besthaps"] for t in dip])
        res = [rc.phase(t) for t in range(nt)]
        out[pre + "mat"] = np.stack([r[0] for r in res])
        out[pre + "pat"] = np.stack([r[1] for r in res])
        out[pre + "dos_mat"] = np.stack([r[2] for r in res])
        out[pre + "dos_pat"] = np.stack([r[3] for r in res])
        out[pre + "totalconf"] = np.array([r[4] for r in res], np.float32)
        out[pre + "ncallsites"] = np.array([r[5] for r in res], np.int64)
        if K == 64:
            ph = np.zeros((2 * nt, W(rc.M)), np.uint64)
            ph[0::2] = out[pre + "mat"]
            ph[1::2] = out[pre + "pat"]
            imp = rc.imputer(ph, 1)
            compr, absperm = imp.refpbwt()
            out["imp_phased"] = ph
            out["imp_K"] = imp.K
            out["imp_compr"] = compr
            out["imp_absperm"] = absperm
            ms = [imp.matches(h) for h in range(imp.ntargethaps)]
            out["imp_nmatches"] = np.array([len(m) for m in ms], np.int64)
            out["imp_matches"] = np.concatenate(ms) if ms else np.zeros((0, 4), np.int64)
            bits, dos = imp.bunch(rc.Mref, 1)
            out["imp_bits"] = bits
            out["imp_dos"] = dos
            imp.close()
    path = os.path.join(HERE, "golden_haploid.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    if sys.argv[1:] != ["haploid"]:
        main()
    main_haploid()
