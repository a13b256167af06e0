"""Haploid samples and targets (chrX and other haploid regions) on the GPU,
bit-exact against the reference's own code: the fixture
tests/golden/golden_haploid.npz made by tests/golden/make_golden.py from
oracle/_ref, and a larger case run through oracle/_ref here.

* phasing: a haploid reference sample's second column is never chosen and K
  is clamped to the haplotypes that exist (Target.cpp:798-838,
  PBWTPhaser.cpp:210); haploid targets are not phased (Target.cpp:166-203);
* imputation: the PBWT holds only the existing haplotypes and the dosages
  read the panel through the column map (PBWTImputer.cpp:31-34, 67-114,
  TargetImp.cpp:536); a haploid target's single haplotype is imputed
  (PBWTImputer.cpp:130, 202)."""
import os

import numpy as np
import pytest

from conftest import golden_path
from eimp_b200.bits import W, unpack_rows

pytestmark = pytest.mark.gpu

DOSAGE_TOL = 1e-5


@pytest.fixture(scope="module")
def g():
    return np.load(golden_path("golden_haploid.npz"))


def hapmap(tgt_hap):
    m = []
    for t, h in enumerate(tgt_hap):
        m.append(2 * t)
        if not h:
            m.append(2 * t + 1)
    return np.array(m)


@pytest.mark.parametrize("K", [64, 200])
def test_phasing_haploid_golden(ctx, g, K):
    from eimp_b200.engine import PhaseParams, Phaser
    pre = f"K{K}_"
    ph = Phaser(ctx, g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"])
    ph.setHaploidRef(g["ref_haploid"])
    pp = PhaseParams(K=K, beamwidth=16)
    dip = np.flatnonzero(g["tgt_haploid"] == 0)
    prep = ph.prep(pp, g["gt"][dip])
    np.testing.assert_array_equal(prep["besthaps"], g[pre + "besthaps"])
    ph.setHaploidTargets(g["tgt_haploid"])
    mats, pats, dm, dp, tc, nc = ph.phase(pp, g["gt"])
    ph.setHaploidTargets(None)
    np.testing.assert_array_equal(mats, g[pre + "mat"])
    np.testing.assert_array_equal(pats, g[pre + "pat"])
    np.testing.assert_array_equal(dm, g[pre + "dos_mat"])
    np.testing.assert_array_equal(dp, g[pre + "dos_pat"])
    np.testing.assert_array_equal(tc, g[pre + "totalconf"])
    np.testing.assert_array_equal(nc, g[pre + "ncallsites"])


def test_imputation_haploid_golden(ctx, g):
    from eimp_b200.engine import PBWTImputer
    imp = PBWTImputer(ctx, g["sitemajor_full"], g["af_full"], g["typed"], g["sitemajor_typed"], int(g["nhaps"]),
                      haploid_ref=g["ref_haploid"])
    assert imp.K == int(g["imp_K"])
    imp.prepareImputation(g["imp_phased"], g["gt"], haploid_targets=g["tgt_haploid"])
    compr, ap = imp.refpbwt()
    np.testing.assert_array_equal(compr, g["imp_compr"])
    np.testing.assert_array_equal(ap, g["imp_absperm"])
    off = np.concatenate([[0], np.cumsum(g["imp_nmatches"])])
    hm = hapmap(g["tgt_haploid"])
    for j, h in enumerate(hm):
        np.testing.assert_array_equal(imp.matches(int(h)).astype(np.int64), g["imp_matches"][off[j]:off[j + 1]])
    Mref, M = int(g["Mref"]), int(g["M"])
    bits, dos = imp.impute_window(0, Mref)
    # the sites the reference writes: untyped, and missing typed ones
    sel = np.ones((g["gt"].shape[0], Mref), bool)
    sel[:, g["typed"]] = g["gt"] == 3
    for h in hm:
        s = sel[h // 2]
        np.testing.assert_array_equal(dos[h][s], g["imp_dos"][h][s])
        np.testing.assert_array_equal(unpack_rows(bits[h], Mref)[s], unpack_rows(g["imp_bits"][h], Mref)[s])
    for t in np.flatnonzero(g["tgt_haploid"]):   # the second haplotype is not imputed
        assert not dos[2 * t + 1].any() and not bits[2 * t + 1].any()
        assert imp.matches(2 * t + 1).shape[0] == 0


def test_haploid_het_is_an_error(ctx, g):
    from eimp_b200._lib import EimpError
    from eimp_b200.engine import PhaseParams, Phaser
    ph = Phaser(ctx, g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"])
    gt = g["gt"].copy()
    t = int(np.flatnonzero(g["tgt_haploid"])[0])
    gt[t, 5] = 1
    ph.setHaploidTargets(g["tgt_haploid"])
    with pytest.raises(EimpError, match="heterozygous genotype in haploid target"):
        ph.phase(PhaseParams(K=64, beamwidth=16), gt)
    ph.setHaploidTargets(None)


def test_haploid_vs_reference_cfg1(ctx):
    """cfg1 panel (5000 haplotypes, 2000 typed sites), every third reference
    sample haploid and 5 of 16 targets haploid: phasing at K=1024 (below the
    4,167 existing haplotypes) and beam 64, and imputation of all 27 existing
    target haplotypes at every panel site, bit-exact against oracle/_ref."""
    from eimp_b200 import synth
    from eimp_b200.bits import pack_rows, transpose_bits
    from eimp_b200.engine import PBWTImputer, PhaseParams, Phaser
    from oracle import refcore
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    nt = 16
    nh, Mref = panel.nhaps, panel.nsites
    ref_hap = (np.arange(nh // 2) % 3 == 1).astype(np.uint8)
    dense = unpack_rows(panel.hapmajor, Mref)
    dense[2 * np.flatnonzero(ref_hap) + 1] = dense[2 * np.flatnonzero(ref_hap)]
    hm_full = pack_rows(dense, W(Mref))
    sm_full = transpose_bits(hm_full, nh, Mref)
    af = (dense.sum(axis=0) / nh).astype(np.float32)
    panel = synth.Panel(nh, Mref, panel.pos, panel.cm, af, hm_full, sm_full)
    tgt_hap = np.zeros(nt, np.uint8)
    tgt_hap[[0, 3, 7, 8, 15]] = 1
    gt = tg.gt[:nt].copy()
    truth = tg.truth[:2 * nt].copy()
    for t in np.flatnonzero(tgt_hap):
        miss = gt[t] == 3
        gt[t] = 2 * truth[2 * t]
        gt[t][miss] = 3
    sub = synth.Targets(tg.typed, gt, truth)
    hm, sm, cm = synth.typed_views(panel, tg.typed)
    rc = refcore.RefCore(panel, sub)
    rc.set_haploids(ref_hap, tgt_hap)
    rc.set_params(refcore.PhaseParams(K=1024, beamwidth=64))
    rm, rp, rdm, rdp = rc.phase_range(0, nt, os.cpu_count() or 1)
    ph = Phaser(ctx, hm, sm, cm)
    ph.setHaploidRef(ref_hap)
    ph.setHaploidTargets(tgt_hap)
    mats, pats, dm, dp, tc, nc = ph.phase(PhaseParams(K=1024, beamwidth=64), gt)
    ph.setHaploidTargets(None)
    bad = [t for t in range(nt) if not (np.array_equal(mats[t], rm[t]) and np.array_equal(pats[t], rp[t])
                                        and np.array_equal(dm[t], rdm[t]) and np.array_equal(dp[t], rdp[t]))]
    assert not bad, f"targets differing from the reference: {bad}"
    M = len(tg.typed)
    phased = np.zeros((2 * nt, W(M)), np.uint64)
    phased[0::2], phased[1::2] = mats, pats
    rimp = rc.imputer(phased, os.cpu_count() or 1)
    rbits, rdos = rimp.bunch(Mref, os.cpu_count() or 1)
    imp = PBWTImputer(ctx, panel.sitemajor, panel.af, tg.typed, sm, nh, haploid_ref=ref_hap)
    imp.prepareImputation(phased, gt, haploid_targets=tgt_hap)
    bits, dos = imp.impute_window(0, Mref)
    hmap = hapmap(tgt_hap)
    assert rimp.ntargethaps == len(hmap) == 27 and rimp.K == imp.K
    sel = np.ones((nt, Mref), bool)
    sel[:, tg.typed] = gt == 3
    for j, h in enumerate(hmap):
        np.testing.assert_array_equal(imp.matches(int(h)).astype(np.int64), rimp.matches(j))
        s = sel[h // 2]
        np.testing.assert_array_equal(dos[h][s], rdos[h][s])
        assert np.max(np.abs(dos[h][s] - rdos[h][s]), initial=0) <= DOSAGE_TOL
        np.testing.assert_array_equal(unpack_rows(bits[h], Mref)[s], unpack_rows(rbits[h], Mref)[s])
    rimp.close()
    rc.close()
