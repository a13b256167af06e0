"""The FP64 dosage oracle on a sample of sites (oracle/restate.py
impute_fp64_sites, used on the large panel where the whole prefix-array set
cannot go to the host) equals the C oracle's FP64 output over all sites
(eo_impute, TargetImp.cpp:474-558) at every untyped site, on the reference-made
golden matches and prefix arrays and on a panel where the low-frequency
shortcut (TargetImp.cpp:522-531) and uncovered sites occur."""
import numpy as np

from conftest import golden_path
from eimp_b200.bits import W, pack_rows


def _check(matches, absperm, sm_full, typed, af, nrefhaps, miss, hw):
    from oracle import restate as R
    Mref = sm_full.shape[0]
    _, dos, _, d64 = R.impute(matches, absperm, sm_full, typed, af, nrefhaps, miss, hw, fp64=True)
    sites = np.setdiff1d(np.arange(Mref), typed)

    def prefix_slice(en, rs, re):
        return absperm[en, rs:re + 1]

    def site_bits(j, refs):
        row = sm_full[sites[j]]
        return (row[refs >> 6] >> (refs & 63).astype(np.uint64)) & np.uint64(1)

    got = R.impute_fp64_sites(matches, sites, typed, af, nrefhaps, prefix_slice, site_bits)
    np.testing.assert_array_equal(got, d64[sites])
    cov = got >= 0
    np.testing.assert_array_equal(got[cov].astype(np.float32), dos[sites][cov])
    return got


def test_fp64_sample_golden():
    g = np.load(golden_path("golden_tiny.npz"))
    counts = g["imp_nmatches"]
    off = np.concatenate([[0], np.cumsum(counts)])
    nh = int(g["nhaps"])
    for h in range(len(counts)):
        miss = np.flatnonzero(g["gt"][h // 2] == 3).astype(np.int64)
        _check(g["imp_matches"][off[h]:off[h + 1]], g["imp_absperm"], g["sitemajor_full"], g["typed"],
               g["af_full"], nh, miss, g["imp_phased"][h])


def test_fp64_sample_shortcut_and_conflicts():
    """A panel of 600 haplotypes with many rare sites (the shortcut's height
    threshold 100 * maf * 600 is below the taller intervals there) and a
    target whose matches leave sites uncovered."""
    from oracle import restate as R
    rng = np.random.default_rng(3)
    nh, Mref = 600, 3000
    af_true = np.where(rng.random(Mref) < 0.5, 0.002, rng.uniform(0.05, 0.5, Mref))
    dense = (rng.random((nh, Mref)) < af_true[None, :]).astype(np.uint8)
    dense[:, :] = dense[rng.integers(0, 40, nh)]       # 40 founders: long shared intervals
    flip = rng.random((nh, Mref)) < 0.001
    dense ^= flip.astype(np.uint8)
    sm_full = pack_rows(np.ascontiguousarray(dense.T), W(nh))
    af = dense.mean(axis=0).astype(np.float32)
    typed = np.sort(rng.choice(Mref, 300, replace=False)).astype(np.int64)
    compr, c0, ap = R.pbwt(np.ascontiguousarray(sm_full[typed]), nh, absperm=True)
    seen_short = seen_conf = False
    for t in range(4):
        hap = dense[rng.integers(0, nh)].copy()
        hap[rng.random(Mref) < 0.01] ^= 1
        hw = pack_rows(hap[typed][None, :], W(len(typed)))[0]
        miss = np.sort(rng.choice(len(typed), 3, replace=False)).astype(np.int64)
        m = R.smmatches(compr, c0, len(typed), nh, hw, miss, 0)
        got = _check(m, ap, sm_full, typed, af, nh, miss, hw)
        seen_conf |= bool((got < 0).any())
        maf = np.minimum(af, 1 - af)
        seen_short |= bool(((m[:, 3] - m[:, 2] + 1)[:, None] > 100 * maf[None, :] * nh).any())
    assert seen_short
