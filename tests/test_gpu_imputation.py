"""GPU parity: PBWT imputation (reference PBWT + prefix arrays, set-maximal
matches, dosages) against the golden fixtures made by the reference and
against the oracle restatement.  Matches and bits must be bit-exact; dosages
are bit-exact too (integer score/sum and one double division), the tolerance
asked for is 1e-5 absolute."""
import numpy as np
import pytest

from conftest import golden_path
from eimp_b200.bits import W, pack_rows, unpack_rows

pytestmark = pytest.mark.gpu

DOSAGE_TOL = 1e-5


@pytest.fixture(scope="module")
def g():
    return np.load(golden_path("golden_tiny.npz"))


def split_rows(a, counts):
    out, o = [], 0
    for c in counts:
        out.append(a[o:o + c])
        o += c
    return out


@pytest.fixture(scope="module")
def imp(ctx, g):
    from eimp_b200.engine import PBWTImputer
    i = PBWTImputer(ctx, g["sitemajor_full"], g["af_full"], g["typed"], g["sitemajor_typed"], int(g["nhaps"]))
    i.prepareImputation(g["imp_phased"], g["gt"])
    return i


def test_refpbwt_golden(imp, g):
    compr, ap = imp.refpbwt()
    np.testing.assert_array_equal(compr, g["imp_compr"])
    np.testing.assert_array_equal(ap, g["imp_absperm"])


def test_matches_golden(imp, g):
    ms = split_rows(g["imp_matches"], g["imp_nmatches"])
    for h in range(g["imp_phased"].shape[0]):
        np.testing.assert_array_equal(imp.matches(h).astype(np.int64), ms[h])


def test_dosages_golden(imp, g):
    from oracle import restate as R
    Mref = int(g["Mref"])
    bits, dos = imp.impute_window(0, Mref)
    gt = g["gt"]
    nh = int(g["nhaps"])
    compr, c0, ap = R.pbwt(g["sitemajor_typed"], nh, absperm=True)
    for h in range(g["imp_phased"].shape[0]):
        miss = np.where(gt[h // 2] == 3)[0].astype(np.int64)
        _, _, imputed = R.impute(imp.matches(h).astype(np.int64), ap, g["sitemajor_full"], g["typed"],
                                 g["af_full"], nh, miss, g["imp_phased"][h])
        sel = imputed.astype(bool)
        rb = unpack_rows(g["imp_bits"][h], Mref)
        ob = unpack_rows(bits[h], Mref)
        np.testing.assert_array_equal(ob[sel], rb[sel])
        np.testing.assert_array_equal(dos[h][sel], g["imp_dos"][h][sel])
        assert np.max(np.abs(dos[h][sel] - g["imp_dos"][h][sel]), initial=0) <= DOSAGE_TOL
        # sites the reference leaves unwritten carry the phased allele
        k = np.searchsorted(g["typed"], np.arange(Mref), side="right") - 1
        ph = unpack_rows(g["imp_phased"][h], int(g["M"]))
        np.testing.assert_array_equal(ob[~sel], ph[k[~sel]])
        np.testing.assert_array_equal(dos[h][~sel], ph[k[~sel]].astype(np.float32))


def test_windows_and_bunches(imp, g):
    """imputeBunch over blocks/bunches = one whole window (stateless windows,
    unaligned starts included)."""
    Mref = int(g["Mref"])
    bits, dos = imp.impute_window(0, Mref)
    full = unpack_rows(bits, Mref)
    for b0, n in ((0, 64), (37, 500), (1000, 1999), (Mref - 10, 10)):
        bb, dd = imp.impute_window(b0, n)
        np.testing.assert_array_equal(dd, dos[:, b0:b0 + n])
        np.testing.assert_array_equal(unpack_rows(bb, n), full[:, b0:b0 + n])
    imp.prepareImputation(g["imp_phased"], g["gt"], num_sites_per_block=[100, 1400, Mref - 1500, 0])
    d0 = np.concatenate([imp.imputeBunch(0, 700)[1], imp.imputeBunch(0, 700)[1]], axis=1)
    np.testing.assert_array_equal(d0, dos[:, 100:1500])
    d1 = imp.imputeBunch(1, Mref)[1]
    np.testing.assert_array_equal(d1[:, :Mref - 1500], dos[:, 1500:])


def test_imputation_vs_oracle_cfg1_sample(ctx):
    """cfg1 panel (5000 haplotypes x 20000 sites, 2000 typed), 40 target
    haplotypes from the true haplotypes: matches and dosages bit-exact against
    the oracle; max |error| against an FP64 score/sum stated."""
    from eimp_b200 import synth
    from eimp_b200.engine import PBWTImputer
    from eimp_b200.synth import typed_views
    from oracle import restate as R
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    nt = 20
    hm, sm, cm = typed_views(panel, tg.typed)
    M = len(tg.typed)
    phased = pack_rows(tg.truth[:2 * nt], W(M))
    imp = PBWTImputer(ctx, panel.sitemajor, panel.af, tg.typed, sm, panel.nhaps)
    imp.prepareImputation(phased, tg.gt[:nt])
    bits, dos = imp.impute_window(0, panel.nsites)
    compr, c0, ap = R.pbwt(sm, panel.nhaps, absperm=True)
    gc, ga = imp.refpbwt()
    np.testing.assert_array_equal(gc, compr)
    np.testing.assert_array_equal(ga, ap)
    worst = 0.0
    for h in range(2 * nt):
        miss = np.where(tg.gt[h // 2] == 3)[0].astype(np.int64)
        om = R.smmatches(compr, c0, M, panel.nhaps, phased[h], miss)
        np.testing.assert_array_equal(imp.matches(h).astype(np.int64), om)
        ob, od, oi, o64 = R.impute(om, ap, panel.sitemajor, tg.typed, panel.af, panel.nhaps, miss, phased[h],
                                   fp64=True)
        np.testing.assert_array_equal(dos[h], od)
        np.testing.assert_array_equal(bits[h], ob)
        cov = oi.astype(bool) & (o64 >= 0)
        err = np.abs(dos[h][cov].astype(np.float64) - o64[cov])
        assert err.max(initial=0.0) <= DOSAGE_TOL
        worst = max(worst, float(err.max(initial=0.0)))
    print(f"largest |dosage - FP64 score/sum| over {2 * nt} haplotypes x {panel.nsites} sites: {worst:.3e}")


@pytest.mark.parametrize("setmaxerrors", [1, 2, 3])
def test_setmaxerrors_vs_oracle_cfg1(ctx, setmaxerrors):
    """Set-maximal matches with tolerated errors (--setmaxerrors): the match
    trees grow past the first launch's node pool (up to 718, 1733 and 3093
    nodes at 1, 2 and 3 errors on this panel) and those haplotypes are redone
    by the retry launch.  Matches and dosages bit-exact against the oracle."""
    from eimp_b200 import synth
    from eimp_b200.engine import PBWTImputer
    from eimp_b200.synth import typed_views
    from oracle import restate as R
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    nt = 16
    _, sm, _ = typed_views(panel, tg.typed)
    M = len(tg.typed)
    phased = pack_rows(tg.truth[:2 * nt], W(M))
    imp = PBWTImputer(ctx, panel.sitemajor, panel.af, tg.typed, sm, panel.nhaps, setmaxerrors=setmaxerrors)
    imp.prepareImputation(phased, tg.gt[:nt])
    bits, dos = imp.impute_window(0, panel.nsites)
    compr, c0, ap = R.pbwt(sm, panel.nhaps, absperm=True)
    for h in range(2 * nt):
        miss = np.where(tg.gt[h // 2] == 3)[0].astype(np.int64)
        om = R.smmatches(compr, c0, M, panel.nhaps, phased[h], miss, setmaxerrors)
        np.testing.assert_array_equal(imp.matches(h).astype(np.int64), om)
        ob, od, oi = R.impute(om, ap, panel.sitemajor, tg.typed, panel.af, panel.nhaps, miss, phased[h])
        np.testing.assert_array_equal(dos[h], od)
        np.testing.assert_array_equal(bits[h], ob)


def test_many_typed_sites_wide_tree(ctx):
    """70000 typed sites (more than the compact tree's 16-bit depths hold):
    the match search runs on the wide-tree kernel.  Panel of 512 haplotypes
    copied in segments from 40 founders with 0.2 % mutations; targets copied
    the same way, 2 % of their genotypes missing.  Matches and dosages
    bit-exact against the oracle."""
    from eimp_b200.engine import PBWTImputer
    from oracle import restate as R
    rng = np.random.default_rng(70000)
    M, K, nt, nf, seg = 70000, 512, 3, 40, 2500
    founders = (rng.random((nf, M)) < rng.beta(0.5, 0.5, M)).astype(np.uint8)

    def mosaic(n):
        src = rng.integers(0, nf, (n, (M + seg - 1) // seg)).repeat(seg, axis=1)[:, :M]
        h = founders[src, np.arange(M)]
        return h ^ (rng.random((n, M)) < 0.002).astype(np.uint8)

    ref = mosaic(K)
    tgt = mosaic(2 * nt)
    gt = (tgt[0::2] + tgt[1::2]).astype(np.uint8)
    gt[rng.random(gt.shape) < 0.02] = 3
    sm = pack_rows(ref.T.copy(), W(K))
    af = ref.mean(axis=0).astype(np.float32)
    typed = np.arange(M, dtype=np.int64)
    phased = pack_rows(tgt, W(M))
    imp = PBWTImputer(ctx, sm, af, typed, sm, K)
    imp.prepareImputation(phased, gt)
    bits, dos = imp.impute_window(0, M)
    compr, c0, ap = R.pbwt(sm, K, absperm=True)
    for h in range(2 * nt):
        miss = np.where(gt[h // 2] == 3)[0].astype(np.int64)
        om = R.smmatches(compr, c0, M, K, phased[h], miss)
        assert len(om) > 0
        np.testing.assert_array_equal(imp.matches(h).astype(np.int64), om)
        ob, od, oi = R.impute(om, ap, sm, typed, af, K, miss, phased[h])
        np.testing.assert_array_equal(dos[h], od)
        np.testing.assert_array_equal(bits[h], ob)
