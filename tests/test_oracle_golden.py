"""The C restatement oracle against the golden fixtures made by the reference's
own code (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from conftest import golden_path
from eimp_b200.bits import W, pack_genotypes, unpack_rows
from oracle import restate as R


@pytest.fixture(scope="module")
def g():
    return np.load(golden_path("golden_tiny.npz"))


def split_rows(z, key, counts):
    a = z[key]
    out, o = [], 0
    for c in counts:
        out.append(a[o:o + c])
        o += c
    return out


@pytest.mark.parametrize("K", [64, 50, 200])
def test_prep_cref_pbwt(g, K):
    pre = f"K{K}_"
    nh, M = int(g["nhaps"]), int(g["M"])
    gt = g["gt"]
    splits = split_rows(g, pre + "splits", g[pre + "nsplits"])
    calls = split_rows(g, pre + "calls", g[pre + "ncalls"])
    cmd = split_rows(g, pre + "cmdiffs", [s + 1 if s else 0 for s in g[pre + "nsplits"]])
    crefs = split_rows(g, pre + "cref", g[pre + "rows"])
    c0s = split_rows(g, pre + "count0", g[pre + "rows"])
    pbs = split_rows(g, pre + "pbwt", 2 * g[pre + "rows"])
    for t in range(gt.shape[0]):
        bh, _ = R.besthaps(gt[t], g["hapmajor_typed"], K)
        np.testing.assert_array_equal(bh, g[pre + "besthaps"][t])
        mo = R.monos(g["hapmajor_typed"], M, bh)
        np.testing.assert_array_equal(mo, g[pre + "monos"][t])
        sp, ca, cd = R.calllocs(gt[t], mo, g["cm_typed"])
        np.testing.assert_array_equal(sp, splits[t])
        if len(sp):
            np.testing.assert_array_equal(ca, calls[t])
            np.testing.assert_array_equal(cd, cmd[t])
        cr, c0 = R.cref(gt[t], g["sitemajor_typed"], nh, bh, sp)
        np.testing.assert_array_equal(cr, crefs[t])
        np.testing.assert_array_equal(c0, c0s[t])
        Kc = min(K, nh)
        fw, _, _ = R.pbwt(cr, Kc)
        bw, _, _ = R.pbwt(cr, Kc, reverse=True)
        np.testing.assert_array_equal(np.concatenate([fw, bw]), pbs[t])


@pytest.mark.parametrize("K", [64, 50, 200])
def test_phasing(g, K):
    pre = f"K{K}_"
    P = R.params_c(K=K, beamwidth=16)
    gt = g["gt"]
    for t in range(gt.shape[0]):
        mat, pat, dm, dp, tc, nc = R.phase(gt[t], g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"], P)
        np.testing.assert_array_equal(mat, g[pre + "mat"][t])
        np.testing.assert_array_equal(pat, g[pre + "pat"][t])
        np.testing.assert_array_equal(dm, g[pre + "dos_mat"][t])
        np.testing.assert_array_equal(dp, g[pre + "dos_pat"][t])
        assert np.float32(tc) == g[pre + "totalconf"][t]
        assert nc == g[pre + "ncallsites"][t]


def test_imputation(g):
    nh, M, Mref = int(g["nhaps"]), int(g["M"]), int(g["Mref"])
    compr, c0, ap = R.pbwt(g["sitemajor_typed"], nh, absperm=True)
    np.testing.assert_array_equal(compr, g["imp_compr"])
    np.testing.assert_array_equal(ap, g["imp_absperm"])
    ph = g["imp_phased"]
    ms = split_rows(g, "imp_matches", g["imp_nmatches"])
    gt = g["gt"]
    for h in range(ph.shape[0]):
        miss = np.where(gt[h // 2] == 3)[0].astype(np.int64)
        m = R.smmatches(compr, c0, M, nh, ph[h], miss)
        np.testing.assert_array_equal(m, ms[h])
        bits, dos, imp = R.impute(m, ap, g["sitemajor_full"], g["typed"], g["af_full"], nh, miss, ph[h])
        sel = imp.astype(bool)
        rb = unpack_rows(g["imp_bits"][h], Mref)
        ob = unpack_rows(bits, Mref)
        np.testing.assert_array_equal(ob[sel], rb[sel])
        np.testing.assert_array_equal(dos[sel], g["imp_dos"][h][sel])
        # a 60 %-missing target yields no matches and only dosage conflicts
        if h // 2 == gt.shape[0] - 1:
            assert len(m) == 0 and np.all(dos[sel] == -1.0)


def test_transpose_bits_round_trip():
    """The host transposition used to build the panel of a phasing iteration."""
    from eimp_b200.bits import pack_rows, unpack_rows
    from eimp_b200.engine import _transpose_bits
    rng = np.random.default_rng(3)
    b = (rng.random((37, 1000)) < 0.3).astype(np.uint8)
    rows = pack_rows(b, W(1000))
    t = _transpose_bits(rows, 1000)
    assert t.shape == (1000, W(37))
    np.testing.assert_array_equal(unpack_rows(t, 37), b.T)


def test_reference_iteration_excludes_own_sample():
    """The reference's findBestHaps in an iteration after the first
    (Target.cpp:791-841), run from its own sources: a target never picks its
    own two haplotypes from the panel of reference + phased targets, and with
    K at least the other haplotypes it takes all of those in order."""
    from oracle import refcore
    if not refcore.available():
        pytest.skip("reference sources not compiled (oracle/_ref)")
    from eimp_b200.engine import _transpose_bits
    g = np.load(golden_path("golden_tiny.npz"))
    hm, cm, gt = g["hapmajor_typed"], g["cm_typed"], g["gt"]
    n, M = gt.shape
    nh = hm.shape[0]
    tgt = np.empty((2 * n, hm.shape[1]), np.uint64)
    tgt[0::2], tgt[1::2] = g["K64_mat"], g["K64_pat"]
    aug = np.concatenate([hm, tgt])
    rc = refcore.RefCore.typed_only(aug, _transpose_bits(aug, M), cm, gt, g["af_full"][g["typed"]])
    rc.set_iteration(nh, True)
    for K in (64, 1000):
        rc.set_params(refcore.PhaseParams(K=K))
        for t in range(n):
            bh = rc.prep(t)["besthaps"]
            assert nh + 2 * t not in bh and nh + 2 * t + 1 not in bh
            if K == 1000:
                np.testing.assert_array_equal(bh, [h for h in range(nh + 2 * n) if h // 2 != nh // 2 + t])
    rc.close()


def test_determine_start_phases():
    """VCFData::determineStartPhases (VCFData.cpp:2802-2816): the maternal
    allele at the first heterozygous site from the overlap start on, else at
    the last site."""
    from eimp_b200.bits import pack_rows
    from eimp_b200.engine import determine_start_phases
    M = 10
    mats = np.array([[0, 0, 1, 1, 0, 0, 0, 0, 0, 0],    # het at 4 (mat 0)
                     [0, 0, 0, 0, 0, 1, 0, 0, 0, 0],    # het at 5 (mat 1)
                     [1, 1, 1, 1, 1, 1, 1, 1, 1, 1]], np.uint8)   # no het: mat at the last site
    pats = np.array([[0, 0, 1, 1, 1, 0, 0, 0, 0, 0],
                     [0, 0, 0, 0, 0, 0, 0, 0, 0, 0],
                     [1, 1, 1, 1, 1, 1, 1, 1, 1, 1]], np.uint8)
    got = determine_start_phases(pack_rows(mats, W(M)), pack_rows(pats, W(M)), 3, M)
    np.testing.assert_array_equal(got, [0, 1, 1])
