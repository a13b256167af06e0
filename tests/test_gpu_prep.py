"""GPU parity: condensed-reference preparation, condensed reference and PBWT
(Target::prepPhase, condensedReferenceT, PBWT) against the golden fixtures made
by the reference and against the oracle restatement at larger sizes.  Integer
and bit outputs must be bit-exact."""
import numpy as np
import pytest

from conftest import golden_path
from eimp_b200.bits import W, pack_genotypes

pytestmark = pytest.mark.gpu


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
def phaser(ctx, g):
    from eimp_b200.engine import Phaser
    return Phaser(ctx, g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"])


@pytest.mark.parametrize("K", [64, 50, 200])
def test_prep_golden(phaser, g, K):
    from eimp_b200.engine import PhaseParams
    pre = f"K{K}_"
    gt = g["gt"]
    r = phaser.prep(PhaseParams(K=K, beamwidth=16), gt)
    np.testing.assert_array_equal(r["besthaps"], g[pre + "besthaps"].astype(np.int32))
    np.testing.assert_array_equal(r["monos"], g[pre + "monos"])
    ns = g[pre + "nsplits"]
    np.testing.assert_array_equal(r["nsplits"], ns)
    splits = split_rows(g[pre + "splits"], ns)
    calls = split_rows(g[pre + "calls"], g[pre + "ncalls"])
    cmd = split_rows(g[pre + "cmdiffs"], [s + 1 if s else 0 for s in ns])
    for t in range(gt.shape[0]):
        S = int(ns[t])
        np.testing.assert_array_equal(r["splits"][t, :S], splits[t])
        if S:
            assert r["ncalls"][t] == len(calls[t])
            np.testing.assert_array_equal(r["calls"][t, :len(calls[t])], calls[t])
            np.testing.assert_array_equal(r["cmdiffs"][t, :S + 1], cmd[t])
        # best-haplotype flags = the best haplotypes as a bit vector
        nh = int(g["nhaps"])
        fl = np.zeros(nh, np.uint8)
        fl[g[pre + "besthaps"][t]] = 1
        np.testing.assert_array_equal(np.unpackbits(r["flags"][t].view(np.uint8), bitorder="little")[:nh], fl)


@pytest.mark.parametrize("K", [64, 50, 200])
def test_cref_pbwt_golden(phaser, g, K):
    from eimp_b200.engine import PhaseParams
    pre = f"K{K}_"
    gt = g["gt"]
    rowoff, cref, c0, pb = phaser.cref_pbwt(PhaseParams(K=K, beamwidth=16), gt)
    rows = g[pre + "rows"]
    np.testing.assert_array_equal(np.diff(rowoff), rows)
    np.testing.assert_array_equal(cref, g[pre + "cref"])
    np.testing.assert_array_equal(c0, g[pre + "count0"])
    np.testing.assert_array_equal(pb, g[pre + "pbwt"])


def test_gpuengine_dropin_golden(ctx, g):
    """GPUEngine::runCrefPBWTKernel contract: GenotypeVector words, split flags
    and best-hap flags in; 4*Kwords-stride PBWT (fwd then bck) + count0 out."""
    from eimp_b200.engine import GPUEngine
    K = 64
    pre = f"K{K}_"
    nh, M = int(g["nhaps"]), int(g["M"])
    eng = GPUEngine(0, ctx=ctx)
    Kwords = W(K)
    eng.initialize(K, Kwords, M, nh, nh, W(nh) * 8, g["sitemajor_typed"])
    gt = g["gt"]
    ns = g[pre + "nsplits"]
    splits = split_rows(g[pre + "splits"], ns)
    tgt, spl, bhf, outs, c0s = [], [], [], [], []
    for t in range(gt.shape[0]):
        tgt.append(pack_genotypes(gt[t]))
        sw = np.zeros(W(M), np.uint64)
        for s in splits[t]:
            sw[s // 64] |= np.uint64(1) << np.uint64(s % 64)
        spl.append(sw)
        fw = np.zeros(W(nh), np.uint64)
        for h in g[pre + "besthaps"][t]:
            fw[h // 64] |= np.uint64(1) << np.uint64(h % 64)
        bhf.append(fw)
        nr = 2 * int(ns[t]) + 1
        outs.append(np.zeros(2 * nr * 4 * Kwords, np.uint32))
        c0s.append(np.zeros(nr, np.int32))
    off = np.concatenate([[0], np.cumsum(2 * ns + 1)]).astype(np.uint32)
    eng.runCrefPBWTKernel(tgt, spl, bhf, off, outs, c0s)
    pbs = split_rows(g[pre + "pbwt"], 2 * g[pre + "rows"])
    c0g = split_rows(g[pre + "count0"], g[pre + "rows"])
    kw = 2 * ((K + 31) // 32)
    for t in range(gt.shape[0]):
        o = outs[t].reshape(-1, 4 * Kwords)
        np.testing.assert_array_equal(o[:, :kw], pbs[t])
        assert not o[:, kw:].any()
        np.testing.assert_array_equal(c0s[t], c0g[t])


def test_prep_cref_pbwt_vs_oracle_larger(ctx, smalltest):
    """small-test panel (600 haplotypes, 800 typed sites, K=200): every stage
    bit-exact against the oracle restatement."""
    from eimp_b200.engine import PhaseParams, Phaser
    from eimp_b200.synth import typed_views
    from oracle import restate as R
    panel, groups = smalltest
    tg = groups[0]
    hm, sm, cm = typed_views(panel, tg.typed)
    ph = Phaser(ctx, hm, sm, cm)
    K = 200
    r = ph.prep(PhaseParams(K=K), tg.gt)
    rowoff, cref, c0, pb = ph.cref_pbwt(PhaseParams(K=K), tg.gt)
    kw = 2 * ((K + 31) // 32)
    for t in range(tg.gt.shape[0]):
        bh, _ = R.besthaps(tg.gt[t], hm, K)
        np.testing.assert_array_equal(r["besthaps"][t], bh)
        mo = R.monos(hm, len(tg.typed), bh)
        np.testing.assert_array_equal(r["monos"][t], mo)
        sp, ca, cd = R.calllocs(tg.gt[t], mo, cm)
        assert r["nsplits"][t] == len(sp)
        np.testing.assert_array_equal(r["splits"][t, :len(sp)], sp)
        ocr, oc0 = R.cref(tg.gt[t], sm, panel.nhaps, bh, sp)
        a, b = rowoff[t], rowoff[t + 1]
        np.testing.assert_array_equal(cref[a:b], ocr)
        np.testing.assert_array_equal(c0[a:b], oc0)
        fw, _, _ = R.pbwt(ocr, K)
        bw, _, _ = R.pbwt(ocr, K, reverse=True)
        np.testing.assert_array_equal(pb[2 * a:2 * a + (b - a)], fw)
        np.testing.assert_array_equal(pb[2 * a + (b - a):2 * b], bw)
