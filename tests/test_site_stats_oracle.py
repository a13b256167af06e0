"""The oracle restatement of the output statistics of an imputed bunch
(VCFData::writeVCFImputedBunch, VCFData.cpp:3068-3446), checked by a case
worked by hand and by a second, element-by-element restatement in Python with
explicit float32/float64 scalars in the reference's order of operations, over
random inputs with conflicts, missing calls and the --overwriteCalls /
--improveCalls / filter options.  The pin against the reference's own writer
is tests/test_site_stats_reference_writer.py."""
import numpy as np
import pytest

from eimp_b200.bits import W, pack_rows, unpack_rows

f32, f64 = np.float32, np.float64


def python_stats(mref_begin, bits, dos, phased, pdm, pdp, gt, typed, af_full, overwrite, improve, r2f_thr,
                 maf_thr):
    nh, nsites = dos.shape
    N, M = gt.shape
    ub = unpack_rows(bits, nsites)
    up = unpack_rows(phased, M)
    typed = list(typed)
    tset = {m: k for k, m in enumerate(typed)}
    out = dict(ads=np.zeros((nh, nsites), f32), gt=np.zeros((nh, nsites), np.uint8), ds=np.zeros((N, nsites), f32),
               gp=np.zeros((3 * N, nsites), f32), r2=np.zeros(nsites, f32), af=np.zeros(nsites, f32),
               maf=np.zeros(nsites, f32), ac=np.zeros(nsites, np.int32), an=np.zeros(nsites, np.int32),
               passed=np.zeros(nsites, np.uint8))
    conf = 0
    for s in range(nsites):
        mref = mref_begin + s
        rpaf = f32(af_full[mref])
        isimp = mref not in tset
        psite = tset.get(mref, 0)
        adsum, ad2sum, nval, ac1, an = f64(0), f64(0), 0, 0, 0
        for i in range(N):
            h0, h1 = 2 * i, 2 * i + 1
            miss = (not isimp) and gt[i, psite] == 3
            if isimp or miss or overwrite:
                hp = [int(ub[h0, s]), int(ub[h1, s])]
                a = [f32(dos[h0, s]), f32(dos[h1, s])]
                for j in range(2):
                    if a[j] < 0:
                        a[j] = rpaf
                        hp[j] = int(rpaf > 0.5)
                        conf += 1
            else:
                hp = [int(up[h0, psite]), int(up[h1, psite])]
                a = [f32(pdm[i, psite]), f32(pdp[i, psite])]
                if improve:
                    raw = [f32(dos[h0, s]), f32(dos[h1, s])]
                    idos = [rpaf if x < 0 else x for x in raw]
                    idos = [f32(f64(1.0) - f64(x)) if x > 0.5 else x for x in idos]
                    pd = [f32(f64(1.0) - f64(x)) if x > 0.5 else x for x in a]
                    imp = [f32(pd[j] - idos[j]) for j in range(2)]
                    if f32(imp[0] + imp[1]) > 0:
                        conf += int(raw[0] < 0) + int(raw[1] < 0)
                        hp = [int(ub[h0, s]), int(ub[h1, s])]
                        a = [f32(f64(1.0) - f64(idos[j])) if hp[j] else idos[j] for j in range(2)]
            out["ads"][h0, s], out["ads"][h1, s] = a
            out["gt"][h0, s], out["gt"][h1, s] = hp
            adsum = f64(adsum + f64(f32(a[0] + a[1])))
            ad2sum = f64(ad2sum + f64(f32(f32(a[0] * a[0]) + f32(a[1] * a[1]))))
            out["ds"][i, s] = f32(a[0] + a[1])
            g0 = f64((f64(1.0) - f64(a[0])) * (f64(1.0) - f64(a[1])))
            g2 = f64(f32(a[0] * a[1]))
            g1 = f64(f64(f64(1.0) - g0) - g2)
            out["gp"][3 * i, s], out["gp"][3 * i + 1, s], out["gp"][3 * i + 2, s] = f32(g0), f32(g1), f32(g2)
            ac1 += hp[0] + hp[1]
            an += 2
            nval += 2
        r2, af = f64(1.0), f64(0.0)
        if nval:
            af = f64(adsum / f64(nval))
            evar = f64(af * f64(f64(1.0) - af))
            ovar = f64(f64(ad2sum - f64(adsum * af)) / f64(nval))
            r2 = f64(ovar / evar) if (evar > 0 and ovar > 0) else f64(0.0)
        r2f, aff = f32(r2), f32(af)
        maff = f32(f32(1.0) - aff) if aff > 0.5 else aff
        out["r2"][s], out["af"][s], out["maf"][s] = r2f, aff, maff
        out["ac"][s], out["an"][s] = ac1, an
        out["passed"][s] = int(not (r2f < f32(r2f_thr) or maff < f32(maf_thr)))
    return out, conf


def random_case(seed, N=5, M=12, Mref=40, nsites=30, mref_begin=6):
    rng = np.random.default_rng(seed)
    typed = np.sort(rng.choice(Mref, M, replace=False)).astype(np.int64)
    af_full = rng.random(Mref).astype(np.float32)
    gt = rng.integers(0, 3, (N, M)).astype(np.uint8)
    gt[rng.random((N, M)) < 0.25] = 3
    dos = rng.random((2 * N, nsites)).astype(np.float32)
    dos[rng.random(dos.shape) < 0.15] = -1.0
    dos[rng.random(dos.shape) < 0.1] = 1.0
    bits = pack_rows((rng.random((2 * N, nsites)) < 0.5).astype(np.uint8), W(nsites))
    phased = pack_rows((rng.random((2 * N, M)) < 0.5).astype(np.uint8), W(M))
    pdm = rng.random((N, M)).astype(np.float32)
    pdp = rng.random((N, M)).astype(np.float32)
    pdm[rng.random(pdm.shape) < 0.3] = 0.0
    pdp[rng.random(pdp.shape) < 0.3] = 1.0
    return mref_begin, bits, dos, phased, pdm, pdp, gt, typed, Mref, af_full


def test_hand_worked_case():
    """Two targets, three reference sites of one bunch (all imputed):
    site 0 dosages (1, 0 | 1, 1) -> AF 0.75, r2 1, AC 3, AN 4, MAF 0.25;
    site 1 dosages (0.5, 0.5 | 0.5, 0.5) -> AF 0.5, observed variance 0, r2 0;
    site 2 dosages (conflict, 1 | 0, 0) with RefPanelAF 0.25 -> the conflict
    becomes 0.25 with allele 0: AF 1.25/4, AC 1, one conflict."""
    from oracle import restate as R
    dos = np.array([[1, 0.5, -1], [0, 0.5, 1], [1, 0.5, 0], [1, 0.5, 0]], np.float32)
    alleles = np.array([[1, 0, 1], [0, 1, 1], [1, 1, 0], [1, 0, 0]], np.uint8)
    bits = pack_rows(alleles, W(3))
    gt = np.zeros((2, 1), np.uint8)
    phased = np.zeros((4, W(1)), np.uint64)
    pd = np.zeros((2, 1), np.float32)
    af_full = np.array([0.5, 0.5, 0.25, 0.9], np.float32)
    r = R.site_stats(0, bits, dos, phased, pd, pd, gt, [3], 4, af_full, want_ds=True, want_gp=True)
    np.testing.assert_array_equal(r["ac"], [3, 2, 1])
    np.testing.assert_array_equal(r["an"], [4, 4, 4])
    assert r["conflicts"] == 1
    assert r["ads"][0, 2] == np.float32(0.25)
    assert unpack_rows(r["gtbits"], 3)[0, 2] == 0
    np.testing.assert_array_equal(r["af"], np.float32([0.75, 0.5, 1.25 / 4]))
    np.testing.assert_array_equal(r["maf"], np.float32([0.25, 0.5, 1.25 / 4]))
    assert r["r2"][0] == 1.0 and r["r2"][1] == 0.0
    # site 2: mean 0.3125, E[x^2] = (0.0625 + 1)/4, r2 = (E[x^2] - mean^2) / (mean (1 - mean))
    m, e2 = 1.25 / 4, 1.0625 / 4
    assert abs(float(r["r2"][2]) - (e2 - m * m) / (m * (1 - m))) < 1e-6
    np.testing.assert_array_equal(r["ds"][:, 0], np.float32([1, 2]))
    np.testing.assert_array_equal(r["gp"][:3, 0], np.float32([0, 1, 0]))   # dosages 1 and 0: heterozygous
    np.testing.assert_array_equal(r["passed"], [1, 1, 1])


@pytest.mark.parametrize("overwrite,improve", [(False, False), (True, False), (False, True)])
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_vs_python_restatement(seed, overwrite, improve):
    from oracle import restate as R
    mref_begin, bits, dos, phased, pdm, pdp, gt, typed, Mref, af_full = random_case(seed)
    r = R.site_stats(mref_begin, bits, dos, phased, pdm, pdp, gt, typed, Mref, af_full, overwrite, improve,
                     0.3, 0.1, want_ds=True, want_gp=True)
    p, conf = python_stats(mref_begin, bits, dos, phased, pdm, pdp, gt, typed, af_full, overwrite, improve, 0.3, 0.1)
    assert r["conflicts"] == conf
    for k in ("ads", "ds", "gp", "r2", "af", "maf", "ac", "an", "passed"):
        np.testing.assert_array_equal(r[k], p[k], err_msg=k)
    np.testing.assert_array_equal(unpack_rows(r["gtbits"], dos.shape[1]), p["gt"])
    assert 0 < r["passed"].sum() < len(r["passed"])   # the filters cut some records, not all
