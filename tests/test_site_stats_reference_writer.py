"""The output statistics of an imputed bunch against the reference's own
writer: VCFData::writeVCFImputedBunch (VCFData.cpp:3068-3446) compiled from the
reference tree into oracle/_ref/libeimp_refwriter.so (``make -C oracle
refwriter``), with the records it builds read back field by field.  The oracle
restatement (oracle/restate.py site_stats, eo_site_stats) must give the same
ADS, GT, DS, GP, RefPanelAF, AF, MAF, R2, AC, AN, TYPED and filter decision for
every site, bit for bit, and the same run statistics (conflicts, the
--improveCalls categories and their totals), for diploid and haploid targets
and every option.  The GPU kernel is checked against the same writer in
tests/test_gpu_site_stats.py."""
import numpy as np
import pytest

from eimp_b200.bits import W, pack_rows, unpack_rows

pytestmark = pytest.mark.skipif("not __import__('oracle.refwriter', fromlist=['x']).available()",
                                reason="reference writer harness not built (make -C oracle refwriter)")

u32 = lambda a: np.asarray(a, np.float32).view(np.uint32)  # noqa: E731


def random_case(seed, N=7, M=14, Mref=48, nsites=36, mref_begin=7, haploid_frac=0.0):
    rng = np.random.default_rng(seed)
    typed = np.sort(rng.choice(Mref, M, replace=False)).astype(np.int64)
    af_full = rng.random(Mref).astype(np.float32)
    af_full[rng.random(Mref) < 0.1] = 0.5          # the RefPanelAF > 0.5 boundary
    gt = rng.integers(0, 3, (N, M)).astype(np.uint8)
    gt[rng.random((N, M)) < 0.25] = 3
    dos = rng.random((2 * N, nsites)).astype(np.float32)
    dos[rng.random(dos.shape) < 0.15] = -1.0
    dos[rng.random(dos.shape) < 0.1] = 1.0
    dos[rng.random(dos.shape) < 0.05] = 0.5
    bits = pack_rows((rng.random((2 * N, nsites)) < 0.5).astype(np.uint8), W(nsites))
    phased = pack_rows((rng.random((2 * N, M)) < 0.5).astype(np.uint8), W(M))
    pdm = rng.random((N, M)).astype(np.float32)
    pdp = rng.random((N, M)).astype(np.float32)
    pdm[rng.random(pdm.shape) < 0.3] = 0.0
    pdp[rng.random(pdp.shape) < 0.3] = 1.0
    haploid = (rng.random(N) < haploid_frac).astype(np.uint8)
    if haploid_frac:
        haploid[0] = 1
        haploid[-1] = 0
        # a haploid target's genotypes are homozygous
        gt[haploid == 1] = np.where(gt[haploid == 1] == 1, 2, gt[haploid == 1])
    return dict(mref_begin=mref_begin, bits=bits, dos=dos, phased=phased, pdm=pdm, pdp=pdp, gt=gt, typed=typed,
                Mref=Mref, af_full=af_full, haploid=haploid if haploid_frac else None)


def both(case, **opt):
    from oracle import refwriter as RW
    from oracle import restate as R
    c = dict(case)
    hap = c.pop("haploid")
    args = (c["mref_begin"], c["bits"], c["dos"], c["phased"], c["pdm"], c["pdp"], c["gt"], c["typed"], c["Mref"],
            c["af_full"])
    o = R.site_stats(*args, opt.get("overwriteCalls", False), opt.get("improveCalls", False),
                     opt.get("r2filter", 0.0), opt.get("maffilter", 0.0), want_ds=True, want_gp=True, haploid=hap)
    w = RW.write_bunch(*args, haploid=hap, **opt)
    return o, w


def unset_typed_haploid(case):
    """(target, site) pairs where the reference's writer leaves DS and GP
    unset: haploid targets at typed, non-missing sites (VCFData.cpp:3428-3432)."""
    N, nsites = case["gt"].shape[0], case["dos"].shape[1]
    mask = np.zeros((N, nsites), bool)
    if case["haploid"] is None:
        return mask
    tset = {int(m): k for k, m in enumerate(case["typed"])}
    for s in range(nsites):
        k = tset.get(case["mref_begin"] + s)
        if k is None:
            continue
        mask[:, s] = (case["haploid"] == 1) & (case["gt"][:, k] != 3)
    return mask


def check(case, o, w, overwrite=False):
    from oracle import refwriter as RW
    nsites = case["dos"].shape[1]
    np.testing.assert_array_equal(o["passed"], w["written"])
    sel = w["written"] == 1
    assert sel.any()
    np.testing.assert_array_equal(u32(o["ads"][:, sel]), u32(w["ads"][:, sel]))
    # GT: the allele bits, and the vector end of a haploid target's second entry
    g = unpack_rows(o["gtbits"], nsites).astype(np.int32)
    exp = np.where(w["gtv"] == RW.INT32_VECTOR_END, 0, (w["gtv"] >> 1) - 1)
    np.testing.assert_array_equal(g[:, sel], exp[:, sel])
    if case["haploid"] is not None:
        hrows = 2 * np.flatnonzero(case["haploid"]) + 1
        assert (w["gtv"][hrows][:, sel] == RW.INT32_VECTOR_END).all()
    for k in ("r2", "af", "maf"):
        np.testing.assert_array_equal(u32(o[k][sel]), u32(w[k][sel]), err_msg=k)
    np.testing.assert_array_equal(o["ac"][sel], w["ac"][sel])
    np.testing.assert_array_equal(o["an"][sel], w["an"][sel])
    np.testing.assert_array_equal(u32(w["refpanelaf"][sel]), u32(case["af_full"][case["mref_begin"]:][:nsites][sel]))
    tset = set(int(m) for m in case["typed"])
    np.testing.assert_array_equal(w["typed"][sel], [int(case["mref_begin"] + s in tset) for s in np.flatnonzero(sel)])
    # DS and GP, except where the writer leaves them unset (the oracle writes
    # a missing DS and GP (missing, end, end) there)
    unset = unset_typed_haploid(case) if not overwrite else np.zeros((case["gt"].shape[0], nsites), bool)
    keep = ~unset & sel[None, :]
    np.testing.assert_array_equal(u32(o["ds"])[keep], u32(w["ds"])[keep])
    gkeep = np.repeat(keep, 3, axis=0)
    np.testing.assert_array_equal(u32(o["gp"])[gkeep], u32(w["gp"])[gkeep])
    if unset.any():
        assert (u32(o["ds"])[unset] == RW.FLOAT_MISSING.view(np.uint32)).all()
        assert (u32(o["gp"][0::3])[unset] == RW.FLOAT_MISSING.view(np.uint32)).all()
        assert (u32(o["gp"][1::3])[unset] == RW.FLOAT_VECTOR_END.view(np.uint32)).all()
    assert o["conflicts"] == w["conflicts"]
    np.testing.assert_array_equal(o["improve_counts"], w["improve_counts"])
    np.testing.assert_array_equal(o["improve_totals"], w["improve_totals"])


@pytest.mark.parametrize("opts", [dict(), dict(overwriteCalls=True), dict(improveCalls=True),
                                  dict(r2filter=0.3, maffilter=0.1), dict(improveCalls=True, r2filter=0.5)])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_diploid(seed, opts):
    case = random_case(seed)
    o, w = both(case, **opts)
    check(case, o, w, opts.get("overwriteCalls", False))
    if opts.get("improveCalls"):
        assert o["improve_counts"].sum() > 0


@pytest.mark.parametrize("opts", [dict(), dict(overwriteCalls=True), dict(improveCalls=True),
                                  dict(r2filter=0.3, maffilter=0.1)])
@pytest.mark.parametrize("seed", [4, 5])
def test_haploid_targets(seed, opts):
    case = random_case(seed, N=9, haploid_frac=0.4)
    o, w = both(case, **opts)
    check(case, o, w, opts.get("overwriteCalls", False))
    assert unset_typed_haploid(case).any()


def test_all_haploid_typed_site_has_no_values():
    """Every target haploid and called at a typed site: the writer adds
    nothing for that site (AN 0), so AF is 0 and r2 keeps its default 1."""
    case = random_case(6, N=4, haploid_frac=1.0)
    case["haploid"][:] = 1
    case["gt"][case["gt"] == 3] = 0
    o, w = both(case)
    check(case, o, w)
    tset = set(int(m) for m in case["typed"])
    for s in range(case["dos"].shape[1]):
        if case["mref_begin"] + s in tset:
            assert w["an"][s] == 0 and o["an"][s] == 0 and o["r2"][s] == 1.0 and o["af"][s] == 0.0
