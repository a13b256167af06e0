"""GPU parity at the benchmarked setting against the reference's own code.

The full phase+impute configuration: 10,000 reference haplotypes x 100,000
sites, targets typed at 5,000 sites with 2 % missing, K = 4096, beam width 128
(the reference's default, Args.cpp:293, and the largest the beam kernel
holds), history 100.  The first 24 targets run through the CUDA path and
through the reference's own Target::phase and PBWTImputer compiled from its
sources (oracle/_ref).  Phased haplotypes, phasing dosages, call confidences,
set-maximal matches, imputed alleles and dosages must be bit-exact; dosages
are also held to 1e-5 absolute against the reference, and their largest error
against the FP64 dosage oracle (score/sum in double, TargetImp.cpp:546-548
without the rounding to float) is printed and bounded by half a float ulp."""
import os

import numpy as np
import pytest

from eimp_b200.bits import W, unpack_rows

pytestmark = pytest.mark.gpu

NT = 24
K, BEAM = 4096, 128
DOSAGE_TOL = 1e-5


@pytest.fixture(scope="module")
def bench_case():
    from eimp_b200 import synth
    from oracle import refcore
    assert refcore.available(), "the reference-compiled oracle (oracle/_ref) is missing"
    panel, groups = synth.generate("cfg2")
    tg = groups[0]
    sub = synth.Targets(tg.typed, np.ascontiguousarray(tg.gt[:NT]), np.ascontiguousarray(tg.truth[:2 * NT]))
    rc = refcore.RefCore(panel, sub)
    rc.set_params(refcore.PhaseParams(K=K, beamwidth=BEAM))
    yield panel, sub, rc
    rc.close()


@pytest.fixture(scope="module")
def phased(ctx, bench_case):
    from eimp_b200.engine import PhaseParams, Phaser
    from eimp_b200.synth import typed_views
    panel, sub, rc = bench_case
    hm, sm, cm = typed_views(panel, sub.typed)
    ph = Phaser(ctx, hm, sm, cm)
    gpu = ph.phase(PhaseParams(K=K, beamwidth=BEAM), sub.gt)
    ref = rc.phase_range(0, NT, os.cpu_count() or 1)
    return gpu, ref


def test_phasing_bit_exact_vs_reference(phased):
    (mats, pats, dm, dp, tc, nc), (rm, rp, rdm, rdp) = phased
    bad = [t for t in range(NT) if not (np.array_equal(mats[t], rm[t]) and np.array_equal(pats[t], rp[t]))]
    assert not bad, f"targets whose phased haplotypes differ from the reference: {bad}"
    np.testing.assert_array_equal(dm, rdm)
    np.testing.assert_array_equal(dp, rdp)


def test_call_confidences_vs_reference(phased, bench_case):
    """Target::getTotalConfidence / getNCallSites of four targets."""
    _, _, rc = bench_case
    (_, _, _, _, tc, nc), _ = phased
    for t in range(4):
        _, _, _, _, rtc, rnc = rc.phase(t)
        assert tc[t] == np.float32(rtc) and nc[t] == rnc, t


def test_imputation_bit_exact_vs_reference(ctx, phased, bench_case):
    from eimp_b200.engine import PBWTImputer
    from oracle import restate as R
    panel, sub, rc = bench_case
    (mats, pats, *_), _ = phased
    M, Mref = len(sub.typed), panel.nsites
    hap = np.zeros((2 * NT, W(M)), np.uint64)
    hap[0::2], hap[1::2] = mats, pats
    from eimp_b200.synth import typed_views
    _, sm, _ = typed_views(panel, sub.typed)
    imp = PBWTImputer(ctx, panel.sitemajor, panel.af, sub.typed, sm, panel.nhaps)
    imp.prepareImputation(hap, sub.gt)
    bits, dos = imp.impute_window(0, Mref)
    rimp = rc.imputer(hap, os.cpu_count() or 1)
    rbits, rdos = rimp.bunch(Mref, os.cpu_count() or 1)
    compr, ap = rimp.refpbwt()
    gc, ga = imp.refpbwt()
    np.testing.assert_array_equal(gc, compr)
    np.testing.assert_array_equal(ga, ap)
    worst64 = 0.0
    for h in range(2 * NT):
        rm = rimp.matches(h)
        np.testing.assert_array_equal(imp.matches(h).astype(np.int64), rm)
        miss = np.where(sub.gt[h // 2] == 3)[0].astype(np.int64)
        _, _, imputed, d64 = R.impute(rm, ap, panel.sitemajor, sub.typed, panel.af, panel.nhaps, miss, hap[h],
                                      fp64=True)
        sel = imputed.astype(bool)
        np.testing.assert_array_equal(unpack_rows(bits[h], Mref)[sel], unpack_rows(rbits[h], Mref)[sel])
        np.testing.assert_array_equal(dos[h][sel], rdos[h][sel])
        assert np.max(np.abs(dos[h][sel] - rdos[h][sel]), initial=0.0) <= DOSAGE_TOL
        cov = sel & (d64 >= 0)
        err = np.abs(dos[h][cov].astype(np.float64) - d64[cov])
        assert np.all(err <= np.spacing(np.float32(1.0)) / 2), h   # half a float ulp at 1
        worst64 = max(worst64, float(err.max(initial=0.0)))
    rimp.close()
    print(f"largest |dosage - FP64 score/sum| over {2 * NT} haplotypes x {Mref} sites: {worst64:.3e}")
