"""GPU parity: phasing iterations (PBWTPhaser.cpp:406-476, --phaseIters)
against the reference's own Target::phase (oracle/_ref) over the same
augmented panels: after the first iteration the panel is the reference
followed by the phased targets, each target leaves its own haplotypes out of
its best haplotypes (Target.cpp:791-811), and reverse phasing runs in the last
iteration only.  Phased haplotypes, dosages and confidences bit-exact."""
import numpy as np
import pytest

from conftest import golden_path
from eimp_b200.bits import W

pytestmark = pytest.mark.gpu


def reference_iterations(hm, sm, cm, gt, af_common, K, beam, iters, ref_hap=None, tgt_hap=None):
    from eimp_b200.engine import _transpose_bits
    from oracle import refcore
    n, M = gt.shape
    nh = hm.shape[0]
    panel = (hm, sm)
    out = None
    for it in range(1, iters + 1):
        last = it == iters
        if it > 1:
            mats, pats = out[0], out[1]
            tgt = np.empty((2 * n, mats.shape[1]), np.uint64)
            tgt[0::2], tgt[1::2] = mats, pats
            aug = np.concatenate([hm, tgt])
            panel = (aug, _transpose_bits(aug, M))
        rc = refcore.RefCore.typed_only(panel[0], panel[1], cm, gt, af_common)
        rc.set_iteration(nh if it > 1 else 0, last)
        if ref_hap is not None:
            # iterations after the first: the phased targets join the panel
            # with their ploidy (VCFData.cpp:1926-1931)
            rc.set_haploids(ref_hap if it == 1 else np.concatenate([ref_hap, tgt_hap]), tgt_hap)
        rc.set_params(refcore.PhaseParams(K=K, beamwidth=beam, doRevPhasing=last))
        res = [rc.phase(t) for t in range(n)]
        rc.close()
        out = [np.stack([r[i] for r in res]) for i in range(4)] + [np.array([r[4] for r in res], np.float32),
                                                                    np.array([r[5] for r in res])]
    return out


@pytest.mark.parametrize("K,iters", [(64, 2), (64, 3), (400, 2)])
def test_phasing_iterations_vs_reference(ctx, K, iters):
    from eimp_b200.engine import PhaseParams, phase_iterations
    from oracle import refcore
    if not refcore.available():
        pytest.skip("reference sources not compiled (oracle/_ref)")
    g = np.load(golden_path("golden_tiny.npz"))
    hm, sm, cm, gt = g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"], g["gt"]
    af_common = g["af_full"][g["typed"]]
    got = phase_iterations(ctx, hm, sm, cm, PhaseParams(K=K, beamwidth=16), gt, iters)
    want = reference_iterations(hm, sm, cm, gt, af_common, K, 16, iters)
    for name, a, b in zip(("mats", "pats", "dm", "dp", "totalconf", "ncallsites"), got, want):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b).astype(np.asarray(a).dtype), err_msg=name)


def test_best_haps_leave_own_sample_out(ctx):
    """Iteration 2 best haplotypes: never the target's own two haplotypes,
    and the same set as the reference's findBestHaps."""
    from eimp_b200.engine import PhaseParams, Phaser, _transpose_bits
    from oracle import refcore
    if not refcore.available():
        pytest.skip("reference sources not compiled (oracle/_ref)")
    g = np.load(golden_path("golden_tiny.npz"))
    hm, cm, gt = g["hapmajor_typed"], g["cm_typed"], g["gt"]
    n, M = gt.shape
    nh = hm.shape[0]
    tgt = np.concatenate([g["K64_mat"], g["K64_pat"]])[np.argsort(np.r_[0:2 * n:2, 1:2 * n:2])]
    aug = np.concatenate([hm, tgt])
    ph = Phaser(ctx, aug, _transpose_bits(aug, M), cm)
    ph.excludeSelf(nh // 2)
    got = ph.prep(PhaseParams(K=64), gt)["besthaps"]
    rc = refcore.RefCore.typed_only(aug, _transpose_bits(aug, M), cm, gt, g["af_full"][g["typed"]])
    rc.set_iteration(nh, True)
    rc.set_params(refcore.PhaseParams(K=64))
    for t in range(n):
        own = {nh + 2 * t, nh + 2 * t + 1}
        assert not own & set(got[t].tolist())
        np.testing.assert_array_equal(got[t], rc.prep(t)["besthaps"])
    rc.close()


@pytest.mark.parametrize("K", [64, 400])
def test_phasing_iterations_haploid_vs_reference(ctx, K):
    """Two iterations over a panel with haploid samples and haploid targets
    (golden_haploid.npz): the grown panel carries the targets' ploidy, K is
    clamped to the haplotypes that exist (PBWTPhaser.cpp:159)."""
    from eimp_b200.engine import PhaseParams, phase_iterations
    g = np.load(golden_path("golden_haploid.npz"))
    hm, sm, cm, gt = g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"], g["gt"]
    af_common = g["af_full"][g["typed"]]
    rh, th = g["ref_haploid"], g["tgt_haploid"]
    got = phase_iterations(ctx, hm, sm, cm, PhaseParams(K=K, beamwidth=16), gt, 2, haploid_ref=rh, haploid_tgt=th)
    want = reference_iterations(hm, sm, cm, gt, af_common, K, 16, 2, rh, th)
    for name, a, b in zip(("mats", "pats", "dm", "dp", "totalconf", "ncallsites"), got, want):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b).astype(np.asarray(a).dtype), err_msg=name)
